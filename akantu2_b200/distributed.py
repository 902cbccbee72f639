"""One mesh over several subdomains: the explicit step of a partitioned mesh.

The reference distributes a mesh with a graph partitioner
(src/mesh_utils/mesh_partition/mesh_partition_scotch.cc) and, every step,
sends the stresses of ghost elements to the processes that hold them
(SynchronizationTag::_smm_stress, solid_mechanics_model.cc:333-370).  Here
(libakb, partition.cc):

- the elements are split by recursive coordinate bisection of their centroids;
- a node belongs to the lowest part among its elements, and a subdomain holds
  every element with a node it owns (a ghost layer evaluated redundantly) and
  every node of those elements; ghost nodes are blocked locally;
- before every step each owner sends the predicted displacement of its nodes
  that are ghosts elsewhere, the holders write it into their prediction, and
  the step runs: one exchange per step.  (Exchanging before rather than after
  the step also covers host writes between steps, after which every model
  predicts again from its own state.)

Each owned node sums the same elemental forces in the same order as the whole
mesh on one GPU, so a partitioned run is bit-identical to the serial one
(FP64 and mixed alike).

PartitionedModel advances all subdomains on the current GPU through the
library's exchange (akb_exchange: per-step gather / scatter between the
subdomain models on their own streams, ordered by events, replayed as CUDA
graphs of 100 steps).  DistributedModel is one
subdomain per torch.distributed rank: with NCCL the halo buffers stay on the
device and the send/receive run on the model's stream; with gloo they are
staged through host memory.
"""
import ctypes

import numpy as np

from . import _capi
from .mesh import Mesh, TYPE_IDS
from .model import SolidMechanicsModel, _explicit_lumped_mass


def partition_elements(mesh, nparts):
    """Part of every element, [E] int32 (akb_partition_elements)."""
    part = np.zeros(mesh.getNbElement(), dtype=np.int32)
    _capi.check(_capi.lib().akb_partition_elements(
        TYPE_IDS[mesh.element_type], _capi.ptr(mesh.nodes), mesh.getNbNodes(),
        _capi.ptr(mesh.connectivity), mesh.getNbElement(), int(nparts), _capi.ptr(part)))
    return part


class Subdomain:
    """Rank `rank`'s part of the mesh: local mesh (owned nodes first, then
    ghosts), global ids of local nodes and elements, and per neighbor the
    local nodes to send and to receive (the same global nodes in the same
    order on both sides)."""

    def __init__(self, mesh, part, nparts, rank):
        L = _capi.lib()
        part = np.ascontiguousarray(part, dtype=np.int32)
        h = ctypes.c_void_p()
        _capi.check(L.akb_subdomain_create(
            TYPE_IDS[mesh.element_type], _capi.ptr(mesh.nodes), mesh.getNbNodes(),
            _capi.ptr(mesh.connectivity), mesh.getNbElement(), _capi.ptr(part), int(nparts),
            int(rank), ctypes.byref(h)))
        try:
            nl, no, el, nb = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int()
            _capi.check(L.akb_subdomain_sizes(h, ctypes.byref(nl), ctypes.byref(no),
                                              ctypes.byref(el), ctypes.byref(nb)))
            d = mesh.spatial_dimension
            nodes = np.zeros((nl.value, d))
            conn = np.zeros((el.value, mesh.connectivity.shape[1]), dtype=np.int32)
            self.node_global = np.zeros(nl.value, dtype=np.int64)
            self.element_global = np.zeros(el.value, dtype=np.int64)
            _capi.check(L.akb_subdomain_mesh(h, _capi.ptr(nodes), _capi.ptr(conn),
                                             _capi.ptr(self.node_global),
                                             _capi.ptr(self.element_global)))
            self.neighbors = []
            for k in range(nb.value):
                r, ns, nr = ctypes.c_int(), ctypes.c_int64(), ctypes.c_int64()
                _capi.check(L.akb_subdomain_neighbor(h, k, ctypes.byref(r), ctypes.byref(ns),
                                                     ctypes.byref(nr)))
                send = np.zeros(ns.value, dtype=np.int32)
                recv = np.zeros(nr.value, dtype=np.int32)
                _capi.check(L.akb_subdomain_lists(h, k, _capi.ptr(send), _capi.ptr(recv)))
                self.neighbors.append((r.value, send, recv))
        finally:
            L.akb_subdomain_destroy(h)
        self.rank = rank
        self.n_owned = no.value
        self.mesh = Mesh(d, nodes, conn, mesh.element_type)

    @property
    def owned_global(self):
        return self.node_global[:self.n_owned]


class _Local:
    """A subdomain's model with its ghost nodes blocked."""

    def __init__(self, sub, dim):
        self.sub = sub
        self.model = SolidMechanicsModel(sub.mesh)
        self.dim = dim

    def set_blocked(self, blocked_global):
        b = np.asarray(blocked_global)[self.sub.node_global].astype(np.uint8)
        b[self.sub.n_owned:] = 1  # ghosts: moved only by their owner
        self.model.setNodal("blocked_dofs", b)

    def pack(self, idx_dev, buf_dev, n):
        _capi.check(_capi.lib().akb_model_halo_pack(self.model._h, ctypes.c_void_p(idx_dev), n,
                                                    ctypes.c_void_p(buf_dev)))

    def unpack(self, idx_dev, buf_dev, n):
        _capi.check(_capi.lib().akb_model_halo_unpack(self.model._h, ctypes.c_void_p(idx_dev),
                                                      n, ctypes.c_void_p(buf_dev)))


class _PartitionBase:
    """Global-array view over a list of local subdomain models."""

    def _setup(self, mesh, subs):
        self.mesh = mesh
        self.dim = mesh.spatial_dimension
        self.locals = [_Local(s, self.dim) for s in subs]
        self._blocked = np.zeros((mesh.getNbNodes(), self.dim), dtype=np.bool_)

    # -- set-up ------------------------------------------------------------------
    def addMaterial(self, type, **params):
        for lc in self.locals:
            lc.model.addMaterial(type, **params)

    def setElementMaterials(self, material_of_element):
        mat = np.asarray(material_of_element, dtype=np.int32)
        for lc in self.locals:
            lc.model.setElementMaterials(mat[lc.sub.element_global])

    def _init_locals(self, method, precision):
        for lc in self.locals:
            lc.model.initFull(method, precision=precision)
            lc.set_blocked(self._blocked)
        self.precision = precision

    # -- nodal arrays --------------------------------------------------------------
    def setNodal(self, name, values):
        values = np.asarray(values)
        if name == "blocked_dofs":
            self._blocked = values.astype(np.bool_).reshape(-1, self.dim).copy()
            for lc in self.locals:
                lc.set_blocked(self._blocked)
            return
        for lc in self.locals:
            lc.model.setNodal(name, values.reshape(-1, self.dim)[lc.sub.node_global])

    def _owned(self, name):
        """(global ids, values) of the owned nodes of the local subdomains,
        read without handing out the models' host mirrors (a mirror handed
        out is uploaded again before the next step, which would discard the
        exchanged ghost predictions)."""
        from .model import _FIELDS
        ids, vals = [], []
        L = _capi.lib()
        for lc in self.locals:
            m = lc.model
            m._sync_up()
            a = np.zeros((lc.sub.mesh.getNbNodes(), self.dim))
            _capi.check(L.akb_model_get_nodal(m._h, _FIELDS[name], _capi.ptr(a), a.nbytes))
            ids.append(lc.sub.owned_global)
            vals.append(a[:lc.sub.n_owned])
        return np.concatenate(ids), np.concatenate(vals)

    def getBlockedDOFs(self):
        return self._blocked

    def setPrescribedVelocityRamp(self, nodes, axis, v_max, ramp_steps):
        nodes = np.asarray(nodes)
        if nodes.dtype == np.bool_:
            nodes = np.nonzero(nodes)[0]
        self._blocked[nodes, axis] = True
        for lc in self.locals:
            local = np.nonzero(np.isin(lc.sub.node_global, nodes))[0]
            lc.model.setPrescribedVelocityRamp(local, axis, v_max, ramp_steps)
            lc.set_blocked(self._blocked)

    def setTimeStep(self, dt):
        for lc in self.locals:
            lc.model.setTimeStep(dt)

    def getTimeStep(self):
        return self.locals[0].model.getTimeStep()


class PartitionedModel(_PartitionBase):
    """The mesh split into nparts subdomains, all advanced on the current GPU
    with the per-step halo exchange of a multi-GPU run (device gather and
    scatter between the subdomain models).  Results are bit-identical to a
    SolidMechanicsModel of the whole mesh."""

    def __init__(self, mesh, nparts, part=None):
        self.nparts = int(nparts)
        self.part = partition_elements(mesh, nparts) if part is None else np.asarray(part, np.int32)
        self._setup(mesh, [Subdomain(mesh, self.part, nparts, r) for r in range(nparts)])

    def initFull(self, _analysis_method=_explicit_lumped_mass, precision="fp64"):
        self._init_locals(_analysis_method, precision)
        # the per-step exchange in the library (akb_exchange): one link per
        # directed pair (owner r -> holder s), the send list of r and the
        # receive list of s naming the same global nodes in the same order
        L = _capi.lib()
        handles = (ctypes.c_void_p * len(self.locals))(*[lc.model._h.value for lc in self.locals])
        self._x = ctypes.c_void_p()
        _capi.check(L.akb_exchange_create(handles, len(self.locals), ctypes.byref(self._x)))
        recv_of = {}
        for lc in self.locals:
            for r, send, recv in lc.sub.neighbors:
                recv_of[(r, lc.sub.rank)] = recv
        for lc in self.locals:
            r = lc.sub.rank
            for s, send, _ in lc.sub.neighbors:
                recv = np.ascontiguousarray(recv_of[(r, s)], dtype=np.int32)
                send = np.ascontiguousarray(send, dtype=np.int32)
                assert len(send) == len(recv)
                _capi.check(L.akb_exchange_add_link(self._x, r, s, _capi.ptr(send),
                                                    _capi.ptr(recv), len(send)))

    def setGraphSteps(self, steps):
        _capi.check(_capi.lib().akb_exchange_set_graph_steps(self._x, int(steps)))

    def getStableTimeStep(self):
        return min(lc.model.getStableTimeStep() for lc in self.locals)

    def solveStep(self, nsteps=1):
        for lc in self.locals:
            lc.model._sync_up()
        _capi.check(_capi.lib().akb_exchange_solve_step(self._x, int(nsteps)))
        for lc in self.locals:
            lc.model._invalidate()

    def timeSteps(self, nsteps):
        """nsteps steps of all subdomains timed on the device (ms), between
        events on the first subdomain's stream after a full synchronisation"""
        import torch
        L = _capi.lib()
        _capi.check(L.akb_exchange_synchronize(self._x))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        sp = ctypes.c_void_p()
        _capi.check(L.akb_model_stream(self.locals[0].model._h, ctypes.byref(sp)))
        st = torch.cuda.ExternalStream(sp.value)
        e0.record(st)
        # every subdomain's stream starts after e0 through the exchange's fork
        self.solveStep(nsteps)
        for lc in self.locals[1:]:
            sp2 = ctypes.c_void_p()
            _capi.check(L.akb_model_stream(lc.model._h, ctypes.byref(sp2)))
            ev = torch.cuda.Event()
            ev.record(torch.cuda.ExternalStream(sp2.value))
            st.wait_event(ev)
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1)

    def __del__(self):
        x = getattr(self, "_x", None)
        if x:
            _capi.lib().akb_exchange_destroy(x)
            self._x = None

    def getNodal(self, name):
        ids, vals = self._owned(name)
        out = np.zeros((self.mesh.getNbNodes(), self.dim))
        out[ids] = vals
        return out

    def getDisplacement(self):
        return self.getNodal("displacement")

    def getVelocity(self):
        return self.getNodal("velocity")

    def getAcceleration(self):
        return self.getNodal("acceleration")

    def getInternalForce(self):
        return self.getNodal("internal_force")

    def getMass(self):
        return self.getNodal("mass")


class DistributedModel(_PartitionBase):
    """Rank `torch.distributed.get_rank()`'s subdomain of the mesh (every rank
    partitions the whole mesh the same way, into world-size parts).  The
    per-step exchange runs over the process group: NCCL with device buffers
    on the model's stream, or gloo through host memory.  Getters return the
    whole-mesh array on every rank (gathered from the owners)."""

    def __init__(self, mesh, group=None, device=None):
        import torch
        import torch.distributed as dist
        self.dist, self.group = dist, group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.nccl = dist.get_backend(group) == "nccl"
        self.device = int(device) if device is not None else torch.cuda.current_device()
        _capi.check(_capi.lib().akb_set_device(self.device))
        torch.cuda.set_device(self.device)
        self.part = partition_elements(mesh, self.world)
        self._setup(mesh, [Subdomain(mesh, self.part, self.world, self.rank)])

    @property
    def local(self):
        return self.locals[0]

    def initFull(self, _analysis_method=_explicit_lumped_mass, precision="fp64"):
        import torch
        self._init_locals(_analysis_method, precision)
        dev = torch.device("cuda", self.device)
        self._lists = []
        for s, send, recv in self.local.sub.neighbors:
            self._lists.append((s, torch.from_numpy(send).to(dev), len(send),
                                torch.from_numpy(recv).to(dev), len(recv),
                                torch.empty(max(len(send), 1) * self.dim, dtype=torch.float64,
                                            device=dev),
                                torch.empty(max(len(recv), 1) * self.dim, dtype=torch.float64,
                                            device=dev)))
        torch.cuda.synchronize(self.device)
        sp = ctypes.c_void_p()
        _capi.check(_capi.lib().akb_model_stream(self.local.model._h, ctypes.byref(sp)))
        self._stream = torch.cuda.ExternalStream(sp.value, device=dev)
        # every rank takes part in the group's first collective before the
        # point-to-point exchanges between neighbors only
        self.dist.barrier(group=self.group)

    def getStableTimeStep(self):
        import torch
        dt = torch.tensor([self.local.model.getStableTimeStep()], dtype=torch.float64)
        if self.nccl:
            dt = dt.cuda(self.device)
        self.dist.all_reduce(dt, op=self.dist.ReduceOp.MIN, group=self.group)
        return float(dt.cpu()[0])

    def _exchange(self):
        import torch
        lc, dist = self.local, self.dist
        for s, send, ns, _, _, sbuf, _ in self._lists:
            lc.pack(send.data_ptr(), sbuf.data_ptr(), ns)
        if self.nccl:
            # the transfers are ordered after the packs on the model's stream,
            # and the unpacks after the transfers
            with torch.cuda.stream(self._stream):
                ops = []
                for s, _, ns, _, nr, sbuf, rbuf in self._lists:
                    ops.append(dist.P2POp(dist.isend, sbuf[:ns * self.dim], s, self.group))
                    ops.append(dist.P2POp(dist.irecv, rbuf[:nr * self.dim], s, self.group))
                if ops:
                    for w in dist.batch_isend_irecv(ops):
                        w.wait()
        else:
            lc.model.synchronize()
            reqs, hosts = [], []
            for s, _, ns, _, nr, sbuf, rbuf in self._lists:
                hs = sbuf[:ns * self.dim].cpu()
                hr = torch.empty(nr * self.dim, dtype=torch.float64)
                reqs.append(dist.isend(hs, s, group=self.group))
                reqs.append(dist.irecv(hr, s, group=self.group))
                hosts.append((hr, rbuf))
            for q in reqs:
                q.wait()
            for hr, rbuf in hosts:
                rbuf[:hr.numel()].copy_(hr)
            torch.cuda.synchronize(self.device)
        for s, _, _, recv, nr, _, rbuf in self._lists:
            lc.unpack(recv.data_ptr(), rbuf.data_ptr(), nr)

    def solveStep(self, nsteps=1):
        for _ in range(int(nsteps)):
            self._exchange()
            self.local.model.solveStep(1)
        self.local.model.synchronize()

    def getNodal(self, name):
        ids, vals = self._owned(name)
        parts = [None] * self.world
        self.dist.all_gather_object(parts, (ids, vals), group=self.group)
        out = np.zeros((self.mesh.getNbNodes(), self.dim))
        for i, v in parts:
            out[i] = v
        return out

    def getDisplacement(self):
        return self.getNodal("displacement")

    def getVelocity(self):
        return self.getNodal("velocity")

    def getAcceleration(self):
        return self.getNodal("acceleration")

    def getInternalForce(self):
        return self.getNodal("internal_force")

"""Partitioned meshes on the CPU: the partition and subdomain rules of
libakb (host code, no GPU), and the halo-exchange scheme run by gloo ranks
with the oracle as each rank's solver, compared bit for bit with the oracle
on the whole mesh."""
import multiprocessing as mp
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import akantu2_b200 as akb  # noqa: E402


def _meshes():
    return [("tet", akb.box_tet4(5, 4, 3)), ("hex", akb.box_hex8(6, 3, 4)),
            ("tri6", akb.square_tri6(7, 5))]


@pytest.mark.parametrize("nparts", [1, 2, 3, 5])
def test_partition_is_balanced_and_deterministic(nparts):
    for _, mesh in _meshes():
        p1 = akb.partition_elements(mesh, nparts)
        p2 = akb.partition_elements(mesh, nparts)
        assert np.array_equal(p1, p2)
        counts = np.bincount(p1, minlength=nparts)
        assert counts.sum() == mesh.getNbElement()
        assert counts.max() - counts.min() <= 1 + nparts  # bisection rounding


@pytest.mark.parametrize("nparts", [2, 3, 4])
def test_subdomains_cover_the_mesh_and_agree_on_halos(nparts):
    for _, mesh in _meshes():
        part = akb.partition_elements(mesh, nparts)
        subs = [akb.Subdomain(mesh, part, nparts, r) for r in range(nparts)]
        owned = np.concatenate([s.owned_global for s in subs])
        assert np.array_equal(np.sort(owned), np.arange(mesh.getNbNodes()))
        assert np.array_equal(np.unique(np.concatenate([s.element_global for s in subs])),
                              np.arange(mesh.getNbElement()))
        node_elems = [[] for _ in range(mesh.getNbNodes())]
        for e, row in enumerate(mesh.connectivity):
            for n in row:
                node_elems[n].append(e)
        for s in subs:
            # elements ascending; local connectivity maps back to the global one
            assert np.all(np.diff(s.element_global) > 0)
            assert np.array_equal(s.node_global[s.mesh.connectivity],
                                  mesh.connectivity[s.element_global])
            assert np.allclose(s.mesh.nodes, mesh.nodes[s.node_global])
            # every element of an owned node is local
            local = set(s.element_global.tolist())
            for n in s.owned_global:
                assert set(node_elems[n]) <= local
            for r, send, recv in s.neighbors:
                back = [x for x in subs[r].neighbors if x[0] == s.rank][0]
                assert np.array_equal(s.node_global[send], subs[r].node_global[back[2]])
                assert np.array_equal(s.node_global[recv], subs[r].node_global[back[1]])
                assert np.all(np.diff(s.node_global[send]) > 0)
            ghosts = s.node_global[s.n_owned:]
            recv_all = np.concatenate([s.node_global[recv] for _, _, recv in s.neighbors]) \
                if s.neighbors else np.zeros(0, np.int64)
            assert np.array_equal(np.sort(recv_all), np.sort(ghosts))


def test_bad_arguments_are_rejected():
    mesh = akb.box_tet4(2)
    with pytest.raises(akb.AkbError):
        akb.partition_elements(mesh, 0)
    part = akb.partition_elements(mesh, 2)
    with pytest.raises(akb.AkbError):
        akb.Subdomain(mesh, part, 2, 2)
    bad = part.copy()
    bad[0] = 7
    with pytest.raises(akb.AkbError):
        akb.Subdomain(mesh, bad, 2, 0)


# -- the exchange scheme with gloo ranks, the oracle solving each subdomain -------------
MAT = dict(type="neohookean", rho=1.0, E=1.0, nu=0.3)


def _problem(kind):
    from oracle import oracle as orc
    mesh = {"tet": lambda: akb.box_tet4(6, 5, 4), "hex": lambda: akb.box_hex8(6, 4, 5)}[kind]()
    otype = {"tet": orc.TET4, "hex": orc.HEX8}[kind]
    x = mesh.nodes
    v0 = np.zeros_like(x)
    v0[:, 2] = 0.02 * np.sin(np.pi * x[:, 0]) * np.sin(2 * np.pi * x[:, 1]) * x[:, 2]
    v0[:, 0] = 0.01 * np.cos(np.pi * x[:, 2])
    bl = np.zeros(x.shape, np.uint8)
    bl[np.isclose(x[:, 2], 0.0)] = 1
    return mesh, otype, v0, bl


def _serial(kind, steps):
    from oracle import oracle as orc
    mesh, otype, v0, bl = _problem(kind)
    o = orc.OracleModel(otype, mesh.nodes, mesh.connectivity, [MAT])
    o.set(orc.V, v0)
    o.set(orc.BLOCKED, bl)
    dt = 0.8 * o.stable_dt()
    o.set_dt(dt)
    o.step(steps)
    return dt, o.get(orc.U), o.get(orc.V), o.get(orc.FINT)


def _rank(rank, world, port, kind, steps, dt, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    from oracle import oracle as orc
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mesh, otype, v0, bl = _problem(kind)
        part = akb.partition_elements(mesh, world)
        sub = akb.Subdomain(mesh, part, world, rank)
        g = sub.node_global
        o = orc.OracleModel(otype, sub.mesh.nodes, sub.mesh.connectivity, [MAT])
        o.set(orc.V, v0[g])
        o.set(orc.BLOCKED, bl[g])
        o.set_dt(dt)
        fields = (orc.U, orc.V, orc.A)
        for _ in range(steps):
            o.step(1)
            # owners send u, v, a of their nodes that are ghosts elsewhere;
            # ghosts take them (the ghost's own update used partial forces)
            state = [o.get(f) for f in fields]
            reqs, incoming = [], []
            for r, send, recv in sub.neighbors:
                buf = torch.from_numpy(np.concatenate([s[send] for s in state], axis=1).copy())
                reqs.append(dist.isend(buf, r))
                rb = torch.empty((len(recv), 3 * sub.mesh.spatial_dimension), dtype=torch.float64)
                reqs.append(dist.irecv(rb, r))
                incoming.append((recv, rb))
            for q in reqs:
                q.wait()
            d = sub.mesh.spatial_dimension
            for recv, rb in incoming:
                for k, f in enumerate(fields):
                    state[k][recv] = rb.numpy()[:, k * d:(k + 1) * d]
            for k, f in enumerate(fields):
                o.set(f, state[k])
        n = sub.n_owned
        out.put((rank, g[:n], o.get(orc.U)[:n], o.get(orc.V)[:n], o.get(orc.FINT)[:n]))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("kind,world", [("tet", 2), ("hex", 3)])
def test_gloo_ranks_match_the_whole_mesh_bit_for_bit(kind, world):
    steps = 40
    dt, u, v, f = _serial(kind, steps)
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, kind, steps, dt, out))
             for r in range(world)]
    for p in procs:
        p.start()
    res = [out.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    U, V, F = np.full_like(u, np.nan), np.full_like(v, np.nan), np.full_like(f, np.nan)
    for _, ids, uu, vv, ff in res:
        U[ids], V[ids], F[ids] = uu, vv, ff
    assert np.max(np.abs(u)) > 0
    assert np.array_equal(U, u) and np.array_equal(V, v) and np.array_equal(F, f)

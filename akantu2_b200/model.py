"""SolidMechanicsModel for the explicit lumped-mass path, over libakb.

Mirrors the reference's Python binding (python/py_solid_mechanics_model.cc:
57-173, python/py_model.cc:131-137): initFull, getStableTimeStep,
setTimeStep, solveStep and the nodal-array getters.  The arrays live on the
GPU; the getters return host copies that the model refreshes after each step
and uploads again before the next step, so a script that edits the array it
got (boundary values, initial velocity, external force) behaves as with the
reference's zero-copy views.
"""
import ctypes

import numpy as np

from . import _capi
from .mesh import Mesh, TYPE_IDS

_explicit_lumped_mass = "_explicit_lumped_mass"
_x, _y, _z = 0, 1, 2

_FIELDS = {
    "displacement": _capi.DISPLACEMENT, "velocity": _capi.VELOCITY,
    "acceleration": _capi.ACCELERATION, "external_force": _capi.EXTERNAL_FORCE,
    "internal_force": _capi.INTERNAL_FORCE, "mass": _capi.MASS,
    "blocked_dofs": _capi.BLOCKED_DOFS, "current_position": _capi.CURRENT_POSITION,
    "previous_displacement": _capi.PREVIOUS_DISPLACEMENT,
    "displacement_increment": _capi.DISPLACEMENT_INCREMENT,
}
_LAW_IDS = {"elastic": 0, "neohookean": 1, "plastic_linear_isotropic_hardening": 2,
            "plastic": 2}
_WRITABLE = ("displacement", "velocity", "acceleration", "external_force", "blocked_dofs")


class _Parser:
    """getStaticParser(): the parsed .dat texts, in parse order."""

    def __init__(self):
        self.texts = []

    def parse(self, path):
        with open(path) as f:
            self.texts.append(f.read())

    def parse_text(self, text):
        self.texts.append(text)

    def clear(self):
        self.texts = []


_static_parser = _Parser()


def getStaticParser():
    return _static_parser


def parseInput(path):
    """akantu.parseInput: add the sections of a .dat file to the static parser."""
    _static_parser.parse(path)


class FixedValue:
    """BC::Dirichlet::FixedValue(value, axis)  (boundary_condition_functor_inline_impl.hh:53-61)."""

    def __init__(self, value, axis):
        self.value = value
        self.axis = axis


class FromHigherDim:
    """BC::Neumann::FromHigherDim(stress): the traction stress . n on the
    boundary facets of a group (boundary_condition_functor.hh)."""

    def __init__(self, stress):
        self.stress = np.asarray(stress, dtype=np.float64)


def neumann_forces(mesh, group_nodes, stress):
    """Nodal forces [N, dim] of FromHigherDim(stress) on the boundary facets
    whose nodes all belong to group_nodes (akb_mesh_neumann_forces)."""
    d = mesh.spatial_dimension
    nodes = np.ascontiguousarray(group_nodes, dtype=np.int32)
    sig = np.asfortranarray(np.asarray(stress, dtype=np.float64).reshape(d, d))
    sig_cm = np.ascontiguousarray(sig.T).reshape(-1)  # column-major
    out = np.zeros((mesh.getNbNodes(), d))
    _capi.check(_capi.lib().akb_mesh_neumann_forces(
        TYPE_IDS[mesh.element_type], _capi.ptr(mesh.nodes), mesh.getNbNodes(),
        _capi.ptr(mesh.connectivity), mesh.getNbElement(), _capi.ptr(nodes), nodes.size,
        _capi.ptr(sig_cm), _capi.ptr(out)))
    return out


class MaterialSelector:
    """Element -> material index (ConstitutiveLawSelector,
    src/model/common/constitutive_laws/constitutive_law_selector.hh:45-86):
    the fallback value, or a fallback selector, for every element."""

    def __init__(self):
        self.fallback_value = 0
        self.fallback_selector = None

    def setFallback(self, f):
        if isinstance(f, MaterialSelector):
            self.fallback_selector = f
        else:
            self.fallback_value = int(f)

    def getFallbackValue(self):
        return self.fallback_value

    def _fallback(self, model, elements):
        if self.fallback_selector is not None:
            return self.fallback_selector.select(model)[elements]
        return np.full(len(elements), self.fallback_value, dtype=np.int32)

    def select(self, model):
        """the material index of every element of the model's mesh"""
        return self._fallback(model, np.arange(model.mesh.getNbElement()))


class ElementDataMaterialSelector(MaterialSelector):
    """ElementDataConstitutiveLawSelector (constitutive_law_selector.hh:119-142,
    constitutive_law_selector_tmpl.hh:8-20): a string datum is the name of the
    element's material, an integer datum its index; an element whose name
    names no material takes the fallback."""

    def __init__(self, element_data, model=None, first_index=1):
        super().__init__()
        self.element_data = np.asarray(element_data)
        self.first_index = first_index

    def _data(self, model):
        return self.element_data

    def select(self, model):
        data = self._data(model)
        n = model.mesh.getNbElement()
        if len(data) != n:
            raise ValueError("element data must have one entry per element")
        if data.dtype.kind in "iu":
            return data.astype(np.int32)
        index = {model.getMaterial(i).getName(): i for i in range(model.getNbMaterials())}
        out = np.array([index.get(str(d), -1) for d in data], dtype=np.int32)
        miss = np.nonzero(out < 0)[0]
        if len(miss):
            out[miss] = self._fallback(model, miss)
        return out


class MeshDataMaterialSelector(ElementDataMaterialSelector):
    """MeshDataConstitutiveLawSelector (constitutive_law_selector.hh:144-150):
    the selector of the mesh's element data of that name, e.g.
    MeshDataMaterialSelector("physical_names", model) for a gmsh file whose
    physical names are the material names."""

    def __init__(self, name, model, first_index=1):
        super().__init__(model.mesh.getData(name), model, first_index)
        self.name = name


# the reference's Python names (python/py_constitutive_law_selector.cc:95-96)
MeshDataMaterialSelectorString = MeshDataMaterialSelector
MeshDataMaterialSelectorInt = MeshDataMaterialSelector


class Material:
    """View of one material of a model (src/model/solid_mechanics/material.hh)."""

    def __init__(self, model, index):
        self._model = model
        self._index = index

    def get(self, name):
        v = ctypes.c_double()
        _capi.check(_capi.lib().akb_model_get_material_param(
            self._model._h, self._index, name.encode(), ctypes.byref(v)))
        return v.value

    getParam = get

    def getRho(self):
        return self.get("rho")

    def getName(self):
        buf = ctypes.create_string_buffer(256)
        _capi.check(_capi.lib().akb_model_get_material_name(self._model._h, self._index, buf, 256))
        return buf.value.decode()

    def _qp(self, field):
        m = self._model
        m._sync_up()
        n = ctypes.c_int64()
        L = _capi.lib()
        _capi.check(L.akb_model_qp_field_size(m._h, field, self._index, ctypes.byref(n)))
        out = np.zeros(n.value)
        _capi.check(L.akb_model_get_qp_field(m._h, field, self._index, _capi.ptr(out), n.value))
        if field in (_capi.ISO_HARDENING, _capi.PLASTIC_ENERGY):
            return out.reshape(-1, 1)
        return out.reshape(-1, m.dim * m.dim)

    def getElementFilter(self, element_type=None):
        """elements of the mesh that this material holds"""
        return np.nonzero(self._model._element_materials() == self._index)[0]

    def getStress(self, element_type=None):
        return self._qp(_capi.STRESS)

    def getGradU(self, element_type=None):
        return self._qp(_capi.GRAD_U)

    _INTERNALS = {"stress": _capi.STRESS, "grad_u": _capi.GRAD_U,
                  "piola_kirchhoff_2": _capi.PIOLA_KIRCHHOFF_2,
                  "inelastic_strain": _capi.INELASTIC_STRAIN,
                  "iso_hardening": _capi.ISO_HARDENING, "plastic_energy": _capi.PLASTIC_ENERGY,
                  "eigen_grad_u": _capi.EIGEN_GRAD_U}

    def getInternal(self, name):
        fid = self._INTERNALS[name]
        return lambda element_type=None: self._qp(fid)

    def setInternal(self, name, values, element_type=None):
        """Writes a quadrature-point internal ([points][dim*dim], the getter's
        layout); the reference assigns getInternal<Real>(name)(type) in place
        (test_solid_mechanics_model_material_eigenstrain.cc:127-136).  Only
        "eigen_grad_u" is writable."""
        m = self._model
        fid = self._INTERNALS[name]
        n = ctypes.c_int64()
        L = _capi.lib()
        _capi.check(L.akb_model_qp_field_size(m._h, fid, self._index, ctypes.byref(n)))
        a = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
        if a.size != n.value:
            raise ValueError(f"{name} holds {n.value} values, got {a.size}")
        _capi.check(L.akb_model_set_qp_field(m._h, fid, self._index, _capi.ptr(a), n.value))


class SolidMechanicsModel:
    """Explicit lumped-mass SolidMechanicsModel on one GPU."""

    def __init__(self, mesh, dim=None, id="solid_mechanics_model"):
        if not isinstance(mesh, Mesh):
            raise TypeError("mesh must be an akantu2_b200.Mesh")
        self.mesh = mesh
        self.dim = mesh.spatial_dimension if dim is None else dim
        self.id = id
        L = _capi.lib()
        h = ctypes.c_void_p()
        _capi.check(L.akb_model_create(self.dim, TYPE_IDS[mesh.element_type],
                                       _capi.ptr(mesh.nodes), mesh.getNbNodes(),
                                       _capi.ptr(mesh.connectivity), mesh.getNbElement(),
                                       ctypes.byref(h)))
        self._h = h
        self._mirrors = {}
        self._handed_out = set()
        self._initialized = False
        self._materials_added = False

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _capi.lib().akb_model_destroy(h)
            self._h = None

    # -- set-up ------------------------------------------------------------------
    def addMaterial(self, type, **params):
        """Adds one material (alternative to a parsed .dat file)."""
        def fmt(v):
            if isinstance(v, (bool, np.bool_)):
                return "true" if v else "false"
            if isinstance(v, (list, tuple, np.ndarray)):  # a matrix: rows in brackets
                rows = np.atleast_2d(np.asarray(v, dtype=np.float64))
                return "[" + ", ".join("[" + ", ".join(repr(float(x)) for x in r) + "]"
                                       for r in rows) + "]"
            return repr(float(v)) if isinstance(v, (int, float, np.floating)) else str(v)
        text = "\n".join(f"{k} = {fmt(v)}" for k, v in params.items())
        _capi.check(_capi.lib().akb_model_add_material(self._h, type.encode(), text.encode()))
        self._materials_added = True

    def setElementMaterials(self, material_of_element):
        self._mat = np.ascontiguousarray(material_of_element, dtype=np.int32)
        _capi.check(_capi.lib().akb_model_set_element_materials(self._h, _capi.ptr(self._mat)))

    def setMaterialSelector(self, selector):
        """setMaterialSelector (constitutive_laws_handler.hh:251): applied at
        initFull, once the materials are known"""
        if self._initialized:
            raise _capi.AkbError(7, "the material selector must be set before initFull")
        self._selector = selector

    def getMaterialSelector(self):
        return getattr(self, "_selector", None)

    def _element_materials(self):
        mat = getattr(self, "_mat", None)
        return np.zeros(self.mesh.getNbElement(), np.int32) if mat is None else mat

    def setQuadratureRule(self, rule):
        """0: the reference's default order; 1: the 6-point rule of _triangle_6."""
        _capi.check(_capi.lib().akb_model_set_quadrature_rule(self._h, rule))

    def initFull(self, _analysis_method=_explicit_lumped_mass, precision="fp64"):
        if _analysis_method != _explicit_lumped_mass:
            raise _capi.AkbError(8, "only _explicit_lumped_mass is provided")
        L = _capi.lib()
        if not self._materials_added:
            for text in _static_parser.texts:
                _capi.check(L.akb_model_load_materials(self._h, text.encode()))
        if getattr(self, "_selector", None) is not None:
            self.setElementMaterials(self._selector.select(self))
        prec = {"fp64": _capi.PRECISION_FP64, "mixed": _capi.PRECISION_MIXED,
                "fp64_fast": _capi.PRECISION_FP64_FAST}[precision]
        _capi.check(L.akb_model_init_full(self._h, _capi.EXPLICIT_LUMPED_MASS, prec))
        self._initialized = True
        self.precision = precision

    # -- nodal arrays ----------------------------------------------------------------
    def _get(self, name):
        a = self._mirrors.get(name)
        if a is None:
            shape = (self.mesh.getNbNodes(), self.dim)
            a = np.zeros(shape, dtype=np.bool_ if name == "blocked_dofs" else np.float64)
            view = a.view(np.uint8) if name == "blocked_dofs" else a
            _capi.check(_capi.lib().akb_model_get_nodal(self._h, _FIELDS[name], _capi.ptr(view),
                                                        view.nbytes))
            self._mirrors[name] = a
        if name in _WRITABLE:
            self._handed_out.add(name)
        return a

    def _sync_up(self):
        """Uploads the host arrays handed out since the last step."""
        L = _capi.lib()
        for name in list(self._handed_out):
            a = self._mirrors[name]
            view = np.ascontiguousarray(a).view(np.uint8) if name == "blocked_dofs" else \
                np.ascontiguousarray(a, dtype=np.float64)
            _capi.check(L.akb_model_set_nodal(self._h, _FIELDS[name], _capi.ptr(view), view.nbytes))
        self._handed_out.clear()

    def _invalidate(self, names=None):
        if names is None:
            self._mirrors.clear()
        else:
            for n in names:
                self._mirrors.pop(n, None)

    def getDisplacement(self):
        return self._get("displacement")

    def getVelocity(self):
        return self._get("velocity")

    def getAcceleration(self):
        return self._get("acceleration")

    def getExternalForce(self):
        return self._get("external_force")

    def getInternalForce(self):
        self._sync_up()
        return self._get("internal_force")

    def getMass(self):
        return self._get("mass")

    def getBlockedDOFs(self):
        return self._get("blocked_dofs")

    def setAffineKernel(self, on=True):
        """Mixed hexahedra of a mesh of parallelepipeds: the element kernel
        compiled without per-point geometry (True or 1), the same reading each
        element's adjugate and 1/det from a table formed once (2), or the
        general kernel (False or 0); the same numbers in every mode."""
        mode = on if isinstance(on, int) and not isinstance(on, bool) else int(bool(on))
        _capi.check(_capi.lib().akb_model_set_affine_kernel(self._h, mode))

    def getAffineKernel(self):
        """0 (general kernel), 1 or 2 (the modes of setAffineKernel)"""
        on = ctypes.c_int()
        _capi.check(_capi.lib().akb_model_get_affine_kernel(self._h, ctypes.byref(on)))
        return on.value

    def setIncrementTracking(self, on=True):
        """Keep the displacement each step starts from and its increment
        (getPreviousDisplacement, getIncrement); off by default, one extra
        launch per step when on (akb_model_set_increment_tracking)."""
        self._sync_up()
        _capi.check(_capi.lib().akb_model_set_increment_tracking(self._h, int(bool(on))))
        self._invalidate(["previous_displacement", "displacement_increment"])

    def getPreviousDisplacement(self):
        """SolidMechanicsModel::getPreviousDisplacement: u at the start of
        the last step (increment tracking on)."""
        self._sync_up()
        return self._get("previous_displacement")

    def getIncrement(self):
        """SolidMechanicsModel::getIncrement: u_{n+1} - u_n of the last step
        (increment tracking on)."""
        self._sync_up()
        return self._get("displacement_increment")

    def getCurrentPosition(self):
        self._sync_up()
        self._invalidate(["current_position"])
        return self._get("current_position")

    def setNodalAsync(self, name, pinned):
        """Asynchronous upload of a whole nodal array from a pinned host array
        (akb_model_set_nodal_async); the array may be reused once a read
        enqueued after the next step has been waited for, or after the next
        synchronize()."""
        self._sync_up()
        _capi.check(_capi.lib().akb_model_set_nodal_async(self._h, _FIELDS[name], _capi.ptr(pinned),
                                                          pinned.nbytes))
        self._invalidate([name, "current_position"])

    def getNodalAsync(self, name, pinned):
        """Asynchronous read of a nodal array into a pinned host array; returns
        a ticket for waitNodalAsync (akb_model_get_nodal_async).  The
        ASYNC_READS_IN_FLIGHT most recent tickets can be waited on one by one:
        waiting for each step's read that many steps minus one later lets the
        copies of consecutive steps run back to back."""
        t = ctypes.c_int64()
        _capi.check(_capi.lib().akb_model_get_nodal_async(self._h, _FIELDS[name], _capi.ptr(pinned),
                                                          pinned.nbytes, ctypes.byref(t)))
        return t.value

    def waitNodalAsync(self, ticket):
        _capi.check(_capi.lib().akb_model_wait_nodal_async(self._h, int(ticket)))

    def setNodal(self, name, values):
        """Direct upload of a whole nodal array."""
        self._sync_up()
        a = np.ascontiguousarray(values, dtype=np.uint8 if name == "blocked_dofs" else np.float64)
        _capi.check(_capi.lib().akb_model_set_nodal(self._h, _FIELDS[name], _capi.ptr(a), a.nbytes))
        self._invalidate([name, "current_position"])

    def applyBC(self, bc, group):
        """applyBC(FixedValue(v, axis), group): blocks the axis of the group's
        nodes and sets their displacement; applyBC(FromHigherDim(stress),
        group): adds the boundary traction to the external force
        (boundary_condition_tmpl.hh)."""
        nodes = self.mesh.getNodeGroup(group) if isinstance(group, str) else np.asarray(group)
        if isinstance(bc, FromHigherDim):
            self.getExternalForce()[:] += neumann_forces(self.mesh, nodes, bc.stress)
            return
        if not isinstance(bc, FixedValue):
            raise TypeError("applyBC takes FixedValue or FromHigherDim")
        self.getBlockedDOFs()[nodes, bc.axis] = True
        self.getDisplacement()[nodes, bc.axis] = bc.value

    # -- time stepping -----------------------------------------------------------------
    def getStableTimeStep(self):
        self._sync_up()
        dt = ctypes.c_double()
        _capi.check(_capi.lib().akb_model_get_stable_time_step(self._h, ctypes.byref(dt)))
        return dt.value

    def setTimeStep(self, dt, solver_id=""):
        _capi.check(_capi.lib().akb_model_set_time_step(self._h, float(dt)))

    def getTimeStep(self, solver_id=""):
        dt = ctypes.c_double()
        _capi.check(_capi.lib().akb_model_get_time_step(self._h, ctypes.byref(dt)))
        return dt.value

    def solveStep(self, nsteps=1):
        """ModelSolver::solveStep; nsteps > 1 enqueues several steps at once."""
        self._sync_up()
        _capi.check(_capi.lib().akb_model_solve_step(self._h, int(nsteps)))
        self._invalidate()

    def timeSteps(self, nsteps):
        """Runs nsteps steps between two CUDA events on the model's stream;
        returns the device time in milliseconds."""
        self._sync_up()
        ms = ctypes.c_double()
        _capi.check(_capi.lib().akb_model_time_steps(self._h, int(nsteps), ctypes.byref(ms)))
        self._invalidate()
        return ms.value

    def profileSteps(self, nsteps):
        """Like timeSteps with events between phases; returns (total_ms,
        [predictor_ms, element_forces_ms, node_update_ms]) summed over steps."""
        self._sync_up()
        total = ctypes.c_double()
        phases = (ctypes.c_double * 3)()
        _capi.check(_capi.lib().akb_model_profile_steps(self._h, int(nsteps), ctypes.byref(total),
                                                        phases))
        self._invalidate()
        return total.value, list(phases)

    def setPersistent(self, mode):
        """0: never, 1: small single-law meshes (default), 2: whenever allowed
        -- whole step sequences in one persistent launch (akb_model_set_persistent)."""
        _capi.check(_capi.lib().akb_model_set_persistent(self._h, int(mode)))

    def persistentActive(self):
        a = ctypes.c_int()
        _capi.check(_capi.lib().akb_model_persistent_active(self._h, ctypes.byref(a)))
        return bool(a.value)

    def prepareGraphs(self):
        """Captures the step graph the next solveStep launches, so that the
        capture is not paid inside a timed run (akb_model_prepare_graphs)."""
        self._sync_up()
        _capi.check(_capi.lib().akb_model_prepare_graphs(self._h))

    def setGraphSteps(self, steps):
        """Multi-step runs are replayed as CUDA graphs of `steps` steps (even; 0 disables)."""
        _capi.check(_capi.lib().akb_model_set_graph_steps(self._h, int(steps)))

    def synchronize(self):
        _capi.check(_capi.lib().akb_model_synchronize(self._h))

    def assembleInternalForces(self):
        self._sync_up()
        _capi.check(_capi.lib().akb_model_assemble_internal_forces(self._h))
        self._invalidate(["internal_force"])

    def getEnergy(self, energy_id):
        self._sync_up()
        v = ctypes.c_double()
        _capi.check(_capi.lib().akb_model_get_energy(self._h, energy_id.encode(), ctypes.byref(v)))
        return v.value

    def setPrescribedVelocityRamp(self, nodes, axis, v_max, ramp_steps):
        """Blocks `axis` of `nodes` and, before every later step k, sets their
        displacement to u_now + sum_{j<=k} dt v_max min(1, j / ramp_steps) on
        the device (akb_model_set_prescribed_velocity_ramp)."""
        self._sync_up()
        nodes = np.asarray(nodes)
        if nodes.dtype == np.bool_:
            nodes = np.nonzero(nodes)[0]
        dofs = np.ascontiguousarray(nodes.astype(np.int64) * self.dim + int(axis))
        _capi.check(_capi.lib().akb_model_set_prescribed_velocity_ramp(
            self._h, _capi.ptr(dofs), dofs.size, float(v_max), int(ramp_steps)))
        self._invalidate(["blocked_dofs"])

    def autotune(self, repeats=5):
        """Picks the fastest launch shapes of the step kernels on the current
        state (akb_model_autotune); results are unchanged by the choice."""
        self._sync_up()
        _capi.check(_capi.lib().akb_model_autotune(self._h, int(repeats)))

    def getLaunchShape(self, law):
        """(element threads per block, points per iteration, min blocks per SM,
        node threads per block) of the law group `law` ("elastic",
        "neohookean", "plastic...")."""
        b, q, mb, n = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _capi.check(_capi.lib().akb_model_get_launch_shape(
            self._h, _LAW_IDS[law], ctypes.byref(b), ctypes.byref(q), ctypes.byref(mb),
            ctypes.byref(n)))
        return b.value, q.value, mb.value, n.value

    def setLaunchShape(self, law, element_block, points_per_iteration, node_block, min_blocks=1):
        _capi.check(_capi.lib().akb_model_set_launch_shape(self._h, _LAW_IDS[law],
                                                           int(element_block),
                                                           int(points_per_iteration),
                                                           int(min_blocks), int(node_block)))

    def setPrefetch(self, law, waves):
        """L2 prefetch distance (waves of resident blocks, 0 = off) of the
        packed hexahedron kernel of the law group `law`; results are
        unchanged by it."""
        _capi.check(_capi.lib().akb_model_set_prefetch(self._h, _LAW_IDS[law], int(waves)))

    def getPrefetch(self, law):
        w = ctypes.c_int()
        _capi.check(_capi.lib().akb_model_get_prefetch(self._h, _LAW_IDS[law], ctypes.byref(w)))
        return w.value

    def setRecomputeGeometry(self, law, on=True):
        """Tetrahedra and triangles: recompute dN/dx and det J w from the
        coordinates every step (the precomputation's arithmetic) instead of
        streaming the tables; results are unchanged by it."""
        _capi.check(_capi.lib().akb_model_set_recompute_geometry(self._h, _LAW_IDS[law],
                                                                 int(bool(on))))

    def getRecomputeGeometry(self, law):
        w = ctypes.c_int()
        _capi.check(_capi.lib().akb_model_get_recompute_geometry(self._h, _LAW_IDS[law],
                                                                 ctypes.byref(w)))
        return bool(w.value)

    def setStreamedPoints(self, law, on=True):
        """Plain FP64 hexahedra: the per-point kernel with the streamed law
        (dN/dx rows loaded where used, forces sent to shared memory as formed;
        fewer registers) or with the point's row and forces held in
        registers; results are unchanged by it."""
        _capi.check(_capi.lib().akb_model_set_streamed_points(self._h, _LAW_IDS[law],
                                                              int(bool(on))))

    def getStreamedPoints(self, law):
        w = ctypes.c_int()
        _capi.check(_capi.lib().akb_model_get_streamed_points(self._h, _LAW_IDS[law],
                                                              ctypes.byref(w)))
        return bool(w.value)

    def setNodeShape(self, node_block, staged=0):
        """Threads per block of the node update, and its form: 0 the direct
        gather, 1 (True) the gather staged through shared memory, 2 the direct
        gather with each node's state read first; results are unchanged by
        either."""
        _capi.check(_capi.lib().akb_model_set_node_shape(self._h, int(node_block), int(staged)))

    def getNodeShape(self):
        b, st = ctypes.c_int(), ctypes.c_int()
        _capi.check(_capi.lib().akb_model_get_node_shape(self._h, ctypes.byref(b), ctypes.byref(st)))
        return b.value, st.value

    def setDependentLaunch(self, on=True):
        """Step kernels launched with programmatic stream serialization (each
        scheduled while its predecessor drains); results are unchanged."""
        _capi.check(_capi.lib().akb_model_set_dependent_launch(self._h, int(bool(on))))

    def getDependentLaunch(self):
        on = ctypes.c_int()
        _capi.check(_capi.lib().akb_model_get_dependent_launch(self._h, ctypes.byref(on)))
        return bool(on.value)

    def getDeviceBytes(self):
        """Device memory held by the model."""
        b = ctypes.c_int64()
        _capi.check(_capi.lib().akb_model_device_bytes(self._h, ctypes.byref(b)))
        return b.value

    def getStatus(self):
        f = ctypes.c_int()
        _capi.check(_capi.lib().akb_model_get_status(self._h, ctypes.byref(f)))
        return f.value

    def getFEData(self):
        """(dN/dx [E, nq, n, dim], det J * w [E, nq]) in user element order."""
        L = _capi.lib()
        nq = ctypes.c_int()
        _capi.check(L.akb_model_nb_quadrature_points(self._h, ctypes.byref(nq)))
        E, n = self.mesh.getNbElement(), self.mesh.connectivity.shape[1]
        B = np.zeros((E, nq.value, n, self.dim))
        j = np.zeros((E, nq.value))
        _capi.check(L.akb_model_get_fe_data(self._h, 0, _capi.ptr(B), B.size))
        _capi.check(L.akb_model_get_fe_data(self._h, 1, _capi.ptr(j), j.size))
        return B, j

    # -- materials ------------------------------------------------------------------
    def getNbMaterials(self):
        c = ctypes.c_int()
        _capi.check(_capi.lib().akb_model_nb_materials(self._h, ctypes.byref(c)))
        return c.value

    def getMaterial(self, which=0):
        if isinstance(which, str):
            for i in range(self.getNbMaterials()):
                if Material(self, i).getName() == which:
                    return Material(self, i)
            raise _capi.AkbError(10, f"no material named '{which}'")
        return Material(self, which)

    def getSpatialDimension(self):
        return self.dim


class BatchModel(SolidMechanicsModel):
    """Many independent meshes of one element type advanced together
    (akb_batch_create).  The nodal arrays are the instances' arrays one after
    the other; ``instance_nodes(k)`` / ``instance_elements(k)`` give the
    slices of instance k.  Each instance may have its own material
    (``setInstanceMaterials``) and its own time step (``setTimeSteps``)."""

    def __init__(self, meshes, dim=None, id="solid_mechanics_batch"):
        meshes = list(meshes)
        if not meshes or not all(isinstance(m, Mesh) for m in meshes):
            raise TypeError("meshes must be a non-empty list of akantu2_b200.Mesh")
        et = meshes[0].element_type
        if any(m.element_type != et for m in meshes):
            raise ValueError("all instances of a batch have the same element type")
        sd = meshes[0].spatial_dimension
        nn = np.array([m.getNbNodes() for m in meshes], dtype=np.int64)
        ne = np.array([m.getNbElement() for m in meshes], dtype=np.int64)
        self.node_offsets = np.concatenate([[0], np.cumsum(nn)]).astype(np.int64)
        self.element_offsets = np.concatenate([[0], np.cumsum(ne)]).astype(np.int64)
        nodes = np.ascontiguousarray(np.concatenate([m.nodes for m in meshes]), dtype=np.float64)
        local = np.ascontiguousarray(np.concatenate([m.connectivity for m in meshes]),
                                     dtype=np.int32)
        combined = Mesh(sd)
        combined.set(nodes, local + np.repeat(self.node_offsets[:-1], ne)[:, None].astype(np.int32),
                     et)
        self.mesh = combined
        self.meshes = meshes
        self.dim = sd if dim is None else dim
        self.id = id
        L = _capi.lib()
        h = ctypes.c_void_p()
        _capi.check(L.akb_batch_create(self.dim, TYPE_IDS[et], len(meshes), _capi.ptr(nn),
                                       _capi.ptr(ne), _capi.ptr(nodes), _capi.ptr(local),
                                       ctypes.byref(h)))
        self._h = h
        self._mirrors = {}
        self._handed_out = set()
        self._initialized = False
        self._materials_added = False

    @property
    def nb_instances(self):
        return len(self.meshes)

    def instance_nodes(self, k):
        return slice(int(self.node_offsets[k]), int(self.node_offsets[k + 1]))

    def instance_elements(self, k):
        return slice(int(self.element_offsets[k]), int(self.element_offsets[k + 1]))

    def setInstanceMaterials(self, material_of_instance):
        self._imat = np.ascontiguousarray(material_of_instance, dtype=np.int32)
        _capi.check(_capi.lib().akb_batch_set_instance_materials(self._h, _capi.ptr(self._imat)))

    def getStableTimeSteps(self):
        self._sync_up()
        dt = np.zeros(self.nb_instances)
        _capi.check(_capi.lib().akb_batch_get_stable_time_steps(self._h, _capi.ptr(dt)))
        return dt

    def setTimeSteps(self, dt):
        dt = np.ascontiguousarray(dt, dtype=np.float64)
        if dt.shape != (self.nb_instances,):
            raise ValueError("one time step per instance")
        _capi.check(_capi.lib().akb_batch_set_time_steps(self._h, _capi.ptr(dt)))

    def getTimeSteps(self):
        dt = np.zeros(self.nb_instances)
        _capi.check(_capi.lib().akb_batch_get_time_steps(self._h, _capi.ptr(dt)))
        return dt

    def setInstanceSteps(self, steps):
        """From the current step on, instance k advances exactly steps[k] more
        steps (negative: its limit stays as it is, initially none), then
        keeps its u, v and a while the others go on
        (akb_batch_set_instance_steps)."""
        self._sync_up()
        st = np.ascontiguousarray(steps, dtype=np.int64)
        if st.shape != (self.nb_instances,):
            raise ValueError("one step count per instance")
        _capi.check(_capi.lib().akb_batch_set_instance_steps(self._h, _capi.ptr(st)))

    def getInstanceStepsLeft(self):
        left = np.zeros(self.nb_instances, dtype=np.int64)
        _capi.check(_capi.lib().akb_batch_instance_steps_left(self._h, _capi.ptr(left)))
        return left

    def getInstanceNodal(self, field, k):
        """one instance's displacement, velocity or acceleration, copied
        after the steps enqueued so far"""
        sl = self.instance_nodes(k)
        out = np.zeros((sl.stop - sl.start, self.dim))
        L = _capi.lib()
        _capi.check(L.akb_batch_copy_instance_nodal(self._h, _FIELDS[field], int(k),
                                                    _capi.ptr(out), out.nbytes))
        _capi.check(L.akb_model_synchronize(self._h))
        return out

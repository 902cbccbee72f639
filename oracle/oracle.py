"""ctypes wrapper of the CPU oracle (liboracle.so).

Test infrastructure only: imported by tests/, by __graft_entry__.smoke() and by
the CPU-baseline leg of bench.py, always as the checker or the timed CPU
reference, never by the product package.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

TET4, HEX8, TRI6 = 0, 1, 2
ELASTIC, NEOHOOKEAN, PLASTIC, ELASTIC_FD = 0, 1, 2, 3
U, V, A, FEXT, FINT, MASS, BLOCKED = range(7)
GRAD_U, STRESS, PK2, EPS_P, ISO, PLASTIC_ENERGY = range(6)
EKIN, EPOT, EXT_WORK, EPLASTIC = range(4)

_LAWS = {"elastic": ELASTIC, "neohookean": NEOHOOKEAN,
         "plastic_linear_isotropic_hardening": PLASTIC}

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        vp = ctypes.c_void_p
        L.or_model_create.restype = vp
        L.or_model_create.argtypes = [ctypes.c_int, ctypes.c_int, vp, ctypes.c_long,
                                      vp, ctypes.c_long]
        L.or_model_destroy.argtypes = [vp]
        L.or_model_add_material.argtypes = [vp, ctypes.c_int] + [ctypes.c_double] * 7 + [ctypes.c_int]
        L.or_model_set_element_material.argtypes = [vp, vp]
        L.or_model_init.restype = ctypes.c_long
        L.or_model_init.argtypes = [vp]
        L.or_model_stable_dt.restype = ctypes.c_double
        L.or_model_stable_dt.argtypes = [vp]
        L.or_model_set_dt.argtypes = [vp, ctypes.c_double]
        L.or_model_set_nodal.argtypes = [vp, ctypes.c_int, vp]
        L.or_model_get_nodal.argtypes = [vp, ctypes.c_int, vp]
        L.or_model_qp_size.restype = ctypes.c_long
        L.or_model_qp_size.argtypes = [vp, ctypes.c_int]
        L.or_model_get_qp.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp]
        L.or_model_set_eigen_grad_u.argtypes = [vp, ctypes.c_int, vp]
        L.or_model_set_threads.argtypes = [vp, ctypes.c_int]
        L.or_model_solve_step.argtypes = [vp, ctypes.c_long]
        L.or_model_assemble_internal_forces.argtypes = [vp]
        L.or_model_energy.restype = ctypes.c_double
        L.or_model_energy.argtypes = [vp, ctypes.c_int]
        L.or_precompute.restype = ctypes.c_long
        L.or_precompute.argtypes = [ctypes.c_int, ctypes.c_int, vp, ctypes.c_long, vp, vp, vp]
        L.or_inradius.restype = ctypes.c_double
        L.or_inradius.argtypes = [ctypes.c_int, vp]
        L.or_nb_quad.restype = ctypes.c_int
        L.or_nb_quad.argtypes = [ctypes.c_int, ctypes.c_int]
        L.or_quadrature.argtypes = [ctypes.c_int, ctypes.c_int, vp, vp]
        L.or_elastic_stress.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_int, vp, ctypes.c_double, vp]
        L.or_neohookean_stress.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                           vp, ctypes.c_double, vp]
        L.or_plastic_stress.argtypes = [ctypes.c_int] + [ctypes.c_double] * 4 + [vp] * 4 + \
            [ctypes.c_double] * 3 + [vp] * 3
        del dp
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _nnodes(t):
    return {TET4: 4, HEX8: 8, TRI6: 6}[t]


def _dim(t):
    return 2 if t == TRI6 else 3


# ---- element level ---------------------------------------------------------
def quadrature(etype, rule=0):
    L = lib()
    nq = L.or_nb_quad(etype, rule)
    d = _dim(etype)
    pts = np.zeros((nq, d))
    w = np.zeros(nq)
    L.or_quadrature(etype, rule, _p(pts), _p(w))
    return pts, w


def precompute(etype, Xe, rule=0):
    """Xe [E, n, dim] -> (N [E,nq,n], B [E,nq,n,dim], j [E,nq], status)."""
    L = lib()
    Xe = np.ascontiguousarray(Xe, dtype=np.float64)
    E, n, d = Xe.shape
    nq = L.or_nb_quad(etype, rule)
    N = np.zeros((E, nq, n))
    B = np.zeros((E, nq, n, d))
    j = np.zeros((E, nq))
    rc = L.or_precompute(etype, rule, _p(Xe), E, _p(N), _p(B), _p(j))
    return N, B, j, rc


def inradius(etype, Xe):
    Xe = np.ascontiguousarray(Xe, dtype=np.float64)
    return lib().or_inradius(etype, _p(Xe))


def elastic_stress(grad_u, E, nu, sigma_th=0.0, plane_stress=False):
    g = np.asfortranarray(grad_u, dtype=np.float64)
    d = g.shape[0]
    s = np.zeros((d, d), order="F")
    lib().or_elastic_stress(d, E, nu, int(plane_stress), _p(g), sigma_th, _p(s))
    return s


def neohookean_stress(grad_u, E, nu, C33=1.0):
    g = np.asfortranarray(grad_u, dtype=np.float64)
    d = g.shape[0]
    S = np.zeros((d, d), order="F")
    lib().or_neohookean_stress(d, E, nu, _p(g), C33, _p(S))
    return S


def plastic_stress(grad_u, prev_grad_u, prev_sigma, prev_eps_p, iso, prev_iso,
                   E, nu, sigma_y, h, delta_sigma_th=0.0):
    f = lambda a: np.asfortranarray(a, dtype=np.float64)
    g, gp, sp, ep = f(grad_u), f(prev_grad_u), f(prev_sigma), f(prev_eps_p)
    d = g.shape[0]
    s = np.zeros((d, d), order="F")
    e = np.zeros((d, d), order="F")
    iso_out = np.zeros(1)
    lib().or_plastic_stress(d, E, nu, sigma_y, h, _p(g), _p(gp), _p(sp), _p(ep),
                            iso, prev_iso, delta_sigma_th, _p(s), _p(e), _p(iso_out))
    return s, e, float(iso_out[0])


# ---- model level -------------------------------------------------------------
class OracleModel:
    """Explicit lumped-mass model on the CPU (the reference algorithm)."""

    def __init__(self, etype, nodes, conn, materials, mat_of_elem=None, qp_rule=0,
                 threads=1):
        L = lib()
        self.etype = etype
        self.dim = _dim(etype)
        self.nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        self.conn = np.ascontiguousarray(conn, dtype=np.int32)
        self.N = self.nodes.shape[0]
        self.E = self.conn.shape[0]
        self._m = L.or_model_create(etype, qp_rule, _p(self.nodes), self.N,
                                    _p(self.conn), self.E)
        for mat in materials:
            law = _LAWS[mat["type"]] if isinstance(mat["type"], str) else mat["type"]
            if law == ELASTIC and mat.get("finite_deformation", False):
                law = ELASTIC_FD
            L.or_model_add_material(self._m, law, mat.get("rho", 0.0), mat.get("E", 0.0),
                                    mat.get("nu", 0.5), mat.get("sigma_y", 0.0),
                                    mat.get("h", 0.0), mat.get("alpha", 0.0),
                                    mat.get("delta_T", 0.0),
                                    int(mat.get("Plane_Stress", False)))
        if mat_of_elem is not None:
            self._mat = np.ascontiguousarray(mat_of_elem, dtype=np.int32)
            L.or_model_set_element_material(self._m, _p(self._mat))
        L.or_model_set_threads(self._m, threads)
        rc = L.or_model_init(self._m)
        if rc != 0:
            L.or_model_destroy(self._m)
            self._m = None
            raise RuntimeError(f"oracle init failed ({rc})")
        self.nb_materials = len(materials)
        # eigen_grad_u parameter: every point of the material starts from it
        # (Material::updateInternalParameters); its leading d x d block is used
        for k, mat in enumerate(materials):
            if "eigen_grad_u" in mat:
                M = np.asarray(mat["eigen_grad_u"], dtype=np.float64)[:self.dim, :self.dim]
                col = M.reshape(self.dim, self.dim).ravel(order="F")
                n = lib().or_model_qp_size(self._m, k)
                self.set_eigen_grad_u(k, np.tile(col, (n, 1)))

    def __del__(self):
        if getattr(self, "_m", None):
            lib().or_model_destroy(self._m)
            self._m = None

    def set_threads(self, t):
        lib().or_model_set_threads(self._m, t)

    def stable_dt(self):
        return lib().or_model_stable_dt(self._m)

    def set_dt(self, dt):
        lib().or_model_set_dt(self._m, dt)

    def set(self, field, arr):
        if field == BLOCKED:
            a = np.ascontiguousarray(arr, dtype=np.uint8).reshape(self.N, self.dim)
        else:
            a = np.ascontiguousarray(arr, dtype=np.float64).reshape(self.N, self.dim)
        lib().or_model_set_nodal(self._m, field, _p(a))

    def get(self, field):
        if field == BLOCKED:
            a = np.zeros((self.N, self.dim), dtype=np.uint8)
        else:
            a = np.zeros((self.N, self.dim))
        lib().or_model_get_nodal(self._m, field, _p(a))
        return a

    def qp(self, mat, field):
        n = lib().or_model_qp_size(self._m, mat)
        comp = 1 if field in (ISO, PLASTIC_ENERGY) else self.dim * self.dim
        a = np.zeros((n, comp))
        lib().or_model_get_qp(self._m, mat, field, _p(a))
        return a

    def set_eigen_grad_u(self, mat, values):
        """per-point eigen gradient of one material, [points][dim*dim]"""
        a = np.ascontiguousarray(values, dtype=np.float64)
        assert a.size == lib().or_model_qp_size(self._m, mat) * self.dim * self.dim
        lib().or_model_set_eigen_grad_u(self._m, mat, _p(a))

    def step(self, n=1):
        lib().or_model_solve_step(self._m, n)

    def assemble_internal_forces(self):
        lib().or_model_assemble_internal_forces(self._m)

    def energy(self, which):
        return lib().or_model_energy(self._m, which)

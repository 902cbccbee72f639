"""The bounds-checking build (libakb_checked.so, AKB_BOUNDS_CHECK): every index
the step kernels read is checked before it is used.  Indices are corrupted on
the host (akb_model_debug_write_index writes one entry of an index array);
the kernels only report it: the element or node with the bad index is
skipped, status bit 2 is set, the launch completes and the context stays
usable.  Runs in a child process that loads the checked library."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import sys
sys.path.insert(0, ROOT)
import numpy as np
import akantu2_b200 as akb
from akantu2_b200 import _capi
L = _capi.lib()
assert _capi.LIB_PATH.endswith("libakb_checked.so"), _capi.LIB_PATH
assert L.akb_bounds_checked() == 1

def model(mesh, mat, precision):
    m = akb.SolidMechanicsModel(mesh)
    m.addMaterial(mat["type"], **{k: v for k, v in mat.items() if k != "type"})
    m.initFull(akb._explicit_lumped_mass, precision=precision)
    x = mesh.nodes
    d = x.shape[1]
    v = np.zeros_like(x)
    v[:, d - 1] = 0.02 * np.sin(np.pi * x[:, 0])
    b = np.zeros(x.shape, dtype=np.uint8)
    b[np.isclose(x[:, d - 1], 0.0)] = 1
    m.setNodal("velocity", v)
    m.setNodal("blocked_dofs", b)
    m.setTimeStep(0.8 * m.getStableTimeStep())
    return m

EL = dict(type="elastic", rho=1.0, E=1.0, nu=0.3)
NEO = dict(type="neohookean", rho=1.0, E=1.0, nu=0.3)
PL = dict(type="plastic_linear_isotropic_hardening", rho=1.0, E=1.0, nu=0.3, sigma_y=1e-3, h=0.1)
cases = [(akb.box_tet4(4), EL, "fp64"), (akb.box_tet4(4), EL, "mixed"),
         (akb.box_hex8(4), NEO, "fp64"), (akb.box_hex8(4), NEO, "mixed"),
         (akb.box_hex8(4), EL, "fp64_fast"), (akb.square_tri6(5), PL, "mixed")]
for mesh, mat, prec in cases:
    E, N, n = mesh.getNbElement(), mesh.getNbNodes(), mesh.connectivity.shape[1]
    for which, position, value in ((0, 2 * E + 5, N + 7), (0, E + 3, -2),
                                   (1, 1 * E + 7, E * n + 3), (2, 10, 1 << 30)):
        m = model(mesh, mat, prec)
        m.solveStep(4)
        assert m.getStatus() == 0
        _capi.check(L.akb_model_debug_write_index(m._h, which, position, value))
        m.solveStep(3)
        st = m.getStatus()
        assert st & 4, (mesh.element_type, prec, which, st)
        del m
    # the context is still usable: a fresh model steps with no status
    m = model(mesh, mat, prec)
    m.solveStep(5)
    assert m.getStatus() == 0 and np.all(np.isfinite(m.getDisplacement()))
print("checked build OK")
"""


def test_bounds_checking_build_reports_corrupted_indices():
    env = dict(os.environ, AKB_BOUNDS_CHECK="1")
    code = "ROOT = %r\n" % ROOT + CHILD
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "checked build OK" in r.stdout


def test_index_writes_need_the_checked_build():
    import akantu2_b200 as akb
    from akantu2_b200 import _capi
    if _capi.LIB_PATH.endswith("libakb_checked.so"):
        pytest.skip("this process loaded the checked build")
    assert _capi.lib().akb_bounds_checked() == 0
    m = akb.SolidMechanicsModel(akb.box_tet4(2))
    m.addMaterial("elastic", rho=1.0, E=1.0, nu=0.3)
    m.initFull()
    rc = _capi.lib().akb_model_debug_write_index(m._h, 0, 0, 5)
    assert _capi.ERRORS[rc] == "AKB_EUNSUPPORTED"

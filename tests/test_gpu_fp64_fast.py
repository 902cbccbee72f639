"""The fast FP64 path (AKB_PRECISION_FP64_FAST): FP64 state and element math,
hexahedra by the sum-factorised element kernel with contraction allowed.  It
does not keep the CPU path's operation order, so it is held to a 1e-12
relative bar against the oracle (max |gpu - cpu| / max
|cpu| over each nodal array) after 1,000 steps, on a box of parallelepipeds
(the per-element adjugate table) and on a distorted box (geometry per point),
for the elastic and neohookean laws; the plastic law, whose yield test can
turn on a last-bit difference, over 200 steps."""
import numpy as np
import pytest

import akantu2_b200 as akb
from oracle import oracle as orc
from scenarios import (UNIT_ELASTIC, UNIT_NEOHOOKEAN, UNIT_PLASTIC, blocked_face,
                       random_field_velocity, sinusoidal_velocity)
from test_gpu_parity import compare, setup_pair

pytestmark = pytest.mark.gpu


def _mesh(distorted):
    mesh = akb.box_hex8(7)
    if distorted:
        x = mesh.nodes
        rng = np.random.default_rng(5)
        inner = np.all((x > 1e-9) & (x < 1 - 1e-9), axis=1)
        x[inner] += rng.uniform(-0.1, 0.1, size=(inner.sum(), 3)) / 7
    return mesh


@pytest.mark.parametrize("distorted", [False, True])
@pytest.mark.parametrize("mat,steps", [(UNIT_ELASTIC, 1000), (UNIT_NEOHOOKEAN, 1000),
                                       (dict(UNIT_PLASTIC, sigma_y=2e-3), 200)])
def test_fp64_fast_within_1e12_of_the_oracle(mat, steps, distorted):
    mesh = _mesh(distorted)
    v0 = sinusoidal_velocity(mesh.nodes, 0.03) if distorted else \
        random_field_velocity(mesh.nodes, seed=9, corr_length=0.3, std=0.01)
    g, o = setup_pair(mesh, [mat], v0, blocked_face(mesh.nodes), precision="fp64_fast")
    g.solveStep(steps)
    o.step(steps)
    assert np.max(np.abs(o.get(orc.U))) > 0
    errs = compare(g, o, exact=False, tol=1e-12)
    assert max(errs.values()) > 0  # a different evaluation, not the same one
    if mat["type"].startswith("plastic"):
        assert np.max(np.abs(o.qp(0, orc.EPS_P))) > 0, "must yield"


def test_fp64_fast_register_caps_are_bit_identical():
    mesh = _mesh(False)
    v0, bl = sinusoidal_velocity(mesh.nodes, 0.03), blocked_face(mesh.nodes)
    runs = []
    for minb in (1, 2, 3):
        m = akb.SolidMechanicsModel(mesh)
        m.addMaterial("neohookean", rho=1.0, E=1.0, nu=0.3)
        m.initFull(akb._explicit_lumped_mass, precision="fp64_fast")
        assert m.getLaunchShape("neohookean")[1:3] == (2, 3)
        m.setLaunchShape("neohookean", 128, 2, 256, minb)
        m.setNodal("velocity", v0)
        m.setNodal("blocked_dofs", bl)
        m.setTimeStep(0.8 * m.getStableTimeStep())
        m.solveStep(150)
        runs.append((m.getDisplacement().copy(), m.getVelocity().copy()))
    for other in runs[1:]:
        assert np.array_equal(runs[0][0], other[0]) and np.array_equal(runs[0][1], other[1])


def test_fp64_fast_leaves_other_elements_on_the_plain_path():
    """tetrahedra and triangles have no sum-factorised kernel: the fast FP64
    path runs them exactly as the plain one (bit-identical to the oracle)"""
    mesh = akb.box_tet4(4)
    g, o = setup_pair(mesh, [UNIT_ELASTIC], sinusoidal_velocity(mesh.nodes),
                      blocked_face(mesh.nodes), precision="fp64_fast")
    g.solveStep(120)
    o.step(120)
    compare(g, o, exact=True)

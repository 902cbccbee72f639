"""Eigen gradient of the displacement and thermal stress with plasticity on
the GPU, against the CPU oracle.

- eigen_grad_u (material.cc:35-51,147): the material parameter fills every
  quadrature point, setInternal("eigen_grad_u") writes them point by point;
  the gradient minus it enters every law, and is what getGradU returns.
- sigma_th of a plastic material (material_thermal.cc:33-34,
  material_linear_isotropic_hardening_inline_impl.hh:31-34): the trial
  stress takes previous minus current sigma_th, nonzero on the first stress
  evaluation after initFull.

FP64 runs are bit-identical to the oracle (the neohookean law within 1e-12
relative: it calls log), mixed runs within 1e-5 relative L2 displacement.
"""
import numpy as np
import pytest

import akantu2_b200 as akb
from oracle import oracle as orc
from scenarios import (STEEL_PLANE_STRAIN, UNIT_ELASTIC, UNIT_NEOHOOKEAN, UNIT_PLASTIC,
                       blocked_face, linear_field, oracle_model, random_field_velocity,
                       sinusoidal_velocity)
from test_gpu_parity import compare, gpu_model, setup_pair
from test_oracle_golden import _eigen_prescribed_stress, _patch_mesh

pytestmark = pytest.mark.gpu

EIG3 = np.array([[1e-3, 2e-4, -1e-4], [3e-4, -2e-3, 5e-4], [-2e-4, 1e-4, 1.5e-3]])


def _l2(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("etype", ["_tetrahedron_4", "_hexahedron_8", "_triangle_6"])
@pytest.mark.parametrize("per_point", [False, True])
def test_eigen_stress_check_of_the_reference(etype, per_point):
    """test_solid_mechanics_model_material_eigenstrain.cc: linear field,
    eigen_grad_u = 0.1 everywhere, stress within 1e-13 of the analytic one;
    bit-identical to the oracle"""
    mesh = _patch_mesh(etype)
    d = mesh.spatial_dimension
    eig = np.full((d, d), 0.1)
    mat = dict(STEEL_PLANE_STRAIN)
    if not per_point:
        mat["eigen_grad_u"] = eig
    g = gpu_model(mesh, [mat])
    o = oracle_model(mesh, [mat])
    if per_point:
        n = g.getMaterial(0).getInternal("eigen_grad_u")().shape[0]
        assert np.all(g.getMaterial(0).getInternal("eigen_grad_u")() == 0)
        vals = np.tile(eig.ravel(order="F"), (n, 1))
        g.getMaterial(0).setInternal("eigen_grad_u", vals)
        o.set_eigen_grad_u(0, vals)
    assert np.array_equal(g.getMaterial(0).getInternal("eigen_grad_u")(),
                          np.tile(eig.ravel(order="F"), (g.getMaterial(0).getGradU().shape[0], 1)))
    u = linear_field(mesh.nodes)
    g.setNodal("displacement", u)
    o.set(orc.U, u)
    g.assembleInternalForces()
    o.assemble_internal_forces()
    stress = g.getMaterial(0).getStress()
    expected = _eigen_prescribed_stress(eig, d)
    for s in stress:
        S = s.reshape(d, d, order="F")
        assert np.max(np.abs(S - expected)) / np.max(np.abs(S)) <= 1e-13
    assert np.array_equal(stress, o.qp(0, orc.STRESS))
    assert np.array_equal(g.getMaterial(0).getGradU(), o.qp(0, orc.GRAD_U))
    assert np.array_equal(g.getInternalForce(), o.get(orc.FINT))


def _eig(d, scale=1.0):
    return scale * EIG3[:d, :d]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", ["tet4_elastic", "hex8_neohookean", "tri6_plastic"])
def test_eigen_dynamics_match_oracle(case, precision):
    etype, law = case.split("_")
    if etype == "tet4":
        mesh, mat = akb.box_tet4(5), dict(UNIT_ELASTIC)
    elif etype == "hex8":
        mesh, mat = akb.box_hex8(5), dict(UNIT_NEOHOOKEAN)
    else:
        mesh, mat = akb.square_tri6(6), dict(UNIT_PLASTIC, sigma_y=2e-3)
    d = mesh.spatial_dimension
    mat["eigen_grad_u"] = _eig(d, 5.0 if law == "plastic" else 1.0)
    v0 = sinusoidal_velocity(mesh.nodes, 0.02) if d == 3 else np.zeros_like(mesh.nodes)
    blocked = blocked_face(mesh.nodes, axis=d - 1)
    g, o = setup_pair(mesh, [mat], v0, blocked, precision=precision)
    g.solveStep(150)  # one graph of 100 steps and plain launches
    o.step(150)
    if law == "plastic":
        assert np.max(np.abs(o.qp(0, orc.EPS_P))) > 0, "the eigen gradient must make it yield"
    if precision == "fp64":
        compare(g, o, exact=law != "neohookean")
        if law != "neohookean":
            assert np.array_equal(g.getMaterial(0).getGradU(), o.qp(0, orc.GRAD_U))
    else:
        assert _l2(g.getDisplacement(), o.get(orc.U)) <= 1e-5


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_eigen_field_written_between_steps(precision):
    """a per-point eigen gradient written after steps (captured graphs read
    none before): the following steps use it, the hexahedral mixed path
    included (its sum-factorised kernel)"""
    mesh = akb.box_hex8(5)
    v0 = random_field_velocity(mesh.nodes, seed=5, corr_length=0.3, std=0.004)
    g, o = setup_pair(mesh, [UNIT_ELASTIC], v0, blocked_face(mesh.nodes), precision=precision)
    g.solveStep(120)
    o.step(120)
    n = o.qp(0, orc.GRAD_U).shape[0]
    rng = np.random.default_rng(4)
    vals = 1e-3 * rng.standard_normal((n, 9))
    g.getMaterial(0).setInternal("eigen_grad_u", vals)
    o.set_eigen_grad_u(0, vals)
    assert np.array_equal(g.getMaterial(0).getInternal("eigen_grad_u")(), vals)
    g.solveStep(130)
    o.step(130)
    if precision == "fp64":
        compare(g, o, exact=True)
    else:
        assert _l2(g.getDisplacement(), o.get(orc.U)) <= 1e-5
    with pytest.raises(akb.AkbError):
        g.getMaterial(0).setInternal("grad_u", vals)


def test_eigen_parameter_needs_the_dimension():
    mesh = akb.box_tet4(2)
    m = akb.SolidMechanicsModel(mesh)
    m.addMaterial("elastic", rho=1.0, E=1.0, nu=0.3, eigen_grad_u=np.eye(2))
    with pytest.raises(akb.AkbError):
        m.initFull()


@pytest.mark.parametrize("graph_steps", [0, 10])
def test_thermal_plasticity_bitwise(graph_steps):
    """two heated plastic materials (one law group, per-element parameter
    table) and an elastic one in a plane-strain square: the first step's
    thermal term makes the plastic points yield; a standalone assembly in the
    middle takes none; bit-identical to the oracle, plastic internals too"""
    mesh = akb.square_tri6(6)
    E = mesh.getNbElement()
    mat_of_elem = (np.arange(E) % 3).astype(np.int32)
    mats = [dict(UNIT_PLASTIC, name="p0", sigma_y=1e-3, alpha=1e-3, delta_T=2.0),
            dict(UNIT_ELASTIC, name="e1", alpha=2e-3, delta_T=-1.0),
            dict(UNIT_PLASTIC, name="p2", E=0.7, sigma_y=5e-4, h=0.2, alpha=-1e-3, delta_T=1.5)]
    x = mesh.nodes
    blocked = np.zeros(x.shape, dtype=np.uint8)
    blocked[np.isclose(x[:, 0], 0.0)] = 1
    g, o = setup_pair(mesh, mats, np.zeros_like(x), blocked, mat_of_elem=mat_of_elem)
    g.setGraphSteps(graph_steps)
    g.solveStep(25)
    o.step(25)
    compare(g, o, exact=True)
    g.assembleInternalForces()
    o.assemble_internal_forces()
    compare(g, o, exact=True)
    g.solveStep(37)
    o.step(37)
    compare(g, o, exact=True)
    for k in (0, 2):
        mk = g.getMaterial(k)
        assert np.max(np.abs(o.qp(k, orc.EPS_P))) > 0, f"material {k} must yield"
        assert np.array_equal(mk.getInternal("inelastic_strain")(), o.qp(k, orc.EPS_P))
        assert np.array_equal(mk.getInternal("iso_hardening")(), o.qp(k, orc.ISO))
        assert np.array_equal(mk.getStress(), o.qp(k, orc.STRESS))
    assert np.array_equal(g.getMaterial(1).getStress(), o.qp(1, orc.STRESS))

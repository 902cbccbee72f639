"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

The FP64 kernels are compiled without contraction and follow the oracle's
operation order, so elastic and plastic runs are expected to be bit-identical;
the neohookean law calls log(), whose last bit may differ between the CUDA
and glibc implementations, so those runs are held to a 1e-12 relative bar
(max |gpu - cpu| / max |cpu| over each nodal array).
"""
import numpy as np
import pytest

import akantu2_b200 as akb
from oracle import oracle as orc
from scenarios import (OR_TYPE, STEEL_PLANE_STRAIN, STEEL_PLANE_STRESS, UNIT_ELASTIC,
                       UNIT_NEOHOOKEAN, UNIT_PLASTIC, blocked_face, golden, oracle_model,
                       random_field_velocity, sinusoidal_velocity)
from test_oracle_golden import _patch_mesh, check_patch_results, run_patch_test

pytestmark = pytest.mark.gpu

REL = 1e-12
NODAL = [("displacement", orc.U), ("velocity", orc.V), ("acceleration", orc.A),
         ("internal_force", orc.FINT)]


def rel_err(a, b):
    scale = np.max(np.abs(b))
    return np.max(np.abs(a - b)) / scale if scale > 0 else np.max(np.abs(a - b))


def gpu_model(mesh, materials, mat_of_elem=None, precision="fp64", qp_rule=0):
    m = akb.SolidMechanicsModel(mesh)
    for mat in materials:
        params = {k: v for k, v in mat.items() if k != "type"}
        m.addMaterial(mat["type"], **params)
    if mat_of_elem is not None:
        m.setElementMaterials(mat_of_elem)
    if qp_rule:
        m.setQuadratureRule(qp_rule)
    m.initFull(akb._explicit_lumped_mass, precision=precision)
    return m


def setup_pair(mesh, materials, v0, blocked, mat_of_elem=None, qp_rule=0, precision="fp64",
               dt_factor=0.8):
    g = gpu_model(mesh, materials, mat_of_elem, precision, qp_rule)
    o = oracle_model(mesh, materials, mat_of_elem, qp_rule)
    g.setNodal("velocity", v0)
    g.setNodal("blocked_dofs", blocked)
    o.set(orc.V, v0)
    o.set(orc.BLOCKED, blocked)
    dt_g, dt_o = g.getStableTimeStep(), o.stable_dt()
    assert dt_g == dt_o
    g.setTimeStep(dt_factor * dt_g)
    o.set_dt(dt_factor * dt_o)
    return g, o


def compare(g, o, exact, tol=REL):
    errs = {}
    for name, fid in NODAL:
        a, b = getattr(g, "get" + "".join(w.capitalize() for w in name.split("_")))(), o.get(fid)
        if exact:
            assert np.array_equal(a, b), f"{name} differs: rel {rel_err(a, b):.3e}"
        errs[name] = rel_err(a, b)
        assert errs[name] <= tol, f"{name}: {errs[name]:.3e}"
    return errs


# ---- element data -----------------------------------------------------------------
@pytest.mark.parametrize("etype", ["_tetrahedron_4", "_hexahedron_8", "_triangle_6"])
def test_fe_data_bitwise_and_py_engine(etype):
    gold = golden(f"fe{etype}.npz")
    mesh = akb.Mesh(gold["nodes"].shape[1], gold["nodes"], gold["conn"], etype)
    m = gpu_model(mesh, [UNIT_ELASTIC])
    B, j = m.getFEData()
    _, Bo, jo, _ = orc.precompute(OR_TYPE[etype], mesh.nodes[mesh.connectivity])
    assert np.array_equal(B, Bo) and np.array_equal(j, jo)
    assert np.max(np.abs(B - gold["B"])) < 1e-10 and np.max(np.abs(j - gold["j"])) < 1e-10


@pytest.mark.parametrize("etype", ["_tetrahedron_4", "_hexahedron_8", "_triangle_6"])
def test_mass_and_stable_dt_bitwise(etype):
    mesh = {"_tetrahedron_4": akb.box_tet4(4), "_hexahedron_8": akb.box_hex8(4),
            "_triangle_6": akb.square_tri6(5)}[etype]
    mesh.nodes += 0.01 * np.sin(7 * mesh.nodes)  # distorted, still valid
    g = gpu_model(mesh, [UNIT_ELASTIC])
    o = oracle_model(mesh, [UNIT_ELASTIC])
    assert np.array_equal(g.getMass(), o.get(orc.MASS))
    assert g.getStableTimeStep() == o.stable_dt()


def test_inradius_fixtures_through_stable_dt():
    for etype in ["_tetrahedron_4", "_hexahedron_8", "_triangle_6"]:
        gold = golden(f"fe{etype}.npz")
        mesh = akb.Mesh(gold["nodes"].shape[1], gold["nodes"], gold["conn"], etype)
        m = gpu_model(mesh, [dict(UNIT_ELASTIC, nu=0.0)])  # celerity 1
        assert abs(m.getStableTimeStep() - gold["inradius"].min()) < 1e-6


# ---- trajectories -------------------------------------------------------------------
def test_tet4_elastic_bitwise():
    mesh = akb.box_tet4(5)
    g, o = setup_pair(mesh, [UNIT_ELASTIC], sinusoidal_velocity(mesh.nodes),
                      blocked_face(mesh.nodes))
    g.solveStep(150)
    o.step(150)
    compare(g, o, exact=True)
    for f in (orc.GRAD_U, orc.STRESS):
        got = g.getMaterial(0).getGradU() if f == orc.GRAD_U else g.getMaterial(0).getStress()
        assert np.array_equal(got, o.qp(0, f))


def test_hex8_neohookean_parity():
    mesh = akb.box_hex8(6)
    v0 = random_field_velocity(mesh.nodes, seed=7, corr_length=0.3, std=0.004)
    g, o = setup_pair(mesh, [UNIT_NEOHOOKEAN], v0, blocked_face(mesh.nodes))
    g.solveStep(150)
    o.step(150)
    assert np.all(np.isfinite(o.get(orc.U)))
    # large enough to leave the linear regime: |grad u| of order 1e-2
    assert np.max(np.abs(o.qp(0, orc.GRAD_U))) > 1e-2
    compare(g, o, exact=False)
    assert rel_err(g.getMaterial(0).getInternal("piola_kirchhoff_2")(), o.qp(0, orc.PK2)) < REL
    assert rel_err(g.getMaterial(0).getGradU(), o.qp(0, orc.GRAD_U)) < REL


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_graph_replay_matches_plain_launches(precision):
    """Multi-step runs replayed as CUDA graphs give the same state as one
    launch sequence per step (both buffer parities, host edits in between)."""
    mesh = akb.box_tet4(4)
    v0, bl = sinusoidal_velocity(mesh.nodes, 0.05), blocked_face(mesh.nodes)
    runs = []
    for graph_steps in (0, 2, 100):
        m = gpu_model(mesh, [UNIT_ELASTIC], precision=precision)
        m.setGraphSteps(graph_steps)
        m.setNodal("velocity", v0)
        m.setNodal("blocked_dofs", bl)
        m.setTimeStep(0.8 * m.getStableTimeStep())
        m.solveStep(233)
        f = m.getExternalForce()
        f[:, 0] = 1e-4  # host edit: the next step re-predicts, graphs see f_ext != 0
        m.solveStep(301)
        runs.append((m.getDisplacement().copy(), m.getVelocity().copy(),
                     m.getInternalForce().copy()))
    for other in runs[1:]:
        for a, b in zip(runs[0], other):
            assert np.array_equal(a, b)


def test_hex8_elastic_bitwise():
    mesh = akb.box_hex8(5)
    v0 = random_field_velocity(mesh.nodes, seed=3)
    g, o = setup_pair(mesh, [UNIT_ELASTIC], v0, blocked_face(mesh.nodes))
    g.solveStep(100)
    o.step(100)
    compare(g, o, exact=True)


@pytest.mark.parametrize("qp_rule", [0, 1])
def test_tri6_plastic_ramp_bitwise(qp_rule):
    """Left edge blocked, right edge pulled with a velocity ramp written
    into the displacement before every step (the imposed-motion loop of
    test_solid_mechanics_model_dynamics.cc:243-244)."""
    mesh = akb.square_tri6(6)
    x = mesh.nodes
    left, right = np.isclose(x[:, 0], 0.0), np.isclose(x[:, 0], 1.0)
    blocked = np.zeros(x.shape, dtype=np.uint8)
    blocked[left] = 1
    blocked[right, 0] = 1
    mat = dict(UNIT_PLASTIC, sigma_y=2e-3)
    g, o = setup_pair(mesh, [mat], np.zeros_like(x), blocked, qp_rule=qp_rule)
    nsteps, target = 120, 2e-2
    u = np.zeros_like(x)
    for s in range(nsteps):
        u = o.get(orc.U)
        u[right, 0] = target * min(1.0, (s + 1) / nsteps)
        o.set(orc.U, u)
        g.setNodal("displacement", u)
        g.solveStep()
        o.step()
    compare(g, o, exact=True)
    mg, eps = g.getMaterial(0), o.qp(0, orc.EPS_P)
    assert np.max(np.abs(eps)) > 0, "the ramp must reach the yield stress"
    assert np.array_equal(mg.getInternal("inelastic_strain")(), eps)
    assert np.array_equal(mg.getInternal("iso_hardening")(), o.qp(0, orc.ISO))
    assert np.array_equal(mg.getStress(), o.qp(0, orc.STRESS))
    assert np.array_equal(mg.getInternal("plastic_energy")(), o.qp(0, orc.PLASTIC_ENERGY))


def test_multi_material_hex8():
    mesh = akb.box_hex8(4)
    centers = mesh.nodes[mesh.connectivity].mean(axis=1)
    mat_of_elem = (centers[:, 0] > 0.5).astype(np.int32)  # elements interleaved by x
    mats = [dict(UNIT_ELASTIC, name="soft", E=0.5), dict(UNIT_ELASTIC, name="stiff", E=2.0)]
    v0 = random_field_velocity(mesh.nodes, seed=11)
    g, o = setup_pair(mesh, mats, v0, blocked_face(mesh.nodes), mat_of_elem=mat_of_elem)
    g.solveStep(80)
    o.step(80)
    compare(g, o, exact=True)
    for k in range(2):
        assert np.array_equal(g.getMaterial(k).getStress(), o.qp(k, orc.STRESS))


def test_energies_match_oracle():
    mesh = akb.box_tet4(4)
    f_ext = np.zeros_like(mesh.nodes)
    f_ext[:, 0] = 1e-4
    g, o = setup_pair(mesh, [UNIT_ELASTIC], sinusoidal_velocity(mesh.nodes),
                      blocked_face(mesh.nodes))
    g.setNodal("external_force", f_ext)
    o.set(orc.FEXT, f_ext)
    g.solveStep(60)
    o.step(60)
    for name, which in [("kinetic", orc.EKIN), ("potential", orc.EPOT),
                        ("external work", orc.EXT_WORK)]:
        a, b = g.getEnergy(name), o.energy(which)
        assert abs(a - b) <= 1e-12 * abs(b), name


def test_plastic_energy_matches_oracle():
    mesh = akb.square_tri6(4)
    x = mesh.nodes
    blocked = np.zeros(x.shape, dtype=np.uint8)
    blocked[np.isclose(x[:, 0], 0.0)] = 1
    v0 = np.zeros_like(x)
    v0[:, 0] = 0.02 * x[:, 0]
    g, o = setup_pair(mesh, [UNIT_PLASTIC], v0, blocked)
    g.solveStep(80)
    o.step(80)
    for name, which in [("plastic", orc.EPLASTIC), ("potential", orc.EPOT)]:
        a, b = g.getEnergy(name), o.energy(which)
        assert b != 0 and abs(a - b) <= 1e-12 * abs(b), name


@pytest.mark.parametrize("etype,material", [
    ("_tetrahedron_4", STEEL_PLANE_STRAIN), ("_hexahedron_8", STEEL_PLANE_STRAIN),
    ("_triangle_6", STEEL_PLANE_STRAIN), ("_triangle_6", STEEL_PLANE_STRESS)])
def test_gpu_explicit_patch_test(etype, material):
    mesh, model, blocked, u = run_patch_test(lambda m, mat: gpu_model(m, [mat]), etype, material)
    model.getBlockedDOFs()[:] = blocked.astype(bool)
    model.getDisplacement()[:] = u
    model.setTimeStep(0.8 * model.getStableTimeStep())
    for _ in range(100):
        model.solveStep()
    check_patch_results(mesh, model.getDisplacement(), model.getMaterial(0).getGradU(),
                        model.getMaterial(0).getStress(), material, model.getInternalForce(),
                        model.getEnergy("kinetic"))


# ---- full-size tet-cube configuration ---------------------------------------------------
def test_tet_cube_48k_1000_steps():
    """Unit cube, 20^3 cells x 6 tetrahedra, elastic, z = 0 blocked,
    v_z = 0.01 sin(pi x) sin(pi y) z, dt = 0.8 stable, 1000 steps."""
    mesh = akb.box_tet4(20)
    assert mesh.getNbElement() == 48000 and mesh.getNbNodes() == 9261
    g, o = setup_pair(mesh, [UNIT_ELASTIC], sinusoidal_velocity(mesh.nodes),
                      blocked_face(mesh.nodes))
    g.solveStep(1000)
    o.step(1000)
    errs = compare(g, o, exact=True)
    assert max(errs.values()) == 0.0


def test_mixed_precision_error_tet_cube():
    mesh = akb.box_tet4(12)
    v0, bl = sinusoidal_velocity(mesh.nodes), blocked_face(mesh.nodes)
    g, o = setup_pair(mesh, [UNIT_ELASTIC], v0, bl, precision="mixed")
    g.solveStep(1000)
    o.step(1000)
    u, uo = g.getDisplacement(), o.get(orc.U)
    l2 = np.linalg.norm(u - uo) / np.linalg.norm(uo)
    assert l2 < 1e-5


# ---- edge cases ---------------------------------------------------------------------------
def test_negative_jacobian_is_reported():
    mesh = akb.box_tet4(2)
    c = mesh.connectivity
    c[3, [1, 2]] = c[3, [2, 1]]  # invert one element
    with pytest.raises(akb.AkbError) as e:
        gpu_model(mesh, [UNIT_ELASTIC])
    assert e.value.name == "AKB_ENEGJAC" and ":3)" in str(e.value)


def test_empty_mesh():
    mesh = akb.Mesh(3, np.zeros((0, 3)), np.zeros((0, 4), np.int32), "_tetrahedron_4")
    m = gpu_model(mesh, [UNIT_ELASTIC])
    m.setTimeStep(1e-3)
    m.solveStep(3)
    assert m.getDisplacement().shape == (0, 3)
    assert m.getEnergy("kinetic") == 0.0


def test_single_element_and_unconnected_node():
    nodes = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [5, 5, 5]], dtype=float)
    conn = np.array([[0, 1, 2, 3]], dtype=np.int32)
    mesh = akb.Mesh(3, nodes, conn, "_tetrahedron_4")
    g = gpu_model(mesh, [UNIT_ELASTIC])
    o = oracle_model(mesh, [UNIT_ELASTIC])
    assert np.array_equal(g.getMass(), o.get(orc.MASS))
    v0 = np.zeros((5, 3))
    v0[1, 0] = 0.1
    for m in (g,):
        m.setNodal("velocity", v0)
    o.set(orc.V, v0)
    dt = 0.5 * g.getStableTimeStep()
    g.setTimeStep(dt)
    o.set_dt(dt)
    g.solveStep(10)
    o.step(10)
    # node 4 has zero mass: its acceleration is r / 0 (non-finite) in both
    a_g, a_o = g.getAcceleration(), o.get(orc.A)
    assert np.array_equal(np.isfinite(a_g), np.isfinite(a_o))
    fin = np.isfinite(a_o)
    assert np.array_equal(a_g[fin], a_o[fin])
    assert g.getStatus() & 1


def test_nonfinite_state_sets_status():
    mesh = akb.box_tet4(2)
    m = gpu_model(mesh, [UNIT_ELASTIC])
    v0 = np.zeros_like(mesh.nodes)
    m.setTimeStep(0.5 * m.getStableTimeStep())
    m.solveStep(2)
    assert m.getStatus() == 0
    v0[3, 1] = np.nan
    m.setNodal("velocity", v0)
    m.solveStep(2)
    assert m.getStatus() & 1
    assert m.getStatus() == 0  # reading clears the flag


def test_user_writes_between_steps_keep_reference_semantics():
    """Elastic grad_u / stress are those of the last force assembly even
    if the displacement array is written afterwards."""
    mesh = akb.box_tet4(3)
    g, o = setup_pair(mesh, [UNIT_ELASTIC], sinusoidal_velocity(mesh.nodes, 0.1),
                      blocked_face(mesh.nodes))
    g.solveStep(5)
    o.step(5)
    u = g.getDisplacement()
    u[:] += 0.01
    ref = o.qp(0, orc.GRAD_U)
    assert np.array_equal(g.getMaterial(0).getGradU(), ref)


@pytest.mark.parametrize("graph_steps", [0, 10])
def test_device_prescribed_velocity_ramp_bitwise(graph_steps):
    """the right edge pulled by a velocity ramp prescribed on the device
    matches the host writing the same displacement before every step"""
    mesh = akb.square_tri6(6)
    x = mesh.nodes
    left, right = np.isclose(x[:, 0], 0.0), np.isclose(x[:, 0], 1.0)
    blocked = np.zeros(x.shape, dtype=np.uint8)
    blocked[left] = 1
    mat = dict(UNIT_PLASTIC, sigma_y=2e-3)
    g, o = setup_pair(mesh, [mat], np.zeros_like(x), blocked)
    g.setGraphSteps(graph_steps)
    nsteps, ramp, v_max = 130, 60, 0.4
    dt = g.getTimeStep()
    g.setPrescribedVelocityRamp(right, 0, v_max, ramp)
    ob = blocked.copy()
    ob[right, 0] = 1
    o.set(orc.BLOCKED, ob)
    assert np.array_equal(g.getBlockedDOFs(), ob.astype(bool))
    u0 = o.get(orc.U)[right, 0].copy()
    acc = 0.0
    for k in range(1, nsteps + 1):
        acc = acc + dt * (v_max * min(1.0, k / ramp))
        u = o.get(orc.U)
        u[right, 0] = u0 + acc
        o.set(orc.U, u)
        o.step()
    g.solveStep(nsteps)
    compare(g, o, exact=True)
    assert np.max(np.abs(o.qp(0, orc.EPS_P))) > 0, "the ramp must reach the yield stress"
    assert np.array_equal(g.getMaterial(0).getInternal("inelastic_strain")(), o.qp(0, orc.EPS_P))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_ramp_survives_host_writes(precision):
    """a host write between steps makes the model predict again; the ramp
    then applies the coming step's value again instead of advancing twice"""
    mesh = akb.square_tri6(6)
    x = mesh.nodes
    right = np.flatnonzero(np.isclose(x[:, 0], 1.0))
    blocked = np.zeros(x.shape, dtype=np.uint8)
    blocked[np.isclose(x[:, 0], 0.0)] = 1
    runs = []
    for writes in (False, True):
        g = gpu_model(mesh, [dict(UNIT_PLASTIC, sigma_y=2e-3)], precision=precision)
        g.setNodal("blocked_dofs", blocked)
        g.setTimeStep(0.8 * g.getStableTimeStep())
        g.setPrescribedVelocityRamp(right, 0, 0.4, 30)
        for chunk in (7, 1, 20, 45):
            if writes:
                g.setNodal("velocity", g.getVelocity().copy())
            g.solveStep(chunk)
        runs.append((g.getDisplacement().copy(), g.getVelocity().copy()))
    assert np.array_equal(runs[0][0], runs[1][0]) and np.array_equal(runs[0][1], runs[1][1])


UNIT_ELASTIC_FD = dict(type="elastic", name="svk", rho=1.0, E=1.0, nu=0.3,
                       finite_deformation=True)


@pytest.mark.parametrize("etype,plane_stress", [("_tetrahedron_4", False),
                                                ("_hexahedron_8", False),
                                                ("_triangle_6", False), ("_triangle_6", True)])
def test_finite_deformation_elastic_bitwise(etype, plane_stress):
    """`elastic` with finite_deformation = true (the JOSS benchmark's material
    path): FP64 bit-identical to the oracle, mixed within 1e-5"""
    mesh = {"_tetrahedron_4": lambda: akb.box_tet4(4), "_hexahedron_8": lambda: akb.box_hex8(4),
            "_triangle_6": lambda: akb.square_tri6(5)}[etype]()
    mat = dict(UNIT_ELASTIC_FD, Plane_Stress=plane_stress) if plane_stress else UNIT_ELASTIC_FD
    d = mesh.spatial_dimension
    v0 = random_field_velocity(mesh.nodes, seed=8) * 5 if d == 3 else \
        np.stack([0.1 * mesh.nodes[:, 0], 0.05 * mesh.nodes[:, 1]], axis=1)
    bl = blocked_face(mesh.nodes, axis=2 if d == 3 else 0)
    g, o = setup_pair(mesh, [mat], v0, bl)
    g.solveStep(60)
    o.step(60)
    compare(g, o, exact=True)
    assert np.array_equal(g.getMaterial(0).getInternal("piola_kirchhoff_2")(), o.qp(0, orc.PK2))
    assert np.max(np.abs(g.getMaterial(0).getStress())) == 0.0  # Cauchy: filled on dump only
    a, b = g.getEnergy("potential"), o.energy(orc.EPOT)
    assert b > 0 and abs(a - b) <= 1e-12 * b
    gm, _ = setup_pair(mesh, [mat], v0, bl, precision="mixed")
    gm.solveStep(60)
    uo = o.get(orc.U)
    assert np.linalg.norm(gm.getDisplacement() - uo) / np.linalg.norm(uo) < 1e-5


def test_finite_deformation_elastic_shares_the_finite_strain_launch():
    """neohookean and finite-deformation elastic materials interleaved: one
    finite-strain law group with per-element parameters, bit-identical"""
    mesh = akb.box_hex8(4)
    mat_of_elem = (np.arange(mesh.getNbElement()) % 2).astype(np.int32)
    mats = [dict(UNIT_NEOHOOKEAN, name="nh"), dict(UNIT_ELASTIC_FD, E=2.0)]
    v0 = random_field_velocity(mesh.nodes, seed=12)
    g, o = setup_pair(mesh, mats, v0, blocked_face(mesh.nodes), mat_of_elem=mat_of_elem)
    g.solveStep(40)
    o.step(40)
    compare(g, o, exact=False)
    for k in range(2):
        assert np.array_equal(g.getMaterial(k).getInternal("piola_kirchhoff_2")(),
                              o.qp(k, orc.PK2)) or k == 0


@pytest.mark.parametrize("kind", ["tet_cube_48k", "hex8_neohookean_64"])
def test_mixed_precision_error_after_ten_thousand_steps(kind):
    """FP32 element math with FP64 state against the plain FP64 path after
    10^4 steps: relative L2 displacement <= 1e-5, and both paths conserve the
    total energy of the free vibration to the same degree.  (The difference
    is a phase drift that grows with the number of periods simulated: a 16^3
    hexahedral box run for 10^4 steps covers eight times more periods of its
    lowest mode than the 128^3 benchmark box and ends near 2.4e-5.)"""
    if kind == "tet_cube_48k":
        mesh, mat = akb.box_tet4(20), UNIT_ELASTIC
        v0 = sinusoidal_velocity(mesh.nodes)
    else:
        mesh, mat = akb.box_hex8(64), UNIT_NEOHOOKEAN
        v0 = random_field_velocity(mesh.nodes, seed=2024)
    bl = blocked_face(mesh.nodes)
    res = {}
    for prec in ("mixed", "fp64"):
        m = gpu_model(mesh, [mat], precision=prec)
        m.setNodal("velocity", v0)
        m.setNodal("blocked_dofs", bl)
        m.setTimeStep(0.8 * m.getStableTimeStep())
        e0 = m.getEnergy("kinetic") + m.getEnergy("potential")
        m.solveStep(10000)
        e1 = m.getEnergy("kinetic") + m.getEnergy("potential")
        res[prec] = (m.getDisplacement(), (e1 - e0) / e0)
    u, ud = res["mixed"][0], res["fp64"][0]
    assert np.linalg.norm(u - ud) / np.linalg.norm(ud) < 1e-5
    assert abs(res["mixed"][1] - res["fp64"][1]) < 1e-6


def test_plane_stress_neohookean_parity():
    """plane-stress neohookean on _triangle_6: the per-point C33 Newton solve
    (state carried between steps) against the oracle"""
    mesh = akb.square_tri6(6)
    x = mesh.nodes
    mat = dict(UNIT_NEOHOOKEAN, Plane_Stress=True)
    v0 = np.stack([0.2 * x[:, 0], -0.05 * x[:, 0] * x[:, 1]], axis=1)
    bl = blocked_face(x, axis=0)
    g, o = setup_pair(mesh, [mat], v0, bl)
    g.solveStep(80)
    o.step(80)
    errs = compare(g, o, exact=False)
    assert max(errs.values()) <= 1e-12
    pk2, opk2 = g.getMaterial(0).getInternal("piola_kirchhoff_2")(), o.qp(0, orc.PK2)
    assert np.max(np.abs(pk2 - opk2)) <= 1e-12 * np.max(np.abs(opk2))
    gm, _ = setup_pair(mesh, [mat], v0, bl, precision="mixed")
    gm.solveStep(80)
    uo = o.get(orc.U)
    assert np.linalg.norm(gm.getDisplacement() - uo) / np.linalg.norm(uo) < 1e-5


def test_neumann_stress_adds_to_external_force():
    mesh = akb.box_hex8(3)
    g = gpu_model(mesh, [UNIT_ELASTIC])
    sigma = np.array([[1e-3, 2e-4, 0.0], [2e-4, -5e-4, 1e-4], [0.0, 1e-4, 3e-4]])
    top = np.nonzero(np.isclose(mesh.nodes[:, 2], 1.0))[0]
    g.getExternalForce()[:] = 1.0
    g.applyBC(akb.FromHigherDim(sigma), top)
    g.solveStep(0)
    expected = 1.0 + akb.neumann_forces(mesh, top, sigma)
    assert np.array_equal(g.getExternalForce(), expected)
    # the top face's normal is +z: the resultant is the third column times the area
    assert np.allclose((expected - 1.0).sum(axis=0), sigma[:, 2], rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("lag", [1, 3])
def test_async_nodal_io_matches_synchronous_calls(lag):
    """per-step uploads and reads through the asynchronous forms give the
    state and the host copies of the synchronous set / get sequence, each
    read waited for lag steps later (up to AKB_ASYNC_READS_IN_FLIGHT - 1;
    lag + 1 host buffers per direction)"""
    from akantu2_b200._capi import PinnedArray
    mesh = akb.box_tet4(6)
    v0, bl = sinusoidal_velocity(mesh.nodes, 0.05), blocked_face(mesh.nodes)
    rng = np.random.default_rng(4)
    forces = [1e-4 * rng.standard_normal(mesh.nodes.shape) for _ in range(12)]
    out = {}
    for mode in ("sync", "async"):
        m = gpu_model(mesh, [UNIT_ELASTIC], precision="mixed")
        m.setNodal("velocity", v0)
        m.setNodal("blocked_dofs", bl)
        m.setTimeStep(0.8 * m.getStableTimeStep())
        fin = [PinnedArray(mesh.nodes.shape) for _ in range(lag + 1)]
        uo = [PinnedArray(mesh.nodes.shape) for _ in range(lag + 1)]
        seen = []
        pending = []
        for j, f in enumerate(forces):
            if mode == "sync":
                m.setNodal("external_force", f)
                m.solveStep(1)
                seen.append(m.getDisplacement().copy())
            else:
                b = j % (lag + 1)
                fin[b].array[:] = f
                m.setNodalAsync("external_force", fin[b].array)
                m.solveStep(1)
                pending.append((m.getNodalAsync("displacement", uo[b].array), b))
                if len(pending) > lag:
                    t, bo = pending.pop(0)
                    m.waitNodalAsync(t)
                    seen.append(uo[bo].array.copy())
        if mode == "async":
            m.synchronize()
            seen += [uo[bo].array.copy() for _, bo in pending]
        out[mode] = (seen, m.getVelocity().copy())
    assert len(out["sync"][0]) == len(out["async"][0])
    for a, b in zip(out["sync"][0], out["async"][0]):
        assert np.array_equal(a, b)
    assert np.array_equal(out["sync"][1], out["async"][1])


def test_async_reads_in_flight_limit():
    """the AKB_ASYNC_READS_IN_FLIGHT most recent reads can be waited on one
    by one; an older ticket is rejected (akb_model_synchronize covers it)"""
    from akantu2_b200 import _capi
    from akantu2_b200._capi import PinnedArray
    n = _capi.ASYNC_READS_IN_FLIGHT
    mesh = akb.box_tet4(4)
    m = gpu_model(mesh, [UNIT_ELASTIC], precision="mixed")
    m.setTimeStep(0.8 * m.getStableTimeStep())
    bufs = [PinnedArray(mesh.nodes.shape) for _ in range(n + 1)]
    tickets = []
    for b in bufs:
        m.solveStep(1)
        tickets.append(m.getNodalAsync("displacement", b.array))
    with pytest.raises(akb.AkbError) as e:
        m.waitNodalAsync(tickets[0])
    assert e.value.name == "AKB_EINVAL"
    for t in tickets[1:]:
        m.waitNodalAsync(t)
    m.synchronize()
    assert np.array_equal(bufs[-1].array, m.getDisplacement())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_previous_displacement_and_increment(precision):
    """TimeStepSolverDefault's bookkeeping (time_step_solver_default.cc:171-221):
    the previous displacement is u at the start of the last step and the
    increment u_{n+1} - u_n, through single steps, a 100-step graph and a
    host write between steps; tracking changes no state"""
    mesh = akb.box_tet4(5)
    v0, bl = sinusoidal_velocity(mesh.nodes, 0.03), blocked_face(mesh.nodes)

    def model(track):
        m = gpu_model(mesh, [UNIT_NEOHOOKEAN], precision=precision)
        m.setNodal("velocity", v0)
        m.setNodal("blocked_dofs", bl)
        m.setTimeStep(0.8 * m.getStableTimeStep())
        if track:
            m.setIncrementTracking(True)
        return m

    plain = model(False)
    with pytest.raises(akb.AkbError):
        plain.getIncrement()
    history = [plain.getDisplacement().copy()]
    for _ in range(152):
        plain.solveStep(1)
        history.append(plain.getDisplacement().copy())
    tracked = model(True)
    assert not np.any(tracked.getIncrement())
    tracked.solveStep(1)
    assert np.array_equal(tracked.getPreviousDisplacement(), history[0])
    assert np.array_equal(tracked.getIncrement(), history[1] - history[0])
    tracked.solveStep(150)  # one 100-step graph and 50 single steps
    assert np.array_equal(tracked.getDisplacement(), history[151])
    assert np.array_equal(tracked.getPreviousDisplacement(), history[150])
    assert np.array_equal(tracked.getIncrement(), history[151] - history[150])
    # a host write: the next step starts from the written displacement
    u = tracked.getDisplacement()
    u[:, 0] += 1e-4
    written = u.copy()
    tracked.solveStep(1)
    assert np.array_equal(tracked.getPreviousDisplacement(), written)
    assert np.array_equal(tracked.getIncrement(), tracked.getDisplacement() - written)


@pytest.mark.parametrize("etype", ["_tetrahedron_4", "_hexahedron_8", "_triangle_6"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_travelling_wave_bar(etype, precision):
    """the reference's explicit dynamics test (test_solid_mechanics_model_dynamics.cc)
    through the C ABI, the boundary written by the host before every step:
    error at most 2e-3, and the FP64 path equal to the oracle's run"""
    from scenarios import WAVE_MAT, run_wave, wave_bar
    mesh = wave_bar(etype)
    g = gpu_model(mesh, [WAVE_MAT], precision=precision)
    dt = g.getStableTimeStep() / 10
    g.setTimeStep(dt)
    err, steps = run_wave(mesh, g.setNodal,
                          lambda: (g.getDisplacement().copy(), g.getVelocity().copy()),
                          lambda: g.solveStep(1), dt)
    assert steps >= 100 and 0 < err < 2e-3
    if precision == "fp64":
        fields = {"displacement": orc.U, "velocity": orc.V, "blocked_dofs": orc.BLOCKED}
        o = oracle_model(mesh, [WAVE_MAT])
        o.set_dt(dt)
        err_o, _ = run_wave(mesh, lambda n, a: o.set(fields[n], a),
                            lambda: (o.get(orc.U), o.get(orc.V)), lambda: o.step(1), dt)
        assert err == err_o
        assert np.array_equal(g.getDisplacement(), o.get(orc.U))


def test_nodes_with_many_elements_fp64_bitwise():
    """a fan of 300 tetrahedra around one axis: two nodes with 300 slots each
    (long node-CSR rows), the oracle's trajectory bit for bit"""
    n = 300
    th = 2 * np.pi * np.arange(n) / n
    ring = np.stack([np.cos(th), np.sin(th), np.zeros(n)], axis=1)
    nodes = np.vstack([[0.0, 0.0, 0.0], [0.0, 0.0, 1.0], ring])
    conn = np.array([[0, 2 + k, 2 + (k + 1) % n, 1] for k in range(n)], dtype=np.int32)
    X = nodes[conn]
    vol = np.einsum("ij,ij->i", X[:, 1] - X[:, 0], np.cross(X[:, 2] - X[:, 0], X[:, 3] - X[:, 0]))
    conn[vol < 0] = conn[vol < 0][:, [0, 2, 1, 3]]
    mesh = akb.Mesh(3, nodes, conn, "_tetrahedron_4")
    v0 = np.zeros_like(nodes)
    v0[2:, 2] = 0.01 * np.sin(3 * th)
    bl = np.zeros(nodes.shape, np.uint8)
    bl[0] = 1
    g, o = setup_pair(mesh, [UNIT_ELASTIC], v0, bl)
    g.solveStep(60)
    o.step(60)
    compare(g, o, exact=True)

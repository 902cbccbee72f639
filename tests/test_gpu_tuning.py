"""Launch shapes and the autotuner: every candidate shape computes the same
numbers, the autotuner leaves the model's state alone, and the sum-factorised
mixed-precision hexahedron kernel agrees with the dN/dx form and with the
FP64 oracle."""
import numpy as np
import pytest

import akantu2_b200 as akb
from oracle import oracle as orc
from scenarios import (UNIT_ELASTIC, UNIT_NEOHOOKEAN, UNIT_PLASTIC, blocked_face,
                       random_field_velocity, sinusoidal_velocity)
from test_gpu_parity import gpu_model, setup_pair

pytestmark = pytest.mark.gpu

LAW_NAME = {"elastic": "elastic", "neohookean": "neohookean",
            "plastic_linear_isotropic_hardening": "plastic"}


def _run(mesh, mat, precision, v0, bl, steps, shape=None, autotune_at=None):
    m = gpu_model(mesh, [mat], precision=precision)
    m.setNodal("velocity", v0)
    m.setNodal("blocked_dofs", bl)
    m.setTimeStep(0.8 * m.getStableTimeStep())
    if shape is not None:
        m.setLaunchShape(mat["type"], *shape)
    if autotune_at is None:
        m.solveStep(steps)
    else:
        m.solveStep(autotune_at)
        m.autotune(2)
        m.solveStep(steps - autotune_at)
    return m


HEX_SHAPES = [(128, 8, 256), (64, 8, 128), (256, 8, 512)]
PE_SHAPES = [(64, 8, 128), (128, 8, 256), (256, 8, 1024)]


@pytest.mark.parametrize("mat", [UNIT_ELASTIC, UNIT_NEOHOOKEAN, UNIT_PLASTIC])
@pytest.mark.parametrize("qu", [8, 2, 1])
def test_hex8_mixed_shapes_are_bit_identical(mat, qu):
    """threads per block change nothing (points per iteration are a separate,
    untuned choice)"""
    mesh = akb.box_hex8(5)
    v0, bl = random_field_velocity(mesh.nodes, seed=4), blocked_face(mesh.nodes)
    ref = None
    shapes = [(b, qu, n, 1) for b, _, n in HEX_SHAPES] if qu != 1 else [(128, 1, 256, 1),
                                                                          (128, 1, 1024, 1)]
    shapes.append((128, qu, 256, 5))  # registers capped for 5 blocks per SM
    if qu == 2:
        shapes.append((128, qu, 256, 4))  # capped for 4 blocks per SM
    for shape in shapes:
        m = _run(mesh, mat, "mixed", v0, bl, 120, shape)
        got = (m.getDisplacement(), m.getVelocity(), m.getInternalForce())
        if ref is None:
            ref = got
        else:
            for a, b in zip(ref, got):
                assert np.array_equal(a, b), shape


@pytest.mark.parametrize("mat", [UNIT_ELASTIC, UNIT_NEOHOOKEAN, UNIT_PLASTIC])
def test_hex8_affine_and_general_elements(mat):
    """a box whose upper half is distorted: parallelepipeds (geometry formed
    once per element) and general hexahedra (per point) side by side, also
    within a warp, against the FP64 oracle"""
    mesh = akb.box_hex8(8)
    x = mesh.nodes
    rng = np.random.default_rng(17)
    inner = np.all((x > 1e-9) & (x < 1 - 1e-9), axis=1) & (x[:, 2] > 0.5) & (x[:, 0] > 0.3)
    x[inner] += rng.uniform(-0.12, 0.12, size=(inner.sum(), 3)) / 8
    v0, bl = sinusoidal_velocity(x, 0.03), blocked_face(x)
    g, o = setup_pair(mesh, [dict(mat, sigma_y=2e-3) if "sigma_y" in mat else mat], v0, bl,
                      precision="mixed")
    g.solveStep(400)
    o.step(400)
    uo = o.get(orc.U)
    assert np.linalg.norm(g.getDisplacement() - uo) / np.linalg.norm(uo) < 1e-5


@pytest.mark.parametrize("etype,precision,mat", [
    ("_tetrahedron_4", "fp64", UNIT_ELASTIC), ("_tetrahedron_4", "mixed", UNIT_NEOHOOKEAN),
    ("_triangle_6", "fp64", UNIT_PLASTIC), ("_triangle_6", "mixed", UNIT_PLASTIC)])
def test_block_sizes_are_bit_identical(etype, precision, mat):
    mesh = akb.box_tet4(4) if etype == "_tetrahedron_4" else akb.square_tri6(6)
    v0 = sinusoidal_velocity(mesh.nodes) if mesh.spatial_dimension == 3 else \
        np.stack([0.02 * mesh.nodes[:, 0], np.zeros(mesh.getNbNodes())], axis=1)
    bl = blocked_face(mesh.nodes, axis=mesh.spatial_dimension - 1 if etype != "_triangle_6" else 0)
    ref = None
    for shape in PE_SHAPES:
        m = _run(mesh, mat, precision, v0, bl, 90, shape)
        got = (m.getDisplacement(), m.getVelocity())
        if ref is None:
            ref = got
        else:
            for a, b in zip(ref, got):
                assert np.array_equal(a, b), shape


@pytest.mark.parametrize("etype,precision,mat", [
    ("_hexahedron_8", "mixed", UNIT_NEOHOOKEAN), ("_hexahedron_8", "fp64", UNIT_ELASTIC),
    ("_triangle_6", "mixed", UNIT_PLASTIC), ("_tetrahedron_4", "fp64", UNIT_ELASTIC)])
def test_autotune_leaves_the_state_alone(etype, precision, mat):
    mesh = {"_hexahedron_8": lambda: akb.box_hex8(4), "_triangle_6": lambda: akb.square_tri6(6),
            "_tetrahedron_4": lambda: akb.box_tet4(4)}[etype]()
    d = mesh.spatial_dimension
    v0 = sinusoidal_velocity(mesh.nodes) if d == 3 else \
        np.stack([0.02 * mesh.nodes[:, 0], np.zeros(mesh.getNbNodes())], axis=1)
    bl = blocked_face(mesh.nodes, axis=2 if d == 3 else 0)
    plain = _run(mesh, mat, precision, v0, bl, 150)
    tuned = _run(mesh, mat, precision, v0, bl, 150, autotune_at=70)
    for name in ("getDisplacement", "getVelocity", "getAcceleration", "getInternalForce"):
        assert np.array_equal(getattr(plain, name)(), getattr(tuned, name)()), name
    if mat is UNIT_PLASTIC:
        for f in ("inelastic_strain", "iso_hardening", "plastic_energy"):
            assert np.array_equal(plain.getMaterial(0).getInternal(f)(),
                                  tuned.getMaterial(0).getInternal(f)()), f
    b, q, mb, n = tuned.getLaunchShape(mat["type"])
    assert b in (64, 128, 256) and mb in (1, 4, 5, 6, 7, 8) and n in (128, 256, 512, 1024)


@pytest.mark.parametrize("mat", [UNIT_ELASTIC, UNIT_NEOHOOKEAN])
def test_hex8_sum_factorisation_accuracy(mat):
    """the sum-factorised FP32 kernel against the dN/dx FP32 form and the FP64
    oracle after 500 steps (relative L2 of the displacement)"""
    mesh = akb.box_hex8(8)
    v0, bl = random_field_velocity(mesh.nodes, seed=21), blocked_face(mesh.nodes)
    g, o = setup_pair(mesh, [mat], v0, bl, precision="mixed")
    g.solveStep(500)
    o.step(500)
    uo = o.get(orc.U)
    u = g.getDisplacement()
    assert np.linalg.norm(u - uo) / np.linalg.norm(uo) < 1e-5
    for qu in (0, 1, 2):  # the dN/dx form, and 1 or 2 points per iteration
        other = _run(mesh, mat, "mixed", v0, bl, 500, shape=(128, qu, 256)).getDisplacement()
        assert np.linalg.norm(other - uo) / np.linalg.norm(uo) < 1e-5, qu
        assert np.linalg.norm(other - u) / np.linalg.norm(uo) < 1e-5, qu


@pytest.mark.parametrize("etype,precision,mat", [
    ("_tetrahedron_4", "fp64", UNIT_ELASTIC), ("_tetrahedron_4", "mixed", UNIT_ELASTIC),
    ("_hexahedron_8", "mixed", UNIT_NEOHOOKEAN), ("_hexahedron_8", "fp64", UNIT_NEOHOOKEAN),
    ("_hexahedron_8", "mixed", UNIT_PLASTIC),
    ("_triangle_6", "fp64", UNIT_PLASTIC), ("_triangle_6", "mixed", UNIT_PLASTIC)])
def test_persistent_kernel_is_bit_identical(etype, precision, mat):
    """whole step sequences in one persistent launch give the state of the
    two-kernel graphs, including an odd step count and a host edit between"""
    mesh = {"_hexahedron_8": lambda: akb.box_hex8(5), "_triangle_6": lambda: akb.square_tri6(6),
            "_tetrahedron_4": lambda: akb.box_tet4(5)}[etype]()
    d = mesh.spatial_dimension
    v0 = sinusoidal_velocity(mesh.nodes, 0.03) if d == 3 else \
        np.stack([0.02 * mesh.nodes[:, 0], np.zeros(mesh.getNbNodes())], axis=1)
    bl = blocked_face(mesh.nodes, axis=2 if d == 3 else 0)
    runs = []
    for mode in (0, 2):  # graphs, cooperative grid
        m = gpu_model(mesh, [mat], precision=precision)
        if etype == "_hexahedron_8" and precision == "mixed" and mat is not UNIT_PLASTIC:
            # the persistent kernel has the scalar forms (1 or 2 points per
            # iteration), not the packed pairs of the default shape
            m.setLaunchShape(mat["type"], 128, 2, 256, 4)
        m.setPersistent(mode)
        assert m.persistentActive() == (mode != 0)
        m.setNodal("velocity", v0)
        m.setNodal("blocked_dofs", bl)
        m.setTimeStep(0.8 * m.getStableTimeStep())
        m.solveStep(137)
        f = m.getExternalForce()
        f[:, 0] = 1e-4
        m.solveStep(100)
        assert m.getStatus() == 0
        got = [m.getDisplacement().copy(), m.getVelocity().copy(), m.getAcceleration().copy(),
               m.getInternalForce().copy()]
        if mat is UNIT_PLASTIC:
            got += [m.getMaterial(0).getInternal(f)() for f in ("inelastic_strain",
                                                                "iso_hardening", "plastic_energy")]
        runs.append(got)
    for other in runs[1:]:
        for a, b in zip(runs[0], other):
            assert np.array_equal(a, b)


def test_persistent_batch_with_instance_time_steps():
    meshes = [akb.box_tet4(n) for n in (2, 3, 4)]
    outs = []
    for mode in (0, 2):
        b = akb.BatchModel(meshes)
        for k in range(3):
            b.addMaterial("elastic", name=f"m{k}", rho=1.0, E=0.5 + k, nu=0.3)
        b.setInstanceMaterials(np.arange(3))
        b.initFull(akb._explicit_lumped_mass, precision="mixed")
        b.setPersistent(mode)
        assert b.persistentActive() == (mode != 0)
        b.setNodal("velocity", np.concatenate([sinusoidal_velocity(m.nodes) for m in meshes]))
        b.setNodal("blocked_dofs", np.concatenate([blocked_face(m.nodes) for m in meshes]))
        b.setTimeSteps(0.8 * b.getStableTimeSteps())
        b.solveStep(251)
        outs.append((b.getDisplacement().copy(), b.getVelocity().copy()))
    for other in outs[1:]:
        for a, c in zip(outs[0], other):
            assert np.array_equal(a, c)


@pytest.mark.parametrize("etype,precision,mat", [
    ("_tetrahedron_4", "mixed", UNIT_ELASTIC), ("_tetrahedron_4", "fp64", UNIT_ELASTIC),
    ("_hexahedron_8", "mixed", UNIT_NEOHOOKEAN), ("_hexahedron_8", "fp64", UNIT_ELASTIC),
    ("_triangle_6", "mixed", UNIT_PLASTIC), ("_triangle_6", "fp64", UNIT_PLASTIC)])
def test_staged_node_gather_is_bit_identical(etype, precision, mat):
    """the shared-memory staged gather, and the direct gather with the node's
    state read first (form 2), sum every node's slots in the order of the
    direct gather: identical states, for every block size (small chunks are
    exercised by the 512-thread blocks of tetrahedra, 24 slots a node)"""
    mesh = {"_hexahedron_8": lambda: akb.box_hex8(6), "_triangle_6": lambda: akb.square_tri6(8),
            "_tetrahedron_4": lambda: akb.box_tet4(8)}[etype]()
    d = mesh.spatial_dimension
    v0 = sinusoidal_velocity(mesh.nodes, 0.03) if d == 3 else \
        np.stack([0.02 * mesh.nodes[:, 0], np.zeros(mesh.getNbNodes())], axis=1)
    bl = blocked_face(mesh.nodes, axis=2 if d == 3 else 0)
    runs = []
    for shape in [(128, 0), (128, 1), (256, 1), (512, 1), (128, 2), (512, 2)]:
        m = gpu_model(mesh, [mat], precision=precision)
        m.setNodeShape(*shape)
        assert m.getNodeShape() == shape
        m.setNodal("velocity", v0)
        m.setNodal("blocked_dofs", bl)
        m.setTimeStep(0.8 * m.getStableTimeStep())
        m.solveStep(123)
        runs.append((m.getDisplacement().copy(), m.getVelocity().copy(),
                     m.getInternalForce().copy()))
    for other in runs[1:]:
        for a, b in zip(runs[0], other):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("etype,precision,mat", [
    ("_tetrahedron_4", "mixed", UNIT_ELASTIC), ("_tetrahedron_4", "fp64", UNIT_PLASTIC),
    ("_hexahedron_8", "mixed", UNIT_NEOHOOKEAN), ("_hexahedron_8", "fp64", UNIT_ELASTIC),
    ("_triangle_6", "mixed", UNIT_PLASTIC), ("_triangle_6", "fp64", UNIT_NEOHOOKEAN)])
def test_dependent_launch_is_bit_identical(etype, precision, mat):
    """programmatic stream serialization only changes when a step kernel is
    scheduled, not what it computes: identical states with and without it,
    through graphs, single steps, a velocity ramp on blocked dofs (one more
    kernel per step) and both node-update forms"""
    mesh = {"_hexahedron_8": lambda: akb.box_hex8(6), "_triangle_6": lambda: akb.square_tri6(8),
            "_tetrahedron_4": lambda: akb.box_tet4(8)}[etype]()
    d = mesh.spatial_dimension
    v0 = sinusoidal_velocity(mesh.nodes, 0.03) if d == 3 else \
        np.stack([0.02 * mesh.nodes[:, 0], np.zeros(mesh.getNbNodes())], axis=1)
    bl = blocked_face(mesh.nodes, axis=2 if d == 3 else 0)
    top = np.flatnonzero(np.isclose(mesh.nodes[:, d - 1], mesh.nodes[:, d - 1].max()))
    runs = []
    for pdl, staged in [(False, 0), (True, 0), (True, 1), (True, 2), (False, 2)]:
        m = gpu_model(mesh, [mat], precision=precision)
        m.setDependentLaunch(pdl)
        assert m.getDependentLaunch() == pdl
        m.setNodeShape(128, staged)
        m.setNodal("velocity", v0)
        m.setNodal("blocked_dofs", bl)
        m.setTimeStep(0.8 * m.getStableTimeStep())
        m.setPrescribedVelocityRamp(top, d - 1, 0.05, 40)
        m.solveStep(3)
        m.solveStep(207)
        runs.append((m.getDisplacement().copy(), m.getVelocity().copy(),
                     m.getInternalForce().copy(), m.getMaterial(0).getStress().copy()))
    for other in runs[1:]:
        for a, b in zip(runs[0], other):
            assert np.array_equal(a, b)


def test_dependent_launch_batch_is_bit_identical():
    meshes = [akb.box_tet4(n) for n in (3, 5, 4)]
    runs = []
    for pdl in (False, True):
        b = akb.BatchModel(meshes)
        for e in (0.5, 1.0, 2.0):
            b.addMaterial("elastic", rho=1.0, E=e, nu=0.3)
        b.setInstanceMaterials(np.arange(3))
        b.initFull(akb._explicit_lumped_mass, precision="mixed")
        b.setDependentLaunch(pdl)
        x = np.concatenate([m.nodes for m in meshes])
        b.setNodal("velocity", sinusoidal_velocity(x, 0.03))
        b.setNodal("blocked_dofs", blocked_face(x, axis=2))
        b.setTimeSteps(0.8 * b.getStableTimeSteps())
        b.solveStep(250)
        runs.append((b.getDisplacement().copy(), b.getVelocity().copy()))
    for a, c in zip(*runs):
        assert np.array_equal(a, c)


@pytest.mark.parametrize("etype,precision", [
    ("_tetrahedron_4", "fp64"), ("_tetrahedron_4", "mixed"), ("_triangle_6", "fp64"),
    ("_triangle_6", "mixed")])
def test_plastic_register_caps_are_bit_identical(etype, precision):
    """128-thread plastic kernels with registers capped for 5 to 8 resident
    blocks per SM compute the same numbers, and so does the streamed law of
    plastic triangles with each cap"""
    mesh = {"_triangle_6": lambda: akb.square_tri6(8), "_tetrahedron_4": lambda: akb.box_tet4(6)}[etype]()
    d = mesh.spatial_dimension
    mat = dict(UNIT_PLASTIC, sigma_y=2e-3)
    v0 = sinusoidal_velocity(mesh.nodes, 0.05) if d == 3 else \
        np.stack([0.05 * mesh.nodes[:, 0], np.zeros(mesh.getNbNodes())], axis=1)
    bl = blocked_face(mesh.nodes, axis=2 if d == 3 else 0)
    runs = []
    shapes = [(mb, False) for mb in (1, 5, 6, 7, 8)]
    if etype == "_triangle_6":
        shapes += [(mb, True) for mb in (1, 5, 6, 7, 8)]
    for mb, streamed in shapes:
        m = gpu_model(mesh, [mat], precision=precision)
        m.setLaunchShape(mat["type"], 128, 8, 128, mb)
        m.setPrefetch(mat["type"], 0)
        m.setRecomputeGeometry(mat["type"], False)
        m.setStreamedPoints(mat["type"], streamed)
        assert m.getLaunchShape(mat["type"])[2] == mb
        assert m.getStreamedPoints(mat["type"]) == streamed
        m.setNodal("velocity", v0)
        m.setNodal("blocked_dofs", bl)
        m.setTimeStep(0.8 * m.getStableTimeStep())
        m.solveStep(150)
        runs.append((m.getDisplacement().copy(), m.getVelocity().copy(),
                     m.getMaterial(0).getInternal("inelastic_strain")().copy()))
    assert np.max(np.abs(runs[0][2])) > 0, "the run must yield"
    for other in runs[1:]:
        for a, b in zip(runs[0], other):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("mat", [UNIT_ELASTIC, UNIT_NEOHOOKEAN, UNIT_PLASTIC])
def test_affine_kernel_is_bit_identical(mat):
    """a box of parallelepipeds runs the element kernel compiled without
    per-point geometry by default; that kernel reading the geometry table
    (mode 2) and the general kernel compute the same numbers in every launch
    shape"""
    mesh = akb.box_hex8(5, 4, 6, lengths=(1.0, 0.7, 1.3))
    v0, bl = sinusoidal_velocity(mesh.nodes, 0.03), blocked_face(mesh.nodes)
    mat = dict(mat, sigma_y=2e-3) if "sigma_y" in mat else mat
    runs = []
    for affine in (2, 1, 0):
        for shape in ((128, 2, 4), (128, 2, 5), (128, 2, 6), (128, 1, 5), (128, 1, 6),
                      (128, 8, 1)):
            m = gpu_model(mesh, [mat], precision="mixed")
            assert m.getAffineKernel() in (1, 2)
            m.setAffineKernel(affine)
            assert m.getAffineKernel() == affine
            m.setLaunchShape(mat["type"], shape[0], shape[1], 128, shape[2])
            m.setNodal("velocity", v0)
            m.setNodal("blocked_dofs", bl)
            m.setTimeStep(0.8 * m.getStableTimeStep())
            m.solveStep(130)
            runs.append(((affine,) + shape, m.getDisplacement().copy(), m.getVelocity().copy()))
    for qu in (2, 1, 8):
        same = [r for r in runs if r[0][2] == qu]
        for other in same[1:]:
            assert np.array_equal(same[0][1], other[1]), (same[0][0], other[0])
            assert np.array_equal(same[0][2], other[2]), (same[0][0], other[0])


def test_affine_kernel_only_for_parallelepipeds():
    mesh = akb.box_hex8(4)
    mesh.nodes[np.all((mesh.nodes > 0.1) & (mesh.nodes < 0.9), axis=1)] += 0.01
    m = gpu_model(mesh, [UNIT_ELASTIC], precision="mixed")
    assert not m.getAffineKernel()
    for mode in (True, 2):
        with pytest.raises(akb.AkbError):
            m.setAffineKernel(mode)
    assert not gpu_model(akb.box_hex8(3), [UNIT_ELASTIC], precision="fp64").getAffineKernel()
    assert not gpu_model(akb.box_tet4(3), [UNIT_ELASTIC], precision="mixed").getAffineKernel()


PACK = 256  # AKB_POINTS_PACKED


@pytest.mark.parametrize("mat", [UNIT_ELASTIC, UNIT_NEOHOOKEAN])
def test_hex8_packed_pairs_are_the_default_and_bit_identical(mat):
    """meshes of parallelepipeds evaluate elastic and neohookean points as
    packed FP32 pairs by default; every packed shape (points per iteration,
    register cap) and both affine kernel modes give the same numbers"""
    mesh = akb.box_hex8(5, 4, 6, lengths=(1.0, 0.7, 1.3))
    v0, bl = sinusoidal_velocity(mesh.nodes, 0.03), blocked_face(mesh.nodes)
    m = gpu_model(mesh, [mat], precision="mixed")
    b, q, mb, n = m.getLaunchShape(mat["type"])
    assert q == PACK | 8 and b == 128
    assert m.getPrefetch(mat["type"]) == 0
    runs = []
    shapes = [(affine, PACK | pts, minb) for affine in (2, 1) for pts in (2, 4, 8)
              for minb in (1, 4, 5)]
    for affine, q, minb in shapes:
        m = gpu_model(mesh, [mat], precision="mixed")
        m.setAffineKernel(affine)
        m.setLaunchShape(mat["type"], 128, q, 128, minb)
        m.setNodal("velocity", v0)
        m.setNodal("blocked_dofs", bl)
        m.setTimeStep(0.8 * m.getStableTimeStep())
        m.solveStep(130)
        runs.append(((affine, q, minb), m.getDisplacement().copy(), m.getVelocity().copy(),
                     m.getInternalForce().copy()))
    for other in runs[1:]:
        for a, b_ in zip(runs[0][1:], other[1:]):
            assert np.array_equal(a, b_), (runs[0][0], other[0])


@pytest.mark.parametrize("mat", [UNIT_ELASTIC, UNIT_NEOHOOKEAN])
def test_hex8_packed_pairs_accuracy(mat):
    """the packed form against the FP64 oracle and the scalar form after 500
    steps (relative L2 of the displacement)"""
    mesh = akb.box_hex8(8)
    v0, bl = random_field_velocity(mesh.nodes, seed=21), blocked_face(mesh.nodes)
    g, o = setup_pair(mesh, [mat], v0, bl, precision="mixed")
    assert g.getLaunchShape(mat["type"])[1] & PACK
    g.solveStep(500)
    o.step(500)
    uo = o.get(orc.U)
    u = g.getDisplacement()
    assert np.linalg.norm(u - uo) / np.linalg.norm(uo) < 1e-5
    scalar = _run(mesh, mat, "mixed", v0, bl, 500, shape=(128, 2, 256, 5)).getDisplacement()
    assert np.linalg.norm(scalar - u) / np.linalg.norm(uo) < 1e-5


def test_hex8_packed_l2_prefetch_is_bit_identical():
    """the L2 prefetch distance of the packed kernel (0 = off, 1, 2 and 4
    waves of resident blocks) changes no number: a box large enough for the
    prefetching warps to exist, two law groups (the second starting past
    element 0, a table offset), the default shapes and both register caps"""
    mesh = akb.box_hex8(60)
    E = mesh.getNbElement()
    assert E > 2 * 148 * 5 * 128  # two waves of the 5-block cap
    mat_of_elem = (np.arange(E) >= E // 3).astype(np.int32)
    mats = [UNIT_ELASTIC, UNIT_NEOHOOKEAN]
    v0, bl = sinusoidal_velocity(mesh.nodes, 0.03), blocked_face(mesh.nodes)
    runs = []
    for minb in (4, 5):
        for pf in (0, 1, 2, 4):
            m = gpu_model(mesh, mats, mat_of_elem=mat_of_elem, precision="mixed")
            for law in ("elastic", "neohookean"):
                m.setLaunchShape(law, 128, PACK | 8, 128, minb)
                m.setPrefetch(law, pf)
                assert m.getPrefetch(law) == pf
            m.setNodal("velocity", v0)
            m.setNodal("blocked_dofs", bl)
            m.setTimeStep(0.8 * m.getStableTimeStep())
            m.solveStep(130)
            runs.append(((minb, pf), m.getDisplacement().copy(), m.getVelocity().copy(),
                         m.getInternalForce().copy()))
            del m
    for other in runs[1:]:
        for a, b_ in zip(runs[0][1:], other[1:]):
            assert np.array_equal(a, b_), (runs[0][0], other[0])


@pytest.mark.parametrize("case", ["tet4_elastic", "tet4_neohookean", "tri6_plastic3",
                                  "tri6_plastic6", "tri6_elastic6"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_recomputed_geometry_and_prefetch_are_bit_identical(case, precision):
    """tetrahedra and triangles: dN/dx and det J w recomputed from the
    coordinates every step (the precomputation's explicitly rounded FP64
    arithmetic) instead of streamed, and the L2 prefetch of later warps' rows,
    on or off: every combination, with the plastic register caps, gives the
    same nodal fields and plastic internals"""
    etype, law = case.split("_")
    qp_rule = 1 if law.endswith("6") else 0
    law = law.rstrip("36")
    if etype == "tet4":
        mesh = akb.box_tet4(30)  # 162,000 elements: the prefetching warps exist
        mat = dict(UNIT_ELASTIC if law == "elastic" else UNIT_NEOHOOKEAN)
        v0 = sinusoidal_velocity(mesh.nodes, 0.02)
        bl = blocked_face(mesh.nodes)
    else:
        mesh = akb.square_tri6(200)  # 80,000 elements
        mat = dict(UNIT_PLASTIC, sigma_y=2e-3) if law == "plastic" else dict(UNIT_ELASTIC)
        x = mesh.nodes
        v0 = np.zeros_like(x)
        v0[:, 0] = 0.05 * x[:, 0] * x[:, 1]
        bl = np.zeros(x.shape, dtype=np.uint8)
        bl[np.isclose(x[:, 0], 0.0)] = 1
    name = LAW_NAME[mat["type"]]
    shapes = [(128, 8, 1, 0, 0), (128, 8, 1, 1, 0), (128, 8, 1, 0, 1), (128, 8, 1, 1, 1),
              (64, 8, 1, 1, 1), (256, 8, 1, 1, 1)]
    if law == "plastic":
        shapes += [(128, 8, 5, 1, 1), (128, 8, 6, 1, 1), (128, 8, 6, 0, 1)]
    if etype == "tet4" and precision == "fp64":
        # FP64 elastic and neohookean tetrahedra: the recomputed-geometry kernel
        # with registers capped for 6 and 7 blocks, with and without prefetch
        shapes += [(128, 8, 6, 1, 1), (128, 8, 6, 1, 0), (128, 8, 7, 1, 1), (128, 8, 7, 1, 0)]
    runs = []
    for block, q, minb, rec, pf in shapes:
        m = gpu_model(mesh, [mat], precision=precision, qp_rule=qp_rule)
        m.setLaunchShape(mat["type"], block, q, 256, minb)
        m.setRecomputeGeometry(mat["type"], rec)
        m.setPrefetch(mat["type"], pf)
        assert m.getRecomputeGeometry(mat["type"]) == bool(rec)
        m.setNodal("velocity", v0)
        m.setNodal("blocked_dofs", bl)
        m.setTimeStep(0.8 * m.getStableTimeStep())
        m.solveStep(120)
        fields = [m.getDisplacement().copy(), m.getVelocity().copy(),
                  m.getAcceleration().copy(), m.getInternalForce().copy()]
        if name == "plastic":
            mt = m.getMaterial(0)
            fields += [mt.getStress().copy(), mt.getInternal("inelastic_strain")().copy()]
        runs.append(((block, q, minb, rec, pf), fields))
        del m
    if name == "plastic":
        assert np.max(np.abs(runs[0][1][5])) > 0, "the square must yield"
    for other in runs[1:]:
        for a, b_ in zip(runs[0][1], other[1]):
            assert np.array_equal(a, b_), (runs[0][0], other[0])


def test_recomputed_geometry_batch_is_bit_identical():
    """a tetrahedral batch (per-instance materials and time steps) with the
    geometry recomputed and the prefetch on, against the streamed tables"""
    import bench
    meshes, mats, vels, blocks = bench.batch_workload(12)
    runs = []
    for rec, pf in ((0, 0), (1, 1), (1, 0)):
        for precision in ("fp64", "mixed"):
            b = bench.build_batch(akb, meshes, mats, vels, blocks, precision)
            b.setRecomputeGeometry("elastic", rec)
            b.setPrefetch("elastic", pf)
            b.solveStep(130)
            runs.append(((rec, pf, precision), b.getDisplacement().copy(), b.getVelocity().copy()))
            del b
    for other in runs[2:]:
        ref = runs[0] if other[0][2] == "fp64" else runs[1]
        for a, b_ in zip(ref[1:], other[1:]):
            assert np.array_equal(a, b_), (ref[0], other[0])


def test_geometry_and_prefetch_defaults():
    """FP64 elastic and neohookean tetrahedra recompute the geometry and
    prefetch the next wave's rows; mixed tetrahedra and plastic triangles do
    neither"""
    for precision in ("fp64", "mixed"):
        t = gpu_model(akb.box_tet4(3), [UNIT_ELASTIC], precision=precision)
        assert t.getPrefetch("elastic") == (1 if precision == "fp64" else 0)
        assert t.getRecomputeGeometry("elastic") == (precision == "fp64")
        p = gpu_model(akb.square_tri6(3), [UNIT_PLASTIC], precision=precision)
        law = UNIT_PLASTIC["type"]
        assert p.getPrefetch(law) == 0 and not p.getRecomputeGeometry(law)


def test_recomputed_geometry_setting_rules():
    h = gpu_model(akb.box_hex8(3), [UNIT_ELASTIC], precision="fp64")
    with pytest.raises(akb.AkbError):
        h.setRecomputeGeometry("elastic", True)
    t = gpu_model(akb.box_tet4(3), [UNIT_ELASTIC], precision="mixed")
    assert not t.getRecomputeGeometry("elastic")
    t.setRecomputeGeometry("elastic", True)
    t.setLaunchShape("elastic", 128, 0, 128, 1)  # the FP32 recomputed form
    with pytest.raises(akb.AkbError):
        t.setRecomputeGeometry("elastic", True)


def test_l2_prefetch_setting_rules():
    m = gpu_model(akb.box_hex8(3), [UNIT_NEOHOOKEAN], precision="mixed")
    with pytest.raises(akb.AkbError):
        m.setPrefetch("neohookean", 5)
    with pytest.raises(akb.AkbError):
        m.setPrefetch("elastic", 1)  # no such law group
    m.setLaunchShape("neohookean", 128, 2, 128, 5)  # the scalar kernel: no prefetch
    assert m.getPrefetch("neohookean") == 0
    with pytest.raises(akb.AkbError):
        m.setPrefetch("neohookean", 1)
    m.setPrefetch("neohookean", 0)
    f = gpu_model(akb.box_hex8(3), [UNIT_ELASTIC], precision="fp64")  # per-point kernel
    with pytest.raises(akb.AkbError):
        f.setPrefetch("elastic", 1)


def test_hex8_packed_shape_rules():
    mesh = akb.box_hex8(3)
    m = gpu_model(mesh, [UNIT_NEOHOOKEAN], precision="mixed")
    with pytest.raises(akb.AkbError):
        m.setLaunchShape("neohookean", 64, PACK | 8, 128, 1)  # 128 threads only
    with pytest.raises(akb.AkbError):
        m.setLaunchShape("neohookean", 128, PACK | 3, 128, 1)
    m.setAffineKernel(0)  # no packed form for the general kernel: scalar again
    b, q, mb, n = m.getLaunchShape("neohookean")
    assert not (q & PACK)
    with pytest.raises(akb.AkbError):
        m.setLaunchShape("neohookean", 128, PACK | 8, 128, 4)
    p = gpu_model(mesh, [UNIT_PLASTIC], precision="mixed")
    with pytest.raises(akb.AkbError):
        p.setLaunchShape("plastic_linear_isotropic_hardening", 128, PACK | 2, 128, 5)


def test_persistent_barrier_wait_runs_out_and_reports():
    """the failure path of the persistent kernel's grid barrier: with a short
    bound on its waits and one block arriving late, a wait runs out, the
    launch ends and status bit 1 reports it; the context stays usable and the
    default bound steps normally again (bit-identical to the step graphs from
    the same state)"""
    import time
    from akantu2_b200 import _capi
    mesh = akb.box_tet4(10)  # 6,000 elements: 24 blocks of the persistent grid
    v0, bl = sinusoidal_velocity(mesh.nodes, 0.03), blocked_face(mesh.nodes)
    m = gpu_model(mesh, [UNIT_ELASTIC])
    m.setPersistent(2)
    assert m.persistentActive()
    m.setNodal("velocity", v0)
    m.setNodal("blocked_dofs", bl)
    dt = 0.8 * m.getStableTimeStep()
    m.setTimeStep(dt)
    L = _capi.lib()
    # waits bounded at 64 sleeps (about 2 us); block 1 starts 20 ms late
    _capi.check(L.akb_model_set_persistent_wait_test(m._h, 64, 1, 20000))
    t0 = time.perf_counter()
    m.solveStep(5)
    status = m.getStatus()
    assert status & 2, status
    assert time.perf_counter() - t0 < 10.0
    _capi.check(L.akb_model_set_persistent_wait_test(m._h, 0, -1, 0))
    # a fresh state written by the host, then steps with the default bound
    zero = np.zeros_like(mesh.nodes)
    for name, val in (("displacement", zero), ("velocity", v0), ("acceleration", zero)):
        m.setNodal(name, val)
    m.solveStep(40)
    assert m.getStatus() == 0
    ref = gpu_model(mesh, [UNIT_ELASTIC])
    ref.setNodal("velocity", v0)
    ref.setNodal("blocked_dofs", bl)
    ref.setTimeStep(dt)
    ref.solveStep(40)
    assert np.array_equal(m.getDisplacement(), ref.getDisplacement())
    assert np.array_equal(m.getVelocity(), ref.getVelocity())


@pytest.mark.parametrize("mat", [UNIT_ELASTIC, UNIT_NEOHOOKEAN, UNIT_PLASTIC])
@pytest.mark.parametrize("eigen", [False, True])
def test_hex8_fp64_streamed_points_are_bit_identical(mat, eigen):
    """plain FP64 hexahedra: the per-point kernel with the streamed law (dN/dx
    rows loaded where used, forces written to shared memory as formed) and
    with the point's row and forces held in registers give the same nodal
    fields and internals, on a partly distorted box with two materials of
    the law, with and without an eigen gradient; the streamed form is the
    default of the neohookean and plastic laws"""
    mesh = akb.box_hex8(9)  # 729 elements: 23 blocks of 32, the last one partial
    x = mesh.nodes
    rng = np.random.default_rng(5)
    inner = np.all((x > 1e-9) & (x < 1 - 1e-9), axis=1) & (x[:, 2] > 0.4)
    x[inner] += rng.uniform(-0.1, 0.1, size=(inner.sum(), 3)) / 9
    v0, bl = sinusoidal_velocity(x, 0.04), blocked_face(x)
    m1 = dict(mat, sigma_y=2e-3) if "sigma_y" in mat else dict(mat)
    m2 = dict(m1, name=m1["name"] + "_b", E=1.7, nu=0.25)
    if eigen:
        m1["eigen_grad_u"] = 0.01 * np.arange(9.0).reshape(3, 3)
    mat_of_elem = (np.arange(mesh.connectivity.shape[0]) % 3 == 0).astype(np.int32)
    name = LAW_NAME[mat["type"]]
    runs = []
    for streamed in (True, False):
        m = gpu_model(mesh, [m1, m2], mat_of_elem=mat_of_elem, precision="fp64")
        assert m.getStreamedPoints(mat["type"]) == (name != "elastic")
        m.setStreamedPoints(mat["type"], streamed)
        assert m.getStreamedPoints(mat["type"]) == streamed
        m.setNodal("velocity", v0)
        m.setNodal("blocked_dofs", bl)
        m.setTimeStep(0.8 * m.getStableTimeStep())
        m.solveStep(37)    # single launches, then a 100-step graph
        m.solveStep(100)
        fields = [m.getDisplacement().copy(), m.getVelocity().copy(),
                  m.getAcceleration().copy(), m.getInternalForce().copy()]
        for k in range(2):
            mt = m.getMaterial(k)
            fields.append(mt.getGradU().copy())
            if name == "plastic":
                fields += [mt.getStress().copy(), mt.getInternal("inelastic_strain")().copy()]
        runs.append(fields)
        del m
    if name == "plastic":
        assert np.max(np.abs(runs[0][6])) > 0, "the box must yield"
    for a, b_ in zip(runs[0], runs[1]):
        assert np.array_equal(a, b_)


def test_hex8_fp64_streamed_points_setting_rules():
    """the streamed law is a setting of plain FP64 hexahedra only; the
    autotuner keeps the state and picks one of the two forms"""
    for etype, precision in (("hex8", "mixed"), ("hex8", "fp64_fast"), ("tet4", "fp64"),
                             ("tri6", "mixed")):
        mesh = {"hex8": akb.box_hex8, "tet4": akb.box_tet4, "tri6": akb.square_tri6}[etype](3)
        m = gpu_model(mesh, [UNIT_ELASTIC], precision=precision)
        assert not m.getStreamedPoints("elastic")
        with pytest.raises(akb.AkbError):
            m.setStreamedPoints("elastic", True)
        m.setStreamedPoints("elastic", False)
    # plastic triangles: 128 threads and the streamed tables; a prefetch turns it off
    p = gpu_model(akb.square_tri6(3), [UNIT_PLASTIC], precision="mixed")
    law = UNIT_PLASTIC["type"]
    p.setStreamedPoints(law, True)
    assert p.getStreamedPoints(law)
    p.setPrefetch(law, 1)
    assert not p.getStreamedPoints(law)
    p.setPrefetch(law, 0)
    p.setLaunchShape(law, 64, 8, 128, 1)
    with pytest.raises(akb.AkbError):
        p.setStreamedPoints(law, True)
    mesh = akb.box_hex8(6)
    v0, bl = sinusoidal_velocity(mesh.nodes, 0.03), blocked_face(mesh.nodes)
    ref = _run(mesh, UNIT_NEOHOOKEAN, "fp64", v0, bl, 60)
    tuned = _run(mesh, UNIT_NEOHOOKEAN, "fp64", v0, bl, 60, autotune_at=20)
    assert np.array_equal(ref.getDisplacement(), tuned.getDisplacement())
    assert np.array_equal(ref.getVelocity(), tuned.getVelocity())

"""Several constitutive laws in one mesh, and batches of independent meshes.

A law group runs the elements of all its materials in one launch (per-element
parameters); a batch advances many meshes in the same launches, each with its
own time step.  Both must give exactly the results of the reference's order
of operations: the oracle for FP64, and the same mesh run alone for either
precision.
"""
import numpy as np
import pytest

import akantu2_b200 as akb
from oracle import oracle as orc
from scenarios import (UNIT_ELASTIC, UNIT_NEOHOOKEAN, UNIT_PLASTIC, blocked_face, oracle_model,
                       sinusoidal_velocity)
from test_gpu_parity import NODAL, compare, gpu_model, rel_err, setup_pair

pytestmark = pytest.mark.gpu


def _getter(name):
    return "get" + "".join(w.capitalize() for w in name.split("_"))


def test_interleaved_laws_tet4_bitwise():
    """plastic / elastic / plastic materials interleaved element by element:
    two law groups, the plastic one with two parameter sets."""
    mesh = akb.box_tet4(4)
    E = mesh.getNbElement()
    mat_of_elem = (np.arange(E) % 3).astype(np.int32)
    mats = [dict(UNIT_PLASTIC, name="p0"), dict(UNIT_ELASTIC, name="e1", E=1.5, nu=0.25),
            dict(UNIT_PLASTIC, name="p2", E=0.7, sigma_y=5e-4, h=0.2)]
    v0 = sinusoidal_velocity(mesh.nodes, amplitude=0.05)
    g, o = setup_pair(mesh, mats, v0, blocked_face(mesh.nodes), mat_of_elem=mat_of_elem)
    assert np.array_equal(g.getMass(), o.get(orc.MASS))
    g.setGraphSteps(10)
    g.solveStep(61)
    o.step(61)
    compare(g, o, exact=True)
    for k in (0, 2):
        mk = g.getMaterial(k)
        assert np.array_equal(mk.getInternal("inelastic_strain")(), o.qp(k, orc.EPS_P))
        assert np.array_equal(mk.getInternal("iso_hardening")(), o.qp(k, orc.ISO))
        assert np.array_equal(mk.getStress(), o.qp(k, orc.STRESS))
    assert np.max(np.abs(o.qp(0, orc.EPS_P))) > 0, "material 0 must yield"
    # energies are sums over all quadrature points: the reduction order differs
    for name, which in [("plastic", orc.EPLASTIC), ("potential", orc.EPOT)]:
        a, b = g.getEnergy(name), o.energy(which)
        assert b != 0 and abs(a - b) <= 1e-12 * abs(b), name


def test_interleaved_laws_mass_order_with_shared_nodes():
    """two densities on elements sharing nodes: the lumped mass sums in element
    order, the internal force material by material"""
    mesh = akb.box_hex8(3)
    E = mesh.getNbElement()
    mat_of_elem = (np.arange(E) % 2).astype(np.int32)
    mats = [dict(UNIT_ELASTIC, name="a", rho=1.0 / 3.0), dict(UNIT_NEOHOOKEAN, name="b", rho=0.7)]
    v0 = sinusoidal_velocity(mesh.nodes, amplitude=0.02)
    g, o = setup_pair(mesh, mats, v0, blocked_face(mesh.nodes), mat_of_elem=mat_of_elem)
    assert np.array_equal(g.getMass(), o.get(orc.MASS))
    g.solveStep(20)
    o.step(20)
    compare(g, o, exact=False)


def _instances(seed, count=4):
    rng = np.random.default_rng(seed)
    meshes, mats, vels = [], [], []
    for k in range(count):
        n = int(rng.integers(2, 5))
        mesh = akb.box_tet4(n)
        meshes.append(mesh)
        mats.append(dict(UNIT_ELASTIC, name=f"inst{k}", E=float(np.exp(rng.uniform(np.log(0.5),
                                                                                  np.log(2.0)))),
                         nu=float(rng.uniform(0.2, 0.4))))
        kx, ky = rng.integers(1, 5, size=2)
        v = np.zeros_like(mesh.nodes)
        v[:, 2] = 0.01 * np.sin(kx * np.pi * mesh.nodes[:, 0]) * np.sin(ky * np.pi * mesh.nodes[:, 1])
        vels.append(v)
    return meshes, mats, vels


def _batch(meshes, mats, vels, precision):
    b = akb.BatchModel(meshes)
    for mat in mats:
        b.addMaterial(mat["type"], **{k: v for k, v in mat.items() if k != "type"})
    b.setInstanceMaterials(np.arange(len(meshes)))
    b.initFull(akb._explicit_lumped_mass, precision=precision)
    b.setNodal("velocity", np.concatenate(vels))
    b.setNodal("blocked_dofs", np.concatenate([blocked_face(m.nodes) for m in meshes]))
    return b


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_matches_instances_alone(precision):
    meshes, mats, vels = _instances(seed=5)
    b = _batch(meshes, mats, vels, precision)
    dts = b.getStableTimeSteps()
    b.setTimeSteps(0.8 * dts)
    b.setGraphSteps(10)
    b.solveStep(45)
    for k, mesh in enumerate(meshes):
        alone = gpu_model(mesh, [mats[k]], precision=precision)
        alone.setNodal("velocity", vels[k])
        alone.setNodal("blocked_dofs", blocked_face(mesh.nodes))
        assert alone.getStableTimeStep() == dts[k]
        alone.setTimeStep(0.8 * dts[k])
        alone.solveStep(45)
        sl = b.instance_nodes(k)
        for name, _ in NODAL + [("mass", None)]:
            a = getattr(b, _getter(name))()[sl]
            c = getattr(alone, _getter(name))()
            assert np.array_equal(a, c), f"instance {k} {name}: rel {rel_err(a, c):.3e}"
        if precision == "fp64":
            o = oracle_model(mesh, [mats[k]])
            o.set(orc.V, vels[k])
            o.set(orc.BLOCKED, blocked_face(mesh.nodes))
            o.set_dt(0.8 * dts[k])
            o.step(45)
            for name, fid in NODAL:
                assert np.array_equal(getattr(b, _getter(name))()[sl], o.get(fid)), (k, name)


def test_batch_time_steps_and_offsets():
    meshes, mats, vels = _instances(seed=9, count=3)
    b = _batch(meshes, mats, vels, "fp64")
    assert b.nb_instances == 3
    assert b.getMass().shape == (sum(m.getNbNodes() for m in meshes), 3)
    dts = b.getStableTimeSteps()
    assert np.all(dts > 0)
    assert b.getStableTimeStep() == dts.min()
    b.setTimeStep(0.5 * dts.min())
    assert np.all(b.getTimeSteps() == 0.5 * dts.min())
    b.setTimeSteps(0.8 * dts)
    assert np.array_equal(b.getTimeSteps(), 0.8 * dts)
    with pytest.raises(ValueError):
        b.setTimeSteps(dts[:2])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("graph_steps", [0, 10])
def test_instances_stop_after_their_own_steps(precision, graph_steps):
    """a batch whose instances stop after their own step counts (the serving
    loop's batches): each instance's u, v and a equal the same mesh run
    alone for exactly that many steps, bit for bit, while the others go on;
    limits set again later count from then"""
    meshes, mats, vels = _instances(seed=13, count=5)
    b = _batch(meshes, mats, vels, precision)
    dts = b.getStableTimeSteps()
    b.setTimeSteps(0.8 * dts)
    b.setGraphSteps(graph_steps)
    steps = np.array([7, 33, 0, -1, 24], dtype=np.int64)
    b.setInstanceSteps(steps)
    assert np.array_equal(b.getInstanceStepsLeft(), [7, 33, 0, np.iinfo(np.int64).max, 24])
    b.solveStep(29)
    left = b.getInstanceStepsLeft()
    assert np.array_equal(left[[0, 1, 2, 4]], [0, 4, 0, 0])
    b.solveStep(21)  # 50 steps in all
    # instance 3 has no limit: 50 steps; a new limit for it from now on
    b.setInstanceSteps(np.array([-1, -1, -1, 6, -1], dtype=np.int64))
    b.solveStep(13)
    expected = {0: 7, 1: 33, 2: 0, 3: 56, 4: 24}
    for k, mesh in enumerate(meshes):
        alone = gpu_model(mesh, [mats[k]], precision=precision)
        alone.setNodal("velocity", vels[k])
        alone.setNodal("blocked_dofs", blocked_face(mesh.nodes))
        alone.setTimeStep(0.8 * dts[k])
        alone.solveStep(expected[k])
        sl = b.instance_nodes(k)
        for name in ("displacement", "velocity", "acceleration"):
            got = getattr(b, _getter(name))()[sl]
            assert np.array_equal(got, getattr(alone, _getter(name))()), (k, name)
            assert np.array_equal(b.getInstanceNodal(name, k), got), (k, name)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_single_instance_batch_stops_after_its_steps(precision):
    """a batch of one instance (no node -> instance table) with a step limit,
    as the serving loop builds when one request arrives alone"""
    meshes, mats, vels = _instances(seed=21, count=1)
    b = _batch(meshes, mats, vels, precision)
    dt = b.getStableTimeSteps()
    b.setTimeSteps(0.8 * dt)
    b.setInstanceSteps(np.array([37], dtype=np.int64))
    b.solveStep(150)
    alone = gpu_model(meshes[0], [mats[0]], precision=precision)
    alone.setNodal("velocity", vels[0])
    alone.setNodal("blocked_dofs", blocked_face(meshes[0].nodes))
    alone.setTimeStep(0.8 * dt[0])
    alone.solveStep(37)
    for name in ("displacement", "velocity", "acceleration"):
        assert np.array_equal(getattr(b, _getter(name))(), getattr(alone, _getter(name))()), name

"""Parity with the CPU oracle at the benchmark configurations' full sizes.

The other parity tests run small meshes; these run the meshes the benchmark
measures, for a few steps each, against the oracle on all host threads:

- the 128^3 _hexahedron_8 neohookean box (2,097,152 elements), plain FP64
  and fast FP64 within 1e-12 relative (the law calls log; the fast path
  evaluates in another order) and the mixed path within 1e-5 relative L2
  displacement, 10 steps;
- the 512^2 x 2 _triangle_6 plastic square (524,288 elements), its right edge
  pulled by the velocity ramp prescribed on the device: the configuration's
  own ramp (1e-3 over 5000 steps: elastic over the first steps), and a steep
  ramp that yields within the run, with the 3-point and the 6-point rules;
  FP64 bit-identical, plastic internals included;
- the 256-mesh tetrahedral batch (16.9 M elements): the smallest, a median
  and the largest instance compared with the oracle run alone, FP64
  bit-identical, mixed within 1e-5.
"""
import os

import numpy as np
import pytest

import akantu2_b200 as akb
from oracle import oracle as orc
from scenarios import UNIT_NEOHOOKEAN, UNIT_PLASTIC, blocked_face, oracle_model
from test_gpu_parity import NODAL, compare, gpu_model, rel_err

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1


def _l2(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_hex8_neohookean_128_full_size():
    from akantu2_b200 import gaussian_random_field
    mesh = akb.box_hex8(128)
    assert mesh.getNbElement() == 2_097_152 and mesh.getNbNodes() == 2_146_689
    v0 = gaussian_random_field(mesh.nodes, seed=2024, corr_length=0.1, std=0.02)
    blocked = blocked_face(mesh.nodes)
    o = oracle_model(mesh, [UNIT_NEOHOOKEAN], threads=THREADS)
    o.set(orc.V, v0)
    o.set(orc.BLOCKED, blocked)
    dt = 0.8 * o.stable_dt()
    o.set_dt(dt)
    nsteps = 10
    o.step(nsteps)
    for precision in ("fp64", "fp64_fast", "mixed"):
        g = gpu_model(mesh, [UNIT_NEOHOOKEAN], precision=precision)
        g.setNodal("velocity", v0)
        g.setNodal("blocked_dofs", blocked)
        if precision != "mixed":
            assert g.getStableTimeStep() == dt / 0.8
        g.setTimeStep(dt)
        g.solveStep(nsteps)
        if precision != "mixed":
            compare(g, o, exact=False)
            assert np.array_equal(g.getMass(), o.get(orc.MASS))
        else:
            err = _l2(g.getDisplacement(), o.get(orc.U))
            assert err <= 1e-5, err
        del g


def _tri6_square_pair(qp_rule, nsteps, v_max, ramp_steps):
    """512^2 x 2 plastic square, left edge blocked, right edge's x motion
    prescribed: the GPU by its device ramp, the oracle by the host writing
    the same displacement before every step (the ramp's arithmetic)."""
    mesh = akb.square_tri6(512)
    assert mesh.getNbElement() == 524_288 and mesh.getNbNodes() == 1_050_625
    x = mesh.nodes
    left, right = np.isclose(x[:, 0], 0.0), np.isclose(x[:, 0], 1.0)
    blocked = np.zeros(x.shape, dtype=np.uint8)
    blocked[left] = 1
    g = gpu_model(mesh, [UNIT_PLASTIC], precision="fp64", qp_rule=qp_rule)
    o = oracle_model(mesh, [UNIT_PLASTIC], qp_rule=qp_rule, threads=THREADS)
    v0 = np.zeros_like(x)
    v0[:, 0] = v_max * x[:, 0]
    g.setNodal("velocity", v0)
    g.setNodal("blocked_dofs", blocked)
    o.set(orc.V, v0)
    dt = g.getStableTimeStep()
    assert dt == o.stable_dt()
    g.setTimeStep(0.8 * dt)
    o.set_dt(0.8 * dt)
    dt = 0.8 * dt
    g.setPrescribedVelocityRamp(right, 0, v_max, ramp_steps)
    ob = blocked.copy()
    ob[right, 0] = 1
    o.set(orc.BLOCKED, ob)
    u0 = o.get(orc.U)[right, 0].copy()
    acc = 0.0
    for k in range(1, nsteps + 1):
        acc = acc + dt * (v_max * min(1.0, k / ramp_steps))
        u = o.get(orc.U)
        u[right, 0] = u0 + acc
        o.set(orc.U, u)
        o.step()
    g.solveStep(nsteps)
    return g, o


def _check_plastic_internals(g, o):
    mg = g.getMaterial(0)
    assert np.array_equal(mg.getInternal("inelastic_strain")(), o.qp(0, orc.EPS_P))
    assert np.array_equal(mg.getInternal("iso_hardening")(), o.qp(0, orc.ISO))
    assert np.array_equal(mg.getStress(), o.qp(0, orc.STRESS))
    assert np.array_equal(mg.getGradU(), o.qp(0, orc.GRAD_U))
    assert np.array_equal(mg.getInternal("plastic_energy")(), o.qp(0, orc.PLASTIC_ENERGY))


def test_tri6_plastic_512_configuration_ramp():
    """the configuration's own ramp (end velocity 1e-3 reached after 5000
    steps), first 150 steps: bit-identical, state still elastic"""
    g, o = _tri6_square_pair(qp_rule=0, nsteps=150, v_max=1e-3, ramp_steps=5000)
    compare(g, o, exact=True)
    _check_plastic_internals(g, o)


@pytest.mark.parametrize("qp_rule", [0, 1])
def test_tri6_plastic_512_yielding(qp_rule):
    """a steep ramp (0.05 over 50 steps) on the full-size square: the pulled
    edge yields within the run; 3-point and 6-point rules, bit-identical"""
    g, o = _tri6_square_pair(qp_rule=qp_rule, nsteps=120, v_max=0.05, ramp_steps=50)
    compare(g, o, exact=True)
    eps = o.qp(0, orc.EPS_P)
    assert np.count_nonzero(np.any(eps != 0, axis=1)) > 1000, "the edge must yield"
    _check_plastic_internals(g, o)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_256_tet_cubes_full_size(precision):
    import bench
    meshes, mats, vels, blocks = bench.batch_workload(256)
    assert sum(m.getNbElement() for m in meshes) == 16_883_406
    b = bench.build_batch(akb, meshes, mats, vels, blocks, precision)
    dts = b.getTimeSteps()
    nsteps = 100
    b.solveStep(nsteps)
    sizes = np.array([m.getNbElement() for m in meshes])
    order = np.argsort(sizes, kind="stable")
    picks = [int(order[0]), int(order[len(order) // 2]), int(order[-1])]
    for k in picks:
        mesh = meshes[k]
        o = oracle_model(mesh, [mats[k]], threads=THREADS)
        o.set(orc.V, vels[k])
        o.set(orc.BLOCKED, blocks[k])
        if precision == "fp64":
            assert o.stable_dt() * 0.8 == dts[k]
        o.set_dt(dts[k])
        o.step(nsteps)
        sl = b.instance_nodes(k)
        if precision == "fp64":
            for name, fid in NODAL:
                got = getattr(b, "get" + "".join(w.capitalize() for w in name.split("_")))()[sl]
                assert np.array_equal(got, o.get(fid)), (k, name, rel_err(got, o.get(fid)))
        else:
            err = _l2(b.getDisplacement()[sl], o.get(orc.U))
            assert err <= 1e-5, (k, err)

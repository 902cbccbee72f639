"""The serving loop: admission by device-memory footprint, overlap of resident
solves, and results that do not depend on what else was running."""
import time

import numpy as np
import pytest

import akantu2_b200 as akb
from scenarios import UNIT_ELASTIC, UNIT_NEOHOOKEAN, UNIT_PLASTIC

pytestmark = pytest.mark.gpu

LAWS = [UNIT_ELASTIC, UNIT_NEOHOOKEAN, UNIT_PLASTIC]


def _request(k, rng):
    kind = ("tet", "hex", "tri6")[k % 3]
    n = int(rng.integers(2, 7))
    mesh = {"tet": akb.box_tet4, "hex": akb.box_hex8, "tri6": akb.square_tri6}[kind](n)
    mat = dict(LAWS[int(rng.integers(0, 3))])
    mat.pop("name")
    x = mesh.nodes
    d = x.shape[1]
    v = np.zeros_like(x)
    v[:, d - 1] = 0.01 * np.sin(np.pi * x[:, 0]) * x[:, d - 1]
    if kind == "tri6":
        v[:, 0] = 0.02 * x[:, 0]
    b = np.zeros(x.shape, dtype=np.uint8)
    b[np.isclose(x[:, d - 1 if kind != "tri6" else 0], 0.0)] = 1
    steps = int(rng.integers(50, 450))
    precision = ("fp64", "mixed")[int(rng.integers(0, 2))]
    return dict(mesh=mesh, material=mat, steps=steps, velocity=v, blocked=b, precision=precision)


def _alone(req):
    m = akb.SolidMechanicsModel(req["mesh"])
    mat = req["material"]
    m.addMaterial(mat["type"], **{k: v for k, v in mat.items() if k != "type"})
    m.initFull(akb._explicit_lumped_mass, precision=req["precision"])
    m.setNodal("velocity", req["velocity"])
    m.setNodal("blocked_dofs", req["blocked"])
    m.setTimeStep(0.8 * m.getStableTimeStep())
    m.solveStep(req["steps"])
    return m.getDisplacement(), m.getVelocity()


@pytest.mark.parametrize("batching", [True, False])
def test_results_same_alone_and_in_the_mix(batching):
    """every result equals the same solve run by a model of its own, bit for
    bit, whether it ran as an instance of a batch (requests of one kind
    sharing a batch model, each stopping after its own step count) or alone"""
    rng = np.random.default_rng(3)
    # seven pairs of one kind each (element type, law, precision) arriving
    # together: a solve with no queued partner of its kind runs alone
    reqs = []
    for k in range(14):
        r = _request(k // 2, rng)
        if k % 2:
            r["material"], r["precision"] = reqs[-1]["material"], reqs[-1]["precision"]
        reqs.append(r)
    srv = akb.Server(max_active=5, chunk_steps=100, builders=3, batching=batching)
    ids = {}
    for k, r in enumerate(reqs):
        rid, out = srv.submit(r["mesh"], r["material"], r["steps"], velocity=r["velocity"],
                              blocked=r["blocked"], precision=r["precision"], want_velocity=True)
        ids[rid] = (k, out)
        if k == 6:
            time.sleep(0.05)  # later arrivals join a running set
    done = srv.drain(timeout=300)
    srv.close()
    assert sorted(c["id"] for c in done) == sorted(ids)
    assert any(c["batched"] for c in done) == batching
    for c in done:
        assert c["status"] == 0, c["message"]
        assert c["t_submit"] <= c["t_admit"] <= c["t_start"] <= c["t_end"]
        k, out = ids[c["id"]]
        u, v = _alone(reqs[k])
        assert np.array_equal(out["displacement"], u), f"request {k}"
        assert np.array_equal(out["velocity"], v), f"request {k}"
        assert np.abs(u).max() > 0


def test_admission_respects_the_memory_budget():
    rng = np.random.default_rng(8)
    reqs = [_request(3 * k, rng) for k in range(8)]  # tet meshes
    for r in reqs:
        r["steps"] = 400
    est = [akb.Server.estimate_bytes(r["mesh"], r["material"], r["precision"]) for r in reqs]
    budget = int(2.5 * max(est))
    srv = akb.Server(max_active=16, device_bytes=budget, chunk_steps=100)
    for r in reqs:
        srv.submit(r["mesh"], r["material"], r["steps"], velocity=r["velocity"],
                   blocked=r["blocked"], precision=r["precision"])
    peak = 0
    done = []
    while len(done) < len(reqs):
        st = srv.stats()
        assert st["device_bytes_reserved"] <= budget
        peak = max(peak, st["device_bytes_reserved"])
        done += srv.poll(wait=0.002)
    srv.close()
    assert all(c["status"] == 0 for c in done)
    assert 0 < peak <= budget
    too_big = akb.box_tet4(8)
    srv = akb.Server(device_bytes=1 << 16)
    with pytest.raises(akb.AkbError) as e:
        srv.submit(too_big, dict(type="elastic", E=1.0, nu=0.3, rho=1.0), 10)
    assert e.value.name == "AKB_ENOMEM"
    srv.close()


def test_estimate_bounds_the_allocation():
    for mesh, mat, prec in [(akb.box_tet4(5), UNIT_ELASTIC, "fp64"),
                            (akb.box_hex8(4), UNIT_NEOHOOKEAN, "mixed"),
                            (akb.square_tri6(6), UNIT_PLASTIC, "mixed"),
                            (akb.square_tri6(6), UNIT_PLASTIC, "fp64")]:
        m = akb.SolidMechanicsModel(mesh)
        m.addMaterial(mat["type"], **{k: v for k, v in mat.items() if k != "type"})
        m.initFull(akb._explicit_lumped_mass, precision=prec)
        used = m.getDeviceBytes()
        est = akb.Server.estimate_bytes(mesh, mat, prec)
        assert used <= est <= used + 4096, (mesh.element_type, prec, used, est)


def test_failed_solves_are_reported_and_do_not_disturb_others():
    """a solve whose model cannot be built (an inverted element) completes
    with the library's status and message; the others complete normally"""
    good = akb.box_tet4(3)
    bad = akb.box_tet4(3)
    bad.connectivity[0, [1, 2]] = bad.connectivity[0, [2, 1]]  # negative Jacobian
    mat = dict(type="elastic", E=1.0, nu=0.3, rho=1.0)
    srv = akb.Server(max_active=4)
    v = 0.01 * np.ones_like(good.nodes)
    ids = {}
    for name, mesh in (("good1", good), ("bad", bad), ("good2", good)):
        rid, _ = srv.submit(mesh, mat, 150, velocity=v)
        ids[rid] = name
    done = {ids[c["id"]]: c for c in srv.drain(timeout=120)}
    srv.close()
    assert done["bad"]["status"] == 4 and "Negative jacobian" in done["bad"]["message"]
    assert done["good1"]["status"] == 0 and done["good2"]["status"] == 0
    assert np.array_equal(done["good1"]["outputs"]["displacement"],
                          done["good2"]["outputs"]["displacement"])


def test_submit_rejects_unknown_material():
    srv = akb.Server()
    with pytest.raises(akb.AkbError) as e:
        srv.submit(akb.box_tet4(2), dict(type="no_such_law", E=1.0), 10)
    assert e.value.name == "AKB_EMATERIAL"
    srv.close()


def test_batched_admission_of_many_small_solves():
    """40 small solves of a few kinds arriving together: they share batch
    models (up to the instance limit), each result bit-identical to the solve
    alone, reported as soon as its own steps are done"""
    rng = np.random.default_rng(11)
    reqs = []
    for k in range(40):
        r = _request(3 * (k % 2), rng)  # tetrahedra (k even) and hexahedra
        r["precision"] = ("fp64", "mixed")[(k // 2) % 2]
        reqs.append(r)
    srv = akb.Server(max_active=40, chunk_steps=500, builders=2, batch_max_instances=12)
    ids = {}
    for k, r in enumerate(reqs):
        rid, out = srv.submit(r["mesh"], r["material"], r["steps"], velocity=r["velocity"],
                              blocked=r["blocked"], precision=r["precision"], want_velocity=True)
        ids[rid] = (k, out)
    done = srv.drain(timeout=300)
    srv.close()
    assert sum(c["batched"] for c in done) >= 30
    for c in done:
        assert c["status"] == 0, c["message"]
        k, out = ids[c["id"]]
        u, v = _alone(reqs[k])
        assert np.array_equal(out["displacement"], u), f"request {k}"
        assert np.array_equal(out["velocity"], v), f"request {k}"


def test_batch_estimate_bounds_the_allocation():
    import ctypes
    from akantu2_b200 import _capi
    for meshes, mat, prec in [([akb.box_tet4(n) for n in (2, 3, 4)], UNIT_ELASTIC, "fp64"),
                              ([akb.box_hex8(n) for n in (2, 4)], UNIT_NEOHOOKEAN, "mixed"),
                              ([akb.square_tri6(n) for n in (3, 5)], UNIT_PLASTIC, "mixed")]:
        b = akb.BatchModel(meshes)
        for k in range(len(meshes)):
            b.addMaterial(mat["type"], **{kk: v for kk, v in mat.items() if kk != "type"})
        b.setInstanceMaterials(np.arange(len(meshes)))
        b.initFull(akb._explicit_lumped_mass, precision=prec)
        b.setInstanceSteps(np.full(len(meshes), 10, dtype=np.int64))
        used = b.getDeviceBytes()
        est = ctypes.c_int64()
        law = {"elastic": 0, "neohookean": 1, "plastic_linear_isotropic_hardening": 2}[mat["type"]]
        _capi.check(_capi.lib().akb_estimate_batch_device_bytes(
            _capi.TETRAHEDRON_4 if meshes[0].element_type == "_tetrahedron_4" else
            (_capi.HEXAHEDRON_8 if meshes[0].element_type == "_hexahedron_8" else
             _capi.TRIANGLE_6), 0, b.mesh.getNbNodes(), b.mesh.getNbElement(), len(meshes),
            law, 0 if prec == "fp64" else 1, ctypes.byref(est)))
        assert used <= est.value <= used + 8192, (meshes[0].element_type, prec, used, est.value)

"""A partitioned mesh on the GPU: subdomain models with the per-step halo
exchange (all on one GPU, and as gloo ranks that each drive a model on the
GPU) give exactly the state of one model of the whole mesh."""
import multiprocessing as mp
import os
import socket
import sys

import numpy as np
import pytest

import akantu2_b200 as akb

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PLASTIC = dict(type="plastic_linear_isotropic_hardening", rho=1.0, E=1.0, nu=0.3, sigma_y=2e-3,
               h=0.1)
CASES = {
    "tet_elastic": (lambda: akb.box_tet4(8, 6, 5), [dict(type="elastic", rho=1.0, E=1.0, nu=0.3)]),
    "hex_neohookean": (lambda: akb.box_hex8(10, 8, 6),
                       [dict(type="neohookean", rho=1.0, E=1.0, nu=0.3)]),
    "tri6_plastic": (lambda: akb.square_tri6(12, 9), [PLASTIC]),
    "tet_two_materials": (lambda: akb.box_tet4(7, 5, 6),
                          [dict(type="elastic", name="soft", rho=1.0, E=0.5, nu=0.3),
                           dict(type="neohookean", name="stiff", rho=2.0, E=2.0, nu=0.25)]),
}


def _state(mesh):
    x = mesh.nodes
    d = mesh.spatial_dimension
    v0 = np.zeros_like(x)
    if d == 3:
        v0[:, 2] = 0.02 * np.sin(np.pi * x[:, 0]) * np.sin(2 * np.pi * x[:, 1]) * x[:, 2]
        v0[:, 0] = 0.01 * np.cos(np.pi * x[:, 2])
    else:
        v0[:, 0] = 0.02 * x[:, 0]
        v0[:, 1] = 0.01 * np.sin(np.pi * x[:, 0])
    bl = np.zeros(x.shape, np.uint8)
    bl[np.isclose(x[:, d - 1], 0.0)] = 1
    return v0, bl


def _materials_of(mesh, mats):
    if len(mats) == 1:
        return None
    return (mesh.nodes[mesh.connectivity].mean(axis=1)[:, 0] > 0.5).astype(np.int32)


def _setup(model, mesh, mats, precision, ramp):
    for mat in mats:
        model.addMaterial(mat["type"], **{k: v for k, v in mat.items() if k != "type"})
    which = _materials_of(mesh, mats)
    if which is not None:
        model.setElementMaterials(which)
    model.initFull(akb._explicit_lumped_mass, precision=precision)
    v0, bl = _state(mesh)
    model.setNodal("velocity", v0)
    model.setNodal("blocked_dofs", bl)
    model.setTimeStep(0.8 * model.getStableTimeStep())
    if ramp:
        d = mesh.spatial_dimension
        top = np.flatnonzero(np.isclose(mesh.nodes[:, d - 1], mesh.nodes[:, d - 1].max()))
        model.setPrescribedVelocityRamp(top, 0, 0.05, 30)


def _serial(case, precision, ramp, steps):
    make, mats = CASES[case]
    mesh = make()
    m = akb.SolidMechanicsModel(mesh)
    _setup(m, mesh, mats, precision, ramp)
    m.solveStep(steps)
    return mesh, m


@pytest.mark.parametrize("case,precision,nparts", [
    ("tet_elastic", "fp64", 2), ("tet_elastic", "mixed", 3), ("hex_neohookean", "mixed", 4),
    ("hex_neohookean", "fp64", 2), ("tri6_plastic", "fp64", 3), ("tri6_plastic", "mixed", 2),
    ("tet_two_materials", "fp64", 4)])
def test_partitioned_model_is_bit_identical(case, precision, nparts):
    ramp = case == "tri6_plastic"
    steps = 60
    mesh, ref = _serial(case, precision, ramp, steps)
    make, mats = CASES[case]
    pm = akb.PartitionedModel(mesh, nparts)
    _setup(pm, mesh, mats, precision, ramp)
    assert pm.getTimeStep() == ref.getTimeStep()
    pm.solveStep(25)
    # a host write between steps: the prediction is made again everywhere
    v = pm.getVelocity()
    pm.setNodal("velocity", v)
    pm.solveStep(steps - 25)
    u = ref.getDisplacement()
    assert np.max(np.abs(u)) > 0
    assert np.array_equal(pm.getDisplacement(), u)
    assert np.array_equal(pm.getVelocity(), ref.getVelocity())
    assert np.array_equal(pm.getAcceleration(), ref.getAcceleration())
    assert np.array_equal(pm.getInternalForce(), ref.getInternalForce())
    assert np.array_equal(pm.getMass(), ref.getMass())


@pytest.mark.parametrize("case,precision,nparts", [
    ("hex_neohookean", "mixed", 4), ("tri6_plastic", "fp64", 3), ("tet_elastic", "fp64", 2)])
def test_partitioned_exchange_graphs_are_bit_identical(case, precision, nparts):
    """the exchange's captured graphs (100 steps of every subdomain with their
    halo packs and unpacks as graph edges) against the whole mesh, with a
    host write between two graph runs and steps that are not whole graphs"""
    ramp = case == "tri6_plastic"
    mesh, ref = _serial(case, precision, ramp, 0)
    make, mats = CASES[case]
    pm = akb.PartitionedModel(mesh, nparts)
    _setup(pm, mesh, mats, precision, ramp)
    for n in (203, 17, 100):
        if n == 17:
            v = pm.getVelocity()
            pm.setNodal("velocity", v)
            ref.setNodal("velocity", ref.getVelocity())
        pm.solveStep(n)
        ref.solveStep(n)
    assert np.array_equal(pm.getDisplacement(), ref.getDisplacement())
    assert np.array_equal(pm.getVelocity(), ref.getVelocity())
    assert np.array_equal(pm.getInternalForce(), ref.getInternalForce())


def test_partitioned_step_cost_on_one_gpu():
    """64^3 hexahedra (neohookean, mixed) in 4 subdomains on the one GPU: the
    step of the four models with their exchange, replayed as graphs, within
    1.4x of one model of the whole mesh"""
    mesh = akb.box_hex8(64)
    mat = dict(type="neohookean", rho=1.0, E=1.0, nu=0.3)
    v0, bl = _state(mesh)
    whole = akb.SolidMechanicsModel(mesh)
    _setup(whole, mesh, [mat], "mixed", False)
    whole.solveStep(200)
    t_whole = min(whole.timeSteps(200) for _ in range(3)) / 200
    pm = akb.PartitionedModel(mesh, 4)
    _setup(pm, mesh, [mat], "mixed", False)
    pm.solveStep(200)
    t_part = min(pm.timeSteps(200) for _ in range(3)) / 200
    print(f"whole {t_whole * 1e3:.1f} us, 4 parts {t_part * 1e3:.1f} us per step")
    assert t_part <= 1.4 * t_whole, (t_part, t_whole)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, case, precision, steps, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import akantu2_b200 as akb_
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        make, mats = CASES[case]
        mesh = make()
        dm = akb_.DistributedModel(mesh, device=0)
        _setup(dm, mesh, mats, precision, False)
        dm.solveStep(steps)
        u, v = dm.getDisplacement(), dm.getVelocity()
        if rank == 0:
            out.put((dm.getTimeStep(), u, v))
    finally:
        dist.destroy_process_group()


def test_distributed_model_over_gloo_ranks():
    """two processes, each driving its subdomain's model on the GPU, the halo
    staged through host memory over gloo"""
    steps = 50
    mesh, ref = _serial("hex_neohookean", "mixed", False, steps)
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, "hex_neohookean", "mixed", steps, out))
             for r in range(2)]
    for p in procs:
        p.start()
    dt, u, v = out.get(timeout=600)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert dt == ref.getTimeStep()
    assert np.array_equal(u, ref.getDisplacement())
    assert np.array_equal(v, ref.getVelocity())

"""Benchmark of the explicit solid-dynamics step (element-steps/s).

Workload (default): the single-large-mesh configuration -- a 128 x 128 x 128
structured _hexahedron_8 box (2,097,152 elements, 2,146,689 nodes, 8 Gauss
points), neohookean (rho = 1, E = 1, nu = 0.3), z = 0 face blocked, seeded
Gaussian random initial velocity (correlation length 0.1, std 0.02),
dt = 0.8 x stable.  One step = one central-difference step of the whole mesh.

  value      device time (CUDA events on the model's stream) of K steps of the
             mixed-precision path (FP32 element math, FP64 state); inputs are
             resident in HBM and far larger than L2 (no flush needed).  A
             model that fits in L2 (the 48k-tet cube of --config tet) is
             timed step by step instead, each step after an L2 flush; its
             L2-resident rate is reported beside it
  fp64       the same for the plain FP64 path
  e2e        through the C ABI with host buffers: every step uploads the
             external force from pinned memory, runs the step and reads the
             displacement back (wall clock, synchronised); pcie_bound: the
             same two copies alone, issued together, as the floor of that step
  roofline   element-force kernel: algorithmic bytes / its event-timed duration
  cpu_baseline  the CPU oracle (restatement of the reference path) on the host
             cores, bounded sample of the same workload

--config batch: 256 independent linear-elastic tet cubes, n cells per edge
with n uniform in 8..32 (seeded), E log-uniform in [0.5, 2], nu uniform in
[0.2, 0.4], rho = 1, z = 0 blocked, sinusoidal initial velocity modes with
wavenumbers 1..4, each instance at 0.8 x its own stable dt, all advanced
together (one element launch and one node launch per step, 100-step CUDA
graphs).  Beside the batched mixed and FP64 rates it times the instances one
model at a time (FP64, a sample of 16 instances) as the unbatched baseline.

--config serve: a stream of solve requests with Poisson arrivals (rate
--rate per second, seeded).  Each request is a tet4 or hex8 box with an
element count log-uniform in [1e3, 1e6], a material drawn uniformly among
elastic, neohookean and plastic_linear_isotropic_hardening (rho = 1, E = 1,
nu = 0.3; sigma_y = 1e-3, h = 0.1), z = 0 blocked, a sinusoidal initial
velocity and a step count uniform in 500..5000 at 0.8 x its stable dt.  The
server admits requests by device-memory footprint and advances the resident
ones together; value = element-steps/s of the whole stream, with p50 / p99
of the arrival-to-result latency.

--impl reference times the reference's CPU algorithm (the oracle: the
reference cannot be built here) on all host threads and prints its line.
N > 1 (torchrun): independent replicas, one mesh per GPU, weak scaling.
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "element-steps/s"
UNIT = "element-steps/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--config", default="hex8",
                   choices=["hex8", "tet", "tri6", "batch", "serve"])
    p.add_argument("--instances", type=int, default=256, help="batch: number of meshes")
    p.add_argument("--requests", type=int, default=200, help="serve: number of requests")
    p.add_argument("--rate", type=float, default=20.0, help="serve: arrivals per second")
    p.add_argument("--max-active", type=int, default=64, help="serve: resident solves")
    p.add_argument("--builders", type=int, default=8, help="serve: host build threads")
    p.add_argument("--no-batching", action="store_true",
                   help="serve: every request gets a model of its own")
    p.add_argument("--cells", type=int, default=0, help="override the mesh resolution")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    p.add_argument("--e2e-lag", type=int, default=3,
                   help="end-to-end leg: steps between a step's read and the wait for it "
                        "(1 .. AKB_ASYNC_READS_IN_FLIGHT - 1)")
    p.add_argument("--no-e2e-fp64", action="store_true",
                   help="skip the end-to-end leg of the FP64 path")
    p.add_argument("--no-extras", action="store_true",
                   help="default configuration: skip the compact tri6 and batch records")
    p.add_argument("--precisions", default="mixed,fp64,fp64_fast")
    p.add_argument("--accuracy-steps", type=int, default=10000,
                   help="steps of the mixed-vs-FP64 accuracy leg (0: skip)")
    p.add_argument("--no-autotune", action="store_true",
                   help="keep the default launch shapes (profiling captures)")
    p.add_argument("--mode", default="replicas", choices=["replicas", "partitioned"],
                   help="N > 1: independent replicas (weak scaling), or one mesh split over "
                        "the ranks with a halo exchange every step (strong scaling)")
    p.add_argument("--qp-rule", type=int, default=0,
                   help="tri6: quadrature rule (0: the reference's default, 3 points; 1: 6 points)")
    p.add_argument("--parts", type=int, default=0,
                   help="partitioned, one process: subdomains advanced on the one GPU")
    args = p.parse_args()
    # the library keeps AKB_ASYNC_READS_IN_FLIGHT reads waitable one by one
    if not 1 <= args.e2e_lag <= 3:
        p.error("--e2e-lag must be in 1 .. 3 (AKB_ASYNC_READS_IN_FLIGHT - 1)")
    return args


# ---- workloads ---------------------------------------------------------------------
def workload(config, cells):
    import akantu2_b200 as akb
    if config == "hex8":
        n = cells or 128
        mesh = akb.box_hex8(n)
        mat = dict(type="neohookean", rho=1.0, E=1.0, nu=0.3)
        desc = f"hex8 neohookean {n}^3 box"
    elif config == "tet":
        n = cells or 20
        mesh = akb.box_tet4(n)
        mat = dict(type="elastic", rho=1.0, E=1.0, nu=0.3)
        desc = f"tet4 elastic {n}^3 x 6 cube"
    else:
        n = cells or 512
        mesh = akb.square_tri6(n)
        mat = dict(type="plastic_linear_isotropic_hardening", rho=1.0, E=1.0, nu=0.3,
                   sigma_y=1e-3, h=0.1)
        desc = (f"tri6 plastic {n}^2 x 2 square, plane strain, right edge pulled by a "
                "velocity ramp to 1e-3 over 5000 steps (prescribed on the device)")
    return mesh, mat, desc


def initial_state(config, mesh):
    from akantu2_b200 import gaussian_random_field
    x = mesh.nodes
    blocked = np.zeros(x.shape, dtype=np.uint8)
    if config == "tri6":
        # left edge blocked; the right edge's x motion is prescribed (run_ours)
        blocked[np.isclose(x[:, 0], 0.0)] = 1
        blocked[np.isclose(x[:, 0], 1.0), 0] = 1
        v0 = np.zeros_like(x)
        v0[:, 0] = 1e-3 * x[:, 0]  # the ramp's end velocity, linear in x
    else:
        blocked[np.isclose(x[:, 2], 0.0)] = 1
        if config == "hex8":
            v0 = gaussian_random_field(x, seed=2024, corr_length=0.1, std=0.02)
        else:
            v0 = np.zeros_like(x)
            v0[:, 2] = 0.01 * np.sin(np.pi * x[:, 0]) * np.sin(np.pi * x[:, 1]) * x[:, 2]
    return v0, blocked


def batch_workload(count, seed=7, n_range=(8, 32)):
    """The batched-instance configuration: meshes, materials, initial states."""
    import akantu2_b200 as akb
    rng = np.random.default_rng(seed)
    meshes, mats, vels, blocks = [], [], [], []
    for k in range(count):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        mesh = akb.box_tet4(n)
        E = float(np.exp(rng.uniform(np.log(0.5), np.log(2.0))))
        nu = float(rng.uniform(0.2, 0.4))
        mats.append(dict(type="elastic", name=f"instance{k}", rho=1.0, E=E, nu=nu))
        x = mesh.nodes
        v = np.zeros_like(x)
        for _ in range(2):  # two modes per component, wavenumbers 1..4
            kx, ky, kz = rng.integers(1, 5, size=3)
            amp = 0.01 * rng.uniform(-1.0, 1.0, size=3)
            mode = (np.sin(kx * np.pi * x[:, 0]) * np.sin(ky * np.pi * x[:, 1]) *
                    np.sin(0.5 * kz * np.pi * x[:, 2]))
            v += amp[None, :] * mode[:, None]
        b = np.zeros(x.shape, dtype=np.uint8)
        b[np.isclose(x[:, 2], 0.0)] = 1
        meshes.append(mesh)
        vels.append(v)
        blocks.append(b)
    return meshes, mats, vels, blocks


SERVE_MATERIALS = [
    dict(type="elastic", rho=1.0, E=1.0, nu=0.3),
    dict(type="neohookean", rho=1.0, E=1.0, nu=0.3),
    dict(type="plastic_linear_isotropic_hardening", rho=1.0, E=1.0, nu=0.3, sigma_y=1e-3,
         h=0.1),
]


def serve_requests(count, rate, seed=11):
    """Seeded request stream: (arrival time, kind, cells, material, steps)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for _ in range(count):
        t += rng.exponential(1.0 / rate)
        kind = ("tet", "hex")[int(rng.integers(0, 2))]
        target = float(np.exp(rng.uniform(np.log(1e3), np.log(1e6))))
        per_cell = 6 if kind == "tet" else 1
        n = max(2, int(round((target / per_cell) ** (1.0 / 3.0))))
        nz = max(1, int(round(target / (per_cell * n * n))))
        mat = SERVE_MATERIALS[int(rng.integers(0, 3))]
        steps = int(rng.integers(500, 5001))
        out.append((t, kind, (n, n, nz), mat, steps))
    return out


_MESH_CACHE = {}


def serve_mesh(kind, cells):
    import akantu2_b200 as akb
    key = (kind, cells)
    if key not in _MESH_CACHE:
        nx, ny, nz = cells
        mesh = (akb.box_tet4 if kind == "tet" else akb.box_hex8)(nx, ny, nz)
        x = mesh.nodes
        v = np.zeros_like(x)
        v[:, 2] = 0.01 * np.sin(np.pi * x[:, 0]) * np.sin(np.pi * x[:, 1]) * x[:, 2]
        b = np.zeros(x.shape, dtype=np.uint8)
        b[np.isclose(x[:, 2], 0.0)] = 1
        _MESH_CACHE[key] = (mesh, v, b)
    return _MESH_CACHE[key]


# algorithmic bytes per element-step (fixed formula over the arrays the step
# must read and write), and the element-force kernel's own share
def quadrature_points(config, qp_rule=0):
    return {"hex8": 8, "tet": 1, "tri6": 6 if qp_rule else 3, "batch": 1}[config]


def algorithmic_bytes(config, mesh, precision, qp_rule=0):
    E, N = mesh.getNbElement(), mesh.getNbNodes()
    n = mesh.connectivity.shape[1]
    d = mesh.spatial_dimension
    Q = quadrature_points(config, qp_rule)
    s_e = 8 if precision.startswith("fp64") else 4
    S = (3 * d * d + 1) * 8 if config == "tri6" else 0
    elem = E * (4 * n + Q * (d * n + 1) * s_e + 2 * Q * S)
    nodal = N * (64 * d + 9)
    step = elem + nodal
    kernel = elem + N * 8 * d  # the element kernel also gathers u
    return step, kernel


def read_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def read_traffic(config, precision):
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            t = json.load(f)
        return t.get(f"{config}_{precision}")
    except Exception:
        return None


def roofline_entry(kern_bytes, elem_ms, peak, peak_kind, traffic):
    """the element-force kernel against the measured HBM peak: the formula's
    algorithmic bytes per launch, and (when an ncu capture gave the kernel's
    DRAM bytes per launch) the measured DRAM traffic per launch time"""
    secs = elem_ms / 1e3
    r = {"bound": "hbm", "kernel": "k_element_forces",
         "achieved": kern_bytes / secs / 1e9, "peak": peak, "unit": "GB/s",
         "frac": kern_bytes / secs / 1e9 / peak, "traffic": traffic,
         "peak_source": f"{peak_kind} hbm_gbs"}
    if traffic:
        r["dram_achieved"] = traffic / secs / 1e9
        r["dram_frac"] = traffic / secs / 1e9 / peak
    return r


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, device):
        self.device = device
        self.proc = None
        # the raw samples (the line carries their summary); AKB_CLOCKS_DIR
        # keeps them somewhere else than the system's temporary directory
        import tempfile
        self.path = os.path.join(os.environ.get("AKB_CLOCKS_DIR", tempfile.gettempdir()),
                                 f"akb_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device),
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.f, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None:
            return None
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx.append(float(parts[2]))
                except ValueError:
                    continue
                for name, val in zip(names, parts[5:9]):
                    if val.lower() == "active":
                        reasons.add(name)
        except Exception:
            return None
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(mx), "samples": len(sm),
                "reasons": sorted(reasons)}


class Replicas:
    """One process per GPU (torchrun): rank and world size from the
    environment, a process group when world > 1, the barrier and the maximum
    over ranks of a device-timed value.  The replicas share no data: the only
    collectives are this barrier and this maximum."""

    def __init__(self, backend="nccl"):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import datetime
            import torch
            import torch.distributed as dist
            if backend == "nccl":
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
            self.dist = dist

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()
            if self.backend == "nccl":
                import torch
                torch.cuda.synchronize()

    def max(self, x):
        if self.dist is None:
            return x
        import torch
        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None


def aggregate_rate(units_per_rank, world, ms_max):
    """whole-job units/s: every rank processed units_per_rank in at most ms_max"""
    return world * units_per_rank / (ms_max / 1e3)


# ---- CPU legs --------------------------------------------------------------------------
def cpu_rate(config, mesh, mat, v0, blocked, budget_s, max_steps, threads):
    """Element-steps/s of the oracle on `threads` host threads."""
    from oracle import oracle as orc
    otype = {"hex8": orc.HEX8, "tet": orc.TET4, "tri6": orc.TRI6}[config]
    o = orc.OracleModel(otype, mesh.nodes, mesh.connectivity, [mat], threads=threads)
    o.set(orc.V, v0)
    o.set(orc.BLOCKED, blocked)
    o.set_dt(0.8 * o.stable_dt())
    o.step(1)  # warm
    t0 = time.perf_counter()
    steps = 0
    while steps < max_steps:
        o.step(1)
        steps += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return mesh.getNbElement() * steps / dt, steps, dt


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    if args.config == "batch":
        meshes, mats, vels, blocks = batch_workload(args.instances)
        cpu = cpu_batch_rate(meshes, mats, vels, blocks, threads, budget_s=60.0)
        E = sum(m.getNbElement() for m in meshes)
        line = {
            "impl": "reference", "metric": METRIC, "value": cpu["value"], "unit": UNIT,
            "n_gpus": args.gpus, "steps": 20, "warmup": 1, "ms_per_step": 1e3 * E / cpu["value"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": f"{len(meshes)} tet4 elastic cubes, n in 8..32",
                       "elements": E, "parallelism": f"{threads} host threads"},
            "cpu_baseline": cpu,
            "e2e": {"value": cpu["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return
    if args.config == "serve":
        cpu = cpu_serve_rate(serve_requests(args.requests, args.rate), threads, budget_s=60.0)
        line = {
            "impl": "reference", "metric": METRIC, "value": cpu["value"], "unit": UNIT,
            "n_gpus": args.gpus, "steps": 20, "warmup": 1, "ms_per_step": None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": "serving request stream (sample)",
                                            "parallelism": f"{threads} host threads"},
            "cpu_baseline": cpu,
            "e2e": {"value": cpu["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return
    mesh, mat, desc = workload(args.config, args.cells)
    v0, blocked = initial_state(args.config, mesh)
    # each timed step is one full step of the workload; the count is bounded
    # so that the whole run stays within a few minutes
    rate, steps, secs = cpu_rate(args.config, mesh, mat, v0, blocked, budget_s=60.0,
                                 max_steps=max(1, args.steps), threads=threads)
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT,
        "n_gpus": args.gpus, "steps": steps, "warmup": 1,
        "ms_per_step": 1e3 * secs / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": desc, "elements": mesh.getNbElement(),
                   "nodes": mesh.getNbNodes(), "parallelism": f"{threads} host threads"},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{steps} full steps of the {desc} (oracle restatement; "
                                   "the reference cannot be built without Eigen/Boost)"},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---- GPU leg ----------------------------------------------------------------------------
def run_ours(args, rep=None, emit=True, extra=False):
    own = rep is None
    rep = rep or Replicas("nccl")
    world, rank, local = rep.world, rep.rank, rep.local
    barrier, max_over_ranks = rep.barrier, rep.max
    import akantu2_b200 as akb
    from akantu2_b200 import _capi
    _capi.check(_capi.lib().akb_set_device(local))

    mesh, mat, desc = workload(args.config, args.cells)
    if args.config == "tri6":
        desc += f", {quadrature_points('tri6', args.qp_rule)} Gauss points per triangle"
    v0, blocked = initial_state(args.config, mesh)
    E = mesh.getNbElement()
    results = {}
    precisions = [p for p in args.precisions.split(",") if p]

    for prec in precisions:
        m = akb.SolidMechanicsModel(mesh)
        m.addMaterial(mat["type"], **{k: v for k, v in mat.items() if k != "type"})
        if args.config == "tri6" and args.qp_rule:
            m.setQuadratureRule(args.qp_rule)
        m.initFull(akb._explicit_lumped_mass, precision=prec)
        m.setNodal("velocity", v0)
        m.setNodal("blocked_dofs", blocked)
        m.setTimeStep(0.8 * m.getStableTimeStep())
        if args.config == "tri6":
            m.setPrescribedVelocityRamp(np.isclose(mesh.nodes[:, 0], 1.0), 0, 1e-3, 5000)
        m.timeSteps(max(3, args.warmup))
        # launch shapes timed on this state (none of them changes results)
        if not args.no_autotune:
            m.autotune(5)
        m.prepareGraphs()  # the step graph is captured before the clock starts
        footprint = m.getDeviceBytes()
        fits_l2 = footprint < L2_BYTES
        barrier()
        with ClockSampler(local) as clk:
            ms_resident = m.timeSteps(args.steps)
            # a model that fits in L2: every timed step starts from a flushed
            # L2 (the flush is outside the per-step events)
            ms = flushed_steps(m, args.steps, local) if fits_l2 else ms_resident
        barrier()
        ms = max_over_ranks(ms)
        nprof = min(args.steps, 20)
        tot, phases = m.profileSteps(nprof)
        step_b, kern_b = algorithmic_bytes(args.config, mesh, prec, args.qp_rule)
        elem_ms = phases[1] / nprof
        peak, peak_kind = read_peaks()
        results[prec] = {
            "ms_per_step": ms / args.steps,
            "value": aggregate_rate(E * args.steps, world, ms),
            "phase_ms_per_step": {"predictor": phases[0] / nprof,
                                  "element_forces": phases[1] / nprof,
                                  "node_update": phases[2] / nprof},
            "roofline": roofline_entry(kern_b, elem_ms, peak, peak_kind,
                                       None if args.qp_rule else
                                       read_traffic(args.config, prec)),
            "roofline_step": {"bytes_per_element_step": step_b / E,
                              "achieved": step_b / (ms / args.steps / 1e3) / 1e9,
                              "frac": step_b / (ms / args.steps / 1e3) / 1e9 / peak},
            "clocks": clk.summary(),
            "tuning": {"element": list(m.getLaunchShape(mat["type"])),
                       "node": list(m.getNodeShape()),
                       "dependent_launch": m.getDependentLaunch()},
            "l2": (f"model fits in L2 ({footprint / 1e6:.1f} MB on the device): L2 flushed "
                   f"(512 MB write) before every timed step, each step timed alone; "
                   f"{ms_resident / args.steps:.5f} ms per step with the model L2-resident "
                   "(100-step graphs)") if fits_l2 else
                  f"inputs larger than L2 ({footprint / 1e6:.0f} MB on the device; no flush)",
            # per step: the element-force kernel, the node update (with the next
            # predictor) and, for the ramp, the prescribed-motion kernel
            "gpu_launches": args.steps * (3 if args.config == "tri6" else 2),
            # the state after the timed steps must be finite (device status word)
            "state_finite": m.getStatus() == 0 and bool(np.all(np.isfinite(m.getDisplacement()))),
        }
        if (prec == precisions[0] and not extra) or (prec == "fp64" and not args.no_e2e_fp64):
            # end to end through the C ABI with pinned host buffers
            nb = int(np.prod(mesh.nodes.shape)) * 8
            k_e2e = max(1, min(args.steps, 100 if prec == precisions[0] else 20))
            secs_sync, secs_async = e2e_legs(m, mesh.nodes.shape, k_e2e, barrier,
                                             args.e2e_lag)
            secs_sync, secs_async = max_over_ranks(secs_sync), max_over_ranks(secs_async)
            results[prec]["e2e"] = {"value": world * E * k_e2e / secs_async, "unit": UNIT,
                                    "steps": k_e2e, "h2d_bytes_per_step": nb,
                                    "d2h_bytes_per_step": nb,
                                    "mode": "pipelined: the external force of every step uploaded "
                                            "and its displacement read back through the async "
                                            f"C ABI, each result waited for {args.e2e_lag} "
                                            "step(s) later, all copies complete inside the "
                                            "timed region",
                                    "synchronous_value": world * E * k_e2e / secs_sync,
                                    "pcie_bound": e2e_bound(nb, nb, secs_async, k_e2e)}
        del m
    head = results[precisions[0]]
    accuracy = None
    if rank == 0 and not extra and args.accuracy_steps > 0 and \
            set(precisions) >= {"mixed", "fp64"}:
        accuracy = accuracy_leg(akb, args.config, mesh, mat, v0, blocked, args.accuracy_steps)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu and not extra:
        threads = os.cpu_count() or 1
        rate, steps, secs = cpu_rate(args.config, mesh, mat, v0, blocked, budget_s=20.0,
                                     max_steps=50, threads=threads)
        # one thread, as the reference runs per MPI rank (a short sample)
        rate1, steps1, secs1 = cpu_rate(args.config, mesh, mat, v0, blocked, budget_s=5.0,
                                        max_steps=50, threads=1)
        cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{steps} steps of the full {desc} in {secs:.1f} s "
                         f"(CPU oracle, {threads} threads)",
               "one_thread": {"value": rate1, "unit": UNIT, "cores": 1,
                              "sample": f"{steps1} steps in {secs1:.1f} s"}}
    if rank == 0:
        line = {
            "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": max(3, args.warmup),
            "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 element math / f64 state" if precisions[0] == "mixed" else "f64",
            "data": "synthetic (seeded random-field initial velocity)",
            "precisions": {"mixed": "FP32 element math, FP64 state, Kahan gather",
                           "fp64": "plain FP64, the CPU path's operation order (bit-identical "
                                   "up to log ulps)",
                           "fp64_fast": "FP64, hexahedra by the sum-factorised kernel with "
                                        "contraction (within 1e-12 of the CPU path)"},
            "config": {"workload": desc, "elements": E, "nodes": mesh.getNbNodes(),
                       "quadrature_points": quadrature_points(args.config, args.qp_rule),
                       "precision": precisions[0], "parallelism": f"replicas x{world}",
                       "l2": head["l2"]},
            "e2e": head.get("e2e"), "roofline": head["roofline"],
            "roofline_step": head["roofline_step"], "clocks": head["clocks"],
            "gpu_launches": head["gpu_launches"], "state_finite": head["state_finite"],
            "phase_ms_per_step": head["phase_ms_per_step"],
            "tuning": head["tuning"],
            "cpu_baseline": cpu,
            "accuracy": accuracy,
        }
        for prec in precisions[1:]:
            r = results[prec]
            line[prec] = {"value": r["value"], "ms_per_step": r["ms_per_step"],
                          "roofline": r["roofline"], "roofline_step": r["roofline_step"],
                          "phase_ms_per_step": r["phase_ms_per_step"]}
            if "e2e" in r:
                line[prec]["e2e"] = r["e2e"]
        if "fp64" in results and precisions[0] != "fp64":
            line["speedup_vs_fp64"] = head["value"] / results["fp64"]["value"]
        if emit:
            print(json.dumps(line), flush=True)
    if own:
        rep.close()
    return line if rank == 0 else None


L2_BYTES = 126 * 10**6  # B200 L2


def flushed_steps(m, k, device):
    """k steps, each timed alone on the model's stream right after a 512 MB
    write has evicted the model from L2; returns the summed device time (ms)."""
    import torch
    buf = torch.empty(512 * 2**20 // 4, dtype=torch.float32, device=f"cuda:{device}")
    total = 0.0
    for _ in range(k):
        buf.fill_(1.0)
        torch.cuda.synchronize(device)
        total += m.timeSteps(1)
    del buf
    return total


def e2e_legs(m, shape, k, barrier, lag=None):
    """End to end through the C ABI with pinned host buffers, k steps: every
    step uploads the external force and reads the displacement back.
    Synchronous: set_nodal / solve_step / get_nodal.  Pipelined: the async
    forms, the result of step j waited for after step j + lag is enqueued
    (lag + 1 host buffers per direction; by default lag =
    AKB_ASYNC_READS_IN_FLIGHT - 1, so that the copies of consecutive steps
    run back to back).  Returns both wall times (seconds)."""
    from akantu2_b200 import _capi
    from akantu2_b200._capi import PinnedArray
    L = _capi.lib()
    if lag is None:
        lag = _capi.ASYNC_READS_IN_FLIGHT - 1
    fext = [PinnedArray(shape) for _ in range(lag + 1)]
    uout = [PinnedArray(shape) for _ in range(lag + 1)]
    for f in fext:
        f.array[:] = 0.0
    nb = fext[0].array.nbytes
    import ctypes
    ticket = ctypes.c_int64()

    def sync_steps(n):
        for _ in range(n):
            _capi.check(L.akb_model_set_nodal(m._h, _capi.EXTERNAL_FORCE,
                                              _capi.ptr(fext[0].array), nb))
            _capi.check(L.akb_model_solve_step(m._h, 1))
            _capi.check(L.akb_model_get_nodal(m._h, _capi.DISPLACEMENT,
                                              _capi.ptr(uout[0].array), nb))

    def async_steps(n):
        issued = []
        for j in range(n):
            b = j % (lag + 1)
            _capi.check(L.akb_model_set_nodal_async(m._h, _capi.EXTERNAL_FORCE,
                                                    _capi.ptr(fext[b].array), nb))
            _capi.check(L.akb_model_solve_step(m._h, 1))
            _capi.check(L.akb_model_get_nodal_async(m._h, _capi.DISPLACEMENT,
                                                    _capi.ptr(uout[b].array), nb,
                                                    ctypes.byref(ticket)))
            issued.append(ticket.value)
            if len(issued) > lag:
                _capi.check(L.akb_model_wait_nodal_async(m._h, issued.pop(0)))
        _capi.check(L.akb_model_synchronize(m._h))

    # untimed warm-up of both legs: the first asynchronous call creates the
    # copy streams and the staging buffers, and the first touches of the
    # pinned buffers fault their pages in
    sync_steps(3)
    async_steps(3)
    barrier()
    t0 = time.perf_counter()
    sync_steps(k)
    secs_sync = time.perf_counter() - t0
    barrier()
    t0 = time.perf_counter()
    async_steps(k)
    secs_async = time.perf_counter() - t0
    return secs_sync, secs_async


def pcie_bound(h2d_bytes, d2h_bytes, reps=20):
    """The end-to-end leg's copy floor on this box: one host-to-device and
    one device-to-host copy of the step's sizes, pinned, issued together on
    two streams, timed with CUDA events; milliseconds per pair."""
    import torch
    h = [torch.empty(b, dtype=torch.uint8, pin_memory=True) for b in (h2d_bytes, d2h_bytes)]
    d = [torch.empty(b, dtype=torch.uint8, device="cuda") for b in (h2d_bytes, d2h_bytes)]
    up, down = torch.cuda.Stream(), torch.cuda.Stream()
    main = torch.cuda.current_stream()

    def pairs(n):
        up.wait_stream(main)
        down.wait_stream(main)
        for _ in range(n):
            with torch.cuda.stream(up):
                d[0].copy_(h[0], non_blocking=True)
            with torch.cuda.stream(down):
                h[1].copy_(d[1], non_blocking=True)
        main.wait_stream(up)
        main.wait_stream(down)

    pairs(3)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    pairs(reps)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def e2e_bound(nb_up, nb_down, secs, steps):
    """the copy floor against the measured end-to-end step"""
    floor = pcie_bound(nb_up, nb_down)
    step_ms = 1e3 * secs / steps
    return {"copy_pair_ms": floor, "step_ms": step_ms, "frac": floor / step_ms,
            "gbs_per_direction": max(nb_up, nb_down) / floor / 1e6,
            "how": "one pinned host-to-device and one device-to-host copy of the step's sizes "
                   "issued together on two streams, CUDA-event timed: the floor of a step "
                   "that moves both"}


def accuracy_leg(akb, config, mesh, mat, v0, blocked, nsteps):
    """The mixed path against the plain FP64 path (bit-identical to the CPU
    oracle for elastic / plastic, within 1e-12 for neohookean) after nsteps
    steps from the same state: relative L2 of the displacement, and the drift
    of the total energy (kinetic + potential) of each path."""
    models = {}
    e0 = {}
    for prec in ("mixed", "fp64"):
        m = akb.SolidMechanicsModel(mesh)
        m.addMaterial(mat["type"], **{k: v for k, v in mat.items() if k != "type"})
        m.initFull(akb._explicit_lumped_mass, precision=prec)
        m.setNodal("velocity", v0)
        m.setNodal("blocked_dofs", blocked)
        m.setTimeStep(0.8 * m.getStableTimeStep())
        if config == "tri6":
            m.setPrescribedVelocityRamp(np.isclose(mesh.nodes[:, 0], 1.0), 0, 1e-3, 5000)
        e0[prec] = m.getEnergy("kinetic") + m.getEnergy("potential")
        models[prec] = m
    out = {"steps": nsteps}
    for prec, m in models.items():
        m.solveStep(nsteps)
        e = m.getEnergy("kinetic") + m.getEnergy("potential")
        out[f"energy_drift_{prec}"] = (e - e0[prec]) / e0[prec]
        out[f"energy_{prec}"] = e
    u, ud = models["mixed"].getDisplacement(), models["fp64"].getDisplacement()
    out["rel_l2_displacement"] = float(np.linalg.norm(u - ud) / np.linalg.norm(ud))
    out["energy_rel_diff"] = abs(out["energy_mixed"] - out["energy_fp64"]) / abs(out["energy_fp64"])
    out["note"] = ("prescribed edge motion: the energy is not conserved, drift is the work of the "
                   "pulled edge" if config == "tri6" else "free vibration: drift is the "
                   "integration error of each path")
    return out


def build_batch(akb, meshes, mats, vels, blocks, precision):
    b = akb.BatchModel(meshes)
    for mat in mats:
        b.addMaterial(mat["type"], **{k: v for k, v in mat.items() if k != "type"})
    b.setInstanceMaterials(np.arange(len(meshes)))
    b.initFull(akb._explicit_lumped_mass, precision=precision)
    b.setNodal("velocity", np.concatenate(vels))
    b.setNodal("blocked_dofs", np.concatenate(blocks))
    b.setTimeSteps(0.8 * b.getStableTimeSteps())
    return b


def run_batch(args, rep=None, emit=True, extra=False):
    own = rep is None
    rep = rep or Replicas("nccl")
    world, rank, local = rep.world, rep.rank, rep.local
    barrier, max_over_ranks = rep.barrier, rep.max
    import akantu2_b200 as akb
    from akantu2_b200 import _capi
    _capi.check(_capi.lib().akb_set_device(local))

    meshes, mats, vels, blocks = batch_workload(args.instances)
    E = sum(m.getNbElement() for m in meshes)
    N = sum(m.getNbNodes() for m in meshes)
    desc = (f"{len(meshes)} tet4 elastic cubes, n in 8..32 cells per edge "
            f"({E} elements, {N} nodes)")
    peak, peak_kind = read_peaks()
    precisions = [p for p in args.precisions.split(",") if p]
    results = {}
    for prec in precisions:
        b = build_batch(akb, meshes, mats, vels, blocks, prec)
        b.timeSteps(max(3, args.warmup))
        if not args.no_autotune:
            b.autotune(5)
        b.prepareGraphs()
        barrier()
        with ClockSampler(local) as clk:
            ms = b.timeSteps(args.steps)
        barrier()
        ms = max_over_ranks(ms)
        nprof = min(args.steps, 20)
        _, phases = b.profileSteps(nprof)
        step_b, kern_b = algorithmic_bytes("batch", b.mesh, prec)
        elem_ms = phases[1] / nprof
        results[prec] = {
            "ms_per_step": ms / args.steps,
            "value": aggregate_rate(E * args.steps, world, ms),
            "phase_ms_per_step": {"predictor": phases[0] / nprof,
                                  "element_forces": phases[1] / nprof,
                                  "node_update": phases[2] / nprof},
            "roofline": roofline_entry(kern_b, elem_ms, peak, peak_kind,
                                       read_traffic("batch", prec)),
            "roofline_step": {"bytes_per_element_step": step_b / E,
                              "achieved": step_b / (ms / args.steps / 1e3) / 1e9,
                              "frac": step_b / (ms / args.steps / 1e3) / 1e9 / peak},
            "clocks": clk.summary(),
            "gpu_launches": args.steps * 2,
            "state_finite": b.getStatus() == 0 and bool(np.all(np.isfinite(b.getDisplacement()))),
        }
        if prec == precisions[0] and not extra:
            nb = N * 3 * 8
            k_e2e = max(1, min(args.steps, 100))
            secs_sync, secs_async = e2e_legs(b, (N, 3), k_e2e, barrier, args.e2e_lag)
            secs_sync, secs_async = max_over_ranks(secs_sync), max_over_ranks(secs_async)
            results[prec]["e2e"] = {"value": world * E * k_e2e / secs_async, "unit": UNIT,
                                    "steps": k_e2e, "h2d_bytes_per_step": nb,
                                    "d2h_bytes_per_step": nb,
                                    "mode": "pipelined async C ABI copies (see e2e_legs)",
                                    "synchronous_value": world * E * k_e2e / secs_sync,
                                    "pcie_bound": e2e_bound(nb, nb, secs_async, k_e2e)}
        del b
    # unbatched baseline: every 16th instance alone (sizes spread over the
    # range), FP64, same step count with the same graphs
    alone_e, alone_ms = 0, 0.0
    for k in (range(0, len(meshes), max(1, len(meshes) // 16)) if not extra else []):
        m = akb.SolidMechanicsModel(meshes[k])
        m.addMaterial(mats[k]["type"], **{kk: v for kk, v in mats[k].items() if kk != "type"})
        m.initFull(akb._explicit_lumped_mass, precision="fp64")
        m.setNodal("velocity", vels[k])
        m.setNodal("blocked_dofs", blocks[k])
        m.setTimeStep(0.8 * m.getStableTimeStep())
        m.timeSteps(max(3, args.warmup))
        if not args.no_autotune:
            m.autotune(5)
        m.prepareGraphs()
        alone_ms += m.timeSteps(args.steps)
        alone_e += meshes[k].getNbElement()
        del m
    unbatched = alone_e * args.steps / (alone_ms / 1e3) if alone_ms > 0 else None
    head = results[precisions[0]]
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu and not extra:
        threads = os.cpu_count() or 1
        cpu = cpu_batch_rate(meshes, mats, vels, blocks, threads, budget_s=20.0)
    if rank == 0:
        line = {
            "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": max(3, args.warmup),
            "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 element math / f64 state" if precisions[0] == "mixed" else "f64",
            "data": "synthetic (seeded meshes, materials and sinusoidal modes)",
            "config": {"workload": desc, "instances": len(meshes), "elements": E, "nodes": N,
                       "quadrature_points": 1, "precision": precisions[0],
                       "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (no flush)"},
            "e2e": head.get("e2e"), "roofline": head["roofline"],
            "roofline_step": head["roofline_step"], "clocks": head["clocks"],
            "gpu_launches": head["gpu_launches"], "state_finite": head["state_finite"],
            "phase_ms_per_step": head["phase_ms_per_step"],
            "unbatched_fp64": {"value": unbatched, "unit": UNIT,
                               "sample": "every 16th instance run alone, FP64"},
            "cpu_baseline": cpu,
        }
        for prec in precisions[1:]:
            r = results[prec]
            line[prec] = {"value": r["value"], "ms_per_step": r["ms_per_step"],
                          "roofline": r["roofline"], "roofline_step": r["roofline_step"],
                          "phase_ms_per_step": r["phase_ms_per_step"]}
        if "fp64" in results and precisions[0] != "fp64":
            line["speedup_vs_fp64"] = head["value"] / results["fp64"]["value"]
        if unbatched:
            line["speedup_vs_unbatched_fp64"] = head["value"] / unbatched
        if emit:
            print(json.dumps(line), flush=True)
    if own:
        rep.close()
    return line if rank == 0 else None


def cpu_serve_rate(reqs, threads, budget_s):
    """Oracle element-steps/s over the first requests of the stream, 20 steps
    of each (bounded time)."""
    from oracle import oracle as orc
    elems, secs, done = 0, 0.0, 0
    for (_, kind, cells, mat, _) in reqs:
        mesh, v, b = serve_mesh(kind, cells)
        o = orc.OracleModel(orc.TET4 if kind == "tet" else orc.HEX8, mesh.nodes,
                            mesh.connectivity, [mat], threads=threads)
        o.set(orc.V, v)
        o.set(orc.BLOCKED, b)
        o.set_dt(0.8 * o.stable_dt())
        o.step(1)
        t0 = time.perf_counter()
        o.step(20)
        secs += time.perf_counter() - t0
        elems += mesh.getNbElement() * 20
        done += 1
        if secs > budget_s:
            break
    return {"value": elems / secs, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"20 steps of each of the first {done} requests "
                      f"(CPU oracle, {threads} threads, {secs:.1f} s)"}


def cpu_batch_rate(meshes, mats, vels, blocks, threads, budget_s):
    """Oracle element-steps/s over the instances in turn (bounded time)."""
    from oracle import oracle as orc
    elems, secs, steps_total, done = 0, 0.0, 0, 0
    for k in range(len(meshes)):
        o = orc.OracleModel(orc.TET4, meshes[k].nodes, meshes[k].connectivity, [mats[k]],
                            threads=threads)
        o.set(orc.V, vels[k])
        o.set(orc.BLOCKED, blocks[k])
        o.set_dt(0.8 * o.stable_dt())
        o.step(1)
        t0 = time.perf_counter()
        o.step(20)
        secs += time.perf_counter() - t0
        elems += meshes[k].getNbElement() * 20
        steps_total += 20
        done += 1
        if secs > budget_s:
            break
    rate = elems / secs
    return {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"20 steps of each of the first {done} instances "
                      f"(CPU oracle, {threads} threads, {secs:.1f} s)"}


def run_serve(args):
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    import akantu2_b200 as akb
    from akantu2_b200 import _capi
    _capi.check(_capi.lib().akb_set_device(local))
    reqs = serve_requests(args.requests, args.rate)
    precision = [p for p in args.precisions.split(",") if p][0]
    # meshes are generated before the clock starts (the client's work)
    for _, kind, cells, _, _ in reqs:
        serve_mesh(kind, cells)
    # warm the library (context, module load) outside the timed stream
    warm = akb.Server(device=local, max_active=2)
    m0, v0, b0 = serve_mesh("tet", (2, 2, 2))
    warm.submit(m0, SERVE_MATERIALS[0], 100, velocity=v0, blocked=b0, precision=precision)
    warm.drain()
    warm.close()
    srv = akb.Server(device=local, max_active=args.max_active, chunk_steps=500,
                     builders=args.builders, batching=not args.no_batching)
    done = []
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        for (t_arr, kind, cells, mat, steps) in reqs:
            while True:
                now = time.perf_counter() - t0
                if now >= t_arr:
                    break
                done += srv.poll(wait=min(0.002, t_arr - now))
            mesh, v, b = serve_mesh(kind, cells)
            srv.submit(mesh, mat, steps, velocity=v, blocked=b, precision=precision)
        done += srv.drain(timeout=3600)
        wall = time.perf_counter() - t0
    srv.close()
    bad = [c for c in done if c["status"] != 0]
    lat = np.array([c["t_end"] - c["t_submit"] for c in done])
    wait = np.array([c["t_admit"] - c["t_submit"] for c in done])
    build = np.array([c["t_start"] - c["t_admit"] for c in done])
    run = np.array([c["t_end"] - c["t_start"] for c in done])
    work = float(sum(c["nb_elements"] * c["nb_steps"] for c in done))
    span = max(c["t_end"] for c in done) - min(c["t_submit"] for c in done)
    if rank == 0:
        line = {
            "metric": METRIC, "value": world * work / span, "unit": UNIT, "n_gpus": world,
            "steps": len(done), "warmup": 1, "ms_per_step": 1e3 * span / max(1, len(done)),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 element math / f64 state" if precision == "mixed" else "f64",
            "data": "synthetic (seeded request stream)",
            "config": {"workload": f"{len(reqs)} solve requests, Poisson arrivals at "
                                   f"{args.rate}/s, tet4/hex8 boxes of 1e3..1e6 elements, "
                                   "3 laws, 500..5000 steps",
                       "precision": precision, "max_active": args.max_active,
                       "batching": not args.no_batching,
                       "chunk_steps": 500, "parallelism": f"replicas x{world}"},
            "latency_s": {"p50": float(np.percentile(lat, 50)),
                          "p99": float(np.percentile(lat, 99)),
                          "mean": float(lat.mean()), "max": float(lat.max())},
            "queue_wait_s": {"p50": float(np.percentile(wait, 50)),
                             "p99": float(np.percentile(wait, 99))},
            "build_s": {"p50": float(np.percentile(build, 50)),
                        "p99": float(np.percentile(build, 99))},
            "run_s": {"p50": float(np.percentile(run, 50)), "p99": float(np.percentile(run, 99))},
            "requests_per_s": len(done) / span, "element_steps": work, "wall_s": wall,
            "batched_requests": int(sum(c.get("batched", False) for c in done)),
            "batching": not args.no_batching,
            "failed": len(bad),
            "failures": [{k: c.get(k) for k in ("status", "message", "nb_elements", "nb_steps",
                                                "batched")} for c in bad[:5]],
            "clocks": clk.summary(),
            "e2e": {"value": world * work / span, "unit": UNIT,
                    "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                    "note": "each request uploads its mesh and initial state and reads its "
                            "final displacement; value covers arrival to result"},
        }
        print(json.dumps(line), flush=True)


def run_partitioned(args):
    """One mesh of the configuration split into subdomains (coordinate
    bisection, ghost layer, per-step halo exchange of the predicted
    displacement).  Under torchrun: one subdomain per rank, the exchange over
    NCCL on each model's stream, device time of the K steps (events on the
    model's stream) taken as the maximum over ranks; strong scaling.  In one
    process with --parts P: P subdomains advanced on the one GPU."""
    rep = Replicas("nccl")
    world, rank, local = rep.world, rep.rank, rep.local
    import torch
    import akantu2_b200 as akb
    from akantu2_b200 import _capi
    _capi.check(_capi.lib().akb_set_device(local))
    mesh, mat, desc = workload(args.config, args.cells)
    v0, blocked = initial_state(args.config, mesh)
    prec = [p for p in args.precisions.split(",") if p][0]
    if world > 1:
        pm = akb.DistributedModel(mesh, device=local)
        nparts = world
    else:
        nparts = max(1, args.parts)
        pm = akb.PartitionedModel(mesh, nparts)
    pm.addMaterial(mat["type"], **{k: v for k, v in mat.items() if k != "type"})
    pm.initFull(akb._explicit_lumped_mass, precision=prec)
    pm.setNodal("velocity", v0)
    pm.setNodal("blocked_dofs", blocked)
    pm.setTimeStep(0.8 * pm.getStableTimeStep())
    if args.config == "tri6":
        pm.setPrescribedVelocityRamp(np.isclose(mesh.nodes[:, 0], 1.0), 0, 1e-3, 5000)
    pm.solveStep(max(3, args.warmup))
    E = mesh.getNbElement()
    models = [lc.model for lc in pm.locals]
    for m in models:
        m.synchronize()
    rep.barrier()
    # events on the first local model's stream
    sp = ctypes_stream(models[0])
    stream = torch.cuda.ExternalStream(sp, device=torch.device("cuda", local))
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        if world == 1:
            # all subdomains on this GPU: device time of the exchange's steps
            # (its graphs fork into and join from every subdomain's stream)
            ms = pm.timeSteps(args.steps)
        else:
            t0.record(stream)
            pm.solveStep(args.steps)
            t1.record(stream)
            t1.synchronize()
            ms = t0.elapsed_time(t1)
    ms = rep.max(ms)
    rep.barrier()
    local_elems = [len(lc.sub.element_global) for lc in pm.locals]
    if rank == 0:
        line = {
            "metric": METRIC, "value": E * args.steps / (ms / 1e3), "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": max(3, args.warmup),
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None,
            "dtype": "f32 element math / f64 state" if prec == "mixed" else "f64",
            "data": "synthetic (seeded random-field initial velocity)",
            "config": {"workload": desc, "elements": E, "nodes": mesh.getNbNodes(),
                       "precision": prec, "parallelism": f"partitioned x{nparts}",
                       "subdomain_elements_rank0": local_elems,
                       "l2": "inputs larger than L2 (no flush)"},
            "clocks": clk.summary(),
            # per step and subdomain: element forces, node update, the ramp
            # (tri6), one halo pack and one unpack per neighbor (rank 0's
            # subdomains)
            "gpu_launches": args.steps * sum(2 + (1 if args.config == "tri6" else 0) +
                                             2 * len(lc.sub.neighbors) for lc in pm.locals),
        }
        print(json.dumps(line), flush=True)
    rep.close()


def ctypes_stream(model):
    import ctypes
    from akantu2_b200 import _capi
    sp = ctypes.c_void_p()
    _capi.check(_capi.lib().akb_model_stream(model._h, ctypes.byref(sp)))
    return sp.value


def compact(line):
    """the figures of a configuration's line kept as a sub-record"""
    keys = ("value", "ms_per_step", "roofline", "roofline_step", "phase_ms_per_step",
            "speedup_vs_fp64", "clocks", "state_finite", "tuning")
    out = {k: line[k] for k in keys if k in line}
    out["workload"] = line["config"]["workload"]
    out["elements"] = line["config"]["elements"]
    if "fp64" in line:
        out["fp64"] = {k: line["fp64"][k] for k in ("value", "ms_per_step", "roofline")
                       if k in line["fp64"]}
    return out


def run_default_with_extras(args):
    """The default run on one GPU: the hexahedral configuration's line, with
    compact records of the plastic triangle square and of the 256-mesh batch
    (mixed and FP64 each, 20 timed steps after the same warm-up, autotuned
    shapes; no CPU, accuracy or end-to-end legs for those two) appended to
    the same JSON line."""
    import copy
    rep = Replicas("nccl")
    line = run_ours(args, rep=rep, emit=False)
    extras = {}
    # the plastic square with the reference's default 3-point rule and with
    # the 6-point rule its configuration names
    for name, config, rule, runner in (("tri6", "tri6", 0, run_ours),
                                       ("tri6_6points", "tri6", 1, run_ours),
                                       ("batch", "batch", 0, run_batch)):
        a = copy.copy(args)
        a.config, a.steps, a.no_cpu, a.accuracy_steps, a.no_e2e_fp64 = config, 20, True, 0, True
        a.precisions = "mixed,fp64"
        a.qp_rule = rule
        extras[name] = compact(runner(a, rep=rep, emit=False, extra=True))
    line["configs"] = extras
    print(json.dumps(line), flush=True)
    rep.close()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.mode == "partitioned" and args.config in ("hex8", "tet", "tri6"):
        run_partitioned(args)
    elif args.config == "serve":
        run_serve(args)
    elif args.config == "batch":
        run_batch(args)
    elif args.config == "hex8" and not args.no_extras and not args.cells and \
            int(os.environ.get("WORLD_SIZE", "1")) == 1:
        run_default_with_extras(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

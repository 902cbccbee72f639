"""The multi-GPU path of bench.py is independent replicas: each rank runs its
own copy of the workload, the only collectives are a barrier and the maximum
of the device-timed durations.  This runs that host logic with two gloo
ranks on the CPU."""
import json
import multiprocessing as mp
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    rep = bench.Replicas("gloo")
    rep.barrier()
    ms = rep.max(10.0 + rank)  # rank 1 is the slower one
    value = bench.aggregate_rate(1000, rep.world, ms)
    rep.barrier()
    rep.close()
    out.put((rank, ms, value))


def test_two_gloo_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [11.0, 11.0]
    # whole-job rate: both ranks' units over the slowest rank's time
    assert res[0][2] == pytest.approx(2 * 1000 / 0.011)


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    rep = bench.Replicas("gloo")
    assert rep.world == 1 and rep.dist is None
    assert rep.max(3.5) == 3.5
    rep.barrier()
    rep.close()


def test_reference_arm_runs_on_rank_zero_only():
    """under torchrun every rank but 0 exits at once without output"""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1"], env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0
    assert r.stdout.strip() == ""


def test_reference_arm_line_on_a_small_case():
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--config", "tet", "--cells", "4", "--steps", "2"], env=env,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] == "port"

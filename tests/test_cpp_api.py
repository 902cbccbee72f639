"""The C++ drop-in API (include/akantu_b200/solid_mechanics_model.hh) used by a
driver written like the reference's explicit examples (examples/
explicit_dynamic.cc): it compiles against the header and libakb.so, and on a
GPU its results match the CPU oracle."""
import os
import subprocess

import numpy as np
import pytest

import akantu2_b200 as akb
from oracle import oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def build_example(tmp_path):
    exe = tmp_path / "explicit_dynamic"
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror",
           "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "examples", "explicit_dynamic.cc"),
           "-L", os.path.join(ROOT, "akantu2_b200"), "-lakb",
           "-Wl,-rpath," + os.path.join(ROOT, "akantu2_b200"), "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


MATERIAL = "material elastic [\n  name = unit\n  rho = 1\n  E = 1\n  nu = 0.3\n]\n"


def test_example_compiles(tmp_path):
    exe = build_example(tmp_path)
    assert exe.exists()


def build_serving_example(tmp_path):
    exe = tmp_path / "serve_boxes"
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror",
           "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "examples", "serve_boxes.cc"),
           "-L", os.path.join(ROOT, "akantu2_b200"), "-lakb",
           "-Wl,-rpath," + os.path.join(ROOT, "akantu2_b200"), "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_serving_example_compiles(tmp_path):
    assert build_serving_example(tmp_path).exists()


@pytest.mark.gpu
def test_serving_example_runs(tmp_path):
    """every submitted solve completes, and solves of the same box agree"""
    exe = build_serving_example(tmp_path)
    out = subprocess.run([str(exe), "8", "200"], check=True, capture_output=True,
                         text=True).stdout.splitlines()
    assert len(out) == 8 and all(" failed " not in line for line in out)
    by_size = {}
    for line in out:
        f = line.split()
        by_size.setdefault(f[3], set()).add(f[7])
    assert all(len(v) == 1 for v in by_size.values())  # same box, same result


def _oracle_run(kind, cells, steps):
    mesh = akb.box_hex8(cells) if kind == "hex8" else akb.box_tet4(cells)
    x = mesh.nodes
    o = orc.OracleModel(orc.HEX8 if kind == "hex8" else orc.TET4, x, mesh.connectivity,
                        [dict(type="elastic", rho=1.0, E=1.0, nu=0.3)])
    bl = np.zeros(x.shape, dtype=np.uint8)
    bl[x[:, 2] == 0.0] = 1
    v = np.zeros_like(x)
    v[:, 2] = 0.01 * np.sin(np.pi * x[:, 0]) * np.sin(np.pi * x[:, 1]) * x[:, 2]
    o.set(orc.BLOCKED, bl)
    o.set(orc.V, v)
    o.set_dt(0.8 * o.stable_dt())
    o.step(steps)
    return np.max(np.abs(o.get(orc.U))), o.energy(orc.EKIN), o.energy(orc.EPOT)


@pytest.mark.gpu
@pytest.mark.parametrize("kind,cells,steps", [("hex8", 5, 80), ("tet4", 4, 80)])
def test_example_matches_oracle(tmp_path, kind, cells, steps):
    exe = build_example(tmp_path)
    dat = tmp_path / "material.dat"
    dat.write_text(MATERIAL)
    out = subprocess.run([str(exe), str(dat), kind, str(cells), str(steps)], check=True,
                         capture_output=True, text=True).stdout.split()
    got = dict(zip(out[0::2], out[1::2]))
    umax, ekin, epot = _oracle_run(kind, cells, steps)
    assert float(got["u_max"]) == umax
    assert abs(float(got["ekin"]) - ekin) <= 1e-12 * ekin
    assert abs(float(got["epot"]) - epot) <= 1e-12 * epot

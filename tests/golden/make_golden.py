"""Generates the golden fixtures of tests/golden/ from the reference's own test
data.  Run once in a container that has the reference tree, giving its root
as the argument; the fixtures it writes are committed, the GPU host never
reads the reference.

  fe_<type>.npz     meshes of test/test_fe_engine/_<type>.msh with
                    - the per-element inradius of test/test_fe_engine/_<type>.csv
                      (checked by test_fe_engine_inradius.cc to 1e-6)
                    - N, B = dN/dx and j = det J * w computed by the reference's
                      independent numpy engine test/test_fe_engine/py_engine/
                      py_engine.py (the cross-check of
                      test_fe_engine_precomputation.cc, tolerance 1e-10)
  patch_<type>.npz  meshes of test/test_model/patch_tests/data/_<type>.msh
                    (patch tests and lumped-mass test)

usage: python tests/golden/make_golden.py REFERENCE_ROOT
"""
import contextlib
import io
import os
import sys

import numpy as np

if len(sys.argv) != 2:
    sys.exit("usage: python tests/golden/make_golden.py REFERENCE_ROOT")
REF = sys.argv[1]
OUT = os.path.dirname(os.path.abspath(__file__))

GMSH_TYPE = {"_tetrahedron_4": (4, 4, 3), "_hexahedron_8": (5, 8, 3), "_triangle_6": (9, 6, 2)}


def read_msh(path, etype):
    """Minimal gmsh 2.x ASCII reader: nodes in file order, elements of one type."""
    gtype, nn, dim = GMSH_TYPE[etype]
    with open(path) as f:
        lines = [l.strip() for l in f]
    i = lines.index("$Nodes")
    n = int(lines[i + 1])
    ids, nodes = {}, []
    for k in range(n):
        parts = lines[i + 2 + k].split()
        ids[int(parts[0])] = k
        nodes.append([float(x) for x in parts[1:1 + dim]])
    i = lines.index("$Elements")
    m = int(lines[i + 1])
    conn = []
    for k in range(m):
        parts = [int(x) for x in lines[i + 2 + k].split()]
        if parts[1] != gtype:
            continue
        ntags = parts[2]
        conn.append([ids[x] for x in parts[3 + ntags:3 + ntags + nn]])
    return np.array(nodes, dtype=np.float64), np.array(conn, dtype=np.int32)


def main():
    sys.path.insert(0, os.path.join(REF, "test", "test_fe_engine", "py_engine"))
    import py_engine  # noqa: E402  (reference's independent numpy engine)

    for etype in GMSH_TYPE:
        nodes, conn = read_msh(os.path.join(REF, "test/test_fe_engine", etype + ".msh"), etype)
        radii = np.zeros(len(conn))
        with open(os.path.join(REF, "test/test_fe_engine", etype + ".csv")) as f:
            for line in f:
                if line.strip():
                    k, r = line.split(",")
                    radii[int(k)] = float(r)
        dim = nodes.shape[1]
        nn = conn.shape[1]
        X = nodes[conn].reshape(len(conn), nn * dim)
        shapes = py_engine.Shapes(etype)
        nq = len(shapes._g)
        N = np.zeros((len(conn) * nq, nn))
        B = np.zeros((len(conn) * nq, nn * dim))
        j = np.zeros((len(conn) * nq, 1))
        # py_engine prints a line for every N that differs from its own; the
        # arrays passed in are zeros, so silence that
        with contextlib.redirect_stdout(io.StringIO()):
            shapes.precompute(X=X, N=N, B=B, j=j, Q=shapes._g.T)
        np.savez_compressed(os.path.join(OUT, f"fe{etype}.npz"), nodes=nodes, conn=conn,
                            inradius=radii, N=N.reshape(len(conn), nq, nn),
                            B=B.reshape(len(conn), nq, nn, dim), j=j.reshape(len(conn), nq),
                            quad_points=shapes._g, quad_weights=shapes._w)
        pnodes, pconn = read_msh(
            os.path.join(REF, "test/test_model/patch_tests/data", etype + ".msh"), etype)
        np.savez_compressed(os.path.join(OUT, f"patch{etype}.npz"), nodes=pnodes, conn=pconn)
        print(etype, "fe mesh", conn.shape, "patch mesh", pconn.shape)


if __name__ == "__main__":
    main()

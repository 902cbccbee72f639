"""gmsh reading in formats 2.2, 4.0 and 4.1 (src/io/mesh_io/mesh_io_msh.cc,
populateReaders2 / populateReaders4) and the node groups made from the file's
physical groups.  Each test writes one box of hexahedra in the three formats,
with a named volume group, a named bottom-face group, a named corner point and
an unnamed top-face group, and node ids that are neither contiguous nor sorted.
"""
import os
import subprocess

import numpy as np
import pytest

import akantu2_b200 as akb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

NAMES = {1: "body", 2: "bottom", 4: "corner"}  # physical tag 3 has no name
VOLUME, BOTTOM, TOP, POINT = 7, 5, 6, 9       # entity tags


def _box():
    mesh = akb.box_hex8(2, 3, 2)
    x, conn = mesh.nodes, mesh.connectivity
    # the element faces as quadrangles (gmsh type 3); those on z = 0 and z = max
    faces = np.concatenate([conn[:, [0, 1, 5, 4]], conn[:, [1, 2, 6, 5]], conn[:, [2, 3, 7, 6]],
                            conn[:, [3, 0, 4, 7]], conn[:, [0, 3, 2, 1]], conn[:, [4, 5, 6, 7]]])
    on = lambda z: faces[np.all(np.isclose(x[faces, 2], z), axis=1)]
    ids = 1000 - 7 * np.arange(len(x))  # gmsh ids of the nodes, decreasing
    return x, conn, on(0.0), on(x[:, 2].max()), ids


def _entities(version):
    """one point, two surfaces and one volume, of physical tags 4, 2, 3 and 1"""
    point = f"{POINT} 0 0 0" + ("" if version == "4.1" else " 0 0 0") + " 1 4"
    return ["$Entities", "1 0 2 1", point,
            f"{BOTTOM} 0 0 0 1 1 0 1 2 0", f"{TOP} 0 0 1 1 1 1 1 3 0",
            f"{VOLUME} 0 0 0 1 1 1 1 1 0", "$EndEntities"]


def write_msh(path, version, names=True):
    x, conn, bottom, top, ids = _box()
    out = ["$MeshFormat", f"{version} 0 8", "$EndMeshFormat"]
    if names:
        out += ["$PhysicalNames", str(len(NAMES))]
        dims = {1: 3, 2: 2, 4: 0}
        out += [f'{dims[t]} {t} "{n}"' for t, n in NAMES.items()]
        out += ["$EndPhysicalNames"]
    fmt = lambda v: " ".join("%.17g" % c for c in v)
    blocks = [(0, POINT, 15, np.array([[0]])), (2, BOTTOM, 3, bottom), (2, TOP, 3, top),
              (3, VOLUME, 5, conn)]
    phys = {POINT: 4, BOTTOM: 2, TOP: 3, VOLUME: 1}
    if version == "2.2":
        out += ["$Nodes", str(len(x))]
        out += [f"{ids[i]} {fmt(x[i])}" for i in range(len(x))]
        out += ["$EndNodes", "$Elements", str(sum(len(b[3]) for b in blocks))]
        k = 1
        for _, tag, gtype, el in blocks:
            for c in el:
                out.append(f"{k} {gtype} 2 {phys[tag]} {tag} " + " ".join(str(ids[n]) for n in c))
                k += 1
        out += ["$EndElements"]
    else:
        out += _entities(version)
        # nodes in two blocks: the corner point's node, then the rest
        parts = [(0, POINT, np.array([0])), (3, VOLUME, np.arange(1, len(x)))]
        head = f"{len(parts)} {len(x)}" + (f" {ids.min()} {ids.max()}" if version == "4.1" else "")
        out += ["$Nodes", head]
        for dim, tag, nodes in parts:
            if version == "4.1":
                out.append(f"{dim} {tag} 0 {len(nodes)}")
                out += [str(ids[n]) for n in nodes]
                out += [fmt(x[n]) for n in nodes]
            else:
                out.append(f"{tag} {dim} 0 {len(nodes)}")
                out += [f"{ids[n]} {fmt(x[n])}" for n in nodes]
        out += ["$EndNodes"]
        ne = sum(len(b[3]) for b in blocks)
        out += ["$Elements", f"{len(blocks)} {ne}" + (f" 1 {ne}" if version == "4.1" else "")]
        k = 1
        for dim, tag, gtype, el in blocks:
            out.append(f"{dim} {tag} {gtype} {len(el)}" if version == "4.1"
                       else f"{tag} {dim} {gtype} {len(el)}")
            for c in el:
                out.append(f"{k} " + " ".join(str(ids[n]) for n in c))
                k += 1
        out += ["$EndElements"]
    path.write_text("\n".join(out) + "\n")
    return x, conn, bottom, top


@pytest.mark.parametrize("version", ["2.2", "4.0", "4.1"])
def test_nodes_elements_and_tags(tmp_path, version):
    p = tmp_path / "box.msh"
    x, conn, _, _ = write_msh(p, version)
    mesh = akb.Mesh(3).read(p)
    assert mesh.element_type == "_hexahedron_8"
    assert np.array_equal(mesh.nodes, x)
    assert np.array_equal(mesh.connectivity, conn)
    assert np.all(mesh.physical_tags == 1)


@pytest.mark.parametrize("version", ["2.2", "4.0", "4.1"])
def test_named_groups(tmp_path, version):
    p = tmp_path / "box.msh"
    x, conn, bottom, top = write_msh(p, version)
    g = akb.Mesh(3).read(p).node_groups
    assert np.array_equal(g["body"], np.arange(len(x)))
    assert np.array_equal(g["bottom"], np.nonzero(x[:, 2] == 0.0)[0])
    assert np.array_equal(g["bottom"], np.unique(bottom))
    assert np.array_equal(g["corner"], [0])
    # the unnamed tag: format 2 names the group by the tag's number and fills
    # it; format 4 creates "msh_block_3" and leaves it empty
    if version == "2.2":
        assert set(g) == {"body", "bottom", "corner", "3"}
        assert np.array_equal(g["3"], np.unique(top))
    else:
        assert set(g) == {"body", "bottom", "corner", "msh_block_3"}
        assert len(g["msh_block_3"]) == 0


@pytest.mark.parametrize("version", ["2.2", "4.0", "4.1"])
def test_groups_without_physical_names(tmp_path, version):
    p = tmp_path / "box.msh"
    write_msh(p, version, names=False)
    g = akb.Mesh(3).read(p).node_groups
    if version == "2.2":
        assert g == {}  # format 2 makes groups only from $PhysicalNames
    else:
        assert set(g) == {"msh_block_1", "msh_block_2", "msh_block_3", "msh_block_4"}
        assert all(len(v) == 0 for v in g.values())


def test_formats_agree(tmp_path):
    meshes = []
    for v in ("2.2", "4.0", "4.1"):
        p = tmp_path / f"box{v}.msh"
        write_msh(p, v)
        meshes.append(akb.Mesh(3).read(p))
    for m in meshes[1:]:
        assert np.array_equal(m.nodes, meshes[0].nodes)
        assert np.array_equal(m.connectivity, meshes[0].connectivity)
        for name in ("body", "bottom", "corner"):
            assert np.array_equal(m.node_groups[name], meshes[0].node_groups[name])


def test_group_bc_on_read_mesh(tmp_path):
    """a group read from the file drives a Dirichlet condition on the host"""
    p = tmp_path / "box.msh"
    x, _, _, _ = write_msh(p, "4.1")
    mesh = akb.Mesh(3).read(p)
    assert np.all(x[mesh.getNodeGroup("bottom"), 2] == 0.0)


def test_malformed_files(tmp_path):
    p = tmp_path / "bad.msh"
    write_msh(p, "4.1")
    text = p.read_text()
    p.write_text(text.replace("$MeshFormat\n4.1 0 8", "$MeshFormat\n3.0 0 8"))
    with pytest.raises(akb.AkbError) as e:
        akb.Mesh(3).read(p)
    assert e.value.name == "AKB_EUNSUPPORTED"
    p.write_text(text.replace("$MeshFormat\n4.1 0 8", "$MeshFormat\n4.1 1 8"))
    with pytest.raises(akb.AkbError) as e:
        akb.Mesh(3).read(p)
    assert e.value.name == "AKB_EUNSUPPORTED"
    # an element that names a node the file does not have
    lines = text.splitlines()
    last = max(i for i, line in enumerate(lines) if not line.startswith("$"))
    lines[last] = lines[last].rsplit(" ", 1)[0] + " 123456"
    p.write_text("\n".join(lines) + "\n")
    with pytest.raises(akb.AkbError) as e:
        akb.Mesh(3).read(p)
    assert e.value.name == "AKB_EPARSE"


CPP = r"""
#include <akantu_b200/solid_mechanics_model.hh>
#include <cstdio>
using namespace akantu_b200;
int main(int, char **argv) {
  Mesh mesh(3);
  mesh.read(argv[1]);
  std::printf("%d %d %zu %zu %zu\n", (int)mesh.getNbNodes(), (int)mesh.getNbElement(),
              mesh.getNodeGroup("body").size(), mesh.getNodeGroup("bottom").size(),
              mesh.getNodeGroup("corner").size());
  return 0;
}
"""


def test_cpp_mesh_read_groups(tmp_path):
    src = tmp_path / "read.cc"
    src.write_text(CPP)
    exe = tmp_path / "read"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I",
                    os.path.join(ROOT, "include"), str(src), "-L",
                    os.path.join(ROOT, "akantu2_b200"), "-lakb",
                    "-Wl,-rpath," + os.path.join(ROOT, "akantu2_b200"), "-o", str(exe)],
                   check=True, capture_output=True, text=True)
    p = tmp_path / "box.msh"
    x, conn, _, _ = write_msh(p, "4.1")
    out = subprocess.run([str(exe), str(p)], check=True, capture_output=True,
                         text=True).stdout.split()
    assert [int(v) for v in out] == [len(x), len(conn), len(x), int(np.sum(x[:, 2] == 0)), 1]

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


# -- material selection by physical name ------------------------------------------
REGIONS = {1: "steel", 2: "rubber", 3: "glass"}  # physical tag 4 has no name


def write_regions(path, version):
    """a row of 8 hexahedra in four volume entities (physical tags 1 2 3 4,
    two elements each): element k lies in entity k // 2 + 1"""
    mesh = akb.box_hex8(8, 1, 1)
    x, conn = mesh.nodes, mesh.connectivity
    fmt = lambda v: " ".join("%.17g" % c for c in v)
    out = ["$MeshFormat", f"{version} 0 8", "$EndMeshFormat",
           "$PhysicalNames", str(len(REGIONS))]
    out += [f'3 {t} "{n}"' for t, n in REGIONS.items()] + ["$EndPhysicalNames"]
    if version == "2.2":
        out += ["$Nodes", str(len(x))] + [f"{i + 1} {fmt(x[i])}" for i in range(len(x))]
        out += ["$EndNodes", "$Elements", str(len(conn))]
        out += [f"{k + 1} 5 2 {k // 2 + 1} {k // 2 + 1} " + " ".join(str(n + 1) for n in c)
                for k, c in enumerate(conn)]
    else:
        out += ["$Entities", "0 0 0 4"]
        out += [f"{t} 0 0 0 1 1 1 1 {t} 0" for t in range(1, 5)] + ["$EndEntities"]
        out += ["$Nodes", f"1 {len(x)} 1 {len(x)}", f"3 1 0 {len(x)}"]
        out += [str(i + 1) for i in range(len(x))] + [fmt(v) for v in x] + ["$EndNodes"]
        out += ["$Elements", f"4 {len(conn)} 1 {len(conn)}"]
        for t in range(1, 5):
            out.append(f"3 {t} 5 2")
            out += [f"{k + 1} " + " ".join(str(n + 1) for n in conn[k])
                    for k in (2 * t - 2, 2 * t - 1)]
    out += ["$EndElements"]
    path.write_text("\n".join(out) + "\n")


def _model_with_materials(mesh):
    model = akb.SolidMechanicsModel(mesh)
    for name, E in (("steel", 2.0), ("rubber", 0.5), ("glass", 1.5)):
        model.addMaterial("elastic", name=name, rho=1.0, E=E, nu=0.3)
    return model


@pytest.mark.parametrize("version", ["2.2", "4.1"])
def test_physical_names_data(tmp_path, version):
    p = tmp_path / "regions.msh"
    write_regions(p, version)
    mesh = akb.Mesh(3).read(p)
    names = list(mesh.getData("physical_names"))
    unnamed = "4" if version == "2.2" else ""  # format 4 leaves it empty
    assert names == ["steel"] * 2 + ["rubber"] * 2 + ["glass"] * 2 + [unnamed] * 2
    assert list(mesh.getData("tag_0")) == [1, 1, 2, 2, 3, 3, 4, 4]


def test_no_physical_names_data_in_format_2(tmp_path):
    p = tmp_path / "box.msh"
    write_msh(p, "2.2", names=False)
    mesh = akb.Mesh(3).read(p)
    with pytest.raises(KeyError):
        mesh.getData("physical_names")


@pytest.mark.parametrize("version", ["2.2", "4.1"])
def test_mesh_data_material_selector(tmp_path, version):
    p = tmp_path / "regions.msh"
    write_regions(p, version)
    model = _model_with_materials(akb.Mesh(3).read(p))
    sel = akb.MeshDataMaterialSelector("physical_names", model)
    # the unnamed region names no material: the fallback value, then a
    # fallback selector
    assert list(sel.select(model)) == [0, 0, 1, 1, 2, 2, 0, 0]
    sel.setFallback(2)
    assert list(sel.select(model)) == [0, 0, 1, 1, 2, 2, 2, 2]
    by_tag = akb.MeshDataMaterialSelectorInt("tag_0", model)
    assert list(by_tag.select(model)) == [1, 1, 2, 2, 3, 3, 4, 4]
    fb = akb.ElementDataMaterialSelector(np.array([1, 1, 1, 1, 1, 1, 2, 1]))
    sel.setFallback(fb)
    assert list(sel.select(model)) == [0, 0, 1, 1, 2, 2, 2, 1]


@pytest.mark.gpu
@pytest.mark.parametrize("version", ["2.2", "4.1"])
def test_selector_at_init_full(tmp_path, version):
    """initFull applies the selector: each material holds its region's
    elements, and the run is bit-identical to one given the same element
    materials directly"""
    p = tmp_path / "regions.msh"
    write_regions(p, version)
    runs = []
    for use_selector in (True, False):
        mesh = akb.Mesh(3).read(p)
        model = _model_with_materials(mesh)
        if use_selector:
            model.setMaterialSelector(akb.MeshDataMaterialSelector("physical_names", model))
        else:
            model.setElementMaterials([0, 0, 1, 1, 2, 2, 0, 0])
        model.initFull(_analysis_method=akb._explicit_lumped_mass)
        if use_selector:
            assert list(model.getMaterial("steel").getElementFilter()) == [0, 1, 6, 7]
            assert list(model.getMaterial("rubber").getElementFilter()) == [2, 3]
            assert list(model.getMaterial("glass").getElementFilter()) == [4, 5]
        x = mesh.nodes
        model.getBlockedDOFs()[x[:, 0] == 0.0] = True
        model.getVelocity()[:, 0] = 0.01 * x[:, 0]
        model.setTimeStep(0.5 * model.getStableTimeStep())
        model.solveStep(50)
        runs.append(model.getDisplacement().copy())
    assert np.array_equal(runs[0], runs[1])
    assert np.abs(runs[0]).max() > 0


CPP_SELECTOR = r"""
#include <akantu_b200/solid_mechanics_model.hh>
#include <cstdio>
#include <cstring>
using namespace akantu_b200;
int main(int argc, char **argv) {
  Mesh mesh(3);
  mesh.read(argv[1]);
  for (const auto &n : mesh.getData<std::string>("physical_names")) std::printf("[%s]", n.c_str());
  for (Idx t : mesh.getData<Idx>("tag_0")) std::printf(" %d", (int)t);
  std::printf("\n");
  if (argc < 3) return 0;
  initialize(argv[2], argc, argv);
  SolidMechanicsModel model(mesh);
  auto selector = std::make_shared<MeshDataMaterialSelector<std::string>>("physical_names", model);
  model.setMaterialSelector(selector);
  model.initFull(_analysis_method = _explicit_lumped_mass);
  for (const char *name : {"steel", "rubber", "glass"}) {
    auto filter = model.getMaterial(name).getElementFilter(_hexahedron_8);
    std::printf("%s", name);
    for (Int k = 0; k < filter.size(); ++k) std::printf(" %d", (int)filter(k, 0));
    std::printf("\n");
  }
  return 0;
}
"""

DAT = "".join(f"material elastic [\n  name = {n}\n  rho = 1\n  E = {E}\n  nu = 0.3\n]\n"
              for n, E in (("steel", 2.0), ("rubber", 0.5), ("glass", 1.5)))


def _build_selector_example(tmp_path):
    src = tmp_path / "selector.cc"
    src.write_text(CPP_SELECTOR)
    exe = tmp_path / "selector"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I",
                    os.path.join(ROOT, "include"), str(src), "-L",
                    os.path.join(ROOT, "akantu2_b200"), "-lakb",
                    "-Wl,-rpath," + os.path.join(ROOT, "akantu2_b200"), "-o", str(exe)],
                   check=True, capture_output=True, text=True)
    return exe


def test_cpp_mesh_data(tmp_path):
    exe = _build_selector_example(tmp_path)
    p = tmp_path / "regions.msh"
    write_regions(p, "4.1")
    out = subprocess.run([str(exe), str(p)], check=True, capture_output=True, text=True).stdout
    assert out.strip() == "[steel][steel][rubber][rubber][glass][glass][][] 1 1 2 2 3 3 4 4"


@pytest.mark.gpu
def test_cpp_selector_at_init_full(tmp_path):
    exe = _build_selector_example(tmp_path)
    p = tmp_path / "regions.msh"
    write_regions(p, "2.2")
    dat = tmp_path / "materials.dat"
    dat.write_text(DAT)
    out = subprocess.run([str(exe), str(p), str(dat)], check=True, capture_output=True,
                         text=True).stdout.splitlines()
    assert out[1:] == ["steel 0 1 6 7", "rubber 2 3", "glass 4 5"]

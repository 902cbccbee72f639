"""Host-side logic of libakb that runs without a GPU: the exported C ABI,
the .dat parser, the gmsh reader, the mesh generators, and the refusal to
compute without a CUDA device (no CPU fallback)."""
import os
import re

import numpy as np
import pytest

import akantu2_b200 as akb
from akantu2_b200 import _capi
from oracle import oracle as orc
from scenarios import OR_TYPE, TYPES, golden

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "akb_capi.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(akb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = _capi.lib()
    names = header_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert missing == []


def _tiny_model(dim=3):
    mesh = akb.box_tet4(1) if dim == 3 else akb.square_tri6(1)
    return mesh, akb.SolidMechanicsModel(mesh)


DAT = """
# parser subset exercised by the reference's test inputs
permissive_parser = true

material elastic [
   name = steel
   rho = 7800   # density
   E   = 2.1e11 # young's modulus
   nu  = 0.3    # poisson's ratio
   Plane_Stress = false # plane strain
   finite_deformation = false
]

material plastic_linear_isotropic_hardening [
   name = metal
   rho = 2 * (0.5 + 0.5)
   E = 1e3 / 10^3
   nu = -(-0.3)
   sigma_y = 1e-3
   h = 0.1
]

solver_options [
   nested_section foo [
      a = 1
   ]
]
"""


def test_dat_parser_reads_materials_and_expressions():
    _, m = _tiny_model()
    L = _capi.lib()
    _capi.check(L.akb_model_load_materials(m._h, DAT.encode()))
    assert m.getNbMaterials() == 2
    steel, metal = m.getMaterial("steel"), m.getMaterial("metal")
    assert steel.get("rho") == 7800.0 and steel.get("E") == 2.1e11 and steel.get("nu") == 0.3
    lam = 0.3 * 2.1e11 / ((1 + 0.3) * (1 - 2 * 0.3))
    assert steel.get("lambda") == lam
    assert metal.get("rho") == 2.0 and metal.get("E") == 1.0 and metal.get("nu") == 0.3
    assert metal.get("sigma_y") == 1e-3 and metal.get("h") == 0.1


@pytest.mark.parametrize("text,code", [
    ("material unknown_law [ E = 1 ]", 10),
    ("material elastic [ E = 1 ", 6),
    ("material elastic [ E = abc ]", 6),
    ("material elastic [ Youngs = 1 ]", 6),
    ("material plastic_linear_isotropic_hardening [ E = 1\n finite_deformation = true ]", 8),
])
def test_dat_parser_errors(text, code):
    _, m = _tiny_model()
    rc = _capi.lib().akb_model_load_materials(m._h, text.encode())
    assert rc == code
    assert _capi.lib().akb_last_error()


def test_finite_deformation_elastic_is_accepted():
    _, m = _tiny_model()
    text = "material elastic [\n name = svk\n E = 2\n nu = 0.25\n finite_deformation = true\n]\n"
    _capi.check(_capi.lib().akb_model_load_materials(m._h, text.encode()))
    mat = m.getMaterial(0)
    assert mat.get("finite_deformation") == 1.0 and mat.get("E") == 2.0


def test_permissive_parser_ignores_unknown_parameters():
    _, m = _tiny_model()
    text = "permissive_parser = true\nmaterial elastic [\n E = 1\n foo = 3\n]\n"
    _capi.check(_capi.lib().akb_model_load_materials(m._h, text.encode()))
    assert m.getNbMaterials() == 1


def test_compute_refuses_without_device():
    count = _capi.ctypes.c_int()
    if _capi.lib().akb_device_count(_capi.ctypes.byref(count)) == 0 and count.value > 0:
        pytest.skip("a CUDA device is present")
    _, m = _tiny_model()
    m.addMaterial("elastic", E=1.0, nu=0.3, rho=1.0)
    with pytest.raises(akb.AkbError) as e:
        m.initFull()
    assert e.value.name == "AKB_ECUDA"


def test_create_rejects_bad_connectivity():
    mesh = akb.box_tet4(1)
    mesh.connectivity[0, 0] = mesh.getNbNodes() + 5
    with pytest.raises(akb.AkbError) as e:
        akb.SolidMechanicsModel(mesh)
    assert e.value.name == "AKB_EINVAL"


def test_batch_offsets_and_local_connectivity():
    meshes = [akb.box_tet4(1), akb.box_tet4(2), akb.box_hex8(1)]
    with pytest.raises(ValueError):
        akb.BatchModel(meshes)  # mixed element types
    b = akb.BatchModel(meshes[:2])
    assert b.nb_instances == 2
    off_n = np.zeros(3, dtype=np.int64)
    off_e = np.zeros(3, dtype=np.int64)
    _capi.check(_capi.lib().akb_batch_instance_offsets(b._h, _capi.ptr(off_n), _capi.ptr(off_e)))
    assert list(off_n) == [0, 8, 35] and list(off_e) == [0, 6, 54]
    assert np.array_equal(off_n, b.node_offsets) and np.array_equal(off_e, b.element_offsets)
    # the combined mesh refers to global node ids
    assert b.mesh.connectivity[b.instance_elements(1)].min() == 8
    # an instance-local id past its own nodes is rejected, even when it would
    # be a valid id of the concatenated array
    bad = akb.Mesh(3).set(meshes[1].nodes, meshes[1].connectivity, akb._tetrahedron_4)
    bad.connectivity[0, 0] = meshes[1].getNbNodes()
    with pytest.raises(akb.AkbError) as e:
        akb.BatchModel([bad, meshes[0]])
    assert e.value.name == "AKB_EINVAL"


def _write_msh(path, nodes, conn, gtype):
    with open(path, "w") as f:
        f.write("$MeshFormat\n2.1 0 8\n$EndMeshFormat\n$Nodes\n%d\n" % len(nodes))
        for i, x in enumerate(nodes):
            xyz = list(x) + [0.0] * (3 - len(x))
            f.write("%d %.17g %.17g %.17g\n" % (i + 1, *xyz))
        f.write("$EndNodes\n$Elements\n%d\n" % (len(conn) + 1))
        f.write("1 15 2 0 1 1\n")  # a point element, to be skipped
        for k, c in enumerate(conn):
            f.write("%d %d 2 7 1 %s\n" % (k + 2, gtype, " ".join(str(n + 1) for n in c)))
        f.write("$EndElements\n")


@pytest.mark.parametrize("etype,gtype", [("_tetrahedron_4", 4), ("_hexahedron_8", 5),
                                         ("_triangle_6", 9)])
def test_msh_reader_roundtrip(tmp_path, etype, gtype):
    g = golden(f"patch{etype}.npz")
    p = tmp_path / "m.msh"
    _write_msh(p, g["nodes"], g["conn"], gtype)
    mesh = akb.Mesh(g["nodes"].shape[1]).read(p)
    assert mesh.element_type == etype
    assert np.array_equal(mesh.nodes, g["nodes"])
    assert np.array_equal(mesh.connectivity, g["conn"])
    assert np.all(mesh.physical_tags == 7)


@pytest.mark.parametrize("gen,etype,n", [(akb.box_tet4, "_tetrahedron_4", 3),
                                         (akb.box_hex8, "_hexahedron_8", 3),
                                         (akb.square_tri6, "_triangle_6", 4)])
def test_generators_are_positively_oriented(gen, etype, n):
    mesh = gen(n)
    _, _, j, rc = orc.precompute(OR_TYPE[etype], mesh.nodes[mesh.connectivity])
    assert rc == 0 and np.all(j > 0)
    assert abs(j.sum() - 1.0) < 1e-14
    counts = {"_tetrahedron_4": 6 * n ** 3, "_hexahedron_8": n ** 3, "_triangle_6": 2 * n * n}
    assert mesh.getNbElement() == counts[etype]
    nb = {"_tetrahedron_4": (n + 1) ** 3 - (n - 1) ** 3, "_hexahedron_8": (n + 1) ** 3 - (n - 1) ** 3,
          "_triangle_6": (2 * n + 1) ** 2 - (2 * n - 1) ** 2}
    assert len(akb.boundary_nodes(etype, mesh.connectivity)) == nb[etype]


def test_boundary_of_reference_patch_meshes():
    for etype in TYPES:
        g = golden(f"patch{etype}.npz")
        b = akb.boundary_nodes(etype, g["conn"])
        x = g["nodes"]
        on_hull = np.any(np.isclose(x, x.min(0)) | np.isclose(x, x.max(0)), axis=1)
        assert set(b) == set(np.nonzero(on_hull)[0])


def test_both_library_builds_export_the_checked_entry_points():
    import ctypes
    import os
    here = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                        "akantu2_b200")
    for name, checked in (("libakb.so", 0), ("libakb_checked.so", 1)):
        L = ctypes.CDLL(os.path.join(here, name))
        assert L.akb_bounds_checked() == checked
        for sym in ("akb_model_debug_write_index", "akb_exchange_create",
                    "akb_batch_set_instance_steps", "akb_model_set_qp_field"):
            assert hasattr(L, sym), (name, sym)

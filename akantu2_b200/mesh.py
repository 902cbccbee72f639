"""Meshes for the explicit path: the Mesh container, the gmsh reader (through
libakb) and structured generators of positively oriented meshes.

Element node orders follow the reference element classes:
  _tetrahedron_4  src/fe_engine/element_classes/element_class_tetrahedron_4_inline_impl.hh
  _hexahedron_8   .../element_class_hexahedron_8_inline_impl.hh:21-41
  _triangle_6     .../element_class_triangle_6_inline_impl.hh:21-50
"""
import ctypes

import numpy as np

from . import _capi

_tetrahedron_4 = "_tetrahedron_4"
_hexahedron_8 = "_hexahedron_8"
_triangle_6 = "_triangle_6"

TYPE_IDS = {_tetrahedron_4: _capi.TETRAHEDRON_4, _hexahedron_8: _capi.HEXAHEDRON_8,
            _triangle_6: _capi.TRIANGLE_6}
NODES_PER_ELEMENT = {_tetrahedron_4: 4, _hexahedron_8: 8, _triangle_6: 6}
DIM = {_tetrahedron_4: 3, _hexahedron_8: 3, _triangle_6: 2}


class Mesh:
    """Nodes, one element type and named node groups (src/mesh/mesh.hh)."""

    def __init__(self, spatial_dimension, nodes=None, connectivity=None, element_type=None):
        self.spatial_dimension = spatial_dimension
        self.nodes = np.zeros((0, spatial_dimension))
        self.element_type = None
        self.connectivity = np.zeros((0, 0), dtype=np.int32)
        self.physical_tags = np.zeros(0, dtype=np.int32)
        self.node_groups = {}
        self.mesh_data = {}
        if nodes is not None:
            self.set(nodes, connectivity, element_type)

    def set(self, nodes, connectivity, element_type, physical_tags=None):
        if DIM[element_type] != self.spatial_dimension:
            raise ValueError("element type does not match the spatial dimension")
        self.nodes = np.ascontiguousarray(nodes, dtype=np.float64).reshape(-1, self.spatial_dimension)
        self.connectivity = np.ascontiguousarray(connectivity, dtype=np.int32).reshape(
            -1, NODES_PER_ELEMENT[element_type])
        self.element_type = element_type
        self.physical_tags = (np.zeros(len(self.connectivity), dtype=np.int32)
                              if physical_tags is None else np.asarray(physical_tags, np.int32))
        return self

    def read(self, path, element_type=None):
        """Mesh::read for gmsh 2.x and 4.x ASCII files (src/io/mesh_io/mesh_io_msh.cc);
        the file's physical groups become node groups (getNodeGroup)."""
        types = [element_type] if element_type else [t for t, d in DIM.items()
                                                     if d == self.spatial_dimension]
        L = _capi.lib()
        for t in types:
            h = ctypes.c_void_p()
            _capi.check(L.akb_mesh_read_msh(str(path).encode(), self.spatial_dimension,
                                            TYPE_IDS[t], ctypes.byref(h)))
            try:
                nn, ne, npe = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int()
                _capi.check(L.akb_mesh_sizes(h, ctypes.byref(nn), ctypes.byref(ne),
                                             ctypes.byref(npe)))
                if ne.value == 0 and len(types) > 1:
                    continue
                nodes = np.zeros((nn.value, self.spatial_dimension))
                conn = np.zeros((ne.value, npe.value), dtype=np.int32)
                tags = np.zeros(ne.value, dtype=np.int32)
                _capi.check(L.akb_mesh_copy(h, _capi.ptr(nodes), _capi.ptr(conn), _capi.ptr(tags)))
                ng = ctypes.c_int()
                _capi.check(L.akb_mesh_nb_groups(h, ctypes.byref(ng)))
                groups = {}
                for k in range(ng.value):
                    name = ctypes.create_string_buffer(256)
                    gdim, count = ctypes.c_int(), ctypes.c_int64()
                    _capi.check(L.akb_mesh_group(h, k, name, 256, ctypes.byref(gdim),
                                                 ctypes.byref(count), None))
                    members = np.zeros(count.value, dtype=np.int32)
                    _capi.check(L.akb_mesh_group(h, k, None, 0, None, None, _capi.ptr(members)))
                    groups[name.value.decode()] = members.astype(np.int64)
                nb_names = ctypes.c_int()
                _capi.check(L.akb_mesh_nb_element_names(h, ctypes.byref(nb_names)))
                names = None
                if nb_names.value >= 0:
                    table = []
                    for k in range(nb_names.value):
                        buf = ctypes.create_string_buffer(256)
                        _capi.check(L.akb_mesh_element_names(h, k, buf, 256, None))
                        table.append(buf.value.decode())
                    index = np.zeros(ne.value, dtype=np.int32)
                    _capi.check(L.akb_mesh_element_names(h, 0, None, 0, _capi.ptr(index)))
                    names = np.array(table, dtype=object)[index] if table else \
                        np.zeros(0, dtype=object)
            finally:
                L.akb_mesh_free(h)
            self.set(nodes, conn, t, tags)
            self.node_groups.update(groups)
            self.mesh_data = {"tag_0": self.physical_tags}
            if names is not None:
                self.mesh_data["physical_names"] = names
            return self
        raise ValueError(f"{path}: no element of a supported type")

    # -- akantu-style accessors ------------------------------------------------
    def getNodes(self):
        return self.nodes

    def getNbNodes(self):
        return self.nodes.shape[0]

    def getConnectivity(self, element_type=None):
        return self.connectivity

    def getNbElement(self, element_type=None):
        return self.connectivity.shape[0]

    def getSpatialDimension(self):
        return self.spatial_dimension

    def getLowerBounds(self):
        return self.nodes.min(axis=0)

    def getUpperBounds(self):
        return self.nodes.max(axis=0)

    def getData(self, name, element_type=None):
        """Element data read from the file (Mesh::getData): "tag_0", the first
        physical tag, and "physical_names", each element's physical name."""
        if name not in self.mesh_data:
            raise KeyError(f"the mesh has no element data '{name}'")
        return self.mesh_data[name]

    def createNodeGroup(self, name, nodes):
        self.node_groups[name] = np.unique(np.asarray(nodes, dtype=np.int64))
        return self.node_groups[name]

    def getNodeGroup(self, name):
        return self.node_groups[name]

    def createBoundaryGroupFromGeometry(self, name="boundary"):
        """Nodes of the facets that belong to a single element."""
        return self.createNodeGroup(name, boundary_nodes(self.element_type, self.connectivity))


# -- boundary facets -------------------------------------------------------------
_FACETS = {
    _tetrahedron_4: [(0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)],
    _hexahedron_8: [(0, 1, 2, 3), (4, 5, 6, 7), (0, 1, 5, 4), (1, 2, 6, 5), (2, 3, 7, 6),
                    (3, 0, 4, 7)],
    _triangle_6: [(0, 1, 3), (1, 2, 4), (2, 0, 5)],
}
# corner nodes that identify a facet (the mid-side node of _triangle_6 is not)
_FACET_KEY = {_tetrahedron_4: 3, _hexahedron_8: 4, _triangle_6: 2}


def boundary_nodes(element_type, conn):
    conn = np.asarray(conn)
    facets = np.concatenate([conn[:, list(f)] for f in _FACETS[element_type]], axis=0)
    key = np.sort(facets[:, :_FACET_KEY[element_type]], axis=1)
    _, inv, counts = np.unique(key, axis=0, return_inverse=True, return_counts=True)
    on_boundary = counts[inv.ravel()] == 1
    return np.unique(facets[on_boundary].ravel())


# -- structured generators -------------------------------------------------------
def box_tet4(nx, ny=None, nz=None, lengths=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0)):
    """Box of nx*ny*nz cells, each split into 6 Kuhn tetrahedra (shared main
    diagonal), positively oriented; nodes lexicographic with x fastest."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    xs = origin[0] + lengths[0] * np.arange(nx + 1) / nx
    ys = origin[1] + lengths[1] * np.arange(ny + 1) / ny
    zs = origin[2] + lengths[2] * np.arange(nz + 1) / nz
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    nodes = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    base = (i + (nx + 1) * (j + (ny + 1) * k)).ravel()
    step = np.array([1, nx + 1, (nx + 1) * (ny + 1)])
    tets = []
    for perm, odd in (((0, 1, 2), False), ((1, 2, 0), False), ((2, 0, 1), False),
                      ((0, 2, 1), True), ((2, 1, 0), True), ((1, 0, 2), True)):
        v0 = base
        v1 = v0 + step[perm[0]]
        v2 = v1 + step[perm[1]]
        v3 = v2 + step[perm[2]]
        tets.append(np.stack([v0, v2, v1, v3] if odd else [v0, v1, v2, v3], axis=1))
    conn = np.stack(tets, axis=1).reshape(-1, 4).astype(np.int32)
    return Mesh(3, nodes, conn, _tetrahedron_4)


def box_hex8(nx, ny=None, nz=None, lengths=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0)):
    """Box of nx*ny*nz hexahedra, nodes lexicographic with x fastest."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    xs = origin[0] + lengths[0] * np.arange(nx + 1) / nx
    ys = origin[1] + lengths[1] * np.arange(ny + 1) / ny
    zs = origin[2] + lengths[2] * np.arange(nz + 1) / nz
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    nodes = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    n0 = (i + (nx + 1) * (j + (ny + 1) * k)).ravel()
    sx, sy = 1, nx + 1
    sz = (nx + 1) * (ny + 1)
    conn = np.stack([n0, n0 + sx, n0 + sx + sy, n0 + sy,
                     n0 + sz, n0 + sz + sx, n0 + sz + sx + sy, n0 + sz + sy], axis=1)
    return Mesh(3, nodes, conn.astype(np.int32), _hexahedron_8)


def square_tri6(nx, ny=None, lengths=(1.0, 1.0), origin=(0.0, 0.0)):
    """nx*ny cells split along the (0,0)-(1,1) diagonal into two quadratic
    triangles; nodes on the (2nx+1) x (2ny+1) grid, x fastest."""
    ny = nx if ny is None else ny
    mx, my = 2 * nx + 1, 2 * ny + 1
    xs = origin[0] + lengths[0] * np.arange(mx) / (2 * nx)
    ys = origin[1] + lengths[1] * np.arange(my) / (2 * ny)
    Y, X = np.meshgrid(ys, xs, indexing="ij")
    nodes = np.stack([X.ravel(), Y.ravel()], axis=1)
    j, i = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    g = lambda a, b: ((2 * j + b) * mx + (2 * i + a)).ravel()
    A, B, C, D = g(0, 0), g(2, 0), g(2, 2), g(0, 2)
    t1 = np.stack([A, B, C, g(1, 0), g(2, 1), g(1, 1)], axis=1)
    t2 = np.stack([A, C, D, g(1, 1), g(1, 2), g(0, 1)], axis=1)
    conn = np.stack([t1, t2], axis=1).reshape(-1, 6).astype(np.int32)
    return Mesh(2, nodes, conn, _triangle_6)


# -- seeded initial fields --------------------------------------------------------
def gaussian_random_field(nodes, seed, corr_length=0.1, std=0.02):
    """Smooth random vector field on the nodes of a structured grid: seeded
    white noise per component, filtered in Fourier space by a Gaussian of the
    given correlation length, rescaled to the given standard deviation."""
    rng = np.random.default_rng(seed)
    d = nodes.shape[1]
    lo, hi = nodes.min(0), nodes.max(0)
    shape = [len(np.unique(nodes[:, k])) for k in range(d)]
    if int(np.prod(shape)) != nodes.shape[0]:
        raise ValueError("gaussian_random_field needs a structured node grid")
    dims = shape[::-1]  # nodes are x-fastest: array index order (z, y, x)
    freqs = np.meshgrid(*[np.fft.fftfreq(n, d=(hi[k] - lo[k]) / max(n - 1, 1))
                          for k, n in zip(reversed(range(d)), dims)], indexing="ij")
    k2 = sum(f ** 2 for f in freqs)
    filt = np.exp(-0.5 * (2 * np.pi) ** 2 * k2 * corr_length ** 2)
    v = np.zeros_like(nodes)
    for c in range(d):
        noise = rng.standard_normal(dims)
        field = np.real(np.fft.ifftn(np.fft.fftn(noise) * filt))
        v[:, c] = (field / (field.std() + 1e-300) * std).ravel()
    return v

// gmsh 2.x ASCII reader for the explicit path (src/io/mesh_io/mesh_io_msh.cc).
// Keeps the nodes in file order and the elements of one akantu type, in order
// of appearance, with their first (physical) tag.  _tetrahedron_4,
// _hexahedron_8 and _triangle_6 use gmsh's node order unchanged
// (mesh_io_msh.cc:211-263 permutes only higher-order types).
#include <cstdint>
#include <fstream>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "akb_capi.h"
#include "host_common.h"

struct akb_mesh {
  int dim = 0, nn = 0;
  std::vector<double> nodes;
  std::vector<int32_t> conn;
  std::vector<int32_t> tag;
};

namespace {
// gmsh element type ids
int gmsh_type_of(int et) {
  switch (et) {
  case AKB_TETRAHEDRON_4: return 4;
  case AKB_HEXAHEDRON_8: return 5;
  case AKB_TRIANGLE_6: return 9;
  default: return -1;
  }
}
int nodes_of(int et) { return et == AKB_TETRAHEDRON_4 ? 4 : (et == AKB_HEXAHEDRON_8 ? 8 : 6); }
}  // namespace

extern "C" int akb_mesh_read_msh(const char *path, int dim, int et, akb_mesh **out) {
  if (!path || !out) return akb::fail(AKB_EINVAL, "null argument");
  const int gt = gmsh_type_of(et);
  if (gt < 0) return akb::fail(AKB_EINVAL, "unsupported element type");
  if ((et == AKB_TRIANGLE_6 && dim != 2) || (et != AKB_TRIANGLE_6 && dim != 3))
    return akb::fail(AKB_EINVAL, "spatial dimension does not match the element type");
  std::ifstream f(path);
  if (!f) return akb::fail(AKB_EIO, std::string("cannot open ") + path);
  auto *m = new akb_mesh();
  m->dim = dim;
  m->nn = nodes_of(et);
  std::unordered_map<long, int32_t> id2idx;
  std::string line;
  bool have_format = false;
  while (std::getline(f, line)) {
    if (line.rfind("$MeshFormat", 0) == 0) {
      double version = 0;
      int file_type = 0, data_size = 0;
      f >> version >> file_type >> data_size;
      if (version < 2.0 || version >= 3.0 || file_type != 0) {
        delete m;
        return akb::fail(AKB_EUNSUPPORTED, "only gmsh 2.x ASCII files are read");
      }
      have_format = true;
    } else if (line.rfind("$Nodes", 0) == 0) {
      long n = 0;
      f >> n;
      m->nodes.resize((size_t)n * dim);
      for (long i = 0; i < n; ++i) {
        long id;
        double x[3];
        if (!(f >> id >> x[0] >> x[1] >> x[2])) {
          delete m;
          return akb::fail(AKB_EPARSE, "truncated $Nodes block");
        }
        id2idx[id] = (int32_t)i;
        for (int c = 0; c < dim; ++c) m->nodes[(size_t)i * dim + c] = x[c];
      }
    } else if (line.rfind("$Elements", 0) == 0) {
      long n = 0;
      f >> n;
      std::getline(f, line);
      for (long i = 0; i < n; ++i) {
        if (!std::getline(f, line)) {
          delete m;
          return akb::fail(AKB_EPARSE, "truncated $Elements block");
        }
        std::istringstream ls(line);
        long id;
        int type, ntags;
        ls >> id >> type >> ntags;
        std::vector<long> tags(ntags);
        for (int t = 0; t < ntags; ++t) ls >> tags[t];
        if (type != gt) continue;
        for (int a = 0; a < m->nn; ++a) {
          long nid;
          if (!(ls >> nid) || !id2idx.count(nid)) {
            delete m;
            return akb::fail(AKB_EPARSE, "element refers to an unknown node");
          }
          m->conn.push_back(id2idx[nid]);
        }
        m->tag.push_back(ntags > 0 ? (int32_t)tags[0] : 0);
      }
    }
  }
  if (!have_format) {
    delete m;
    return akb::fail(AKB_EPARSE, "missing $MeshFormat");
  }
  *out = m;
  return AKB_OK;
}

extern "C" int akb_mesh_sizes(const akb_mesh *m, int64_t *nb_nodes, int64_t *nb_elements,
                              int *npe) {
  if (!m) return akb::fail(AKB_EINVAL, "null mesh");
  if (nb_nodes) *nb_nodes = (int64_t)(m->nodes.size() / m->dim);
  if (nb_elements) *nb_elements = (int64_t)m->tag.size();
  if (npe) *npe = m->nn;
  return AKB_OK;
}

extern "C" int akb_mesh_copy(const akb_mesh *m, double *nodes, int32_t *conn, int32_t *tag) {
  if (!m) return akb::fail(AKB_EINVAL, "null mesh");
  if (nodes) std::copy(m->nodes.begin(), m->nodes.end(), nodes);
  if (conn) std::copy(m->conn.begin(), m->conn.end(), conn);
  if (tag) std::copy(m->tag.begin(), m->tag.end(), tag);
  return AKB_OK;
}

extern "C" void akb_mesh_free(akb_mesh *m) { delete m; }

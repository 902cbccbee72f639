// gmsh ASCII reader for the explicit path (src/io/mesh_io/mesh_io_msh.cc):
// formats 2.x and 4.0 / 4.1 (the two families the reference reads, its
// populateReaders2 / populateReaders4).  Keeps the nodes in file order and the
// elements of one akantu type, in order of appearance, with their first
// physical tag (the reference's "tag_0" data).  Physical groups become node
// groups (the nodes of the reference's element groups), following the
// reference's rules for each format:
//   2.x  only when the file has $PhysicalNames (mesh_io_msh.cc:913-916); every
//        element of any type joins the group of its first tag, named by
//        $PhysicalNames or by the tag's decimal number (mesh_io.cc:89-113);
//   4.x  every physical tag of an entity creates a group, named by
//        $PhysicalNames or "msh_block_<tag>" (mesh_io_msh.cc:507-521), and an
//        element joins only the groups whose tag has a name (:669-681), so
//        the "msh_block_" groups stay empty.
// _tetrahedron_4, _hexahedron_8 and _triangle_6 use gmsh's node order
// unchanged (mesh_io_msh.cc:211-263 permutes only higher-order types).
#include <algorithm>
#include <cstdint>
#include <fstream>
#include <map>
#include <set>
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
  // physical groups: name -> (dimension, node indices)
  std::map<std::string, std::pair<int, std::set<int32_t>>> groups;
  // the "physical_names" element data of the read type: distinct names, and
  // each element's index into them; absent (has_names false) for a format 2
  // file without $PhysicalNames, as in the reference
  bool has_names = false;
  std::vector<std::string> names;
  std::vector<int32_t> name_of;
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

// dimension of a gmsh element type (for groups of elements whose entity
// dimension the file does not give, format 2)
int dim_of_gmsh(int type) {
  switch (type) {
  case 15: return 0;                                        // point
  case 1: case 8: case 26: case 27: case 28: return 1;      // lines
  case 2: case 3: case 9: case 10: case 16: case 20: case 21: case 22: case 23: case 24:
  case 25: return 2;                                        // triangles, quadrangles
  default: return 3;
  }
}

struct Reader {
  akb_mesh *m;
  int gt;
  int version = 0;  // 2000 + minor, 4000 + minor
  std::unordered_map<long, int32_t> id2idx;
  std::map<int, std::string> names;          // physical tag -> name
  std::map<std::pair<int, int>, std::vector<int>> entity_phys;  // (dim, entity) -> tags

  // format 4: the group of one entity physical tag, created empty
  void declare_group(int phys, int dim) {
    auto it = names.find(phys);
    auto &g = m->groups[it != names.end() ? it->second : "msh_block_" + std::to_string(phys)];
    g.first = std::max(g.first, dim);
  }
  // one element: its nodes (file ids), physical tags and type
  int element(int type, int dim, const std::vector<int> &phys, const std::vector<long> &ids) {
    std::vector<int32_t> idx(ids.size());
    for (size_t k = 0; k < ids.size(); ++k) {
      auto it = id2idx.find(ids[k]);
      if (it == id2idx.end()) return akb::fail(AKB_EPARSE, "element refers to an unknown node");
      idx[k] = it->second;
    }
    for (int p : phys) {
      auto it = names.find(p);
      std::string name;
      if (it != names.end())
        name = it->second;
      else if (version < 4000 && !names.empty())
        name = std::to_string(p);
      else
        continue;
      auto &g = m->groups[name];
      g.first = std::max(g.first, dim);
      g.second.insert(idx.begin(), idx.end());
    }
    if (type == gt) {
      if ((int)idx.size() != m->nn) return akb::fail(AKB_EPARSE, "wrong number of element nodes");
      m->conn.insert(m->conn.end(), idx.begin(), idx.end());
      const int first = phys.empty() ? 0 : phys[0];
      m->tag.push_back(first);
      // the element's physical name: format 2 names every tag, unnamed ones
      // by their number (mesh_io.cc:97-110); format 4 names an element only
      // when its entity's first tag has a name (mesh_io_msh.cc:669-676)
      auto it = names.find(first);
      std::string name;
      if (it != names.end() && !phys.empty())
        name = it->second;
      else if (version < 4000)
        name = std::to_string(first);
      auto pos = std::find(m->names.begin(), m->names.end(), name);
      m->name_of.push_back((int32_t)(pos - m->names.begin()));
      if (pos == m->names.end()) m->names.push_back(name);
    }
    return AKB_OK;
  }
};

bool next_line(std::ifstream &f, std::istringstream &ls) {
  std::string line;
  if (!std::getline(f, line)) return false;
  ls.clear();
  ls.str(line);
  return true;
}
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
  Reader rd{m, gt};
  auto bail = [&](int code, const std::string &msg) {
    delete m;
    return akb::fail(code, msg);
  };
  std::string line;
  std::istringstream ls;
  int &version = rd.version;
  while (std::getline(f, line)) {
    if (line.rfind("$MeshFormat", 0) == 0) {
      double v = 0;
      int file_type = 0;
      if (!next_line(f, ls) || !(ls >> v >> file_type)) return bail(AKB_EPARSE, "bad $MeshFormat");
      if (file_type != 0) return bail(AKB_EUNSUPPORTED, "only ASCII gmsh files are read");
      const int major = (int)v, minor = (int)(10 * (v - major) + 0.5);
      if (major != 2 && major != 4) return bail(AKB_EUNSUPPORTED, "gmsh format 2.x or 4.x only");
      version = major * 1000 + minor;
    } else if (line.rfind("$PhysicalNames", 0) == 0) {
      long n = 0;
      if (!next_line(f, ls) || !(ls >> n)) return bail(AKB_EPARSE, "bad $PhysicalNames");
      for (long i = 0; i < n; ++i) {
        int pdim = 0, tag = 0;
        if (!next_line(f, ls) || !(ls >> pdim >> tag)) return bail(AKB_EPARSE, "bad physical name");
        std::string rest;
        std::getline(ls, rest);
        const auto a = rest.find('"'), b = rest.rfind('"');
        rd.names[tag] = (a != std::string::npos && b > a) ? rest.substr(a + 1, b - a - 1) : rest;
      }
    } else if (line.rfind("$Entities", 0) == 0) {
      long num[4] = {0, 0, 0, 0};
      if (!next_line(f, ls) || !(ls >> num[0] >> num[1] >> num[2] >> num[3]))
        return bail(AKB_EPARSE, "bad $Entities");
      for (int edim = 0; edim < 4; ++edim)
        for (long i = 0; i < num[edim]; ++i) {
          int tag = 0;
          double box[6];
          if (!next_line(f, ls) || !(ls >> tag)) return bail(AKB_EPARSE, "bad entity");
          // points of format 4.1 give one position, other entities a box
          const int nb = (edim == 0 && version >= 4001) ? 3 : 6;
          for (int k = 0; k < nb; ++k) ls >> box[k];
          long np = 0;
          ls >> np;
          std::vector<int> &phys = rd.entity_phys[{edim, tag}];
          for (long k = 0; k < np; ++k) {
            int p = 0;
            ls >> p;
            phys.push_back(p);
            rd.declare_group(p, edim);
          }
        }
    } else if (line.rfind("$Nodes", 0) == 0) {
      if (version == 0) return bail(AKB_EPARSE, "missing $MeshFormat");
      if (version < 4000) {
        long n = 0;
        if (!next_line(f, ls) || !(ls >> n)) return bail(AKB_EPARSE, "bad $Nodes");
        m->nodes.resize((size_t)n * dim);
        for (long i = 0; i < n; ++i) {
          long id;
          double x[3];
          if (!next_line(f, ls) || !(ls >> id >> x[0] >> x[1] >> x[2]))
            return bail(AKB_EPARSE, "truncated $Nodes block");
          rd.id2idx[id] = (int32_t)i;
          for (int c = 0; c < dim; ++c) m->nodes[(size_t)i * dim + c] = x[c];
        }
      } else {
        long blocks = 0, n = 0;
        if (!next_line(f, ls) || !(ls >> blocks >> n)) return bail(AKB_EPARSE, "bad $Nodes");
        m->nodes.resize((size_t)n * dim);
        long idx = 0;
        for (long b = 0; b < blocks; ++b) {
          long a0 = 0, a1 = 0, param = 0, count = 0;
          if (!next_line(f, ls) || !(ls >> a0 >> a1 >> param >> count))
            return bail(AKB_EPARSE, "bad node block");
          if (param != 0) return bail(AKB_EUNSUPPORTED, "parametric nodes are not read");
          std::vector<long> ids((size_t)count);
          if (version >= 4001) {  // the block's tags, then its coordinates
            for (long k = 0; k < count; ++k)
              if (!next_line(f, ls) || !(ls >> ids[k])) return bail(AKB_EPARSE, "bad node tag");
          }
          for (long k = 0; k < count; ++k) {
            double x[3];
            if (!next_line(f, ls)) return bail(AKB_EPARSE, "truncated $Nodes block");
            if (version < 4001) ls >> ids[k];
            if (!(ls >> x[0] >> x[1] >> x[2])) return bail(AKB_EPARSE, "bad node coordinates");
            if (idx >= n) return bail(AKB_EPARSE, "more nodes than announced");
            rd.id2idx[ids[k]] = (int32_t)idx;
            for (int c = 0; c < dim; ++c) m->nodes[(size_t)idx * dim + c] = x[c];
            ++idx;
          }
        }
      }
    } else if (line.rfind("$Elements", 0) == 0) {
      if (version == 0) return bail(AKB_EPARSE, "missing $MeshFormat");
      if (version < 4000) {
        long n = 0;
        if (!next_line(f, ls) || !(ls >> n)) return bail(AKB_EPARSE, "bad $Elements");
        for (long i = 0; i < n; ++i) {
          long id;
          int type, ntags;
          if (!next_line(f, ls) || !(ls >> id >> type >> ntags))
            return bail(AKB_EPARSE, "truncated $Elements block");
          std::vector<long> tags(ntags);
          for (int t = 0; t < ntags; ++t) ls >> tags[t];
          std::vector<int> phys;
          if (ntags > 0) phys.push_back((int)tags[0]);
          std::vector<long> ids;
          long nid;
          while (ls >> nid) ids.push_back(nid);
          const int rc = rd.element(type, dim_of_gmsh(type), phys, ids);
          if (rc != AKB_OK) {
            delete m;
            return rc;
          }
        }
      } else {
        long blocks = 0, n = 0;
        if (!next_line(f, ls) || !(ls >> blocks >> n)) return bail(AKB_EPARSE, "bad $Elements");
        for (long b = 0; b < blocks; ++b) {
          long a0 = 0, a1 = 0, type = 0, count = 0;
          if (!next_line(f, ls) || !(ls >> a0 >> a1 >> type >> count))
            return bail(AKB_EPARSE, "bad element block");
          // format 4.1: entity dimension, entity tag; 4.0: tag, dimension
          const int edim = (int)(version >= 4001 ? a0 : a1);
          const int etag = (int)(version >= 4001 ? a1 : a0);
          auto it = rd.entity_phys.find({edim, etag});
          const std::vector<int> phys = it != rd.entity_phys.end() ? it->second : std::vector<int>{};
          for (long k = 0; k < count; ++k) {
            long id;
            if (!next_line(f, ls) || !(ls >> id)) return bail(AKB_EPARSE, "truncated element block");
            std::vector<long> ids;
            long nid;
            while (ls >> nid) ids.push_back(nid);
            const int rc = rd.element((int)type, edim, phys, ids);
            if (rc != AKB_OK) {
              delete m;
              return rc;
            }
          }
        }
      }
    }
  }
  if (version == 0) return bail(AKB_EPARSE, "missing $MeshFormat");
  m->has_names = version >= 4000 || !rd.names.empty();
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

extern "C" int akb_mesh_nb_groups(const akb_mesh *m, int *count) {
  if (!m || !count) return akb::fail(AKB_EINVAL, "null argument");
  *count = (int)m->groups.size();
  return AKB_OK;
}

extern "C" int akb_mesh_group(const akb_mesh *m, int k, char *name, size_t name_size, int *dim,
                              int64_t *nb_nodes, int32_t *nodes) {
  if (!m) return akb::fail(AKB_EINVAL, "null mesh");
  if (k < 0 || k >= (int)m->groups.size()) return akb::fail(AKB_EINVAL, "group index out of range");
  auto it = m->groups.begin();
  std::advance(it, k);
  if (name && name_size > 0) {
    const size_t n = std::min(name_size - 1, it->first.size());
    std::copy(it->first.begin(), it->first.begin() + n, name);
    name[n] = '\0';
  }
  if (dim) *dim = it->second.first;
  if (nb_nodes) *nb_nodes = (int64_t)it->second.second.size();
  if (nodes) std::copy(it->second.second.begin(), it->second.second.end(), nodes);
  return AKB_OK;
}

extern "C" int akb_mesh_nb_element_names(const akb_mesh *m, int *count) {
  if (!m || !count) return akb::fail(AKB_EINVAL, "null argument");
  *count = m->has_names ? (int)m->names.size() : -1;
  return AKB_OK;
}

extern "C" int akb_mesh_element_names(const akb_mesh *m, int k, char *name, size_t name_size,
                                      int32_t *name_of_element) {
  if (!m) return akb::fail(AKB_EINVAL, "null mesh");
  if (!m->has_names) return akb::fail(AKB_EINVAL, "the file gives no physical names");
  if (name && name_size > 0) {
    if (k < 0 || k >= (int)m->names.size()) return akb::fail(AKB_EINVAL, "name index out of range");
    const std::string &s = m->names[k];
    const size_t n = std::min(name_size - 1, s.size());
    std::copy(s.begin(), s.begin() + n, name);
    name[n] = '\0';
  }
  if (name_of_element) std::copy(m->name_of.begin(), m->name_of.end(), name_of_element);
  return AKB_OK;
}

extern "C" void akb_mesh_free(akb_mesh *m) { delete m; }

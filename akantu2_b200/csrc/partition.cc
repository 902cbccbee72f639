// Partition of one mesh across ranks (one GPU each) for the explicit step.
//
// The reference distributes a mesh with a graph partitioner
// (src/mesh_utils/mesh_partition/mesh_partition_scotch.cc) and keeps, on each
// process, its local elements plus a layer of ghost elements whose stresses
// arrive from their owner every step (SynchronizationTag::_smm_stress,
// solid_mechanics_model.cc:333-370; element_synchronizer.cc).  Here:
//
//  - elements are split by recursive coordinate bisection of their centroids
//    (akb_partition_elements): balanced counts, deterministic, no library;
//  - node n is owned by the lowest part among its elements; rank r keeps
//    every element that has a node it owns (its own elements and the ghost
//    layer, evaluated redundantly), and every node of those elements;
//  - each owned node therefore has all of its elements locally, in global
//    order, so its internal force is the sum of the same slots in the same
//    order as on one GPU: a partitioned run is bit-identical to the serial
//    run.  Ghost nodes (owned elsewhere) are blocked locally and receive the
//    owner's predicted displacement after every step: one exchange per step,
//    owned node -> every rank that holds it as a ghost.
//
// Every rank builds its own subdomain from the whole mesh with the same
// deterministic rules, so the send list of r -> s and the receive list of
// s <- r are the same global nodes in the same (ascending) order without any
// message.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <numeric>
#include <set>
#include <vector>

#include "akb_capi.h"
#include "host_common.h"

using namespace akb;

namespace {

int nodes_per(int et) {
  return et == AKB_TETRAHEDRON_4 ? 4 : (et == AKB_HEXAHEDRON_8 ? 8 : 6);
}
int dim_of_type(int et) { return et == AKB_TRIANGLE_6 ? 2 : 3; }

// elements [lo, hi) of order, split into nparts parts starting at part0
void bisect(std::vector<int64_t> &order, int64_t lo, int64_t hi, int part0, int nparts,
            const std::vector<double> &cen, int d, int32_t *part) {
  if (nparts == 1 || hi - lo <= 1) {
    for (int64_t k = lo; k < hi; ++k) part[order[k]] = part0;
    return;
  }
  // the axis of the largest centroid extent
  int axis = 0;
  double best = -1.;
  for (int j = 0; j < d; ++j) {
    double mn = INFINITY, mx = -INFINITY;
    for (int64_t k = lo; k < hi; ++k) {
      const double c = cen[order[k] * d + j];
      mn = std::min(mn, c);
      mx = std::max(mx, c);
    }
    if (mx - mn > best) {
      best = mx - mn;
      axis = j;
    }
  }
  const int left = nparts / 2;
  const int64_t mid = lo + (hi - lo) * left / nparts;
  // ties broken by element id: the split is deterministic
  auto less = [&](int64_t a, int64_t b) {
    const double ca = cen[a * d + axis], cb = cen[b * d + axis];
    return ca < cb || (ca == cb && a < b);
  };
  std::nth_element(order.begin() + lo, order.begin() + mid, order.begin() + hi, less);
  bisect(order, lo, mid, part0, left, cen, d, part);
  bisect(order, mid, hi, part0 + left, nparts - left, cen, d, part);
}

}  // namespace

extern "C" int akb_partition_elements(int et, const double *nodes, int64_t N,
                                      const int32_t *conn, int64_t E, int nparts,
                                      int32_t *part) {
  if (et < AKB_TETRAHEDRON_4 || et > AKB_TRIANGLE_6) return fail(AKB_EINVAL, "unknown element type");
  if (nparts < 1) return fail(AKB_EINVAL, "nparts must be >= 1");
  if (N < 0 || E < 0 || (E > 0 && (!nodes || !conn || !part)))
    return fail(AKB_EINVAL, "bad arguments");
  const int nn = nodes_per(et), d = dim_of_type(et);
  std::vector<double> cen((size_t)E * d, 0.);
  for (int64_t e = 0; e < E; ++e)
    for (int a = 0; a < nn; ++a) {
      const int32_t n = conn[e * nn + a];
      if (n < 0 || n >= N) return fail(AKB_EINVAL, "connectivity refers to a missing node");
      for (int j = 0; j < d; ++j) cen[e * d + j] += nodes[(int64_t)n * d + j] / nn;
    }
  std::vector<int64_t> order(E);
  std::iota(order.begin(), order.end(), 0);
  bisect(order, 0, E, 0, nparts, cen, d, part);
  return AKB_OK;
}

struct akb_subdomain {
  int rank = 0, nparts = 1, d = 3, nn = 4;
  std::vector<int64_t> node_global;  // local node -> global: owned (ascending), then ghosts
  int64_t n_owned = 0;
  std::vector<int64_t> elem_global;  // local element -> global, ascending
  std::vector<double> nodes;         // [n_local][d]
  std::vector<int32_t> conn;         // [e_local][nn], local node ids
  std::vector<int> neighbors;        // ranks exchanged with, ascending
  std::vector<std::vector<int32_t>> send, recv;  // local node ids, by ascending global id
};

extern "C" int akb_subdomain_create(int et, const double *nodes, int64_t N, const int32_t *conn,
                                    int64_t E, const int32_t *part, int nparts, int rank,
                                    akb_subdomain **out) {
  if (!out) return fail(AKB_EINVAL, "null argument");
  *out = nullptr;
  if (et < AKB_TETRAHEDRON_4 || et > AKB_TRIANGLE_6) return fail(AKB_EINVAL, "unknown element type");
  if (nparts < 1 || rank < 0 || rank >= nparts) return fail(AKB_EINVAL, "bad rank or nparts");
  if (N < 0 || E < 0 || (E > 0 && (!nodes || !conn || !part)))
    return fail(AKB_EINVAL, "bad arguments");
  const int nn = nodes_per(et), d = dim_of_type(et);
  for (int64_t e = 0; e < E; ++e) {
    if (part[e] < 0 || part[e] >= nparts) return fail(AKB_EINVAL, "part out of range");
    for (int a = 0; a < nn; ++a)
      if (conn[e * nn + a] < 0 || conn[e * nn + a] >= N)
        return fail(AKB_EINVAL, "connectivity refers to a missing node");
  }
  // owner of each node: the lowest part among its elements (nodes of no
  // element belong to rank 0, which keeps them as isolated nodes)
  std::vector<int32_t> owner(N, nparts);
  for (int64_t e = 0; e < E; ++e)
    for (int a = 0; a < nn; ++a) {
      int32_t &o = owner[conn[e * nn + a]];
      o = std::min(o, part[e]);
    }
  for (auto &o : owner)
    if (o == nparts) o = 0;
  auto sd = new akb_subdomain;
  sd->rank = rank;
  sd->nparts = nparts;
  sd->d = d;
  sd->nn = nn;
  // ranks holding each element: the owners of its nodes.  Element e is local
  // to rank r if r owns one of its nodes; every node of e is then local to r,
  // and a ghost there unless r owns it: (owner -> r) pairs to exchange.
  std::vector<uint8_t> local_node(N, 0);
  std::map<int, std::set<int64_t>> send_g, recv_g;  // global node ids
  int holders[8];
  for (int64_t e = 0; e < E; ++e) {
    int nh = 0;
    for (int a = 0; a < nn; ++a) {
      const int o = owner[conn[e * nn + a]];
      bool seen = false;
      for (int k = 0; k < nh; ++k) seen |= holders[k] == o;
      if (!seen) holders[nh++] = o;
    }
    bool mine = false;
    for (int k = 0; k < nh; ++k) mine |= holders[k] == rank;
    if (mine) {
      sd->elem_global.push_back(e);
      for (int a = 0; a < nn; ++a) {
        const int32_t n = conn[e * nn + a];
        local_node[n] = 1;
        if (owner[n] != rank) recv_g[owner[n]].insert(n);
      }
    }
    // nodes this rank owns that are ghosts of another holder of e
    for (int k = 0; k < nh; ++k) {
      const int r = holders[k];
      if (r == rank) continue;
      for (int a = 0; a < nn; ++a) {
        const int32_t n = conn[e * nn + a];
        if (owner[n] == rank) send_g[r].insert(n);
      }
    }
  }
  for (int64_t n = 0; n < N; ++n)
    if (owner[n] == rank && !local_node[n]) local_node[n] = 1;  // isolated owned nodes
  for (int64_t n = 0; n < N; ++n)
    if (local_node[n] && owner[n] == rank) sd->node_global.push_back(n);
  sd->n_owned = (int64_t)sd->node_global.size();
  for (int64_t n = 0; n < N; ++n)
    if (local_node[n] && owner[n] != rank) sd->node_global.push_back(n);
  std::vector<int32_t> g2l(N, -1);
  for (size_t k = 0; k < sd->node_global.size(); ++k) g2l[sd->node_global[k]] = (int32_t)k;
  sd->nodes.resize(sd->node_global.size() * d);
  for (size_t k = 0; k < sd->node_global.size(); ++k)
    for (int j = 0; j < d; ++j) sd->nodes[k * d + j] = nodes[sd->node_global[k] * d + j];
  sd->conn.resize(sd->elem_global.size() * nn);
  for (size_t k = 0; k < sd->elem_global.size(); ++k)
    for (int a = 0; a < nn; ++a) sd->conn[k * nn + a] = g2l[conn[sd->elem_global[k] * nn + a]];
  std::set<int> nb;
  for (auto &x : send_g) nb.insert(x.first);
  for (auto &x : recv_g) nb.insert(x.first);
  for (int r : nb) {
    sd->neighbors.push_back(r);
    std::vector<int32_t> s, q;
    for (int64_t n : send_g[r]) s.push_back(g2l[n]);
    for (int64_t n : recv_g[r]) q.push_back(g2l[n]);
    sd->send.push_back(std::move(s));
    sd->recv.push_back(std::move(q));
  }
  *out = sd;
  return AKB_OK;
}

extern "C" int akb_subdomain_sizes(const akb_subdomain *sd, int64_t *n_local, int64_t *n_owned,
                                   int64_t *e_local, int *n_neighbors) {
  if (!sd || !n_local || !n_owned || !e_local || !n_neighbors)
    return fail(AKB_EINVAL, "null argument");
  *n_local = (int64_t)sd->node_global.size();
  *n_owned = sd->n_owned;
  *e_local = (int64_t)sd->elem_global.size();
  *n_neighbors = (int)sd->neighbors.size();
  return AKB_OK;
}

extern "C" int akb_subdomain_mesh(const akb_subdomain *sd, double *nodes, int32_t *conn,
                                  int64_t *node_global, int64_t *elem_global) {
  if (!sd) return fail(AKB_EINVAL, "null subdomain");
  if (nodes) std::memcpy(nodes, sd->nodes.data(), sizeof(double) * sd->nodes.size());
  if (conn) std::memcpy(conn, sd->conn.data(), sizeof(int32_t) * sd->conn.size());
  if (node_global)
    std::memcpy(node_global, sd->node_global.data(), sizeof(int64_t) * sd->node_global.size());
  if (elem_global)
    std::memcpy(elem_global, sd->elem_global.data(), sizeof(int64_t) * sd->elem_global.size());
  return AKB_OK;
}

extern "C" int akb_subdomain_neighbor(const akb_subdomain *sd, int k, int *rank, int64_t *n_send,
                                      int64_t *n_recv) {
  if (!sd || !rank || !n_send || !n_recv) return fail(AKB_EINVAL, "null argument");
  if (k < 0 || k >= (int)sd->neighbors.size()) return fail(AKB_EINVAL, "neighbor index out of range");
  *rank = sd->neighbors[k];
  *n_send = (int64_t)sd->send[k].size();
  *n_recv = (int64_t)sd->recv[k].size();
  return AKB_OK;
}

extern "C" int akb_subdomain_lists(const akb_subdomain *sd, int k, int32_t *send_local,
                                   int32_t *recv_local) {
  if (!sd) return fail(AKB_EINVAL, "null subdomain");
  if (k < 0 || k >= (int)sd->neighbors.size()) return fail(AKB_EINVAL, "neighbor index out of range");
  if (send_local) std::memcpy(send_local, sd->send[k].data(), sizeof(int32_t) * sd->send[k].size());
  if (recv_local) std::memcpy(recv_local, sd->recv[k].data(), sizeof(int32_t) * sd->recv[k].size());
  return AKB_OK;
}

extern "C" void akb_subdomain_destroy(akb_subdomain *sd) { delete sd; }

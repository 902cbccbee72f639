// Neumann boundary condition from a stress tensor (BC::Neumann::FromHigherDim,
// boundary_condition_functor.hh; applied by boundary_condition_tmpl.hh:100-164):
// on every boundary facet whose nodes all belong to the group, the traction
// t = sigma n (n the outward unit normal) is integrated against the facet's
// shape functions and added to the external force.  Facets: the triangles of
// _tetrahedron_4 (_triangle_3, 1 point), the quadrangles of _hexahedron_8
// (_quadrangle_4, 2 x 2 points) and the edges of _triangle_6 (_segment_3,
// 2 points); the facet rules integrate the constant-traction loads exactly.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "akb_capi.h"
#include "host_common.h"

using namespace akb;

namespace {

struct FacetType {
  int nf;                  // facets per element
  int nn;                  // nodes per facet
  int corners;             // corner nodes (the rest are mid-side)
  std::vector<std::array<int, 4>> local;  // local node ids of each facet
};

const FacetType &facets_of(int et) {
  static const FacetType tet{4, 3, 3, {{0, 1, 2, 0}, {0, 1, 3, 0}, {0, 2, 3, 0}, {1, 2, 3, 0}}};
  // hexahedron nodes 0..7 at (-,-,-), (+,-,-), (+,+,-), (-,+,-), (-,-,+), (+,-,+), (+,+,+), (-,+,+)
  static const FacetType hex{6, 4, 4, {{0, 1, 2, 3}, {4, 5, 6, 7}, {0, 1, 5, 4},
                                       {1, 2, 6, 5}, {2, 3, 7, 6}, {3, 0, 4, 7}}};
  // triangle_6: corners 0, 1, 2; mid-sides 3 (0-1), 4 (1-2), 5 (2-0)
  static const FacetType tri{3, 3, 2, {{0, 1, 3, 0}, {1, 2, 4, 0}, {2, 0, 5, 0}}};
  return et == AKB_TETRAHEDRON_4 ? tet : (et == AKB_HEXAHEDRON_8 ? hex : tri);
}

int nodes_per_elem(int et) {
  return et == AKB_TETRAHEDRON_4 ? 4 : (et == AKB_HEXAHEDRON_8 ? 8 : 6);
}

void cross(const double *a, const double *b, double *c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

}  // namespace

extern "C" int akb_mesh_neumann_forces(int et, const double *nodes, int64_t N,
                                       const int32_t *conn, int64_t E,
                                       const int32_t *group_nodes, int64_t count,
                                       const double *stress, double *forces) {
  if (et < AKB_TETRAHEDRON_4 || et > AKB_TRIANGLE_6) return fail(AKB_EINVAL, "unknown element type");
  if (N < 0 || E < 0 || count < 0 || !stress || !forces || (N > 0 && !nodes) ||
      (E > 0 && !conn) || (count > 0 && !group_nodes))
    return fail(AKB_EINVAL, "bad arguments");
  const int d = et == AKB_TRIANGLE_6 ? 2 : 3;
  const int ne = nodes_per_elem(et);
  const FacetType &ft = facets_of(et);
  std::vector<uint8_t> in_group(N, 0);
  for (int64_t k = 0; k < count; ++k) {
    if (group_nodes[k] < 0 || group_nodes[k] >= N) return fail(AKB_EINVAL, "group node out of range");
    in_group[group_nodes[k]] = 1;
  }
  for (int64_t k = 0; k < E * ne; ++k)
    if (conn[k] < 0 || conn[k] >= N) return fail(AKB_EINVAL, "connectivity refers to a missing node");
  // facets on the boundary: their sorted corner set appears in one element
  std::map<std::array<int32_t, 4>, int> uses;
  auto key = [&](const int32_t *c, const std::array<int, 4> &loc) {
    std::array<int32_t, 4> k{-1, -1, -1, -1};
    for (int i = 0; i < ft.corners; ++i) k[i] = c[loc[i]];
    std::sort(k.begin(), k.begin() + ft.corners);
    return k;
  };
  for (int64_t e = 0; e < E; ++e)
    for (int f = 0; f < ft.nf; ++f) uses[key(conn + e * ne, ft.local[f])]++;
  for (int64_t e = 0; e < E; ++e) {
    const int32_t *c = conn + e * ne;
    double centroid[3] = {0., 0., 0.};
    for (int a = 0; a < ne; ++a)
      for (int i = 0; i < d; ++i) centroid[i] += nodes[(int64_t)c[a] * d + i] / ne;
    for (int f = 0; f < ft.nf; ++f) {
      const auto &loc = ft.local[f];
      bool all = true;
      for (int i = 0; i < ft.nn; ++i) all = all && in_group[c[loc[i]]];
      if (!all || uses[key(c, loc)] != 1) continue;
      double X[4][3] = {{0.}};
      double fc[3] = {0., 0., 0.};
      for (int i = 0; i < ft.nn; ++i)
        for (int j = 0; j < d; ++j) {
          X[i][j] = nodes[(int64_t)c[loc[i]] * d + j];
          fc[j] += X[i][j] / ft.nn;
        }
      // quadrature: points, weights, shape values and the area-scaled normal
      std::vector<std::array<double, 4>> Nq;
      std::vector<std::array<double, 3>> Jn;  // normal times |J| at each point
      std::vector<double> w;
      if (et == AKB_TETRAHEDRON_4) {
        double t1[3], t2[3], n[3];
        for (int j = 0; j < 3; ++j) {
          t1[j] = X[1][j] - X[0][j];
          t2[j] = X[2][j] - X[0][j];
        }
        cross(t1, t2, n);
        Nq.push_back({1. / 3., 1. / 3., 1. / 3., 0.});
        Jn.push_back({n[0], n[1], n[2]});
        w.push_back(0.5);
      } else if (et == AKB_HEXAHEDRON_8) {
        const double g = 1. / std::sqrt(3.);
        const double s[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
        for (int q = 0; q < 4; ++q) {
          const double xi = s[q][0] * g, eta = s[q][1] * g;
          std::array<double, 4> Nv;
          double dxi[3] = {0., 0., 0.}, deta[3] = {0., 0., 0.}, n[3];
          for (int a = 0; a < 4; ++a) {
            Nv[a] = .25 * (1 + s[a][0] * xi) * (1 + s[a][1] * eta);
            for (int j = 0; j < 3; ++j) {
              dxi[j] += .25 * s[a][0] * (1 + s[a][1] * eta) * X[a][j];
              deta[j] += .25 * s[a][1] * (1 + s[a][0] * xi) * X[a][j];
            }
          }
          cross(dxi, deta, n);
          Nq.push_back(Nv);
          Jn.push_back({n[0], n[1], n[2]});
          w.push_back(1.);
        }
      } else {
        // _segment_3: nodes at xi = -1, 1 and 0
        const double g = 1. / std::sqrt(3.);
        for (int q = 0; q < 2; ++q) {
          const double xi = q == 0 ? -g : g;
          std::array<double, 4> Nv{xi * (xi - 1) / 2., xi * (xi + 1) / 2., 1 - xi * xi, 0.};
          const double dN[3] = {xi - .5, xi + .5, -2 * xi};
          double t[2] = {0., 0.};
          for (int a = 0; a < 3; ++a)
            for (int j = 0; j < 2; ++j) t[j] += dN[a] * X[a][j];
          Nq.push_back(Nv);
          Jn.push_back({t[1], -t[0], 0.});
          w.push_back(1.);
        }
      }
      // orient every normal away from the element
      double out[3] = {0., 0., 0.};
      for (int j = 0; j < d; ++j) out[j] = fc[j] - centroid[j];
      for (size_t q = 0; q < Nq.size(); ++q) {
        double *n = Jn[q].data();
        double dot = 0.;
        for (int j = 0; j < d; ++j) dot += n[j] * out[j];
        if (dot < 0)
          for (int j = 0; j < d; ++j) n[j] = -n[j];
        // traction times |J|: sigma (n |J|), sigma column-major [d][d]
        double t[3] = {0., 0., 0.};
        for (int i = 0; i < d; ++i)
          for (int j = 0; j < d; ++j) t[i] += stress[i + d * j] * n[j];
        for (int a = 0; a < ft.nn; ++a)
          for (int i = 0; i < d; ++i)
            forces[(int64_t)c[loc[a]] * d + i] += Nq[q][a] * t[i] * w[q];
      }
    }
  }
  return AKB_OK;
}

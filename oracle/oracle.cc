// CPU oracle (test infrastructure only) -- see oracle.h for the list of
// reference files this restates.  Compiled with -ffp-contract=off so that every
// product and sum is rounded separately, in the order written here.
#include "oracle.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

#include <thread>

namespace {

// static block partition of [0, n) over nthreads std::threads; the work of
// each index is independent, so results do not depend on the thread count
template <class F> void parallel_for(long n, int nthreads, F &&f) {
  if (nthreads <= 1 || n < 2 * nthreads) {
    for (long i = 0; i < n; ++i) f(i);
    return;
  }
  std::vector<std::thread> pool;
  long chunk = (n + nthreads - 1) / nthreads;
  for (int t = 0; t < nthreads; ++t) {
    long b = t * chunk, e = std::min(n, b + chunk);
    if (b >= e) break;
    pool.emplace_back([b, e, &f] {
      for (long i = b; i < e; ++i) f(i);
    });
  }
  for (auto &th : pool) th.join();
}

/* ------------------------------------------------------------------------ */
/* element classes                                                          */
/* ------------------------------------------------------------------------ */
int nnodes(int t) { return t == OR_TET4 ? 4 : (t == OR_HEX8 ? 8 : 6); }
int sdim(int t) { return t == OR_TRI6 ? 2 : 3; }

// quadrature, gauss_integration.cc:42-43,62-65,75-86,109-110 and the tensor
// product of gauss_integration_tmpl.hh:129-180 (xi varies fastest)
int quad(int t, int rule, double *pts, double *w) {
  if (t == OR_TET4) {
    pts[0] = 1. / 4.; pts[1] = 1. / 4.; pts[2] = 1. / 4.;
    w[0] = 1. / 6.;
    return 1;
  }
  if (t == OR_HEX8) {
    const double g[2] = {-1. / std::sqrt(3.), 1. / std::sqrt(3.)};
    for (int q = 0; q < 8; ++q) {
      pts[q * 3 + 0] = g[q & 1];
      pts[q * 3 + 1] = g[(q >> 1) & 1];
      pts[q * 3 + 2] = g[(q >> 2) & 1];
      w[q] = 1.;
    }
    return 8;
  }
  if (rule == 0) {  // triangle, degree 2 -> 3 points
    const double p[6] = {1. / 6., 1. / 6., 2. / 3., 1. / 6., 1. / 6., 2. / 3.};
    for (int i = 0; i < 6; ++i) pts[i] = p[i];
    w[0] = w[1] = w[2] = 1. / 6.;
    return 3;
  }
  // triangle, degree 4 -> 6 points
  const double a = (8. - std::sqrt(10.) + std::sqrt(38. - 44. * std::sqrt(2. / 5.))) / 18.;
  const double b = (8. - std::sqrt(10.) - std::sqrt(38. - 44. * std::sqrt(2. / 5.))) / 18.;
  const double w1 = (620. - std::sqrt(213125. - 53320. * std::sqrt(10.))) / 7440.;
  const double w2 = (620. + std::sqrt(213125. - 53320. * std::sqrt(10.))) / 7440.;
  const double p[12] = {b, b, 1. - 2. * b, b, b, 1. - 2. * b,
                        a, 1. - 2. * a, a, a, 1. - 2. * a, a};
  for (int i = 0; i < 12; ++i) pts[i] = p[i];
  w[0] = w[1] = w[2] = w1;
  w[3] = w[4] = w[5] = w2;
  return 6;
}

// shape functions (computeShapes of the element files)
void shapes(int t, const double *c, double *N) {
  if (t == OR_TET4) {
    double c0 = 1 - c[0] - c[1] - c[2];
    N[0] = c0; N[1] = c[1]; N[2] = c[2]; N[3] = c[0];
  } else if (t == OR_HEX8) {
    N[0] = .125 * (1 - c[0]) * (1 - c[1]) * (1 - c[2]);
    N[1] = .125 * (1 + c[0]) * (1 - c[1]) * (1 - c[2]);
    N[2] = .125 * (1 + c[0]) * (1 + c[1]) * (1 - c[2]);
    N[3] = .125 * (1 - c[0]) * (1 + c[1]) * (1 - c[2]);
    N[4] = .125 * (1 - c[0]) * (1 - c[1]) * (1 + c[2]);
    N[5] = .125 * (1 + c[0]) * (1 - c[1]) * (1 + c[2]);
    N[6] = .125 * (1 + c[0]) * (1 + c[1]) * (1 + c[2]);
    N[7] = .125 * (1 - c[0]) * (1 + c[1]) * (1 + c[2]);
  } else {
    double c0 = 1 - c[0] - c[1], c1 = c[0], c2 = c[1];
    N[0] = c0 * (2 * c0 - 1.);
    N[1] = c1 * (2 * c1 - 1.);
    N[2] = c2 * (2 * c2 - 1.);
    N[3] = 4 * c0 * c1;
    N[4] = 4 * c1 * c2;
    N[5] = 4 * c2 * c0;
  }
}

// dN/ds, row k (natural direction), column a (node): d[k*n + a]
void dnds(int t, const double *c, double *d) {
  if (t == OR_TET4) {
    const double v[12] = {-1., 0., 0., 1., -1., 1., 0., 0., -1., 0., 1., 0.};
    for (int i = 0; i < 12; ++i) d[i] = v[i];
  } else if (t == OR_HEX8) {
    double *r0 = d, *r1 = d + 8, *r2 = d + 16;
    r0[0] = -.125 * (1 - c[1]) * (1 - c[2]);
    r0[1] = .125 * (1 - c[1]) * (1 - c[2]);
    r0[2] = .125 * (1 + c[1]) * (1 - c[2]);
    r0[3] = -.125 * (1 + c[1]) * (1 - c[2]);
    r0[4] = -.125 * (1 - c[1]) * (1 + c[2]);
    r0[5] = .125 * (1 - c[1]) * (1 + c[2]);
    r0[6] = .125 * (1 + c[1]) * (1 + c[2]);
    r0[7] = -.125 * (1 + c[1]) * (1 + c[2]);
    r1[0] = -.125 * (1 - c[0]) * (1 - c[2]);
    r1[1] = -.125 * (1 + c[0]) * (1 - c[2]);
    r1[2] = .125 * (1 + c[0]) * (1 - c[2]);
    r1[3] = .125 * (1 - c[0]) * (1 - c[2]);
    r1[4] = -.125 * (1 - c[0]) * (1 + c[2]);
    r1[5] = -.125 * (1 + c[0]) * (1 + c[2]);
    r1[6] = .125 * (1 + c[0]) * (1 + c[2]);
    r1[7] = .125 * (1 - c[0]) * (1 + c[2]);
    r2[0] = -.125 * (1 - c[0]) * (1 - c[1]);
    r2[1] = -.125 * (1 + c[0]) * (1 - c[1]);
    r2[2] = -.125 * (1 + c[0]) * (1 + c[1]);
    r2[3] = -.125 * (1 - c[0]) * (1 + c[1]);
    r2[4] = .125 * (1 - c[0]) * (1 - c[1]);
    r2[5] = .125 * (1 + c[0]) * (1 - c[1]);
    r2[6] = .125 * (1 + c[0]) * (1 + c[1]);
    r2[7] = .125 * (1 - c[0]) * (1 + c[1]);
  } else {
    double c0 = 1 - c[0] - c[1], c1 = c[0], c2 = c[1];
    double *r0 = d, *r1 = d + 6;
    r0[0] = 1 - 4 * c0; r0[1] = 4 * c1 - 1.; r0[2] = 0.;
    r0[3] = 4 * (c0 - c1); r0[4] = 4 * c2; r0[5] = -4 * c2;
    r1[0] = 1 - 4 * c0; r1[1] = 0.; r1[2] = 4 * c2 - 1.;
    r1[3] = -4 * c1; r1[4] = 4 * c1; r1[5] = 4 * (c0 - c2);
  }
}

/* small dense helpers, column-major m[i + j*d] ------------------------------ */
inline double det2(const double *m) { return m[0] * m[3] - m[1] * m[2]; }
inline double det3(const double *m) {
  // first-row expansion
  return m[0] * (m[4] * m[8] - m[7] * m[5]) - m[3] * (m[1] * m[8] - m[7] * m[2]) +
         m[6] * (m[1] * m[5] - m[4] * m[2]);
}
// cofactor c(i,j) of a 3x3 (column-major): m(i1,j1) m(i2,j2) - m(i1,j2) m(i2,j1)
inline double cof3(const double *m, int i, int j) {
  int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
  return m[i1 + 3 * j1] * m[i2 + 3 * j2] - m[i1 + 3 * j2] * m[i2 + 3 * j1];
}
// inverse by cofactors: det = c00 m00 + c10 m10 + c20 m20, inv(i,j) = c(j,i)/det
inline void inv3(const double *m, double *r) {
  double c0 = cof3(m, 0, 0), c1 = cof3(m, 1, 0), c2 = cof3(m, 2, 0);
  double det = c0 * m[0] + c1 * m[1] + c2 * m[2];
  double id = 1. / det;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r[i + 3 * j] = cof3(m, j, i) * id;
}
inline void inv2(const double *m, double *r) {
  double id = 1. / det2(m);
  r[0] = m[3] * id;
  r[1] = -m[1] * id;
  r[2] = -m[2] * id;
  r[3] = m[0] * id;
}

// J = dN/ds X^T, det J, dN/dx = J^-1 dN/ds for one element and one point.
// X is [n][dim]; B out is [n][dim] (dN_a/dx_j at B[a*dim + j]).
double jac_and_dndx(int t, const double *xi, const double *X, double *B) {
  const int n = nnodes(t), d = sdim(t);
  double dn[24];
  dnds(t, xi, dn);
  double J[9], Ji[9];
  for (int k = 0; k < d; ++k)
    for (int j = 0; j < d; ++j) {
      double s = dn[k * n] * X[j];
      for (int a = 1; a < n; ++a) s = s + dn[k * n + a] * X[a * d + j];
      J[k + d * j] = s;
    }
  double det;
  if (d == 3) { det = det3(J); inv3(J, Ji); }
  else { det = det2(J); inv2(J, Ji); }
  for (int a = 0; a < n; ++a)
    for (int j = 0; j < d; ++j) {
      double s = Ji[j] * dn[a];
      for (int k = 1; k < d; ++k) s = s + Ji[j + d * k] * dn[k * n + a];
      B[a * d + j] = s;
    }
  return det;
}

inline double dist(const double *a, const double *b, int d) {
  double s = 0;
  for (int i = 0; i < d; ++i) { double t = a[i] - b[i]; s += t * t; }
  return std::sqrt(s);
}
double tri_inradius(const double *p1, const double *p2, const double *p3, int d) {
  double a = dist(p1, p2, d), b = dist(p2, p3, d), c = dist(p1, p3, d);
  double s = (a + b + c) / 2.;
  return std::sqrt((s - a) * (s - b) * (s - c) / s);
}
double det3cols(const double *c0, const double *c1, const double *c2) {
  double m[9] = {c0[0], c0[1], c0[2], c1[0], c1[1], c1[2], c2[0], c2[1], c2[2]};
  return det3(m);
}
double tet_inradius(const double *p1, const double *p2, const double *p3, const double *p4) {
  double l12 = dist(p1, p2, 3), l13 = dist(p1, p3, 3), l14 = dist(p1, p4, 3);
  double l23 = dist(p2, p3, 3), l24 = dist(p2, p4, 3), l34 = dist(p3, p4, 3);
  double s1 = (l12 + l23 + l13) * 0.5;
  s1 = std::sqrt(s1 * (s1 - l12) * (s1 - l23) * (s1 - l13));
  double s2 = (l12 + l24 + l14) * 0.5;
  s2 = std::sqrt(s2 * (s2 - l12) * (s2 - l24) * (s2 - l14));
  double s3 = (l23 + l34 + l24) * 0.5;
  s3 = std::sqrt(s3 * (s3 - l23) * (s3 - l34) * (s3 - l24));
  double s4 = (l13 + l34 + l14) * 0.5;
  s4 = std::sqrt(s4 * (s4 - l13) * (s4 - l34) * (s4 - l14));
  // signed volume by the four-determinant expansion (aka_math_tmpl.hh:70-95)
  double vol = det3cols(p2, p3, p4);
  vol -= det3cols(p1, p3, p4);
  vol += det3cols(p1, p2, p4);
  vol -= det3cols(p1, p2, p3);
  vol /= 6;
  return 3 * vol / (s1 + s2 + s3 + s4);
}
double inradius(int t, const double *X) {
  if (t == OR_TET4) return 2. * tet_inradius(X, X + 3, X + 6, X + 9);
  if (t == OR_HEX8) {
    static const int ed[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {0, 4}, {1, 5},
                                  {2, 6}, {3, 7}, {4, 5}, {5, 6}, {6, 7}, {7, 4}};
    double p = dist(X + 3 * ed[0][0], X + 3 * ed[0][1], 3);
    for (int k = 1; k < 12; ++k) p = std::min(p, dist(X + 3 * ed[k][0], X + 3 * ed[k][1], 3));
    return p;
  }
  static const int tr[4][3] = {{0, 3, 5}, {3, 1, 4}, {3, 4, 5}, {5, 4, 2}};
  double r = std::numeric_limits<double>::max();
  for (int k = 0; k < 4; ++k)
    r = std::min(tri_inradius(X + 2 * tr[k][0], X + 2 * tr[k][1], X + 2 * tr[k][2], 2), r);
  return 2. * r;
}

/* ------------------------------------------------------------------------ */
/* constitutive laws                                                        */
/* ------------------------------------------------------------------------ */
struct Mat {
  int law;
  double rho, E, nu, sigma_y, h, alpha, delta_T;
  int plane_stress;
  double lambda, mu, sigma_th;
  // sigma_th internal and its saved previous value (material_thermal.cc:33-34)
  double th_prev = 0., th_cur = 0.;
  void update() {
    lambda = nu * E / ((1 + nu) * (1 - 2 * nu));
    mu = E / (2 * (1 + nu));
    if (plane_stress && law != OR_NEOHOOKEAN) lambda = nu * E / ((1 + nu) * (1 - nu));
    sigma_th = -E / (1. - 2. * nu) * alpha * delta_T;
  }
  bool finite() const { return law == OR_NEOHOOKEAN || law == OR_ELASTIC_FD; }
  double celerity() const { return std::sqrt((lambda + 2 * mu) / rho); }
};

// material_elastic_inline_impl.hh:31-48
inline void elastic(int d, double lambda, double mu, const double *g, double sth,
                    double *s) {
  double tr = g[0];
  for (int i = 1; i < d; ++i) tr = tr + g[i * (d + 1)];
  double dia = lambda * tr + sth;
  for (int j = 0; j < d; ++j)
    for (int i = 0; i < d; ++i) {
      double eps = .5 * (g[j + d * i] + g[i + d * j]);
      double v = 2. * mu * eps;
      s[i + d * j] = (i == j) ? v + dia : v;
    }
}

// material_neohookean_inline_impl.hh:37-48 with gradUToF / rightCauchy
// Green-Lagrange strain E = (g^T g + g^T + g) / 2 (material_inline_impl.hh:127-130)
inline void green_lagrange(int d, const double *g, double *E) {
  for (int j = 0; j < d; ++j)
    for (int i = 0; i < d; ++i) {
      double s = g[0 + d * i] * g[0 + d * j];
      for (int k = 1; k < d; ++k) s = s + g[k + d * i] * g[k + d * j];
      E[i + d * j] = ((s + g[j + d * i]) + g[i + d * j]) / 2.;
    }
}

inline void neohookean(int d, double lambda, double mu, const double *g, double C33,
                       double *S) {
  double F[9], C[9], Ci[9];
  for (int j = 0; j < d; ++j)
    for (int i = 0; i < d; ++i) F[i + d * j] = (i == j ? 1. : 0.) + g[i + d * j];
  for (int j = 0; j < d; ++j)
    for (int i = 0; i < d; ++i) {
      double s = F[0 + d * i] * F[0 + d * j];
      for (int k = 1; k < d; ++k) s = s + F[k + d * i] * F[k + d * j];
      C[i + d * j] = s;
    }
  double J;
  if (d == 3) { J = det3(F) * std::sqrt(C33); inv3(C, Ci); }
  else { J = det2(F) * std::sqrt(C33); inv2(C, Ci); }
  double c = lambda * std::log(J) - mu;
  for (int j = 0; j < d; ++j)
    for (int i = 0; i < d; ++i) {
      double t = c * Ci[i + d * j];
      S[i + d * j] = (i == j) ? mu + t : t;
    }
}

// material_linear_isotropic_hardening_inline_impl.hh:28-84 followed by
// MaterialPlastic::computeStressAndInelasticStrainOnQuad (material_plastic.hh)
inline void plastic(int d, double lambda, double mu, double sigma_y, double h,
                    const double *g, const double *gp, const double *sp,
                    const double *ep_prev, double iso_cur, double iso_prev,
                    double dsth, double *s, double *ep, double *iso) {
  const int dd = d * d;
  double gdu[9] = {0.}, str[9] = {0.}, dev[9], deps[9];
  for (int k = 0; k < dd; ++k) gdu[k] = g[k] - gp[k];
  elastic(d, lambda, mu, gdu, dsth, str);
  for (int k = 0; k < dd; ++k) str[k] = str[k] + sp[k];
  double tr = str[0];
  for (int i = 1; i < d; ++i) tr = tr + str[i * (d + 1)];
  for (int k = 0; k < 9; ++k) dev[k] = 0.;
  for (int j = 0; j < d; ++j)
    for (int i = 0; i < d; ++i) dev[i + 3 * j] = str[i + d * j];
  double t3 = tr / 3.0;
  for (int i = 0; i < 3; ++i) dev[i * 4] = dev[i * 4] - t3;
  double ss = dev[0] * dev[0];
  for (int k = 1; k < 9; ++k) ss = ss + dev[k] * dev[k];
  double eff = std::sqrt(3. / 2. * ss);
  bool yield = (eff - iso_cur - sigma_y) > 0;
  double dp = yield ? (eff - sigma_y - iso_prev) / (3 * mu + h) : 0;
  *iso = iso_prev + h * dp;
  double nrm = std::sqrt(ss);
  const double tol = 1e2 * std::numeric_limits<double>::epsilon();
  for (int k = 0; k < dd; ++k) deps[k] = 0.;
  if (std::abs(eff) > nrm * tol) {
    for (int j = 0; j < d; ++j)
      for (int i = 0; i < d; ++i)
        deps[i + d * j] = dev[i + 3 * j] * 3. / 2. * dp / eff;
  }
  double ge[9], sel[9];
  for (int k = 0; k < dd; ++k) ge[k] = gdu[k] - deps[k];
  elastic(d, lambda, mu, ge, 0., sel);
  for (int k = 0; k < dd; ++k) {
    s[k] = sp[k] + sel[k];
    ep[k] = ep_prev[k] + deps[k];
  }
}

/* ------------------------------------------------------------------------ */
/* model                                                                    */
/* ------------------------------------------------------------------------ */
struct MatState {
  std::vector<int> elems;  // filter: global element ids, ascending
  long offset = 0;         // first slot (element) of this material in r_e
  std::vector<double> grad_u, grad_u_prev, stress, stress_prev, pk2;
  std::vector<double> eps_p, eps_p_prev, iso, iso_prev, pe;
  std::vector<double> c33;  // plane-stress neohookean out-of-plane stretch, initially 1
  std::vector<double> eig;  // eigen_grad_u per point [qp][d*d], empty when zero
};

}  // namespace

struct or_model {
  int type, rule, d, n, nq;
  long N, E;
  std::vector<double> X;
  std::vector<int32_t> conn;
  std::vector<int32_t> mat_of_elem;
  std::vector<Mat> mats;
  std::vector<MatState> st;
  double qpts[24], qw[8];
  std::vector<double> Nq, B, wJ;  // per global element
  std::vector<double> u, v, a, fext, fint, mass;
  std::vector<uint8_t> blocked;
  std::vector<double> re;  // [slot][n][d]
  std::vector<int64_t> node_ptr;
  std::vector<int64_t> node_ent;       // internal-force scatter order
  std::vector<int64_t> node_ent_mass;  // lumped-mass scatter order
  double dt = 0.;
  int threads = 1;
};

namespace {

void assign_materials(or_model *m) {
  int nm = (int)m->mats.size();
  m->st.assign(nm, MatState());
  for (long e = 0; e < m->E; ++e) {
    int k = m->mat_of_elem.empty() ? 0 : m->mat_of_elem[e];
    m->st[k].elems.push_back((int)e);
  }
  long off = 0;
  const int dd = m->d * m->d;
  for (int k = 0; k < nm; ++k) {
    MatState &s = m->st[k];
    s.offset = off;
    off += (long)s.elems.size();
    size_t nqp = s.elems.size() * (size_t)m->nq;
    s.grad_u.assign(nqp * dd, 0.);
    s.grad_u_prev.assign(nqp * dd, 0.);
    s.stress.assign(nqp * dd, 0.);
    s.stress_prev.assign(nqp * dd, 0.);
    if (m->mats[k].finite()) s.pk2.assign(nqp * dd, 0.);
    if (m->mats[k].law == OR_NEOHOOKEAN && m->mats[k].plane_stress && m->d == 2)
      s.c33.assign(nqp, 1.);
    if (m->mats[k].law == OR_PLASTIC) {
      s.eps_p.assign(nqp * dd, 0.);
      s.eps_p_prev.assign(nqp * dd, 0.);
      s.iso.assign(nqp, 0.);
      s.iso_prev.assign(nqp, 0.);
      s.pe.assign(nqp, 0.);
    }
  }
  // node -> slot lists, slot = (material offset + local element) * n + a;
  // pushed in increasing slot order, which is the reference scatter order
  m->node_ptr.assign(m->N + 1, 0);
  for (int k = 0; k < nm; ++k)
    for (int e : m->st[k].elems)
      for (int a = 0; a < m->n; ++a) m->node_ptr[m->conn[(long)e * m->n + a] + 1]++;
  for (long i = 0; i < m->N; ++i) m->node_ptr[i + 1] += m->node_ptr[i];
  m->node_ent.assign(m->node_ptr[m->N], 0);
  std::vector<int64_t> fill(m->node_ptr.begin(), m->node_ptr.end() - 1);
  for (int k = 0; k < nm; ++k) {
    const MatState &s = m->st[k];
    for (size_t le = 0; le < s.elems.size(); ++le) {
      long e = s.elems[le];
      for (int a = 0; a < m->n; ++a) {
        long node = m->conn[e * m->n + a];
        m->node_ent[fill[node]++] = (int64_t)(s.offset + (long)le) * m->n + a;
      }
    }
  }
  // the lumped mass is assembled over all elements of the type in element
  // order, whatever their material (solid_mechanics_model_mass.cc:115-128)
  std::vector<int64_t> slot_of_elem(m->E);
  for (int k = 0; k < nm; ++k)
    for (size_t le = 0; le < m->st[k].elems.size(); ++le)
      slot_of_elem[m->st[k].elems[le]] = m->st[k].offset + (long)le;
  m->node_ent_mass.assign(m->node_ptr[m->N], 0);
  std::copy(m->node_ptr.begin(), m->node_ptr.end() - 1, fill.begin());
  for (long e = 0; e < m->E; ++e)
    for (int a = 0; a < m->n; ++a)
      m->node_ent_mass[fill[m->conn[e * m->n + a]]++] = slot_of_elem[e] * m->n + a;
  m->re.assign((size_t)m->E * m->n * m->d, 0.);
}

// gather r_e into a nodal array with factor -1 (internal force) or +1 (mass)
void gather(or_model *m, double scale, std::vector<double> &out, int ncomp_src,
            int ncomp_dst, const std::vector<int64_t> &ent) {
parallel_for(m->N, m->threads, [&](long i) {
    double acc[3] = {0., 0., 0.};
    for (int64_t p = m->node_ptr[i]; p < m->node_ptr[i + 1]; ++p) {
      const double *r = &m->re[(size_t)ent[p] * ncomp_src];
      for (int c = 0; c < ncomp_src; ++c) acc[c] += scale * r[c];
    }
    for (int c = 0; c < ncomp_dst; ++c)
      out[(size_t)i * ncomp_dst + c] = acc[ncomp_src == 1 ? 0 : c];
  });
}

void lumped_mass(or_model *m) {
  const int n = m->n, nq = m->nq;
  for (size_t k = 0; k < m->st.size(); ++k) {
    const MatState &s = m->st[k];
    double rho = m->mats[k].rho;
parallel_for((long)s.elems.size(), m->threads, [&](long le) {
      long e = s.elems[le];
      double *r = &m->re[(size_t)(s.offset + le) * n];
      if (m->type == OR_TRI6) {
        // fe_engine_template_tmpl_field.hh:144-242: rho V_e scaled per node
        double vol = rho * m->wJ[e * nq];
        for (int q = 1; q < nq; ++q) vol = vol + rho * m->wJ[e * nq + q];
        for (int a = 0; a < n; ++a) r[a] = vol * (a < 3 ? 1. / 12. : 1. / 4.);
      } else {
        // row sum: sum_q (rho N_a(q)) wJ_q
        for (int a = 0; a < n; ++a) {
          double acc = rho * m->Nq[(e * nq) * n + a] * m->wJ[e * nq];
          for (int q = 1; q < nq; ++q)
            acc = acc + rho * m->Nq[(e * nq + q) * n + a] * m->wJ[e * nq + q];
          r[a] = acc;
        }
      }
    });
  }
  m->mass.assign((size_t)m->N * m->d, 0.);
  gather(m, 1., m->mass, 1, m->d, m->node_ent_mass);
}

// gradient, stress and elemental force of one material's elements
void element_forces(or_model *m, int k, bool history_step) {
  const int n = m->n, nq = m->nq, d = m->d, dd = d * d;
  MatState &s = m->st[k];
  Mat &mat = m->mats[k];
  const long ne = (long)s.elems.size();
  // MaterialThermal::computeStress sets the current sigma_th
  // (material_thermal.hh:89-95); the plastic trial stress takes the saved
  // previous value minus it (material_linear_isotropic_hardening_inline_impl.hh:31-34)
  mat.th_cur = mat.sigma_th;
  const double dsth = mat.th_prev - mat.th_cur;
parallel_for(ne, m->threads, [&](long le) {
    const long e = s.elems[le];
    const int32_t *cn = &m->conn[e * n];
    double ue[24];
    for (int a = 0; a < n; ++a)
      for (int i = 0; i < d; ++i) ue[a * d + i] = m->u[(size_t)cn[a] * d + i];
    double re[24];
    for (int c = 0; c < n * d; ++c) re[c] = 0.;
    for (int q = 0; q < nq; ++q) {
      const size_t qp = (size_t)le * nq + q;
      const double *B = &m->B[((size_t)e * nq + q) * n * d];
      const double w = m->wJ[(size_t)e * nq + q];
      double *g = &s.grad_u[qp * dd];
      // grad u = u B^T  (shape_functions_inline_impl.hh:303-310)
      for (int j = 0; j < d; ++j)
        for (int i = 0; i < d; ++i) {
          double t = ue[i] * B[j];
          for (int a = 1; a < n; ++a) t = t + ue[a * d + i] * B[a * d + j];
          g[i + d * j] = t;
        }
      // gradu -= eigengradu (material.cc:147)
      if (!s.eig.empty())
        for (int c = 0; c < dd; ++c) g[c] = g[c] - s.eig[qp * dd + c];
      double rq[24];
      if (!mat.finite()) {
        double *sig = &s.stress[qp * dd];
        if (mat.law == OR_ELASTIC) {
          elastic(d, mat.lambda, mat.mu, g, mat.sigma_th, sig);
        } else {
          plastic(d, mat.lambda, mat.mu, mat.sigma_y, mat.h, g,
                  &s.grad_u_prev[qp * dd], &s.stress_prev[qp * dd],
                  &s.eps_p_prev[qp * dd], s.iso[qp], s.iso_prev[qp], dsth,
                  sig, &s.eps_p[qp * dd], &s.iso[qp]);
          if (history_step) {
            // MaterialPlastic::updateEnergies (material_plastic.cc:85-103)
            double wp = 0.;
            for (int c = 0; c < dd; ++c) {
              double de = s.eps_p[qp * dd + c] - s.eps_p_prev[qp * dd + c];
              double sh = sig[c] + s.stress_prev[qp * dd + c];
              wp = (c == 0) ? sh * de : wp + sh * de;
            }
            wp = wp / 2.;
            s.pe[qp] += wp;
          }
        }
        // sigma B (shape_lagrange_inline_impl.hh:402-408), d x n
        for (int a = 0; a < n; ++a)
          for (int i = 0; i < d; ++i) {
            double t = sig[i] * B[a * d];
            for (int j = 1; j < d; ++j) t = t + sig[i + d * j] * B[a * d + j];
            rq[a * d + i] = t;
          }
      } else {
        double *S = &s.pk2[qp * dd];
        if (mat.law == OR_ELASTIC_FD) {
          // MaterialElastic::computeStress, finite deformation (material_elastic.cc:82-101)
          double Egl[9];
          green_lagrange(d, g, Egl);
          elastic(d, mat.lambda, mat.mu, Egl, mat.sigma_th, S);
        } else if (!s.c33.empty()) {
          // plane stress: C33 by Newton iterations from the stored value on
          // f(x) = lambda/2 (log x + log(C00 C11 - C01^2)) + mu (x - 1)
          // (material_neohookean_inline_impl.hh:52-92, aka_math_tmpl.hh:191-208),
          // then J = det F sqrt(C33)
          const double F00 = 1. + g[0], F10 = g[1], F01 = g[2], F11 = 1. + g[3];
          const double C00 = F00 * F00 + F10 * F10, C11 = F01 * F01 + F11 * F11;
          const double C01 = F00 * F01 + F10 * F11;
          const double lc = std::log(C00 * C11 - C01 * C01);
          double x = s.c33[qp];
          double fx = mat.lambda / 2. * (std::log(x) + lc) + mat.mu * (x - 1.);
          for (int it = 0; std::fabs(fx) > 1e-5 && it < 100; ++it) {
            x -= fx / (mat.lambda / (2. * x) + mat.mu);
            fx = mat.lambda / 2. * (std::log(x) + lc) + mat.mu * (x - 1.);
          }
          s.c33[qp] = x;
          neohookean(d, mat.lambda, mat.mu, g, x, S);
        } else {
          neohookean(d, mat.lambda, mat.mu, g, 1., S);
        }
        // r_q = (B_L0 + B_L2(grad u))^T S_voigt  (material.cc:547-565)
        const int nv = d == 3 ? 6 : 3;
        double Sv[6];
        if (d == 3) {
          Sv[0] = S[0]; Sv[1] = S[4]; Sv[2] = S[8];
          Sv[3] = S[1 + 3 * 2]; Sv[4] = S[0 + 3 * 2]; Sv[5] = S[0 + 3 * 1];
        } else {
          Sv[0] = S[0]; Sv[1] = S[3]; Sv[2] = S[0 + 2 * 1];
        }
        for (int a = 0; a < n; ++a)
          for (int kk = 0; kk < d; ++kk) {
            const int col = a * d + kk;
            double acc = 0.;
            for (int I = 0; I < nv; ++I) {
              double bl0 = 0., bl2 = 0.;
              if (d == 3) {
                const double *b = &B[a * 3];
                if (I < 3) {
                  if (kk == I) bl0 = b[I];
                  bl2 = g[kk + 3 * I] * b[I];
                } else {
                  if (I == 3) { if (kk == 1) bl0 = b[2]; else if (kk == 2) bl0 = b[1]; }
                  if (I == 4) { if (kk == 0) bl0 = b[2]; else if (kk == 2) bl0 = b[0]; }
                  if (I == 5) { if (kk == 0) bl0 = b[1]; else if (kk == 1) bl0 = b[0]; }
                  const int aux = I - 3;
                  bl2 = 0.;
                  for (int mm = 0; mm < 3; ++mm)
                    if (mm != aux) bl2 += g[kk + 3 * mm] * b[3 - mm - aux];
                }
              } else {
                const double *b = &B[a * 2];
                if (I < 2) {
                  if (kk == I) bl0 = b[I];
                  bl2 = g[kk + 2 * I] * b[I];
                } else {
                  if (kk == 1) bl0 = b[0]; else bl0 = b[1];
                  bl2 = 0.;
                  for (int mm = 0; mm < 2; ++mm) bl2 += g[kk + 2 * mm] * b[1 - mm];
                }
              }
              double bf = bl0 + bl2;
              acc = (I == 0) ? bf * Sv[I] : acc + bf * Sv[I];
            }
            rq[col] = acc;
          }
      }
      // integrate: r_e = sum_q rq * wJ_q
      for (int c = 0; c < n * d; ++c) re[c] = (q == 0) ? rq[c] * w : re[c] + rq[c] * w;
    }
    double *out = &m->re[(size_t)(s.offset + le) * n * d];
    for (int c = 0; c < n * d; ++c) out[c] = re[c];
  });
}

void internal_forces(or_model *m, bool history_step) {
  for (size_t k = 0; k < m->st.size(); ++k) element_forces(m, (int)k, history_step);
  gather(m, -1., m->fint, m->d, m->d, m->node_ent);
}

void save_previous(or_model *m) {
  for (auto &mt : m->mats) mt.th_prev = mt.th_cur;
  for (auto &s : m->st) {
    s.grad_u_prev = s.grad_u;
    s.stress_prev = s.stress;
    if (!s.iso.empty()) {
      s.eps_p_prev = s.eps_p;
      s.iso_prev = s.iso;
    }
  }
}

void one_step(or_model *m) {
  const long nd = m->N * m->d;
  const double dt = m->dt;
  save_previous(m);
  // NewmarkBeta::predictor with alpha = 0, beta = 1/2, k = h = 0
parallel_for(nd, m->threads, [&](long i) {
    if (!m->blocked[i]) {
      double dta = dt * m->a[i];
      m->u[i] += (1 - 0. * 0.) * dt * m->v[i] + (.5 - 0. * 0. * .5) * dt * dta;
      m->v[i] = (1 - 0.) * m->v[i] + (1 - 0. * .5) * dta;
    }
  });
  internal_forces(m, true);
  // residual r = (0 + f_ext + f_int) + M (-a); x = r / M; corrector c=1, d=dt/2
  const double dcoef = .5 * dt;
parallel_for(nd, m->threads, [&](long i) {
    double r = 0. + 1. * m->fext[i];
    r = r + 1. * m->fint[i];
    double ma = 0. + -1. * m->a[i];  // DOFManagerDefault::assembleLumpedMatMulVectToResidual
    r = r + m->mass[i] * ma;
    if (!m->blocked[i]) {
      double x = 1. * (r / m->mass[i]);
      m->v[i] += dcoef * x;
      m->a[i] += 1. * x;
    }
  });
}

}  // namespace

/* ------------------------------------------------------------------------ */
/* C API                                                                    */
/* ------------------------------------------------------------------------ */
extern "C" {

int or_nb_nodes_per_element(int type) { return nnodes(type); }
int or_dim(int type) { return sdim(type); }
int or_nb_quad(int type, int rule) {
  double p[24], w[8];
  return quad(type, rule, p, w);
}
void or_quadrature(int type, int rule, double *pts, double *w) { quad(type, rule, pts, w); }
void or_shapes(int type, const double *xi, double *N) { shapes(type, xi, N); }
double or_inradius(int type, const double *Xe) { return inradius(type, Xe); }

long or_precompute(int type, int rule, const double *Xe, long E, double *N, double *B,
                   double *j) {
  double p[24], w[8];
  const int nq = quad(type, rule, p, w), n = nnodes(type), d = sdim(type);
  long bad = 0;
  for (long e = 0; e < E; ++e)
    for (int q = 0; q < nq; ++q) {
      const double *xi = &p[q * d];
      shapes(type, xi, &N[(e * nq + q) * n]);
      double det = jac_and_dndx(type, xi, &Xe[e * n * d], &B[(e * nq + q) * n * d]);
      if (det < 0 && bad == 0) bad = -(1 + e * nq + q);
      j[e * nq + q] = det * w[q];
    }
  return bad;
}

void or_elastic_stress(int dim, double E, double nu, int plane_stress, const double *g,
                       double sigma_th, double *s) {
  Mat m{OR_ELASTIC, 1., E, nu, 0., 0., 0., 0., plane_stress, 0., 0., 0.};
  m.update();
  elastic(dim, m.lambda, m.mu, g, sigma_th, s);
}
void or_neohookean_stress(int dim, double E, double nu, const double *g, double C33,
                          double *S) {
  Mat m{OR_NEOHOOKEAN, 1., E, nu, 0., 0., 0., 0., 0, 0., 0., 0.};
  m.update();
  neohookean(dim, m.lambda, m.mu, g, C33, S);
}
void or_plastic_stress(int dim, double E, double nu, double sigma_y, double h,
                       const double *g, const double *gp, const double *sp,
                       const double *epp, double iso_cur, double iso_prev, double dsth,
                       double *s, double *ep, double *iso) {
  Mat m{OR_PLASTIC, 1., E, nu, sigma_y, h, 0., 0., 0, 0., 0., 0.};
  m.update();
  plastic(dim, m.lambda, m.mu, sigma_y, h, g, gp, sp, epp, iso_cur, iso_prev, dsth, s, ep,
          iso);
}

or_model *or_model_create(int type, int rule, const double *X, long N, const int32_t *conn,
                          long E) {
  or_model *m = new or_model();
  m->type = type;
  m->rule = rule;
  m->d = sdim(type);
  m->n = nnodes(type);
  m->nq = quad(type, rule, m->qpts, m->qw);
  m->N = N;
  m->E = E;
  m->X.assign(X, X + N * m->d);
  m->conn.assign(conn, conn + E * m->n);
  size_t nd = (size_t)N * m->d;
  m->u.assign(nd, 0.); m->v.assign(nd, 0.); m->a.assign(nd, 0.);
  m->fext.assign(nd, 0.); m->fint.assign(nd, 0.); m->mass.assign(nd, 0.);
  m->blocked.assign(nd, 0);
  return m;
}
void or_model_destroy(or_model *m) { delete m; }

int or_model_add_material(or_model *m, int law, double rho, double E, double nu,
                          double sigma_y, double h, double alpha, double delta_T,
                          int plane_stress) {
  Mat mt{law, rho, E, nu, sigma_y, h, alpha, delta_T, plane_stress, 0., 0., 0.};
  mt.update();
  m->mats.push_back(mt);
  return (int)m->mats.size() - 1;
}
void or_model_set_element_material(or_model *m, const int32_t *mat) {
  m->mat_of_elem.assign(mat, mat + m->E);
}
void or_model_set_threads(or_model *m, int t) { m->threads = t < 1 ? 1 : t; }

long or_model_init(or_model *m) {
  const int n = m->n, d = m->d, nq = m->nq;
  std::vector<double> Xe((size_t)m->E * n * d);
  for (long e = 0; e < m->E; ++e)
    for (int a = 0; a < n; ++a)
      for (int i = 0; i < d; ++i)
        Xe[((size_t)e * n + a) * d + i] = m->X[(size_t)m->conn[e * n + a] * d + i];
  m->Nq.assign((size_t)m->E * nq * n, 0.);
  m->B.assign((size_t)m->E * nq * n * d, 0.);
  m->wJ.assign((size_t)m->E * nq, 0.);
  long rc = or_precompute(m->type, m->rule, Xe.data(), m->E, m->Nq.data(), m->B.data(),
                          m->wJ.data());
  if (rc != 0) return rc;
  if (m->mats.empty()) return -1;
  assign_materials(m);
  lumped_mass(m);
  return 0;
}

double or_model_stable_dt(or_model *m) {
  const int n = m->n, d = m->d;
  double min_dt = std::numeric_limits<double>::max();
  for (size_t k = 0; k < m->st.size(); ++k) {
    double c = m->mats[k].celerity();
    for (int e : m->st[k].elems) {
      double Xe[24];
      for (int a = 0; a < n; ++a)
        for (int i = 0; i < d; ++i) {
          size_t idx = (size_t)m->conn[(long)e * n + a] * d + i;
          Xe[a * d + i] = m->X[idx] + m->u[idx];
        }
      min_dt = std::min(min_dt, inradius(m->type, Xe) / c);
    }
  }
  return min_dt;
}
void or_model_set_dt(or_model *m, double dt) { m->dt = dt; }

void or_model_set_nodal(or_model *m, int field, const void *data) {
  size_t nd = (size_t)m->N * m->d;
  const double *p = (const double *)data;
  switch (field) {
  case OR_U: m->u.assign(p, p + nd); break;
  case OR_V: m->v.assign(p, p + nd); break;
  case OR_A: m->a.assign(p, p + nd); break;
  case OR_FEXT: m->fext.assign(p, p + nd); break;
  case OR_BLOCKED: {
    const uint8_t *b = (const uint8_t *)data;
    m->blocked.assign(b, b + nd);
  } break;
  default: break;
  }
}
void or_model_get_nodal(or_model *m, int field, void *data) {
  size_t nd = (size_t)m->N * m->d;
  const std::vector<double> *src = nullptr;
  switch (field) {
  case OR_U: src = &m->u; break;
  case OR_V: src = &m->v; break;
  case OR_A: src = &m->a; break;
  case OR_FEXT: src = &m->fext; break;
  case OR_FINT: src = &m->fint; break;
  case OR_MASS: src = &m->mass; break;
  case OR_BLOCKED: std::memcpy(data, m->blocked.data(), nd); return;
  default: return;
  }
  std::memcpy(data, src->data(), nd * sizeof(double));
}
long or_model_qp_size(or_model *m, int mat) {
  return (long)m->st[mat].elems.size() * m->nq;
}
void or_model_set_eigen_grad_u(or_model *m, int mat, const double *values) {
  MatState &s = m->st[mat];
  const size_t n = s.elems.size() * (size_t)m->nq * m->d * m->d;
  s.eig.assign(values, values + n);
}

void or_model_get_qp(or_model *m, int mat, int field, double *out) {
  const MatState &s = m->st[mat];
  const std::vector<double> *src = nullptr;
  switch (field) {
  case OR_GRAD_U: src = &s.grad_u; break;
  case OR_STRESS: src = &s.stress; break;
  case OR_PK2: src = &s.pk2; break;
  case OR_EPS_P: src = &s.eps_p; break;
  case OR_ISO: src = &s.iso; break;
  case OR_PLASTIC_ENERGY: src = &s.pe; break;
  default: return;
  }
  if (!src->empty()) std::memcpy(out, src->data(), src->size() * sizeof(double));
}

void or_model_solve_step(or_model *m, long nsteps) {
  for (long s = 0; s < nsteps; ++s) one_step(m);
}
void or_model_assemble_internal_forces(or_model *m) { internal_forces(m, false); }

double or_model_energy(or_model *m, int which) {
  const int d = m->d, nq = m->nq, dd = d * d;
  if (which == OR_EKIN) {
    double ekin = 0.;
    for (long i = 0; i < m->N; ++i) {
      double mv2 = 0.;
      for (int c = 0; c < d; ++c) {
        double mm = m->mass[i * d + c], vv = m->v[i * d + c];
        if (mm > std::numeric_limits<double>::epsilon()) mv2 += vv * vv * mm;
      }
      ekin += mv2;
    }
    return ekin / 2.;
  }
  if (which == OR_EXT_WORK) {
    double w = 0.;
    for (long i = 0; i < m->N * d; ++i) {
      if (m->blocked[i]) w -= m->fint[i] * m->v[i];
      else w += m->fext[i] * m->v[i];
    }
    return w * m->dt;
  }
  double total = 0.;
  for (size_t k = 0; k < m->st.size(); ++k) {
    const MatState &s = m->st[k];
    const Mat &mat = m->mats[k];
    double acc = 0.;
    for (size_t le = 0; le < s.elems.size(); ++le) {
      long e = s.elems[le];
      double el = 0.;
      for (int q = 0; q < nq; ++q) {
        size_t qp = le * nq + q;
        double dens = 0.;
        if (which == OR_EPLASTIC) {
          if (mat.law != OR_PLASTIC) continue;
          dens = s.pe[qp];
        } else if (mat.law == OR_ELASTIC_FD) {
          // .5 S : E (material_elastic.cc:140-157)
          const double *g = &s.grad_u[qp * dd];
          const double *S = &s.pk2[qp * dd];
          double Egl[9];
          green_lagrange(d, g, Egl);
          double dot = 0.;
          for (int c = 0; c < dd; ++c) dot = (c == 0) ? S[c] * Egl[c] : dot + S[c] * Egl[c];
          dens = .5 * dot;
        } else if (mat.law == OR_NEOHOOKEAN) {
          const double *g = &s.grad_u[qp * dd];
          double F[9];
          for (int j = 0; j < d; ++j)
            for (int i = 0; i < d; ++i) F[i + d * j] = (i == j ? 1. : 0.) + g[i + d * j];
          double trC = 0.;
          for (int i = 0; i < d; ++i) {
            double t = F[0 + d * i] * F[0 + d * i];
            for (int kk = 1; kk < d; ++kk) t = t + F[kk + d * i] * F[kk + d * i];
            trC = (i == 0) ? t : trC + t;
          }
          double J = d == 3 ? det3(F) : det2(F);
          dens = mat.lambda * std::pow(std::log(J), 2.) +
                 mat.mu * (-std::log(J) + (trC - d) / 2.) / 2.;
        } else {
          const double *g = &s.grad_u[qp * dd];
          const double *sg = &s.stress[qp * dd];
          double dot = 0.;
          for (int c = 0; c < dd; ++c) {
            double ge = g[c];
            if (mat.law == OR_PLASTIC) ge = g[c] - s.eps_p[qp * dd + c];
            dot = (c == 0) ? sg[c] * ge : dot + sg[c] * ge;
          }
          dens = .5 * dot;
        }
        el = (q == 0) ? dens * m->wJ[e * nq + q] : el + dens * m->wJ[e * nq + q];
      }
      acc += el;
    }
    total += acc;
  }
  return total;
}

}  // extern "C"

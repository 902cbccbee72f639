// Device-side element and constitutive arithmetic of the explicit step.
//
// Every function keeps the operand order of the reference expression it
// restates (file:line given per function).  The FP64 kernels that include this
// header are compiled with --fmad=false, so each product and sum is rounded on
// its own exactly as the CPU path rounds it.  T is the element-math type
// (double for the plain path, float for the mixed path).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace akb {

enum { ET_TET4 = 0, ET_HEX8 = 1, ET_TRI6 = 2 };
enum { LAW_ELASTIC = 0, LAW_NEOHOOKEAN = 1, LAW_PLASTIC = 2 };

// Lame constants and the per-material scalars the laws read.  svk selects,
// in the finite-strain kernels, the finite-deformation elastic law
// (`elastic` with finite_deformation = true) instead of the neohookean one.
struct MatParams {
  double lambda, mu, sigma_y, h, sigma_th, rho;
  int svk;
  int c33;  // plane-stress neohookean: J includes the out-of-plane stretch sqrt(C33)
  // plastic law: thermal term of the trial stress, previous sigma_th minus
  // current sigma_th (material_linear_isotropic_hardening_inline_impl.hh:31-34)
  double dsth;
};

// ---- small dense algebra, column-major m[i + j*D] ---------------------------
template <class T> __device__ __forceinline__ T det2(const T *m) {
  return m[0] * m[3] - m[1] * m[2];
}
// first-row expansion, Eigen's bruteforce 3x3 determinant
template <class T> __device__ __forceinline__ T det3(const T *m) {
  return m[0] * (m[4] * m[8] - m[7] * m[5]) - m[3] * (m[1] * m[8] - m[7] * m[2]) +
         m[6] * (m[1] * m[5] - m[4] * m[2]);
}
template <class T> __device__ __forceinline__ T cof3(const T *m, int i, int j) {
  const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
  return m[i1 + 3 * j1] * m[i2 + 3 * j2] - m[i1 + 3 * j2] * m[i2 + 3 * j1];
}
// inverse through the adjugate: det from the first-column cofactors
template <class T> __device__ __forceinline__ void inv3(const T *m, T *r) {
  const T c0 = cof3(m, 0, 0), c1 = cof3(m, 1, 0), c2 = cof3(m, 2, 0);
  const T det = c0 * m[0] + c1 * m[1] + c2 * m[2];
  const T id = T(1) / det;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) r[i + 3 * j] = cof3(m, j, i) * id;
}
// adjugate r = det(m) m^-1 (r[i + 3 j] = cofactor (j, i)); returns det(m)
// from the first-column cofactors
template <class T> __device__ __forceinline__ T adj3(const T *m, T *r) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) r[i + 3 * j] = cof3(m, j, i);
  return r[0] * m[0] + r[3] * m[1] + r[6] * m[2];
}
template <class T> __device__ __forceinline__ void inv2(const T *m, T *r) {
  const T id = T(1) / det2(m);
  r[0] = m[3] * id;
  r[1] = -m[1] * id;
  r[2] = -m[2] * id;
  r[3] = m[0] * id;
}

// ---- constitutive laws --------------------------------------------------------
// sigma = 2 mu eps(g) + (lambda tr g + sigma_th) I
// (material_elastic_inline_impl.hh:31-48)
template <int D, class T>
__device__ __forceinline__ void elastic_stress(T lambda, T mu, const T *g, T sth, T *s) {
  T tr = g[0];
#pragma unroll
  for (int i = 1; i < D; ++i) tr = tr + g[i * (D + 1)];
  const T dia = lambda * tr + sth;
  const T two_mu = T(2) * mu;
#pragma unroll
  for (int j = 0; j < D; ++j)
#pragma unroll
    for (int i = 0; i < D; ++i) {
      const T eps = T(.5) * (g[j + D * i] + g[i + D * j]);
      const T v = two_mu * eps;
      s[i + D * j] = (i == j) ? v + dia : v;
    }
}

// S = mu I + (lambda ln J - mu) C^-1, F = I + grad u, C = F^T F, J = det F
// (times sqrt(C33) in plane stress, c33 > 0)
// (material_neohookean_inline_impl.hh:37-48, material_inline_impl.hh:33-81)
template <int D, class T>
__device__ __forceinline__ void neohookean_pk2(T lambda, T mu, const T *g, T *S, double c33 = 0.) {
  T F[D * D], C[D * D], Ci[D * D];
#pragma unroll
  for (int j = 0; j < D; ++j)
#pragma unroll
    for (int i = 0; i < D; ++i) F[i + D * j] = (i == j ? T(1) : T(0)) + g[i + D * j];
  // C is symmetric term by term (same products, same order): fill j >= i
#pragma unroll
  for (int j = 0; j < D; ++j)
#pragma unroll
    for (int i = 0; i <= j; ++i) {
      T s = F[0 + D * i] * F[0 + D * j];
#pragma unroll
      for (int k = 1; k < D; ++k) s = s + F[k + D * i] * F[k + D * j];
      C[i + D * j] = s;
      C[j + D * i] = s;
    }
  T J;
  if constexpr (D == 3) {
    J = det3(F);
    inv3(C, Ci);
  } else {
    J = det2(F);
    inv2(C, Ci);
  }
  // J * sqrt(C33); C33 = 1 in plane strain and 3D (the product is exact then)
  if (c33 > 0.) J = J * (T)sqrt(c33);
  const T c = lambda * log(J) - mu;
#pragma unroll
  for (int j = 0; j < D; ++j)
#pragma unroll
    for (int i = 0; i < D; ++i) {
      const T t = c * Ci[i + D * j];
      S[i + D * j] = (i == j) ? mu + t : t;
    }
}

// Green-Lagrange strain E = (g^T g + g^T + g) / 2 (material_inline_impl.hh:127-130)
template <int D, class T>
__device__ __forceinline__ void green_lagrange(const T *g, T *E) {
#pragma unroll
  for (int j = 0; j < D; ++j)
#pragma unroll
    for (int i = 0; i < D; ++i) {
      T s = g[0 + D * i] * g[0 + D * j];
#pragma unroll
      for (int k = 1; k < D; ++k) s = s + g[k + D * i] * g[k + D * j];
      E[i + D * j] = ((s + g[j + D * i]) + g[i + D * j]) / T(2);
    }
}

// out-of-plane right Cauchy-Green stretch of a plane-stress neohookean
// point: Newton iterations from the stored value x on
//   f(x) = lambda/2 (log x + log(C00 C11 - C01^2)) + mu (x - 1),
//   f'(x) = lambda / (2 x) + mu, tolerance 1e-5, at most 100 iterations
// (material_neohookean_inline_impl.hh:52-92, aka_math_tmpl.hh:191-208)
__device__ __forceinline__ double solve_c33(double lambda, double mu, double C00, double C11,
                                            double C01, double x) {
  const double lc = log(C00 * C11 - C01 * C01);
  double fx = lambda / 2. * (log(x) + lc) + mu * (x - 1.);
  for (int it = 0; fabs(fx) > 1e-5 && it < 100; ++it) {
    x -= fx / (lambda / (2. * x) + mu);
    fx = lambda / 2. * (log(x) + lc) + mu * (x - 1.);
  }
  return x;
}

// right Cauchy-Green entries of a 2D point, C = F^T F
template <class T>
__device__ __forceinline__ void right_cauchy2(const T *g, double *c00, double *c11, double *c01) {
  const T F00 = T(1) + g[0], F10 = g[1], F01 = g[2], F11 = T(1) + g[3];
  *c00 = (double)(F00 * F00 + F10 * F10);
  *c11 = (double)(F01 * F01 + F11 * F11);
  *c01 = (double)(F00 * F01 + F10 * F11);
}

// second Piola-Kirchhoff stress of a finite-strain material: the elastic law
// applied to E (MaterialElastic::computeStress with finite_deformation,
// material_elastic.cc:82-101), or the neohookean law (c33 > 0: plane stress)
template <int D, class T>
__device__ __forceinline__ void finite_pk2(const MatParams &mp, const T *g, T *S,
                                           double c33 = 0.) {
  if (mp.svk) {
    T E[D * D];
    green_lagrange<D, T>(g, E);
    elastic_stress<D, T>((T)mp.lambda, (T)mp.mu, E, (T)mp.sigma_th, S);
  } else {
    neohookean_pk2<D, T>((T)mp.lambda, (T)mp.mu, g, S, c33);
  }
}

// radial return with linear isotropic hardening, small strain
// (material_linear_isotropic_hardening_inline_impl.hh:28-84 and
//  material_plastic.hh computeStressAndInelasticStrainOnQuad)
template <int D>
__device__ __forceinline__ void plastic_update(double lambda, double mu, double sigma_y,
                                               double h, const double *g, const double *gp,
                                               const double *sp, const double *epp,
                                               double iso_cur, double iso_prev, double dsth,
                                               double *s, double *ep, double *iso) {
  constexpr int DD = D * D;
  double gdu[DD], str[DD], dev[9], deps[DD];
#pragma unroll
  for (int k = 0; k < DD; ++k) gdu[k] = g[k] - gp[k];
  elastic_stress<D, double>(lambda, mu, gdu, dsth, str);
#pragma unroll
  for (int k = 0; k < DD; ++k) str[k] = str[k] + sp[k];
  double tr = str[0];
#pragma unroll
  for (int i = 1; i < D; ++i) tr = tr + str[i * (D + 1)];
#pragma unroll
  for (int k = 0; k < 9; ++k) dev[k] = 0.;
#pragma unroll
  for (int j = 0; j < D; ++j)
#pragma unroll
    for (int i = 0; i < D; ++i) dev[i + 3 * j] = str[i + D * j];
  const double t3 = tr / 3.0;
#pragma unroll
  for (int i = 0; i < 3; ++i) dev[i * 4] = dev[i * 4] - t3;
  double ss = dev[0] * dev[0];
#pragma unroll
  for (int k = 1; k < 9; ++k) ss = ss + dev[k] * dev[k];
  const double eff = sqrt(3. / 2. * ss);
  const bool yield = (eff - iso_cur - sigma_y) > 0;
  const double dp = yield ? (eff - sigma_y - iso_prev) / (3 * mu + h) : 0.;
  *iso = iso_prev + h * dp;
  const double nrm = sqrt(ss);
  const double tol = 1e2 * 2.220446049250313080847e-16;  // Math::tolerance
#pragma unroll
  for (int k = 0; k < DD; ++k) deps[k] = 0.;
  if (fabs(eff) > nrm * tol) {
#pragma unroll
    for (int j = 0; j < D; ++j)
#pragma unroll
      for (int i = 0; i < D; ++i) deps[i + D * j] = dev[i + 3 * j] * 3. / 2. * dp / eff;
  }
  double ge[DD], sel[DD];
#pragma unroll
  for (int k = 0; k < DD; ++k) ge[k] = gdu[k] - deps[k];
  elastic_stress<D, double>(lambda, mu, ge, 0., sel);
#pragma unroll
  for (int k = 0; k < DD; ++k) {
    s[k] = sp[k] + sel[k];
    ep[k] = epp[k] + deps[k];
  }
}

// r_q(a*D + k) = sum_I (B_L0 + B_L2(grad u))(I, a*D + k) S_voigt(I)
// (material.cc:547-565, aka_voigthelper_tmpl.hh:99-140,180-235).
// The reference builds the full 6 x 3n matrices; here the entries that are
// structurally zero are not added (x + 0 == x), every non-zero term keeps its
// operand order, so the result is the same number.  k must be a compile-time
// constant after unrolling.
template <int D, class T>
__device__ __forceinline__ T finite_force_component(const T *b /* dN_a/dx */, const T *g,
                                                    const T *Sv, int k) {
  if constexpr (D == 3) {
    // rows 0..2: B_L0(I, k) = b_I if k == I; B_L2(I, k) = g(k, I) b_I
    T bf[6];
#pragma unroll
    for (int I = 0; I < 3; ++I) {
      const T bl2 = g[k + 3 * I] * b[I];
      bf[I] = (k == I) ? b[I] + bl2 : bl2;
    }
    // shear rows: B_L2(3+aux, k) = sum_{m != aux} g(k, m) b_{3-m-aux}
    const T s3 = g[k + 3 * 1] * b[2] + g[k + 3 * 2] * b[1];
    const T s4 = g[k + 3 * 0] * b[2] + g[k + 3 * 2] * b[0];
    const T s5 = g[k + 3 * 0] * b[1] + g[k + 3 * 1] * b[0];
    bf[3] = (k == 1) ? b[2] + s3 : ((k == 2) ? b[1] + s3 : s3);
    bf[4] = (k == 0) ? b[2] + s4 : ((k == 2) ? b[0] + s4 : s4);
    bf[5] = (k == 0) ? b[1] + s5 : ((k == 1) ? b[0] + s5 : s5);
    T acc = bf[0] * Sv[0];
#pragma unroll
    for (int I = 1; I < 6; ++I) acc = acc + bf[I] * Sv[I];
    return acc;
  } else {
    T bf[3];
#pragma unroll
    for (int I = 0; I < 2; ++I) {
      const T bl2 = g[k + 2 * I] * b[I];
      bf[I] = (k == I) ? b[I] + bl2 : bl2;
    }
    const T s2 = g[k + 2 * 0] * b[1] + g[k + 2 * 1] * b[0];
    bf[2] = ((k == 1) ? b[0] : b[1]) + s2;
    T acc = bf[0] * Sv[0];
    acc = acc + bf[1] * Sv[1];
    acc = acc + bf[2] * Sv[2];
    return acc;
  }
}

// first Piola-Kirchhoff form of the same force, P = F S, r(a, k) = P(k, :) . dN_a/dx,
// used by the mixed-precision path (equal in exact arithmetic, fewer operations)
template <int D, class T>
__device__ __forceinline__ void first_piola(const T *g, const T *S, T w, T *P) {
#pragma unroll
  for (int J = 0; J < D; ++J)
#pragma unroll
    for (int k = 0; k < D; ++k) {
      T s = S[k + D * J];
#pragma unroll
      for (int m = 0; m < D; ++m) s += g[k + D * m] * S[m + D * J];
      P[k + D * J] = s * w;
    }
}

// Weighted first Piola-Kirchhoff stress of the neohookean law for the
// mixed-precision path,
//   P = F S = mu F + (lambda ln J - mu) F^-T = mu F + c cof(F),
//   c = (lambda ln J - mu) / det F   (F C^-1 = F^-T = cof(F) / det F),
// the same tensor as first_piola(g, neohookean_pk2(g)) in exact arithmetic,
// written in the displacement gradient H = F - I so that the O(1) parts
// cancel analytically and small strains keep FP32's relative precision
// (forming mu F and c cof(F) separately loses it: their identity parts cancel
// to O(|H|)).  With t = tr H:
//   3D (Cayley-Hamilton): cof(I + H) = I + K^T, K = (t + i2) I - (1 + t) H + H^2,
//      i2 = (t^2 - tr H^2) / 2,  det F - 1 = t + i2 + det H;
//   2D: cof(I + H) = I + K^T, K = t I - H,  det F - 1 = t + det H;
//   P = (mu + c) I + mu H + c K^T,  mu + c = (mu (det F - 1) + lambda ln J) / det F,
//   ln J = log1p(det F - 1) (+ ln C33 / 2 in plane stress).
// explicitly rounded operations (never contracted or split by the compiler,
// whatever the launch shape's register budget), FP32 and FP64
__device__ __forceinline__ float op_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float op_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float op_fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double op_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double op_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double op_fma(double a, double b, double c) { return __fma_rn(a, b, c); }

template <int D, class T>
__device__ __forceinline__ void neohookean_piola(T lambda, T mu, const T *g, T w, T *P,
                                                 double c33 = 0.) {
  T K[D * D];
  T dm1;
  if constexpr (D == 3) {
    T H2[9];
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
      for (int i = 0; i < 3; ++i)
        H2[i + 3 * j] = op_fma(g[i + 6], g[2 + 3 * j],
                               op_fma(g[i + 3], g[1 + 3 * j], op_mul(g[i], g[3 * j])));
    const T t = op_add(op_add(g[0], g[4]), g[8]);
    const T trH2 = op_add(op_add(H2[0], H2[4]), H2[8]);
    const T i2 = op_mul(T(0.5), op_fma(t, t, -trH2));
    const T m0 = op_fma(g[4], g[8], -op_mul(g[5], g[7]));
    const T m1 = op_fma(g[1], g[8], -op_mul(g[2], g[7]));
    const T m2 = op_fma(g[1], g[5], -op_mul(g[2], g[4]));
    const T detH = op_fma(g[6], m2, op_fma(-g[3], m1, op_mul(g[0], m0)));
    dm1 = op_add(op_add(t, i2), detH);
    const T a = op_add(t, i2), b = op_add(T(1), t);
#pragma unroll
    for (int k = 0; k < 9; ++k) K[k] = op_fma(-b, g[k], H2[k]);
    K[0] = op_add(K[0], a);
    K[4] = op_add(K[4], a);
    K[8] = op_add(K[8], a);
  } else {
    const T t = op_add(g[0], g[3]);
    dm1 = op_add(t, op_fma(g[0], g[3], -op_mul(g[1], g[2])));
#pragma unroll
    for (int k = 0; k < 4; ++k) K[k] = -g[k];
    K[0] = op_add(K[0], t);
    K[3] = op_add(K[3], t);
  }
  const T det = op_add(T(1), dm1);
  T lnJ = log1p(dm1);
  if (c33 > 0.) lnJ = op_add(lnJ, (T)(0.5 * log(c33)));
  const T rdet = T(1) / det;
  const T c = op_mul(op_fma(lambda, lnJ, -mu), rdet);
  const T a0 = op_mul(op_fma(mu, dm1, op_mul(lambda, lnJ)), rdet);
#pragma unroll
  for (int j = 0; j < D; ++j)
#pragma unroll
    for (int i = 0; i < D; ++i) {
      T p = op_fma(c, K[j + D * i], op_mul(mu, g[i + D * j]));
      if (i == j) p = op_add(p, a0);
      P[i + D * j] = op_mul(w, p);
    }
}

template <int D, class T> __device__ __forceinline__ void to_voigt(const T *S, T *Sv) {
  if constexpr (D == 3) {
    Sv[0] = S[0]; Sv[1] = S[4]; Sv[2] = S[8];
    Sv[3] = S[1 + 3 * 2]; Sv[4] = S[0 + 3 * 2]; Sv[5] = S[0 + 3 * 1];
  } else {
    Sv[0] = S[0]; Sv[1] = S[3]; Sv[2] = S[0 + 2 * 1];
  }
}

}  // namespace akb

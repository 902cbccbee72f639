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

// Lame constants and the per-material scalars the laws read
struct MatParams {
  double lambda, mu, sigma_y, h, sigma_th, rho;
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

// S = mu I + (lambda ln J - mu) C^-1, F = I + grad u, C = F^T F
// (material_neohookean_inline_impl.hh:37-48, material_inline_impl.hh:33-81)
template <int D, class T>
__device__ __forceinline__ void neohookean_pk2(T lambda, T mu, const T *g, T *S) {
  T F[D * D], C[D * D], Ci[D * D];
#pragma unroll
  for (int j = 0; j < D; ++j)
#pragma unroll
    for (int i = 0; i < D; ++i) F[i + D * j] = (i == j ? T(1) : T(0)) + g[i + D * j];
#pragma unroll
  for (int j = 0; j < D; ++j)
#pragma unroll
    for (int i = 0; i < D; ++i) {
      T s = F[0 + D * i] * F[0 + D * j];
#pragma unroll
      for (int k = 1; k < D; ++k) s = s + F[k + D * i] * F[k + D * j];
      C[i + D * j] = s;
    }
  T J;
  if constexpr (D == 3) {
    J = det3(F);
    inv3(C, Ci);
  } else {
    J = det2(F);
    inv2(C, Ci);
  }
  // J * sqrt(C33) with C33 = 1 (plane strain / 3D)
  const T c = lambda * log(J) - mu;
#pragma unroll
  for (int j = 0; j < D; ++j)
#pragma unroll
    for (int i = 0; i < D; ++i) {
      const T t = c * Ci[i + D * j];
      S[i + D * j] = (i == j) ? mu + t : t;
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
// (material.cc:547-565, aka_voigthelper_tmpl.hh:99-140,180-235)
template <int D, class T>
__device__ __forceinline__ T finite_force_component(const T *b /* dN_a/dx */, const T *g,
                                                    const T *Sv, int k) {
  T acc = T(0);
  if constexpr (D == 3) {
#pragma unroll
    for (int I = 0; I < 6; ++I) {
      T bl0 = T(0), bl2;
      if (I < 3) {
        if (k == I) bl0 = b[I];
        bl2 = g[k + 3 * I] * b[I];
      } else {
        if (I == 3) { if (k == 1) bl0 = b[2]; else if (k == 2) bl0 = b[1]; }
        if (I == 4) { if (k == 0) bl0 = b[2]; else if (k == 2) bl0 = b[0]; }
        if (I == 5) { if (k == 0) bl0 = b[1]; else if (k == 1) bl0 = b[0]; }
        const int aux = I - 3;
        bl2 = T(0);
#pragma unroll
        for (int m = 0; m < 3; ++m)
          if (m != aux) bl2 += g[k + 3 * m] * b[3 - m - aux];
      }
      const T bf = bl0 + bl2;
      acc = (I == 0) ? bf * Sv[I] : acc + bf * Sv[I];
    }
  } else {
#pragma unroll
    for (int I = 0; I < 3; ++I) {
      T bl0 = T(0), bl2;
      if (I < 2) {
        if (k == I) bl0 = b[I];
        bl2 = g[k + 2 * I] * b[I];
      } else {
        bl0 = (k == 1) ? b[0] : b[1];
        bl2 = T(0);
#pragma unroll
        for (int m = 0; m < 2; ++m) bl2 += g[k + 2 * m] * b[1 - m];
      }
      const T bf = bl0 + bl2;
      acc = (I == 0) ? bf * Sv[I] : acc + bf * Sv[I];
    }
  }
  return acc;
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

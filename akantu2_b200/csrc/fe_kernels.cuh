// Kernel templates of the explicit step.  Instantiated by kernels_fp64.cu
// (T = double, compiled --fmad=false) and kernels_mixed.cu (T = float).
//
// HBM layout (all arrays in internal element order: elements grouped by
// material, ascending original id inside a material):
//   conn  int32 [NN][E]              node ids, component-major
//   B     T     [NQ][NN*D][E]        dN_a/dx_j of point q at ((q*NN + a)*D + j)*E + e
//   wJ    T     [NQ][E]              det J * w_q
//   per-material quadrature-point internals [NQ][comp][ne] (element fastest)
//   re    RT    [E*NN][D]            elemental internal force, read by the
//                                    node gather in ascending slot order
//   u,v,a,fext,fint double [N][D]    user node order (reference layout)
//   mass  double [N]                 one lumped mass per node
//   blocked uint8 [N]                bit c = component c blocked
// The node -> slot CSR (ptr [N+1], ent [E*NN]) lists slots (e*NN + a) in
// increasing order, which is the order of the reference's serial scatter
// (dof_manager.cc:65-120), so the gather reproduces its sums exactly.
#pragma once

#include "fe_device.cuh"

namespace akb {

constexpr int kMaxNQ = 8;
constexpr int kMaxNN = 8;

// Programmatic dependent launch of the step kernels: a step kernel launched
// with the programmatic-serialization attribute may start while the kernel
// before it on the stream finishes; it waits here (griddepcontrol.wait)
// until that kernel has completed and its writes are visible, before it
// reads anything.  Kernels of at most kEarlyTriggerBlocks blocks (one wave)
// let the next kernel launch at once; larger grids let it launch when they
// end, so that its waiting blocks do not hold SM slots their later waves
// need.  Without the attribute both instructions do nothing.
constexpr unsigned kEarlyTriggerBlocks = 1184;  // 148 SMs x 8
__device__ __forceinline__ void pdl_begin() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  if (gridDim.x * gridDim.y <= kEarlyTriggerBlocks)
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// L2 prefetch (cp.async.bulk.prefetch.L2: nothing reaches the SM) of the
// bytes [lo, hi) of an array occupying [base, end).  The range is widened to
// 16-byte boundaries, as the instruction requires, and clipped to the
// array's own 16-byte-aligned span, so no byte outside the array is named.
__device__ __forceinline__ void prefetch_l2(const void *base, const void *end, const void *lo,
                                            const void *hi) {
  const uint64_t b0 = ((uint64_t)__cvta_generic_to_global(base) + 15) & ~(uint64_t)15;
  const uint64_t b1 = (uint64_t)__cvta_generic_to_global(end) & ~(uint64_t)15;
  uint64_t a = (uint64_t)__cvta_generic_to_global(lo) & ~(uint64_t)15;
  uint64_t z = ((uint64_t)__cvta_generic_to_global(hi) + 15) & ~(uint64_t)15;
  if (a < b0) a = b0;
  if (z > b1) z = b1;
  if (z > a)
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"((unsigned)(z - a))
                 : "memory");
}

// natural-coordinate tables evaluated on the host (passed by value: they sit
// in the kernel-parameter constant bank)
struct QuadTable {
  double dnds[kMaxNQ * 3 * kMaxNN];  // [q][k][a]
  double N[kMaxNQ * kMaxNN];         // [q][a]
  double w[kMaxNQ];
  float fdnds[kMaxNQ * 3 * kMaxNN];  // FP32 copies for the mixed path
  float fw[kMaxNQ];
};

// elemental-force slots: the D components of one (element, node) force at
// slot p.  FP32 3D slots are padded to one 16-byte float4 (one vector store
// in the element kernel, one vector load in the node gather); the others
// hold D values without padding.  Unpadded 12-byte slots (three scalar
// stores, the node's range read in aligned 16-byte chunks) were measured: the
// element launches took 58 % (128^3 hexahedra) and 55 % (tet batch) longer,
// for a 5 % shorter hexahedral node update and a 15 % longer batch one.
template <int D, class RT> struct SlotStride {
  static constexpr int value = (D == 3 && sizeof(RT) == 4) ? 4 : D;
};

template <int D, class RT, class V>
__device__ __forceinline__ void store_slot(RT *re, int64_t p, const V *v) {
  if constexpr (SlotStride<D, RT>::value == 4) {
    reinterpret_cast<float4 *>(re)[p] = make_float4((float)v[0], (float)v[1], (float)v[2], 0.f);
  } else {
#pragma unroll
    for (int i = 0; i < D; ++i) re[p * D + i] = (RT)v[i];
  }
}
// plain loads: the compiler uses the read-only path where the kernel's
// parameters allow it, and coherent loads in the persistent kernel, which
// writes the slots in the same launch
template <int D, class RT>
__device__ __forceinline__ void load_slot(const RT *re, int64_t p, double *v) {
  if constexpr (SlotStride<D, RT>::value == 4) {
    const float4 f = reinterpret_cast<const float4 *>(re)[p];
    v[0] = (double)f.x;
    v[1] = (double)f.y;
    v[2] = (double)f.z;
  } else {
#pragma unroll
    for (int i = 0; i < D; ++i) v[i] = (double)re[p * D + i];
  }
}

// per-material plastic internals, [q][comp][ne], ping-pong prev/cur
// One launch covers a law group: the elements of all materials with the same
// law, contiguous in internal order.  With several materials, each element
// reads its parameters from mtab[mslot[le]]; with one, from the launch's
// MatParams.  Plastic internals of the group are [q][comp][ne] arrays,
// ping-pong prev / cur.  The stress and the plastic strain are symmetric
// term by term (every expression that forms them is), so they keep their
// SymComps<D> independent components; the previous displacement gradient
// is stored in the element-math type (FP32 on the mixed path, where it is
// an FP32 value to begin with).
struct GroupArgs {
  const MatParams *mtab;     // per-material parameters, or null
  const int32_t *mslot;      // [ne] index into mtab
  const double *sig_prev, *eps_prev, *iso_prev;
  const void *gu_prev;       // double (FP64 path) or float (mixed path)
  const double *iso_cur_in;  // "current" hardening read by the yield test
  double *sig, *eps, *iso;
  void *gu;
  double *pe;                // cumulative plastic energy density
  double *c33;               // [q][ne] plane-stress neohookean out-of-plane stretch
                             // (updated in place by every stress evaluation), or null
  int update_energy;         // 1 inside solveStep (afterSolveStep), 0 otherwise
  // eigen gradient of the displacement [q][d*d][ne] (double), subtracted from
  // the gradient before the law (material.cc:147), or null when zero
  const double *eig;
  // batches whose instances stop after their own step counts: instance of
  // each element of the launch [ne], the step count at which each instance
  // stops, and the device's step counter (all null otherwise)
  const int32_t *einst;
  const int64_t *inst_end;
  const int64_t *step;
  // index checks of the bounds-checking build (AKB_BOUNDS_CHECK): node count,
  // slot count and the model's status word
  int64_t nb_nodes, nb_slots;
  unsigned int *status;
};

// AKB_BOUNDS_CHECK builds check every index an element reads before using it:
// node ids in [0, nb_nodes), slot positions in [0, nb_slots); an element with
// an index out of range sets status bit 2 and is skipped (no access through
// the bad index)
constexpr unsigned int ST_INDEX_RANGE = 4u;
template <int NN>
__device__ __forceinline__ bool element_indices_ok(const GroupArgs &ps, const int32_t *conn,
                                                   const int32_t *pos, int64_t E, int64_t e) {
#ifdef AKB_BOUNDS_CHECK
  bool ok = true;
#pragma unroll
  for (int a = 0; a < NN; ++a) {
    const int32_t n = conn[(int64_t)a * E + e], p = pos[(int64_t)a * E + e];
    ok = ok && n >= 0 && n < ps.nb_nodes && p >= 0 && p < ps.nb_slots;
  }
  if (!ok && ps.status) atomicOr(ps.status, ST_INDEX_RANGE);
  return ok;
#else
  (void)ps, (void)conn, (void)pos, (void)E, (void)e;
  return true;
#endif
}

// the element's instance still advances in this step
__device__ __forceinline__ bool element_active(const GroupArgs &ps, int64_t le) {
  return !ps.inst_end || *ps.step < ps.inst_end[ps.einst[le]];
}

// grad u -= eigen_grad_u at point (le, q) of a launch over ne elements
template <int D, class T>
__device__ __forceinline__ void subtract_eigen(const GroupArgs &ps, int64_t ne, int64_t le, int q,
                                               T *g) {
  if (ps.eig) {
#pragma unroll
    for (int k = 0; k < D * D; ++k) g[k] = g[k] - (T)ps.eig[(int64_t)(q * D * D + k) * ne + le];
  }
}

// plane-stress C33 of point (le, q), solved from its stored value and stored
// back (PlaneStressToolbox::computeStress runs computeThirdAxisDeformation on
// every stress evaluation, plane_stress_toolbox_tmpl.hh:68-74); 0 otherwise
template <int D, class T>
__device__ __forceinline__ double point_c33(const MatParams &mp, const GroupArgs &ps, int64_t ne,
                                            int64_t le, int q, const T *g) {
  if constexpr (D == 2) {
    if (mp.c33 && ps.c33) {
      double c00, c11, c01;
      right_cauchy2<T>(g, &c00, &c11, &c01);
      double *p = ps.c33 + (int64_t)q * ne + le;
      const double x = solve_c33(mp.lambda, mp.mu, c00, c11, c01, *p);
      *p = x;
      return x;
    }
  }
  return 0.;
}

// symmetric d x d tensors: components (0,0), (1,1), (2,2), (1,2), (0,2), (0,1)
// in 3D, (0,0), (1,1), (0,1) in 2D
template <int D> struct SymComps { static constexpr int value = D == 3 ? 6 : 3; };
// component of column-major entry k = i + D j
template <int D> __host__ __device__ constexpr int sym_of(int k) {
  return D == 3 ? (k == 0 ? 0 : k == 4 ? 1 : k == 8 ? 2 : (k == 5 || k == 7) ? 3
                  : (k == 2 || k == 6) ? 4 : 5)
                : (k == 0 ? 0 : k == 3 ? 1 : 2);
}
// column-major entry stored for component c
template <int D> __host__ __device__ constexpr int full_of(int c) {
  return D == 3 ? (c == 0 ? 0 : c == 1 ? 4 : c == 2 ? 8 : c == 3 ? 7 : c == 4 ? 6 : 3)
                : (c == 0 ? 0 : c == 1 ? 3 : 2);
}

__device__ __forceinline__ MatParams group_params(const MatParams &mp, const GroupArgs &ga,
                                                  int64_t le) {
  return ga.mtab ? ga.mtab[ga.mslot[le]] : mp;
}

// ---------------------------------------------------------------------------
// K0: dN/dx and det J * w  (element_class_tmpl.hh:296-395,
// integrator_gauss_inline_impl.hh:176-195,378-398).
//
// point_geometry: one quadrature point from the element's nodal coordinates
// Xe [NN][D] and dN/ds at the point, dn(k, a): J = dN/ds X, det J
// by first-row expansion, J^-1 through the adjugate (det from the
// first-column cofactors), dN/dx = J^-1 dN/ds, wJ = det J w.  Every product,
// sum and quotient is explicitly rounded, so the translation units built with
// and without contraction compute the same bits: the step kernels that
// recompute the geometry instead of streaming it reproduce the precomputed
// tables exactly.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double cof3_rn(const double *m, int i, int j) {
  const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
  return sub_rn(mul_rn(m[i1 + 3 * j1], m[i2 + 3 * j2]), mul_rn(m[i1 + 3 * j2], m[i2 + 3 * j1]));
}
template <int D, int NN, class DN>
__device__ __forceinline__ double point_geometry(const double *Xe, const DN &dn, double w,
                                                 double *Bq, double *wJq) {
  double J[D * D], Ji[D * D];
#pragma unroll
  for (int k = 0; k < D; ++k)
#pragma unroll
    for (int j = 0; j < D; ++j) {
      double s = mul_rn(dn(k, 0), Xe[j]);
#pragma unroll
      for (int a = 1; a < NN; ++a) s = add_rn(s, mul_rn(dn(k, a), Xe[a * D + j]));
      J[k + D * j] = s;
    }
  double det;
  if constexpr (D == 3) {
    const double *m = J;
    det = add_rn(sub_rn(mul_rn(m[0], sub_rn(mul_rn(m[4], m[8]), mul_rn(m[7], m[5]))),
                        mul_rn(m[3], sub_rn(mul_rn(m[1], m[8]), mul_rn(m[7], m[2])))),
                 mul_rn(m[6], sub_rn(mul_rn(m[1], m[5]), mul_rn(m[4], m[2]))));
    const double c0 = cof3_rn(m, 0, 0), c1 = cof3_rn(m, 1, 0), c2 = cof3_rn(m, 2, 0);
    const double dc = add_rn(add_rn(mul_rn(c0, m[0]), mul_rn(c1, m[1])), mul_rn(c2, m[2]));
    const double id = __ddiv_rn(1., dc);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) Ji[i + 3 * j] = mul_rn(cof3_rn(m, j, i), id);
  } else {
    det = sub_rn(mul_rn(J[0], J[3]), mul_rn(J[1], J[2]));
    const double id = __ddiv_rn(1., det);
    Ji[0] = mul_rn(J[3], id);
    Ji[1] = mul_rn(-J[1], id);
    Ji[2] = mul_rn(-J[2], id);
    Ji[3] = mul_rn(J[0], id);
  }
#pragma unroll
  for (int a = 0; a < NN; ++a)
#pragma unroll
    for (int j = 0; j < D; ++j) {
      double s = mul_rn(Ji[j], dn(0, a));
#pragma unroll
      for (int k = 1; k < D; ++k) s = add_rn(s, mul_rn(Ji[j + D * k], dn(k, a)));
      Bq[a * D + j] = s;
    }
  *wJq = mul_rn(det, w);
  return det;
}

// dN/ds at one point: the host-evaluated table of the element type
struct TableDn {
  const double *p;  // dnds of the point, [k][kMaxNN]
  __device__ __forceinline__ double operator()(int k, int a) const { return p[k * kMaxNN + a]; }
};
// dN/ds of the linear tetrahedron (the same at every point; N3 = xi, N1 =
// eta, N2 = zeta, N0 = 1 - xi - eta - zeta) at compile time: the products
// with its 1 and -1 entries fold to exact copies and negations, its 0 entries
// stay multiplications (0 x X keeps the signs of zeros the table-driven sums
// give), so it computes what TableDn over the tetrahedron's table computes
struct Tet4Dn {
  __device__ __forceinline__ constexpr double operator()(int k, int a) const {
    return a == 0 ? -1. : (a == (k == 0 ? 3 : k) ? 1. : 0.);
  }
};

// One thread per (e, q), element fastest.  bad receives the smallest
// e*NQ + q with det J < 0.
template <int D, int NN, int NQ>
__global__ void k_precompute(const double *__restrict__ X, const int32_t *__restrict__ conn,
                             int64_t E, QuadTable tab, double *__restrict__ B,
                             double *__restrict__ wJ, unsigned long long *__restrict__ bad) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= E * NQ) return;
  const int q = (int)(t / E);
  const int64_t e = t - (int64_t)q * E;
  double Xe[NN * D];
#pragma unroll
  for (int a = 0; a < NN; ++a) {
    const int64_t node = conn[(int64_t)a * E + e];
#pragma unroll
    for (int i = 0; i < D; ++i) Xe[a * D + i] = X[node * D + i];
  }
  double Bq[NN * D], wq;
  const double det =
      point_geometry<D, NN>(Xe, TableDn{&tab.dnds[q * 3 * kMaxNN]}, tab.w[q], Bq, &wq);
#pragma unroll
  for (int c = 0; c < NN * D; ++c) B[(int64_t)(q * NN * D + c) * E + e] = Bq[c];
  if (det < 0) atomicMin(bad, (unsigned long long)(e * NQ + q));
  wJ[t] = wq;
}

// ---------------------------------------------------------------------------
// K1a: elemental lumped mass into the slot array (ncomp 1)
// row sum sum_q (rho N_a(q)) wJ_q, or for _triangle_6 rho V_e * (1/12 | 1/4)
// (fe_engine_template_tmpl_field.hh:112-242)
template <int NN, int NQ, bool DIAG>
__global__ void k_mass_elem(int64_t e_begin, int64_t e_count, int64_t E, double rho,
                            QuadTable tab, const double *__restrict__ wJ,
                            double *__restrict__ me) {
  const int64_t le = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (le >= e_count) return;
  const int64_t e = e_begin + le;
  if constexpr (DIAG) {
    double vol = rho * wJ[e];
#pragma unroll
    for (int q = 1; q < NQ; ++q) vol = vol + rho * wJ[q * E + e];
#pragma unroll
    for (int a = 0; a < NN; ++a) me[e * NN + a] = vol * (a < 3 ? 1. / 12. : 1. / 4.);
  } else {
#pragma unroll
    for (int a = 0; a < NN; ++a) {
      double acc = rho * tab.N[a] * wJ[e];
#pragma unroll
      for (int q = 1; q < NQ; ++q) acc = acc + rho * tab.N[q * kMaxNN + a] * wJ[q * E + e];
      me[e * NN + a] = acc;
    }
  }
}

// K1b: M_i = sum over the node's slots, ascending
static __global__ void k_gather_scalar(int64_t N, const int32_t *__restrict__ ptr,
                                const int32_t *__restrict__ ent, const double *__restrict__ me,
                                double *__restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double acc = 0.;
  for (int32_t p = ptr[i]; p < ptr[i + 1]; ++p) acc += 1. * me[ent[p]];
  out[i] = acc;
}

// ---------------------------------------------------------------------------
// K2: element inradius / celerity at the current position X + u
// (solid_mechanics_model.cc:436-473, fe_engine_inline_impl.hh:35-45)
__device__ __forceinline__ double dist3(const double *a, const double *b) {
  double s = 0;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    double t = a[i] - b[i];
    s += t * t;
  }
  return sqrt(s);
}
__device__ __forceinline__ double dist2(const double *a, const double *b) {
  double s = 0;
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    double t = a[i] - b[i];
    s += t * t;
  }
  return sqrt(s);
}
__device__ __forceinline__ double det3cols(const double *c0, const double *c1,
                                           const double *c2) {
  double m[9] = {c0[0], c0[1], c0[2], c1[0], c1[1], c1[2], c2[0], c2[1], c2[2]};
  return det3(m);
}
template <int ET> __device__ double element_inradius(const double *X);
template <> __device__ inline double element_inradius<ET_TET4>(const double *X) {
  const double *p1 = X, *p2 = X + 3, *p3 = X + 6, *p4 = X + 9;
  double l12 = dist3(p1, p2), l13 = dist3(p1, p3), l14 = dist3(p1, p4);
  double l23 = dist3(p2, p3), l24 = dist3(p2, p4), l34 = dist3(p3, p4);
  double s1 = (l12 + l23 + l13) * 0.5;
  s1 = sqrt(s1 * (s1 - l12) * (s1 - l23) * (s1 - l13));
  double s2 = (l12 + l24 + l14) * 0.5;
  s2 = sqrt(s2 * (s2 - l12) * (s2 - l24) * (s2 - l14));
  double s3 = (l23 + l34 + l24) * 0.5;
  s3 = sqrt(s3 * (s3 - l23) * (s3 - l34) * (s3 - l24));
  double s4 = (l13 + l34 + l14) * 0.5;
  s4 = sqrt(s4 * (s4 - l13) * (s4 - l34) * (s4 - l14));
  double vol = det3cols(p2, p3, p4);
  vol -= det3cols(p1, p3, p4);
  vol += det3cols(p1, p2, p4);
  vol -= det3cols(p1, p2, p3);
  vol /= 6;
  return 2. * (3 * vol / (s1 + s2 + s3 + s4));
}
template <> __device__ inline double element_inradius<ET_HEX8>(const double *X) {
  const int ed[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {0, 4}, {1, 5},
                         {2, 6}, {3, 7}, {4, 5}, {5, 6}, {6, 7}, {7, 4}};
  double p = dist3(X + 3 * ed[0][0], X + 3 * ed[0][1]);
#pragma unroll
  for (int k = 1; k < 12; ++k) p = fmin(p, dist3(X + 3 * ed[k][0], X + 3 * ed[k][1]));
  return p;
}
template <> __device__ inline double element_inradius<ET_TRI6>(const double *X) {
  const int tr[4][3] = {{0, 3, 5}, {3, 1, 4}, {3, 4, 5}, {5, 4, 2}};
  double r = 1.7976931348623157e308;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const double *p1 = X + 2 * tr[k][0], *p2 = X + 2 * tr[k][1], *p3 = X + 2 * tr[k][2];
    double a = dist2(p1, p2), b = dist2(p2, p3), c = dist2(p1, p3);
    double s = (a + b + c) / 2.;
    r = fmin(sqrt((s - a) * (s - b) * (s - c) / s), r);
  }
  return 2. * r;
}

// out[perm ? perm[e] : e] = h_e / c
template <int ET, int D, int NN>
__global__ void k_element_dt(int64_t e_begin, int64_t e_count, int64_t E, double celerity,
                             const int32_t *__restrict__ conn, const double *__restrict__ X,
                             const double *__restrict__ u, const int32_t *__restrict__ perm,
                             double *__restrict__ out) {
  const int64_t le = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (le >= e_count) return;
  const int64_t e = e_begin + le;
  double Xe[NN * D];
#pragma unroll
  for (int a = 0; a < NN; ++a) {
    const int64_t node = conn[(int64_t)a * E + e];
#pragma unroll
    for (int i = 0; i < D; ++i) Xe[a * D + i] = X[node * D + i] + u[node * D + i];
  }
  out[perm ? (int64_t)perm[e] : e] = element_inradius<ET>(Xe) / celerity;
}

// minimum of each segment [off[k], off[k+1]) of x, one block per segment
static __global__ void k_segment_min(const double *__restrict__ x, const int64_t *__restrict__ off,
                                     double *__restrict__ out) {
  __shared__ double sm[256];
  const int k = blockIdx.x;
  double acc = 1.7976931348623157e308;
  for (int64_t i = off[k] + threadIdx.x; i < off[k + 1]; i += blockDim.x) acc = fmin(acc, x[i]);
  sm[threadIdx.x] = acc;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sm[threadIdx.x] = fmin(sm[threadIdx.x], sm[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[k] = sm[0];
}

// time step of node i: one value for the model, or the value of the node's
// instance when several independent meshes advance together
__device__ __forceinline__ double node_dt(double dt, const int32_t *node_inst,
                                          const double *inst_dt, int64_t i) {
  return node_inst ? inst_dt[node_inst[i]] : dt;
}

// ---------------------------------------------------------------------------
// K3: NewmarkBeta::predictor, alpha = 0, beta = 1/2 (newmark-beta.cc:47-76)
//   u_pred = u + (dt v + (dt/2)(dt a)) on non-blocked dofs, u elsewhere.
// The displacement goes to a second buffer; the predicted velocity v + dt a is
// formed again by the node update (same arithmetic), so v and a keep the
// corrected values of the last step.  Only launched when the prediction made
// by the previous node update is not valid (first step, or the host wrote u,
// v, a, the blocked dofs or the time step in between).
template <int D>
__global__ void k_predict(int64_t N, const uint8_t *__restrict__ blocked,
                          const double *__restrict__ u, const double *__restrict__ v,
                          const double *__restrict__ a, double dt,
                          const int32_t *__restrict__ node_inst,
                          const double *__restrict__ inst_dt, double *__restrict__ u_pred) {
  pdl_begin();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N * D) return;
  const int64_t node = i / D;
  const int c = (int)(i - node * D);
  if ((blocked[node] >> c) & 1) {
    u_pred[i] = u[i];
    return;
  }
  dt = node_dt(dt, node_inst, inst_dt, node);
  const double hdt = .5 * dt;
  const double dta = dt * a[i];
  u_pred[i] = u[i] + (dt * v[i] + hdt * dta);
}

// ---------------------------------------------------------------------------
// K4: gradient at quadrature points, material law, B^T sigma integration.
//
// element_law<...>() evaluates one (element, quadrature point): the gradient
// u B^T, the law, and the weighted elemental force t = (B^T sigma or
// B(grad u)^T S) * wJ_q.  Two launch shapes use it:
//  - k_element_forces_pe: one thread per element, loop over q, accumulate t
//    in registers in increasing q (mixed tetrahedra and triangles; FP64 tet4
//    / tri6);
//  - k_element_forces_pq: one thread per (element, q) for FP64 hexahedra,
//    32 elements per warp (lanes = elements, warps = quadrature points), the
//    per-q contributions summed in increasing q through shared memory laid
//    out [q][component][lane], which is free of bank conflicts.

// plastic internals of one quadrature point: loads previous state, runs the
// radial return, stores the new state (and the plastic energy in a step)
// GT: storage type of the displacement gradient (the element-math type)
template <int D, class GT>
__device__ __forceinline__ void plastic_point(const MatParams &mp, const GroupArgs &ps,
                                              int64_t ne, int64_t le, int q,
                                              const double *gd, double *s) {
  constexpr int DD = D * D, NS = SymComps<D>::value;
  const GT *gu_prev = static_cast<const GT *>(ps.gu_prev);
  double gp[DD], sp[DD], epp[DD], ep[DD], iso;
  double sps[NS], epps[NS];
#pragma unroll
  for (int k = 0; k < DD; ++k) gp[k] = (double)gu_prev[(int64_t)(q * DD + k) * ne + le];
#pragma unroll
  for (int c = 0; c < NS; ++c) {
    const int64_t idx = (int64_t)(q * NS + c) * ne + le;
    sps[c] = ps.sig_prev[idx];
    epps[c] = ps.eps_prev[idx];
  }
#pragma unroll
  for (int k = 0; k < DD; ++k) {
    sp[k] = sps[sym_of<D>(k)];
    epp[k] = epps[sym_of<D>(k)];
  }
  const int64_t qi = (int64_t)q * ne + le;
  plastic_update<D>(mp.lambda, mp.mu, mp.sigma_y, mp.h, gd, gp, sp, epp, ps.iso_cur_in[qi],
                    ps.iso_prev[qi], mp.dsth, s, ep, &iso);
  if (ps.update_energy) {
    // MaterialPlastic::updateEnergies (material_plastic.cc:85-103)
    double wp = 0.;
#pragma unroll
    for (int k = 0; k < DD; ++k) {
      const double de = ep[k] - epp[k];
      const double sh = s[k] + sp[k];
      wp = (k == 0) ? sh * de : wp + sh * de;
    }
    wp = wp / 2.;
    ps.pe[qi] = ps.pe[qi] + wp;
  }
  GT *gu = static_cast<GT *>(ps.gu);
#pragma unroll
  for (int k = 0; k < DD; ++k) gu[(int64_t)(q * DD + k) * ne + le] = (GT)gd[k];
#pragma unroll
  for (int c = 0; c < NS; ++c) {
    const int64_t idx = (int64_t)(q * NS + c) * ne + le;
    ps.sig[idx] = s[full_of<D>(c)];
    ps.eps[idx] = ep[full_of<D>(c)];
  }
  ps.iso[qi] = iso;
}

template <int D, int NN, int LAW, class T, bool REL>
__device__ __forceinline__ void element_law(const T *ue, const T *b, T w, const MatParams &mp,
                                            const GroupArgs &ps, int64_t ne, int64_t le,
                                            int q, T *t) {
  // grad u = u B^T  (shape_functions_inline_impl.hh:303-310)
  T g[D * D];
#pragma unroll
  for (int j = 0; j < D; ++j)
#pragma unroll
    for (int i = 0; i < D; ++i) {
      T s = ue[i] * b[j];
#pragma unroll
      for (int a = 1; a < NN; ++a) s = s + ue[a * D + i] * b[a * D + j];
      g[i + D * j] = s;
    }
  subtract_eigen<D, T>(ps, ne, le, q, g);
  if constexpr (LAW == LAW_NEOHOOKEAN) {
    if constexpr (REL) {
      // mixed path: r = (F S w) . dN/dx with F S formed in the displacement gradient
      T P[D * D];
      if (mp.svk) {
        T S[D * D];
        finite_pk2<D, T>(mp, g, S);
        first_piola<D, T>(g, S, w, P);
      } else {
        const double c33 = point_c33<D, T>(mp, ps, ne, le, q, g);
        neohookean_piola<D, T>((T)mp.lambda, (T)mp.mu, g, w, P, c33);
      }
#pragma unroll
      for (int a = 0; a < NN; ++a)
#pragma unroll
        for (int k = 0; k < D; ++k) {
          T s = P[k] * b[a * D];
#pragma unroll
          for (int J = 1; J < D; ++J) s += P[k + D * J] * b[a * D + J];
          t[a * D + k] = s;
        }
    } else {
      T S[D * D];
      finite_pk2<D, T>(mp, g, S, point_c33<D, T>(mp, ps, ne, le, q, g));
      T Sv[D == 3 ? 6 : 3];
      to_voigt<D, T>(S, Sv);
#pragma unroll
      for (int a = 0; a < NN; ++a)
#pragma unroll
        for (int k = 0; k < D; ++k)
          t[a * D + k] = finite_force_component<D, T>(&b[a * D], g, Sv, k) * w;
    }
  } else {
    T sig[D * D];
    if constexpr (LAW == LAW_ELASTIC) {
      elastic_stress<D, T>((T)mp.lambda, (T)mp.mu, g, (T)mp.sigma_th, sig);
    } else {
      double gd[D * D], s[D * D];
#pragma unroll
      for (int k = 0; k < D * D; ++k) gd[k] = (double)g[k];
      plastic_point<D, T>(mp, ps, ne, le, q, gd, s);
#pragma unroll
      for (int k = 0; k < D * D; ++k) sig[k] = (T)s[k];
    }
    // sigma B, d x n  (shape_lagrange_inline_impl.hh:402-408), times wJ_q
    if constexpr (REL) {
#pragma unroll
      for (int k = 0; k < D * D; ++k) sig[k] *= w;
#pragma unroll
      for (int a = 0; a < NN; ++a)
#pragma unroll
        for (int i = 0; i < D; ++i) {
          T s = sig[i] * b[a * D];
#pragma unroll
          for (int j = 1; j < D; ++j) s += sig[i + D * j] * b[a * D + j];
          t[a * D + i] = s;
        }
    } else {
#pragma unroll
      for (int a = 0; a < NN; ++a)
#pragma unroll
        for (int i = 0; i < D; ++i) {
          T s = sig[i] * b[a * D];
#pragma unroll
          for (int j = 1; j < D; ++j) s = s + sig[i + D * j] * b[a * D + j];
          t[a * D + i] = s * w;
        }
    }
  }
}

// element le of a launch over [e_begin, e_begin + e_count): dN/dx and
// det J w streamed from the precomputed tables B, wJ, or with REC recomputed
// from the nodal coordinates X by the precomputation's own arithmetic
// (point_geometry, FP64, then rounded to T like the tables' FP32 copies):
// the same numbers either way, REC reading the L2-resident coordinates
// instead of streaming (NQ x NN x D + NQ) values per element from DRAM
template <int D, int NN, int NQ, int LAW, class T, class RT, bool REC = false>
__device__ __forceinline__ void element_pe(int64_t le, int64_t e_begin, int64_t e_count,
                                           int64_t E, const int32_t *conn,
                                           const int32_t *pos,
                                           const T *B, const T *wJ,
                                           const double *u, const MatParams &mp,
                                           const GroupArgs &ps, RT *re,
                                           const double *X = nullptr,
                                           const QuadTable *tab = nullptr) {
  constexpr int ND = NN * D;
  constexpr bool REL = !std::is_same<T, double>::value;  // relative gather in FP32
  const int64_t e = e_begin + le;
  const MatParams mpe = group_params(mp, ps, le);
  T ue[ND];
  double u0[D];
  double Xe[REC ? ND : 1];
#pragma unroll
  for (int a = 0; a < NN; ++a) {
    const int64_t node = conn[(int64_t)a * E + e];
#pragma unroll
    for (int i = 0; i < D; ++i) {
      const double x = u[node * D + i];
      if constexpr (REL) {
        if (a == 0) u0[i] = x;
        ue[a * D + i] = (T)(x - u0[i]);
      } else {
        ue[a * D + i] = x;
      }
      if constexpr (REC) Xe[a * D + i] = X[node * D + i];
    }
  }
  // mixed tetrahedra stream dN/dx of nodes 1..3 only ([9][E]); node 0's are
  // minus their sum (its relative displacement is zero, so only its force
  // uses them)
  constexpr bool TET_COMPACT = D == 3 && NN == 4 && NQ == 1 && REL;
  T r[ND];
#pragma unroll 1
  for (int q = 0; q < NQ; ++q) {
    T b[ND];
    T w;
    if constexpr (REC) {
      double Bq[ND], wq;
      if constexpr (D == 3 && NN == 4)
        point_geometry<D, NN>(Xe, Tet4Dn{}, tab->w[q], Bq, &wq);
      else
        point_geometry<D, NN>(Xe, TableDn{&tab->dnds[q * 3 * kMaxNN]}, tab->w[q], Bq, &wq);
#pragma unroll
      for (int c = TET_COMPACT ? 3 : 0; c < ND; ++c) b[c] = (T)Bq[c];
      w = (T)wq;
    } else {
      if constexpr (TET_COMPACT) {
#pragma unroll
        for (int c = 3; c < ND; ++c) b[c] = B[(int64_t)(c - 3) * E + e];
      } else {
#pragma unroll
        for (int c = 0; c < ND; ++c) b[c] = B[(int64_t)(q * ND + c) * E + e];
      }
      w = wJ[(int64_t)q * E + e];
    }
    if constexpr (TET_COMPACT) {
#pragma unroll
      for (int j = 0; j < 3; ++j) b[j] = -((b[3 + j] + b[6 + j]) + b[9 + j]);
    }
    T t[ND];
    element_law<D, NN, LAW, T, REL>(ue, b, w, mpe, ps, e_count, le, q, t);
    // integrate: sum over q in increasing order (integrator_gauss_inline_impl.hh:401-418)
#pragma unroll
    for (int c = 0; c < ND; ++c) r[c] = (q == 0) ? t[c] : r[c] + t[c];
  }
  // elemental force of node a goes to its position in the node CSR
#pragma unroll
  for (int a = 0; a < NN; ++a) store_slot<D>(re, pos[(int64_t)a * E + e], &r[a * D]);
}

// one value of a dN/dx table, loaded where it is used: the asm keeps the
// compiler from holding a point's whole row in registers between the
// gradient and the force, which read it at two places
__device__ __forceinline__ float ld_table(const float *p) {
  float v;
  asm volatile("ld.global.nc.f32 %0, [%1];" : "=f"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ double ld_table(const double *p) {
  double v;
  asm volatile("ld.global.nc.f64 %0, [%1];" : "=d"(v) : "l"(p));
  return v;
}

// element_pe for the plastic law, streamed: the same operations in the same
// order, with less held in registers across the radial return (its FP64
// state is the register peak of the kernel): each point gathers the nodal
// displacements again (the same values: u does not change within the step),
// loads its dN/dx row node by node where the gradient and the force use it,
// and the element's force sum over the points lives in shared memory
// rs[c sst] instead of registers
template <int D, int NN, int NQ, class T, class RT>
__device__ __forceinline__ void element_pe_plastic_streamed(int64_t le, int64_t e_begin,
                                                            int64_t e_count, int64_t E,
                                                            const int32_t *conn,
                                                            const int32_t *pos, const T *B,
                                                            const T *wJ, const double *u,
                                                            const MatParams &mp,
                                                            const GroupArgs &ps, RT *re, T *rs,
                                                            int sst) {
  constexpr int ND = NN * D;
  constexpr bool REL = !std::is_same<T, double>::value;
  const int64_t e = e_begin + le;
  const MatParams mpe = group_params(mp, ps, le);
#pragma unroll 1
  for (int q = 0; q < NQ; ++q) {
    T ue[ND];
    double u0[D];
#pragma unroll
    for (int a = 0; a < NN; ++a) {
      const int64_t node = conn[(int64_t)a * E + e];
#pragma unroll
      for (int i = 0; i < D; ++i) {
        const double x = u[node * D + i];
        if constexpr (REL) {
          if (a == 0) u0[i] = x;
          ue[a * D + i] = (T)(x - u0[i]);
        } else {
          ue[a * D + i] = x;
        }
      }
    }
    const T *Bq = B + (int64_t)q * ND * E + e;
    // grad u = u B^T, s = u_0 b_0 then s + u_a b_a (the expression of element_law)
    T g[D * D];
#pragma unroll
    for (int a = 0; a < NN; ++a) {
      T ba[D];
#pragma unroll
      for (int j = 0; j < D; ++j) ba[j] = Bq[(int64_t)(a * D + j) * E];
#pragma unroll
      for (int j = 0; j < D; ++j)
#pragma unroll
        for (int i = 0; i < D; ++i)
          g[i + D * j] = (a == 0) ? ue[i] * ba[j] : g[i + D * j] + ue[a * D + i] * ba[j];
    }
    subtract_eigen<D, T>(ps, e_count, le, q, g);
    T sig[D * D];
    {
      double gd[D * D], sd[D * D];
#pragma unroll
      for (int k = 0; k < D * D; ++k) gd[k] = (double)g[k];
      plastic_point<D, T>(mpe, ps, e_count, le, q, gd, sd);
#pragma unroll
      for (int k = 0; k < D * D; ++k) sig[k] = (T)sd[k];
    }
    const T w = wJ[(int64_t)q * E + e];
    if constexpr (REL) {
#pragma unroll
      for (int k = 0; k < D * D; ++k) sig[k] *= w;
    }
#pragma unroll
    for (int a = 0; a < NN; ++a) {
      T ba[D];
#pragma unroll
      for (int j = 0; j < D; ++j) ba[j] = ld_table(Bq + (int64_t)(a * D + j) * E);
#pragma unroll
      for (int i = 0; i < D; ++i) {
        T t;
        if constexpr (REL) {
          T s = sig[i] * ba[0];
#pragma unroll
          for (int j = 1; j < D; ++j) s += sig[i + D * j] * ba[j];
          t = s;
        } else {
          T s = sig[i] * ba[0];
#pragma unroll
          for (int j = 1; j < D; ++j) s = s + sig[i + D * j] * ba[j];
          t = s * w;
        }
        // integrate: sum over q in increasing order
        T &r = rs[(a * D + i) * sst];
        r = (q == 0) ? t : r + t;
      }
    }
  }
#pragma unroll
  for (int a = 0; a < NN; ++a) {
    T ra[D];
#pragma unroll
    for (int i = 0; i < D; ++i) ra[i] = rs[(a * D + i) * sst];
    store_slot<D>(re, pos[(int64_t)a * E + e], ra);
  }
}

// k_element_forces_pe with the streamed plastic law (the same numbers)
template <int D, int NN, int NQ, class T, class RT, int BLOCK, int MINB = 1>
__global__ void __launch_bounds__(BLOCK, MINB)
    k_element_forces_pe_streamed(int64_t e_begin, int64_t e_count, int64_t E,
                                 const int32_t *__restrict__ conn,
                                 const int32_t *__restrict__ pos, const T *__restrict__ B,
                                 const T *__restrict__ wJ, const double *__restrict__ u,
                                 MatParams mp, GroupArgs ps, RT *__restrict__ re, int64_t pf) {
  (void)pf;
  __shared__ T s_r[NN * D * BLOCK];
  pdl_begin();
  const int64_t le = (int64_t)blockIdx.x * BLOCK + threadIdx.x;
  if (le >= e_count || !element_active(ps, le)) return;
  if (!element_indices_ok<NN>(ps, conn, pos, E, e_begin + le)) return;
  element_pe_plastic_streamed<D, NN, NQ, T, RT>(le, e_begin, e_count, E, conn, pos, B, wJ, u, mp,
                                                ps, re, s_r + threadIdx.x, BLOCK);
}

// The element-indexed rows the warp pf elements further on reads, prefetched
// into L2 (one row segment of 32 elements per lane and pass): connectivity,
// slot positions, dN/dx and det J w, the material slot, and the previous
// plastic state of every point ([row][e_count] arrays of the group).  L2 is
// the device's point of coherence, so a prefetch can never return stale
// data: it is issued before the dependent-launch wait.
template <int D, int NN, int NQ, int LAW, class T>
__device__ __forceinline__ void prefetch_pe_rows(int64_t pf, int64_t e_begin, int64_t e_count,
                                                 int64_t E, const int32_t *conn,
                                                 const int32_t *pos, const T *B, const T *wJ,
                                                 const GroupArgs &ps) {
  constexpr int ND = NN * D, DD = D * D, NS = SymComps<D>::value;
  constexpr bool TET_COMPACT = D == 3 && NN == 4 && NQ == 1 && !std::is_same<T, double>::value;
  constexpr int NB = TET_COMPACT ? 9 : NQ * ND;
  constexpr int NPL = LAW == LAW_PLASTIC ? NQ * (2 * NS + DD + 2) : 0;
  constexpr int kRows = 2 * NN + NB + NQ + 1 + NPL;
  const int64_t w0 = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31) + pf;
  if (w0 >= e_count) return;
  const int64_t w1 = w0 + 32 < e_count ? w0 + 32 : e_count;
  for (int r = threadIdx.x & 31; r < kRows; r += 32) {
    // array, its entry count and size, and the entry of local element 0
    const char *b = nullptr;
    int64_t n = 0, at = 0;
    int esz = 4;
    int k = r;
    if (k < NN) {
      b = (const char *)conn, n = NN * E, at = k * E + e_begin;
    } else if ((k -= NN) < NN) {
      b = (const char *)pos, n = NN * E, at = k * E + e_begin;
    } else if ((k -= NN) < NB) {
      b = (const char *)B, n = NB * E, at = k * E + e_begin, esz = sizeof(T);
    } else if ((k -= NB) < NQ) {
      b = (const char *)wJ, n = NQ * E, at = k * E + e_begin, esz = sizeof(T);
    } else if ((k -= NQ) < 1) {
      b = (const char *)ps.mslot, n = e_count;  // per-element material slot, or none
    } else if (LAW == LAW_PLASTIC) {
      k -= 1;
      esz = 8;
      if (k < NQ * NS) {
        b = (const char *)ps.sig_prev, n = NQ * NS * e_count, at = k * e_count;
      } else if ((k -= NQ * NS) < NQ * NS) {
        b = (const char *)ps.eps_prev, n = NQ * NS * e_count, at = k * e_count;
      } else if ((k -= NQ * NS) < NQ * DD) {
        esz = sizeof(T);
        b = (const char *)ps.gu_prev, n = NQ * DD * e_count, at = k * e_count;
      } else if ((k -= NQ * DD) < NQ) {
        b = (const char *)ps.iso_prev, n = NQ * e_count, at = k * e_count;
      } else {
        k -= NQ;
        b = (const char *)ps.iso_cur_in, n = NQ * e_count, at = k * e_count;
      }
    }
    if (b) prefetch_l2(b, b + n * esz, b + (at + w0) * esz, b + (at + w1) * esz);
  }
}

// BLOCK: threads (= elements) per block, one of the launch shapes the
// autotuner chooses from; MINB > 1 caps the registers for that many resident
// blocks per SM (plastic groups, whose state loads want more warps in flight)
// PF: the instance with the L2 prefetch (pf > 0); the one without has no
// prefetch code at all
template <int D, int NN, int NQ, int LAW, class T, class RT, int BLOCK, int MINB = 1,
          bool PF = false>
__global__ void __launch_bounds__(BLOCK, MINB)
    k_element_forces_pe(int64_t e_begin, int64_t e_count, int64_t E,
                        const int32_t *__restrict__ conn, const int32_t *__restrict__ pos,
                        const T *__restrict__ B, const T *__restrict__ wJ,
                        const double *__restrict__ u, MatParams mp, GroupArgs ps,
                        RT *__restrict__ re, int64_t pf) {
  if constexpr (PF)
    prefetch_pe_rows<D, NN, NQ, LAW, T>(pf, e_begin, e_count, E, conn, pos, B, wJ, ps);
  pdl_begin();
  const int64_t le = (int64_t)blockIdx.x * BLOCK + threadIdx.x;
  if (le >= e_count || !element_active(ps, le)) return;
  if (!element_indices_ok<NN>(ps, conn, pos, E, e_begin + le)) return;
  element_pe<D, NN, NQ, LAW, T, RT>(le, e_begin, e_count, E, conn, pos, B, wJ, u, mp, ps, re);
}

// k_element_forces_pe with the geometry recomputed from the coordinates
// (element_pe REC): the same numbers, no dN/dx and det J w streamed
template <int D, int NN, int NQ, int LAW, class T, class RT, int BLOCK, int MINB = 1,
          bool PF = false>
__global__ void __launch_bounds__(BLOCK, MINB)
    k_element_forces_pr(int64_t e_begin, int64_t e_count, int64_t E,
                        const int32_t *__restrict__ conn, const int32_t *__restrict__ pos,
                        const double *__restrict__ X, const QuadTable tab,
                        const double *__restrict__ u, MatParams mp, GroupArgs ps,
                        RT *__restrict__ re, int64_t pf) {
  if constexpr (PF)
    prefetch_pe_rows<D, NN, NQ, LAW, T>(pf, e_begin, e_count, E, conn, pos, nullptr, nullptr, ps);
  pdl_begin();
  const int64_t le = (int64_t)blockIdx.x * BLOCK + threadIdx.x;
  if (le >= e_count || !element_active(ps, le)) return;
  if (!element_indices_ok<NN>(ps, conn, pos, E, e_begin + le)) return;
  element_pe<D, NN, NQ, LAW, T, RT, true>(le, e_begin, e_count, E, conn, pos, nullptr, nullptr, u,
                                          mp, ps, re, X, &tab);
}

// Mixed path: FP32 element math with the shape derivatives recomputed from
// the gathered nodal coordinates instead of streamed from HBM.  Per point:
// J = dN/ds X^T, dN/dx = J^-1 dN/ds, w = det J * w_q (the arithmetic of
// k_precompute, in FP32, with coordinates and displacements taken relative
// to the element's first node -- dN/ds sums to zero over the nodes, so the
// Jacobian and the gradient are unchanged in exact arithmetic).
template <int D, int NN, int NQ, int LAW>
__device__ __forceinline__ void element_geo(int64_t le, int64_t e_begin, int64_t e_count,
                                            int64_t E, const int32_t *conn,
                                            const int32_t *pos,
                                            const double *X, const QuadTable &tab,
                                            const double *u, const MatParams &mp,
                                            const GroupArgs &ps, float *re) {
  constexpr int ND = NN * D;
  const int64_t e = e_begin + le;
  const MatParams mpe = group_params(mp, ps, le);
  float xe[ND], ue[ND];
  double x0[D], u0[D];
#pragma unroll
  for (int a = 0; a < NN; ++a) {
    const int64_t node = conn[(int64_t)a * E + e];
#pragma unroll
    for (int i = 0; i < D; ++i) {
      const double x = X[node * D + i], uu = u[node * D + i];
      if (a == 0) {
        x0[i] = x;
        u0[i] = uu;
      }
      xe[a * D + i] = (float)(x - x0[i]);
      ue[a * D + i] = (float)(uu - u0[i]);
    }
  }
  float r[ND];
#pragma unroll 1
  for (int q = 0; q < NQ; ++q) {
    const float *dn = &tab.fdnds[q * 3 * kMaxNN];
    float J[D * D], Ji[D * D];
#pragma unroll
    for (int k = 0; k < D; ++k)
#pragma unroll
      for (int j = 0; j < D; ++j) {
        float s = dn[k * kMaxNN] * xe[j];
#pragma unroll
        for (int a = 1; a < NN; ++a) s += dn[k * kMaxNN + a] * xe[a * D + j];
        J[k + D * j] = s;
      }
    float det;
    if constexpr (D == 3) {
      det = det3(J);
      inv3(J, Ji);
    } else {
      det = det2(J);
      inv2(J, Ji);
    }
    float b[ND];
#pragma unroll
    for (int a = 0; a < NN; ++a)
#pragma unroll
      for (int j = 0; j < D; ++j) {
        float s = Ji[j] * dn[a];
#pragma unroll
        for (int k = 1; k < D; ++k) s += Ji[j + D * k] * dn[k * kMaxNN + a];
        b[a * D + j] = s;
      }
    const float w = det * tab.fw[q];
    float t[ND];
    element_law<D, NN, LAW, float, true>(ue, b, w, mpe, ps, e_count, le, q, t);
#pragma unroll
    for (int c = 0; c < ND; ++c) r[c] = (q == 0) ? t[c] : r[c] + t[c];
  }
#pragma unroll
  for (int a = 0; a < NN; ++a) store_slot<D>(re, pos[(int64_t)a * E + e], &r[a * D]);
}

template <int D, int NN, int NQ, int LAW, int BLOCK>
__global__ void __launch_bounds__(BLOCK)
    k_element_forces_geo(int64_t e_begin, int64_t e_count, int64_t E,
                         const int32_t *__restrict__ conn, const int32_t *__restrict__ pos,
                         const double *__restrict__ X, QuadTable tab,
                         const double *__restrict__ u, MatParams mp, GroupArgs ps,
                         float *__restrict__ re) {
  pdl_begin();
  const int64_t le = (int64_t)blockIdx.x * BLOCK + threadIdx.x;
  if (le >= e_count || !element_active(ps, le)) return;
  if (!element_indices_ok<NN>(ps, conn, pos, E, e_begin + le)) return;
  element_geo<D, NN, NQ, LAW>(le, e_begin, e_count, E, conn, pos, X, tab, u, mp, ps, re);
}

// Mixed path, _hexahedron_8: sum factorisation of the trilinear element.
// With node a at signs (sx, sy, sz) in {-1, 1}^3, N_a = (1 + sx xi)(1 + sy eta)
// (1 + sz zeta) / 8, so a nodal field f has the modal form
//   f(xi) = (W_0 + W_1 xi + W_2 eta + W_3 xi eta + W_4 zeta + W_5 xi zeta
//            + W_6 eta zeta + W_7 xi eta zeta) / 8,
// W_m = sum_a f_a prod_{d in m} s_{a,d} (m a bit set over x, y, z): an 8-point
// Walsh-Hadamard transform of the nodal values.  The Jacobian and the
// displacement derivative at a Gauss point (all coordinates +-1/sqrt(3)) are
// then a few signed sums of the W_m, and the elemental force
//   r_a = sum_q P_q J_q^-1 dN_a/dxi(q)
// (P_q the weighted flux: w sigma, or w F S) is accumulated in the same modal
// basis and brought back to the nodes by the inverse transform.  Equal to the
// dN/dx form of k_element_forces_geo in exact arithmetic, with about 40% fewer
// floating-point operations per point.  The factors 1/8 cancel between the
// Jacobian and its inverse and are folded into det J.
template <class T> __device__ __forceinline__ void wht8(T (*v)[3]) {
#pragma unroll
  for (int d = 0; d < 3; ++d)
#pragma unroll
    for (int l = 0; l < 8; ++l)
      if (!(l & (1 << d))) {
        const int h = l | (1 << d);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const T a = v[l][c], b = v[h][c];
          v[l][c] = a + b;
          v[h][c] = b - a;
        }
      }
}
template <class T> __device__ __forceinline__ void iwht8(T (*v)[3]) {
#pragma unroll
  for (int d = 0; d < 3; ++d)
#pragma unroll
    for (int l = 0; l < 8; ++l)
      if (!(l & (1 << d))) {
        const int h = l | (1 << d);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const T a = v[l][c], b = v[h][c];
          v[l][c] = a - b;
          v[h][c] = a + b;
        }
      }
}

// weighted flux P of one point for the sum-factorised kernels: r_a = P . dN_a/dx
// (FP32 element math on the mixed path, FP64 on the fast FP64 path: the
// same formulas, first Piola-Kirchhoff stress in the displacement gradient)
template <int D, int LAW, class T = float>
__device__ __forceinline__ void mixed_flux(const T *g, T w, const MatParams &mp,
                                           const GroupArgs &ps, int64_t ne, int64_t le, int q,
                                           T *P) {
  if constexpr (LAW == LAW_NEOHOOKEAN) {
    if (mp.svk) {
      T S[D * D];
      finite_pk2<D, T>(mp, g, S);
      first_piola<D, T>(g, S, w, P);
    } else {
      neohookean_piola<D, T>((T)mp.lambda, (T)mp.mu, g, w, P);
    }
  } else if constexpr (LAW == LAW_ELASTIC) {
    T sig[D * D];
    elastic_stress<D, T>((T)mp.lambda, (T)mp.mu, g, (T)mp.sigma_th, sig);
#pragma unroll
    for (int k = 0; k < D * D; ++k) P[k] = sig[k] * w;
  } else {
    double gd[D * D], sd[D * D];
#pragma unroll
    for (int k = 0; k < D * D; ++k) gd[k] = (double)g[k];
    plastic_point<D, T>(mp, ps, ne, le, q, gd, sd);
#pragma unroll
    for (int k = 0; k < D * D; ++k) P[k] = (T)sd[k] * w;
  }
}

// relative FP32 coordinates of a hexahedron's nodes in the modal
// (Walsh-Hadamard) basis, lexicographic corner order
template <class T>
__device__ __forceinline__ void hex8_geometry_modes(int64_t e, int64_t E, const int32_t *conn,
                                                    const double *X, T (*wx)[3]) {
  constexpr int lex[8] = {0, 1, 3, 2, 4, 5, 7, 6};
  double x0[3];
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const int64_t node = conn[(int64_t)a * E + e];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const double x = X[node * 3 + i];
      if (a == 0) x0[i] = x;
      wx[lex[a]][i] = (T)(x - x0[i]);
    }
  }
  wht8(wx);
}

// the Jacobian adjugate and 1/det of a parallelepiped from its geometry
// modes (wx after wht8: modes 1, 2 and 4 are 8 dX/dxi, 8 dX/deta, 8 dX/dzeta)
template <class T>
__device__ __forceinline__ T hex8_affine_adjugate(const T (*wx)[3], T *Ja) {
  T Jp[9];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    Jp[0 + 3 * j] = wx[1][j];
    Jp[1 + 3 * j] = wx[2][j];
    Jp[2 + 3 * j] = wx[4][j];
  }
  return T(1) / adj3(Jp, Ja);
}

// QU: quadrature points per unrolled iteration (1, 2, 4 or 8).  AFF: every
// element of the launch is a parallelepiped (checked once per mesh), so the
// per-point geometry and its registers are compiled out; the same arithmetic
// as the general kernel's affine branch.  GEO (with AFF): the adjugate and
// 1/det of each element are read from geo [10][E], formed once by
// k_hex8_affine_geometry with the same arithmetic, instead of gathering the
// element's coordinates every step
template <int LAW, int QU, bool AFF = false, bool GEO = false, class T = float>
__device__ __forceinline__ void element_hex8sf(int64_t le, int64_t e_begin, int64_t e_count,
                                               int64_t E, const int32_t *conn,
                                               const int32_t *pos,
                                               const double *X, const T *geo,
                                               const double *u, const MatParams &mp,
                                               const GroupArgs &ps, T *re) {
  static_assert(AFF || !GEO, "the geometry table holds parallelepipeds only");
  const int64_t e = e_begin + le;
  const MatParams mpe = group_params(mp, ps, le);
  // reference node a sits at lexicographic corner lex[a] = [sx>0] + 2[sy>0] + 4[sz>0]
  constexpr int lex[8] = {0, 1, 3, 2, 4, 5, 7, 6};
  T wx[8][3], wu[8][3];
  double x0[3], u0[3];
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const int64_t node = conn[(int64_t)a * E + e];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const double uu = u[node * 3 + i];
      if (a == 0) u0[i] = uu;
      wu[lex[a]][i] = (T)(uu - u0[i]);
      if constexpr (!GEO) {
        const double x = X[node * 3 + i];
        if (a == 0) x0[i] = x;
        wx[lex[a]][i] = (T)(x - x0[i]);
      }
    }
  }
  T Ja[9], rdet_a = T(0);
  if constexpr (GEO) {
#pragma unroll
    for (int k = 0; k < 9; ++k) Ja[k] = geo[(int64_t)k * E + e];
    rdet_a = geo[(int64_t)9 * E + e];
  } else {
    wht8(wx);
  }
  wht8(wu);
  // Gauss coordinate 1/sqrt(3), rounded once to T
  constexpr T g1 = std::is_same<T, float>::value ? T(0.577350269189625764509f)
                                                 : T(0.577350269189625764509);
  constexpr T g2 = T(1) / T(3);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if constexpr (!GEO) {
      wx[3][c] *= g1; wx[5][c] *= g1; wx[6][c] *= g1; wx[7][c] *= g2;
    }
    wu[3][c] *= g1; wu[5][c] *= g1; wu[6][c] *= g1; wu[7][c] *= g2;
  }
  T A[8][3];
#pragma unroll
  for (int m = 0; m < 8; ++m)
#pragma unroll
    for (int c = 0; c < 3; ++c) A[m][c] = T(0);
  // a parallelepiped (affine element: no bilinear or trilinear geometry
  // mode) has the same Jacobian at every point; its adjugate and 1/det are
  // formed once.  The modes are tested for exact zeros, so the point-wise
  // formulas below would give the same values at every point anyway.
  bool affine = true;
  if constexpr (!AFF) {
#pragma unroll
    for (int c = 0; c < 3; ++c)
      affine = affine && wx[3][c] == T(0) && wx[5][c] == T(0) && wx[6][c] == T(0) &&
               wx[7][c] == T(0);
  }
  if constexpr (!GEO)
    if (affine) rdet_a = hex8_affine_adjugate(wx, Ja);
#pragma unroll 1
  for (int qo = 0; qo < 8; qo += QU)
#pragma unroll
  for (int qi = 0; qi < QU; ++qi) {
    const int q = qo + qi;
    // point q at (xi, eta, zeta) = g1 (sx, sy, sz), the order of the rule
    const T sx = (q & 1) ? T(1) : T(-1), sy = (q & 2) ? T(1) : T(-1), sz = (q & 4) ? T(1) : T(-1);
    T Dp[9], Ji[9];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      // 8 d(u_j)/d(xi_k) at row k
      Dp[0 + 3 * j] = wu[1][j] + sy * wu[3][j] + sz * wu[5][j] + sy * sz * wu[7][j];
      Dp[1 + 3 * j] = wu[2][j] + sx * wu[3][j] + sz * wu[6][j] + sx * sz * wu[7][j];
      Dp[2 + 3 * j] = wu[4][j] + sx * wu[5][j] + sy * wu[6][j] + sx * sy * wu[7][j];
    }
    T rdet;
    if (affine) {
#pragma unroll
      for (int k = 0; k < 9; ++k) Ji[k] = Ja[k];
      rdet = rdet_a;
    } else if constexpr (!AFF) {
      // 8 d(X_j)/d(xi_k) at row k
      T Jp[9];
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        Jp[0 + 3 * j] = wx[1][j] + sy * wx[3][j] + sz * wx[5][j] + sy * sz * wx[7][j];
        Jp[1 + 3 * j] = wx[2][j] + sx * wx[3][j] + sz * wx[6][j] + sx * sz * wx[7][j];
        Jp[2 + 3 * j] = wx[4][j] + sx * wx[5][j] + sy * wx[6][j] + sx * sy * wx[7][j];
      }
      // adjugate: (8 J)^-1 = adj / det8, det8 = 512 det J
      rdet = T(1) / adj3(Jp, Ji);
    }
    // grad u (i, j) = sum_k J^-1(j, k) du_i/dxi_k  (the factors 8 cancel)
    T gr[9];
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
      for (int i = 0; i < 3; ++i)
        gr[i + 3 * j] = (Ji[j] * Dp[0 + 3 * i] + Ji[j + 3] * Dp[1 + 3 * i] +
                         Ji[j + 6] * Dp[2 + 3 * i]) * rdet;
    subtract_eigen<3, T>(ps, e_count, le, q, gr);
    // the weight w = det J (2 x 2 x 2 Gauss weights are 1) cancels the 1/det
    // of J^-1 in H = w P J^-1: the unweighted flux times the adjugate is
    // accumulated and the remaining 1/512 applied once per element
    T P[9];
    mixed_flux<3, LAW, T>(gr, T(1), mpe, ps, e_count, le, q, P);
    // H(k, m) = sum_J P(k, J) adj(J, m), accumulated per mode
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const T H0 = P[k] * Ji[0] + P[k + 3] * Ji[1] + P[k + 6] * Ji[2];
      const T H1 = P[k] * Ji[3] + P[k + 3] * Ji[4] + P[k + 6] * Ji[5];
      const T H2 = P[k] * Ji[6] + P[k + 3] * Ji[7] + P[k + 6] * Ji[8];
      A[1][k] += H0;
      A[2][k] += H1;
      A[4][k] += H2;
      A[3][k] += sy * H0 + sx * H1;
      A[5][k] += sz * H0 + sx * H2;
      A[6][k] += sz * H1 + sy * H2;
      A[7][k] += sy * sz * H0 + sx * sz * H1 + sx * sy * H2;
    }
  }
  constexpr T s0 = T(1) / T(512), s1 = g1 / T(512), s2 = g2 / T(512);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    A[1][c] *= s0; A[2][c] *= s0; A[4][c] *= s0;
    A[3][c] *= s1; A[5][c] *= s1; A[6][c] *= s1; A[7][c] *= s2;
  }
  iwht8(A);
#pragma unroll
  for (int a = 0; a < 8; ++a) store_slot<3>(re, pos[(int64_t)a * E + e], A[lex[a]]);
}

// ---- sum-factorised hexahedra on packed FP32 pairs ---------------------------
// sm_100 executes two FP32 operations of one thread as one packed
// instruction (add / mul / fma .rn .f32x2), each lane rounded exactly like
// the scalar operation.  The two Gauss points of an element that differ only
// in xi (q and q + 1: the same eta and zeta) are evaluated as the two lanes
// of one pair: their derivative rows, gradient, flux and projection are
// packed operations, the per-element constants (adjugate, Lame constants)
// broadcast to both lanes.  Lane x is the point at xi = -1/sqrt(3), lane y
// the point at +1/sqrt(3).
__device__ __forceinline__ float2 pb(float x) { return make_float2(x, x); }
__device__ __forceinline__ float2 padd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 pmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 pfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 pneg(float2 a) { return make_float2(-a.x, -a.y); }

// weighted first Piola-Kirchhoff stress of the neohookean law for a pair of
// points (weight 1), P = mu F + c cof(F), written in the displacement
// gradient H = F - I like neohookean_piola, with the cofactor expansion
//   adj(I + H) = I + t I - H + adj(H)       (t = tr H; Cayley-Hamilton)
// whose quadratic part adj(H) is formed from the 2 x 2 minors of H directly
// (18 operations instead of the 27 of H^2), and
//   det F - 1 = t + i2 + det H,  i2 = tr adj(H),  det H = H(0, :) . adj(H)(:, 0)
__device__ __forceinline__ void neohookean_piola_x2(float lambda, float mu, const float2 *g,
                                                    float2 *P) {
  float2 adj[9];
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      // adj(H)(i, j) = cofactor (j, i) of H
      const int j1 = (j + 1) % 3, j2 = (j + 2) % 3, i1 = (i + 1) % 3, i2 = (i + 2) % 3;
      adj[i + 3 * j] = pfma(g[j1 + 3 * i1], g[j2 + 3 * i2], pneg(pmul(g[j1 + 3 * i2], g[j2 + 3 * i1])));
    }
  const float2 t = padd(padd(g[0], g[4]), g[8]);
  const float2 i2 = padd(padd(adj[0], adj[4]), adj[8]);
  const float2 detH = pfma(g[6], adj[2], pfma(g[3], adj[1], pmul(g[0], adj[0])));
  const float2 dm1 = padd(padd(t, i2), detH);
  // K = adj(I + H) - I = adj(H) - H + t I; cof(F) = I + K^T
  float2 K[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) K[k] = padd(adj[k], pneg(g[k]));
  K[0] = padd(K[0], t);
  K[4] = padd(K[4], t);
  K[8] = padd(K[8], t);
  const float2 det = padd(pb(1.f), dm1);
  const float2 lnJ = make_float2(log1pf(dm1.x), log1pf(dm1.y));
  const float2 rdet = make_float2(1.f / det.x, 1.f / det.y);
  const float2 c = pmul(pfma(pb(lambda), lnJ, pb(-mu)), rdet);
  const float2 a0 = pmul(pfma(pb(mu), dm1, pmul(pb(lambda), lnJ)), rdet);
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      float2 p = pfma(c, K[j + 3 * i], pmul(pb(mu), g[i + 3 * j]));
      if (i == j) p = padd(p, a0);
      P[i + 3 * j] = p;
    }
}

// Cauchy stress of the elastic law for a pair of points
// (material_elastic_inline_impl.hh:31-48), sigma_th included
__device__ __forceinline__ void elastic_stress_x2(float lambda, float mu, float sth,
                                                  const float2 *g, float2 *s) {
  const float2 tr = padd(padd(g[0], g[4]), g[8]);
  const float2 dia = pfma(pb(lambda), tr, pb(sth));
  const float2 two_mu = pb(__fmul_rn(2.f, mu));
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const float2 v = pmul(two_mu, pmul(pb(.5f), padd(g[j + 3 * i], g[i + 3 * j])));
      s[i + 3 * j] = (i == j) ? padd(v, dia) : v;
    }
}

// PU pairs per unrolled iteration (1, 2 or 4); meshes of parallelepipeds
// only (one adjugate per element, from the geometry table with GEO); the
// elastic and neohookean laws (the plastic state is FP64 per point).  Every
// FP32 operation is explicitly rounded (scalar __f*_rn or packed .rn), so
// neither the points per iteration nor the register cap changes a result.
// the element's work once its relative nodal displacements wu (lexicographic
// corner order, FP32) are known
// The element's per-element table entries come as views: node a is cn[a cs],
// its slot position pv[a ps], adjugate entry k gv[k gs] (the global [row][E]
// tables at the element, or a block's staged copies in shared memory).
template <int LAW, int PU, bool GEO>
__device__ __forceinline__ void element_hex8sf_x2_core(float (*wu)[3], int64_t le,
                                                       int64_t e_count, const int32_t *cn,
                                                       int64_t cs, const int32_t *pv,
                                                       int64_t pvs, const double *X,
                                                       const float *gv, int64_t gs,
                                                       const MatParams &mp, const GroupArgs &ps,
                                                       float *re) {
  static_assert(LAW != LAW_PLASTIC, "plastic hexahedra use the scalar kernel");
  const MatParams mpe = group_params(mp, ps, le);
  constexpr int lex[8] = {0, 1, 3, 2, 4, 5, 7, 6};
  float Ja[9], rdet;
  if constexpr (GEO) {
#pragma unroll
    for (int k = 0; k < 9; ++k) Ja[k] = gv[k * gs];
    rdet = gv[9 * gs];
  } else {
    float wx[8][3];
    hex8_geometry_modes(0, cs, cn, X, wx);
    rdet = hex8_affine_adjugate(wx, Ja);
  }
  wht8(wu);
  constexpr float g1 = 0.577350269189625764509f;
  constexpr float g2 = 1.f / 3.f;
  // the modes carry the 1/det of the gradient (adj / det) and the Gauss
  // coordinates of their bilinear and trilinear terms
  const float rg1 = __fmul_rn(rdet, g1), rg2 = __fmul_rn(rdet, g2);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    wu[1][c] = __fmul_rn(wu[1][c], rdet);
    wu[2][c] = __fmul_rn(wu[2][c], rdet);
    wu[4][c] = __fmul_rn(wu[4][c], rdet);
    wu[3][c] = __fmul_rn(wu[3][c], rg1);
    wu[5][c] = __fmul_rn(wu[5][c], rg1);
    wu[6][c] = __fmul_rn(wu[6][c], rg1);
    wu[7][c] = __fmul_rn(wu[7][c], rg2);
  }
  float A[8][3];
#pragma unroll
  for (int m = 0; m < 8; ++m)
#pragma unroll
    for (int c = 0; c < 3; ++c) A[m][c] = 0.f;
  const float lam = (float)mpe.lambda, mu = (float)mpe.mu, sth = (float)mpe.sigma_th;
#pragma unroll 1
  for (int po = 0; po < 4; po += PU)
#pragma unroll
  for (int pi = 0; pi < PU; ++pi) {
    const int pr = po + pi;  // pair: points 2 pr (lane x) and 2 pr + 1 (lane y)
    // sign products are exact: sy, sz = +-1
    const float sy = (pr & 1) ? 1.f : -1.f, sz = (pr & 2) ? 1.f : -1.f;
    // du_j/dxi_k (times 8 / det): row 0 is the same for both points; rows 1
    // and 2 are r -+ s (xi = -+1/sqrt(3))
    float2 D1[3], D2[3];
    float D0[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      D0[j] = __fadd_rn(__fadd_rn(wu[1][j], sy * wu[3][j]),
                        sz * __fadd_rn(wu[5][j], sy * wu[7][j]));
      const float r1 = __fadd_rn(wu[2][j], sz * wu[6][j]), s1 = __fadd_rn(wu[3][j], sz * wu[7][j]);
      const float r2 = __fadd_rn(wu[4][j], sy * wu[6][j]), s2 = __fadd_rn(wu[5][j], sy * wu[7][j]);
      D1[j] = make_float2(__fadd_rn(r1, -s1), __fadd_rn(r1, s1));
      D2[j] = make_float2(__fadd_rn(r2, -s2), __fadd_rn(r2, s2));
    }
    // grad u (i, j) = sum_k adj(j, k) du_i/dxi_k / det
    float2 gr[9];
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
      for (int i = 0; i < 3; ++i)
        gr[i + 3 * j] = pfma(pb(Ja[j + 6]), D2[i],
                             pfma(pb(Ja[j + 3]), D1[i], pb(__fmul_rn(Ja[j], D0[i]))));
    if (ps.eig) {
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        const int64_t i0 = (int64_t)((2 * pr) * 9 + k) * e_count + le;
        gr[k] = make_float2(__fadd_rn(gr[k].x, -(float)ps.eig[i0]),
                            __fadd_rn(gr[k].y, -(float)ps.eig[i0 + 9 * e_count]));
      }
    }
    float2 P[9];
    if constexpr (LAW == LAW_NEOHOOKEAN) {
      if (mpe.svk) {
#pragma unroll
        for (int l = 0; l < 2; ++l) {
          float gl[9], S[9], Pl[9];
#pragma unroll
          for (int k = 0; k < 9; ++k) gl[k] = l ? gr[k].y : gr[k].x;
          finite_pk2<3, float>(mpe, gl, S);
          first_piola<3, float>(gl, S, 1.f, Pl);
#pragma unroll
          for (int k = 0; k < 9; ++k) (l ? P[k].y : P[k].x) = Pl[k];
        }
      } else {
        neohookean_piola_x2(lam, mu, gr, P);
      }
    } else {
      elastic_stress_x2(lam, mu, sth, gr, P);
    }
    // H(k, m) = sum_J P(k, J) adj(J, m), folded into the modes: with
    // S = H.x + H.y and T = H.y - H.x (the xi sign of lane y is +1)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float2 H0 = pfma(P[k + 6], pb(Ja[2]), pfma(P[k + 3], pb(Ja[1]), pmul(P[k], pb(Ja[0]))));
      const float2 H1 = pfma(P[k + 6], pb(Ja[5]), pfma(P[k + 3], pb(Ja[4]), pmul(P[k], pb(Ja[3]))));
      const float2 H2 = pfma(P[k + 6], pb(Ja[8]), pfma(P[k + 3], pb(Ja[7]), pmul(P[k], pb(Ja[6]))));
      const float S0 = __fadd_rn(H0.x, H0.y), S1 = __fadd_rn(H1.x, H1.y),
                  S2 = __fadd_rn(H2.x, H2.y);
      const float T1 = __fadd_rn(H1.y, -H1.x), T2 = __fadd_rn(H2.y, -H2.x);
      A[1][k] = __fadd_rn(A[1][k], S0);
      A[2][k] = __fadd_rn(A[2][k], S1);
      A[4][k] = __fadd_rn(A[4][k], S2);
      A[3][k] = __fadd_rn(A[3][k], __fadd_rn(sy * S0, T1));
      A[5][k] = __fadd_rn(A[5][k], __fadd_rn(sz * S0, T2));
      A[6][k] = __fadd_rn(A[6][k], __fadd_rn(sz * S1, sy * S2));
      A[7][k] = __fadd_rn(A[7][k], __fadd_rn(__fadd_rn((sy * sz) * S0, sz * T1), sy * T2));
    }
  }
  constexpr float s0 = 1.f / 512.f, s1 = g1 / 512.f, s2 = g2 / 512.f;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    A[1][c] = __fmul_rn(A[1][c], s0);
    A[2][c] = __fmul_rn(A[2][c], s0);
    A[4][c] = __fmul_rn(A[4][c], s0);
    A[3][c] = __fmul_rn(A[3][c], s1);
    A[5][c] = __fmul_rn(A[5][c], s1);
    A[6][c] = __fmul_rn(A[6][c], s1);
    A[7][c] = __fmul_rn(A[7][c], s2);
  }
  iwht8(A);
#pragma unroll
  for (int a = 0; a < 8; ++a) store_slot<3>(re, pv[a * pvs], A[lex[a]]);
}

// the element's relative nodal displacements gathered from global memory
template <int LAW, int PU, bool GEO>
__device__ __forceinline__ void element_hex8sf_x2(int64_t le, int64_t e_begin, int64_t e_count,
                                                  int64_t E, const int32_t *conn,
                                                  const int32_t *pos, const double *X,
                                                  const float *geo, const double *u,
                                                  const MatParams &mp, const GroupArgs &ps,
                                                  float *re) {
  constexpr int lex[8] = {0, 1, 3, 2, 4, 5, 7, 6};
  const int64_t e = e_begin + le;
  float wu[8][3];
  double u0[3];
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const int64_t node = conn[(int64_t)a * E + e];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const double uu = u[node * 3 + i];
      if (a == 0) u0[i] = uu;
      wu[lex[a]][i] = (float)(uu - u0[i]);
    }
  }
  element_hex8sf_x2_core<LAW, PU, GEO>(wu, le, e_count, conn + e, E, pos + e, E, X,
                                       GEO ? geo + e : nullptr, E, mp, ps, re);
}

// The rows of the per-element tables (connectivity and slot positions, 8
// each; with GEO the 10 of the adjugate table) that the warp pf elements
// further on will read, prefetched into L2 by one lane per row: with pf one
// wave of resident blocks, the blocks that follow find them there instead
// of in DRAM.  L2 is the device's point of coherence, so the prefetch is
// issued before the dependent-launch wait.
template <bool GEO>
__device__ __forceinline__ void prefetch_hex8_rows(int64_t pf, int64_t e_begin, int64_t e_count,
                                                   int64_t E, const int32_t *conn,
                                                   const int32_t *pos, const float *geo) {
  const int lane = threadIdx.x & 31;
  constexpr int kRows = GEO ? 26 : 16;
  const int64_t w0 = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31) + pf;
  if (lane >= kRows || w0 >= e_count) return;
  const int64_t w1 = w0 + 32 < e_count ? w0 + 32 : e_count;
  const char *b;
  int64_t r, n;
  if (lane < 8) {
    b = (const char *)conn, r = lane, n = 8;
  } else if (lane < 16) {
    b = (const char *)pos, r = lane - 8, n = 8;
  } else {
    b = (const char *)geo, r = lane - 16, n = 10;
  }
  static_assert(sizeof(int32_t) == 4 && sizeof(float) == 4, "4-byte table entries");
  prefetch_l2(b, b + n * E * 4, b + (r * E + e_begin + w0) * 4, b + (r * E + e_begin + w1) * 4);
}

// PF: the instance with the prefetch (pf > 0); the one without has no
// prefetch code at all
template <int LAW, int BLOCK, int PU, int MINB, bool GEO, bool PF = false>
__global__ void __launch_bounds__(BLOCK, MINB)
    k_element_forces_hex8sf_x2(int64_t e_begin, int64_t e_count, int64_t E,
                               const int32_t *__restrict__ conn, const int32_t *__restrict__ pos,
                               const double *__restrict__ X, const float *__restrict__ geo,
                               const double *__restrict__ u, MatParams mp, GroupArgs ps,
                               float *__restrict__ re, int64_t pf) {
  if constexpr (PF) prefetch_hex8_rows<GEO>(pf, e_begin, e_count, E, conn, pos, geo);
  pdl_begin();
  const int64_t le = (int64_t)blockIdx.x * BLOCK + threadIdx.x;
  if (le >= e_count || !element_active(ps, le)) return;
  if (!element_indices_ok<8>(ps, conn, pos, E, e_begin + le)) return;
  element_hex8sf_x2<LAW, PU, GEO>(le, e_begin, e_count, E, conn, pos, X, geo, u, mp, ps, re);
}

// MINB: blocks per SM the register allocation must allow (1: the compiler's
// choice)
template <int LAW, int BLOCK, int QU, int MINB, bool AFF = false, bool GEO = false,
          class T = float>
__global__ void __launch_bounds__(BLOCK, MINB)
    k_element_forces_hex8sf(int64_t e_begin, int64_t e_count, int64_t E,
                            const int32_t *__restrict__ conn, const int32_t *__restrict__ pos,
                            const double *__restrict__ X, const T *__restrict__ geo,
                            const double *__restrict__ u, MatParams mp, GroupArgs ps,
                            T *__restrict__ re) {
  pdl_begin();
  const int64_t le = (int64_t)blockIdx.x * BLOCK + threadIdx.x;
  if (le >= e_count || !element_active(ps, le)) return;
  if (!element_indices_ok<8>(ps, conn, pos, E, e_begin + le)) return;
  element_hex8sf<LAW, QU, AFF, GEO, T>(le, e_begin, e_count, E, conn, pos, X, geo, u, mp, ps,
                                       re);
}

// One thread per (element, q): blockDim = 32 * NQ, warp w = point q, lane =
// element; FP64 hexahedra.  The warps gather the element's nodal
// displacements into shared memory (FP64; with an FP32 element type T they
// are taken relative to node 0 there, as the per-element kernel does), each
// thread evaluates its point, and the points' contributions are summed in
// increasing q through shared memory laid out [q][component][lane] (free of
// bank conflicts): the per-element kernel's sums, bit for bit.  One thread
// per point of plastic triangles, in either precision, was measured slower
// than the per-element kernel (0.152 against 0.091 ms mixed, 0.181 against
// 0.126 ms FP64 on the 512^2 square: a third of the elements in flight per
// SM) and is not offered.
template <int D, int NN, int NQ, int LAW, class T = double, class RT = double>
__global__ void __launch_bounds__(32 * NQ)
    k_element_forces_pq(int64_t e_begin, int64_t e_count, int64_t E,
                        const int32_t *__restrict__ conn, const int32_t *__restrict__ pos,
                        const T *__restrict__ B, const T *__restrict__ wJ,
                        const double *__restrict__ u, MatParams mp, GroupArgs ps,
                        RT *__restrict__ re) {
  pdl_begin();
  constexpr int ND = NN * D;
  constexpr bool REL = !std::is_same<T, double>::value;  // relative gather in FP32
  constexpr int CH = (ND + NQ - 1) / NQ;  // components reduced per round and thread
  __shared__ double us[ND][32];
  __shared__ T red[NQ][NQ][32];
  const int lane = threadIdx.x & 31;
  const int q = threadIdx.x >> 5;
  const int64_t le = (int64_t)blockIdx.x * 32 + lane;
  const bool active = le < e_count && element_active(ps, le) &&
                      element_indices_ok<NN>(ps, conn, pos, E, e_begin + le);
  const int64_t e = e_begin + le;
  if (active) {
    for (int a = q; a < NN; a += NQ) {
      const int64_t node = conn[(int64_t)a * E + e];
#pragma unroll
      for (int i = 0; i < D; ++i) us[a * D + i][lane] = u[node * D + i];
    }
  }
  __syncthreads();
  T t[ND];
  if (active) {
    T ue[ND], b[ND];
#pragma unroll
    for (int c = 0; c < ND; ++c) {
      if constexpr (REL)
        ue[c] = (T)(us[c][lane] - us[c % D][lane]);
      else
        ue[c] = us[c][lane];
      b[c] = B[(int64_t)(q * ND + c) * E + e];
    }
    const T w = wJ[(int64_t)q * E + e];
    const MatParams mpe = group_params(mp, ps, le);
    element_law<D, NN, LAW, T, REL>(ue, b, w, mpe, ps, e_count, le, q, t);
  }
  // sum over q in increasing order, NQ components per round
#pragma unroll
  for (int round = 0; round < CH; ++round) {
    if (active) {
#pragma unroll
      for (int k = 0; k < NQ; ++k) {
        const int c = round * NQ + k;
        if (c < ND) red[q][k][lane] = t[c];
      }
    }
    __syncthreads();
    const int c = round * NQ + q;
    if (active && c < ND) {
      T s = red[0][q][lane];
#pragma unroll
      for (int qq = 1; qq < NQ; ++qq) s = s + red[qq][q][lane];
      const int a = c / D;
      re[(int64_t)pos[(int64_t)a * E + e] * SlotStride<D, RT>::value + (c - a * D)] = (RT)s;
    }
    __syncthreads();
  }
}

// The FP64 law of one (element, point), the operations of
// element_law<D, NN, LAW, double, false> in the same order, streamed: the
// nodal displacements are read from the block's staging us[c][lane], the
// point's dN/dx row b_a = B[(q ND + a D + j) E + e] is loaded node by node
// where the gradient and the force use it, and each force component c is
// handed to put(c, value) as soon as it is formed.  Nothing of size NN x D
// stays in registers, which leaves room for more resident warps.
template <int D, int NN, int LAW, class Put>
__device__ __forceinline__ void element_law_streamed(const double (*us)[32], int lane,
                                                     const double *Bq, int64_t E, double w,
                                                     const MatParams &mp, const GroupArgs &ps,
                                                     int64_t ne, int64_t le, int q, Put put) {
  // grad u = u B^T (shape_functions_inline_impl.hh:303-310): g(i, j) =
  // u_0,i b_0,j, then + u_a,i b_a,j for a ascending
  double g[D * D];
#pragma unroll
  for (int a = 0; a < NN; ++a) {
    double ba[D];
#pragma unroll
    for (int j = 0; j < D; ++j) ba[j] = Bq[(int64_t)(a * D + j) * E];
#pragma unroll
    for (int j = 0; j < D; ++j)
#pragma unroll
      for (int i = 0; i < D; ++i) {
        const double p = us[a * D + i][lane] * ba[j];
        g[i + D * j] = (a == 0) ? p : g[i + D * j] + p;
      }
  }
  subtract_eigen<D, double>(ps, ne, le, q, g);
  if constexpr (LAW == LAW_NEOHOOKEAN) {
    double S[D * D];
    finite_pk2<D, double>(mp, g, S, point_c33<D, double>(mp, ps, ne, le, q, g));
    double Sv[D == 3 ? 6 : 3];
    to_voigt<D, double>(S, Sv);
#pragma unroll
    for (int a = 0; a < NN; ++a) {
      double ba[D];
#pragma unroll
      for (int j = 0; j < D; ++j) ba[j] = ld_table(Bq + (int64_t)(a * D + j) * E);
#pragma unroll
      for (int k = 0; k < D; ++k) put(a * D + k, finite_force_component<D, double>(ba, g, Sv, k) * w);
    }
  } else {
    double sig[D * D];
    if constexpr (LAW == LAW_ELASTIC) {
      elastic_stress<D, double>(mp.lambda, mp.mu, g, mp.sigma_th, sig);
    } else {
      plastic_point<D, double>(mp, ps, ne, le, q, g, sig);
    }
    // sigma B, d x n (shape_lagrange_inline_impl.hh:402-408), times wJ_q
#pragma unroll
    for (int a = 0; a < NN; ++a) {
      double ba[D];
#pragma unroll
      for (int j = 0; j < D; ++j) ba[j] = ld_table(Bq + (int64_t)(a * D + j) * E);
#pragma unroll
      for (int i = 0; i < D; ++i) {
        double s = sig[i] * ba[0];
#pragma unroll
        for (int j = 1; j < D; ++j) s = s + sig[i + D * j] * ba[j];
        put(a * D + i, s * w);
      }
    }
  }
}

// k_element_forces_pq with the streamed law: the same thread layout (warp =
// point, lane = element), the same gather, the same sums over q in
// increasing order, bit for bit; every point's NN x D force components go to
// shared memory [q][component][lane] as they are formed and are summed in
// one round.  Dynamic shared memory: (NN D + NQ NN D) x 32 doubles (55,296
// bytes for hexahedra in 3D, above the 48 KB of static shared memory).
template <int D, int NN, int NQ, int LAW>
__global__ void __launch_bounds__(32 * NQ)
    k_element_forces_pqs(int64_t e_begin, int64_t e_count, int64_t E,
                         const int32_t *__restrict__ conn, const int32_t *__restrict__ pos,
                         const double *__restrict__ B, const double *__restrict__ wJ,
                         const double *__restrict__ u, MatParams mp, GroupArgs ps,
                         double *__restrict__ re) {
  pdl_begin();
  constexpr int ND = NN * D;
  extern __shared__ double pqs_smem[];
  double(*us)[32] = reinterpret_cast<double(*)[32]>(pqs_smem);
  double(*red)[ND][32] = reinterpret_cast<double(*)[ND][32]>(pqs_smem + ND * 32);
  const int lane = threadIdx.x & 31;
  const int q = threadIdx.x >> 5;
  const int64_t le = (int64_t)blockIdx.x * 32 + lane;
  const bool active = le < e_count && element_active(ps, le) &&
                      element_indices_ok<NN>(ps, conn, pos, E, e_begin + le);
  const int64_t e = e_begin + le;
  if (active) {
    for (int a = q; a < NN; a += NQ) {
      const int64_t node = conn[(int64_t)a * E + e];
#pragma unroll
      for (int i = 0; i < D; ++i) us[a * D + i][lane] = u[node * D + i];
    }
  }
  __syncthreads();
  if (active) {
    const double w = wJ[(int64_t)q * E + e];
    const MatParams mpe = group_params(mp, ps, le);
    element_law_streamed<D, NN, LAW>(us, lane, B + (int64_t)q * ND * E + e, E, w, mpe, ps,
                                     e_count, le, q,
                                     [&](int c, double v) { red[q][c][lane] = v; });
  }
  __syncthreads();
  if (active) {
#pragma unroll
    for (int c = q; c < ND; c += NQ) {
      double s = red[0][c][lane];
#pragma unroll
      for (int qq = 1; qq < NQ; ++qq) s = s + red[qq][c][lane];
      const int a = c / D;
      re[(int64_t)pos[(int64_t)a * E + e] * SlotStride<D, double>::value + (c - a * D)] = s;
    }
  }
}

// ---------------------------------------------------------------------------
// K5: node gather + residual + lumped solve + corrector
//   f_int = sum_slots (-1) r_e           (dof_manager.cc:65-120)
//   r = (0 + f_ext + f_int) + M (0 - a)  (solid_mechanics_model.cc:235-249,
//                                         dof_manager_default.cc:260-277)
//   x = r / M; v += (dt/2) x; a += x     (non_linear_solver_lumped.cc:76-87,
//                                         newmark-beta.cc:163-197)
// The displacement coefficient of the corrector is alpha*beta*dt^2 = 0.
// The elemental forces are stored in node-CSR order, so node i reads slots
// ptr[i] .. ptr[i+1] contiguously, in increasing slot order.
// flags: NU_CORRECT   residual, solve and corrector; the predicted velocity
//                     v + dt a of the reference predictor is formed here
//        NU_PREDICT   + the predictor of the next step,
//                     u_next = u + (dt v + (dt/2)(dt a))
//        NU_FINT      store the internal force (else it is gathered again on
//                     request by a flags == NU_FINT launch)
//        NU_FEXT_ZERO the external force is identically zero: not read
//                     (0 + f_ext + f_int == f_int)
// KAHAN selects a compensated FP64 sum (mixed path).
enum { NU_CORRECT = 1, NU_PREDICT = 2, NU_FINT = 4, NU_FEXT_ZERO = 8 };

// one slot into the internal-force sum, sign -1 (dof_manager.cc:65-120),
// optionally compensated
template <int D, bool KAHAN>
__device__ __forceinline__ void accumulate_slot(const double *rv, double *acc, double *comp) {
#pragma unroll
  for (int c = 0; c < D; ++c) {
    const double val = -1. * rv[c];
    if constexpr (KAHAN) {
      const double y = val - comp[c];
      const double tt = acc[c] + y;
      comp[c] = (tt - acc[c]) - y;
      acc[c] = tt;
    } else {
      acc[c] = acc[c] + val;
    }
  }
}

// the node update after the gather: f_int = acc, residual, solve, corrector
// and predictor of node i (its nodal state is loaded after the gather: loaded
// before it, with the slots, the update was measured slower, 0.120 against
// 0.107 ms on the 128^3 hexahedral box, at 66 instead of 50 registers)
template <int D>
__device__ __forceinline__ void node_apply(int64_t i, const double *acc, const double *fext,
                                           const double *mass, const uint8_t *blocked,
                                           double *fint, double *a, double *v, const double *u,
                                           double *u_next, double dt, const int32_t *node_inst,
                                           const double *inst_dt, int flags,
                                           unsigned int *status) {
  if (flags & NU_FINT) {
#pragma unroll
    for (int c = 0; c < D; ++c) fint[i * D + c] = acc[c];
  }
  if (!(flags & NU_CORRECT)) return;
  const double m = mass[i];
  const uint8_t bl = blocked[i];
  dt = node_dt(dt, node_inst, inst_dt, i);
  const double hdt = __dmul_rn(.5, dt);
  bool bad = false;
  // explicit round-to-nearest products and sums: the nodal state arithmetic is
  // the same (no contraction) in the FP64 and the mixed translation units,
  // and the fused predictor equals k_predict
#pragma unroll
  for (int c = 0; c < D; ++c) {
    const int64_t k = i * D + c;
    const bool free_dof = !((bl >> c) & 1);
    const double ak = a[k];
    double vk = v[k];
    if (free_dof) vk = __dadd_rn(vk, __dmul_rn(dt, ak));  // predicted velocity (newmark-beta.cc:69)
    double r;
    if (flags & NU_FEXT_ZERO) {
      r = acc[c];
    } else {
      r = __dadd_rn(0., __dmul_rn(1., fext[k]));
      r = __dadd_rn(r, __dmul_rn(1., acc[c]));
    }
    const double ma = __dadd_rn(0., __dmul_rn(-1., ak));
    r = __dadd_rn(r, __dmul_rn(m, ma));
    double an = ak;
    if (free_dof) {
      const double x = __dmul_rn(1., __ddiv_rn(r, m));
      vk = __dadd_rn(vk, __dmul_rn(hdt, x));
      an = __dadd_rn(ak, __dmul_rn(1., x));
      v[k] = vk;
      a[k] = an;
      bad |= !isfinite(an);
    }
    if (flags & NU_PREDICT) {
      const double uk = u[k];
      u_next[k] = free_dof ? __dadd_rn(uk, __dadd_rn(__dmul_rn(dt, vk),
                                                     __dmul_rn(hdt, __dmul_rn(dt, an))))
                           : uk;
    }
  }
  if (bad) atomicOr(status, 1u);
}

// 32 bytes of the slot array as one load (sm_100 256-bit global load): two
// float4 slots of 3D or four float2 slots of 2D; the address 32-byte aligned
__device__ __forceinline__ void load_32b(const float *q, float *f) {
  asm volatile("ld.global.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=f"(f[0]), "=f"(f[1]), "=f"(f[2]), "=f"(f[3]), "=f"(f[4]), "=f"(f[5]),
                 "=f"(f[6]), "=f"(f[7])
               : "l"(q));
}

__device__ __forceinline__ void load_32b(const double *q, double *f) {
  asm volatile("ld.global.v4.f64 {%0, %1, %2, %3}, [%4];"
               : "=d"(f[0]), "=d"(f[1]), "=d"(f[2]), "=d"(f[3])
               : "l"(q));
}

// AKB_BOUNDS_CHECK builds: node i's slot range lies within the CSR
// (0 <= ptr[i] <= ptr[i + 1] <= ptr[N]); a node whose range does not sets
// status bit 2 and is skipped
__device__ __forceinline__ bool node_range_ok(const int32_t *ptr, int64_t N, int64_t i,
                                              unsigned int *status) {
#ifdef AKB_BOUNDS_CHECK
  const int32_t p0 = ptr[i], p1 = ptr[i + 1], pn = ptr[N];
  if (p0 >= 0 && p0 <= p1 && p1 <= pn) return true;
  atomicOr(status, 4u);
  return false;
#else
  (void)ptr, (void)N, (void)i, (void)status;
  return true;
#endif
}

// A node's inputs to the update, loaded ahead of its slot gather by the
// state-first node update (the values node_apply reads itself)
template <int D> struct NodeState {
  double m;
  uint8_t bl;
  double a[D], v[D], f[D], u[D];
};

template <int D>
__device__ __forceinline__ void load_node_state(NodeState<D> &st, int64_t i, const double *fext,
                                                const double *a, const double *v,
                                                const double *u, int flags) {
#pragma unroll
  for (int c = 0; c < D; ++c) {
    const int64_t k = i * D + c;
    st.a[c] = a[k];
    st.v[c] = v[k];
    st.f[c] = (flags & NU_FEXT_ZERO) ? 0. : fext[k];
    st.u[c] = (flags & NU_PREDICT) ? u[k] : 0.;
  }
}

// node_apply on preloaded inputs: the same operations in the same order
template <int D>
__device__ __forceinline__ void node_apply_state(int64_t i, const double *acc,
                                                 const NodeState<D> &st, double *fint, double *a,
                                                 double *v, double *u_next, double dt,
                                                 const int32_t *node_inst,
                                                 const double *inst_dt, int flags,
                                                 unsigned int *status) {
  if (flags & NU_FINT) {
#pragma unroll
    for (int c = 0; c < D; ++c) fint[i * D + c] = acc[c];
  }
  if (!(flags & NU_CORRECT)) return;
  const double m = st.m;
  const uint8_t bl = st.bl;
  dt = node_dt(dt, node_inst, inst_dt, i);
  const double hdt = __dmul_rn(.5, dt);
  bool bad = false;
#pragma unroll
  for (int c = 0; c < D; ++c) {
    const int64_t k = i * D + c;
    const bool free_dof = !((bl >> c) & 1);
    const double ak = st.a[c];
    double vk = st.v[c];
    if (free_dof) vk = __dadd_rn(vk, __dmul_rn(dt, ak));
    double r;
    if (flags & NU_FEXT_ZERO) {
      r = acc[c];
    } else {
      r = __dadd_rn(0., __dmul_rn(1., st.f[c]));
      r = __dadd_rn(r, __dmul_rn(1., acc[c]));
    }
    const double ma = __dadd_rn(0., __dmul_rn(-1., ak));
    r = __dadd_rn(r, __dmul_rn(m, ma));
    double an = ak;
    if (free_dof) {
      const double x = __dmul_rn(1., __ddiv_rn(r, m));
      vk = __dadd_rn(vk, __dmul_rn(hdt, x));
      an = __dadd_rn(ak, __dmul_rn(1., x));
      v[k] = vk;
      a[k] = an;
      bad |= !isfinite(an);
    }
    if (flags & NU_PREDICT) {
      const double uk = st.u[c];
      u_next[k] = free_dof ? __dadd_rn(uk, __dadd_rn(__dmul_rn(dt, vk),
                                                     __dmul_rn(hdt, __dmul_rn(dt, an))))
                           : uk;
    }
  }
  if (bad) atomicOr(status, 1u);
}

// the node's slots p0 .. p1 summed in increasing slot order into acc (comp:
// the compensation of the Kahan sum); WIDE: slots read 32 bytes at a time
// (the launcher checks the slot array's alignment), same slots, same order
template <int D, class RT, bool KAHAN, bool WIDE>
__device__ __forceinline__ void gather_slots(int32_t p0, int32_t p1, const RT *re, double *acc,
                                             double *comp) {
  if constexpr (WIDE && std::is_same<RT, float>::value) {
    // floats per slot and slots per 32-byte load
    constexpr int FS = SlotStride<D, RT>::value, PER = 8 / FS;
    int32_t p = p0;
    for (; (p % PER) != 0 && p < p1; ++p) {
      double rv[D];
      load_slot<D>(re, p, rv);
      accumulate_slot<D, KAHAN>(rv, acc, comp);
    }
#pragma unroll 2
    for (; p + PER <= p1; p += PER) {
      float f[8];
      load_32b(reinterpret_cast<const float *>(re) + (int64_t)FS * p, f);
#pragma unroll
      for (int k = 0; k < PER; ++k) {
        double rv[D];
#pragma unroll
        for (int c = 0; c < D; ++c) rv[c] = (double)f[k * FS + c];
        accumulate_slot<D, KAHAN>(rv, acc, comp);
      }
    }
    for (; p < p1; ++p) {
      double rv[D];
      load_slot<D>(re, p, rv);
      accumulate_slot<D, KAHAN>(rv, acc, comp);
    }
  } else if constexpr (WIDE && std::is_same<RT, double>::value) {
    // FP64 slots of D doubles: G slots fill D * G / 4 loads of 32 bytes
    constexpr int G = D == 3 ? 4 : 2, NL = D * G / 4;
    int32_t p = p0;
    for (; (p % G) != 0 && p < p1; ++p) {
      double rv[D];
      load_slot<D>(re, p, rv);
      accumulate_slot<D, KAHAN>(rv, acc, comp);
    }
    for (; p + G <= p1; p += G) {
      double f[4 * NL];
#pragma unroll
      for (int l = 0; l < NL; ++l)
        load_32b(reinterpret_cast<const double *>(re) + (int64_t)D * p + 4 * l, f + 4 * l);
#pragma unroll
      for (int k = 0; k < G; ++k) {
        double rv[D];
#pragma unroll
        for (int c = 0; c < D; ++c) rv[c] = f[k * D + c];
        accumulate_slot<D, KAHAN>(rv, acc, comp);
      }
    }
    for (; p < p1; ++p) {
      double rv[D];
      load_slot<D>(re, p, rv);
      accumulate_slot<D, KAHAN>(rv, acc, comp);
    }
  } else {
#pragma unroll 4
    for (int32_t p = p0; p < p1; ++p) {
      double rv[D];
      load_slot<D>(re, p, rv);
      accumulate_slot<D, KAHAN>(rv, acc, comp);
    }
  }
}

// the gather and the node update of node i (WIDE: 32-byte slot loads)
template <int D, class RT, bool KAHAN, bool WIDE = false>
__device__ __forceinline__ void node_body(int64_t i, const int32_t *ptr,
                                          const RT *re,
                                          const double *fext,
                                          const double *mass,
                                          const uint8_t *blocked,
                                          double *fint, double *a,
                                          double *v, const double *u,
                                          double *u_next, double dt,
                                          const int32_t *node_inst,
                                          const double *inst_dt, int flags,
                                          unsigned int *status) {
  double acc[D], comp[D];
#pragma unroll
  for (int c = 0; c < D; ++c) {
    acc[c] = 0.;
    comp[c] = 0.;
  }
  const int32_t p0 = ptr[i], p1 = ptr[i + 1];
  gather_slots<D, RT, KAHAN, WIDE>(p0, p1, re, acc, comp);
  node_apply<D>(i, acc, fext, mass, blocked, fint, a, v, u, u_next, dt, node_inst, inst_dt, flags,
                status);
}


// launched with up to 1024 threads per block (the autotuner's candidates):
// at most 64 registers
template <int D, class RT, bool KAHAN, bool WIDE = false>
__global__ void __launch_bounds__(1024) k_node_update(int64_t N, const int32_t *__restrict__ ptr,
                              const RT *__restrict__ re, const double *__restrict__ fext,
                              const double *__restrict__ mass,
                              const uint8_t *__restrict__ blocked, double *__restrict__ fint,
                              double *__restrict__ a, double *__restrict__ v,
                              const double *__restrict__ u, double *__restrict__ u_next,
                              double dt, const int32_t *__restrict__ node_inst,
                              const double *__restrict__ inst_dt, int flags,
                              unsigned int *__restrict__ status) {
  pdl_begin();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N || !node_range_ok(ptr, N, i, status)) return;
  node_body<D, RT, KAHAN, WIDE>(i, ptr, re, fext, mass, blocked, fint, a, v, u, u_next, dt,
                                node_inst, inst_dt, flags, status);
}

// State-first form of k_node_update (the same numbers): the node's slot
// range, mass and blocked flags, which no step changes, are read before the
// wait on the preceding kernel (a dependent launch starts them under that
// kernel's tail), and its a, v, f_ext and u before the slot gather, so that
// they are in flight together with it rather than after it
template <int D, class RT, bool KAHAN, bool WIDE = false>
__global__ void __launch_bounds__(1024)
    k_node_update_early(int64_t N, const int32_t *__restrict__ ptr, const RT *__restrict__ re,
                        const double *__restrict__ fext, const double *__restrict__ mass,
                        const uint8_t *__restrict__ blocked, double *__restrict__ fint,
                        double *__restrict__ a, double *__restrict__ v,
                        const double *__restrict__ u, double *__restrict__ u_next, double dt,
                        const int32_t *__restrict__ node_inst, const double *__restrict__ inst_dt,
                        int flags, unsigned int *__restrict__ status) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool in = i < N;
  int32_t p0 = 0, p1 = 0;
  NodeState<D> st;
  st.m = 1.;
  st.bl = 0;
  if (in) {
    p0 = ptr[i];
    p1 = ptr[i + 1];
    st.m = mass[i];
    st.bl = blocked[i];
  }
  pdl_begin();
  if (!in || !node_range_ok(ptr, N, i, status)) return;
  if (flags & NU_CORRECT) load_node_state<D>(st, i, fext, a, v, u, flags);
  double acc[D], comp[D];
#pragma unroll
  for (int c = 0; c < D; ++c) {
    acc[c] = 0.;
    comp[c] = 0.;
  }
  gather_slots<D, RT, KAHAN, WIDE>(p0, p1, re, acc, comp);
  node_apply_state<D>(i, acc, st, fint, a, v, u_next, dt, node_inst, inst_dt, flags, status);
}

// Node update of a batch whose instances stop after their own step counts:
// a node of a stopped instance keeps its state; the displacement buffer that
// becomes the model's displacement after this step (u, the prediction's
// buffer) takes the value of the other one (u_next), which holds the
// instance's last displacement, so that both buffers hold it from then on
template <int D, class RT, bool KAHAN>
__global__ void __launch_bounds__(1024) k_node_update_retire(int64_t N, const int32_t *__restrict__ ptr,
                                     const RT *__restrict__ re, const double *__restrict__ fext,
                                     const double *__restrict__ mass,
                                     const uint8_t *__restrict__ blocked,
                                     double *__restrict__ fint, double *__restrict__ a,
                                     double *__restrict__ v, double *u, double *u_next, double dt,
                                     const int32_t *__restrict__ node_inst,
                                     const double *__restrict__ inst_dt,
                                     const int64_t *__restrict__ inst_end,
                                     const int64_t *__restrict__ step, int flags,
                                     unsigned int *__restrict__ status) {
  pdl_begin();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N || !node_range_ok(ptr, N, i, status)) return;
  // a batch of one instance has no node -> instance table
  if (*step >= inst_end[node_inst ? node_inst[i] : 0]) {
    if (flags & NU_PREDICT) {
#pragma unroll
      for (int c = 0; c < D; ++c) u[i * D + c] = u_next[i * D + c];
    }
    return;
  }
  node_body<D, RT, KAHAN, false>(i, ptr, re, fext, mass, blocked, fint, a, v, u, u_next, dt,
                                 node_inst, inst_dt, flags, status);
}

// the step counter of a batch with stopping instances, after each step
static __global__ void k_step_advance(int64_t *step) {
  pdl_begin();
  *step += 1;
}

// Node update with the gather staged through shared memory: the slots of
// BLOCK consecutive nodes are one contiguous range of the slot array, loaded
// in chunks with coalesced vector loads (the direct form makes each thread
// read its own node's slots, which a warp spreads over 32 separate ranges);
// each thread then sums its node's slots from shared memory in the same order
// as the direct form, so the results are identical.  Slot vectors are stored
// at an XOR-swizzled index so that threads reading ranges a multiple of 8
// vectors apart hit different banks.
template <int D, class RT> struct SlotVec;
template <> struct SlotVec<3, float> { using type = float4; static constexpr int per_slot = 1; };
template <> struct SlotVec<2, float> { using type = float2; static constexpr int per_slot = 1; };
template <> struct SlotVec<2, double> { using type = double2; static constexpr int per_slot = 1; };
template <> struct SlotVec<3, double> { using type = double; static constexpr int per_slot = 3; };

constexpr int kStagedBytes = 32768;

__device__ __forceinline__ int swizzle(int w) { return w ^ ((w >> 3) & 7); }

template <int D, class RT, bool KAHAN, int BLOCK>
__global__ void __launch_bounds__(BLOCK)
    k_node_update_staged(int64_t N, const int32_t *__restrict__ ptr, const RT *__restrict__ re,
                         const double *__restrict__ fext, const double *__restrict__ mass,
                         const uint8_t *__restrict__ blocked, double *__restrict__ fint,
                         double *__restrict__ a, double *__restrict__ v,
                         const double *__restrict__ u, double *__restrict__ u_next, double dt,
                         const int32_t *__restrict__ node_inst,
                         const double *__restrict__ inst_dt, int flags,
                         unsigned int *__restrict__ status) {
  pdl_begin();
  using V = typename SlotVec<D, RT>::type;
  constexpr int WPS = SlotVec<D, RT>::per_slot;  // vectors per slot
  constexpr int CAPW = kStagedBytes / (int)sizeof(V);
  constexpr int CAP = CAPW / WPS;               // slots per chunk
  __shared__ V sm[CAPW];
  const int64_t i0 = (int64_t)blockIdx.x * BLOCK;
  const int64_t i = i0 + threadIdx.x;
  const int64_t iend = i0 + BLOCK < N ? i0 + BLOCK : N;
  const int32_t pb = ptr[i0], pe = ptr[iend];
  const int32_t p0 = i < N ? ptr[i] : pe, p1 = i < N ? ptr[i + 1] : pe;
  const V *src = reinterpret_cast<const V *>(re);
  double acc[D], comp[D];
#pragma unroll
  for (int c = 0; c < D; ++c) {
    acc[c] = 0.;
    comp[c] = 0.;
  }
  for (int32_t cb = pb; cb < pe; cb += CAP) {
    const int32_t ce = cb + CAP < pe ? cb + CAP : pe;
    __syncthreads();
    const int nw = (ce - cb) * WPS;
    for (int w = threadIdx.x; w < nw; w += BLOCK) sm[swizzle(w)] = src[(int64_t)cb * WPS + w];
    __syncthreads();
    const int32_t lo = p0 > cb ? p0 : cb, hi = p1 < ce ? p1 : ce;
    for (int32_t p = lo; p < hi; ++p) {
      double rv[D];
      const int w = (p - cb) * WPS;
      if constexpr (WPS == 1) {
        const V x = sm[swizzle(w)];
        rv[0] = (double)x.x;
        rv[1] = (double)x.y;
        if constexpr (D == 3) rv[2] = (double)reinterpret_cast<const float4 &>(x).z;
      } else {
#pragma unroll
        for (int c = 0; c < D; ++c) rv[c] = (double)sm[swizzle(w + c)];
      }
      accumulate_slot<D, KAHAN>(rv, acc, comp);
    }
  }
  if (i >= N) return;
  node_apply<D>(i, acc, fext, mass, blocked, fint, a, v, u, u_next, dt, node_inst, inst_dt, flags,
                status);
}

// ---------------------------------------------------------------------------
// Persistent multi-step kernel for small meshes of one law group.  All
// blocks are resident (cooperative launch); each step runs the element phase
// and the node phase over grid-stride loops, separated by grid barriers, with
// the same per-element and per-node functions as the two-kernel path, so the
// results are bit-identical to it.  The pointers below carry no __restrict__:
// the displacement, the slots and the state are written and read again in the
// same launch, so their loads must not take the read-only path.
struct StepArgs {
  int64_t E, N;
  const int32_t *conn, *pos, *ptr;
  const void *B, *wJ;  // streamed dN/dx and det J w, element-math type
  const double *X;
  MatParams mp;
  GroupArgs ps;        // state buffers of the first step
  void *re;
  const double *fext, *mass;
  const uint8_t *blocked;
  double *fint, *a, *v;
  double *u_pred;      // displacement the first step starts from
  double *u_other;     // receives the prediction of the step after it
  double dt;
  const int32_t *node_inst;
  const double *inst_dt;
  int flags;           // node-update flags of a step (NU_CORRECT | NU_PREDICT ...)
  int plastic;         // swap the plastic state buffers after each step
  int64_t nsteps;
  unsigned int *status;
  unsigned int *bar;   // [1 + blocks]: release generation, then one arrival flag per block
  // the barrier's bound on its waits (sleeps of about 32 ns each), and a
  // failure-path setting: block late_block (>= 0) first sleeps late_us
  // microseconds, so that a short bound runs out (status bit 1)
  unsigned int spin_limit;
  int late_block;
  unsigned int late_us;
};

constexpr int kPersistentThreads = 256;
constexpr unsigned int kBarrierSpinLimit = 1u << 24;  // x 64 ns sleeps: about a second
constexpr unsigned int ST_BARRIER_TIMEOUT = 2u;

// grid-wide barrier number `gen` (1, 2, ... within a launch) with bounded
// waits: every block publishes its arrival in its own flag (no contended
// atomic), the first warp of block 0 waits for all flags and then publishes
// the release, which the other blocks wait for.  Returns false (status bit 1
// set) when a wait ran out.
__device__ __forceinline__ bool grid_barrier(unsigned int *bar, unsigned int gen,
                                             unsigned int *status, unsigned int spin_limit) {
  __shared__ int ok;
  volatile unsigned int *release = bar;
  volatile unsigned int *arrive = bar + 1;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    __threadfence();
    arrive[blockIdx.x] = gen;
  }
  if (blockIdx.x == 0) {
    if (threadIdx.x < 32) {
      bool fine = true;
      for (unsigned int b = threadIdx.x; b < gridDim.x && fine; b += 32) {
        unsigned int spins = 0;
        while (arrive[b] != gen) {
          if (++spins > spin_limit) {
            fine = false;
            break;
          }
          __nanosleep(32);
        }
      }
      fine = __all_sync(0xffffffffu, fine);
      if (threadIdx.x == 0) {
        if (!fine) atomicOr(status, ST_BARRIER_TIMEOUT);
        __threadfence();
        *release = gen;  // released even after a timeout, so no block waits on
      }
    }
  } else if (threadIdx.x == 0) {
    unsigned int spins = 0;
    while (*release != gen) {
      if (++spins > spin_limit) {
        atomicOr(status, ST_BARRIER_TIMEOUT);
        break;
      }
      __nanosleep(32);
    }
  }
  if (threadIdx.x == 0) {
    __threadfence();
    if (*(volatile unsigned int *)status & ST_BARRIER_TIMEOUT) ok = 0;
  }
  __syncthreads();
  return ok != 0;
}

__device__ __forceinline__ void swap_state(GroupArgs &ps) {
  const double *t;
  t = ps.sig_prev; ps.sig_prev = ps.sig; ps.sig = const_cast<double *>(t);
  t = ps.eps_prev; ps.eps_prev = ps.eps; ps.eps = const_cast<double *>(t);
  t = ps.iso_prev; ps.iso_prev = ps.iso; ps.iso = const_cast<double *>(t);
  const void *tg = ps.gu_prev; ps.gu_prev = ps.gu; ps.gu = const_cast<void *>(tg);
  ps.iso_cur_in = ps.iso_prev;
}

// FORM: 0 streamed dN/dx (element_pe, T), 1 recomputed in FP32
// (element_geo), 2 sum-factorised hexahedron with QU points per iteration
template <int D, int NN, int NQ, int LAW, int FORM, class T, class RT, bool KAHAN, int QU>
__global__ void __launch_bounds__(kPersistentThreads)
    k_persistent_steps(StepArgs sa, QuadTable tab) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  GroupArgs ps = sa.ps;
  double *up = sa.u_pred, *uo = sa.u_other;
  RT *re = static_cast<RT *>(sa.re);
  unsigned int gen = 0;
  if ((int)blockIdx.x == sa.late_block && threadIdx.x == 0)
    for (unsigned int k = 0; k < sa.late_us; ++k) __nanosleep(1000);
  for (int64_t s = 0; s < sa.nsteps; ++s) {
    for (int64_t le = t0; le < sa.E; le += stride) {
      const MatParams &mp = sa.mp;
      if constexpr (FORM == 0)
        element_pe<D, NN, NQ, LAW, T, RT>(le, 0, sa.E, sa.E, sa.conn, sa.pos,
                                          static_cast<const T *>(sa.B),
                                          static_cast<const T *>(sa.wJ), up, mp, ps, re);
      else if constexpr (FORM == 1)
        element_geo<D, NN, NQ, LAW>(le, 0, sa.E, sa.E, sa.conn, sa.pos, sa.X, tab, up, mp, ps,
                                    reinterpret_cast<float *>(re));
      else
        element_hex8sf<LAW, QU, false, false, float>(le, 0, sa.E, sa.E, sa.conn, sa.pos, sa.X,
                                                     static_cast<const float *>(nullptr), up,
                                                     mp, ps, reinterpret_cast<float *>(re));
    }
    if (!grid_barrier(sa.bar, ++gen, sa.status, sa.spin_limit)) return;
    for (int64_t i = t0; i < sa.N; i += stride)
      node_body<D, RT, KAHAN>(i, sa.ptr, re, sa.fext, sa.mass, sa.blocked, sa.fint, sa.a, sa.v,
                              up, uo, sa.dt, sa.node_inst, sa.inst_dt, sa.flags, sa.status);
    if (!grid_barrier(sa.bar, ++gen, sa.status, sa.spin_limit)) return;
    double *tu = up;
    up = uo;
    uo = tu;
    if (sa.plastic) swap_state(ps);
  }
}

// ---------------------------------------------------------------------------
// quadrature-point fields of elastic / neohookean materials, evaluated from a
// displacement snapshot (the reference keeps them as internals,
// material.cc:128-154).  Output [q][D*D][ne].
template <int D, int NN, int NQ, int LAW>
// c33: the stored plane-stress stretches of the material's points at
// c33[q * c33_ld + le] (read only: the getter reports the stress of the last
// evaluation), or null
__global__ void k_qp_fields(int64_t e_begin, int64_t e_count, int64_t E,
                            const int32_t *__restrict__ conn, const double *__restrict__ B,
                            const double *__restrict__ u, MatParams mp,
                            const double *__restrict__ c33, int64_t c33_ld,
                            const double *__restrict__ eig,
                            double *__restrict__ grad_out, double *__restrict__ stress_out) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= e_count * NQ) return;
  const int q = (int)(t / e_count);
  const int64_t le = t - (int64_t)q * e_count;
  const int64_t e = e_begin + le;
  double ue[NN * D], b[NN * D];
#pragma unroll
  for (int a = 0; a < NN; ++a) {
    const int64_t node = conn[(int64_t)a * E + e];
#pragma unroll
    for (int i = 0; i < D; ++i) ue[a * D + i] = u[node * D + i];
  }
#pragma unroll
  for (int c = 0; c < NN * D; ++c) b[c] = B[(int64_t)(q * NN * D + c) * E + e];
  double g[D * D], s[D * D];
#pragma unroll
  for (int j = 0; j < D; ++j)
#pragma unroll
    for (int i = 0; i < D; ++i) {
      double acc = ue[i] * b[j];
#pragma unroll
      for (int a = 1; a < NN; ++a) acc = acc + ue[a * D + i] * b[a * D + j];
      g[i + D * j] = acc;
    }
  if (eig) {
#pragma unroll
    for (int k = 0; k < D * D; ++k) g[k] = g[k] - eig[(int64_t)(q * D * D + k) * c33_ld + le];
  }
  if constexpr (LAW == LAW_NEOHOOKEAN)
    finite_pk2<D, double>(mp, g, s, (c33 && mp.c33) ? c33[(int64_t)q * c33_ld + le] : 0.);
  else
    elastic_stress<D, double>(mp.lambda, mp.mu, g, mp.sigma_th, s);
#pragma unroll
  for (int k = 0; k < D * D; ++k) {
    grad_out[(int64_t)(q * D * D + k) * e_count + le] = g[k];
    stress_out[(int64_t)(q * D * D + k) * e_count + le] = s[k];
  }
}

}  // namespace akb

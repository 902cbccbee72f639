// FP64 kernels and their launchers.  Built with --fmad=false: no contraction,
// so the arithmetic matches the CPU path operation for operation.
#include <type_traits>

#include "dispatch.cuh"

namespace akb {

// ---- init ------------------------------------------------------------------
cudaError_t launch_precompute(const DevGeom &g, const QuadTable &tab, double *B, double *wJ,
                              unsigned long long *bad, cudaStream_t s) {
  if (g.E == 0) return cudaSuccess;
  AKB_DISPATCH_ELEM(g, {
    (void)ET;
    k_precompute<D, NN, NQ><<<grid_for(g.E * NQ), kThreads, 0, s>>>(g.X, g.conn, g.E, tab, B,
                                                                      wJ, bad);
  });
  return cudaGetLastError();
}

cudaError_t launch_mass_elem(const DevGeom &g, int64_t e0, int64_t ne, double rho,
                             const QuadTable &tab, const double *wJ, double *me,
                             cudaStream_t s) {
  if (ne == 0) return cudaSuccess;
  AKB_DISPATCH_ELEM(g, {
    (void)D;
    k_mass_elem<NN, NQ, ET == ET_TRI6><<<grid_for(ne), kThreads, 0, s>>>(e0, ne, g.E, rho, tab,
                                                                         wJ, me);
  });
  return cudaGetLastError();
}

cudaError_t launch_gather_scalar(const DevGeom &g, const double *me, double *out,
                                 cudaStream_t s) {
  if (g.N == 0) return cudaSuccess;
  k_gather_scalar<<<grid_for(g.N), kThreads, 0, s>>>(g.N, g.ptr, g.ent, me, out);
  return cudaGetLastError();
}

cudaError_t launch_element_dt(const DevGeom &g, int64_t e0, int64_t ne, double celerity,
                              const double *u, const int32_t *perm, double *out,
                              cudaStream_t s) {
  if (ne == 0) return cudaSuccess;
  AKB_DISPATCH_ELEM(g, {
    (void)NQ;
    k_element_dt<ET, D, NN><<<grid_for(ne), kThreads, 0, s>>>(e0, ne, g.E, celerity, g.conn,
                                                              g.X, u, perm, out);
  });
  return cudaGetLastError();
}

cudaError_t launch_segment_min(const double *x, const int64_t *off, int nseg, double *out,
                               cudaStream_t s) {
  if (nseg == 0) return cudaSuccess;
  k_segment_min<<<nseg, 256, 0, s>>>(x, off, out);
  return cudaGetLastError();
}

__global__ void k_fill(double *__restrict__ out, double v, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = v;
}
cudaError_t launch_fill(double *out, double v, int64_t n, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_fill<<<grid_for(n), kThreads, 0, s>>>(out, v, n);
  return cudaGetLastError();
}

__global__ void k_to_float(const double *__restrict__ in, float *__restrict__ out, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (float)in[i];
}
cudaError_t launch_to_float(const double *in, float *out, int64_t n, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_to_float<<<grid_for(n), kThreads, 0, s>>>(in, out, n);
  return cudaGetLastError();
}

// ---- step ------------------------------------------------------------------
cudaError_t launch_predict(const DevGeom &g, const uint8_t *blocked, const double *u,
                           const double *v, const double *a, double dt, double *u_pred,
                           cudaStream_t s) {
  if (g.N == 0) return cudaSuccess;
  auto kern = g.D == 3 ? k_predict<3> : k_predict<2>;
  return launch_step(g.pdl, kern, grid_for(g.N * g.D), kThreads, s, g.N, blocked, u, v, a, dt,
                     g.node_inst, g.inst_dt, u_pred);
}

cudaError_t launch_element_forces_fp64(const DevGeom &g, int law, int64_t e0, int64_t ne,
                                       const double *B, const double *wJ, const double *u,
                                       const MatParams &mp, const GroupArgs &ps,
                                       double *re, const ElemTuning &tn, const QuadTable &tab,
                                       cudaStream_t s) {
  return element_forces_impl<double, double>(g, law, e0, ne, B, wJ, u, mp, ps, re, tn, &tab, s);
}

cudaError_t launch_persistent_fp64(const DevGeom &g, int law, int qu, const StepArgs &sa,
                                   const QuadTable &tab, cudaStream_t s) {
  (void)qu;
  const int64_t work = std::max(g.E, g.N);
  AKB_DISPATCH_ELEM(g, {
    (void)ET;
    if (law == LAW_ELASTIC)
      return launch_cooperative(
          k_persistent_steps<D, NN, NQ, LAW_ELASTIC, 0, double, double, false, 1>, work, sa,
          tab, s);
    if (law == LAW_NEOHOOKEAN)
      return launch_cooperative(
          k_persistent_steps<D, NN, NQ, LAW_NEOHOOKEAN, 0, double, double, false, 1>, work, sa,
          tab, s);
    return launch_cooperative(
        k_persistent_steps<D, NN, NQ, LAW_PLASTIC, 0, double, double, false, 1>, work, sa, tab,
        s);
  });
  return cudaErrorInvalidValue;
}

cudaError_t launch_node_update_fp64(const DevGeom &g, const double *re, const double *fext,
                                    const double *mass, const uint8_t *blocked, double *fint,
                                    double *a, double *v, const double *u, double *u_next,
                                    double dt, int flags, unsigned int *status, int node_block,
                                    int form, cudaStream_t s) {
  if (g.N > 0 && g.inst_end) {
    auto kern = g.D == 3 ? k_node_update_retire<3, double, false> : k_node_update_retire<2, double, false>;
    return launch_step(g.pdl, kern, grid_for(g.N, node_block), node_block, s, g.N, g.ptr, re,
                       fext, mass, blocked, fint, a, v, const_cast<double *>(u), u_next, dt,
                       g.node_inst, g.inst_dt, g.inst_end, (const int64_t *)g.step, flags, status);
  }
  if (g.N == 0) return cudaSuccess;
#ifdef AKB_BOUNDS_CHECK
  if (form == 1) form = 0;  // the bounds-checking build checks each node's own slot range
#endif
  if (form == 1) {
    AKB_DISPATCH_NODE_BLOCK(node_block, {
      auto kern = g.D == 3 ? k_node_update_staged<3, double, false, NB>
                           : k_node_update_staged<2, double, false, NB>;
      return launch_step(g.pdl, kern, grid_for(g.N, NB), NB, s, g.N, g.ptr, re, fext, mass,
                         blocked, fint, a, v, u, u_next, dt, g.node_inst, g.inst_dt, flags,
                         status);
    });
  }
  // slots read 32 bytes at a time when the array's alignment allows it
  const bool wide = ((uintptr_t)re & 31) == 0;
  auto kern = g.D == 3 ? (wide ? k_node_update<3, double, false, true>
                               : k_node_update<3, double, false>)
                       : (wide ? k_node_update<2, double, false, true>
                               : k_node_update<2, double, false>);
  if (form == 2)
    kern = g.D == 3 ? (wide ? k_node_update_early<3, double, false, true>
                            : k_node_update_early<3, double, false>)
                    : (wide ? k_node_update_early<2, double, false, true>
                            : k_node_update_early<2, double, false>);
  return launch_step(g.pdl, kern, grid_for(g.N, node_block), node_block, s, g.N, g.ptr, re,
                     fext, mass, blocked, fint, a, v, u, u_next, dt, g.node_inst, g.inst_dt,
                     flags, status);
}

// prescribed motion: before step k (k = 1, 2, ... since the motion was set)
// the listed dofs get u = u0 + sum_{j <= k} dt v_max min(1, j / ramp_steps),
// the cumulative displacement of a velocity ramped linearly to v_max over
// ramp_steps steps.  One block: thread 0 advances the step counter and the
// running sum (advance != 0; else the sum of the coming step is applied
// again), then the block writes the dofs into the displacement the coming
// step starts from.
__global__ void k_prescribe(int64_t count, const int64_t *__restrict__ dofs,
                            const double *__restrict__ u0, double v_max, double ramp_steps,
                            double dt, double *__restrict__ acc, int64_t *__restrict__ step,
                            double *__restrict__ u, int advance) {
  pdl_begin();
  __shared__ double a_sh;
  if (threadIdx.x == 0) {
    double a = *acc;
    if (advance) {
      const int64_t k = *step + 1;
      const double vk = v_max * fmin(1.0, (double)k / ramp_steps);
      a = a + dt * vk;
      *step = k;
      *acc = a;
    }
    a_sh = a;
  }
  __syncthreads();
  const double a = a_sh;
  for (int64_t i = threadIdx.x; i < count; i += blockDim.x) u[dofs[i]] = u0[i] + a;
}
cudaError_t launch_prescribe(int64_t count, const int64_t *dofs, const double *u0, double v_max,
                             int64_t ramp_steps, double dt, double *acc, int64_t *step,
                             double *u, bool advance, bool pdl, cudaStream_t s) {
  return launch_step(pdl, k_prescribe, 1, 512, s, count, dofs, u0, v_max, (double)ramp_steps,
                     dt, acc, step, u, advance ? 1 : 0);
}

cudaError_t launch_step_advance(const DevGeom &g, cudaStream_t s) {
  return launch_step(g.pdl, k_step_advance, 1, 1, s, g.step);
}

// ---- fields and energies ---------------------------------------------------
cudaError_t launch_qp_fields(const DevGeom &g, int law, int64_t e0, int64_t ne,
                             const double *B, const double *u, const MatParams &mp,
                             const double *c33, int64_t c33_ld, const double *eig,
                             double *grad, double *stress, cudaStream_t s) {
  if (ne == 0) return cudaSuccess;
  AKB_DISPATCH_ELEM(g, {
    (void)ET;
    if (law == LAW_NEOHOOKEAN)
      k_qp_fields<D, NN, NQ, LAW_NEOHOOKEAN><<<grid_for(ne * NQ), kThreads, 0, s>>>(
          e0, ne, g.E, g.conn, B, u, mp, c33, c33_ld, eig, grad, stress);
    else
      k_qp_fields<D, NN, NQ, LAW_ELASTIC><<<grid_for(ne * NQ), kThreads, 0, s>>>(
          e0, ne, g.E, g.conn, B, u, mp, c33, c33_ld, eig, grad, stress);
  });
  return cudaGetLastError();
}

// kinetic energy terms (solid_mechanics_model.cc:476-527): per node
// mv2 = sum_c (m > eps ? v v m : 0)
template <int D>
__global__ void k_ekin_terms(int64_t N, const double *__restrict__ v,
                             const double *__restrict__ mass, double *__restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double m = mass[i];
  double mv2 = 0.;
#pragma unroll
  for (int c = 0; c < D; ++c) {
    const double vv = v[i * D + c];
    if (m > 2.220446049250313080847e-16) mv2 += vv * vv * m;
  }
  out[i] = mv2;
}
cudaError_t launch_ekin_terms(const DevGeom &g, const double *v, const double *mass,
                              double *out, cudaStream_t s) {
  if (g.N == 0) return cudaSuccess;
  if (g.D == 3)
    k_ekin_terms<3><<<grid_for(g.N), kThreads, 0, s>>>(g.N, v, mass, out);
  else
    k_ekin_terms<2><<<grid_for(g.N), kThreads, 0, s>>>(g.N, v, mass, out);
  return cudaGetLastError();
}

// external work terms (solid_mechanics_model.cc:556-598)
template <int D>
__global__ void k_work_terms(int64_t N, const double *__restrict__ fext,
                             const double *__restrict__ fint, const double *__restrict__ v,
                             const uint8_t *__restrict__ blocked, double *__restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double w = 0.;
  const uint8_t bl = blocked[i];
#pragma unroll
  for (int c = 0; c < D; ++c) {
    const int64_t k = i * D + c;
    if ((bl >> c) & 1)
      w -= fint[k] * v[k];
    else
      w += fext[k] * v[k];
  }
  out[i] = w;
}
cudaError_t launch_work_terms(const DevGeom &g, const double *fext, const double *fint,
                              const double *v, const uint8_t *blocked, double *out,
                              cudaStream_t s) {
  if (g.N == 0) return cudaSuccess;
  if (g.D == 3)
    k_work_terms<3><<<grid_for(g.N), kThreads, 0, s>>>(g.N, fext, fint, v, blocked, out);
  else
    k_work_terms<2><<<grid_for(g.N), kThreads, 0, s>>>(g.N, fext, fint, v, blocked, out);
  return cudaGetLastError();
}

// per-element integral of an energy density (Material::getPotentialEnergy,
// material.cc:604-619; MaterialPlastic::getPlasticEnergy, material_plastic.cc:47-69).
// Quadrature-point inputs are [q][comp][ld]; wJ is [q][E].  Plastic inputs
// are the group's internals: the gradient in GT, stress and plastic strain
// as symmetric components.
template <int D, int NQ, int LAW, class GT>
__global__ void k_energy_elem(int which, int64_t e0, int64_t ne, int64_t ld, int64_t E,
                              const double *__restrict__ wJ, const GT *__restrict__ grad,
                              const double *__restrict__ stress,
                              const double *__restrict__ eps_p, const double *__restrict__ pe,
                              MatParams mp, double *__restrict__ out) {
  const int64_t le = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (le >= ne) return;
  constexpr int DD = D * D, NS = SymComps<D>::value;
  double el = 0.;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    auto at = [&](int k) { return (int64_t)(q * DD + k) * ld + le; };
    auto sym = [&](int k) { return (int64_t)(q * NS + sym_of<D>(k)) * ld + le; };
    double dens;
    if (which == 1) {
      dens = pe[(int64_t)q * ld + le];
    } else if (LAW == LAW_NEOHOOKEAN) {
      double F[DD];
#pragma unroll
      for (int j = 0; j < D; ++j)
#pragma unroll
        for (int i = 0; i < D; ++i) F[i + D * j] = (i == j ? 1. : 0.) + (double)grad[at(i + D * j)];
      double trC = 0.;
#pragma unroll
      for (int i = 0; i < D; ++i) {
        double tt = F[0 + D * i] * F[0 + D * i];
#pragma unroll
        for (int k = 1; k < D; ++k) tt = tt + F[k + D * i] * F[k + D * i];
        trC = (i == 0) ? tt : trC + tt;
      }
      if (mp.svk) {
        // finite-deformation elastic: .5 S : E (material_elastic.cc:140-157,
        // material_elastic_inline_impl.hh:113-116), S the stored PK2 stress
        double g[DD], E[DD];
#pragma unroll
        for (int k = 0; k < DD; ++k) g[k] = (double)grad[at(k)];
        green_lagrange<D, double>(g, E);
        double dot = 0.;
#pragma unroll
        for (int k = 0; k < DD; ++k) {
          const double sk = stress[at(k)];
          dot = (k == 0) ? sk * E[k] : dot + sk * E[k];
        }
        dens = .5 * dot;
      } else {
        double J;
        if constexpr (D == 3) J = det3(F); else J = det2(F);
        dens = mp.lambda * pow(log(J), 2.) + mp.mu * (-log(J) + (trC - D) / 2.) / 2.;
      }
    } else {
      double dot = 0.;
#pragma unroll
      for (int k = 0; k < DD; ++k) {
        double ge = (double)grad[at(k)];
        if (LAW == LAW_PLASTIC) ge = ge - eps_p[sym(k)];
        const double sk = LAW == LAW_PLASTIC ? stress[sym(k)] : stress[at(k)];
        dot = (k == 0) ? sk * ge : dot + sk * ge;
      }
      dens = .5 * dot;
    }
    const double w = wJ[(int64_t)q * E + e0 + le];
    el = (q == 0) ? dens * w : el + dens * w;
  }
  out[le] = el;
}
cudaError_t launch_energy_elem(const DevGeom &g, int law, int which, int64_t e0, int64_t ne,
                               int64_t ld, const double *wJ, const void *grad,
                               bool grad_float, const double *stress, const double *eps_p,
                               const double *pe, const MatParams &mp, double *out,
                               cudaStream_t s) {
  if (ne == 0) return cudaSuccess;
  const double *gd = static_cast<const double *>(grad);
  AKB_DISPATCH_ELEM(g, {
    (void)ET;
    (void)NN;
    if (law == LAW_NEOHOOKEAN)
      k_energy_elem<D, NQ, LAW_NEOHOOKEAN, double><<<grid_for(ne), kThreads, 0, s>>>(
          which, e0, ne, ld, g.E, wJ, gd, stress, eps_p, pe, mp, out);
    else if (law == LAW_PLASTIC && grad_float)
      k_energy_elem<D, NQ, LAW_PLASTIC, float><<<grid_for(ne), kThreads, 0, s>>>(
          which, e0, ne, ld, g.E, wJ, static_cast<const float *>(grad), stress, eps_p, pe, mp,
          out);
    else if (law == LAW_PLASTIC)
      k_energy_elem<D, NQ, LAW_PLASTIC, double><<<grid_for(ne), kThreads, 0, s>>>(
          which, e0, ne, ld, g.E, wJ, gd, stress, eps_p, pe, mp, out);
    else
      k_energy_elem<D, NQ, LAW_ELASTIC, double><<<grid_for(ne), kThreads, 0, s>>>(
          which, e0, ne, ld, g.E, wJ, gd, stress, eps_p, pe, mp, out);
  });
  return cudaGetLastError();
}

// deterministic two-level reduction: block b sums the strided set
// {i : i % gridDim == b} in increasing i per thread, then a fixed smem tree
template <int OPMIN>
__global__ void k_reduce_partial(const double *__restrict__ x, int64_t n,
                                 double *__restrict__ partials) {
  __shared__ double sm[256];
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  double acc = OPMIN ? 1.7976931348623157e308 : 0.;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    acc = OPMIN ? fmin(acc, x[i]) : acc + x[i];
  sm[threadIdx.x] = acc;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      sm[threadIdx.x] = OPMIN ? fmin(sm[threadIdx.x], sm[threadIdx.x + w])
                              : sm[threadIdx.x] + sm[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = sm[0];
}
template <int OPMIN>
__global__ void k_reduce_final(const double *__restrict__ partials, int np,
                               double *__restrict__ out) {
  __shared__ double sm[1024];
  double acc = OPMIN ? 1.7976931348623157e308 : 0.;
  for (int i = threadIdx.x; i < np; i += blockDim.x)
    acc = OPMIN ? fmin(acc, partials[i]) : acc + partials[i];
  sm[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      sm[threadIdx.x] = OPMIN ? fmin(sm[threadIdx.x], sm[threadIdx.x + w])
                              : sm[threadIdx.x] + sm[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sm[0];
}
cudaError_t launch_reduce(const double *x, int64_t n, int op_min, double *partials,
                          double *out, cudaStream_t s) {
  const int nb = kReducePartials;
  if (op_min) {
    k_reduce_partial<1><<<nb, 256, 0, s>>>(x, n, partials);
    k_reduce_final<1><<<1, 1024, 0, s>>>(partials, nb, out);
  } else {
    k_reduce_partial<0><<<nb, 256, 0, s>>>(x, n, partials);
    k_reduce_final<0><<<1, 1024, 0, s>>>(partials, nb, out);
  }
  return cudaGetLastError();
}

// ---- halo of a partitioned mesh: the predicted displacement of listed nodes --
__global__ void k_halo(int64_t n, int d, bool unpack, const int32_t *__restrict__ idx,
                       double *__restrict__ u, double *__restrict__ buf) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n * d) return;
  const int64_t node = idx[k / d], c = k % d;
  if (unpack)
    u[node * d + c] = buf[k];
  else
    buf[k] = u[node * d + c];
}

cudaError_t launch_halo(bool unpack, int d, int64_t n, const int32_t *idx, double *u, double *buf,
                        cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_halo<<<(unsigned)((n * d + 255) / 256), 256, 0, s>>>(n, d, unpack, idx, u, buf);
  return cudaGetLastError();
}

// ---- previous displacement and increment of a step ---------------------------
// u_n is the displacement the step starts from, u_np1 its prediction, which
// the corrector does not change (its displacement coefficient is zero)
__global__ void k_history(int64_t n, const double *__restrict__ u_n,
                          const double *__restrict__ u_np1, double *__restrict__ prev,
                          double *__restrict__ incr) {
  pdl_begin();
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double a = u_n[k];
  prev[k] = a;
  incr[k] = u_np1[k] - a;
}

cudaError_t launch_history(const DevGeom &g, const double *u_n, const double *u_np1,
                           double *prev, double *incr, cudaStream_t s) {
  const int64_t n = g.N * g.D;
  if (n == 0) return cudaSuccess;
  return launch_step(g.pdl, k_history, (unsigned)((n + 255) / 256), 256, s, n, u_n, u_np1, prev,
                     incr);
}

}  // namespace akb

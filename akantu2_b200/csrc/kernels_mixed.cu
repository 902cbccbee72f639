// Mixed-precision kernels: FP32 element kinematics, stress and B^T sigma,
// FP64 nodal state with a compensated (Kahan) FP64 gather of the FP32
// elemental forces.  Contraction (FMA) is allowed in this translation unit.
#include "dispatch.cuh"

namespace akb {

namespace {

template <int LAW, int BLOCK, int QU, int MINB = 1, bool AFF = false, bool GEO = false>
void launch_hex8sf(const DevGeom &g, int64_t e0, int64_t ne, const double *u,
                   const MatParams &mp, const GroupArgs &ps, float *re, cudaStream_t s) {
  const unsigned grid = (unsigned)((ne + BLOCK - 1) / BLOCK);
  launch_step(g.pdl, k_element_forces_hex8sf<LAW, BLOCK, QU, MINB, AFF, GEO>, grid, BLOCK, s, e0,
              ne, g.E, g.conn, g.pos, g.X, g.geo, u, mp, ps, re);
}

// the shapes of the sum-factorised kernel: 64, 128 or 256 threads with 8 or
// 2 points per iteration, 128 threads with 1
template <int LAW, int QU, bool AFF, bool GEO>
void dispatch_hex8sf_block(int block, const DevGeom &g, int64_t e0, int64_t ne,
                           const double *u, const MatParams &mp, const GroupArgs &ps, float *re,
                           cudaStream_t s) {
  if (block == 64)
    launch_hex8sf<LAW, 64, QU, 1, AFF, GEO>(g, e0, ne, u, mp, ps, re, s);
  else if (block == 256)
    launch_hex8sf<LAW, 256, QU, 1, AFF, GEO>(g, e0, ne, u, mp, ps, re, s);
  else
    launch_hex8sf<LAW, 128, QU, 1, AFF, GEO>(g, e0, ne, u, mp, ps, re, s);
}
template <int LAW, bool AFF, bool GEO>
void dispatch_hex8sf(const ElemTuning &tn, const DevGeom &g, int64_t e0, int64_t ne,
                     const double *u, const MatParams &mp, const GroupArgs &ps, float *re,
                     cudaStream_t s) {
  // 128 threads with the registers capped for 6 or 5 resident blocks (24 or
  // 20 warps)
  if (tn.minb == 6 && tn.qu == 1)
    launch_hex8sf<LAW, 128, 1, 6, AFF, GEO>(g, e0, ne, u, mp, ps, re, s);
  else if (tn.minb == 6 && tn.qu == 2)
    launch_hex8sf<LAW, 128, 2, 6, AFF, GEO>(g, e0, ne, u, mp, ps, re, s);
  else if (tn.minb == 5 && tn.qu == 1)
    launch_hex8sf<LAW, 128, 1, 5, AFF, GEO>(g, e0, ne, u, mp, ps, re, s);
  else if (tn.minb == 5 && tn.qu == 2)
    launch_hex8sf<LAW, 128, 2, 5, AFF, GEO>(g, e0, ne, u, mp, ps, re, s);
  else if (tn.minb == 5)
    launch_hex8sf<LAW, 128, 8, 5, AFF, GEO>(g, e0, ne, u, mp, ps, re, s);
  // 128 threads capped at 128 registers for 4 resident blocks (16 warps)
  else if (tn.minb == 4 && tn.qu == 2)
    launch_hex8sf<LAW, 128, 2, 4, AFF, GEO>(g, e0, ne, u, mp, ps, re, s);
  else if (tn.qu == 1)
    launch_hex8sf<LAW, 128, 1, 1, AFF, GEO>(g, e0, ne, u, mp, ps, re, s);
  else if (tn.qu == 2)
    dispatch_hex8sf_block<LAW, 2, AFF, GEO>(tn.block, g, e0, ne, u, mp, ps, re, s);
  else
    dispatch_hex8sf_block<LAW, 8, AFF, GEO>(tn.block, g, e0, ne, u, mp, ps, re, s);
}
template <int LAW>
void dispatch_hex8sf_mesh(const ElemTuning &tn, const DevGeom &g, int64_t e0, int64_t ne,
                          const double *u, const MatParams &mp, const GroupArgs &ps, float *re,
                          cudaStream_t s) {
  if (g.affine && g.geo)
    dispatch_hex8sf<LAW, true, true>(tn, g, e0, ne, u, mp, ps, re, s);
  else if (g.affine)
    dispatch_hex8sf<LAW, true, false>(tn, g, e0, ne, u, mp, ps, re, s);
  else
    dispatch_hex8sf<LAW, false, false>(tn, g, e0, ne, u, mp, ps, re, s);
}

// a hexahedron is a parallelepiped when its bilinear and trilinear geometry
// modes are zero (the test of the element kernel, on the same FP32 values)
template <class T>
__global__ void k_hex8_affine(int64_t E, const int32_t *__restrict__ conn,
                              const double *__restrict__ X, unsigned int *__restrict__ flag) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  T wx[8][3];
  hex8_geometry_modes(e, E, conn, X, wx);
  constexpr T g1 = std::is_same<T, float>::value ? T(0.577350269189625764509f)
                                                 : T(0.577350269189625764509);
  constexpr T g2 = T(1) / T(3);
  bool affine = true;
#pragma unroll
  for (int c = 0; c < 3; ++c)
    affine = affine && wx[3][c] * g1 == T(0) && wx[5][c] * g1 == T(0) &&
             wx[6][c] * g1 == T(0) && wx[7][c] * g2 == T(0);
  if (!affine) atomicOr(flag, 1u);
}

// the adjugate and 1/det of every element of a mesh of parallelepipeds, into
// geo [10][E]: the values the element kernel forms from the same modes
template <class T>
__global__ void k_hex8_affine_geometry(int64_t E, const int32_t *__restrict__ conn,
                                       const double *__restrict__ X, T *__restrict__ geo) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  T wx[8][3], Ja[9];
  hex8_geometry_modes(e, E, conn, X, wx);
  const T rdet = hex8_affine_adjugate(wx, Ja);
#pragma unroll
  for (int k = 0; k < 9; ++k) geo[(int64_t)k * E + e] = Ja[k];
  geo[(int64_t)9 * E + e] = rdet;
}

}  // namespace

cudaError_t launch_element_forces_mixed(const DevGeom &g, int law, int64_t e0, int64_t ne,
                                        const QuadTable &tab, const float *fB,
                                        const float *fwJ, const double *u,
                                        const MatParams &mp, const GroupArgs &ps,
                                        float *re, const ElemTuning &tn, cudaStream_t s) {
  if (ne == 0) return cudaSuccess;
  // 2D elements and tetrahedra stream the FP32 copies of dN/dx (tetrahedra:
  // unless the recomputed form is selected, points_per_iteration 0)
  if (g.D == 2 || (g.et == ET_TET4 && fB && tn.qu != 0))
    return element_forces_impl<float, float>(g, law, e0, ne, fB, fwJ, u, mp, ps, re, tn, &tab,
                                              s);
  if (g.et == ET_HEX8 && (tn.qu & kPackedPoints))
    return launch_element_forces_hex8_x2(g, law, e0, ne, u, mp, ps, re, tn.qu & 0xff, tn.minb,
                                         tn.pf, s);
  if (g.et == ET_HEX8 && tn.qu > 0) {
    if (law == LAW_ELASTIC)
      dispatch_hex8sf_mesh<LAW_ELASTIC>(tn, g, e0, ne, u, mp, ps, re, s);
    else if (law == LAW_NEOHOOKEAN)
      dispatch_hex8sf_mesh<LAW_NEOHOOKEAN>(tn, g, e0, ne, u, mp, ps, re, s);
    else
      dispatch_hex8sf_mesh<LAW_PLASTIC>(tn, g, e0, ne, u, mp, ps, re, s);
    return cudaGetLastError();
  }
  AKB_DISPATCH_ELEM(g, {
    (void)ET;
    AKB_DISPATCH_BLOCK(tn.block, {
      const unsigned grid = (unsigned)((ne + BLOCK - 1) / BLOCK);
      auto kern = law == LAW_ELASTIC      ? k_element_forces_geo<D, NN, NQ, LAW_ELASTIC, BLOCK>
                  : law == LAW_NEOHOOKEAN ? k_element_forces_geo<D, NN, NQ, LAW_NEOHOOKEAN, BLOCK>
                                          : k_element_forces_geo<D, NN, NQ, LAW_PLASTIC, BLOCK>;
      return launch_step(g.pdl, kern, grid, BLOCK, s, e0, ne, g.E, g.conn, g.pos, g.X, tab, u,
                         mp, ps, re);
    });
  });
  return cudaGetLastError();
}

namespace {
template <int LAW>
cudaError_t persistent_mixed_law(const DevGeom &g, int qu, const StepArgs &sa,
                                 const QuadTable &tab, cudaStream_t s) {
  const int64_t work = std::max(g.E, g.N);
  if (g.et == ET_TET4 && qu == 0)
    return launch_cooperative(k_persistent_steps<3, 4, 1, LAW, 1, float, float, true, 1>, work,
                              sa, tab, s);
  if (g.et == ET_TET4)
    return launch_cooperative(k_persistent_steps<3, 4, 1, LAW, 0, float, float, true, 1>, work,
                              sa, tab, s);
  if (g.et == ET_HEX8 && qu == 1)
    return launch_cooperative(k_persistent_steps<3, 8, 8, LAW, 2, float, float, true, 1>, work,
                              sa, tab, s);
  if (g.et == ET_HEX8)
    return launch_cooperative(k_persistent_steps<3, 8, 8, LAW, 2, float, float, true, 2>, work,
                              sa, tab, s);
  if (g.NQ == 3)
    return launch_cooperative(k_persistent_steps<2, 6, 3, LAW, 0, float, float, true, 1>, work,
                              sa, tab, s);
  return launch_cooperative(k_persistent_steps<2, 6, 6, LAW, 0, float, float, true, 1>, work, sa,
                            tab, s);
}
}  // namespace

cudaError_t launch_persistent_mixed(const DevGeom &g, int law, int qu, const StepArgs &sa,
                                    const QuadTable &tab, cudaStream_t s) {
  if (law == LAW_ELASTIC) return persistent_mixed_law<LAW_ELASTIC>(g, qu, sa, tab, s);
  if (law == LAW_NEOHOOKEAN) return persistent_mixed_law<LAW_NEOHOOKEAN>(g, qu, sa, tab, s);
  return persistent_mixed_law<LAW_PLASTIC>(g, qu, sa, tab, s);
}

cudaError_t launch_node_update_mixed(const DevGeom &g, const float *re, const double *fext,
                                     const double *mass, const uint8_t *blocked,
                                     double *fint, double *a, double *v, const double *u,
                                     double *u_next, double dt, int flags,
                                     unsigned int *status, int node_block, int form,
                                     cudaStream_t s) {
  if (g.N > 0 && g.inst_end) {
    auto kern = g.D == 3 ? k_node_update_retire<3, float, true> : k_node_update_retire<2, float, true>;
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
      auto kern = g.D == 3 ? k_node_update_staged<3, float, true, NB>
                           : k_node_update_staged<2, float, true, NB>;
      return launch_step(g.pdl, kern, grid_for(g.N, NB), NB, s, g.N, g.ptr, re, fext, mass,
                         blocked, fint, a, v, u, u_next, dt, g.node_inst, g.inst_dt, flags,
                         status);
    });
  }
  // slots read 32 bytes at a time when the array's alignment allows it
  const bool wide = ((uintptr_t)re & 31) == 0;
  auto kern = g.D == 3 ? (wide ? k_node_update<3, float, true, true> : k_node_update<3, float, true>)
                       : (wide ? k_node_update<2, float, true, true> : k_node_update<2, float, true>);
  if (form == 2)
    kern = g.D == 3 ? (wide ? k_node_update_early<3, float, true, true>
                            : k_node_update_early<3, float, true>)
                    : (wide ? k_node_update_early<2, float, true, true>
                            : k_node_update_early<2, float, true>);
  return launch_step(g.pdl, kern, grid_for(g.N, node_block), node_block, s, g.N, g.ptr, re,
                     fext, mass, blocked, fint, a, v, u, u_next, dt, g.node_inst, g.inst_dt,
                     flags, status);
}

cudaError_t launch_hex8_affine_geometry(const DevGeom &g, float *geo, cudaStream_t s) {
  if (g.E == 0) return cudaSuccess;
  k_hex8_affine_geometry<float><<<(unsigned)((g.E + 255) / 256), 256, 0, s>>>(g.E, g.conn, g.X,
                                                                             geo);
  return cudaGetLastError();
}

cudaError_t launch_hex8_affine_geometry_fp64(const DevGeom &g, double *geo, cudaStream_t s) {
  if (g.E == 0) return cudaSuccess;
  k_hex8_affine_geometry<double><<<(unsigned)((g.E + 255) / 256), 256, 0, s>>>(g.E, g.conn, g.X,
                                                                              geo);
  return cudaGetLastError();
}

// FP64 hexahedra by the sum-factorised kernel with contraction allowed (the
// fast FP64 path): 128 threads, QU points per unrolled iteration, registers
// capped for MINB blocks; meshes of parallelepipeds read their FP64 adjugate
// table, the others form their geometry per point
template <int LAW, int QU, int MINB>
cudaError_t launch_sf64(const DevGeom &g, int64_t e0, int64_t ne, const double *u,
                        const MatParams &mp, const GroupArgs &ps, double *re, const double *geo,
                        cudaStream_t s) {
  const unsigned grid = (unsigned)((ne + 127) / 128);
  if (geo)
    return launch_step(g.pdl, k_element_forces_hex8sf<LAW, 128, QU, MINB, true, true, double>,
                       grid, 128, s, e0, ne, g.E, g.conn, g.pos, g.X, geo, u, mp, ps, re);
  return launch_step(g.pdl, k_element_forces_hex8sf<LAW, 128, QU, MINB, false, false, double>,
                     grid, 128, s, e0, ne, g.E, g.conn, g.pos, g.X, geo, u, mp, ps, re);
}

template <int LAW>
cudaError_t dispatch_sf64(const ElemTuning &tn, const DevGeom &g, int64_t e0, int64_t ne,
                          const double *u, const MatParams &mp, const GroupArgs &ps, double *re,
                          const double *geo, cudaStream_t s) {
  if (tn.qu == 1) return launch_sf64<LAW, 1, 1>(g, e0, ne, u, mp, ps, re, geo, s);
  if (tn.qu == 8) return launch_sf64<LAW, 8, 1>(g, e0, ne, u, mp, ps, re, geo, s);
  if (tn.minb == 2) return launch_sf64<LAW, 2, 2>(g, e0, ne, u, mp, ps, re, geo, s);
  if (tn.minb == 3) return launch_sf64<LAW, 2, 3>(g, e0, ne, u, mp, ps, re, geo, s);
  return launch_sf64<LAW, 2, 1>(g, e0, ne, u, mp, ps, re, geo, s);
}

cudaError_t launch_element_forces_fp64_sf(const DevGeom &g, int law, int64_t e0, int64_t ne,
                                          const double *u, const MatParams &mp,
                                          const GroupArgs &ps, double *re, const double *geo,
                                          const ElemTuning &tn, cudaStream_t s) {
  if (ne == 0) return cudaSuccess;
  if (g.et != ET_HEX8) return cudaErrorInvalidValue;
  if (law == LAW_ELASTIC) return dispatch_sf64<LAW_ELASTIC>(tn, g, e0, ne, u, mp, ps, re, geo, s);
  if (law == LAW_NEOHOOKEAN)
    return dispatch_sf64<LAW_NEOHOOKEAN>(tn, g, e0, ne, u, mp, ps, re, geo, s);
  return dispatch_sf64<LAW_PLASTIC>(tn, g, e0, ne, u, mp, ps, re, geo, s);
}

cudaError_t launch_hex8_affine_check(const DevGeom &g, unsigned int *flag, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(flag, 0, sizeof(unsigned int), s);
  if (e != cudaSuccess || g.E == 0) return e;
  k_hex8_affine<float><<<(unsigned)((g.E + 255) / 256), 256, 0, s>>>(g.E, g.conn, g.X, flag);
  return cudaGetLastError();
}

cudaError_t launch_hex8_affine_check_fp64(const DevGeom &g, unsigned int *flag, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(flag, 0, sizeof(unsigned int), s);
  if (e != cudaSuccess || g.E == 0) return e;
  k_hex8_affine<double><<<(unsigned)((g.E + 255) / 256), 256, 0, s>>>(g.E, g.conn, g.X, flag);
  return cudaGetLastError();
}

}  // namespace akb

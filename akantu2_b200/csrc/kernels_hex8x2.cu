// Mixed-precision hexahedra on packed FP32 pairs (sm_100 add / mul / fma
// .f32x2): the sum-factorised element kernel with the two Gauss points of
// equal eta and zeta evaluated as the two lanes of each packed operation.
// Meshes of parallelepipeds, elastic and neohookean laws.  A translation
// unit of its own so that it compiles in parallel with the others.
#include "dispatch.cuh"

namespace akb {

namespace {

template <int LAW, int BLOCK, int PU, int MINB, bool GEO>
cudaError_t launch_x2(const DevGeom &g, int64_t e0, int64_t ne, const double *u,
                      const MatParams &mp, const GroupArgs &ps, float *re, int pf_waves,
                      cudaStream_t s) {
  const unsigned grid = (unsigned)((ne + BLOCK - 1) / BLOCK);
  constexpr auto k0 = k_element_forces_hex8sf_x2<LAW, BLOCK, PU, MINB, GEO, false>;
  constexpr auto k1 = k_element_forces_hex8sf_x2<LAW, BLOCK, PU, MINB, GEO, true>;
  const int64_t pf = prefetch_distance<k1>(pf_waves, BLOCK);
  return launch_step(g.pdl, pf > 0 ? k1 : k0, grid, BLOCK, s, e0, ne, g.E, g.conn, g.pos, g.X,
                     g.geo, u, mp, ps, re, pf);
}

// 128 threads, registers capped for minb resident blocks per SM (1: the
// compiler's choice); pu pairs per unrolled iteration
template <int LAW, bool GEO>
cudaError_t dispatch_x2(int pu, int minb, const DevGeom &g, int64_t e0, int64_t ne,
                        const double *u, const MatParams &mp, const GroupArgs &ps, float *re,
                        int pf, cudaStream_t s) {
#define AKB_X2(PU, MINB)                                                      \
  if (pu == PU && minb == MINB) return launch_x2<LAW, 128, PU, MINB, GEO>(g, e0, ne, u, mp, ps, re, pf, s);
  AKB_X2(1, 1) AKB_X2(2, 1) AKB_X2(4, 1)
  AKB_X2(1, 4) AKB_X2(2, 4) AKB_X2(4, 4)
  AKB_X2(1, 5) AKB_X2(2, 5) AKB_X2(4, 5)
#undef AKB_X2
  return cudaErrorInvalidValue;
}

}  // namespace

cudaError_t launch_element_forces_hex8_x2(const DevGeom &g, int law, int64_t e0, int64_t ne,
                                          const double *u, const MatParams &mp,
                                          const GroupArgs &ps, float *re, int points,
                                          int minb, int pf_waves, cudaStream_t s) {
  if (ne == 0) return cudaSuccess;
  if (!g.affine || law == LAW_PLASTIC) return cudaErrorInvalidValue;
  const int pu = points / 2;
  const bool geo = g.geo != nullptr;
  if (law == LAW_ELASTIC)
    return geo ? dispatch_x2<LAW_ELASTIC, true>(pu, minb, g, e0, ne, u, mp, ps, re, pf_waves, s)
               : dispatch_x2<LAW_ELASTIC, false>(pu, minb, g, e0, ne, u, mp, ps, re, pf_waves, s);
  return geo ? dispatch_x2<LAW_NEOHOOKEAN, true>(pu, minb, g, e0, ne, u, mp, ps, re, pf_waves, s)
             : dispatch_x2<LAW_NEOHOOKEAN, false>(pu, minb, g, e0, ne, u, mp, ps, re, pf_waves, s);
}

}  // namespace akb

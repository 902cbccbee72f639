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
                      const MatParams &mp, const GroupArgs &ps, float *re, cudaStream_t s) {
  const unsigned grid = (unsigned)((ne + BLOCK - 1) / BLOCK);
  return launch_step(g.pdl, k_element_forces_hex8sf_x2<LAW, BLOCK, PU, MINB, GEO>, grid, BLOCK,
                     s, e0, ne, g.E, g.conn, g.pos, g.X, g.geo, u, mp, ps, re);
}

// 128 threads, registers capped for minb resident blocks per SM (1: the
// compiler's choice); pu pairs per unrolled iteration
template <int LAW, bool GEO>
cudaError_t dispatch_x2(int pu, int minb, const DevGeom &g, int64_t e0, int64_t ne,
                        const double *u, const MatParams &mp, const GroupArgs &ps, float *re,
                        cudaStream_t s) {
#define AKB_X2(PU, MINB)                                                      \
  if (pu == PU && minb == MINB) return launch_x2<LAW, 128, PU, MINB, GEO>(g, e0, ne, u, mp, ps, re, s);
  AKB_X2(1, 1) AKB_X2(2, 1) AKB_X2(4, 1)
  AKB_X2(1, 4) AKB_X2(2, 4) AKB_X2(4, 4)
  AKB_X2(1, 5) AKB_X2(2, 5) AKB_X2(4, 5)
#undef AKB_X2
  return cudaErrorInvalidValue;
}

// the pipelined form: a grid of resident blocks (minb per SM)
template <int LAW, int PU, int MINB>
cudaError_t launch_x2p(const DevGeom &g, int64_t e0, int64_t ne, const double *u,
                       const MatParams &mp, const GroupArgs &ps, float *re, cudaStream_t s) {
  static int sms = 0;
  if (sms == 0) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    // the shared-memory share of the unified L1 that lets MINB blocks of
    // 48 KB reside
    cudaFuncSetAttribute(k_element_forces_hex8sf_x2p<LAW, PU, MINB>,
                         cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  }
  const int64_t want = (ne + kPipeThreads - 1) / kPipeThreads;
  const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)sms * MINB));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kPipeThreads);
  cfg.dynamicSmemBytes = kPipeSmem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = g.pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, k_element_forces_hex8sf_x2p<LAW, PU, MINB>, e0, ne, g.E,
                            g.conn, g.pos, g.geo, u, mp, ps, re);
}

template <int LAW>
cudaError_t dispatch_x2p(int pu, int minb, const DevGeom &g, int64_t e0, int64_t ne,
                         const double *u, const MatParams &mp, const GroupArgs &ps, float *re,
                         cudaStream_t s) {
#define AKB_X2P(PU, MINB) \
  if (pu == PU && minb == MINB) return launch_x2p<LAW, PU, MINB>(g, e0, ne, u, mp, ps, re, s);
  AKB_X2P(1, 4) AKB_X2P(2, 4) AKB_X2P(4, 4)
  AKB_X2P(1, 3) AKB_X2P(2, 3) AKB_X2P(4, 3)
#undef AKB_X2P
  return cudaErrorInvalidValue;
}

}  // namespace

cudaError_t launch_element_forces_hex8_x2(const DevGeom &g, int law, int64_t e0, int64_t ne,
                                          const double *u, const MatParams &mp,
                                          const GroupArgs &ps, float *re, int points,
                                          int minb, cudaStream_t s) {
  if (ne == 0) return cudaSuccess;
  if (!g.affine || law == LAW_PLASTIC) return cudaErrorInvalidValue;
  const bool pipelined = (points & kPipelinedPoints) != 0;
  points &= ~kPipelinedPoints;
  const int pu = points / 2;
  const bool geo = g.geo != nullptr;
#ifdef AKB_BOUNDS_CHECK
  const bool pipe_ok = false;  // the checked build gathers through checked indices only
#else
  const bool pipe_ok = geo;
#endif
  if (pipelined && pipe_ok)
    return law == LAW_ELASTIC ? dispatch_x2p<LAW_ELASTIC>(pu, minb, g, e0, ne, u, mp, ps, re, s)
                              : dispatch_x2p<LAW_NEOHOOKEAN>(pu, minb, g, e0, ne, u, mp, ps, re, s);
  if (law == LAW_ELASTIC)
    return geo ? dispatch_x2<LAW_ELASTIC, true>(pu, minb, g, e0, ne, u, mp, ps, re, s)
               : dispatch_x2<LAW_ELASTIC, false>(pu, minb, g, e0, ne, u, mp, ps, re, s);
  return geo ? dispatch_x2<LAW_NEOHOOKEAN, true>(pu, minb, g, e0, ne, u, mp, ps, re, s)
             : dispatch_x2<LAW_NEOHOOKEAN, false>(pu, minb, g, e0, ne, u, mp, ps, re, s);
}

}  // namespace akb

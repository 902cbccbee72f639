// Dispatch from runtime (element type, quadrature rule, law) to the kernel
// template instances; shared by the FP64 and the mixed translation units.
#pragma once

#include <algorithm>
#include <atomic>
#include <type_traits>

#include "fe_kernels.cuh"
#include "launch.h"

namespace akb {

namespace {
constexpr int kThreads = 256;
inline unsigned grid_for(int64_t n, int threads = kThreads) {
  return (unsigned)((n + threads - 1) / threads);
}
}  // namespace

// a step kernel launch, with the programmatic-serialization attribute when pdl
// is set (the kernel then overlaps the end of the previous kernel on the
// stream; it waits for it in pdl_begin)
// (smem: bytes of dynamic shared memory)
template <class... KArgs, class... Args>
inline cudaError_t launch_step_smem(bool pdl, void (*kernel)(KArgs...), unsigned grid,
                                    unsigned block, size_t smem, cudaStream_t s,
                                    Args... args) {
  if (!pdl) {
    kernel<<<grid, block, smem, s>>>(args...);
    return cudaGetLastError();
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

template <class... KArgs, class... Args>
inline cudaError_t launch_step(bool pdl, void (*kernel)(KArgs...), unsigned grid,
                               unsigned block, cudaStream_t s, Args... args) {
  return launch_step_smem(pdl, kernel, grid, block, 0, s, args...);
}

// ---- dispatch helpers ------------------------------------------------------
#define AKB_DISPATCH_ELEM(g, ...)                                        \
  do {                                                                    \
    if ((g).et == ET_TET4) {                                              \
      constexpr int ET = ET_TET4, D = 3, NN = 4, NQ = 1;                  \
      __VA_ARGS__;                                                        \
    } else if ((g).et == ET_HEX8) {                                       \
      constexpr int ET = ET_HEX8, D = 3, NN = 8, NQ = 8;                  \
      __VA_ARGS__;                                                        \
    } else if ((g).et == ET_TRI6 && (g).NQ == 3) {                        \
      constexpr int ET = ET_TRI6, D = 2, NN = 6, NQ = 3;                  \
      __VA_ARGS__;                                                        \
    } else if ((g).et == ET_TRI6 && (g).NQ == 6) {                        \
      constexpr int ET = ET_TRI6, D = 2, NN = 6, NQ = 6;                  \
      __VA_ARGS__;                                                        \
    } else {                                                              \
      return cudaErrorInvalidValue;                                       \
    }                                                                     \
  } while (0)

// threads per block of the per-element kernels: 64, 128 or 256
#define AKB_DISPATCH_BLOCK(b, ...)                                       \
  do {                                                                    \
    if ((b) == 64) {                                                      \
      constexpr int BLOCK = 64;                                           \
      __VA_ARGS__;                                                        \
    } else if ((b) == 256) {                                              \
      constexpr int BLOCK = 256;                                          \
      __VA_ARGS__;                                                        \
    } else {                                                              \
      constexpr int BLOCK = 128;                                          \
      __VA_ARGS__;                                                        \
    }                                                                     \
  } while (0)

// threads per block of the staged node update: 128, 256 or 512
#define AKB_DISPATCH_NODE_BLOCK(b, ...)                                  \
  do {                                                                    \
    if ((b) <= 128) {                                                     \
      constexpr int NB = 128;                                             \
      __VA_ARGS__;                                                        \
    } else if ((b) <= 256) {                                              \
      constexpr int NB = 256;                                             \
      __VA_ARGS__;                                                        \
    } else {                                                              \
      constexpr int NB = 512;                                             \
      __VA_ARGS__;                                                        \
    }                                                                     \
  } while (0)

// cooperative launch of a persistent step kernel: as many blocks as fit on
// the device at once (all resident, so the grid barrier can complete), fewer
// when the mesh needs fewer
template <class K>
inline cudaError_t launch_cooperative(K kernel, int64_t work, const StepArgs &sa,
                                      const QuadTable &tab, cudaStream_t s) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kPersistentThreads, 0);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  const int64_t want = (work + kPersistentThreads - 1) / kPersistentThreads;
  const unsigned grid = (unsigned)std::max<int64_t>(
      1, std::min<int64_t>(std::min<int64_t>(want, (int64_t)per_sm * sms), 8192));
  StepArgs a = sa;
  QuadTable t = tab;
  void *args[] = {&a, &t};
  return cudaLaunchCooperativeKernel((const void *)kernel, grid, kPersistentThreads, args, 0, s);
}

// elements one wave of resident blocks of kernel covers: its occupancy
// times the SM count (0 if the query fails)
template <class K>
int64_t wave_elements(K kernel, int block) {
  int dev = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0) != cudaSuccess)
    return 0;
  return (int64_t)sms * per_sm * block;
}

// L2 prefetch distance, in elements, of `waves` waves of resident blocks of
// the kernel K (0: none); the wave is queried once per kernel (the GPUs of a
// node are of one model)
template <auto K>
int64_t prefetch_distance(int waves, int block) {
  if (waves <= 0) return 0;
  static std::atomic<int64_t> wave{-1};
  int64_t w = wave.load(std::memory_order_relaxed);
  if (w < 0) wave.store(w = wave_elements(K, block), std::memory_order_relaxed);
  return waves * w;
}

// tab: the quadrature tables, for the kernels that recompute dN/dx and
// det J w from the coordinates (tn.rec; tetrahedra and triangles)
template <class T, class RT>
inline cudaError_t element_forces_impl(const DevGeom &g, int law, int64_t e0, int64_t ne,
                                       const T *B, const T *wJ, const double *u,
                                       const MatParams &mp, const GroupArgs &ps, RT *re,
                                       const ElemTuning &tn, const QuadTable *tab,
                                       cudaStream_t s) {
  if (ne == 0) return cudaSuccess;
  AKB_DISPATCH_ELEM(g, {
    (void)ET;
    // FP64 hexahedra: one thread per (element, point); otherwise one thread
    // per element looping over its points
    constexpr bool PQ = std::is_same<T, double>::value && NQ == 8;
    if constexpr (PQ) {
      const unsigned grid = (unsigned)((ne + 31) / 32);
      if (tn.pqs) {
        auto kern = law == LAW_ELASTIC      ? k_element_forces_pqs<D, NN, NQ, LAW_ELASTIC>
                    : law == LAW_NEOHOOKEAN ? k_element_forces_pqs<D, NN, NQ, LAW_NEOHOOKEAN>
                                            : k_element_forces_pqs<D, NN, NQ, LAW_PLASTIC>;
        constexpr size_t smem = sizeof(double) * 32 * (NN * D) * (1 + NQ);
        // above the 48 KB default: allowed once per kernel and device (a
        // host-side attribute of the current device, no stream work)
        static std::atomic<unsigned long long> opted[3] = {0ull, 0ull, 0ull};
        const int li = law == LAW_ELASTIC ? 0 : law == LAW_NEOHOOKEAN ? 1 : 2;
        int dev = 0;
        const cudaError_t ed = cudaGetDevice(&dev);
        if (ed != cudaSuccess) return ed;
        const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
        if (!(opted[li].load(std::memory_order_relaxed) & bit)) {
          const cudaError_t ea =
              cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
          if (ea != cudaSuccess) return ea;
          opted[li].fetch_or(bit, std::memory_order_relaxed);
        }
        return launch_step_smem(g.pdl, kern, grid, 32 * NQ, smem, s, e0, ne, g.E, g.conn, g.pos,
                                B, wJ, u, mp, ps, re);
      }
      auto kern = law == LAW_ELASTIC      ? k_element_forces_pq<D, NN, NQ, LAW_ELASTIC>
                  : law == LAW_NEOHOOKEAN ? k_element_forces_pq<D, NN, NQ, LAW_NEOHOOKEAN>
                                          : k_element_forces_pq<D, NN, NQ, LAW_PLASTIC>;
      return launch_step(g.pdl, kern, grid, 32 * NQ, s, e0, ne, g.E, g.conn, g.pos, B, wJ, u,
                         mp, ps, re);
    } else {
      AKB_DISPATCH_BLOCK(tn.block, {
        const unsigned grid = (unsigned)((ne + BLOCK - 1) / BLOCK);
        if constexpr (ET == ET_TRI6 && BLOCK == 128) {
          // plastic triangles, streamed law: 128 threads, registers capped
          // for 1 (none), 5, 6, 7 or 8 resident blocks; tables streamed
          if (law == LAW_PLASTIC && tn.pqs && !tn.rec) {
            auto kern = tn.minb >= 8   ? k_element_forces_pe_streamed<D, NN, NQ, T, RT, 128, 8>
                        : tn.minb == 7 ? k_element_forces_pe_streamed<D, NN, NQ, T, RT, 128, 7>
                        : tn.minb == 6 ? k_element_forces_pe_streamed<D, NN, NQ, T, RT, 128, 6>
                        : tn.minb == 5 ? k_element_forces_pe_streamed<D, NN, NQ, T, RT, 128, 5>
                                       : k_element_forces_pe_streamed<D, NN, NQ, T, RT, 128, 1>;
            return launch_step(g.pdl, kern, grid, 128, s, e0, ne, g.E, g.conn, g.pos, B, wJ, u,
                               mp, ps, re, (int64_t)0);
          }
        }
        if constexpr (ET != ET_HEX8) {
          if (tn.rec && tab) {
            if constexpr (BLOCK == 128) {
              if (law == LAW_PLASTIC && tn.minb > 1) {
                constexpr auto k6 = k_element_forces_pr<D, NN, NQ, LAW_PLASTIC, T, RT, 128, 6>;
                constexpr auto k5 = k_element_forces_pr<D, NN, NQ, LAW_PLASTIC, T, RT, 128, 5>;
                constexpr auto k6p =
                    k_element_forces_pr<D, NN, NQ, LAW_PLASTIC, T, RT, 128, 6, true>;
                constexpr auto k5p =
                    k_element_forces_pr<D, NN, NQ, LAW_PLASTIC, T, RT, 128, 5, true>;
                const int64_t pf = tn.minb >= 6 ? prefetch_distance<k6p>(tn.pf, 128)
                                                : prefetch_distance<k5p>(tn.pf, 128);
                auto kern = tn.minb >= 6 ? (pf > 0 ? k6p : k6) : (pf > 0 ? k5p : k5);
                return launch_step(g.pdl, kern, grid, 128, s, e0, ne, g.E, g.conn, g.pos, g.X,
                                   *tab, u, mp, ps, re, pf);
              }
            }
            if constexpr (ET == ET_TET4 && BLOCK == 128 && std::is_same<T, double>::value) {
              // FP64 elastic and neohookean tetrahedra: registers capped for 6
              // or 7 resident blocks (80 / 72 instead of 90 registers)
              if (law != LAW_PLASTIC && (tn.minb == 6 || tn.minb == 7)) {
                const bool el = law == LAW_ELASTIC, m7 = tn.minb == 7;
                constexpr auto e6 = k_element_forces_pr<D, NN, NQ, LAW_ELASTIC, T, RT, 128, 6>;
                constexpr auto e7 = k_element_forces_pr<D, NN, NQ, LAW_ELASTIC, T, RT, 128, 7>;
                constexpr auto n6 = k_element_forces_pr<D, NN, NQ, LAW_NEOHOOKEAN, T, RT, 128, 6>;
                constexpr auto n7 = k_element_forces_pr<D, NN, NQ, LAW_NEOHOOKEAN, T, RT, 128, 7>;
                constexpr auto e6p =
                    k_element_forces_pr<D, NN, NQ, LAW_ELASTIC, T, RT, 128, 6, true>;
                constexpr auto e7p =
                    k_element_forces_pr<D, NN, NQ, LAW_ELASTIC, T, RT, 128, 7, true>;
                constexpr auto n6p =
                    k_element_forces_pr<D, NN, NQ, LAW_NEOHOOKEAN, T, RT, 128, 6, true>;
                constexpr auto n7p =
                    k_element_forces_pr<D, NN, NQ, LAW_NEOHOOKEAN, T, RT, 128, 7, true>;
                const int64_t pf = el ? (m7 ? prefetch_distance<e7p>(tn.pf, 128)
                                            : prefetch_distance<e6p>(tn.pf, 128))
                                      : (m7 ? prefetch_distance<n7p>(tn.pf, 128)
                                            : prefetch_distance<n6p>(tn.pf, 128));
                auto kern = el ? (m7 ? (pf > 0 ? e7p : e7) : (pf > 0 ? e6p : e6))
                               : (m7 ? (pf > 0 ? n7p : n7) : (pf > 0 ? n6p : n6));
                return launch_step(g.pdl, kern, grid, 128, s, e0, ne, g.E, g.conn, g.pos, g.X,
                                   *tab, u, mp, ps, re, pf);
              }
            }
            constexpr auto ke = k_element_forces_pr<D, NN, NQ, LAW_ELASTIC, T, RT, BLOCK>;
            constexpr auto kn = k_element_forces_pr<D, NN, NQ, LAW_NEOHOOKEAN, T, RT, BLOCK>;
            constexpr auto kp = k_element_forces_pr<D, NN, NQ, LAW_PLASTIC, T, RT, BLOCK>;
            constexpr auto kep = k_element_forces_pr<D, NN, NQ, LAW_ELASTIC, T, RT, BLOCK, 1, true>;
            constexpr auto knp =
                k_element_forces_pr<D, NN, NQ, LAW_NEOHOOKEAN, T, RT, BLOCK, 1, true>;
            constexpr auto kpp = k_element_forces_pr<D, NN, NQ, LAW_PLASTIC, T, RT, BLOCK, 1, true>;
            const int64_t pf = law == LAW_ELASTIC      ? prefetch_distance<kep>(tn.pf, BLOCK)
                               : law == LAW_NEOHOOKEAN ? prefetch_distance<knp>(tn.pf, BLOCK)
                                                       : prefetch_distance<kpp>(tn.pf, BLOCK);
            auto kern = law == LAW_ELASTIC      ? (pf > 0 ? kep : ke)
                        : law == LAW_NEOHOOKEAN ? (pf > 0 ? knp : kn)
                                                : (pf > 0 ? kpp : kp);
            return launch_step(g.pdl, kern, grid, BLOCK, s, e0, ne, g.E, g.conn, g.pos, g.X,
                               *tab, u, mp, ps, re, pf);
          }
        }
        if constexpr (BLOCK == 128) {
          // plastic groups: 128 threads with registers capped for 5 to 8 blocks per
          // SM (7 and 8 without the prefetch)
          if (law == LAW_PLASTIC && tn.minb >= 7 && tn.pf == 0) {
            auto kern = tn.minb >= 8 ? k_element_forces_pe<D, NN, NQ, LAW_PLASTIC, T, RT, 128, 8>
                                     : k_element_forces_pe<D, NN, NQ, LAW_PLASTIC, T, RT, 128, 7>;
            return launch_step(g.pdl, kern, grid, 128, s, e0, ne, g.E, g.conn, g.pos, B, wJ, u,
                               mp, ps, re, (int64_t)0);
          }
          if (law == LAW_PLASTIC && tn.minb > 1) {
            constexpr auto k6 = k_element_forces_pe<D, NN, NQ, LAW_PLASTIC, T, RT, 128, 6>;
            constexpr auto k5 = k_element_forces_pe<D, NN, NQ, LAW_PLASTIC, T, RT, 128, 5>;
            constexpr auto k6p = k_element_forces_pe<D, NN, NQ, LAW_PLASTIC, T, RT, 128, 6, true>;
            constexpr auto k5p = k_element_forces_pe<D, NN, NQ, LAW_PLASTIC, T, RT, 128, 5, true>;
            const int64_t pf = tn.minb >= 6 ? prefetch_distance<k6p>(tn.pf, 128)
                                            : prefetch_distance<k5p>(tn.pf, 128);
            auto kern = tn.minb >= 6 ? (pf > 0 ? k6p : k6) : (pf > 0 ? k5p : k5);
            return launch_step(g.pdl, kern, grid, 128, s, e0, ne, g.E, g.conn, g.pos, B, wJ, u,
                               mp, ps, re, pf);
          }
        }
        constexpr auto ke = k_element_forces_pe<D, NN, NQ, LAW_ELASTIC, T, RT, BLOCK>;
        constexpr auto kn = k_element_forces_pe<D, NN, NQ, LAW_NEOHOOKEAN, T, RT, BLOCK>;
        constexpr auto kp = k_element_forces_pe<D, NN, NQ, LAW_PLASTIC, T, RT, BLOCK>;
        constexpr auto kep = k_element_forces_pe<D, NN, NQ, LAW_ELASTIC, T, RT, BLOCK, 1, true>;
        constexpr auto knp = k_element_forces_pe<D, NN, NQ, LAW_NEOHOOKEAN, T, RT, BLOCK, 1, true>;
        constexpr auto kpp = k_element_forces_pe<D, NN, NQ, LAW_PLASTIC, T, RT, BLOCK, 1, true>;
        const int64_t pf = law == LAW_ELASTIC      ? prefetch_distance<kep>(tn.pf, BLOCK)
                           : law == LAW_NEOHOOKEAN ? prefetch_distance<knp>(tn.pf, BLOCK)
                                                   : prefetch_distance<kpp>(tn.pf, BLOCK);
        auto kern = law == LAW_ELASTIC      ? (pf > 0 ? kep : ke)
                    : law == LAW_NEOHOOKEAN ? (pf > 0 ? knp : kn)
                                            : (pf > 0 ? kpp : kp);
        return launch_step(g.pdl, kern, grid, BLOCK, s, e0, ne, g.E, g.conn, g.pos, B, wJ, u,
                           mp, ps, re, pf);
      });
    }
  });
  return cudaGetLastError();
}


}  // namespace akb

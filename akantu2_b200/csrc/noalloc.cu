// Stable time step without any device allocation by the library.
//
// The model entry point akb_model_get_stable_time_step keeps its per-element
// values and its reduction partials in buffers the model allocated with
// cudaMalloc.  This variant keeps that scratch in a file-scope __device__
// array instead, for callers that must not allocate: applications whose
// device memory is owned by their own pool or arena (no cudaMalloc behind
// their back), and code that computes the time step inside a loop where a
// runtime allocation is not allowed.  The caller passes the inputs and the
// output; the library allocates nothing.
#include <mutex>

#include "akb_capi.h"
#include "fe_kernels.cuh"
#include "host_common.h"
#include "launch.h"

namespace akb {
namespace {

constexpr int64_t kMaxElements = AKB_NOALLOC_MAX_ELEMENTS;

// per-element h/c values, then the reduction partials; every device that
// loads the library holds it until the process exits
__device__ __align__(256) double g_noalloc_scratch[kMaxElements + kReducePartials];

constexpr int kMaxDevices = 64;
double *g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mutex;

// device address of g_noalloc_scratch on the current device (the host-side
// name is only a stand-in; a kernel must get this address)
int scratch_address(double **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(AKB_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(AKB_EINVAL, "device index out of range");
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      return fail(AKB_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_scratch_addr[dev] = static_cast<double *>(p);
  }
  *out = g_scratch_addr[dev];
  return AKB_OK;
}

// h_e / c at X + u for connectivity in the reference layout [E][n]
template <int ET, int D, int NN>
__global__ void k_noalloc_element_dt(int64_t E, double celerity, const int32_t *__restrict__ conn,
                                     const double *__restrict__ X, const double *__restrict__ u,
                                     double *__restrict__ out) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  double Xe[NN * D];
#pragma unroll
  for (int a = 0; a < NN; ++a) {
    const int64_t node = conn[e * NN + a];
#pragma unroll
    for (int i = 0; i < D; ++i) Xe[a * D + i] = X[node * D + i] + u[node * D + i];
  }
  out[e] = element_inradius<ET>(Xe) / celerity;
}

}  // namespace
}  // namespace akb

using namespace akb;

extern "C" int akb_stable_time_step_noalloc(int element_type, const double *nodes,
                                            const double *displacement,
                                            const int32_t *connectivity, int64_t nb_elements,
                                            double celerity, double *dt_out, void *stream) {
  if (!dt_out) return fail(AKB_EINVAL, "null output pointer");
  if (nb_elements < 0) return fail(AKB_EINVAL, "negative element count");
  if (nb_elements > kMaxElements)
    return fail(AKB_EINVAL, "nb_elements (" + std::to_string(nb_elements) +
                                ") exceeds AKB_NOALLOC_MAX_ELEMENTS (" +
                                std::to_string(kMaxElements) + ")");
  if (nb_elements > 0 && (!nodes || !displacement || !connectivity))
    return fail(AKB_EINVAL, "null input pointer");
  if (element_type < AKB_TETRAHEDRON_4 || element_type > AKB_TRIANGLE_6)
    return fail(AKB_EINVAL, "unknown element type");
  double *scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc != AKB_OK) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double *partials = scratch + kMaxElements;
  if (nb_elements > 0) {
    const unsigned grid = (unsigned)((nb_elements + 255) / 256);
    if (element_type == AKB_TETRAHEDRON_4)
      k_noalloc_element_dt<ET_TET4, 3, 4><<<grid, 256, 0, s>>>(nb_elements, celerity,
                                                               connectivity, nodes,
                                                               displacement, scratch);
    else if (element_type == AKB_HEXAHEDRON_8)
      k_noalloc_element_dt<ET_HEX8, 3, 8><<<grid, 256, 0, s>>>(nb_elements, celerity,
                                                               connectivity, nodes,
                                                               displacement, scratch);
    else
      k_noalloc_element_dt<ET_TRI6, 2, 6><<<grid, 256, 0, s>>>(nb_elements, celerity,
                                                               connectivity, nodes,
                                                               displacement, scratch);
  }
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = launch_reduce(scratch, nb_elements, 1, partials, dt_out, s);
  if (e != cudaSuccess)
    return fail(AKB_ECUDA, std::string("stable time step: ") + cudaGetErrorString(e));
  return AKB_OK;
}

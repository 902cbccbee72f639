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
#include <climits>
#include <cmath>
#include <mutex>

#include "akb_capi.h"
#include "fe_kernels.cuh"
#include "host_common.h"
#include "launch.h"

namespace akb {
namespace {

constexpr int64_t kMaxElements = AKB_NOALLOC_MAX_ELEMENTS;

// per-element h/c values, then the reduction partials, then one status word
// (set when a connectivity index lies outside [0, nb_nodes)); every device
// that loads the library holds it until the process exits
__device__ __align__(256) double g_noalloc_scratch[kMaxElements + kReducePartials + 1];

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

// h_e / c at X + u for connectivity in the reference layout [E][n].  An
// element with a node index outside [0, N) reads no node: it sets *bad and
// contributes +inf (the largest double) to the minimum.
template <int ET, int D, int NN>
__global__ void k_noalloc_element_dt(int64_t E, int64_t N, double celerity,
                                     const int32_t *__restrict__ conn,
                                     const double *__restrict__ X, const double *__restrict__ u,
                                     double *__restrict__ out, double *__restrict__ bad) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  int32_t nodes[NN];
  bool ok = true;
#pragma unroll
  for (int a = 0; a < NN; ++a) {
    nodes[a] = conn[e * NN + a];
    ok = ok && nodes[a] >= 0 && (int64_t)nodes[a] < N;
  }
  if (!ok) {
    *bad = 1.;
    out[e] = 1.7976931348623157e308;
    return;
  }
  double Xe[NN * D];
#pragma unroll
  for (int a = 0; a < NN; ++a) {
    const int64_t node = nodes[a];
#pragma unroll
    for (int i = 0; i < D; ++i) Xe[a * D + i] = X[node * D + i] + u[node * D + i];
  }
  out[e] = element_inradius<ET>(Xe) / celerity;
}

// the result becomes NaN when an element had a node index out of range
__global__ void k_noalloc_finish(const double *__restrict__ bad, double *__restrict__ dt_out) {
  if (*bad != 0.) *dt_out = __longlong_as_double(0x7ff8000000000000LL);
}

}  // namespace
}  // namespace akb

using namespace akb;

extern "C" int akb_stable_time_step_noalloc(int element_type, const double *nodes,
                                            const double *displacement, int64_t nb_nodes,
                                            const int32_t *connectivity, int64_t nb_elements,
                                            double celerity, double *dt_out, void *stream) {
  if (!dt_out) return fail(AKB_EINVAL, "null output pointer");
  if (nb_elements < 0) return fail(AKB_EINVAL, "negative element count");
  if (nb_nodes < 0 || nb_nodes > INT32_MAX) return fail(AKB_EINVAL, "node count out of range");
  if (!(celerity > 0.) || !std::isfinite(celerity))
    return fail(AKB_EINVAL, "celerity must be finite and positive");
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
  double *bad = partials + kReducePartials;
  // the status word keeps the last call's value: clear it first
  cudaError_t e = cudaMemsetAsync(bad, 0, sizeof(double), s);
  if (e != cudaSuccess)
    return fail(AKB_ECUDA, std::string("stable time step: ") + cudaGetErrorString(e));
  if (nb_elements > 0) {
    const unsigned grid = (unsigned)((nb_elements + 255) / 256);
    if (element_type == AKB_TETRAHEDRON_4)
      k_noalloc_element_dt<ET_TET4, 3, 4><<<grid, 256, 0, s>>>(nb_elements, nb_nodes,
                                                               celerity, connectivity, nodes,
                                                               displacement, scratch, bad);
    else if (element_type == AKB_HEXAHEDRON_8)
      k_noalloc_element_dt<ET_HEX8, 3, 8><<<grid, 256, 0, s>>>(nb_elements, nb_nodes,
                                                               celerity, connectivity, nodes,
                                                               displacement, scratch, bad);
    else
      k_noalloc_element_dt<ET_TRI6, 2, 6><<<grid, 256, 0, s>>>(nb_elements, nb_nodes,
                                                               celerity, connectivity, nodes,
                                                               displacement, scratch, bad);
  }
  e = cudaGetLastError();
  if (e == cudaSuccess) e = launch_reduce(scratch, nb_elements, 1, partials, dt_out, s);
  if (e == cudaSuccess) {
    k_noalloc_finish<<<1, 1, 0, s>>>(bad, dt_out);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess)
    return fail(AKB_ECUDA, std::string("stable time step: ") + cudaGetErrorString(e));
  return AKB_OK;
}

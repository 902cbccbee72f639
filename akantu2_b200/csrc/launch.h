// Host-side launchers of the explicit-step kernels (one translation unit per
// arithmetic: kernels_fp64.cu is built with --fmad=false, kernels_mixed.cu
// with contraction allowed).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fe_device.cuh"

namespace akb {

struct QuadTable;
struct GroupArgs;

// launch shape of the element-force kernel of one law group: threads per
// block (64, 128 or 256) and, for the mixed _hexahedron_8 kernel, the
// quadrature points per unrolled iteration (1, 2 or 8; 0 selects the dN/dx
// form) and the resident blocks per SM its registers are capped for (1: the
// compiler's choice; 5 with 128 threads).  Threads per block and the
// register cap leave the arithmetic unchanged; the points per iteration do
// not (FP32 contraction differs).
struct ElemTuning {
  int block = 128;
  int qu = 8;
  int minb = 1;
  // packed hexahedron kernel and the one-thread-per-element kernel of
  // tetrahedra and triangles: distance, in waves of resident blocks, at which
  // each warp prefetches the per-element table rows of a later warp into L2
  // (0: no prefetch); the results do not depend on it
  int pf = 0;
  // tetrahedra and triangles (one thread per element): 1 recomputes dN/dx and
  // det J w from the coordinates by the precomputation's arithmetic instead
  // of streaming the tables (the same numbers)
  int rec = 0;
  // the streamed law (the same numbers): plain FP64 hexahedra, one thread
  // per point (k_element_forces_pqs: dN/dx rows loaded node by node where
  // used, force components sent to shared memory as formed); plastic
  // triangles, one thread per element (k_element_forces_pe_streamed: the
  // displacements gathered per point, dN/dx loaded where used, the force sum
  // in shared memory), with the streamed tables (rec 0, no prefetch)
  int pqs = 0;
};
// points_per_iteration flag of the mixed hexahedron kernel: the points are
// evaluated as packed FP32 pairs (2, 4 or 8 points per iteration)
constexpr int kPackedPoints = 256;

// device view of the mesh, internal element order
struct DevGeom {
  int et, D, NN, NQ;
  int64_t E, N;
  const int32_t *conn;  // [NN][E]
  const double *X;      // [N][D]
  const int32_t *ptr;   // [N+1]
  const int32_t *ent;   // [E*NN] slot (e*NN + a) of each CSR position
  const int32_t *pos;   // [NN][E] CSR position of each slot
  // several independent meshes in one model: instance of each node and the
  // time step of each instance (both null for a single mesh)
  const int32_t *node_inst = nullptr;  // [N]
  const double *inst_dt = nullptr;     // [instances]
  // launch the step kernels with programmatic dependent launch (pdl_begin)
  int pdl = 0;
  // every element is a parallelepiped (mixed hexahedra: the element kernel
  // compiled without per-point geometry)
  int affine = 0;
  // with affine: the adjugate and 1/det of each element [10][E], or null
  const float *geo = nullptr;
  // batch whose instances stop after their own step counts: the step count
  // at which each instance stops and the device step counter (null otherwise)
  const int64_t *inst_end = nullptr;
  int64_t *step = nullptr;
};

// ---- init ------------------------------------------------------------------
cudaError_t launch_precompute(const DevGeom &g, const QuadTable &tab, double *B, double *wJ,
                              unsigned long long *bad, cudaStream_t s);
cudaError_t launch_mass_elem(const DevGeom &g, int64_t e0, int64_t ne, double rho,
                             const QuadTable &tab, const double *wJ, double *me,
                             cudaStream_t s);
cudaError_t launch_gather_scalar(const DevGeom &g, const double *me, double *out,
                                 cudaStream_t s);
// out[perm ? perm[e] : e] = h_e / celerity for the elements e0 .. e0 + ne
cudaError_t launch_element_dt(const DevGeom &g, int64_t e0, int64_t ne, double celerity,
                              const double *u, const int32_t *perm, double *out,
                              cudaStream_t s);
// out[k] = min of x[off[k] .. off[k+1]) (off on the device)
cudaError_t launch_segment_min(const double *x, const int64_t *off, int nseg, double *out,
                               cudaStream_t s);
cudaError_t launch_to_float(const double *in, float *out, int64_t n, cudaStream_t s);
cudaError_t launch_fill(double *out, double v, int64_t n, cudaStream_t s);

// ---- step ------------------------------------------------------------------
// u_pred = predictor displacement of (u, v, a); v and a are not modified
cudaError_t launch_predict(const DevGeom &g, const uint8_t *blocked, const double *u,
                           const double *v, const double *a, double dt, double *u_pred,
                           cudaStream_t s);
cudaError_t launch_element_forces_fp64(const DevGeom &g, int law, int64_t e0, int64_t ne,
                                       const double *B, const double *wJ, const double *u,
                                       const MatParams &mp, const GroupArgs &ps,
                                       double *re, const ElemTuning &tn, const QuadTable &tab,
                                       cudaStream_t s);
// mixed path: 3D elements recompute their shape derivatives in FP32 from g.X
// and the table; 2D elements stream FP32 copies (fB, fwJ) of the precomputed
// ones (their state traffic dominates, the recomputation would not pay)
cudaError_t launch_element_forces_mixed(const DevGeom &g, int law, int64_t e0, int64_t ne,
                                        const QuadTable &tab, const float *fB,
                                        const float *fwJ, const double *u,
                                        const MatParams &mp, const GroupArgs &ps,
                                        float *re, const ElemTuning &tn, cudaStream_t s);
// mixed hexahedra of a mesh of parallelepipeds, elastic or neohookean law:
// the sum-factorised kernel on packed FP32 pairs of points; points per
// unrolled iteration 2, 4 or 8; minb: resident blocks per SM the registers
// are capped for (1, 4 or 5); 128 threads
cudaError_t launch_element_forces_hex8_x2(const DevGeom &g, int law, int64_t e0, int64_t ne,
                                          const double *u, const MatParams &mp,
                                          const GroupArgs &ps, float *re, int points,
                                          int minb, int pf_waves, cudaStream_t s);
// flags: NU_CORRECT | NU_PREDICT | NU_FINT | NU_FEXT_ZERO (fe_kernels.cuh);
// the predictor of the next step reads u and writes u_next
// node_block: threads per block of the node update (any multiple of 32 up to
// 1024; 128, 256 or 512 when staged); form: 0 the direct gather, 1 the gather
// staged through shared memory (k_node_update_staged), 2 the direct gather
// with the node's state read first (k_node_update_early); same arithmetic
cudaError_t launch_node_update_fp64(const DevGeom &g, const double *re, const double *fext,
                                    const double *mass, const uint8_t *blocked, double *fint,
                                    double *a, double *v, const double *u, double *u_next,
                                    double dt, int flags, unsigned int *status, int node_block,
                                    int form, cudaStream_t s);
cudaError_t launch_node_update_mixed(const DevGeom &g, const float *re, const double *fext,
                                     const double *mass, const uint8_t *blocked,
                                     double *fint, double *a, double *v, const double *u,
                                     double *u_next, double dt, int flags,
                                     unsigned int *status, int node_block, int form,
                                     cudaStream_t s);

// the device step counter of a batch with stopping instances, + 1
cudaError_t launch_step_advance(const DevGeom &g, cudaStream_t s);

// prescribed velocity ramp on a set of dofs (u indices node * D + c), written
// into the displacement the next step starts from; acc and step live on the
// device so that captured graphs replay it
cudaError_t launch_prescribe(int64_t count, const int64_t *dofs, const double *u0, double v_max,
                             int64_t ramp_steps, double dt, double *acc, int64_t *step,
                             double *u, bool advance, bool pdl, cudaStream_t s);

// persistent multi-step kernel (one law group; sa describes the steps);
// qu: points per iteration of mixed hexahedra (1 or 2)
struct StepArgs;
cudaError_t launch_persistent_fp64(const DevGeom &g, int law, int qu, const StepArgs &sa,
                                   const QuadTable &tab, cudaStream_t s);
cudaError_t launch_persistent_mixed(const DevGeom &g, int law, int qu, const StepArgs &sa,
                                    const QuadTable &tab, cudaStream_t s);

// ---- fields and energies ---------------------------------------------------
// c33: stored plane-stress stretches of the material's points ([q][c33_ld]),
// eig: their eigen gradients ([q][d*d][c33_ld]); either may be null
cudaError_t launch_qp_fields(const DevGeom &g, int law, int64_t e0, int64_t ne,
                             const double *B, const double *u, const MatParams &mp,
                             const double *c33, int64_t c33_ld, const double *eig,
                             double *grad, double *stress, cudaStream_t s);
// per-dof kinetic terms (m > eps ? v v m : 0) summed per node -> out[N]
cudaError_t launch_ekin_terms(const DevGeom &g, const double *v, const double *mass,
                              double *out, cudaStream_t s);
// per-dof external work terms -> out[N]
cudaError_t launch_work_terms(const DevGeom &g, const double *fext, const double *fint,
                              const double *v, const uint8_t *blocked, double *out,
                              cudaStream_t s);
// per-element sum_q density_q wJ_q of one material -> out[ne]; the
// quadrature-point inputs are [q][comp][ld] with the material's elements at
// 0 .. ne (plastic: grad in float when grad_float, stress and eps_p as
// symmetric components).  which: 0 potential, 1 plastic
cudaError_t launch_energy_elem(const DevGeom &g, int law, int which, int64_t e0, int64_t ne,
                               int64_t ld, const double *wJ, const void *grad, bool grad_float,
                               const double *stress, const double *eps_p, const double *pe,
                               const MatParams &mp, double *out, cudaStream_t s);
// deterministic reductions (fixed grid, fixed tree): result written to *out
// (device); partials needs kReducePartials doubles
constexpr int kReducePartials = 1024;
cudaError_t launch_reduce(const double *x, int64_t n, int op_min, double *partials,
                          double *out, cudaStream_t s);

// buf[k d + c] = u[idx[k] d + c] (pack) or the reverse (unpack), k < n
cudaError_t launch_halo(bool unpack, int d, int64_t n, const int32_t *idx, double *u, double *buf,
                        cudaStream_t s);
// prev = u_n, incr = u_np1 - u_n over the N * D dofs
cudaError_t launch_history(const DevGeom &g, const double *u_n, const double *u_np1,
                           double *prev, double *incr, cudaStream_t s);
// flag = 1 if some hexahedron is not a parallelepiped (FP32 modal test)
// adjugate and 1/det of every element of a mesh of parallelepipeds, [10][E]
cudaError_t launch_hex8_affine_geometry(const DevGeom &g, float *geo, cudaStream_t s);
cudaError_t launch_hex8_affine_check(const DevGeom &g, unsigned int *flag, cudaStream_t s);
// the same check and table in FP64 (fast FP64 path)
cudaError_t launch_hex8_affine_check_fp64(const DevGeom &g, unsigned int *flag, cudaStream_t s);
cudaError_t launch_hex8_affine_geometry_fp64(const DevGeom &g, double *geo, cudaStream_t s);
// fast FP64 path, hexahedra: the sum-factorised element kernel in FP64 with
// contraction allowed (not the operation order of the CPU path: within
// 1e-12 of it); geo: the FP64 adjugate table of a mesh of parallelepipeds,
// or null (geometry formed per point); tn.qu 1, 2 or 8 points per
// iteration, tn.minb 1, 2 or 3 (with 2 points)
cudaError_t launch_element_forces_fp64_sf(const DevGeom &g, int law, int64_t e0, int64_t ne,
                                          const double *u, const MatParams &mp,
                                          const GroupArgs &ps, double *re, const double *geo,
                                          const ElemTuning &tn, cudaStream_t s);
}  // namespace akb

// Mixed-precision kernels: FP32 element kinematics, stress and B^T sigma,
// FP64 nodal state with a compensated (Kahan) FP64 gather of the FP32
// elemental forces.  Contraction (FMA) is allowed in this translation unit.
#include "dispatch.cuh"

namespace akb {

cudaError_t launch_element_forces_mixed(const DevGeom &g, int law, int64_t e0, int64_t ne,
                                        const QuadTable &tab, const float *fB,
                                        const float *fwJ, const double *u,
                                        const MatParams &mp, const GroupArgs &ps,
                                        float *re, cudaStream_t s) {
  if (ne == 0) return cudaSuccess;
  if (g.D == 2) return element_forces_impl<float, float>(g, law, e0, ne, fB, fwJ, u, mp, ps, re, s);
  AKB_DISPATCH_ELEM(g, {
    (void)ET;
    const unsigned grid = (unsigned)((ne + kPeThreads - 1) / kPeThreads);
    if (law == LAW_ELASTIC)
      k_element_forces_geo<D, NN, NQ, LAW_ELASTIC>
          <<<grid, kPeThreads, 0, s>>>(e0, ne, g.E, g.conn, g.pos, g.X, tab, u, mp, ps, re);
    else if (law == LAW_NEOHOOKEAN)
      k_element_forces_geo<D, NN, NQ, LAW_NEOHOOKEAN>
          <<<grid, kPeThreads, 0, s>>>(e0, ne, g.E, g.conn, g.pos, g.X, tab, u, mp, ps, re);
    else
      k_element_forces_geo<D, NN, NQ, LAW_PLASTIC>
          <<<grid, kPeThreads, 0, s>>>(e0, ne, g.E, g.conn, g.pos, g.X, tab, u, mp, ps, re);
  });
  return cudaGetLastError();
}

cudaError_t launch_node_update_mixed(const DevGeom &g, const float *re, const double *fext,
                                     const double *mass, const uint8_t *blocked,
                                     double *fint, double *a, double *v, const double *u,
                                     double *u_next, double dt, int flags,
                                     unsigned int *status, cudaStream_t s) {
  if (g.N == 0) return cudaSuccess;
  if (g.D == 3)
    k_node_update<3, float, true><<<grid_for(g.N), kThreads, 0, s>>>(
        g.N, g.ptr, re, fext, mass, blocked, fint, a, v, u, u_next, dt, g.node_inst, g.inst_dt,
        flags, status);
  else
    k_node_update<2, float, true><<<grid_for(g.N), kThreads, 0, s>>>(
        g.N, g.ptr, re, fext, mass, blocked, fint, a, v, u, u_next, dt, g.node_inst, g.inst_dt,
        flags, status);
  return cudaGetLastError();
}

}  // namespace akb

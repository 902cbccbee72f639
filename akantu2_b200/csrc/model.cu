// Host runtime behind the C ABI (include/akb_capi.h): model construction,
// material instantiation from .dat sections, device memory, the explicit
// step pipeline and the field / energy getters.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <limits>
#include <string>
#include <vector>

#include "akb_capi.h"
#include "dat_parser.h"
#include "fe_kernels.cuh"
#include "host_common.h"
#include "launch.h"

namespace akb {
static thread_local std::string g_last_error;
int fail(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}
}  // namespace akb

using namespace akb;

#define AKB_CUDA(call)                                                                   \
  do {                                                                                   \
    cudaError_t err_ = (call);                                                           \
    if (err_ != cudaSuccess)                                                             \
      return fail(AKB_ECUDA, std::string(#call) + ": " + cudaGetErrorString(err_));      \
  } while (0)

#define AKB_TRY(call)                                                                    \
  do {                                                                                   \
    int rc_ = (call);                                                                    \
    if (rc_ != AKB_OK) return rc_;                                                       \
  } while (0)

namespace {

struct Material {
  std::string type, name;
  int law = LAW_ELASTIC;
  double rho = 0., E = 0., nu = 0.5, sigma_y = 0., h = 0., alpha = 0., delta_T = 0.;
  bool plane_stress = false, finite_deformation = false;
  // `elastic` with finite_deformation: runs in the finite-strain (neohookean)
  // kernels with the elastic law applied to the Green-Lagrange strain
  bool svk = false;
  double lambda = 0., mu = 0., sigma_th = 0.;
  // eigen_grad_u parameter (material.cc:35-51), column-major d x d; every
  // point of the material starts from it (Material::updateInternalParameters)
  double eig[9] = {0., 0., 0., 0., 0., 0., 0., 0., 0.};
  bool has_eig = false;
  double eig_in[9] = {0., 0., 0., 0., 0., 0., 0., 0., 0.};  // as parsed, 3 x 3
  int eig_rows = 0, eig_cols = 0;                           // parsed size
  // sigma_th internal and its saved previous value (material_thermal.cc:33-34):
  // a stress evaluation sets th_cur = sigma_th, the start of a step saves
  // th_prev = th_cur; the plastic trial stress takes th_prev - th_cur
  double th_prev = 0., th_cur = 0., dsth = 0.;
  int64_t e_begin = 0, e_count = 0;  // internal element range
  int group = 0;                     // law group holding the range

  // Lame update (material_elastic.cc:53-78, material_neohookean.cc:61-67),
  // thermal stress (material_thermal.hh:89-95)
  void update(int dim) {
    lambda = nu * E / ((1 + nu) * (1 - 2 * nu));
    mu = E / (2 * (1 + nu));
    if (dim == 2 && plane_stress && (law != LAW_NEOHOOKEAN || svk))
      lambda = nu * E / ((1 + nu) * (1 - nu));
    sigma_th = -E / (1. - 2. * nu) * alpha * delta_T;
  }
  MatParams params() const {
    return MatParams{lambda, mu, sigma_y, h, sigma_th, rho, svk ? 1 : 0, c33 ? 1 : 0, dsth};
  }
  bool c33 = false;  // plane-stress neohookean (set by initFull in 2D)
  double celerity() const { return std::sqrt((lambda + 2 * mu) / rho); }
};

// Law group: the elements of all materials with one constitutive law, one
// contiguous internal range, advanced by one kernel launch per step.  Its
// plastic internals are [q][comp][e_count] arrays (group-local element
// fastest), ping-pong prev / cur; a material's part starts at column
// (material e_begin - group e_begin).
struct Group {
  int law = LAW_ELASTIC;
  ElemTuning tune;  // launch shape of the group's element-force kernel
  int mat0 = 0;  // first material of the group
  int nmat = 0;
  int64_t e_begin = 0, e_count = 0;
  // stress and plastic strain as symmetric components, the gradient in the
  // element-math type (float on the mixed path)
  double *sig[2] = {nullptr, nullptr}, *eps[2] = {nullptr, nullptr};
  void *gu[2] = {nullptr, nullptr};
  double *iso[2] = {nullptr, nullptr};
  double *pe = nullptr;
  // plane-stress neohookean: out-of-plane stretch C33 per point, initially 1
  // (third_axis_deformation, plane_stress_toolbox_tmpl.hh:46)
  double *c33 = nullptr;
  // eigen gradient of every point [q][d*d][e_count], or null while every
  // material of the group has a zero one
  double *eig = nullptr;
};

// independent components of a symmetric d x d tensor, and the map from
// column-major entry k to component (the device-side SymComps / sym_of)
int sym_comps(int d) { return d == 3 ? 6 : 3; }
int sym_component(int d, int k) {
  if (d == 3) {
    static const int m[9] = {0, 5, 4, 5, 1, 3, 4, 3, 2};
    return m[k];
  }
  static const int m2[4] = {0, 2, 2, 1};
  return m2[k];
}

int nodes_per_element(int et) {
  return et == AKB_TETRAHEDRON_4 ? 4 : (et == AKB_HEXAHEDRON_8 ? 8 : 6);
}
int dim_of(int et) { return et == AKB_TRIANGLE_6 ? 2 : 3; }

// quadrature tables (gauss_integration.cc) and the natural-coordinate shape
// functions / derivatives of the element files, evaluated at the points
int quadrature(int et, int rule, double *pts, double *w) {
  if (et == AKB_TETRAHEDRON_4) {
    pts[0] = pts[1] = pts[2] = 1. / 4.;
    w[0] = 1. / 6.;
    return 1;
  }
  if (et == AKB_HEXAHEDRON_8) {
    const double g[2] = {-1. / std::sqrt(3.), 1. / std::sqrt(3.)};
    for (int q = 0; q < 8; ++q) {
      pts[q * 3 + 0] = g[q & 1];
      pts[q * 3 + 1] = g[(q >> 1) & 1];
      pts[q * 3 + 2] = g[(q >> 2) & 1];
      w[q] = 1.;
    }
    return 8;
  }
  if (rule == 0) {
    const double p[6] = {1. / 6., 1. / 6., 2. / 3., 1. / 6., 1. / 6., 2. / 3.};
    std::copy(p, p + 6, pts);
    w[0] = w[1] = w[2] = 1. / 6.;
    return 3;
  }
  const double a = (8. - std::sqrt(10.) + std::sqrt(38. - 44. * std::sqrt(2. / 5.))) / 18.;
  const double b = (8. - std::sqrt(10.) - std::sqrt(38. - 44. * std::sqrt(2. / 5.))) / 18.;
  const double w1 = (620. - std::sqrt(213125. - 53320. * std::sqrt(10.))) / 7440.;
  const double w2 = (620. + std::sqrt(213125. - 53320. * std::sqrt(10.))) / 7440.;
  const double p[12] = {b, b, 1. - 2. * b, b, b, 1. - 2. * b, a, 1. - 2. * a, a, a, 1. - 2. * a, a};
  std::copy(p, p + 12, pts);
  w[0] = w[1] = w[2] = w1;
  w[3] = w[4] = w[5] = w2;
  return 6;
}

void fill_tables(int et, int rule, QuadTable &tab, int &nq) {
  std::memset(&tab, 0, sizeof(tab));
  double pts[24], w[8];
  nq = quadrature(et, rule, pts, w);
  const int d = dim_of(et);
  for (int q = 0; q < nq; ++q) {
    const double *c = &pts[q * d];
    double *N = &tab.N[q * kMaxNN];
    double *r0 = &tab.dnds[q * 3 * kMaxNN], *r1 = r0 + kMaxNN, *r2 = r1 + kMaxNN;
    tab.w[q] = w[q];
    if (et == AKB_TETRAHEDRON_4) {
      double c0 = 1 - c[0] - c[1] - c[2];
      N[0] = c0; N[1] = c[1]; N[2] = c[2]; N[3] = c[0];
      const double v0[4] = {-1., 0., 0., 1.}, v1[4] = {-1., 1., 0., 0.}, v2[4] = {-1., 0., 1., 0.};
      for (int a = 0; a < 4; ++a) { r0[a] = v0[a]; r1[a] = v1[a]; r2[a] = v2[a]; }
    } else if (et == AKB_HEXAHEDRON_8) {
      // node a at (sx, sy, sz) in {-1, 1}^3, element_class_hexahedron_8_inline_impl.hh
      static const int s[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                  {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
      for (int a = 0; a < 8; ++a) {
        const double fx = s[a][0] < 0 ? (1 - c[0]) : (1 + c[0]);
        const double fy = s[a][1] < 0 ? (1 - c[1]) : (1 + c[1]);
        const double fz = s[a][2] < 0 ? (1 - c[2]) : (1 + c[2]);
        N[a] = .125 * fx * fy * fz;
        r0[a] = (s[a][0] < 0 ? -.125 : .125) * fy * fz;
        r1[a] = (s[a][1] < 0 ? -.125 : .125) * fx * fz;
        r2[a] = (s[a][2] < 0 ? -.125 : .125) * fx * fy;
      }
    } else {
      double c0 = 1 - c[0] - c[1], c1 = c[0], c2 = c[1];
      N[0] = c0 * (2 * c0 - 1.); N[1] = c1 * (2 * c1 - 1.); N[2] = c2 * (2 * c2 - 1.);
      N[3] = 4 * c0 * c1; N[4] = 4 * c1 * c2; N[5] = 4 * c2 * c0;
      r0[0] = 1 - 4 * c0; r0[1] = 4 * c1 - 1.; r0[2] = 0.;
      r0[3] = 4 * (c0 - c1); r0[4] = 4 * c2; r0[5] = -4 * c2;
      r1[0] = 1 - 4 * c0; r1[1] = 0.; r1[2] = 4 * c2 - 1.;
      r1[3] = -4 * c1; r1[4] = 4 * c1; r1[5] = 4 * (c0 - c2);
    }
  }
  for (int k = 0; k < kMaxNQ * 3 * kMaxNN; ++k) tab.fdnds[k] = (float)tab.dnds[k];
  for (int q = 0; q < kMaxNQ; ++q) tab.fw[q] = (float)tab.w[q];
}

}  // namespace

struct akb_model {
  int dim = 3, et = 0, nn = 4, nq = 1, rule = 0, precision = AKB_PRECISION_FP64;
  int64_t N = 0, E = 0;
  std::vector<double> X;
  std::vector<int32_t> conn;        // user order [E][nn]
  std::vector<int32_t> mat_user;    // user element -> material
  std::vector<Material> mats;
  std::vector<Group> groups;
  std::vector<int64_t> perm;        // internal element -> user element
  // independent meshes advanced together (batch): node and element ranges of
  // each instance in user order, and the time step of each
  int ninst = 1;
  bool is_batch = false;  // made by akb_batch_create
  std::vector<int64_t> inst_node_off{0, 0}, inst_elem_off{0, 0};
  std::vector<double> inst_dt;
  bool initialized = false, forces_evaluated = false, snap_valid = false;
  int cur = 0;  // ping-pong index of the latest plastic state
  int64_t steps_done = 0;
  double dt = 0.;
  int device = 0;
  cudaStream_t stream = nullptr;
  // device arrays
  double *dX = nullptr, *dB = nullptr, *dwJ = nullptr;
  float *fB = nullptr, *fwJ = nullptr;  // FP32 copies (mixed path, 2D elements)
  QuadTable tab;  // quadrature tables of the element type
  int32_t *dconn = nullptr, *dptr = nullptr, *dent = nullptr, *dpos = nullptr;
  MatParams *dmtab = nullptr;  // all materials, for groups of several
  std::vector<double> mtab_dsth;  // the dsth values dmtab holds
  int32_t *dmslot = nullptr;   // [E] material of each internal element
  int32_t *dnode_inst = nullptr, *dperm = nullptr;  // batch: [N] instance, [E] user id
  double *dinst_dt = nullptr, *dinst_min = nullptr;  // batch: [ninst]
  int64_t *dinst_eoff = nullptr;                     // batch: [ninst + 1]
  // batch whose instances stop after their own step counts
  // (akb_batch_set_instance_steps): the step count at which each stops, the
  // device step counter and the instance of each internal element
  int64_t *dinst_end = nullptr, *dstep = nullptr;
  int32_t *delem_inst = nullptr;
  std::vector<int64_t> inst_end;
  // displacement ping-pong: dU[ucur] is the model's u, dU[1 - ucur] the
  // prediction of the next step (valid when `predicted`)
  double *dU[2] = {nullptr, nullptr};
  int ucur = 0;
  bool predicted = false;
  bool fint_valid = true;  // dfint holds the internal force of the last evaluation
  bool fext_zero = true;   // the external force is identically zero
  double *dv = nullptr, *da = nullptr, *dfext = nullptr, *dfint = nullptr;
  double *dmass = nullptr, *dusnap = nullptr;
  uint8_t *dblocked = nullptr;
  void *dre = nullptr;
  double *dscratch = nullptr, *dpartials = nullptr, *dresult = nullptr;
  double *dqp_a = nullptr, *dqp_b = nullptr;
  int64_t qp_scratch_size = 0;
  unsigned int *dstatus = nullptr;
  unsigned long long *dbad = nullptr;
  std::vector<void *> allocs;
  // captured multi-step graphs, keyed by the buffer parities they start from
  // (an even number of steps returns to the same parities) and by the values
  // baked into their launches
  struct StepGraph {
    cudaGraphExec_t exec = nullptr;
    int ucur = 0, cur = 0;
    double dt = 0.;
    bool fext_zero = true;
    int64_t steps = 0;
  };
  std::vector<StepGraph> graphs;
  int64_t graph_steps = 100;  // steps per captured graph (even; 0 disables)
  int stream_priority = 0;    // of the model's stream, when priority_set
  bool priority_set = false;
  int node_block = 128;       // threads per block of the node update
  int node_form = 0;  // node update: 0 direct, 1 staged gather, 2 state first
  // mixed hexahedra: every element a parallelepiped (found at initFull), and
  // the kernel in use: 0 the general one, 1 the one compiled for such meshes,
  // 2 the same reading each element's adjugate and 1/det from dgeo [10][E]
  bool all_affine = false;
  int affine_kernel = 0;
  float *dgeo = nullptr;
  // fast FP64 path (AKB_PRECISION_FP64_FAST): FP64 state and element math,
  // hexahedra by the sum-factorised kernel with contraction allowed, reading
  // the FP64 adjugate table of a mesh of parallelepipeds (dgeo64) or forming
  // their geometry per point
  bool fast64 = false;
  double *dgeo64 = nullptr;
  // previous displacement and increment of the last step, when tracked
  bool track_history = false;
  double *dprev = nullptr, *dincr = nullptr;
  // step kernels launched with programmatic stream serialization: each one
  // is scheduled while its predecessor drains and waits for it on the device
  bool pdl = false;
  // persistent multi-step kernel: 0 never (default: on B200 the 100-step
  // graphs of the two-kernel step are faster at every measured size), 1 for
  // small single-group meshes, 2 whenever the model allows it
  int persistent = 0;
  unsigned int *dbar = nullptr;  // grid-barrier counters
  // the persistent kernel's bound on a barrier wait, and the failure-path
  // setting that makes one block arrive late (akb_model_set_persistent_wait_test)
  unsigned int bar_spin_limit = kBarrierSpinLimit;
  int bar_late_block = -1;
  unsigned int bar_late_us = 0;
  // prescribed velocity ramp on a set of dofs (akb_model_set_prescribed_velocity_ramp)
  int64_t presc_count = 0, presc_ramp = 1;
  double presc_vmax = 0.;
  int64_t *dpresc_dofs = nullptr, *dpresc_step = nullptr;
  double *dpresc_u0 = nullptr, *dpresc_acc = nullptr;
  // the prescribed value of the coming step is in place (a prediction made
  // again after a host write re-applies it instead of advancing the ramp)
  bool presc_ahead = false;

  double *u() const { return dU[ucur]; }
  double *u_pred() const { return dU[1 - ucur]; }
  DevGeom geom() const {
    DevGeom g;
    g.et = et; g.D = dim; g.NN = nn; g.NQ = nq; g.E = E; g.N = N;
    g.conn = dconn; g.X = dX; g.ptr = dptr; g.ent = dent; g.pos = dpos;
    g.node_inst = dnode_inst;
    g.inst_dt = dinst_dt;
    g.pdl = pdl ? 1 : 0;
    g.affine = affine_kernel ? 1 : 0;
    g.geo = affine_kernel == 2 ? dgeo : nullptr;
    g.inst_end = dinst_end;
    g.step = dstep;
    return g;
  }
  // stream-ordered allocations on the model's stream: neither allocating
  // nor freeing waits for the work of other models on the device
  template <class P> int alloc(P **p, size_t bytes) {
    void *q = nullptr;
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMallocAsync(&q, bytes, stream);
    if (e != cudaSuccess)
      return fail(e == cudaErrorMemoryAllocation ? AKB_ENOMEM : AKB_ECUDA,
                  std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
    allocs.push_back(q);
    device_bytes += bytes;
    *p = (P *)q;
    return AKB_OK;
  }
  size_t device_bytes = 0;
  // asynchronous nodal I/O: copy streams, device staging (two upload
  // buffers, AKB_ASYNC_READS_IN_FLIGHT read buffers) and the events that
  // order them against the step stream
  struct AsyncIO {
    static constexpr int kIn = 2, kOut = AKB_ASYNC_READS_IN_FLIGHT;
    cudaStream_t in = nullptr, out = nullptr;
    double *stage_in[kIn] = {}, *stage_out[kOut] = {};
    cudaEvent_t in_ready[kIn] = {}, in_used[kIn] = {};
    cudaEvent_t out_ready[kOut] = {}, out_done[kOut] = {};
    int in_k = 0;
    int64_t out_tickets = 0;  // copies issued so far
  } aio;
  ~akb_model() {
    if (aio.in) cudaStreamSynchronize(aio.in);
    if (aio.out) cudaStreamSynchronize(aio.out);
    for (auto &g : graphs) cudaGraphExecDestroy(g.exec);
    for (void *p : allocs) cudaFreeAsync(p, stream);
    for (int k = 0; k < AsyncIO::kIn; ++k)
      for (cudaEvent_t e : {aio.in_ready[k], aio.in_used[k]})
        if (e) cudaEventDestroy(e);
    for (int k = 0; k < AsyncIO::kOut; ++k)
      for (cudaEvent_t e : {aio.out_ready[k], aio.out_done[k]})
        if (e) cudaEventDestroy(e);
    if (aio.in) cudaStreamDestroy(aio.in);
    if (aio.out) cudaStreamDestroy(aio.out);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

// a matrix parameter, rows of a bracketed list "[[a, b, c], [d, e, f], ...]"
// (the .dat grammar of parsable matrices, algebraic_parser.hh:363-380);
// entries are expressions.  rows[i][j] is entry (i, j).
bool parse_matrix(const std::string &val, std::vector<std::vector<double>> &rows) {
  size_t p = 0;
  auto ws = [&]() {
    while (p < val.size() && std::isspace((unsigned char)val[p])) ++p;
  };
  ws();
  if (p >= val.size() || val[p] != '[') return false;
  ++p;
  rows.clear();
  for (;;) {
    ws();
    if (p >= val.size() || val[p] != '[') return false;
    ++p;
    std::vector<double> row;
    for (;;) {
      size_t b = p;
      int depth = 0;
      while (p < val.size() && !(depth == 0 && (val[p] == ',' || val[p] == ']'))) {
        if (val[p] == '(') ++depth;
        if (val[p] == ')') --depth;
        ++p;
      }
      if (p >= val.size()) return false;
      double x;
      if (!eval_value(val.substr(b, p - b), x)) return false;
      row.push_back(x);
      if (val[p++] == ']') break;
    }
    rows.push_back(row);
    ws();
    if (p < val.size() && val[p] == ',') {
      ++p;
      continue;
    }
    if (p < val.size() && val[p] == ']') {
      ++p;
      break;
    }
    return false;
  }
  ws();
  return p == val.size();
}

int apply_param(Material &m, const std::string &key, const std::string &val) {
  if (key == "name") {
    m.name = val;
    return AKB_OK;
  }
  if (key == "eigen_grad_u") {
    // a matrix (its leading d x d block is used, ParameterTyped<Matrix>::setAuto,
    // parameter_registry_tmpl.hh:203-217), or a scalar 0
    std::vector<std::vector<double>> rows;
    double z;
    if (parse_matrix(val, rows)) {
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          const double x = (i < (int)rows.size() && j < (int)rows[i].size()) ? rows[i][j] : 0.;
          m.eig_in[i + 3 * j] = x;  // column-major; the d x d block is taken at initFull
        }
      m.eig_rows = (int)rows.size();
      m.eig_cols = 3;
      for (auto &r : rows) m.eig_cols = std::min(m.eig_cols, (int)r.size());
      return AKB_OK;
    }
    if (eval_value(val, z) && z == 0.) return AKB_OK;
    return fail(AKB_EPARSE, "eigen_grad_u must be a matrix [[...], ...] (got '" + val + "')");
  }
  double v;
  if (!eval_value(val, v))
    return fail(AKB_EPARSE, "material parameter '" + key + "' has a non-numeric value '" + val + "'");
  if (key == "rho") m.rho = v;
  else if (key == "E") m.E = v;
  else if (key == "nu") m.nu = v;
  else if (key == "sigma_y") m.sigma_y = v;
  else if (key == "h") m.h = v;
  else if (key == "alpha") m.alpha = v;
  else if (key == "delta_T") m.delta_T = v;
  else if (key == "Plane_Stress") m.plane_stress = v != 0.;
  else if (key == "finite_deformation") m.finite_deformation = v != 0.;
  else
    return fail(AKB_EPARSE, "unknown material parameter '" + key + "'");
  return AKB_OK;
}

int make_material(akb_model *m, const std::string &type, const std::string &name,
                  const std::vector<std::pair<std::string, std::string>> &kv, bool permissive) {
  Material mat;
  mat.type = type;
  if (type == "elastic") mat.law = LAW_ELASTIC;
  else if (type == "neohookean") { mat.law = LAW_NEOHOOKEAN; mat.finite_deformation = true; }
  else if (type == "plastic_linear_isotropic_hardening") mat.law = LAW_PLASTIC;
  else return fail(AKB_EMATERIAL, "unknown material type '" + type + "'");
  mat.name = name;
  for (auto &p : kv) {
    int rc = apply_param(mat, p.first, p.second);
    if (rc == AKB_EPARSE && permissive && p.first != "rho" && p.first != "E" && p.first != "nu")
      continue;
    if (rc != AKB_OK) return rc;
  }
  if (mat.law == LAW_ELASTIC && mat.finite_deformation) {
    mat.law = LAW_NEOHOOKEAN;
    mat.svk = true;
  }
  if (mat.law == LAW_PLASTIC && mat.finite_deformation)
    return fail(AKB_EUNSUPPORTED, "finite-strain plasticity is not supported by this path");
  m->mats.push_back(mat);
  return AKB_OK;
}

// every double of x is +0.0 (a -0.0 counts as nonzero, which only costs the
// step the read of f_ext): an OR over 64-bit words, 512 at a time
bool all_zero_bits(const void *x, size_t n) {
  const uint64_t *w = static_cast<const uint64_t *>(x);
  size_t i = 0;
  for (; i + 512 <= n; i += 512) {
    uint64_t acc = 0;
    for (size_t j = 0; j < 512; ++j) acc |= w[i + j];
    if (acc) return false;
  }
  uint64_t acc = 0;
  for (; i < n; ++i) acc |= w[i];
  return acc == 0;
}

int check_model(akb_model *m, bool need_init) {
  if (!m) return fail(AKB_EINVAL, "null model");
  if (need_init && !m->initialized) return fail(AKB_ESTATE, "initFull has not been called");
  return AKB_OK;
}

int64_t nodal_doubles(const akb_model *m) { return m->N * m->dim; }

// snapshot of u used by the elastic / neohookean quadrature-point getters
// when the displacement is overwritten after the last force evaluation
int snapshot_u(akb_model *m) {
  if (!m->forces_evaluated || m->snap_valid) return AKB_OK;
  bool need = false;
  for (auto &mt : m->mats) need |= mt.law != LAW_PLASTIC;
  if (!need) return AKB_OK;
  if (!m->dusnap) AKB_TRY(m->alloc(&m->dusnap, sizeof(double) * nodal_doubles(m)));
  AKB_CUDA(cudaMemcpyAsync(m->dusnap, m->u(), sizeof(double) * nodal_doubles(m),
                           cudaMemcpyDeviceToDevice, m->stream));
  m->snap_valid = true;
  return AKB_OK;
}

GroupArgs group_args(akb_model *m, const Group &mt, bool in_step) {
  GroupArgs ps;
  std::memset(&ps, 0, sizeof(ps));
  if (mt.nmat > 1) {
    ps.mtab = m->dmtab;
    ps.mslot = m->dmslot + mt.e_begin;
  }
  ps.c33 = mt.c33;
  ps.eig = mt.eig;
  ps.nb_nodes = m->N;
  ps.nb_slots = m->E * m->nn;
  ps.status = m->dstatus;
  if (m->dinst_end) {
    ps.einst = m->delem_inst + mt.e_begin;
    ps.inst_end = m->dinst_end;
    ps.step = m->dstep;
  }
  if (mt.law != LAW_PLASTIC) return ps;
  const int c = m->cur;
  // inside a step the new state goes to the other buffer; a standalone
  // assembly recomputes the current state from the previous one
  const int prev = in_step ? c : 1 - c;
  const int out = in_step ? 1 - c : c;
  ps.sig_prev = mt.sig[prev];
  ps.gu_prev = mt.gu[prev];
  ps.eps_prev = mt.eps[prev];
  ps.iso_prev = mt.iso[prev];
  ps.iso_cur_in = mt.iso[c];
  ps.sig = mt.sig[out];
  ps.gu = mt.gu[out];
  ps.eps = mt.eps[out];
  ps.iso = mt.iso[out];
  ps.pe = mt.pe;
  ps.update_energy = in_step ? 1 : 0;
  return ps;
}

// the device table of per-material parameters (groups of several materials)
// follows the materials' dsth values
int sync_mtab(akb_model *m) {
  if (!m->dmtab) return AKB_OK;
  const size_t nm = m->mats.size();
  bool same = m->mtab_dsth.size() == nm;
  for (size_t k = 0; same && k < nm; ++k)
    same = std::memcmp(&m->mtab_dsth[k], &m->mats[k].dsth, sizeof(double)) == 0;
  if (same) return AKB_OK;
  std::vector<MatParams> tab(nm);
  m->mtab_dsth.resize(nm);
  for (size_t k = 0; k < nm; ++k) {
    tab[k] = m->mats[k].params();
    m->mtab_dsth[k] = m->mats[k].dsth;
  }
  // pageable source: the call returns once the data is staged
  AKB_CUDA(cudaMemcpyAsync(m->dmtab, tab.data(), sizeof(MatParams) * nm, cudaMemcpyHostToDevice,
                           m->stream));
  return AKB_OK;
}

// sigma_th of the plastic materials for one stress evaluation: a step first
// saves the previous value (Material::savePreviousState, material.cc:737),
// then MaterialThermal::computeStress sets the current one
// (material_thermal.hh:89-95); the trial stress of the radial return takes
// previous - current (material_linear_isotropic_hardening_inline_impl.hh:31-34)
int thermal_eval(akb_model *m, bool in_step) {
  for (auto &mt : m->mats) {
    if (mt.law != LAW_PLASTIC) continue;
    if (in_step) mt.th_prev = mt.th_cur;
    mt.th_cur = mt.sigma_th;
    mt.dsth = mt.th_prev - mt.th_cur;
  }
  return sync_mtab(m);
}

// every step from now on has a zero thermal term (the current sigma_th is
// the material's and the last evaluation had none): steps may be replayed
// from captured graphs, whose launches bake the parameters in
bool thermal_steady(const akb_model *m) {
  for (auto &mt : m->mats)
    if (mt.law == LAW_PLASTIC && (mt.th_cur != mt.sigma_th || mt.dsth != 0.)) return false;
  return true;
}

// elemental forces at the predicted displacement (inside a step) or at the
// model's displacement (standalone assembly)
int element_forces(akb_model *m, bool in_step) {
  AKB_TRY(thermal_eval(m, in_step));
  DevGeom g = m->geom();
  const double *u = in_step ? m->u_pred() : m->u();
  for (auto &gr : m->groups) {
    GroupArgs ps = group_args(m, gr, in_step);
    const MatParams mp = m->mats[gr.mat0].params();
    cudaError_t e;
    if (m->precision == AKB_PRECISION_MIXED)
      e = launch_element_forces_mixed(g, gr.law, gr.e_begin, gr.e_count, m->tab, m->fB, m->fwJ,
                                      u, mp, ps, (float *)m->dre, gr.tune, m->stream);
    else if (m->fast64 && m->et == AKB_HEXAHEDRON_8)
      e = launch_element_forces_fp64_sf(g, gr.law, gr.e_begin, gr.e_count, u, mp, ps,
                                        (double *)m->dre, m->dgeo64, gr.tune, m->stream);
    else
      e = launch_element_forces_fp64(g, gr.law, gr.e_begin, gr.e_count, m->dB, m->dwJ, u, mp,
                                     ps, (double *)m->dre, gr.tune, m->tab, m->stream);
    if (e != cudaSuccess) return fail(AKB_ECUDA, std::string("element forces: ") + cudaGetErrorString(e));
  }
  return AKB_OK;
}

// the prescribed dofs of the step that starts from u_start: advanced to the
// next step of the ramp, or the value of the coming step applied again
int prescribe(akb_model *m, double *u_start, bool advance) {
  if (m->presc_count == 0) return AKB_OK;
  AKB_CUDA(launch_prescribe(m->presc_count, m->dpresc_dofs, m->dpresc_u0, m->presc_vmax,
                            m->presc_ramp, m->dt, m->dpresc_acc, m->dpresc_step, u_start,
                            advance, m->pdl, m->stream));
  m->presc_ahead = true;
  return AKB_OK;
}

// predictor of the coming step from the model's state (when the prediction
// made by the last node update is stale)
int predict(akb_model *m) {
  AKB_CUDA(launch_predict(m->geom(), m->dblocked, m->u(), m->dv, m->da, m->dt, m->u_pred(),
                          m->stream));
  AKB_TRY(prescribe(m, m->u_pred(), !m->presc_ahead));
  m->predicted = true;
  return AKB_OK;
}

// node update after the element forces.  In a step (correct == true): the
// corrector, then the predictor of the next step from the new displacement
// u_pred into the other buffer (which held the displacement of the previous
// step); the internal force is only gathered when asked for (ensure_fint).
// Standalone (correct == false): the internal force only.
int node_update(akb_model *m, bool correct) {
  DevGeom g = m->geom();
  cudaError_t e;
  int flags = correct ? (NU_CORRECT | NU_PREDICT) : NU_FINT;
  if (correct && m->fext_zero) flags |= NU_FEXT_ZERO;
  const double *u = m->u_pred();
  double *u_next = m->u();
  if (m->precision == AKB_PRECISION_MIXED)
    e = launch_node_update_mixed(g, (const float *)m->dre, m->dfext, m->dmass, m->dblocked,
                                 m->dfint, m->da, m->dv, u, u_next, m->dt, flags, m->dstatus,
                                 m->node_block, m->node_form, m->stream);
  else
    e = launch_node_update_fp64(g, (const double *)m->dre, m->dfext, m->dmass, m->dblocked,
                                m->dfint, m->da, m->dv, u, u_next, m->dt, flags, m->dstatus,
                                m->node_block, m->node_form, m->stream);
  if (e != cudaSuccess) return fail(AKB_ECUDA, std::string("node update: ") + cudaGetErrorString(e));
  if (correct) AKB_TRY(prescribe(m, u_next, true));
  m->fint_valid = !correct;
  return AKB_OK;
}

// the internal force of the last force evaluation, gathered again from the
// elemental forces it left in the slot array
int ensure_fint(akb_model *m) {
  if (m->fint_valid || !m->forces_evaluated) return AKB_OK;
  AKB_TRY(node_update(m, false));
  return AKB_OK;
}

// one explicit step: [predictor,] element forces, node update (+ next
// predictor); afterwards the prediction buffer becomes the model's u
int one_step(akb_model *m, bool any_plastic, cudaEvent_t e1 = nullptr,
             cudaEvent_t e2 = nullptr) {
  if (!m->predicted) AKB_TRY(predict(m));
  // previous displacement and increment: the step goes from u() to its
  // prediction u_pred()
  if (m->track_history)
    AKB_CUDA(launch_history(m->geom(), m->u(), m->u_pred(), m->dprev, m->dincr, m->stream));
  if (e1) AKB_CUDA(cudaEventRecord(e1, m->stream));
  AKB_TRY(element_forces(m, true));
  if (e2) AKB_CUDA(cudaEventRecord(e2, m->stream));
  AKB_TRY(node_update(m, true));
  if (m->dstep) AKB_CUDA(launch_step_advance(m->geom(), m->stream));
  m->ucur = 1 - m->ucur;  // u_{n+1} is now the model's displacement
  if (any_plastic) m->cur = 1 - m->cur;
  m->steps_done++;
  return AKB_OK;
}

// graph_steps steps (even) as one CUDA graph launch.  The graph is captured
// from one_step the first time a (parity, dt, f_ext == 0) combination is
// met; capturing does not execute, so the host-side step state is restored
// afterwards and advanced when the graph is launched.
// the graph for the model's current parities, dt and f_ext flag, captured
// (not launched) if it does not exist yet
int capture_graph(akb_model *m, bool any_plastic, akb_model::StepGraph **out = nullptr) {
  akb_model::StepGraph *g = nullptr;
  // a batch reads its time steps from device memory: they are not baked in
  const double key_dt = m->ninst > 1 ? 0. : m->dt;
  for (auto &x : m->graphs)
    if (x.ucur == m->ucur && x.cur == m->cur && x.dt == key_dt && x.fext_zero == m->fext_zero &&
        x.steps == m->graph_steps)
      g = &x;
  if (!g) {
    const int ucur0 = m->ucur, cur0 = m->cur;
    const int64_t steps0 = m->steps_done;
    // graphs replay steps without a thermal term (thermal_steady): capture
    // them from that state, with the device table already matching it
    std::vector<Material> mats0 = m->mats;
    for (auto &mt : m->mats)
      if (mt.law == LAW_PLASTIC) {
        mt.th_prev = mt.th_cur = mt.sigma_th;
        mt.dsth = 0.;
      }
    AKB_TRY(sync_mtab(m));
    AKB_CUDA(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
    int rc = AKB_OK;
    for (int64_t s = 0; s < m->graph_steps && rc == AKB_OK; ++s) rc = one_step(m, any_plastic);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(m->stream, &graph);
    m->ucur = ucur0;
    m->cur = cur0;
    m->steps_done = steps0;
    for (size_t k = 0; k < m->mats.size(); ++k) {
      m->mats[k].th_prev = mats0[k].th_prev;
      m->mats[k].th_cur = mats0[k].th_cur;
      m->mats[k].dsth = mats0[k].dsth;
    }
    if (rc != AKB_OK || e != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      if (rc != AKB_OK) return rc;
      return fail(AKB_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    }
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess)
      return fail(AKB_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    // uploaded now, so that its first launch costs what the later ones do
    e = cudaGraphUpload(exec, m->stream);
    if (e != cudaSuccess) {
      cudaGraphExecDestroy(exec);
      return fail(AKB_ECUDA, std::string("graph upload: ") + cudaGetErrorString(e));
    }
    if (m->graphs.size() >= 8) {  // keep the cache small: drop the oldest
      cudaGraphExecDestroy(m->graphs.front().exec);
      m->graphs.erase(m->graphs.begin());
    }
    m->graphs.push_back({exec, ucur0, cur0, key_dt, m->fext_zero, m->graph_steps});
    g = &m->graphs.back();
  }
  if (out) *out = g;
  return AKB_OK;
}

int run_graph(akb_model *m, bool any_plastic) {
  akb_model::StepGraph *g = nullptr;
  AKB_TRY(capture_graph(m, any_plastic, &g));
  // the steps of the graph leave the sigma_th history steady
  for (auto &mt : m->mats)
    if (mt.law == LAW_PLASTIC) {
      mt.th_prev = mt.th_cur = mt.sigma_th;
      mt.dsth = 0.;
    }
  AKB_TRY(sync_mtab(m));
  AKB_CUDA(cudaGraphLaunch(g->exec, m->stream));
  m->steps_done += g->steps;
  m->fint_valid = false;
  return AKB_OK;
}

// release word + one arrival flag per block of a persistent launch (its grid
// is at most the resident-block capacity, far below this)
constexpr int kBarrierWords = 1 + 8192;

// small meshes of one law group run whole step sequences in one persistent
// launch (launch latency dominates the two-kernel step below about this size)
constexpr int64_t kPersistentMaxElements = 1 << 18;

bool use_persistent(const akb_model *m) {
#ifdef AKB_BOUNDS_CHECK
  return false;  // the bounds-checking build runs the checked two-kernel step only
#endif
  if (m->persistent == 0 || m->groups.size() != 1 || m->presc_count > 0 || m->E == 0 ||
      m->track_history || m->dinst_end || m->fast64) return false;
  const Group &gr = m->groups[0];
  // mixed hexahedra: the persistent kernel has the 1- and 2-point forms
  if (m->et == AKB_HEXAHEDRON_8 && m->precision == AKB_PRECISION_MIXED && gr.tune.qu != 1 &&
      gr.tune.qu != 2)
    return false;
  static int coop = -1;
  if (coop < 0) {
    int dev = 0, v = 0;
    coop = (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&v, cudaDevAttrCooperativeLaunch, dev) == cudaSuccess && v)
               ? 1
               : 0;
  }
  if (!coop) return false;
  return m->persistent == 2 || m->E <= kPersistentMaxElements;
}

// nsteps steps in persistent launches (up to 10,000 steps each)
int run_persistent(akb_model *m, int64_t nsteps, bool any_plastic) {
  if (!m->predicted) AKB_TRY(predict(m));
  const Group &gr = m->groups[0];
  DevGeom g = m->geom();
  int64_t left = nsteps;
  while (left > 0) {
    const int64_t n = std::min<int64_t>(left, 10000);
    StepArgs sa;
    std::memset(&sa, 0, sizeof(sa));
    sa.E = m->E;
    sa.N = m->N;
    sa.conn = m->dconn;
    sa.pos = m->dpos;
    sa.ptr = m->dptr;
    if (m->precision == AKB_PRECISION_MIXED) {
      sa.B = m->fB;
      sa.wJ = m->fwJ;
    } else {
      sa.B = m->dB;
      sa.wJ = m->dwJ;
    }
    sa.X = m->dX;
    sa.mp = m->mats[gr.mat0].params();
    sa.ps = group_args(m, gr, true);
    sa.re = m->dre;
    sa.fext = m->dfext;
    sa.mass = m->dmass;
    sa.blocked = m->dblocked;
    sa.fint = m->dfint;
    sa.a = m->da;
    sa.v = m->dv;
    sa.u_pred = m->u_pred();
    sa.u_other = m->u();
    sa.dt = m->dt;
    sa.node_inst = m->dnode_inst;
    sa.inst_dt = m->dinst_dt;
    sa.flags = NU_CORRECT | NU_PREDICT | (m->fext_zero ? NU_FEXT_ZERO : 0);
    sa.plastic = any_plastic ? 1 : 0;
    sa.nsteps = n;
    sa.status = m->dstatus;
    sa.bar = m->dbar;
    sa.spin_limit = m->bar_spin_limit;
    sa.late_block = m->bar_late_block;
    sa.late_us = m->bar_late_us;
    AKB_CUDA(cudaMemsetAsync(m->dbar, 0, kBarrierWords * sizeof(unsigned int), m->stream));
    cudaError_t e = m->precision == AKB_PRECISION_MIXED
                        ? launch_persistent_mixed(g, gr.law, gr.tune.qu, sa, m->tab, m->stream)
                        : launch_persistent_fp64(g, gr.law, gr.tune.qu, sa, m->tab, m->stream);
    if (e != cudaSuccess)
      return fail(AKB_ECUDA, std::string("persistent steps: ") + cudaGetErrorString(e));
    if (n & 1) m->ucur = 1 - m->ucur;
    if (any_plastic && (n & 1)) m->cur = 1 - m->cur;
    m->steps_done += n;
    left -= n;
  }
  m->fint_valid = false;
  return AKB_OK;
}

int ensure_qp_scratch(akb_model *m) {
  int64_t need = 0;
  for (auto &mt : m->mats) need = std::max(need, mt.e_count * m->nq * m->dim * m->dim);
  if (need <= m->qp_scratch_size) return AKB_OK;
  AKB_TRY(m->alloc(&m->dqp_a, sizeof(double) * need));
  AKB_TRY(m->alloc(&m->dqp_b, sizeof(double) * need));
  m->qp_scratch_size = need;
  return AKB_OK;
}

// grad u and stress (or PK2) of an elastic / neohookean material into the
// qp scratch buffers, SoA [dd][nqp]
int eval_qp_fields(akb_model *m, const Material &mt) {
  AKB_TRY(ensure_qp_scratch(m));
  const int64_t n = mt.e_count * m->nq * m->dim * m->dim;
  if (!m->forces_evaluated) {
    AKB_CUDA(cudaMemsetAsync(m->dqp_a, 0, sizeof(double) * std::max<int64_t>(n, 1), m->stream));
    AKB_CUDA(cudaMemsetAsync(m->dqp_b, 0, sizeof(double) * std::max<int64_t>(n, 1), m->stream));
    return AKB_OK;
  }
  const double *u = m->snap_valid ? m->dusnap : m->u();
  const Group &gr = m->groups[mt.group];
  const double *c33 = gr.c33 ? gr.c33 + (mt.e_begin - gr.e_begin) : nullptr;
  const double *eig = gr.eig ? gr.eig + (mt.e_begin - gr.e_begin) : nullptr;
  AKB_CUDA(launch_qp_fields(m->geom(), mt.law, mt.e_begin, mt.e_count, m->dB, u, mt.params(),
                            c33, gr.e_count, eig, m->dqp_a, m->dqp_b, m->stream));
  return AKB_OK;
}

// the group's eigen-gradient array [q][d*d][e_count], allocated if needed
// and set to each material's eigen_grad_u parameter at every point.  Graphs
// captured before the array existed read no eigen gradient: they are dropped.
int fill_group_eigen(akb_model *m, int gi) {
  Group &gr = m->groups[gi];
  const int dd = m->dim * m->dim;
  const int64_t ne = gr.e_count, rows = (int64_t)m->nq * dd;
  if (!gr.eig) {
    AKB_TRY(m->alloc(&gr.eig, sizeof(double) * std::max<int64_t>(rows * ne, 1)));
    for (auto &g : m->graphs) cudaGraphExecDestroy(g.exec);
    m->graphs.clear();
  }
  std::vector<double> h((size_t)(rows * ne), 0.);
  for (auto &mt : m->mats) {
    if (mt.group != gi || !mt.has_eig) continue;
    const int64_t off = mt.e_begin - gr.e_begin;
    for (int q = 0; q < m->nq; ++q)
      for (int k = 0; k < dd; ++k)
        std::fill(h.begin() + (size_t)((q * dd + k) * ne + off),
                  h.begin() + (size_t)((q * dd + k) * ne + off + mt.e_count), mt.eig[k]);
  }
  if (!h.empty())
    AKB_CUDA(cudaMemcpyAsync(gr.eig, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice,
                             m->stream));
  AKB_CUDA(cudaStreamSynchronize(m->stream));
  return AKB_OK;
}

int reduce_to_host(akb_model *m, const double *x, int64_t n, bool op_min, double *out) {
  AKB_CUDA(launch_reduce(x, n, op_min ? 1 : 0, m->dpartials, m->dresult, m->stream));
  AKB_CUDA(cudaMemcpyAsync(out, m->dresult, sizeof(double), cudaMemcpyDeviceToHost, m->stream));
  AKB_CUDA(cudaStreamSynchronize(m->stream));
  return AKB_OK;
}

}  // namespace

/* ------------------------------------------------------------------------ */
/* C ABI                                                                    */
/* ------------------------------------------------------------------------ */
extern "C" {

const char *akb_last_error(void) { return g_last_error.c_str(); }
int akb_version(void) { return 100; }

int akb_device_count(int *count) {
  if (!count) return fail(AKB_EINVAL, "null argument");
  int c = 0;
  cudaError_t e = cudaGetDeviceCount(&c);
  if (e != cudaSuccess) {
    *count = 0;
    return fail(AKB_ECUDA, std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
  }
  *count = c;
  return AKB_OK;
}

int akb_set_device(int device) {
  AKB_CUDA(cudaSetDevice(device));
  return AKB_OK;
}

int akb_host_alloc(size_t bytes, void **ptr) {
  if (!ptr) return fail(AKB_EINVAL, "null argument");
  AKB_CUDA(cudaHostAlloc(ptr, bytes ? bytes : 16, cudaHostAllocDefault));
  return AKB_OK;
}

int akb_host_free(void *ptr) {
  if (ptr) AKB_CUDA(cudaFreeHost(ptr));
  return AKB_OK;
}

int akb_model_create(int dim, int et, const double *nodes, int64_t N, const int32_t *conn,
                     int64_t E, akb_model **out) {
  if (!out) return fail(AKB_EINVAL, "null output pointer");
  *out = nullptr;
  if (et < AKB_TETRAHEDRON_4 || et > AKB_TRIANGLE_6) return fail(AKB_EINVAL, "unknown element type");
  if (dim != dim_of(et)) return fail(AKB_EINVAL, "spatial dimension does not match the element type");
  if (N < 0 || E < 0 || (N > 0 && !nodes) || (E > 0 && !conn))
    return fail(AKB_EINVAL, "bad mesh arrays");
  const int nn = nodes_per_element(et);
  if (E * nn >= (int64_t)std::numeric_limits<int32_t>::max())
    return fail(AKB_EINVAL, "mesh too large for 32-bit slot indices");
  for (int64_t k = 0; k < E * nn; ++k)
    if (conn[k] < 0 || conn[k] >= N) return fail(AKB_EINVAL, "connectivity refers to a missing node");
  auto *m = new akb_model();
  m->dim = dim;
  m->et = et;
  m->nn = nn;
  m->N = N;
  m->E = E;
  m->X.assign(nodes, nodes + N * dim);
  m->conn.assign(conn, conn + E * nn);
  m->inst_node_off = {0, N};
  m->inst_elem_off = {0, E};
  *out = m;
  return AKB_OK;
}

int akb_batch_create(int dim, int et, int nb_instances, const int64_t *nb_nodes,
                     const int64_t *nb_elements, const double *nodes, const int32_t *conn,
                     akb_model **out) {
  if (!out) return fail(AKB_EINVAL, "null output pointer");
  *out = nullptr;
  if (nb_instances < 1 || !nb_nodes || !nb_elements)
    return fail(AKB_EINVAL, "a batch needs at least one instance and its sizes");
  if (et < AKB_TETRAHEDRON_4 || et > AKB_TRIANGLE_6) return fail(AKB_EINVAL, "unknown element type");
  const int nn = nodes_per_element(et);
  std::vector<int64_t> noff(nb_instances + 1, 0), eoff(nb_instances + 1, 0);
  for (int k = 0; k < nb_instances; ++k) {
    if (nb_nodes[k] < 0 || nb_elements[k] < 0) return fail(AKB_EINVAL, "negative instance size");
    noff[k + 1] = noff[k] + nb_nodes[k];
    eoff[k + 1] = eoff[k] + nb_elements[k];
  }
  const int64_t N = noff.back(), E = eoff.back();
  if (N >= (int64_t)std::numeric_limits<int32_t>::max())
    return fail(AKB_EINVAL, "batch too large for 32-bit node indices");
  if ((N > 0 && !nodes) || (E > 0 && !conn)) return fail(AKB_EINVAL, "bad mesh arrays");
  // instance-local node ids -> ids in the concatenated node array
  std::vector<int32_t> gconn((size_t)E * nn);
  for (int k = 0; k < nb_instances; ++k)
    for (int64_t j = eoff[k] * nn; j < eoff[k + 1] * nn; ++j) {
      if (conn[j] < 0 || conn[j] >= nb_nodes[k])
        return fail(AKB_EINVAL, "instance " + std::to_string(k) +
                                    ": connectivity refers to a missing node");
      gconn[j] = (int32_t)(conn[j] + noff[k]);
    }
  akb_model *m = nullptr;
  AKB_TRY(akb_model_create(dim, et, nodes, N, gconn.data(), E, &m));
  m->ninst = nb_instances;
  m->is_batch = true;
  m->inst_node_off = noff;
  m->inst_elem_off = eoff;
  m->inst_dt.assign(nb_instances, 0.);
  *out = m;
  return AKB_OK;
}

int akb_batch_nb_instances(const akb_model *m, int *count) {
  if (!m || !count) return fail(AKB_EINVAL, "null argument");
  *count = m->ninst;
  return AKB_OK;
}

int akb_batch_instance_offsets(const akb_model *m, int64_t *node_offsets,
                               int64_t *element_offsets) {
  if (!m) return fail(AKB_EINVAL, "null model");
  if (node_offsets) std::copy(m->inst_node_off.begin(), m->inst_node_off.end(), node_offsets);
  if (element_offsets)
    std::copy(m->inst_elem_off.begin(), m->inst_elem_off.end(), element_offsets);
  return AKB_OK;
}

int akb_batch_set_instance_materials(akb_model *m, const int32_t *material_of_instance) {
  AKB_TRY(check_model(m, false));
  if (!material_of_instance) return fail(AKB_EINVAL, "null array");
  std::vector<int32_t> mat(m->E);
  for (int k = 0; k < m->ninst; ++k)
    for (int64_t e = m->inst_elem_off[k]; e < m->inst_elem_off[k + 1]; ++e)
      mat[e] = material_of_instance[k];
  return akb_model_set_element_materials(m, mat.data());
}

int akb_model_destroy(akb_model *m) {
  if (!m) return AKB_OK;
  if (m->stream) cudaStreamSynchronize(m->stream);
  delete m;
  return AKB_OK;
}

int akb_model_load_materials(akb_model *m, const char *text) {
  AKB_TRY(check_model(m, false));
  if (!text) return fail(AKB_EINVAL, "null text");
  if (m->initialized) return fail(AKB_ESTATE, "materials must be loaded before initFull");
  ParsedFile pf;
  std::string err;
  if (!parse_dat(text, pf, err)) return fail(AKB_EPARSE, ".dat: " + err);
  bool permissive = false;
  auto it = pf.globals.find("permissive_parser");
  if (it != pf.globals.end()) {
    double v;
    permissive = eval_value(it->second, v) && v != 0.;
  }
  for (auto &pm : pf.materials) {
    std::vector<std::pair<std::string, std::string>> kv(pm.raw.begin(), pm.raw.end());
    AKB_TRY(make_material(m, pm.type, pm.name, kv, permissive));
  }
  return AKB_OK;
}

int akb_model_add_material(akb_model *m, const char *type, const char *params) {
  AKB_TRY(check_model(m, false));
  if (!type) return fail(AKB_EINVAL, "null type");
  if (m->initialized) return fail(AKB_ESTATE, "materials must be added before initFull");
  std::string text = std::string("material ") + type + " [\n";
  if (params) {
    for (const char *p = params; *p; ++p) text.push_back(*p == ';' ? '\n' : *p);
  }
  text += "\n]\n";
  ParsedFile pf;
  std::string err;
  if (!parse_dat(text, pf, err)) return fail(AKB_EPARSE, "material parameters: " + err);
  auto &pm = pf.materials.at(0);
  std::vector<std::pair<std::string, std::string>> kv(pm.raw.begin(), pm.raw.end());
  return make_material(m, pm.type, pm.name, kv, false);
}

int akb_model_set_element_materials(akb_model *m, const int32_t *mat) {
  AKB_TRY(check_model(m, false));
  if (m->initialized) return fail(AKB_ESTATE, "element materials must be set before initFull");
  if (!mat && m->E > 0) return fail(AKB_EINVAL, "null array");
  m->mat_user.assign(mat, mat + m->E);
  return AKB_OK;
}

int akb_model_set_quadrature_rule(akb_model *m, int rule) {
  AKB_TRY(check_model(m, false));
  if (m->initialized) return fail(AKB_ESTATE, "the quadrature rule must be set before initFull");
  if (rule != 0 && !(rule == 1 && m->et == AKB_TRIANGLE_6))
    return fail(AKB_EUNSUPPORTED, "only _triangle_6 has an alternative (6-point) rule");
  m->rule = rule;
  return AKB_OK;
}

int akb_model_init_full(akb_model *m, int method, int precision) {
  AKB_TRY(check_model(m, false));
  if (m->initialized) return fail(AKB_ESTATE, "initFull called twice");
  if (method != AKB_EXPLICIT_LUMPED_MASS)
    return fail(AKB_EUNSUPPORTED, "only _explicit_lumped_mass is provided");
  if (precision != AKB_PRECISION_FP64 && precision != AKB_PRECISION_MIXED &&
      precision != AKB_PRECISION_FP64_FAST)
    return fail(AKB_EINVAL, "unknown precision");
  // the fast FP64 path is the FP64 path everywhere but in the element
  // kernel of hexahedra
  m->fast64 = precision == AKB_PRECISION_FP64_FAST;
  if (m->fast64) precision = AKB_PRECISION_FP64;
  if (m->mats.empty()) return fail(AKB_EMATERIAL, "no material defined (parse a .dat first)");
  if (m->mat_user.empty()) m->mat_user.assign(m->E, 0);
  for (int32_t k : m->mat_user)
    if (k < 0 || k >= (int32_t)m->mats.size()) return fail(AKB_EINVAL, "element material index out of range");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(AKB_ECUDA, "no CUDA device available");
  for (auto &mt : m->mats) {
    mt.update(m->dim);
    mt.c33 = m->dim == 2 && mt.law == LAW_NEOHOOKEAN && !mt.svk && mt.plane_stress;
    if (mt.eig_rows > 0) {
      const int d = m->dim;
      if (mt.eig_rows < d || mt.eig_cols < d)
        return fail(AKB_EINVAL, "material '" + mt.name + "': eigen_grad_u needs at least " +
                                    std::to_string(d) + " x " + std::to_string(d) + " entries");
      mt.has_eig = false;
      for (int j = 0; j < d; ++j)
        for (int i = 0; i < d; ++i) {
          mt.eig[i + d * j] = mt.eig_in[i + 3 * j];
          mt.has_eig |= mt.eig[i + d * j] != 0.;
        }
    }
  }
  m->precision = precision;
  AKB_CUDA(cudaGetDevice(&m->device));
  if (m->priority_set)
    AKB_CUDA(cudaStreamCreateWithPriority(&m->stream, cudaStreamNonBlocking, m->stream_priority));
  else
    AKB_CUDA(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));

  const int nn = m->nn, d = m->dim;
  const int64_t E = m->E, N = m->N;
  QuadTable &tab = m->tab;
  fill_tables(m->et, m->rule, tab, m->nq);
  const int nq = m->nq;

  // internal element order: grouped by law, then material, ascending user
  // id inside a material; a law group is one launch per step
  const int nm = (int)m->mats.size();
  std::vector<int> mat_order(nm);  // materials sorted by (law, index)
  for (int k = 0; k < nm; ++k) mat_order[k] = k;
  std::stable_sort(mat_order.begin(), mat_order.end(),
                   [&](int x, int y) { return m->mats[x].law < m->mats[y].law; });
  m->perm.resize(E);
  {
    std::vector<int64_t> count(nm, 0), start(nm, 0);
    for (int64_t e = 0; e < E; ++e) count[m->mat_user[e]]++;
    int64_t off = 0;
    m->groups.clear();
    for (int k : mat_order) {
      Material &mt = m->mats[k];
      start[k] = off;
      mt.e_begin = off;
      mt.e_count = count[k];
      off += count[k];
      if (m->groups.empty() || m->groups.back().law != mt.law) {
        Group gr;
        gr.law = mt.law;
        gr.mat0 = k;
        gr.e_begin = mt.e_begin;
        m->groups.push_back(gr);
      }
      Group &gr = m->groups.back();
      // mixed hexahedra, fastest forms measured at 128^3 on B200: all 8
      // points unrolled (elastic); 2 points per iteration with registers
      // capped for 4 blocks per SM (neohookean); 1 point capped for 5 blocks
      // (plastic, whose state loads need latency hiding more than registers)
      if (m->et == AKB_HEXAHEDRON_8 && precision == AKB_PRECISION_MIXED)
        gr.tune = gr.law == LAW_PLASTIC      ? ElemTuning{128, 1, 5}
                  : gr.law == LAW_NEOHOOKEAN ? ElemTuning{128, 2, 4}
                                             : ElemTuning{128, 8, 1};
      // plastic quadratic triangles: registers capped for 6 (mixed) or 5
      // (FP64) resident blocks, 22-24 % shorter element launches measured on
      // the 512^2 square than uncapped
      if (m->et == AKB_TRIANGLE_6 && gr.law == LAW_PLASTIC)
        gr.tune = ElemTuning{128, 8, precision == AKB_PRECISION_MIXED ? 6 : 5};
      // mixed plastic triangles: the streamed law with 7 blocks, measured on
      // the 512^2 square: 0.0845 against 0.0875 ms (3 points), 0.1434 against
      // 0.1481 ms (6 points); FP64 keeps the held form (0.1246 ms, 5 blocks)
      if (m->et == AKB_TRIANGLE_6 && gr.law == LAW_PLASTIC && precision == AKB_PRECISION_MIXED) {
        gr.tune.minb = 7;
        gr.tune.pqs = 1;
      }
      // FP64 elastic and neohookean tetrahedra: the geometry recomputed from
      // the coordinates instead of streaming 104 bytes of dN/dx and det J w
      // per element, and the next wave's table rows prefetched into L2
      // (256-cube batch, element launch 0.835 against 0.993 ms).  Mixed
      // tetrahedra keep the streamed FP32 copies without prefetch (0.455 ms;
      // prefetching 0.476, recomputing 0.538: 80 instead of 56 registers),
      // and so do triangles (the prefetch made their launches a third longer:
      // one wave of the plastic per-point state is most of L2)
      if (m->et == AKB_TETRAHEDRON_4 && gr.law != LAW_PLASTIC &&
          precision == AKB_PRECISION_FP64) {
        gr.tune.pf = 1;
        gr.tune.rec = 1;
        // registers capped for 6 resident blocks (80 instead of 90, no
        // spill): 256-cube batch element launch 0.781-0.802 against
        // 0.836-0.865 ms
        gr.tune.minb = 6;
      }
      // plain FP64 hexahedra, neohookean and plastic: the streamed per-point
      // law (64 instead of 126 and 128 instead of 168 registers), measured on
      // B200: 128^3 neohookean element launch 1.342 against 1.572 ms, 48^3
      // plastic 0.119 against 0.199 ms; elastic keeps the form holding its
      // values in registers (1.277 against 1.316 ms streamed)
      if (m->et == AKB_HEXAHEDRON_8 && precision == AKB_PRECISION_FP64 && gr.law != LAW_ELASTIC)
        gr.tune.pqs = 1;
      gr.nmat++;
      gr.e_count += mt.e_count;
      mt.group = (int)m->groups.size() - 1;
    }
    for (int64_t e = 0; e < E; ++e) m->perm[start[m->mat_user[e]]++] = e;
  }
  // dependent launches: measured on B200 from 3k to 2M elements, 4-15 %
  // shorter steps on meshes below ~50k elements and even above, except FP64
  // hexahedra (the per-point kernel), whose 16^3 and 32^3 steps were slower
  m->pdl = !(m->et == AKB_HEXAHEDRON_8 && precision == AKB_PRECISION_FP64);
  std::vector<int64_t> iperm(E);  // user element -> internal element
  for (int64_t ie = 0; ie < E; ++ie) iperm[m->perm[ie]] = ie;
  std::vector<int32_t> conn_soa((size_t)nn * E);
  for (int64_t ie = 0; ie < E; ++ie)
    for (int a = 0; a < nn; ++a) conn_soa[(size_t)a * E + ie] = m->conn[m->perm[ie] * nn + a];
  // node -> slot CSR.  A node's slots follow the reference's scatter order of
  // the internal force: material by material in index order, ascending user
  // element inside a material (dof_manager.cc:65-120 called per material from
  // solid_mechanics_model.cc:333-370).  pos: CSR position of slot (a, e),
  // where the element kernel writes the force of its node a, so the node
  // gather reads its forces contiguously.  ent: the slots of each node in
  // the order of the lumped-mass assembly, which runs over all elements of
  // the type in user order (solid_mechanics_model_mass.cc:115-128).
  std::vector<int32_t> ptr(N + 1, 0), ent((size_t)E * nn), pos((size_t)E * nn);
  for (int64_t ie = 0; ie < E; ++ie)
    for (int a = 0; a < nn; ++a) ptr[conn_soa[(size_t)a * E + ie] + 1]++;
  for (int64_t i = 0; i < N; ++i) ptr[i + 1] += ptr[i];
  {
    std::vector<int32_t> fill(ptr.begin(), ptr.end() - 1);
    for (int k = 0; k < nm; ++k) {
      const Material &mt = m->mats[k];
      for (int64_t ie = mt.e_begin; ie < mt.e_begin + mt.e_count; ++ie)
        for (int a = 0; a < nn; ++a) pos[(size_t)a * E + ie] = fill[conn_soa[(size_t)a * E + ie]]++;
    }
    std::copy(ptr.begin(), ptr.end() - 1, fill.begin());
    for (int64_t e = 0; e < E; ++e) {
      const int64_t ie = iperm[e];
      for (int a = 0; a < nn; ++a) ent[fill[conn_soa[(size_t)a * E + ie]]++] = (int32_t)(ie * nn + a);
    }
  }

  AKB_TRY(m->alloc(&m->dX, sizeof(double) * N * d));
  AKB_TRY(m->alloc(&m->dconn, sizeof(int32_t) * E * nn));
  AKB_TRY(m->alloc(&m->dptr, sizeof(int32_t) * (N + 1)));
  AKB_TRY(m->alloc(&m->dent, sizeof(int32_t) * E * nn));
  AKB_TRY(m->alloc(&m->dpos, sizeof(int32_t) * E * nn));
  AKB_TRY(m->alloc(&m->dB, sizeof(double) * E * nq * nn * d));
  AKB_TRY(m->alloc(&m->dwJ, sizeof(double) * E * nq));
  for (double **p : {&m->dU[0], &m->dU[1], &m->dv, &m->da, &m->dfext, &m->dfint})
    AKB_TRY(m->alloc(p, sizeof(double) * N * d));
  AKB_TRY(m->alloc(&m->dmass, sizeof(double) * N));
  AKB_TRY(m->alloc(&m->dblocked, N));
  // one slot per (element, node): FP32 3D slots are padded to 4 values
  // (SlotStride); the slot array first holds the elemental lumped masses
  const size_t slot_vals = (precision == AKB_PRECISION_MIXED && d == 3) ? 4 : (size_t)d;
  const size_t re_bytes = (precision == AKB_PRECISION_MIXED ? sizeof(float) : sizeof(double)) *
                          (size_t)E * nn * slot_vals;
  AKB_TRY(m->alloc(&m->dre, std::max(re_bytes, sizeof(double) * (size_t)E * nn)));
  AKB_TRY(m->alloc(&m->dscratch, sizeof(double) * std::max<int64_t>(std::max(E, N), 1)));
  AKB_TRY(m->alloc(&m->dpartials, sizeof(double) * kReducePartials));
  AKB_TRY(m->alloc(&m->dresult, sizeof(double)));
  AKB_TRY(m->alloc(&m->dstatus, sizeof(unsigned int)));
  AKB_TRY(m->alloc(&m->dbar, kBarrierWords * sizeof(unsigned int)));
  AKB_TRY(m->alloc(&m->dbad, sizeof(unsigned long long)));
  cudaStream_t s = m->stream;
  AKB_CUDA(cudaMemcpyAsync(m->dX, m->X.data(), sizeof(double) * N * d, cudaMemcpyHostToDevice, s));
  AKB_CUDA(cudaMemcpyAsync(m->dconn, conn_soa.data(), sizeof(int32_t) * E * nn, cudaMemcpyHostToDevice, s));
  AKB_CUDA(cudaMemcpyAsync(m->dptr, ptr.data(), sizeof(int32_t) * (N + 1), cudaMemcpyHostToDevice, s));
  AKB_CUDA(cudaMemcpyAsync(m->dent, ent.data(), sizeof(int32_t) * E * nn, cudaMemcpyHostToDevice, s));
  AKB_CUDA(cudaMemcpyAsync(m->dpos, pos.data(), sizeof(int32_t) * E * nn, cudaMemcpyHostToDevice, s));
  for (double *p : {m->dU[0], m->dU[1], m->dv, m->da, m->dfext, m->dfint})
    AKB_CUDA(cudaMemsetAsync(p, 0, sizeof(double) * N * d, s));
  AKB_CUDA(cudaMemsetAsync(m->dblocked, 0, N, s));
  AKB_CUDA(cudaMemsetAsync(m->dstatus, 0, sizeof(unsigned int), s));
  AKB_CUDA(cudaMemsetAsync(m->dbad, 0xff, sizeof(unsigned long long), s));

  DevGeom g = m->geom();
  AKB_CUDA(launch_precompute(g, tab, m->dB, m->dwJ, m->dbad, s));
  unsigned long long bad = 0;
  AKB_CUDA(cudaMemcpyAsync(&bad, m->dbad, sizeof(bad), cudaMemcpyDeviceToHost, s));
  AKB_CUDA(cudaStreamSynchronize(s));
  if (bad != ~0ull) {
    const int64_t ie = (int64_t)(bad / nq);
    return fail(AKB_ENEGJAC, "Negative jacobian computed, possible problem in the element node "
                             "ordering (Quadrature Point " + std::to_string(bad % nq) + ":" +
                             std::to_string(m->perm[ie]) + ")");
  }
  // lumped mass
  double *me = (double *)m->dre;
  for (auto &mt : m->mats)
    AKB_CUDA(launch_mass_elem(g, mt.e_begin, mt.e_count, mt.rho, tab, m->dwJ, me, s));
  AKB_CUDA(launch_gather_scalar(g, me, m->dmass, s));
  // FP32 copies of dN/dx and det J w: streamed by the mixed kernels of 2D
  // elements and tetrahedra (a copy of the FP64 values, rounded once, is both
  // as fast as recomputing the geometry in FP32 and more accurate).
  // Tetrahedra keep nodes 1..3 only, rows 3..11 of the [12][E] FP64 array:
  // node 0's derivatives are minus their sum (the shape functions sum to 1)
  if (precision == AKB_PRECISION_MIXED && (d == 2 || m->et == AKB_TETRAHEDRON_4)) {
    const int64_t rows0 = m->et == AKB_TETRAHEDRON_4 ? 3 : 0;
    const int64_t nb = E * (nq * nn * d - rows0);
    AKB_TRY(m->alloc(&m->fB, sizeof(float) * nb));
    AKB_TRY(m->alloc(&m->fwJ, sizeof(float) * E * nq));
    AKB_CUDA(launch_to_float(m->dB + rows0 * E, m->fB, nb, s));
    AKB_CUDA(launch_to_float(m->dwJ, m->fwJ, E * nq, s));
  }
  // a mesh of parallelepipeds (structured and voxel meshes) runs the mixed
  // hexahedron kernel compiled for them
  if (precision == AKB_PRECISION_MIXED && m->et == AKB_HEXAHEDRON_8) {
    unsigned int *flag = reinterpret_cast<unsigned int *>(m->dscratch), h = 1;
    AKB_CUDA(launch_hex8_affine_check(g, flag, s));
    AKB_CUDA(cudaMemcpyAsync(&h, flag, sizeof(h), cudaMemcpyDeviceToHost, s));
    AKB_CUDA(cudaStreamSynchronize(s));
    m->all_affine = h == 0;
    m->affine_kernel = 0;
    // without per-point geometry the kernel fits 5 blocks per SM without
    // spilling: the fastest shape for the elastic and neohookean laws
    // (measured on the 128^3 box: 11 % and 7 % shorter launches).  Reading
    // each element's adjugate and 1/det from a table formed here, instead of
    // gathering its coordinates every step, shortens the neohookean launch
    // by a further 4 % for 40 bytes per element
    // The elastic and neohookean laws then evaluate their points as packed
    // FP32 pairs, all 8 unrolled: measured on the 128^3 box, 0.149 instead
    // of 0.167 ms (elastic, registers capped for 5 blocks) and 0.178 instead
    // of 0.196 ms (neohookean, capped for 4) against the best scalar shapes.
    // The L2 prefetch of the next wave's table rows made both launches
    // longer (0.218 against 0.184 ms neohookean, 0.171 against 0.147
    // elastic): off
    if (m->all_affine) {
      AKB_TRY(m->alloc(&m->dgeo, sizeof(float) * 10 * m->E));
      AKB_CUDA(launch_hex8_affine_geometry(g, m->dgeo, s));
      m->affine_kernel = 2;
      for (auto &gr : m->groups)
        if (gr.law == LAW_ELASTIC) gr.tune = ElemTuning{128, AKB_POINTS_PACKED | 8, 5};
        else if (gr.law == LAW_NEOHOOKEAN) gr.tune = ElemTuning{128, AKB_POINTS_PACKED | 8, 4};
    }
  }
  if (m->fast64 && m->et == AKB_HEXAHEDRON_8) {
    unsigned int *flag = reinterpret_cast<unsigned int *>(m->dscratch), h = 1;
    AKB_CUDA(launch_hex8_affine_check_fp64(g, flag, s));
    AKB_CUDA(cudaMemcpyAsync(&h, flag, sizeof(h), cudaMemcpyDeviceToHost, s));
    AKB_CUDA(cudaStreamSynchronize(s));
    if (h == 0) {
      AKB_TRY(m->alloc(&m->dgeo64, sizeof(double) * 10 * m->E));
      AKB_CUDA(launch_hex8_affine_geometry_fp64(g, m->dgeo64, s));
    }
    // 2 points per iteration, registers capped for 3 blocks per SM: measured
    // on the 128^3 box, element launch 0.417 ms (neohookean) and 0.299 ms
    // (elastic) against 0.517 and 0.396 uncapped (2 blocks of 192 registers)
    for (auto &gr : m->groups) gr.tune = ElemTuning{128, 2, 3};
    m->pdl = true;
  }
  const size_t gu_size = precision == AKB_PRECISION_MIXED ? sizeof(float) : sizeof(double);
  for (auto &mt : m->groups) {
    if (mt.law != LAW_PLASTIC) continue;
    const int64_t nqp = mt.e_count * nq, dd = (int64_t)d * d, ns = sym_comps(d);
    for (int b = 0; b < 2; ++b) {
      AKB_TRY(m->alloc(&mt.sig[b], sizeof(double) * nqp * ns));
      AKB_TRY(m->alloc(&mt.gu[b], gu_size * nqp * dd));
      AKB_TRY(m->alloc(&mt.eps[b], sizeof(double) * nqp * ns));
      AKB_TRY(m->alloc(&mt.iso[b], sizeof(double) * nqp));
      for (double *p : {mt.sig[b], mt.eps[b]})
        AKB_CUDA(cudaMemsetAsync(p, 0, sizeof(double) * std::max<int64_t>(nqp * ns, 1), s));
      AKB_CUDA(cudaMemsetAsync(mt.gu[b], 0, gu_size * std::max<int64_t>(nqp * dd, 1), s));
      AKB_CUDA(cudaMemsetAsync(mt.iso[b], 0, sizeof(double) * std::max<int64_t>(nqp, 1), s));
    }
    AKB_TRY(m->alloc(&mt.pe, sizeof(double) * nqp));
    AKB_CUDA(cudaMemsetAsync(mt.pe, 0, sizeof(double) * std::max<int64_t>(nqp, 1), s));
  }
  // plane-stress neohookean points keep their out-of-plane stretch
  for (auto &gr : m->groups) {
    bool need = false;
    for (auto &mt : m->mats) need |= mt.group == (int)(&gr - m->groups.data()) && mt.c33;
    if (!need) continue;
    const int64_t nqp = gr.e_count * nq;
    AKB_TRY(m->alloc(&gr.c33, sizeof(double) * nqp));
    AKB_CUDA(launch_fill(gr.c33, 1.0, nqp, s));
  }
  // eigen gradients: every point of a material starts from its parameter
  // (Material::updateInternalParameters, material.cc:61-71)
  for (size_t gi = 0; gi < m->groups.size(); ++gi) {
    bool need = false;
    for (auto &mt : m->mats) need |= mt.group == (int)gi && mt.has_eig;
    if (need) AKB_TRY(fill_group_eigen(m, (int)gi));
  }
  // groups of several materials read per-element parameters
  bool multi = false;
  for (auto &gr : m->groups) multi |= gr.nmat > 1;
  if (multi) {
    std::vector<MatParams> mtab(nm);
    for (int k = 0; k < nm; ++k) mtab[k] = m->mats[k].params();
    m->mtab_dsth.assign(nm, 0.);
    for (int k = 0; k < nm; ++k) m->mtab_dsth[k] = m->mats[k].dsth;
    std::vector<int32_t> mslot(E);
    for (int64_t ie = 0; ie < E; ++ie) mslot[ie] = m->mat_user[m->perm[ie]];
    AKB_TRY(m->alloc(&m->dmtab, sizeof(MatParams) * nm));
    AKB_TRY(m->alloc(&m->dmslot, sizeof(int32_t) * E));
    AKB_CUDA(cudaMemcpyAsync(m->dmtab, mtab.data(), sizeof(MatParams) * nm, cudaMemcpyHostToDevice, s));
    AKB_CUDA(cudaMemcpyAsync(m->dmslot, mslot.data(), sizeof(int32_t) * E, cudaMemcpyHostToDevice, s));
    AKB_CUDA(cudaStreamSynchronize(s));
  }
  // batch: instance of each node, per-instance time steps, element ranges
  if (m->ninst > 1) {
    const int ni = m->ninst;
    std::vector<int32_t> node_inst(N), perm32(E);
    for (int k = 0; k < ni; ++k)
      for (int64_t i = m->inst_node_off[k]; i < m->inst_node_off[k + 1]; ++i) node_inst[i] = k;
    for (int64_t ie = 0; ie < E; ++ie) perm32[ie] = (int32_t)m->perm[ie];
    AKB_TRY(m->alloc(&m->dnode_inst, sizeof(int32_t) * N));
    AKB_TRY(m->alloc(&m->dperm, sizeof(int32_t) * E));
    AKB_TRY(m->alloc(&m->dinst_dt, sizeof(double) * ni));
    AKB_TRY(m->alloc(&m->dinst_min, sizeof(double) * ni));
    AKB_TRY(m->alloc(&m->dinst_eoff, sizeof(int64_t) * (ni + 1)));
    AKB_CUDA(cudaMemcpyAsync(m->dnode_inst, node_inst.data(), sizeof(int32_t) * N, cudaMemcpyHostToDevice, s));
    AKB_CUDA(cudaMemcpyAsync(m->dperm, perm32.data(), sizeof(int32_t) * E, cudaMemcpyHostToDevice, s));
    AKB_CUDA(cudaMemcpyAsync(m->dinst_dt, m->inst_dt.data(), sizeof(double) * ni, cudaMemcpyHostToDevice, s));
    AKB_CUDA(cudaMemcpyAsync(m->dinst_eoff, m->inst_elem_off.data(), sizeof(int64_t) * (ni + 1),
                             cudaMemcpyHostToDevice, s));
    AKB_CUDA(cudaStreamSynchronize(s));
  }
  AKB_CUDA(cudaStreamSynchronize(s));
  m->initialized = true;
  return AKB_OK;
}

int akb_model_nb_materials(const akb_model *m, int *count) {
  if (!m || !count) return fail(AKB_EINVAL, "null argument");
  *count = (int)m->mats.size();
  return AKB_OK;
}

int akb_model_get_material_param(const akb_model *m, int k, const char *name, double *v) {
  if (!m || !name || !v) return fail(AKB_EINVAL, "null argument");
  if (k < 0 || k >= (int)m->mats.size()) return fail(AKB_EINVAL, "material index out of range");
  Material mt = m->mats[k];
  mt.update(m->dim);
  std::string n(name);
  if (n == "rho") *v = mt.rho;
  else if (n == "E") *v = mt.E;
  else if (n == "nu") *v = mt.nu;
  else if (n == "lambda") *v = mt.lambda;
  else if (n == "mu") *v = mt.mu;
  else if (n == "sigma_y") *v = mt.sigma_y;
  else if (n == "h") *v = mt.h;
  else if (n == "alpha") *v = mt.alpha;
  else if (n == "delta_T") *v = mt.delta_T;
  else if (n == "kapa") *v = mt.lambda + 2. / 3. * mt.mu;
  else if (n == "Plane_Stress") *v = mt.plane_stress ? 1. : 0.;
  else if (n == "finite_deformation") *v = mt.finite_deformation ? 1. : 0.;
  else return fail(AKB_EINVAL, "unknown parameter '" + n + "'");
  return AKB_OK;
}

int akb_model_get_material_name(const akb_model *m, int k, char *buf, size_t size) {
  if (!m || !buf || size == 0) return fail(AKB_EINVAL, "null argument");
  if (k < 0 || k >= (int)m->mats.size()) return fail(AKB_EINVAL, "material index out of range");
  std::snprintf(buf, size, "%s", m->mats[k].name.c_str());
  return AKB_OK;
}

int akb_model_nb_quadrature_points(const akb_model *m, int *nq) {
  if (!m || !nq) return fail(AKB_EINVAL, "null argument");
  if (!m->initialized) return fail(AKB_ESTATE, "initFull has not been called");
  *nq = m->nq;
  return AKB_OK;
}

int akb_model_get_fe_data(akb_model *m, int which, double *host, int64_t count) {
  AKB_TRY(check_model(m, true));
  const int64_t EQ = m->E * m->nq, comps = which == 0 ? (int64_t)m->nn * m->dim : 1;
  if (which != 0 && which != 1) return fail(AKB_EINVAL, "which must be 0 (dN/dx) or 1 (det J w)");
  if (count != EQ * comps) return fail(AKB_EINVAL, "count does not match the field size");
  if (!host && count > 0) return fail(AKB_EINVAL, "null host buffer");
  std::vector<double> soa((size_t)EQ * comps);
  AKB_CUDA(cudaMemcpyAsync(soa.data(), which == 0 ? m->dB : m->dwJ, sizeof(double) * soa.size(),
                           cudaMemcpyDeviceToHost, m->stream));
  AKB_CUDA(cudaStreamSynchronize(m->stream));
  for (int64_t ie = 0; ie < m->E; ++ie) {
    const int64_t ue = m->perm[ie];
    for (int q = 0; q < m->nq; ++q)
      for (int64_t c = 0; c < comps; ++c)
        host[(ue * m->nq + q) * comps + c] = soa[(size_t)(q * comps + c) * m->E + ie];
  }
  return AKB_OK;
}

int akb_model_get_stable_time_step(akb_model *m, double *dt) {
  AKB_TRY(check_model(m, true));
  if (!dt) return fail(AKB_EINVAL, "null argument");
  DevGeom g = m->geom();
  for (auto &mt : m->mats)
    AKB_CUDA(launch_element_dt(g, mt.e_begin, mt.e_count, mt.celerity(), m->u(), nullptr,
                               m->dscratch, m->stream));
  return reduce_to_host(m, m->dscratch, m->E, true, dt);
}

int akb_batch_get_stable_time_steps(akb_model *m, double *dt) {
  AKB_TRY(check_model(m, true));
  if (!dt) return fail(AKB_EINVAL, "null argument");
  if (m->ninst == 1) return akb_model_get_stable_time_step(m, dt);
  DevGeom g = m->geom();
  // per-element values in user order, then the minimum over each instance
  for (auto &mt : m->mats)
    AKB_CUDA(launch_element_dt(g, mt.e_begin, mt.e_count, mt.celerity(), m->u(), m->dperm,
                               m->dscratch, m->stream));
  AKB_CUDA(launch_segment_min(m->dscratch, m->dinst_eoff, m->ninst, m->dinst_min, m->stream));
  AKB_CUDA(cudaMemcpyAsync(dt, m->dinst_min, sizeof(double) * m->ninst, cudaMemcpyDeviceToHost,
                           m->stream));
  AKB_CUDA(cudaStreamSynchronize(m->stream));
  return AKB_OK;
}

int akb_batch_set_time_steps(akb_model *m, const double *dt) {
  AKB_TRY(check_model(m, false));
  if (!dt) return fail(AKB_EINVAL, "null argument");
  if (m->ninst == 1) return akb_model_set_time_step(m, dt[0]);
  if (m->inst_dt.empty() || !std::equal(m->inst_dt.begin(), m->inst_dt.end(), dt))
    m->predicted = false;
  m->inst_dt.assign(dt, dt + m->ninst);
  m->dt = *std::min_element(m->inst_dt.begin(), m->inst_dt.end());
  if (m->dinst_dt) {
    AKB_CUDA(cudaMemcpyAsync(m->dinst_dt, m->inst_dt.data(), sizeof(double) * m->ninst,
                             cudaMemcpyHostToDevice, m->stream));
    AKB_CUDA(cudaStreamSynchronize(m->stream));
  }
  return AKB_OK;
}

int akb_batch_get_time_steps(const akb_model *m, double *dt) {
  if (!m || !dt) return fail(AKB_EINVAL, "null argument");
  if (m->ninst == 1) {
    dt[0] = m->dt;
    return AKB_OK;
  }
  std::copy(m->inst_dt.begin(), m->inst_dt.end(), dt);
  return AKB_OK;
}

int akb_batch_set_instance_steps(akb_model *m, const int64_t *steps) {
  AKB_TRY(check_model(m, true));
  if (!m->is_batch) return fail(AKB_EINVAL, "not a batch (akb_batch_create)");
  if (!steps) return fail(AKB_EINVAL, "null argument");
  const int ni = m->ninst;
  if (!m->dinst_end) {
    // instance of each internal element, from the user order offsets
    std::vector<int32_t> einst(m->E);
    for (int64_t ie = 0; ie < m->E; ++ie) {
      const int64_t ue = m->perm[ie];
      einst[ie] = (int32_t)(std::upper_bound(m->inst_elem_off.begin(), m->inst_elem_off.end(), ue) -
                            m->inst_elem_off.begin() - 1);
    }
    AKB_TRY(m->alloc(&m->dinst_end, sizeof(int64_t) * ni));
    AKB_TRY(m->alloc(&m->dstep, sizeof(int64_t)));
    AKB_TRY(m->alloc(&m->delem_inst, sizeof(int32_t) * std::max<int64_t>(m->E, 1)));
    if (m->E > 0)
      AKB_CUDA(cudaMemcpyAsync(m->delem_inst, einst.data(), sizeof(int32_t) * m->E,
                               cudaMemcpyHostToDevice, m->stream));
    AKB_CUDA(cudaMemcpyAsync(m->dstep, &m->steps_done, sizeof(int64_t), cudaMemcpyHostToDevice,
                             m->stream));
    AKB_CUDA(cudaStreamSynchronize(m->stream));
    // captured graphs and the persistent kernel know no stopping instances
    for (auto &x : m->graphs) cudaGraphExecDestroy(x.exec);
    m->graphs.clear();
    m->inst_end.assign(ni, std::numeric_limits<int64_t>::max());
  }
  for (int k = 0; k < ni; ++k)
    if (steps[k] >= 0) m->inst_end[k] = m->steps_done + steps[k];
  AKB_CUDA(cudaMemcpyAsync(m->dinst_end, m->inst_end.data(), sizeof(int64_t) * ni,
                           cudaMemcpyHostToDevice, m->stream));
  AKB_CUDA(cudaStreamSynchronize(m->stream));
  return AKB_OK;
}

int akb_batch_instance_steps_left(const akb_model *m, int64_t *left) {
  if (!m || !left) return fail(AKB_EINVAL, "null argument");
  for (int k = 0; k < m->ninst; ++k)
    left[k] = m->inst_end.empty() ? -1 : std::max<int64_t>(0, m->inst_end[k] - m->steps_done);
  return AKB_OK;
}

int akb_batch_copy_instance_nodal(akb_model *m, int field, int k, void *host, int64_t nbytes) {
  AKB_TRY(check_model(m, true));
  if (!m->is_batch) return fail(AKB_EINVAL, "not a batch (akb_batch_create)");
  if (k < 0 || k >= m->ninst) return fail(AKB_EINVAL, "instance index out of range");
  const int64_t n0 = m->inst_node_off[k], nn = m->inst_node_off[k + 1] - n0;
  const int64_t nd = nn * m->dim;
  if (nbytes != nd * (int64_t)sizeof(double)) return fail(AKB_EINVAL, "size must be N_k*dim doubles");
  if (!host && nd > 0) return fail(AKB_EINVAL, "null host buffer");
  const double *src = nullptr;
  switch (field) {
  case AKB_DISPLACEMENT: src = m->u(); break;
  case AKB_VELOCITY: src = m->dv; break;
  case AKB_ACCELERATION: src = m->da; break;
  default: return fail(AKB_EINVAL, "field is not one of displacement, velocity, acceleration");
  }
  if (nd > 0)
    AKB_CUDA(cudaMemcpyAsync(host, src + n0 * m->dim, sizeof(double) * nd, cudaMemcpyDeviceToHost,
                             m->stream));
  return AKB_OK;
}

int akb_model_set_time_step(akb_model *m, double dt) {
  AKB_TRY(check_model(m, false));
  if (m->ninst > 1) {
    std::vector<double> all(m->ninst, dt);
    return akb_batch_set_time_steps(m, all.data());
  }
  if (dt != m->dt) m->predicted = false;
  m->dt = dt;
  return AKB_OK;
}
int akb_model_get_time_step(const akb_model *m, double *dt) {
  if (!m || !dt) return fail(AKB_EINVAL, "null argument");
  *dt = m->dt;
  return AKB_OK;
}

int akb_model_set_nodal(akb_model *m, int field, const void *host, int64_t nbytes) {
  AKB_TRY(check_model(m, true));
  const int64_t nd = nodal_doubles(m);
  if (!host && nd > 0) return fail(AKB_EINVAL, "null host buffer");
  if (field == AKB_BLOCKED_DOFS) {
    if (nbytes != nd) return fail(AKB_EINVAL, "blocked dofs: size must be N*dim bytes");
    const uint8_t *b = (const uint8_t *)host;
    std::vector<uint8_t> mask(m->N, 0);
    for (int64_t i = 0; i < m->N; ++i)
      for (int c = 0; c < m->dim; ++c)
        if (b[i * m->dim + c]) mask[i] |= (uint8_t)(1u << c);
    AKB_CUDA(cudaMemcpyAsync(m->dblocked, mask.data(), m->N, cudaMemcpyHostToDevice, m->stream));
    AKB_CUDA(cudaStreamSynchronize(m->stream));
    m->predicted = false;
    return AKB_OK;
  }
  if (nbytes != nd * (int64_t)sizeof(double)) return fail(AKB_EINVAL, "size must be N*dim doubles");
  double *dst = nullptr;
  switch (field) {
  case AKB_DISPLACEMENT:
    AKB_TRY(snapshot_u(m));
    dst = m->u();
    m->predicted = false;
    break;
  case AKB_VELOCITY: dst = m->dv; m->predicted = false; break;
  case AKB_ACCELERATION: dst = m->da; m->predicted = false; break;
  case AKB_EXTERNAL_FORCE:
    dst = m->dfext;
    m->fext_zero = all_zero_bits(host, (size_t)nd);
    break;
  default: return fail(AKB_EINVAL, "field is read-only or unknown");
  }
  AKB_CUDA(cudaMemcpyAsync(dst, host, nbytes, cudaMemcpyHostToDevice, m->stream));
  AKB_CUDA(cudaStreamSynchronize(m->stream));
  return AKB_OK;
}

int akb_model_get_nodal(akb_model *m, int field, void *host, int64_t nbytes) {
  AKB_TRY(check_model(m, true));
  const int64_t nd = nodal_doubles(m);
  if (!host && nd > 0) return fail(AKB_EINVAL, "null host buffer");
  cudaStream_t s = m->stream;
  if (field == AKB_BLOCKED_DOFS) {
    if (nbytes != nd) return fail(AKB_EINVAL, "blocked dofs: size must be N*dim bytes");
    std::vector<uint8_t> mask(m->N);
    AKB_CUDA(cudaMemcpyAsync(mask.data(), m->dblocked, m->N, cudaMemcpyDeviceToHost, s));
    AKB_CUDA(cudaStreamSynchronize(s));
    uint8_t *b = (uint8_t *)host;
    for (int64_t i = 0; i < m->N; ++i)
      for (int c = 0; c < m->dim; ++c) b[i * m->dim + c] = (mask[i] >> c) & 1;
    return AKB_OK;
  }
  if (nbytes != nd * (int64_t)sizeof(double)) return fail(AKB_EINVAL, "size must be N*dim doubles");
  double *out = (double *)host;
  switch (field) {
  case AKB_MASS: {
    std::vector<double> mass(m->N);
    AKB_CUDA(cudaMemcpyAsync(mass.data(), m->dmass, sizeof(double) * m->N, cudaMemcpyDeviceToHost, s));
    AKB_CUDA(cudaStreamSynchronize(s));
    for (int64_t i = 0; i < m->N; ++i)
      for (int c = 0; c < m->dim; ++c) out[i * m->dim + c] = mass[i];
    return AKB_OK;
  }
  case AKB_CURRENT_POSITION: {
    AKB_CUDA(cudaMemcpyAsync(out, m->u(), nbytes, cudaMemcpyDeviceToHost, s));
    AKB_CUDA(cudaStreamSynchronize(s));
    for (int64_t k = 0; k < nd; ++k) out[k] = m->X[k] + out[k];
    return AKB_OK;
  }
  default: break;
  }
  const double *src = nullptr;
  switch (field) {
  case AKB_DISPLACEMENT: src = m->u(); break;
  case AKB_VELOCITY: src = m->dv; break;
  case AKB_ACCELERATION: src = m->da; break;
  case AKB_EXTERNAL_FORCE: src = m->dfext; break;
  case AKB_INTERNAL_FORCE:
    AKB_TRY(ensure_fint(m));
    src = m->dfint;
    break;
  case AKB_PREVIOUS_DISPLACEMENT:
  case AKB_DISPLACEMENT_INCREMENT:
    if (!m->track_history)
      return fail(AKB_ESTATE, "increment tracking is off (akb_model_set_increment_tracking)");
    src = field == AKB_PREVIOUS_DISPLACEMENT ? m->dprev : m->dincr;
    break;
  default: return fail(AKB_EINVAL, "unknown nodal field");
  }
  AKB_CUDA(cudaMemcpyAsync(out, src, nbytes, cudaMemcpyDeviceToHost, s));
  AKB_CUDA(cudaStreamSynchronize(s));
  return AKB_OK;
}

int akb_model_nodal_device_pointer(akb_model *m, int field, void **p) {
  AKB_TRY(check_model(m, true));
  if (!p) return fail(AKB_EINVAL, "null argument");
  switch (field) {
  case AKB_DISPLACEMENT: *p = m->u(); break;
  case AKB_VELOCITY: *p = m->dv; break;
  case AKB_ACCELERATION: *p = m->da; break;
  case AKB_EXTERNAL_FORCE: *p = m->dfext; break;
  case AKB_INTERNAL_FORCE:
    AKB_TRY(ensure_fint(m));
    AKB_CUDA(cudaStreamSynchronize(m->stream));
    *p = m->dfint;
    break;
  case AKB_PREVIOUS_DISPLACEMENT:
  case AKB_DISPLACEMENT_INCREMENT:
    if (!m->track_history)
      return fail(AKB_ESTATE, "increment tracking is off (akb_model_set_increment_tracking)");
    *p = field == AKB_PREVIOUS_DISPLACEMENT ? m->dprev : m->dincr;
    break;
  default: return fail(AKB_EINVAL, "no device pointer for this field");
  }
  return AKB_OK;
}

int akb_model_qp_field_size(akb_model *m, int field, int k, int64_t *count) {
  AKB_TRY(check_model(m, true));
  if (!count) return fail(AKB_EINVAL, "null argument");
  if (k < 0 || k >= (int)m->mats.size()) return fail(AKB_EINVAL, "material index out of range");
  const int64_t nqp = m->mats[k].e_count * m->nq;
  switch (field) {
  case AKB_GRAD_U: case AKB_STRESS: case AKB_PIOLA_KIRCHHOFF_2: case AKB_INELASTIC_STRAIN:
  case AKB_EIGEN_GRAD_U:
    *count = nqp * m->dim * m->dim;
    return AKB_OK;
  case AKB_ISO_HARDENING: case AKB_PLASTIC_ENERGY:
    *count = nqp;
    return AKB_OK;
  default: return fail(AKB_EINVAL, "unknown quadrature-point field");
  }
}

int akb_model_get_qp_field(akb_model *m, int field, int k, double *host, int64_t count) {
  int64_t need = 0;
  AKB_TRY(akb_model_qp_field_size(m, field, k, &need));
  if (count != need) return fail(AKB_EINVAL, "count does not match the field size");
  if (!host && need > 0) return fail(AKB_EINVAL, "null host buffer");
  const Material &mt = m->mats[k];
  const int64_t nqp = mt.e_count * m->nq;
  const int dd = m->dim * m->dim;
  const double *src = nullptr;
  int comps = dd;
  int64_t ld = mt.e_count;  // row length of the device array [q][comp][ld]
  if (field == AKB_EIGEN_GRAD_U) {
    const Group &gr = m->groups[mt.group];
    if (!gr.eig) {  // never set: every point holds the (zero) parameter
      for (int64_t p = 0; p < nqp; ++p)
        for (int kk = 0; kk < dd; ++kk) host[p * dd + kk] = mt.eig[kk];
      return AKB_OK;
    }
    src = gr.eig + (mt.e_begin - gr.e_begin);
    ld = gr.e_count;
  } else if (mt.law == LAW_PLASTIC) {
    const Group &gr = m->groups[mt.group];
    const int c = m->cur;
    const int64_t off = mt.e_begin - gr.e_begin, ns = sym_comps(m->dim);
    const double *sym = nullptr;
    switch (field) {
    case AKB_GRAD_U: break;
    case AKB_STRESS: sym = gr.sig[c]; break;
    case AKB_INELASTIC_STRAIN: sym = gr.eps[c]; break;
    case AKB_ISO_HARDENING: src = gr.iso[c]; comps = 1; break;
    case AKB_PLASTIC_ENERGY: src = gr.pe; comps = 1; break;
    default: return fail(AKB_EINVAL, "field not defined for plastic_linear_isotropic_hardening");
    }
    const int64_t ne = mt.e_count;
    if (field == AKB_GRAD_U || sym) {
      // gradient rows in the storage type, or symmetric rows, then expanded
      const bool f32 = field == AKB_GRAD_U && m->precision == AKB_PRECISION_MIXED;
      const size_t es = f32 ? sizeof(float) : sizeof(double);
      const int64_t rows = (int64_t)m->nq * (field == AKB_GRAD_U ? dd : ns);
      std::vector<char> raw((size_t)(rows * ne) * es);
      const char *base = field == AKB_GRAD_U ? static_cast<const char *>(gr.gu[c])
                                             : reinterpret_cast<const char *>(sym);
      if (ne > 0)
        AKB_CUDA(cudaMemcpy2DAsync(raw.data(), es * ne, base + es * off, es * gr.e_count, es * ne,
                                   (size_t)rows, cudaMemcpyDeviceToHost, m->stream));
      AKB_CUDA(cudaStreamSynchronize(m->stream));
      auto at = [&](int64_t row, int64_t le) {
        return f32 ? (double)reinterpret_cast<const float *>(raw.data())[row * ne + le]
                   : reinterpret_cast<const double *>(raw.data())[row * ne + le];
      };
      for (int64_t le = 0; le < ne; ++le)
        for (int q = 0; q < m->nq; ++q)
          for (int kk = 0; kk < dd; ++kk) {
            const int64_t row = field == AKB_GRAD_U ? (int64_t)q * dd + kk
                                                    : (int64_t)q * ns + sym_component(m->dim, kk);
            host[(le * m->nq + q) * dd + kk] = at(row, le);
          }
      return AKB_OK;
    }
    src += off;
    ld = gr.e_count;
  } else {
    if (field != AKB_GRAD_U && field != AKB_STRESS && field != AKB_PIOLA_KIRCHHOFF_2)
      return fail(AKB_EINVAL, "field not defined for this material");
    if (field == AKB_PIOLA_KIRCHHOFF_2 && mt.law != LAW_NEOHOOKEAN)
      return fail(AKB_EINVAL, "piola_kirchhoff_2 exists only for finite deformation");
    if (field == AKB_STRESS && mt.law == LAW_NEOHOOKEAN) {
      // the Cauchy stress of a finite-deformation material is only filled
      // on dump (Material::onDump); the internal stays zero during stepping
      std::fill(host, host + need, 0.);
      return AKB_OK;
    }
    AKB_TRY(eval_qp_fields(m, mt));
    src = (field == AKB_GRAD_U) ? m->dqp_a : m->dqp_b;
  }
  std::vector<double> soa((size_t)nqp * comps);
  if (nqp > 0)
    AKB_CUDA(cudaMemcpy2DAsync(soa.data(), sizeof(double) * mt.e_count, src, sizeof(double) * ld,
                               sizeof(double) * mt.e_count, (size_t)m->nq * comps,
                               cudaMemcpyDeviceToHost, m->stream));
  AKB_CUDA(cudaStreamSynchronize(m->stream));
  // device [q][comp][ne] -> reference order [element][q][comp]
  const int64_t ne = mt.e_count;
  for (int64_t le = 0; le < ne; ++le)
    for (int q = 0; q < m->nq; ++q)
      for (int c = 0; c < comps; ++c)
        host[(le * m->nq + q) * comps + c] = soa[(size_t)(q * comps + c) * ne + le];
  return AKB_OK;
}

int akb_model_set_qp_field(akb_model *m, int field, int k, const double *host, int64_t count) {
  int64_t need = 0;
  AKB_TRY(akb_model_qp_field_size(m, field, k, &need));
  if (field != AKB_EIGEN_GRAD_U)
    return fail(AKB_EINVAL, "only eigen_grad_u can be written");
  if (count != need) return fail(AKB_EINVAL, "count does not match the field size");
  if (!host && need > 0) return fail(AKB_EINVAL, "null host buffer");
  const Material &mt = m->mats[k];
  Group &gr = m->groups[mt.group];
  if (!gr.eig) AKB_TRY(fill_group_eigen(m, mt.group));
  const int dd = m->dim * m->dim;
  const int64_t ne = mt.e_count, rows = (int64_t)m->nq * dd;
  // reference order [element][q][comp] -> device [q][comp][element]
  std::vector<double> soa((size_t)(rows * ne));
  for (int64_t le = 0; le < ne; ++le)
    for (int q = 0; q < m->nq; ++q)
      for (int c = 0; c < dd; ++c)
        soa[(size_t)((q * dd + c) * ne + le)] = host[(le * m->nq + q) * dd + c];
  if (ne > 0)
    AKB_CUDA(cudaMemcpy2DAsync(gr.eig + (mt.e_begin - gr.e_begin), sizeof(double) * gr.e_count,
                               soa.data(), sizeof(double) * ne, sizeof(double) * ne,
                               (size_t)rows, cudaMemcpyHostToDevice, m->stream));
  AKB_CUDA(cudaStreamSynchronize(m->stream));
  return AKB_OK;
}

int akb_model_solve_step(akb_model *m, int64_t nsteps) {
  AKB_TRY(check_model(m, true));
  if (nsteps < 0) return fail(AKB_EINVAL, "negative step count");
  bool any_plastic = false;
  for (auto &mt : m->mats) any_plastic |= mt.law == LAW_PLASTIC;
  // a step with a thermal term in the plastic trial stress (the first after
  // initFull or a standalone assembly of a heated material) runs eagerly
  if (nsteps > 0 && !thermal_steady(m)) {
    AKB_TRY(one_step(m, any_plastic));
    --nsteps;
    m->forces_evaluated = true;
    m->snap_valid = false;
  }
  if (nsteps > 0 && use_persistent(m)) {
    AKB_TRY(run_persistent(m, nsteps, any_plastic));
    m->forces_evaluated = true;
    m->snap_valid = false;
    return AKB_OK;
  }
  int64_t left = nsteps;
  // a step whose prediction is stale runs eagerly (it launches the predictor)
  if (left > 0 && !m->predicted) {
    AKB_TRY(one_step(m, any_plastic));
    --left;
  }
  const int64_t G = m->graph_steps;
  while (G > 0 && left >= G) {
    AKB_TRY(run_graph(m, any_plastic));
    left -= G;
  }
  for (; left > 0; --left) AKB_TRY(one_step(m, any_plastic));
  if (nsteps > 0) {
    m->forces_evaluated = true;
    m->snap_valid = false;
  }
  return AKB_OK;
}

int akb_model_prepare_graphs(akb_model *m) {
  AKB_TRY(check_model(m, true));
  if (use_persistent(m)) {  // persistent launches need no graph, only the prediction
    if (!m->predicted) AKB_TRY(predict(m));
    return AKB_OK;
  }
  if (m->graph_steps == 0) return AKB_OK;
  bool any_plastic = false;
  for (auto &mt : m->mats) any_plastic |= mt.law == LAW_PLASTIC;
  if (!m->predicted) AKB_TRY(predict(m));
  // captured, not launched: the next solve_step launches it
  return capture_graph(m, any_plastic);
}

int akb_model_stream(const akb_model *m, void **stream) {
  if (!m || !stream) return fail(AKB_EINVAL, "null argument");
  if (!m->initialized) return fail(AKB_ESTATE, "initFull has not been called");
  *stream = m->stream;
  return AKB_OK;
}

int akb_model_device_bytes(const akb_model *m, int64_t *bytes) {
  if (!m || !bytes) return fail(AKB_EINVAL, "null argument");
  *bytes = (int64_t)m->device_bytes;
  return AKB_OK;
}

int akb_estimate_device_bytes(int et, int rule, int64_t N, int64_t E, int law, int precision,
                              int64_t *bytes) {
  if (!bytes) return fail(AKB_EINVAL, "null argument");
  if (et < AKB_TETRAHEDRON_4 || et > AKB_TRIANGLE_6) return fail(AKB_EINVAL, "unknown element type");
  if (law < LAW_ELASTIC || law > LAW_PLASTIC) return fail(AKB_EINVAL, "unknown law");
  if (N < 0 || E < 0) return fail(AKB_EINVAL, "negative size");
  const int64_t nn = nodes_per_element(et), d = dim_of(et);
  QuadTable tab;
  int nq = 0;
  fill_tables(et, rule, tab, nq);
  // mirrors the allocations of akb_model_init_full (16-byte minimum each)
  auto r = [](int64_t b) { return std::max<int64_t>(b, 16); };
  int64_t t = 0;
  t += r(8 * N * d) + 3 * r(4 * E * nn) + r(4 * (N + 1));
  t += r(8 * E * nq * nn * d) + r(8 * E * nq);
  t += 6 * r(8 * N * d) + r(8 * N) + r(N);
  const int64_t slot_vals = (precision == AKB_PRECISION_MIXED && d == 3) ? 4 : d;
  const int64_t re_bytes = (precision == AKB_PRECISION_MIXED ? 4 : 8) * E * nn * slot_vals;
  t += r(std::max(re_bytes, 8 * E * nn));
  t += r(8 * std::max<int64_t>(std::max(E, N), 1)) + 8 * kReducePartials + 4 * 16;
  t += 4 * kBarrierWords;
  if (precision == AKB_PRECISION_MIXED && (d == 2 || et == AKB_TETRAHEDRON_4))
    t += r(4 * E * (nq * nn * d - (et == AKB_TETRAHEDRON_4 ? 3 : 0))) + r(4 * E * nq);
  const int64_t gs = precision == AKB_PRECISION_MIXED ? 4 : 8, ns = sym_comps((int)d);
  if (law == LAW_PLASTIC)
    t += 2 * (2 * r(8 * E * nq * ns) + r(gs * E * nq * d * d) + r(8 * E * nq)) + r(8 * E * nq);
  if (law == LAW_NEOHOOKEAN && d == 2) t += r(8 * E * nq);  // plane-stress C33
  // mixed hexahedra: the adjugate table of a mesh of parallelepipeds
  if (precision == AKB_PRECISION_MIXED && et == AKB_HEXAHEDRON_8) t += r(4 * 10 * E);
  *bytes = t;
  return AKB_OK;
}

int akb_estimate_batch_device_bytes(int et, int rule, int64_t N, int64_t E, int nb_instances,
                                    int law, int precision, int64_t *bytes) {
  AKB_TRY(akb_estimate_device_bytes(et, rule, N, E, law, precision, bytes));
  if (nb_instances < 1) return fail(AKB_EINVAL, "a batch has at least one instance");
  auto r = [](int64_t b) { return std::max<int64_t>(b, 16); };
  const int64_t ni = nb_instances;
  // instance of each node, user id and instance of each element, material
  // slot of each element; per-instance time steps, minima, element offsets,
  // stop steps; the material table and the step counter
  *bytes += r(4 * N) + 3 * r(4 * E) + 3 * r(8 * ni) + r(8 * (ni + 1)) +
            r((int64_t)sizeof(MatParams) * ni) + r(8);
  return AKB_OK;
}

int akb_model_apply_neumann_stress(akb_model *m, const int32_t *group_nodes, int64_t count,
                                   const double *stress) {
  AKB_TRY(check_model(m, true));
  const int64_t nd = nodal_doubles(m);
  std::vector<double> f(nd);
  AKB_CUDA(cudaMemcpyAsync(f.data(), m->dfext, sizeof(double) * nd, cudaMemcpyDeviceToHost,
                           m->stream));
  AKB_CUDA(cudaStreamSynchronize(m->stream));
  AKB_TRY(akb_mesh_neumann_forces(m->et, m->X.data(), m->N, m->conn.data(), m->E, group_nodes,
                                  count, stress, f.data()));
  return akb_model_set_nodal(m, AKB_EXTERNAL_FORCE, f.data(), nd * (int64_t)sizeof(double));
}

int akb_model_set_prescribed_velocity_ramp(akb_model *m, const int64_t *dofs, int64_t count,
                                           double v_max, int64_t ramp_steps) {
  AKB_TRY(check_model(m, true));
  if (m->ninst > 1) return fail(AKB_EUNSUPPORTED, "prescribed motion is not provided for batches");
  if (count < 0 || (count > 0 && !dofs)) return fail(AKB_EINVAL, "bad dof list");
  if (ramp_steps < 1) return fail(AKB_EINVAL, "ramp_steps must be >= 1");
  const int64_t nd = nodal_doubles(m);
  for (int64_t k = 0; k < count; ++k)
    if (dofs[k] < 0 || dofs[k] >= nd) return fail(AKB_EINVAL, "dof index out of range");
  cudaStream_t s = m->stream;
  AKB_CUDA(cudaStreamSynchronize(s));
  for (auto &x : m->graphs) cudaGraphExecDestroy(x.exec);
  m->graphs.clear();
  m->presc_count = 0;
  if (count == 0) return AKB_OK;
  // the dofs are blocked from now on
  std::vector<uint8_t> mask(m->N);
  AKB_CUDA(cudaMemcpyAsync(mask.data(), m->dblocked, m->N, cudaMemcpyDeviceToHost, s));
  AKB_CUDA(cudaStreamSynchronize(s));
  for (int64_t k = 0; k < count; ++k) mask[dofs[k] / m->dim] |= (uint8_t)(1u << (dofs[k] % m->dim));
  AKB_CUDA(cudaMemcpyAsync(m->dblocked, mask.data(), m->N, cudaMemcpyHostToDevice, s));
  // starting displacement of the dofs
  std::vector<double> u(nd), u0(count);
  AKB_CUDA(cudaMemcpyAsync(u.data(), m->u(), sizeof(double) * nd, cudaMemcpyDeviceToHost, s));
  AKB_CUDA(cudaStreamSynchronize(s));
  for (int64_t k = 0; k < count; ++k) u0[k] = u[dofs[k]];
  // buffers are kept for the model's lifetime; a longer list reallocates
  AKB_TRY(m->alloc(&m->dpresc_dofs, sizeof(int64_t) * count));
  AKB_TRY(m->alloc(&m->dpresc_u0, sizeof(double) * count));
  if (!m->dpresc_acc) {
    AKB_TRY(m->alloc(&m->dpresc_acc, sizeof(double)));
    AKB_TRY(m->alloc(&m->dpresc_step, sizeof(int64_t)));
  }
  AKB_CUDA(cudaMemcpyAsync(m->dpresc_dofs, dofs, sizeof(int64_t) * count, cudaMemcpyHostToDevice, s));
  AKB_CUDA(cudaMemcpyAsync(m->dpresc_u0, u0.data(), sizeof(double) * count, cudaMemcpyHostToDevice, s));
  AKB_CUDA(cudaMemsetAsync(m->dpresc_acc, 0, sizeof(double), s));
  AKB_CUDA(cudaMemsetAsync(m->dpresc_step, 0, sizeof(int64_t), s));
  AKB_CUDA(cudaStreamSynchronize(s));
  m->presc_count = count;
  m->presc_vmax = v_max;
  m->presc_ramp = ramp_steps;
  m->presc_ahead = false;
  m->predicted = false;
  return AKB_OK;
}

int akb_model_set_persistent(akb_model *m, int mode) {
  AKB_TRY(check_model(m, false));
  if (mode < 0 || mode > 2) return fail(AKB_EINVAL, "mode must be 0, 1 or 2");
  m->persistent = mode;
  return AKB_OK;
}

int akb_model_set_persistent_wait_test(akb_model *m, unsigned int spin_limit, int late_block,
                                       unsigned int late_us) {
  AKB_TRY(check_model(m, true));
  if (late_us > 1000000u) return fail(AKB_EINVAL, "late_us is at most one second");
  m->bar_spin_limit = spin_limit ? spin_limit : kBarrierSpinLimit;
  m->bar_late_block = late_block;
  m->bar_late_us = late_block >= 0 ? late_us : 0u;
  return AKB_OK;
}

int akb_model_persistent_active(const akb_model *m, int *active) {
  if (!m || !active) return fail(AKB_EINVAL, "null argument");
  if (!m->initialized) return fail(AKB_ESTATE, "initFull has not been called");
  *active = use_persistent(m) ? 1 : 0;
  return AKB_OK;
}

// the element kernels with an L2 prefetch of later warps' rows: the packed
// hexahedron kernel, and the one-thread-per-element kernel of tetrahedra
// and triangles (not its recomputed-geometry form, points_per_iteration 0)
static bool prefetching_kernel(const akb_model *m, const Group &gr) {
  if (m->et == AKB_HEXAHEDRON_8) return (gr.tune.qu & AKB_POINTS_PACKED) != 0;
  return !(m->et == AKB_TETRAHEDRON_4 && m->precision == AKB_PRECISION_MIXED && gr.tune.qu == 0);
}

int akb_model_autotune(akb_model *m, int repeats) {
  AKB_TRY(check_model(m, true));
  if (repeats < 1) return fail(AKB_EINVAL, "repeats must be >= 1");
  DevGeom g = m->geom();
  // the timed node updates write scratch outputs only: the plain kernels
  // (a stopping batch's kernel would write the model's displacement)
  g.inst_end = nullptr;
  g.step = nullptr;
  const int64_t nd = nodal_doubles(m);
  cudaStream_t s = m->stream;
  // scratch: plastic outputs of the timed element launches, and a, v, u_next
  // and the status word of the timed node updates (the model is not touched)
  int64_t state_n = 0;
  for (auto &gr : m->groups)
    if (gr.law == LAW_PLASTIC) state_n = std::max(state_n, gr.e_count * m->nq);
  const int64_t dd = (int64_t)m->dim * m->dim, ns = sym_comps(m->dim);
  double *tmp = nullptr;
  const size_t tmp_doubles = (size_t)(state_n * (2 * ns + dd + 1) + 3 * nd + 1);
  AKB_CUDA(cudaMallocAsync((void **)&tmp, sizeof(double) * tmp_doubles, s));
  double *t_sig = tmp, *t_gu = t_sig + state_n * ns, *t_eps = t_gu + state_n * dd;
  double *t_iso = t_eps + state_n * ns, *t_a = t_iso + state_n, *t_v = t_a + nd;
  double *t_u = t_v + nd;
  unsigned int *t_status = (unsigned int *)(t_u + nd);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = AKB_OK;
  auto check = [&](cudaError_t e, const char *what) {
    if (e != cudaSuccess && rc == AKB_OK)
      rc = fail(AKB_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return rc == AKB_OK;
  };
  check(cudaEventCreate(&e0), "cudaEventCreate");
  check(cudaEventCreate(&e1), "cudaEventCreate");
  auto time_it = [&](const std::function<cudaError_t()> &launch, float *ms) {
    if (!check(launch(), "autotune launch")) return false;  // warm-up
    check(cudaEventRecord(e0, s), "cudaEventRecord");
    for (int r = 0; r < repeats && rc == AKB_OK; ++r) check(launch(), "autotune launch");
    check(cudaEventRecord(e1, s), "cudaEventRecord");
    check(cudaEventSynchronize(e1), "cudaEventSynchronize");
    if (check(cudaEventElapsedTime(ms, e0, e1), "cudaEventElapsedTime")) *ms /= repeats;
    return rc == AKB_OK;
  };
  // the stress evaluations of the timed launches update C33 in place: they
  // get a copy
  int64_t c33_n = 0;
  for (auto &gr : m->groups)
    if (gr.c33) c33_n = std::max(c33_n, gr.e_count * m->nq);
  double *t_c33 = nullptr;
  if (c33_n > 0) AKB_CUDA(cudaMallocAsync((void **)&t_c33, sizeof(double) * c33_n, s));
  auto elem_launch = [&](Group &gr, const ElemTuning &tn) {
    GroupArgs ps = group_args(m, gr, false);
    if (gr.c33) ps.c33 = t_c33;
    if (gr.law == LAW_PLASTIC) {
      ps.sig = t_sig;
      ps.gu = t_gu;
      ps.eps = t_eps;
      ps.iso = t_iso;
      ps.update_energy = 0;
    }
    const MatParams mp = m->mats[gr.mat0].params();
    if (m->precision == AKB_PRECISION_MIXED)
      return launch_element_forces_mixed(g, gr.law, gr.e_begin, gr.e_count, m->tab, m->fB,
                                         m->fwJ, m->u(), mp, ps, (float *)m->dre, tn, s);
    if (m->fast64 && m->et == AKB_HEXAHEDRON_8)
      return launch_element_forces_fp64_sf(g, gr.law, gr.e_begin, gr.e_count, m->u(), mp, ps,
                                           (double *)m->dre, m->dgeo64, tn, s);
    return launch_element_forces_fp64(g, gr.law, gr.e_begin, gr.e_count, m->dB, m->dwJ,
                                      m->u(), mp, ps, (double *)m->dre, tn, m->tab, s);
  };
  for (auto &gr : m->groups) {
    if (rc != AKB_OK) break;
    if (gr.c33)
      check(cudaMemcpyAsync(t_c33, gr.c33, sizeof(double) * gr.e_count * m->nq,
                            cudaMemcpyDeviceToDevice, s), "copy");
    // threads per block only: the points per iteration of the mixed
    // hexahedron kernel change the FP32 rounding and stay as set
    std::vector<ElemTuning> cand;
    if (m->fast64 && m->et == AKB_HEXAHEDRON_8) {
      // the register cap only (points per iteration change the rounding)
      const int q = gr.tune.qu;
      cand = {{128, q, 1}};
      if (q == 2) cand.insert(cand.end(), {{128, 2, 2}, {128, 2, 3}});
    } else if (m->et == AKB_HEXAHEDRON_8 && m->precision == AKB_PRECISION_MIXED &&
        (gr.tune.qu & AKB_POINTS_PACKED)) {
      // points per iteration and register cap (every FP32 operation of the
      // packed form is explicitly rounded: the same numbers in every shape),
      // and the L2 prefetch of the shape in use
      cand = {gr.tune};
      for (int pts : {2, 4, 8})
        for (int minb : {1, 4, 5}) cand.push_back({128, AKB_POINTS_PACKED | pts, minb, 0});
      cand.push_back(gr.tune);
      cand.back().pf = gr.tune.pf ? 0 : 1;
    } else if (m->et == AKB_HEXAHEDRON_8 && m->precision == AKB_PRECISION_MIXED) {
      const int q = gr.tune.qu;
      cand = {{128, q, 1}, {128, q, 5}};
      if (q == 1 || q == 2) cand.push_back({128, q, 6});
      if (q != 1) cand.insert(cand.end(), {{64, q, 1}, {256, q, 1}});
      if (q == 2) cand.push_back({128, q, 4});
      if (q == 0) cand = {{128, 0, 1}, {64, 0, 1}, {256, 0, 1}};
    } else if (m->et == AKB_HEXAHEDRON_8 && m->precision == AKB_PRECISION_FP64) {
      // plain FP64 hexahedra: the per-point kernel with and without the
      // streamed law (the same numbers), the form in use first
      cand = {gr.tune, gr.tune};
      cand[1].pqs = !gr.tune.pqs;
    } else {
      const int q = gr.tune.qu;
      cand = {{64, q, 1}, {128, q, 1}, {256, q, 1}};
      if (gr.law == LAW_PLASTIC && m->et != AKB_HEXAHEDRON_8)
        cand.insert(cand.end(), {{128, q, 5}, {128, q, 6}, {128, q, 7}, {128, q, 8}});
      // FP64 elastic and neohookean tetrahedra: register caps of the kernel
      // with the recomputed geometry (the streamed form ignores them)
      if (gr.law != LAW_PLASTIC && m->et == AKB_TETRAHEDRON_4 &&
          m->precision == AKB_PRECISION_FP64)
        cand.insert(cand.end(), {{128, q, 6}, {128, q, 7}});
      // plastic triangles: the streamed law with each register cap
      std::vector<ElemTuning> streamed;
      if (gr.law == LAW_PLASTIC && m->et == AKB_TRIANGLE_6)
        for (int mb : {1, 5, 6, 7, 8}) {
          streamed.push_back({128, q, mb});
          streamed.back().pqs = 1;
        }
      // each with and without the L2 prefetch of the next wave's rows, and
      // (tetrahedra and triangles) with the geometry streamed or recomputed
      Group probe = gr;
      probe.tune = cand[0];
      if (prefetching_kernel(m, probe)) {
        const size_t n = cand.size();
        for (size_t k = 0; k < n; ++k) {
          cand[k].pf = 0;
          cand[k].rec = 0;
          // the 7- and 8-block caps of plastic groups: streamed tables, no prefetch
          if (cand[k].minb >= 7 && gr.law == LAW_PLASTIC) continue;
          for (int v = 1; v < 4; ++v) {
            cand.push_back(cand[k]);
            cand.back().pf = v & 1;
            cand.back().rec = v >> 1;
          }
        }
      }
      cand.insert(cand.end(), streamed.begin(), streamed.end());
      // the shape in use first (kept on ties)
      cand.insert(cand.begin(), gr.tune);
    }
    float best = 0.f;
    for (size_t k = 0; k < cand.size() && rc == AKB_OK; ++k) {
      float ms = 0.f;
      if (!time_it([&] { return elem_launch(gr, cand[k]); }, &ms)) break;
      if (k == 0 || ms < best) {
        best = ms;
        gr.tune = cand[k];
      }
    }
  }
  if (rc == AKB_OK) {
    const int flags = NU_CORRECT | NU_PREDICT | (m->fext_zero ? NU_FEXT_ZERO : 0);
    check(cudaMemcpyAsync(t_a, m->da, sizeof(double) * nd, cudaMemcpyDeviceToDevice, s), "copy");
    check(cudaMemcpyAsync(t_v, m->dv, sizeof(double) * nd, cudaMemcpyDeviceToDevice, s), "copy");
    // direct gather with 128 .. 1024 threads, staged gather with 128 .. 512,
    // state first with 128 .. 512
    const int blocks[10] = {128, 256, 512, 1024, 128, 256, 512, 128, 256, 512};
    const int forms[10] = {0, 0, 0, 0, 1, 1, 1, 2, 2, 2};
    float best = 0.f;
    for (int k = 0; k < 10 && rc == AKB_OK; ++k) {
      float ms = 0.f;
      const int form = forms[k];
      auto launch = [&]() {
        if (m->precision == AKB_PRECISION_MIXED)
          return launch_node_update_mixed(g, (const float *)m->dre, m->dfext, m->dmass,
                                          m->dblocked, m->dfint, t_a, t_v, m->u(), t_u, m->dt,
                                          flags, t_status, blocks[k], form, s);
        return launch_node_update_fp64(g, (const double *)m->dre, m->dfext, m->dmass,
                                       m->dblocked, m->dfint, t_a, t_v, m->u(), t_u, m->dt,
                                       flags, t_status, blocks[k], form, s);
      };
      if (!time_it(launch, &ms)) break;
      if (k == 0 || ms < best) {
        best = ms;
        m->node_block = blocks[k];
        m->node_form = form;
      }
    }
  }
  // dependent launch on or off: whole steps (element forces of every group,
  // node update into the scratch state) in the chosen shapes
  if (rc == AKB_OK) {
    const int flags = NU_CORRECT | NU_PREDICT | (m->fext_zero ? NU_FEXT_ZERO : 0);
    float ms[2] = {0.f, 0.f};
    for (int pdl = 0; pdl < 2 && rc == AKB_OK; ++pdl) {
      g.pdl = pdl;
      auto step = [&]() {
        cudaError_t e = cudaSuccess;
        for (int r = 0; r < 8 && e == cudaSuccess; ++r) {
          for (auto &gr : m->groups)
            if (e == cudaSuccess) e = elem_launch(gr, gr.tune);
          if (e != cudaSuccess) break;
          if (m->precision == AKB_PRECISION_MIXED)
            e = launch_node_update_mixed(g, (const float *)m->dre, m->dfext, m->dmass,
                                         m->dblocked, m->dfint, t_a, t_v, m->u(), t_u, m->dt,
                                         flags, t_status, m->node_block, m->node_form, s);
          else
            e = launch_node_update_fp64(g, (const double *)m->dre, m->dfext, m->dmass,
                                        m->dblocked, m->dfint, t_a, t_v, m->u(), t_u, m->dt,
                                        flags, t_status, m->node_block, m->node_form, s);
        }
        return e;
      };
      time_it(step, &ms[pdl]);
    }
    if (rc == AKB_OK) m->pdl = ms[1] < ms[0];
    g.pdl = m->pdl ? 1 : 0;
  }
  // the slot array again holds the forces of the current state, computed
  // with the chosen shapes
  for (auto &gr : m->groups)
    if (rc == AKB_OK) check(elem_launch(gr, gr.tune), "autotune launch");
  check(cudaStreamSynchronize(s), "cudaStreamSynchronize");
  cudaFreeAsync(tmp, s);
  if (t_c33) cudaFreeAsync(t_c33, s);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  // captured graphs hold the old launch shapes
  for (auto &x : m->graphs) cudaGraphExecDestroy(x.exec);
  m->graphs.clear();
  return rc;
}

int akb_model_set_node_shape(akb_model *m, int node_block, int staged) {
  AKB_TRY(check_model(m, true));
  if (staged < 0 || staged > 2) return fail(AKB_EINVAL, "staged must be 0, 1 or 2");
  if (staged == 1 && node_block != 128 && node_block != 256 && node_block != 512)
    return fail(AKB_EINVAL, "the staged gather runs with 128, 256 or 512 threads");
  if (node_block < 32 || node_block > 1024 || node_block % 32)
    return fail(AKB_EINVAL, "node_block must be a multiple of 32 in [32, 1024]");
  AKB_CUDA(cudaStreamSynchronize(m->stream));
  m->node_block = node_block;
  m->node_form = staged;
  for (auto &x : m->graphs) cudaGraphExecDestroy(x.exec);
  m->graphs.clear();
  return AKB_OK;
}

// halo of a partitioned mesh: the prediction of the coming step (the
// displacement its element forces read) of the listed local nodes
int akb_model_halo_pack(akb_model *m, const int32_t *idx, int64_t n, double *buf) {
  AKB_TRY(check_model(m, true));
  if (n < 0 || (n > 0 && (!idx || !buf))) return fail(AKB_EINVAL, "bad arguments");
  if (!m->predicted) AKB_TRY(predict(m));
  AKB_CUDA(launch_halo(false, m->dim, n, idx, m->u_pred(), buf, m->stream));
  return AKB_OK;
}

int akb_model_halo_unpack(akb_model *m, const int32_t *idx, int64_t n, const double *buf) {
  AKB_TRY(check_model(m, true));
  if (n < 0 || (n > 0 && (!idx || !buf))) return fail(AKB_EINVAL, "bad arguments");
  if (!m->predicted) AKB_TRY(predict(m));
  AKB_CUDA(launch_halo(true, m->dim, n, idx, m->u_pred(), const_cast<double *>(buf), m->stream));
  return AKB_OK;
}

int akb_model_set_increment_tracking(akb_model *m, int on) {
  AKB_TRY(check_model(m, true));
  AKB_CUDA(cudaStreamSynchronize(m->stream));
  if (on && !m->dprev) {
    AKB_TRY(m->alloc(&m->dprev, sizeof(double) * nodal_doubles(m)));
    AKB_TRY(m->alloc(&m->dincr, sizeof(double) * nodal_doubles(m)));
  }
  if (on && !m->track_history) {
    AKB_CUDA(cudaMemsetAsync(m->dprev, 0, sizeof(double) * nodal_doubles(m), m->stream));
    AKB_CUDA(cudaMemsetAsync(m->dincr, 0, sizeof(double) * nodal_doubles(m), m->stream));
    AKB_CUDA(cudaStreamSynchronize(m->stream));
  }
  m->track_history = on != 0;
  // captured steps hold the launches of the previous setting
  for (auto &x : m->graphs) cudaGraphExecDestroy(x.exec);
  m->graphs.clear();
  return AKB_OK;
}

int akb_model_set_affine_kernel(akb_model *m, int on) {
  AKB_TRY(check_model(m, true));
  if (on < 0 || on > 2) return fail(AKB_EINVAL, "affine kernel mode is 0, 1 or 2");
  if (on && !m->all_affine)
    return fail(AKB_EUNSUPPORTED, "the mesh is not made of parallelepipeds only (or is not a "
                                  "mixed-precision hexahedral mesh)");
  if (on == 2 && !m->dgeo) {
    AKB_TRY(m->alloc(&m->dgeo, sizeof(float) * 10 * m->E));
    AKB_CUDA(launch_hex8_affine_geometry(m->geom(), m->dgeo, m->stream));
  }
  AKB_CUDA(cudaStreamSynchronize(m->stream));
  m->affine_kernel = on;
  // the packed form exists for meshes of parallelepipeds only: without the
  // kernel compiled for them, the scalar form with the same points per
  // iteration (2 or 8; 4 becomes 2) and a register cap that does not spill
  for (auto &gr : m->groups)
    if (!on && (gr.tune.qu & AKB_POINTS_PACKED)) {
      const int pts = gr.tune.qu & 0xff;
      gr.tune = ElemTuning{128, pts == 8 ? 8 : 2, pts == 8 ? 1 : 4};
    }
  for (auto &x : m->graphs) cudaGraphExecDestroy(x.exec);
  m->graphs.clear();
  return AKB_OK;
}

int akb_model_get_affine_kernel(const akb_model *m, int *on) {
  if (!m || !on) return fail(AKB_EINVAL, "null argument");
  *on = m->affine_kernel;
  return AKB_OK;
}

int akb_model_set_dependent_launch(akb_model *m, int on) {
  AKB_TRY(check_model(m, true));
  AKB_CUDA(cudaStreamSynchronize(m->stream));
  m->pdl = on != 0;
  for (auto &x : m->graphs) cudaGraphExecDestroy(x.exec);
  m->graphs.clear();
  return AKB_OK;
}

int akb_model_get_dependent_launch(const akb_model *m, int *on) {
  if (!m || !on) return fail(AKB_EINVAL, "null argument");
  *on = m->pdl ? 1 : 0;
  return AKB_OK;
}

int akb_model_get_node_shape(const akb_model *m, int *node_block, int *staged) {
  if (!m || !node_block || !staged) return fail(AKB_EINVAL, "null argument");
  *node_block = m->node_block;
  *staged = m->node_form;
  return AKB_OK;
}

int akb_model_get_launch_shape(const akb_model *m, int law, int *element_block,
                               int *points_per_iteration, int *min_blocks, int *node_block) {
  if (!m) return fail(AKB_EINVAL, "null model");
  if (!m->initialized) return fail(AKB_ESTATE, "initFull has not been called");
  for (auto &gr : m->groups)
    if (gr.law == law) {
      if (element_block) *element_block = gr.tune.block;
      if (points_per_iteration) *points_per_iteration = gr.tune.qu;
      if (min_blocks) *min_blocks = gr.tune.minb;
      if (node_block) *node_block = m->node_block;
      return AKB_OK;
    }
  return fail(AKB_EINVAL, "no material of this law in the model");
}

int akb_model_set_launch_shape(akb_model *m, int law, int element_block,
                               int points_per_iteration, int min_blocks, int node_block) {
  AKB_TRY(check_model(m, true));
  if (element_block != 64 && element_block != 128 && element_block != 256)
    return fail(AKB_EINVAL, "element_block must be 64, 128 or 256");
  const int q = points_per_iteration;
  if (m->fast64 && m->et == AKB_HEXAHEDRON_8) {
    // the FP64 sum-factorised kernel: 128 threads, 1, 2 or 8 points per
    // iteration, registers capped for 2 or 3 blocks with 2 points
    if (element_block != 128 || (q != 1 && q != 2 && q != 8) ||
        (min_blocks != 1 && !(q == 2 && (min_blocks == 2 || min_blocks == 3))))
      return fail(AKB_EINVAL, "fast FP64 hexahedra: 128 threads, 1, 2 or 8 points per "
                              "iteration, min_blocks 1 (or 2, 3 with 2 points)");
    if (node_block < 32 || node_block > 1024 || node_block % 32)
      return fail(AKB_EINVAL, "node_block must be a multiple of 32 in [32, 1024]");
    bool found = false;
    for (auto &gr : m->groups)
      if (gr.law == law) {
        gr.tune = ElemTuning{element_block, q, min_blocks};
        found = true;
      }
    if (!found) return fail(AKB_EINVAL, "no material of this law in the model");
    m->node_block = node_block;
    AKB_CUDA(cudaStreamSynchronize(m->stream));
    for (auto &x : m->graphs) cudaGraphExecDestroy(x.exec);
    m->graphs.clear();
    return AKB_OK;
  }
  const bool sf = m->et == AKB_HEXAHEDRON_8 && m->precision == AKB_PRECISION_MIXED;
  const bool tet_mixed = m->et == AKB_TETRAHEDRON_4 && m->precision == AKB_PRECISION_MIXED;
  if (q & AKB_POINTS_PACKED) {
    // packed FP32 pairs: mixed hexahedra of a mesh of parallelepipeds with the
    // kernel compiled for them, elastic or neohookean, 128 threads
    const int pts = q & ~AKB_POINTS_PACKED;
    if (!sf || !m->affine_kernel || law == LAW_PLASTIC)
      return fail(AKB_EINVAL, "packed points need mixed hexahedra of a mesh of parallelepipeds "
                              "(affine kernel on), elastic or neohookean");
    if (pts != 2 && pts != 4 && pts != 8)
      return fail(AKB_EINVAL, "packed points per iteration must be 2, 4 or 8");
    if (element_block != 128 || (min_blocks != 1 && min_blocks != 4 && min_blocks != 5))
      return fail(AKB_EINVAL, "packed points run with 128 threads and min_blocks 1, 4 or 5");
  } else if (!sf && q != 8 && !(tet_mixed && q == 0))
    return fail(AKB_EINVAL, "points_per_iteration is 8 (or 0 for the recomputed form of mixed "
                            "tetrahedra and hexahedra)");
  if (sf && !(q & AKB_POINTS_PACKED) && q != 0 && q != 1 && q != 2 && q != 8)
    return fail(AKB_EINVAL, "points_per_iteration must be 0, 1, 2 or 8");
  if (sf && q == 1 && element_block != 128)
    return fail(AKB_EINVAL, "1 point per iteration runs with 128 threads");
  const bool capped_sf = sf && q != 0 && element_block == 128 && !(q & AKB_POINTS_PACKED) &&
                         (min_blocks == 5 || (min_blocks == 4 && q == 2) ||
                          (min_blocks == 6 && (q == 1 || q == 2)));
  const bool capped_plastic = m->et != AKB_HEXAHEDRON_8 && law == LAW_PLASTIC &&
                              min_blocks >= 5 && min_blocks <= 8 && element_block == 128;
  // FP64 elastic and neohookean tetrahedra with the recomputed geometry
  const bool capped_tet64 = m->et == AKB_TETRAHEDRON_4 && m->precision == AKB_PRECISION_FP64 &&
                            law != LAW_PLASTIC && (min_blocks == 6 || min_blocks == 7) &&
                            element_block == 128;
  if (min_blocks != 1 && !capped_sf && !capped_plastic && !capped_tet64 &&
      !(q & AKB_POINTS_PACKED))
    return fail(AKB_EINVAL, "min_blocks is 1; 5 (or 4 with 2 points per iteration, 6 with 1 or "
                            "2) for the 128-thread mixed hexahedron kernel; 5 to 8 for "
                            "128-thread plastic tetrahedra and triangles; 6 or 7 for 128-thread "
                            "FP64 elastic and neohookean tetrahedra");
  if (node_block < 32 || node_block > 1024 || node_block % 32)
    return fail(AKB_EINVAL, "node_block must be a multiple of 32 in [32, 1024]");
  bool found = false;
  for (auto &gr : m->groups)
    if (gr.law == law) {
      // the L2 prefetch and the recomputed geometry carry over where the new
      // shape's kernel has them
      const ElemTuning old = gr.tune;
      gr.tune = ElemTuning{element_block, q, min_blocks, old.pf, old.rec, old.pqs};
      // the streamed law of plastic triangles runs with 128 threads
      if (m->et == AKB_TRIANGLE_6 && element_block != 128) gr.tune.pqs = 0;
      if (!prefetching_kernel(m, gr)) gr.tune.pf = 0;
      if (!prefetching_kernel(m, gr) || m->et == AKB_HEXAHEDRON_8) gr.tune.rec = 0;
      found = true;
    }
  if (!found) return fail(AKB_EINVAL, "no material of this law in the model");
  m->node_block = node_block;
  AKB_CUDA(cudaStreamSynchronize(m->stream));
  for (auto &x : m->graphs) cudaGraphExecDestroy(x.exec);
  m->graphs.clear();
  return AKB_OK;
}

int akb_model_set_prefetch(akb_model *m, int law, int waves) {
  AKB_TRY(check_model(m, true));
  if (waves < 0 || waves > 4) return fail(AKB_EINVAL, "waves must be in [0, 4]");
  bool found = false;
  for (auto &gr : m->groups)
    if (gr.law == law) {
      if (!prefetching_kernel(m, gr) && waves != 0)
        return fail(AKB_EINVAL, "the L2 prefetch is a setting of the packed hexahedron kernel "
                                "(points_per_iteration with AKB_POINTS_PACKED) and of the "
                                "tetrahedron and triangle kernels");
      gr.tune.pf = waves;
      // a prefetching kernel replaces the streamed law of plastic triangles
      if (waves > 0 && m->et == AKB_TRIANGLE_6) gr.tune.pqs = 0;
      found = true;
    }
  if (!found) return fail(AKB_EINVAL, "no material of this law in the model");
  AKB_CUDA(cudaStreamSynchronize(m->stream));
  for (auto &x : m->graphs) cudaGraphExecDestroy(x.exec);
  m->graphs.clear();
  return AKB_OK;
}

int akb_model_set_recompute_geometry(akb_model *m, int law, int on) {
  AKB_TRY(check_model(m, true));
  if (on != 0 && on != 1) return fail(AKB_EINVAL, "on must be 0 or 1");
  bool found = false;
  for (auto &gr : m->groups)
    if (gr.law == law) {
      if (on && (m->et == AKB_HEXAHEDRON_8 || !prefetching_kernel(m, gr)))
        return fail(AKB_EINVAL, "the recomputed geometry is a setting of the tetrahedron and "
                                "triangle kernels that stream dN/dx");
      gr.tune.rec = on;
      // so does the recomputed geometry
      if (on && m->et == AKB_TRIANGLE_6) gr.tune.pqs = 0;
      found = true;
    }
  if (!found) return fail(AKB_EINVAL, "no material of this law in the model");
  AKB_CUDA(cudaStreamSynchronize(m->stream));
  for (auto &x : m->graphs) cudaGraphExecDestroy(x.exec);
  m->graphs.clear();
  return AKB_OK;
}

int akb_model_set_streamed_points(akb_model *m, int law, int on) {
  AKB_TRY(check_model(m, true));
  if (on != 0 && on != 1) return fail(AKB_EINVAL, "on must be 0 or 1");
  const bool hex64 = m->et == AKB_HEXAHEDRON_8 && m->precision == AKB_PRECISION_FP64 && !m->fast64;
  const bool tri_plastic = m->et == AKB_TRIANGLE_6 && law == LAW_PLASTIC;
  if (on && !hex64 && !tri_plastic)
    return fail(AKB_EINVAL, "the streamed law is a setting of plain FP64 hexahedra and of plastic "
                            "triangles");
  bool found = false;
  for (auto &gr : m->groups)
    if (gr.law == law) {
      if (on && tri_plastic && (gr.tune.block != 128 || gr.tune.rec))
        return fail(AKB_EINVAL, "the streamed law of plastic triangles runs with 128 threads and "
                                "the streamed dN/dx tables (recompute_geometry 0)");
      gr.tune.pqs = on;
      if (on && tri_plastic) gr.tune.pf = 0;
      found = true;
    }
  if (!found) return fail(AKB_EINVAL, "no material of this law in the model");
  AKB_CUDA(cudaStreamSynchronize(m->stream));
  for (auto &x : m->graphs) cudaGraphExecDestroy(x.exec);
  m->graphs.clear();
  return AKB_OK;
}

int akb_model_get_streamed_points(const akb_model *m, int law, int *on) {
  if (!m) return fail(AKB_EINVAL, "null model");
  if (!m->initialized) return fail(AKB_ESTATE, "initFull has not been called");
  for (auto &gr : m->groups)
    if (gr.law == law) {
      if (on) *on = gr.tune.pqs;
      return AKB_OK;
    }
  return fail(AKB_EINVAL, "no material of this law in the model");
}

int akb_model_get_recompute_geometry(const akb_model *m, int law, int *on) {
  if (!m) return fail(AKB_EINVAL, "null model");
  if (!m->initialized) return fail(AKB_ESTATE, "initFull has not been called");
  for (auto &gr : m->groups)
    if (gr.law == law) {
      if (on) *on = gr.tune.rec;
      return AKB_OK;
    }
  return fail(AKB_EINVAL, "no material of this law in the model");
}

int akb_model_get_prefetch(const akb_model *m, int law, int *waves) {
  if (!m) return fail(AKB_EINVAL, "null model");
  if (!m->initialized) return fail(AKB_ESTATE, "initFull has not been called");
  for (auto &gr : m->groups)
    if (gr.law == law) {
      if (waves) *waves = gr.tune.pf;
      return AKB_OK;
    }
  return fail(AKB_EINVAL, "no material of this law in the model");
}

int akb_model_set_stream_priority(akb_model *m, int priority) {
  AKB_TRY(check_model(m, false));
  if (m->initialized) return fail(AKB_ESTATE, "the stream priority is set before initFull");
  int least = 0, greatest = 0;
  AKB_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
  m->stream_priority = std::min(std::max(priority, greatest), least);
  m->priority_set = true;
  return AKB_OK;
}

int akb_model_set_graph_steps(akb_model *m, int64_t steps) {
  AKB_TRY(check_model(m, false));
  if (steps < 0 || steps % 2) return fail(AKB_EINVAL, "graph length must be even and >= 0");
  m->graph_steps = steps;
  return AKB_OK;
}

int akb_model_time_steps(akb_model *m, int64_t nsteps, double *ms) {
  AKB_TRY(check_model(m, true));
  if (!ms || nsteps < 0) return fail(AKB_EINVAL, "bad argument");
  cudaEvent_t e0, e1;
  AKB_CUDA(cudaEventCreate(&e0));
  AKB_CUDA(cudaEventCreate(&e1));
  AKB_CUDA(cudaEventRecord(e0, m->stream));
  int rc = akb_model_solve_step(m, nsteps);
  cudaError_t e = cudaEventRecord(e1, m->stream);
  if (e == cudaSuccess) e = cudaEventSynchronize(e1);
  float f = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&f, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != AKB_OK) return rc;
  if (e != cudaSuccess) return fail(AKB_ECUDA, std::string("timing: ") + cudaGetErrorString(e));
  *ms = f;
  return AKB_OK;
}

int akb_model_profile_steps(akb_model *m, int64_t nsteps, double *total_ms, double *phase_ms) {
  AKB_TRY(check_model(m, true));
  if (!total_ms || !phase_ms || nsteps < 1 || nsteps > 4096) return fail(AKB_EINVAL, "bad argument");
  std::vector<cudaEvent_t> ev((size_t)nsteps * 3 + 1);
  for (auto &x : ev) AKB_CUDA(cudaEventCreate(&x));
  bool any_plastic = false;
  for (auto &mt : m->mats) any_plastic |= mt.law == LAW_PLASTIC;
  int rc = AKB_OK;
  AKB_CUDA(cudaEventRecord(ev[0], m->stream));
  for (int64_t s = 0; s < nsteps && rc == AKB_OK; ++s) {
    // phases: [predictor if needed], element forces, node update (+ predictor)
    rc = one_step(m, any_plastic, ev[s * 3 + 1], ev[s * 3 + 2]);
    if (rc == AKB_OK) cudaEventRecord(ev[s * 3 + 3], m->stream);
  }
  cudaError_t e = cudaStreamSynchronize(m->stream);
  if (rc == AKB_OK && e == cudaSuccess) {
    m->forces_evaluated = true;
    m->snap_valid = false;
    phase_ms[0] = phase_ms[1] = phase_ms[2] = 0.;
    for (int64_t s = 0; s < nsteps; ++s)
      for (int p = 0; p < 3; ++p) {
        float f = 0.f;
        cudaEventElapsedTime(&f, ev[s * 3 + p], ev[s * 3 + p + 1]);
        phase_ms[p] += f;
      }
    float f = 0.f;
    cudaEventElapsedTime(&f, ev[0], ev[(size_t)nsteps * 3]);
    *total_ms = f;
  }
  for (auto &x : ev) cudaEventDestroy(x);
  if (rc != AKB_OK) return rc;
  if (e != cudaSuccess) return fail(AKB_ECUDA, std::string("profile: ") + cudaGetErrorString(e));
  return AKB_OK;
}

int akb_model_synchronize(akb_model *m) {
  AKB_TRY(check_model(m, true));
  AKB_CUDA(cudaStreamSynchronize(m->stream));
  if (m->aio.in) AKB_CUDA(cudaStreamSynchronize(m->aio.in));
  if (m->aio.out) AKB_CUDA(cudaStreamSynchronize(m->aio.out));
  return AKB_OK;
}

namespace {
int ensure_async_io(akb_model *m) {
  auto &io = m->aio;
  if (io.in) return AKB_OK;
  const size_t bytes = sizeof(double) * (size_t)std::max<int64_t>(nodal_doubles(m), 1);
  for (int k = 0; k < akb_model::AsyncIO::kIn; ++k) {
    AKB_TRY(m->alloc(&io.stage_in[k], bytes));
    for (cudaEvent_t *e : {&io.in_ready[k], &io.in_used[k]})
      AKB_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  }
  for (int k = 0; k < akb_model::AsyncIO::kOut; ++k) {
    AKB_TRY(m->alloc(&io.stage_out[k], bytes));
    for (cudaEvent_t *e : {&io.out_ready[k], &io.out_done[k]})
      AKB_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  }
  AKB_CUDA(cudaStreamSynchronize(m->stream));  // staging allocated before the copy streams use it
  AKB_CUDA(cudaStreamCreateWithFlags(&io.out, cudaStreamNonBlocking));
  AKB_CUDA(cudaStreamCreateWithFlags(&io.in, cudaStreamNonBlocking));
  return AKB_OK;
}
}  // namespace

int akb_model_set_nodal_async(akb_model *m, int field, const void *host, int64_t nbytes) {
  AKB_TRY(check_model(m, true));
  const int64_t nd = nodal_doubles(m);
  if (nbytes != nd * (int64_t)sizeof(double)) return fail(AKB_EINVAL, "size must be N*dim doubles");
  if (!host && nd > 0) return fail(AKB_EINVAL, "null host buffer");
  double *dst = nullptr;
  switch (field) {
  case AKB_DISPLACEMENT:
    AKB_TRY(snapshot_u(m));
    dst = m->u();
    m->predicted = false;
    break;
  case AKB_VELOCITY: dst = m->dv; m->predicted = false; break;
  case AKB_ACCELERATION: dst = m->da; m->predicted = false; break;
  case AKB_EXTERNAL_FORCE: dst = m->dfext; m->fext_zero = false; break;
  default: return fail(AKB_EINVAL, "field is read-only or unknown");
  }
  AKB_TRY(ensure_async_io(m));
  auto &io = m->aio;
  const int k = io.in_k;
  io.in_k ^= 1;
  // the staging buffer k is free once the step stream consumed its last upload
  AKB_CUDA(cudaStreamWaitEvent(io.in, io.in_used[k], 0));
  AKB_CUDA(cudaMemcpyAsync(io.stage_in[k], host, nbytes, cudaMemcpyHostToDevice, io.in));
  AKB_CUDA(cudaEventRecord(io.in_ready[k], io.in));
  AKB_CUDA(cudaStreamWaitEvent(m->stream, io.in_ready[k], 0));
  AKB_CUDA(cudaMemcpyAsync(dst, io.stage_in[k], nbytes, cudaMemcpyDeviceToDevice, m->stream));
  AKB_CUDA(cudaEventRecord(io.in_used[k], m->stream));
  return AKB_OK;
}

int akb_model_get_nodal_async(akb_model *m, int field, void *host, int64_t nbytes,
                              int64_t *ticket) {
  AKB_TRY(check_model(m, true));
  const int64_t nd = nodal_doubles(m);
  if (nbytes != nd * (int64_t)sizeof(double)) return fail(AKB_EINVAL, "size must be N*dim doubles");
  if (!host && nd > 0) return fail(AKB_EINVAL, "null host buffer");
  const double *src = nullptr;
  switch (field) {
  case AKB_DISPLACEMENT: src = m->u(); break;
  case AKB_VELOCITY: src = m->dv; break;
  case AKB_ACCELERATION: src = m->da; break;
  case AKB_EXTERNAL_FORCE: src = m->dfext; break;
  case AKB_INTERNAL_FORCE:
    AKB_TRY(ensure_fint(m));
    src = m->dfint;
    break;
  default: return fail(AKB_EINVAL, "field cannot be read asynchronously");
  }
  AKB_TRY(ensure_async_io(m));
  auto &io = m->aio;
  const int64_t t = io.out_tickets++;
  const int k = (int)(t % akb_model::AsyncIO::kOut);
  // snapshot on the step stream (the field's buffer is reused by later
  // steps), then the host copy on the copy stream, overlapping those steps
  AKB_CUDA(cudaStreamWaitEvent(m->stream, io.out_done[k], 0));
  AKB_CUDA(cudaMemcpyAsync(io.stage_out[k], src, nbytes, cudaMemcpyDeviceToDevice, m->stream));
  AKB_CUDA(cudaEventRecord(io.out_ready[k], m->stream));
  AKB_CUDA(cudaStreamWaitEvent(io.out, io.out_ready[k], 0));
  AKB_CUDA(cudaMemcpyAsync(host, io.stage_out[k], nbytes, cudaMemcpyDeviceToHost, io.out));
  AKB_CUDA(cudaEventRecord(io.out_done[k], io.out));
  if (ticket) *ticket = t;
  return AKB_OK;
}

int akb_model_wait_nodal_async(akb_model *m, int64_t ticket) {
  AKB_TRY(check_model(m, true));
  auto &io = m->aio;
  if (ticket < 0 || ticket >= io.out_tickets) return fail(AKB_EINVAL, "unknown ticket");
  constexpr int kOut = akb_model::AsyncIO::kOut;
  if (ticket < io.out_tickets - kOut)
    return fail(AKB_EINVAL, "ticket older than the reads in flight: use akb_model_synchronize");
  AKB_CUDA(cudaEventSynchronize(io.out_done[ticket % kOut]));
  return AKB_OK;
}

int akb_model_assemble_internal_forces(akb_model *m) {
  AKB_TRY(check_model(m, true));
  AKB_TRY(element_forces(m, false));
  AKB_TRY(node_update(m, false));
  m->forces_evaluated = true;
  m->snap_valid = false;
  AKB_CUDA(cudaStreamSynchronize(m->stream));
  return AKB_OK;
}

int akb_model_get_energy(akb_model *m, const char *id, double *value) {
  AKB_TRY(check_model(m, true));
  if (!id || !value) return fail(AKB_EINVAL, "null argument");
  std::string which(id);
  DevGeom g = m->geom();
  if (which == "kinetic") {
    AKB_CUDA(launch_ekin_terms(g, m->dv, m->dmass, m->dscratch, m->stream));
    double s = 0.;
    AKB_TRY(reduce_to_host(m, m->dscratch, m->N, false, &s));
    *value = s / 2.;
    return AKB_OK;
  }
  if (which == "external work") {
    AKB_TRY(ensure_fint(m));
    AKB_CUDA(launch_work_terms(g, m->dfext, m->dfint, m->dv, m->dblocked, m->dscratch, m->stream));
    double s = 0.;
    AKB_TRY(reduce_to_host(m, m->dscratch, m->N, false, &s));
    *value = s * m->dt;
    return AKB_OK;
  }
  if (which != "potential" && which != "plastic")
    return fail(AKB_EINVAL, "unknown energy '" + which + "'");
  const int kind = which == "plastic" ? 1 : 0;
  double total = 0.;
  for (auto &mt : m->mats) {
    if (kind == 1 && mt.law != LAW_PLASTIC) continue;
    const void *grad = nullptr;
    const double *stress = nullptr, *eps = nullptr, *pe = nullptr;
    int64_t ld = mt.e_count;
    bool grad_float = false;
    if (mt.law == LAW_PLASTIC) {
      const Group &gr = m->groups[mt.group];
      const int64_t off = mt.e_begin - gr.e_begin;
      grad_float = m->precision == AKB_PRECISION_MIXED;
      grad = grad_float ? (const void *)(static_cast<const float *>(gr.gu[m->cur]) + off)
                        : (const void *)(static_cast<const double *>(gr.gu[m->cur]) + off);
      stress = gr.sig[m->cur] + off;
      eps = gr.eps[m->cur] + off;
      pe = gr.pe + off;
      ld = gr.e_count;
    } else {
      AKB_TRY(eval_qp_fields(m, mt));
      grad = m->dqp_a;
      stress = m->dqp_b;
    }
    AKB_CUDA(launch_energy_elem(g, mt.law, kind, mt.e_begin, mt.e_count, ld, m->dwJ, grad,
                                grad_float, stress, eps, pe, mt.params(), m->dscratch,
                                m->stream));
    double s = 0.;
    AKB_TRY(reduce_to_host(m, m->dscratch, mt.e_count, false, &s));
    total += s;
  }
  *value = total;
  return AKB_OK;
}

int akb_bounds_checked(void) {
#ifdef AKB_BOUNDS_CHECK
  return 1;
#else
  return 0;
#endif
}

int akb_model_debug_write_index(akb_model *m, int which, int64_t position, int32_t value) {
#ifndef AKB_BOUNDS_CHECK
  (void)m, (void)which, (void)position, (void)value;
  return fail(AKB_EUNSUPPORTED, "index writes exist in the bounds-checking build only");
#else
  AKB_TRY(check_model(m, true));
  int32_t *arr = nullptr;
  int64_t n = 0;
  if (which == 0) {
    arr = m->dconn;
    n = m->E * m->nn;
  } else if (which == 1) {
    arr = m->dpos;
    n = m->E * m->nn;
  } else if (which == 2) {
    arr = m->dptr;
    n = m->N + 1;
  } else {
    return fail(AKB_EINVAL, "which is 0 (connectivity), 1 (slot positions) or 2 (CSR offsets)");
  }
  if (position < 0 || position >= n) return fail(AKB_EINVAL, "position out of range");
  AKB_CUDA(cudaMemcpyAsync(arr + position, &value, sizeof(int32_t), cudaMemcpyHostToDevice,
                           m->stream));
  AKB_CUDA(cudaStreamSynchronize(m->stream));
  // graphs and predictions stay valid: the kernels read the array in place
  return AKB_OK;
#endif
}

int akb_model_get_status(akb_model *m, int *flags) {
  AKB_TRY(check_model(m, true));
  if (!flags) return fail(AKB_EINVAL, "null argument");
  unsigned int st = 0;
  AKB_CUDA(cudaMemcpyAsync(&st, m->dstatus, sizeof(st), cudaMemcpyDeviceToHost, m->stream));
  AKB_CUDA(cudaMemsetAsync(m->dstatus, 0, sizeof(st), m->stream));
  AKB_CUDA(cudaStreamSynchronize(m->stream));
  *flags = (int)st;
  return AKB_OK;
}

}  // extern "C"

/* ------------------------------------------------------------------------ */
/* Halo exchange between the subdomain models of one process                */
/* ------------------------------------------------------------------------ */
// Replaces the reference's per-step ElementSynchronizer exchange
// (solid_mechanics_model.cc:333-370, _smm_stress) for subdomains that one
// process drives, on one or several GPUs.  Every step, for each directed
// link (owner -> holder): the owner's stream gathers the prediction of the
// listed nodes into the link buffer (and copies it to the holder's GPU when
// the two differ), records an event; the holder's stream waits for it and
// scatters the values into its own prediction; then every model runs its
// step on its own stream.  The subdomains' kernels overlap on the device: a
// model waits only for its own neighbors' packs.  A link's buffer is reused
// the next step only after the holder has read it (a second event).  With all
// models on one GPU, runs of graph_steps steps are captured as one CUDA graph
// (fork from a stream of the exchange into the models' streams, join back),
// so a step costs no host work at all.
namespace {

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) == cudaSuccess && prev != dev) cudaSetDevice(dev);
    else prev = -1;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

}  // namespace

struct akb_exchange {
  std::vector<akb_model *> parts;  // not owned
  struct Link {
    int from = 0, to = 0;
    int64_t n = 0;
    int32_t *send_idx = nullptr, *recv_idx = nullptr;  // on the owner's / holder's GPU
    double *send_buf = nullptr, *recv_buf = nullptr;   // the same buffer on one GPU
    cudaEvent_t packed = nullptr, consumed = nullptr;
    bool consumed_pending = false;  // `consumed` recorded since the last pack
  };
  std::vector<Link> links;
  std::vector<void *> dev_allocs;  // (device, pointer) freed at destruction
  std::vector<int> dev_of_alloc;
  int device = 0;
  bool one_device = true;
  cudaStream_t main = nullptr;
  cudaEvent_t fork = nullptr, done = nullptr;
  std::vector<cudaEvent_t> joins;
  int64_t graph_steps = 100;
  struct Graph {
    cudaGraphExec_t exec = nullptr;
    std::vector<int> ucur, cur;
    std::vector<double> dt;
    std::vector<char> fext_zero;
    int64_t steps = 0;
  };
  std::vector<Graph> graphs;
  ~akb_exchange() {
    if (main) cudaStreamSynchronize(main);
    for (auto *m : parts)
      if (m && m->stream) cudaStreamSynchronize(m->stream);
    for (auto &g : graphs) cudaGraphExecDestroy(g.exec);
    for (auto &l : links) {
      if (l.packed) cudaEventDestroy(l.packed);
      if (l.consumed) cudaEventDestroy(l.consumed);
    }
    for (size_t k = 0; k < dev_allocs.size(); ++k) {
      DeviceGuard g(dev_of_alloc[k]);
      cudaFree(dev_allocs[k]);
    }
    for (auto e : joins) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
    if (done) cudaEventDestroy(done);
    if (main) cudaStreamDestroy(main);
  }
  template <class P> int alloc(int dev, P **p, size_t bytes) {
    DeviceGuard g(dev);
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, bytes ? bytes : 16);
    if (e != cudaSuccess)
      return fail(e == cudaErrorMemoryAllocation ? AKB_ENOMEM : AKB_ECUDA,
                  std::string("cudaMalloc: ") + cudaGetErrorString(e));
    dev_allocs.push_back(q);
    dev_of_alloc.push_back(dev);
    *p = (P *)q;
    return AKB_OK;
  }
};

namespace {

bool any_plastic_of(const akb_model *m) {
  for (auto &mt : m->mats)
    if (mt.law == LAW_PLASTIC) return true;
  return false;
}

// one step of every model with its halo exchange, enqueued on the models'
// streams (inside or outside a capture)
int exchange_step(akb_exchange *x) {
  for (auto *m : x->parts) {
    DeviceGuard g(m->device);
    if (!m->predicted) AKB_TRY(predict(m));
  }
  for (auto &l : x->links) {
    akb_model *a = x->parts[l.from], *b = x->parts[l.to];
    DeviceGuard g(a->device);
    if (l.consumed_pending) AKB_CUDA(cudaStreamWaitEvent(a->stream, l.consumed, 0));
    AKB_CUDA(launch_halo(false, a->dim, l.n, l.send_idx, a->u_pred(), l.send_buf, a->stream));
    if (l.recv_buf != l.send_buf)
      AKB_CUDA(cudaMemcpyPeerAsync(l.recv_buf, b->device, l.send_buf, a->device,
                                   sizeof(double) * l.n * a->dim, a->stream));
    AKB_CUDA(cudaEventRecord(l.packed, a->stream));
  }
  for (auto &l : x->links) {
    akb_model *b = x->parts[l.to];
    DeviceGuard g(b->device);
    AKB_CUDA(cudaStreamWaitEvent(b->stream, l.packed, 0));
    AKB_CUDA(launch_halo(true, b->dim, l.n, l.recv_idx, b->u_pred(), l.recv_buf, b->stream));
    AKB_CUDA(cudaEventRecord(l.consumed, b->stream));
    l.consumed_pending = true;
  }
  for (auto *m : x->parts) {
    DeviceGuard g(m->device);
    AKB_TRY(one_step(m, any_plastic_of(m)));
  }
  return AKB_OK;
}

// graph_steps steps of every model as one graph (one GPU), captured when
// the models' parities, time steps and external-force flags are new
int exchange_graph(akb_exchange *x) {
  const size_t P = x->parts.size();
  akb_exchange::Graph *g = nullptr;
  for (auto &c : x->graphs) {
    bool same = c.steps == x->graph_steps;
    for (size_t k = 0; same && k < P; ++k) {
      const akb_model *m = x->parts[k];
      same = c.ucur[k] == m->ucur && c.cur[k] == m->cur && c.dt[k] == m->dt &&
             c.fext_zero[k] == (char)m->fext_zero;
    }
    if (same) g = &c;
  }
  DeviceGuard dg(x->device);
  if (!g) {
    akb_exchange::Graph ng;
    for (auto *m : x->parts) {
      ng.ucur.push_back(m->ucur);
      ng.cur.push_back(m->cur);
      ng.dt.push_back(m->dt);
      ng.fext_zero.push_back((char)m->fext_zero);
    }
    ng.steps = x->graph_steps;
    std::vector<int64_t> steps0(P);
    for (size_t k = 0; k < P; ++k) steps0[k] = x->parts[k]->steps_done;
    std::vector<bool> pending0;
    for (auto &l : x->links) {
      pending0.push_back(l.consumed_pending);
      l.consumed_pending = false;  // the fork orders the graph after earlier work
    }
    AKB_CUDA(cudaStreamBeginCapture(x->main, cudaStreamCaptureModeThreadLocal));
    int rc = AKB_OK;
    if (cudaEventRecord(x->fork, x->main) != cudaSuccess) rc = fail(AKB_ECUDA, "capture fork");
    for (auto *m : x->parts)
      if (rc == AKB_OK && cudaStreamWaitEvent(m->stream, x->fork, 0) != cudaSuccess)
        rc = fail(AKB_ECUDA, "capture fork");
    for (int64_t s = 0; s < x->graph_steps && rc == AKB_OK; ++s) rc = exchange_step(x);
    for (size_t k = 0; k < P && rc == AKB_OK; ++k)
      if (cudaEventRecord(x->joins[k], x->parts[k]->stream) != cudaSuccess ||
          cudaStreamWaitEvent(x->main, x->joins[k], 0) != cudaSuccess)
        rc = fail(AKB_ECUDA, "capture join");
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(x->main, &graph);
    // capturing executes nothing: the models' step state goes back
    for (size_t k = 0; k < P; ++k) {
      akb_model *m = x->parts[k];
      m->ucur = ng.ucur[k];
      m->cur = ng.cur[k];
      m->steps_done = steps0[k];
    }
    for (size_t k = 0; k < x->links.size(); ++k) x->links[k].consumed_pending = pending0[k];
    if (rc != AKB_OK || e != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      if (rc != AKB_OK) return rc;
      return fail(AKB_ECUDA, std::string("exchange capture: ") + cudaGetErrorString(e));
    }
    e = cudaGraphInstantiate(&ng.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e == cudaSuccess) e = cudaGraphUpload(ng.exec, x->main);
    if (e != cudaSuccess)
      return fail(AKB_ECUDA, std::string("exchange graph: ") + cudaGetErrorString(e));
    if (x->graphs.size() >= 8) {
      cudaGraphExecDestroy(x->graphs.front().exec);
      x->graphs.erase(x->graphs.begin());
    }
    x->graphs.push_back(std::move(ng));
    g = &x->graphs.back();
  }
  // the graph after everything enqueued on the models' streams, and their
  // later work after the graph
  for (size_t k = 0; k < P; ++k) {
    AKB_CUDA(cudaEventRecord(x->joins[k], x->parts[k]->stream));
    AKB_CUDA(cudaStreamWaitEvent(x->main, x->joins[k], 0));
  }
  AKB_CUDA(cudaGraphLaunch(g->exec, x->main));
  AKB_CUDA(cudaEventRecord(x->done, x->main));
  for (auto *m : x->parts) {
    AKB_CUDA(cudaStreamWaitEvent(m->stream, x->done, 0));
    m->steps_done += g->steps;
    m->fint_valid = false;
  }
  // the graph's last unpacks precede its end, which the models' streams wait for
  for (auto &l : x->links) l.consumed_pending = false;
  return AKB_OK;
}

bool exchange_steady(const akb_exchange *x) {
  for (auto *m : x->parts)
    if (!thermal_steady(m) || !m->predicted) return false;
  return true;
}

}  // namespace

extern "C" {

int akb_exchange_create(akb_model *const *parts, int nparts, akb_exchange **out) {
  if (!out || !parts || nparts < 1) return fail(AKB_EINVAL, "bad arguments");
  *out = nullptr;
  for (int k = 0; k < nparts; ++k) {
    AKB_TRY(check_model(parts[k], true));
    if (parts[k]->is_batch) return fail(AKB_EINVAL, "a batch cannot be a subdomain");
    if (parts[k]->dim != parts[0]->dim) return fail(AKB_EINVAL, "subdomains of different dimensions");
  }
  auto *x = new akb_exchange();
  x->parts.assign(parts, parts + nparts);
  x->device = parts[0]->device;
  for (auto *m : x->parts) x->one_device = x->one_device && m->device == x->device;
  int rc = AKB_OK;
  {
    DeviceGuard g(x->device);
    if (cudaStreamCreateWithFlags(&x->main, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&x->fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&x->done, cudaEventDisableTiming) != cudaSuccess)
      rc = fail(AKB_ECUDA, "exchange stream / events");
    x->joins.assign(nparts, nullptr);
    for (auto &e : x->joins)
      if (rc == AKB_OK && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
        rc = fail(AKB_ECUDA, "exchange events");
  }
  if (rc != AKB_OK) {
    delete x;
    return rc;
  }
  *out = x;
  return AKB_OK;
}

int akb_exchange_add_link(akb_exchange *x, int from, int to, const int32_t *send_local,
                          const int32_t *recv_local, int64_t count) {
  if (!x) return fail(AKB_EINVAL, "null exchange");
  const int P = (int)x->parts.size();
  if (from < 0 || from >= P || to < 0 || to >= P || from == to)
    return fail(AKB_EINVAL, "link ends out of range");
  if (count < 0 || (count > 0 && (!send_local || !recv_local)))
    return fail(AKB_EINVAL, "bad node lists");
  akb_model *a = x->parts[from], *b = x->parts[to];
  for (int64_t i = 0; i < count; ++i)
    if (send_local[i] < 0 || send_local[i] >= a->N || recv_local[i] < 0 || recv_local[i] >= b->N)
      return fail(AKB_EINVAL, "node list refers to a missing node");
  akb_exchange::Link l;
  l.from = from;
  l.to = to;
  l.n = count;
  const size_t bytes = sizeof(double) * (size_t)std::max<int64_t>(count * a->dim, 1);
  AKB_TRY(x->alloc(a->device, &l.send_idx, sizeof(int32_t) * std::max<int64_t>(count, 1)));
  AKB_TRY(x->alloc(b->device, &l.recv_idx, sizeof(int32_t) * std::max<int64_t>(count, 1)));
  AKB_TRY(x->alloc(a->device, &l.send_buf, bytes));
  if (a->device == b->device) {
    l.recv_buf = l.send_buf;
  } else {
    AKB_TRY(x->alloc(b->device, &l.recv_buf, bytes));
  }
  {
    DeviceGuard g(a->device);
    if (count > 0)
      AKB_CUDA(cudaMemcpy(l.send_idx, send_local, sizeof(int32_t) * count, cudaMemcpyHostToDevice));
    AKB_CUDA(cudaEventCreateWithFlags(&l.packed, cudaEventDisableTiming));
  }
  {
    DeviceGuard g(b->device);
    if (count > 0)
      AKB_CUDA(cudaMemcpy(l.recv_idx, recv_local, sizeof(int32_t) * count, cudaMemcpyHostToDevice));
    AKB_CUDA(cudaEventCreateWithFlags(&l.consumed, cudaEventDisableTiming));
  }
  x->links.push_back(l);
  for (auto &g : x->graphs) cudaGraphExecDestroy(g.exec);
  x->graphs.clear();
  return AKB_OK;
}

int akb_exchange_set_graph_steps(akb_exchange *x, int64_t steps) {
  if (!x) return fail(AKB_EINVAL, "null exchange");
  if (steps < 0 || (steps & 1)) return fail(AKB_EINVAL, "graph steps must be even and >= 0");
  x->graph_steps = steps;
  return AKB_OK;
}

int akb_exchange_solve_step(akb_exchange *x, int64_t nsteps) {
  if (!x) return fail(AKB_EINVAL, "null exchange");
  if (nsteps < 0) return fail(AKB_EINVAL, "negative step count");
  int64_t left = nsteps;
  const int64_t G = x->graph_steps;
  // steps whose models must first predict, or whose plastic trial stress
  // has a thermal term, run eagerly; then whole graphs on one GPU
  while (left > 0 && (!x->one_device || G == 0 || left < G || !exchange_steady(x))) {
    AKB_TRY(exchange_step(x));
    --left;
    if (x->one_device && G > 0 && left >= G && exchange_steady(x)) break;
  }
  while (G > 0 && left >= G && x->one_device) {
    AKB_TRY(exchange_graph(x));
    left -= G;
  }
  for (; left > 0; --left) AKB_TRY(exchange_step(x));
  if (nsteps > 0)
    for (auto *m : x->parts) {
      m->forces_evaluated = true;
      m->snap_valid = false;
    }
  return AKB_OK;
}

int akb_exchange_synchronize(akb_exchange *x) {
  if (!x) return fail(AKB_EINVAL, "null exchange");
  for (auto *m : x->parts) {
    DeviceGuard g(m->device);
    AKB_CUDA(cudaStreamSynchronize(m->stream));
  }
  DeviceGuard g(x->device);
  AKB_CUDA(cudaStreamSynchronize(x->main));
  return AKB_OK;
}

int akb_exchange_destroy(akb_exchange *x) {
  delete x;
  return AKB_OK;
}

}  // extern "C"

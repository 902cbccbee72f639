/*
 * akb_capi.h -- C ABI of the B200 explicit solid-dynamics step.
 *
 * This is the drop-in boundary for the explicit, lumped-mass, central-
 * difference time step of Akantu's SolidMechanicsModel.  Every entry point is
 * `extern "C"`, takes plain pointers and sizes, and returns an int status
 * (AKB_OK == 0).  On error, akb_last_error() returns a thread-local message.
 *
 * Each function names the reference interface it replaces (paths relative to
 * the Akantu source tree).  Host buffers are owned by the caller, device
 * memory by the library.  One model belongs to one host thread and one CUDA
 * stream; different models may be driven from different threads.  There is
 * no CPU fallback: without a usable CUDA device every compute entry point
 * fails with AKB_ECUDA.
 */
#ifndef AKB_CAPI_H_
#define AKB_CAPI_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define AKB_OK 0
#define AKB_EINVAL 1       /* bad argument (size, index, enum)                 */
#define AKB_ENOMEM 2       /* device or host allocation failed                 */
#define AKB_ECUDA 3        /* CUDA runtime error / no device                   */
#define AKB_ENEGJAC 4      /* negative Jacobian at initialisation              */
#define AKB_ENAN 5         /* non-finite value detected on the device          */
#define AKB_EPARSE 6       /* .dat or .msh syntax error                        */
#define AKB_ESTATE 7       /* call out of order (e.g. step before init)        */
#define AKB_EUNSUPPORTED 8 /* option the explicit path does not provide        */
#define AKB_EIO 9          /* file could not be read                           */
#define AKB_EMATERIAL 10   /* unknown material type / name                     */

/* ---- enumerations ------------------------------------------------------- */
/* element types, src/common/aka_element_classes_info.hh (_tetrahedron_4 ...) */
enum akb_element_type {
  AKB_TETRAHEDRON_4 = 0,
  AKB_HEXAHEDRON_8 = 1,
  AKB_TRIANGLE_6 = 2
};

/* src/model/model_solver.hh AnalysisMethod: only _explicit_lumped_mass */
enum akb_analysis_method { AKB_EXPLICIT_LUMPED_MASS = 0 };

/* arithmetic of the element kernels; nodal state is FP64 in both */
enum akb_precision {
  AKB_PRECISION_FP64 = 0,  /* plain FP64, same operation order as the CPU path */
  AKB_PRECISION_MIXED = 1, /* FP32 element math, FP64 nodal state + gather   */
  /* FP64 everywhere; hexahedra by a sum-factorised FP64 element kernel with
   * contraction allowed: not the CPU path's operation order, within 1e-12 of
   * it, faster (the plain FP64 path streams dN/dx; this one reads a
   * per-element adjugate table or recomputes the geometry) */
  AKB_PRECISION_FP64_FAST = 2
};

/* nodal arrays, src/model/solid_mechanics/solid_mechanics_model.hh:270-321 */
enum akb_nodal_field {
  AKB_DISPLACEMENT = 0,     /* double [N][dim] getDisplacement()             */
  AKB_VELOCITY = 1,         /* double [N][dim] getVelocity()                 */
  AKB_ACCELERATION = 2,     /* double [N][dim] getAcceleration()             */
  AKB_EXTERNAL_FORCE = 3,   /* double [N][dim] getExternalForce()            */
  AKB_INTERNAL_FORCE = 4,   /* double [N][dim] getInternalForce() (read only)*/
  AKB_MASS = 5,             /* double [N][dim] getMass()         (read only) */
  AKB_BLOCKED_DOFS = 6,     /* uint8  [N][dim] getBlockedDOFs()              */
  AKB_CURRENT_POSITION = 7, /* double [N][dim] getCurrentPosition() (r/o)    */
  /* displacement at the start of the last step and its change over it
   * (getPreviousDisplacement / getIncrement, solid_mechanics_model.hh:284-293);
   * read only, kept while increment tracking is on */
  AKB_PREVIOUS_DISPLACEMENT = 8,
  AKB_DISPLACEMENT_INCREMENT = 9
};

/* quadrature-point internals of one material, material-local element order,
 * src/model/solid_mechanics/material.hh getStress / getGradU / getInternal */
enum akb_qp_field {
  AKB_GRAD_U = 0,               /* [nq_m][dim*dim] column-major               */
  AKB_STRESS = 1,               /* [nq_m][dim*dim] Cauchy (small strain)      */
  AKB_PIOLA_KIRCHHOFF_2 = 2,    /* [nq_m][dim*dim] neohookean                 */
  AKB_INELASTIC_STRAIN = 3,     /* [nq_m][dim*dim] plastic                    */
  AKB_ISO_HARDENING = 4,        /* [nq_m]          plastic                    */
  AKB_PLASTIC_ENERGY = 5,       /* [nq_m]          plastic, cumulative        */
  /* [nq_m][dim*dim] eigen gradient subtracted from grad u before the law
   * (material.cc:147); initially the material's eigen_grad_u parameter at
   * every point (material.cc:61-71), writable per point */
  AKB_EIGEN_GRAD_U = 6
};

/* ---- library ------------------------------------------------------------ */
/* thread-local description of the last failed call on this thread */
const char *akb_last_error(void);
/* library version, e.g. 100 for 0.1.0 */
int akb_version(void);
/* number of CUDA devices visible to the library */
int akb_device_count(int *count);

/* selects the CUDA device used by models created afterwards on this thread */
int akb_set_device(int device);
/* page-locked host buffers, for host <-> device copies at full PCIe rate */
int akb_host_alloc(size_t bytes, void **ptr);
int akb_host_free(void *ptr);

/* ---- mesh input (src/io/mesh_io/mesh_io_msh.cc, gmsh 2.x and 4.x ASCII) -- */
typedef struct akb_mesh akb_mesh;
/* reads the nodes and the elements of `element_type` from a .msh file of
 * format 2.x, 4.0 or 4.1 (Mesh::read, src/mesh/mesh.hh:121; the reference's
 * populateReaders2 / populateReaders4); node order is the file's, elements are
 * numbered in order of appearance; the first physical tag is kept per
 * element.  Every element of any type with a physical tag (volumes, facets,
 * edges, points) adds its nodes to that physical group, named by
 * $PhysicalNames or "msh_block_<tag>" (mesh_io_msh.cc:483-529). */
int akb_mesh_read_msh(const char *path, int spatial_dimension, int element_type,
                      akb_mesh **mesh);
int akb_mesh_sizes(const akb_mesh *mesh, int64_t *nb_nodes, int64_t *nb_elements,
                   int *nodes_per_element);
/* copies nodes [N][dim], connectivity [E][n] and physical tag [E] */
int akb_mesh_copy(const akb_mesh *mesh, double *nodes, int32_t *connectivity,
                  int32_t *physical_tag);
/* physical groups of the file, in name order: name, dimension and nodes
 * (0-based node indices; any output may be null, query nb_nodes first) */
int akb_mesh_nb_groups(const akb_mesh *mesh, int *count);
int akb_mesh_group(const akb_mesh *mesh, int k, char *name, size_t name_size, int *dimension,
                   int64_t *nb_nodes, int32_t *nodes);
/* the "physical_names" element data of the read type (mesh_io_msh.cc:669-676,
 * mesh_io.cc:89-113, read by MeshDataMaterialSelector<std::string>): count =
 * the number of distinct names, -1 when the file gives none (format 2 without
 * $PhysicalNames); akb_mesh_element_names copies name k and/or, for each
 * element, the index of its name [E] */
int akb_mesh_nb_element_names(const akb_mesh *mesh, int *count);
int akb_mesh_element_names(const akb_mesh *mesh, int k, char *name, size_t name_size,
                           int32_t *name_of_element);
void akb_mesh_free(akb_mesh *mesh);

/* ---- model --------------------------------------------------------------- */
typedef struct akb_model akb_model;

/* SolidMechanicsModel(Mesh &, Int dim)  solid_mechanics_model.hh:61-64.
 * nodes [N][dim] double, connectivity [E][n] int32 (reference node order) */
int akb_model_create(int spatial_dimension, int element_type, const double *nodes,
                     int64_t nb_nodes, const int32_t *connectivity,
                     int64_t nb_elements, akb_model **model);
int akb_model_destroy(akb_model *model);

/* material sections of a .dat text (getStaticParser().parse(file),
 * src/io/parser/parser.hh:344-432); types: elastic, neohookean,
 * plastic_linear_isotropic_hardening.  Materials are appended in file order. */
int akb_model_load_materials(akb_model *model, const char *dat_text);
/* one material, params as "name = value" pairs separated by newlines or ';' */
int akb_model_add_material(akb_model *model, const char *type, const char *params);
/* element -> material index (ConstitutiveLawSelector, default all 0) */
int akb_model_set_element_materials(akb_model *model, const int32_t *material_of_element);
/* quadrature rule of _triangle_6: 0 = reference default (3 points), 1 = 6 points */
int akb_model_set_quadrature_rule(akb_model *model, int rule);

/* Model::initFull(_analysis_method = _explicit_lumped_mass)
 * src/model/model.hh:74-131, solid_mechanics_model.cc:123-232.
 * Precomputes dN/dx and det J w (AKB_ENEGJAC on an inverted element,
 * integrator_gauss_inline_impl.hh:176-195) and assembles the lumped mass. */
int akb_model_init_full(akb_model *model, int analysis_method, int precision);

int akb_model_nb_materials(const akb_model *model, int *count);
/* Material::getParam / get("E"), returns the parsed or derived value
 * (rho, E, nu, lambda, mu, sigma_y, h, alpha, delta_T) */
int akb_model_get_material_param(const akb_model *model, int material, const char *name,
                                 double *value);
int akb_model_get_material_name(const akb_model *model, int material, char *buffer,
                                size_t size);

/* precomputed element data in user element order
 * (ShapeLagrange::getShapesDerivatives, shape_lagrange.hh, and
 * IntegratorGauss::getJacobians, integrator_gauss.hh):
 * which 0: dN/dx  [E][nq][n][dim] (dN_a/dx_j at a*dim + j), which 1: det J * w [E][nq] */
int akb_model_get_fe_data(akb_model *model, int which, double *host, int64_t count);
/* number of quadrature points per element */
int akb_model_nb_quadrature_points(const akb_model *model, int *nq);

/* SolidMechanicsModel::getStableTimeStep  solid_mechanics_model.cc:423-473 */
int akb_model_get_stable_time_step(akb_model *model, double *dt);
/* Model::setTimeStep / getTimeStep */
int akb_model_set_time_step(akb_model *model, double dt);
int akb_model_get_time_step(const akb_model *model, double *dt);

/* host <-> device copies of a nodal array (the getters of
 * solid_mechanics_model.hh:270-321 return the same arrays by reference);
 * nbytes must be N*dim*sizeof(double), or N*dim for AKB_BLOCKED_DOFS */
int akb_model_set_nodal(akb_model *model, int field, const void *host, int64_t nbytes);
int akb_model_get_nodal(akb_model *model, int field, void *host, int64_t nbytes);
/* device address of a nodal array, for callers that keep data on the GPU.
 * The displacement alternates between two buffers (the step writes the next
 * step's prediction into the other one): its address is valid until the next
 * akb_model_solve_step; the other arrays keep their address. */
int akb_model_nodal_device_pointer(akb_model *model, int field, void **device_ptr);
/* asynchronous forms of set/get, for drivers that stream inputs and results
 * every step (pinned host buffers, akb_host_alloc): the copies run on two
 * copy streams of the model through device staging (two upload buffers,
 * AKB_ASYNC_READS_IN_FLIGHT read buffers), so that they overlap the steps
 * enqueued after them.  set: takes effect before the next step; the host
 * buffer may be reused once a read enqueued after that step has been waited
 * for, or after the next akb_model_synchronize (an external force set this
 * way is not tested for zero).  get: snapshots the field as of the steps
 * enqueued so far and returns a ticket; the host buffer holds it once
 * akb_model_wait_nodal_async(ticket) or akb_model_synchronize returns (only
 * the AKB_ASYNC_READS_IN_FLIGHT most recent tickets can be waited on
 * individually).  A driver that waits for each step's read one step later
 * leaves the copies of a single step to overlap the computation; waiting
 * AKB_ASYNC_READS_IN_FLIGHT - 1 steps later lets the copies of consecutive
 * steps run back to back, so that a step costs the slower of its copies and
 * its computation. */
#define AKB_ASYNC_READS_IN_FLIGHT 4
int akb_model_set_nodal_async(akb_model *model, int field, const void *host, int64_t nbytes);
int akb_model_get_nodal_async(akb_model *model, int field, void *host, int64_t nbytes,
                              int64_t *ticket);
int akb_model_wait_nodal_async(akb_model *model, int64_t ticket);

/* Material::getStress/getGradU/getInternal<Real>(id)(type): count is the
 * number of doubles (akb_model_qp_field_size) */
int akb_model_qp_field_size(akb_model *model, int field, int material, int64_t *count);
int akb_model_get_qp_field(akb_model *model, int field, int material, double *host,
                           int64_t count);
/* writes a quadrature-point internal of one material, the same layout as the
 * getter: Material::getInternal<Real>("eigen_grad_u")(type) assigned in
 * place (e.g. test_solid_mechanics_model_material_eigenstrain.cc:127-136);
 * only AKB_EIGEN_GRAD_U is writable (AKB_EINVAL otherwise) */
int akb_model_set_qp_field(akb_model *model, int field, int material, const double *host,
                           int64_t count);

/* prescribed motion on the device, for the imposed-displacement loop of a
 * driver (a velocity ramp written into the displacement before each step,
 * e.g. test_solid_mechanics_model_dynamics.cc:243-244) without a host round
 * trip per step: the dofs (node * dim + component) become blocked and,
 * before each later step k = 1, 2, ..., get
 *   u = u_set + sum_{j=1..k} dt * v_max * min(1, j / ramp_steps)
 * (u_set: their displacement at this call; the sum is accumulated in that
 * order).  count == 0 removes the motion (the dofs stay blocked).  Not
 * available for batches. */
int akb_model_set_prescribed_velocity_ramp(akb_model *model, const int64_t *dofs,
                                           int64_t count, double v_max, int64_t ramp_steps);
/* BC::Neumann::FromHigherDim(stress) on a node group (boundary_condition_tmpl.hh:100-164):
 * the traction stress * n is integrated over every boundary facet whose nodes
 * all belong to the group (n the outward normal) and added to forces
 * [N][dim] (host arithmetic, no device needed).  stress: dim x dim,
 * column-major. */
int akb_mesh_neumann_forces(int element_type, const double *nodes, int64_t nb_nodes,
                            const int32_t *connectivity, int64_t nb_elements,
                            const int32_t *group_nodes, int64_t count, const double *stress,
                            double *forces);
/* the same added to the model's external force */
int akb_model_apply_neumann_stress(akb_model *model, const int32_t *group_nodes, int64_t count,
                                   const double *stress);

/* ---- one mesh over several GPUs ----------------------------------------------
 * Replaces the reference's distributed mesh (MeshPartitionScotch,
 * mesh_partition_scotch.cc; ElementSynchronizer with the _smm_stress exchange,
 * solid_mechanics_model.cc:333-370).  akb_partition_elements splits the
 * elements by recursive coordinate bisection of their centroids (part[E],
 * balanced counts, deterministic).  A node belongs to the lowest part among
 * its elements; rank r's subdomain holds every element with a node r owns
 * (a ghost layer evaluated redundantly) and every node of those elements,
 * owned nodes first, then ghosts, each in ascending global order; elements in
 * ascending global order.  Each owned node then sums the same slots in the
 * same order as the whole mesh on one GPU, so a partitioned run is
 * bit-identical to it when ghost nodes are blocked and, after every step,
 * receive their owner's prediction: akb_model_halo_pack (the prediction of
 * the coming step of the listed local nodes into buf[n][dim], device
 * pointers, on the model's stream) on the owner, akb_model_halo_unpack on the
 * holder.  Neighbor k's send list of rank r and receive list of the neighbor
 * name the same global nodes in the same order. */
int akb_partition_elements(int element_type, const double *nodes, int64_t nb_nodes,
                           const int32_t *connectivity, int64_t nb_elements, int nparts,
                           int32_t *part);
typedef struct akb_subdomain akb_subdomain;
int akb_subdomain_create(int element_type, const double *nodes, int64_t nb_nodes,
                         const int32_t *connectivity, int64_t nb_elements, const int32_t *part,
                         int nparts, int rank, akb_subdomain **out);
int akb_subdomain_sizes(const akb_subdomain *sd, int64_t *nb_local_nodes, int64_t *nb_owned_nodes,
                        int64_t *nb_local_elements, int *nb_neighbors);
/* local nodes [n_local][dim], local connectivity [e_local][nodes per element]
 * (local ids), and the global id of each local node and element; any output
 * may be null */
int akb_subdomain_mesh(const akb_subdomain *sd, double *nodes, int32_t *connectivity,
                       int64_t *node_global, int64_t *element_global);
int akb_subdomain_neighbor(const akb_subdomain *sd, int k, int *rank, int64_t *nb_send,
                           int64_t *nb_recv);
int akb_subdomain_lists(const akb_subdomain *sd, int k, int32_t *send_local,
                        int32_t *recv_local);
void akb_subdomain_destroy(akb_subdomain *sd);
int akb_model_halo_pack(akb_model *model, const int32_t *local_nodes, int64_t count, double *buf);
int akb_model_halo_unpack(akb_model *model, const int32_t *local_nodes, int64_t count,
                          const double *buf);
/* The per-step halo exchange of subdomain models driven by one process
 * (replaces the reference's ElementSynchronizer _smm_stress exchange,
 * solid_mechanics_model.cc:333-370): the models, initialised with their
 * ghost nodes blocked, are advanced together; every step each link gathers
 * the owner's prediction of its send list (akb_subdomain_lists) and scatters
 * it into the holder's prediction of its receive list, on the models' streams
 * ordered by events (peer copies between GPUs), the subdomains' kernels
 * overlapping on the device.  With all models on one GPU, runs of
 * graph_steps (even, default 100) steps are captured as one CUDA graph.  The
 * models are not owned and must outlive the exchange; while it is in use,
 * step them only through it.  Bit-identical to the whole mesh on one model. */
typedef struct akb_exchange akb_exchange;
int akb_exchange_create(akb_model *const *models, int nb_models, akb_exchange **out);
/* owner `from` sends the prediction of its local nodes send_local[count] to
 * model `to`, which writes it to its local nodes recv_local[count] (host
 * arrays, copied) */
int akb_exchange_add_link(akb_exchange *exchange, int from, int to, const int32_t *send_local,
                          const int32_t *recv_local, int64_t count);
int akb_exchange_set_graph_steps(akb_exchange *exchange, int64_t steps);
/* enqueues nsteps steps of every model (asynchronous) */
int akb_exchange_solve_step(akb_exchange *exchange, int64_t nsteps);
int akb_exchange_synchronize(akb_exchange *exchange);
int akb_exchange_destroy(akb_exchange *exchange);

/* ModelSolver::solveStep  model_solver.cc:267-280: enqueues nsteps explicit
 * steps on the model's stream (asynchronous; getters synchronise) */
int akb_model_solve_step(akb_model *model, int64_t nsteps);
/* runs of solve_step are issued as CUDA graphs of `steps` steps (even; 0 =
 * plain launches; default 100).  A graph is captured once per (buffer
 * parity, dt, zero external force) and replayed; steps that follow a host
 * edit of u, v, a, the blocked dofs or dt run eagerly first. */
int akb_model_set_graph_steps(akb_model *model, int64_t steps);
/* priority of the model's CUDA stream (cudaStreamCreateWithPriority; lower
 * numbers run first, clamped to the device's range), before initFull; the
 * serving loop gives short solves the higher priority */
int akb_model_set_stream_priority(akb_model *model, int priority);
/* persistent multi-step kernel: a model of one law group runs a whole
 * solve_step in one cooperative launch (all blocks resident, grid barriers
 * between the element and node phases, bounded waits reported in bit 1 of
 * the status word), with the arithmetic of the two-kernel step.  mode 0
 * (default): never -- on B200 the 100-step graphs of the two-kernel step
 * measured faster at every mesh size (6k to 1.6M elements); 1: meshes of at
 * most 2^18 elements; 2: whenever the model allows it.  Not used with a
 * prescribed motion or several constitutive laws. */
int akb_model_set_persistent(akb_model *model, int mode);
/* Failure path of the persistent kernel's grid barrier, for tests: every
 * wait of the barrier gives up after spin_limit sleeps of about 32 ns (0: the
 * default bound, about a second), sets bit 1 of the status word
 * (akb_model_get_status) and ends the launch; block late_block (>= 0; -1:
 * none) first sleeps late_us microseconds (at most 10^6), so that a short
 * bound runs out.  The state of a launch that gave up is not a step's. */
int akb_model_set_persistent_wait_test(akb_model *model, unsigned int spin_limit,
                                       int late_block, unsigned int late_us);
int akb_model_persistent_active(const akb_model *model, int *active);
/* autotuner: times the candidate launch shapes of each law group's
 * element-force kernel (threads per block 64 / 128 / 256; for mixed
 * hexahedra also a register cap for 5 resident blocks of 128; the L2
 * prefetch; for tetrahedra and triangles the recomputed geometry) and of the node
 * update (direct gather with 128 .. 1024 threads per block, staged gather
 * with 128 .. 512) on the model's current state,
 * `repeats` launches each, and keeps the fastest.  The candidates compute
 * the same numbers, so the choice changes only the timing; the model's state
 * is not modified.  Captured step graphs are rebuilt.  The points per
 * iteration of the mixed hexahedron kernel (set_launch_shape) are not tuned:
 * they change the FP32 rounding; those of its packed form
 * (AKB_POINTS_PACKED), whose every operation is explicitly rounded, are. */
int akb_model_autotune(akb_model *model, int repeats);
/* the launch shape in use for the law group of `law` (0 elastic, 1
 * neohookean, 2 plastic); points_per_iteration is 8 except for mixed
 * hexahedra, where 0 selects the dN/dx form of the kernel instead of the
 * sum-factorised one (not bit-identical to it: a different FP32 evaluation);
 * min_blocks is 1 except for 128-thread kernels that cap their registers
 * for that many resident blocks per SM: 5 for the mixed hexahedron kernel
 * (4 with 2 points per iteration, 6 with 1 or 2), 5 or 6 for plastic
 * tetrahedra and triangles (same results) */
/* flag of points_per_iteration (mixed hexahedra of a mesh of parallelepipeds,
 * elastic or neohookean, 128 threads, min_blocks 1, 4 or 5): the Gauss
 * points are evaluated as packed FP32 pairs, 2, 4 or 8 points per iteration
 * (e.g. AKB_POINTS_PACKED | 2); a different FP32 evaluation order again */
#define AKB_POINTS_PACKED 256
/* L2 prefetch of the packed hexahedron kernel (points_per_iteration with
 * AKB_POINTS_PACKED): each warp prefetches into L2 the connectivity,
 * slot-position and adjugate rows that the warp `waves` waves of resident
 * blocks further on reads (0: none; at most 4).  The results do not depend
 * on it; the autotuner also tries 0, 1 and 2.  Captured step graphs are
 * rebuilt.  No reference counterpart (a launch setting of this library). */
int akb_model_set_prefetch(akb_model *model, int law, int waves);
int akb_model_get_prefetch(const akb_model *model, int law, int *waves);
/* geometry of the tetrahedron and triangle element kernels (one thread per
 * element): 0 streams the precomputed dN/dx and det J w every step (FP32
 * copies on the mixed path), 1 recomputes them from the nodal coordinates
 * with the precomputation's own FP64 arithmetic (explicitly rounded, then
 * rounded to FP32 on the mixed path), reading the coordinates instead of the
 * tables.  The same numbers either way; the autotuner tries both.  Not for
 * hexahedra, nor for the FP32 recomputed form of mixed tetrahedra
 * (points_per_iteration 0).  No reference counterpart (a launch setting of
 * this library; the reference precomputes, fe_engine_template_tmpl.hh). */
int akb_model_set_recompute_geometry(akb_model *model, int law, int on);
int akb_model_get_recompute_geometry(const akb_model *model, int law, int *on);
/* streamed form of an element kernel, for plain FP64 hexahedra and for
 * plastic triangles.  Plain FP64 hexahedra (one thread per Gauss point): 1
 * (the default of the neohookean and plastic laws; elastic 0) evaluates the
 * law streamed, each point's dN/dx row loaded node by node where the
 * gradient and the force read it and every force component written to
 * shared memory as soon as it is formed, which needs about half the
 * registers; 0 holds the point's row and forces in registers.  Plastic
 * triangles (one thread per element, 128 threads, the streamed dN/dx
 * tables): 1 gathers the displacements again for each point, loads dN/dx
 * where used and keeps the element's force sum in shared memory, so that
 * less stays in registers across the FP64 radial return; setting the L2
 * prefetch or the recomputed geometry turns it off.  The same operations in
 * the same order either way (bit-identical); the autotuner tries both.  No
 * reference counterpart (a launch setting of this library). */
int akb_model_set_streamed_points(akb_model *model, int law, int on);
int akb_model_get_streamed_points(const akb_model *model, int law, int *on);
int akb_model_get_launch_shape(const akb_model *model, int law, int *element_block,
                               int *points_per_iteration, int *min_blocks, int *node_block);
int akb_model_set_launch_shape(akb_model *model, int law, int element_block,
                               int points_per_iteration, int min_blocks, int node_block);
/* node update shape: threads per block, and its form: staged = 1 stages
 * each block's slot range through shared memory (coalesced loads; 128, 256
 * or 512 threads); staged = 2 keeps the direct gather but reads each node's
 * slot range, mass and blocked flags before the wait on the preceding kernel
 * and its state (a, v, u, f_ext) before the gather; 0 the direct gather.
 * Every form sums every node's slots in the same order. */
int akb_model_set_node_shape(akb_model *model, int node_block, int staged);
int akb_model_get_node_shape(const akb_model *model, int *node_block, int *staged);
/* TimeStepSolverDefault::predictor / corrector bookkeeping
 * (time_step_solver_default.cc:171-221): with tracking on, every step also
 * stores the displacement it starts from (AKB_PREVIOUS_DISPLACEMENT) and
 * u_{n+1} - u_n (AKB_DISPLACEMENT_INCREMENT), both FP64, one extra launch per
 * step; off (the default) the step does neither and those fields are not
 * available (AKB_ESTATE).  Turning it on zeroes both arrays. */
int akb_model_set_increment_tracking(akb_model *model, int on);
/* mixed-precision hexahedra: a mesh made of parallelepipeds only (found at
 * init_full; structured and voxel meshes) runs an element kernel compiled
 * without per-point geometry, which needs fewer registers (on = 1); on = 2
 * also forms each element's Jacobian adjugate and 1/det once, into a table
 * of 40 bytes per element that the kernel streams instead of gathering the
 * element's coordinates every step; on = 0 returns to the general kernel.
 * All three compute the same numbers.  AKB_EUNSUPPORTED for other meshes. */
int akb_model_set_affine_kernel(akb_model *model, int on);
int akb_model_get_affine_kernel(const akb_model *model, int *on);
/* on = 1 launches the step kernels with programmatic stream serialization:
 * a kernel is scheduled while the previous one drains and waits for its
 * completion on the device before touching memory, which hides part of the
 * launch gap on small meshes.  Results do not change. */
int akb_model_set_dependent_launch(akb_model *model, int on);
int akb_model_get_dependent_launch(const akb_model *model, int *on);
/* captures the graph that the next solve_step will launch (and enqueues the
 * predictor it starts from), so that the capture cost is not paid inside the
 * first solve_step; optional */
int akb_model_prepare_graphs(akb_model *model);
/* the model's CUDA stream (a cudaStream_t), for callers that order their own
 * work after the model's: every model call enqueues on it */
int akb_model_stream(const akb_model *model, void **stream);
/* device memory held by the model (bytes allocated so far) */
int akb_model_device_bytes(const akb_model *model, int64_t *bytes);
/* upper bound of the device memory akb_model_init_full allocates for a mesh
 * of one material of law `law` (0 elastic, 1 neohookean, 2 plastic); used
 * for admission by memory footprint */
int akb_estimate_device_bytes(int element_type, int quadrature_rule, int64_t nb_nodes,
                              int64_t nb_elements, int law, int precision, int64_t *bytes);
/* the same for a batch of nb_instances meshes with N nodes and E elements in
 * all, one material per instance, instances stopping after their own step
 * counts (akb_batch_set_instance_steps) */
int akb_estimate_batch_device_bytes(int element_type, int quadrature_rule, int64_t nb_nodes,
                                    int64_t nb_elements, int nb_instances, int law,
                                    int precision, int64_t *bytes);
int akb_model_synchronize(akb_model *model);
/* SolidMechanicsModel::assembleInternalForces  solid_mechanics_model.cc:333-370 */
int akb_model_assemble_internal_forces(akb_model *model);
/* SolidMechanicsModel::getEnergy("kinetic" | "potential" | "external work" |
 * "plastic")  solid_mechanics_model.cc:601-621 */
int akb_model_get_energy(akb_model *model, const char *energy_id, double *value);
/* timing on the device: enqueues nsteps steps between two CUDA events
 * recorded on the model's stream and returns the elapsed milliseconds */
int akb_model_time_steps(akb_model *model, int64_t nsteps, double *elapsed_ms);
/* the same with an event between the phases of every step; phase_ms[0..2]
 * receive the summed durations of the standalone predictor (only run when the
 * host changed u, v, a, the blocked dofs or dt since the last step), element
 * forces (all materials) and node update (gather, corrector and the next
 * step's predictor); nsteps <= 4096 */
int akb_model_profile_steps(akb_model *model, int64_t nsteps, double *total_ms,
                            double *phase_ms);
/* device status word: bit 0 = non-finite acceleration seen since the last
 * call, bit 1 = a grid barrier of the persistent kernel timed out (the
 * launch stopped early); the word is cleared by reading it */
int akb_model_get_status(akb_model *model, int *flags);

/* ---- batches of independent meshes --------------------------------------- */
/* A batch is a model whose mesh is the disjoint union of nb_instances
 * independent meshes of one element type (no reference counterpart: the
 * reference advances one SolidMechanicsModel per mesh).  Every model entry
 * point applies to it; the nodal arrays are the instances' arrays one after
 * the other (akb_batch_instance_offsets).  Each step advances all instances
 * with one element-force launch per constitutive law and one node-update
 * launch, each instance with its own time step; the result of an instance is
 * the result of the same mesh run alone (same kernels, same summation order).
 *   nb_nodes[k], nb_elements[k]: sizes of instance k;
 *   nodes: [sum N_k][dim], instance after instance;
 *   connectivity: [sum E_k][n], instance-local node ids (0 .. N_k - 1). */
int akb_batch_create(int spatial_dimension, int element_type, int nb_instances,
                     const int64_t *nb_nodes, const int64_t *nb_elements, const double *nodes,
                     const int32_t *connectivity, akb_model **model);
int akb_batch_nb_instances(const akb_model *model, int *count);
/* first node / element of each instance, arrays of nb_instances + 1 (either
 * may be NULL) */
int akb_batch_instance_offsets(const akb_model *model, int64_t *node_offsets,
                               int64_t *element_offsets);
/* material index of every element of instance k (before initFull) */
int akb_batch_set_instance_materials(akb_model *model, const int32_t *material_of_instance);
/* Instances that stop after their own step counts (the serving loop's
 * batches): from the current step on, instance k advances exactly steps[k]
 * more steps (steps[k] < 0: its limit stays as it is, initially none) and
 * then keeps its state (u, v, a;
 * its plastic internals are not maintained) while the others go on; the
 * captured step graphs stay valid (each step's kernels read the device's
 * step counter).  Called again, it sets new counts from the current step. */
int akb_batch_set_instance_steps(akb_model *model, const int64_t *steps);
/* steps each instance still advances (-1: no limit set) */
int akb_batch_instance_steps_left(const akb_model *model, int64_t *left);
/* enqueues on the model's stream a copy of one instance's nodal field
 * (AKB_DISPLACEMENT, AKB_VELOCITY or AKB_ACCELERATION; N_k * dim doubles) to
 * host memory, after the steps enqueued so far; synchronise the model's
 * stream (or an event recorded on it) before reading the buffer, which
 * should be pinned for the copy to be asynchronous */
int akb_batch_copy_instance_nodal(akb_model *model, int field, int instance, void *host,
                                  int64_t nbytes);
/* getStableTimeStep of every instance -> dt[nb_instances] */
int akb_batch_get_stable_time_steps(akb_model *model, double *dt);
/* setTimeStep per instance (akb_model_set_time_step sets them all) */
int akb_batch_set_time_steps(akb_model *model, const double *dt);
int akb_batch_get_time_steps(const akb_model *model, double *dt);

/* ---- bounds-checking build ----------------------------------------------- */
/* libakb_checked.so is this library built with AKB_BOUNDS_CHECK: its step
 * kernels check every index they read (node ids of the connectivity, slot
 * positions, each node's CSR slot range) before using it; an element or node
 * with an index out of range is skipped and sets bit 2 of the status word
 * (akb_model_get_status).  It stands in for a memory checker.  The persistent
 * kernel and the staged node gather are not used by it.  1 in that build. */
int akb_bounds_checked(void);
/* bounds-checking build only (AKB_EUNSUPPORTED otherwise): overwrites one
 * entry of an index array on the device from the host, for tests of the
 * checks: which 0 connectivity [n][E] (internal order), 1 slot positions
 * [n][E], 2 CSR offsets [N + 1] */
int akb_model_debug_write_index(akb_model *model, int which, int64_t position, int32_t value);

/* ---- serving: many solves resident on one GPU ---------------------------- */
/* No reference counterpart (the reference runs one model per process).  A
 * server admits submitted solves in arrival order while their estimated
 * device memory (akb_estimate_device_bytes, akb_estimate_batch_device_bytes)
 * fits in its budget and fewer than max_active are resident.  Solves of at
 * most batch_max_request_elements elements are admitted in batches: the
 * queue's head with every queued solve of the same element type, quadrature
 * rule, law and precision (limits above) becomes one batch model whose
 * instances each stop after their own step count
 * (akb_batch_set_instance_steps) and are reported as soon as they end, while
 * the batch goes on; larger solves, and a solve with no queued partner of its
 * kind, get a model of their own.  Builder threads
 * prepare the models (tables, lumped mass, stable time steps, step graphs),
 * the scheduler thread advances every resident batch and solve chunk by chunk
 * on its own stream, so that their kernels overlap on the device; arrivals are
 * admitted as soon as memory and a slot are free.  A solve's result does not
 * depend on what else runs (each is computed exactly as by a model of its
 * own). */
typedef struct akb_server akb_server;
typedef struct {
  int device;            /* CUDA device                                        */
  int max_active;        /* resident solves at most (<= 0: 64)                 */
  int64_t device_bytes;  /* admission budget (<= 0: 80% of the free memory)    */
  int64_t chunk_steps;   /* steps enqueued per solve and scheduling pass
                            (<= 0: 500; multiples of 100 use the step graphs)  */
  int builders;          /* host threads preparing and finishing solves (<= 0: 4) */
  double short_work;     /* solves of fewer element-steps (elements x steps) run on
                            high-priority streams (<= 0: 1e8)                   */
  int no_batching;       /* 1: every solve gets a model of its own             */
  int batch_max_instances;            /* solves per batch (<= 0: 256)          */
  int64_t batch_max_request_elements; /* larger solves run alone (<= 0: 2^17)  */
  int64_t batch_max_elements;         /* elements per batch (<= 0: 2^23)       */
} akb_server_config;

typedef struct {
  int element_type, quadrature_rule, precision;
  int64_t nb_nodes, nb_elements;
  const double *nodes;           /* [N][dim]                                   */
  const int32_t *connectivity;   /* [E][n]                                     */
  const char *material_type;     /* elastic | neohookean | plastic_linear_...  */
  const char *material_params;   /* "E = 1; nu = 0.3; rho = 1" (may be NULL)   */
  const double *displacement;    /* initial u [N][dim] or NULL (zero)          */
  const double *velocity;        /* initial v [N][dim] or NULL (zero)          */
  const uint8_t *blocked_dofs;   /* [N][dim] or NULL (none)                    */
  double dt_factor;              /* dt = dt_factor * stable dt (<= 0: 0.8)     */
  int64_t nb_steps;
  double *displacement_out;      /* [N][dim] final u, or NULL; caller-owned,
                                    written before the completion is reported */
  double *velocity_out;          /* [N][dim] final v, or NULL                 */
} akb_request;

typedef struct {
  int64_t id;
  int status;                    /* AKB_OK or the error of the failed step     */
  char message[256];
  double t_submit, t_admit, t_start, t_end; /* seconds on the server's clock   */
  int64_t nb_elements, nb_steps, device_bytes;
  double dt;
  int batched;                   /* 1: advanced as an instance of a batch      */
} akb_completion;

typedef struct {
  int64_t queued, building, running, finishing, completed_unpolled;
  int64_t device_bytes_reserved, device_bytes_budget;
  double now;                    /* the server's clock, seconds                */
} akb_server_stats;

int akb_server_create(const akb_server_config *config, akb_server **server);
/* copies the request's inputs; AKB_ENOMEM if it can never fit the budget */
int akb_server_submit(akb_server *server, const akb_request *request, int64_t *id);
/* up to `capacity` completions, waiting at most wait_seconds for the first */
int akb_server_poll(akb_server *server, akb_completion *out, int capacity, int *count,
                    double wait_seconds);
int akb_server_get_stats(akb_server *server, akb_server_stats *stats);
/* drops queued solves, waits for the admitted ones, joins the threads */
int akb_server_destroy(akb_server *server);

/* ---- stable time step without allocation -------------------------------- */
/* This entry point has no counterpart in the reference.  It computes the
 * same value as akb_model_get_stable_time_step for the elements of one
 * material, for callers that cannot let the library call cudaMalloc: an
 * application whose device memory all comes from its own pool or arena, or
 * code computing the time step inside a loop where runtime allocation is not
 * allowed.  All arrays are device pointers owned by the caller:
 *   nodes, displacement  double [nb_nodes][dim]; connectivity int32 [E][n]
 *   (the reference's node order); dt_out one double, receives
 *   min_e h_e / celerity (DBL_MAX when nb_elements == 0); stream a
 *   cudaStream_t (NULL: the default stream).
 * Every connectivity index must lie in [0, nb_nodes).  An element with an
 * index outside that range reads no node, and dt_out then receives NaN
 * (the check runs on the device, so the call itself still returns AKB_OK).
 * celerity must be finite and positive (AKB_EINVAL otherwise).
 * The work is enqueued on `stream`; synchronise it before reading dt_out.
 * The scratch (per-element values, reduction partials and the index-check
 * word) is a file-scope device array of AKB_NOALLOC_MAX_ELEMENTS + 1025
 * doubles (8 MiB) that every GPU loading the library holds until the
 * process exits; larger element counts are rejected with AKB_EINVAL.  Every
 * call shares that array and clears or overwrites all of it that it reads,
 * so nothing carries over between calls, but calls that overlap on the GPU
 * (different streams, threads or processes sharing the module) race on it.
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress, with that device current) and keeps it; make that
 * first call before any stream capture begins.  cudaDeviceReset unloads the
 * module and invalidates the kept address: do not call this entry point
 * again in a process after resetting a device it ran on. */
#define AKB_NOALLOC_MAX_ELEMENTS (1 << 20)
int akb_stable_time_step_noalloc(int element_type, const double *nodes,
                                 const double *displacement, int64_t nb_nodes,
                                 const int32_t *connectivity, int64_t nb_elements,
                                 double celerity, double *dt_out, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* AKB_CAPI_H_ */

/*
 * CPU oracle for the explicit lumped-mass central-difference step of Akantu's
 * SolidMechanicsModel.  TEST INFRASTRUCTURE ONLY: the parity tests, smoke()
 * and the CPU-baseline leg of bench.py link it as the checker.  The product
 * (akantu2_b200/libakb.so) never calls it.
 *
 * It restates, in plain C++17, the reference algorithm of
 *   src/fe_engine/element_classes/element_class_{tetrahedron_4,hexahedron_8,
 *       triangle_6}_inline_impl.hh      (shapes, dN/ds, inradius)
 *   src/fe_engine/gauss_integration.cc, gauss_integration_tmpl.hh (quadrature)
 *   src/fe_engine/element_class_tmpl.hh:296-395 (J = dN/ds X^T, dN/dx = J^-1 dN/ds)
 *   src/fe_engine/integrator_gauss_inline_impl.hh:176-195,378-441 (det J * w)
 *   src/fe_engine/shape_functions_inline_impl.hh:266-315 (grad u = u B^T)
 *   src/fe_engine/shape_lagrange_inline_impl.hh:373-410 (sigma B)
 *   src/model/solid_mechanics/material.cc:128-154,467-584 (stress / forces)
 *   src/model/solid_mechanics/materials/... (elastic, neohookean, plastic)
 *   src/model/common/dof_manager/dof_manager.cc:65-120 (scatter, ascending e)
 *   src/model/common/integration_scheme/newmark-beta.cc:47-197 (central diff.)
 *   src/model/common/non_linear_solver/non_linear_solver_lumped.cc:48-87
 *   src/fe_engine/fe_engine_template_tmpl_field.hh:59-242 (lumped mass)
 *   src/model/solid_mechanics/solid_mechanics_model.cc:423-621 (dt, energies)
 * Every floating-point expression keeps the operand order written in those
 * files; reductions that Eigen performs internally (matrix products, traces,
 * double dots) are summed left to right.  Build with -ffp-contract=off.
 */
#ifndef AKB_ORACLE_H_
#define AKB_ORACLE_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* element types (same numbering as the product's C-ABI) */
enum { OR_TET4 = 0, OR_HEX8 = 1, OR_TRI6 = 2 };
/* constitutive laws */
// OR_ELASTIC_FD: `elastic` with finite_deformation = true (the elastic law
// applied to the Green-Lagrange strain, finite-strain assembly)
enum { OR_ELASTIC = 0, OR_NEOHOOKEAN = 1, OR_PLASTIC = 2, OR_ELASTIC_FD = 3 };
/* nodal fields */
enum {
  OR_U = 0, OR_V = 1, OR_A = 2, OR_FEXT = 3, OR_FINT = 4, OR_MASS = 5,
  OR_BLOCKED = 6
};
/* quadrature-point fields */
enum {
  OR_GRAD_U = 0, OR_STRESS = 1, OR_PK2 = 2, OR_EPS_P = 3, OR_ISO = 4,
  OR_PLASTIC_ENERGY = 5
};
/* energies */
enum { OR_EKIN = 0, OR_EPOT = 1, OR_EXT_WORK = 2, OR_EPLASTIC = 3 };

typedef struct or_model or_model;

/* ---- element level ------------------------------------------------------ */
int or_nb_nodes_per_element(int type);
int or_dim(int type);
/* qp_rule 0 = the reference default order, 1 = the 6-point triangle rule */
int or_nb_quad(int type, int qp_rule);
void or_quadrature(int type, int qp_rule, double *pts /* [nq][dim] */,
                   double *w /* [nq] */);
void or_shapes(int type, const double *xi, double *N /* [n] */);
/* precompute for E elements; Xe is [E][n][dim]; outputs
 *   N [E][nq][n], B [E][nq][n][dim] (dN_a/dx_j), j [E][nq] (det J * w).
 * returns 0, or -(1 + first e*nq+q) with a negative Jacobian */
long or_precompute(int type, int qp_rule, const double *Xe, long E, double *N,
                   double *B, double *j);
double or_inradius(int type, const double *Xe /* [n][dim] */);

/* ---- material level (single quadrature point) --------------------------- */
/* grad_u, sigma, ... are dim x dim, column-major (i + j*dim) */
void or_elastic_stress(int dim, double E, double nu, int plane_stress,
                       const double *grad_u, double sigma_th, double *sigma);
void or_neohookean_stress(int dim, double E, double nu, const double *grad_u,
                          double C33, double *S);
void or_plastic_stress(int dim, double E, double nu, double sigma_y, double h,
                       const double *grad_u, const double *prev_grad_u,
                       const double *prev_sigma, const double *prev_eps_p,
                       double iso_current, double prev_iso,
                       double delta_sigma_th, double *sigma, double *eps_p,
                       double *iso);

/* ---- model level --------------------------------------------------------- */
or_model *or_model_create(int type, int qp_rule, const double *X, long N,
                          const int32_t *conn, long E);
void or_model_destroy(or_model *m);
/* returns the material index */
int or_model_add_material(or_model *m, int law, double rho, double E,
                          double nu, double sigma_y, double h, double alpha,
                          double delta_T, int plane_stress);
void or_model_set_element_material(or_model *m, const int32_t *mat_of_elem);
/* precompute shapes, jacobians, lumped mass; returns 0 or the precompute
 * error code */
long or_model_init(or_model *m);
double or_model_stable_dt(or_model *m);
void or_model_set_dt(or_model *m, double dt);
void or_model_set_nodal(or_model *m, int field, const void *data);
void or_model_get_nodal(or_model *m, int field, void *data);
long or_model_qp_size(or_model *m, int mat);
void or_model_get_qp(or_model *m, int mat, int field, double *out);
/* eigen_grad_u of every point of material mat, [qp][dim*dim] in the qp
 * getter's order (material.cc:35-51,147: subtracted from grad u) */
void or_model_set_eigen_grad_u(or_model *m, int mat, const double *values);
void or_model_set_threads(or_model *m, int nthreads);
void or_model_solve_step(or_model *m, long nsteps);
/* recompute internal forces (and stresses) at the current displacement */
void or_model_assemble_internal_forces(or_model *m);
double or_model_energy(or_model *m, int which);

#ifdef __cplusplus
}
#endif

#endif

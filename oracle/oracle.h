/*
 * oracle.h — CPU FP64 restatement of FELSPA's level-set hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  The product (felspa_b200/libflsp_dg.so) never
 * links, loads or calls this code.  Only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline / reference arm use it, as the checker and
 * as the CPU baseline.
 *
 * Parity status: UNPINNED.  The reference needs deal.II >= 9.3, Boost and
 * TBB, none of which is available here, and its own tests hold no golden
 * vectors.  This restatement follows the reference source line by line
 * (citations at every function) and is pinned by analytic known-answer
 * tests (tests/test_oracle.py) and by the committed fixtures under
 * tests/golden/ (regression pins of this file, generated by
 * tests/golden/make_golden.py).
 *
 * Conventions shared with the product:
 *   - cells are numbered lexicographically (x fastest);
 *   - within a cell, DoFs follow deal.II's order: FE_DGQLegendre is
 *     lexicographic in (a,b,c) with a fastest; FE_DGP (PolynomialSpace)
 *     loops c outer, b middle, a inner with a+b+c <= p;
 *   - the basis is the Legendre basis orthonormal on [0,1]^dim.
 */
#ifndef FLSP_ORACLE_H
#define FLSP_ORACLE_H

#include "flsp_dg.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_problem orc_problem;

/* advection clock: simulation time, running CFL maximum (the reference's
   CFLEstimator never resets its velo_diam member, pde_tools.implement.h:60-64),
   substeps since the last reinit */
typedef struct orc_clock {
  double t;
  double vd_run;
  int n_since_reinit;
  int n_substeps;
} orc_clock;

int orc_create(const flsp_mesh_desc* mesh, int degree, int basis,
               orc_problem** out);
void orc_destroy(orc_problem* pr);
/* LevelSetSurface::append_boundary_condition with a Dirichlet condition of
   constant value on the boundary faces of id boundary_id (> 0), as
   flsp_set_dirichlet                                                  */
int orc_set_dirichlet(orc_problem* pr, int boundary_id, double value);
void orc_clear_dirichlet(orc_problem* pr);
long orc_n_dofs(const orc_problem* pr);
int orc_dofs_per_cell(const orc_problem* pr);
void orc_set_threads(int n);

/* basis / quadrature known-answer hooks */
void orc_gauss(int n, double* x, double* w);
void orc_legendre(int n, double x, double* v, double* d, double* dd);
/* values (nb*npts) and reference-coordinate gradients (nb*npts*dim) */
void orc_shape(const orc_problem* pr, int npts, const double* xi,
               double* val, double* grad);

int orc_set_velocity(orc_problem* pr, const flsp_velocity_desc* v);
/* velocity of a coupled FE simulator: continuous nodal field of degree
   1..3 on the Gauss-Lobatto lattice (layout of flsp_set_velocity_fe) */
int orc_set_velocity_fe(orc_problem* pr, int degree, const double* values, long n);
void orc_eval_velocity(const orc_problem* pr, const double* x, double t,
                       double* u);
double orc_eval_ic(const flsp_ic_desc* ic, int dim, const double* x);

int orc_project_ic(orc_problem* pr, const flsp_ic_desc* ic, double* phi);

/* advection */
int orc_advect_rhs(orc_problem* pr, const double* phi, double t,
                   double* phidot);
double orc_advect_cfl(orc_problem* pr, double t);
int orc_advance(orc_problem* pr, double* phi, orc_clock* clk, int rk_order,
                double cfl_max, double time_step, int single_cycle,
                double* advanced);

/* Hamilton-Jacobi reinitialization */
int orc_hj_gradients(orc_problem* pr, const double* phi, double* gl,
                     double* gr);
int orc_hj_rhs(orc_problem* pr, const double* phi, const double* phi0,
               double viscosity, double* phidot);
double orc_hj_cfl(orc_problem* pr, const double* phi_grad_src,
                  const double* phi0);
int orc_reinit(orc_problem* pr, double* phi, const flsp_reinit_opts* o,
               int* n_iter);
int orc_weno(orc_problem* pr, double* phi, int* n_troubled);
/* curvature estimate (level_set.implement.h:600-812), lexicographic cells;
   order: the CellId order of the cells (NULL = lexicographic);
   to_neighbour: exterior face terms to the neighbour (0: to the owner, as
   the reference)                                                         */
int orc_curvature(orc_problem* pr, const double* phi, const int64_t* order, int to_neighbour,
                  double* kappa);
int orc_minmod_flags(orc_problem* pr, const double* phi, int* flags);

/* level-set driver */
int orc_ls_advance(orc_problem* pr, double* phi, orc_clock* clk, int rk_order,
                   double cfl_max, const flsp_ls_opts* o, double time_step,
                   int single_step, double* advanced);

/* reductions (flsp_reduce_kind) */
/* MaterialStack mixing of constant material scalars at QGauss(nq) points
   (as flsp_material_mix): out[k * nq^dim + j], k in the cell order
   `order` (NULL: lexicographic) */
int orc_material_mix(int n, orc_problem* const* prs, const double* const* phis, const double* values, int nq,
                     int smoothing, const int64_t* order, double* out);
int orc_reduce(orc_problem* pr, int which, const double* phi,
               const double* phi_ref, const flsp_ic_desc* ic, double* out);

/* learned reinit: FP64 reference MLP (82 -> 256 x4 GELU -> 9) */
int orc_mlp_forward(int n_layers, const int* widths, const double* const* W,
                    const double* const* b, int batch, const double* x,
                    double* y);
int orc_mlp_backward(int n_layers, const int* widths, const double* const* W,
                     const double* const* b, int batch, const double* x,
                     const double* dy, double* const* dW, double* const* db);

#ifdef __cplusplus
}
#endif
#endif

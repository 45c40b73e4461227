/*
 * flsp_dg.h — C ABI of the B200 level-set hot path (DG advection + HJ
 * reinitialization) of FELSPA.
 *
 * One handle = one level-set problem on a uniform Cartesian mesh, resident
 * on one GPU, driven through one CUDA stream.  Host pointers passed to any
 * call are borrowed for the duration of that call only.  Every call returns
 * an int status (FLSP_OK == 0); flsp_last_error() gives a thread-local
 * message.  No C++ exception crosses this boundary.
 *
 * Reference interfaces each entry point replaces (paths inside the FELSPA
 * source tree):
 *   flsp_create / flsp_destroy     dg::AdvectSimulator ctor + do_initialize
 *                                  (include/felspa/pde/src/advection.implement.h:22-83)
 *   flsp_project_ic                AdvectSimulator::discretize_function_to_solution
 *                                  (src/pde/advection.cc:145-169)
 *   flsp_set_state / flsp_get_state  AdvectSimulator::initialize(vector) and
 *                                  get_solution_vector (advection.implement.h:119-131)
 *   flsp_set_velocity              AdvectSimulator::initialize(..., ptr_velocity_field)
 *                                  (advection.implement.h:86-115)
 *   flsp_set_velocity_fe           the same with a simulator as the velocity field
 *                                  (VelocityExtractor, advection.implement.h:472-477,891-905)
 *   flsp_advect_rhs                AdvectSimulator::explicit_time_derivative
 *                                  (src/pde/advection.cc:269-296)
 *   flsp_advance                   AdvectSimulator::advance_time(dt, single)
 *                                  (src/pde/advection.cc:359-426)
 *   flsp_reinit                    ReinitSimulatorLDG::initialize + run_iteration
 *                                  (src/level_set/reinit.cc:386-393,529-637)
 *   flsp_ls_advance                LevelSetSurface::advance_time(dt, single)
 *                                  (include/felspa/level_set/src/level_set.implement.h:180-205)
 *   flsp_hj_gradients              HJSimulator::local_left_right_gradients
 *                                  (src/pde/hamilton_jacobi.cc:462-511)
 *   flsp_weno_limit                dg::apply_weno_limiter
 *                                  (include/felspa/pde/src/pde_tools.implement.h:977-1004)
 *   flsp_reduce                    LevelSetSurface::compute_mass_error / integrate_mass
 *                                  (level_set.implement.h:215-295), AdvectSimulator::
 *                                  compute_error (advection.cc:452-484),
 *                                  ReinitSimulatorLDG::gradient_deviation (reinit.cc:491-526)
 *   flsp_curvature                 LevelSetSurface::CurvatureEstimator::estimate
 *                                  (level_set.implement.h:600-812)
 *   flsp_eval_patches /            SimulatorBase::export_solutions (src/pde/pde_base.cc:93-115),
 *   flsp_export_solutions          LevelSetSurface::export_solution (level_set.implement.h:313-342),
 *                                  PVDCollector (src/base/io.cc:110-166)
 */
#ifndef FLSP_DG_H
#define FLSP_DG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* status codes                                                        */
/* ------------------------------------------------------------------ */
enum flsp_status {
  FLSP_OK = 0,
  FLSP_ERR_CUDA = 1,              /* a CUDA runtime call failed          */
  FLSP_ERR_NONFINITE = 2,         /* NaN/Inf found in state or input     */
  FLSP_ERR_BAD_ARG = 3,           /* invalid argument / size mismatch    */
  FLSP_ERR_BAD_MESH = 4,          /* mesh / permutation failed checks    */
  FLSP_ERR_TIMEOUT = 5,           /* bounded device loop gave up         */
  FLSP_ERR_BAND_NOT_REACHED = 6,  /* reinit hit max_iter (ExcNotEnoughStepsForWidth) */
  FLSP_ERR_UNSUPPORTED = 7,       /* (dim, degree, basis) not compiled   */
  FLSP_ERR_NO_DEVICE = 8,         /* no CUDA device visible              */
  FLSP_ERR_OOM = 9                /* device allocation failed            */
};

enum flsp_basis {
  FLSP_BASIS_P = 0, /* FE_DGP: Legendre, total degree <= p (reference)  */
  FLSP_BASIS_Q = 1  /* FE_DGQLegendre: Legendre tensor product          */
};

enum flsp_precision {
  FLSP_FP64 = 0, /* parity mode: every operation in double             */
  FLSP_FP32 = 1  /* production: stencil arithmetic in float; clocks,
                    CFL and all reductions in double                    */
};

/* ------------------------------------------------------------------ */
/* mesh: uniform Cartesian box, cells numbered lexicographically       */
/* (x fastest) on the device.                                          */
/* ------------------------------------------------------------------ */
typedef struct flsp_mesh_desc {
  int dim;          /* 2 or 3                                            */
  int n[3];         /* cells per axis                                    */
  double lo[3];     /* lower corner                                      */
  double hi[3];     /* upper corner                                      */
  /* Optional host cell order: host_cell_order[k] = lexicographic lattice
     index of the k-th cell of the host DoF vector (for example the active
     cell order of a refined deal.II hyper cube).  NULL = lexicographic.
     Must be a permutation of 0..n_cells-1 (checked at create).          */
  const int64_t* host_cell_order;
  /* Optional boundary ids (deal.II types::boundary_id, >= 0) of the
     domain-boundary faces: side by side in the order x-, x+, y-, y+
     (, z-, z+), each side's faces lexicographic in the other axes (lower
     axis fastest), 2 * sum_d prod_{e != d} n[e] entries.  NULL = every
     boundary face has id 0, as deal.II's hyper_cube without colorize
     (with colorize the sides carry ids 0..2 dim-1 in this order).       */
  const int32_t* boundary_ids;
} flsp_mesh_desc;

typedef struct flsp_dg_opts {
  int degree;      /* 1..3 (3D: 1..2)                                    */
  int basis;       /* flsp_basis                                         */
  int precision;   /* flsp_precision                                     */
  int rk_order;    /* advection SSP-RK order 1..3, reference default 3   */
  double cfl_max;  /* advection CFL upper bound, reference default 0.9   */
  int device;      /* CUDA device ordinal                                */
} flsp_dg_opts;

/* ------------------------------------------------------------------ */
/* prescribed velocity: a sum of separable terms                       */
/*   u_comp(x,t) += coeff * f_0(x_0) f_1(x_1) f_2(x_2) * c(t)           */
/* every field the reference and the benchmark configurations use      */
/* (rigid rotation, single vortex, 3D deformation, Fourier stream      */
/* function, plume rolls, constant) is such a sum.                     */
/* ------------------------------------------------------------------ */
enum flsp_factor_kind {
  FLSP_F_ONE = 0,      /* 1                          */
  FLSP_F_LIN = 1,      /* a*x + b                    */
  FLSP_F_SIN = 2,      /* sin(a*x + b)               */
  FLSP_F_COS = 3,      /* cos(a*x + b)               */
  FLSP_F_SINSQ = 4,    /* sin(a*x + b)^2             */
  FLSP_F_SINPI = 5,    /* sin(pi*(a*x + b))          */
  FLSP_F_COSPI = 6,    /* cos(pi*(a*x + b))          */
  FLSP_F_SINPISQ = 7   /* sin(pi*(a*x + b))^2        */
};

enum flsp_time_kind {
  FLSP_T_ONE = 0,           /* 1                     */
  FLSP_T_COS = 1,           /* cos(a*t + b)          */
  FLSP_T_COSPI = 2,         /* cos(pi*(a*t + b))     */
  FLSP_T_ONE_MINUS_EXP = 3  /* 1 - exp(-a*t)         */
};

typedef struct flsp_factor {
  int kind;
  double a, b;
} flsp_factor;

#define FLSP_MAX_VEL_TERMS 24
typedef struct flsp_vel_term {
  int comp;            /* velocity component 0..dim-1 */
  double coeff;
  flsp_factor f[3];    /* factor per axis (axis 2 ignored in 2D) */
} flsp_vel_term;

typedef struct flsp_velocity_desc {
  int n_terms;
  flsp_vel_term terms[FLSP_MAX_VEL_TERMS];
  int time_kind;       /* flsp_time_kind, one factor for all components */
  double ta, tb;
} flsp_velocity_desc;

/* ------------------------------------------------------------------ */
/* initial condition: small CSG tree of signed-distance primitives     */
/* (reference: include/felspa/level_set/geometry.h:80-160)             */
/* ------------------------------------------------------------------ */
enum flsp_ic_kind {
  FLSP_IC_SPHERE = 0,     /* p[0..2] centre, p[3] radius: |x-c| - r            */
  FLSP_IC_RECT = 1,       /* p[0..2] lower, p[3..5] upper corner: box SDF      */
  FLSP_IC_HEIGHT = 2,     /* x_axis - (p[1] + sum_m w0 cos(2 pi (w1 x_u + w2 x_v) + w3)),
                             axis = (int)p[0]; u,v = the other axes           */
  FLSP_IC_UNION = 3,      /* min(a, b)                                         */
  FLSP_IC_DIFF = 4,       /* max(a, -b)                                        */
  FLSP_IC_INTERSECT = 5   /* max(a, b)                                         */
};

#define FLSP_MAX_IC_NODES 32
#define FLSP_MAX_IC_WAVES 32
typedef struct flsp_ic_node {
  int kind;
  int a, b;            /* child node indices (CSG ops) */
  double p[6];
} flsp_ic_node;

typedef struct flsp_ic_desc {
  int n_nodes;
  int root;
  int exact;           /* reference ICBase::exact; non-exact ICs get a
                          global reinit at initialisation              */
  flsp_ic_node nodes[FLSP_MAX_IC_NODES];
  int n_waves;         /* shared by FLSP_IC_HEIGHT nodes */
  double waves[FLSP_MAX_IC_WAVES][4];
} flsp_ic_desc;

/* ------------------------------------------------------------------ */
/* reinitialization options (reference: src/level_set/reinit.h:276-341) */
/* ------------------------------------------------------------------ */
enum flsp_reinit_mode {
  FLSP_REINIT_BAND = 0,   /* iterate while pseudo-time < band_width_coeff * min_diam */
  FLSP_REINIT_GLOBAL = 1, /* iterate while pseudo-time < 1.2 * max|coeff|            */
  FLSP_REINIT_FIXED = 2   /* exactly n_pseudo_steps pseudo-steps (device resident)   */
};

typedef struct flsp_reinit_opts {
  int mode;                /* flsp_reinit_mode, reference default BAND   */
  int n_pseudo_steps;      /* FIXED mode                                 */
  double band_width_coeff; /* reference default 4.0                      */
  int max_iter;            /* reference default 1000                     */
  double cfl_max;          /* reference ReinitControl default 0.2        */
  double viscosity;        /* LDG artificial viscosity, default 0        */
  int rk_order;            /* reference default 1                        */
  int limiter;             /* 2D WENO limiter: -1 = reference (on in 2D) */
  int narrow_band;         /* 1 = only cells within band_cells of the
                              interface are updated (not in reference)   */
  double band_cells;       /* compute band half-width, in cell diameters */
} flsp_reinit_opts;

/* level-set driver options (reference: level_set.h:108-166) */
typedef struct flsp_ls_opts {
  int reinit_frequency;    /* reference default 10 */
  int execute_reinit;      /* reference default 1  */
  flsp_reinit_opts reinit;
} flsp_ls_opts;

/* reductions (flsp_reduce `which`) */
enum flsp_reduce_kind {
  FLSP_RED_MASS = 0,          /* sum H_eps(-phi) JxW, QGauss(p+1), sine Heaviside,
                                 eps = 1.5 min_diam (integrate_mass)               */
  FLSP_RED_MASS_ERROR = 1,    /* (mass(phi) - mass(ic)) / mass(ic) vs flsp_ic_desc  */
  FLSP_RED_L1_INTERFACE = 2,  /* int |H(-phi) - H(-phi_ref)| dx, sharp H, QGauss(p+2);
                                 reference = the saved snapshot                     */
  FLSP_RED_MEAN_ABS_DIFF = 3, /* mean |coeff - coeff_ref| (compute_error(vector))    */
  FLSP_RED_GRAD_DEVIATION = 4,/* mean over domain of ||grad phi| - 1|, QGauss(p+1)   */
  FLSP_RED_MAX_ABS = 5,       /* max |coeff|                                         */
  FLSP_RED_L2_ERROR_IC = 6,   /* L2 norm of phi - ic, QGauss(p+1)                    */
  FLSP_RED_L1_INTERFACE_IC = 7,/* int |H(-phi) - H(-ic)| dx, sharp H, QGauss(p+2)    */
  FLSP_RED_MASS_SHARP = 8     /* sum H(-phi) JxW with the sharp Heaviside, QGauss(p+2) */
};

typedef struct flsp_handle flsp_handle;

/* lifetime ----------------------------------------------------------- */
int flsp_create(const flsp_mesh_desc* mesh, const flsp_dg_opts* opts,
                flsp_handle** out);
void flsp_destroy(flsp_handle* h);
const char* flsp_last_error(void);
int flsp_version(void);

/* sizes -------------------------------------------------------------- */
int flsp_n_dofs(const flsp_handle* h, int64_t* n_dofs);
int flsp_dofs_per_cell(const flsp_handle* h, int* n);

/* state -------------------------------------------------------------- */
/* A velocity whose components are single terms runs the separable stage
   kernel.  Any other (several terms for a component; every member of a
   batch) is tabulated once here: its spatial part at every cell's
   QGauss(p+2) points and its normal component at every face's, in the
   state precision, read by the stage kernel times the time factor.  The
   tables take dim (p+2)^dim values per cell plus (p+2)^(dim-1) per face
   (3D Q2 FP32: ~1 KB per cell), allocated on the first such velocity and
   kept until flsp_destroy; where they do not fit in device memory the
   stage kernel sums the terms at every point instead (batch members
   fail with FLSP_ERR_OOM).                                              */
int flsp_set_velocity(flsp_handle* h, const flsp_velocity_desc* v);
/* Velocity from a coupled finite-element simulator (the advection
   assembler's simulator branch, advection.implement.h:472-477,891-905;
   the Stokes extractor, stokes_common.implement.h:583-591): a continuous
   nodal field of degree `degree` (1..FLSP_MAX_FE_VEL_DEGREE) per axis,
   the FE_Q field of the coupled simulator on this mesh, evaluated at the
   advection's own quadrature points in every cell.
   `values` holds the field at the Gauss-Lobatto support points of every
   cell (for degree 1 and 2 the equispaced vertices / edge midpoints):
   on axis e node I sits at lo[e] + h[e]*(I/degree + x_{I%degree}), x the
   degree+1 Gauss-Lobatto points on [0,1], I = 0..degree*n[e]; nodes x
   fastest, then y (then z), one block per component: n = dim *
   prod_e (degree*n[e] + 1).  A face's velocity is the same from both of
   its cells (the nodes on the face are shared): the call tabulates the
   field once at every cell's and every face's quadrature points (in the
   state precision), which the stage kernel reads.  The field is constant
   in time.  The CFL estimate is the largest node |u| at a cell vertex
   over the cell diameter (CFLEstimator, pde_tools.implement.h:18-67).
   Setting a field of the same degree again rewrites the device copy in
   place (on the problem's stream): captured graphs stay valid, so a
   coupled loop updates the velocity between advance calls without
   re-capture.  flsp_set_velocity replaces an FE field.  Not supported for
   members of a batch.                                                    */
#define FLSP_MAX_FE_VEL_DEGREE 3
int flsp_set_velocity_fe(flsp_handle* h, int degree, const double* values, int64_t n);
int flsp_project_ic(flsp_handle* h, const flsp_ic_desc* ic);
int flsp_set_state(flsp_handle* h, const double* coeffs, int64_t n);
int flsp_get_state(flsp_handle* h, double* coeffs, int64_t n);
int flsp_set_time(flsp_handle* h, double t);
int flsp_get_time(const flsp_handle* h, double* t);
/* advection substeps executed since create (the reference keeps no such
   counter; its drivers count their advance_time calls)                 */
int flsp_get_step_count(const flsp_handle* h, int64_t* n_substeps);
/* save the current state as the comparison snapshot of the reductions */
int flsp_snapshot(flsp_handle* h);

/* boundary conditions ------------------------------------------------ */
/* LevelSetSurface::append_boundary_condition (level_set.implement.h:
   384-392) with a Dirichlet condition of constant value: on every
   boundary face of id `boundary_id` (> 0; id 0 never takes a condition,
   advection.implement.h:723, ldg.cc:588) the advection inflow
   (advection.implement.h:719-741) and the reinitialisation's LDG left /
   right gradients (ldg.cc:551-620, :686-740) take `value` as the exterior
   trace; the other boundary faces keep the zero-Neumann interior trace.
   Setting an id again replaces its value.  Not supported for members of
   a batch (flsp_batch_run_steps fails).                                */
int flsp_set_dirichlet(flsp_handle* h, int boundary_id, double value);
/* remove every Dirichlet condition                                    */
int flsp_clear_dirichlet(flsp_handle* h);

/* advection ---------------------------------------------------------- */
/* phidot = M^-1 R(phi, t) of the current state, in host DoF order */
int flsp_advect_rhs(flsp_handle* h, double t, double* phidot, int64_t n);
/* AdvectSimulator::advance_time(time_step, single_cycle): CFL-limited
   SSP-RK substeps until time_step is consumed (or one substep).        */
int flsp_advance(flsp_handle* h, double time_step, int single_cycle,
                 double* advanced);
/* n_steps CFL-limited substeps with no host synchronisation in between
   (dt is computed on the device), optionally clamped at t_end.        */
int flsp_advance_steps(flsp_handle* h, int n_steps, double t_end);

/* reinitialization ---------------------------------------------------- */
int flsp_reinit(flsp_handle* h, const flsp_reinit_opts* o, int* n_iter);
/* left/right LDG gradients of the current state: 2*dim blocks of n dofs,
   left blocks first, host DoF order                                    */
int flsp_hj_gradients(flsp_handle* h, double* grads, int64_t n);
/* one application of the 2D minmod detector + WENO limiter             */
int flsp_weno_limit(flsp_handle* h, int* n_troubled);

/* level-set driver ---------------------------------------------------- */
int flsp_ls_advance(flsp_handle* h, const flsp_ls_opts* o, double time_step,
                    int single_step, double* advanced);
/* n_steps advection substeps with a reinit every reinit_frequency steps
   (fixed-count reinit), replayed from a captured CUDA graph.  Returns once
   the work is enqueued on the handle's stream; flsp_sync() waits for it
   (flsp_get_state and the reductions synchronise by themselves).        */
int flsp_ls_run_steps(flsp_handle* h, const flsp_ls_opts* o, int n_steps);
int flsp_sync(flsp_handle* h);
/* the handle's cudaStream_t (for callers that order their own work or
   record CUDA events against the library's work)                       */
int flsp_stream(const flsp_handle* h, void** stream);

/* measurement helper, no counterpart in the reference: average device
   time (ms, CUDA events on the handle's stream) of one launch of a
   hot-path kernel over `reps` back-to-back repetitions; the state is not
   modified.  which: 0 = advection stage kernel (the three SSP-RK3 stages
   per repetition), 1 = reinit pseudo-step kernel.                      */
int flsp_time_kernel(flsp_handle* h, int which, int reps, double* ms_per_launch);

/* Tile autotuner of the advection stage kernel (no counterpart in the
   reference, whose assembly has no tiles): times every CTA tile shape the
   stage kernel is built with on this problem (flsp_time_kernel, `reps`
   RK3 steps each; the state and the device clock are kept) and keeps the
   fastest; `tile` (3 ints, or NULL) receives it.  Optional reports:
   cand_tiles (3 x FLSP_MAX_TILE_CANDIDATES ints) the shapes tried,
   cand_ms (FLSP_MAX_TILE_CANDIDATES) their ms per stage launch (NaN where a
   shape does not fit), n_cand their count.  Captured graphs are dropped.
   flsp_stage_tile reports the tile in force (set at flsp_set_velocity to
   the first shape with two CTAs per SM).                                */
#define FLSP_MAX_TILE_CANDIDATES 8
int flsp_autotune(flsp_handle* h, int reps, int* tile, int* cand_tiles, double* cand_ms,
                  int* n_cand);
int flsp_stage_tile(const flsp_handle* h, int* tile);

/* reductions ---------------------------------------------------------- */
int flsp_reduce(flsp_handle* h, int which, const flsp_ic_desc* ic,
                double* out);

/* curvature ------------------------------------------------------------ */
/* LevelSetSurface::CurvatureEstimator::estimate
   (include/felspa/level_set/src/level_set.implement.h:600-812): the weak
   divergence of grad phi / |grad phi| of the current state with QGauss(p+1)
   cell and face rules and the upwind-by-"shock speed" face flux, divided by
   |K| (the mass solve), then the absolute value of every coefficient.
   FLSP_CURV_REFERENCE reproduces the reference, whose face loop binds the
   exterior face term to the face's owner (the cell with the lower CellId,
   i.e. the earlier one in the host cell order; level_set.implement.h:731):
   both face terms go to the owner and the neighbour gets none, so the
   cell-mean coefficient vanishes away from the boundary.
   FLSP_CURV_NEIGHBOUR gives the exterior term to the neighbour (a standard
   DG divergence; its cell means approach the mean curvature, e.g. 1/r for
   a circle in 2D).  kappa: n_dofs values, host DoF order, FP64.          */
enum flsp_curvature_mode {
  FLSP_CURV_REFERENCE = 0,
  FLSP_CURV_NEIGHBOUR = 1
};
int flsp_curvature(flsp_handle* h, int mode, double* kappa, int64_t n);

/* output --------------------------------------------------------------- */
/* Values of the state at the (n_sub+1)^dim equispaced vertices of every
   cell: the patch deal.II's DataOut::build_patches(n_sub) builds, which
   LevelSetSurface::export_solution uses with n_sub = 1
   (include/felspa/level_set/src/level_set.implement.h:313-342).
   n = n_cells (n_sub+1)^dim values, cells in host order, vertices x
   fastest; evaluated on the device in FP64 from the state (FP64 or FP32).
   1 <= n_sub <= 16.                                                     */
int flsp_eval_patches(flsp_handle* h, int n_sub, double* values, int64_t n);
/* SimulatorBase::export_solutions(path) (src/pde/pde_base.cc:93-115):
   writes <path><label>_<9-digit export count>.vtu (ASCII VTK unstructured
   grid, one patch of corner values per cell, point data named `label`)
   and records (time, file name); <path><label>.pvd is rewritten with every
   record so far on each call (the reference's PVDCollector,
   src/base/io.cc:142-166, writes it once, at destruction).  `path` is a
   prefix (a directory ends with '/'); `label` holds letters, digits, '_',
   '-' and '.' only (it names files and XML attributes).  As the reference, the last
   flsp_curvature result is written too, as `<label>Curvature`, when its
   time equals the state's (within 1e-12, numerics::is_nearly_equal).   */
int flsp_export_solutions(flsp_handle* h, const char* path, const char* label);
/* The host-side writers behind flsp_export_solutions; they need no GPU.
   flsp_write_vtu: `values` as flsp_eval_patches returns them for `mesh`
   (its host_cell_order gives the cell of each patch).  flsp_write_pvd:
   n records (time, VTU file name), deal.II's write_pvd_record layout.  */
int flsp_write_vtu(const flsp_mesh_desc* mesh, int n_sub, const double* values,
                   const char* label, const char* filename);
int flsp_write_pvd(const char* filename, int n, const double* times,
                   const char* const* files);

/* MaterialStack mixing: MaterialAccessor<MaterialStack>::reinit and
   eval_scalars (include/felspa/level_set/src/material_stack.implement.h:
   320-470) for materials with one constant scalar each (a viscosity, a
   density).  At every point of QGauss(n_qpts_1d) of every cell, the level
   sets level_sets[0..n) in stack order each take the share
   rest * H(-phi_i) of what the earlier ones left (rest starts at 1), the
   background material the remaining rest, where H is the level set's
   domain identity (level_set.implement.h:356-380) with `smoothing`
   (flsp_heaviside) over eps = 1.5 min_diameter; shares and rests of
   magnitude <= DBL_EPSILON count as zero (numerics::is_zero).  values[i]
   is material i's scalar, values[n] the background's.  out[k * npt + j]
   = the mixed scalar at point j (x fastest) of host cell k (the first
   handle's cell order), npt = n_qpts_1d^dim.  Every handle must be on the
   same mesh (dim, cells, box) and device; degrees, bases and precisions
   may differ.  The reference sums the shares in the order of its
   material map; here they are summed in stack order, then the
   background.                                                         */
#define FLSP_MAX_MATERIALS 8
#define FLSP_MAX_MIX_QPTS 8
enum flsp_heaviside {
  FLSP_HEAVISIDE_NONE = 0,    /* sharp: 1, 0, 1/2 at zero                */
  FLSP_HEAVISIDE_LINEAR = 1,  /* linear ramp over [-eps, eps]            */
  FLSP_HEAVISIDE_SINE = 2     /* sine smoothing (LevelSetControl default) */
};
int flsp_material_mix(flsp_handle* const* level_sets, int n, const double* values,
                      int n_qpts_1d, int smoothing, double* out, int64_t n_out);

/* Allocation-free reduction.  No counterpart in the reference: FELSPA
   computes these diagnostics on the host.  Same arithmetic as flsp_reduce,
   but for callers that cannot allocate device memory: host codes that own
   all device memory through their own pool or arena and forbid driver
   allocations outside it.  It takes no handle: the
   state is the caller's device array (lexicographic cells, deal.II DoF
   order inside a cell, double for FLSP_FP64 / float for FLSP_FP32),
   `ref_state` the caller's device array for the snapshot reductions (or
   NULL), `ic` a host IC description (or NULL; it is passed to the device
   as a kernel argument, so the caller may free it when the call
   returns), and the scalar result is written to the caller's device
   double `result`.  Work is enqueued on `stream` (a cudaStream_t, NULL =
   default stream) and not waited for.  Scratch space is a file-scope
   device array of 1 MiB (partial sums of at most FLSP_NOALLOC_MAX_CELLS
   cells); larger meshes are rejected with FLSP_ERR_BAD_ARG.  The first
   call on a device (and the first call after cudaDeviceReset, which gives
   the device a new context) uploads the basis tables and looks up the
   array's device address (synchronous); make that first call before any
   stream capture.  All calls on a device share the array and it keeps
   the last call's contents: calls that overlap on the GPU race.          */
#define FLSP_NOALLOC_MAX_CELLS (65536LL * 128LL)
int flsp_reduce_noalloc(const flsp_mesh_desc* mesh, int degree, int basis,
                        int precision, const void* state,
                        const void* ref_state, int which,
                        const flsp_ic_desc* ic, double* result,
                        void* stream);

/* ------------------------------------------------------------------
   Learned reinitialisation (no counterpart in the reference: its
   ReinitSimulatorLDG, src/level_set/reinit.cc:386-637, only has the HJ
   sweep, which stays here as the fallback and as the source of the
   training targets).  2D, degree 2, Q basis.  Input of the network: the
   3 x 3 patch of cells around a cell, 9 coefficients each, divided by the
   cell size h, plus 64 h (82 values, cell rows y outer, x inner; cells
   outside the domain repeat the nearest inside cell).  Output: the change
   of the centre cell's 9 coefficients under the reinitialisation, divided
   by h.  82 -> 256 -> 256 -> 256 -> 256 -> 9, GELU hidden layers, BF16
   weights on the tensor cores, FP32 accumulation and master weights.
   Parameters: W1 [256][82], b1[256], W2 [256][256], b2, W3, b3, W4, b4,
   W5 [9][256], b5[9] (row-major W[out][in]).
   ------------------------------------------------------------------ */
#define FLSP_MLP_IN 82
#define FLSP_MLP_HIDDEN 256
#define FLSP_MLP_OUT 9
/* The 3D variant: 3 x 3 x 3 cells of a 3D degree-2 Q
   state, 27 coefficients each, divided by h, plus 64 h (730 values, cells
   z outer, y, x inner), to the change of the centre cell's 27
   coefficients divided by h: 730 -> 256 x 4 -> 27, same layout rules. */
#define FLSP_MLP3_IN 730
#define FLSP_MLP3_OUT 27
/* patch kinds of flsp_mlp_create_patch */
#define FLSP_PATCH_2D_Q2 0
#define FLSP_PATCH_3D_Q2 1

typedef struct flsp_mlp flsp_mlp;

typedef struct flsp_train_opts {
  int64_t steps;           /* Adam steps                                  */
  int batch;               /* pairs per step (default 8192)               */
  double lr;               /* default 1e-3                                */
  double beta1, beta2, eps;/* default 0.9, 0.999, 1e-8                    */
  uint64_t seed;           /* batch sampling                              */
} flsp_train_opts;

typedef struct flsp_learned_opts {
  double band_cells;       /* cells with |mean phi| <= band_cells * h are
                              redistanced by the network (default 6)      */
  double max_residual;     /* a cell whose mean ||grad phi| - 1| after the
                              network exceeds this takes the HJ result
                              (default 0.05)                              */
  flsp_reinit_opts fallback;   /* the HJ sweep used for those cells; a
                              narrow-band sweep covers exactly them (and the
                              tiles within two cells of them), the rest of
                              the mesh frozen at the pre-reinit state      */
} flsp_learned_opts;

typedef struct flsp_learned_stats {
  int64_t n_band;          /* cells the network redistanced               */
  int64_t n_fallback;      /* of those, cells that took the HJ result     */
  int hj_ran;              /* the fallback sweep ran                      */
} flsp_learned_stats;

int flsp_mlp_create(int device, uint64_t seed, flsp_mlp** out);   /* 2D patch */
int flsp_mlp_create_patch(int patch, int device, uint64_t seed, flsp_mlp** out);
void flsp_mlp_destroy(flsp_mlp* net);
int flsp_mlp_n_params(int64_t* n);   /* of the 2D network */
/* input / output widths and parameter count of a network */
int flsp_mlp_info(const flsp_mlp* net, int* n_in, int* n_out, int64_t* n_params);
int flsp_mlp_get_params(flsp_mlp* net, float* params, int64_t n);
int flsp_mlp_set_params(flsp_mlp* net, const float* params, int64_t n);
/* y[batch][n_out] = net(x[batch][n_in]), host arrays */
int flsp_mlp_forward(flsp_mlp* net, const float* x, int64_t batch, float* y);
/* gradient of sum_b dy[b] . y[b] w.r.t. every parameter (summed over the
   batch, parameter layout above), host arrays */
int flsp_mlp_backward(flsp_mlp* net, const float* x, const float* dy, int64_t batch,
                      float* grad);
/* training pairs from a handle (degree 2, Q basis, square / cubic cells,
   the network's dimension): the
   band cells' patches of the current state, then the handle is
   reinitialised with `target` and the centre cells' changes are the
   targets.  The handle is left reinitialised. */
int flsp_mlp_collect(flsp_mlp* net, flsp_handle* h, double band_cells,
                     const flsp_reinit_opts* target, int64_t* n_added);
int flsp_mlp_n_pairs(const flsp_mlp* net, int64_t* n);
int flsp_mlp_clear_pairs(flsp_mlp* net);
/* Adam on the MSE of the collected pairs; *loss = mean loss of the last
   steps (may be NULL) */
int flsp_mlp_train(flsp_mlp* net, const flsp_train_opts* o, double* loss);
/* mean squared error of the network on the collected pairs */
int flsp_mlp_eval(flsp_mlp* net, double* loss);
/* learned reinitialisation of the handle's state (replaces flsp_reinit) */
int flsp_reinit_learned(flsp_handle* h, flsp_mlp* net, const flsp_learned_opts* o,
                        flsp_learned_stats* stats);
/* n_steps advection substeps with a learned reinitialisation every
   reinit_frequency steps, each period replayed from a captured CUDA graph
   (like flsp_ls_run_steps).  No counterpart in the reference.  With a
   finite o->max_residual > 0 each period carries the residual test and
   the HJ fallback of flsp_reinit_learned, decided on the device: the
   fallback sweep (o->fallback, which must be a fixed-count narrow-band
   sweep) is always enqueued, over the failed cells only, and finds no
   tile to sweep when no band cell failed the test, so the results equal
   flsp_reinit_learned's.  With
   o->max_residual = infinity the network's result is taken in every band
   cell.  Enqueued; flsp_sync waits.  The first period of each buffer role
   sizes the network's work buffers for every cell of the mesh.         */
int flsp_ls_run_steps_learned(flsp_handle* h, flsp_mlp* net, const flsp_learned_opts* o,
                              int reinit_frequency, int n_steps);
/* running totals over the handle's learned reinitialisations (host loop,
   graph-replayed periods, groups): band cells the network redistanced
   and, of those, cells that took the fallback sweep's result (periods
   without a fallback add to the first only); reset != 0 zeroes them.
   Synchronises the handle's stream.                                    */
int flsp_learned_totals(flsp_handle* h, int64_t* n_band, int64_t* n_fallback, int reset);
void flsp_default_train_opts(flsp_train_opts* o);
void flsp_default_learned_opts(flsp_learned_opts* o);

/* ------------------------------------------------------------------
   Batched problems (no counterpart in the reference, where one simulator
   object holds one problem).  Many independent 2D Q-basis problems (own
   meshes, degrees 1..3, velocities, ICs and clocks; one precision and RK
   order) advance together: one persistent launch per RK stage and per
   reinit pseudo-step covers every problem, a reinit period is replayed from
   a captured CUDA graph, and the tile shapes come from flsp_batch_autotune
   (run on first use if not called).  Problem i is a regular handle
   (flsp_batch_problem) for set-up, state exchange and reductions; the
   batch owns it.
   ------------------------------------------------------------------ */
typedef struct flsp_batch flsp_batch;

typedef struct flsp_batch_tuning {
  int adv_tile[2];          /* chosen advection-stage tile (cells x, y)    */
  int hj_tile[2];           /* chosen reinit-step tile                     */
  int n_adv, n_hj;          /* candidates timed                            */
  int adv_cand[8][2];
  int hj_cand[8][2];
  double adv_ms[8];         /* ms per batched launch of each candidate     */
  double hj_ms[8];
} flsp_batch_tuning;

int flsp_batch_create(int n, const flsp_mesh_desc* meshes, const flsp_dg_opts* opts,
                      flsp_batch** out);
void flsp_batch_destroy(flsp_batch* b);
int flsp_batch_size(const flsp_batch* b, int* n);
int flsp_batch_problem(flsp_batch* b, int i, flsp_handle** h);
int flsp_batch_autotune(flsp_batch* b, flsp_batch_tuning* out);
/* n_steps substeps of every problem with a fixed-count reinit every
   reinit_frequency steps (no viscosity, no narrow band); enqueued, returns
   without waiting */
int flsp_batch_run_steps(flsp_batch* b, const flsp_ls_opts* o, int n_steps);
int flsp_batch_sync(flsp_batch* b);
int flsp_batch_stream(const flsp_batch* b, void** stream);

/* ------------------------------------------------------------------
   Groups.  No counterpart in the reference (FELSPA advances one problem
   per simulator object).  A group holds several independent problems of
   any dimension, mesh size or degree (regular handles, still owned by the
   caller); a reinit period of every member (reinit_frequency substeps and
   a fixed-count reinit) is captured into ONE CUDA graph with one branch
   per member, so that small members fill the device beside a large one.
   Every member must be at the start of a reinit period.  Work is enqueued
   on the group's stream, ordered after the members' earlier work and
   before their later work; flsp_group_sync waits for it.
   ------------------------------------------------------------------ */
typedef struct flsp_group flsp_group;

int flsp_group_create(flsp_handle* const* handles, int n, flsp_group** out);
void flsp_group_destroy(flsp_group* g);
int flsp_group_run_periods(flsp_group* g, const flsp_ls_opts* o, int n_periods);
/* the same with the learned reinitialisation, the residual fallback
   decided on the device as in flsp_ls_run_steps_learned (none for
   o->max_residual = infinity): every member advances reinit_frequency
   substeps and takes the network's result in its band, its failed cells
   the result of its own fallback sweep; the members' network passes
   follow one another on the network's stream                            */
int flsp_group_run_periods_learned(flsp_group* g, flsp_mlp* net, const flsp_learned_opts* o,
                                   int reinit_frequency, int n_periods);
int flsp_group_sync(flsp_group* g);
int flsp_group_stream(const flsp_group* g, void** stream);

/* default option structs (reference defaults) */
void flsp_default_dg_opts(flsp_dg_opts* o);
void flsp_default_reinit_opts(flsp_reinit_opts* o);
void flsp_default_ls_opts(flsp_ls_opts* o);

#ifdef __cplusplus
}
#endif
#endif /* FLSP_DG_H */

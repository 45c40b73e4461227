// flsp_api.cu — C ABI of the B200 level-set hot path (include/flsp_dg.h).
//
// Host side of the drop-in: one handle per level-set problem, resident on
// one GPU, driven through one CUDA stream.  The host mirrors the control
// flow of the reference simulators (AdvectSimulator::advance_time,
// ReinitSimulatorLDG::run_iteration*, LevelSetSurface::advance_time); all
// arithmetic on the state runs in the kernels of flsp_k_*.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "flsp_dg.h"
#include "flsp_launch.h"
#include "flsp_mlp.h"
#include "flsp_tables.h"

using namespace flsp;

namespace {
thread_local std::string g_err;
}

namespace flsp {
int set_error(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
}  // namespace flsp

namespace {

int fail(int code, const std::string& msg) { return set_error(code, msg); }

#define CU(call)                                                                         \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return fail(e_ == cudaErrorMemoryAllocation ? FLSP_ERR_OOM : FLSP_ERR_CUDA,        \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                   \
  } while (0)

#define ST(call)                  \
  do {                            \
    int s_ = (call);              \
    if (s_ != FLSP_OK) return s_; \
  } while (0)

double host_factor(const flsp_factor& f, double x) {
  const double kPi = 3.14159265358979323846;
  switch (f.kind) {
    case FLSP_F_ONE: return 1.0;
    case FLSP_F_LIN: return f.a * x + f.b;
    case FLSP_F_SIN: return std::sin(f.a * x + f.b);
    case FLSP_F_COS: return std::cos(f.a * x + f.b);
    case FLSP_F_SINSQ: { double s = std::sin(f.a * x + f.b); return s * s; }
    case FLSP_F_SINPI: return std::sin(kPi * (f.a * x + f.b));
    case FLSP_F_COSPI: return std::cos(kPi * (f.a * x + f.b));
    case FLSP_F_SINPISQ: { double s = std::sin(kPi * (f.a * x + f.b)); return s * s; }
  }
  return 0.0;
}

double host_time_factor(const flsp_velocity_desc& v, double t) {
  const double kPi = 3.14159265358979323846;
  switch (v.time_kind) {
    case FLSP_T_COS: return std::cos(v.ta * t + v.tb);
    case FLSP_T_COSPI: return std::cos(kPi * (v.ta * t + v.tb));
    case FLSP_T_ONE_MINUS_EXP: return 1.0 - std::exp(-v.ta * t);
    default: return 1.0;
  }
}

double adv_cfl_scaling(int p) {  // AdvectSimulator::cfl_scaling (advection.cc:487-496)
  const double pp = p;
  double c = 4.0 / (2.0 + pp) / (2.0 + pp) + 1.0;
  c *= (2.0 * pp + 1.0);
  return c;
}

bool g_tables_ready[64] = {false};

int upload_tables(int dev) {
  if (dev >= 0 && dev < 64 && g_tables_ready[dev]) return FLSP_OK;
  ST(upload_tables_adv());
  ST(upload_tables_hj());
  ST(upload_tables_misc());
  ST(upload_tables_sep2());
  ST(upload_tables_sep3());
  ST(upload_tables_batch());
  ST(upload_tables_io());
  if (dev >= 0 && dev < 64) g_tables_ready[dev] = true;
  return FLSP_OK;
}

}  // namespace

// ------------------------------------------------------------------
// handle
// ------------------------------------------------------------------
struct GraphEntry {
  cudaGraphExec_t exec = nullptr;
  int cur_after = 0;
};

struct flsp_handle {
  int dim = 2, p = 1, basis = 1, prec = 0, rk = 3;
  double cfl_max = 0.9;
  int dev = 0;
  cudaStream_t stream = nullptr;
  MeshArgs m;
  long long ndofs = 0;
  size_t tsize = 8;
  void* buf[3] = {nullptr, nullptr, nullptr};
  int cur = 0;
  void* snap = nullptr;
  bool has_snap = false;
  void* vtab = nullptr;
  double* vtab64 = nullptr;
  void* optab = nullptr;          // separable-operator rows (sep1 velocities)
  int opstride = 0;               // rows per (component, axis) in optab
  bool has_vel = false;
  flsp_velocity_desc vel;
  int nmax = 1, npt = 1;
  // velocity of a coupled FE simulator (fe_pv > 0): the nodal lattice (FP64)
  int fe_pv = 0;
  double* fe_u64 = nullptr;
  // velocity tables at the cells' and faces' quadrature points (state
  // precision; layouts of VelArgs::tab_q / tab_f): the FE field, or a
  // velocity of several terms per component (the point-wise stage kernel's
  // input); tab_ok when they hold the current velocity
  void* tab_q = nullptr;
  void* tab_f = nullptr;
  long long tab_foff[3] = {0, 0, 0}, tab_nf[3] = {0, 0, 0};
  bool tab_ok = false;
  DevClock* clk = nullptr;
  DevClock* clk_host = nullptr;   // pinned mirror
  int64_t* perm = nullptr;
  double* stage64 = nullptr;      // FP64 device staging (2 * dim * ndofs)
  double* partial = nullptr;
  int partial_n = 0;
  double* red_out = nullptr;
  flsp_ic_desc* ic_dev = nullptr;
  unsigned int* flag_dev = nullptr;
  int2* weno_list = nullptr;      // 2D: troubled cells of a limiter pass
  unsigned int* weno_n = nullptr;
  int n_since_reinit = 0;
  void* qbuf = nullptr;     // LDG alternating gradient (dim blocks)
  void* rdiff = nullptr;    // LDG diffusion RHS
  int adv_tile[3] = {0, 0, 0};
  int hj_tile[3] = {0, 0, 0};
  void* hj_stab = nullptr;   // smooth-sign table of the tensor-product reinit kernel
  size_t hj_stab_bytes = 0;
  // learned reinitialisation scratch (allocated on first use)
  int* lrn_flags = nullptr;   // ncell band flags, then per-band-cell fallback flags
  int* lrn_work = nullptr;    // block counts / offsets of the band compaction
  int* lrn_cells = nullptr;   // band cells (ncell)
  int* lrn_count = nullptr;   // [0] band cells, [1] fallback cells
  int* lrn_count_host = nullptr;   // pinned mirror
  unsigned long long* lrn_tot = nullptr;   // running totals: band cells, fallback cells
  void* lrn_save = nullptr;   // one state vector
  float* lrn_feat = nullptr;  // band patch features
  int64_t lrn_feat_cap = 0;
  cudaEvent_t lrn_ev = nullptr;   // orders the network's stream with the handle's
  // compute-restricted narrow band of the reinitialisation
  int* nb_flags = nullptr;    // ncell band flags
  int* nb_lists = nullptr;    // 3 tile lists of ncell entries (HJ, LDG, WENO)
  int* nb_counts = nullptr;   // their device counts
  bool nb_use[3] = {false, false, false};   // lists in force for the launches
  std::map<unsigned long long, GraphEntry> graphs;
  unsigned long long gen = 0;     // bumped whenever captured graphs go stale
  // boundary conditions: id of every domain-boundary face (empty: all 0),
  // Dirichlet value per id, and the per-face values on the device
  std::vector<int32_t> bid;
  std::map<int, double> dirichlet;
  double* bc_dev = nullptr;
  long long nbf = 0;
  bool batch_member = false;      // owned by a batch (no Dirichlet conditions)
  // exported files (PVDCollector: time and VTU name of every export)
  std::vector<std::pair<double, std::string>> pvd;
  // last curvature estimate (host DoF order, FP64) and the time it belongs to
  double* curv = nullptr;
  bool has_curv = false;
  double curv_time = 0.0;

  Ctx ctx() const {
    Ctx c;
    c.dim = dim;
    c.p = p;
    c.prec = prec;
    c.basis = basis;
    c.m = m;
    c.m.tiles = nullptr;
    c.m.n_tiles = nullptr;
    c.stream = stream;
    for (int k = 0; k < 3; ++k) {
      c.nb_tiles[k] = nb_use[k] ? nb_lists + (size_t)k * m.ncell : nullptr;
      c.nb_count[k] = nb_use[k] ? nb_counts + k : nullptr;
    }
    c.hj_stab = hj_stab;
    return c;
  }
  flsp_velocity_desc vel_dev;   // terms as laid out in the device tables
  VelDev veldev() const {
    VelDev v;
    std::memset(&v, 0, sizeof(v));
    v.vtab = vtab;
    v.n_terms = vel_dev.n_terms;
    v.nmax = nmax;
    v.npt = npt;
    for (int k = 0; k < vel_dev.n_terms; ++k) v.comp[k] = vel_dev.terms[k].comp;
    v.sep1 = vel_dev.n_terms == dim;
    for (int k = 0; k < vel_dev.n_terms; ++k) v.sep1 = v.sep1 && vel_dev.terms[k].comp == k;
    v.optab = v.sep1 ? optab : nullptr;
    v.opstride = opstride;
    v.err = clk ? &clk->err : nullptr;
    if (fe_pv > 0) {
      v.sep1 = false;
      v.optab = nullptr;
      v.fe_pv = fe_pv;
    }
    // tables of a velocity the separable kernel does not take
    if (tab_ok && !use_sep_kernel(v)) {
      v.tab = true;
      v.tab_q = tab_q;
      v.tab_f = tab_f;
      for (int e = 0; e < 3; ++e) {
        v.tab_foff[e] = tab_foff[e];
        v.tab_nf[e] = tab_nf[e];
      }
    }
    return v;
  }
};

namespace {

void clear_graphs(flsp_handle* h) {
  for (auto& kv : h->graphs)
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
  h->graphs.clear();
  h->gen++;
}

// per-face Dirichlet values from the face ids and the conditions (NaN: none)
int rebuild_bc(flsp_handle* h) {
  std::vector<double> v((size_t)h->nbf, std::nan(""));
  bool any = false;
  for (long long k = 0; k < h->nbf; ++k) {
    const int id = h->bid.empty() ? 0 : h->bid[k];
    if (id <= 0) continue;
    auto it = h->dirichlet.find(id);
    if (it == h->dirichlet.end()) continue;
    v[k] = it->second;
    any = true;
  }
  CU(cudaSetDevice(h->dev));
  CU(cudaStreamSynchronize(h->stream));
  if (any) {
    if (!h->bc_dev && cudaMalloc(&h->bc_dev, sizeof(double) * (size_t)h->nbf) != cudaSuccess) {
      h->bc_dev = nullptr;
      return fail(FLSP_ERR_OOM, "boundary values allocation failed");
    }
    CU(cudaMemcpy(h->bc_dev, v.data(), sizeof(double) * (size_t)h->nbf, cudaMemcpyHostToDevice));
  }
  h->m.bc_face = any ? h->bc_dev : nullptr;
  clear_graphs(h);
  return FLSP_OK;
}

int ensure_partial(flsp_handle* h, int n) {
  if (h->partial_n >= n) return FLSP_OK;
  if (h->partial) cudaFree(h->partial);
  h->partial = nullptr;
  CU(cudaMalloc(&h->partial, sizeof(double) * 2 * (size_t)n));
  h->partial_n = n;
  return FLSP_OK;
}

int device_error(int err) {
  if (err & kErrCopyTimeout)
    return fail(FLSP_ERR_TIMEOUT, "a kernel's wait for its bulk copies ran out (results invalid)");
  return FLSP_OK;
}

int sync_clock(flsp_handle* h) {
  CU(cudaMemcpyAsync(h->clk_host, h->clk, sizeof(DevClock), cudaMemcpyDeviceToHost, h->stream));
  CU(cudaStreamSynchronize(h->stream));
  return device_error(h->clk_host->err);
}

// kernel configuration of this handle (tiles, shared-memory attributes);
// done outside any stream capture
int prepare_kernels(flsp_handle* h) {
  Ctx c = h->ctx();
  ST(adv_default_tile(c, h->veldev(), h->adv_tile));
  ST(adv_prepare(c, h->veldev(), h->adv_tile));
  ST(hj_default_tile(c, h->hj_tile));
  ST(hj_prepare(c, h->hj_tile));
  if (h->basis == FLSP_BASIS_Q) {
    size_t bytes = 0;
    ST(hj_table_bytes(c, h->hj_tile, &bytes));
    if (bytes != h->hj_stab_bytes) {
      if (h->hj_stab) cudaFree(h->hj_stab);
      h->hj_stab = nullptr;
      h->hj_stab_bytes = 0;
      CU(cudaMalloc(&h->hj_stab, bytes));
      h->hj_stab_bytes = bytes;
    }
  }
  ST(ldg_prepare(c));
  if (h->dim == 2) ST(weno_prepare(c));
  return FLSP_OK;
}

// LDG viscosity buffers (allocated outside any stream capture)
int ensure_ldg_buffers(flsp_handle* h) {
  if (!h->qbuf) CU(cudaMalloc(&h->qbuf, (size_t)h->dim * h->ndofs * h->tsize));
  if (!h->rdiff) CU(cudaMalloc(&h->rdiff, (size_t)h->ndofs * h->tsize));
  return FLSP_OK;
}

int other(int a, int b) {  // the buffer index that is neither a nor b
  for (int i = 0; i < 3; ++i)
    if (i != a && i != b) return i;
  return -1;
}

int stage(flsp_handle* h, const void* in, const void* phin, void* out, int st, int combine) {
  return launch_adv_stage(h->ctx(), h->veldev(), in, phin, out, h->clk, st, combine, 0.0, h->adv_tile);
}

// one SSP-RK substep on the device clock (no host synchronisation)
// step_count: a step-count run (flsp_advance_steps, graph periods) rather
// than a call for a time step (flsp_advance, the reference's advance_time)
int enqueue_adv_step(flsp_handle* h, bool step_count = true) {
  AdvClockArgs ca;
  ca.cfl_max = h->cfl_max;
  ca.scale = adv_cfl_scaling(h->p);
  ca.tkind = h->vel.time_kind;
  ca.ta = h->vel.ta;
  ca.tb = h->vel.tb;
  ca.rk = h->rk;
  ca.step_count = step_count ? 1 : 0;
  ST(launch_adv_clock_begin(h->stream, h->clk, ca));
  const int x = h->cur, y = (h->cur + 1) % 3, z = (h->cur + 2) % 3;
  void* X = h->buf[x];
  void* Y = h->buf[y];
  void* Z = h->buf[z];
  if (h->rk == 1) {
    ST(stage(h, X, X, Y, 0, kRK1));
    h->cur = y;
  } else if (h->rk == 2) {
    ST(stage(h, X, X, Y, 0, kRK2a));
    ST(stage(h, Y, X, Z, 1, kRK2b));
    h->cur = z;
  } else {
    ST(stage(h, X, X, Y, 0, kRK3a));
    ST(stage(h, Y, X, Z, 1, kRK3b));
    ST(stage(h, Z, X, Y, 2, kRK3c));
    h->cur = y;
  }
  return launch_adv_clock_end(h->stream, h->clk);
}

bool reinit_limiter(const flsp_handle* h, const flsp_reinit_opts* o) {
  if (h->dim != 2) return false;
  return o->limiter < 0 ? true : o->limiter != 0;
}

// one reinitialisation pseudo-step: reads cur and phi0, writes a free buffer
int enqueue_hj_step(flsp_handle* h, const flsp_reinit_opts* o, int phi0_idx, bool limiter) {
  ST(launch_hj_clock_begin(h->stream, h->clk, o->cfl_max, h->p, o->viscosity, h->m.min_diam,
                           adv_cfl_scaling(h->p)));
  const int src = h->cur;
  const int dst = (src == phi0_idx) ? (phi0_idx + 1) % 3 : other(src, phi0_idx);
  const void* rdiff = nullptr;
  if (o->viscosity > 0.0) {   // LDGDiffusionTerm of the current solution (ldg.cc:249-298)
    ST(launch_ldg(h->ctx(), h->buf[src], h->qbuf, h->ndofs, o->viscosity, 0));
    ST(launch_ldg(h->ctx(), h->qbuf, h->rdiff, h->ndofs, o->viscosity, 1));
    rdiff = h->rdiff;
  }
  ST(launch_hj(h->ctx(), h->buf[src], h->buf[phi0_idx], h->buf[dst], h->clk, kHJStep, o->rk_order, 0.0,
               h->ndofs, h->hj_tile, rdiff));
  int res = dst;
  if (limiter) {
    const int lim = other(dst, phi0_idx);
    ST(launch_weno(h->ctx(), h->buf[dst], h->buf[lim], nullptr, h->weno_list, h->weno_n));
    res = lim;
  }
  h->cur = res;
  return launch_hj_clock_end(h->stream, h->clk);
}

int reduce_dev(flsp_handle* h, int which, const void* phi, const void* ref, bool with_ic, double* out2) {
  Ctx c = h->ctx();
  ST(ensure_partial(h, reduce_blocks(c)));
  ST(launch_reduce(c, which, phi, ref, with_ic ? h->ic_dev : nullptr, h->partial, h->red_out));
  CU(cudaMemcpyAsync(out2, h->red_out, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CU(cudaStreamSynchronize(h->stream));
  return FLSP_OK;
}

int check_finite(flsp_handle* h, const void* x) {
  CU(cudaMemsetAsync(h->flag_dev, 0, sizeof(unsigned int), h->stream));
  ST(launch_nonfinite(h->ctx(), x, h->ndofs, h->flag_dev));
  unsigned int cnt = 0;
  CU(cudaMemcpyAsync(&cnt, h->flag_dev, sizeof(cnt), cudaMemcpyDeviceToHost, h->stream));
  CU(cudaStreamSynchronize(h->stream));
  if (cnt) return fail(FLSP_ERR_NONFINITE, std::to_string(cnt) + " non-finite coefficients");
  return FLSP_OK;
}

void fill_reinit_defaults(flsp_reinit_opts* o) {
  o->mode = FLSP_REINIT_BAND;
  o->n_pseudo_steps = 5;
  o->band_width_coeff = 4.0;
  o->max_iter = 1000;
  o->cfl_max = 0.2;
  o->viscosity = 0.0;
  o->rk_order = 1;
  o->limiter = -1;
  o->narrow_band = 0;
  o->band_cells = 6.0;
}

int validate_reinit(const flsp_handle* h, const flsp_reinit_opts* o) {
  if (!o) return fail(FLSP_ERR_BAD_ARG, "null reinit options");
  if (o->mode < 0 || o->mode > 2) return fail(FLSP_ERR_BAD_ARG, "bad reinit mode");
  if (!(o->cfl_max > 0.0)) return fail(FLSP_ERR_BAD_ARG, "reinit cfl_max must be positive");
  if (o->mode == FLSP_REINIT_BAND && !(o->band_width_coeff > 1.0))
    return fail(FLSP_ERR_BAD_ARG, "band_width_coeff must be greater than 1 (reinit.cc:597-598)");
  if (o->mode == FLSP_REINIT_FIXED && (o->n_pseudo_steps < 0 || o->n_pseudo_steps > 100000))
    return fail(FLSP_ERR_BAD_ARG, "bad n_pseudo_steps");
  if (o->max_iter < 0) return fail(FLSP_ERR_BAD_ARG, "negative max_iter");
  if (o->viscosity < 0.0) return fail(FLSP_ERR_BAD_ARG, "negative viscosity");
  if (o->rk_order < 1 || o->rk_order > 3) return fail(FLSP_ERR_BAD_ARG, "reinit rk_order must be 1..3");
  if (o->narrow_band && !(o->band_cells > 0.0)) return fail(FLSP_ERR_BAD_ARG, "narrow band needs band_cells > 0");
  (void)h;
  return FLSP_OK;
}

// Compute-restricted narrow band (flsp_reinit_opts::narrow_band): only the
// tiles within two cells of the band |mean phi0| <= band_cells * min_diam
// are swept (kernel grids keep their size, blocks past the device-side tile
// count return at once, so nothing here waits for the host); the other
// state buffers start as copies of phi0 so that untouched tiles stay
// consistent, and at the end the cells outside the band get phi0 back.
// Enqueue only: usable inside a stream capture.
int ensure_band_buffers(flsp_handle* h) {
  if (!h->nb_flags) {
    CU(cudaMalloc(&h->nb_flags, (size_t)h->m.ncell * sizeof(int)));
    CU(cudaMalloc(&h->nb_lists, 3 * (size_t)h->m.ncell * sizeof(int)));
    CU(cudaMalloc(&h->nb_counts, 3 * sizeof(int)));
  }
  return FLSP_OK;
}

// The cells a narrow-band sweep covers, when they are not the band of phi0:
// the listed cells (cells[i], i < min(n, *n_dev)) whose flag is set.
struct SweepCells {
  const int* cells;
  const int* flags;
  long long n;
  const int* n_dev;
};

// (buffers allocated beforehand by ensure_band_buffers); `only`: the band is
// that cell list instead of |mean phi0| <= band_cells * min_diam
int band_begin(flsp_handle* h, const flsp_reinit_opts* o, int phi0, bool limiter, const SweepCells* only = nullptr) {
  Ctx c = h->ctx();
  if (only)
    ST(launch_band_flags_from_list(c, only->cells, only->flags, only->n, only->n_dev, h->nb_flags));
  else
    ST(launch_band_flags(c, h->buf[phi0], o->band_cells * h->m.min_diam, h->nb_flags));
  const int margin = 2;
  ST(launch_band_tiles(c, h->nb_flags, h->hj_tile, margin, h->nb_lists, h->nb_counts));
  h->nb_use[kNbHJ] = true;
  if (o->viscosity > 0.0) {
    ST(launch_band_tiles(c, h->nb_flags, h->dim == 2 ? kLdgTile2 : kLdgTile3, margin,
                         h->nb_lists + (size_t)kNbLdg * h->m.ncell, h->nb_counts + kNbLdg));
    h->nb_use[kNbLdg] = true;
    CU(cudaMemsetAsync(h->qbuf, 0, (size_t)h->dim * h->ndofs * h->tsize, h->stream));
    CU(cudaMemsetAsync(h->rdiff, 0, (size_t)h->ndofs * h->tsize, h->stream));
  }
  if (limiter) {
    ST(launch_band_tiles(c, h->nb_flags, kWenoTile, margin, h->nb_lists + (size_t)kNbWeno * h->m.ncell,
                         h->nb_counts + kNbWeno));
    h->nb_use[kNbWeno] = true;
  }
  for (int i = 0; i < 3; ++i)
    if (i != phi0)
      CU(cudaMemcpyAsync(h->buf[i], h->buf[phi0], (size_t)h->ndofs * h->tsize, cudaMemcpyDeviceToDevice, h->stream));
  return FLSP_OK;
}

int band_end(flsp_handle* h, int phi0) {
  for (int k = 0; k < 3; ++k) h->nb_use[k] = false;
  return launch_band_restore(h->ctx(), h->buf[phi0], h->buf[h->cur], h->nb_flags);
}

// ReinitSimulatorLDG::initialize + run_iteration (reinit.cc:386-393, 529-637);
// a narrow-band sweep given `only` covers those cells (none listed: no tile)
int run_reinit(flsp_handle* h, const flsp_reinit_opts* o, int* n_iter, const SweepCells* only = nullptr) {
  ST(validate_reinit(h, o));
  if (o->viscosity > 0.0) ST(ensure_ldg_buffers(h));
  const bool limiter = reinit_limiter(h, o);
  const int phi0 = h->cur;
  const bool narrow = o->narrow_band != 0;
  if (narrow) {
    ST(ensure_band_buffers(h));
    const int st = band_begin(h, o, phi0, limiter, only);
    if (st) {
      for (int k = 0; k < 3; ++k) h->nb_use[k] = false;
      return st;
    }
  }
  auto sweep = [&]() -> int {
    ST(launch_hj_clock_reset(h->stream, h->clk));
    // CFL estimate of the first pseudo-step: gradients of the initial state
    ST(launch_hj(h->ctx(), h->buf[phi0], h->buf[phi0], nullptr, h->clk, kHJCflOnly, o->rk_order, 0.0,
                 h->ndofs, h->hj_tile));
    int it = 0;
    if (o->mode == FLSP_REINIT_FIXED) {
      for (it = 0; it < o->n_pseudo_steps; ++it) ST(enqueue_hj_step(h, o, phi0, limiter));
    } else {
      double horizon;
      if (o->mode == FLSP_REINIT_GLOBAL) {
        double r[2];
        ST(reduce_dev(h, FLSP_RED_MAX_ABS, h->buf[phi0], nullptr, false, r));
        horizon = 1.2 * r[0];
      } else {
        horizon = o->band_width_coeff * h->m.min_diam;
      }
      double cum = 0.0;
      while (cum < horizon && it <= o->max_iter) {
        ST(enqueue_hj_step(h, o, phi0, limiter));
        ++it;
        ST(sync_clock(h));
        cum = h->clk_host->hj_cum;
        if (!std::isfinite(cum) || !(h->clk_host->hj_dt > 0.0))
          return fail(FLSP_ERR_NONFINITE, "reinit pseudo-time step is not positive/finite");
      }
    }
    if (n_iter) *n_iter = it;
    if (o->mode == FLSP_REINIT_BAND && it == o->max_iter)
      return fail(FLSP_ERR_BAND_NOT_REACHED, "reinit reached max_iter before the band width");
    return FLSP_OK;
  };
  int st = sweep();
  if (narrow) {
    const int st2 = band_end(h, phi0);
    if (st == FLSP_OK) st = st2;
  }
  return st;
}

// Lay the velocity terms out for the device: when every component has at
// most one term, term k becomes component k (a zero term stands in for a
// missing component), which selects the stage kernel's fast path.
void layout_velocity(flsp_handle* h) {
  const flsp_velocity_desc& v = h->vel;
  int count[3] = {0, 0, 0};
  for (int k = 0; k < v.n_terms; ++k) count[v.terms[k].comp]++;
  bool sep = true;
  for (int d = 0; d < h->dim; ++d) sep = sep && count[d] <= 1;
  h->vel_dev = v;
  if (!sep) {
    // terms grouped by component (stable: each component keeps its own
    // order, so its sum is formed in the same order)
    std::stable_sort(h->vel_dev.terms, h->vel_dev.terms + h->vel_dev.n_terms,
                     [](const flsp_vel_term& x, const flsp_vel_term& y) { return x.comp < y.comp; });
    return;
  }
  flsp_velocity_desc r = v;
  r.n_terms = h->dim;
  for (int d = 0; d < h->dim; ++d) {
    flsp_vel_term zero;
    std::memset(&zero, 0, sizeof(zero));
    zero.comp = d;
    zero.coeff = 0.0;
    r.terms[d] = zero;
  }
  for (int k = 0; k < v.n_terms; ++k) r.terms[v.terms[k].comp] = v.terms[k];
  h->vel_dev = r;
}

// Per-axis operator rows of a velocity whose component d is the single
// separable term d (the stage kernel's separable path, flsp_advsep.cuh).
// For component d, axis e and cell index i along e, with g = the term's
// axis-e factor at the cell's QGauss(p+2) points:
//   A[a][b] = sum_q w_q g(x_q) L_b(x_q) (e == d ? L_a'(x_q) : L_a(x_q))
//   e != d: B[a][b] = sum_q w_q |g(x_q)| L_a(x_q) L_b(x_q)  (at element boff),
//           and at element (p+1)^2 the sign of g over the points (0: mixed)
//   e == d: g(0), g(1)                                      (at element boff)
// All in FP64 (long double sums) from the same factor values as the
// point-wise tables, stored in the state precision.
int build_optab(flsp_handle* h, const std::vector<double>& tabd) {
  if (h->optab) cudaFree(h->optab);
  h->optab = nullptr;
  VelDev vd = h->veldev();
  if (!vd.sep1) return FLSP_OK;
  const int n1 = h->p + 1, nq = h->p + 2, nn = n1 * n1;
  const int boff = ((nn + 1 + 3) / 4) * 4, opw = 2 * boff;   // spare element nn: sign of g
  // a tile copies its rows in one piece: pad each (d, e) block past the mesh
  const int stride = h->nmax + kOpRowPad;
  const size_t nrow = (size_t)h->dim * 3 * stride;
  std::vector<double> op(nrow * opw, 0.0);
  double x[8], w[8], lv[8][8], ld[8][8];
  gauss_rule(nq, x, w);
  for (int q = 0; q < nq; ++q) {
    double dd[8];
    leg_all(n1, x[q], lv[q], ld[q], dd);
  }
  for (int d = 0; d < h->dim; ++d)
    for (int e = 0; e < h->dim; ++e)
      for (int i = 0; i < h->m.n[e]; ++i) {
        const size_t r = ((size_t)d * 3 + e) * h->nmax + i;
        const double* gq = &tabd[r * h->npt];   // term d == component d
        double* row = &op[(((size_t)d * 3 + e) * stride + i) * opw];
        for (int al = 0; al < n1; ++al)
          for (int be = 0; be < n1; ++be) {
            long double sa = 0.0L, sb = 0.0L;
            for (int q = 0; q < nq; ++q) {
              const long double t = (long double)w[q] * gq[q] * lv[q][be];
              sa += t * (e == d ? ld[q][al] : lv[q][al]);
              sb += (long double)w[q] * std::fabs(gq[q]) * lv[q][be] * lv[q][al];
            }
            row[al * n1 + be] = (double)sa;
            if (e != d) row[boff + al * n1 + be] = (double)sb;
          }
        if (e != d) {   // sign of g over the Gauss points (0: changes sign)
          bool pos = true, neg = true;
          for (int q = 0; q < nq; ++q) {
            pos = pos && gq[q] >= 0.0;
            neg = neg && gq[q] <= 0.0;
          }
          row[nn] = pos ? 1.0 : (neg ? -1.0 : 0.0);
        }
        if (e == d) {
          row[boff] = gq[nq];          // xi = 0
          row[boff + 1] = gq[nq + 1];  // xi = 1
        }
      }
  const size_t n = op.size();
  if (h->prec == FLSP_FP64) {
    CU(cudaMalloc(&h->optab, n * sizeof(double)));
    CU(cudaMemcpy(h->optab, op.data(), n * sizeof(double), cudaMemcpyHostToDevice));
  } else {
    std::vector<float> of(n);
    for (size_t i = 0; i < n; ++i) of[i] = (float)op[i];
    CU(cudaMalloc(&h->optab, n * sizeof(float)));
    CU(cudaMemcpy(h->optab, of.data(), n * sizeof(float), cudaMemcpyHostToDevice));
  }
  h->opstride = stride;
  return FLSP_OK;
}

// Gauss-Lobatto points of degree pv on [0, 1] (the support points of FE_Q(pv))
void gauss_lobatto01(int pv, double* x) {
  x[0] = 0.0;
  x[pv] = 1.0;
  if (pv == 2) x[1] = 0.5;
  if (pv == 3) {
    const double r = 0.5 / std::sqrt(5.0);
    x[1] = 0.5 - r;
    x[2] = 0.5 + r;
  }
}

// Lagrange basis a of the nodes x[0..pv] at t; exactly 1 / 0 at the nodes
// (numerator and denominator are the same products there)
double lagrange(int pv, const double* x, int a, double t) {
  double num = 1.0, den = 1.0;
  for (int b = 0; b <= pv; ++b) {
    if (b == a) continue;
    num *= t - x[b];
    den *= x[a] - x[b];
  }
  return num / den;
}

void free_fe_velocity(flsp_handle* h) {
  if (h->fe_u64) cudaFree(h->fe_u64);
  h->fe_u64 = nullptr;
  h->fe_pv = 0;
  h->tab_ok = false;
}

// the velocity tables (sizes fixed by the mesh and the degree)
int ensure_vel_tables(flsp_handle* h) {
  if (h->tab_q) return FLSP_OK;
  const int nq = h->p + 2;
  const long long nqd = h->dim > 2 ? (long long)nq * nq * nq : (long long)nq * nq;
  const long long nqf = h->dim > 2 ? (long long)nq * nq : nq;
  long long off = 0;
  for (int e = 0; e < 3; ++e) {
    long long nf = e < h->dim ? 1 : 0;
    for (int d = 0; d < h->dim && e < h->dim; ++d) nf *= h->m.n[d] + (d == e);
    h->tab_foff[e] = off;
    h->tab_nf[e] = nf;
    off += nqf * nf;
  }
  if (cudaMalloc(&h->tab_q, (size_t)(h->dim * nqd * h->m.ncell) * h->tsize) != cudaSuccess ||
      cudaMalloc(&h->tab_f, (size_t)off * h->tsize) != cudaSuccess) {
    if (h->tab_q) cudaFree(h->tab_q);
    h->tab_q = nullptr;
    return fail(FLSP_ERR_OOM, "velocity table allocation failed");
  }
  return FLSP_OK;
}

void free_vel_tables(flsp_handle* h) {
  if (h->tab_q) cudaFree(h->tab_q);
  if (h->tab_f) cudaFree(h->tab_f);
  h->tab_q = h->tab_f = nullptr;
  h->tab_ok = false;
}

// tables: tabulate a velocity of several terms per component (the
// point-wise stage kernel reads the tables instead of summing the terms at
// every point of every stage; batch members always)
int build_vtab(flsp_handle* h, bool tables = true) {
  const int dim = h->dim;
  layout_velocity(h);
  const int nq = h->p + 2;
  h->npt = nq + 2;
  h->nmax = std::max(h->m.n[0], std::max(h->m.n[1], h->m.n[2]));
  const int nt = std::max(h->vel_dev.n_terms, 1);
  const size_t n = (size_t)nt * 3 * h->nmax * h->npt;
  std::vector<double> tabd(n, 0.0);
  double x[8], w[8];
  gauss_rule(nq, x, w);
  for (int k = 0; k < h->vel_dev.n_terms; ++k) {
    const flsp_vel_term& tm = h->vel_dev.terms[k];
    for (int ax = 0; ax < 3; ++ax)
      for (int i = 0; i < h->nmax; ++i)
        for (int j = 0; j < h->npt; ++j) {
          double v = 1.0;
          if (ax < dim && i < h->m.n[ax]) {
            const double xi = j < nq ? x[j] : (double)(j - nq);
            const double X0 = h->m.lo[ax] + i * h->m.h[ax];
            // a face's coordinate by one expression from both of its cells
            // (cell i's upper face = cell i + 1's lower face, bit for bit)
            const double xx = j == nq + 1 ? h->m.lo[ax] + (i + 1) * h->m.h[ax] : X0 + h->m.h[ax] * xi;
            // coefficient folded into the x factor: ((coeff f0) f1) f2
            v = (ax == 0) ? tm.coeff * host_factor(tm.f[0], xx) : host_factor(tm.f[ax], xx);
          }
          tabd[(((size_t)k * 3 + ax) * h->nmax + i) * h->npt + j] = v;
        }
  }
  if (h->vtab) cudaFree(h->vtab);
  if (h->vtab64) cudaFree(h->vtab64);
  h->vtab = nullptr;
  h->vtab64 = nullptr;
  CU(cudaMalloc(&h->vtab64, n * sizeof(double)));
  CU(cudaMemcpy(h->vtab64, tabd.data(), n * sizeof(double), cudaMemcpyHostToDevice));
  if (h->prec == FLSP_FP64) {
    CU(cudaMalloc(&h->vtab, n * sizeof(double)));
    CU(cudaMemcpy(h->vtab, tabd.data(), n * sizeof(double), cudaMemcpyHostToDevice));
  } else {
    std::vector<float> tf(n);
    for (size_t i = 0; i < n; ++i) tf[i] = (float)tabd[i];
    CU(cudaMalloc(&h->vtab, n * sizeof(float)));
    CU(cudaMemcpy(h->vtab, tf.data(), n * sizeof(float), cudaMemcpyHostToDevice));
  }
  ST(build_optab(h, tabd));
  int comp[kMaxTerms];
  for (int k = 0; k < h->vel_dev.n_terms; ++k) comp[k] = h->vel_dev.terms[k].comp;
  h->tab_ok = false;
  if (tables && (h->batch_member || !use_sep_kernel(h->veldev()))) {
    const int st = ensure_vel_tables(h);
    if (st == FLSP_OK) {
      ST(launch_vel_tabulate(h->ctx(), h->vtab64, h->vel_dev.n_terms, comp, h->nmax, h->npt, h->tab_q, h->tab_f,
                             h->tab_foff, h->tab_nf));
      h->tab_ok = true;
    } else if (h->batch_member) {
      return st;   // the batched stage kernel reads tables only
    } else {
      cudaGetLastError();   // no room for the tables: the stage kernel sums the terms at every point
    }
  }
  // static CFL part: max over vertices of |u_spatial| / diam
  CU(cudaMemsetAsync(&h->clk->vd_static, 0, sizeof(double), h->stream));
  ST(launch_static_cfl(h->ctx(), h->vtab64, h->vel_dev.n_terms, comp, h->nmax, h->npt, h->clk));
  CU(cudaStreamSynchronize(h->stream));
  return FLSP_OK;
}

// ---- learned reinitialisation helpers
int learned_check(const flsp_handle* h, const flsp_mlp* net) {
  if (h->p != 2 || h->basis != FLSP_BASIS_Q)
    return fail(FLSP_ERR_UNSUPPORTED, "learned reinitialisation: degree 2, Q basis only");
  for (int d = 1; d < h->dim; ++d)
    if (std::fabs(h->m.h[0] - h->m.h[d]) > 1e-12 * h->m.h[0])
      return fail(FLSP_ERR_UNSUPPORTED, "learned reinitialisation: square / cubic cells only");
  if (net && net->dev != h->dev) return fail(FLSP_ERR_BAD_ARG, "network and problem on different devices");
  if (net && (h->dim == 3) != (net->patch == FLSP_PATCH_3D_Q2))
    return fail(FLSP_ERR_BAD_ARG, "the network's patch is not of the problem's dimension");
  return FLSP_OK;
}

// network input width for the handle's dimension
int learned_n_in(const flsp_handle* h) { return h->dim == 3 ? FLSP_MLP3_IN : FLSP_MLP_IN; }

int ensure_learned_buffers(flsp_handle* h, int64_t nfeat) {
  const int64_t ncell = h->m.ncell;
  if (!h->lrn_flags) {
    const int64_t nblk = (ncell + 255) / 256;
    CU(cudaMalloc(&h->lrn_flags, (size_t)ncell * sizeof(int)));
    CU(cudaMalloc(&h->lrn_work, (size_t)(2 * nblk + 2) * sizeof(int)));
    CU(cudaMalloc(&h->lrn_cells, (size_t)ncell * sizeof(int)));
    CU(cudaMalloc(&h->lrn_count, 2 * sizeof(int)));
    CU(cudaMalloc(&h->lrn_tot, 2 * sizeof(unsigned long long)));
    CU(cudaMemsetAsync(h->lrn_tot, 0, 2 * sizeof(unsigned long long), h->stream));
    CU(cudaMallocHost(&h->lrn_count_host, 4 * sizeof(int)));
    CU(cudaEventCreateWithFlags(&h->lrn_ev, cudaEventDisableTiming));
    CU(cudaMalloc(&h->lrn_save, (size_t)h->ndofs * h->tsize + kStatePad));
  }
  if (h->lrn_feat_cap < nfeat) {
    if (h->lrn_feat) cudaFree(h->lrn_feat);
    h->lrn_feat = nullptr;
    CU(cudaMalloc(&h->lrn_feat, (size_t)nfeat * learned_n_in(h) * sizeof(float)));
    h->lrn_feat_cap = nfeat;
  }
  return FLSP_OK;
}

// The network's part of a learned reinitialisation, enqueued on the
// handle's stream without a host wait (graph-capturable once the buffers
// exist): band cells of buf[pre], their patch features, the network (on its
// own stream, ordered by an event both ways), and buf[out] = buf[pre] with
// the band cells corrected.  Every launch is sized for all cells; the band's
// size stays on the device.
int enqueue_learned(flsp_handle* h, flsp_mlp* net, double band_cells, int pre, int out) {
  const int64_t ncell = h->m.ncell;
  const double hh = h->m.h[0];
  const int* nband = h->lrn_count;
  ST(launch_band_select(h->stream, h->prec, h->m.nb, h->buf[pre], ncell, band_cells * hh, h->lrn_flags,
                        h->lrn_work, h->lrn_cells, h->lrn_count));
  ST(launch_patch_features(h->stream, h->prec, h->dim, h->buf[pre], h->m.n, hh, h->lrn_cells, ncell, nband,
                           h->lrn_feat));
  CU(cudaEventRecord(h->lrn_ev, h->stream));
  CU(cudaStreamWaitEvent(net->stream, h->lrn_ev, 0));
  int st = mlp_pack_input(net, h->lrn_feat, nullptr, ncell, nband);
  if (st == FLSP_OK) st = mlp_forward_dev(net, ncell, false, nband);
  // join back even after a failed launch, so that a capture stays joined
  const cudaError_t e1 = cudaEventRecord(h->lrn_ev, net->stream);
  const cudaError_t e2 = cudaStreamWaitEvent(h->stream, h->lrn_ev, 0);
  ST(st);
  if (e1 != cudaSuccess || e2 != cudaSuccess) return fail(FLSP_ERR_CUDA, "learned reinit: stream join failed");
  ST(launch_apply_delta(h->stream, h->prec, h->m.nb, h->buf[pre], h->buf[out], h->ndofs, hh, h->lrn_cells,
                        ncell, nband, net->y, net->y_ld));
  // the network's next pass (another handle's, in a group) overwrites its
  // output: it waits until this apply has read it
  CU(cudaEventRecord(h->lrn_ev, h->stream));
  CU(cudaStreamWaitEvent(net->stream, h->lrn_ev, 0));
  return FLSP_OK;
}

// A learned reinitialisation with its residual fallback, enqueued without
// a host wait (graph-capturable): the network's result from buf[cur], the
// band cells whose mean ||grad phi| - 1| exceeds o->max_residual, the
// narrow-band HJ sweep (o->fallback, fixed count) from buf[cur] over those
// failed cells (tiles within the narrow band's margin of them; none failed:
// no tile, the launches return at once), and the network's result
// everywhere but the failed cells, which take the sweep's.  The operations
// of flsp_reinit_learned, whose host decides whether to sweep at all;
// h->cur ends on the result.  Band, learned and LDG buffers are allocated
// beforehand.
int enqueue_learned_fallback(flsp_handle* h, flsp_mlp* net, const flsp_learned_opts* o) {
  const int64_t ncell = h->m.ncell;
  const int pre = h->cur, out = other(pre, -1);
  ST(enqueue_learned(h, net, o->band_cells, pre, out));
  ST(launch_residual_flags(h->stream, h->prec, h->dim, h->buf[out], h->m.h[0], h->lrn_cells, ncell,
                           h->lrn_count, o->max_residual, h->lrn_flags, h->lrn_count + 1));
  CU(cudaMemcpyAsync(h->lrn_save, h->buf[out], (size_t)h->ndofs * h->tsize, cudaMemcpyDeviceToDevice, h->stream));
  h->cur = pre;
  int nit = 0;
  const SweepCells failed = {h->lrn_cells, h->lrn_flags, ncell, h->lrn_count};
  ST(run_reinit(h, &o->fallback, &nit, &failed));
  const int hj = h->cur, res = other(hj, -1);
  CU(cudaMemcpyAsync(h->buf[res], h->lrn_save, (size_t)h->ndofs * h->tsize, cudaMemcpyDeviceToDevice, h->stream));
  ST(launch_merge_cells(h->stream, h->prec, h->m.nb, h->buf[hj], h->buf[res], h->lrn_cells, h->lrn_flags, ncell,
                        h->lrn_count));
  ST(launch_learned_totals(h->stream, h->lrn_count, h->lrn_tot, 1));
  h->cur = res;
  return FLSP_OK;
}

// a fallback that graph-replayed periods can carry: enabled by a finite
// positive max_residual, a fixed-count narrow-band sweep (the other modes
// need host decisions)
int learned_graph_fallback(flsp_handle* h, const flsp_learned_opts* o, bool* on) {
  *on = std::isfinite(o->max_residual) && o->max_residual > 0.0;
  if (!*on) return FLSP_OK;
  ST(validate_reinit(h, &o->fallback));
  if (o->fallback.mode != FLSP_REINIT_FIXED || !o->fallback.narrow_band)
    return fail(FLSP_ERR_BAD_ARG, "graph-replayed learned periods need a fixed-count narrow-band fallback sweep "
                                  "(or max_residual = infinity for none)");
  ST(ensure_band_buffers(h));
  if (o->fallback.viscosity > 0.0) ST(ensure_ldg_buffers(h));
  return FLSP_OK;
}

// band cells of the current state: |mean phi| <= band_cells * h; returns the count
int select_band(flsp_handle* h, double band_cells, int64_t* n) {
  ST(ensure_learned_buffers(h, 0));
  ST(launch_band_select(h->stream, h->prec, h->m.nb, h->buf[h->cur], h->m.ncell, band_cells * h->m.h[0],
                        h->lrn_flags, h->lrn_work, h->lrn_cells, h->lrn_count));
  CU(cudaMemcpyAsync(h->lrn_count_host, h->lrn_count, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CU(cudaStreamSynchronize(h->stream));
  *n = h->lrn_count_host[0];
  return FLSP_OK;
}

}  // namespace

// ==================================================================
// C ABI
// ==================================================================
extern "C" {

const char* flsp_last_error(void) { return g_err.c_str(); }
int flsp_version(void) { return 1; }

void flsp_default_dg_opts(flsp_dg_opts* o) {
  if (!o) return;
  o->degree = 1;
  o->basis = FLSP_BASIS_P;
  o->precision = FLSP_FP64;
  o->rk_order = 3;
  o->cfl_max = 0.9;   // AdvectControl: TempoControl(rktvd3, exp, 0.5, 0.9)
  o->device = 0;
}
void flsp_default_reinit_opts(flsp_reinit_opts* o) {
  if (o) fill_reinit_defaults(o);
}
void flsp_default_ls_opts(flsp_ls_opts* o) {
  if (!o) return;
  o->reinit_frequency = 10;
  o->execute_reinit = 1;
  fill_reinit_defaults(&o->reinit);
}

int flsp_create(const flsp_mesh_desc* mesh, const flsp_dg_opts* opts, flsp_handle** out) {
  if (!mesh || !opts || !out) return fail(FLSP_ERR_BAD_ARG, "null argument");
  *out = nullptr;
  if (mesh->dim < 2 || mesh->dim > 3) return fail(FLSP_ERR_BAD_ARG, "dim must be 2 or 3");
  if (!supported_config(mesh->dim, opts->degree))
    return fail(FLSP_ERR_UNSUPPORTED, "degree " + std::to_string(opts->degree) + " not built for dim " +
                                          std::to_string(mesh->dim));
  if (opts->basis != FLSP_BASIS_P && opts->basis != FLSP_BASIS_Q) return fail(FLSP_ERR_BAD_ARG, "bad basis");
  if (opts->precision != FLSP_FP64 && opts->precision != FLSP_FP32) return fail(FLSP_ERR_BAD_ARG, "bad precision");
  if (opts->rk_order < 1 || opts->rk_order > 3) return fail(FLSP_ERR_BAD_ARG, "rk_order must be 1..3");
  if (!(opts->cfl_max > 0.0)) return fail(FLSP_ERR_BAD_ARG, "cfl_max must be positive");
  long long ncell = 1;
  for (int d = 0; d < mesh->dim; ++d) {
    if (mesh->n[d] < 1 || mesh->n[d] > (1 << 20)) return fail(FLSP_ERR_BAD_MESH, "bad cell count");
    if (!(mesh->hi[d] > mesh->lo[d])) return fail(FLSP_ERR_BAD_MESH, "empty box");
    ncell *= mesh->n[d];
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(FLSP_ERR_NO_DEVICE, "no CUDA device visible");
  if (opts->device < 0 || opts->device >= ndev) return fail(FLSP_ERR_BAD_ARG, "bad device ordinal");
  CU(cudaSetDevice(opts->device));
  ST(upload_tables(opts->device));

  flsp_handle* h = new flsp_handle();
  h->dim = mesh->dim;
  h->p = opts->degree;
  h->basis = opts->basis;
  h->prec = opts->precision;
  h->rk = opts->rk_order;
  h->cfl_max = opts->cfl_max;
  h->dev = opts->device;
  h->tsize = h->prec == FLSP_FP64 ? 8 : 4;
  std::memset(&h->m, 0, sizeof(h->m));
  double d2 = 0.0, vol = 1.0;
  for (int d = 0; d < 3; ++d) {
    h->m.n[d] = d < h->dim ? mesh->n[d] : 1;
    h->m.lo[d] = d < h->dim ? mesh->lo[d] : 0.0;
    h->m.h[d] = d < h->dim ? (mesh->hi[d] - mesh->lo[d]) / mesh->n[d] : 1.0;
    if (d < h->dim) { d2 += h->m.h[d] * h->m.h[d]; vol *= h->m.h[d]; }
  }
  h->m.ncell = ncell;
  h->m.vol = vol;
  h->m.diam = std::sqrt(d2);   // cell diagonal (mesh.implement.h:60-71)
  h->m.min_diam = h->m.diam;
  // DoF order inside a cell and its Q-layout map
  const int n1 = h->p + 1, cz = h->dim > 2 ? h->p : 0;
  std::memset(h->m.q2g, -1, sizeof(h->m.q2g));
  std::memset(h->m.g2q, 0, sizeof(h->m.g2q));
  int nb = 0;
  if (h->basis == FLSP_BASIS_Q) {
    for (int c = 0; c <= cz; ++c)
      for (int b = 0; b <= h->p; ++b)
        for (int a = 0; a <= h->p; ++a) {
          const int q = a + n1 * (b + n1 * c);
          h->m.q2g[q] = (signed char)nb;
          h->m.g2q[nb++] = (signed char)q;
        }
  } else {
    for (int c = 0; c <= cz; ++c)
      for (int b = 0; b <= h->p - c; ++b)
        for (int a = 0; a <= h->p - b - c; ++a) {
          const int q = a + n1 * (b + n1 * c);
          h->m.q2g[q] = (signed char)nb;
          h->m.g2q[nb++] = (signed char)q;
        }
  }
  h->m.nb = nb;
  h->ndofs = ncell * nb;

  auto cleanup_fail = [&](int code) {
    flsp_destroy(h);
    return code;
  };
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
    return cleanup_fail(fail(FLSP_ERR_CUDA, "stream creation failed"));
  for (int i = 0; i < 3; ++i)
    // padded: the stage kernel's bulk row copies round their ends up to 16 bytes
    if (cudaMalloc(&h->buf[i], h->ndofs * h->tsize + kStatePad) != cudaSuccess)
      return cleanup_fail(fail(FLSP_ERR_OOM, "state allocation failed"));
  if (cudaMalloc(&h->clk, sizeof(DevClock)) != cudaSuccess ||
      cudaMallocHost(&h->clk_host, sizeof(DevClock)) != cudaSuccess ||
      cudaMalloc(&h->stage64, sizeof(double) * (size_t)h->ndofs * 2 * h->dim) != cudaSuccess ||
      cudaMalloc(&h->red_out, 2 * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&h->ic_dev, sizeof(flsp_ic_desc)) != cudaSuccess ||
      cudaMalloc(&h->flag_dev, sizeof(unsigned int)) != cudaSuccess)
    return cleanup_fail(fail(FLSP_ERR_OOM, "allocation failed"));
  if (h->dim == 2 && (cudaMalloc(&h->weno_list, sizeof(int2) * (size_t)ncell) != cudaSuccess ||
                      cudaMalloc(&h->weno_n, sizeof(unsigned int)) != cudaSuccess))
    return cleanup_fail(fail(FLSP_ERR_OOM, "allocation failed"));
  cudaMemset(h->clk, 0, sizeof(DevClock));
  cudaMemset(h->buf[0], 0, h->ndofs * h->tsize);
  if (mesh->host_cell_order) {
    std::vector<char> seen(ncell, 0);
    for (long long k = 0; k < ncell; ++k) {
      const int64_t v = mesh->host_cell_order[k];
      if (v < 0 || v >= ncell || seen[v]) return cleanup_fail(fail(FLSP_ERR_BAD_MESH, "host_cell_order is not a permutation"));
      seen[v] = 1;
    }
    if (cudaMalloc(&h->perm, sizeof(int64_t) * ncell) != cudaSuccess)
      return cleanup_fail(fail(FLSP_ERR_OOM, "allocation failed"));
    cudaMemcpy(h->perm, mesh->host_cell_order, sizeof(int64_t) * ncell, cudaMemcpyHostToDevice);
  }
  for (int d = 0; d < h->dim; ++d) {
    long long side = 1;
    for (int e = 0; e < h->dim; ++e)
      if (e != d) side *= h->m.n[e];
    h->nbf += 2 * side;
  }
  if (mesh->boundary_ids) {
    h->bid.assign(mesh->boundary_ids, mesh->boundary_ids + h->nbf);
    for (int32_t id : h->bid)
      if (id < 0) return cleanup_fail(fail(FLSP_ERR_BAD_MESH, "negative boundary id"));
  }
  std::memset(&h->vel, 0, sizeof(h->vel));
  std::memset(&h->vel_dev, 0, sizeof(h->vel_dev));
  {
    int st = prepare_kernels(h);
    if (st) return cleanup_fail(st);
  }
  if (cudaDeviceSynchronize() != cudaSuccess) return cleanup_fail(fail(FLSP_ERR_CUDA, "device sync failed"));
  *out = h;
  return FLSP_OK;
}

void flsp_destroy(flsp_handle* h) {
  if (!h) return;
  cudaSetDevice(h->dev);
  if (h->stream) cudaStreamSynchronize(h->stream);
  clear_graphs(h);
  for (int i = 0; i < 3; ++i) if (h->buf[i]) cudaFree(h->buf[i]);
  if (h->snap) cudaFree(h->snap);
  if (h->qbuf) cudaFree(h->qbuf);
  if (h->rdiff) cudaFree(h->rdiff);
  if (h->hj_stab) cudaFree(h->hj_stab);
  if (h->vtab) cudaFree(h->vtab);
  if (h->vtab64) cudaFree(h->vtab64);
  free_fe_velocity(h);
  free_vel_tables(h);
  if (h->optab) cudaFree(h->optab);
  void* lrn[] = {h->lrn_flags, h->lrn_work, h->lrn_cells, h->lrn_count, h->lrn_tot, h->lrn_save, h->lrn_feat,
                 h->nb_flags, h->nb_lists, h->nb_counts};
  for (void* q : lrn)
    if (q) cudaFree(q);
  if (h->lrn_count_host) cudaFreeHost(h->lrn_count_host);
  if (h->lrn_ev) cudaEventDestroy(h->lrn_ev);
  if (h->clk) cudaFree(h->clk);
  if (h->clk_host) cudaFreeHost(h->clk_host);
  if (h->perm) cudaFree(h->perm);
  if (h->curv) cudaFree(h->curv);
  if (h->bc_dev) cudaFree(h->bc_dev);
  if (h->stage64) cudaFree(h->stage64);
  if (h->partial) cudaFree(h->partial);
  if (h->red_out) cudaFree(h->red_out);
  if (h->ic_dev) cudaFree(h->ic_dev);
  if (h->flag_dev) cudaFree(h->flag_dev);
  if (h->weno_list) cudaFree(h->weno_list);
  if (h->weno_n) cudaFree(h->weno_n);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

int flsp_n_dofs(const flsp_handle* h, int64_t* n) {
  if (!h || !n) return fail(FLSP_ERR_BAD_ARG, "null argument");
  *n = h->ndofs;
  return FLSP_OK;
}

int flsp_dofs_per_cell(const flsp_handle* h, int* n) {
  if (!h || !n) return fail(FLSP_ERR_BAD_ARG, "null argument");
  *n = h->m.nb;
  return FLSP_OK;
}

int flsp_set_velocity(flsp_handle* h, const flsp_velocity_desc* v) {
  if (!h || !v) return fail(FLSP_ERR_BAD_ARG, "null argument");
  if (v->n_terms < 0 || v->n_terms > FLSP_MAX_VEL_TERMS) return fail(FLSP_ERR_BAD_ARG, "bad n_terms");
  for (int k = 0; k < v->n_terms; ++k) {
    if (v->terms[k].comp < 0 || v->terms[k].comp >= h->dim) return fail(FLSP_ERR_BAD_ARG, "bad velocity component");
    for (int a = 0; a < 3; ++a)
      if (v->terms[k].f[a].kind < 0 || v->terms[k].f[a].kind > FLSP_F_SINPISQ)
        return fail(FLSP_ERR_BAD_ARG, "bad factor kind");
  }
  if (v->time_kind < 0 || v->time_kind > FLSP_T_ONE_MINUS_EXP) return fail(FLSP_ERR_BAD_ARG, "bad time kind");
  CU(cudaSetDevice(h->dev));
  CU(cudaStreamSynchronize(h->stream));
  free_fe_velocity(h);
  h->vel = *v;
  ST(build_vtab(h));
  h->has_vel = true;
  clear_graphs(h);
  return prepare_kernels(h);
}

int flsp_set_velocity_fe(flsp_handle* h, int degree, const double* values, int64_t n) {
  if (!h || !values) return fail(FLSP_ERR_BAD_ARG, "null argument");
  if (degree < 1 || degree > FLSP_MAX_FE_VEL_DEGREE) return fail(FLSP_ERR_BAD_ARG, "FE velocity degree out of range");
  if (h->batch_member) return fail(FLSP_ERR_UNSUPPORTED, "FE velocity on a batch member");
  long long nn = 1;
  for (int d = 0; d < h->dim; ++d) nn *= (long long)degree * h->m.n[d] + 1;
  if (n != (int64_t)h->dim * nn) return fail(FLSP_ERR_BAD_ARG, "FE velocity size mismatch");
  for (int64_t i = 0; i < n; ++i)
    if (!std::isfinite(values[i])) return fail(FLSP_ERR_BAD_ARG, "non-finite FE velocity value");
  CU(cudaSetDevice(h->dev));
  const bool same = h->fe_pv == degree && h->fe_u64 != nullptr;
  if (!same) {
    // an FE field has no analytic terms: zero tables, time factor 1
    CU(cudaStreamSynchronize(h->stream));
    free_fe_velocity(h);
    std::memset(&h->vel, 0, sizeof(h->vel));
    h->vel.time_kind = FLSP_T_ONE;
    ST(build_vtab(h, false));
    CU(cudaMalloc(&h->fe_u64, (size_t)n * sizeof(double)));
    ST(ensure_vel_tables(h));
    h->fe_pv = degree;
  }
  double gl[kMaxFeVel + 1], xq[8], wq[8], gb[kMaxFeVel + 1][kMaxNQ + 2];
  gauss_lobatto01(degree, gl);
  gauss_rule(h->p + 2, xq, wq);
  std::memset(gb, 0, sizeof(gb));
  for (int a = 0; a <= degree; ++a)
    for (int j = 0; j < h->p + 2; ++j) gb[a][j] = lagrange(degree, gl, a, xq[j]);
  // in place: ordered after the work already queued on the problem's stream
  CU(cudaMemcpyAsync(h->fe_u64, values, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  Ctx c = h->ctx();
  ST(launch_fe_tabulate(c, h->fe_u64, degree, gb, h->tab_q, h->tab_f, h->tab_foff, h->tab_nf));
  CU(cudaMemsetAsync(&h->clk->vd_static, 0, sizeof(double), h->stream));
  ST(launch_fe_static_cfl(c, h->fe_u64, degree, h->clk));
  CU(cudaStreamSynchronize(h->stream));
  h->tab_ok = true;
  h->has_vel = true;
  if (same) return FLSP_OK;
  clear_graphs(h);
  return prepare_kernels(h);
}

int flsp_set_state(flsp_handle* h, const double* coeffs, int64_t n) {
  if (!h || !coeffs) return fail(FLSP_ERR_BAD_ARG, "null argument");
  if (n != h->ndofs) return fail(FLSP_ERR_BAD_ARG, "size mismatch");
  CU(cudaSetDevice(h->dev));
  CU(cudaMemcpyAsync(h->stage64, coeffs, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
  ST(launch_scatter(h->ctx(), h->stage64, h->buf[h->cur], h->perm));
  CU(cudaStreamSynchronize(h->stream));
  return check_finite(h, h->buf[h->cur]);
}

int flsp_get_state(flsp_handle* h, double* coeffs, int64_t n) {
  if (!h || !coeffs) return fail(FLSP_ERR_BAD_ARG, "null argument");
  if (n != h->ndofs) return fail(FLSP_ERR_BAD_ARG, "size mismatch");
  CU(cudaSetDevice(h->dev));
  ST(launch_gather(h->ctx(), h->buf[h->cur], h->stage64, h->perm));
  CU(cudaMemcpyAsync(coeffs, h->stage64, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
  CU(cudaStreamSynchronize(h->stream));
  return FLSP_OK;
}

int flsp_eval_patches(flsp_handle* h, int n_sub, double* values, int64_t n) {
  if (!h || !values) return fail(FLSP_ERR_BAD_ARG, "null argument");
  if (n_sub < 1 || n_sub > 16) return fail(FLSP_ERR_BAD_ARG, "n_sub must be in 1..16");
  const long long ns1 = n_sub + 1, npt = h->dim == 3 ? ns1 * ns1 * ns1 : ns1 * ns1;
  if (n != h->m.ncell * npt) return fail(FLSP_ERR_BAD_ARG, "size mismatch");
  CU(cudaSetDevice(h->dev));
  // the FP64 staging buffer (2 dim n_dofs doubles) holds the corner values
  // of every degree; finer patches may need a buffer of their own
  const bool own = n > (long long)h->ndofs * 2 * h->dim;
  double* dev = h->stage64;
  if (own) CU(cudaMalloc(&dev, sizeof(double) * (size_t)n));
  int st = launch_eval_patches(h->ctx(), h->buf[h->cur], h->perm, n_sub, dev);
  if (st == FLSP_OK) {
    cudaError_t e = cudaMemcpyAsync(values, dev, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) st = fail(FLSP_ERR_CUDA, std::string("eval_patches copy: ") + cudaGetErrorString(e));
  }
  if (own) cudaFree(dev);
  return st;
}

int flsp_material_mix(flsp_handle* const* ls, int n, const double* values, int nq, int smoothing, double* out,
                      int64_t n_out) {
  if (!ls || !values || !out) return fail(FLSP_ERR_BAD_ARG, "null argument");
  if (n < 1 || n > FLSP_MAX_MATERIALS) return fail(FLSP_ERR_BAD_ARG, "1..FLSP_MAX_MATERIALS level sets");
  if (nq < 1 || nq > FLSP_MAX_MIX_QPTS) return fail(FLSP_ERR_BAD_ARG, "n_qpts_1d must be in 1..FLSP_MAX_MIX_QPTS");
  if (smoothing < FLSP_HEAVISIDE_NONE || smoothing > FLSP_HEAVISIDE_SINE)
    return fail(FLSP_ERR_BAD_ARG, "bad Heaviside smoothing");
  const flsp_handle* h0 = ls[0];
  for (int i = 0; i < n; ++i) {
    const flsp_handle* h = ls[i];
    if (!h) return fail(FLSP_ERR_BAD_ARG, "null handle");
    bool same = h->dim == h0->dim && h->dev == h0->dev;
    for (int d = 0; d < 3 && same; ++d)
      same = h->m.n[d] == h0->m.n[d] && h->m.lo[d] == h0->m.lo[d] && h->m.h[d] == h0->m.h[d];
    if (!same) return fail(FLSP_ERR_BAD_ARG, "the level sets of a material stack must share mesh and device");
  }
  for (int i = 0; i <= n; ++i)
    if (!std::isfinite(values[i])) return fail(FLSP_ERR_BAD_ARG, "non-finite material value");
  const long long npt = h0->dim == 3 ? (long long)nq * nq * nq : (long long)nq * nq;
  if (n_out != h0->m.ncell * npt) return fail(FLSP_ERR_BAD_ARG, "size mismatch (n_cells * n_qpts_1d^dim)");
  CU(cudaSetDevice(h0->dev));
  MixArgs a;
  std::memset(&a, 0, sizeof(a));
  double x[FLSP_MAX_MIX_QPTS], w[FLSP_MAX_MIX_QPTS], v[8], dv[8], ddv[8];
  gauss_rule(nq, x, w);
  for (int q = 0; q < nq; ++q) {
    leg_all(kMaxN1, x[q], v, dv, ddv);
    for (int k = 0; k < kMaxN1; ++k) a.L[k][q] = v[k];
  }
  a.perm = h0->perm;
  a.ncell = h0->m.ncell;
  a.n = n;
  a.dim = h0->dim;
  a.nq = nq;
  a.smoothing = smoothing;
  for (int i = 0; i <= n; ++i) a.value[i] = values[i];
  // the kernel runs on the first handle's stream, after that handle's
  // earlier work; the other handles' streams are drained first
  for (int i = 0; i < n; ++i) {
    flsp_handle* h = ls[i];
    MixLevelSet& m = a.ls[i];
    m.phi = h->buf[h->cur];
    m.prec = h->prec;
    m.n1 = h->p + 1;
    m.nb = h->m.nb;
    m.eps = 1.5 * h->m.min_diam;
    std::memcpy(m.q2g, h->m.q2g, sizeof(m.q2g));
    if (i > 0) CU(cudaStreamSynchronize(h->stream));
  }
  // results in the first handle's FP64 staging buffer when it is large
  // enough (2 dim n_dofs doubles), else in a buffer of their own
  flsp_handle* hs = ls[0];
  const bool own = n_out > (long long)hs->ndofs * 2 * hs->dim;
  double* dev = hs->stage64;
  if (own) CU(cudaMalloc(&dev, sizeof(double) * (size_t)n_out));
  int st = launch_material_mix(a, hs->stream, dev);
  if (st == FLSP_OK) {
    cudaError_t e = cudaMemcpyAsync(out, dev, sizeof(double) * (size_t)n_out, cudaMemcpyDeviceToHost, hs->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(hs->stream);
    if (e != cudaSuccess) st = fail(FLSP_ERR_CUDA, std::string("material mix copy: ") + cudaGetErrorString(e));
  }
  if (own) cudaFree(dev);
  return st;
}

int flsp_curvature(flsp_handle* h, int mode, double* kappa, int64_t n) {
  if (!h || !kappa) return fail(FLSP_ERR_BAD_ARG, "null argument");
  if (mode != FLSP_CURV_REFERENCE && mode != FLSP_CURV_NEIGHBOUR) return fail(FLSP_ERR_BAD_ARG, "bad curvature mode");
  if (n != h->ndofs) return fail(FLSP_ERR_BAD_ARG, "size mismatch");
  CU(cudaSetDevice(h->dev));
  double t = 0.0;
  ST(flsp_get_time(h, &t));
  // kept on the device for the exports (CurvatureEstimator's vector)
  if (!h->curv) CU(cudaMalloc(&h->curv, sizeof(double) * (size_t)h->ndofs));
  h->has_curv = false;
  // FP64 staging (2 dim n_dofs doubles) holds the inverse permutation
  int64_t* pos = reinterpret_cast<int64_t*>(h->stage64 + h->ndofs);
  ST(launch_curvature(h->ctx(), h->buf[h->cur], h->perm, pos, mode, h->curv));
  CU(cudaMemcpyAsync(kappa, h->curv, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, h->stream));
  CU(cudaStreamSynchronize(h->stream));
  h->has_curv = true;
  h->curv_time = t;
  return FLSP_OK;
}

int flsp_export_solutions(flsp_handle* h, const char* path, const char* label) {
  if (!h || !path || !label || !label[0]) return fail(FLSP_ERR_BAD_ARG, "null or empty argument");
  for (const char* c = label; *c; ++c)
    if (!((*c >= 'a' && *c <= 'z') || (*c >= 'A' && *c <= 'Z') || (*c >= '0' && *c <= '9') || *c == '_' ||
          *c == '-' || *c == '.'))
      return fail(FLSP_ERR_BAD_ARG, "labels may hold letters, digits, '_', '-' and '.' only");
  CU(cudaSetDevice(h->dev));
  double t = 0.0;
  ST(flsp_get_time(h, &t));
  if (!(t >= 0.0)) return fail(FLSP_ERR_BAD_ARG, "negative time (PVDCollector::append_record)");
  char num[32];
  std::snprintf(num, sizeof(num), "%09zu", h->pvd.size() + 1);
  const std::string master = std::string(label) + "_" + num + ".vtu";
  std::vector<double> values((size_t)h->m.ncell << h->dim);
  ST(flsp_eval_patches(h, 1, values.data(), (int64_t)values.size()));
  flsp_mesh_desc md;
  std::memset(&md, 0, sizeof(md));
  md.dim = h->dim;
  for (int e = 0; e < 3; ++e) {
    md.n[e] = e < h->dim ? h->m.n[e] : 1;
    md.lo[e] = e < h->dim ? h->m.lo[e] : 0.0;
    md.hi[e] = e < h->dim ? h->m.lo[e] + h->m.n[e] * h->m.h[e] : 1.0;
  }
  std::vector<int64_t> order;
  if (h->perm) {
    order.resize((size_t)h->m.ncell);
    CU(cudaMemcpy(order.data(), h->perm, sizeof(int64_t) * order.size(), cudaMemcpyDeviceToHost));
    md.host_cell_order = order.data();
  }
  // the curvature goes along when it belongs to the current time
  // (level_set.implement.h:325-330; TimedPhysicsObject::is_synced_with,
  // numerics::is_nearly_equal with tolerance 1e-12)
  std::vector<double> kvals;
  const double tc = h->curv_time;
  const bool synced = (t < 1.0 && tc < 1.0) ? std::fabs(t - tc) < 1e-12
                                            : std::fabs(t - tc) < 1e-12 * std::max(std::fabs(t), std::fabs(tc));
  if (h->has_curv && synced) {
    kvals.resize(values.size());
    Ctx c64 = h->ctx();
    c64.prec = FLSP_FP64;   // the curvature vector is FP64, already in host cell order
    ST(launch_eval_patches(c64, h->curv, nullptr, 1, h->stage64));
    CU(cudaMemcpyAsync(kvals.data(), h->stage64, sizeof(double) * kvals.size(), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
  }
  const std::string klabel = std::string(label) + "Curvature";
  ST(write_vtu_file(&md, 1, values.data(), label, (std::string(path) + master).c_str(),
                    kvals.empty() ? nullptr : kvals.data(), klabel.c_str()));
  h->pvd.emplace_back(t, master);
  std::vector<double> times;
  std::vector<const char*> files;
  for (const auto& r : h->pvd) {
    times.push_back(r.first);
    files.push_back(r.second.c_str());
  }
  return write_pvd_file((std::string(path) + label + ".pvd").c_str(), (int)h->pvd.size(), times.data(), files.data());
}

int flsp_set_time(flsp_handle* h, double t) {
  if (!h) return fail(FLSP_ERR_BAD_ARG, "null handle");
  CU(cudaSetDevice(h->dev));
  ST(sync_clock(h));
  h->clk_host->t = t;
  CU(cudaMemcpyAsync(h->clk, h->clk_host, sizeof(DevClock), cudaMemcpyHostToDevice, h->stream));
  CU(cudaStreamSynchronize(h->stream));
  return FLSP_OK;
}

int flsp_get_time(const flsp_handle* hc, double* t) {
  flsp_handle* h = const_cast<flsp_handle*>(hc);
  if (!h || !t) return fail(FLSP_ERR_BAD_ARG, "null argument");
  CU(cudaSetDevice(h->dev));
  ST(sync_clock(h));
  *t = h->clk_host->t;
  return FLSP_OK;
}

int flsp_set_dirichlet(flsp_handle* h, int boundary_id, double value) {
  if (!h) return fail(FLSP_ERR_BAD_ARG, "null handle");
  if (boundary_id <= 0)
    return fail(FLSP_ERR_BAD_ARG, "Dirichlet conditions need a boundary id > 0 (id 0 never takes one)");
  if (!std::isfinite(value)) return fail(FLSP_ERR_BAD_ARG, "non-finite boundary value");
  if (h->batch_member) return fail(FLSP_ERR_UNSUPPORTED, "Dirichlet conditions on a batch member");
  h->dirichlet[boundary_id] = value;
  return rebuild_bc(h);
}

int flsp_clear_dirichlet(flsp_handle* h) {
  if (!h) return fail(FLSP_ERR_BAD_ARG, "null handle");
  h->dirichlet.clear();
  return rebuild_bc(h);
}

int flsp_get_step_count(const flsp_handle* hc, int64_t* n_substeps) {
  flsp_handle* h = const_cast<flsp_handle*>(hc);
  if (!h || !n_substeps) return fail(FLSP_ERR_BAD_ARG, "null argument");
  CU(cudaSetDevice(h->dev));
  ST(sync_clock(h));
  *n_substeps = h->clk_host->n_substeps;
  return FLSP_OK;
}

int flsp_project_ic(flsp_handle* h, const flsp_ic_desc* ic) {
  if (!h || !ic) return fail(FLSP_ERR_BAD_ARG, "null argument");
  if (ic->n_nodes < 1 || ic->n_nodes > FLSP_MAX_IC_NODES || ic->root < 0 || ic->root >= ic->n_nodes ||
      ic->n_waves < 0 || ic->n_waves > FLSP_MAX_IC_WAVES)
    return fail(FLSP_ERR_BAD_ARG, "bad IC description");
  for (int k = 0; k < ic->n_nodes; ++k) {
    const flsp_ic_node& nd = ic->nodes[k];
    if (nd.kind < 0 || nd.kind > FLSP_IC_INTERSECT) return fail(FLSP_ERR_BAD_ARG, "bad IC node kind");
    if (nd.kind >= FLSP_IC_UNION && (nd.a < 0 || nd.a >= k || nd.b < 0 || nd.b >= k))
      return fail(FLSP_ERR_BAD_ARG, "IC operands must precede their node");
    if (nd.kind == FLSP_IC_HEIGHT && ((int)nd.p[0] < 0 || (int)nd.p[0] >= h->dim))
      return fail(FLSP_ERR_BAD_ARG, "bad height-function axis");
  }
  CU(cudaSetDevice(h->dev));
  CU(cudaMemcpyAsync(h->ic_dev, ic, sizeof(flsp_ic_desc), cudaMemcpyHostToDevice, h->stream));
  ST(launch_project_ic(h->ctx(), h->ic_dev, h->buf[h->cur]));
  CU(cudaStreamSynchronize(h->stream));
  return FLSP_OK;
}

int flsp_snapshot(flsp_handle* h) {
  if (!h) return fail(FLSP_ERR_BAD_ARG, "null handle");
  CU(cudaSetDevice(h->dev));
  if (!h->snap) CU(cudaMalloc(&h->snap, h->ndofs * h->tsize));
  CU(cudaMemcpyAsync(h->snap, h->buf[h->cur], h->ndofs * h->tsize, cudaMemcpyDeviceToDevice, h->stream));
  CU(cudaStreamSynchronize(h->stream));
  h->has_snap = true;
  return FLSP_OK;
}

int flsp_advect_rhs(flsp_handle* h, double t, double* phidot, int64_t n) {
  if (!h || !phidot) return fail(FLSP_ERR_BAD_ARG, "null argument");
  if (n != h->ndofs) return fail(FLSP_ERR_BAD_ARG, "size mismatch");
  if (!h->has_vel) return fail(FLSP_ERR_BAD_ARG, "velocity not set");
  CU(cudaSetDevice(h->dev));
  const int tmp = (h->cur + 1) % 3;
  ST(launch_adv_stage(h->ctx(), h->veldev(), h->buf[h->cur], h->buf[h->cur], h->buf[tmp], nullptr, 0,
                      kRhsOnly, host_time_factor(h->vel, t), h->adv_tile));
  ST(launch_gather(h->ctx(), h->buf[tmp], h->stage64, h->perm));
  CU(cudaMemcpyAsync(phidot, h->stage64, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
  CU(cudaStreamSynchronize(h->stream));
  return FLSP_OK;
}

// AdvectSimulator::advance_time(time_step, compute_single_cycle)
int flsp_advance(flsp_handle* h, double time_step, int single_cycle, double* advanced) {
  if (!h) return fail(FLSP_ERR_BAD_ARG, "null handle");
  if (!h->has_vel) return fail(FLSP_ERR_BAD_ARG, "velocity not set");
  if (!(time_step >= 0.0) || !std::isfinite(time_step)) return fail(FLSP_ERR_BAD_ARG, "bad time step");
  CU(cudaSetDevice(h->dev));
  ST(launch_adv_clock_horizon(h->stream, h->clk, time_step));
  double cum = 0.0;
  long long guard = 0;
  do {
    ST(enqueue_adv_step(h, false));
    ST(sync_clock(h));
    cum = h->clk_host->scratch[1];
    if (!std::isfinite(h->clk_host->dt)) return fail(FLSP_ERR_NONFINITE, "non-finite time step");
    if (single_cycle) break;
    if (++guard > 100000000LL) return fail(FLSP_ERR_TIMEOUT, "substep loop did not terminate");
  } while (!(std::fabs(cum - time_step) <= 2.220446049250313e-16));
  if (advanced) *advanced = cum;
  return FLSP_OK;
}

int flsp_advance_steps(flsp_handle* h, int n_steps, double t_end) {
  if (!h) return fail(FLSP_ERR_BAD_ARG, "null handle");
  if (!h->has_vel) return fail(FLSP_ERR_BAD_ARG, "velocity not set");
  if (n_steps < 0) return fail(FLSP_ERR_BAD_ARG, "negative step count");
  CU(cudaSetDevice(h->dev));
  ST(sync_clock(h));
  const double horizon = std::isfinite(t_end) ? t_end - h->clk_host->t : INFINITY;
  ST(launch_adv_clock_horizon(h->stream, h->clk, horizon));
  for (int i = 0; i < n_steps; ++i) ST(enqueue_adv_step(h));
  CU(cudaStreamSynchronize(h->stream));
  return FLSP_OK;
}

int flsp_reinit(flsp_handle* h, const flsp_reinit_opts* o, int* n_iter) {
  if (!h) return fail(FLSP_ERR_BAD_ARG, "null handle");
  CU(cudaSetDevice(h->dev));
  int st = run_reinit(h, o, n_iter);
  cudaStreamSynchronize(h->stream);
  return st;
}

int flsp_hj_gradients(flsp_handle* h, double* grads, int64_t n) {
  if (!h || !grads) return fail(FLSP_ERR_BAD_ARG, "null argument");
  if (n != 2 * h->dim * h->ndofs) return fail(FLSP_ERR_BAD_ARG, "size mismatch (2*dim*n_dofs)");
  CU(cudaSetDevice(h->dev));
  void* tmp = nullptr;
  CU(cudaMalloc(&tmp, (size_t)n * h->tsize));
  int st = launch_hj(h->ctx(), h->buf[h->cur], h->buf[h->cur], tmp, nullptr, kHJGradients, 1, 0.0,
                     h->ndofs, h->hj_tile);
  for (int b = 0; b < 2 * h->dim && st == FLSP_OK; ++b)
    st = launch_gather(h->ctx(), (const char*)tmp + (size_t)b * h->ndofs * h->tsize,
                       h->stage64 + b * h->ndofs, h->perm);
  if (st == FLSP_OK) {
    cudaMemcpyAsync(grads, h->stage64, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) st = fail(FLSP_ERR_CUDA, "sync failed");
  }
  cudaFree(tmp);
  return st;
}

int flsp_weno_limit(flsp_handle* h, int* n_troubled) {
  if (!h) return fail(FLSP_ERR_BAD_ARG, "null handle");
  CU(cudaSetDevice(h->dev));
  CU(cudaMemsetAsync(h->flag_dev, 0, sizeof(unsigned int), h->stream));
  const int dst = (h->cur + 1) % 3;
  ST(launch_weno(h->ctx(), h->buf[h->cur], h->buf[dst], h->flag_dev, h->weno_list, h->weno_n));
  unsigned int cnt = 0;
  CU(cudaMemcpyAsync(&cnt, h->flag_dev, sizeof(cnt), cudaMemcpyDeviceToHost, h->stream));
  CU(cudaStreamSynchronize(h->stream));
  h->cur = dst;
  if (n_troubled) *n_troubled = (int)cnt;
  return FLSP_OK;
}

// LevelSetSurface::advance_time(time_step, compute_single_step)
int flsp_ls_advance(flsp_handle* h, const flsp_ls_opts* o, double time_step, int single_step,
                    double* advanced) {
  if (!h || !o) return fail(FLSP_ERR_BAD_ARG, "null argument");
  if (o->reinit_frequency < 1) return fail(FLSP_ERR_BAD_ARG, "reinit_frequency must be >= 1");
  double cum = 0.0;
  long long guard = 0;
  do {
    double sub = 0.0;
    ST(flsp_advance(h, time_step, 1, &sub));
    h->n_since_reinit++;
    if (o->execute_reinit && h->n_since_reinit == o->reinit_frequency) {
      int nit = 0;
      ST(flsp_reinit(h, &o->reinit, &nit));
      if (nit) h->n_since_reinit = 0;
    }
    cum += sub;
    time_step -= sub;
    if (++guard > 100000000LL) return fail(FLSP_ERR_TIMEOUT, "level-set loop did not terminate");
  } while (!(std::fabs(time_step) <= 2.220446049250313e-16) && !single_step);
  if (advanced) *advanced = cum;
  return FLSP_OK;
}

// n_steps advection substeps, fixed-count reinit every reinit_frequency
// steps; one reinit period is captured into a CUDA graph and replayed
// one reinit period on the handle's stream: `steps` advection substeps, then
// the fixed-count reinit (graph-capturable; band buffers allocated before)
int enqueue_period(flsp_handle* h, const flsp_reinit_opts* ro, int steps) {
  for (int s = 0; s < steps; ++s) ST(enqueue_adv_step(h));
  const bool limiter = reinit_limiter(h, ro);
  const int phi0 = h->cur;
  if (ro->narrow_band) {
    const int stb = band_begin(h, ro, phi0, limiter);
    if (stb) {
      for (int k = 0; k < 3; ++k) h->nb_use[k] = false;
      return stb;
    }
  }
  int st = launch_hj_clock_reset(h->stream, h->clk);
  if (st == FLSP_OK)
    st = launch_hj(h->ctx(), h->buf[phi0], h->buf[phi0], nullptr, h->clk, kHJCflOnly, ro->rk_order, 0.0,
                   h->ndofs, h->hj_tile);
  for (int k = 0; k < ro->n_pseudo_steps && st == FLSP_OK; ++k) st = enqueue_hj_step(h, ro, phi0, limiter);
  if (ro->narrow_band) {
    const int st2 = band_end(h, phi0);
    if (st == FLSP_OK) st = st2;
  }
  return st;
}

int flsp_ls_run_steps(flsp_handle* h, const flsp_ls_opts* o, int n_steps) {
  if (!h || !o) return fail(FLSP_ERR_BAD_ARG, "null argument");
  if (!h->has_vel) return fail(FLSP_ERR_BAD_ARG, "velocity not set");
  if (n_steps < 0 || o->reinit_frequency < 1) return fail(FLSP_ERR_BAD_ARG, "bad step counts");
  flsp_reinit_opts ro = o->reinit;
  if (o->execute_reinit) {
    if (ro.mode != FLSP_REINIT_FIXED)
      return fail(FLSP_ERR_BAD_ARG, "flsp_ls_run_steps needs a fixed-count reinit (FLSP_REINIT_FIXED)");
    ST(validate_reinit(h, &ro));
    if (ro.viscosity > 0.0) ST(ensure_ldg_buffers(h));
  }
  CU(cudaSetDevice(h->dev));
  ST(launch_adv_clock_horizon(h->stream, h->clk, INFINITY));
  int done = 0;
  while (done < n_steps) {
    const int to_reinit = o->execute_reinit ? o->reinit_frequency - h->n_since_reinit : n_steps - done;
    if (to_reinit <= 0) { h->n_since_reinit = 0; continue; }
    if (done + to_reinit <= n_steps && o->execute_reinit) {
      // a full period: replay (or capture) the graph for this buffer role
      // graph key: buffer role, period length and every reinit option
      // (kernel arguments are baked into the captured graph)
      unsigned long long key = 1469598103934665603ull;
      auto mix = [&key](const void* p, size_t n) {
        const unsigned char* b = (const unsigned char*)p;
        for (size_t i = 0; i < n; ++i) { key ^= b[i]; key *= 1099511628211ull; }
      };
      mix(&h->cur, sizeof(h->cur));
      mix(&to_reinit, sizeof(to_reinit));
      mix(&ro, sizeof(ro));
      auto it = h->graphs.find(key);
      if (it == h->graphs.end()) {
        const int cur0 = h->cur;
        if (ro.narrow_band) ST(ensure_band_buffers(h));
        cudaGraph_t g = nullptr;
        CU(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        const int st = enqueue_period(h, &ro, to_reinit);
        cudaError_t ce = cudaStreamEndCapture(h->stream, &g);
        if (st != FLSP_OK) { if (g) cudaGraphDestroy(g); h->cur = cur0; return st; }
        if (ce != cudaSuccess) return fail(FLSP_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
        GraphEntry ge;
        ge.cur_after = h->cur;
        h->cur = cur0;
        CU(cudaGraphInstantiate(&ge.exec, g, 0));
        cudaGraphDestroy(g);
        it = h->graphs.emplace(key, ge).first;
      }
      CU(cudaGraphLaunch(it->second.exec, h->stream));
      h->cur = it->second.cur_after;
      done += to_reinit;
      h->n_since_reinit = 0;
    } else {
      const int k = std::min(to_reinit, n_steps - done);
      for (int s = 0; s < k; ++s) ST(enqueue_adv_step(h));
      done += k;
      h->n_since_reinit += k;
    }
  }
  return FLSP_OK;
}

int flsp_sync(flsp_handle* h) {
  if (!h) return fail(FLSP_ERR_BAD_ARG, "null handle");
  CU(cudaSetDevice(h->dev));
  return sync_clock(h);
}

int flsp_stream(const flsp_handle* h, void** stream) {
  if (!h || !stream) return fail(FLSP_ERR_BAD_ARG, "null argument");
  *stream = (void*)h->stream;
  return FLSP_OK;
}

int flsp_time_kernel(flsp_handle* h, int which, int reps, double* ms_per_launch) {
  if (!h || !ms_per_launch || reps < 1) return fail(FLSP_ERR_BAD_ARG, "bad argument");
  if (which == 0 && !h->has_vel) return fail(FLSP_ERR_BAD_ARG, "velocity not set");
  CU(cudaSetDevice(h->dev));
  CU(cudaStreamSynchronize(h->stream));
  const int x = h->cur, y = (h->cur + 1) % 3, z = (h->cur + 2) % 3;
  if (which == 0) {
    // a valid substep on the clock (idempotent: the CFL maximum is a max)
    AdvClockArgs ca;
    ca.cfl_max = h->cfl_max;
    ca.scale = adv_cfl_scaling(h->p);
    ca.tkind = h->vel.time_kind;
    ca.ta = h->vel.ta;
    ca.tb = h->vel.tb;
    ca.rk = h->rk;
    ca.step_count = 1;
    ST(launch_adv_clock_horizon(h->stream, h->clk, INFINITY));
    ST(launch_adv_clock_begin(h->stream, h->clk, ca));
  } else {
    ST(launch_hj_clock_reset(h->stream, h->clk));
    // the pseudo-steps' smooth-sign table (phi0 = the timed input)
    ST(launch_hj(h->ctx(), h->buf[x], h->buf[x], nullptr, h->clk, kHJCflOnly, 1, 0.0, h->ndofs, h->hj_tile));
  }
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0));
  CU(cudaEventCreate(&e1));
  int st = FLSP_OK;
  // one untimed round, then the timed repetitions
  for (int pass = 0; pass < 2 && st == FLSP_OK; ++pass) {
    if (pass == 1) cudaEventRecord(e0, h->stream);
    const int n = pass == 0 ? 1 : reps;
    for (int r = 0; r < n && st == FLSP_OK; ++r) {
      if (which == 0) {
        st = stage(h, h->buf[x], h->buf[x], h->buf[y], 0, kRK3a);
        if (st == FLSP_OK) st = stage(h, h->buf[y], h->buf[x], h->buf[z], 1, kRK3b);
        if (st == FLSP_OK) st = stage(h, h->buf[z], h->buf[x], h->buf[y], 2, kRK3c);
      } else {
        st = launch_hj(h->ctx(), h->buf[x], h->buf[x], h->buf[y], h->clk, kHJStep, 1, 0.0, h->ndofs,
                       h->hj_tile);
      }
    }
  }
  cudaEventRecord(e1, h->stream);
  cudaError_t ce = cudaEventSynchronize(e1);
  float ms = 0.f;
  if (st == FLSP_OK && ce == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st) return st;
  if (ce != cudaSuccess) return fail(FLSP_ERR_CUDA, cudaGetErrorString(ce));
  *ms_per_launch = (double)ms / (double)(reps * (which == 0 ? 3 : 1));
  return FLSP_OK;
}

int flsp_autotune(flsp_handle* h, int reps, int* tile, int* cand_tiles, double* cand_ms, int* n_cand) {
  if (!h || reps < 1) return fail(FLSP_ERR_BAD_ARG, "bad argument");
  if (!h->has_vel) return fail(FLSP_ERR_BAD_ARG, "velocity not set");
  CU(cudaSetDevice(h->dev));
  // the timing runs advance the device clock's substep state: keep a copy
  ST(sync_clock(h));
  const DevClock saved_clk = *h->clk_host;
  const int saved[3] = {h->adv_tile[0], h->adv_tile[1], h->adv_tile[2]};
  int cand[FLSP_MAX_TILE_CANDIDATES][3], nc = 0, best = -1;
  double best_ms = INFINITY;
  const Ctx c = h->ctx();
  ST(adv_tile_candidates(c, h->veldev(), cand, &nc));
  int st = FLSP_OK;
  for (int i = 0; i < nc && st == FLSP_OK; ++i) {
    if (cand_tiles)
      for (int d = 0; d < 3; ++d) cand_tiles[3 * i + d] = cand[i][d];
    if (cand_ms) cand_ms[i] = NAN;
    if (adv_prepare(c, h->veldev(), cand[i]) != FLSP_OK) continue;   // does not fit this GPU
    for (int d = 0; d < 3; ++d) h->adv_tile[d] = cand[i][d];
    double ms = 0.0;
    st = flsp_time_kernel(h, 0, reps, &ms);
    if (cand_ms && st == FLSP_OK) cand_ms[i] = ms;
    if (st == FLSP_OK && ms < best_ms) {
      best_ms = ms;
      best = i;
    }
  }
  const int* pick = (st == FLSP_OK && best >= 0) ? cand[best] : saved;
  for (int d = 0; d < 3; ++d) h->adv_tile[d] = pick[d];
  const int st2 = adv_prepare(c, h->veldev(), h->adv_tile);
  clear_graphs(h);
  *h->clk_host = saved_clk;
  CU(cudaMemcpyAsync(h->clk, h->clk_host, sizeof(DevClock), cudaMemcpyHostToDevice, h->stream));
  CU(cudaStreamSynchronize(h->stream));
  if (st) return st;
  if (best < 0) return fail(FLSP_ERR_UNSUPPORTED, "no stage tile fits");
  if (st2) return st2;
  if (tile)
    for (int d = 0; d < 3; ++d) tile[d] = h->adv_tile[d];
  if (n_cand) *n_cand = nc;
  return FLSP_OK;
}

int flsp_stage_tile(const flsp_handle* h, int* tile) {
  if (!h || !tile) return fail(FLSP_ERR_BAD_ARG, "null argument");
  for (int d = 0; d < 3; ++d) tile[d] = h->adv_tile[d];
  return FLSP_OK;
}

int flsp_reduce(flsp_handle* h, int which, const flsp_ic_desc* ic, double* out) {
  if (!h || !out) return fail(FLSP_ERR_BAD_ARG, "null argument");
  CU(cudaSetDevice(h->dev));
  const bool need_ic = which == FLSP_RED_MASS_ERROR || which == FLSP_RED_L2_ERROR_IC ||
                       which == FLSP_RED_L1_INTERFACE_IC;
  const bool need_ref = which == FLSP_RED_L1_INTERFACE || which == FLSP_RED_MEAN_ABS_DIFF;
  if (which < 0 || which > FLSP_RED_MASS_SHARP) return fail(FLSP_ERR_BAD_ARG, "bad reduction kind");
  if (need_ic) {
    if (!ic) return fail(FLSP_ERR_BAD_ARG, "reduction needs an IC");
    CU(cudaMemcpyAsync(h->ic_dev, ic, sizeof(flsp_ic_desc), cudaMemcpyHostToDevice, h->stream));
  }
  if (need_ref && !h->has_snap) return fail(FLSP_ERR_BAD_ARG, "reduction needs flsp_snapshot first");
  double r[2];
  ST(reduce_dev(h, which, h->buf[h->cur], need_ref ? h->snap : nullptr, need_ic, r));
  switch (which) {
    case FLSP_RED_MASS_ERROR: *out = (r[0] - r[1]) / r[1]; break;
    case FLSP_RED_MEAN_ABS_DIFF: *out = r[0] / (double)h->ndofs; break;
    case FLSP_RED_GRAD_DEVIATION: *out = r[0] / r[1]; break;
    case FLSP_RED_L2_ERROR_IC: *out = std::sqrt(r[0]); break;
    default: *out = r[0];
  }
  return FLSP_OK;
}

// ---- learned reinitialisation (no counterpart in the reference)
int flsp_mlp_collect(flsp_mlp* net, flsp_handle* h, double band_cells, const flsp_reinit_opts* target,
                     int64_t* n_added) {
  if (!net || !h || !target) return fail(FLSP_ERR_BAD_ARG, "null argument");
  if (!(band_cells > 0.0)) return fail(FLSP_ERR_BAD_ARG, "band_cells must be positive");
  CU(cudaSetDevice(h->dev));
  ST(learned_check(h, net));
  ST(validate_reinit(h, target));
  int64_t n = 0;
  ST(select_band(h, band_cells, &n));
  ST(mlp_ensure_pairs(net, net->n_pairs + n));
  const double hh = h->m.h[0];
  ST(launch_patch_features(h->stream, h->prec, h->dim, h->buf[h->cur], h->m.n, hh, h->lrn_cells, n, nullptr,
                           net->feat + net->n_pairs * net->n_in));
  CU(cudaMemcpyAsync(h->lrn_save, h->buf[h->cur], (size_t)h->ndofs * h->tsize, cudaMemcpyDeviceToDevice, h->stream));
  int nit = 0;
  ST(run_reinit(h, target, &nit));
  ST(launch_patch_targets(h->stream, h->prec, h->m.nb, h->lrn_save, h->buf[h->cur], hh, h->lrn_cells, n,
                          net->targ + net->n_pairs * net->n_out));
  CU(cudaStreamSynchronize(h->stream));
  net->n_pairs += n;
  if (n_added) *n_added = n;
  return FLSP_OK;
}

void flsp_default_learned_opts(flsp_learned_opts* o) {
  if (!o) return;
  o->band_cells = 6.0;
  o->max_residual = 0.05;
  fill_reinit_defaults(&o->fallback);
  o->fallback.mode = FLSP_REINIT_FIXED;
  o->fallback.n_pseudo_steps = 20;
  o->fallback.narrow_band = 1;   // the sweep only needs to cover the band
  o->fallback.band_cells = o->band_cells;
}

int flsp_reinit_learned(flsp_handle* h, flsp_mlp* net, const flsp_learned_opts* o, flsp_learned_stats* stats) {
  if (!h || !net || !o) return fail(FLSP_ERR_BAD_ARG, "null argument");
  if (!(o->band_cells > 0.0) || !(o->max_residual > 0.0)) return fail(FLSP_ERR_BAD_ARG, "bad learned options");
  CU(cudaSetDevice(h->dev));
  ST(learned_check(h, net));
  ST(validate_reinit(h, &o->fallback));
  // every launch is sized for all cells; the band's size stays on the device
  // (kernels past it return at once), so the host waits only once, for the
  // counts that decide the fallback
  const int64_t ncell = h->m.ncell;
  ST(ensure_learned_buffers(h, ncell));
  ST(mlp_ensure_cap(net, ncell));
  const double hh = h->m.h[0];
  const int pre = h->cur;
  const int out = other(pre, -1);
  const int* nband = h->lrn_count;
  ST(enqueue_learned(h, net, o->band_cells, pre, out));
  // band cells whose result is not distance-like enough take the HJ sweep
  ST(launch_residual_flags(h->stream, h->prec, h->dim, h->buf[out], hh, h->lrn_cells, ncell, nband,
                           o->max_residual, h->lrn_flags, h->lrn_count + 1));
  ST(launch_learned_totals(h->stream, h->lrn_count, h->lrn_tot, 1));
  CU(cudaMemcpyAsync(h->lrn_count_host, h->lrn_count, 2 * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CU(cudaMemcpyAsync(h->lrn_count_host + 2, net->err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CU(cudaStreamSynchronize(h->stream));
  if (h->lrn_count_host[2]) return fail(FLSP_ERR_TIMEOUT, "a tensor-core kernel's pipeline wait ran out");
  flsp_learned_stats stl = {h->lrn_count_host[0], h->lrn_count_host[1], 0};
  if (stl.n_fallback > 0) {
    // keep the network's result, run the sweep from the pre-reinit state,
    // then put the network's result back everywhere but the flagged cells
    CU(cudaMemcpyAsync(h->lrn_save, h->buf[out], (size_t)h->ndofs * h->tsize, cudaMemcpyDeviceToDevice, h->stream));
    h->cur = pre;
    int nit = 0;
    const SweepCells failed = {h->lrn_cells, h->lrn_flags, stl.n_band, nullptr};
    ST(run_reinit(h, &o->fallback, &nit, o->fallback.narrow_band ? &failed : nullptr));
    const int hj = h->cur;
    const int res = other(hj, -1);
    CU(cudaMemcpyAsync(h->buf[res], h->lrn_save, (size_t)h->ndofs * h->tsize, cudaMemcpyDeviceToDevice, h->stream));
    ST(launch_merge_cells(h->stream, h->prec, h->m.nb, h->buf[hj], h->buf[res], h->lrn_cells, h->lrn_flags,
                          stl.n_band, nullptr));
    h->cur = res;
    stl.hj_ran = 1;
    CU(cudaStreamSynchronize(h->stream));
  } else {
    h->cur = out;
  }
  h->n_since_reinit = 0;
  if (stats) *stats = stl;
  return FLSP_OK;
}

int flsp_learned_totals(flsp_handle* h, int64_t* n_band, int64_t* n_fallback, int reset) {
  if (!h) return fail(FLSP_ERR_BAD_ARG, "null handle");
  CU(cudaSetDevice(h->dev));
  unsigned long long t[2] = {0, 0};
  if (h->lrn_tot) {
    CU(cudaMemcpyAsync(t, h->lrn_tot, sizeof(t), cudaMemcpyDeviceToHost, h->stream));
    if (reset) CU(cudaMemsetAsync(h->lrn_tot, 0, sizeof(t), h->stream));
    CU(cudaStreamSynchronize(h->stream));
  }
  if (n_band) *n_band = (int64_t)t[0];
  if (n_fallback) *n_fallback = (int64_t)t[1];
  return FLSP_OK;
}

int flsp_ls_run_steps_learned(flsp_handle* h, flsp_mlp* net, const flsp_learned_opts* o, int reinit_frequency,
                              int n_steps) {
  if (!h || !net || !o) return fail(FLSP_ERR_BAD_ARG, "null argument");
  if (!h->has_vel) return fail(FLSP_ERR_BAD_ARG, "velocity not set");
  if (n_steps < 0 || reinit_frequency < 1) return fail(FLSP_ERR_BAD_ARG, "bad step counts");
  if (!(o->band_cells > 0.0)) return fail(FLSP_ERR_BAD_ARG, "bad learned options");
  CU(cudaSetDevice(h->dev));
  ST(learned_check(h, net));
  // buffers and attributes before any capture
  ST(ensure_learned_buffers(h, h->m.ncell));
  ST(mlp_ensure_cap(net, h->m.ncell));
  bool fb = false;
  ST(learned_graph_fallback(h, o, &fb));
  ST(launch_adv_clock_horizon(h->stream, h->clk, INFINITY));
  int done = 0;
  while (done < n_steps) {
    const int to_reinit = reinit_frequency - h->n_since_reinit;
    if (to_reinit <= 0) { h->n_since_reinit = 0; continue; }
    if (done + to_reinit <= n_steps) {
      // a full period, replayed from its graph (key: buffer role, period,
      // band width, the network and its buffers)
      unsigned long long key = 0x6c6561726e656421ull;
      auto mix = [&key](const void* p, size_t n) {
        const unsigned char* b = (const unsigned char*)p;
        for (size_t i = 0; i < n; ++i) { key ^= b[i]; key *= 1099511628211ull; }
      };
      mix(&h->cur, sizeof(h->cur));
      mix(&to_reinit, sizeof(to_reinit));
      mix(&o->band_cells, sizeof(o->band_cells));
      mix(&net->uid, sizeof(net->uid));
      mix(&net->cap, sizeof(net->cap));
      mix(&fb, sizeof(fb));
      if (fb) {
        mix(&o->max_residual, sizeof(o->max_residual));
        mix(&o->fallback, sizeof(o->fallback));
      }
      auto it = h->graphs.find(key);
      if (it == h->graphs.end()) {
        const int cur0 = h->cur;
        cudaGraph_t g = nullptr;
        CU(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        int st = FLSP_OK;
        for (int s = 0; s < to_reinit && st == FLSP_OK; ++s) st = enqueue_adv_step(h);
        if (st == FLSP_OK && fb) {
          st = enqueue_learned_fallback(h, net, o);
        } else if (st == FLSP_OK) {
          const int pre = h->cur, out = other(pre, -1);
          st = enqueue_learned(h, net, o->band_cells, pre, out);
          if (st == FLSP_OK) st = launch_learned_totals(h->stream, h->lrn_count, h->lrn_tot, 0);
          if (st == FLSP_OK) h->cur = out;
        }
        cudaError_t ce = cudaStreamEndCapture(h->stream, &g);
        if (st != FLSP_OK) { if (g) cudaGraphDestroy(g); h->cur = cur0; return st; }
        if (ce != cudaSuccess) { h->cur = cur0; return fail(FLSP_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce)); }
        GraphEntry ge;
        ge.cur_after = h->cur;
        h->cur = cur0;
        CU(cudaGraphInstantiate(&ge.exec, g, 0));
        cudaGraphDestroy(g);
        it = h->graphs.emplace(key, ge).first;
      }
      CU(cudaGraphLaunch(it->second.exec, h->stream));
      h->cur = it->second.cur_after;
      done += to_reinit;
      h->n_since_reinit = 0;
    } else {
      const int k = n_steps - done;
      for (int s = 0; s < k; ++s) ST(enqueue_adv_step(h));
      done += k;
      h->n_since_reinit += k;
    }
  }
  return FLSP_OK;
}

// ---- batched problems (no counterpart in the reference: one problem per
// simulator object there).  Many independent 2D problems advance in one
// persistent launch per RK stage and per reinit pseudo-step, periods
// replayed from captured CUDA graphs, tile shapes from the autotuner.
}  // extern "C"

struct flsp_batch {
  int dev = 0, prec = 0, rk = 3;
  cudaStream_t stream = nullptr;
  std::vector<flsp_handle*> h;
  int cur = 0;             // common buffer role of every problem
  int n_since_reinit = 0;
  bool tuned = false;
  int adv_tile[3] = {16, 16, 1}, hj_tile[3] = {16, 8, 1};
  flsp_batch_tuning tuning;
  // device descriptors and work lists for the current tiles
  BatchProb* probs = nullptr;
  int2* items_adv = nullptr;
  int2* items_hj = nullptr;
  int2* items_weno = nullptr;
  int n_adv = 0, n_hj = 0, n_weno = 0;
  // per kernel kind (adv, hj, weno) and degree 1..3: the items' range in the
  // kind's list (sorted by degree), shared memory, persistent grid
  int deg_off[3][4] = {}, deg_cnt[3][4] = {};
  int prob_off[4] = {}, prob_cnt[4] = {};   // per degree: its range of the descriptors
  size_t deg_smem[3][4] = {};
  int deg_grid[3][4] = {};
  bool built = false;
  std::map<unsigned long long, GraphEntry> graphs;
  // the degrees' launches of a stage run side by side: one stream per
  // degree, forked from and joined back into the batch stream
  cudaStream_t side[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t ev_fork = nullptr;
  cudaEvent_t ev_join[3] = {nullptr, nullptr, nullptr};
  // per degree: the troubled cells of a limiter pass (the cells of the
  // degree's problems) and their counter (weno_n[p])
  int2* weno_list[4] = {nullptr, nullptr, nullptr, nullptr};
  long long deg_cells[4] = {0, 0, 0, 0};
  unsigned int* weno_n = nullptr;
};

namespace {

void batch_free_plan(flsp_batch* b) {
  if (b->probs) cudaFree(b->probs);
  if (b->items_adv) cudaFree(b->items_adv);
  if (b->items_hj) cudaFree(b->items_hj);
  if (b->items_weno) cudaFree(b->items_weno);
  b->probs = nullptr;
  b->items_adv = b->items_hj = b->items_weno = nullptr;
  b->built = false;
  for (auto& kv : b->graphs)
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
  b->graphs.clear();
}

// descriptors and work lists of every problem for tiles (adv, hj)
int batch_build(flsp_batch* b, const int* adv_tile, const int* hj_tile) {
  batch_free_plan(b);
  const int n = (int)b->h.size();
  std::vector<BatchProb> pr((size_t)n);
  std::vector<int2> ia, ih, iw;
  size_t sa[4] = {0, 0, 0, 0}, sh[4] = {0, 0, 0, 0}, sw[4] = {0, 0, 0, 0};
  // descriptors sorted by degree (descending): each degree's problems are one
  // range of the array (its chain's clocks), items refer to the sorted index
  std::vector<int> order((size_t)n);
  for (int i = 0; i < n; ++i) order[(size_t)i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return b->h[x]->p > b->h[y]->p; });
  for (int p = 0; p < 4; ++p) b->prob_off[p] = b->prob_cnt[p] = 0;
  for (int i = 0; i < n; ++i) {
    flsp_handle* h = b->h[(size_t)order[(size_t)i]];
    if (h->p >= 1 && h->p <= 3) {
      if (b->prob_cnt[h->p] == 0) b->prob_off[h->p] = i;
      ++b->prob_cnt[h->p];
    }
    BatchProb& q = pr[(size_t)i];
    std::memset(&q, 0, sizeof(q));
    q.m_adv = h->m;
    q.m_adv.tiles = nullptr;
    q.m_adv.n_tiles = nullptr;
    q.m_hj = q.m_adv;
    q.m_weno = q.m_adv;
    set_tile(q.m_adv, 2, adv_tile);
    set_tile(q.m_hj, 2, hj_tile);
    set_tile(q.m_weno, 2, kWenoTile);
    for (int k = 0; k < 3; ++k) q.buf[k] = h->buf[k];
    q.clk = h->clk;
    VelDev v = h->veldev();
    if (!h->tab_ok) return fail(FLSP_ERR_BAD_ARG, "batched problem without velocity tables");
    q.tab_q = h->tab_q;
    q.tab_f = h->tab_f;
    for (int e = 0; e < 3; ++e) {
      q.tab_foff[e] = h->tab_foff[e];
      q.tab_nf[e] = h->tab_nf[e];
    }
    q.vtab = v.vtab;
    q.n_terms = v.n_terms;
    q.nmax = v.nmax;
    q.npt = v.npt;
    for (int k = 0; k < kMaxTerms; ++k) q.comp[k] = v.comp[k];
    q.p = h->p;
    q.ca.cfl_max = h->cfl_max;
    q.ca.scale = adv_cfl_scaling(h->p);
    q.ca.tkind = h->vel.time_kind;
    q.ca.ta = h->vel.ta;
    q.ca.tb = h->vel.tb;
    q.ca.rk = h->rk;
    q.ca.step_count = 1;
    q.adv_scale = adv_cfl_scaling(h->p);
    auto add = [&](const MeshArgs& m, std::vector<int2>& it) {
      const long long nt = nblocks(m);
      for (long long t = 0; t < nt; ++t) it.push_back(make_int2(i, (int)t));
    };
    add(q.m_adv, ia);
    add(q.m_hj, ih);
    add(q.m_weno, iw);
    if (h->p < 1 || h->p > 3) return fail(FLSP_ERR_UNSUPPORTED, "batched problems: degree 1..3");
    size_t x = 0;
    ST(batch_smem(kBatchKindAdv, h->p, b->prec, adv_tile, v.n_terms, &x));
    sa[h->p] = std::max(sa[h->p], x);
    ST(batch_smem(kBatchKindHJ, h->p, b->prec, hj_tile, 0, &x));
    sh[h->p] = std::max(sh[h->p], x);
    ST(batch_smem(kBatchKindWeno, h->p, b->prec, kWenoTile, 0, &x));
    sw[h->p] = std::max(sw[h->p], x);
  }
  // most expensive items first (higher degree, more velocity terms): blocks
  // take items round-robin, so the long ones spread over the whole grid and
  // the short ones fill in at the end
  auto by_cost = [&](std::vector<int2>& it) {
    std::stable_sort(it.begin(), it.end(), [&](const int2& x, const int2& y) {
      const long long cx = (long long)pr[(size_t)x.x].p * 64 + pr[(size_t)x.x].n_terms;
      const long long cy = (long long)pr[(size_t)y.x].p * 64 + pr[(size_t)y.x].n_terms;
      return cx > cy;
    });
  };
  by_cost(ia);
  by_cost(ih);
  by_cost(iw);
  CU(cudaMalloc(&b->probs, sizeof(BatchProb) * (size_t)n));
  CU(cudaMalloc(&b->items_adv, sizeof(int2) * ia.size()));
  CU(cudaMalloc(&b->items_hj, sizeof(int2) * ih.size()));
  CU(cudaMalloc(&b->items_weno, sizeof(int2) * iw.size()));
  CU(cudaMemcpy(b->probs, pr.data(), sizeof(BatchProb) * (size_t)n, cudaMemcpyHostToDevice));
  CU(cudaMemcpy(b->items_adv, ia.data(), sizeof(int2) * ia.size(), cudaMemcpyHostToDevice));
  CU(cudaMemcpy(b->items_hj, ih.data(), sizeof(int2) * ih.size(), cudaMemcpyHostToDevice));
  CU(cudaMemcpy(b->items_weno, iw.data(), sizeof(int2) * iw.size(), cudaMemcpyHostToDevice));
  b->n_adv = (int)ia.size();
  b->n_hj = (int)ih.size();
  b->n_weno = (int)iw.size();
  // the lists are sorted by degree (descending): one range, one launch per degree
  const std::vector<int2>* lists[3] = {&ia, &ih, &iw};
  const size_t* smems[3] = {sa, sh, sw};
  const int threads[3] = {adv_tile[0] * adv_tile[1], hj_tile[0] * hj_tile[1], kWenoTile[0] * kWenoTile[1]};
  for (int k = 0; k < 3; ++k) {
    for (int p = 0; p < 4; ++p) b->deg_off[k][p] = b->deg_cnt[k][p] = b->deg_grid[k][p] = 0;
    const std::vector<int2>& it = *lists[k];
    for (size_t j = 0; j < it.size(); ++j) {
      const int p = pr[(size_t)it[j].x].p;
      if (b->deg_cnt[k][p] == 0) b->deg_off[k][p] = (int)j;
      ++b->deg_cnt[k][p];
    }
    for (int p = 1; p <= 3; ++p) {
      b->deg_smem[k][p] = smems[k][p];
      if (b->deg_cnt[k][p] > 0)
        ST(batch_prepare(k, b->prec, p, smems[k][p], threads[k], b->deg_cnt[k][p], &b->deg_grid[k][p]));
    }
  }
  for (int d = 0; d < 3; ++d) {
    b->adv_tile[d] = adv_tile[d];
    b->hj_tile[d] = hj_tile[d];
  }
  b->built = true;
  return FLSP_OK;
}

int batch_sync_problems(flsp_batch* b) {
  for (flsp_handle* h : b->h) CU(cudaStreamSynchronize(h->stream));
  // a common buffer role: move a problem's state where the others' is
  for (flsp_handle* h : b->h)
    if (h->cur != b->cur) {
      CU(cudaMemcpy(h->buf[b->cur], h->buf[h->cur], (size_t)h->ndofs * h->tsize, cudaMemcpyDeviceToDevice));
      h->cur = b->cur;
    }
  return FLSP_OK;
}

// the stage / reinit step / limiter of every problem: one launch per degree
// one launch per degree present, side by side when there are several:
// each degree's launch on its own stream forked from the batch stream and
// joined back (graph branches under capture), so that one degree's tail
// overlaps the others' work
template <typename F>
int batch_each_degree(flsp_batch* b, int kind, F&& launch) {
  int n = 0;
  for (int p = 1; p <= 3; ++p) n += b->deg_cnt[kind][p] > 0;
  if (n <= 1) {
    for (int p = 3; p >= 1; --p)
      if (b->deg_cnt[kind][p] > 0) ST(launch(p, b->stream));
    return FLSP_OK;
  }
  CU(cudaEventRecord(b->ev_fork, b->stream));
  int st = FLSP_OK;
  for (int p = 3; p >= 1; --p) {
    if (b->deg_cnt[kind][p] == 0) continue;
    cudaStream_t s = b->side[p - 1];
    CU(cudaStreamWaitEvent(s, b->ev_fork, 0));
    if (st == FLSP_OK) st = launch(p, s);
    // join even after a failed launch, so that a capture stays joined
    CU(cudaEventRecord(b->ev_join[p - 1], s));
    CU(cudaStreamWaitEvent(b->stream, b->ev_join[p - 1], 0));
  }
  return st;
}

int batch_adv_all(flsp_batch* b, int thr, int in, int pn, int out, int stage, int combine) {
  return batch_each_degree(b, kBatchKindAdv, [&](int p, cudaStream_t s) {
    return launch_batch_adv(s, b->prec, p, b->probs, b->items_adv + b->deg_off[kBatchKindAdv][p],
                            b->deg_cnt[kBatchKindAdv][p], b->deg_grid[kBatchKindAdv][p], thr,
                            b->deg_smem[kBatchKindAdv][p], in, pn, out, stage, combine);
  });
}

int batch_hj_all(flsp_batch* b, int thr, int src, int phi0, int dst, int mode, int rk) {
  return batch_each_degree(b, kBatchKindHJ, [&](int p, cudaStream_t s) {
    return launch_batch_hj(s, b->prec, p, b->probs, b->items_hj + b->deg_off[kBatchKindHJ][p],
                           b->deg_cnt[kBatchKindHJ][p], b->deg_grid[kBatchKindHJ][p], thr,
                           b->deg_smem[kBatchKindHJ][p], src, phi0, dst, mode, rk);
  });
}

// One degree's chain on stream s: `steps` substeps of the degree's problems
// and, with ro, their reinitialisation; the buffer roles advance from *cur
// (the same sequence for every degree).
int batch_chain(flsp_batch* b, int p, cudaStream_t s, int steps, const flsp_reinit_opts* ro, bool limiter,
                int* cur) {
  const BatchProb* probs = b->probs + b->prob_off[p];
  const int np = b->prob_cnt[p];
  const int kA = kBatchKindAdv, kH = kBatchKindHJ, kW = kBatchKindWeno;
  const int thr = b->adv_tile[0] * b->adv_tile[1];
  auto stage = [&](int in, int pn, int out, int k, int comb) {
    return launch_batch_adv(s, b->prec, p, b->probs, b->items_adv + b->deg_off[kA][p], b->deg_cnt[kA][p],
                            b->deg_grid[kA][p], thr, b->deg_smem[kA][p], in, pn, out, k, comb);
  };
  for (int k = 0; k < steps; ++k) {
    ST(launch_batch_clock(s, probs, np, kBatchAdvBegin, 0.0));
    const int x = *cur, y = (x + 1) % 3, z = (x + 2) % 3;
    if (b->rk == 1) {
      ST(stage(x, x, y, 0, kRK1));
      *cur = y;
    } else if (b->rk == 2) {
      ST(stage(x, x, y, 0, kRK2a));
      ST(stage(y, x, z, 1, kRK2b));
      *cur = z;
    } else {
      ST(stage(x, x, y, 0, kRK3a));
      ST(stage(y, x, z, 1, kRK3b));
      ST(stage(z, x, y, 2, kRK3c));
      *cur = y;
    }
    ST(launch_batch_clock(s, probs, np, kBatchAdvEnd, 0.0));
  }
  if (!ro) return FLSP_OK;
  const int hthr = b->hj_tile[0] * b->hj_tile[1];
  auto hj = [&](int src, int phi0, int dst, int mode) {
    return launch_batch_hj(s, b->prec, p, b->probs, b->items_hj + b->deg_off[kH][p], b->deg_cnt[kH][p],
                           b->deg_grid[kH][p], hthr, b->deg_smem[kH][p], src, phi0, dst, mode, ro->rk_order);
  };
  const int phi0 = *cur;
  ST(launch_batch_clock(s, probs, np, kBatchHjReset, 0.0));
  ST(hj(phi0, phi0, -1, kHJCflOnly));
  for (int k = 0; k < ro->n_pseudo_steps; ++k) {
    ST(launch_batch_clock(s, probs, np, kBatchHjBegin, ro->cfl_max));
    const int src = *cur;
    const int dst = (src == phi0) ? (phi0 + 1) % 3 : other(src, phi0);
    ST(hj(src, phi0, dst, kHJStep));
    int res = dst;
    if (limiter) {
      const int lim = other(dst, phi0);
      ST(launch_batch_weno(s, b->prec, p, b->probs, b->items_weno + b->deg_off[kW][p], b->deg_cnt[kW][p],
                           b->deg_grid[kW][p], kWenoTile[0] * kWenoTile[1], b->deg_smem[kW][p], dst, lim,
                           b->weno_list[p], b->weno_n + p, b->deg_cells[p]));
      res = lim;
    }
    *cur = res;
    ST(launch_batch_clock(s, probs, np, kBatchHjEnd, 0.0));
  }
  return FLSP_OK;
}

// `steps` substeps and, with ro, a reinitialisation of every problem: one
// chain per degree, the chains side by side on their own streams, forked
// from the batch stream once and joined back once (a degree waits only for
// its own problems between stages)
int batch_enqueue_chains(flsp_batch* b, int steps, const flsp_reinit_opts* ro, bool limiter) {
  int n = 0;
  for (int p = 1; p <= 3; ++p) n += b->prob_cnt[p] > 0;
  const int cur0 = b->cur;
  int cur_end = cur0;
  if (n <= 1) {
    for (int p = 3; p >= 1; --p)
      if (b->prob_cnt[p] > 0) ST(batch_chain(b, p, b->stream, steps, ro, limiter, &cur_end));
    b->cur = cur_end;
    return FLSP_OK;
  }
  CU(cudaEventRecord(b->ev_fork, b->stream));
  int st = FLSP_OK;
  for (int p = 3; p >= 1; --p) {
    if (b->prob_cnt[p] == 0) continue;
    cudaStream_t s = b->side[p - 1];
    CU(cudaStreamWaitEvent(s, b->ev_fork, 0));
    int cur = cur0;
    if (st == FLSP_OK) st = batch_chain(b, p, s, steps, ro, limiter, &cur);
    cur_end = cur;
    // join even after a failed launch, so that a capture stays joined
    CU(cudaEventRecord(b->ev_join[p - 1], s));
    CU(cudaStreamWaitEvent(b->stream, b->ev_join[p - 1], 0));
  }
  if (st == FLSP_OK) b->cur = cur_end;
  return st;
}

}  // namespace

extern "C" {

void flsp_batch_destroy(flsp_batch* b) {
  if (!b) return;
  cudaSetDevice(b->dev);
  if (b->stream) cudaStreamSynchronize(b->stream);
  batch_free_plan(b);
  for (flsp_handle* h : b->h) flsp_destroy(h);
  for (int i = 0; i < 3; ++i) {
    if (b->side[i]) cudaStreamDestroy(b->side[i]);
    if (b->ev_join[i]) cudaEventDestroy(b->ev_join[i]);
  }
  if (b->ev_fork) cudaEventDestroy(b->ev_fork);
  if (b->stream) cudaStreamDestroy(b->stream);
  for (int p = 0; p < 4; ++p)
    if (b->weno_list[p]) cudaFree(b->weno_list[p]);
  if (b->weno_n) cudaFree(b->weno_n);
  delete b;
}

int flsp_batch_create(int n, const flsp_mesh_desc* meshes, const flsp_dg_opts* opts, flsp_batch** out) {
  if (!out || !meshes || !opts) return fail(FLSP_ERR_BAD_ARG, "null argument");
  *out = nullptr;
  if (n < 1 || n > (1 << 20)) return fail(FLSP_ERR_BAD_ARG, "bad batch size");
  for (int i = 0; i < n; ++i) {
    if (meshes[i].dim != 2) return fail(FLSP_ERR_UNSUPPORTED, "batched problems are 2D");
    if (opts[i].basis != FLSP_BASIS_Q) return fail(FLSP_ERR_UNSUPPORTED, "batched problems use the Q basis");
    if (opts[i].precision != opts[0].precision || opts[i].rk_order != opts[0].rk_order ||
        opts[i].device != opts[0].device)
      return fail(FLSP_ERR_BAD_ARG, "batched problems share precision, RK order and device");
  }
  flsp_batch* b = new flsp_batch();
  std::memset(&b->tuning, 0, sizeof(b->tuning));
  b->dev = opts[0].device;
  b->prec = opts[0].precision;
  b->rk = opts[0].rk_order;
  for (int i = 0; i < n; ++i) {
    flsp_handle* h = nullptr;
    const int st = flsp_create(&meshes[i], &opts[i], &h);
    if (st) {
      flsp_batch_destroy(b);
      return st;
    }
    h->batch_member = true;
    b->h.push_back(h);
  }
  bool ok = cudaSetDevice(b->dev) == cudaSuccess &&
            cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming) == cudaSuccess;
  for (int i = 0; i < 3 && ok; ++i)
    ok = cudaStreamCreateWithFlags(&b->side[i], cudaStreamNonBlocking) == cudaSuccess &&
         cudaEventCreateWithFlags(&b->ev_join[i], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    flsp_batch_destroy(b);
    return fail(FLSP_ERR_CUDA, "batch stream creation failed");
  }
  for (flsp_handle* h : b->h) b->deg_cells[h->p] += h->m.ncell;
  ok = cudaMalloc(&b->weno_n, 4 * sizeof(unsigned int)) == cudaSuccess;
  for (int p = 1; p <= 3 && ok; ++p)
    if (b->deg_cells[p] > 0) ok = cudaMalloc(&b->weno_list[p], sizeof(int2) * (size_t)b->deg_cells[p]) == cudaSuccess;
  if (!ok) {
    flsp_batch_destroy(b);
    return fail(FLSP_ERR_OOM, "batch allocation failed");
  }
  *out = b;
  return FLSP_OK;
}

int flsp_batch_size(const flsp_batch* b, int* n) {
  if (!b || !n) return fail(FLSP_ERR_BAD_ARG, "null argument");
  *n = (int)b->h.size();
  return FLSP_OK;
}

int flsp_batch_problem(flsp_batch* b, int i, flsp_handle** h) {
  if (!b || !h) return fail(FLSP_ERR_BAD_ARG, "null argument");
  if (i < 0 || i >= (int)b->h.size()) return fail(FLSP_ERR_BAD_ARG, "problem index out of range");
  *h = b->h[(size_t)i];
  return FLSP_OK;
}

int flsp_batch_autotune(flsp_batch* b, flsp_batch_tuning* out) {
  if (!b) return fail(FLSP_ERR_BAD_ARG, "null argument");
  CU(cudaSetDevice(b->dev));
  for (flsp_handle* h : b->h)
    if (!h->has_vel) return fail(FLSP_ERR_BAD_ARG, "velocity not set for every problem");
  ST(batch_sync_problems(b));
  static const int ca[][3] = {{32, 8, 1}, {16, 16, 1}, {16, 8, 1}, {8, 8, 1}};
  static const int ch[][3] = {{16, 8, 1}, {8, 16, 1}, {8, 8, 1}};
  flsp_batch_tuning t;
  std::memset(&t, 0, sizeof(t));
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0));
  CU(cudaEventCreate(&e1));
  auto time_it = [&](auto&& launch, double* ms) -> int {
    for (int r = 0; r < 2; ++r) ST(launch());
    CU(cudaEventRecord(e0, b->stream));
    const int reps = 5;
    for (int r = 0; r < reps; ++r) ST(launch());
    CU(cudaEventRecord(e1, b->stream));
    CU(cudaEventSynchronize(e1));
    float f = 0.0f;
    CU(cudaEventElapsedTime(&f, e0, e1));
    *ms = f / reps;
    return FLSP_OK;
  };
  // the stage: clock set-up at the current time (harmless: the step's own
  // set-up recomputes it), the first RK stage into a free buffer
  double best = 1e300;
  int bi = 0;
  for (int c = 0; c < 4; ++c) {
    ST(batch_build(b, ca[c], ch[0]));
    ST(launch_batch_clock(b->stream, b->probs, (int)b->h.size(), kBatchAdvBegin, 0.0));
    const int x = b->cur, y = (x + 1) % 3;
    double ms = 0.0;
    ST(time_it([&]() {
      return batch_adv_all(b, ca[c][0] * ca[c][1], x, x, y, 0, kRK3a);
    }, &ms));
    t.adv_cand[c][0] = ca[c][0];
    t.adv_cand[c][1] = ca[c][1];
    t.adv_ms[c] = ms;
    if (ms < best) { best = ms; bi = c; }
  }
  t.n_adv = 4;
  // the reinit step: the CFL pass (reads the state, writes only the clock's
  // CFL slot, which every reinit resets)
  best = 1e300;
  int bj = 0;
  for (int c = 0; c < 3; ++c) {
    ST(batch_build(b, ca[bi], ch[c]));
    const int x = b->cur;
    double ms = 0.0;
    ST(time_it([&]() {
      return batch_hj_all(b, ch[c][0] * ch[c][1], x, x, -1, kHJCflOnly, 1);
    }, &ms));
    t.hj_cand[c][0] = ch[c][0];
    t.hj_cand[c][1] = ch[c][1];
    t.hj_ms[c] = ms;
    if (ms < best) { best = ms; bj = c; }
  }
  t.n_hj = 3;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ST(batch_build(b, ca[bi], ch[bj]));
  t.adv_tile[0] = ca[bi][0];
  t.adv_tile[1] = ca[bi][1];
  t.hj_tile[0] = ch[bj][0];
  t.hj_tile[1] = ch[bj][1];
  b->tuning = t;
  b->tuned = true;
  if (out) *out = t;
  return FLSP_OK;
}

int flsp_batch_run_steps(flsp_batch* b, const flsp_ls_opts* o, int n_steps) {
  if (!b || !o) return fail(FLSP_ERR_BAD_ARG, "null argument");
  if (n_steps < 0 || o->reinit_frequency < 1) return fail(FLSP_ERR_BAD_ARG, "bad step counts");
  const flsp_reinit_opts ro = o->reinit;
  if (o->execute_reinit) {
    if (ro.mode != FLSP_REINIT_FIXED) return fail(FLSP_ERR_BAD_ARG, "batched reinit is fixed-count (FLSP_REINIT_FIXED)");
    if (ro.viscosity != 0.0 || ro.narrow_band) return fail(FLSP_ERR_UNSUPPORTED, "batched reinit: no viscosity, no narrow band");
    ST(validate_reinit(b->h[0], &ro));
  }
  CU(cudaSetDevice(b->dev));
  if (!b->tuned) ST(flsp_batch_autotune(b, nullptr));
  ST(batch_sync_problems(b));
  const bool limiter = ro.limiter != 0;   // 2D: on unless switched off (reinit.cc:475-478)
  const int n = (int)b->h.size();
  ST(launch_batch_clock(b->stream, b->probs, n, kBatchAdvHorizon, 0.0));
  int done = 0;
  while (done < n_steps) {
    const int to_reinit = o->execute_reinit ? o->reinit_frequency - b->n_since_reinit : n_steps - done;
    if (to_reinit <= 0) { b->n_since_reinit = 0; continue; }
    if (done + to_reinit <= n_steps && o->execute_reinit) {
      unsigned long long key = 1469598103934665603ull;
      auto mix = [&](const void* p, size_t nb) {
        const unsigned char* c = static_cast<const unsigned char*>(p);
        for (size_t i = 0; i < nb; ++i) { key ^= c[i]; key *= 1099511628211ull; }
      };
      mix(&b->cur, sizeof(b->cur));
      mix(&to_reinit, sizeof(to_reinit));
      mix(&ro, sizeof(ro));
      auto it = b->graphs.find(key);
      if (it == b->graphs.end()) {
        const int cur0 = b->cur;
        cudaGraph_t g = nullptr;
        CU(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        int st = FLSP_OK;
        st = batch_enqueue_chains(b, to_reinit, &ro, limiter);
        cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
        if (st != FLSP_OK) { if (g) cudaGraphDestroy(g); b->cur = cur0; return st; }
        if (ce != cudaSuccess) return fail(FLSP_ERR_CUDA, std::string("batch graph capture: ") + cudaGetErrorString(ce));
        GraphEntry ge;
        ge.cur_after = b->cur;
        b->cur = cur0;
        CU(cudaGraphInstantiate(&ge.exec, g, 0));
        cudaGraphDestroy(g);
        it = b->graphs.emplace(key, ge).first;
      }
      CU(cudaGraphLaunch(it->second.exec, b->stream));
      b->cur = it->second.cur_after;
      b->n_since_reinit = 0;
      done += to_reinit;
    } else {
      const int k = std::min(to_reinit, n_steps - done);
      ST(batch_enqueue_chains(b, k, nullptr, false));
      b->n_since_reinit += k;
      done += k;
    }
  }
  for (flsp_handle* h : b->h) {
    h->cur = b->cur;
    h->n_since_reinit = b->n_since_reinit;
  }
  return FLSP_OK;
}

int flsp_batch_sync(flsp_batch* b) {
  if (!b) return fail(FLSP_ERR_BAD_ARG, "null argument");
  CU(cudaSetDevice(b->dev));
  CU(cudaStreamSynchronize(b->stream));
  for (flsp_handle* h : b->h) ST(sync_clock(h));
  return FLSP_OK;
}

int flsp_batch_stream(const flsp_batch* b, void** stream) {
  if (!b || !stream) return fail(FLSP_ERR_BAD_ARG, "null argument");
  *stream = (void*)b->stream;
  return FLSP_OK;
}


// ---------------------------------------------------------------------
// Groups: several independent problems (any dimension, size or degree)
// whose reinit periods are captured into ONE CUDA graph, one branch per
// problem, so that their kernels run side by side on the device.
// ---------------------------------------------------------------------
}  // extern "C"

struct GroupGraph {
  cudaGraphExec_t exec = nullptr;
  std::vector<int> cur_after;
};

struct flsp_group {
  int dev = 0;
  std::vector<flsp_handle*> h;
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  std::map<unsigned long long, GroupGraph> graphs;
};

extern "C" {

int flsp_group_create(flsp_handle* const* handles, int n, flsp_group** out) {
  if (!handles || n < 1 || !out) return fail(FLSP_ERR_BAD_ARG, "bad argument");
  *out = nullptr;
  for (int i = 0; i < n; ++i) {
    if (!handles[i]) return fail(FLSP_ERR_BAD_ARG, "null handle");
    if (handles[i]->dev != handles[0]->dev) return fail(FLSP_ERR_BAD_ARG, "group members on different devices");
    for (int j = 0; j < i; ++j)
      if (handles[j] == handles[i]) return fail(FLSP_ERR_BAD_ARG, "a handle appears twice in the group");
  }
  flsp_group* g = new flsp_group();
  g->dev = handles[0]->dev;
  g->h.assign(handles, handles + n);
  g->join.assign(n, nullptr);
  cudaError_t e = cudaSetDevice(g->dev);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->fork, cudaEventDisableTiming);
  for (int i = 0; i < n && e == cudaSuccess; ++i) e = cudaEventCreateWithFlags(&g->join[i], cudaEventDisableTiming);
  if (e != cudaSuccess) {
    flsp_group_destroy(g);
    return fail(FLSP_ERR_CUDA, std::string("group: ") + cudaGetErrorString(e));
  }
  *out = g;
  return FLSP_OK;
}

void flsp_group_destroy(flsp_group* g) {
  if (!g) return;
  cudaSetDevice(g->dev);
  if (g->stream) cudaStreamSynchronize(g->stream);
  for (auto& kv : g->graphs)
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
  for (cudaEvent_t ev : g->join)
    if (ev) cudaEventDestroy(ev);
  if (g->fork) cudaEventDestroy(g->fork);
  if (g->stream) cudaStreamDestroy(g->stream);
  delete g;
}

}  // extern "C"

namespace {

// what a group period runs: the fixed-count plain reinit (ro) or the
// learned reinit without fallback (net, lo)
struct GroupMode {
  int freq = 0;
  const flsp_reinit_opts* ro = nullptr;
  flsp_mlp* net = nullptr;
  const flsp_learned_opts* lo = nullptr;
  bool fallback = false;   // learned with its residual fallback
};

int group_run(flsp_group* g, const GroupMode& gm, int n_periods) {
  const int n = (int)g->h.size();
  // the group's stream waits for every member's earlier work
  for (int i = 0; i < n; ++i) {
    CU(cudaEventRecord(g->join[i], g->h[i]->stream));
    CU(cudaStreamWaitEvent(g->stream, g->join[i], 0));
  }
  for (int it = 0; it < n_periods; ++it) {
    unsigned long long key = 1469598103934665603ull;
    auto mix = [&key](const void* p, size_t nb) {
      const unsigned char* b = (const unsigned char*)p;
      for (size_t i = 0; i < nb; ++i) { key ^= b[i]; key *= 1099511628211ull; }
    };
    for (flsp_handle* h : g->h) {
      mix(&h->cur, sizeof(h->cur));
      mix(&h->gen, sizeof(h->gen));   // a member's velocity or conditions changed
    }
    mix(&gm.freq, sizeof(gm.freq));
    if (gm.ro) mix(gm.ro, sizeof(*gm.ro));
    if (gm.net) {
      mix(&gm.net->uid, sizeof(gm.net->uid));
      mix(&gm.net->cap, sizeof(gm.net->cap));
      mix(&gm.lo->band_cells, sizeof(gm.lo->band_cells));
      mix(&gm.fallback, sizeof(gm.fallback));
      if (gm.fallback) {
        mix(&gm.lo->max_residual, sizeof(gm.lo->max_residual));
        mix(&gm.lo->fallback, sizeof(gm.lo->fallback));
      }
    }
    auto gi = g->graphs.find(key);
    if (gi == g->graphs.end()) {
      std::vector<int> cur0(n);
      for (int i = 0; i < n; ++i) cur0[i] = g->h[i]->cur;
      cudaGraph_t graph = nullptr;
      CU(cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal));
      int st = FLSP_OK;
      cudaError_t ce = cudaEventRecord(g->fork, g->stream);
      for (int i = 0; i < n && st == FLSP_OK && ce == cudaSuccess; ++i) {
        flsp_handle* h = g->h[i];
        ce = cudaStreamWaitEvent(h->stream, g->fork, 0);   // the member's stream joins the capture
        if (ce == cudaSuccess) st = launch_adv_clock_horizon(h->stream, h->clk, INFINITY);
        if (ce == cudaSuccess && st == FLSP_OK) {
          if (gm.net) {
            // the members' network passes share the network's buffers: they
            // follow one another on its stream (member order)
            for (int s = 0; s < gm.freq && st == FLSP_OK; ++s) st = enqueue_adv_step(h);
            if (st == FLSP_OK && gm.fallback) {
              st = enqueue_learned_fallback(h, gm.net, gm.lo);
            } else if (st == FLSP_OK) {
              const int pre = h->cur, out = other(pre, -1);
              st = enqueue_learned(h, gm.net, gm.lo->band_cells, pre, out);
              if (st == FLSP_OK) st = launch_learned_totals(h->stream, h->lrn_count, h->lrn_tot, 0);
              if (st == FLSP_OK) h->cur = out;
            }
          } else {
            st = enqueue_period(h, gm.ro, gm.freq);
          }
        }
        if (ce == cudaSuccess) ce = cudaEventRecord(g->join[i], h->stream);
        if (ce == cudaSuccess) ce = cudaStreamWaitEvent(g->stream, g->join[i], 0);
      }
      const cudaError_t ce2 = cudaStreamEndCapture(g->stream, &graph);
      if (st != FLSP_OK || ce != cudaSuccess || ce2 != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        for (int i = 0; i < n; ++i) g->h[i]->cur = cur0[i];
        if (st != FLSP_OK) return st;
        return fail(FLSP_ERR_CUDA, std::string("group capture: ") + cudaGetErrorString(ce != cudaSuccess ? ce : ce2));
      }
      GroupGraph gg;
      gg.cur_after.resize(n);
      for (int i = 0; i < n; ++i) {
        gg.cur_after[i] = g->h[i]->cur;
        g->h[i]->cur = cur0[i];
      }
      const cudaError_t ci = cudaGraphInstantiate(&gg.exec, graph, 0);
      cudaGraphDestroy(graph);
      if (ci != cudaSuccess) return fail(FLSP_ERR_CUDA, std::string("group graph: ") + cudaGetErrorString(ci));
      gi = g->graphs.emplace(key, gg).first;
    }
    CU(cudaGraphLaunch(gi->second.exec, g->stream));
    for (int i = 0; i < n; ++i) g->h[i]->cur = gi->second.cur_after[i];
  }
  // every member's stream waits for the group's work
  CU(cudaEventRecord(g->fork, g->stream));
  for (flsp_handle* h : g->h) CU(cudaStreamWaitEvent(h->stream, g->fork, 0));
  return FLSP_OK;
}

}  // namespace

extern "C" {

int flsp_group_run_periods(flsp_group* g, const flsp_ls_opts* o, int n_periods) {
  if (!g || !o || n_periods < 0) return fail(FLSP_ERR_BAD_ARG, "bad argument");
  if (o->reinit_frequency < 1 || !o->execute_reinit || o->reinit.mode != FLSP_REINIT_FIXED)
    return fail(FLSP_ERR_BAD_ARG, "group periods need a fixed-count reinit (FLSP_REINIT_FIXED)");
  const flsp_reinit_opts ro = o->reinit;
  CU(cudaSetDevice(g->dev));
  for (flsp_handle* h : g->h) {
    if (!h->has_vel) return fail(FLSP_ERR_BAD_ARG, "velocity not set");
    if (h->n_since_reinit != 0) return fail(FLSP_ERR_BAD_ARG, "a group member is inside a reinit period");
    ST(validate_reinit(h, &ro));
    if (ro.viscosity > 0.0) ST(ensure_ldg_buffers(h));
    if (ro.narrow_band) ST(ensure_band_buffers(h));
  }
  GroupMode gm;
  gm.freq = o->reinit_frequency;
  gm.ro = &ro;
  return group_run(g, gm, n_periods);
}

int flsp_group_run_periods_learned(flsp_group* g, flsp_mlp* net, const flsp_learned_opts* o, int reinit_frequency,
                                   int n_periods) {
  if (!g || !net || !o || n_periods < 0 || reinit_frequency < 1) return fail(FLSP_ERR_BAD_ARG, "bad argument");
  if (!(o->band_cells > 0.0)) return fail(FLSP_ERR_BAD_ARG, "bad learned options");
  CU(cudaSetDevice(g->dev));
  int64_t max_cells = 0;
  bool fb = false;
  for (flsp_handle* h : g->h) {
    if (!h->has_vel) return fail(FLSP_ERR_BAD_ARG, "velocity not set");
    if (h->n_since_reinit != 0) return fail(FLSP_ERR_BAD_ARG, "a group member is inside a reinit period");
    ST(learned_check(h, net));
    ST(ensure_learned_buffers(h, h->m.ncell));
    ST(learned_graph_fallback(h, o, &fb));
    max_cells = std::max<int64_t>(max_cells, h->m.ncell);
  }
  ST(mlp_ensure_cap(net, max_cells));
  GroupMode gm;
  gm.freq = reinit_frequency;
  gm.net = net;
  gm.lo = o;
  gm.fallback = fb;
  return group_run(g, gm, n_periods);
}

int flsp_group_sync(flsp_group* g) {
  if (!g) return fail(FLSP_ERR_BAD_ARG, "null group");
  CU(cudaSetDevice(g->dev));
  CU(cudaStreamSynchronize(g->stream));
  for (flsp_handle* h : g->h) ST(sync_clock(h));
  return FLSP_OK;
}

int flsp_group_stream(const flsp_group* g, void** stream) {
  if (!g || !stream) return fail(FLSP_ERR_BAD_ARG, "null argument");
  *stream = (void*)g->stream;
  return FLSP_OK;
}

}  // extern "C"

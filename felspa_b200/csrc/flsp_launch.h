// flsp_launch.h — host launchers exported by the kernel units
// (flsp_k_adv.cu, flsp_k_hj.cu, flsp_k_misc.cu) to the C-ABI unit.
// Launchers return a flsp_status and leave a message through set_error().
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <type_traits>

#include "flsp_device.cuh"
#include "flsp_dg.h"

namespace flsp {

int set_error(int code, const std::string& msg);

// narrow-band tile lists, one per kernel family (their tile shapes differ)
enum NarrowBandKind : int { kNbHJ = 0, kNbLdg = 1, kNbWeno = 2 };

struct Ctx {
  int dim, p, prec, basis;
  MeshArgs m;          // tile fields are filled by the launchers
  cudaStream_t stream;
  const int* nb_tiles[3];   // active tile lists (null: every tile)
  const int* nb_count[3];   // device counts of the lists
  void* hj_stab;            // smooth-sign table of the tensor-product reinit kernel
};

// tile shapes of the LDG viscosity and WENO limiter kernels
inline constexpr int kLdgTile2[3] = {16, 16, 1};
inline constexpr int kLdgTile3[3] = {8, 8, 4};
inline constexpr int kWenoTile[3] = {16, 16, 1};

// narrow band: flags[c] = 1 for cells with |mean phi0| <= thr; then the
// list of tiles of shape `tile` that hold a flagged cell within `margin`
// cells of the tile (device count in *count, order of the list arbitrary:
// each tile is computed independently)
int launch_band_flags(const Ctx& c, const void* phi0, double thr, int* flags);
int launch_band_tiles(const Ctx& c, const int* flags, const int* tile, int margin, int* list, int* count);
// out[c] = phi0[c] for cells with flags[c] == 0
int launch_band_restore(const Ctx& c, const void* phi0, void* out, const int* flags);
// band flags of the listed cells whose list flag is set (all others 0); the
// list holds min(n, *n_dev) cells
int launch_band_flags_from_list(const Ctx& c, const int* cells, const int* list_flags, long long n, const int* n_dev,
                                int* flags);
// tot[0] += counts[0] (band cells); tot[1] += counts[1] (fallback cells) if with_fallback
int launch_learned_totals(cudaStream_t s, const int* counts, unsigned long long* tot, int with_fallback);

// ---------------- batched problems (flsp_k_batch.cu) ----------------
// one problem of a batch, as the batched kernels see it (2D, Q basis)
struct BatchProb {
  MeshArgs m_adv, m_hj, m_weno;   // the batch's tile shapes, no narrow band
  void* buf[3];                   // state buffers (roles are launch parameters)
  DevClock* clk;
  const void* vtab;               // velocity table (state precision)
  int n_terms, nmax, npt;
  int comp[kMaxTerms];
  const void* tab_q;              // velocity tables of the problem (VelArgs::tab_q / tab_f)
  const void* tab_f;
  long long tab_foff[3], tab_nf[3];
  int p;                          // degree 1..3
  AdvClockArgs ca;                // advection clock parameters
  double adv_scale;               // advection CFL scaling of the degree
};
enum BatchKernelKind : int { kBatchKindAdv = 0, kBatchKindHJ = 1, kBatchKindWeno = 2 };
enum BatchClockOp : int {
  kBatchAdvBegin = 0, kBatchAdvEnd = 1, kBatchAdvHorizon = 2, kBatchHjReset = 3, kBatchHjBegin = 4, kBatchHjEnd = 5
};
int upload_tables_batch();
// shared memory one problem needs for a tile of the given kind
int batch_smem(int kind, int p, int prec, const int* tile, int n_terms, size_t* bytes);
// kernel attributes of the degree-p kernel for `smem` and its persistent
// grid for n_items (every item of a launch has degree p)
int batch_prepare(int kind, int prec, int p, size_t smem, int threads, int n_items, int* grid);
int launch_batch_clock(cudaStream_t s, const BatchProb* probs, int n, int what, double cfl_max);
int launch_batch_adv(cudaStream_t s, int prec, int p, const BatchProb* probs, const int2* items, int n_items,
                     int grid, int threads, size_t smem, int ix, int in_n, int iout, int stage, int combine);
int launch_batch_hj(cudaStream_t s, int prec, int p, const BatchProb* probs, const int2* items, int n_items,
                    int grid, int threads, size_t smem, int isrc, int iphi0, int idst, int mode, int rk);
int launch_batch_weno(cudaStream_t s, int prec, int p, const BatchProb* probs, const int2* items, int n_items,
                      int grid, int threads, size_t smem, int iin, int iout, int2* list, unsigned int* list_n,
                      long long n_cells);

// restrict a launch's MeshArgs to the narrow-band tile list of `kind`
inline void apply_band(const Ctx& c, int kind, MeshArgs& m) {
  m.tiles = c.nb_tiles[kind];
  m.n_tiles = c.nb_count[kind];
}

inline bool supported_config(int dim, int p) {
  return (dim == 2 && p >= 1 && p <= 3) || (dim == 3 && p >= 1 && p <= 2);
}

// compile-time dispatch over the built (dim, degree, precision) variants
template <typename F>
int dispatch(const Ctx& c, F&& f) {
#define FLSP_CASE(D, PP)                                                                      \
  if (c.dim == D && c.p == PP) {                                                              \
    if (c.prec == FLSP_FP64)                                                                  \
      return f(std::integral_constant<int, D>(), std::integral_constant<int, PP>(), (double)0); \
    return f(std::integral_constant<int, D>(), std::integral_constant<int, PP>(), (float)0);  \
  }
  FLSP_CASE(2, 1)
  FLSP_CASE(2, 2)
  FLSP_CASE(2, 3)
  FLSP_CASE(3, 1)
  FLSP_CASE(3, 2)
#undef FLSP_CASE
  return set_error(FLSP_ERR_UNSUPPORTED, "unsupported (dim, degree)");
}

inline void set_tile(MeshArgs& m, int dim, const int* t) {
  for (int d = 0; d < 3; ++d) {
    m.tile[d] = d < dim ? t[d] : 1;
    m.ntile[d] = (m.n[d] + m.tile[d] - 1) / m.tile[d];
  }
}
inline long long nblocks(const MeshArgs& m) { return (long long)m.ntile[0] * m.ntile[1] * m.ntile[2]; }

inline int launch_status(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(FLSP_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return FLSP_OK;
}

// ---------------- tables (one per unit) ----------------
int upload_tables_adv();
int upload_tables_hj();
int upload_tables_misc();
int upload_tables_sep2();
int upload_tables_sep3();



// ---------------- advection (flsp_k_adv.cu) ----------------
struct VelDev {
  const void* vtab;    // T-precision table
  int n_terms, nmax, npt;
  int comp[kMaxTerms];
  bool sep1;           // term k is the only term of component k
  const void* optab;   // per-axis operator rows of a sep1 velocity (T precision), or null
  int opstride;        // operator rows per (component, axis) in optab
  int* err;            // device error word (DevClock::err)
  // velocity tables (tab): T-precision values at the cells' and faces'
  // quadrature points (VelArgs::tab_q / tab_f), made from the terms or from
  // the FE field of a coupled simulator (fe_pv > 0: its lattice degree)
  bool tab;
  int fe_pv;
  const void* tab_q;
  const void* tab_f;
  long long tab_foff[3], tab_nf[3];
};
// stage kernel of this velocity: separable-operator kernel when optab is set
inline bool use_sep_kernel(const VelDev& v) { return v.sep1 && v.optab != nullptr; }
// separable stage kernel units: what = 0 shared-memory bytes of the tile,
// 1 kernel attributes, 2 launch (flsp_k_sep.cuh)
int sep2_call(int what, const Ctx& c, const VelDev* v, const int* tile, size_t* bytes, const void* in,
              const void* phin, void* out, const DevClock* clk, int stage, int combine, double ct_explicit);
int sep3_call(int what, const Ctx& c, const VelDev* v, const int* tile, size_t* bytes, const void* in,
              const void* phin, void* out, const DevClock* clk, int stage, int combine, double ct_explicit);
// tile: cells per CTA (nullptr = default); smem attribute is set on first use
int adv_default_tile(const Ctx& c, const VelDev& v, int* tile);
int adv_prepare(const Ctx& c, const VelDev& v, const int* tile);
// the tile shapes the stage kernel for this velocity is built with (at most 8)
int adv_tile_candidates(const Ctx& c, const VelDev& v, int (*out)[3], int* n);
int launch_adv_stage(const Ctx& c, const VelDev& v, const void* in, const void* phin, void* out,
                     const DevClock* clk, int stage, int combine, double ct_explicit,
                     const int* tile);

// ---------------- reinitialisation (flsp_k_hj.cu) ----------------
int hj_default_tile(const Ctx& c, int* tile);
int hj_prepare(const Ctx& c, const int* tile);
// bytes of the tensor-product reinit kernel's smooth-sign table for `tile`
int hj_table_bytes(const Ctx& c, const int* tile, size_t* bytes);
int launch_hj(const Ctx& c, const void* phi, const void* phi0, void* out, DevClock* clk, int mode,
              int rk, double dt_explicit, long long block, const int* tile,
              const void* rdiff = nullptr);
// LDG artificial viscosity: mode 0 = alternating gradient q (DIM blocks)
// from phi, mode 1 = diffusion RHS (per unit volume) from q
int ldg_prepare(const Ctx& c);
int launch_ldg(const Ctx& c, const void* in, void* out, long long block, double nu, int mode);

// ---------------- misc (flsp_k_misc.cu) ----------------
int weno_prepare(const Ctx& c);
// detection over the tiles (untroubled cells copied), then the WENO
// reconstruction of the troubled cells listed in `list` (ncell entries,
// counter list_n)
int launch_weno(const Ctx& c, const void* in, void* out, unsigned int* count, int2* list, unsigned int* list_n);
int launch_project_ic(const Ctx& c, const flsp_ic_desc* ic_dev, void* out);
int launch_static_cfl(const Ctx& c, const double* vtab64, int n_terms, const int* comp, int nmax,
                      int npt, DevClock* clk);
// static CFL part of an FE velocity lattice (FP64, degree pv), max-ed into clk->vd_static
int launch_fe_static_cfl(const Ctx& c, const double* u64, int pv, DevClock* clk);
// the spatial part of a sum of separable terms (FP64 term tables of
// build_vtab, terms sorted by component) at every cell's QGauss(p+2) points
// and every face's, in the state precision (layouts of VelArgs::tab_q / tab_f)
int launch_vel_tabulate(const Ctx& c, const double* vtab64, int n_terms, const int* comp, int nmax, int npt,
                        void* tab_q, void* tab_f, const long long* foff, const long long* nf);
// the FE velocity lattice (FP64, degree pv) at every cell's QGauss(p+2)
// points and every face's, in the state precision (layouts of VelArgs::
// tab_q / tab_f); gb[a][q] = Lagrange basis a at Gauss point q
int launch_fe_tabulate(const Ctx& c, const double* u64, int pv, const double (*gb)[kMaxNQ + 2], void* tab_q,
                       void* tab_f, const long long* foff, const long long* nf);
// two-level FP64 reduction; partial holds 2 * reduce_blocks(c) doubles,
// out_dev receives two doubles (sum pair, or max)
int launch_reduce(const Ctx& c, int which, const void* phi, const void* ref,
                  const flsp_ic_desc* ic_dev, double* partial, double* out_dev);
int reduce_blocks(const Ctx& c);
int launch_scatter(const Ctx& c, const double* src, void* dst, const int64_t* perm);
int launch_gather(const Ctx& c, const void* src, double* dst, const int64_t* perm);
int launch_nonfinite(const Ctx& c, const void* x, long long n, unsigned int* count);

int launch_adv_clock_begin(cudaStream_t s, DevClock* clk, const AdvClockArgs& a);
int launch_adv_clock_end(cudaStream_t s, DevClock* clk);
int launch_adv_clock_horizon(cudaStream_t s, DevClock* clk, double time_step);
int launch_hj_clock_reset(cudaStream_t s, DevClock* clk);
int launch_hj_clock_begin(cudaStream_t s, DevClock* clk, double cfl_max, int p, double nu,
                          double min_diam, double adv_scale);
int launch_hj_clock_end(cudaStream_t s, DevClock* clk);

// ---------------- output (flsp_io.cu) ----------------
// out[k * (n_sub+1)^dim + j] = the state of host cell k at its patch vertex j
int launch_eval_patches(const Ctx& c, const void* phi, const int64_t* perm, int n_sub, double* out);

// MaterialStack mixing (flsp_io.cu): one level set of the stack
struct MixLevelSet {
  const void* phi;        // state, lexicographic cells
  int prec, n1, nb;
  double eps;             // Heaviside smoothing width, 1.5 min_diameter
  signed char q2g[64];    // Q-layout mode -> in-cell DoF (-1: absent)
};
struct MixArgs {
  MixLevelSet ls[FLSP_MAX_MATERIALS];
  double value[FLSP_MAX_MATERIALS + 1];   // stack entries, then the background
  double L[kMaxN1][FLSP_MAX_MIX_QPTS];    // Legendre values at the Gauss points
  const int64_t* perm;                    // output cell order (null: lexicographic)
  long long ncell;
  int n, dim, nq, smoothing;
};
int launch_material_mix(const MixArgs& a, cudaStream_t s, double* out);
// values2 / label2 (or NULL): a second point-data array
int write_vtu_file(const flsp_mesh_desc* mesh, int n_sub, const double* values, const char* label,
                   const char* filename, const double* values2, const char* label2);
int write_pvd_file(const char* filename, int n, const double* times, const char* const* files);
int upload_tables_io();
// curvature estimate of the state into out (host DoF order, FP64);
// pos_scratch: n_cells int64 for the inverse permutation (used when perm)
int launch_curvature(const Ctx& c, const void* phi, const int64_t* perm, int64_t* pos_scratch, int mode,
                     double* out);

}  // namespace flsp

// flsp_k_misc.cu — limiter, projection, reductions, clocks, DoF order
// (instantiations + launchers).
#include <cuda.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "flsp_launch.h"
#include "flsp_misc.cuh"
#include "flsp_tables.h"
#include "flsp_weno.cuh"

namespace flsp {

int upload_tables_misc() {
  cudaError_t e = upload_tables_here();
  if (e != cudaSuccess) return set_error(FLSP_ERR_CUDA, std::string("tables: ") + cudaGetErrorString(e));
  return FLSP_OK;
}


int weno_prepare(const Ctx& c) {
  if (c.dim != 2) return set_error(FLSP_ERR_UNSUPPORTED, "WENO limiter is 2D only (reinit.cc:475-478)");
  return dispatch(c, [&](auto D, auto PP, auto tz) -> int {
    constexpr int P = decltype(PP)::value;
    using T = decltype(tz);
    if constexpr (decltype(D)::value != 2) {
      return set_error(FLSP_ERR_UNSUPPORTED, "WENO limiter is 2D only");
    } else {
      const size_t smem = weno_smem_bytes<P, T>(kWenoTile);
      cudaError_t e = cudaFuncSetAttribute(weno_kernel<P, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return set_error(FLSP_ERR_CUDA, std::string("weno attr: ") + cudaGetErrorString(e));
      return FLSP_OK;
    }
  });
}

int launch_weno(const Ctx& c, const void* in, void* out, unsigned int* count, int2* list, unsigned int* list_n) {
  if (c.dim != 2) return set_error(FLSP_ERR_UNSUPPORTED, "WENO limiter is 2D only (reinit.cc:475-478)");
  return dispatch(c, [&](auto D, auto PP, auto tz) -> int {
    constexpr int P = decltype(PP)::value;
    using T = decltype(tz);
    if constexpr (decltype(D)::value != 2) {
      return set_error(FLSP_ERR_UNSUPPORTED, "WENO limiter is 2D only");
    } else {
      WenoArgs<T> a;
      std::memset(&a, 0, sizeof(a));
      a.m = c.m;
      set_tile(a.m, 2, kWenoTile);
      apply_band(c, kNbWeno, a.m);
      a.in = reinterpret_cast<const T*>(in);
      a.out = reinterpret_cast<T*>(out);
      a.count = count;
      a.list = list;
      a.list_n = list_n;
      a.problem = 0;
      cudaError_t e = cudaMemsetAsync(list_n, 0, sizeof(unsigned int), c.stream);
      if (e != cudaSuccess) return set_error(FLSP_ERR_CUDA, std::string("weno list: ") + cudaGetErrorString(e));
      const size_t smem = weno_smem_bytes<P, T>(a.m.tile);
      weno_kernel<P, T><<<(unsigned)nblocks(a.m), kWenoTile[0] * kWenoTile[1], smem, c.stream>>>(a);
      // the troubled cells: a warp each, at most one warp per cell
      const long long want = (c.m.ncell + 7) / 8;
      const int grid = (int)std::max<long long>(1, std::min<long long>(want, 148LL * 4));
      weno_fix_kernel<P, T><<<grid, 256, 0, c.stream>>>(a);
      return launch_status("weno_kernel");
    }
  });
}

int launch_project_ic(const Ctx& c, const flsp_ic_desc* ic_dev, void* out) {
  const int threads = 128;
  const int blocks = (int)((c.m.ncell + threads - 1) / threads);
  return dispatch(c, [&](auto D, auto PP, auto tz) -> int {
    constexpr int DIM = decltype(D)::value, P = decltype(PP)::value;
    using T = decltype(tz);
    project_ic_kernel<DIM, P, T><<<blocks, threads, 0, c.stream>>>(c.m, ic_dev, reinterpret_cast<T*>(out));
    return launch_status("project_ic_kernel");
  });
}

int launch_static_cfl(const Ctx& c, const double* vtab64, int n_terms, const int* comp, int nmax,
                      int npt, DevClock* clk) {
  VelArgs<double> va;
  std::memset(&va, 0, sizeof(va));
  va.vtab = vtab64;
  va.n_terms = n_terms;
  va.nmax = nmax;
  va.npt = npt;
  for (int k = 0; k < n_terms; ++k) va.comp[k] = comp[k];
  const int threads = 256;
  const int blocks = (int)((c.m.ncell + threads - 1) / threads);
  if (c.dim == 2) static_cfl_kernel<2><<<blocks, threads, 0, c.stream>>>(c.m, va, clk);
  else static_cfl_kernel<3><<<blocks, threads, 0, c.stream>>>(c.m, va, clk);
  return launch_status("static_cfl_kernel");
}

int launch_fe_static_cfl(const Ctx& c, const double* u64, int pv, DevClock* clk) {
  const int nx = pv * c.m.n[0] + 1, ny = pv * c.m.n[1] + 1, nz = c.dim > 2 ? pv * c.m.n[2] + 1 : 1;
  const int threads = 256;
  const int blocks = (int)((c.m.ncell + threads - 1) / threads);
  if (c.dim == 2) fe_static_cfl_kernel<2><<<blocks, threads, 0, c.stream>>>(c.m, u64, pv, nx, ny, nz, clk);
  else fe_static_cfl_kernel<3><<<blocks, threads, 0, c.stream>>>(c.m, u64, pv, nx, ny, nz, clk);
  return launch_status("fe_static_cfl_kernel");
}

int launch_vel_tabulate(const Ctx& c, const double* vtab64, int n_terms, const int* comp, int nmax, int npt,
                        void* tab_q, void* tab_f, const long long* foff, const long long* nf) {
  VelTerms vt;
  term_ranges(comp, n_terms, vt.cstart);
  const int nq = c.p + 2;
  const int threads = 256;
  auto grid = [&](long long n) { return (int)std::max<long long>(1, std::min<long long>((n + threads - 1) / threads, 148LL * 32)); };
  const long long nqd = c.dim > 2 ? (long long)nq * nq * nq : (long long)nq * nq;
  const long long nqf = c.dim > 2 ? (long long)nq * nq : nq;
  auto run = [&](auto tz) -> int {
    using T = decltype(tz);
    T* q = static_cast<T*>(tab_q);
    T* f = static_cast<T*>(tab_f);
    if (c.dim == 2)
      vel_tabulate_cells<2, T><<<grid(nqd * c.m.ncell), threads, 0, c.stream>>>(c.m, vtab64, nmax, npt, vt, nq, q);
    else
      vel_tabulate_cells<3, T><<<grid(nqd * c.m.ncell), threads, 0, c.stream>>>(c.m, vtab64, nmax, npt, vt, nq, q);
    for (int e = 0; e < c.dim; ++e) {
      if (c.dim == 2)
        vel_tabulate_faces<2, T><<<grid(nqf * nf[e]), threads, 0, c.stream>>>(c.m, vtab64, nmax, npt, vt, nq, e, nf[e],
                                                                              f + foff[e]);
      else
        vel_tabulate_faces<3, T><<<grid(nqf * nf[e]), threads, 0, c.stream>>>(c.m, vtab64, nmax, npt, vt, nq, e, nf[e],
                                                                              f + foff[e]);
    }
    return launch_status("vel_tabulate");
  };
  return c.prec == FLSP_FP64 ? run(double(0)) : run(float(0));
}

int launch_fe_tabulate(const Ctx& c, const double* u64, int pv, const double (*gb)[kMaxNQ + 2], void* tab_q,
                       void* tab_f, const long long* foff, const long long* nf) {
  FeBasis fb;
  std::memcpy(fb.b, gb, sizeof(fb.b));
  const int nq = c.p + 2;
  const int threads = 256;
  auto grid = [&](long long n) { return (int)std::max<long long>(1, std::min<long long>((n + threads - 1) / threads, 148LL * 32)); };
  const long long nqd = c.dim > 2 ? (long long)nq * nq * nq : (long long)nq * nq;
  const long long nqf = c.dim > 2 ? (long long)nq * nq : nq;
  auto run = [&](auto tz) -> int {
    using T = decltype(tz);
    T* q = static_cast<T*>(tab_q);
    T* f = static_cast<T*>(tab_f);
    if (c.dim == 2) fe_tabulate_cells<2, T><<<grid(nqd * c.m.ncell), threads, 0, c.stream>>>(c.m, u64, pv, nq, fb, q);
    else fe_tabulate_cells<3, T><<<grid(nqd * c.m.ncell), threads, 0, c.stream>>>(c.m, u64, pv, nq, fb, q);
    for (int e = 0; e < c.dim; ++e) {
      if (c.dim == 2)
        fe_tabulate_faces<2, T><<<grid(nqf * nf[e]), threads, 0, c.stream>>>(c.m, u64, pv, nq, fb, e, nf[e], f + foff[e]);
      else
        fe_tabulate_faces<3, T><<<grid(nqf * nf[e]), threads, 0, c.stream>>>(c.m, u64, pv, nq, fb, e, nf[e], f + foff[e]);
    }
    return launch_status("fe_tabulate");
  };
  return c.prec == FLSP_FP64 ? run(double(0)) : run(float(0));
}

int reduce_blocks(const Ctx& c) { return (int)((c.m.ncell + 127) / 128); }

int launch_reduce(const Ctx& c, int which, const void* phi, const void* ref,
                  const flsp_ic_desc* ic_dev, double* partial, double* out_dev) {
  const int blocks = reduce_blocks(c);
  int st = dispatch(c, [&](auto D, auto PP, auto tz) -> int {
    constexpr int DIM = decltype(D)::value, P = decltype(PP)::value;
    using T = decltype(tz);
    RedArgs<T> a;
    std::memset(&a, 0, sizeof(a));
    a.m = c.m;
    a.phi = reinterpret_cast<const T*>(phi);
    a.ref = reinterpret_cast<const T*>(ref);
    a.ic = ic_dev;
    a.which = which;
    a.partial = partial;
    reduce_kernel<DIM, P, T><<<blocks, 128, 0, c.stream>>>(a);
    return launch_status("reduce_kernel");
  });
  if (st) return st;
  reduce_final<<<1, 256, 0, c.stream>>>(partial, blocks, which == FLSP_RED_MAX_ABS, out_dev);
  return launch_status("reduce_final");
}

static int grid_for(long long n) { return (int)std::min<long long>((n + 255) / 256, 148 * 16); }

int launch_scatter(const Ctx& c, const double* src, void* dst, const int64_t* perm) {
  const long long n = c.m.ncell * c.m.nb;
  if (c.prec == FLSP_FP64)
    scatter_state<double><<<grid_for(n), 256, 0, c.stream>>>(src, (double*)dst, perm, c.m.ncell, c.m.nb);
  else
    scatter_state<float><<<grid_for(n), 256, 0, c.stream>>>(src, (float*)dst, perm, c.m.ncell, c.m.nb);
  return launch_status("scatter_state");
}

int launch_gather(const Ctx& c, const void* src, double* dst, const int64_t* perm) {
  const long long n = c.m.ncell * c.m.nb;
  if (c.prec == FLSP_FP64)
    gather_state<double><<<grid_for(n), 256, 0, c.stream>>>((const double*)src, dst, perm, c.m.ncell, c.m.nb);
  else
    gather_state<float><<<grid_for(n), 256, 0, c.stream>>>((const float*)src, dst, perm, c.m.ncell, c.m.nb);
  return launch_status("gather_state");
}

int launch_nonfinite(const Ctx& c, const void* x, long long n, unsigned int* count) {
  if (c.prec == FLSP_FP64)
    nonfinite_kernel<double><<<grid_for(n), 256, 0, c.stream>>>((const double*)x, n, count);
  else
    nonfinite_kernel<float><<<grid_for(n), 256, 0, c.stream>>>((const float*)x, n, count);
  return launch_status("nonfinite_kernel");
}

int launch_adv_clock_begin(cudaStream_t s, DevClock* clk, const AdvClockArgs& a) {
  adv_clock_begin<<<1, 1, 0, s>>>(clk, a);
  return launch_status("adv_clock_begin");
}
int launch_adv_clock_end(cudaStream_t s, DevClock* clk) {
  adv_clock_end<<<1, 1, 0, s>>>(clk);
  return launch_status("adv_clock_end");
}
int launch_adv_clock_horizon(cudaStream_t s, DevClock* clk, double time_step) {
  adv_clock_horizon<<<1, 1, 0, s>>>(clk, time_step);
  return launch_status("adv_clock_horizon");
}
int launch_hj_clock_reset(cudaStream_t s, DevClock* clk) {
  hj_clock_reset<<<1, 1, 0, s>>>(clk);
  return launch_status("hj_clock_reset");
}
int launch_hj_clock_begin(cudaStream_t s, DevClock* clk, double cfl_max, int p, double nu,
                          double min_diam, double adv_scale) {
  hj_clock_begin<<<1, 1, 0, s>>>(clk, cfl_max, p, nu, min_diam, adv_scale);
  return launch_status("hj_clock_begin");
}
int launch_hj_clock_end(cudaStream_t s, DevClock* clk) {
  hj_clock_end<<<1, 1, 0, s>>>(clk);
  return launch_status("hj_clock_end");
}

}  // namespace flsp

// ======================================================================
// Allocation-free reduction (flsp_reduce_noalloc in include/flsp_dg.h).
//
// For callers that cannot allocate device memory (all their device memory
// comes from their own pool / arena): the partial sums live in a file-scope
// device array instead of a handle's buffer.  Host code must not use the
// array's name as an address (it is a host-side stand-in), so the device
// address is looked up once per device with cudaGetSymbolAddress while that
// device is current, and that pointer is passed to the kernels.  Every call
// on a device shares the array; each launch writes every partial slot it
// reads, so nothing has to be cleared between calls, but calls that overlap
// on the GPU race.
// ======================================================================
namespace {

constexpr int kNoAllocBlocks = 65536;                 // 128 cells per block
constexpr long long kNoAllocDoubles = 2LL * kNoAllocBlocks + 2;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];   // ~1 MiB
static __device__ __align__(256) flsp_ic_desc g_noalloc_ic;

// Set-up state per device ordinal, valid for the CUDA context it was made
// in: after cudaDeviceReset the next call on that device runs in a new
// primary context (new module, zeroed constant tables, possibly another
// symbol address), so the context's unique id is part of the key.
struct NoAllocDevice {
  unsigned long long ctx_id = 0;   // 0: not set up
  double* scratch = nullptr;
  flsp_ic_desc* ic = nullptr;
};
NoAllocDevice g_noalloc_dev[64];
std::mutex g_noalloc_mu[64];

// unique id of the calling thread's current CUDA context (driver entry
// points fetched through the runtime, so the library does not link libcuda)
int current_context_id(int dev, unsigned long long* id) {
  typedef CUresult (*GetCurrent)(CUcontext*);
  typedef CUresult (*GetId)(CUcontext, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", (void**)&get_current, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      get_current = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", (void**)&get_id, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      get_id = nullptr;
  });
  if (!get_current || !get_id) return flsp::set_error(FLSP_ERR_CUDA, "driver entry points cuCtxGetCurrent/cuCtxGetId");
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS) return flsp::set_error(FLSP_ERR_CUDA, "cuCtxGetCurrent failed");
  if (!ctx) {   // no context yet on this thread: make the device's primary context current
    cudaError_t e = cudaSetDevice(dev);
    if (e != cudaSuccess) return flsp::set_error(FLSP_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return flsp::set_error(FLSP_ERR_CUDA, "no current CUDA context");
  }
  if (get_id(ctx, id) != CUDA_SUCCESS) return flsp::set_error(FLSP_ERR_CUDA, "cuCtxGetId failed");
  return FLSP_OK;
}

// the IC description travels as a kernel parameter (copied at launch, so
// the caller's host struct is not read after the call returns)
__global__ void noalloc_set_ic(const flsp_ic_desc ic, flsp_ic_desc* dst) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *dst = ic;
}

__global__ void noalloc_finalize(const double* sums, int which, long long ndofs, double* result) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double r0 = sums[0], r1 = sums[1];
  double v = r0;
  if (which == FLSP_RED_MASS_ERROR) v = (r0 - r1) / r1;
  else if (which == FLSP_RED_MEAN_ABS_DIFF) v = r0 / (double)ndofs;
  else if (which == FLSP_RED_GRAD_DEVIATION) v = r0 / r1;
  else if (which == FLSP_RED_L2_ERROR_IC) v = sqrt(r0);
  *result = v;
}

}  // namespace

extern "C" int flsp_reduce_noalloc(const flsp_mesh_desc* mesh, int degree, int basis, int precision,
                                   const void* state, const void* ref_state, int which,
                                   const flsp_ic_desc* ic, double* result, void* stream) {
  using namespace flsp;
  if (!mesh || !state || !result) return set_error(FLSP_ERR_BAD_ARG, "null argument");
  if (mesh->dim < 2 || mesh->dim > 3) return set_error(FLSP_ERR_BAD_ARG, "dim must be 2 or 3");
  if (!supported_config(mesh->dim, degree)) return set_error(FLSP_ERR_UNSUPPORTED, "unsupported (dim, degree)");
  if (basis != FLSP_BASIS_P && basis != FLSP_BASIS_Q) return set_error(FLSP_ERR_BAD_ARG, "bad basis");
  if (precision != FLSP_FP64 && precision != FLSP_FP32) return set_error(FLSP_ERR_BAD_ARG, "bad precision");
  if (which < 0 || which > FLSP_RED_MASS_SHARP) return set_error(FLSP_ERR_BAD_ARG, "bad reduction kind");
  const bool need_ic = which == FLSP_RED_MASS_ERROR || which == FLSP_RED_L2_ERROR_IC ||
                       which == FLSP_RED_L1_INTERFACE_IC;
  const bool need_ref = which == FLSP_RED_L1_INTERFACE || which == FLSP_RED_MEAN_ABS_DIFF;
  if (need_ic && !ic) return set_error(FLSP_ERR_BAD_ARG, "this reduction needs an IC");
  if (need_ref && !ref_state) return set_error(FLSP_ERR_BAD_ARG, "this reduction needs ref_state");
  if (ic && (ic->n_nodes < 1 || ic->n_nodes > FLSP_MAX_IC_NODES || ic->root < 0 || ic->root >= ic->n_nodes ||
             ic->n_waves < 0 || ic->n_waves > FLSP_MAX_IC_WAVES))
    return set_error(FLSP_ERR_BAD_ARG, "bad IC description");
  long long ncell = 1;
  for (int d = 0; d < mesh->dim; ++d) {
    if (mesh->n[d] < 1 || !(mesh->hi[d] > mesh->lo[d])) return set_error(FLSP_ERR_BAD_MESH, "bad mesh");
    ncell *= mesh->n[d];
  }
  if (ncell > FLSP_NOALLOC_MAX_CELLS)
    return set_error(FLSP_ERR_BAD_ARG, "mesh has " + std::to_string(ncell) + " cells; flsp_reduce_noalloc "
                     "supports at most " + std::to_string(FLSP_NOALLOC_MAX_CELLS) + " (fixed scratch size)");

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_error(FLSP_ERR_NO_DEVICE, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= 64) return set_error(FLSP_ERR_BAD_ARG, "device ordinal out of range");
  unsigned long long ctx_id = 0;
  {
    const int st = current_context_id(dev, &ctx_id);
    if (st) return st;
  }
  double* scratch = nullptr;
  flsp_ic_desc* ic_dev = nullptr;
  {
    // once per device and context, with that device current
    std::lock_guard<std::mutex> lock(g_noalloc_mu[dev]);
    NoAllocDevice& nd = g_noalloc_dev[dev];
    if (nd.ctx_id != ctx_id) {
      nd.ctx_id = 0;
      int st = upload_tables_misc();
      if (st) return st;
      e = cudaGetSymbolAddress((void**)&nd.scratch, g_noalloc_scratch);
      if (e != cudaSuccess) return set_error(FLSP_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      e = cudaGetSymbolAddress((void**)&nd.ic, g_noalloc_ic);
      if (e != cudaSuccess) return set_error(FLSP_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      nd.ctx_id = ctx_id;
    }
    scratch = nd.scratch;
    ic_dev = nd.ic;
  }

  Ctx c;
  std::memset(&c, 0, sizeof(c));
  c.dim = mesh->dim;
  c.p = degree;
  c.prec = precision;
  c.basis = basis;
  c.stream = (cudaStream_t)stream;
  MeshArgs& m = c.m;
  double d2 = 0.0, vol = 1.0;
  for (int d = 0; d < 3; ++d) {
    m.n[d] = d < mesh->dim ? mesh->n[d] : 1;
    m.lo[d] = d < mesh->dim ? mesh->lo[d] : 0.0;
    m.h[d] = d < mesh->dim ? (mesh->hi[d] - mesh->lo[d]) / mesh->n[d] : 1.0;
    if (d < mesh->dim) { d2 += m.h[d] * m.h[d]; vol *= m.h[d]; }
  }
  m.ncell = ncell;
  m.vol = vol;
  m.diam = std::sqrt(d2);
  m.min_diam = m.diam;
  const int n1 = degree + 1, cz = mesh->dim > 2 ? degree : 0;
  std::memset(m.q2g, -1, sizeof(m.q2g));
  std::memset(m.g2q, 0, sizeof(m.g2q));
  int nb = 0;   // in-cell DoF order: lexicographic (Q) or PolynomialSpace (P: c outer, b, a inner)
  for (int cc = 0; cc <= cz; ++cc)
    for (int b = 0; b <= degree; ++b)
      for (int a = 0; a <= degree; ++a) {
        if (basis == FLSP_BASIS_P && a + b + cc > degree) continue;
        const int q = a + n1 * (b + n1 * cc);
        m.q2g[q] = (signed char)nb;
        m.g2q[nb++] = (signed char)q;
      }
  m.nb = nb;

  if (need_ic) {
    noalloc_set_ic<<<1, 1, 0, c.stream>>>(*ic, ic_dev);
    const int st = launch_status("noalloc_set_ic");
    if (st) return st;
  }
  double* partial = scratch;
  double* sums = scratch + 2LL * kNoAllocBlocks;
  int st = launch_reduce(c, which, state, need_ref ? ref_state : nullptr, need_ic ? ic_dev : nullptr, partial, sums);
  if (st) return st;
  noalloc_finalize<<<1, 1, 0, c.stream>>>(sums, which, ncell * nb, result);
  return launch_status("noalloc_finalize");
}

// ======================================================================
// Compute-restricted narrow band of the reinitialisation (no counterpart
// in the reference, whose sweep covers every cell).
// ======================================================================
namespace flsp {
namespace {

template <typename T>
__global__ void band_flags_kernel(const T* __restrict__ phi0, long long ncell, int nb, double thr,
                                  int* __restrict__ flags) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell;
       c += (long long)gridDim.x * blockDim.x)
    flags[c] = fabs((double)phi0[c * nb]) <= thr ? 1 : 0;
}

// one thread per tile: any flagged cell in the tile grown by `margin`?
__global__ void band_tiles_kernel(const int* __restrict__ flags, MeshArgs m, int dim, int margin,
                                  int* __restrict__ list, int* __restrict__ count) {
  const long long ntiles = (long long)m.ntile[0] * m.ntile[1] * m.ntile[2];
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ntiles;
       t += (long long)gridDim.x * blockDim.x) {
    const int bx = (int)(t % m.ntile[0]), by = (int)((t / m.ntile[0]) % m.ntile[1]),
              bz = (int)(t / ((long long)m.ntile[0] * m.ntile[1]));
    const int lo[3] = {bx * m.tile[0] - margin, by * m.tile[1] - margin, dim > 2 ? bz * m.tile[2] - margin : 0};
    const int hi[3] = {(bx + 1) * m.tile[0] + margin, (by + 1) * m.tile[1] + margin,
                       dim > 2 ? (bz + 1) * m.tile[2] + margin : 1};
    bool any = false;
    for (int z = max(lo[2], 0); z < min(hi[2], m.n[2]) && !any; ++z)
      for (int y = max(lo[1], 0); y < min(hi[1], m.n[1]) && !any; ++y)
        for (int x = max(lo[0], 0); x < min(hi[0], m.n[0]); ++x)
          if (flags[x + (long long)m.n[0] * (y + (long long)m.n[1] * z)]) {
            any = true;
            break;
          }
    if (any) list[atomicAdd(count, 1)] = (int)t;
  }
}

template <typename T>
__global__ void band_restore_kernel(const T* __restrict__ phi0, T* __restrict__ out, const int* __restrict__ flags,
                                    long long ncell, int nb) {
  const long long total = ncell * nb;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x)
    if (!flags[e / nb]) out[e] = phi0[e];
}

}  // namespace

int launch_band_flags(const Ctx& c, const void* phi0, double thr, int* flags) {
  const int blocks = grid_for(c.m.ncell);
  if (c.prec == FLSP_FP64)
    band_flags_kernel<double><<<blocks, 256, 0, c.stream>>>((const double*)phi0, c.m.ncell, c.m.nb, thr, flags);
  else
    band_flags_kernel<float><<<blocks, 256, 0, c.stream>>>((const float*)phi0, c.m.ncell, c.m.nb, thr, flags);
  return launch_status("band_flags_kernel");
}

int launch_band_tiles(const Ctx& c, const int* flags, const int* tile, int margin, int* list, int* count) {
  MeshArgs m = c.m;
  m.tiles = nullptr;
  m.n_tiles = nullptr;
  set_tile(m, c.dim, tile);
  cudaError_t e = cudaMemsetAsync(count, 0, sizeof(int), c.stream);
  if (e != cudaSuccess) return set_error(FLSP_ERR_CUDA, std::string("band tiles: ") + cudaGetErrorString(e));
  band_tiles_kernel<<<grid_for(nblocks(m)), 256, 0, c.stream>>>(flags, m, c.dim, margin, list, count);
  return launch_status("band_tiles_kernel");
}

namespace {
// running totals of the learned reinitialisation: band cells, and fallback
// cells when `with_fallback`
__global__ void learned_totals_kernel(const int* counts, unsigned long long* tot, int with_fallback) {
  if (threadIdx.x != 0) return;
  tot[0] += (unsigned long long)counts[0];
  if (with_fallback) tot[1] += (unsigned long long)counts[1];
}
}  // namespace

int launch_learned_totals(cudaStream_t s, const int* counts, unsigned long long* tot, int with_fallback) {
  learned_totals_kernel<<<1, 32, 0, s>>>(counts, tot, with_fallback);
  return launch_status("learned_totals_kernel");
}

namespace {
// flags[cells[i]] = list_flags[i] for the listed cells (the others zeroed before)
__global__ void band_flags_from_list_kernel(const int* __restrict__ cells, const int* __restrict__ list_flags,
                                            long long n, const int* __restrict__ n_dev, int* __restrict__ flags) {
  if (n_dev) n = min(n, (long long)*n_dev);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    if (list_flags[i]) flags[cells[i]] = 1;
}
}  // namespace

int launch_band_flags_from_list(const Ctx& c, const int* cells, const int* list_flags, long long n, const int* n_dev,
                                int* flags) {
  cudaError_t e = cudaMemsetAsync(flags, 0, (size_t)c.m.ncell * sizeof(int), c.stream);
  if (e != cudaSuccess) return set_error(FLSP_ERR_CUDA, std::string("band flags: ") + cudaGetErrorString(e));
  if (n <= 0) return FLSP_OK;
  band_flags_from_list_kernel<<<grid_for(n), 256, 0, c.stream>>>(cells, list_flags, n, n_dev, flags);
  return launch_status("band_flags_from_list_kernel");
}

int launch_band_restore(const Ctx& c, const void* phi0, void* out, const int* flags) {
  const int blocks = grid_for(c.m.ncell * c.m.nb);
  if (c.prec == FLSP_FP64)
    band_restore_kernel<double><<<blocks, 256, 0, c.stream>>>((const double*)phi0, (double*)out, flags, c.m.ncell,
                                                              c.m.nb);
  else
    band_restore_kernel<float><<<blocks, 256, 0, c.stream>>>((const float*)phi0, (float*)out, flags, c.m.ncell,
                                                             c.m.nb);
  return launch_status("band_restore_kernel");
}

}  // namespace flsp

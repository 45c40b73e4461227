// flsp_k_misc.cu — limiter, projection, reductions, clocks, DoF order
// (instantiations + launchers).
#include <algorithm>
#include <cstring>

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

static const int kWenoTile[3] = {16, 16, 1};

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

int launch_weno(const Ctx& c, const void* in, void* out, unsigned int* count) {
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
      a.in = reinterpret_cast<const T*>(in);
      a.out = reinterpret_cast<T*>(out);
      a.count = count;
      const size_t smem = weno_smem_bytes<P, T>(a.m.tile);
      weno_kernel<P, T><<<(unsigned)nblocks(a.m), kWenoTile[0] * kWenoTile[1], smem, c.stream>>>(a);
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

// flsp_k_batch.cu — batched problems: many independent 2D level-set
// problems (their own meshes, degrees 1..3, velocities and clocks) advance
// in ONE persistent launch per RK stage (and one per reinit pseudo-step and
// limiter pass) per degree.  A block walks a list of work items (problem,
// tile) of one degree and runs the same per-tile bodies as the
// single-problem kernels (adv_stage_tile, hjq_tile, weno_tile); each degree
// has its own instantiation, so its registers, shared memory and occupancy
// are its own, not those of the most demanding degree in the batch.  The
// tile shapes are launch parameters picked by the batch autotuner.
#include <algorithm>
#include <cstring>
#include <string>
#include <type_traits>

#include "flsp_advect.cuh"
#include "flsp_clock.cuh"
#include "flsp_hjq.cuh"
#include "flsp_launch.h"
#include "flsp_tables.h"
#include "flsp_weno.cuh"

namespace flsp {

int upload_tables_batch() {
  cudaError_t e = upload_tables_here();
  if (e != cudaSuccess) return set_error(FLSP_ERR_CUDA, std::string("tables: ") + cudaGetErrorString(e));
  return FLSP_OK;
}

namespace {

// per-item argument structs are assembled (in shared memory, by one
// thread) from the problem's descriptor and the launch's buffer roles
template <typename T>
__device__ __forceinline__ void make_adv_args(const BatchProb& pr, int ix, int in_n, int iout, int stage, int combine,
                                              AdvArgs<T>& a) {
  a.m = pr.m_adv;
  a.v.vtab = reinterpret_cast<const T*>(pr.vtab);
  a.v.n_terms = pr.n_terms;
  a.v.nmax = pr.nmax;
  a.v.npt = pr.npt;
#pragma unroll 1
  for (int k = 0; k < kMaxTerms; ++k) a.v.comp[k] = pr.comp[k];
  term_ranges(pr.comp, pr.n_terms, a.v.cstart);
  a.v.tab_q = reinterpret_cast<const T*>(pr.tab_q);
  a.v.tab_f = reinterpret_cast<const T*>(pr.tab_f);
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    a.v.tab_foff[e] = pr.tab_foff[e];
    a.v.tab_nf[e] = pr.tab_nf[e];
  }
  a.phi_s = reinterpret_cast<const T*>(pr.buf[ix]);
  a.phi_n = reinterpret_cast<const T*>(pr.buf[in_n]);
  a.out = reinterpret_cast<T*>(pr.buf[iout]);
  a.clk = pr.clk;
  a.stage = stage;
  a.combine = combine;
  a.ct_explicit = 0.0;
  a.dt_explicit = 0.0;
}

template <typename T, int P>
__global__ void __launch_bounds__(256, 2)
    batch_adv_kernel(const BatchProb* __restrict__ probs, const int2* __restrict__ items, int n_items, int ix,
                     int in_n, int iout, int stage, int combine) {
  // the item's arguments are assembled once per block in shared memory
  // (every thread reads them, like a plain launch's kernel parameters)
  __shared__ AdvArgs<T> a;
  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const int2 w = items[it];
    if (threadIdx.x == 0) make_adv_args<T>(probs[w.x], ix, in_n, iout, stage, combine, a);
    __syncthreads();
    adv_stage_tile<2, P, T, true>(a, w.y);   // velocity from the problem's tables
    __syncthreads();   // shared memory is reused by the next item
  }
}

template <typename T, int P>
__global__ void __launch_bounds__(128)
    batch_hj_kernel(const BatchProb* __restrict__ probs, const int2* __restrict__ items, int n_items, int isrc,
                    int iphi0, int idst, int mode, int rk) {
  __shared__ HJArgs<T> a;
  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const int2 w = items[it];
    if (threadIdx.x == 0) {
      const BatchProb& pr = probs[w.x];
      a.m = pr.m_hj;
      a.phi = reinterpret_cast<const T*>(pr.buf[isrc]);
      a.phi0 = reinterpret_cast<const T*>(pr.buf[iphi0]);
      a.out = idst >= 0 ? reinterpret_cast<T*>(pr.buf[idst]) : nullptr;
      a.clk = pr.clk;
      a.mode = mode;
      a.rk = rk;
      a.dt_explicit = 0.0;
      a.block = pr.m_hj.ncell * pr.m_hj.nb;
      a.rdiff = nullptr;
    }
    __syncthreads();
    hjq_tile<2, P, T>(a, w.y);
    __syncthreads();
  }
}

template <typename T, int P>
__global__ void __launch_bounds__(256, 2)
    batch_weno_kernel(const BatchProb* __restrict__ probs, const int2* __restrict__ items, int n_items, int iin,
                      int iout, int2* list, unsigned int* list_n) {
  __shared__ WenoArgs<T> a;
  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const int2 w = items[it];
    if (threadIdx.x == 0) {
      const BatchProb& pr = probs[w.x];
      a.m = pr.m_weno;
      a.in = reinterpret_cast<const T*>(pr.buf[iin]);
      a.out = reinterpret_cast<T*>(pr.buf[iout]);
      a.count = nullptr;
      a.list = list;
      a.list_n = list_n;
      a.problem = w.x;
    }
    __syncthreads();
    weno_tile<P, T>(a, w.y);
    __syncthreads();
  }
}

// the troubled cells of every problem of the launch's degree: a warp each
template <typename T, int P>
__global__ void __launch_bounds__(256)
    batch_weno_fix_kernel(const BatchProb* __restrict__ probs, const int2* __restrict__ list,
                          const unsigned int* __restrict__ list_n, int iin, int iout) {
  constexpr int NM = (P + 1) * (P + 1);
  __shared__ T sh[8][5 * NM];
  const int wl = threadIdx.x >> 5;
  const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  const unsigned int n = *list_n;
  for (unsigned int i = warp; i < n; i += nwarps) {
    const int2 e = list[i];
    const BatchProb& pr = probs[e.x];
    weno_fix<P, T>(pr.m_weno, reinterpret_cast<const T*>(pr.buf[iin]), reinterpret_cast<T*>(pr.buf[iout]), e.y,
                   sh[wl]);
  }
}

// clocks: one thread per problem
__global__ void batch_clock_kernel(const BatchProb* __restrict__ probs, int n, int what, double cfl_max) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const BatchProb& pr = probs[i];
  switch (what) {
    case kBatchAdvBegin: adv_clock_begin_body(pr.clk, pr.ca); break;
    case kBatchAdvEnd: adv_clock_end_body(pr.clk); break;
    case kBatchAdvHorizon: adv_clock_horizon_body(pr.clk, __longlong_as_double(0x7ff0000000000000LL)); break;
    case kBatchHjReset: hj_clock_reset_body(pr.clk); break;
    case kBatchHjBegin: hj_clock_begin_body(pr.clk, cfl_max, pr.p, 0.0, pr.m_hj.min_diam, pr.adv_scale); break;
    default: hj_clock_end_body(pr.clk); break;
  }
}

template <typename K>
int persistent_grid(K kern, int threads, size_t smem, int n_items) {
  int per_sm = 0, dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  return std::max(1, std::min(n_items, nsm * per_sm));
}

}  // namespace

int batch_smem(int kind, int p, int prec, const int* tile, int n_terms, size_t* bytes) {
  auto go = [&](auto tz) -> size_t {
    using T = decltype(tz);
    if (kind == kBatchKindAdv) {
      switch (p) {
        case 1: return adv_smem_bytes<2, 1, T>(tile, std::max(n_terms, 1), true);
        case 2: return adv_smem_bytes<2, 2, T>(tile, std::max(n_terms, 1), true);
        default: return adv_smem_bytes<2, 3, T>(tile, std::max(n_terms, 1), true);
      }
    } else if (kind == kBatchKindHJ) {
      switch (p) {
        case 1: return hjq_smem_bytes<2, 1, T>(tile);
        case 2: return hjq_smem_bytes<2, 2, T>(tile);
        default: return hjq_smem_bytes<2, 3, T>(tile);
      }
    }
    switch (p) {
      case 1: return weno_smem_bytes<1, T>(tile);
      case 2: return weno_smem_bytes<2, T>(tile);
      default: return weno_smem_bytes<3, T>(tile);
    }
  };
  *bytes = prec == FLSP_FP64 ? go((double)0) : go((float)0);
  return FLSP_OK;
}

int launch_batch_clock(cudaStream_t s, const BatchProb* probs, int n, int what, double cfl_max) {
  batch_clock_kernel<<<(n + 127) / 128, 128, 0, s>>>(probs, n, what, cfl_max);
  return launch_status("batch_clock_kernel");
}

// f(integral_constant<int, p>) for the degree p in 1..3
template <typename F>
int with_degree(int p, F&& f) {
  switch (p) {
    case 1: return f(std::integral_constant<int, 1>());
    case 2: return f(std::integral_constant<int, 2>());
    case 3: return f(std::integral_constant<int, 3>());
  }
  return set_error(FLSP_ERR_UNSUPPORTED, "batched problems: degree 1..3");
}

template <typename T, int P>
static int batch_attr(int kind, size_t smem) {
  cudaError_t e = cudaSuccess;
  const int s = (int)smem;
  if (kind == kBatchKindAdv) e = cudaFuncSetAttribute(batch_adv_kernel<T, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, s);
  else if (kind == kBatchKindHJ) e = cudaFuncSetAttribute(batch_hj_kernel<T, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, s);
  else e = cudaFuncSetAttribute(batch_weno_kernel<T, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, s);
  if (e != cudaSuccess) return set_error(FLSP_ERR_CUDA, std::string("batch attr: ") + cudaGetErrorString(e));
  return FLSP_OK;
}

int batch_prepare(int kind, int prec, int p, size_t smem, int threads, int n_items, int* grid) {
  if (smem > 227 * 1024) return set_error(FLSP_ERR_BAD_ARG, "batch tile too large for shared memory");
  return with_degree(p, [&](auto PC) -> int {
    constexpr int P = decltype(PC)::value;
    int st = prec == FLSP_FP64 ? batch_attr<double, P>(kind, smem) : batch_attr<float, P>(kind, smem);
    if (st) return st;
    auto g = [&](auto tz) -> int {
      using T = decltype(tz);
      if (kind == kBatchKindAdv) return persistent_grid(batch_adv_kernel<T, P>, threads, smem, n_items);
      if (kind == kBatchKindHJ) return persistent_grid(batch_hj_kernel<T, P>, threads, smem, n_items);
      return persistent_grid(batch_weno_kernel<T, P>, threads, smem, n_items);
    };
    *grid = prec == FLSP_FP64 ? g((double)0) : g((float)0);
    return FLSP_OK;
  });
}

int launch_batch_adv(cudaStream_t s, int prec, int p, const BatchProb* probs, const int2* items, int n_items,
                     int grid, int threads, size_t smem, int ix, int in_n, int iout, int stage, int combine) {
  return with_degree(p, [&](auto PC) -> int {
    constexpr int P = decltype(PC)::value;
    if (prec == FLSP_FP64)
      batch_adv_kernel<double, P><<<grid, threads, smem, s>>>(probs, items, n_items, ix, in_n, iout, stage, combine);
    else
      batch_adv_kernel<float, P><<<grid, threads, smem, s>>>(probs, items, n_items, ix, in_n, iout, stage, combine);
    return launch_status("batch_adv_kernel");
  });
}

int launch_batch_hj(cudaStream_t s, int prec, int p, const BatchProb* probs, const int2* items, int n_items,
                    int grid, int threads, size_t smem, int isrc, int iphi0, int idst, int mode, int rk) {
  return with_degree(p, [&](auto PC) -> int {
    constexpr int P = decltype(PC)::value;
    if (prec == FLSP_FP64)
      batch_hj_kernel<double, P><<<grid, threads, smem, s>>>(probs, items, n_items, isrc, iphi0, idst, mode, rk);
    else
      batch_hj_kernel<float, P><<<grid, threads, smem, s>>>(probs, items, n_items, isrc, iphi0, idst, mode, rk);
    return launch_status("batch_hj_kernel");
  });
}

int launch_batch_weno(cudaStream_t s, int prec, int p, const BatchProb* probs, const int2* items, int n_items,
                      int grid, int threads, size_t smem, int iin, int iout, int2* list, unsigned int* list_n,
                      long long n_cells) {
  cudaError_t e = cudaMemsetAsync(list_n, 0, sizeof(unsigned int), s);
  if (e != cudaSuccess) return set_error(FLSP_ERR_CUDA, std::string("batch weno list: ") + cudaGetErrorString(e));
  const int fix_grid = (int)std::max<long long>(1, std::min<long long>((n_cells + 7) / 8, 148LL * 4));
  return with_degree(p, [&](auto PC) -> int {
    constexpr int P = decltype(PC)::value;
    if (prec == FLSP_FP64) {
      batch_weno_kernel<double, P><<<grid, threads, smem, s>>>(probs, items, n_items, iin, iout, list, list_n);
      batch_weno_fix_kernel<double, P><<<fix_grid, 256, 0, s>>>(probs, list, list_n, iin, iout);
    } else {
      batch_weno_kernel<float, P><<<grid, threads, smem, s>>>(probs, items, n_items, iin, iout, list, list_n);
      batch_weno_fix_kernel<float, P><<<fix_grid, 256, 0, s>>>(probs, list, list_n, iin, iout);
    }
    return launch_status("batch_weno_kernel");
  });
}

}  // namespace flsp

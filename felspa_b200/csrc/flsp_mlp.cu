// flsp_mlp.cu — the learned reinitialisation's network: BF16 tensor-core
// forward / backward (tcgen05 GEMMs, flsp_tc.cuh), Adam, the patch
// features of a level-set state, band selection and the fallback merge.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "flsp_launch.h"
#include "flsp_mlp.h"
#include "flsp_tc.cuh"

namespace flsp {

#define MCU(x)                                                                          \
  do {                                                                                  \
    cudaError_t e_ = (x);                                                               \
    if (e_ != cudaSuccess) return set_error(FLSP_ERR_CUDA, std::string(#x ": ") + cudaGetErrorString(e_)); \
  } while (0)
#define MST(x)                 \
  do {                         \
    int s_ = (x);              \
    if (s_ != FLSP_OK) return s_; \
  } while (0)

static int grid_of(long long n, int threads = 256) {
  return (int)std::max(1LL, std::min<long long>((n + threads - 1) / threads, 148LL * 32));
}

// ------------------------------------------------------------------ kernels
// dst(r, k) of a packed R x K operand = scale * src[(idx ? idx[r] : r) * ld_r
// + k * ld_c] inside rows x cols, zero in the padding
__global__ void k_pack(const float* __restrict__ src, const int* __restrict__ idx, long long ld_r,
                       long long ld_c, int rows, int cols, float scale, __nv_bfloat16* __restrict__ dst,
                       int R, int K, const int* __restrict__ rows_dev) {
  // with a device-side row count only the 128-row tiles that hold rows are written
  if (rows_dev) rows = min(rows, *rows_dev);
  const int Rw = rows_dev ? min(R, ((rows + 127) / 128) * 128) : R;
  const long long total = (long long)Rw * K;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(e / K), k = (int)(e % K);
    float v = 0.0f;
    if (r < rows && k < cols) {
      const long long sr = idx ? idx[r] : r;
      v = scale * src[sr * ld_r + (long long)k * ld_c];
    }
    dst[packed_off(r, k, R)] = __float2bfloat16_rn(v);
  }
}

// packed R x C -> packed dst_rows x R (transpose); rows C..dst_rows-1 zero.
// One thread per 8 x 8 core matrix.
__global__ void k_transpose_packed(const __nv_bfloat16* __restrict__ src, int R, int C,
                                   __nv_bfloat16* __restrict__ dst, int dst_rows) {
  const long long total = (long long)(dst_rows / 8) * (R / 8);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int cg = (int)(t % (dst_rows / 8)), rg = (int)(t / (dst_rows / 8));
    uint4* d = reinterpret_cast<uint4*>(dst + packed_off((long long)cg * 8, (long long)rg * 8, dst_rows));
    if (cg >= C / 8) {
#pragma unroll
      for (int i = 0; i < 8; ++i) d[i] = make_uint4(0, 0, 0, 0);
      continue;
    }
    const uint4* s = reinterpret_cast<const uint4*>(src + packed_off((long long)rg * 8, (long long)cg * 8, R));
    unsigned short in[64], out[64];
#pragma unroll
    for (int i = 0; i < 8; ++i) *reinterpret_cast<uint4*>(&in[8 * i]) = s[i];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) out[8 * j + i] = in[8 * i + j];
#pragma unroll
    for (int i = 0; i < 8; ++i) d[i] = *reinterpret_cast<const uint4*>(&out[8 * i]);
  }
}

// output-layer gradient, packed R x 64: g = dy[r][n] (given) or
// 2 (y - t) / (B * OUT) (MSE of the batch); per-block loss and column sums
// (col_part row stride ldy)
template <int OUT>
__global__ void k_out_grad(const float* __restrict__ y, int ldy, const float* __restrict__ dy,
                           const float* __restrict__ targ, const int* __restrict__ idx, int B, int R,
                           __nv_bfloat16* __restrict__ gout, double* __restrict__ loss_part,
                           float* __restrict__ col_part) {
  constexpr int kMlpOut = OUT;
  static_assert(OUT <= 64, "output gradient rows are 64 wide");
  __shared__ double sl[256];
  __shared__ float sc[256][kMlpOut];
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  double l = 0.0;
  __align__(16) __nv_bfloat16 row[64];
#pragma unroll
  for (int k = 0; k < 64; ++k) row[k] = __float2bfloat16_rn(0.0f);
  float gv[kMlpOut];
#pragma unroll
  for (int n = 0; n < kMlpOut; ++n) gv[n] = 0.0f;
  if (r < B) {
    const long long tr = idx ? idx[r] : r;
#pragma unroll
    for (int n = 0; n < kMlpOut; ++n) {
      float g;
      if (dy) {
        g = dy[(long long)r * kMlpOut + n];
      } else {
        const float d = y[(long long)r * ldy + n] - targ[tr * kMlpOut + n];
        l += (double)d * d;
        g = 2.0f * d / (float)((double)B * kMlpOut);
      }
      gv[n] = g;
      row[n] = __float2bfloat16_rn(g);
    }
  }
  if (r < R) {
#pragma unroll
    for (int kb = 0; kb < 8; ++kb)
      *reinterpret_cast<uint4*>(gout + packed_off(r, kb * 8, R)) = *reinterpret_cast<const uint4*>(&row[kb * 8]);
  }
  sl[threadIdx.x] = l;
#pragma unroll
  for (int n = 0; n < kMlpOut; ++n) sc[threadIdx.x][n] = gv[n];
  __syncthreads();
  if (threadIdx.x < kMlpOut + 1) {
    // fixed-order sums: thread n < OUT sums column n, thread OUT the loss
    double s = 0.0;
    for (int i = 0; i < (int)blockDim.x; ++i) s += threadIdx.x < kMlpOut ? (double)sc[i][threadIdx.x] : sl[i];
    if (threadIdx.x < kMlpOut) col_part[(long long)blockIdx.x * ldy + threadIdx.x] = (float)s;
    else loss_part[blockIdx.x] = s;
  }
}

// out[n] = sum_p part[p * ld + n] in a fixed order, n < n_valid
__global__ void k_colsum(const float* __restrict__ part, int P, int ld, int n_valid, float* __restrict__ out) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= n_valid) return;
  double s = 0.0;
  for (int p = 0; p < P; ++p) s += part[(long long)p * ld + n];
  out[n] = (float)s;
}

__global__ void k_sum_double(const double* __restrict__ part, int P, double* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s = 0.0;
  for (int p = 0; p < P; ++p) s += part[p];
  *out = s;
}

__global__ void k_adam(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ g, long long n, float lr, float b1, float b2, float eps,
                       float bc1, float bc2) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  }
}

// ---- level-set patch kernels (degree 2, Q basis: NB = 3^dim coefficients
// per cell, lexicographic cells)
// one thread per (listed cell, patch cell): the patch cell's coefficients
// over h; the centre cell also writes 64 h at the end of the row.  Patch
// cells outside the domain repeat the nearest inside cell.
template <int DIM, typename T>
__global__ void k_patch_features(const T* __restrict__ s, int nx, int ny, int nz, float ih, float hfeat,
                                 const int* __restrict__ cells, long long n, const int* __restrict__ n_dev,
                                 float* __restrict__ feat) {
  constexpr int NB = DIM == 2 ? 9 : 27, NP = DIM == 2 ? 9 : 27, NIN = NP * NB + 1;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n_dev) n = min(n, (long long)*n_dev);
  if (t >= n * NP) return;
  const long long i = t / NP;
  const int j = (int)(t % NP);   // patch cell: z outer, y, x inner
  const long long c = cells[i];
  const int cx = (int)(c % nx), cy = (int)((c / nx) % ny), cz = DIM > 2 ? (int)(c / ((long long)nx * ny)) : 0;
  const int px = min(max(cx + j % 3 - 1, 0), nx - 1), py = min(max(cy + (j / 3) % 3 - 1, 0), ny - 1);
  const int pz = DIM > 2 ? min(max(cz + j / 9 - 1, 0), nz - 1) : 0;
  const T* src = s + (((long long)pz * ny + py) * nx + px) * NB;
  float* dst = feat + i * NIN + j * NB;
#pragma unroll
  for (int q = 0; q < NB; ++q) dst[q] = (float)src[q] * ih;
  if (j == NP / 2) feat[i * NIN + NIN - 1] = hfeat;
}

template <typename T>
__global__ void k_patch_targets(const T* __restrict__ pre, const T* __restrict__ post, int nb, float ih,
                                const int* __restrict__ cells, long long n, float* __restrict__ targ) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n * nb) return;
  const long long i = t / nb;
  const int q = (int)(t % nb);
  const long long c = cells[i];
  targ[i * nb + q] = (float)((double)post[c * nb + q] - (double)pre[c * nb + q]) * ih;
}

template <typename T>
__global__ void k_apply_delta(T* __restrict__ out, int nb, double h, const int* __restrict__ cells, long long n,
                              const int* __restrict__ n_dev, const float* __restrict__ y, int ldy) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n_dev) n = min(n, (long long)*n_dev);
  if (t >= n * nb) return;
  const long long i = t / nb;
  const int q = (int)(t % nb);
  const long long c = cells[i];
  out[c * nb + q] = (T)((double)out[c * nb + q] + h * (double)y[i * ldy + q]);
}

// band flags and per-block counts (256 cells per block)
template <typename T>
__global__ void k_band_count(const T* __restrict__ s, long long ncell, int nb, double thr, int* __restrict__ flags,
                             int* __restrict__ bcount) {
  const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int f = (c < ncell && fabs((double)s[c * nb]) <= thr) ? 1 : 0;
  if (c < ncell) flags[c] = f;
  const int w = __syncthreads_count(f);
  if (threadIdx.x == 0) bcount[blockIdx.x] = w;
}
// exclusive scan of the block counts (one block, fixed order); total -> *count
__global__ void k_scan_counts(const int* __restrict__ bcount, int nblk, int* __restrict__ boff, int* __restrict__ count) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int s = 0;
  for (int b = 0; b < nblk; ++b) {
    boff[b] = s;
    s += bcount[b];
  }
  *count = s;
}
__global__ void k_band_compact(const int* __restrict__ flags, long long ncell, const int* __restrict__ boff,
                               int* __restrict__ cells) {
  __shared__ int wsum[8];
  const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int f = c < ncell ? flags[c] : 0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned ball = __ballot_sync(0xffffffffu, f);
  if (lane == 0) wsum[warp] = __popc(ball);
  __syncthreads();
  int base = boff[blockIdx.x];
  for (int w = 0; w < warp; ++w) base += wsum[w];
  if (f) cells[base + __popc(ball & ((1u << lane) - 1u))] = (int)c;
}

// mean of ||grad phi| - 1| over the 3 x 3 Gauss points of each listed cell
// mean over the cell's 3^dim Gauss points of ||grad phi| - 1| (degree-2
// Legendre modes on [0,1] per axis, Q layout a + 3 b (+ 9 c))
template <int DIM, typename T>
__global__ void k_residual(const T* __restrict__ s, double ih, const int* __restrict__ cells, long long n,
                           const int* __restrict__ n_dev, double thr, int* __restrict__ flags, int* __restrict__ count) {
  constexpr int NB = DIM == 2 ? 9 : 27;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n_dev) n = min(n, (long long)*n_dev);
  if (i >= n) return;
  const T* c = s + (long long)cells[i] * NB;
  const double g[3] = {0.5 - 0.5 * 0.7745966692414834, 0.5, 0.5 + 0.5 * 0.7745966692414834};
  const double w[3] = {5.0 / 18.0, 8.0 / 18.0, 5.0 / 18.0};
  const double r3 = 1.7320508075688772, r5 = 2.23606797749979;
  double Lv[3][3], Dv[3][3];   // [point][mode]
  for (int k = 0; k < 3; ++k) {
    const double x = g[k];
    Lv[k][0] = 1.0;
    Lv[k][1] = r3 * (2 * x - 1);
    Lv[k][2] = r5 * (6 * x * x - 6 * x + 1);
    Dv[k][0] = 0.0;
    Dv[k][1] = 2 * r3;
    Dv[k][2] = r5 * (12 * x - 6);
  }
  double acc = 0.0;
  for (int qz = 0; qz < (DIM > 2 ? 3 : 1); ++qz)
    for (int qy = 0; qy < 3; ++qy)
      for (int qx = 0; qx < 3; ++qx) {
        double gx = 0.0, gy = 0.0, gz = 0.0;
        for (int cc = 0; cc < (DIM > 2 ? 3 : 1); ++cc) {
          const double lz = DIM > 2 ? Lv[qz][cc] : 1.0, dz = DIM > 2 ? Dv[qz][cc] : 0.0;
          for (int b = 0; b < 3; ++b)
            for (int a = 0; a < 3; ++a) {
              const double v = (double)c[a + 3 * b + 9 * cc];
              gx += v * Dv[qx][a] * Lv[qy][b] * lz;
              gy += v * Lv[qx][a] * Dv[qy][b] * lz;
              gz += v * Lv[qx][a] * Lv[qy][b] * dz;
            }
        }
        const double wq = w[qx] * w[qy] * (DIM > 2 ? w[qz] : 1.0);
        acc += wq * fabs(sqrt(gx * gx + gy * gy + gz * gz) * ih - 1.0);
      }
  const int f = acc > thr ? 1 : 0;
  flags[i] = f;
  if (f) atomicAdd(count, 1);
}

template <typename T>
__global__ void k_merge(const T* __restrict__ src, T* __restrict__ out, int nb, const int* __restrict__ cells,
                        const int* __restrict__ flags, long long n, const int* __restrict__ n_dev) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n_dev) n = min(n, (long long)*n_dev);
  if (t >= n * nb) return;
  const long long i = t / nb;
  if (!flags[i]) return;
  const long long c = cells[i];
  const int q = (int)(t % nb);
  out[c * nb + q] = src[c * nb + q];
}

// y[r][c] = sum_s part[s][r][c] (fixed order) for r < rows, c < cols
__global__ void k_split_sum(const float* __restrict__ part, int splits, long long stride, int rows, int cols,
                            int ldp, float* __restrict__ y, int ldy) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)rows * cols) return;
  const int r = (int)(t / cols), c = (int)(t % cols);
  float acc = 0.0f;
  for (int s = 0; s < splits; ++s) acc += part[s * stride + (long long)r * ldp + c];
  y[(long long)r * ldy + c] = acc;
}

// ------------------------------------------------------------------ GEMM launch
// the kernel's shared-memory attribute, once per epilogue and device
template <int EPI>
static int gemm_attr() {
  static bool attr_done[4][64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && !attr_done[EPI][dev]) {
    MCU(cudaFuncSetAttribute(tc_gemm_kernel<EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)tc_gemm_smem(256)));
    attr_done[EPI][dev] = true;
  }
  return FLSP_OK;
}

template <int EPI>
static int gemm(cudaStream_t st, const TcGemmArgs& a, int ksplit = 1) {
  if (a.M % kTcBM || a.N % 16 || a.N > 256 || a.N < 16 || a.K % kTcBK || a.K <= 0)
    return set_error(FLSP_ERR_BAD_ARG, "tensor-core GEMM: unsupported shape");
  if (ksplit < 1 || ksplit > a.K / kTcBK || (ksplit > 1 && EPI != kEpiStoreF32))
    return set_error(FLSP_ERR_BAD_ARG, "tensor-core GEMM: bad K split");
  const size_t smem = tc_gemm_smem(a.N);
  MST(gemm_attr<EPI>());
  tc_gemm_kernel<EPI><<<dim3(a.M / kTcBM, ksplit), 128, smem, st>>>(a);
  return launch_status("tc_gemm_kernel");
}

static int transpose(cudaStream_t st, const __nv_bfloat16* src, int R, int C, __nv_bfloat16* dst, int dst_rows) {
  const long long total = (long long)(dst_rows / 8) * (R / 8);
  k_transpose_packed<<<grid_of(total), 256, 0, st>>>(src, R, C, dst, dst_rows);
  return launch_status("k_transpose_packed");
}

static long long round128(long long n) { return ((n + 127) / 128) * 128; }

// ------------------------------------------------------------------ host side
int mlp_ensure_cap(flsp_mlp* net, int64_t rows) {
  // kernel attributes here too: callers size the buffers before a capture
  MST(gemm_attr<kEpiHidden>());
  MST(gemm_attr<kEpiOutput>());
  MST(gemm_attr<kEpiBackAct>());
  MST(gemm_attr<kEpiStoreF32>());
  const int64_t need = round128(std::max<int64_t>(rows, 128));
  if (net->cap >= need) return FLSP_OK;
  auto fr = [](void* p) { if (p) cudaFree(p); };
  fr(net->x);
  for (int i = 0; i < 4; ++i) { fr(net->act[i]); fr(net->gd[i]); }
  fr(net->y); fr(net->gout); fr(net->gh[0]); fr(net->gh[1]); fr(net->tA); fr(net->tG);
  fr(net->colsum); fr(net->loss_part);
  net->cap = 0;
  const size_t c = (size_t)need;
  MCU(cudaMalloc(&net->x, c * net->k_in * 2));
  for (int i = 0; i < 4; ++i) {
    MCU(cudaMalloc(&net->act[i], c * 256 * 2));
    MCU(cudaMalloc(&net->gd[i], c * 256 * 4));
  }
  MCU(cudaMalloc(&net->y, c * net->y_ld * 4));
  MCU(cudaMalloc(&net->gout, c * 64 * 2));
  MCU(cudaMalloc(&net->gh[0], c * 256 * 2));
  MCU(cudaMalloc(&net->gh[1], c * 256 * 2));
  MCU(cudaMalloc(&net->tA, c * std::max(256, net->k_in) * 2));
  MCU(cudaMalloc(&net->tG, c * 256 * 2));
  MCU(cudaMalloc(&net->colsum, (c / 32 + 1) * 256 * 4));
  if (!net->split) MCU(cudaMalloc(&net->split, (size_t)kMlpSplits * 256 * 256 * 4));
  MCU(cudaMalloc(&net->loss_part, (c / 256 + 1) * 8));
  net->cap = need;
  return FLSP_OK;
}

int mlp_ensure_pairs(flsp_mlp* net, int64_t n) {
  if (net->pair_cap >= n) return FLSP_OK;
  const int64_t cap = std::max<int64_t>(n, std::max<int64_t>(2 * net->pair_cap, 1 << 16));
  float *f = nullptr, *t = nullptr;
  MCU(cudaMalloc(&f, (size_t)cap * net->n_in * 4));
  MCU(cudaMalloc(&t, (size_t)cap * net->n_out * 4));
  if (net->n_pairs) {
    MCU(cudaMemcpyAsync(f, net->feat, (size_t)net->n_pairs * net->n_in * 4, cudaMemcpyDeviceToDevice, net->stream));
    MCU(cudaMemcpyAsync(t, net->targ, (size_t)net->n_pairs * net->n_out * 4, cudaMemcpyDeviceToDevice,
                        net->stream));
    MCU(cudaStreamSynchronize(net->stream));
  }
  if (net->feat) cudaFree(net->feat);
  if (net->targ) cudaFree(net->targ);
  net->feat = f;
  net->targ = t;
  net->pair_cap = cap;
  return FLSP_OK;
}

// packed BF16 weights and their transposes from the FP32 master copy
static int repack(flsp_mlp* net) {
  for (int l = 0; l < kMlpLayers; ++l) {
    const MlpLayer& L = net->L[l];
    const float* W = net->p + L.w_off;
    const long long nw = (long long)L.n_pad * L.k_pad;
    k_pack<<<grid_of(nw), 256, 0, net->stream>>>(W, nullptr, L.n_in, 1, L.n_out, L.n_in, 1.0f, net->wp[l], L.n_pad,
                                                L.k_pad, nullptr);
    MST(launch_status("k_pack"));
    if (net->wtp[l]) {
      const long long nt = (long long)net->wt_rows[l] * net->wt_k[l];
      // W^T: rows = inputs, K = outputs
      k_pack<<<grid_of(nt), 256, 0, net->stream>>>(W, nullptr, 1, L.n_in, L.n_in, L.n_out, 1.0f, net->wtp[l],
                                                  net->wt_rows[l], net->wt_k[l], nullptr);
      MST(launch_status("k_pack"));
    }
    MCU(cudaMemsetAsync(net->bp[l], 0, (size_t)L.n_pad * 4, net->stream));
    MCU(cudaMemcpyAsync(net->bp[l], net->p + L.b_off, (size_t)L.n_out * 4, cudaMemcpyDeviceToDevice, net->stream));
  }
  return FLSP_OK;
}

int mlp_pack_input(flsp_mlp* net, const float* feat, const int* idx, int64_t n, const int* rows_dev) {
  const long long R = round128(n);
  k_pack<<<grid_of(R * net->k_in), 256, 0, net->stream>>>(feat, idx, net->n_in, 1, (int)n, net->n_in, 1.0f, net->x,
                                                          (int)R, net->k_in,
                                                    rows_dev);
  return launch_status("k_pack");
}

int mlp_forward_dev(flsp_mlp* net, int64_t n, bool train, const int* rows_dev) {
  const int R = (int)round128(n);
  const __nv_bfloat16* in = net->x;
  for (int l = 0; l < 4; ++l) {
    TcGemmArgs a;
    std::memset(&a, 0, sizeof(a));
    a.A = in;
    a.B = net->wp[l];
    a.M = R;
    a.N = net->L[l].n_pad;
    a.K = net->L[l].k_pad;
    a.bias = net->bp[l];
    a.out_bf16 = net->act[l];
    a.out_k = 256;
    a.gd_out = train ? net->gd[l] : nullptr;
    a.err = net->err;
    a.rows_dev = rows_dev;
    MST(gemm<kEpiHidden>(net->stream, a));
    in = net->act[l];
  }
  TcGemmArgs a;
  std::memset(&a, 0, sizeof(a));
  a.A = in;
  a.B = net->wp[4];
  a.M = R;
  a.N = net->L[4].n_pad;
  a.K = net->L[4].k_pad;
  a.bias = net->bp[4];
  a.y = net->y;
  a.ldy = net->y_ld;
  a.n_valid = net->y_ld;
  a.m_valid = R;
  a.err = net->err;
  a.rows_dev = rows_dev;
  return gemm<kEpiOutput>(net->stream, a);
}

// backward from the packed output gradient net->gout (rows R): parameter
// gradients into net->g (the output-layer bias gradient must already be there)
static int mlp_backward_dev(flsp_mlp* net, int64_t n) {
  const int R = (int)round128(n);
  cudaStream_t st = net->stream;
  const __nv_bfloat16* G = net->gout;
  int gk = 64;          // K extent of G
  int cur = 0;
  for (int l = kMlpLayers - 1; l >= 0; --l) {
    const MlpLayer& L = net->L[l];
    // dW_l = G^T A_{l-1}
    const int grows = l == kMlpLayers - 1 ? 128 : 256;   // padded output rows (M of the GEMM)
    MST(transpose(st, G, R, l == kMlpLayers - 1 ? 64 : 256, net->tG, grows));
    const __nv_bfloat16* Ain = l == 0 ? net->x : net->act[l - 1];
    const int ain_k = l == 0 ? net->k_in : 256;
    MST(transpose(st, Ain, R, ain_k, net->tA, ain_k));
    // wide inputs (the 3D patch): column blocks of at most 256 inputs, each
    // a row block of the transposed input
    for (int c0 = 0; c0 < ain_k; c0 += 256) {
      TcGemmArgs a;
      std::memset(&a, 0, sizeof(a));
      a.A = net->tG;
      a.B = net->tA;
      a.b_rows = ain_k;
      a.b_row0 = c0;
      a.M = grows;
      a.N = std::min(256, ain_k - c0);
      a.K = R;
      a.n_valid = std::min(a.N, L.n_in - c0);
      a.m_valid = L.n_out;
      a.err = net->err;
      if (a.n_valid <= 0) continue;
      // the batch is the GEMM's K: split it over up to kMlpSplits CTA rows
      // (partial products, then a fixed-order sum) so that the few output
      // tiles still fill the GPU
      const int ks = std::max(1, std::min(kMlpSplits, (R / kTcBK) / 2));
      if (ks == 1) {
        a.y = net->g + L.w_off + c0;
        a.ldy = L.n_in;
        MST(gemm<kEpiStoreF32>(st, a));
      } else {
        a.y = net->split;
        a.ldy = a.N;
        a.split_stride = (long long)a.M * a.N;
        MST(gemm<kEpiStoreF32>(st, a, ks));
        const long long nt = (long long)a.m_valid * a.n_valid;
        k_split_sum<<<(int)((nt + 255) / 256), 256, 0, st>>>(net->split, ks, a.split_stride, a.m_valid, a.n_valid,
                                                           a.N, net->g + L.w_off + c0, L.n_in);
        MST(launch_status("k_split_sum"));
      }
    }
    if (l == 0) break;
    // G_{l-1} = (G W_l) * GELU'(z_{l-1}), with its column sums -> db_{l-1}
    TcGemmArgs b;
    std::memset(&b, 0, sizeof(b));
    b.A = G;
    b.B = net->wtp[l];
    b.M = R;
    b.N = 256;
    b.K = gk;
    b.gd_in = net->gd[l - 1];
    b.out_bf16 = net->gh[cur];
    b.out_k = 256;
    b.colsum = net->colsum;
    b.err = net->err;
    MST(gemm<kEpiBackAct>(st, b));
    k_colsum<<<1, 256, 0, st>>>(net->colsum, R / 32, 256, net->L[l - 1].n_out, net->g + net->L[l - 1].b_off);
    MST(launch_status("k_colsum"));
    G = net->gh[cur];
    gk = 256;
    cur ^= 1;
  }
  return FLSP_OK;
}

// the output-layer gradient kernel for the network's width
static void out_grad_launch(flsp_mlp* net, int nblk, const float* dy, const float* targ, const int* idx, int n,
                            int R) {
  if (net->n_out == FLSP_MLP3_OUT)
    k_out_grad<FLSP_MLP3_OUT><<<nblk, 256, 0, net->stream>>>(net->y, net->y_ld, dy, targ, idx, n, R, net->gout,
                                                             net->loss_part, net->colsum);
  else
    k_out_grad<kMlpOut><<<nblk, 256, 0, net->stream>>>(net->y, net->y_ld, dy, targ, idx, n, R, net->gout,
                                                       net->loss_part, net->colsum);
}

static int output_grad(flsp_mlp* net, int64_t n, const float* dy_dev, const int* idx) {
  const int R = (int)round128(n);
  const int nblk = R / 256 + 1;
  out_grad_launch(net, nblk, dy_dev, net->targ, idx, (int)n, R);
  MST(launch_status("k_out_grad"));
  k_colsum<<<1, 32, 0, net->stream>>>(net->colsum, nblk, net->y_ld, net->n_out, net->g + net->L[4].b_off);
  MST(launch_status("k_colsum"));
  k_sum_double<<<1, 1, 0, net->stream>>>(net->loss_part, nblk, net->loss_dev);
  return launch_status("k_sum_double");
}

static int check_err(flsp_mlp* net) {
  int e = 0;
  MCU(cudaMemcpyAsync(&e, net->err, sizeof(int), cudaMemcpyDeviceToHost, net->stream));
  MCU(cudaStreamSynchronize(net->stream));
  if (e) return set_error(FLSP_ERR_TIMEOUT, "a tensor-core kernel's pipeline wait ran out");
  return FLSP_OK;
}

static int ensure_hbuf(flsp_mlp* net, size_t bytes) {
  if (net->hbuf_bytes >= bytes) return FLSP_OK;
  if (net->hbuf) cudaFreeHost(net->hbuf);
  net->hbuf = nullptr;
  MCU(cudaMallocHost(&net->hbuf, bytes));
  net->hbuf_bytes = bytes;
  return FLSP_OK;
}

}  // namespace flsp

using namespace flsp;

extern "C" {

int flsp_mlp_n_params(int64_t* n) {
  if (!n) return set_error(FLSP_ERR_BAD_ARG, "null argument");
  *n = (int64_t)kMlpHidden * kMlpIn + kMlpHidden + 3 * ((int64_t)kMlpHidden * kMlpHidden + kMlpHidden) +
       (int64_t)kMlpOut * kMlpHidden + kMlpOut;
  return FLSP_OK;
}

void flsp_mlp_destroy(flsp_mlp* net) {
  if (!net) return;
  cudaSetDevice(net->dev);
  if (net->stream) cudaStreamSynchronize(net->stream);
  if (net->split) cudaFree(net->split);
  void* ps[] = {net->p, net->m, net->v, net->g, net->x, net->y, net->gout, net->gh[0], net->gh[1], net->tA,
                net->tG, net->colsum, net->loss_part, net->loss_dev, net->err, net->feat, net->targ, net->idx};
  for (void* q : ps)
    if (q) cudaFree(q);
  for (int i = 0; i < 4; ++i) {
    if (net->act[i]) cudaFree(net->act[i]);
    if (net->gd[i]) cudaFree(net->gd[i]);
  }
  for (int l = 0; l < kMlpLayers; ++l) {
    if (net->wp[l]) cudaFree(net->wp[l]);
    if (net->wtp[l]) cudaFree(net->wtp[l]);
    if (net->bp[l]) cudaFree(net->bp[l]);
  }
  if (net->hbuf) cudaFreeHost(net->hbuf);
  if (net->stream) cudaStreamDestroy(net->stream);
  delete net;
}

int flsp_mlp_create(int device, uint64_t seed, flsp_mlp** out) {
  return flsp_mlp_create_patch(FLSP_PATCH_2D_Q2, device, seed, out);
}

int flsp_mlp_info(const flsp_mlp* net, int* n_in, int* n_out, int64_t* n_params) {
  if (!net) return set_error(FLSP_ERR_BAD_ARG, "null argument");
  if (n_in) *n_in = net->n_in;
  if (n_out) *n_out = net->n_out;
  if (n_params) *n_params = net->n_params;
  return FLSP_OK;
}

int flsp_mlp_create_patch(int patch, int device, uint64_t seed, flsp_mlp** out) {
  if (!out) return set_error(FLSP_ERR_BAD_ARG, "null argument");
  *out = nullptr;
  if (patch != FLSP_PATCH_2D_Q2 && patch != FLSP_PATCH_3D_Q2) return set_error(FLSP_ERR_BAD_ARG, "bad patch kind");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return set_error(FLSP_ERR_NO_DEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) return set_error(FLSP_ERR_BAD_ARG, "bad device ordinal");
  int major = 0;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device);
  if (major != 10) return set_error(FLSP_ERR_UNSUPPORTED, "the tensor-core MLP needs an sm_100 GPU");
  MCU(cudaSetDevice(device));
  flsp_mlp* net = new flsp_mlp();
  net->dev = device;
  static uint64_t next_uid = 1;   // graph keys of the learned periods tell networks apart by it
  net->uid = next_uid++;
  net->patch = patch;
  net->n_in = patch == FLSP_PATCH_3D_Q2 ? FLSP_MLP3_IN : kMlpIn;
  net->n_out = patch == FLSP_PATCH_3D_Q2 ? FLSP_MLP3_OUT : kMlpOut;
  net->k_in = ((net->n_in + 63) / 64) * 64;
  net->y_ld = ((net->n_out + 15) / 16) * 16;
  auto fail_destroy = [&](int code) { flsp_mlp_destroy(net); return code; };
  if (cudaStreamCreateWithFlags(&net->stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail_destroy(set_error(FLSP_ERR_CUDA, "stream creation failed"));
  const int nin[kMlpLayers] = {net->n_in, kMlpHidden, kMlpHidden, kMlpHidden, kMlpHidden};
  const int nout[kMlpLayers] = {kMlpHidden, kMlpHidden, kMlpHidden, kMlpHidden, net->n_out};
  size_t off = 0;
  for (int l = 0; l < kMlpLayers; ++l) {
    MlpLayer& L = net->L[l];
    L.n_in = nin[l];
    L.n_out = nout[l];
    L.k_pad = (int)(((nin[l] + 63) / 64) * 64);
    L.n_pad = (int)(((nout[l] + 15) / 16) * 16);
    L.w_off = off;
    off += (size_t)L.n_in * L.n_out;
    L.b_off = off;
    off += (size_t)L.n_out;
  }
  net->n_params = (int64_t)off;
  const size_t pb = off * sizeof(float);
  if (cudaMalloc(&net->p, pb) || cudaMalloc(&net->m, pb) || cudaMalloc(&net->v, pb) || cudaMalloc(&net->g, pb) ||
      cudaMalloc(&net->loss_dev, sizeof(double)) || cudaMalloc(&net->err, sizeof(int)))
    return fail_destroy(set_error(FLSP_ERR_OOM, "allocation failed"));
  for (int l = 0; l < kMlpLayers; ++l) {
    const MlpLayer& L = net->L[l];
    if (cudaMalloc(&net->wp[l], (size_t)L.n_pad * L.k_pad * 2) || cudaMalloc(&net->bp[l], (size_t)L.n_pad * 4))
      return fail_destroy(set_error(FLSP_ERR_OOM, "allocation failed"));
    if (l > 0) {   // transposes for dA_{l-1} = G_l W_l: rows = inputs (256), K = outputs padded to 64
      net->wt_rows[l] = ((L.n_in + 7) / 8) * 8;
      net->wt_k[l] = ((L.n_out + 63) / 64) * 64;
      if (cudaMalloc(&net->wtp[l], (size_t)net->wt_rows[l] * net->wt_k[l] * 2))
        return fail_destroy(set_error(FLSP_ERR_OOM, "allocation failed"));
    }
  }
  // initial weights: U(-1/sqrt(fan_in), 1/sqrt(fan_in)), output layer scaled
  // by 0.1 so that the initial correction is small; zero biases
  std::vector<float> h((size_t)off, 0.0f);
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> U(-1.0, 1.0);
  for (int l = 0; l < kMlpLayers; ++l) {
    const MlpLayer& L = net->L[l];
    const double s = (l == kMlpLayers - 1 ? 0.1 : 1.0) / std::sqrt((double)L.n_in);
    for (size_t i = 0; i < (size_t)L.n_in * L.n_out; ++i) h[L.w_off + i] = (float)(s * U(rng));
  }
  if (cudaMemcpy(net->p, h.data(), pb, cudaMemcpyHostToDevice) || cudaMemset(net->m, 0, pb) ||
      cudaMemset(net->v, 0, pb) || cudaMemset(net->err, 0, sizeof(int)))
    return fail_destroy(set_error(FLSP_ERR_CUDA, "initialisation failed"));
  int st = repack(net);
  if (st == FLSP_OK) st = mlp_ensure_cap(net, 128);
  if (st == FLSP_OK && cudaStreamSynchronize(net->stream) != cudaSuccess) st = set_error(FLSP_ERR_CUDA, "sync failed");
  if (st != FLSP_OK) return fail_destroy(st);
  *out = net;
  return FLSP_OK;
}

int flsp_mlp_get_params(flsp_mlp* net, float* params, int64_t n) {
  if (!net || !params) return set_error(FLSP_ERR_BAD_ARG, "null argument");
  if (n != net->n_params) return set_error(FLSP_ERR_BAD_ARG, "size mismatch");
  MCU(cudaSetDevice(net->dev));
  MCU(cudaMemcpyAsync(params, net->p, (size_t)n * 4, cudaMemcpyDeviceToHost, net->stream));
  MCU(cudaStreamSynchronize(net->stream));
  return FLSP_OK;
}

int flsp_mlp_set_params(flsp_mlp* net, const float* params, int64_t n) {
  if (!net || !params) return set_error(FLSP_ERR_BAD_ARG, "null argument");
  if (n != net->n_params) return set_error(FLSP_ERR_BAD_ARG, "size mismatch");
  for (int64_t i = 0; i < n; ++i)
    if (!std::isfinite(params[i])) return set_error(FLSP_ERR_NONFINITE, "non-finite parameter");
  MCU(cudaSetDevice(net->dev));
  MCU(cudaMemcpyAsync(net->p, params, (size_t)n * 4, cudaMemcpyHostToDevice, net->stream));
  MCU(cudaMemsetAsync(net->m, 0, (size_t)n * 4, net->stream));
  MCU(cudaMemsetAsync(net->v, 0, (size_t)n * 4, net->stream));
  net->adam_t = 0;
  MST(repack(net));
  MCU(cudaStreamSynchronize(net->stream));
  return FLSP_OK;
}

int flsp_mlp_forward(flsp_mlp* net, const float* x, int64_t batch, float* y) {
  if (!net || !x || !y) return set_error(FLSP_ERR_BAD_ARG, "null argument");
  if (batch <= 0 || batch > (1LL << 24)) return set_error(FLSP_ERR_BAD_ARG, "bad batch size");
  MCU(cudaSetDevice(net->dev));
  MST(mlp_ensure_cap(net, batch));
  const size_t xb = (size_t)batch * net->n_in * 4;
  MST(ensure_hbuf(net, xb));
  float* fdev = nullptr;
  MCU(cudaMallocAsync(&fdev, xb, net->stream));
  std::memcpy(net->hbuf, x, xb);
  cudaMemcpyAsync(fdev, net->hbuf, xb, cudaMemcpyHostToDevice, net->stream);
  int st = mlp_pack_input(net, fdev, nullptr, batch, nullptr);
  if (st == FLSP_OK) st = mlp_forward_dev(net, batch, false, nullptr);
  cudaFreeAsync(fdev, net->stream);
  MST(st);
  MST(check_err(net));
  MCU(cudaMemcpy2DAsync(y, net->n_out * 4, net->y, net->y_ld * 4, net->n_out * 4, (size_t)batch, cudaMemcpyDeviceToHost,
                        net->stream));
  MCU(cudaStreamSynchronize(net->stream));
  return FLSP_OK;
}

int flsp_mlp_backward(flsp_mlp* net, const float* x, const float* dy, int64_t batch, float* grad) {
  if (!net || !x || !dy || !grad) return set_error(FLSP_ERR_BAD_ARG, "null argument");
  if (batch <= 0 || batch > (1LL << 24)) return set_error(FLSP_ERR_BAD_ARG, "bad batch size");
  MCU(cudaSetDevice(net->dev));
  MST(mlp_ensure_cap(net, batch));
  float *fdev = nullptr, *dydev = nullptr;
  MCU(cudaMallocAsync(&fdev, (size_t)batch * net->n_in * 4, net->stream));
  MCU(cudaMallocAsync(&dydev, (size_t)batch * net->n_out * 4, net->stream));
  MCU(cudaMemcpyAsync(fdev, x, (size_t)batch * net->n_in * 4, cudaMemcpyHostToDevice, net->stream));
  MCU(cudaMemcpyAsync(dydev, dy, (size_t)batch * net->n_out * 4, cudaMemcpyHostToDevice, net->stream));
  int st = mlp_pack_input(net, fdev, nullptr, batch, nullptr);
  if (st == FLSP_OK) st = mlp_forward_dev(net, batch, true, nullptr);
  if (st == FLSP_OK) st = output_grad(net, batch, dydev, nullptr);
  if (st == FLSP_OK) st = mlp_backward_dev(net, batch);
  cudaFreeAsync(fdev, net->stream);
  cudaFreeAsync(dydev, net->stream);
  MST(st);
  MST(check_err(net));
  MCU(cudaMemcpyAsync(grad, net->g, (size_t)net->n_params * 4, cudaMemcpyDeviceToHost, net->stream));
  MCU(cudaStreamSynchronize(net->stream));
  return FLSP_OK;
}

int flsp_mlp_n_pairs(const flsp_mlp* net, int64_t* n) {
  if (!net || !n) return set_error(FLSP_ERR_BAD_ARG, "null argument");
  *n = net->n_pairs;
  return FLSP_OK;
}

int flsp_mlp_clear_pairs(flsp_mlp* net) {
  if (!net) return set_error(FLSP_ERR_BAD_ARG, "null argument");
  net->n_pairs = 0;
  return FLSP_OK;
}

void flsp_default_train_opts(flsp_train_opts* o) {
  if (!o) return;
  o->steps = 1000;
  o->batch = 8192;
  o->lr = 1e-3;
  o->beta1 = 0.9;
  o->beta2 = 0.999;
  o->eps = 1e-8;
  o->seed = 1;
}

int flsp_mlp_train(flsp_mlp* net, const flsp_train_opts* o, double* loss) {
  if (!net || !o) return set_error(FLSP_ERR_BAD_ARG, "null argument");
  if (net->n_pairs <= 0) return set_error(FLSP_ERR_BAD_ARG, "no training pairs collected");
  if (o->batch < 128 || o->batch > (1 << 20) || o->steps < 0) return set_error(FLSP_ERR_BAD_ARG, "bad batch/steps");
  if (!(o->lr > 0.0) || !(o->beta1 >= 0.0 && o->beta1 < 1.0) || !(o->beta2 >= 0.0 && o->beta2 < 1.0) || !(o->eps > 0.0))
    return set_error(FLSP_ERR_BAD_ARG, "bad Adam parameters");
  MCU(cudaSetDevice(net->dev));
  const int64_t B = std::min<int64_t>(o->batch, net->n_pairs);
  MST(mlp_ensure_cap(net, B));
  // one permutation of the pairs per epoch, drawn on the host
  const int64_t np = net->n_pairs;
  if (net->idx_cap < np) {
    if (net->idx) cudaFree(net->idx);
    net->idx = nullptr;
    MCU(cudaMalloc(&net->idx, (size_t)np * 4));
    net->idx_cap = np;
  }
  std::vector<int> perm((size_t)np);
  std::mt19937_64 rng(o->seed);
  int64_t pos = np;   // force a shuffle at the first step
  double last = 0.0;
  for (int64_t step = 0; step < o->steps; ++step) {
    if (pos + B > np) {
      for (int64_t i = 0; i < np; ++i) perm[(size_t)i] = (int)i;
      for (int64_t i = np - 1; i > 0; --i) {
        std::uniform_int_distribution<int64_t> d(0, i);
        std::swap(perm[(size_t)i], perm[(size_t)d(rng)]);
      }
      MCU(cudaMemcpyAsync(net->idx, perm.data(), (size_t)np * 4, cudaMemcpyHostToDevice, net->stream));
      MCU(cudaStreamSynchronize(net->stream));   // perm is reused on the host
      pos = 0;
    }
    const int* bidx = net->idx + pos;
    pos += B;
    MST(mlp_pack_input(net, net->feat, bidx, B, nullptr));
    MST(mlp_forward_dev(net, B, true, nullptr));
    MST(output_grad(net, B, nullptr, bidx));
    MST(mlp_backward_dev(net, B));
    net->adam_t += 1;
    const double bc1 = 1.0 - std::pow(o->beta1, (double)net->adam_t);
    const double bc2 = 1.0 - std::pow(o->beta2, (double)net->adam_t);
    k_adam<<<grid_of(net->n_params), 256, 0, net->stream>>>(net->p, net->m, net->v, net->g, net->n_params,
                                                           (float)o->lr, (float)o->beta1, (float)o->beta2,
                                                           (float)o->eps, (float)bc1, (float)bc2);
    MST(launch_status("k_adam"));
    MST(repack(net));
    if (step + 1 == o->steps) {
      double s = 0.0;
      MCU(cudaMemcpyAsync(&s, net->loss_dev, sizeof(double), cudaMemcpyDeviceToHost, net->stream));
      MCU(cudaStreamSynchronize(net->stream));
      last = s / ((double)B * net->n_out);
    }
  }
  MST(check_err(net));
  if (loss) *loss = last;
  return FLSP_OK;
}

int flsp_mlp_eval(flsp_mlp* net, double* loss) {
  if (!net || !loss) return set_error(FLSP_ERR_BAD_ARG, "null argument");
  if (net->n_pairs <= 0) return set_error(FLSP_ERR_BAD_ARG, "no pairs collected");
  MCU(cudaSetDevice(net->dev));
  const int64_t chunk = 65536;
  MST(mlp_ensure_cap(net, std::min<int64_t>(chunk, net->n_pairs)));
  double total = 0.0;
  for (int64_t p0 = 0; p0 < net->n_pairs; p0 += chunk) {
    const int64_t n = std::min<int64_t>(chunk, net->n_pairs - p0);
    MST(mlp_pack_input(net, net->feat + p0 * net->n_in, nullptr, n, nullptr));
    MST(mlp_forward_dev(net, n, false, nullptr));
    // loss only (the gradient buffers are scratch here)
    const int R = (int)round128(n);
    const int nblk = R / 256 + 1;
    out_grad_launch(net, nblk, nullptr, net->targ + p0 * net->n_out, nullptr, (int)n, R);
    MST(launch_status("k_out_grad"));
    k_sum_double<<<1, 1, 0, net->stream>>>(net->loss_part, nblk, net->loss_dev);
    double s = 0.0;
    MCU(cudaMemcpyAsync(&s, net->loss_dev, sizeof(double), cudaMemcpyDeviceToHost, net->stream));
    MCU(cudaStreamSynchronize(net->stream));
    total += s;
  }
  MST(check_err(net));
  *loss = total / ((double)net->n_pairs * net->n_out);
  return FLSP_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ patch launchers
namespace flsp {

#define DISPATCH_T(prec, F) ((prec) == FLSP_FP64 ? F(double) : F(float))

int launch_patch_features(cudaStream_t s, int prec, int dim, const void* state, const int* n_cells, double h,
                          const int* cells, int64_t n, const int* n_dev, float* feat) {
  if (n <= 0) return FLSP_OK;
  const long long t = n * (dim == 2 ? 9 : 27);
  const int blocks = (int)((t + 255) / 256);
  const int nx = n_cells[0], ny = n_cells[1], nz = dim > 2 ? n_cells[2] : 1;
  const float ih = (float)(1.0 / h), hf = (float)(64.0 * h);
#define L_(T)                                                                                                   \
  (dim == 2 ? (k_patch_features<2, T><<<blocks, 256, 0, s>>>((const T*)state, nx, ny, nz, ih, hf, cells, n, n_dev, \
                                                             feat), 0)                                          \
            : (k_patch_features<3, T><<<blocks, 256, 0, s>>>((const T*)state, nx, ny, nz, ih, hf, cells, n, n_dev, \
                                                             feat), 0))
  DISPATCH_T(prec, L_);
#undef L_
  return launch_status("k_patch_features");
}

int launch_patch_targets(cudaStream_t s, int prec, int nb, const void* pre, const void* post, double h,
                         const int* cells, int64_t n, float* targ) {
  if (n <= 0) return FLSP_OK;
  const int blocks = (int)((n * nb + 255) / 256);
#define L_(T) (k_patch_targets<T><<<blocks, 256, 0, s>>>((const T*)pre, (const T*)post, nb, (float)(1.0 / h), cells, n, targ), 0)
  DISPATCH_T(prec, L_);
#undef L_
  return launch_status("k_patch_targets");
}

int launch_apply_delta(cudaStream_t s, int prec, int nb, const void* pre, void* out, int64_t ndofs, double h,
                       const int* cells, int64_t n, const int* n_dev, const float* y, int ldy) {
  const size_t es = prec == FLSP_FP64 ? 8 : 4;
  if (pre != out) MCU(cudaMemcpyAsync(out, pre, (size_t)ndofs * es, cudaMemcpyDeviceToDevice, s));
  if (n <= 0) return FLSP_OK;
  const int blocks = (int)((n * nb + 255) / 256);
#define L_(T) (k_apply_delta<T><<<blocks, 256, 0, s>>>((T*)out, nb, h, cells, n, n_dev, y, ldy), 0)
  DISPATCH_T(prec, L_);
#undef L_
  return launch_status("k_apply_delta");
}

int launch_band_select(cudaStream_t s, int prec, int nb, const void* state, int64_t ncell, double thr, int* flags,
                       int* work, int* cells, int* count_dev) {
  const int nblk = (int)((ncell + 255) / 256);
  int* bcount = work;
  int* boff = work + nblk;
#define L_(T) (k_band_count<T><<<nblk, 256, 0, s>>>((const T*)state, ncell, nb, thr, flags, bcount), 0)
  DISPATCH_T(prec, L_);
#undef L_
  MST(launch_status("k_band_count"));
  k_scan_counts<<<1, 1, 0, s>>>(bcount, nblk, boff, count_dev);
  MST(launch_status("k_scan_counts"));
  k_band_compact<<<nblk, 256, 0, s>>>(flags, ncell, boff, cells);
  return launch_status("k_band_compact");
}

int launch_residual_flags(cudaStream_t s, int prec, int dim, const void* state, double h, const int* cells,
                          int64_t n, const int* n_dev, double thr, int* flags, int* count_dev) {
  MCU(cudaMemsetAsync(count_dev, 0, sizeof(int), s));
  if (n <= 0) return FLSP_OK;
  const int blocks = (int)((n + 127) / 128);
#define L_(T)                                                                                                   \
  (dim == 2 ? (k_residual<2, T><<<blocks, 128, 0, s>>>((const T*)state, 1.0 / h, cells, n, n_dev, thr, flags,     \
                                                       count_dev), 0)                                          \
            : (k_residual<3, T><<<blocks, 128, 0, s>>>((const T*)state, 1.0 / h, cells, n, n_dev, thr, flags,     \
                                                       count_dev), 0))
  DISPATCH_T(prec, L_);
#undef L_
  return launch_status("k_residual");
}

int launch_merge_cells(cudaStream_t s, int prec, int nb, const void* src, void* out, const int* cells,
                       const int* flags, int64_t n, const int* n_dev) {
  if (n <= 0) return FLSP_OK;
  const int blocks = (int)((n * nb + 255) / 256);
#define L_(T) (k_merge<T><<<blocks, 256, 0, s>>>((const T*)src, (T*)out, nb, cells, flags, n, n_dev), 0)
  DISPATCH_T(prec, L_);
#undef L_
  return launch_status("k_merge");
}

}  // namespace flsp

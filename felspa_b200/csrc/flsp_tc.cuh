// flsp_tc.cuh — BF16 tensor-core GEMM for the learned reinitialisation's
// MLP (5th-generation tensor cores: tcgen05.mma, accumulator in TMEM).
//
//   D[M x N] = A[M x K] * B[N x K]^T     (bf16 operands, fp32 accumulation)
//
// Operands live in HBM in a "packed" K-major order that is the tensor
// cores' canonical no-swizzle shared-memory layout, so that one plain bulk
// copy moves a 128 x 64 (or N x 64) chunk into shared memory unchanged:
//
//   element (r, k) of an R x K operand (R % 8 == 0, K % 64 == 0) sits at
//   (((k / 64) * (R / 8) + r / 8) * 8 + (k % 64) / 8) * 64 + (r % 8) * 8 + k % 8
//
// i.e. 8 x 8 core matrices (8 rows of 16 bytes, 128 contiguous bytes); in
// a chunk, the core matrices of one 8-row group follow each other along K
// (leading-dimension stride 128 B) and 8-row groups are 1024 B apart
// (stride-dimension stride).
//
// One CTA computes a 128 x N tile (N <= 256, N % 16 == 0): warp 0 issues
// the bulk copies of a 3-stage pipeline, one thread of warp 1 issues the
// MMAs (K = 16 per instruction) and commits each stage back to the
// producer through an mbarrier, and all four warps read the accumulator
// out of TMEM (warp w owns lanes 32w..32w+31 = tile rows) for the
// epilogue.  Every wait is bounded; a timeout sets a bit in the error word.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

#include "flsp_device.cuh"

namespace flsp {

constexpr int kTcBM = 128;      // rows per CTA tile (MMA M)
constexpr int kTcBK = 64;       // K per pipeline stage
constexpr int kTcStages = 3;
constexpr int kErrTcTimeout = 2;   // error-word bit: a tensor-core pipeline wait ran out

// offset (elements) of (r, k) in a packed R x K operand
__host__ __device__ inline long long packed_off(long long r, long long k, long long R) {
  return (((k >> 6) * (R >> 3) + (r >> 3)) * 8 + ((k & 63) >> 3)) * 64 + (r & 7) * 8 + (k & 7);
}

// ---------------- tcgen05 / TMEM primitives ----------------
__device__ __forceinline__ void tmem_alloc(uint32_t* slot_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(slot_smem)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}
// shared-memory matrix descriptor, no swizzle, K-major: LBO = 128 B
// (next core matrix along K), SBO = 1024 B (next 8-row group)
__device__ __forceinline__ uint64_t smem_desc(const void* p) {
  const uint64_t a = (uint64_t)(smem_u32(p) & 0x3FFFFu) >> 4;
  return a | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(1024 >> 4) << 32) | (1ull << 46);
}
// instruction descriptor: bf16 x bf16 -> f32, both K-major, M = 128
__host__ __device__ constexpr uint32_t tc_idesc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kTcBM >> 4) << 24);
}
__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
      : "memory");
}
// arrive on `bar` when every tcgen05 operation issued so far by this thread completes
__device__ __forceinline__ void tc_commit(unsigned long long* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                   smem_u32(bar))
               : "memory");
}
// 16 consecutive fp32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

// ---------------- the GEMM ----------------
// Epilogues (fp32 accumulator acc of row r, column n of the tile):
enum TcEpilogue : int {
  kEpiHidden = 0,   // z = acc + bias[n]; out_bf16 = GELU(z) (packed, K = N); gd = GELU'(z) if gd_out
  kEpiOutput = 1,   // y[r][n] = acc + bias[n] for n < n_valid (fp32 row-major, ld = ldy)
  kEpiBackAct = 2,  // g = acc * gd_in[r][n]; out_bf16 = g (packed, K = N); colsum partial of g
  kEpiStoreF32 = 3  // c[r][n] = acc for r < m_valid, n < n_valid (fp32 row-major, ld = ldy)
};

struct TcGemmArgs {
  const __nv_bfloat16* A;     // packed M x K
  const __nv_bfloat16* B;     // packed N x K: rows b_row0 .. b_row0 + N - 1 of a packed b_rows x K
  int b_rows, b_row0;         // matrix (b_rows = 0: B is exactly N x K); both multiples of 8
  int M, N, K;                // M % 128 == 0, N % 16 == 0 (<= 256), K % 64 == 0
  const float* bias;          // [N] (hidden / output)
  __nv_bfloat16* out_bf16;    // packed M x N_pack (hidden / back-act), N_pack = out_k
  int out_k;                  // K extent of the packed output (>= N, multiple of 64)
  float* gd_out;              // [M][N] GELU'(z) (hidden, training only; may be null)
  const float* gd_in;         // [M][N] (back-act)
  float* colsum;              // [M / 128][N] per-tile column sums (back-act; may be null)
  float* y;                   // fp32 row-major output (output / store)
  int ldy, n_valid, m_valid;
  int* err;                   // device error word
  const int* rows_dev;        // if set: only row tiles below this device-side count do work
  long long split_stride;     // store epilogue with a K split (gridDim.y > 1): CTA row y of the
                              // grid sums K chunks [y * nk / gridDim.y, (y + 1) * nk / gridDim.y)
                              // and writes its partial product to y + blockIdx.y * split_stride
};

__device__ __forceinline__ float gelu_f(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d_f(float x) {
  return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

template <int EPI>
__global__ void __launch_bounds__(128, 1) tc_gemm_kernel(const TcGemmArgs a) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // layout: [stages][A chunk 16 KB][B chunk N*128 B] | barriers | TMEM slot
  const int N = a.N;
  const uint32_t a_bytes = kTcBM * kTcBK * 2, b_bytes = (uint32_t)N * kTcBK * 2;
  const uint32_t stage_bytes = a_bytes + b_bytes;
  unsigned char* stages = smem_raw;
  unsigned long long* full = reinterpret_cast<unsigned long long*>(smem_raw + kTcStages * stage_bytes);
  unsigned long long* empty = full + kTcStages;
  unsigned long long* done = empty + kTcStages;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * kTcBM;
  if (a.rows_dev && m0 >= *a.rows_dev) return;   // uniform per CTA, before any barrier or TMEM
  // this CTA's K chunks (all of them without a K split)
  const int nk_all = a.K / kTcBK;
  const int kb = (int)(((long long)blockIdx.y * nk_all) / gridDim.y);
  const int nk = (int)(((long long)(blockIdx.y + 1) * nk_all) / gridDim.y) - kb;
  uint32_t ncols = 32;
  while ((int)ncols < N) ncols <<= 1;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kTcStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
  }
  if (warp == 0) tmem_alloc(tslot, ncols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  bool ok = true;

  if (warp == 0 && lane == 0) {
    // producer: bulk copies of the A and B chunks of every K stage
    const char* ga = reinterpret_cast<const char*>(a.A);
    const char* gb = reinterpret_cast<const char*>(a.B);
    const int rb = a.b_rows > 0 ? a.b_rows : N;
    for (int kc = 0; kc < nk && ok; ++kc) {
      const int s = kc % kTcStages;
      if (kc >= kTcStages) ok = mbar_wait(&empty[s], ((kc / kTcStages) - 1) & 1, 1 << 22);
      if (!ok) break;
      unsigned char* sa = stages + (size_t)s * stage_bytes;
      mbar_arrive_expect_tx(&full[s], stage_bytes);
      // A rows m0.. m0+127 of chunk kc, B rows 0..N-1 of chunk kc: contiguous
      const long long kg = kb + kc;   // global K chunk
      bulk_g2s(sa, ga + (kg * (a.M / 8) + m0 / 8) * 1024, a_bytes, &full[s]);
      bulk_g2s(sa + a_bytes, gb + (kg * (rb / 8) + a.b_row0 / 8) * 1024, b_bytes, &full[s]);
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    const uint32_t idesc = tc_idesc(N);
    for (int kc = 0; kc < nk && ok; ++kc) {
      const int s = kc % kTcStages;
      ok = mbar_wait(&full[s], (kc / kTcStages) & 1, 1 << 22);
      if (!ok) break;
      tc_fence_after();
      unsigned char* sa = stages + (size_t)s * stage_bytes;
      const uint64_t da = smem_desc(sa), db = smem_desc(sa + a_bytes);
#pragma unroll
      for (int j = 0; j < kTcBK / 16; ++j)   // K = 16 per MMA: 2 core matrices = 256 B = 16 descriptor units
        tc_mma(tmem, da + 16ull * j, db + 16ull * j, idesc, (kc > 0 || j > 0) ? 1u : 0u);
      tc_commit(&empty[s]);
    }
    tc_commit(done);
  }
  __syncwarp();
  // epilogue: every warp waits for the accumulator
  if (!mbar_wait(done, 0, 1 << 22)) ok = false;
  if (!ok && a.err && lane == 0) atomicOr(a.err, kErrTcTimeout);
  tc_fence_after();

  const int r = m0 + warp * 32 + lane;   // tile row owned by this thread
  const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
  float csum[16];
  for (int c0 = 0; c0 < N; c0 += 16) {
    float v[16];
    tmem_ld16(trow + (uint32_t)c0, v);
    if (!ok) continue;
    if constexpr (EPI == kEpiHidden) {
      __align__(16) __nv_bfloat16 o[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const float z = v[i] + a.bias[c0 + i];
        o[i] = __float2bfloat16_rn(gelu_f(z));
        if (a.gd_out) a.gd_out[(long long)r * N + c0 + i] = gelu_d_f(z);
      }
      uint4* dst0 = reinterpret_cast<uint4*>(a.out_bf16 + packed_off(r, c0, a.M));
      uint4* dst1 = reinterpret_cast<uint4*>(a.out_bf16 + packed_off(r, c0 + 8, a.M));
      *dst0 = *reinterpret_cast<const uint4*>(&o[0]);
      *dst1 = *reinterpret_cast<const uint4*>(&o[8]);
    } else if constexpr (EPI == kEpiOutput) {
#pragma unroll
      for (int i = 0; i < 16; ++i)
        if (c0 + i < a.n_valid && r < a.m_valid) a.y[(long long)r * a.ldy + c0 + i] = v[i] + a.bias[c0 + i];
    } else if constexpr (EPI == kEpiBackAct) {
      __align__(16) __nv_bfloat16 o[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const float g = v[i] * a.gd_in[(long long)r * N + c0 + i];
        o[i] = __float2bfloat16_rn(g);
        csum[i] = g;
      }
      uint4* dst0 = reinterpret_cast<uint4*>(a.out_bf16 + packed_off(r, c0, a.M));
      uint4* dst1 = reinterpret_cast<uint4*>(a.out_bf16 + packed_off(r, c0 + 8, a.M));
      *dst0 = *reinterpret_cast<const uint4*>(&o[0]);
      *dst1 = *reinterpret_cast<const uint4*>(&o[8]);
      if (a.colsum) {
        // column sums over the tile's 128 rows: warp reduction, then one
        // atomic-free add per warp into shared scratch is avoided by a
        // fixed-order pass: lane 0 of each warp writes its partial
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          float s = csum[i];
#pragma unroll
          for (int o2 = 16; o2 > 0; o2 >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o2);
          csum[i] = s;
        }
        if (lane == 0) {
#pragma unroll
          for (int i = 0; i < 16; ++i)
            a.colsum[((long long)blockIdx.x * 4 + warp) * N + c0 + i] = csum[i];
        }
      }
    } else {
      float* y = a.y + (long long)blockIdx.y * a.split_stride;
#pragma unroll
      for (int i = 0; i < 16; ++i)
        if (c0 + i < a.n_valid && r < a.m_valid) y[(long long)r * a.ldy + c0 + i] = v[i];
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, ncols);
}

// shared memory of one CTA for an N-wide tile
__host__ __device__ inline size_t tc_gemm_smem(int N) {
  return (size_t)kTcStages * (kTcBM * kTcBK * 2 + (size_t)N * kTcBK * 2) + 8 * (2 * kTcStages + 1) + 16;
}

}  // namespace flsp

// flsp_mlp.h — the learned reinitialisation's network (internal).
//
// A 2D degree-2 (Q basis) cell patch of 3 x 3 cells x 9 Legendre
// coefficients, divided by the cell size h, plus 64 h, maps to the change
// of the centre cell's 9 coefficients under the HJ reinitialisation,
// divided by h:
//   82 -> 256 -> 256 -> 256 -> 256 -> 9, GELU after every hidden layer,
// BF16 weights and activations on the tensor cores, FP32 accumulation,
// FP32 master weights and Adam moments.  Parameters are laid out
// W1 [256 x 82], b1 [256], W2 [256 x 256], b2, W3, b3, W4, b4,
// W5 [9 x 256], b5 [9] (row-major W[out][in]).  The 3D variant maps the
// 3 x 3 x 3 patch of a 3D degree-2 cell (27 coefficients each) plus 64 h:
//   730 -> 256 -> 256 -> 256 -> 256 -> 27.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "flsp_dg.h"

namespace flsp {

constexpr int kMlpLayers = 5;
constexpr int kMlpSplits = 32;   // most K splits of a weight-gradient GEMM
constexpr int kMlpIn = FLSP_MLP_IN, kMlpHidden = FLSP_MLP_HIDDEN, kMlpOut = FLSP_MLP_OUT;

struct MlpLayer {
  int n_in, n_out;       // real sizes
  int k_pad, n_pad;      // GEMM K (multiple of 64) and N (multiple of 16)
  size_t w_off, b_off;   // offsets in the parameter vector
};

}  // namespace flsp

struct flsp_mlp {
  int dev = 0;
  uint64_t uid = 0;                    // distinct per network created in this process
  int patch = FLSP_PATCH_2D_Q2;
  int n_in = flsp::kMlpIn, n_out = flsp::kMlpOut;   // network widths
  int k_in = 128;                      // GEMM K of the input (n_in rounded up to 64)
  int y_ld = 16;                       // row stride of y (n_out rounded up to 16)
  cudaStream_t stream = nullptr;
  flsp::MlpLayer L[flsp::kMlpLayers];
  int64_t n_params = 0;
  // parameters (FP32 master), Adam moments, gradients
  float* p = nullptr;
  float* m = nullptr;
  float* v = nullptr;
  float* g = nullptr;
  int64_t adam_t = 0;
  // packed BF16 weights (W: n_pad x k_pad) and transposes for dA (k rows x
  // out-K, layers 2..5), padded biases
  __nv_bfloat16* wp[flsp::kMlpLayers] = {};
  __nv_bfloat16* wtp[flsp::kMlpLayers] = {};
  float* bp[flsp::kMlpLayers] = {};
  int wt_rows[flsp::kMlpLayers] = {}, wt_k[flsp::kMlpLayers] = {};
  // batch work buffers (capacity cap rows, multiple of 128)
  int64_t cap = 0;
  __nv_bfloat16* x = nullptr;          // packed cap x k_in
  __nv_bfloat16* act[4] = {};          // packed cap x 256 (layer outputs 1..4)
  float* gd[4] = {};                   // cap x 256 GELU'(z)
  float* y = nullptr;                  // cap x y_ld
  __nv_bfloat16* gout = nullptr;       // packed cap x 64 (output-layer gradient)
  __nv_bfloat16* gh[2] = {};           // packed cap x 256 (hidden gradients, ping-pong)
  __nv_bfloat16* tA = nullptr;         // packed max(256, k_in) x cap (transposed activation / input)
  __nv_bfloat16* tG = nullptr;         // packed 256 x cap (transposed gradient; 128 rows for the output layer)
  float* colsum = nullptr;             // cap / 32 x 256 per-warp column sums
  float* split = nullptr;              // kMlpSplits x 256 x 256 partial weight gradients
  double* loss_part = nullptr;         // per-block loss partials
  double* loss_dev = nullptr;
  int* err = nullptr;                  // device error word
  float* hbuf = nullptr;               // host staging (pinned)
  size_t hbuf_bytes = 0;
  // training pairs (device): features n x n_in, targets n x n_out
  int64_t n_pairs = 0, pair_cap = 0;
  float* feat = nullptr;
  float* targ = nullptr;
  int* idx = nullptr;                  // batch indices (device)
  int64_t idx_cap = 0;
};

namespace flsp {

int mlp_ensure_cap(flsp_mlp* net, int64_t rows);
int mlp_ensure_pairs(flsp_mlp* net, int64_t n);
// forward of rows [0, n) of net->x (packed); train = keep GELU' for backward.
// rows_dev (optional): a device-side row count <= n; the operand geometry
// stays that of n rows, work past the count is skipped on the device.
int mlp_forward_dev(flsp_mlp* net, int64_t n, bool train, const int* rows_dev);
// pack n feature rows (fp32 n x n_in, row stride n_in; gathered through idx
// if non-null) into net->x (rows_dev as above)
int mlp_pack_input(flsp_mlp* net, const float* feat, const int* idx, int64_t n, const int* rows_dev);

// The list launchers below take an upper bound n for their grids and an
// optional device-side count n_dev <= n of the cells actually listed.
//
// patch features of the listed cells of a degree-2 Q-basis state
// (lexicographic cells n[0] x n[1] (x n[2]), nb = 3^dim coefficients each):
// fp32 rows of 3^dim * nb + 1 values (the patch over h, then 64 h)
int launch_patch_features(cudaStream_t s, int prec, int dim, const void* state, const int* n_cells, double h,
                          const int* cells, int64_t n, const int* n_dev, float* feat);
// targets (post - pre) / h of the listed cells' nb coefficients, fp32 n x nb
int launch_patch_targets(cudaStream_t s, int prec, int nb, const void* pre, const void* post, double h,
                         const int* cells, int64_t n, float* targ);
// out = pre; out[cells] += h * y[:, 0:nb] (y row stride ldy)
int launch_apply_delta(cudaStream_t s, int prec, int nb, const void* pre, void* out, int64_t ndofs, double h,
                       const int* cells, int64_t n, const int* n_dev, const float* y, int ldy);
// band cells |c0| <= band * h (c0 = first of nb coefficients), compacted in
// increasing cell order; count to *count_dev; work holds 2 * ceil(ncell /
// 256) + 1 ints
int launch_band_select(cudaStream_t s, int prec, int nb, const void* state, int64_t ncell, double thr, int* flags,
                       int* work, int* cells, int* count_dev);
// cells of the list whose mean of ||grad phi| - 1| over the 3^dim Gauss
// points exceeds thr: flags[i] = 1 and a count (in *count_dev)
int launch_residual_flags(cudaStream_t s, int prec, int dim, const void* state, double h, const int* cells,
                          int64_t n, const int* n_dev, double thr, int* flags, int* count_dev);
// out[cells[i]] = src[cells[i]] (nb coefficients) where flags[i]
int launch_merge_cells(cudaStream_t s, int prec, int nb, const void* src, void* out, const int* cells,
                       const int* flags, int64_t n, const int* n_dev);

}  // namespace flsp

// flsp_k_hj.cu — reinitialisation pseudo-step kernels (instantiations + launchers).
#include <algorithm>
#include <cstring>

#include "flsp_hj.cuh"
#include "flsp_hjs.cuh"
#include "flsp_ldg.cuh"
#include "flsp_launch.h"
#include "flsp_tables.h"

namespace flsp {

int upload_tables_hj() {
  cudaError_t e = upload_tables_here();
  if (e != cudaSuccess) return set_error(FLSP_ERR_CUDA, std::string("tables: ") + cudaGetErrorString(e));
  return FLSP_OK;
}

int hj_default_tile(const Ctx& c, int* tile) {
  return dispatch(c, [&](auto D, auto PP, auto tz) -> int {
    constexpr int DIM = decltype(D)::value, P = decltype(PP)::value;
    using T = decltype(tz);
    static const int c2[][3] = {{16, 16, 1}, {16, 8, 1}, {8, 8, 1}, {8, 4, 1}};
    static const int c3[][3] = {{8, 8, 4}, {8, 4, 4}, {4, 4, 4}, {4, 4, 2}};
    if (c.basis == FLSP_BASIS_Q) {   // the tensor-product kernel's fixed tile
      tile[0] = HjsTile<DIM>::X;
      tile[1] = HjsTile<DIM>::Y;
      tile[2] = HjsTile<DIM>::Z;
      return FLSP_OK;
    }
    const int(*cand)[3] = DIM == 2 ? c2 : c3;
    int i = 0;
    for (; i < 3; ++i)
      if (hj_smem_bytes<DIM, P, T>(cand[i]) <= 200 * 1024) break;
    tile[0] = cand[i][0];
    tile[1] = cand[i][1];
    tile[2] = cand[i][2];
    return FLSP_OK;
  });
}

int hj_prepare(const Ctx& c, const int* tile) {
  return dispatch(c, [&](auto D, auto PP, auto tz) -> int {
    constexpr int DIM = decltype(D)::value, P = decltype(PP)::value;
    using T = decltype(tz);
    const bool tq = c.basis == FLSP_BASIS_Q;
    const size_t smem = tq ? hjs_smem_bytes<DIM, P, T>(tile) : hj_smem_bytes<DIM, P, T>(tile);
    if (smem > 227 * 1024) return set_error(FLSP_ERR_BAD_ARG, "reinit tile too large for shared memory");
    if (tq && (tile[0] != HjsTile<DIM>::X || tile[1] != HjsTile<DIM>::Y || (DIM > 2 && tile[2] != HjsTile<DIM>::Z)))
      return set_error(FLSP_ERR_BAD_ARG, "the tensor-product reinit kernel has a fixed tile");
    cudaError_t e = cudaFuncSetAttribute(tq ? hjs_kernel<DIM, P, T> : hj_kernel<DIM, P, T>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(tq ? hjs_kernel<DIM, P, T> : hj_kernel<DIM, P, T>,
                               cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e != cudaSuccess) return set_error(FLSP_ERR_CUDA, std::string("hj attr: ") + cudaGetErrorString(e));
    return FLSP_OK;
  });
}

int hj_table_bytes(const Ctx& c, const int* tile, size_t* bytes) {
  return dispatch(c, [&](auto D, auto PP, auto tz) -> int {
    constexpr int DIM = decltype(D)::value, P = decltype(PP)::value;
    using T = decltype(tz);
    MeshArgs m = c.m;
    set_tile(m, DIM, tile);
    const long long nt = (long long)m.tile[0] * m.tile[1] * m.tile[2];
    *bytes = (size_t)nblocks(m) * hjs_ns<DIM, P>() * nt * sizeof(T);
    return FLSP_OK;
  });
}

int ldg_prepare(const Ctx& c) {
  return dispatch(c, [&](auto D, auto PP, auto tz) -> int {
    constexpr int DIM = decltype(D)::value, P = decltype(PP)::value;
    using T = decltype(tz);
    const size_t smem = ldg_smem_bytes<DIM, P, T>(DIM == 2 ? kLdgTile2 : kLdgTile3);
    cudaError_t e = cudaFuncSetAttribute(ldg_kernel<DIM, P, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return set_error(FLSP_ERR_CUDA, std::string("ldg attr: ") + cudaGetErrorString(e));
    return FLSP_OK;
  });
}

int launch_ldg(const Ctx& c, const void* in, void* out, long long block, double nu, int mode) {
  return dispatch(c, [&](auto D, auto PP, auto tz) -> int {
    constexpr int DIM = decltype(D)::value, P = decltype(PP)::value;
    using T = decltype(tz);
    LdgArgs<T> a;
    std::memset(&a, 0, sizeof(a));
    a.m = c.m;
    const int* t = DIM == 2 ? kLdgTile2 : kLdgTile3;
    set_tile(a.m, DIM, t);
    apply_band(c, kNbLdg, a.m);
    a.in = reinterpret_cast<const T*>(in);
    a.out = reinterpret_cast<T*>(out);
    a.block = block;
    a.nu = nu;
    const size_t smem = ldg_smem_bytes<DIM, P, T>(a.m.tile);
    ldg_kernel<DIM, P, T><<<(unsigned)nblocks(a.m), t[0] * t[1] * t[2], smem, c.stream>>>(a, mode);
    return launch_status("ldg_kernel");
  });
}

int launch_hj(const Ctx& c, const void* phi, const void* phi0, void* out, DevClock* clk, int mode,
              int rk, double dt_explicit, long long block, const int* tile, const void* rdiff) {
  return dispatch(c, [&](auto D, auto PP, auto tz) -> int {
    constexpr int DIM = decltype(D)::value, P = decltype(PP)::value;
    using T = decltype(tz);
    HJArgs<T> a;
    std::memset(&a, 0, sizeof(a));
    a.m = c.m;
    int t[3];
    if (tile) { t[0] = tile[0]; t[1] = tile[1]; t[2] = tile[2]; }
    else hj_default_tile(c, t);
    set_tile(a.m, DIM, t);
    a.phi = reinterpret_cast<const T*>(phi);
    a.phi0 = reinterpret_cast<const T*>(phi0);
    a.out = reinterpret_cast<T*>(out);
    a.clk = clk;
    a.mode = mode;
    a.rk = rk;
    a.dt_explicit = dt_explicit;
    a.block = block;
    a.rdiff = reinterpret_cast<const T*>(rdiff);
    // the gradient export mode uses the modal kernel for both bases
    if (mode != kHJGradients) apply_band(c, kNbHJ, a.m);   // the gradient export uses no band
    if (c.basis == FLSP_BASIS_Q && mode != kHJGradients) {
      // the smooth-sign table is filled by the sweep's kHJCflOnly launch,
      // which evaluates phi0 as phi
      if (!c.hj_stab) return set_error(FLSP_ERR_BAD_ARG, "reinit sign table not allocated");
      if (mode == kHJCflOnly && phi != phi0)
        return set_error(FLSP_ERR_BAD_ARG, "the sign-table launch needs phi == phi0");
      if (a.m.tile[0] != HjsTile<DIM>::X || a.m.tile[1] != HjsTile<DIM>::Y || a.m.tile[2] != HjsTile<DIM>::Z)
        return set_error(FLSP_ERR_BAD_ARG, "the tensor-product reinit kernel has a fixed tile");
      a.stab = reinterpret_cast<T*>(c.hj_stab);
      a.err = clk ? &clk->err : nullptr;
      const size_t smem = hjs_smem_bytes<DIM, P, T>(a.m.tile);
      const int threads = HjsTile<DIM>::N * (P + 2);
      hjs_kernel<DIM, P, T><<<(unsigned)nblocks(a.m), threads, smem, c.stream>>>(a);
      return launch_status("hjs_kernel");
    }
    int tm[3];
    if (c.basis == FLSP_BASIS_Q) {  // modal kernel with its own tile
      a.m.tiles = nullptr;
      a.m.n_tiles = nullptr;
      Ctx cp = c;
      cp.basis = FLSP_BASIS_P;
      hj_default_tile(cp, tm);
      set_tile(a.m, DIM, tm);
      const size_t sm2 = hj_smem_bytes<DIM, P, T>(a.m.tile);
      static bool attr_done[2][4][4] = {};
      bool& done = attr_done[sizeof(T) == 8][DIM][P];
      if (!done) {
        cudaFuncSetAttribute(hj_kernel<DIM, P, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2);
        done = true;
      }
      hj_kernel<DIM, P, T><<<(unsigned)nblocks(a.m), tm[0] * tm[1] * tm[2], sm2, c.stream>>>(a);
      return launch_status("hj_kernel");
    }
    const size_t smem = hj_smem_bytes<DIM, P, T>(a.m.tile);
    hj_kernel<DIM, P, T><<<(unsigned)nblocks(a.m), t[0] * t[1] * t[2], smem, c.stream>>>(a);
    return launch_status("hj_kernel");
  });
}

}  // namespace flsp

// flsp_k_hj.cu — reinitialisation pseudo-step kernels (instantiations + launchers).
#include <algorithm>
#include <cstring>

#include "flsp_hj.cuh"
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
    const size_t smem = hj_smem_bytes<DIM, P, T>(tile);
    if (smem > 227 * 1024) return set_error(FLSP_ERR_BAD_ARG, "reinit tile too large for shared memory");
    cudaError_t e = cudaFuncSetAttribute(hj_kernel<DIM, P, T>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return set_error(FLSP_ERR_CUDA, std::string("hj attr: ") + cudaGetErrorString(e));
    return FLSP_OK;
  });
}

int launch_hj(const Ctx& c, const void* phi, const void* phi0, void* out, DevClock* clk, int mode,
              int rk, double dt_explicit, long long block, const int* tile) {
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
    const size_t smem = hj_smem_bytes<DIM, P, T>(a.m.tile);
    hj_kernel<DIM, P, T><<<(unsigned)nblocks(a.m), t[0] * t[1] * t[2], smem, c.stream>>>(a);
    return launch_status("hj_kernel");
  });
}

}  // namespace flsp

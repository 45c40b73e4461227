// flsp_k_adv.cu — advection stage kernels (instantiations + launchers).
#include <algorithm>
#include <cstring>

#include "flsp_advect.cuh"
#include "flsp_advsep.cuh"
#include "flsp_launch.h"
#include "flsp_tables.h"

namespace flsp {

int upload_tables_adv() {
  cudaError_t e = upload_tables_here();
  if (e != cudaSuccess) return set_error(FLSP_ERR_CUDA, std::string("tables: ") + cudaGetErrorString(e));
  return FLSP_OK;
}

// shared memory of the stage kernel that serves velocity v
template <int DIM, int P, typename T>
static size_t stage_smem(const VelDev& v, const int* tile) {
  return use_sep_kernel(v) ? sep_smem_bytes<DIM, P, T>(tile)
                           : adv_smem_bytes<DIM, P, T>(tile, std::max(v.n_terms, 1));
}

int adv_default_tile(const Ctx& c, const VelDev& v, int* tile) {
  return dispatch(c, [&](auto D, auto PP, auto tz) -> int {
    constexpr int DIM = decltype(D)::value, P = decltype(PP)::value;
    using T = decltype(tz);
    static const int c2[][3] = {{32, 8, 1}, {16, 16, 1}, {16, 8, 1}, {8, 8, 1}};
    static const int c3[][3] = {{8, 8, 4}, {8, 4, 4}, {4, 4, 4}, {4, 4, 2}};
    const int(*cand)[3] = DIM == 2 ? c2 : c3;
    int i = 0;
    for (; i < 3; ++i)
      if (stage_smem<DIM, P, T>(v, cand[i]) <= 200 * 1024) break;
    tile[0] = cand[i][0];
    tile[1] = cand[i][1];
    tile[2] = cand[i][2];
    return FLSP_OK;
  });
}

int adv_prepare(const Ctx& c, const VelDev& v, const int* tile) {
  return dispatch(c, [&](auto D, auto PP, auto tz) -> int {
    constexpr int DIM = decltype(D)::value, P = decltype(PP)::value;
    using T = decltype(tz);
    const size_t smem = std::max(adv_smem_bytes<DIM, P, T>(tile, std::max(v.n_terms, 1)),
                                 sep_smem_bytes<DIM, P, T>(tile));
    if (smem > 227 * 1024) return set_error(FLSP_ERR_BAD_ARG, "advection tile too large for shared memory");
    auto attr = [&](auto kern) -> int {
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
      if (e != cudaSuccess) return set_error(FLSP_ERR_CUDA, std::string("adv attr: ") + cudaGetErrorString(e));
      return FLSP_OK;
    };
    int st = attr(adv_stage_kernel<DIM, P, T>);
    if (st == FLSP_OK) st = attr(adv_sep_kernel<DIM, P, T>);
    return st;
  });
}

int launch_adv_stage(const Ctx& c, const VelDev& v, const void* in, const void* phin, void* out,
                     const DevClock* clk, int stage, int combine, double ct_explicit,
                     const int* tile) {
  return dispatch(c, [&](auto D, auto PP, auto tz) -> int {
    constexpr int DIM = decltype(D)::value, P = decltype(PP)::value;
    using T = decltype(tz);
    AdvArgs<T> a;
    std::memset(&a, 0, sizeof(a));
    a.m = c.m;
    int t[3];
    if (tile) { t[0] = tile[0]; t[1] = tile[1]; t[2] = tile[2]; }
    else adv_default_tile(c, v, t);
    set_tile(a.m, DIM, t);
    if (use_sep_kernel(v)) {
      AdvSepArgs<T> b;
      std::memset(&b, 0, sizeof(b));
      b.m = a.m;
      b.optab = reinterpret_cast<const T*>(v.optab);
      b.nmax = v.nmax;
      b.phi_s = reinterpret_cast<const T*>(in);
      b.phi_n = reinterpret_cast<const T*>(phin);
      b.out = reinterpret_cast<T*>(out);
      b.clk = clk;
      b.stage = stage;
      b.combine = combine;
      b.ct_explicit = ct_explicit;
      const size_t smem = sep_smem_bytes<DIM, P, T>(a.m.tile);
      adv_sep_kernel<DIM, P, T><<<(unsigned)nblocks(a.m), t[0] * t[1] * t[2], smem, c.stream>>>(b);
      return launch_status("adv_sep_kernel");
    }
    a.v.vtab = reinterpret_cast<const T*>(v.vtab);
    a.v.n_terms = v.n_terms;
    a.v.nmax = v.nmax;
    a.v.npt = v.npt;
    for (int k = 0; k < v.n_terms; ++k) a.v.comp[k] = v.comp[k];
    a.phi_s = reinterpret_cast<const T*>(in);
    a.phi_n = reinterpret_cast<const T*>(phin);
    a.out = reinterpret_cast<T*>(out);
    a.clk = clk;
    a.stage = stage;
    a.combine = combine;
    a.ct_explicit = ct_explicit;
    const size_t smem = adv_smem_bytes<DIM, P, T>(a.m.tile, std::max(v.n_terms, 1));
    adv_stage_kernel<DIM, P, T><<<(unsigned)nblocks(a.m), t[0] * t[1] * t[2], smem, c.stream>>>(a);
    return launch_status("adv_stage_kernel");
  });
}

}  // namespace flsp

// flsp_k_adv.cu — advection stage kernels (instantiations + launchers).
#include <algorithm>
#include <cstring>

#include "flsp_advect.cuh"
#include "flsp_launch.h"
#include "flsp_tables.h"

namespace flsp {

int upload_tables_adv() {
  cudaError_t e = upload_tables_here();
  if (e != cudaSuccess) return set_error(FLSP_ERR_CUDA, std::string("tables: ") + cudaGetErrorString(e));
  return FLSP_OK;
}

int adv_default_tile(const Ctx& c, int n_terms, int* tile) {
  return dispatch(c, [&](auto D, auto PP, auto tz) -> int {
    constexpr int DIM = decltype(D)::value, P = decltype(PP)::value;
    using T = decltype(tz);
    static const int c2[][3] = {{32, 8, 1}, {16, 16, 1}, {16, 8, 1}, {8, 8, 1}};
    static const int c3[][3] = {{8, 8, 4}, {8, 4, 4}, {4, 4, 4}, {4, 4, 2}};
    const int(*cand)[3] = DIM == 2 ? c2 : c3;
    int i = 0;
    for (; i < 3; ++i)
      if (adv_smem_bytes<DIM, P, T>(cand[i], std::max(n_terms, 1)) <= 200 * 1024) break;
    tile[0] = cand[i][0];
    tile[1] = cand[i][1];
    tile[2] = cand[i][2];
    return FLSP_OK;
  });
}

int adv_prepare(const Ctx& c, int n_terms, const int* tile) {
  return dispatch(c, [&](auto D, auto PP, auto tz) -> int {
    constexpr int DIM = decltype(D)::value, P = decltype(PP)::value;
    using T = decltype(tz);
    const size_t smem = adv_smem_bytes<DIM, P, T>(tile, std::max(n_terms, 1));
    if (smem > 227 * 1024) return set_error(FLSP_ERR_BAD_ARG, "advection tile too large for shared memory");
    for (auto kern : {adv_stage_kernel<DIM, P, true, T>, adv_stage_kernel<DIM, P, false, T>}) {
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
      if (e != cudaSuccess) return set_error(FLSP_ERR_CUDA, std::string("adv attr: ") + cudaGetErrorString(e));
    }
    return FLSP_OK;
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
    else adv_default_tile(c, v.n_terms, t);
    set_tile(a.m, DIM, t);
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
    if (v.sep1)
      adv_stage_kernel<DIM, P, true, T><<<(unsigned)nblocks(a.m), t[0] * t[1] * t[2], smem, c.stream>>>(a);
    else
      adv_stage_kernel<DIM, P, false, T><<<(unsigned)nblocks(a.m), t[0] * t[1] * t[2], smem, c.stream>>>(a);
    return launch_status("adv_stage_kernel");
  });
}

}  // namespace flsp

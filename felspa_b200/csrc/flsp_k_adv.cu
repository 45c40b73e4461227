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

static int sep_unit(int what, const Ctx& c, const VelDev* v, const int* tile, size_t* bytes,
                    const void* in = nullptr, const void* phin = nullptr, void* out = nullptr,
                    const DevClock* clk = nullptr, int stage = 0, int combine = 0, double ct = 0.0) {
  if (c.dim == 2) return sep2_call(what, c, v, tile, bytes, in, phin, out, clk, stage, combine, ct);
  return sep3_call(what, c, v, tile, bytes, in, phin, out, clk, stage, combine, ct);
}

int adv_default_tile(const Ctx& c, const VelDev& v, int* tile) {
  static const int c2[][3] = {{32, 8, 1}, {16, 16, 1}, {16, 8, 1}, {8, 8, 1}};
  static const int c3[][3] = {{8, 8, 4}, {8, 4, 4}, {4, 4, 4}, {4, 4, 2}};
  const int(*cand)[3] = c.dim == 2 ? c2 : c3;
  const int ncand = c.dim == 2 ? 4 : 3;   // 4x4x2 only for the quadrature kernel
  if (use_sep_kernel(v)) {
    // separable kernel: the first shape with two CTAs per SM, else the
    // first that fits
    int pick = -1;
    for (int pass = 0; pass < 2 && pick < 0; ++pass)
      for (int i = 0; i < ncand && pick < 0; ++i) {
        size_t b = 0;
        const int st = sep_unit(0, c, &v, cand[i], &b);
        if (st) return st;
        if (b <= (pass == 0 ? 113u * 1024u : 227u * 1024u)) pick = i;
      }
    if (pick < 0) return set_error(FLSP_ERR_UNSUPPORTED, "no separable tile fits in shared memory");
    for (int d = 0; d < 3; ++d) tile[d] = cand[pick][d];
    return FLSP_OK;
  }
  return dispatch(c, [&](auto D, auto PP, auto tz) -> int {
    constexpr int DIM = decltype(D)::value, P = decltype(PP)::value;
    using T = decltype(tz);
    const int(*cq)[3] = DIM == 2 ? c2 : c3;
    int i = 0;
    for (; i < 3; ++i)
      if (adv_smem_bytes<DIM, P, T>(cq[i], std::max(v.n_terms, 1), v.tab) <= 200 * 1024) break;
    tile[0] = cq[i][0];
    tile[1] = cq[i][1];
    tile[2] = cq[i][2];
    return FLSP_OK;
  });
}

int adv_tile_candidates(const Ctx& c, const VelDev& v, int (*out)[3], int* n) {
  static const int c2[][3] = {{32, 8, 1}, {16, 16, 1}, {16, 8, 1}, {8, 8, 1}};
  static const int c3s[][3] = {{8, 8, 4}, {8, 4, 4}, {4, 4, 4}};
  static const int c3q[][3] = {{8, 8, 4}, {8, 4, 4}, {4, 4, 4}, {4, 4, 2}};
  const int(*cand)[3] = c.dim == 2 ? c2 : (use_sep_kernel(v) ? c3s : c3q);
  *n = c.dim == 2 ? 4 : (use_sep_kernel(v) ? 3 : 4);
  for (int i = 0; i < *n; ++i)
    for (int d = 0; d < 3; ++d) out[i][d] = cand[i][d];
  return FLSP_OK;
}

int adv_prepare(const Ctx& c, const VelDev& v, const int* tile) {
  if (use_sep_kernel(v)) return sep_unit(1, c, &v, tile, nullptr);
  return dispatch(c, [&](auto D, auto PP, auto tz) -> int {
    constexpr int DIM = decltype(D)::value, P = decltype(PP)::value;
    using T = decltype(tz);
    const size_t smem = adv_smem_bytes<DIM, P, T>(tile, std::max(v.n_terms, 1), v.tab);
    if (smem > 227 * 1024) return set_error(FLSP_ERR_BAD_ARG, "advection tile too large for shared memory");
    auto kern = v.tab ? adv_stage_kernel<DIM, P, T, true> : adv_stage_kernel<DIM, P, T, false>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e != cudaSuccess) return set_error(FLSP_ERR_CUDA, std::string("adv attr: ") + cudaGetErrorString(e));
    return FLSP_OK;
  });
}

int launch_adv_stage(const Ctx& c, const VelDev& v, const void* in, const void* phin, void* out,
                     const DevClock* clk, int stage, int combine, double ct_explicit,
                     const int* tile) {
  if (use_sep_kernel(v)) {
    int t[3];
    if (tile) { t[0] = tile[0]; t[1] = tile[1]; t[2] = tile[2]; }
    else {
      const int st = adv_default_tile(c, v, t);
      if (st) return st;
    }
    return sep_unit(2, c, &v, t, nullptr, in, phin, out, clk, stage, combine, ct_explicit);
  }
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
    a.v.vtab = reinterpret_cast<const T*>(v.vtab);
    a.v.n_terms = v.n_terms;
    a.v.nmax = v.nmax;
    a.v.npt = v.npt;
    for (int k = 0; k < v.n_terms; ++k) a.v.comp[k] = v.comp[k];
    term_ranges(a.v.comp, v.n_terms, a.v.cstart);
    if (v.tab) {
      a.v.tab_q = reinterpret_cast<const T*>(v.tab_q);
      a.v.tab_f = reinterpret_cast<const T*>(v.tab_f);
      for (int e = 0; e < 3; ++e) {
        a.v.tab_foff[e] = v.tab_foff[e];
        a.v.tab_nf[e] = v.tab_nf[e];
      }
    }
    a.phi_s = reinterpret_cast<const T*>(in);
    a.phi_n = reinterpret_cast<const T*>(phin);
    a.out = reinterpret_cast<T*>(out);
    a.clk = clk;
    a.stage = stage;
    a.combine = combine;
    a.ct_explicit = ct_explicit;
    const size_t smem = adv_smem_bytes<DIM, P, T>(a.m.tile, std::max(v.n_terms, 1), v.tab);
    if (v.tab)
      adv_stage_kernel<DIM, P, T, true><<<(unsigned)nblocks(a.m), t[0] * t[1] * t[2], smem, c.stream>>>(a);
    else
      adv_stage_kernel<DIM, P, T, false><<<(unsigned)nblocks(a.m), t[0] * t[1] * t[2], smem, c.stream>>>(a);
    return launch_status("adv_stage_kernel");
  });
}

}  // namespace flsp

// flsp_k_sep.cuh — launch side of the separable stage kernel
// (adv_sep_kernel, flsp_advsep.cuh), shared by the per-dimension units
// flsp_k_sep2.cu and flsp_k_sep3.cu.  The tile shape is a template
// parameter; these are the shapes built.
#pragma once
#include <cstring>
#include <type_traits>

#include "flsp_advsep.cuh"
#include "flsp_launch.h"

namespace flsp {

template <int V>
using IC = std::integral_constant<int, V>;

template <int DIM, typename F>
int with_sep_tile(const int* t, F&& f) {
  if constexpr (DIM == 3) {
    if (t[0] == 8 && t[1] == 8 && t[2] == 4) return f(IC<8>(), IC<8>(), IC<4>());
    if (t[0] == 8 && t[1] == 4 && t[2] == 4) return f(IC<8>(), IC<4>(), IC<4>());
    if (t[0] == 4 && t[1] == 4 && t[2] == 4) return f(IC<4>(), IC<4>(), IC<4>());
  } else {
    if (t[0] == 32 && t[1] == 8) return f(IC<32>(), IC<8>(), IC<1>());
    if (t[0] == 16 && t[1] == 16) return f(IC<16>(), IC<16>(), IC<1>());
    if (t[0] == 16 && t[1] == 8) return f(IC<16>(), IC<8>(), IC<1>());
    if (t[0] == 8 && t[1] == 8) return f(IC<8>(), IC<8>(), IC<1>());
  }
  return set_error(FLSP_ERR_UNSUPPORTED, "no separable stage kernel for this tile shape");
}

// what: 0 = shared-memory bytes of the tile (into *bytes), 1 = set the
// kernel's attributes, 2 = launch one stage
template <int DIM>
int sep_call(int what, const Ctx& c, const VelDev* v, const int* tile, size_t* bytes, const void* in,
             const void* phin, void* out, const DevClock* clk, int stage, int combine, double ct_explicit) {
  return dispatch(c, [&](auto D, auto PP, auto tz) -> int {
    constexpr int DD = decltype(D)::value;
    if constexpr (DD != DIM) {
      return set_error(FLSP_ERR_UNSUPPORTED, "separable stage kernel: wrong unit");
    } else {
      constexpr int P = decltype(PP)::value;
      using T = decltype(tz);
      auto body = [&](auto PBC) -> int {
        constexpr bool PB = decltype(PBC)::value;
        return with_sep_tile<DIM>(tile, [&](auto X, auto Y, auto Z) -> int {
          constexpr int TX = decltype(X)::value, TY = decltype(Y)::value, TZ = decltype(Z)::value;
          using PL = SepPlan<DIM, P, PB, TX, TY, TZ, T>;
          // with or without Dirichlet faces (the boundary lookup only where
          // the mesh carries some)
          auto kern = c.m.bc_face ? adv_sep_kernel<DIM, P, PB, TX, TY, TZ, T, true>
                                  : adv_sep_kernel<DIM, P, PB, TX, TY, TZ, T, false>;
          if (what == 0) {
            *bytes = PL::BYTES;
            return FLSP_OK;
          }
          if (what == 1) {
            if (PL::BYTES > 227 * 1024) return set_error(FLSP_ERR_BAD_ARG, "separable tile too large");
            for (auto k : {adv_sep_kernel<DIM, P, PB, TX, TY, TZ, T, true>,
                           adv_sep_kernel<DIM, P, PB, TX, TY, TZ, T, false>}) {
              cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PL::BYTES);
              if (e == cudaSuccess) e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
              if (e != cudaSuccess) return set_error(FLSP_ERR_CUDA, std::string("sep attr: ") + cudaGetErrorString(e));
            }
            return FLSP_OK;
          }
          AdvSepArgs<T> b;
          std::memset(&b, 0, sizeof(b));
          b.m = c.m;
          set_tile(b.m, DIM, tile);
          b.optab = reinterpret_cast<const T*>(v->optab);
          b.nmax = v->opstride;
          b.err = v->err;
          b.phi_s = reinterpret_cast<const T*>(in);
          b.phi_n = reinterpret_cast<const T*>(phin);
          b.out = reinterpret_cast<T*>(out);
          b.clk = clk;
          b.stage = stage;
          b.combine = combine;
          b.ct_explicit = ct_explicit;
          kern<<<(unsigned)nblocks(b.m), TX * TY * TZ, PL::BYTES, c.stream>>>(b);
          return launch_status("adv_sep_kernel");
        });
      };
      if (c.basis == FLSP_BASIS_P) return body(std::true_type());
      return body(std::false_type());
    }
  });
}

}  // namespace flsp

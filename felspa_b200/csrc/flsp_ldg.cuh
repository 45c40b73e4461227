// flsp_ldg.cuh — LDG artificial viscosity of the reinitialisation (nu > 0).
//
// Replaces LDGDiffusionTerm::compute_diffusion_term (src/pde/ldg.cc:249-298):
// the alternating-flux gradient q (LDGGradientAssembler<alternating>,
// ldg.cc:383-504, with beta renormalised to (1,..,1)/sqrt(dim),
// ldg.implement.h:304-313) followed by the diffusion RHS
// (LDGDiffusionAssembler<alternating>, ldg.cc:750-838; no boundary term).
// Every integral is of polynomial products integrated exactly by the
// reference's QGauss(p+1), so both kernels work modally, one line of modes
// along each axis d at a time (faces normal to d are the only ones with
// n_d != 0).  Per axis d, with traces T of the own cell and TnL / TnU of
// the lower / upper neighbour, kp = 1/2 + 1/sqrt(dim), km = 1/2 - 1/sqrt(dim):
//   q_d     = (1/h_d) [ -A c + L(1) phi^_up - L(0) phi^_lo ]
//   phi^_lo = kp T_lo + km TnL   (T_lo on the boundary)
//   phi^_up = km T_up + kp TnU   (T_up on the boundary)
//   R_d     = (nu/h_d) [ -A q_d + L(1) (kp q_up + km q_nU) - L(0) (km q_lo + kp q_nL) ]
// (face terms on interior faces only), all per unit cell volume.
#pragma once
#include "flsp_device.cuh"

namespace flsp {

template <typename T>
struct LdgArgs {
  MeshArgs m;
  const T* __restrict__ in;    // phi (q kernel) or q (diffusion kernel, DIM blocks)
  T* __restrict__ out;         // q (DIM blocks of ncell*nb) or R_diff (ncell*nb)
  long long block;             // ncell * nb
  double nu;
};

template <int DIM, int P, typename T>
__host__ __device__ inline size_t ldg_smem_bytes(const int* tile) {
  constexpr int NM = ipow(P + 1, DIM);
  const int bx = tile[0] + 2, by = DIM > 1 ? tile[1] + 2 : 1, bz = DIM > 2 ? tile[2] + 2 : 1;
  return (size_t)bx * by * bz * NM * sizeof(T);
}

// base index of mode line li along axis d in the Q layout
template <int DIM, int N1>
__device__ __forceinline__ int line_base(int d, int li) {
  constexpr int st[3] = {1, N1, N1 * N1};
  const int i0 = li % N1, i1 = li / N1;
  if constexpr (DIM == 2) return d == 0 ? i0 * st[1] : i0 * st[0];
  return d == 0 ? i0 * st[1] + i1 * st[2] : (d == 1 ? i0 * st[0] + i1 * st[2] : i0 * st[0] + i1 * st[1]);
}

// mode == 0: q from phi;  mode == 1: R_diff from q
template <int DIM, int P, typename T>
__global__ void __launch_bounds__(256) ldg_kernel(const LdgArgs<T> a, int mode) {
  constexpr int N1 = P + 1, NM = ipow(N1, DIM);
  constexpr int st[3] = {1, N1, N1 * N1};
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* box = reinterpret_cast<T*>(smem_raw);
  const MeshArgs& m = a.m;
  const Tab1D<T>& tb = tab<T>(P);
  if (tile_inactive(m)) return;
  const TileCoord tc = tile_coord(m, DIM);
  const T kp = T(0.5 + 1.0 / sqrt((double)DIM)), km = T(0.5 - 1.0 / sqrt((double)DIM));
  const int g[3] = {tc.gx, tc.gy, tc.gz};
  const int l[3] = {tc.lx, tc.ly, tc.lz};
  T acc[NM];
#pragma unroll
  for (int q = 0; q < NM; ++q) acc[q] = T(0);

  // mode 0 reads phi once; mode 1 reads q_d for each axis d in turn
  const int passes = mode == 0 ? 1 : DIM;
#pragma unroll 1
  for (int pass = 0; pass < passes; ++pass) {
    if (pass > 0) __syncthreads();
    load_box<DIM, NM>(m, a.in + (mode == 0 ? 0 : (long long)pass * a.block), box, tc.ox, tc.oy, tc.oz, true);
    cp_async_wait_all();
    __syncthreads();
    if (!tc.valid) continue;
    const T* c = box + (size_t)box_index(m, DIM, l[0], l[1], l[2]) * NM;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      if (mode == 1 && d != pass) continue;
      int ll[3] = {l[0], l[1], l[2]}, lu[3] = {l[0], l[1], l[2]};
      ll[d] -= 1;
      lu[d] += 1;
      const bool has_lo = g[d] > 0, has_hi = g[d] + 1 < m.n[d];
      const T* cL = box + (size_t)box_index(m, DIM, ll[0], ll[1], ll[2]) * NM;
      const T* cU = box + (size_t)box_index(m, DIM, lu[0], lu[1], lu[2]) * NM;
      const T ih = T(1.0 / m.h[d]);
      T out[NM];
#pragma unroll
      for (int li = 0; li < NM / N1; ++li) {
        const int base = line_base<DIM, N1>(d, li);
        T tlo = T(0), tup = T(0), tnl = T(0), tnu = T(0);
#pragma unroll
        for (int b = 0; b < N1; ++b) {
          const T cb = c[base + b * st[d]];
          tlo += tb.L0[b] * cb;
          tup += tb.L1[b] * cb;
          if (has_lo) tnl += tb.L1[b] * cL[base + b * st[d]];
          if (has_hi) tnu += tb.L0[b] * cU[base + b * st[d]];
        }
        T flo, fup;
        if (mode == 0) {
          flo = has_lo ? kp * tlo + km * tnl : tlo;
          fup = has_hi ? km * tup + kp * tnu : tup;
        } else {
          flo = has_lo ? km * tlo + kp * tnl : T(0);
          fup = has_hi ? kp * tup + km * tnu : T(0);
        }
#pragma unroll
        for (int aa = 0; aa < N1; ++aa) {
          T s = T(0);
#pragma unroll
          for (int b = 0; b < N1; ++b) s -= tb.A[aa][b] * c[base + b * st[d]];
          out[base + aa * st[d]] = (s + tb.L1[aa] * fup - tb.L0[aa] * flo) * ih;
        }
      }
      if (mode == 0) {
        const long long cell = (long long)g[0] + (long long)m.n[0] * (g[1] + (long long)m.n[1] * g[2]);
        for (int k = 0; k < m.nb; ++k) a.out[(long long)d * a.block + cell * m.nb + k] = out[m.g2q[k]];
      } else {
#pragma unroll
        for (int q = 0; q < NM; ++q) acc[q] += T(a.nu) * out[q];
      }
    }
  }
  if (mode == 1 && tc.valid) {
    const long long cell = (long long)g[0] + (long long)m.n[0] * (g[1] + (long long)m.n[1] * g[2]);
    for (int k = 0; k < m.nb; ++k) a.out[cell * m.nb + k] = acc[m.g2q[k]];
  }
}

}  // namespace flsp

// flsp_advsep.cuh — DG advection stage kernel for a separable velocity.
//
// Same operator as adv_stage_kernel (AdvectAssembler cell, face and
// boundary terms, include/felspa/pde/src/advection.implement.h:617-744,
// on QGauss(p+2) cell and face rules), evaluated for a velocity whose
// component d is ONE separable term u_d = c(t) g_d0(x) g_d1(y) g_d2(z)
// (coefficient folded into g_d0).  The tensor-product Gauss sum of a
// separable integrand is the product of 1D Gauss sums, so the quadrature
// sums factor exactly into per-axis operators (no approximation):
//
//   cell, component d:  R += c(t)/h_d (A_d0 (x) A_d1 (x) A_d2) phi
//     A_de[a][b] = sum_q w_q g_de(x_q) L_b(x_q) (e == d ? L_a'(x_q) : L_a(x_q))
//   face normal E (flux in +e_E, traces T- of the lower, T+ of the upper cell):
//     u_E phi_upwind = u_E (T- + T+)/2 + |u_E| (T- - T+)/2
//     F = c g_EE (A_Et0 (x) A_Et1) (T- + T+)/2
//       + |c g_EE| (B_Et0 (x) B_Et1) (T- - T+)/2,   B_de = A_de with |g_de|
//   (|u_E| = |c g_EE| |g_Et0| |g_Et1| is separable too; on the domain
//   boundary T+ = T- (own trace, zero-Neumann inflow), so the second term
//   vanishes); R- -= L(1) F / h_E, R+ += L(0) F / h_E.
//
// The per-axis operators are tabulated once per velocity on the host in
// FP64 (optab, one row per component d, axis e and cell index i:
// A_de then, at element BOFF, B_de, or for e == d A_dd then g_dd(0),
// g_dd(1)).  Per cell that
// is ~1.5k FMA for Q2 in 3D instead of the ~4k of point-wise quadrature.
#pragma once
#include "flsp_advect.cuh"

namespace flsp {

// row layout: two (P+1)^2 blocks, each padded to a multiple of 4 elements
// so that every block starts on a 16-byte boundary (FP32 and FP64)
template <int P>
__host__ __device__ constexpr int sep_boff() {
  return (((P + 1) * (P + 1) + 3) / 4) * 4;
}
template <int P>
__host__ __device__ constexpr int sep_opw() {
  return 2 * sep_boff<P>();
}

template <typename T>
struct AdvSepArgs {
  MeshArgs m;
  const T* __restrict__ optab;   // [(d*3 + e) * nmax + i][OPW]
  int nmax;
  const T* __restrict__ phi_s;
  const T* __restrict__ phi_n;
  T* __restrict__ out;
  const DevClock* clk;
  int stage;
  int combine;
  double ct_explicit;
  double dt_explicit;
};

// Face-flux slots of a tile along axis E: every face normal to E that
// touches a tile cell, i.e. tile[E] + 1 faces per line along E.  Slot s of
// a line is the face below tile cell s (s = tile[E]: the tile's top face).
__host__ __device__ inline int sep_face_slots(const int* tile, int dim, int E) {
  int n = 1;
  for (int d = 0; d < dim; ++d) n *= tile[d] + (d == E ? 1 : 0);
  return n;
}

// shared memory: tile box with face halo | operator rows of the tile |
// face fluxes per axis (reused for the tile's R before the store)
template <int DIM, int P, typename T>
__host__ __device__ inline size_t sep_smem_bytes(const int* tile) {
  constexpr int N1 = P + 1, NM = ipow(N1, DIM), NF = ipow(N1, DIM - 1), OPW = sep_opw<P>();
  const int bx = tile[0] + 2, by = DIM > 1 ? tile[1] + 2 : 1, bz = DIM > 2 ? tile[2] + 2 : 1;
  const int nt = tile[0] * tile[1] * (DIM > 2 ? tile[2] : 1);
  const int span = tile[0] + tile[1] + (DIM > 2 ? tile[2] : 0);
  size_t box = (size_t)bx * by * bz * NM * sizeof(T);
  size_t ops = (size_t)DIM * span * OPW * sizeof(T);
  size_t fl = 0;
  for (int E = 0; E < DIM; ++E) fl += (size_t)NF * sep_face_slots(tile, DIM, E);
  fl = (fl > (size_t)nt * NM ? fl : (size_t)nt * NM) * sizeof(T);
  return box + ops + fl + 16;
}

// N1 x N1 operator block from shared memory (16-byte aligned)
template <int N1, typename T>
__device__ __forceinline__ void load_op(const T* __restrict__ src, T (&M)[N1][N1]) {
  constexpr int NN = N1 * N1;
  T v[NN];
  if constexpr (sizeof(T) == 4) {
#pragma unroll
    for (int k = 0; k + 4 <= NN; k += 4) {
      const float4 f = *reinterpret_cast<const float4*>(src + k);
      v[k] = f.x; v[k + 1] = f.y; v[k + 2] = f.z; v[k + 3] = f.w;
    }
#pragma unroll
    for (int k = (NN / 4) * 4; k < NN; ++k) v[k] = src[k];
  } else {
#pragma unroll
    for (int k = 0; k + 2 <= NN; k += 2) {
      const double2 f = *reinterpret_cast<const double2*>(src + k);
      v[k] = f.x; v[k + 1] = f.y;
    }
#pragma unroll
    for (int k = (NN / 2) * 2; k < NN; ++k) v[k] = src[k];
  }
#pragma unroll
  for (int a = 0; a < N1; ++a)
#pragma unroll
    for (int b = 0; b < N1; ++b) M[a][b] = v[a * N1 + b];
}

// R += s * (M0 (x) M1 (x) M2) x, Q layout (index a0 + N1 a1 + N1^2 a2),
// contracted one z-slab of x at a time to keep the partial sums small
template <int DIM, int N1, typename T>
__device__ __forceinline__ void apply_sep_acc(const T (&M0)[N1][N1], const T (&M1)[N1][N1],
                                              const T (&M2)[N1][N1], const T* x, T* R, T s) {
  constexpr int NZ = DIM > 2 ? N1 : 1;
#pragma unroll
  for (int b2 = 0; b2 < NZ; ++b2) {
    T u[N1][N1];   // [a0][b1]
#pragma unroll
    for (int a0 = 0; a0 < N1; ++a0)
#pragma unroll
      for (int b1 = 0; b1 < N1; ++b1) {
        T acc = T(0);
#pragma unroll
        for (int b0 = 0; b0 < N1; ++b0) acc += M0[a0][b0] * x[b0 + N1 * (b1 + N1 * b2)];
        u[a0][b1] = acc;
      }
#pragma unroll
    for (int a1 = 0; a1 < N1; ++a1)
#pragma unroll
      for (int a0 = 0; a0 < N1; ++a0) {
        T acc = T(0);
#pragma unroll
        for (int b1 = 0; b1 < N1; ++b1) acc += M1[a1][b1] * u[a0][b1];
        if constexpr (DIM == 2) {
          R[a0 + N1 * a1] += s * acc;
        } else {
          const T v = s * acc;
#pragma unroll
          for (int a2 = 0; a2 < N1; ++a2) R[a0 + N1 * (a1 + N1 * a2)] += M2[a2][b2] * v;
        }
      }
  }
}

// F = s1 (A0 (x) A1) S + s2 (B0 (x) B1) D on the face modes (m0 + N1 m1);
// in 2D only A0 / B0; the B blocks start BOFF elements after the A blocks
template <int DIM, int N1, int BOFF, typename T>
__device__ __forceinline__ void face_apply(const T* __restrict__ rowA0, const T* __restrict__ rowA1,
                                           const T* S, const T* D, T s1, T s2, bool upwind, T* F) {
  constexpr int NF = DIM > 2 ? N1 * N1 : N1;
  T M0[N1][N1];
  load_op<N1, T>(rowA0, M0);
  if constexpr (DIM == 2) {
#pragma unroll
    for (int a0 = 0; a0 < N1; ++a0) {
      T acc = T(0);
#pragma unroll
      for (int b0 = 0; b0 < N1; ++b0) acc += M0[a0][b0] * S[b0];
      F[a0] = s1 * acc;
    }
    if (upwind) {
      load_op<N1, T>(rowA0 + BOFF, M0);
#pragma unroll
      for (int a0 = 0; a0 < N1; ++a0) {
        T acc = T(0);
#pragma unroll
        for (int b0 = 0; b0 < N1; ++b0) acc += M0[a0][b0] * D[b0];
        F[a0] += s2 * acc;
      }
    }
  } else {
    T M1[N1][N1];
    load_op<N1, T>(rowA1, M1);
    auto apply2 = [&](const T* x, T s, bool acc_into) {
      T u[N1][N1];   // [a0][b1]
#pragma unroll
      for (int a0 = 0; a0 < N1; ++a0)
#pragma unroll
        for (int b1 = 0; b1 < N1; ++b1) {
          T acc = T(0);
#pragma unroll
          for (int b0 = 0; b0 < N1; ++b0) acc += M0[a0][b0] * x[b0 + N1 * b1];
          u[a0][b1] = acc;
        }
#pragma unroll
      for (int a1 = 0; a1 < N1; ++a1)
#pragma unroll
        for (int a0 = 0; a0 < N1; ++a0) {
          T acc = T(0);
#pragma unroll
          for (int b1 = 0; b1 < N1; ++b1) acc += M1[a1][b1] * u[a0][b1];
          if (acc_into) F[a0 + N1 * a1] += s * acc;
          else F[a0 + N1 * a1] = s * acc;
        }
    };
    apply2(S, s1, false);
    if (upwind) {
      load_op<N1, T>(rowA0 + BOFF, M0);
      load_op<N1, T>(rowA1 + BOFF, M1);
      apply2(D, s2, true);
    }
  }
  (void)NF;
}

// trace of the cell polynomial on the face normal to E, in face modes
template <int DIM, int N1, int E, typename T>
__device__ __forceinline__ void face_trace(const T* c, const T* Lside, T* tr) {
  constexpr int NF = DIM > 2 ? N1 * N1 : N1;
  constexpr int t0 = E == 0 ? 1 : 0, t1 = E == 2 ? 1 : 2;
  constexpr int st[3] = {1, N1, N1 * N1};
#pragma unroll
  for (int mf = 0; mf < NF; ++mf) {
    const int m0 = mf % N1, m1 = mf / N1;
    const int base = m0 * st[t0] + (DIM > 2 ? m1 * st[t1] : 0);
    T s = T(0);
#pragma unroll
    for (int a = 0; a < N1; ++a) s += Lside[a] * c[base + a * st[E]];
    tr[mf] = s;
  }
}

// FP32 tiles fit two CTAs per SM (<= 128 registers); an FP64 tile takes most
// of an SM's shared memory, so FP64 gets the full register file
template <int DIM, int P, typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 2 : 1) adv_sep_kernel(const AdvSepArgs<T> a) {
  constexpr int N1 = P + 1, NM = ipow(N1, DIM), NF = ipow(N1, DIM - 1);
  constexpr int OPW = sep_opw<P>(), BOFF = sep_boff<P>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* box = reinterpret_cast<T*>(smem_raw);
  const MeshArgs& m = a.m;
  const int nboxc = box_cells(m, DIM);
  const int tx = m.tile[0], ty = m.tile[1], tz = m.tile[2];
  const int tl[3] = {tx, ty, tz};
  const int nt = tx * ty * tz;
  const int span = tx + ty + (DIM > 2 ? tz : 0);
  const int roff[3] = {0, tx, tx + ty};   // first row of each axis within a component
  // box holds NM values per cell; keep the operator rows 16-byte aligned
  T* ops = align16<T>(box + (size_t)nboxc * NM);
  T* fl = ops + (size_t)DIM * span * OPW;   // face fluxes, then the tile's R
  int flo[3] = {0, 0, 0};                   // section offsets of the face fluxes
  for (int E = 1; E < DIM; ++E) flo[E] = flo[E - 1] + NF * sep_face_slots(m.tile, DIM, E - 1);
  const Tab1D<T>& tb = tab<T>(P);
  const TileCoord tc = tile_coord(m, DIM);

  // ---- operator rows of this tile: ops[(d*span + roff[e] + li)*OPW + k]
  {
    const int total = DIM * span * OPW;
    for (int e2 = threadIdx.x; e2 < total; e2 += blockDim.x) {
      const int k = e2 % OPW;
      const int r = e2 / OPW;
      const int li = r % span;
      const int d = r / span;
      int axis, gi;
      if (li < tx) { axis = 0; gi = tc.ox + li; }
      else if (li < tx + ty) { axis = 1; gi = tc.oy + (li - tx); }
      else { axis = 2; gi = tc.oz + (li - tx - ty); }
      gi = min(gi, m.n[axis] - 1);
      ops[(size_t)r * OPW + k] = a.optab[((size_t)(d * 3 + axis) * a.nmax + gi) * OPW + k];
    }
  }
  load_box<DIM, NM>(m, a.phi_s, box, tc.ox, tc.oy, tc.oz, true);
  cp_async_wait_all();
  __syncthreads();

  const T ct = a.clk ? T(a.clk->ct[a.stage]) : T(a.ct_explicit);
  const T dt = a.clk ? T(a.clk->dt) : T(a.dt_explicit);
  const bool active = a.clk ? (a.clk->active != 0) : true;
  const int cl = tc.lx + tx * (tc.ly + ty * tc.lz);
  const int me = box_index(m, DIM, tc.lx, tc.ly, tc.lz);
  const T ih[3] = {T(1.0 / m.h[0]), T(1.0 / m.h[1]), T(DIM > 2 ? 1.0 / m.h[2] : 1.0)};
  const int g[3] = {tc.gx, tc.gy, tc.gz};
  const int l[3] = {tc.lx, tc.ly, tc.lz};
  const bool work = tc.valid && active;

  auto rowp = [&](int d, int e, int le) -> const T* {
    return ops + (size_t)(d * span + roff[e] + le) * OPW;
  };
  // face-flux slot of the face below local cell lc along E (lc[E] in [0, tile[E]])
  auto slot = [&](int E, const int* lc) -> int {
    const int e0 = tl[0] + (E == 0), e1 = tl[1] + (E == 1);
    return lc[0] + e0 * (lc[1] + (DIM > 2 ? e1 * lc[2] : 0));
  };
  auto flux_at = [&](int E, int mf, int sl) -> T& {
    return fl[flo[E] + (size_t)mf * sep_face_slots(m.tile, DIM, E) + sl];
  };

  // flux through the face normal to E in +e_E between the lower cell (L1
  // trace of cm) and the upper cell (L0 trace of cp); a missing side takes
  // the other side's trace (domain boundary: own trace).  Tangential
  // operator rows at local coordinates lc, g_EE at the face = fe.
  auto face_flux_sep = [&](auto EC, const T* cm, const T* cp, bool has_m, bool has_p, const int* lc,
                           T fe, T* F) {
    constexpr int E = decltype(EC)::value;
    constexpr int t0 = E == 0 ? 1 : 0, t1 = E == 2 ? 1 : 2;
    T Tm[NF], Tp[NF], S[NF], D[NF];
    if (has_m) face_trace<DIM, N1, E, T>(cm, tb.L1, Tm);
    if (has_p) face_trace<DIM, N1, E, T>(cp, tb.L0, Tp);
#pragma unroll
    for (int mf = 0; mf < NF; ++mf) {
      if (!has_m) Tm[mf] = Tp[mf];
      if (!has_p) Tp[mf] = Tm[mf];
      S[mf] = T(0.5) * (Tm[mf] + Tp[mf]);
      D[mf] = T(0.5) * (Tm[mf] - Tp[mf]);
    }
    const T s1 = ct * fe;
    face_apply<DIM, N1, BOFF, T>(rowp(E, t0, lc[t0]), DIM > 2 ? rowp(E, t1, lc[t1]) : nullptr, S, D, s1,
                                 s1 < T(0) ? -s1 : s1, has_m && has_p, F);
  };

  T R[NM];
#pragma unroll
  for (int q = 0; q < NM; ++q) R[q] = T(0);

  if (work) {
    T c[NM];
#pragma unroll
    for (int q = 0; q < NM; ++q) c[q] = box[(size_t)me * NM + q];
    // ============================ cell term ============================
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      T M0[N1][N1], M1[N1][N1], M2[N1][N1];
      load_op<N1, T>(rowp(d, 0, l[0]), M0);
      load_op<N1, T>(rowp(d, 1, l[1]), M1);
      if constexpr (DIM > 2) load_op<N1, T>(rowp(d, 2, l[2]), M2);
      apply_sep_acc<DIM, N1, T>(M0, M1, M2, c, R, ct * ih[d]);
    }
    // ===== upper faces: own flux, shared with the upper neighbour via slot l[E] + 1
    auto do_upper = [&](auto EC) {
      constexpr int E = decltype(EC)::value;
      int nl[3] = {l[0], l[1], l[2]};
      nl[E] += 1;
      const bool has_nb = g[E] + 1 < m.n[E];
      const T* cn = box + (size_t)box_index(m, DIM, nl[0], nl[1], nl[2]) * NM;
      T F[NF];
      face_flux_sep(EC, c, cn, true, has_nb, l, rowp(E, E, l[E])[BOFF + 1], F);
      scatter_face<DIM, P, E, T>(R, tb.L1, F, -ih[E]);
      const int sl = slot(E, nl);
#pragma unroll
      for (int mf = 0; mf < NF; ++mf) flux_at(E, mf, sl) = F[mf];
    };
    do_upper(std::integral_constant<int, 0>());
    do_upper(std::integral_constant<int, 1>());
    if constexpr (DIM == 3) do_upper(std::integral_constant<int, 2>());
  }

  // ===== the tile's lower boundary faces (slot 0 of every line), as work
  // items: axis E's items start at a warp boundary so that a warp serves
  // one axis
  if (active) {
    int nitem[3], ibase[3], tot = 0;
    for (int E = 0; E < DIM; ++E) {
      nitem[E] = nt / tl[E];
      ibase[E] = tot;
      tot += (nitem[E] + 31) & ~31;
    }
    for (int it = threadIdx.x; it < tot; it += blockDim.x) {
      auto do_item = [&](auto EC) {
        constexpr int E = decltype(EC)::value;
        const int k = it - ibase[E];
        if (k < 0 || k >= nitem[E]) return;
        // tile cell with local coordinate 0 along E; the others from k
        constexpr int t0 = E == 0 ? 1 : 0, t1 = E == 2 ? 1 : 2;
        int lc[3] = {0, 0, 0};
        lc[t0] = k % tl[t0];
        if (DIM > 2) lc[t1] = k / tl[t0];
        const int gc[3] = {(E == 0 ? 0 : lc[0]) + tc.ox, (E == 1 ? 0 : lc[1]) + tc.oy,
                           DIM > 2 ? (E == 2 ? 0 : lc[2]) + tc.oz : 0};
        if (gc[0] >= m.n[0] || gc[1] >= m.n[1] || (DIM > 2 && gc[2] >= m.n[2])) return;
        int ll[3] = {lc[0], lc[1], lc[2]};
        ll[E] -= 1;
        const bool has_m = gc[E] > 0;
        const T* cp = box + (size_t)box_index(m, DIM, lc[0], lc[1], lc[2]) * NM;
        const T* cm = box + (size_t)box_index(m, DIM, ll[0], ll[1], ll[2]) * NM;
        T F[NF];
        face_flux_sep(EC, cm, cp, has_m, true, lc, rowp(E, E, 0)[BOFF], F);
        const int sl = slot(E, lc);
#pragma unroll
        for (int mf = 0; mf < NF; ++mf) flux_at(E, mf, sl) = F[mf];
      };
      do_item(std::integral_constant<int, 0>());
      do_item(std::integral_constant<int, 1>());
      if constexpr (DIM == 3) do_item(std::integral_constant<int, 2>());
    }
  }
  __syncthreads();
  // ===== lower faces: every cell reads slot l[E]
  if (work) {
    auto do_lower = [&](auto EC) {
      constexpr int E = decltype(EC)::value;
      const int sl = slot(E, l);
      T F[NF];
#pragma unroll
      for (int mf = 0; mf < NF; ++mf) F[mf] = flux_at(E, mf, sl);
      scatter_face<DIM, P, E, T>(R, tb.L0, F, ih[E]);
    };
    do_lower(std::integral_constant<int, 0>());
    do_lower(std::integral_constant<int, 1>());
    if constexpr (DIM == 3) do_lower(std::integral_constant<int, 2>());
  }
  __syncthreads();   // face fluxes consumed: the region now holds R [cell][NM]
  T* rbuf = fl;
  if (work) {
#pragma unroll
    for (int q = 0; q < NM; ++q) rbuf[(size_t)cl * NM + q] = R[q];
  }
  __syncthreads();

  // ---- RK combination fused into the coalesced store: one warp per row of
  // cells along x; stage input from the box, phi^n straight from HBM
  const bool need_n = a.combine == kRK2b || a.combine == kRK3b || a.combine == kRK3c;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const bool dense = m.nb == NM;
  for (int r = warp; r < ty * tz; r += nw) {
    const int ly = r % ty, lz = r / ty;
    const int gy = tc.oy + ly, gz = tc.oz + lz;
    const int nx = min(tx, m.n[0] - tc.ox);
    if (gy >= m.n[1] || gz >= m.n[2] || nx <= 0) continue;
    const long long gbase = ((long long)m.n[0] * (gy + (long long)m.n[1] * gz) + tc.ox) * m.nb;
    const T* cs = box + (size_t)box_index(m, DIM, 0, ly, lz) * NM;
    const T* rs = rbuf + (size_t)tx * r * NM;
    if (dense) {
#pragma unroll 4
      for (int e = lane; e < nx * NM; e += 32) {
        const T cv = cs[e];
        T res = cv;
        if (active) {
          const T pn = need_n ? __ldg(a.phi_n + gbase + e) : T(0);
          res = combine_value<T>(a.combine, cv, pn, rs[e], dt);
        }
        a.out[gbase + e] = res;
      }
    } else {
      for (int e = lane; e < nx * m.nb; e += 32) {
        const int cx = e / m.nb, k = e - cx * m.nb;
        const int q = cx * NM + m.g2q[k];
        const T cv = cs[q];
        T res = cv;
        if (active) {
          const T pn = need_n ? __ldg(a.phi_n + gbase + e) : T(0);
          res = combine_value<T>(a.combine, cv, pn, rs[q], dt);
        }
        a.out[gbase + e] = res;
      }
    }
  }
}

}  // namespace flsp

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
//   boundary the missing trace is the Dirichlet value of the face, or the
//   own trace (zero-Neumann inflow), when the second term vanishes);
//   R- -= L(1) F / h_E, R+ += L(0) F / h_E.
//
// The CTA's halo box (one bulk copy per row of cells, each row keeping its
// 16-byte phase from HBM so that 27-value cells need no splitting) and its
// operator rows arrive by TMA bulk copies on one mbarrier.  Every face of
// the tile is then one work item of a single routine (runtime axis), its
// flux kept in shared memory; each cell adds its cell term and lifts its
// faces' fluxes; the RK combination is fused into a coalesced store that
// prefetches phi^n into registers (float4 rows where FP32 alignment
// allows).  Tile shapes are compile-time.
//
// The per-axis operators are tabulated once per velocity on the host in
// FP64 (optab, one row per component d, axis e and cell index i:
// A_de then, at element BOFF, B_de, or for e == d A_dd then g_dd(0),
// g_dd(1)).  Per cell that
// is ~1.5k FMA for Q2 in 3D instead of the ~4k of point-wise quadrature.
#pragma once
#include "flsp_advect.cuh"

namespace flsp {

// row layout: two (P+1)^2 blocks, each with one spare element and padded to
// a multiple of 4 elements so that every block starts on a 16-byte boundary
// (FP32 and FP64).  The spare element of the A block of a row with e != d
// holds the sign of g_de over the cell's Gauss points (+1 / -1 if it keeps
// one sign, 0 if it changes sign).
template <int P>
__host__ __device__ constexpr int sep_boff() {
  return (((P + 1) * (P + 1) + 1 + 3) / 4) * 4;
}
template <int P>
__host__ __device__ constexpr int sep_opw() {
  return 2 * sep_boff<P>();
}

template <typename T>
struct AdvSepArgs {
  MeshArgs m;
  const T* __restrict__ optab;   // [(d*3 + e) * nmax + i][OPW]
  int nmax;                      // row stride per (d, e): >= n[e] + kOpRowPad (a tile's
                                 // bulk copy of its rows never leaves the table)
  int* err;                      // device error word (DevClock::err)
  const T* __restrict__ phi_s;
  const T* __restrict__ phi_n;
  T* __restrict__ out;
  const DevClock* clk;
  int stage;
  int combine;
  double ct_explicit;
  double dt_explicit;
};

// In-cell DoF index (HBM order) of Q-layout mode q for FE_DGP
// (PolynomialSpace order: c outer, b, a inner with a + b + c <= P), -1 for a
// mode outside P-space
template <int DIM, int P>
__host__ __device__ constexpr int q2g_ct(int q) {
  const int N1 = P + 1;
  const int a = q % N1, b = (q / N1) % N1, c = DIM > 2 ? q / (N1 * N1) : 0;
  if (a + b + c > P) return -1;
  int idx = 0;
  for (int cc = 0; cc < c; ++cc)
    for (int bb = 0; bb <= P - cc; ++bb) idx += P - bb - cc + 1;
  for (int bb = 0; bb < b; ++bb) idx += P - bb - c + 1;
  return idx + a;
}

// Shared-memory plan of the separable stage kernel for a compile-time tile
// TX x TY x TZ (TZ = 1 in 2D): mbarrier | halo box rows | operator rows |
// face fluxes (reused for the tile's R).  Box rows: (TY+2)(TZ+2) slots of
// SLOT bytes, each holding the row's cells x in [ox-1, ox+TX] from the
// 16-byte-aligned address at or below the first one.
template <int DIM, int P, bool PB, int TX, int TY, int TZ, typename T>
struct SepPlan {
  static constexpr int N1 = P + 1, NM = ipow(N1, DIM), NF = ipow(N1, DIM - 1);
  static constexpr int NBG = PB ? (DIM == 2 ? (P + 1) * (P + 2) / 2 : (P + 1) * (P + 2) * (P + 3) / 6) : NM;
  static constexpr int OPW = sep_opw<P>();
  static constexpr int NT = TX * TY * TZ;
  static constexpr int BY = DIM > 1 ? TY + 2 : 1, BZ = DIM > 2 ? TZ + 2 : 1;
  static constexpr int NROWS = BY * BZ;
  static constexpr int NMB = NBG * (int)sizeof(T);           // bytes per cell in HBM
  static constexpr int SLOT = (((TX + 2) * NMB + 30) + 15) / 16 * 16;
  static constexpr int SPAN = TX + TY + (DIM > 2 ? TZ : 0);
  static constexpr int SL0 = (TX + 1) * TY * TZ, SL1 = TX * (TY + 1) * TZ,
                       SL2 = DIM > 2 ? TX * TY * (TZ + 1) : 0;
  static constexpr int FLN = NF * (SL0 + SL1 + SL2);
  static constexpr int FLE = FLN > NT * NM ? FLN : NT * NM;  // elements
  static constexpr size_t OFF_BOX = 16;
  static constexpr size_t OFF_OPS = OFF_BOX + (size_t)NROWS * SLOT;
  static constexpr size_t OFF_FL = OFF_OPS + (size_t)DIM * SPAN * OPW * sizeof(T);
  static constexpr size_t BYTES = OFF_FL + (size_t)FLE * sizeof(T);
};

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

// trace of a box cell (HBM order) on its face normal to E, in face modes
// (side values Ls = L(0) or L(1)); the P basis reads its modes through the
// Q-layout map
template <int DIM, int P, bool PB, int E, typename T>
__device__ __forceinline__ void face_trace_ct(const T* __restrict__ src, const T* Ls, T* tr) {
  constexpr int N1 = P + 1, NF = DIM > 2 ? N1 * N1 : N1;
  constexpr int t0 = E == 0 ? 1 : 0, t1 = E == 2 ? 1 : 2;
  constexpr int st[3] = {1, N1, N1 * N1};
#pragma unroll
  for (int mf = 0; mf < NF; ++mf) {
    const int m0 = mf % N1, m1 = mf / N1;
    const int base = m0 * st[t0] + (DIM > 2 ? m1 * st[t1] : 0);
    T s = T(0);
#pragma unroll
    for (int aa = 0; aa < N1; ++aa) {
      const int q = base + aa * st[E];
      if constexpr (PB) {
        const int gi = q2g_ct<DIM, P>(q);
        if (gi >= 0) s += Ls[aa] * src[gi];
      } else {
        s += Ls[aa] * src[q];
      }
    }
    tr[mf] = s;
  }
}

// R += s (M0 (x) M1 (x) M2) c (Q layout, index a0 + N1 a1 + N1^2 a2),
// contracted one z-slab of c at a time; M2 read from its shared-memory row
template <int DIM, int P, typename T>
__device__ __forceinline__ void apply_sep_reg(const T (&M0)[P + 1][P + 1], const T (&M1)[P + 1][P + 1],
                                              const T* __restrict__ m2row, const T* c, T* R, T s) {
  constexpr int N1 = P + 1, NZ = DIM > 2 ? N1 : 1;
#pragma unroll
  for (int b2 = 0; b2 < NZ; ++b2) {
    T u[N1][N1];   // [a0][b1]
#pragma unroll
    for (int a0 = 0; a0 < N1; ++a0)
#pragma unroll
      for (int b1 = 0; b1 < N1; ++b1) {
        T acc = T(0);
#pragma unroll
        for (int b0 = 0; b0 < N1; ++b0) acc += M0[a0][b0] * c[b0 + N1 * (b1 + N1 * b2)];
        u[a0][b1] = acc;
      }
    T m2c[N1];   // column b2 of M2
    if constexpr (DIM > 2) {
#pragma unroll
      for (int a2 = 0; a2 < N1; ++a2) m2c[a2] = m2row[a2 * N1 + b2];
    }
#pragma unroll
    for (int a1 = 0; a1 < N1; ++a1)
#pragma unroll
      for (int a0 = 0; a0 < N1; ++a0) {
        T acc = T(0);
#pragma unroll
        for (int b1 = 0; b1 < N1; ++b1) acc += M1[a1][b1] * u[a0][b1];
        const T v = s * acc;
        if constexpr (DIM == 2) {
          R[a0 + N1 * a1] += v;
        } else {
#pragma unroll
          for (int a2 = 0; a2 < N1; ++a2) R[a0 + N1 * (a1 + N1 * a2)] += m2c[a2] * v;
        }
      }
  }
}

// FP32 tiles fit two CTAs per SM (<= 128 registers); an FP64 tile takes most
// of an SM's shared memory, so FP64 gets the full register file.
//
// Phases: (1) every face of the tile (interior, tile boundary, domain
// boundary) is a work item: traces of its two box cells, the separable
// upwind flux, written to the face's slot, so each face's flux is computed
// once per CTA by one routine whatever the tiling;
// (2) every cell: the cell term (one direction at a time) and the lifting of
// its 2 dim face fluxes from the slots; (3) the RK combination fused into
// the coalesced store.  BC: the mesh may carry Dirichlet faces.
template <int DIM, int P, bool PB, int TX, int TY, int TZ, typename T, bool BC>
__global__ void __launch_bounds__(TX * TY * TZ, sizeof(T) == 4 ? 2 : 1)
    adv_sep_kernel(const AdvSepArgs<T> a) {
  using PL = SepPlan<DIM, P, PB, TX, TY, TZ, T>;
  constexpr int N1 = PL::N1, NM = PL::NM, NF = PL::NF, OPW = PL::OPW, BOFF = sep_boff<P>();
  constexpr int NBG = PL::NBG;
  constexpr int NT = PL::NT, NMB = PL::NMB, SPAN = PL::SPAN;
  constexpr int TL[3] = {TX, TY, TZ};
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(smem_raw);
  unsigned char* boxb = smem_raw + PL::OFF_BOX;
  T* ops = reinterpret_cast<T*>(smem_raw + PL::OFF_OPS);
  T* fl = reinterpret_cast<T*>(smem_raw + PL::OFF_FL);
  const MeshArgs& m = a.m;
  const Tab1D<T>& tb = tab<T>(P);

  // tile and cell coordinates
  int b = blockIdx.x;
  const int ox = (b % m.ntile[0]) * TX;
  b /= m.ntile[0];
  const int oy = DIM > 1 ? (b % m.ntile[1]) * TY : 0;
  const int oz = DIM > 2 ? (b / m.ntile[1]) * TZ : 0;
  const int l[3] = {(int)threadIdx.x % TX, ((int)threadIdx.x / TX) % TY, DIM > 2 ? (int)threadIdx.x / (TX * TY) : 0};
  const int g[3] = {ox + l[0], oy + l[1], oz + l[2]};
  const bool valid = g[0] < m.n[0] && g[1] < m.n[1] && (DIM < 3 || g[2] < m.n[2]);
  const int gx0 = max(ox - 1, 0), gx1 = min(ox + TX + 1, m.n[0]);

  // address of the box copy of the cell at local coordinates (lx, ly, lz)
  auto cellp = [&](int lx, int ly, int lz) -> const T* {
    const int rr = DIM > 2 ? (ly + 1) + PL::BY * (lz + 1) : ly + 1;
    const unsigned rowcell = (unsigned)m.n[0] * (unsigned)((oy + ly) + m.n[1] * (DIM > 2 ? oz + lz : 0));
    const unsigned phase = ((rowcell + (unsigned)gx0) * (unsigned)NMB) & 15u;
    return reinterpret_cast<const T*>(boxb + (size_t)rr * PL::SLOT + phase + (ox + lx - gx0) * NMB);
  };
  // operator row of component d, axis e, tile cell le along e
  auto rowp = [&](int d, int e, int le) -> const T* {
    const int roff = e == 0 ? 0 : (e == 1 ? TX : TX + TY);
    return ops + (size_t)(d * SPAN + roff + le) * OPW;
  };

  // ---- staging: box rows and operator rows by bulk copies (warp 0)
  if (threadIdx.x == 0) mbar_init(bar, 1);
  __syncthreads();
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    const char* gsrc = reinterpret_cast<const char*>(a.phi_s);
    // pass 0 counts the bytes, pass 1 issues the copies
    unsigned bytes = 0;
    for (int pass = 0; pass < 2; ++pass) {
      if (pass == 1) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) bytes += __shfl_xor_sync(0xffffffffu, bytes, o);
        if (lane == 0) mbar_arrive_expect_tx(bar, bytes);
        __syncwarp();
      }
      for (int rr = lane; rr < PL::NROWS; rr += 32) {
        const int ly = (DIM > 1 ? rr % PL::BY : 0) - 1, lz = DIM > 2 ? rr / PL::BY - 1 : 0;
        const bool yout = ly < 0 || ly >= TY, zout = DIM > 2 && (lz < 0 || lz >= TZ);
        if (yout && zout) continue;
        const int gy = oy + ly, gz = oz + lz;
        if (gy < 0 || gy >= m.n[1] || (DIM > 2 && (gz < 0 || gz >= m.n[2]))) continue;
        const long long rowcell = (long long)m.n[0] * (gy + (long long)m.n[1] * (DIM > 2 ? gz : 0));
        const long long s0 = (rowcell + gx0) * NMB, s1 = (rowcell + gx1) * NMB;
        const long long a0 = s0 & ~15LL, a1 = (s1 + 15) & ~15LL;
        if (pass == 0) bytes += (unsigned)(a1 - a0);
        else bulk_g2s(boxb + (size_t)rr * PL::SLOT, gsrc + a0, (unsigned)(a1 - a0), bar);
      }
      for (int k = lane; k < DIM * DIM; k += 32) {
        const int d = k / DIM, e = k % DIM;
        const int o = e == 0 ? ox : (e == 1 ? oy : oz);
        const unsigned nbytes = (unsigned)(TL[e] * OPW * sizeof(T));
        if (pass == 0) bytes += nbytes;
        else bulk_g2s(const_cast<T*>(rowp(d, e, 0)), a.optab + ((size_t)(d * 3 + e) * a.nmax + o) * OPW, nbytes, bar);
      }
    }
  }
  if (!mbar_wait(bar, 0, 1 << 22)) {
    if (threadIdx.x == 0 && a.err) atomicOr(a.err, kErrCopyTimeout);
    mbar_wait(bar, 0, 1 << 22);   // give copies in flight a last chance to land
  }

  const T ct = a.clk ? T(a.clk->ct[a.stage]) : T(a.ct_explicit);
  const T dt = a.clk ? T(a.clk->dt) : T(a.dt_explicit);
  const bool active = a.clk ? (a.clk->active != 0) : true;
  const int cl = threadIdx.x;
  const T ih[3] = {T(1.0 / m.h[0]), T(1.0 / m.h[1]), T(DIM > 2 ? 1.0 / m.h[2] : 1.0)};
  const bool work = valid && active;
  constexpr int SL[3] = {PL::SL0, PL::SL1, PL::SL2};
  constexpr int FLO[3] = {0, NF * PL::SL0, NF * (PL::SL0 + PL::SL1)};

  // ===== (1) face fluxes, one work item per face of the tile.  The faces
  // normal to E form a block (TX + (E==0)) x (TY + (E==1)) x (TZ + (E==2))
  // in slot order, x fastest (consecutive lanes read consecutive cells of a
  // box row); the three blocks start on warp boundaries when their sizes are
  // multiples of 32, so a warp serves one axis
  auto face_item = [&](auto EC, int r) {
    constexpr int E = decltype(EC)::value;
    constexpr int t0 = E == 0 ? 1 : 0, t1 = E == 2 ? 1 : 2;
    constexpr int EX = TX + (E == 0), EY = TY + (E == 1);
    const int lx = r % EX, ly = (r / EX) % EY, lz = DIM > 2 ? r / (EX * EY) : 0;
    const int lc[3] = {lx, ly, lz};
    const int gc[3] = {ox + lx, oy + ly, oz + lz};
    if ((E != 0 && gc[0] >= m.n[0]) || (E != 1 && gc[1] >= m.n[1]) || (DIM > 2 && E != 2 && gc[2] >= m.n[2])) return;
    const int f = lc[E], gE = gc[E];
    const bool has_m = gE >= 1 && gE - 1 < m.n[E], has_p = gE < m.n[E];
    if (!has_m && !has_p) return;
    const T* cp = cellp(lx, ly, lz);
    const T* cm = cellp(lx - (E == 0), ly - (E == 1), lz - (E == 2));
    T gd = T(0);
    bool dir = false;
    if constexpr (BC) {
      if (!has_m) dir = bc_dirichlet<DIM>(m, E, 0, gc, gd);
      else if (!has_p) {
        const int gl[3] = {gc[0] - (E == 0), gc[1] - (E == 1), gc[2] - (E == 2)};
        dir = bc_dirichlet<DIM>(m, E, 1, gl, gd);
      }
    }
    // tangential operator rows and the normal factor g_EE at the face: the
    // upper cell's xi = 0 value where that cell is a tile cell of the mesh,
    // else the lower cell's xi = 1 value (the same number, tabulated from
    // one expression; rows past the mesh hold no face values)
    const T* r0 = rowp(E, t0, lc[t0]);
    const T* r1 = DIM > 2 ? rowp(E, t1, lc[t1]) : nullptr;
    const T fe = (f < TL[E] && has_p) ? rowp(E, E, f)[BOFF] : rowp(E, E, f - 1)[BOFF + 1];
    const T s1 = ct * fe;
    T F[NF];
    // tangential factors of one sign over the face: |u_E| = sigma u_E, so
    // the flux is u_E times the upwind trace alone
    const T sigma = DIM > 2 ? r0[N1 * N1] * r1[N1 * N1] : r0[N1 * N1];
    if (sigma != T(0)) {
      const bool flow_up = s1 * sigma > T(0);   // upwind: the lower cell
      T W[NF];
      if (dir && !(flow_up ? has_m : has_p)) {
#pragma unroll
        for (int mf = 0; mf < NF; ++mf) W[mf] = mf == 0 ? gd : T(0);
      } else {
        const bool up_m = flow_up ? has_m : !has_p;
        face_trace_ct<DIM, P, PB, E, T>(up_m ? cm : cp, up_m ? tb.L1 : tb.L0, W);
      }
      face_apply<DIM, N1, BOFF, T>(r0, r1, W, W, s1, T(0), false, F);
    } else {
      T S[NF], D[NF];   // traces Tm / Tp, then their mean / half jump in place
      if (has_m) face_trace_ct<DIM, P, PB, E, T>(cm, tb.L1, S);
      if (has_p) face_trace_ct<DIM, P, PB, E, T>(cp, tb.L0, D);
#pragma unroll
      for (int mf = 0; mf < NF; ++mf) {
        const T ghost = dir ? (mf == 0 ? gd : T(0)) : T(0);
        const T tm = has_m ? S[mf] : (dir ? ghost : D[mf]), tp = has_p ? D[mf] : (dir ? ghost : S[mf]);
        S[mf] = T(0.5) * (tm + tp);
        D[mf] = T(0.5) * (tm - tp);
      }
      face_apply<DIM, N1, BOFF, T>(r0, r1, S, D, s1, s1 < T(0) ? -s1 : s1, (has_m && has_p) || dir, F);
    }
    const int sl = lx + EX * (ly + EY * lz);
#pragma unroll
    for (int mf = 0; mf < NF; ++mf) fl[FLO[E] + mf * SL[E] + sl] = F[mf];
  };
  if (active) {
    constexpr int TOT = PL::SL0 + PL::SL1 + PL::SL2;
    for (int it = threadIdx.x; it < TOT; it += NT) {
      if (it < SL[0]) face_item(std::integral_constant<int, 0>(), it);
      else if (it < SL[0] + SL[1]) face_item(std::integral_constant<int, 1>(), it - SL[0]);
      else if constexpr (DIM > 2) face_item(std::integral_constant<int, 2>(), it - SL[0] - SL[1]);
    }
  }
  __syncthreads();

  // ===== (2) cell term and the lifting of the cell's face fluxes
  T R[NM];
#pragma unroll
  for (int q = 0; q < NM; ++q) R[q] = T(0);
  if (work) {
    // the cell's coefficients in registers (Q layout)
    T c[NM];
    {
      const T* cme = cellp(l[0], l[1], l[2]);
#pragma unroll
      for (int q = 0; q < NM; ++q) {
        if constexpr (PB) {
          const int gi = m.q2g[q];
          c[q] = gi >= 0 ? cme[gi] : T(0);
        } else {
          c[q] = cme[q];
        }
      }
    }
#pragma unroll 1
    for (int d = 0; d < DIM; ++d) {
      T M0[N1][N1], M1[N1][N1];
      load_op<N1, T>(rowp(d, 0, l[0]), M0);
      load_op<N1, T>(rowp(d, 1, l[1]), M1);
      const T ihd = d == 0 ? ih[0] : (d == 1 ? ih[1] : ih[2]);
      apply_sep_reg<DIM, P, T>(M0, M1, DIM > 2 ? rowp(d, 2, l[2]) : nullptr, c, R, ct * ihd);
    }
    auto lift = [&](auto EC) {
      constexpr int E = decltype(EC)::value;
      const int slo = l[0] + (TX + (E == 0)) * (l[1] + (TY + (E == 1)) * l[2]);
      const int sup = slo + (E == 0 ? 1 : (E == 1 ? TX : (TX * (TY + 0)) ));
      T F[NF];
#pragma unroll
      for (int mf = 0; mf < NF; ++mf) F[mf] = fl[FLO[E] + mf * SL[E] + slo];
      scatter_face<DIM, P, E, T>(R, tb.L0, F, ih[E]);
#pragma unroll
      for (int mf = 0; mf < NF; ++mf) F[mf] = fl[FLO[E] + mf * SL[E] + sup];
      scatter_face<DIM, P, E, T>(R, tb.L1, F, -ih[E]);
    };
    lift(std::integral_constant<int, 0>());
    lift(std::integral_constant<int, 1>());
    if constexpr (DIM == 3) lift(std::integral_constant<int, 2>());
  }
  __syncthreads();   // face fluxes consumed: the region now holds R [cell][NM]
  T* rbuf = fl;
  if (work) {
#pragma unroll
    for (int q = 0; q < NM; ++q) rbuf[(size_t)cl * NM + q] = R[q];
  }
  __syncthreads();

  // ---- RK combination fused into the coalesced store: one warp per row of
  // cells along x; stage input from the box, phi^n from HBM, all of a
  // lane's phi^n loads issued before the first use
  const bool need_n = a.combine == kRK2b || a.combine == kRK3b || a.combine == kRK3c;
  constexpr int NW = NT / 32, NROW = TY * TZ, ROWE = TX * NBG;
  constexpr int RPW = (NROW + NW - 1) / NW, KPR = (ROWE + 31) / 32;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nx = min(TX, m.n[0] - ox);
  // FP32 rows of whole tiles start on 16-byte boundaries in HBM, in the box
  // copy (same 16-byte phase) and in the R buffer when TX * NM and the row
  // pitch n[0] * NM are multiples of 4: float4 loads and stores
  constexpr bool VEC = !PB && sizeof(T) == 4 && (TX * NM) % 4 == 0;
  const bool vec_ok = VEC && nx == TX && ((long long)m.n[0] * NM) % 4 == 0 &&
                      ((reinterpret_cast<uintptr_t>(a.out) | reinterpret_cast<uintptr_t>(a.phi_n)) & 15) == 0;
  if (VEC && vec_ok) {
    constexpr int RV = TX * NM / 4, KV = (RV + 31) / 32;   // float4 per row, per lane
    constexpr int CV = RPW;                                 // rows with loads in flight together
#pragma unroll
    for (int j0 = 0; j0 < RPW; j0 += CV) {
      float4 pn[CV][KV];
#pragma unroll
      for (int jj = 0; jj < CV; ++jj) {
        const int r = warp + NW * (j0 + jj);
        const int ly = r % TY, lz = r / TY;
        const bool rok = j0 + jj < RPW && r < NROW && oy + ly < m.n[1] && (DIM < 3 || oz + lz < m.n[2]);
        const long long gbase =
            ((long long)m.n[0] * ((oy + ly) + (long long)m.n[1] * (DIM > 2 ? oz + lz : 0)) + ox) * NM;
        const float4* src = reinterpret_cast<const float4*>(a.phi_n + (rok ? gbase : 0));
#pragma unroll
        for (int k = 0; k < KV; ++k) {
          const int e = lane + 32 * k;
          pn[jj][k] = (need_n && active && rok && e < RV) ? __ldg(src + e) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
      }
#pragma unroll
      for (int jj = 0; jj < CV; ++jj) {
        const int r = warp + NW * (j0 + jj);
        const int ly = r % TY, lz = r / TY;
        if (!(j0 + jj < RPW && r < NROW && oy + ly < m.n[1] && (DIM < 3 || oz + lz < m.n[2]))) continue;
        const long long gbase =
            ((long long)m.n[0] * ((oy + ly) + (long long)m.n[1] * (DIM > 2 ? oz + lz : 0)) + ox) * NM;
        const float4* cs = reinterpret_cast<const float4*>(cellp(0, ly, lz));
        const float4* rs = reinterpret_cast<const float4*>(rbuf + (size_t)TX * r * NM);
        float4* dst = reinterpret_cast<float4*>(a.out + gbase);
#pragma unroll
        for (int k = 0; k < KV; ++k) {
          const int e = lane + 32 * k;
          if (e >= RV) continue;
          const float4 cv = cs[e];
          float4 o = cv;
          if (active) {
            const float4 rv = rs[e], nv = pn[jj][k];
            o.x = combine_value<float>(a.combine, cv.x, nv.x, rv.x, (float)dt);
            o.y = combine_value<float>(a.combine, cv.y, nv.y, rv.y, (float)dt);
            o.z = combine_value<float>(a.combine, cv.z, nv.z, rv.z, (float)dt);
            o.w = combine_value<float>(a.combine, cv.w, nv.w, rv.w, (float)dt);
          }
          dst[e] = o;
        }
      }
    }
  } else if constexpr (!PB) {
    // rows in chunks of CH, a chunk's phi^n loads all in flight together
    constexpr int CH = RPW * KPR > 16 ? (RPW > 2 ? 2 : RPW) : RPW;
#pragma unroll
    for (int j0 = 0; j0 < RPW; j0 += CH) {
      T pn[CH][KPR];
#pragma unroll
      for (int jj = 0; jj < CH; ++jj) {
        const int r = warp + NW * (j0 + jj);
        const int ly = r % TY, lz = r / TY;
        const bool rok = j0 + jj < RPW && r < NROW && oy + ly < m.n[1] && (DIM < 3 || oz + lz < m.n[2]);
        const long long gbase =
            ((long long)m.n[0] * ((oy + ly) + (long long)m.n[1] * (DIM > 2 ? oz + lz : 0)) + ox) * NM;
#pragma unroll
        for (int k = 0; k < KPR; ++k) {
          const int e = lane + 32 * k;
          pn[jj][k] = (need_n && active && rok && e < nx * NM) ? __ldg(a.phi_n + gbase + e) : T(0);
        }
      }
#pragma unroll
      for (int jj = 0; jj < CH; ++jj) {
        const int r = warp + NW * (j0 + jj);
        const int ly = r % TY, lz = r / TY;
        if (!(j0 + jj < RPW && r < NROW && oy + ly < m.n[1] && (DIM < 3 || oz + lz < m.n[2]))) continue;
        const long long gbase =
            ((long long)m.n[0] * ((oy + ly) + (long long)m.n[1] * (DIM > 2 ? oz + lz : 0)) + ox) * NM;
        const T* cs = cellp(0, ly, lz);
        const T* rs = rbuf + (size_t)TX * r * NM;
#pragma unroll
        for (int k = 0; k < KPR; ++k) {
          const int e = lane + 32 * k;
          if (e >= nx * NM) continue;
          const T cv = cs[e];
          a.out[gbase + e] = active ? combine_value<T>(a.combine, cv, pn[jj][k], rs[e], dt) : cv;
        }
      }
    }
  } else {
    for (int r = warp; r < NROW; r += NW) {
      const int ly = r % TY, lz = r / TY;
      const int gy = oy + ly, gz = oz + lz;
      if (gy >= m.n[1] || (DIM > 2 && gz >= m.n[2]) || nx <= 0) continue;
      const long long gbase = ((long long)m.n[0] * (gy + (long long)m.n[1] * (DIM > 2 ? gz : 0)) + ox) * NBG;
      const T* cs = cellp(0, ly, lz);
      const T* rs = rbuf + (size_t)TX * r * NM;
      for (int e = lane; e < nx * NBG; e += 32) {
        const int cx = e / NBG, kk = e - cx * NBG;
        const int q = cx * NM + m.g2q[kk];
        const T cv = cs[e];
        T res = cv;
        if (active) {
          const T pnv = need_n ? __ldg(a.phi_n + gbase + e) : T(0);
          res = combine_value<T>(a.combine, cv, pnv, rs[q], dt);
        }
        a.out[gbase + e] = res;
      }
    }
  }
}

}  // namespace flsp

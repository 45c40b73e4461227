// flsp_hjs.cuh — Hamilton-Jacobi reinitialisation pseudo-step, tensor-
// product (FE_DGQLegendre) basis, with the work of a cell split over its
// Gauss planes.
//
// Same operator and operation order as hjq_tile (flsp_hjq.cuh; the
// reference functions it replaces are listed in flsp_hj.cuh), restated for
// throughput:
//  * the smooth sign S(phi0) (src/level_set/reinit.cc:121-133) depends on
//    phi0 alone, which stays fixed through a reinitialisation sweep.  The
//    sweep's first launch (mode kHJCflOnly, phi == phi0) evaluates it at the
//    cell Gauss points and at the CFL vertices into a per-tile table; every
//    pseudo-step reads it from there instead of evaluating phi0 and its
//    gradient again (the same expression on the same inputs);
//  * NQ threads per cell: thread k of a cell owns the Gauss plane k of the
//    last axis (z in 3D, y in 2D).  Its partial projection onto the modes
//    goes through shared memory, and each thread finishes every NQ-th mode
//    of the cell (the sums over planes keep their order);
//  * the face jumps are formed once per face, not once per cell side.
//
// Table layout: stab[(tile * NS + j) * nt + c], c the cell within the tile;
// j < NQ^dim: the Gauss point qx + NQ (qy + NQ qz), holding w_q S (the
// quadrature weight folded in: w_q H = H with S replaced by w_q S, as
// w_q > 0); j = NQ^dim + v: S at the vertex v (x bit 0, y bit 1, z bit 2).  Tiles are the launch's tiles (the
// narrow band selects among them; the tile index is the global one).
#pragma once
#include "flsp_device.cuh"
#include "flsp_hj.cuh"

namespace flsp {

// the kernel's tile (cells), fixed per dimension so that every shared-
// memory and table offset is a compile-time constant; a multiple of 32
// cells keeps each warp on one Gauss plane
template <int DIM>
struct HjsTile {
  static constexpr int X = DIM == 2 ? 8 : 4, Y = DIM == 2 ? 8 : 4, Z = DIM == 2 ? 1 : 4;
  static constexpr int N = X * Y * Z;
};

// table entries per cell
template <int DIM, int P>
__host__ __device__ constexpr int hjs_ns() {
  return ipow(P + 2, DIM) + (1 << DIM);
}

// shared-memory plan: the halo box as rows of cells along x, each row a
// bulk copy from a 16-byte aligned global address (the row's data starts at
// its slot + the address phase), then the face jumps, the corner jumps,
// the plane projections and the block reduction
template <int DIM, int P, typename T>
struct HjsPlan {
  using TL = HjsTile<DIM>;
  static constexpr int N1 = P + 1, NQ = P + 2, NM = ipow(N1, DIM), NQF = ipow(NQ, DIM - 1);
  static constexpr int NC = 1 << (DIM - 1), NU = ipow(N1, DIM - 1);
  static constexpr int BY = TL::Y + 2, BZ = DIM > 2 ? TL::Z + 2 : 1, NROWS = BY * BZ;
  static constexpr int NMB = NM * (int)sizeof(T);   // bytes per cell
  static constexpr int SLOT = (((TL::X + 2) * NMB + 30) + 15) / 16 * 16;
  static constexpr size_t OFF_BOX = 16;
  static constexpr size_t OFF_JN = OFF_BOX + (size_t)NROWS * SLOT;
  static constexpr size_t OFF_JV = OFF_JN + (size_t)2 * DIM * NQF * TL::N * sizeof(T);
  // the tile's slice of the sign table (pseudo-steps: staged with the box),
  // then, once every thread has read its entries, the plane projections
  static constexpr int NS = ipow(NQ, DIM) + (1 << DIM);
  static constexpr size_t TAB_BYTES = (size_t)NS * TL::N * sizeof(T);
  static constexpr size_t UB_BYTES = (size_t)NQ * NU * TL::N * sizeof(T);
  static constexpr size_t OFF_UB = (OFF_JV + (size_t)2 * DIM * NC * TL::N * sizeof(T) + 15) / 16 * 16;
  static constexpr size_t OFF_RED = (OFF_UB + (TAB_BYTES > UB_BYTES ? TAB_BYTES : UB_BYTES) + 15) / 16 * 16;
  static constexpr size_t BYTES = OFF_RED + 64 * sizeof(double);
};

template <int DIM, int P, typename T>
__host__ __device__ inline size_t hjs_smem_bytes(const int*) {
  return HjsPlan<DIM, P, T>::BYTES;
}

// smooth sign from phi0's value and (scaled) gradient at a point, with the
// pseudo-step kernels' operation sequence
template <typename T>
__device__ __forceinline__ T hjs_sign(T p0, T g2, T hmin) {
  if constexpr (sizeof(T) == 4) {
    return p0 * rsqrtf(p0 * p0 + hmin * hmin * g2);
  } else {
    const T gn = sqrt(g2);
    return p0 / sqrt(p0 * p0 + hmin * hmin * gn * gn);
  }
}

// the jump phi_upper - phi_lower on the faces normal to E (one face per
// call, lower cell at local lc with lc[E] = f - 1), times 1/h_E, written
// nodal at the face Gauss points and at the face corners for both adjacent
// tile cells
template <int DIM, int P, int E, typename T, typename CellP>
__device__ __forceinline__ void hjs_face(const MeshArgs& m, const CellP& cellp, T* jn, T* jv, const int* o,
                                         int r) {
  constexpr int N1 = P + 1, NQ = P + 2, NF = ipow(N1, DIM - 1), NQF = ipow(NQ, DIM - 1), NC = 1 << (DIM - 1);
  constexpr int t0 = E == 0 ? 1 : 0, t1 = E == 2 ? 1 : 2;
  constexpr int st[3] = {1, N1, N1 * N1};
  const Tab1D<T>& tb = tab<T>(P);
  using TL = HjsTile<DIM>;
  constexpr int nt = TL::N, tl[3] = {TL::X, TL::Y, TL::Z};
  const int f = r % (tl[E] + 1);
  const int rest = r / (tl[E] + 1);
  int lu[3];
  lu[E] = f;
  lu[t0] = rest % tl[t0];
  lu[t1] = DIM > 2 ? rest / tl[t0] : 0;
  if (o[t0] + lu[t0] >= m.n[t0] || (DIM > 2 && o[t1] + lu[t1] >= m.n[t1])) return;
  int ll[3] = {lu[0], lu[1], lu[2]};
  ll[E] = f - 1;
  const bool inside = o[E] + f - 1 >= 0 && o[E] + f < m.n[E];
  T J[NF];
  // a domain-boundary face with a Dirichlet value: the missing side's trace
  // is that constant (LDG left / right boundary terms, ldg.cc:551-620,
  // :686-740); without one the jump is zero (interior trace)
  T gd = T(0);
  bool dir = false;
  if (!inside && (o[E] + f == 0 || o[E] + f == m.n[E])) {
    int gcell[3] = {o[0] + lu[0], o[1] + lu[1], o[2] + lu[2]};
    gcell[E] = o[E] + f == 0 ? 0 : m.n[E] - 1;
    dir = bc_dirichlet<DIM>(m, E, o[E] + f == 0 ? 0 : 1, gcell, gd);
  }
  if (dir) {
    const bool lower = o[E] + f == 0;   // the domain's lower side: the cell is above the face
    const T* cc = lower ? cellp(lu[0], lu[1], lu[2]) : cellp(ll[0], ll[1], ll[2]);
#pragma unroll
    for (int mf = 0; mf < NF; ++mf) {
      const int m0 = mf % N1, m1 = mf / N1;
      const int base = m0 * st[t0] + (DIM > 2 ? m1 * st[t1] : 0);
      T tr = T(0);
#pragma unroll
      for (int b = 0; b < N1; ++b) tr += (lower ? tb.L0[b] : tb.L1[b]) * cc[base + b * st[E]];
      const T ghost = mf == 0 ? gd : T(0);
      J[mf] = lower ? tr - ghost : ghost - tr;
    }
  } else if (inside) {
    const T* cu = cellp(lu[0], lu[1], lu[2]);
    const T* cd = cellp(ll[0], ll[1], ll[2]);
#pragma unroll
    for (int mf = 0; mf < NF; ++mf) {
      const int m0 = mf % N1, m1 = mf / N1;
      const int base = m0 * st[t0] + (DIM > 2 ? m1 * st[t1] : 0);
      T tup = T(0), tdn = T(0);
#pragma unroll
      for (int b = 0; b < N1; ++b) {
        tup += tb.L0[b] * cu[base + b * st[E]];
        tdn += tb.L1[b] * cd[base + b * st[E]];
      }
      J[mf] = tup - tdn;
    }
  } else {
#pragma unroll
    for (int mf = 0; mf < NF; ++mf) J[mf] = T(0);
  }
  // the upper cell sees this face as its lower side (slot 2E), the lower
  // cell as its upper side (slot 2E + 1)
  const int cu_l = f < tl[E] ? lu[0] + tl[0] * (lu[1] + tl[1] * lu[2]) : -1;
  const int cd_l = f >= 1 ? ll[0] + tl[0] * (ll[1] + tl[1] * ll[2]) : -1;
  const T ihE = T(1.0 / m.h[E]);
  auto put = [&](int q, T v, bool corner) {
    const int base = corner ? 2 * E * NC : 2 * E * NQF, stride = corner ? NC : NQF;
    T* dst = corner ? jv : jn;
    v *= ihE;
    if (cu_l >= 0) dst[(size_t)(base + q) * nt + cu_l] = v;
    if (cd_l >= 0) dst[(size_t)(base + stride + q) * nt + cd_l] = v;
  };
  if constexpr (DIM == 2) {
#pragma unroll
    for (int q0 = 0; q0 < NQ; ++q0) {
      T s = T(0);
#pragma unroll
      for (int m0 = 0; m0 < N1; ++m0) s += J[m0] * tb.Lq[m0][q0];
      put(q0, s, false);
    }
#pragma unroll
    for (int cr = 0; cr < 2; ++cr) {
      T s = T(0);
#pragma unroll
      for (int m0 = 0; m0 < N1; ++m0) s += J[m0] * (cr ? tb.L1[m0] : tb.L0[m0]);
      put(cr, s, true);
    }
  } else {
    T Pq[NQ][N1];
#pragma unroll
    for (int q0 = 0; q0 < NQ; ++q0)
#pragma unroll
      for (int m1 = 0; m1 < N1; ++m1) {
        T s = T(0);
#pragma unroll
        for (int m0 = 0; m0 < N1; ++m0) s += J[m0 + N1 * m1] * tb.Lq[m0][q0];
        Pq[q0][m1] = s;
      }
#pragma unroll
    for (int q1 = 0; q1 < NQ; ++q1)
#pragma unroll
      for (int q0 = 0; q0 < NQ; ++q0) {
        T s = T(0);
#pragma unroll
        for (int m1 = 0; m1 < N1; ++m1) s += Pq[q0][m1] * tb.Lq[m1][q1];
        put(q0 + NQ * q1, s, false);
      }
#pragma unroll
    for (int cr = 0; cr < 4; ++cr) {
      T s = T(0);
#pragma unroll
      for (int mf = 0; mf < NF; ++mf) {
        const int m0 = mf % N1, m1 = mf / N1;
        s += J[mf] * ((cr & 1) ? tb.L1[m0] : tb.L0[m0]) * ((cr & 2) ? tb.L1[m1] : tb.L0[m1]);
      }
      put(cr, s, true);
    }
  }
}

// values and gradients (reference-cell derivatives) of the modal field c
// at the two vertices (vx = 0, 1) of the x-line with corner bits (vy, vz):
// the y/z reductions are shared by both ends of the line
template <int DIM, int N1, typename T>
__device__ __forceinline__ void hjs_line(const T* c, const Tab1D<T>& tb, int vy, int vz, T* val, T (*gr)[3]) {
  T Y[N1], Yd[N1];
#pragma unroll
  for (int b = 0; b < N1; ++b) {
    Y[b] = vy ? tb.L1[b] : tb.L0[b];
    Yd[b] = vy ? tb.D1[b] : tb.D0[b];
  }
  T V[N1], Vy[N1], Vz[N1];
  if constexpr (DIM == 2) {
#pragma unroll
    for (int a = 0; a < N1; ++a) {
      T s0 = T(0), s1 = T(0);
#pragma unroll
      for (int b = 0; b < N1; ++b) {
        s0 += c[a + N1 * b] * Y[b];
        s1 += c[a + N1 * b] * Yd[b];
      }
      V[a] = s0;
      Vy[a] = s1;
      Vz[a] = T(0);
    }
  } else {
    T Z[N1], Zd[N1];
#pragma unroll
    for (int b = 0; b < N1; ++b) {
      Z[b] = vz ? tb.L1[b] : tb.L0[b];
      Zd[b] = vz ? tb.D1[b] : tb.D0[b];
    }
#pragma unroll
    for (int a = 0; a < N1; ++a) {
      T W[N1], Wd[N1];
#pragma unroll
      for (int b = 0; b < N1; ++b) {
        T s0 = T(0), s1 = T(0);
#pragma unroll
        for (int cc = 0; cc < N1; ++cc) {
          s0 += c[a + N1 * (b + N1 * cc)] * Z[cc];
          s1 += c[a + N1 * (b + N1 * cc)] * Zd[cc];
        }
        W[b] = s0;
        Wd[b] = s1;
      }
      T s0 = T(0), s1 = T(0), s2 = T(0);
#pragma unroll
      for (int b = 0; b < N1; ++b) {
        s0 += W[b] * Y[b];
        s1 += W[b] * Yd[b];
        s2 += Wd[b] * Y[b];
      }
      V[a] = s0;
      Vy[a] = s1;
      Vz[a] = s2;
    }
  }
#pragma unroll
  for (int vx = 0; vx < 2; ++vx) {
    const T* X = vx ? tb.L1 : tb.L0;
    const T* Xd = vx ? tb.D1 : tb.D0;
    T v = T(0), gx = T(0), gy = T(0), gz = T(0);
#pragma unroll
    for (int a = 0; a < N1; ++a) {
      v += V[a] * X[a];
      gx += V[a] * Xd[a];
      gy += Vy[a] * X[a];
      gz += Vz[a] * X[a];
    }
    val[vx] = v;
    gr[vx][0] = gx;
    gr[vx][1] = gy;
    gr[vx][2] = gz;
  }
}

// One block serves one HjsTile of cells (launch slot blockIdx.x) with NQ
// threads per cell (blockDim = cells * NQ); its halo box arrives by bulk
// copies on one mbarrier.  Modes: kHJCflOnly (phi == phi0: fills the sign
// table, CFL estimate of the first pseudo-step) and kHJStep (one pseudo-
// step from the table, CFL estimate of the next).
template <int DIM, int P, typename T>
__global__ void __launch_bounds__(HjsTile<DIM>::N * (P + 2)) hjs_kernel(const HJArgs<T> a) {
  using PL = HjsPlan<DIM, P, T>;
  constexpr int N1 = P + 1, NQ = P + 2, NM = ipow(N1, DIM), NV = 1 << DIM;
  constexpr int NQF = ipow(NQ, DIM - 1), NC = 1 << (DIM - 1);
  constexpr int NU = ipow(N1, DIM - 1), NQV = ipow(NQ, DIM), NS = NQV + NV;
  using TL = HjsTile<DIM>;
  constexpr int TX = TL::X, TY = TL::Y, TZ = TL::Z, NT = TL::N, NMB = PL::NMB;
  static_assert(NM <= 2 * DIM * NQF, "the store staging reuses the face-jump area");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(smem_raw);
  unsigned char* boxb = smem_raw + PL::OFF_BOX;
  T* jn = reinterpret_cast<T*>(smem_raw + PL::OFF_JN);   // [2*DIM*NQF][NT]
  T* jv = reinterpret_cast<T*>(smem_raw + PL::OFF_JV);   // [2*DIM*NC][NT]
  T* ub = reinterpret_cast<T*>(smem_raw + PL::OFF_UB);   // [NQ][NU][NT], after the table slice
  T* stl = ub;                                            // table slice [NS][NT] (pseudo-steps)
  double* red = reinterpret_cast<double*>(smem_raw + PL::OFF_RED);
  const MeshArgs& m = a.m;
  const Tab1D<T>& tb = tab<T>(P);
  const int slot = (int)blockIdx.x;
  if (tile_inactive(m, slot)) return;

  auto origin = [&](int slot, int* o) {
    int b = m.tiles ? m.tiles[slot] : slot;
    o[0] = (b % m.ntile[0]) * TX;
    b /= m.ntile[0];
    o[1] = DIM > 1 ? (b % m.ntile[1]) * TY : 0;
    o[2] = DIM > 2 ? (b / m.ntile[1]) * TZ : 0;
  };
  const bool step = a.mode == kHJStep;
  // halo box of the tile in launch slot `slot`: rows (ly, lz) of cells
  // [max(ox - 1, 0), min(ox + TX + 1, n)) by bulk copies (warp 0); for a
  // pseudo-step also the tile's slice of the sign table (one copy)
  auto issue = [&](int slot) {
    int so[3];
    origin(slot, so);
    const int hx0 = max(so[0] - 1, 0), hx1 = min(so[0] + TX + 1, m.n[0]);
    const int lane = threadIdx.x;
    const char* gsrc = reinterpret_cast<const char*>(a.phi);
    unsigned bytes = 0;
    // pass 0 counts the bytes, pass 1 issues the copies
    for (int pass = 0; pass < 2; ++pass) {
      if (pass == 1) {
#pragma unroll
        for (int w = 16; w > 0; w >>= 1) bytes += __shfl_xor_sync(0xffffffffu, bytes, w);
        if (lane == 0) mbar_arrive_expect_tx(bar, bytes);
        __syncwarp();
      }
      for (int rr = lane; rr < PL::NROWS; rr += 32) {
        const int ly = rr % PL::BY - 1, lz = DIM > 2 ? rr / PL::BY - 1 : 0;
        const bool yout = ly < 0 || ly >= TY, zout = DIM > 2 && (lz < 0 || lz >= TZ);
        if (yout && zout) continue;
        const int gy = so[1] + ly, gz = so[2] + lz;
        if (gy < 0 || gy >= m.n[1] || (DIM > 2 && (gz < 0 || gz >= m.n[2]))) continue;
        const long long rowcell = (long long)m.n[0] * (gy + (long long)m.n[1] * (DIM > 2 ? gz : 0));
        const long long s0 = (rowcell + hx0) * NMB, s1 = (rowcell + hx1) * NMB;
        const long long a0 = s0 & ~15LL, a1 = (s1 + 15) & ~15LL;
        if (pass == 0) bytes += (unsigned)(a1 - a0);
        else bulk_g2s(boxb + (size_t)rr * PL::SLOT, gsrc + a0, (unsigned)(a1 - a0), bar);
      }
      if (step && lane == 0) {
        const int tl = m.tiles ? m.tiles[slot] : slot;
        if (pass == 0) bytes += (unsigned)PL::TAB_BYTES;
        else bulk_g2s(stl, a.stab + (size_t)tl * NS * NT, (unsigned)PL::TAB_BYTES, bar);
      }
    }
  };

  const int cl = (int)threadIdx.x % NT, k = (int)threadIdx.x / NT;   // cell, Gauss plane
  const int l[3] = {cl % TX, (cl / TX) % TY, DIM > 2 ? cl / (TX * TY) : 0};
  const T ih[3] = {T(1.0 / m.h[0]), T(1.0 / m.h[1]), T(DIM > 2 ? 1.0 / m.h[2] : 1.0)};
  const T hmin = T(m.min_diam);
  const bool fill = a.mode == kHJCflOnly;
  // this thread's Gauss plane (uniform per warp): its 1D table entries
  T Lk[N1], Dk[N1];
#pragma unroll
  for (int b = 0; b < N1; ++b) {
    Lk[b] = tb.Lq[b][k];
    Dk[b] = tb.Dq[b][k];
  }
  const T dt = a.clk ? T(a.clk->hj_dt) : T(a.dt_explicit);
  double vmax = 0.0;

  if (threadIdx.x == 0) mbar_init(bar, 1);
  __syncthreads();
  if (threadIdx.x < 32) issue(slot);

  int o[3];
  origin(slot, o);
  const int tile = m.tiles ? m.tiles[slot] : slot;
  const int g[3] = {o[0] + l[0], o[1] + l[1], o[2] + l[2]};
  const bool valid = g[0] < m.n[0] && g[1] < m.n[1] && (DIM < 3 || g[2] < m.n[2]);
  const int gx0 = max(o[0] - 1, 0);
  // box copy of the cell at local coordinates (lx, ly, lz)
  auto cellp = [&](int lx, int ly, int lz) -> const T* {
    const int rr = (ly + 1) + PL::BY * (DIM > 2 ? lz + 1 : 0);
    const unsigned rowcell = (unsigned)m.n[0] * (unsigned)((o[1] + ly) + m.n[1] * (DIM > 2 ? o[2] + lz : 0));
    const unsigned phase = ((rowcell + (unsigned)gx0) * (unsigned)NMB) & 15u;
    return reinterpret_cast<const T*>(boxb + (size_t)rr * PL::SLOT + phase + (o[0] + lx - gx0) * NMB);
  };
  if (!mbar_wait(bar, 0u, 1 << 22)) {
    if (threadIdx.x == 0 && a.err) atomicOr(a.err, kErrCopyTimeout);
  }

  // -------- face jumps, one work item per face of the tile
  {
    constexpr int C0 = (TX + 1) * (NT / TX), C1 = (TY + 1) * (NT / TY);
    constexpr int C2 = DIM > 2 ? (TZ + 1) * (NT / TZ) : 0;
    for (int i = threadIdx.x; i < C0 + C1 + C2; i += NT * NQ) {
      if (i < C0) hjs_face<DIM, P, 0, T>(m, cellp, jn, jv, o, i);
      else if (i < C0 + C1) hjs_face<DIM, P, 1, T>(m, cellp, jn, jv, o, i - C0);
      else if constexpr (DIM > 2) hjs_face<DIM, P, 2, T>(m, cellp, jn, jv, o, i - C0 - C1);
    }
  }
  __syncthreads();

  T* srow = a.stab + (size_t)tile * NS * NT + cl;   // this cell's table column, stride NT
  // the cell's modes projected on this thread's Gauss plane of the last
  // axis: value (PL0) and derivative (PL1) tables, in the modes of the others
  T PL0[NU], PL1[NU];
  const T* c = cellp(l[0], l[1], l[2]);   // the cell's modes (box copy)
  if (valid) {
    T cr[NM];
#pragma unroll
    for (int q = 0; q < NM; ++q) cr[q] = c[q];
    // -------- sign table of this cell's Gauss plane (phi == phi0)
    if (fill) {
      if constexpr (DIM == 2) {
        T P0y[N1], P0dy[N1];
#pragma unroll
        for (int aa = 0; aa < N1; ++aa) {
          T s3 = T(0), s4 = T(0);
#pragma unroll
          for (int b = 0; b < N1; ++b) {
            const T c0v = cr[aa + N1 * b];
            s3 += c0v * Lk[b];
            s4 += c0v * Dk[b];
          }
          P0y[aa] = s3;
          P0dy[aa] = s4;
        }
#pragma unroll
        for (int qx = 0; qx < NQ; ++qx) {
          T p0 = T(0), g0x = T(0), g0y = T(0);
#pragma unroll
          for (int aa = 0; aa < N1; ++aa) {
            p0 += P0y[aa] * tb.Lq[aa][qx];
            g0x += P0y[aa] * tb.Dq[aa][qx];
            g0y += P0dy[aa] * tb.Lq[aa][qx];
          }
          g0x *= ih[0];
          g0y *= ih[1];
          const T g2 = g0x * g0x + g0y * g0y;
          srow[(size_t)(k * NQF + qx) * NT] = tb.wq[qx] * tb.wq[k] * hjs_sign<T>(p0, g2, hmin);
        }
      } else {
        T P0z[N1][N1], D0z[N1][N1];
#pragma unroll
        for (int aa = 0; aa < N1; ++aa)
#pragma unroll
          for (int b = 0; b < N1; ++b) {
            T s3 = T(0), s4 = T(0);
#pragma unroll
            for (int cc = 0; cc < N1; ++cc) {
              const T c0v = cr[aa + N1 * (b + N1 * cc)];
              s3 += c0v * Lk[cc];
              s4 += c0v * Dk[cc];
            }
            P0z[aa][b] = s3;
            D0z[aa][b] = s4;
          }
#pragma unroll
        for (int qy = 0; qy < NQ; ++qy) {
          T P0y[N1], P0dy[N1], D0zy[N1];
#pragma unroll
          for (int aa = 0; aa < N1; ++aa) {
            T s4 = T(0), s5 = T(0), s6 = T(0);
#pragma unroll
            for (int b = 0; b < N1; ++b) {
              s4 += P0z[aa][b] * tb.Lq[b][qy];
              s5 += P0z[aa][b] * tb.Dq[b][qy];
              s6 += D0z[aa][b] * tb.Lq[b][qy];
            }
            P0y[aa] = s4;
            P0dy[aa] = s5;
            D0zy[aa] = s6;
          }
#pragma unroll
          for (int qx = 0; qx < NQ; ++qx) {
            T p0 = T(0), g0x = T(0), g0y = T(0), g0z = T(0);
#pragma unroll
            for (int aa = 0; aa < N1; ++aa) {
              p0 += P0y[aa] * tb.Lq[aa][qx];
              g0x += P0y[aa] * tb.Dq[aa][qx];
              g0y += P0dy[aa] * tb.Lq[aa][qx];
              g0z += D0zy[aa] * tb.Lq[aa][qx];
            }
            g0x *= ih[0];
            g0y *= ih[1];
            g0z *= ih[2];
            T g2 = g0x * g0x + g0y * g0y;
            g2 += g0z * g0z;
            srow[(size_t)(k * NQF + qx + NQ * qy) * NT] =
                tb.wq[qx] * tb.wq[qy] * tb.wq[k] * hjs_sign<T>(p0, g2, hmin);
          }
        }
      }
    }

    // -------- vertex CFL estimate for the next pseudo-step: x-lines of
    // vertices ln = k, k + NQ, ... (corner bits vy = ln & 1, vz = ln >> 1)
#pragma unroll 1
    for (int ln = k; ln < NV / 2; ln += NQ) {
      T vals[2], grs[2][3];
      hjs_line<DIM, N1, T>(cr, tb, ln & 1, ln >> 1, vals, grs);
#pragma unroll
      for (int vx = 0; vx < 2; ++vx) {
      const int v = vx + 2 * ln;
      const int vb[3] = {vx, ln & 1, ln >> 1};
      const T val = vals[vx];
      const T* dphi = grs[vx];
      T S;
      if (fill) {
        T g2 = T(0);
#pragma unroll
        for (int d = 0; d < DIM; ++d) { const T gg = dphi[d] * ih[d]; g2 += gg * gg; }
        const T gn = sqrt(g2);
        S = val / sqrt(val * val + hmin * hmin * gn * gn);
        srow[(size_t)(NQV + v) * NT] = S;
      } else {
        S = stl[(size_t)(NQV + v) * NT + cl];
      }
      T gs[DIM];
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        const int t0 = d == 0 ? 1 : 0, t1 = d == 2 ? 1 : 2;
        const int cr = vb[t0] + (DIM > 2 ? 2 * vb[t1] : 0);
        const T gd = dphi[d] * ih[d];
        const T L = gd + tb.K0v[vb[d]] * jv[(size_t)(2 * d * NC + cr) * NT + cl];
        const T Rr = gd + tb.K1v[vb[d]] * jv[(size_t)((2 * d + 1) * NC + cr) * NT + cl];
        if (S >= T(0)) {
          const T lp = max(L, T(0)), rm = -min(Rr, T(0));
          gs[d] = fabs(lp) > fabs(rm) ? lp : rm;
        } else {
          const T lm = -min(L, T(0)), rp = max(Rr, T(0));
          gs[d] = fabs(lm) > fabs(rp) ? lm : rp;
        }
      }
      T n2 = T(0);
#pragma unroll
      for (int d = 0; d < DIM; ++d) n2 += gs[d] * gs[d];
      const T nrm = sqrt(n2);
      if (!(fabs((double)nrm) <= 2.220446049250313e-16)) {
        const T inv = T(1) / nrm;
#pragma unroll
        for (int d = 0; d < DIM; ++d) gs[d] *= inv;
#pragma unroll
        for (int d = 0; d < DIM; ++d) gs[d] *= S;
      }
      T s2 = T(0);
#pragma unroll
      for (int d = 0; d < DIM; ++d) s2 += gs[d] * gs[d];
      vmax = fmax(vmax, (double)sqrt(s2));
      }
    }
    if (!fill) {
#pragma unroll
      for (int u = 0; u < NU; ++u) {
        T s1 = T(0), s2 = T(0);
#pragma unroll
        for (int cc = 0; cc < N1; ++cc) {
          const T cv = cr[u + NU * cc];
          s1 += cv * Lk[cc];
          s2 += cv * Dk[cc];
        }
        PL0[u] = s1;
        PL1[u] = s2;
      }
    }
  }
  vmax = vmax / m.diam;
  const double bm = block_max(vmax, red);
  if (threadIdx.x == 0 && a.clk) atomic_max_pos(&a.clk->hj_vd_bits, bm);
  if (a.mode != kHJStep) return;

  // -------- pseudo-step: H at this plane's Gauss points, projected onto
  // the modes of the other axes
  auto jnv = [&](int d, int side, int qf) -> T { return jn[(size_t)((2 * d + side) * NQF + qf) * NT + cl]; };
  auto hfun = [&](T S, const T* lft, const T* rgt) -> T {
    T avg2 = T(0);
#pragma unroll
    for (int d = 0; d < DIM; ++d) { const T av = T(0.5) * (lft[d] + rgt[d]); avg2 += av * av; }
    T nrm;
    if constexpr (sizeof(T) == 4) nrm = avg2 * rsqrtf(fmaxf(avg2, 1e-30f));
    else nrm = sqrt(avg2);
    T H = S * (nrm - T(1));
#pragma unroll
    for (int d = 0; d < DIM; ++d) H += T(0.5) * fabs(S) * (lft[d] - rgt[d]);
    return H;
  };
  T Sq[NQF];
  if (valid) {
#pragma unroll
    for (int j = 0; j < NQF; ++j) Sq[j] = stl[(size_t)(k * NQF + j) * NT + cl];
  }
  __syncthreads();   // the table slice is consumed: its region takes the plane projections
  if (valid) {
    const T K0k = tb.K0q[k], K1k = tb.K1q[k];
    if constexpr (DIM == 2) {
      const int qy = k;
      const T* Py = PL0;
      const T* Pdy = PL1;
      const T jlx = jnv(0, 0, qy), jhx = jnv(0, 1, qy);
      T X[N1];
#pragma unroll
      for (int aa = 0; aa < N1; ++aa) X[aa] = T(0);
#pragma unroll
      for (int qx = 0; qx < NQ; ++qx) {
        T gx = T(0), gy = T(0);
#pragma unroll
        for (int aa = 0; aa < N1; ++aa) {
          gx += Py[aa] * tb.Dq[aa][qx];
          gy += Pdy[aa] * tb.Lq[aa][qx];
        }
        gx *= ih[0];
        gy *= ih[1];
        const T jly = jnv(1, 0, qx), jhy = jnv(1, 1, qx);
        const T lft[2] = {gx + tb.K0q[qx] * jlx, gy + K0k * jly};
        const T rgt[2] = {gx + tb.K1q[qx] * jhx, gy + K1k * jhy};
        const T wH = hfun(Sq[qx], lft, rgt);   // weighted sign: w_q H
#pragma unroll
        for (int aa = 0; aa < N1; ++aa) X[aa] += wH * tb.Lq[aa][qx];
      }
#pragma unroll
      for (int aa = 0; aa < N1; ++aa) ub[(size_t)(k * NU + aa) * NT + cl] = X[aa];
    } else {
      T U[N1][N1];
#pragma unroll
      for (int aa = 0; aa < N1; ++aa)
#pragma unroll
        for (int b = 0; b < N1; ++b) U[aa][b] = T(0);
#pragma unroll
      for (int qy = 0; qy < NQ; ++qy) {
        T Py[N1], Pdy[N1], Dzy[N1];
#pragma unroll
        for (int aa = 0; aa < N1; ++aa) {
          T s1 = T(0), s2 = T(0), s3 = T(0);
#pragma unroll
          for (int b = 0; b < N1; ++b) {
            s1 += PL0[aa + N1 * b] * tb.Lq[b][qy];
            s2 += PL0[aa + N1 * b] * tb.Dq[b][qy];
            s3 += PL1[aa + N1 * b] * tb.Lq[b][qy];
          }
          Py[aa] = s1 * ih[0];
          Pdy[aa] = s2 * ih[1];
          Dzy[aa] = s3 * ih[2];
        }
        const T jlx = jnv(0, 0, qy + NQ * k), jhx = jnv(0, 1, qy + NQ * k);
        T X[N1];
#pragma unroll
        for (int aa = 0; aa < N1; ++aa) X[aa] = T(0);
#pragma unroll
        for (int qx = 0; qx < NQ; ++qx) {
          T gx = T(0), gy = T(0), gz = T(0);
#pragma unroll
          for (int aa = 0; aa < N1; ++aa) {
            gx += Py[aa] * tb.Dq[aa][qx];
            gy += Pdy[aa] * tb.Lq[aa][qx];
            gz += Dzy[aa] * tb.Lq[aa][qx];
          }
          const T jly = jnv(1, 0, qx + NQ * k), jhy = jnv(1, 1, qx + NQ * k);
          const T jlz = jnv(2, 0, qx + NQ * qy), jhz = jnv(2, 1, qx + NQ * qy);
          const T lft[3] = {gx + tb.K0q[qx] * jlx, gy + tb.K0q[qy] * jly, gz + K0k * jlz};
          const T rgt[3] = {gx + tb.K1q[qx] * jhx, gy + tb.K1q[qy] * jhy, gz + K1k * jhz};
          const T wH = hfun(Sq[qx + NQ * qy], lft, rgt);   // weighted sign: w_q H
#pragma unroll
          for (int aa = 0; aa < N1; ++aa) X[aa] += wH * tb.Lq[aa][qx];
        }
#pragma unroll
        for (int b = 0; b < N1; ++b)
#pragma unroll
          for (int aa = 0; aa < N1; ++aa) U[aa][b] += X[aa] * tb.Lq[b][qy];
      }
#pragma unroll
      for (int b = 0; b < N1; ++b)
#pragma unroll
        for (int aa = 0; aa < N1; ++aa) ub[(size_t)(k * NU + aa + N1 * b) * NT + cl] = U[aa][b];
    }
  }
  __syncthreads();   // planes done: the face-jump area becomes the store staging

  // -------- modes q = k, k + NQ, ...: sum over the planes, update, stage
  {
  T* sb = jn;   // [NT][NM]
  if (valid) {
    const long long cell = (long long)g[0] + (long long)m.n[0] * (g[1] + (long long)m.n[1] * g[2]);
#pragma unroll 1
    for (int q = k; q < NM; q += NQ) {
      const int u = q % NU, cz = q / NU;   // (aa, b) of the plane projection, last-axis mode
      T R = T(0);
#pragma unroll
      for (int kk = 0; kk < NQ; ++kk) R -= ub[(size_t)(kk * NU + u) * NT + cl] * tb.Lq[cz][kk];
      if (a.rdiff) R += a.rdiff[cell * m.nb + m.q2g[q]];
      sb[(size_t)cl * NM + q] = hj_combine<T>(a.rk, c[q], R, dt);
    }
  }
  __syncthreads();
  store_tile<DIM, NM>(m, sb, a.out, o[0], o[1], o[2]);
  }
}

}  // namespace flsp

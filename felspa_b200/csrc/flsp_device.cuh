// flsp_device.cuh — device-side building blocks shared by every kernel of
// libflsp_dg.so: 1D Legendre/Gauss tables in constant memory, the device
// clock, parameter blocks, small reduction helpers.
//
// Data layout in HBM: one array of n_cells * nb coefficients per state
// vector, cells lexicographic (x fastest), nb DoFs of a cell contiguous in
// deal.II order (FE_DGQLegendre lexicographic, FE_DGP total-degree order).
// Inside a CTA every cell is expanded to the Q layout of (p+1)^dim modes
// (zero where the P space has no mode), so one code path serves both bases.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace flsp {

constexpr int kMaxP = 3;
constexpr int kMaxN1 = kMaxP + 1;   // modes per axis
constexpr int kMaxNQ = kMaxP + 2;   // Gauss points per axis (p+2 rule)
constexpr int kMaxTerms = 24;
constexpr int kMaxFeVel = 3;        // largest degree of an FE velocity field

__host__ __device__ constexpr int ipow(int b, int e) { return e == 0 ? 1 : b * ipow(b, e - 1); }

// 1D tables for one polynomial degree p (entries beyond p unused)
template <typename T>
struct Tab1D {
  T xq[kMaxNQ], wq[kMaxNQ];            // Gauss (p+2) points/weights on [0,1]
  T Lq[kMaxN1][kMaxNQ];                 // L_a(xq)
  T Dq[kMaxN1][kMaxNQ];                 // L_a'(xq)
  T Hq[kMaxN1][kMaxNQ];                 // L_a''(xq)
  T L0[kMaxN1], L1[kMaxN1];             // L_a(0), L_a(1)
  T D0[kMaxN1], D1[kMaxN1];             // L_a'(0), L_a'(1)
  T H0[kMaxN1], H1[kMaxN1];             // L_a''(0), L_a''(1)
  T A[kMaxN1][kMaxN1];                  // int_0^1 L_a' L_b
  T xl[kMaxN1], wl[kMaxN1];             // Gauss (p+1) points/weights
  T Ll[kMaxN1][kMaxN1];                 // L_a(xl)
  T Dl[kMaxN1][kMaxN1];                 // L_a'(xl)
  // LDG lifting kernels K_s(x) = sum_a L_a(x) L_a(s), s = 0, 1, at the
  // Gauss (p+2) points and at x = 0, 1
  T K0q[kMaxNQ], K1q[kMaxNQ];
  T K0v[2], K1v[2];
};

// Every translation unit of the library holds its own copy of the tables
// (no relocatable device code); flsp_upload_tables_<unit>() fills it.
static __constant__ Tab1D<double> c_tab_d[kMaxP + 1];
static __constant__ Tab1D<float> c_tab_f[kMaxP + 1];

template <typename T> __device__ __forceinline__ const Tab1D<T>& tab(int p);
template <> __device__ __forceinline__ const Tab1D<double>& tab<double>(int p) { return c_tab_d[p]; }
template <> __device__ __forceinline__ const Tab1D<float>& tab<float>(int p) { return c_tab_f[p]; }

// ---------------------------------------------------------------------
// device clock: simulation time and CFL state live on the GPU so that a
// whole reinit period can be replayed from a CUDA graph without host
// synchronisation.  All fields in double (clocks are FP64 in both modes).
// ---------------------------------------------------------------------
struct DevClock {
  double t;          // time at the start of the current substep
  double dt;         // current substep
  double vd_run;     // running max of (max vertex |u|)/diam (never reset:
                     // the reference CFLEstimator keeps its maximum)
  double t_end;      // clamp for the substep (time_step - cumulative)
  double ct[3];      // velocity time factor at the RK stage times
  double vd_static;  // max over vertices of |u_spatial| / diam
  int active;        // current substep is non-zero
  int pending;       // dt still to be added to t
  int n_substeps;    // executed substeps
  int err;           // device error word (0 = ok)
  // reinitialisation
  double hj_vd_run;  // running max of characteristic speed / diam
  double hj_dt;      // current pseudo-step
  double hj_cum;     // accumulated pseudo-time (before the current step)
  unsigned long long hj_vd_bits;  // atomicMax slot for the next CFL estimate
  int hj_iter;
  int hj_pending;
  double band_ratio; // accumulated pseudo-time / horizon (host convenience)
  double scratch[4];
};

// stage combinations of the SSP-RK schemes (time_integration.implement.h:141-234)
enum CombineMode : int {
  kRhsOnly = 0,     // out = phidot
  kRK1 = 1,         // out = phidot*dt + phi
  kRK2a = 2,        // out = phi + dt*phidot
  kRK2b = 3,        // out = (phi1 + dt*phidot + phin) * 0.5
  kRK3a = 4,        // out = phi + dt*phidot
  kRK3b = 5,        // out = (phi1 + dt*phidot + 3 phin) * 0.25
  kRK3c = 6         // out = ((phi2 + dt*phidot) * 2 + phin) * (1/3)
};

// modes of the reinitialisation kernel
enum HJMode : int { kHJCflOnly = 0, kHJStep = 1, kHJGradients = 2 };

// advection clock parameters (scale = AdvectSimulator::cfl_scaling(p))
struct AdvClockArgs {
  double cfl_max, scale;
  int tkind;
  double ta, tb;
  int rk;
  int step_count;   // 1: a step-count run (the horizon only caps the time)
};

// time factor kinds (flsp_time_kind)
__device__ __forceinline__ double time_factor(int kind, double a, double b, double t) {
  switch (kind) {
    case 1: return cos(a * t + b);
    case 2: return cospi(a * t + b);
    case 3: return 1.0 - exp(-a * t);
    default: return 1.0;
  }
}

// positive doubles compare like their bit patterns
__device__ __forceinline__ void atomic_max_pos(unsigned long long* slot, double v) {
  if (!(v > 0.0)) return;
  atomicMax(slot, (unsigned long long)__double_as_longlong(v));
}

template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// block-wide max of a non-negative double, result valid in thread 0
__device__ __forceinline__ double block_max(double v, double* red) {
  v = warp_max(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  if (w == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    double x = l < nw ? red[l] : 0.0;
    x = warp_max(x);
    if (l == 0) red[0] = x;
  }
  __syncthreads();
  return red[0];
}

// ---------------------------------------------------------------------
// mesh / tile description passed by value to every stencil kernel
// ---------------------------------------------------------------------
struct MeshArgs {
  int n[3];          // cells per axis (1 for unused axes)
  long long ncell;
  double lo[3], h[3];
  double vol, diam, min_diam;
  int nb;            // DoFs per cell in HBM
  signed char q2g[64];  // Q-layout mode -> in-cell DoF index (-1: absent)
  signed char g2q[64];  // in-cell DoF index -> Q-layout mode
  int tile[3];       // CTA tile in cells
  int ntile[3];      // tiles per axis
  // compute-restricted narrow band: block b serves tile tiles[b]; blocks
  // at or past *n_tiles have no tile (null: block b serves tile b)
  const int* tiles;
  const int* n_tiles;
  // Dirichlet value of every domain-boundary face (NaN: none, the face
  // keeps the zero-Neumann interior trace); null: no Dirichlet face.
  // Faces side by side (x-, x+, y-, y+, z-, z+), each side's faces
  // lexicographic in the other axes (lower axis fastest).
  const double* bc_face;
};

// boundary faces on the sides before side (E, S) and within it
template <int DIM>
__host__ __device__ __forceinline__ long long bc_side_faces(const MeshArgs& m, int E) {
  const int t0 = E == 0 ? 1 : 0, t1 = E == 2 ? 1 : 2;
  return (long long)m.n[t0] * (DIM > 2 ? m.n[t1] : 1);
}

// Dirichlet value g on the domain-boundary face on side S (0: lower, 1:
// upper) of axis E of the cell at lattice position c, when the face's
// boundary id carries one: the exterior trace there is the constant g, a
// face polynomial with g in the constant mode and zeros elsewhere
// (inflow of advection.implement.h:719-741; LDG left / right gradients,
// ldg.cc:551-620 and :686-740).  False: zero-Neumann (interior trace).
template <int DIM, typename T>
__device__ __forceinline__ bool bc_dirichlet(const MeshArgs& m, int E, int S, const int* c, T& g) {
  if (!m.bc_face) return false;
  long long off = 0;
#pragma unroll
  for (int e = 0; e < DIM; ++e)
    if (e < E) off += 2 * bc_side_faces<DIM>(m, e);
  const int t0 = E == 0 ? 1 : 0, t1 = E == 2 ? 1 : 2;
  off += S * bc_side_faces<DIM>(m, E) + c[t0] + (DIM > 2 ? (long long)m.n[t0] * c[t1] : 0);
  const double v = m.bc_face[off];
  if (v != v) return false;   // NaN: no Dirichlet value on this face
  g = T(v);
  return true;
}

// separable velocity: vtab[((k*3 + axis) * nmax + i) * npt + j]
// j < NQ: Gauss (p+2) point j of cell i; j == NQ: xi = 0; j == NQ+1: xi = 1
template <typename T>
struct VelArgs {
  const T* vtab;
  int n_terms;
  int nmax;
  int npt;
  int comp[kMaxTerms];
  int cstart[4];   // terms of component c: [cstart[c], cstart[c+1]) (terms sorted by component)
  // velocity tables (the point-wise kernel's TAB form): the spatial part
  // at the cells' quadrature points, tab_q[comp][point][cell], and its
  // normal component at the faces' points, tab_f[E][point][face] (block E
  // at tab_foff[E], tab_nf[E] faces normal to E)
  const T* tab_q;
  const T* tab_f;
  long long tab_foff[3];
  long long tab_nf[3];
};

// first term of each component in a component-sorted term list
__host__ __device__ inline void term_ranges(const int* comp, int n_terms, int* cstart) {
  for (int c = 0; c < 4; ++c) {
    int k = 0;
    while (k < n_terms && comp[k] < c) ++k;
    cstart[c] = k;
  }
}

// next 16-byte aligned address at or after p (shared-memory sub-buffers)
template <typename U>
__device__ __forceinline__ U* align16(void* p) {
  return reinterpret_cast<U*>((reinterpret_cast<uintptr_t>(p) + 15) & ~uintptr_t(15));
}

// local (tile) coordinates of the thread's cell
struct TileCoord {
  int lx, ly, lz;     // in [0, tile)
  int gx, gy, gz;     // global lattice coordinates
  bool valid;
  int ox, oy, oz;     // tile origin
};

// a launch slot (the block index of a plain launch, a work item of a
// persistent one) with no tile to serve in a narrow-band launch (uniform per block)
__device__ __forceinline__ bool tile_inactive(const MeshArgs& m, int slot) {
  return m.tiles != nullptr && slot >= *m.n_tiles;
}

// tile of launch slot `slot` and this thread's cell in it
__device__ __forceinline__ TileCoord tile_coord(const MeshArgs& m, int dim, int slot) {
  TileCoord c;
  int b = m.tiles ? m.tiles[slot] : slot;
  const int bx = b % m.ntile[0];
  b /= m.ntile[0];
  const int by = dim > 1 ? b % m.ntile[1] : 0;
  const int bz = dim > 2 ? b / m.ntile[1] : 0;
  c.ox = bx * m.tile[0];
  c.oy = by * m.tile[1];
  c.oz = bz * m.tile[2];
  int t = threadIdx.x;
  c.lx = t % m.tile[0];
  t /= m.tile[0];
  c.ly = dim > 1 ? t % m.tile[1] : 0;
  c.lz = dim > 2 ? t / m.tile[1] : 0;
  c.gx = c.ox + c.lx;
  c.gy = c.oy + c.ly;
  c.gz = c.oz + c.lz;
  c.valid = (int)threadIdx.x < m.tile[0] * m.tile[1] * m.tile[2] && c.gx < m.n[0] &&
            c.gy < m.n[1] && c.gz < m.n[2];
  return c;
}

__device__ __forceinline__ bool tile_inactive(const MeshArgs& m) { return tile_inactive(m, (int)blockIdx.x); }
__device__ __forceinline__ TileCoord tile_coord(const MeshArgs& m, int dim) { return tile_coord(m, dim, (int)blockIdx.x); }

// padded smem box (tile + 1 halo layer per axis, edge/corner slots unused)
__device__ __forceinline__ int box_index(const MeshArgs& m, int dim, int lx, int ly, int lz) {
  const int bx = m.tile[0] + 2, by = dim > 1 ? m.tile[1] + 2 : 1;
  return (lx + 1) + bx * ((dim > 1 ? ly + 1 : 0) + by * (dim > 2 ? lz + 1 : 0));
}

__device__ __forceinline__ int box_cells(const MeshArgs& m, int dim) {
  return (m.tile[0] + 2) * (dim > 1 ? m.tile[1] + 2 : 1) * (dim > 2 ? m.tile[2] + 2 : 1);
}

// ---------------------------------------------------------------------
// asynchronous global -> shared copies (cp.async, one element each): a
// thread issues all of its copies before waiting, so the latency of every
// row of a tile overlaps instead of serialising row by row
// ---------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void cp_async_elem(T* smem, const T* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  if constexpr (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Load of the tile and its face halo (no edges/corners) from a cell-major
// vector into the smem box, expanded to the Q layout.  One warp per row of
// cells along x (contiguous in HBM), lanes over the row's elements.  Slots
// of cells outside the domain are not written (boundary faces never read
// them).  Completes with cp_async_wait_all() + __syncthreads() by the caller.
template <int DIM, int NM, typename T>
__device__ __forceinline__ void load_box(const MeshArgs& m, const T* __restrict__ g,
                                         T* __restrict__ sm, int ox, int oy, int oz,
                                         bool with_halo) {
  const int tx = m.tile[0], ty = DIM > 1 ? m.tile[1] : 1, tz = DIM > 2 ? m.tile[2] : 1;
  const int h = with_halo ? 1 : 0;
  const int nry = ty + 2 * (DIM > 1 ? h : 0), nrz = tz + 2 * (DIM > 2 ? h : 0);
  const int ly0 = DIM > 1 ? -h : 0, lz0 = DIM > 2 ? -h : 0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const bool dense = m.nb == NM;   // Q basis: smem row == HBM row
  for (int r = warp; r < nry * nrz; r += nw) {
    const int ly = ly0 + r % nry, lz = lz0 + r / nry;
    const bool yout = ly < 0 || ly >= ty, zout = lz < 0 || lz >= tz;
    if (yout && zout) continue;
    const int gy = oy + ly, gz = oz + lz;
    if (gy < 0 || gy >= m.n[1] || gz < 0 || gz >= m.n[2]) continue;
    const int lx0 = (!yout && !zout) ? -h : 0;
    const int lx1 = (!yout && !zout) ? tx + h : tx;
    const int gx0 = max(ox + lx0, 0), gx1 = min(ox + lx1, m.n[0]);
    if (gx1 <= gx0) continue;
    const long long rowcell = (long long)m.n[0] * (gy + (long long)m.n[1] * gz);
    T* dst = sm + (size_t)box_index(m, DIM, gx0 - ox, ly, lz) * NM;
    const int count = (gx1 - gx0) * NM;
    if (dense) {
      const T* src = g + (rowcell + gx0) * NM;
      for (int e = lane; e < count; e += 32) cp_async_elem(dst + e, src + e);
    } else {
      const T* src = g + (rowcell + gx0) * m.nb;
      for (int e = lane; e < count; e += 32) {
        const int cx = e / NM, q = e - cx * NM;
        const int gi = m.q2g[q];
        if (gi >= 0) cp_async_elem(dst + e, src + (long long)cx * m.nb + gi);
        else dst[e] = T(0);
      }
    }
  }
}

// Load of the tile's own cells (no halo) into [cell][NM] (stride = NM) or,
// with transposed = true, into [NM][ld] (column = tile cell index).
template <int DIM, int NM, typename T>
__device__ __forceinline__ void load_tile(const MeshArgs& m, const T* __restrict__ g,
                                          T* __restrict__ sm, int ox, int oy, int oz,
                                          bool transposed, int ld) {
  const int tx = m.tile[0], ty = DIM > 1 ? m.tile[1] : 1, tz = DIM > 2 ? m.tile[2] : 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int r = warp; r < ty * tz; r += nw) {
    const int ly = r % ty, lz = r / ty;
    const int gy = oy + ly, gz = oz + lz;
    const int nx = min(tx, m.n[0] - ox);
    const int cl0 = tx * r;
    const int count = nx * NM;
    if (gy >= m.n[1] || gz >= m.n[2] || nx <= 0) {
      for (int e = lane; e < tx * NM; e += 32) {
        const int cx = e / NM, q = e - cx * NM;
        if (transposed) sm[(size_t)q * ld + cl0 + cx] = T(0);
        else sm[(size_t)(cl0 + cx) * NM + q] = T(0);
      }
      continue;
    }
    const T* src = g + ((long long)m.n[0] * (gy + (long long)m.n[1] * gz) + ox) * m.nb;
    for (int e = lane; e < count; e += 32) {
      const int cx = e / NM, q = e - cx * NM;
      const int gi = m.q2g[q];
      T* d = transposed ? sm + (size_t)q * ld + cl0 + cx : sm + (size_t)(cl0 + cx) * NM + q;
      if (gi >= 0) cp_async_elem(d, src + (long long)cx * m.nb + gi);
      else *d = T(0);
    }
    for (int e = count + lane; e < tx * NM; e += 32) {   // cells past the domain edge
      const int cx = e / NM, q = e - cx * NM;
      if (transposed) sm[(size_t)q * ld + cl0 + cx] = T(0);
      else sm[(size_t)(cl0 + cx) * NM + q] = T(0);
    }
  }
}

// Store of the tile's own cells from [cell][NM] smem to HBM (nb DoFs per
// cell, g2q maps them to the Q slots), one warp per row.
template <int DIM, int NM, typename T>
__device__ __forceinline__ void store_tile(const MeshArgs& m, const T* __restrict__ sm,
                                           T* __restrict__ g, int ox, int oy, int oz) {
  const int tx = m.tile[0], ty = DIM > 1 ? m.tile[1] : 1, tz = DIM > 2 ? m.tile[2] : 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const bool dense = m.nb == NM;
  for (int r = warp; r < ty * tz; r += nw) {
    const int ly = r % ty, lz = r / ty;
    const int gy = oy + ly, gz = oz + lz;
    const int nx = min(tx, m.n[0] - ox);
    if (gy >= m.n[1] || gz >= m.n[2] || nx <= 0) continue;
    T* dst = g + ((long long)m.n[0] * (gy + (long long)m.n[1] * gz) + ox) * m.nb;
    const T* src = sm + (size_t)tx * r * NM;
    if (dense) {
      for (int e = lane; e < nx * NM; e += 32) dst[e] = src[e];
    } else {
      for (int e = lane; e < nx * m.nb; e += 32) {
        const int cx = e / m.nb, k = e - cx * m.nb;
        dst[e] = src[(size_t)cx * NM + m.g2q[k]];
      }
    }
  }
}

// ---------------------------------------------------------------------
// Bulk asynchronous copies (TMA engine, cp.async.bulk) completing on a
// shared-memory mbarrier.  Copies are plain global -> own-CTA shared
// memory: no cluster multicast.  Both addresses 16-byte aligned, size a
// multiple of 16.
// ---------------------------------------------------------------------
constexpr int kErrCopyTimeout = 1;   // DevClock::err bit: a bulk-copy wait ran out
constexpr int kOpRowPad = 32;        // operator-table rows past the mesh per (d, e) block
constexpr int kStatePad = 256;       // bytes past the end of every state buffer

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
// one arrival that also announces the bytes the phase waits for
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// Wait for phase `parity` of the barrier, at most max_iter polls (each
// try_wait may itself suspend for a while); false when it ran out.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, int max_iter) {
  const unsigned a = smem_u32(bar);
  for (int it = 0; it < max_iter; ++it) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

}  // namespace flsp

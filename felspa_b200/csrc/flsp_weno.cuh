// flsp_weno.cuh — 2D minmod troubled-cell detector + WENO limiter, fused.
//
// Replaces dg::apply_weno_limiter (include/felspa/pde/src/pde_tools.implement.h:977-1004):
// MinmodShockDetector::cell_has_shock (:277-376, beta = 1 + dim) flags cells
// from the state before limiting, then WENOLimiter::apply_limiting_to_cell
// (:557-706) rebuilds each flagged cell from the old copy of the state
// (gamma_neighbour = 0.001, eps = 1e-6, smoothness up to min(2, p)
// derivatives).  Since both read only the pre-limit state, one kernel reads
// `in` (tile + face halo in shared memory) and writes `out`; unflagged
// cells pass through.  The smoothness indicator keeps the reference's
// indexing of the Hessian (hessians[i][j] with i, j < dim indexes the
// quadrature point i, :545-547) and scales neighbour terms by the
// neighbour's cell measure (:524).
#pragma once
#include "flsp_device.cuh"

namespace flsp {

template <typename T>
struct WenoArgs {
  MeshArgs m;
  const T* __restrict__ in;
  T* __restrict__ out;
  unsigned int* count;   // troubled-cell counter (may be null)
  // troubled cells for the reconstruction pass: (problem, cell) entries,
  // *list_n of them
  int2* list;
  unsigned int* list_n;
  int problem;
};

template <int P, typename T>
__host__ __device__ inline size_t weno_smem_bytes(const int* tile) {
  constexpr int NM = (P + 1) * (P + 1);
  return (size_t)(tile[0] + 2) * (tile[1] + 2) * NM * sizeof(T);
}

// Legendre values/derivatives at an arbitrary point (neighbour polynomials
// are evaluated outside their own cell)
template <int N1, typename T>
__device__ __forceinline__ void legendre_at(T x, T* v, T* d, T* dd) {
  const T t = T(2) * x - T(1);
  T P_[N1 + 1], dP[N1 + 1], ddP[N1 + 1];
  P_[0] = T(1); dP[0] = T(0); ddP[0] = T(0);
  if (N1 > 1) { P_[1] = t; dP[1] = T(1); ddP[1] = T(0); }
#pragma unroll
  for (int k = 1; k + 1 < N1; ++k) {
    P_[k + 1] = (T(2 * k + 1) * t * P_[k] - T(k) * P_[k - 1]) / T(k + 1);
    dP[k + 1] = (T(2 * k + 1) * (P_[k] + t * dP[k]) - T(k) * dP[k - 1]) / T(k + 1);
    ddP[k + 1] = (T(2 * k + 1) * (T(2) * dP[k] + t * ddP[k]) - T(k) * ddP[k - 1]) / T(k + 1);
  }
#pragma unroll
  for (int k = 0; k < N1; ++k) {
    const T s = sqrt(T(2 * k + 1));
    v[k] = s * P_[k];
    d[k] = T(2) * s * dP[k];
    dd[k] = T(4) * s * ddP[k];
  }
}

template <int P, typename T>
__device__ __forceinline__ void weno_tile(const WenoArgs<T>& a, int slot) {
  constexpr int N1 = P + 1, NQ = P + 2, NM = N1 * N1, NQV = NQ * NQ;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* box = reinterpret_cast<T*>(smem_raw);
  const MeshArgs& m = a.m;
  const Tab1D<T>& tb = tab<T>(P);
  if (tile_inactive(m, slot)) return;
  const TileCoord tc = tile_coord(m, 2, slot);
  load_box<2, NM>(m, a.in, box, tc.ox, tc.oy, 0, true);
  cp_async_wait_all();
  __syncthreads();
  if (!tc.valid) return;
  const T* c = box + (size_t)box_index(m, 2, tc.lx, tc.ly, 0) * NM;
  const long long cell = (long long)tc.gx + (long long)m.n[0] * tc.gy;
  const T hx = T(m.h[0]), hy = T(m.h[1]);
  const T vol = T(m.vol);

  auto avg_of = [&](const T* cc) -> T {  // compute_cell_average (:960-973)
    T s = T(0);
#pragma unroll
    for (int qy = 0; qy < NQ; ++qy)
#pragma unroll
      for (int qx = 0; qx < NQ; ++qx) {
        T v = T(0);
#pragma unroll
        for (int q = 0; q < NM; ++q) v += cc[q] * (tb.Lq[q % N1][qx] * tb.Lq[q / N1][qy]);
        s += v * (tb.wq[qx] * tb.wq[qy] * vol);
      }
    return s / vol;
  };

  // ---------------- minmod detection ----------------
  const bool nb_ok[4] = {tc.gx > 0, tc.gx + 1 < m.n[0], tc.gy > 0, tc.gy + 1 < m.n[1]};
  const int nbl[4][2] = {{tc.lx - 1, tc.ly}, {tc.lx + 1, tc.ly}, {tc.lx, tc.ly - 1}, {tc.lx, tc.ly + 1}};
  const T* cn[4];
#pragma unroll
  for (int f = 0; f < 4; ++f) cn[f] = box + (size_t)box_index(m, 2, nbl[f][0], nbl[f][1], 0) * NM;
  const T avg = avg_of(c);
  T nav[4];
#pragma unroll
  for (int f = 0; f < 4; ++f) nav[f] = nb_ok[f] ? avg_of(cn[f]) : T(0);
  const int fav[4][2] = {{0, 2}, {2, 1}, {0, 3}, {1, 3}};
  const T beta_mm = T(3);  // 1 + dim
  bool troubled = false;
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    if (!nb_ok[fav[v][0]] || !nb_ok[fav[v][1]]) continue;
    // vertex value
    T val = T(0);
#pragma unroll
    for (int q = 0; q < NM; ++q) {
      const T bx = (v & 1) ? tb.L1[q % N1] : tb.L0[q % N1];
      const T by = (v & 2) ? tb.L1[q / N1] : tb.L0[q / N1];
      val += c[q] * (bx * by);
    }
    // directional coefficients (c_nb - c).(v - c) / |c_nb - c|^2 = 1/2 on a
    // uniform Cartesian mesh
    T interp = T(0);
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int f = fav[v][k];
      const T dxn = (f == 0) ? -hx : (f == 1 ? hx : T(0));
      const T dyn = (f == 2) ? -hy : (f == 3 ? hy : T(0));
      const T vx = (v & 1) ? T(0.5) * hx : T(-0.5) * hx;
      const T vy = (v & 2) ? T(0.5) * hy : T(-0.5) * hy;
      const T coeff = (dxn * vx + dyn * vy) / (dxn * dxn + dyn * dyn);
      interp += (nav[f] - avg) * coeff;
    }
    const T aa = val - avg;
    const T bb = beta_mm * interp;
    const int sa = (aa > T(0)) - (aa < T(0)), sb = (bb > T(0)) - (bb < T(0));
    const T mm = (sa == sb) ? T(sa) * fmin(fabs(aa), fabs(bb)) : T(0);
    if (aa != mm) { troubled = true; break; }
  }

  if (troubled) {
    // the WENO reconstruction runs in a second pass over the troubled
    // cells only (weno_fix), a warp per cell
    if (a.count) atomicAdd(a.count, 1u);
    const unsigned int k = atomicAdd(a.list_n, 1u);
    a.list[k] = make_int2(a.problem, (int)cell);
    return;
  }
  for (int k = 0; k < m.nb; ++k) a.out[cell * m.nb + k] = c[m.g2q[k]];
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// WENO reconstruction of one troubled cell (apply_weno_limiter's troubled
// branch, pde_tools.implement.h:515-720,977-1004), by one warp: lane qp <
// NQV owns home Gauss point qp for the smoothness indicators and the new
// polynomial's values, lane q < NM owns mode q for the projection.  `sh`:
// the warp's 5 * NM values (home cell, then the face neighbours 0..3, Q
// layout).  Every lane of the warp calls it with the same cell.
template <int P, typename T>
__device__ __forceinline__ void weno_fix(const MeshArgs& m, const T* __restrict__ in, T* __restrict__ out, int cell,
                                         T* sh) {
  constexpr int N1 = P + 1, NQ = P + 2, NM = N1 * N1, NQV = NQ * NQ;
  const Tab1D<T>& tb = tab<T>(P);
  const int lane = threadIdx.x & 31;
  const int gx = cell % m.n[0], gy = cell / m.n[0];
  const bool nb_ok[4] = {gx > 0, gx + 1 < m.n[0], gy > 0, gy + 1 < m.n[1]};
  const long long nbc[5] = {cell, (long long)cell - 1, (long long)cell + 1, (long long)cell - m.n[0],
                            (long long)cell + m.n[0]};
  for (int e = lane; e < 5 * NM; e += 32) {
    const int k = e / NM, q = e - k * NM;
    const int gi = m.q2g[q];
    const bool ok = k == 0 || nb_ok[k - 1];
    sh[e] = (ok && gi >= 0) ? in[nbc[k] * m.nb + gi] : T(0);
  }
  __syncwarp();
  const T* c = sh;
  const T hx = T(m.h[0]), hy = T(m.h[1]);
  const T vol = T(m.vol);
  // cell average of the home polynomial, as in the detection pass
  T avg = T(0);
  {
    T s = T(0);
    for (int qy = 0; qy < NQ; ++qy)
      for (int qx = 0; qx < NQ; ++qx) {
        T v = T(0);
#pragma unroll
        for (int q = 0; q < NM; ++q) v += c[q] * (tb.Lq[q % N1][qx] * tb.Lq[q / N1][qy]);
        s += v * (tb.wq[qx] * tb.wq[qy] * vol);
      }
    avg = s / vol;
  }
  const int max_deriv = P < 2 ? P : 2;
  const T gamma_nb = T(0.001), eps = T(1.0e-6);
  const int qx = lane % NQ, qy = lane / NQ;
  const bool own = lane < NQV;
  // smoothness indicator of polynomial cc at the home points shifted by
  // (sx, sy) cells in its own reference coordinates
  auto smooth = [&](const T* cc, T sx, T sy) -> T {
    T part = T(0), hxx = T(0), hxy = T(0), hyy = T(0);
    if (own) {
      T lx[N1], dx[N1], ddx[N1], ly[N1], dy[N1], ddy[N1];
      legendre_at<N1, T>(tb.xq[qx] + sx, lx, dx, ddx);
      legendre_at<N1, T>(tb.xq[qy] + sy, ly, dy, ddy);
      T gxx = T(0), gyy = T(0);
#pragma unroll
      for (int q = 0; q < NM; ++q) {
        const int i0 = q % N1, i1 = q / N1;
        gxx += cc[q] * (dx[i0] * ly[i1] / hx);
        gyy += cc[q] * (lx[i0] * dy[i1] / hy);
        hxx += cc[q] * (ddx[i0] * ly[i1] / (hx * hx));
        hxy += cc[q] * (dx[i0] * dy[i1] / (hx * hy));
        hyy += cc[q] * (lx[i0] * ddy[i1] / (hy * hy));
      }
      if (max_deriv >= 1) part = (gxx * gxx + gyy * gyy) * (tb.wq[qx] * tb.wq[qy] * vol) * vol;
    }
    T beta = warp_sum(part);
    // Hessians at home points 0 and 1 (lanes 0 and 1)
    const T a00 = __shfl_sync(0xffffffffu, hxx, 0), a01 = __shfl_sync(0xffffffffu, hxy, 0);
    const T a11 = __shfl_sync(0xffffffffu, hyy, 0);
    const T b01 = __shfl_sync(0xffffffffu, hxy, 1), b11 = __shfl_sync(0xffffffffu, hyy, 1);
    if (max_deriv >= 2) {
      T ls = T(0);
      ls += a00 * a00 + a01 * a01;
      ls += a01 * a01 + a11 * a11;
      ls += b01 * b01 + b11 * b11;
      for (int py = 0; py < NQ; ++py)
        for (int px = 0; px < NQ; ++px) beta += ls * (tb.wq[px] * tb.wq[py] * vol) * (vol * vol * vol);
    }
    return beta;
  };
  T weights[5];
  int nw = 0;
  T acc = T(0);
#pragma unroll
  for (int f = 0; f < 4; ++f)
    if (nb_ok[f]) acc += gamma_nb;
  {
    const T den = eps + smooth(c, T(0), T(0));
    weights[nw++] = (T(1) - acc) / den / den;
  }
  // neighbour order: faces 0..3 (find_neighbor_cells, :482-508)
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    if (!nb_ok[f]) continue;
    const T sx = (f == 0) ? T(1) : (f == 1 ? T(-1) : T(0));
    const T sy = (f == 2) ? T(1) : (f == 3 ? T(-1) : T(0));
    const T den = eps + smooth(sh + (f + 1) * NM, sx, sy);
    weights[nw++] = gamma_nb / den / den;
  }
  T wsum = T(0);
  for (int i = 0; i < nw; ++i) wsum += weights[i];
  for (int i = 0; i < nw; ++i) weights[i] /= wsum;
  // p_new at the lane's home point: w_home p_home + sum_l w_l (p_l - avg_l + avg_home)
  T pnew = T(0);
  if (own) {
    T v = T(0);
#pragma unroll
    for (int q = 0; q < NM; ++q) v += c[q] * (tb.Lq[q % N1][qx] * tb.Lq[q / N1][qy]);
    pnew = v * weights[0];
  }
  int wi = 1;
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    if (!nb_ok[f]) continue;
    const T sx = (f == 0) ? T(1) : (f == 1 ? T(-1) : T(0));
    const T sy = (f == 2) ? T(1) : (f == 3 ? T(-1) : T(0));
    const T* cn = sh + (f + 1) * NM;
    T val = T(0), part = T(0);
    if (own) {
      T lx[N1], dx[N1], ddx[N1], ly[N1], dy[N1], ddy[N1];
      legendre_at<N1, T>(tb.xq[qx] + sx, lx, dx, ddx);
      legendre_at<N1, T>(tb.xq[qy] + sy, ly, dy, ddy);
#pragma unroll
      for (int q = 0; q < NM; ++q) val += cn[q] * (lx[q % N1] * ly[q / N1]);
      part = val * (tb.wq[qx] * tb.wq[qy] * vol);
    }
    const T this_avg = warp_sum(part) / vol;
    if (own) pnew += (val - this_avg + avg) * weights[wi];
    ++wi;
  }
  // projection c_q = int p_new psi_q / int psi_q^2 (lane q), the points in order
  T num = T(0), den = T(0);
  const int mq = lane < NM ? lane : 0;
  for (int qp = 0; qp < NQV; ++qp) {
    const T pv = __shfl_sync(0xffffffffu, pnew, qp);
    const int px = qp % NQ, py = qp / NQ;
    const T sv = tb.Lq[mq % N1][px] * tb.Lq[mq / N1][py];
    const T jxw = tb.wq[px] * tb.wq[py] * vol;
    num += pv * sv * jxw;
    den += sv * sv * jxw;
  }
  const T outc = (lane < NM && m.q2g[mq] >= 0) ? num / den : T(0);
  const int src = lane < m.nb ? m.g2q[lane] : 0;
  const T w = __shfl_sync(0xffffffffu, outc, src);
  if (lane < m.nb) out[(long long)cell * m.nb + lane] = w;
  __syncwarp();
}

// second pass over the troubled cells of one problem: a warp per cell
template <int P, typename T>
__global__ void __launch_bounds__(256) weno_fix_kernel(const WenoArgs<T> a) {
  constexpr int NM = (P + 1) * (P + 1);
  __shared__ T sh[8][5 * NM];
  const int wl = threadIdx.x >> 5;
  const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  const unsigned int n = *a.list_n;
  for (unsigned int i = warp; i < n; i += nwarps) weno_fix<P, T>(a.m, a.in, a.out, a.list[i].y, sh[wl]);
}

template <int P, typename T>
__global__ void __launch_bounds__(256, 2) weno_kernel(const WenoArgs<T> a) {
  weno_tile<P, T>(a, (int)blockIdx.x);
}

}  // namespace flsp

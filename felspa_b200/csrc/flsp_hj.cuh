// flsp_hj.cuh — Hamilton-Jacobi reinitialisation pseudo-step.
//
// Replaces, per pseudo-step (src/pde/hamilton_jacobi.cc:514-551):
//   local_left_right_gradients  (hamilton_jacobi.cc:462-511; LDG integrators
//                                src/pde/ldg.cc:355-376, 510-740)
//   ReinitOperator::cell_values (src/level_set/reinit.cc:267-301: smooth sign
//                                :121-133, Lax-Friedrichs H :136-191)
//   HJAssemblerWorkStream       (hamilton_jacobi.cc:730-745)
//   the mass solve and the RK update,
// and the characteristic-speed CFL estimate the next pseudo-step uses
// (ReinitOperator::cell_velocities reinit.cc:304-328, characteristic_velocity
// :235-264, CFLEstimator at QTrapezoid vertices).
//
// The LDG one-sided gradients are computed modally and exactly: for the
// orthonormal Legendre basis, QGauss(p+1) integrates every LDG term without
// error, so  g^L_e = (1/h_e) [ -A c + L(1) (x) T_up - L(0) (x) T_lo^left ]
// along each line of axis e (A_ab = int L_a' L_b, T the face traces, the
// left/right flux taking the trace of the lower/upper cell, the interior
// trace on the boundary).  In the P basis the padded Q modes are masked.
#pragma once
#include "flsp_device.cuh"

namespace flsp {


template <typename T>
struct HJArgs {
  MeshArgs m;
  const T* __restrict__ phi;    // phi^k (read with halo)
  const T* __restrict__ phi0;   // phi at reinit start
  T* __restrict__ out;          // phi^{k+1} or gradient blocks
  DevClock* clk;
  int mode;
  int rk;                       // reinit RK order (all stages see the same L)
  double dt_explicit;           // used when clk == nullptr
  long long block;              // gradient block stride (ncell * nb)
  const T* __restrict__ rdiff;  // LDG diffusion RHS per unit volume (nu > 0) or null
  T* stab;                      // smooth-sign table of the tensor-product kernel (hjs_kernel)
  int* err;                     // device error word (DevClock::err) or null
};

// add the cell's LDG diffusion RHS (HBM layout) to R (Q layout)
template <int NM, typename T>
__device__ __forceinline__ void add_rdiff(const MeshArgs& m, const T* rdiff, long long cell, T* R) {
  if (!rdiff) return;
  for (int k = 0; k < m.nb; ++k) {
    const T v = rdiff[cell * m.nb + k];
#pragma unroll
    for (int q = 0; q < NM; ++q)
      if (q == m.g2q[k]) R[q] += v;
  }
}

template <int DIM, int P, typename T>
__host__ __device__ inline size_t hj_smem_bytes(const int* tile) {
  constexpr int N1 = P + 1, NQ = P + 2, NM = ipow(N1, DIM), NQV = ipow(NQ, DIM);
  const int bx = tile[0] + 2, by = DIM > 1 ? tile[1] + 2 : 1, bz = DIM > 2 ? tile[2] + 2 : 1;
  const int nt = tile[0] * tile[1] * (DIM > 2 ? tile[2] : 1);
  size_t box = (size_t)bx * by * bz * NM * sizeof(T);
  size_t own0 = (size_t)nt * NM * sizeof(T);
  size_t acc = (size_t)nt * 2 * NQV * sizeof(T);
  return box + own0 + acc + 64 * sizeof(double) + 16;
}

// RK combinations of ReinitSimulatorLDG::advance_time with the reference's
// operation order; explicit_time_derivative ignores its argument
// (hamilton_jacobi.cc:514-551), so every stage uses the same L.
template <typename T>
__device__ __forceinline__ T hj_combine(int rk, T phi, T L, T dt) {
  if (rk <= 1) { T s = L * dt; return s + phi; }
  if (rk == 2) { T s = phi; s += dt * L; s += dt * L; s += phi; return s * T(0.5); }
  T s = phi;
  s += dt * L; s += dt * L; s += T(3.0) * phi; s *= T(0.25);
  s += dt * L; s *= T(2.0); s += phi;
  return s * (T(1.0) / T(3.0));
}

template <int DIM, int P, typename T>
__global__ void __launch_bounds__(256) hj_kernel(const HJArgs<T> a) {
  constexpr int N1 = P + 1, NQ = P + 2, NM = ipow(N1, DIM), NQV = ipow(NQ, DIM);
  constexpr int NV = 1 << DIM;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const MeshArgs& m = a.m;
  T* box = reinterpret_cast<T*>(smem_raw);
  const int nboxc = box_cells(m, DIM);
  const int tx = m.tile[0], ty = m.tile[1], tz = m.tile[2];
  const int nt = tx * ty * tz;
  T* own0 = box + (size_t)nboxc * NM;
  T* acc = own0 + (size_t)nt * NM;
  double* red = align16<double>(acc + (size_t)nt * 2 * NQV);
  const Tab1D<T>& tb = tab<T>(P);
  if (tile_inactive(m)) return;
  const TileCoord tc = tile_coord(m, DIM);

  load_box<DIM, NM>(m, a.phi, box, tc.ox, tc.oy, tc.oz, true);
  load_tile<DIM, NM>(m, a.phi0, own0, tc.ox, tc.oy, tc.oz, false, NM);
  cp_async_wait_all();
  __syncthreads();

  const int cl = tc.lx + tx * (tc.ly + ty * tc.lz);
  const int st[3] = {1, N1, N1 * N1};
  T c[NM];
  T R[NM];
  double vmax = 0.0;
  const T hmin = T(m.min_diam);
  const T dt = a.clk ? T(a.clk->hj_dt) : T(a.dt_explicit);

  if (tc.valid) {
    const int me = box_index(m, DIM, tc.lx, tc.ly, tc.lz);
#pragma unroll
    for (int q = 0; q < NM; ++q) c[q] = box[(size_t)me * NM + q];
    T* A2 = acc + (size_t)cl * 2 * NQV;
    T* AD = A2 + NQV;
    if (a.mode == kHJStep)
      for (int q = 0; q < NQV; ++q) { A2[q] = T(0); AD[q] = T(0); }
    T vl[NV][DIM], vr[NV][DIM];

#pragma unroll
    for (int e = 0; e < DIM; ++e) {
      const T ih = T(1.0 / m.h[e]);
      int nl[3] = {tc.lx, tc.ly, tc.lz}, nu[3] = {tc.lx, tc.ly, tc.lz};
      int gg[3] = {tc.gx, tc.gy, tc.gz};
      nl[e] -= 1;
      nu[e] += 1;
      const bool has_lo = gg[e] > 0, has_hi = gg[e] + 1 < m.n[e];
      T glo = T(0), ghi = T(0);
      const bool dlo = !has_lo && bc_dirichlet<DIM>(m, e, 0, gg, glo);
      const bool dhi = !has_hi && bc_dirichlet<DIM>(m, e, 1, gg, ghi);
      const T* cL = box + (size_t)box_index(m, DIM, nl[0], nl[1], nl[2]) * NM;
      const T* cU = box + (size_t)box_index(m, DIM, nu[0], nu[1], nu[2]) * NM;
      T gl[NM], gr[NM];
      // lines along axis e: enumerate the other two mode indices
#pragma unroll
      for (int li = 0; li < NM / N1; ++li) {
        const int i0 = li % N1, i1 = li / N1;
        int base;
        if (e == 0) base = i0 * st[1] + i1 * st[2];
        else if (e == 1) base = i0 * st[0] + i1 * st[2];
        else base = i0 * st[0] + i1 * st[1];
        if constexpr (DIM == 2) { base = (e == 0) ? i0 * st[1] : i0 * st[0]; }
        T tup = T(0), tlo = T(0), tnl = T(0), tnu = T(0);
#pragma unroll
        for (int b = 0; b < N1; ++b) {
          const T cb = c[base + b * st[e]];
          tup += tb.L1[b] * cb;
          tlo += tb.L0[b] * cb;
          if (has_lo) tnl += tb.L1[b] * cL[base + b * st[e]];
          if (has_hi) tnu += tb.L0[b] * cU[base + b * st[e]];
        }
        // domain boundary: the Dirichlet value of the face (constant mode
        // only) where it carries one, else the interior trace
        if (!has_lo) tnl = dlo ? (li == 0 ? glo : T(0)) : tlo;
        if (!has_hi) tnu = dhi ? (li == 0 ? ghi : T(0)) : tup;
#pragma unroll
        for (int aa = 0; aa < N1; ++aa) {
          T bs = T(0);
#pragma unroll
          for (int b = 0; b < N1; ++b) bs -= tb.A[aa][b] * c[base + b * st[e]];
          gl[base + aa * st[e]] = (bs + tb.L1[aa] * tup - tb.L0[aa] * tnl) * ih;
          gr[base + aa * st[e]] = (bs + tb.L1[aa] * tnu - tb.L0[aa] * tlo) * ih;
        }
      }
#pragma unroll
      for (int q = 0; q < NM; ++q)
        if (m.q2g[q] < 0) { gl[q] = T(0); gr[q] = T(0); }

      if (a.mode == kHJGradients) {
        const long long cell = (long long)tc.gx + (long long)m.n[0] * (tc.gy + (long long)m.n[1] * tc.gz);
        for (int k = 0; k < m.nb; ++k) {
          a.out[(long long)e * a.block + cell * m.nb + k] = gl[m.g2q[k]];
          a.out[(long long)(DIM + e) * a.block + cell * m.nb + k] = gr[m.g2q[k]];
        }
        continue;
      }
      // values at the 2^dim vertices (QTrapezoid order, x fastest)
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        T sl = T(0), sr = T(0);
#pragma unroll
        for (int q = 0; q < NM; ++q) {
          const int i0 = q % N1, i1 = (q / N1) % N1, i2 = q / (N1 * N1);
          T bw = (v & 1) ? tb.L1[i0] : tb.L0[i0];
          bw = bw * (((v >> 1) & 1) ? tb.L1[i1] : tb.L0[i1]);
          if constexpr (DIM == 3) bw = bw * (((v >> 2) & 1) ? tb.L1[i2] : tb.L0[i2]);
          sl += gl[q] * bw;
          sr += gr[q] * bw;
        }
        vl[v][e] = sl;
        vr[v][e] = sr;
      }
      if (a.mode == kHJStep) {
        // accumulate |avg|^2 and sum (l - r) at the cell quadrature points
#pragma unroll 1
        for (int qp = 0; qp < NQV; ++qp) {
          const int qx = qp % NQ, qy = (qp / NQ) % NQ, qz = qp / (NQ * NQ);
          T sl = T(0), sr = T(0);
#pragma unroll
          for (int q = 0; q < NM; ++q) {
            const int i0 = q % N1, i1 = (q / N1) % N1, i2 = q / (N1 * N1);
            T bw = tb.Lq[i0][qx] * tb.Lq[i1][qy];
            if constexpr (DIM == 3) bw = bw * tb.Lq[i2][qz];
            sl += gl[q] * bw;
            sr += gr[q] * bw;
          }
          const T avg = T(0.5) * (sl + sr);
          A2[qp] += avg * avg;
          AD[qp] += sl - sr;
        }
      }
    }

    if (a.mode != kHJGradients) {
      // smooth sign and characteristic speed at the vertices
      const T* c0 = own0 + (size_t)cl * NM;
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        T p0 = T(0), g[3] = {T(0), T(0), T(0)};
#pragma unroll
        for (int q = 0; q < NM; ++q) {
          const int idx[3] = {q % N1, (q / N1) % N1, q / (N1 * N1)};
          T val = T(1);
          T dv[3];
#pragma unroll
          for (int d = 0; d < DIM; ++d) {
            const bool up = (v >> d) & 1;
            const T lv = up ? tb.L1[idx[d]] : tb.L0[idx[d]];
            val = val * lv;
          }
#pragma unroll
          for (int d = 0; d < DIM; ++d) {
            T pr = T(1);
#pragma unroll
            for (int d2 = 0; d2 < DIM; ++d2) {
              const bool up = (v >> d2) & 1;
              const T lv = (d2 == d) ? (up ? tb.D1[idx[d2]] : tb.D0[idx[d2]])
                                     : (up ? tb.L1[idx[d2]] : tb.L0[idx[d2]]);
              pr = pr * lv;
            }
            dv[d] = pr;
          }
          p0 += c0[q] * val;
#pragma unroll
          for (int d = 0; d < DIM; ++d) g[d] += c0[q] * (dv[d] * T(1.0 / m.h[d]));
        }
        T g2 = T(0);
#pragma unroll
        for (int d = 0; d < DIM; ++d) g2 += g[d] * g[d];
        const T S = p0 / sqrt(p0 * p0 + hmin * hmin * sqrt(g2) * sqrt(g2));
        // characteristic_velocity (reinit.cc:235-264)
        T gs[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
          const T l = vl[v][d], r = vr[v][d];
          if (S >= T(0)) {
            const T lp = max(l, T(0)), rm = -min(r, T(0));
            gs[d] = fabs(lp) > fabs(rm) ? lp : rm;
          } else {
            const T lm = -min(l, T(0)), rp = max(r, T(0));
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
      vmax = vmax / m.diam;

      if (a.mode == kHJStep) {
#pragma unroll
        for (int q = 0; q < NM; ++q) R[q] = T(0);
#pragma unroll 1
        for (int qp = 0; qp < NQV; ++qp) {
          const int qq[3] = {qp % NQ, (qp / NQ) % NQ, qp / (NQ * NQ)};
          T p0 = T(0), g[3] = {T(0), T(0), T(0)};
#pragma unroll
          for (int q = 0; q < NM; ++q) {
            const int idx[3] = {q % N1, (q / N1) % N1, q / (N1 * N1)};
            T val = T(1);
#pragma unroll
            for (int d = 0; d < DIM; ++d) val = val * tb.Lq[idx[d]][qq[d]];
            p0 += c0[q] * val;
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
              T pr = T(1);
#pragma unroll
              for (int d2 = 0; d2 < DIM; ++d2)
                pr = pr * ((d2 == d) ? tb.Dq[idx[d2]][qq[d2]] : tb.Lq[idx[d2]][qq[d2]]);
              g[d] += c0[q] * (pr * T(1.0 / m.h[d]));
            }
          }
          T g2 = T(0);
#pragma unroll
          for (int d = 0; d < DIM; ++d) g2 += g[d] * g[d];
          const T gn = sqrt(g2);
          const T S = p0 / sqrt(p0 * p0 + hmin * hmin * gn * gn);
          T H = S * (sqrt(A2[qp]) - T(1));
          H += T(0.5) * fabs(S) * AD[qp];
          T w = tb.wq[qq[0]] * tb.wq[qq[1]];
          if constexpr (DIM == 3) w = w * tb.wq[qq[2]];
          const T hw = H * w;
#pragma unroll
          for (int q = 0; q < NM; ++q) {
            const int idx[3] = {q % N1, (q / N1) % N1, q / (N1 * N1)};
            T val = T(1);
#pragma unroll
            for (int d = 0; d < DIM; ++d) val = val * tb.Lq[idx[d]][qq[d]];
            R[q] -= val * hw;
          }
        }
      }
    }
  }

  if (a.mode == kHJGradients) return;
  // CFL maximum of this CTA -> device slot
  const double bm = block_max(vmax, red);
  if (threadIdx.x == 0 && a.clk) atomic_max_pos(&a.clk->hj_vd_bits, bm);
  if (a.mode != kHJStep) return;

  // update, staged through shared memory for coalesced stores
  __syncthreads();
  T* sb = box;
  if (tc.valid) {
    add_rdiff<NM>(m, a.rdiff, (long long)tc.gx + (long long)m.n[0] * (tc.gy + (long long)m.n[1] * tc.gz), R);
#pragma unroll
    for (int q = 0; q < NM; ++q) sb[(size_t)cl * NM + q] = hj_combine<T>(a.rk, c[q], R[q], dt);
  }
  __syncthreads();
  store_tile<DIM, NM>(m, sb, a.out, tc.ox, tc.oy, tc.oz);
}

}  // namespace flsp

// flsp_advect.cuh — DG advection: one fused kernel per SSP-RK stage.
//
// Replaces AdvectAssembler<workstream>::cell_assembly / face_assembly /
// boundary_assembly (include/felspa/pde/src/advection.implement.h:617-744),
// the diagonal mass solve (linear_systems.implement.h:30-47) and the stage
// combinations of RungeKuttaTVD<k> (time_integration.implement.h:141-234).
//
// One thread owns one cell.  The CTA stages its tile of cells plus the
// face-neighbour halo in shared memory (Q layout), and the velocity-table
// rows of its tile.  The cell term is sum-factorised (z, then y
// interpolation to a (p+1)(p+2)^2 partial, then x-lines), the upwind face
// flux is evaluated at the (p+2)^(dim-1) face points.  phidot = R / |K| is
// formed in "per volume" units directly (faces scale with 1/h_e).
#pragma once
#include "flsp_device.cuh"

namespace flsp {


template <typename T>
struct AdvArgs {
  MeshArgs m;
  VelArgs<T> v;
  const T* __restrict__ phi_s;   // stage input (read with halo)
  const T* __restrict__ phi_n;   // phi^n for the combinations
  T* __restrict__ out;
  const DevClock* clk;
  int stage;                      // index into clk->ct
  int combine;                    // CombineMode
  double ct_explicit;             // time factor when clk == nullptr
  double dt_explicit;
};

template <typename T>
__device__ __forceinline__ T combine_value(int mode, T phi, T phin, T L, T dt) {
  switch (mode) {
    case kRK1: return L * dt + phi;
    case kRK2a:
    case kRK3a: return phi + dt * L;
    case kRK2b: { T s = phi + dt * L; s += phin; return s * T(0.5); }
    case kRK3b: { T s = phi + dt * L; s += T(3.0) * phin; return s * T(0.25); }
    case kRK3c: { T s = phi + dt * L; s *= T(2.0); s += phin; return s * (T(1.0) / T(3.0)); }
    default: return L;
  }
}

// velocity term value at table columns (jx, jy, jz) in the order the
// separable descriptor defines it: ((coeff f0) f1) f2
template <int DIM, typename T>
__device__ __forceinline__ T term_val(const T* __restrict__ vx, const T* __restrict__ vy,
                                      const T* __restrict__ vz, int jx, int jy, int jz) {
  T v = vx[jx] * vy[jy];
  if constexpr (DIM == 3) v = v * vz[jz];
  return v;
}

// shared-memory footprint of the stage kernel
template <int DIM, int P, typename T>
__host__ __device__ inline size_t adv_smem_bytes(const int* tile, int n_terms) {
  constexpr int N1 = P + 1, NQ = P + 2, NM = ipow(N1, DIM), NPT = NQ + 2;
  const int bx = tile[0] + 2, by = DIM > 1 ? tile[1] + 2 : 1, bz = DIM > 2 ? tile[2] + 2 : 1;
  size_t box = (size_t)bx * by * bz * NM * sizeof(T);
  size_t vt = (size_t)n_terms * (tile[0] + tile[1] + (DIM > 2 ? tile[2] : 0)) * NPT * sizeof(T);
  return box + vt;
}

template <int DIM, int P, typename T>
__global__ void __launch_bounds__(256) adv_stage_kernel(const AdvArgs<T> a) {
  constexpr int N1 = P + 1, NQ = P + 2, NM = ipow(N1, DIM), NPT = NQ + 2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* box = reinterpret_cast<T*>(smem_raw);
  const MeshArgs& m = a.m;
  const int nboxc = box_cells(m, DIM);
  T* vt = box + (size_t)nboxc * NM;
  const Tab1D<T>& tb = tab<T>(P);
  const TileCoord tc = tile_coord(m, DIM);
  const int tx = m.tile[0], ty = m.tile[1], tz = m.tile[2];
  const int nterm = a.v.n_terms;

  // ---- stage velocity-table rows of this tile: vt[(k*3+axis)*span + i]*NPT
  {
    const int span = tx + ty + (DIM > 2 ? tz : 0);
    const int total = nterm * span * NPT;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      const int j = e % NPT;
      int r = e / NPT;
      const int li = r % span;
      const int k = r / span;
      int axis, gi;
      if (li < tx) { axis = 0; gi = tc.ox + li; }
      else if (li < tx + ty) { axis = 1; gi = tc.oy + (li - tx); }
      else { axis = 2; gi = tc.oz + (li - tx - ty); }
      gi = min(gi, m.n[axis] - 1);
      vt[(size_t)(k * span + li) * NPT + j] =
          a.v.vtab[((size_t)(k * 3 + axis) * a.v.nmax + gi) * a.v.npt + j];
    }
  }
  load_box<DIM, NM>(m, a.phi_s, box, tc.ox, tc.oy, tc.oz, true);
  __syncthreads();

  const T ct = a.clk ? T(a.clk->ct[a.stage]) : T(a.ct_explicit);
  const T dt = a.clk ? T(a.clk->dt) : T(a.dt_explicit);
  const bool active = a.clk ? (a.clk->active != 0) : true;

  T R[NM];
  T c[NM];
#pragma unroll
  for (int q = 0; q < NM; ++q) R[q] = T(0);
  const int span = tx + ty + (DIM > 2 ? tz : 0);
  const int me = box_index(m, DIM, tc.lx, tc.ly, tc.lz);
  const T ih0 = T(1.0 / m.h[0]), ih1 = T(1.0 / m.h[1]), ih2 = T(DIM > 2 ? 1.0 / m.h[2] : 1.0);

  if (tc.valid) {
#pragma unroll
    for (int q = 0; q < NM; ++q) c[q] = box[(size_t)me * NM + q];
  }
  if (tc.valid && active) {
    auto vrow = [&](int k, int axis) -> const T* {
      const int li = axis == 0 ? tc.lx : (axis == 1 ? tx + tc.ly : tx + ty + tc.lz);
      return vt + (size_t)(k * span + li) * NPT;
    };

    // ============================ cell term ============================
    if constexpr (DIM == 2) {
      T Pp[N1][NQ];  // Pp[a][qy] = sum_b c[a,b] L_b(y_qy)
#pragma unroll
      for (int aa = 0; aa < N1; ++aa)
#pragma unroll
        for (int qy = 0; qy < NQ; ++qy) {
          T s = T(0);
#pragma unroll
          for (int b = 0; b < N1; ++b) s += c[aa + N1 * b] * tb.Lq[b][qy];
          Pp[aa][qy] = s;
        }
#pragma unroll
      for (int qy = 0; qy < NQ; ++qy) {
        T X1[N1], X2[N1];
#pragma unroll
        for (int aa = 0; aa < N1; ++aa) { X1[aa] = T(0); X2[aa] = T(0); }
#pragma unroll
        for (int qx = 0; qx < NQ; ++qx) {
          T phi = T(0);
#pragma unroll
          for (int aa = 0; aa < N1; ++aa) phi += Pp[aa][qy] * tb.Lq[aa][qx];
          T u0 = T(0), u1 = T(0);
          for (int k = 0; k < nterm; ++k) {
            const T tv = term_val<2>(vrow(k, 0), vrow(k, 1), (const T*)nullptr, qx, qy, 0);
            if (a.v.comp[k] == 0) u0 += tv; else u1 += tv;
          }
          u0 *= ct;
          u1 *= ct;
          const T w = tb.wq[qx] * tb.wq[qy] * phi;
          const T fx = w * u0 * ih0, fy = w * u1 * ih1;
#pragma unroll
          for (int aa = 0; aa < N1; ++aa) {
            X1[aa] += fx * tb.Dq[aa][qx];
            X2[aa] += fy * tb.Lq[aa][qx];
          }
        }
#pragma unroll
        for (int b = 0; b < N1; ++b)
#pragma unroll
          for (int aa = 0; aa < N1; ++aa)
            R[aa + N1 * b] += X1[aa] * tb.Lq[b][qy] + X2[aa] * tb.Dq[b][qy];
      }
    } else {
      // Q1[a][b][qz] = sum_c c[a,b,c] L_c(z); Pp[a][qy][qz] = sum_b Q1 L_b(y)
      T Pp[N1][NQ][NQ];
      {
        T Q1[N1][N1][NQ];
#pragma unroll
        for (int aa = 0; aa < N1; ++aa)
#pragma unroll
          for (int b = 0; b < N1; ++b)
#pragma unroll
            for (int qz = 0; qz < NQ; ++qz) {
              T s = T(0);
#pragma unroll
              for (int cc = 0; cc < N1; ++cc) s += c[aa + N1 * (b + N1 * cc)] * tb.Lq[cc][qz];
              Q1[aa][b][qz] = s;
            }
#pragma unroll
        for (int aa = 0; aa < N1; ++aa)
#pragma unroll
          for (int qy = 0; qy < NQ; ++qy)
#pragma unroll
            for (int qz = 0; qz < NQ; ++qz) {
              T s = T(0);
#pragma unroll
              for (int b = 0; b < N1; ++b) s += Q1[aa][b][qz] * tb.Lq[b][qy];
              Pp[aa][qy][qz] = s;
            }
      }
#pragma unroll 1
      for (int qz = 0; qz < NQ; ++qz) {
        T U1[N1][N1], U3[N1][N1];
#pragma unroll
        for (int aa = 0; aa < N1; ++aa)
#pragma unroll
          for (int b = 0; b < N1; ++b) { U1[aa][b] = T(0); U3[aa][b] = T(0); }
#pragma unroll
        for (int qy = 0; qy < NQ; ++qy) {
          T X1[N1], X2[N1], X3[N1];
#pragma unroll
          for (int aa = 0; aa < N1; ++aa) { X1[aa] = T(0); X2[aa] = T(0); X3[aa] = T(0); }
#pragma unroll
          for (int qx = 0; qx < NQ; ++qx) {
            T phi = T(0);
#pragma unroll
            for (int aa = 0; aa < N1; ++aa) phi += Pp[aa][qy][qz] * tb.Lq[aa][qx];
            T u0 = T(0), u1 = T(0), u2 = T(0);
            for (int k = 0; k < nterm; ++k) {
              const T tv = term_val<3>(vrow(k, 0), vrow(k, 1), vrow(k, 2), qx, qy, qz);
              const int cp = a.v.comp[k];
              if (cp == 0) u0 += tv; else if (cp == 1) u1 += tv; else u2 += tv;
            }
            u0 *= ct;
            u1 *= ct;
            u2 *= ct;
            const T w = tb.wq[qx] * tb.wq[qy] * tb.wq[qz] * phi;
            const T fx = w * u0 * ih0, fy = w * u1 * ih1, fz = w * u2 * ih2;
#pragma unroll
            for (int aa = 0; aa < N1; ++aa) {
              X1[aa] += fx * tb.Dq[aa][qx];
              X2[aa] += fy * tb.Lq[aa][qx];
              X3[aa] += fz * tb.Lq[aa][qx];
            }
          }
#pragma unroll
          for (int b = 0; b < N1; ++b)
#pragma unroll
            for (int aa = 0; aa < N1; ++aa) {
              U1[aa][b] += X1[aa] * tb.Lq[b][qy] + X2[aa] * tb.Dq[b][qy];
              U3[aa][b] += X3[aa] * tb.Lq[b][qy];
            }
        }
#pragma unroll
        for (int cc = 0; cc < N1; ++cc)
#pragma unroll
          for (int b = 0; b < N1; ++b)
#pragma unroll
            for (int aa = 0; aa < N1; ++aa)
              R[aa + N1 * (b + N1 * cc)] += U1[aa][b] * tb.Lq[cc][qz] + U3[aa][b] * tb.Dq[cc][qz];
      }
    }

    // ============================ faces ============================
    constexpr int NF = ipow(N1, DIM - 1);   // face modes
    // fully unrolled: face axis and side are compile-time, so every modal
    // index below is static and c / R stay in registers
#pragma unroll
    for (int f = 0; f < 2 * DIM; ++f) {
      const int e = f >> 1, s = f & 1;
      int nl[3] = {tc.lx, tc.ly, tc.lz};
      int ng[3] = {tc.gx, tc.gy, tc.gz};
      nl[e] += s ? 1 : -1;
      ng[e] += s ? 1 : -1;
      const bool has_nb = ng[e] >= 0 && ng[e] < m.n[e];
      const T* cn = box + (size_t)box_index(m, DIM, nl[0], nl[1], nl[2]) * NM;
      // traces on the face (modes of the tangential axes, t0 < t1)
      const int t0 = e == 0 ? 1 : 0;
      const int t1 = e == 2 ? 1 : 2;
      const int st[3] = {1, N1, N1 * N1};
      T tin[NF], tex[NF];
#pragma unroll
      for (int mf = 0; mf < NF; ++mf) {
        const int m0 = mf % N1, m1 = DIM > 2 ? mf / N1 : 0;
        const int base = m0 * st[t0] + (DIM > 2 ? m1 * st[t1] : 0);
        T si = T(0), sx = T(0);
#pragma unroll
        for (int aa = 0; aa < N1; ++aa) {
          const T li = s ? tb.L1[aa] : tb.L0[aa];
          const T lx = s ? tb.L0[aa] : tb.L1[aa];
          si += li * c[base + aa * st[e]];
          if (has_nb) sx += lx * cn[base + aa * st[e]];
        }
        tin[mf] = si;
        tex[mf] = has_nb ? sx : si;
      }
      // flux at face points, projected back onto the face modes
      T Fm[NF];
#pragma unroll
      for (int mf = 0; mf < NF; ++mf) Fm[mf] = T(0);
      const T ihe = e == 0 ? ih0 : (e == 1 ? ih1 : ih2);
      constexpr int NQF = ipow(NQ, DIM - 1);
#pragma unroll
      for (int qf = 0; qf < NQF; ++qf) {
        const int q0 = qf % NQ, q1 = DIM > 2 ? qf / NQ : 0;
        T pin = T(0), pex = T(0);
#pragma unroll
        for (int mf = 0; mf < NF; ++mf) {
          const int m0 = mf % N1, m1 = DIM > 2 ? mf / N1 : 0;
          T bw = tb.Lq[m0][q0];
          if constexpr (DIM > 2) bw = bw * tb.Lq[m1][q1];
          pin += tin[mf] * bw;
          pex += tex[mf] * bw;
        }
        // normal velocity at the face point
        int j[3];
        j[e] = NQ + s;
        j[t0] = q0;
        if constexpr (DIM > 2) j[t1] = q1;
        T ue = T(0);
        for (int k = 0; k < nterm; ++k) {
          if (a.v.comp[k] != e) continue;
          ue += term_val<DIM>(vrow(k, 0), vrow(k, 1), DIM > 2 ? vrow(k, 2) : nullptr, j[0], j[1],
                              DIM > 2 ? j[2] : 0);
        }
        ue *= ct;
        const T vn = s ? ue : -ue;
        const T up = vn > T(0) ? pin : pex;
        T w = tb.wq[q0];
        if constexpr (DIM > 2) w = w * tb.wq[q1];
        const T F = vn * up * w * ihe;
#pragma unroll
        for (int mf = 0; mf < NF; ++mf) {
          const int m0 = mf % N1, m1 = DIM > 2 ? mf / N1 : 0;
          T bw = tb.Lq[m0][q0];
          if constexpr (DIM > 2) bw = bw * tb.Lq[m1][q1];
          Fm[mf] += F * bw;
        }
      }
#pragma unroll
      for (int mf = 0; mf < NF; ++mf) {
        const int m0 = mf % N1, m1 = DIM > 2 ? mf / N1 : 0;
        const int base = m0 * st[t0] + (DIM > 2 ? m1 * st[t1] : 0);
#pragma unroll
        for (int aa = 0; aa < N1; ++aa) {
          const T li = s ? tb.L1[aa] : tb.L0[aa];
          R[base + aa * st[e]] -= li * Fm[mf];
        }
      }
    }
  }

  // ---- combine with phi^n and store through shared memory (coalesced)
  __syncthreads();
  const int ntile_cells = tx * ty * tz;
  T* stage_buf = box;  // reuse: [tile cell][NM]
  const bool need_n = a.combine == kRK2b || a.combine == kRK3b || a.combine == kRK3c;
  if (need_n) {
    const int total = ntile_cells * NM;
    for (int e2 = threadIdx.x; e2 < total; e2 += blockDim.x) {
      const int q = e2 % NM, cl = e2 / NM;
      const int lx = cl % tx, ly = (cl / tx) % ty, lz = cl / (tx * ty);
      const int gx = tc.ox + lx, gy = tc.oy + ly, gz = tc.oz + lz;
      T v = T(0);
      const int gi = m.q2g[q];
      if (gx < m.n[0] && gy < m.n[1] && gz < m.n[2] && gi >= 0)
        v = a.phi_n[((long long)gx + (long long)m.n[0] * (gy + (long long)m.n[1] * gz)) * m.nb + gi];
      stage_buf[e2] = v;
    }
    __syncthreads();
  }
  if (tc.valid) {
    const int cl = tc.lx + tx * (tc.ly + ty * tc.lz);
#pragma unroll
    for (int q = 0; q < NM; ++q) {
      // an inactive (zero-length) substep passes the stage input through
      T res = c[q];
      if (active) {
        const T pn = need_n ? stage_buf[(size_t)cl * NM + q] : T(0);
        res = combine_value<T>(a.combine, c[q], pn, R[q], dt);
      }
      stage_buf[(size_t)cl * NM + q] = res;
    }
  }
  __syncthreads();
  {
    const int total = ntile_cells * m.nb;
    for (int e2 = threadIdx.x; e2 < total; e2 += blockDim.x) {
      const int k = e2 % m.nb, cl = e2 / m.nb;
      const int lx = cl % tx, ly = (cl / tx) % ty, lz = cl / (tx * ty);
      const int gx = tc.ox + lx, gy = tc.oy + ly, gz = tc.oz + lz;
      if (gx >= m.n[0] || gy >= m.n[1] || gz >= m.n[2]) continue;
      const int q = m.g2q[k];
      a.out[((long long)gx + (long long)m.n[0] * (gy + (long long)m.n[1] * gz)) * m.nb + k] =
          stage_buf[(size_t)cl * NM + q];
    }
  }
}

}  // namespace flsp

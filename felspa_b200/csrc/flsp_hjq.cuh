// flsp_hjq.cuh — Hamilton-Jacobi reinitialisation pseudo-step, tensor-
// product (FE_DGQLegendre) basis, sum-factorised.
//
// Same operator as flsp_hj.cuh (see there for the reference functions it
// replaces) restated for speed.  Integrating the LDG cell term by parts
// (A_ab = L_a(1)L_b(1) - L_a(0)L_b(0) - A_ba) turns the one-sided gradients
// into the broken gradient plus a lifted face jump:
//   g^L_d(x) = d_d phi(x) + (1/h_d) K0(xi_d) [phi]_lo,d(x_perp)
//   g^R_d(x) = d_d phi(x) + (1/h_d) K1(xi_d) [phi]_hi,d(x_perp)
// with K_s(xi) = sum_a L_a(xi) L_a(s), [phi]_lo = phi_own - phi_lower on the
// lower face, [phi]_hi = phi_upper - phi_own on the upper face, both zero on
// the domain boundary (interior trace).  This holds line by line for the Q
// space; the P space has mode-dependent kernels and uses flsp_hj.cuh.
//
// One thread per cell.  Per cell: the 2*dim face jumps at the face Gauss
// points (shared memory, transposed [slot][thread]), the vertex CFL data,
// then one pass over z-planes / y-lines / x-points that builds d phi and
// phi0, grad phi0 by sum factorisation, evaluates H and projects back.
#pragma once
#include "flsp_device.cuh"
#include "flsp_hj.cuh"

namespace flsp {

template <int DIM, int P, typename T>
__host__ __device__ inline size_t hjq_smem_bytes(const int* tile) {
  constexpr int N1 = P + 1, NQ = P + 2, NM = ipow(N1, DIM), NQF = ipow(NQ, DIM - 1);
  const int bx = tile[0] + 2, by = DIM > 1 ? tile[1] + 2 : 1, bz = DIM > 2 ? tile[2] + 2 : 1;
  const int nt = tile[0] * tile[1] * (DIM > 2 ? tile[2] : 1);
  size_t box = (size_t)bx * by * bz * NM * sizeof(T);
  size_t c0 = (size_t)(nt + 1) * NM * sizeof(T);
  size_t jn = (size_t)nt * 2 * DIM * NQF * sizeof(T);
  return box + c0 + jn + 64 * sizeof(double) + 16;
}

// values at the 2^dim vertices of the modal field c (Q layout), each axis
// using the given 1D tables at xi = 0 / xi = 1 (L or L')
template <int DIM, int N1, typename T>
__device__ __forceinline__ void vertex_eval(const T* c, const T* x0, const T* x1, const T* y0,
                                            const T* y1, const T* z0, const T* z1,
                                            T out[1 << DIM]) {
  if constexpr (DIM == 2) {
    T yv[2][N1];
#pragma unroll
    for (int a = 0; a < N1; ++a) {
      T s0 = T(0), s1 = T(0);
#pragma unroll
      for (int b = 0; b < N1; ++b) {
        s0 += c[a + N1 * b] * y0[b];
        s1 += c[a + N1 * b] * y1[b];
      }
      yv[0][a] = s0;
      yv[1][a] = s1;
    }
#pragma unroll
    for (int vy = 0; vy < 2; ++vy) {
      T s0 = T(0), s1 = T(0);
#pragma unroll
      for (int a = 0; a < N1; ++a) {
        s0 += yv[vy][a] * x0[a];
        s1 += yv[vy][a] * x1[a];
      }
      out[0 + 2 * vy] = s0;
      out[1 + 2 * vy] = s1;
    }
  } else {
    T zv[2][N1][N1];
#pragma unroll
    for (int a = 0; a < N1; ++a)
#pragma unroll
      for (int b = 0; b < N1; ++b) {
        T s0 = T(0), s1 = T(0);
#pragma unroll
        for (int cc = 0; cc < N1; ++cc) {
          s0 += c[a + N1 * (b + N1 * cc)] * z0[cc];
          s1 += c[a + N1 * (b + N1 * cc)] * z1[cc];
        }
        zv[0][a][b] = s0;
        zv[1][a][b] = s1;
      }
#pragma unroll
    for (int vz = 0; vz < 2; ++vz)
#pragma unroll
      for (int vy = 0; vy < 2; ++vy) {
        T yv[N1];
#pragma unroll
        for (int a = 0; a < N1; ++a) {
          T s = T(0);
#pragma unroll
          for (int b = 0; b < N1; ++b) s += zv[vz][a][b] * (vy ? y1[b] : y0[b]);
          yv[a] = s;
        }
        T s0 = T(0), s1 = T(0);
#pragma unroll
        for (int a = 0; a < N1; ++a) {
          s0 += yv[a] * x0[a];
          s1 += yv[a] * x1[a];
        }
        out[0 + 2 * vy + 4 * vz] = s0;
        out[1 + 2 * vy + 4 * vz] = s1;
      }
  }
}

template <int DIM, int P, typename T>
__device__ __forceinline__ void hjq_tile(const HJArgs<T>& a, int slot) {
  constexpr int N1 = P + 1, NQ = P + 2, NM = ipow(N1, DIM), NV = 1 << DIM;
  constexpr int NF = ipow(N1, DIM - 1), NQF = ipow(NQ, DIM - 1), NC = 1 << (DIM - 1);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const MeshArgs& m = a.m;
  T* box = reinterpret_cast<T*>(smem_raw);
  const int nboxc = box_cells(m, DIM);
  const int tx = m.tile[0], ty = m.tile[1], tz = m.tile[2];
  const int nt = tx * ty * tz;
  const int ntp = nt + 1;                    // padded stride: conflict-free transposed stores
  T* c0s = box + (size_t)nboxc * NM;        // [NM][nt + 1]
  T* jn = c0s + (size_t)ntp * NM;           // [2*DIM*NQF][nt]
  double* red = align16<double>(jn + (size_t)nt * 2 * DIM * NQF);
  const Tab1D<T>& tb = tab<T>(P);
  if (tile_inactive(m, slot)) return;
  const TileCoord tc = tile_coord(m, DIM, slot);

  load_box<DIM, NM>(m, a.phi, box, tc.ox, tc.oy, tc.oz, true);
  load_tile<DIM, NM>(m, a.phi0, c0s, tc.ox, tc.oy, tc.oz, true, ntp);
  cp_async_wait_all();
  __syncthreads();

  const int cl = tc.lx + tx * (tc.ly + ty * tc.lz);
  constexpr int st[3] = {1, N1, N1 * N1};
  const T ih[3] = {T(1.0 / m.h[0]), T(1.0 / m.h[1]), T(DIM > 2 ? 1.0 / m.h[2] : 1.0)};
  const T hmin = T(m.min_diam);
  const T dt = a.clk ? T(a.clk->hj_dt) : T(a.dt_explicit);
  double vmax = 0.0;
  T R[NM];
  const T* c = box + (size_t)box_index(m, DIM, tc.lx, tc.ly, tc.lz) * NM;

  if (tc.valid) {
    // -------- face jumps: nodal at face points (smem), corners (registers)
    T jv[2 * DIM][NC];
    const int g[3] = {tc.gx, tc.gy, tc.gz};
    const int l[3] = {tc.lx, tc.ly, tc.lz};
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      const int t0 = d == 0 ? 1 : 0, t1 = d == 2 ? 1 : 2;
      int ll[3] = {l[0], l[1], l[2]}, lu[3] = {l[0], l[1], l[2]};
      ll[d] -= 1;
      lu[d] += 1;
      const bool has_lo = g[d] > 0, has_hi = g[d] + 1 < m.n[d];
      T glo = T(0), ghi = T(0);
      const bool dlo = !has_lo && bc_dirichlet<DIM>(m, d, 0, g, glo);
      const bool dhi = !has_hi && bc_dirichlet<DIM>(m, d, 1, g, ghi);
      const T* cL = box + (size_t)box_index(m, DIM, ll[0], ll[1], ll[2]) * NM;
      const T* cU = box + (size_t)box_index(m, DIM, lu[0], lu[1], lu[2]) * NM;
      T jlo[NF], jhi[NF];
#pragma unroll
      for (int mf = 0; mf < NF; ++mf) {
        const int m0 = mf % N1, m1 = mf / N1;
        const int base = m0 * st[t0] + (DIM > 2 ? m1 * st[t1] : 0);
        T tlo = T(0), tup = T(0), tnl = T(0), tnu = T(0);
#pragma unroll
        for (int b = 0; b < N1; ++b) {
          const T cb = c[base + b * st[d]];
          tlo += tb.L0[b] * cb;
          tup += tb.L1[b] * cb;
          if (has_lo) tnl += tb.L1[b] * cL[base + b * st[d]];
          if (has_hi) tnu += tb.L0[b] * cU[base + b * st[d]];
        }
        // domain boundary: jump to the Dirichlet value of the face (constant
        // mode only) where it carries one, else zero (interior trace)
        jlo[mf] = has_lo ? tlo - tnl : (dlo ? tlo - (mf == 0 ? glo : T(0)) : T(0));
        jhi[mf] = has_hi ? tnu - tup : (dhi ? (mf == 0 ? ghi : T(0)) - tup : T(0));
      }
#pragma unroll
      for (int side = 0; side < 2; ++side) {
        const T* J = side ? jhi : jlo;
        // nodal values at the face Gauss points, t0 fastest
        if constexpr (DIM == 2) {
#pragma unroll
          for (int q0 = 0; q0 < NQ; ++q0) {
            T s = T(0);
#pragma unroll
            for (int m0 = 0; m0 < N1; ++m0) s += J[m0] * tb.Lq[m0][q0];
            jn[(size_t)((2 * d + side) * NQF + q0) * nt + cl] = s;
          }
#pragma unroll
          for (int cr = 0; cr < 2; ++cr) {
            T s = T(0);
#pragma unroll
            for (int m0 = 0; m0 < N1; ++m0) s += J[m0] * (cr ? tb.L1[m0] : tb.L0[m0]);
            jv[2 * d + side][cr] = s;
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
              jn[(size_t)((2 * d + side) * NQF + q0 + NQ * q1) * nt + cl] = s;
            }
#pragma unroll
          for (int cr = 0; cr < 4; ++cr) {
            T s = T(0);
#pragma unroll
            for (int mf = 0; mf < NF; ++mf) {
              const int m0 = mf % N1, m1 = mf / N1;
              s += J[mf] * ((cr & 1) ? tb.L1[m0] : tb.L0[m0]) * ((cr & 2) ? tb.L1[m1] : tb.L0[m1]);
            }
            jv[2 * d + side][cr] = s;
          }
        }
      }
    }

    // -------- vertex CFL estimate for the next pseudo-step
    {
      T own[NM], own0[NM];
#pragma unroll
      for (int q = 0; q < NM; ++q) { own[q] = c[q]; own0[q] = c0s[(size_t)q * ntp + cl]; }
      T dphi[DIM][NV], p0v[NV], g0v[DIM][NV];
      vertex_eval<DIM, N1, T>(own, tb.D0, tb.D1, tb.L0, tb.L1, tb.L0, tb.L1, dphi[0]);
      vertex_eval<DIM, N1, T>(own, tb.L0, tb.L1, tb.D0, tb.D1, tb.L0, tb.L1, dphi[1]);
      vertex_eval<DIM, N1, T>(own0, tb.L0, tb.L1, tb.L0, tb.L1, tb.L0, tb.L1, p0v);
      vertex_eval<DIM, N1, T>(own0, tb.D0, tb.D1, tb.L0, tb.L1, tb.L0, tb.L1, g0v[0]);
      vertex_eval<DIM, N1, T>(own0, tb.L0, tb.L1, tb.D0, tb.D1, tb.L0, tb.L1, g0v[1]);
      if constexpr (DIM == 3) {
        vertex_eval<DIM, N1, T>(own, tb.L0, tb.L1, tb.L0, tb.L1, tb.D0, tb.D1, dphi[2]);
        vertex_eval<DIM, N1, T>(own0, tb.L0, tb.L1, tb.L0, tb.L1, tb.D0, tb.D1, g0v[2]);
      }
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        const int vb[3] = {v & 1, (v >> 1) & 1, (v >> 2) & 1};
        T g2 = T(0);
#pragma unroll
        for (int d = 0; d < DIM; ++d) { const T gg = g0v[d][v] * ih[d]; g2 += gg * gg; }
        const T gn = sqrt(g2);
        const T S = p0v[v] / sqrt(p0v[v] * p0v[v] + hmin * hmin * gn * gn);
        T gs[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
          const int t0 = d == 0 ? 1 : 0, t1 = d == 2 ? 1 : 2;
          const int cr = vb[t0] + (DIM > 2 ? 2 * vb[t1] : 0);
          const T gd = dphi[d][v] * ih[d];
          const T L = gd + ih[d] * tb.K0v[vb[d]] * jv[2 * d][cr];
          const T Rr = gd + ih[d] * tb.K1v[vb[d]] * jv[2 * d + 1][cr];
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
      vmax = vmax / m.diam;
    }

    // -------- pseudo-step: H at the cell Gauss points, projected back
    if (a.mode == kHJStep) {
#pragma unroll
      for (int q = 0; q < NM; ++q) R[q] = T(0);
      auto jnv = [&](int d, int side, int qf) -> T { return jn[(size_t)((2 * d + side) * NQF + qf) * nt + cl]; };
      auto hfun = [&](T p0, T g0x, T g0y, T g0z, const T* lft, const T* rgt) -> T {
        T g2 = g0x * g0x + g0y * g0y;
        if constexpr (DIM == 3) g2 += g0z * g0z;
        T S, nrm;
        T avg2 = T(0);
#pragma unroll
        for (int d = 0; d < DIM; ++d) { const T av = T(0.5) * (lft[d] + rgt[d]); avg2 += av * av; }
        if constexpr (sizeof(T) == 4) {
          // production FP32: hardware reciprocal square roots
          S = p0 * rsqrtf(p0 * p0 + hmin * hmin * g2);
          nrm = avg2 * rsqrtf(fmaxf(avg2, 1e-30f));
        } else {
          // FP64: the reference's operation sequence (reinit.cc:121-191)
          const T gn = sqrt(g2);
          S = p0 / sqrt(p0 * p0 + hmin * hmin * gn * gn);
          nrm = sqrt(avg2);
        }
        T H = S * (nrm - T(1));
#pragma unroll
        for (int d = 0; d < DIM; ++d) H += T(0.5) * fabs(S) * (lft[d] - rgt[d]);
        return H;
      };
      if constexpr (DIM == 2) {
#pragma unroll 1
        for (int qy = 0; qy < NQ; ++qy) {
          T Py[N1], Pdy[N1], P0y[N1], P0dy[N1];
#pragma unroll
          for (int aa = 0; aa < N1; ++aa) {
            T s1 = T(0), s2 = T(0), s3 = T(0), s4 = T(0);
#pragma unroll
            for (int b = 0; b < N1; ++b) {
              const T cv = c[aa + N1 * b], c0v = c0s[(size_t)(aa + N1 * b) * ntp + cl];
              s1 += cv * tb.Lq[b][qy];
              s2 += cv * tb.Dq[b][qy];
              s3 += c0v * tb.Lq[b][qy];
              s4 += c0v * tb.Dq[b][qy];
            }
            Py[aa] = s1; Pdy[aa] = s2; P0y[aa] = s3; P0dy[aa] = s4;
          }
          const T jlx = jnv(0, 0, qy), jhx = jnv(0, 1, qy);
          T X[N1];
#pragma unroll
          for (int aa = 0; aa < N1; ++aa) X[aa] = T(0);
#pragma unroll
          for (int qx = 0; qx < NQ; ++qx) {
            T gx = T(0), gy = T(0), p0 = T(0), g0x = T(0), g0y = T(0);
#pragma unroll
            for (int aa = 0; aa < N1; ++aa) {
              gx += Py[aa] * tb.Dq[aa][qx];
              gy += Pdy[aa] * tb.Lq[aa][qx];
              p0 += P0y[aa] * tb.Lq[aa][qx];
              g0x += P0y[aa] * tb.Dq[aa][qx];
              g0y += P0dy[aa] * tb.Lq[aa][qx];
            }
            gx *= ih[0]; gy *= ih[1]; g0x *= ih[0]; g0y *= ih[1];
            const T jly = jnv(1, 0, qx), jhy = jnv(1, 1, qx);
            const T lft[2] = {gx + ih[0] * tb.K0q[qx] * jlx, gy + ih[1] * tb.K0q[qy] * jly};
            const T rgt[2] = {gx + ih[0] * tb.K1q[qx] * jhx, gy + ih[1] * tb.K1q[qy] * jhy};
            const T H = hfun(p0, g0x, g0y, T(0), lft, rgt);
            const T wH = tb.wq[qx] * tb.wq[qy] * H;
#pragma unroll
            for (int aa = 0; aa < N1; ++aa) X[aa] += wH * tb.Lq[aa][qx];
          }
#pragma unroll
          for (int b = 0; b < N1; ++b)
#pragma unroll
            for (int aa = 0; aa < N1; ++aa) R[aa + N1 * b] -= X[aa] * tb.Lq[b][qy];
        }
      } else {
#pragma unroll 1
        for (int qz = 0; qz < NQ; ++qz) {
          T Pz[N1][N1], Dz[N1][N1], P0z[N1][N1], D0z[N1][N1];
#pragma unroll
          for (int aa = 0; aa < N1; ++aa)
#pragma unroll
            for (int b = 0; b < N1; ++b) {
              T s1 = T(0), s2 = T(0), s3 = T(0), s4 = T(0);
#pragma unroll
              for (int cc = 0; cc < N1; ++cc) {
                const int q = aa + N1 * (b + N1 * cc);
                const T cv = c[q], c0v = c0s[(size_t)q * ntp + cl];
                s1 += cv * tb.Lq[cc][qz];
                s2 += cv * tb.Dq[cc][qz];
                s3 += c0v * tb.Lq[cc][qz];
                s4 += c0v * tb.Dq[cc][qz];
              }
              Pz[aa][b] = s1; Dz[aa][b] = s2; P0z[aa][b] = s3; D0z[aa][b] = s4;
            }
          T U[N1][N1];
#pragma unroll
          for (int aa = 0; aa < N1; ++aa)
#pragma unroll
            for (int b = 0; b < N1; ++b) U[aa][b] = T(0);
#pragma unroll 1
          for (int qy = 0; qy < NQ; ++qy) {
            T Py[N1], Pdy[N1], Dzy[N1], P0y[N1], P0dy[N1], D0zy[N1];
#pragma unroll
            for (int aa = 0; aa < N1; ++aa) {
              T s1 = T(0), s2 = T(0), s3 = T(0), s4 = T(0), s5 = T(0), s6 = T(0);
#pragma unroll
              for (int b = 0; b < N1; ++b) {
                s1 += Pz[aa][b] * tb.Lq[b][qy];
                s2 += Pz[aa][b] * tb.Dq[b][qy];
                s3 += Dz[aa][b] * tb.Lq[b][qy];
                s4 += P0z[aa][b] * tb.Lq[b][qy];
                s5 += P0z[aa][b] * tb.Dq[b][qy];
                s6 += D0z[aa][b] * tb.Lq[b][qy];
              }
              Py[aa] = s1; Pdy[aa] = s2; Dzy[aa] = s3; P0y[aa] = s4; P0dy[aa] = s5; D0zy[aa] = s6;
            }
            const T jlx = jnv(0, 0, qy + NQ * qz), jhx = jnv(0, 1, qy + NQ * qz);
            T X[N1];
#pragma unroll
            for (int aa = 0; aa < N1; ++aa) X[aa] = T(0);
#pragma unroll
            for (int qx = 0; qx < NQ; ++qx) {
              T gx = T(0), gy = T(0), gz = T(0), p0 = T(0), g0x = T(0), g0y = T(0), g0z = T(0);
#pragma unroll
              for (int aa = 0; aa < N1; ++aa) {
                gx += Py[aa] * tb.Dq[aa][qx];
                gy += Pdy[aa] * tb.Lq[aa][qx];
                gz += Dzy[aa] * tb.Lq[aa][qx];
                p0 += P0y[aa] * tb.Lq[aa][qx];
                g0x += P0y[aa] * tb.Dq[aa][qx];
                g0y += P0dy[aa] * tb.Lq[aa][qx];
                g0z += D0zy[aa] * tb.Lq[aa][qx];
              }
              gx *= ih[0]; gy *= ih[1]; gz *= ih[2];
              g0x *= ih[0]; g0y *= ih[1]; g0z *= ih[2];
              const T jly = jnv(1, 0, qx + NQ * qz), jhy = jnv(1, 1, qx + NQ * qz);
              const T jlz = jnv(2, 0, qx + NQ * qy), jhz = jnv(2, 1, qx + NQ * qy);
              const T lft[3] = {gx + ih[0] * tb.K0q[qx] * jlx, gy + ih[1] * tb.K0q[qy] * jly,
                                gz + ih[2] * tb.K0q[qz] * jlz};
              const T rgt[3] = {gx + ih[0] * tb.K1q[qx] * jhx, gy + ih[1] * tb.K1q[qy] * jhy,
                                gz + ih[2] * tb.K1q[qz] * jhz};
              const T H = hfun(p0, g0x, g0y, g0z, lft, rgt);
              const T wH = tb.wq[qx] * tb.wq[qy] * tb.wq[qz] * H;
#pragma unroll
              for (int aa = 0; aa < N1; ++aa) X[aa] += wH * tb.Lq[aa][qx];
            }
#pragma unroll
            for (int b = 0; b < N1; ++b)
#pragma unroll
              for (int aa = 0; aa < N1; ++aa) U[aa][b] += X[aa] * tb.Lq[b][qy];
          }
#pragma unroll
          for (int cc = 0; cc < N1; ++cc)
#pragma unroll
            for (int b = 0; b < N1; ++b)
#pragma unroll
              for (int aa = 0; aa < N1; ++aa) R[aa + N1 * (b + N1 * cc)] -= U[aa][b] * tb.Lq[cc][qz];
        }
      }
    }
  }

  const double bm = block_max(vmax, red);
  if (threadIdx.x == 0 && a.clk) atomic_max_pos(&a.clk->hj_vd_bits, bm);
  if (a.mode != kHJStep) return;

  // update, staged through shared memory (the phi0 area) for coalesced stores
  __syncthreads();
  T* sb = c0s;   // [nt][NM] now
  if (tc.valid) {
    add_rdiff<NM>(m, a.rdiff, (long long)tc.gx + (long long)m.n[0] * (tc.gy + (long long)m.n[1] * tc.gz), R);
#pragma unroll
    for (int q = 0; q < NM; ++q) sb[(size_t)cl * NM + q] = hj_combine<T>(a.rk, c[q], R[q], dt);
  }
  __syncthreads();
  store_tile<DIM, NM>(m, sb, a.out, tc.ox, tc.oy, tc.oz);
}

}  // namespace flsp

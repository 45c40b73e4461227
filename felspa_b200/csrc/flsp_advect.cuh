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
#include <type_traits>

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

// shared-memory footprint of the stage kernel: tile box with face halo,
// velocity-table rows of the tile, upper-face fluxes shared with the
// upper neighbours
// tab: the velocity is read from the velocity tables (VelArgs::tab_q /
// tab_f), no velocity rows in shared memory
template <int DIM, int P, typename T>
__host__ __device__ inline size_t adv_smem_bytes(const int* tile, int n_terms, bool tab = false) {
  constexpr int N1 = P + 1, NQ = P + 2, NM = ipow(N1, DIM), NPT = NQ + 2, NF = ipow(N1, DIM - 1);
  const int bx = tile[0] + 2, by = DIM > 1 ? tile[1] + 2 : 1, bz = DIM > 2 ? tile[2] + 2 : 1;
  const int nt = tile[0] * tile[1] * (DIM > 2 ? tile[2] : 1);
  size_t box = (size_t)bx * by * bz * NM * sizeof(T);
  size_t vt = tab ? 0 : (size_t)n_terms * (tile[0] + tile[1] + (DIM > 2 ? tile[2] : 0)) * NPT * sizeof(T);
  size_t fl = (size_t)DIM * NF * nt * sizeof(T);
  return box + vt + fl;
}

// Upwind flux through face (E, S) of a cell (S = 1: upper face, outward
// normal +e_E), projected onto the face modes:
//   Fm[m] = sum_q w_q v_n(q) phi_hat(q) L_m(q),  v_n = (S ? 1 : -1) u_E,
//   phi_hat = v_n > 0 ? own trace : neighbour trace; on the domain
// boundary the neighbour trace is the Dirichlet value `gd` where the face
// carries one (dir), else the own trace (zero-Neumann inflow,
// advection.implement.h:719-741).
// vel_e(q0, q1) returns the weighted normal component u_E(q) w_q (w_q > 0,
// so its sign is the sign of u_E).
template <int DIM, int P, int E, int S, typename T, typename VelE>
__device__ __forceinline__ void face_flux(const Tab1D<T>& tb, const T* c, const T* cn, bool has_nb,
                                          VelE&& vel_e, T* Fm, bool dir = false, T gd = T(0)) {
  constexpr int N1 = P + 1, NQ = P + 2, NF = ipow(N1, DIM - 1);
  constexpr int t0 = E == 0 ? 1 : 0, t1 = E == 2 ? 1 : 2;
  constexpr int st[3] = {1, N1, N1 * N1};
  T tin[NF], tex[NF];
#pragma unroll
  for (int mf = 0; mf < NF; ++mf) {
    const int m0 = mf % N1, m1 = mf / N1;
    const int base = m0 * st[t0] + (DIM > 2 ? m1 * st[t1] : 0);
    T si = T(0), sx = T(0);
#pragma unroll
    for (int a = 0; a < N1; ++a) {
      si += (S ? tb.L1[a] : tb.L0[a]) * c[base + a * st[E]];
      if (has_nb) sx += (S ? tb.L0[a] : tb.L1[a]) * cn[base + a * st[E]];
    }
    tin[mf] = si;
    tex[mf] = has_nb ? sx : (dir ? (mf == 0 ? gd : T(0)) : si);
  }
  if constexpr (DIM == 2) {
#pragma unroll
    for (int m0 = 0; m0 < N1; ++m0) Fm[m0] = T(0);
#pragma unroll
    for (int q0 = 0; q0 < NQ; ++q0) {
      T pin = T(0), pex = T(0);
#pragma unroll
      for (int m0 = 0; m0 < N1; ++m0) {
        pin += tin[m0] * tb.Lq[m0][q0];
        pex += tex[m0] * tb.Lq[m0][q0];
      }
      const T uw = vel_e(q0, 0);
      const T vn = S ? uw : -uw;
      const T up = vn > T(0) ? pin : pex;
      const T F = vn * up;
#pragma unroll
      for (int m0 = 0; m0 < N1; ++m0) Fm[m0] += F * tb.Lq[m0][q0];
    }
  } else {
    T Pi[NQ][N1], Pe[NQ][N1];
#pragma unroll
    for (int q0 = 0; q0 < NQ; ++q0)
#pragma unroll
      for (int m1 = 0; m1 < N1; ++m1) {
        T si = T(0), sx = T(0);
#pragma unroll
        for (int m0 = 0; m0 < N1; ++m0) {
          si += tin[m0 + N1 * m1] * tb.Lq[m0][q0];
          sx += tex[m0 + N1 * m1] * tb.Lq[m0][q0];
        }
        Pi[q0][m1] = si;
        Pe[q0][m1] = sx;
      }
#pragma unroll
    for (int mf = 0; mf < NF; ++mf) Fm[mf] = T(0);
    // one q1 line at a time (not unrolled: the body is inlined for every
    // face of the cell), Fm[m0 + N1 m1] = sum_q1 G[m0](q1) L_m1(q1)
#pragma unroll 1
    for (int q1 = 0; q1 < NQ; ++q1) {
      T G[N1];
#pragma unroll
      for (int m0 = 0; m0 < N1; ++m0) G[m0] = T(0);
#pragma unroll
      for (int q0 = 0; q0 < NQ; ++q0) {
        T pin = T(0), pex = T(0);
#pragma unroll
        for (int m1 = 0; m1 < N1; ++m1) {
          pin += Pi[q0][m1] * tb.Lq[m1][q1];
          pex += Pe[q0][m1] * tb.Lq[m1][q1];
        }
        const T uw = vel_e(q0, q1);
        const T vn = S ? uw : -uw;
        const T up = vn > T(0) ? pin : pex;
        const T F = vn * up;
#pragma unroll
        for (int m0 = 0; m0 < N1; ++m0) G[m0] += F * tb.Lq[m0][q0];
      }
#pragma unroll
      for (int m1 = 0; m1 < N1; ++m1)
#pragma unroll
        for (int m0 = 0; m0 < N1; ++m0) Fm[m0 + N1 * m1] += G[m0] * tb.Lq[m1][q1];
    }
  }
}

// R[.. a along E ..] += coef * L_side[a] * Fm
template <int DIM, int P, int E, typename T>
__device__ __forceinline__ void scatter_face(T* R, const T* Ls, const T* Fm, T coef) {
  constexpr int N1 = P + 1, NF = ipow(N1, DIM - 1);
  constexpr int t0 = E == 0 ? 1 : 0, t1 = E == 2 ? 1 : 2;
  constexpr int st[3] = {1, N1, N1 * N1};
#pragma unroll
  for (int mf = 0; mf < NF; ++mf) {
    const int m0 = mf % N1, m1 = mf / N1;
    const int base = m0 * st[t0] + (DIM > 2 ? m1 * st[t1] : 0);
    const T f = coef * Fm[mf];
#pragma unroll
    for (int a = 0; a < N1; ++a) R[base + a * st[E]] += Ls[a] * f;
  }
}

// General velocity: a runtime sum of separable terms per component.  (A
// velocity whose components are single terms takes adv_sep_kernel.)  TAB:
// the velocity's spatial part read from tables made once per field update
// at every cell's quadrature points and, single-valued, at every face's
// (vel_tabulate_* for a sum of terms, fe_tabulate_* for the velocity of a
// coupled FE simulator, advection.implement.h:891-905), times the time
// factor.
// one tile of a stage (launch slot `slot`); a plain launch serves slot blockIdx.x
template <int DIM, int P, typename T, bool TAB = false>
__device__ __forceinline__ void adv_stage_tile(const AdvArgs<T>& a, int slot) {
  constexpr int N1 = P + 1, NQ = P + 2, NM = ipow(N1, DIM), NPT = NQ + 2, NF = ipow(N1, DIM - 1);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* box = reinterpret_cast<T*>(smem_raw);
  const MeshArgs& m = a.m;
  const int nboxc = box_cells(m, DIM);
  const int tx = m.tile[0], ty = m.tile[1], tz = m.tile[2];
  const int nt = tx * ty * tz;
  const int nterm = a.v.n_terms;
  const int span = tx + ty + (DIM > 2 ? tz : 0);
  T* vt = box + (size_t)nboxc * NM;
  T* fl = vt + (TAB ? 0 : (size_t)max(nterm, 1) * span * NPT);   // [DIM][NF][nt]
  const Tab1D<T>& tb = tab<T>(P);
  const TileCoord tc = tile_coord(m, DIM, slot);

  if constexpr (!TAB) {
    // ---- stage velocity-table rows of this tile: vt[(k*span + li)*NPT + j]
    const int total = nterm * span * NPT;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      const int j = e % NPT;
      const int r = e / NPT;
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
  const int tl[3] = {tx, ty, tz};

  T R[NM];
  T c[NM];
#pragma unroll
  for (int q = 0; q < NM; ++q) R[q] = T(0);
  if (tc.valid) {
#pragma unroll
    for (int q = 0; q < NM; ++q) c[q] = box[(size_t)me * NM + q];
  }
  const bool work = tc.valid && active;

  auto vrow = [&](int k, int axis) -> const T* {
    const int li = axis == 0 ? tc.lx : (axis == 1 ? tx + tc.ly : tx + ty + tc.lz);
    return vt + (size_t)(k * span + li) * NPT;
  };
  // TAB: the tables at this cell's quadrature points ([comp][point][cell],
  // cell lexicographic) and at its faces ([E][point][face], face index
  // lexicographic over n + e_E faces)
  const long long tab_cell = tc.gx + (long long)m.n[0] * (tc.gy + (long long)m.n[1] * tc.gz);
  auto tab_point = [&](int qx, int qy, int qz, T* u) {
    constexpr int NQD = ipow(NQ, DIM);
    const int q = qx + NQ * (qy + NQ * qz);
#pragma unroll
    for (int d = 0; d < DIM; ++d) u[d] = a.v.tab_q[((size_t)d * NQD + q) * m.ncell + tab_cell] * ct;
  };
  auto tab_face = [&](auto EC, int S, int q0, int q1) -> T {
    constexpr int E = decltype(EC)::value;
    int f[3] = {tc.gx, tc.gy, tc.gz};
    f[E] += S;
    const long long nf0 = m.n[0] + (E == 0), nf1 = m.n[1] + (E == 1);
    const long long face = f[0] + nf0 * (f[1] + nf1 * f[2]);
    return a.v.tab_f[a.v.tab_foff[E] + (size_t)(q0 + NQ * q1) * a.v.tab_nf[E] + face] * ct;
  };
  // velocity component `comp` (times the time factor) at table columns
  auto vel = [&](int comp, int jx, int jy, int jz) -> T {
    T u = T(0);
    for (int k = a.v.cstart[comp]; k < a.v.cstart[comp + 1]; ++k) {
      T v = vrow(k, 0)[jx] * vrow(k, 1)[jy];
      if constexpr (DIM == 3) v = v * vrow(k, 2)[jz];
      u += v;
    }
    return u * ct;
  };
  if (work) {
    // ============================ cell term ============================
    if constexpr (DIM == 2) {
#pragma unroll 1
      for (int qy = 0; qy < NQ; ++qy) {
        T Py[N1];
#pragma unroll
        for (int aa = 0; aa < N1; ++aa) {
          T s = T(0);
#pragma unroll
          for (int b = 0; b < N1; ++b) s += c[aa + N1 * b] * tb.Lq[b][qy];
          Py[aa] = s;
        }
        T X1[N1], X2[N1];
#pragma unroll
        for (int aa = 0; aa < N1; ++aa) { X1[aa] = T(0); X2[aa] = T(0); }
#pragma unroll
        for (int qx = 0; qx < NQ; ++qx) {
          T phi = T(0);
#pragma unroll
          for (int aa = 0; aa < N1; ++aa) phi += Py[aa] * tb.Lq[aa][qx];
          T uq[2];
          if constexpr (TAB) tab_point(qx, qy, 0, uq);
          else { uq[0] = vel(0, qx, qy, 0); uq[1] = vel(1, qx, qy, 0); }
          const T u0 = uq[0], u1 = uq[1];
          const T w = tb.wq[qx] * tb.wq[qy] * phi;
          const T fx = w * u0 * ih[0];
          const T fy = w * u1 * ih[1];
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
#pragma unroll 1
      for (int qz = 0; qz < NQ; ++qz) {
        T Pz[N1][N1];
#pragma unroll
        for (int aa = 0; aa < N1; ++aa)
#pragma unroll
          for (int b = 0; b < N1; ++b) {
            T s = T(0);
#pragma unroll
            for (int cc = 0; cc < N1; ++cc) s += c[aa + N1 * (b + N1 * cc)] * tb.Lq[cc][qz];
            Pz[aa][b] = s;
          }
        T U1[N1][N1], U3[N1][N1];
#pragma unroll
        for (int aa = 0; aa < N1; ++aa)
#pragma unroll
          for (int b = 0; b < N1; ++b) { U1[aa][b] = T(0); U3[aa][b] = T(0); }
        // qy not unrolled: the instruction footprint of the unrolled 3D
        // body (every point, every face) misses the instruction cache
#pragma unroll 1
        for (int qy = 0; qy < NQ; ++qy) {
          T Py[N1];
#pragma unroll
          for (int aa = 0; aa < N1; ++aa) {
            T s = T(0);
#pragma unroll
            for (int b = 0; b < N1; ++b) s += Pz[aa][b] * tb.Lq[b][qy];
            Py[aa] = s;
          }
          T X1[N1], X2[N1], X3[N1];
#pragma unroll
          for (int aa = 0; aa < N1; ++aa) { X1[aa] = T(0); X2[aa] = T(0); X3[aa] = T(0); }
#pragma unroll
          for (int qx = 0; qx < NQ; ++qx) {
            T phi = T(0);
#pragma unroll
            for (int aa = 0; aa < N1; ++aa) phi += Py[aa] * tb.Lq[aa][qx];
            T uq[3];
            if constexpr (TAB) tab_point(qx, qy, qz, uq);
            else { uq[0] = vel(0, qx, qy, qz); uq[1] = vel(1, qx, qy, qz); uq[2] = vel(2, qx, qy, qz); }
            const T u0 = uq[0], u1 = uq[1], u2 = uq[2];
            const T w = tb.wq[qx] * tb.wq[qy] * tb.wq[qz] * phi;
            const T fx = w * u0 * ih[0];
            const T fy = w * u1 * ih[1];
            const T fz = w * u2 * ih[2];
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
  }

  // weighted normal velocity on face (E, S): u_E(q) w_q0 w_q1 at the face
  // Gauss point (q0, q1) (tangential axes in increasing order)
  auto face_vel = [&](auto EC, auto SC) {
    constexpr int E = decltype(EC)::value, S = decltype(SC)::value;
    constexpr int t0 = E == 0 ? 1 : 0, t1 = E == 2 ? 1 : 2;
    return [&, E, S](int q0, int q1) -> T {
      int j[3] = {0, 0, 0};
      j[E] = NQ + S;
      j[t0] = q0;
      if (DIM > 2) j[t1] = q1;
      T w = tb.wq[q0];
      if constexpr (DIM > 2) w = w * tb.wq[q1];
      if constexpr (TAB) return tab_face(std::integral_constant<int, E>(), S, q0, q1) * w;
      else return vel(E, j[0], j[1], j[2]) * w;
    };
  };

  // ============ upper faces: computed once, shared with the upper neighbour
  auto do_upper = [&](auto EC) {
    constexpr int E = decltype(EC)::value;
    if (!work) return;
    int nl[3] = {l[0], l[1], l[2]};
    nl[E] += 1;
    const bool has_nb = g[E] + 1 < m.n[E];
    const T* cn = box + (size_t)box_index(m, DIM, nl[0], nl[1], nl[2]) * NM;
    T Fm[NF];
    T gd = T(0);
    const bool dir = !has_nb && bc_dirichlet<DIM>(m, E, 1, g, gd);
    face_flux<DIM, P, E, 1, T>(tb, c, cn, has_nb, face_vel(std::integral_constant<int, E>(),
                                                          std::integral_constant<int, 1>()), Fm, dir, gd);
    scatter_face<DIM, P, E, T>(R, tb.L1, Fm, -ih[E]);
    if (has_nb && l[E] + 1 < tl[E]) {
#pragma unroll
      for (int mf = 0; mf < NF; ++mf) fl[(size_t)(E * NF + mf) * nt + cl] = Fm[mf];
    }
  };
  do_upper(std::integral_constant<int, 0>());
  do_upper(std::integral_constant<int, 1>());
  if constexpr (DIM == 3) do_upper(std::integral_constant<int, 2>());
  __syncthreads();
  // ============ lower faces: shared flux of the lower neighbour, or own
  auto do_lower = [&](auto EC) {
    constexpr int E = decltype(EC)::value;
    if (!work) return;
    T Fm[NF];
    const int stride = E == 0 ? 1 : (E == 1 ? tx : tx * ty);
    if (l[E] > 0 && g[E] > 0) {
#pragma unroll
      for (int mf = 0; mf < NF; ++mf) Fm[mf] = fl[(size_t)(E * NF + mf) * nt + cl - stride];
      scatter_face<DIM, P, E, T>(R, tb.L0, Fm, ih[E]);
    } else {
      int nl[3] = {l[0], l[1], l[2]};
      nl[E] -= 1;
      const bool has_nb = g[E] > 0;
      const T* cn = box + (size_t)box_index(m, DIM, nl[0], nl[1], nl[2]) * NM;
      T gd = T(0);
      const bool dir = !has_nb && bc_dirichlet<DIM>(m, E, 0, g, gd);
      face_flux<DIM, P, E, 0, T>(tb, c, cn, has_nb, face_vel(std::integral_constant<int, E>(),
                                                            std::integral_constant<int, 0>()), Fm, dir, gd);
      scatter_face<DIM, P, E, T>(R, tb.L0, Fm, -ih[E]);
    }
  };
  do_lower(std::integral_constant<int, 0>());
  do_lower(std::integral_constant<int, 1>());
  if constexpr (DIM == 3) do_lower(std::integral_constant<int, 2>());

  // ---- combine with phi^n and store through shared memory (coalesced)
  __syncthreads();
  T* stage_buf = box;  // reuse: [tile cell][NM]
  const bool need_n = a.combine == kRK2b || a.combine == kRK3b || a.combine == kRK3c;
  if (need_n) {
    load_tile<DIM, NM>(m, a.phi_n, stage_buf, tc.ox, tc.oy, tc.oz, false, NM);
    cp_async_wait_all();
    __syncthreads();
  }
  if (tc.valid) {
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
  store_tile<DIM, NM>(m, stage_buf, a.out, tc.ox, tc.oy, tc.oz);
}

template <int DIM, int P, typename T, bool TAB>
__global__ void __launch_bounds__(256, 2) adv_stage_kernel(const AdvArgs<T> a) {
  adv_stage_tile<DIM, P, T, TAB>(a, (int)blockIdx.x);
}

}  // namespace flsp

// flsp_misc.cuh — small kernels around the two stencil kernels: device
// clocks, host<->device DoF order, initial-condition projection, FP64
// diagnostics reductions, the static part of the advection CFL.
#pragma once
#include "flsp_clock.cuh"
#include "flsp_device.cuh"
#include "flsp_dg.h"

namespace flsp {

constexpr double kPiD = 3.14159265358979323846;
constexpr double kEpsD = 2.220446049250313e-16;

// ---------------------------------------------------------------------
// clocks
// ---------------------------------------------------------------------

// clock kernels: one thread (the updates are in flsp_clock.cuh)
__global__ void adv_clock_begin(DevClock* c, const AdvClockArgs a) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  adv_clock_begin_body(c, a);
}
__global__ void adv_clock_end(DevClock* c) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  adv_clock_end_body(c);
}
__global__ void adv_clock_horizon(DevClock* c, double time_step) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  adv_clock_horizon_body(c, time_step);
}
__global__ void hj_clock_reset(DevClock* c) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  hj_clock_reset_body(c);
}
__global__ void hj_clock_begin(DevClock* c, double cfl_max, int p, double nu, double min_diam, double adv_scale) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  hj_clock_begin_body(c, cfl_max, p, nu, min_diam, adv_scale);
}
__global__ void hj_clock_end(DevClock* c) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  hj_clock_end_body(c);
}

// ---------------------------------------------------------------------
// host DoF order <-> device layout (optional cell permutation)
// ---------------------------------------------------------------------
template <typename T>
__global__ void scatter_state(const double* __restrict__ src, T* __restrict__ dst,
                              const int64_t* __restrict__ perm, long long ncell, int nb) {
  const long long n = ncell * nb;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long k = i / nb, j = i - k * nb;
    const long long cell = perm ? perm[k] : k;
    dst[cell * nb + j] = T(src[i]);
  }
}

template <typename T>
__global__ void gather_state(const T* __restrict__ src, double* __restrict__ dst,
                             const int64_t* __restrict__ perm, long long ncell, int nb) {
  const long long n = ncell * nb;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long k = i / nb, j = i - k * nb;
    const long long cell = perm ? perm[k] : k;
    dst[i] = double(src[cell * nb + j]);
  }
}

// ---------------------------------------------------------------------
// initial conditions (src/level_set/geometry.cc:17-235, geometry.h:80-160)
// nodes are evaluated in index order; children precede their parents
// ---------------------------------------------------------------------
__device__ inline double ic_eval(const flsp_ic_desc* ic, int dim, const double* x) {
  double val[FLSP_MAX_IC_NODES];
  for (int k = 0; k < ic->n_nodes; ++k) {
    const flsp_ic_node& nd = ic->nodes[k];
    double r = 0.0;
    switch (nd.kind) {
      case FLSP_IC_SPHERE: {
        double s = 0.0;
        for (int d = 0; d < dim; ++d) { const double e = x[d] - nd.p[d]; s += e * e; }
        r = sqrt(s) - nd.p[3];
        break;
      }
      case FLSP_IC_RECT: {
        double out2 = 0.0;
        bool inside = true;
        for (int d = 0; d < dim; ++d) {
          double e = 0.0;
          if (x[d] < nd.p[d]) { e = x[d] - nd.p[d]; inside = false; }
          else if (x[d] > nd.p[3 + d]) { e = x[d] - nd.p[3 + d]; inside = false; }
          out2 += e * e;
        }
        if (!inside) { r = sqrt(out2); break; }
        double mm = -1e300;
        for (int d = 0; d < dim; ++d) {
          mm = fmax(mm, nd.p[d] - x[d]);
          mm = fmax(mm, x[d] - nd.p[3 + d]);
        }
        r = mm;
        break;
      }
      case FLSP_IC_HEIGHT: {
        const int ax = (int)nd.p[0];
        int u = -1, v = -1;
        for (int d = 0; d < dim; ++d)
          if (d != ax) { if (u < 0) u = d; else v = d; }
        double hgt = nd.p[1];
        for (int w = 0; w < ic->n_waves; ++w) {
          double arg = ic->waves[w][1] * x[u];
          if (v >= 0) arg += ic->waves[w][2] * x[v];
          hgt += ic->waves[w][0] * cos(2.0 * kPiD * arg + ic->waves[w][3]);
        }
        r = x[ax] - hgt;
        break;
      }
      case FLSP_IC_UNION: r = fmin(val[nd.a], val[nd.b]); break;
      case FLSP_IC_DIFF: r = fmax(val[nd.a], -val[nd.b]); break;
      case FLSP_IC_INTERSECT: r = fmax(val[nd.a], val[nd.b]); break;
    }
    val[k] = r;
  }
  return val[ic->root];
}

// evaluate the DG function of one cell at reference point (table columns)
template <int DIM, int P>
__device__ __forceinline__ double eval_modal(const double* c, const double* bx, const double* by,
                                             const double* bz) {
  constexpr int N1 = P + 1;
  double s = 0.0;
  if constexpr (DIM == 2) {
#pragma unroll
    for (int b = 0; b < N1; ++b) {
      double r = 0.0;
#pragma unroll
      for (int a = 0; a < N1; ++a) r += c[a + N1 * b] * bx[a];
      s += r * by[b];
    }
  } else {
#pragma unroll
    for (int cc = 0; cc < N1; ++cc)
#pragma unroll
      for (int b = 0; b < N1; ++b) {
        double r = 0.0;
#pragma unroll
        for (int a = 0; a < N1; ++a) r += c[a + N1 * (b + N1 * cc)] * bx[a];
        s += r * by[b] * bz[cc];
      }
  }
  return s;
}

// L2 projection with QGauss(p+2) (advection.cc:145-161); always in FP64
template <int DIM, int P, typename T>
__global__ void project_ic_kernel(const MeshArgs m, const flsp_ic_desc* __restrict__ ic,
                                  T* __restrict__ out) {
  constexpr int N1 = P + 1, NQ = P + 2, NM = ipow(N1, DIM);
  const Tab1D<double>& tb = c_tab_d[P];
  const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (cell >= m.ncell) return;
  const int gx = (int)(cell % m.n[0]);
  const int gy = (int)((cell / m.n[0]) % m.n[1]);
  const int gz = DIM > 2 ? (int)(cell / ((long long)m.n[0] * m.n[1])) : 0;
  const double x0[3] = {m.lo[0] + gx * m.h[0], m.lo[1] + gy * m.h[1], DIM > 2 ? m.lo[2] + gz * m.h[2] : 0.0};
  double R[NM];
#pragma unroll
  for (int q = 0; q < NM; ++q) R[q] = 0.0;
  const int nqz = DIM > 2 ? NQ : 1;
  for (int qz = 0; qz < nqz; ++qz)
    for (int qy = 0; qy < NQ; ++qy)
      for (int qx = 0; qx < NQ; ++qx) {
        double x[3] = {x0[0] + m.h[0] * tb.xq[qx], x0[1] + m.h[1] * tb.xq[qy],
                       DIM > 2 ? x0[2] + m.h[2] * tb.xq[qz] : 0.0};
        double f = ic_eval(ic, DIM, x);
        double w = tb.wq[qx] * tb.wq[qy];
        if (DIM > 2) w *= tb.wq[qz];
        const double fw = f * w;
#pragma unroll
        for (int q = 0; q < NM; ++q) {
          const int i0 = q % N1, i1 = (q / N1) % N1, i2 = q / (N1 * N1);
          double bw = tb.Lq[i0][qx] * tb.Lq[i1][qy];
          if (DIM > 2) bw *= tb.Lq[i2][qz];
          R[q] += fw * bw;
        }
      }
  for (int k = 0; k < m.nb; ++k) out[cell * m.nb + k] = T(R[m.g2q[k]]);
}

// ---------------------------------------------------------------------
// static CFL part: max over cells and vertices of |u_spatial| / diam
// (CFLEstimator::local_estimate, pde_tools.implement.h:44-57)
// ---------------------------------------------------------------------
template <int DIM>
__global__ void static_cfl_kernel(const MeshArgs m, const VelArgs<double> v, DevClock* clk) {
  __shared__ double red[32];
  const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double best = 0.0;
  if (cell < m.ncell) {
    const int g[3] = {(int)(cell % m.n[0]), (int)((cell / m.n[0]) % m.n[1]),
                      DIM > 2 ? (int)(cell / ((long long)m.n[0] * m.n[1])) : 0};
    const int NQ = v.npt - 2;
    for (int vv = 0; vv < (1 << DIM); ++vv) {
      double u[3] = {0.0, 0.0, 0.0};
      for (int k = 0; k < v.n_terms; ++k) {
        double tv = 1.0;
        for (int d = 0; d < DIM; ++d) {
          const int j = NQ + ((vv >> d) & 1);
          tv *= v.vtab[((size_t)(k * 3 + d) * v.nmax + g[d]) * v.npt + j];
        }
        u[v.comp[k]] += tv;
      }
      double s = 0.0;
      for (int d = 0; d < DIM; ++d) s += u[d] * u[d];
      best = fmax(best, sqrt(s));
    }
    best /= m.diam;
  }
  const double bm = block_max(best, red);
  if (threadIdx.x == 0) {
    unsigned long long* slot = reinterpret_cast<unsigned long long*>(&clk->vd_static);
    atomic_max_pos(slot, bm);
  }
}

// the same estimate for an FE velocity lattice of degree pv (fe_n* nodes per
// axis, FP64): a cell's vertex velocities are its corner nodes
template <int DIM>
__global__ void fe_static_cfl_kernel(const MeshArgs m, const double* __restrict__ u, int pv, int nx, int ny,
                                     int nz, DevClock* clk) {
  __shared__ double red[32];
  const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double best = 0.0;
  if (cell < m.ncell) {
    const int g[3] = {(int)(cell % m.n[0]), (int)((cell / m.n[0]) % m.n[1]),
                      DIM > 2 ? (int)(cell / ((long long)m.n[0] * m.n[1])) : 0};
    const size_t nn = (size_t)nx * ny * nz;
    for (int vv = 0; vv < (1 << DIM); ++vv) {
      const int x = pv * (g[0] + (vv & 1)), y = pv * (g[1] + ((vv >> 1) & 1));
      const int z = DIM > 2 ? pv * (g[2] + ((vv >> 2) & 1)) : 0;
      const size_t node = ((size_t)z * ny + y) * nx + x;
      double s = 0.0;
      for (int d = 0; d < DIM; ++d) s += u[d * nn + node] * u[d * nn + node];
      best = fmax(best, sqrt(s));
    }
    best /= m.diam;
  }
  const double bm = block_max(best, red);
  if (threadIdx.x == 0) {
    unsigned long long* slot = reinterpret_cast<unsigned long long*>(&clk->vd_static);
    atomic_max_pos(slot, bm);
  }
}

// terms of each component in a component-sorted term list
struct VelTerms {
  int cstart[4];
};

// the spatial part of a sum of separable terms at every cell's quadrature
// points: one thread per (point, cell), cell fastest; per term the product
// ((coeff f0) f1) f2 of the term tables' entries, the component's terms in
// order (the point-wise stage kernel's evaluation), in FP64, stored in T
template <int DIM, typename T>
__global__ void vel_tabulate_cells(const MeshArgs m, const double* __restrict__ vtab, int nmax, int npt,
                                   const VelTerms vt, int nq, T* __restrict__ out) {
  const int nqd = DIM > 2 ? nq * nq * nq : nq * nq;
  const long long total = (long long)nqd * m.ncell;
  auto row = [&](int k, int ax, int i) { return vtab + ((size_t)(k * 3 + ax) * nmax + i) * npt; };
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long cell = i % m.ncell;
    const int q = (int)(i / m.ncell);
    const int qx = q % nq, qy = (q / nq) % nq, qz = DIM > 2 ? q / (nq * nq) : 0;
    const int gx = (int)(cell % m.n[0]), gy = (int)((cell / m.n[0]) % m.n[1]);
    const int gz = DIM > 2 ? (int)(cell / ((long long)m.n[0] * m.n[1])) : 0;
    for (int d = 0; d < DIM; ++d) {
      double u = 0.0;
      for (int k = vt.cstart[d]; k < vt.cstart[d + 1]; ++k) {
        double v = row(k, 0, gx)[qx] * row(k, 1, gy)[qy];
        if (DIM == 3) v = v * row(k, 2, gz)[qz];
        u += v;
      }
      out[((size_t)d * nqd + q) * m.ncell + cell] = T(u);
    }
  }
}

// the normal component E at every face's points: from the lower cell's
// upper-face entries (the first face: the upper cell's lower-face entries,
// the same face coordinate bit for bit)
template <int DIM, typename T>
__global__ void vel_tabulate_faces(const MeshArgs m, const double* __restrict__ vtab, int nmax, int npt,
                                   const VelTerms vt, int nq, int E, long long nface, T* __restrict__ out) {
  const int nqf = DIM > 2 ? nq * nq : nq;
  const int nf0 = m.n[0] + (E == 0), nf1 = m.n[1] + (E == 1);
  const int t0 = E == 0 ? 1 : 0, t1 = E == 2 ? 1 : 2;
  const long long total = (long long)nqf * nface;
  auto row = [&](int k, int ax, int i) { return vtab + ((size_t)(k * 3 + ax) * nmax + i) * npt; };
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long face = i % nface;
    const int q = (int)(i / nface);
    const int q0 = q % nq, q1 = DIM > 2 ? q / nq : 0;
    const int f[3] = {(int)(face % nf0), (int)((face / nf0) % nf1), DIM > 2 ? (int)(face / ((long long)nf0 * nf1)) : 0};
    int cidx[3] = {f[0], f[1], f[2]}, j[3] = {0, 0, 0};
    if (f[E] > 0) { cidx[E] = f[E] - 1; j[E] = nq + 1; }
    else j[E] = nq;
    j[t0] = q0;
    if (DIM > 2) j[t1] = q1;
    double u = 0.0;
    for (int k = vt.cstart[E]; k < vt.cstart[E + 1]; ++k) {
      double v = row(k, 0, cidx[0])[j[0]] * row(k, 1, cidx[1])[j[1]];
      if (DIM == 3) v = v * row(k, 2, cidx[2])[j[2]];
      u += v;
    }
    out[(size_t)q * nface + face] = T(u);
  }
}

struct FeBasis {
  double b[kMaxFeVel + 1][kMaxNQ + 2];   // Lagrange basis a at Gauss point q
};

// FE velocity at every cell's quadrature points: one thread per (point,
// cell), cell fastest; the cell's nodes times the basis products, summed x
// fastest, in FP64, stored in T
template <int DIM, typename T>
__global__ void fe_tabulate_cells(const MeshArgs m, const double* __restrict__ u, int pv, int nq,
                                  const FeBasis fb, T* __restrict__ out) {
  const int nx = pv * m.n[0] + 1, ny = pv * m.n[1] + 1, nz = DIM > 2 ? pv * m.n[2] + 1 : 1;
  const size_t nn = (size_t)nx * ny * nz;
  const int nqd = DIM > 2 ? nq * nq * nq : nq * nq;
  const long long total = (long long)nqd * m.ncell;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long cell = i % m.ncell;
    const int q = (int)(i / m.ncell);
    const int qx = q % nq, qy = (q / nq) % nq, qz = DIM > 2 ? q / (nq * nq) : 0;
    const int gx = (int)(cell % m.n[0]), gy = (int)((cell / m.n[0]) % m.n[1]);
    const int gz = DIM > 2 ? (int)(cell / ((long long)m.n[0] * m.n[1])) : 0;
    double acc[3] = {0.0, 0.0, 0.0};
    for (int cz = 0; cz <= (DIM > 2 ? pv : 0); ++cz)
      for (int cy = 0; cy <= pv; ++cy) {
        double byz = fb.b[cy][qy];
        if (DIM > 2) byz *= fb.b[cz][qz];
        for (int cx = 0; cx <= pv; ++cx) {
          const double b = fb.b[cx][qx] * byz;
          const size_t node = ((size_t)(pv * gz + cz) * ny + pv * gy + cy) * nx + pv * gx + cx;
          for (int d = 0; d < DIM; ++d) acc[d] += u[d * nn + node] * b;
        }
      }
    for (int d = 0; d < DIM; ++d) out[((size_t)d * nqd + q) * m.ncell + cell] = T(acc[d]);
  }
}

// the normal component at every face's quadrature points, from the face's
// own nodes (the basis of the others vanishes on it): one value per face
template <int DIM, typename T>
__global__ void fe_tabulate_faces(const MeshArgs m, const double* __restrict__ u, int pv, int nq,
                                  const FeBasis fb, int E, long long nface, T* __restrict__ out) {
  const int nx = pv * m.n[0] + 1, ny = pv * m.n[1] + 1, nz = DIM > 2 ? pv * m.n[2] + 1 : 1;
  const size_t nn = (size_t)nx * ny * nz;
  const int nqf = DIM > 2 ? nq * nq : nq;
  const int nf0 = m.n[0] + (E == 0), nf1 = m.n[1] + (E == 1);
  const int t0 = E == 0 ? 1 : 0, t1 = E == 2 ? 1 : 2;
  const long long total = (long long)nqf * nface;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long face = i % nface;
    const int q = (int)(i / nface);
    const int q0 = q % nq, q1 = DIM > 2 ? q / nq : 0;
    const int f[3] = {(int)(face % nf0), (int)((face / nf0) % nf1), DIM > 2 ? (int)(face / ((long long)nf0 * nf1)) : 0};
    double acc = 0.0;
    for (int c1 = 0; c1 <= (DIM > 2 ? pv : 0); ++c1)
      for (int c0 = 0; c0 <= pv; ++c0) {
        double b = fb.b[c0][q0];
        if (DIM > 2) b *= fb.b[c1][q1];
        int node[3];
        node[E] = pv * f[E];
        node[t0] = pv * f[t0] + c0;
        if (DIM > 2) node[t1] = pv * f[t1] + c1;
        else node[2] = 0;
        acc += u[E * nn + ((size_t)node[2] * ny + node[1]) * nx + node[0]] * b;
      }
    out[(size_t)q * nface + face] = T(acc);
  }
}

// ---------------------------------------------------------------------
// FP64 reductions (level_set.implement.h:215-295, 356-380, 957-993;
// advection.cc:452-484; reinit.cc:491-526).  Two levels, fixed order.
// ---------------------------------------------------------------------
__device__ __forceinline__ double heaviside_sine(double x, double eps) {
  if (x > eps) return 1.0;
  if (x < -eps) return 0.0;
  const double val = 0.5 * (1.0 + x / eps + sin(x * kPiD / eps) / kPiD);
  if (fabs(val) < kEpsD) return 0.0;
  if (fabs(val - 1.0) < kEpsD) return 1.0;
  return val;
}
__device__ __forceinline__ double heaviside_sharp(double x) {
  return x > 0.0 ? 1.0 : (x < 0.0 ? 0.0 : 0.5);
}

template <typename T>
struct RedArgs {
  MeshArgs m;
  const T* phi;
  const T* ref;
  const flsp_ic_desc* ic;
  int which;
  double* partial;   // [gridDim.x][2]
};

template <int DIM, int P, typename T>
__global__ void reduce_kernel(const RedArgs<T> a) {
  constexpr int N1 = P + 1, NQ = P + 2, NM = ipow(N1, DIM);
  __shared__ double red[2][32];
  const MeshArgs& m = a.m;
  const Tab1D<double>& tb = c_tab_d[P];
  const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double s0 = 0.0, s1 = 0.0;
  if (cell < m.ncell) {
    double c[NM], r[NM];
#pragma unroll
    for (int q = 0; q < NM; ++q) {
      const int gi = m.q2g[q];
      c[q] = gi >= 0 ? double(a.phi[cell * m.nb + gi]) : 0.0;
      r[q] = (gi >= 0 && a.ref) ? double(a.ref[cell * m.nb + gi]) : 0.0;
    }
    const int g[3] = {(int)(cell % m.n[0]), (int)((cell / m.n[0]) % m.n[1]),
                      DIM > 2 ? (int)(cell / ((long long)m.n[0] * m.n[1])) : 0};
    const double eps = 1.5 * m.min_diam;
    const int w = a.which;
    if (w == FLSP_RED_MEAN_ABS_DIFF) {
      for (int k = 0; k < m.nb; ++k) s0 += fabs(double(a.phi[cell * m.nb + k]) - double(a.ref[cell * m.nb + k]));
    } else if (w == FLSP_RED_MAX_ABS) {
      for (int k = 0; k < m.nb; ++k) s0 = fmax(s0, fabs(double(a.phi[cell * m.nb + k])));
    } else {
      const bool gauss_p1 = (w == FLSP_RED_MASS || w == FLSP_RED_MASS_ERROR ||
                             w == FLSP_RED_GRAD_DEVIATION || w == FLSP_RED_L2_ERROR_IC);
      const int nq = gauss_p1 ? N1 : NQ;
      const int nqz = DIM > 2 ? nq : 1;
      double cellacc = 0.0;
      for (int qz = 0; qz < nqz; ++qz)
        for (int qy = 0; qy < nq; ++qy)
          for (int qx = 0; qx < nq; ++qx) {
            const int qq[3] = {qx, qy, qz};
            double bx[N1], by[N1], bz[N1], dx[N1], dy[N1], dz[N1], xx[3], wgt = 1.0;
            for (int d = 0; d < 3; ++d) xx[d] = 0.0;
            for (int i = 0; i < N1; ++i) {
              bx[i] = gauss_p1 ? tb.Ll[i][qx] : tb.Lq[i][qx];
              by[i] = gauss_p1 ? tb.Ll[i][qy] : tb.Lq[i][qy];
              bz[i] = DIM > 2 ? (gauss_p1 ? tb.Ll[i][qz] : tb.Lq[i][qz]) : 1.0;
              dx[i] = gauss_p1 ? tb.Dl[i][qx] : tb.Dq[i][qx];
              dy[i] = gauss_p1 ? tb.Dl[i][qy] : tb.Dq[i][qy];
              dz[i] = DIM > 2 ? (gauss_p1 ? tb.Dl[i][qz] : tb.Dq[i][qz]) : 1.0;
            }
            for (int d = 0; d < DIM; ++d) {
              const double xi = gauss_p1 ? tb.xl[qq[d]] : tb.xq[qq[d]];
              xx[d] = (m.lo[d] + g[d] * m.h[d]) + m.h[d] * xi;
              wgt *= gauss_p1 ? tb.wl[qq[d]] : tb.wq[qq[d]];
            }
            const double jxw = wgt * m.vol;
            const double val = eval_modal<DIM, P>(c, bx, by, bz);
            if (w == FLSP_RED_MASS || w == FLSP_RED_MASS_ERROR) {
              s0 += heaviside_sine(-val, eps) * jxw;
              if (w == FLSP_RED_MASS_ERROR) s1 += heaviside_sine(-ic_eval(a.ic, DIM, xx), eps) * jxw;
            } else if (w == FLSP_RED_MASS_SHARP) {
              s0 += heaviside_sharp(-val) * jxw;
            } else if (w == FLSP_RED_L1_INTERFACE) {
              s0 += fabs(heaviside_sharp(-val) - heaviside_sharp(-eval_modal<DIM, P>(r, bx, by, bz))) * jxw;
            } else if (w == FLSP_RED_L1_INTERFACE_IC) {
              s0 += fabs(heaviside_sharp(-val) - heaviside_sharp(-ic_eval(a.ic, DIM, xx))) * jxw;
            } else if (w == FLSP_RED_L2_ERROR_IC) {
              const double diff = val - ic_eval(a.ic, DIM, xx);
              cellacc += diff * diff * jxw;
            } else if (w == FLSP_RED_GRAD_DEVIATION) {
              const double gxv = eval_modal<DIM, P>(c, dx, by, bz) / m.h[0];
              const double gyv = eval_modal<DIM, P>(c, bx, dy, bz) / m.h[1];
              const double gzv = DIM > 2 ? eval_modal<DIM, P>(c, bx, by, dz) / m.h[2] : 0.0;
              const double g2 = gxv * gxv + gyv * gyv + gzv * gzv;
              s0 += fabs(sqrt(g2) - 1.0) * jxw;
            }
          }
      if (w == FLSP_RED_L2_ERROR_IC) s0 += cellacc;
      if (w == FLSP_RED_GRAD_DEVIATION) s1 += m.vol;
    }
  }
  if (a.which == FLSP_RED_MAX_ABS) {
    const double bm = block_max(s0, red[0]);
    if (threadIdx.x == 0) { a.partial[2 * blockIdx.x] = bm; a.partial[2 * blockIdx.x + 1] = 0.0; }
    return;
  }
  s0 = warp_sum(s0);
  s1 = warp_sum(s1);
  const int wi = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { red[0][wi] = s0; red[1][wi] = s1; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t0 = 0.0, t1 = 0.0;
    const int nw = (blockDim.x + 31) >> 5;
    for (int i = 0; i < nw; ++i) { t0 += red[0][i]; t1 += red[1][i]; }
    a.partial[2 * blockIdx.x] = t0;
    a.partial[2 * blockIdx.x + 1] = t1;
  }
}

__global__ void reduce_final(const double* __restrict__ partial, int n, int is_max, double* out) {
  __shared__ double red[2][32];
  double s0 = 0.0, s1 = 0.0;
  // fixed assignment of partials to threads -> deterministic
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    if (is_max) s0 = fmax(s0, partial[2 * i]);
    else { s0 += partial[2 * i]; s1 += partial[2 * i + 1]; }
  }
  if (is_max) {
    const double bm = block_max(s0, red[0]);
    if (threadIdx.x == 0) { out[0] = bm; out[1] = 0.0; }
    return;
  }
  s0 = warp_sum(s0);
  s1 = warp_sum(s1);
  const int wi = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { red[0][wi] = s0; red[1][wi] = s1; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t0 = 0.0, t1 = 0.0;
    for (int i = 0; i < (int)((blockDim.x + 31) >> 5); ++i) { t0 += red[0][i]; t1 += red[1][i]; }
    out[0] = t0;
    out[1] = t1;
  }
}

// finite check of a state vector: counts non-finite entries
template <typename T>
__global__ void nonfinite_kernel(const T* __restrict__ x, long long n, unsigned int* count) {
  unsigned int local = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    if (!isfinite((double)x[i])) ++local;
  if (local) atomicAdd(count, local);
}

}  // namespace flsp

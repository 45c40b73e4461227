// flsp_tables.h — host computation (FP64) of the 1D Legendre / Gauss
// tables every kernel unit uploads into its constant memory.
#pragma once
#include <cmath>
#include <cstring>

#include "flsp_device.cuh"

namespace flsp {

// Legendre polynomials orthonormal on [0,1] (deal.II Polynomials::Legendre):
// L_k(x) = sqrt(2k+1) P_k(2x-1), with first and second derivatives
inline void leg_all(int n, double x, double* v, double* d, double* dd) {
  const double t = 2.0 * x - 1.0;
  double P[8], dP[8], ddP[8];
  P[0] = 1.0; dP[0] = 0.0; ddP[0] = 0.0;
  if (n > 1) { P[1] = t; dP[1] = 1.0; ddP[1] = 0.0; }
  for (int k = 1; k + 1 < n; ++k) {
    P[k + 1] = ((2 * k + 1) * t * P[k] - k * P[k - 1]) / (k + 1);
    dP[k + 1] = ((2 * k + 1) * (P[k] + t * dP[k]) - k * dP[k - 1]) / (k + 1);
    ddP[k + 1] = ((2 * k + 1) * (2.0 * dP[k] + t * ddP[k]) - k * ddP[k - 1]) / (k + 1);
  }
  for (int k = 0; k < n; ++k) {
    const double s = std::sqrt(2.0 * k + 1.0);
    v[k] = s * P[k];
    d[k] = 2.0 * s * dP[k];
    dd[k] = 4.0 * s * ddP[k];
  }
}

// Gauss-Legendre rule on [0,1], points increasing (deal.II QGauss<1>)
inline void gauss_rule(int n, double* x, double* w) {
  for (int i = 0; i < n; ++i) {
    long double z = std::cos(3.14159265358979323846L * (i + 0.75L) / (n + 0.5L));
    long double pp = 0;
    for (int it = 0; it < 100; ++it) {
      long double p1 = 1, p2 = 0;
      for (int j = 0; j < n; ++j) {
        long double p3 = p2;
        p2 = p1;
        p1 = ((2.0L * j + 1.0L) * z * p2 - j * p3) / (j + 1);
      }
      pp = n * (z * p1 - p2) / (z * z - 1.0L);
      long double z1 = z;
      z = z1 - p1 / pp;
      if (std::fabs((double)(z - z1)) < 1e-19) break;
    }
    x[i] = (double)(0.5L - 0.5L * z);
    w[i] = (double)(1.0L / ((1.0L - z * z) * pp * pp));
  }
}

template <typename T>
inline void fill_tab(Tab1D<T>& tb, int p) {
  std::memset(&tb, 0, sizeof(tb));
  const int n1 = p + 1, nq = p + 2;
  double x[8], w[8], v[8], d[8], dd[8];
  gauss_rule(nq, x, w);
  for (int q = 0; q < nq; ++q) {
    tb.xq[q] = T(x[q]);
    tb.wq[q] = T(w[q]);
    leg_all(n1, x[q], v, d, dd);
    for (int a = 0; a < n1; ++a) { tb.Lq[a][q] = T(v[a]); tb.Dq[a][q] = T(d[a]); tb.Hq[a][q] = T(dd[a]); }
  }
  leg_all(n1, 0.0, v, d, dd);
  for (int a = 0; a < n1; ++a) { tb.L0[a] = T(v[a]); tb.D0[a] = T(d[a]); tb.H0[a] = T(dd[a]); }
  leg_all(n1, 1.0, v, d, dd);
  for (int a = 0; a < n1; ++a) { tb.L1[a] = T(v[a]); tb.D1[a] = T(d[a]); tb.H1[a] = T(dd[a]); }
  // A_ab = int_0^1 L_a' L_b (exact with the (p+2)-point rule)
  for (int a = 0; a < n1; ++a)
    for (int b = 0; b < n1; ++b) {
      long double s = 0;
      for (int q = 0; q < nq; ++q) {
        double va[8], da[8], dda[8];
        leg_all(n1, x[q], va, da, dda);
        s += (long double)w[q] * da[a] * va[b];
      }
      tb.A[a][b] = T((double)s);
    }
  {
    double l0[8], l1[8], tmp1[8], tmp2[8];
    leg_all(n1, 0.0, l0, tmp1, tmp2);
    leg_all(n1, 1.0, l1, tmp1, tmp2);
    for (int q = 0; q < nq; ++q) {
      leg_all(n1, x[q], v, d, dd);
      double k0 = 0.0, k1 = 0.0;
      for (int a = 0; a < n1; ++a) { k0 += v[a] * l0[a]; k1 += v[a] * l1[a]; }
      tb.K0q[q] = T(k0);
      tb.K1q[q] = T(k1);
    }
    for (int e = 0; e < 2; ++e) {
      const double* le = e ? l1 : l0;
      double k0 = 0.0, k1 = 0.0;
      for (int a = 0; a < n1; ++a) { k0 += le[a] * l0[a]; k1 += le[a] * l1[a]; }
      tb.K0v[e] = T(k0);
      tb.K1v[e] = T(k1);
    }
  }
  gauss_rule(n1, x, w);
  for (int q = 0; q < n1; ++q) {
    tb.xl[q] = T(x[q]);
    tb.wl[q] = T(w[q]);
    leg_all(n1, x[q], v, d, dd);
    for (int a = 0; a < n1; ++a) { tb.Ll[a][q] = T(v[a]); tb.Dl[a][q] = T(d[a]); }
  }
}

// fills this translation unit's constant tables
inline cudaError_t upload_tables_here() {
  static Tab1D<double> td[kMaxP + 1];
  static Tab1D<float> tf[kMaxP + 1];
  for (int p = 0; p <= kMaxP; ++p) {
    fill_tab(td[p], p);
    fill_tab(tf[p], p);
  }
  cudaError_t e = cudaMemcpyToSymbol(c_tab_d, td, sizeof(td));
  if (e != cudaSuccess) return e;
  return cudaMemcpyToSymbol(c_tab_f, tf, sizeof(tf));
}

}  // namespace flsp

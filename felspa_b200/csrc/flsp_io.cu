// flsp_io.cu — output of the level-set field: point values of every cell's
// polynomial on the device, and the VTU / PVD writers on the host.
//
// FELSPA writes its solutions through deal.II's DataOut
// (LevelSetSurface::export_solution, include/felspa/level_set/src/
// level_set.implement.h:313-342; SimulatorBase::export_solutions,
// src/pde/pde_base.cc:93-115; PVDCollector, src/base/io.cc:110-166).
// DataOut::build_patches(n) turns every cell into one patch of (n+1)^dim
// equispaced vertices (n = 1 by default: the cell's corners) and evaluates
// the DG polynomial of that cell there, so neighbouring patches carry the
// two one-sided values of a discontinuous field.  Here the evaluation is a
// device kernel over all (cell, vertex) pairs in FP64; the host only formats
// the values.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "flsp_launch.h"
#include "flsp_tables.h"

namespace flsp {

int upload_tables_io() {
  cudaError_t e = upload_tables_here();
  if (e != cudaSuccess) return set_error(FLSP_ERR_CUDA, std::string("tables: ") + cudaGetErrorString(e));
  return FLSP_OK;
}

// values of the orthonormal Legendre polynomials L_0..L_{n1-1} on [0,1]
// at s: L_a(s) = sqrt(2a+1) P_a(2s-1), P by Bonnet's recurrence
__device__ __forceinline__ void legendre01(int n1, double s, double* L) {
  const double t = 2.0 * s - 1.0;
  double pm = 1.0, pc = t;
  L[0] = 1.0;
  if (n1 > 1) L[1] = sqrt(3.0) * t;
  for (int k = 1; k + 1 < n1; ++k) {
    const double pn = ((2 * k + 1) * t * pc - k * pm) / (k + 1);
    pm = pc;
    pc = pn;
    L[k + 1] = sqrt(2.0 * (k + 1) + 1.0) * pn;
  }
}

// out[k * npt + j] = phi of host cell k at patch vertex j (x fastest)
template <typename T>
__global__ void __launch_bounds__(256) eval_patch_kernel(const MeshArgs m, int dim, int n1, int n_sub, const T* __restrict__ phi,
                                                         const int64_t* __restrict__ perm, double* __restrict__ out) {
  const int ns1 = n_sub + 1;
  const long long npt = dim == 3 ? (long long)ns1 * ns1 * ns1 : (long long)ns1 * ns1;
  const long long total = m.ncell * npt;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long k = idx / npt;
    const int j = (int)(idx - k * npt);
    const long long c = perm ? perm[k] : k;
    double L[3][kMaxN1];
    legendre01(n1, (double)(j % ns1) / n_sub, L[0]);
    legendre01(n1, (double)((j / ns1) % ns1) / n_sub, L[1]);
    if (dim == 3) legendre01(n1, (double)(j / (ns1 * ns1)) / n_sub, L[2]);
    const T* cc = phi + c * m.nb;
    double v = 0.0;
    const int n3 = dim == 3 ? n1 : 1;
    for (int a2 = 0; a2 < n3; ++a2)
      for (int a1 = 0; a1 < n1; ++a1)
        for (int a0 = 0; a0 < n1; ++a0) {
          const int gi = m.q2g[a0 + n1 * (a1 + n1 * a2)];
          if (gi < 0) continue;
          const double w = L[0][a0] * L[1][a1] * (dim == 3 ? L[2][a2] : 1.0);
          v += (double)cc[gi] * w;
        }
    out[idx] = v;
  }
}

int launch_eval_patches(const Ctx& c, const void* phi, const int64_t* perm, int n_sub, double* out) {
  const long long npt = c.dim == 3 ? (long long)(n_sub + 1) * (n_sub + 1) * (n_sub + 1)
                                   : (long long)(n_sub + 1) * (n_sub + 1);
  const long long total = c.m.ncell * npt;
  const int grid = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
  if (c.prec == FLSP_FP64)
    eval_patch_kernel<double><<<grid, 256, 0, c.stream>>>(c.m, c.dim, c.p + 1, n_sub, (const double*)phi, perm, out);
  else
    eval_patch_kernel<float><<<grid, 256, 0, c.stream>>>(c.m, c.dim, c.p + 1, n_sub, (const float*)phi, perm, out);
  return launch_status("eval_patch_kernel");
}

// ---------------------------------------------------------------------
// MaterialStack mixing, MaterialAccessor<MaterialStack>::reinit +
// eval_scalars (include/felspa/level_set/src/material_stack.implement.h:
// 320-470): at every Gauss point of every cell, the level sets in stack
// order each take the share rest * H(-phi_i) of what the earlier ones left
// (rest starts at 1; a share or rest of magnitude <= DBL_EPSILON counts as
// zero, numerics::is_zero), the background material the remaining rest;
// the mixed scalar is the share-weighted sum of the materials' values.
// H is LevelSetSurface::domain_identity (level_set.implement.h:356-380):
// sharp, linear or sine smoothing over eps = 1.5 min_diameter
// (level_set.implement.h:957-993).  One thread per (cell, point), FP64.
// ---------------------------------------------------------------------
__device__ __forceinline__ double mix_heaviside(double y, double eps, int kind) {
  const double kEpsD = 2.220446049250313e-16;
  if (kind == FLSP_HEAVISIDE_NONE) return y > 0.0 ? 1.0 : (y < 0.0 ? 0.0 : 0.5);
  if (y > eps) return 1.0;
  if (y < -eps) return 0.0;
  if (kind == FLSP_HEAVISIDE_LINEAR) return 0.5 * (y / eps + 1.0);
  const double v = 0.5 * (1.0 + y / eps + sin(y * 3.14159265358979323846 / eps) / 3.14159265358979323846);
  if (fabs(v) < kEpsD) return 0.0;
  if (fabs(v - 1.0) < kEpsD) return 1.0;
  return v;
}

__global__ void __launch_bounds__(256) material_mix_kernel(const MixArgs a, double* __restrict__ out) {
  const double kEpsD = 2.220446049250313e-16;
  const int nq = a.nq;
  const long long npt = a.dim == 3 ? (long long)nq * nq * nq : (long long)nq * nq;
  const long long total = a.ncell * npt;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long k = idx / npt;
    const int j = (int)(idx - k * npt);
    const long long c = a.perm ? a.perm[k] : k;
    const int qx = j % nq, qy = (j / nq) % nq, qz = a.dim == 3 ? j / (nq * nq) : 0;
    double rest = 1.0, v = 0.0;
    for (int i = 0; i < a.n && !(fabs(rest) <= kEpsD); ++i) {
      const MixLevelSet& ls = a.ls[i];
      const int n1 = ls.n1, n3 = a.dim == 3 ? n1 : 1;
      double phi = 0.0;
      for (int a2 = 0; a2 < n3; ++a2)
        for (int a1 = 0; a1 < n1; ++a1)
          for (int a0 = 0; a0 < n1; ++a0) {
            const int gi = ls.q2g[a0 + n1 * (a1 + n1 * a2)];
            if (gi < 0) continue;
            const double cv = ls.prec == FLSP_FP64 ? ((const double*)ls.phi)[c * ls.nb + gi]
                                                   : (double)((const float*)ls.phi)[c * ls.nb + gi];
            phi += cv * a.L[a0][qx] * a.L[a1][qy] * (a.dim == 3 ? a.L[a2][qz] : 1.0);
          }
      const double H = mix_heaviside(-phi, ls.eps, a.smoothing);
      if (!(fabs(H) <= kEpsD)) {
        const double share = rest * H;
        v += a.value[i] * share;
        rest -= share;
      }
    }
    if (!(fabs(rest) <= kEpsD)) v += a.value[a.n] * rest;
    out[idx] = v;
  }
}

int launch_material_mix(const MixArgs& a, cudaStream_t s, double* out) {
  const long long npt = a.dim == 3 ? (long long)a.nq * a.nq * a.nq : (long long)a.nq * a.nq;
  const long long total = a.ncell * npt;
  const int grid = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
  material_mix_kernel<<<grid, 256, 0, s>>>(a, out);
  return launch_status("material_mix_kernel");
}

// ---------------------------------------------------------------------
// Curvature estimate, LevelSetSurface::CurvatureEstimator::estimate
// (include/felspa/level_set/src/level_set.implement.h:600-812): the weak
// divergence of n = grad phi / |grad phi| on QGauss(p+1) cell and face
// rules, the mass solve (|K| I), then |coefficient|.  One thread per cell,
// FP64 arithmetic from the FP64 or FP32 state:
//   cell:     R_i -= sum_q grad psi_i . n JxW                     (:747-763)
//   boundary: R_i += n . normal psi_i JxW                          (:796-811)
//   interior face, per component d (:766-792):
//     s = (n_in[d] - n_ex[d]) / (phi_in - phi_ex),
//     F[d] = s > 0 ? (normal[d] > 0 ? n_in[d] : n_ex[d])
//          : s < 0 ? (normal[d] > 0 ? n_ex[d] : n_in[d]) : 0 (also for NaN);
//     only F along the face normal survives F . normal (the tangential
//     entries are finite or zero).
// mode FLSP_CURV_REFERENCE: the face belongs to the cell with the lower
// CellId (its position in the host order, :717) and both of its terms go
// to that cell's DoFs, psi^in F.normal - psi^ex F.normal with psi^ex the
// same-index basis function of the neighbour at the shared points: the
// reference binds its exterior copy to the cell (copy_ex.reinit(cell),
// :731), so the neighbour receives nothing from that face.
// mode FLSP_CURV_NEIGHBOUR: every cell adds psi_i F.normal_own over each of
// its interior faces (F is the same from either side), the exterior term
// of a standard DG flux.
// ---------------------------------------------------------------------
__global__ void inv_perm_kernel(const int64_t* __restrict__ perm, long long n, int64_t* __restrict__ pos) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    pos[perm[k]] = k;
}

// value and gradient (physical) of a Q-layout cell polynomial from the
// per-axis factors Lx[e][a] (values) and Dx[e][a] (reference derivatives)
template <int DIM, int N1>
__device__ __forceinline__ void eval_point(const double* cq, const double (&Lx)[3][kMaxN1],
                                           const double (&Dx)[3][kMaxN1], const double* ih, double* val,
                                           double* g) {
  constexpr int NZ = DIM > 2 ? N1 : 1;
  double v = 0.0, g0 = 0.0, g1 = 0.0, g2 = 0.0;
#pragma unroll
  for (int a2 = 0; a2 < NZ; ++a2)
#pragma unroll
    for (int a1 = 0; a1 < N1; ++a1)
#pragma unroll
      for (int a0 = 0; a0 < N1; ++a0) {
        const double c = cq[a0 + N1 * (a1 + N1 * a2)];
        const double z = DIM > 2 ? Lx[2][a2] : 1.0, dz = DIM > 2 ? Dx[2][a2] : 0.0;
        v += c * Lx[0][a0] * Lx[1][a1] * z;
        g0 += c * Dx[0][a0] * Lx[1][a1] * z;
        g1 += c * Lx[0][a0] * Dx[1][a1] * z;
        g2 += c * Lx[0][a0] * Lx[1][a1] * dz;
      }
  *val = v;
  g[0] = g0 * ih[0];
  g[1] = g1 * ih[1];
  g[2] = DIM > 2 ? g2 * ih[2] : 0.0;
}

template <int DIM, int P, typename T>
__global__ void __launch_bounds__(128) curvature_kernel(const MeshArgs m, const T* __restrict__ phi,
                                                        const int64_t* __restrict__ pos, int mode,
                                                        double* __restrict__ out) {
  constexpr int N1 = P + 1, NM = DIM > 2 ? N1 * N1 * N1 : N1 * N1, NZ = DIM > 2 ? N1 : 1;
  const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= m.ncell) return;
  const Tab1D<double>& tb = tab<double>(P);
  const int I[3] = {(int)(c % m.n[0]), (int)((c / m.n[0]) % m.n[1]), DIM > 2 ? (int)(c / ((long long)m.n[0] * m.n[1])) : 0};
  const double ih[3] = {1.0 / m.h[0], 1.0 / m.h[1], DIM > 2 ? 1.0 / m.h[2] : 1.0};
  const double vol = m.vol;
  auto load = [&](long long cell, double* cq) {
#pragma unroll
    for (int q = 0; q < NM; ++q) {
      const int gi = m.q2g[q];
      cq[q] = gi >= 0 ? (double)phi[cell * m.nb + gi] : 0.0;
    }
  };
  double cq[NM], R[NM];
  load(c, cq);
#pragma unroll
  for (int q = 0; q < NM; ++q) R[q] = 0.0;
  double Lx[3][kMaxN1], Dx[3][kMaxN1];

  // ---- cell term
  for (int q2 = 0; q2 < NZ; ++q2)
    for (int q1 = 0; q1 < N1; ++q1)
      for (int q0 = 0; q0 < N1; ++q0) {
        const int qq[3] = {q0, q1, q2};
#pragma unroll
        for (int e = 0; e < DIM; ++e)
#pragma unroll
          for (int a = 0; a < N1; ++a) {
            Lx[e][a] = tb.Ll[a][qq[e]];
            Dx[e][a] = tb.Dl[a][qq[e]];
          }
        double val, g[3];
        eval_point<DIM, N1>(cq, Lx, Dx, ih, &val, g);
        const double nrm = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
        const double n0 = g[0] / nrm, n1 = g[1] / nrm, n2 = g[2] / nrm;
        const double jxw = tb.wl[q0] * tb.wl[q1] * (DIM > 2 ? tb.wl[q2] : 1.0) * vol;
#pragma unroll
        for (int a2 = 0; a2 < NZ; ++a2)
#pragma unroll
          for (int a1 = 0; a1 < N1; ++a1)
#pragma unroll
            for (int a0 = 0; a0 < N1; ++a0) {
              const double z = DIM > 2 ? Lx[2][a2] : 1.0;
              double dot = (Dx[0][a0] * Lx[1][a1] * z * ih[0]) * n0 + (Lx[0][a0] * Dx[1][a1] * z * ih[1]) * n1;
              if (DIM > 2) dot += (Lx[0][a0] * Lx[1][a1] * Dx[2][a2] * ih[2]) * n2;
              R[a0 + N1 * (a1 + N1 * a2)] -= dot * jxw;
            }
      }

  // ---- faces
  for (int f = 0; f < 2 * DIM; ++f) {
    const int E = f / 2, side = f % 2;
    const int t0 = E == 0 ? 1 : 0, t1 = E == 2 ? 1 : 2;
    int J[3] = {I[0], I[1], I[2]};
    J[E] += side ? 1 : -1;
    const bool boundary = J[E] < 0 || J[E] >= m.n[E];
    const long long nbc = boundary ? -1 : J[0] + (long long)m.n[0] * (J[1] + (long long)m.n[1] * J[2]);
    if (!boundary && mode == FLSP_CURV_REFERENCE) {
      const long long pc = pos ? pos[c] : c, pn = pos ? pos[nbc] : nbc;
      if (pc > pn) continue;   // the neighbour owns this face
    }
    const double sgn = side ? 1.0 : -1.0;
    const double area = vol * (E == 0 ? ih[0] : (E == 1 ? ih[1] : ih[2]));
    double cn[NM];
    if (!boundary) load(nbc, cn);
    for (int qb = 0; qb < (DIM > 2 ? N1 : 1); ++qb)
      for (int qa = 0; qa < N1; ++qa) {
        const double jxw = tb.wl[qa] * (DIM > 2 ? tb.wl[qb] : 1.0) * area;
#pragma unroll
        for (int a = 0; a < N1; ++a) {
          Lx[t0][a] = tb.Ll[a][qa];
          Dx[t0][a] = tb.Dl[a][qa];
          if (DIM > 2) {
            Lx[t1][a] = tb.Ll[a][qb];
            Dx[t1][a] = tb.Dl[a][qb];
          }
          Lx[E][a] = side ? tb.L1[a] : tb.L0[a];
          Dx[E][a] = side ? tb.D1[a] : tb.D0[a];
        }
        double pin, gin[3];
        eval_point<DIM, N1>(cq, Lx, Dx, ih, &pin, gin);
        const double nin = sqrt(gin[0] * gin[0] + gin[1] * gin[1] + gin[2] * gin[2]);
        double fn;
        if (boundary) {
          fn = gin[E] / nin * sgn;
        } else {
          // the neighbour's trace: its own face on the other side
#pragma unroll
          for (int a = 0; a < N1; ++a) {
            Lx[E][a] = side ? tb.L0[a] : tb.L1[a];
            Dx[E][a] = side ? tb.D0[a] : tb.D1[a];
          }
          double pex, gex[3];
          eval_point<DIM, N1>(cn, Lx, Dx, ih, &pex, gex);
          const double nex = sqrt(gex[0] * gex[0] + gex[1] * gex[1] + gex[2] * gex[2]);
          const double ui = gin[E] / nin, ue = gex[E] / nex;
          const double sh = (ui - ue) / (pin - pex);
          double F = 0.0;
          if (sh > 0.0) F = sgn > 0 ? ui : ue;
          else if (sh < 0.0) F = sgn > 0 ? ue : ui;
          fn = F * sgn;
          // restore the own side's normal factors for the test functions
#pragma unroll
          for (int a = 0; a < N1; ++a) Lx[E][a] = side ? tb.L1[a] : tb.L0[a];
        }
        const double ref_ex = (!boundary && mode == FLSP_CURV_REFERENCE) ? 1.0 : 0.0;
#pragma unroll
        for (int a2 = 0; a2 < NZ; ++a2)
#pragma unroll
          for (int a1 = 0; a1 < N1; ++a1)
#pragma unroll
            for (int a0 = 0; a0 < N1; ++a0) {
              const int aa[3] = {a0, a1, a2};
              double tang = 1.0;
#pragma unroll
              for (int e = 0; e < DIM; ++e)
                if (e != E) tang *= Lx[e][aa[e]];
              const double lin = side ? tb.L1[aa[E]] : tb.L0[aa[E]];
              const double lex = side ? tb.L0[aa[E]] : tb.L1[aa[E]];
              double r = R[a0 + N1 * (a1 + N1 * a2)];
              r += (lin * tang) * fn * jxw;
              if (ref_ex != 0.0) r -= (lex * tang) * fn * jxw;
              R[a0 + N1 * (a1 + N1 * a2)] = r;
            }
      }
  }
  const long long dst = (pos ? pos[c] : c) * m.nb;
#pragma unroll
  for (int q = 0; q < NM; ++q) {
    const int gi = m.q2g[q];
    if (gi >= 0) out[dst + gi] = fabs(R[q] / vol);
  }
}

int launch_curvature(const Ctx& c, const void* phi, const int64_t* perm, int64_t* pos_scratch, int mode,
                     double* out) {
  const int64_t* pos = nullptr;
  if (perm) {
    const int grid = (int)std::min<long long>((c.m.ncell + 255) / 256, 148LL * 16);
    inv_perm_kernel<<<grid, 256, 0, c.stream>>>(perm, c.m.ncell, pos_scratch);
    int st = launch_status("inv_perm_kernel");
    if (st) return st;
    pos = pos_scratch;
  }
  const int blocks = (int)((c.m.ncell + 127) / 128);
  return dispatch(c, [&](auto D, auto PP, auto tz) -> int {
    constexpr int DIM = decltype(D)::value, P = decltype(PP)::value;
    using T = decltype(tz);
    curvature_kernel<DIM, P, T><<<blocks, 128, 0, c.stream>>>(c.m, reinterpret_cast<const T*>(phi), pos, mode, out);
    return launch_status("curvature_kernel");
  });
}

namespace {

// labels become XML attribute values and parts of file names: letters,
// digits, '_', '-' and '.' only
bool plain_label(const char* s) {
  if (!s || !s[0]) return false;
  for (const char* c = s; *c; ++c) {
    const bool ok = (*c >= 'a' && *c <= 'z') || (*c >= 'A' && *c <= 'Z') || (*c >= '0' && *c <= '9') || *c == '_' ||
                    *c == '-' || *c == '.';
    if (!ok) return false;
  }
  return true;
}

bool write_all(FILE* f, const std::string& s) { return std::fwrite(s.data(), 1, s.size(), f) == s.size(); }

}  // namespace

int write_vtu_file(const flsp_mesh_desc* mesh, int n_sub, const double* values, const char* label,
                   const char* filename, const double* values2, const char* label2) {
  if (!mesh || !values || !label || !filename || !label[0] || !filename[0])
    return set_error(FLSP_ERR_BAD_ARG, "null or empty argument");
  if (!plain_label(label) || (values2 && !plain_label(label2)))
    return set_error(FLSP_ERR_BAD_ARG, "labels may hold letters, digits, '_', '-' and '.' only");
  const int dim = mesh->dim;
  if (dim != 2 && dim != 3) return set_error(FLSP_ERR_BAD_ARG, "dim must be 2 or 3");
  if (n_sub < 1 || n_sub > 16) return set_error(FLSP_ERR_BAD_ARG, "n_sub must be in 1..16");
  long long ncell = 1;
  for (int e = 0; e < dim; ++e) {
    if (mesh->n[e] < 1 || !(mesh->hi[e] > mesh->lo[e])) return set_error(FLSP_ERR_BAD_MESH, "bad mesh extent");
    ncell *= mesh->n[e];
  }
  const int ns1 = n_sub + 1;
  const long long npt = dim == 3 ? (long long)ns1 * ns1 * ns1 : (long long)ns1 * ns1;
  const long long nsub = dim == 3 ? (long long)n_sub * n_sub * n_sub : (long long)n_sub * n_sub;
  const long long n_points = ncell * npt, n_cells = ncell * nsub;
  double h[3] = {0, 0, 0};
  for (int e = 0; e < dim; ++e) h[e] = (mesh->hi[e] - mesh->lo[e]) / mesh->n[e];

  FILE* f = std::fopen(filename, "wb");
  if (!f) return set_error(FLSP_ERR_BAD_ARG, std::string("cannot open ") + filename);
  bool ok = true;
  char buf[256];
  std::string s;
  s.reserve(1 << 20);
  auto flush = [&](bool force) {
    if (force || s.size() > (1u << 20)) {
      ok = ok && write_all(f, s);
      s.clear();
    }
  };
  s += "<?xml version=\"1.0\" ?>\n"
       "<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n"
       "<UnstructuredGrid>\n";
  std::snprintf(buf, sizeof(buf), "<Piece NumberOfPoints=\"%lld\" NumberOfCells=\"%lld\">\n", n_points, n_cells);
  s += buf;
  // patch vertices, cells in host order, x fastest inside a patch
  s += "<Points>\n<DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"ascii\">\n";
  for (long long k = 0; k < ncell; ++k) {
    const long long c = mesh->host_cell_order ? mesh->host_cell_order[k] : k;
    if (c < 0 || c >= ncell) {
      std::fclose(f);
      return set_error(FLSP_ERR_BAD_MESH, "host_cell_order entry out of range");
    }
    const long long ix = c % mesh->n[0], iy = (c / mesh->n[0]) % mesh->n[1];
    const long long iz = dim == 3 ? c / ((long long)mesh->n[0] * mesh->n[1]) : 0;
    for (long long j = 0; j < npt; ++j) {
      const int j0 = (int)(j % ns1), j1 = (int)((j / ns1) % ns1), j2 = dim == 3 ? (int)(j / (ns1 * ns1)) : 0;
      const double x = mesh->lo[0] + h[0] * (ix + (double)j0 / n_sub);
      const double y = mesh->lo[1] + h[1] * (iy + (double)j1 / n_sub);
      const double z = dim == 3 ? mesh->lo[2] + h[2] * (iz + (double)j2 / n_sub) : 0.0;
      std::snprintf(buf, sizeof(buf), "%.17g %.17g %.17g\n", x, y, z);
      s += buf;
    }
    flush(false);
  }
  s += "</DataArray>\n</Points>\n<Cells>\n<DataArray type=\"Int64\" Name=\"connectivity\" format=\"ascii\">\n";
  // sub-cells of every patch: VTK_QUAD (counter-clockwise) / VTK_HEXAHEDRON
  // (lower face counter-clockwise, then the upper face)
  for (long long k = 0; k < ncell; ++k) {
    const long long base = k * npt;
    for (long long sc = 0; sc < nsub; ++sc) {
      const int s0 = (int)(sc % n_sub), s1 = (int)((sc / n_sub) % n_sub), s2 = dim == 3 ? (int)(sc / (n_sub * n_sub)) : 0;
      auto v = [&](int a, int b, int cc) -> long long { return base + a + ns1 * (b + (long long)ns1 * cc); };
      if (dim == 2) {
        std::snprintf(buf, sizeof(buf), "%lld %lld %lld %lld\n", v(s0, s1, 0), v(s0 + 1, s1, 0), v(s0 + 1, s1 + 1, 0),
                      v(s0, s1 + 1, 0));
      } else {
        std::snprintf(buf, sizeof(buf), "%lld %lld %lld %lld %lld %lld %lld %lld\n", v(s0, s1, s2), v(s0 + 1, s1, s2),
                      v(s0 + 1, s1 + 1, s2), v(s0, s1 + 1, s2), v(s0, s1, s2 + 1), v(s0 + 1, s1, s2 + 1),
                      v(s0 + 1, s1 + 1, s2 + 1), v(s0, s1 + 1, s2 + 1));
      }
      s += buf;
    }
    flush(false);
  }
  s += "</DataArray>\n<DataArray type=\"Int64\" Name=\"offsets\" format=\"ascii\">\n";
  const int nv = dim == 3 ? 8 : 4;
  for (long long i = 0; i < n_cells; ++i) {
    std::snprintf(buf, sizeof(buf), "%lld\n", (i + 1) * nv);
    s += buf;
    flush(false);
  }
  s += "</DataArray>\n<DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\">\n";
  const char* ty = dim == 3 ? "12\n" : "9\n";
  for (long long i = 0; i < n_cells; ++i) {
    s += ty;
    flush(false);
  }
  s += "</DataArray>\n</Cells>\n";
  s += std::string("<PointData Scalars=\"") + label + "\">\n<DataArray type=\"Float64\" Name=\"" + label +
       "\" format=\"ascii\">\n";
  for (long long i = 0; i < n_points; ++i) {
    std::snprintf(buf, sizeof(buf), "%.17g\n", values[i]);
    s += buf;
    flush(false);
  }
  s += "</DataArray>\n";
  if (values2 && label2 && label2[0]) {
    s += std::string("<DataArray type=\"Float64\" Name=\"") + label2 + "\" format=\"ascii\">\n";
    for (long long i = 0; i < n_points; ++i) {
      std::snprintf(buf, sizeof(buf), "%.17g\n", values2[i]);
      s += buf;
      flush(false);
    }
    s += "</DataArray>\n";
  }
  s += "</PointData>\n</Piece>\n</UnstructuredGrid>\n</VTKFile>\n";
  flush(true);
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) return set_error(FLSP_ERR_BAD_ARG, std::string("write failed: ") + filename);
  return FLSP_OK;
}

int write_pvd_file(const char* filename, int n, const double* times, const char* const* files) {
  if (!filename || !filename[0] || n < 0 || (n > 0 && (!times || !files)))
    return set_error(FLSP_ERR_BAD_ARG, "null or empty argument");
  // every record is checked before the file is opened, so a rejected call
  // leaves an existing collection as it was
  for (int i = 0; i < n; ++i)
    if (!files[i] || !plain_label(files[i]))
      return set_error(FLSP_ERR_BAD_ARG, "PVD records: file names of letters, digits, '_', '-' and '.' only");
  FILE* f = std::fopen(filename, "wb");
  if (!f) return set_error(FLSP_ERR_BAD_ARG, std::string("cannot open ") + filename);
  std::string s =
      "<?xml version=\"1.0\"?>\n"
      "<VTKFile type=\"Collection\" version=\"0.1\" ByteOrder=\"LittleEndian\">\n"
      "  <Collection>\n";
  char buf[64];
  for (int i = 0; i < n; ++i) {
    std::snprintf(buf, sizeof(buf), "%.17g", times[i]);
    s += std::string("    <DataSet timestep=\"") + buf + "\" group=\"\" part=\"0\" file=\"" + files[i] + "\"/>\n";
  }
  s += "  </Collection>\n</VTKFile>\n";
  const bool ok = write_all(f, s);
  if (std::fclose(f) != 0 || !ok) return set_error(FLSP_ERR_BAD_ARG, std::string("write failed: ") + filename);
  return FLSP_OK;
}

}  // namespace flsp

extern "C" int flsp_write_vtu(const flsp_mesh_desc* mesh, int n_sub, const double* values, const char* label,
                              const char* filename) {
  return flsp::write_vtu_file(mesh, n_sub, values, label, filename, nullptr, nullptr);
}

extern "C" int flsp_write_pvd(const char* filename, int n, const double* times, const char* const* files) {
  return flsp::write_pvd_file(filename, n, times, files);
}

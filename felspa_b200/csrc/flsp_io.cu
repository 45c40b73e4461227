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

namespace flsp {

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

namespace {

bool write_all(FILE* f, const std::string& s) { return std::fwrite(s.data(), 1, s.size(), f) == s.size(); }

}  // namespace

int write_vtu_file(const flsp_mesh_desc* mesh, int n_sub, const double* values, const char* label,
                   const char* filename) {
  if (!mesh || !values || !label || !filename || !label[0] || !filename[0])
    return set_error(FLSP_ERR_BAD_ARG, "null or empty argument");
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
  s += "</DataArray>\n</PointData>\n</Piece>\n</UnstructuredGrid>\n</VTKFile>\n";
  flush(true);
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) return set_error(FLSP_ERR_BAD_ARG, std::string("write failed: ") + filename);
  return FLSP_OK;
}

int write_pvd_file(const char* filename, int n, const double* times, const char* const* files) {
  if (!filename || !filename[0] || n < 0 || (n > 0 && (!times || !files)))
    return set_error(FLSP_ERR_BAD_ARG, "null or empty argument");
  FILE* f = std::fopen(filename, "wb");
  if (!f) return set_error(FLSP_ERR_BAD_ARG, std::string("cannot open ") + filename);
  std::string s =
      "<?xml version=\"1.0\"?>\n"
      "<VTKFile type=\"Collection\" version=\"0.1\" ByteOrder=\"LittleEndian\">\n"
      "  <Collection>\n";
  char buf[64];
  for (int i = 0; i < n; ++i) {
    if (!files[i]) {
      std::fclose(f);
      return set_error(FLSP_ERR_BAD_ARG, "null file name");
    }
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
  return flsp::write_vtu_file(mesh, n_sub, values, label, filename);
}

extern "C" int flsp_write_pvd(const char* filename, int n, const double* times, const char* const* files) {
  return flsp::write_pvd_file(filename, n, times, files);
}

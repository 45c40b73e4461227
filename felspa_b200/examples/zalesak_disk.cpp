// zalesak_disk.cpp — C++ driver of the Zalesak slotted-disk level-set test
// on the GPU path, written against the reference-named facade
// (include/flsp_dg.hpp).  It follows tests/test_zalesak_disk.cc of FELSPA:
// [-50, 50]^2 from subdivided_hyper_cube(2) refined 5 times (64 x 64 cells,
// deal.II active-cell order), FE_DGP degree 1, clockwise rigid rotation
// w = pi/314 about the origin, disk r = 15 at (0, 25) minus the slot
// (-2.499999, 15)-(2.499999, 40), reinit every 40 substeps with CFL 0.3,
// 628 calls of advance_time(1.0, false) for one revolution.
//
//   zalesak_disk [n_outer_steps=628] [viscosity=0] [export_prefix]
//
// With an export prefix the solution is written as VTU files (plus a PVD
// collection) before the loop, after the first and after the last outer
// step, as the reference test does.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <vector>

#include "flsp_dg.hpp"

// deal.II active-cell order of subdivided_hyper_cube(nsub) + refine_global(nref)
static std::vector<int64_t> dealii_order(int nsub, int nref) {
  const int N = nsub << nref;
  std::vector<int64_t> order;
  std::function<void(int, int, int)> rec = [&](int ix, int iy, int level) {
    if (level == nref) { order.push_back(ix + (int64_t)N * iy); return; }
    for (int cy = 0; cy < 2; ++cy)
      for (int cx = 0; cx < 2; ++cx) rec(2 * ix + cx, 2 * iy + cy, level + 1);
  };
  for (int ky = 0; ky < nsub; ++ky)
    for (int kx = 0; kx < nsub; ++kx) rec(kx, ky, 0);
  return order;
}

int main(int argc, char** argv) {
  const int n_outer = argc > 1 ? std::atoi(argv[1]) : 628;
  const double viscosity = argc > 2 ? std::atof(argv[2]) : 0.0;
  const char* export_prefix = argc > 3 ? argv[3] : nullptr;
  try {
    flsp::Mesh mesh;
    mesh.dim = 2;
    mesh.n[0] = mesh.n[1] = 64;
    mesh.lo[0] = mesh.lo[1] = -50.0;
    mesh.hi[0] = mesh.hi[1] = 50.0;
    mesh.host_cell_order = dealii_order(2, 5);

    flsp::LevelSetSurface ls(mesh, 1, FLSP_BASIS_P, FLSP_FP64);
    ls.control().reinit_frequency = 40;
    ls.control().reinit.cfl_max = 0.3;
    ls.control().reinit.viscosity = viscosity;
    const flsp_ic_desc ic = flsp::slotted_disk(0.0, 25.0, 15.0, -2.499999, 15.0, 2.499999, 40.0);
    ls.initialize(ic, flsp::rigid_body_rotation(0.0, 0.0, M_PI / 314.0));
    const std::vector<double> initial = ls.get_solution_vector();
    const double mass0 = ls.integrate_mass();

    if (export_prefix) ls.export_solutions(export_prefix);
    for (int i = 0; i < n_outer; ++i) {
      ls.advance_time(1.0, false);
      if (export_prefix && (i == 0 || i == n_outer - 1)) ls.export_solutions(export_prefix);
    }

    std::printf("time %.6f dofs %lld\n", ls.get_time(), (long long)ls.n_dofs());
    std::printf("mean |coeff - initial| %.6e\n", ls.compute_error(initial));
    std::printf("mass error vs exact disk %.6e\n", ls.compute_mass_error(ic));
    std::printf("mass drift %.6e\n", (ls.integrate_mass() - mass0) / mass0);
  } catch (const flsp::Exception& e) {
    std::fprintf(stderr, "error %d: %s\n", e.code(), e.what());
    return 1;
  }
  return 0;
}

// flsp_dg.hpp — header-only C++ facade over the C ABI (flsp_dg.h) with the
// class and method names of FELSPA's level-set simulators, so that a C++
// driver written against the reference reads the same:
//
//   flsp::AdvectSimulator    — dg::AdvectSimulator (include/felspa/pde/advection.h:91-381)
//   flsp::ReinitSimulatorLDG — dg::ReinitSimulatorLDG (include/felspa/level_set/reinit.h:154-268)
//   flsp::LevelSetSurface    — ls::LevelSetSurface (include/felspa/level_set/level_set.h:176-413)
//
// Non-zero library statuses become flsp::Exception (the reference throws
// EXCEPT_MSG exceptions, include/felspa/base/exceptions.h:227-245).  The
// mesh and DoF numbering stay with the caller: the solution vector is in
// the caller's cell order (MeshDesc::host_cell_order) with deal.II's DoF
// order inside each cell.
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "flsp_dg.h"

namespace flsp {

class Exception : public std::runtime_error {
 public:
  Exception(int code, const std::string& what) : std::runtime_error(what), code_(code) {}
  int code() const { return code_; }

 private:
  int code_;
};

inline void check(int status, const char* where) {
  if (status != FLSP_OK)
    throw Exception(status, std::string(where) + ": " + flsp_last_error());
}

struct Mesh {
  int dim = 2;
  int n[3] = {1, 1, 1};
  double lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
  std::vector<int64_t> host_cell_order;   // empty = lexicographic
  std::vector<int32_t> boundary_ids;      // per boundary face (flsp_mesh_desc order); empty = all 0

  flsp_mesh_desc desc() const {
    flsp_mesh_desc d;
    d.dim = dim;
    for (int i = 0; i < 3; ++i) { d.n[i] = n[i]; d.lo[i] = lo[i]; d.hi[i] = hi[i]; }
    d.host_cell_order = host_cell_order.empty() ? nullptr : host_cell_order.data();
    d.boundary_ids = boundary_ids.empty() ? nullptr : boundary_ids.data();
    return d;
  }
};

// one device-resident problem shared by the simulators below
class Problem {
 public:
  Problem(const Mesh& mesh, const flsp_dg_opts& opts) : mesh_(mesh) {
    flsp_mesh_desc d = mesh_.desc();
    check(flsp_create(&d, &opts, &h_), "flsp_create");
    check(flsp_n_dofs(h_, &n_dofs_), "flsp_n_dofs");
  }
  ~Problem() { flsp_destroy(h_); }
  Problem(const Problem&) = delete;
  Problem& operator=(const Problem&) = delete;

  flsp_handle* handle() const { return h_; }
  int64_t n_dofs() const { return n_dofs_; }
  const Mesh& mesh() const { return mesh_; }

 private:
  Mesh mesh_;
  flsp_handle* h_ = nullptr;
  int64_t n_dofs_ = 0;
};

class AdvectSimulator {
 public:
  AdvectSimulator(const Mesh& mesh, unsigned int fe_degree, int basis = FLSP_BASIS_P,
                  int precision = FLSP_FP64, const std::string& label = "Advect")
      : problem_(mesh, make_opts(fe_degree, basis, precision)), label_(label) {}
  virtual ~AdvectSimulator() = default;

  // AdvectSimulator::initialize(ScalarFunction, ptr_velocity_field)
  void initialize(const flsp_ic_desc& ic, const flsp_velocity_desc& velocity) {
    check(flsp_set_velocity(h(), &velocity), "flsp_set_velocity");
    check(flsp_project_ic(h(), &ic), "flsp_project_ic");
  }
  // AdvectSimulator::initialize(vector, ptr_velocity_field)
  void initialize(const std::vector<double>& coeffs, const flsp_velocity_desc& velocity) {
    check(flsp_set_velocity(h(), &velocity), "flsp_set_velocity");
    set_solution_vector(coeffs);
  }
  // the simulator velocity branch (VeloFcnType a simulator, e.g. the Stokes
  // solver of LevelSetStokes): the coupled FE field as nodal values of
  // degree `degree` on the mesh's Gauss-Lobatto lattice, components then
  // z, y, x (flsp_set_velocity_fe); call again after every solve of the
  // coupled simulator
  void set_velocity_field(int degree, const std::vector<double>& nodal_values) {
    check(flsp_set_velocity_fe(h(), degree, nodal_values.data(), (int64_t)nodal_values.size()),
          "flsp_set_velocity_fe");
  }
  // explicit_time_derivative(t, current solution) = M^-1 R(phi, t)
  std::vector<double> explicit_time_derivative(double current_time) const {
    std::vector<double> out(problem_.n_dofs());
    check(flsp_advect_rhs(h(), current_time, out.data(), (int64_t)out.size()), "flsp_advect_rhs");
    return out;
  }
  // advance_time(time_step, compute_single_cycle): CFL-limited SSP-RK substeps
  double advance_time(double time_step, bool compute_single_cycle) {
    double adv = 0.0;
    check(flsp_advance(h(), time_step, compute_single_cycle ? 1 : 0, &adv), "flsp_advance");
    return adv;
  }
  std::vector<double> get_solution_vector() const {
    std::vector<double> out(problem_.n_dofs());
    check(flsp_get_state(h(), out.data(), (int64_t)out.size()), "flsp_get_state");
    return out;
  }
  // append_boundary_condition(bc) for a Dirichlet condition of constant
  // value on the boundary faces of id boundary_id (> 0); a level set's
  // advection and reinitialisation share it (level_set.implement.h:384-392)
  void append_boundary_condition(int boundary_id, double dirichlet_value) {
    check(flsp_set_dirichlet(h(), boundary_id, dirichlet_value), "flsp_set_dirichlet");
  }
  void set_solution_vector(const std::vector<double>& v) {
    check(flsp_set_state(h(), v.data(), (int64_t)v.size()), "flsp_set_state");
  }
  double get_time() const {
    double t = 0.0;
    check(flsp_get_time(h(), &t), "flsp_get_time");
    return t;
  }
  // compute_error(vector): mean |coefficient difference| (advection.cc:471-484)
  double compute_error(const std::vector<double>& reference) const {
    std::vector<double> s = get_solution_vector();
    double acc = 0.0;
    for (size_t i = 0; i < s.size(); ++i) acc += std::abs(s[i] - reference[i]);
    return acc / (double)s.size();
  }
  // SimulatorBase::export_solutions(path) (pde_base.cc:93-115): the
  // solution's cell-corner values as <path><label>_<9-digit count>.vtu and
  // <path><label>.pvd listing every export with its time
  void export_solutions(const std::string& path) const {
    check(flsp_export_solutions(h(), path.c_str(), label_.c_str()), "flsp_export_solutions");
  }
  const std::string& get_label_string() const { return label_; }
  int64_t n_dofs() const { return problem_.n_dofs(); }
  flsp_handle* h() const { return problem_.handle(); }

 protected:
  static flsp_dg_opts make_opts(unsigned int p, int basis, int precision) {
    flsp_dg_opts o;
    flsp_default_dg_opts(&o);
    o.degree = (int)p;
    o.basis = basis;
    o.precision = precision;
    return o;
  }
  Problem problem_;
  std::string label_;
};

class ReinitSimulatorLDG {
 public:
  explicit ReinitSimulatorLDG(flsp_handle* h) : h_(h) { flsp_default_reinit_opts(&control_); }
  flsp_reinit_opts& control() { return control_; }
  // initialize(solution) + run_iteration(): iterations taken
  unsigned int run_iteration() {
    int nit = 0;
    check(flsp_reinit(h_, &control_, &nit), "flsp_reinit");
    return (unsigned int)nit;
  }

 private:
  flsp_handle* h_;
  flsp_reinit_opts control_;
};

class LevelSetSurface : public AdvectSimulator {
 public:
  LevelSetSurface(const Mesh& mesh, unsigned int fe_degree, int basis = FLSP_BASIS_P,
                  int precision = FLSP_FP64, const std::string& label = "LevelSet")
      : AdvectSimulator(mesh, fe_degree, basis, precision, label), reinit_(h()) {
    flsp_default_ls_opts(&control_);
  }
  flsp_ls_opts& control() { return control_; }

  // level_set.implement.h:119-142: project the IC; a non-exact IC gets a
  // global reinitialisation
  void initialize(const flsp_ic_desc& ic, const flsp_velocity_desc& velocity) {
    AdvectSimulator::initialize(ic, velocity);
    if (!ic.exact) {
      flsp_reinit_opts o = control_.reinit;
      o.mode = FLSP_REINIT_GLOBAL;
      int nit = 0;
      check(flsp_reinit(h(), &o, &nit), "flsp_reinit");
    }
  }
  // LevelSetSurface::advance_time(time_step, compute_single_step)
  double advance_time(double time_step, bool compute_single_step) {
    double adv = 0.0;
    check(flsp_ls_advance(h(), &control_, time_step, compute_single_step ? 1 : 0, &adv),
          "flsp_ls_advance");
    return adv;
  }
  double compute_mass_error(const flsp_ic_desc& analytical) const {
    double out = 0.0;
    check(flsp_reduce(h(), FLSP_RED_MASS_ERROR, &analytical, &out), "flsp_reduce");
    return out;
  }
  // CurvatureEstimator::estimate (level_set.implement.h:600-620);
  // FLSP_CURV_NEIGHBOUR gives the exterior face term to the neighbour
  std::vector<double> estimate_curvature(int mode = FLSP_CURV_REFERENCE) const {
    std::vector<double> out((size_t)n_dofs());
    check(flsp_curvature(h(), mode, out.data(), (int64_t)out.size()), "flsp_curvature");
    return out;
  }
  double integrate_mass() const {
    double out = 0.0;
    check(flsp_reduce(h(), FLSP_RED_MASS, nullptr, &out), "flsp_reduce");
    return out;
  }
  ReinitSimulatorLDG& reinit_simulator() { return reinit_; }

 private:
  ReinitSimulatorLDG reinit_;
  flsp_ls_opts control_;
};

// ---------------------------------------------------------------- helpers
inline flsp_velocity_desc rigid_body_rotation(double cx, double cy, double omega) {
  // ls::RigidBodyRotation<2>: u = w (y - cy), v = -w (x - cx)
  flsp_velocity_desc v{};
  v.n_terms = 2;
  v.terms[0].comp = 0;
  v.terms[0].coeff = omega;
  v.terms[0].f[0] = {FLSP_F_ONE, 0, 0};
  v.terms[0].f[1] = {FLSP_F_LIN, 1.0, -cy};
  v.terms[0].f[2] = {FLSP_F_ONE, 0, 0};
  v.terms[1].comp = 1;
  v.terms[1].coeff = -omega;
  v.terms[1].f[0] = {FLSP_F_LIN, 1.0, -cx};
  v.terms[1].f[1] = {FLSP_F_ONE, 0, 0};
  v.terms[1].f[2] = {FLSP_F_ONE, 0, 0};
  v.time_kind = FLSP_T_ONE;
  return v;
}

// HyperSphere(center, r) - HyperRectangle(lo, hi)  (ICDiff, geometry.h:98-112)
inline flsp_ic_desc slotted_disk(double cx, double cy, double r, double x0, double y0, double x1,
                                 double y1) {
  flsp_ic_desc ic{};
  ic.n_nodes = 3;
  ic.root = 2;
  ic.exact = 1;
  ic.nodes[0].kind = FLSP_IC_SPHERE;
  ic.nodes[0].p[0] = cx;
  ic.nodes[0].p[1] = cy;
  ic.nodes[0].p[3] = r;
  ic.nodes[1].kind = FLSP_IC_RECT;
  ic.nodes[1].p[0] = x0;
  ic.nodes[1].p[1] = y0;
  ic.nodes[1].p[3] = x1;
  ic.nodes[1].p[4] = y1;
  ic.nodes[2].kind = FLSP_IC_DIFF;
  ic.nodes[2].a = 0;
  ic.nodes[2].b = 1;
  return ic;
}

}  // namespace flsp

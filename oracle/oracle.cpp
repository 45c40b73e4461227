// oracle.cpp — CPU FP64 restatement of FELSPA's level-set hot path.
//
// TEST INFRASTRUCTURE ONLY (see oracle.h).  Parity status: UNPINNED — the
// reference cannot be built here (deal.II/Boost/TBB absent) and holds no
// golden vectors; this file restates its algorithms with file:line
// citations (paths inside the FELSPA tree) and is pinned by analytic
// known-answer tests plus committed regression fixtures.
//
// The arithmetic deliberately follows the reference's FEValues style:
// basis values at quadrature points, dof-outer / qpt-inner loops as the
// reference assemblers write them, a diagonal mass solve.  The product
// kernels use sum factorisation and modal identities instead, so the two
// computations agree only through the mathematics, not by construction.
#include "oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kEps = 2.220446049250313e-16;  // numeric_limits<double>::epsilon()

// ---------------------------------------------------------------------
// 1D Legendre polynomials orthonormal on [0,1]: L_k(x) = sqrt(2k+1) P_k(2x-1)
// (deal.II Polynomials::Legendre, the 1D factor of FE_DGP / FE_DGQLegendre).
// ---------------------------------------------------------------------
void legendre(int n, double x, double* v, double* d, double* dd) {
  double t = 2.0 * x - 1.0;
  double P[12], dP[12], ddP[12];
  P[0] = 1.0; dP[0] = 0.0; ddP[0] = 0.0;
  if (n > 1) { P[1] = t; dP[1] = 1.0; ddP[1] = 0.0; }
  for (int k = 1; k + 1 < n; ++k) {
    P[k + 1] = ((2 * k + 1) * t * P[k] - k * P[k - 1]) / (k + 1);
    dP[k + 1] = ((2 * k + 1) * (P[k] + t * dP[k]) - k * dP[k - 1]) / (k + 1);
    ddP[k + 1] = ((2 * k + 1) * (2.0 * dP[k] + t * ddP[k]) - k * ddP[k - 1]) / (k + 1);
  }
  for (int k = 0; k < n; ++k) {
    double s = std::sqrt(2.0 * k + 1.0);
    if (v) v[k] = s * P[k];
    if (d) d[k] = 2.0 * s * dP[k];
    if (dd) dd[k] = 4.0 * s * ddP[k];
  }
}

// Gauss-Legendre points on [0,1], increasing (deal.II QGauss<1>).
void gauss(int n, double* x, double* w) {
  for (int i = 0; i < n; ++i) {
    long double z = std::cos(kPi * (i + 0.75) / (n + 0.5));
    long double pp = 0;
    for (int it = 0; it < 100; ++it) {
      long double p1 = 1, p2 = 0;
      for (int j = 0; j < n; ++j) {
        long double p3 = p2; p2 = p1;
        p1 = ((2.0L * j + 1.0L) * z * p2 - j * p3) / (j + 1);
      }
      pp = n * (z * p1 - p2) / (z * z - 1.0L);
      long double z1 = z;
      z = z1 - p1 / pp;
      if (std::fabs((double)(z - z1)) < 1e-19) break;
    }
    // root z in (-1,1) decreasing in i -> map to increasing x
    x[i] = (double)(0.5L - 0.5L * z);
    w[i] = (double)(1.0L / ((1.0L - z * z) * pp * pp));
  }
}

// ---------------------------------------------------------------------
// problem description
// ---------------------------------------------------------------------
struct Quad {  // tensor Gauss rule on the reference cell, x fastest
  int n1 = 0, np = 0;
  std::vector<std::array<double, 3>> xi;
  std::vector<double> w;
};

struct FaceQuad {  // rule on one face, points in cell reference coordinates
  int np = 0;
  std::vector<std::array<double, 3>> xi;
  std::vector<double> w;
};

}  // namespace

struct orc_problem {
  int dim, p, basis, nb;
  int n[3];
  double lo[3], hi[3], h[3];
  long ncell;
  double vol, diam, min_diam;
  std::vector<std::array<int, 3>> modes;
  bool has_vel = false;
  flsp_velocity_desc vel;
  // velocity of a coupled FE simulator: nodal lattice of degree fe_pv (0: none)
  int fe_pv = 0;
  int fe_nn[3] = {1, 1, 1};
  double fe_x[4];                 // Gauss-Lobatto nodes on [0, 1]
  std::vector<double> fe_u;       // [comp][z][y][x]

  Quad qc, ql;           // QGauss(p+2), QGauss(p+1)
  FaceQuad fc[6], fl[6]; // per face: QGauss<dim-1>(p+2) / (p+1)
  // shape tables: val[i*np+q], grad[(i*np+q)*3+d] (reference derivatives)
  std::vector<double> vc, gc, vl, gl;
  std::vector<double> vfc[6], vfl[6];
  std::vector<double> gfl[6];         // reference gradients at the QGauss(p+1) face points
  std::vector<double> vvert, gvert;  // at the 2^dim vertices (QTrapezoid order)
  int nvert;

  void ijk(long c, int* I) const {
    I[0] = (int)(c % n[0]);
    long r = c / n[0];
    I[1] = dim > 1 ? (int)(r % n[1]) : 0;
    I[2] = dim > 2 ? (int)(r / n[1]) : 0;
  }
  long index(const int* I) const {
    return I[0] + (long)n[0] * (I[1] + (long)n[1] * (dim > 2 ? I[2] : 0));
  }
  // neighbour across face f = 2*axis + side; -1 at the boundary
  long neighbor(long c, int f) const {
    int I[3];
    ijk(c, I);
    int ax = f / 2, s = f % 2;
    I[ax] += s ? 1 : -1;
    if (I[ax] < 0 || I[ax] >= n[ax]) return -1;
    return index(I);
  }
  void x0(long c, double* X) const {
    int I[3];
    ijk(c, I);
    for (int d = 0; d < 3; ++d) X[d] = d < dim ? lo[d] + I[d] * h[d] : 0.0;
  }
  // boundary conditions: id of every boundary face (empty: all 0, deal.II's
  // default), the Dirichlet value of each id
  std::vector<int> bid;
  std::map<int, double> dirichlet;
  long side_faces(int ax) const {
    long s = 1;
    for (int e = 0; e < dim; ++e)
      if (e != ax) s *= n[e];
    return s;
  }
  // Dirichlet value on the boundary face f = 2*axis + side of cell c, NaN
  // if none (id 0 or no condition for its id: zero-Neumann).  Faces side by
  // side (x-, x+, y-, y+, z-, z+), each side lexicographic in the other axes.
  double bc_value(long c, int f) const {
    if (dirichlet.empty()) return std::nan("");
    int I[3];
    ijk(c, I);
    const int ax = f / 2, s = f % 2;
    long k = 0;
    for (int e = 0; e < ax; ++e) k += 2 * side_faces(e);
    k += s * side_faces(ax);
    long in_side = 0, stride = 1;
    for (int e = 0; e < dim; ++e) {
      if (e == ax) continue;
      in_side += stride * I[e];
      stride *= n[e];
    }
    const int id = bid.empty() ? 0 : bid[k + in_side];
    if (id <= 0) return std::nan("");
    auto it = dirichlet.find(id);
    return it == dirichlet.end() ? std::nan("") : it->second;
  }
};

namespace {

void shape_eval(const orc_problem* pr, const double* xi, double* val,
                double* grad, double* hess /* dim*dim, may be null */) {
  int n1 = pr->p + 1;
  double v[3][8], d[3][8], dd[3][8];
  for (int a = 0; a < pr->dim; ++a) legendre(n1, xi[a], v[a], d[a], dd[a]);
  for (int i = 0; i < pr->nb; ++i) {
    const auto& m = pr->modes[i];
    double prod = 1.0;
    for (int a = 0; a < pr->dim; ++a) prod *= v[a][m[a]];
    val[i] = prod;
    if (grad) {
      for (int g = 0; g < pr->dim; ++g) {
        double pg = 1.0;
        for (int a = 0; a < pr->dim; ++a) pg *= (a == g) ? d[a][m[a]] : v[a][m[a]];
        grad[i * 3 + g] = pg;
      }
    }
    if (hess) {
      for (int g1 = 0; g1 < pr->dim; ++g1)
        for (int g2 = 0; g2 < pr->dim; ++g2) {
          double ph = 1.0;
          for (int a = 0; a < pr->dim; ++a) {
            int o = (a == g1) + (a == g2);
            ph *= o == 0 ? v[a][m[a]] : (o == 1 ? d[a][m[a]] : dd[a][m[a]]);
          }
          hess[(i * 3 + g1) * 3 + g2] = ph;
        }
    }
  }
}

Quad make_quad(int dim, int n1) {
  Quad q;
  q.n1 = n1;
  double x[16], w[16];
  gauss(n1, x, w);
  int nz = dim > 2 ? n1 : 1, ny = dim > 1 ? n1 : 1;
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < n1; ++i) {
        q.xi.push_back({x[i], dim > 1 ? x[j] : 0.0, dim > 2 ? x[k] : 0.0});
        double ww = w[i];
        if (dim > 1) ww *= w[j];
        if (dim > 2) ww *= w[k];
        q.w.push_back(ww);
      }
  q.np = (int)q.w.size();
  return q;
}

FaceQuad make_face_quad(int dim, int n1, int f) {
  FaceQuad q;
  double x[16], w[16];
  gauss(n1, x, w);
  int ax = f / 2, s = f % 2;
  int t0 = -1, t1 = -1;
  for (int a = 0; a < dim; ++a)
    if (a != ax) { if (t0 < 0) t0 = a; else t1 = a; }
  int n0 = n1, nn1 = (dim > 2) ? n1 : 1;
  for (int j = 0; j < nn1; ++j)
    for (int i = 0; i < n0; ++i) {
      std::array<double, 3> p = {0, 0, 0};
      p[ax] = s ? 1.0 : 0.0;
      p[t0] = x[i];
      double ww = w[i];
      if (t1 >= 0) { p[t1] = x[j]; ww *= w[j]; }
      q.xi.push_back(p);
      q.w.push_back(ww);
    }
  q.np = (int)q.w.size();
  return q;
}

void table(const orc_problem* pr, const std::vector<std::array<double, 3>>& pts,
           std::vector<double>& val, std::vector<double>* grad) {
  int np = (int)pts.size(), nb = pr->nb;
  val.assign((size_t)nb * np, 0.0);
  if (grad) grad->assign((size_t)nb * np * 3, 0.0);
  std::vector<double> v(nb), g(nb * 3);
  for (int q = 0; q < np; ++q) {
    shape_eval(pr, pts[q].data(), v.data(), g.data(), nullptr);
    for (int i = 0; i < nb; ++i) {
      val[(size_t)i * np + q] = v[i];
      if (grad)
        for (int d = 0; d < 3; ++d) (*grad)[((size_t)i * np + q) * 3 + d] = g[i * 3 + d];
    }
  }
}

// ---------------------------------------------------------------------
// velocity: separable sum (reference fields: src/level_set/velocity_field.cc:38-77)
// ---------------------------------------------------------------------
double factor(const flsp_factor& f, double x) {
  switch (f.kind) {
    case FLSP_F_ONE: return 1.0;
    case FLSP_F_LIN: return f.a * x + f.b;
    case FLSP_F_SIN: return std::sin(f.a * x + f.b);
    case FLSP_F_COS: return std::cos(f.a * x + f.b);
    case FLSP_F_SINSQ: { double s = std::sin(f.a * x + f.b); return s * s; }
    case FLSP_F_SINPI: return std::sin(kPi * (f.a * x + f.b));
    case FLSP_F_COSPI: return std::cos(kPi * (f.a * x + f.b));
    case FLSP_F_SINPISQ: { double s = std::sin(kPi * (f.a * x + f.b)); return s * s; }
  }
  return 0.0;
}

double time_factor(const flsp_velocity_desc& v, double t) {
  switch (v.time_kind) {
    case FLSP_T_ONE: return 1.0;
    case FLSP_T_COS: return std::cos(v.ta * t + v.tb);
    case FLSP_T_COSPI: return std::cos(kPi * (v.ta * t + v.tb));
    case FLSP_T_ONE_MINUS_EXP: return 1.0 - std::exp(-v.ta * t);
  }
  return 1.0;
}

// Lagrange basis a of the nodes x[0..pv] at t (1 / 0 at the nodes exactly)
double fe_basis(int pv, const double* x, int a, double t) {
  double num = 1.0, den = 1.0;
  for (int b = 0; b <= pv; ++b)
    if (b != a) {
      num *= t - x[b];
      den *= x[a] - x[b];
    }
  return num / den;
}

// The simulator branch of the advection assembler (advection.implement.h:
// 891-905, stokes_common.implement.h:583-591): the coupled FE field of cell
// c at reference point xi, sum over the cell's nodes (x fastest) of the
// node value times the basis products
void fe_velocity(const orc_problem* pr, long c, const double* xi, double* u) {
  int I[3];
  pr->ijk(c, I);
  const int pv = pr->fe_pv;
  const size_t nn = (size_t)pr->fe_nn[0] * pr->fe_nn[1] * pr->fe_nn[2];
  for (int d = 0; d < 3; ++d) u[d] = 0.0;
  for (int cz = 0; cz <= (pr->dim > 2 ? pv : 0); ++cz)
    for (int cy = 0; cy <= pv; ++cy) {
      double byz = fe_basis(pv, pr->fe_x, cy, xi[1]);
      if (pr->dim > 2) byz *= fe_basis(pv, pr->fe_x, cz, xi[2]);
      for (int cx = 0; cx <= pv; ++cx) {
        const double b = fe_basis(pv, pr->fe_x, cx, xi[0]) * byz;
        const size_t node = ((size_t)(pr->dim > 2 ? pv * I[2] + cz : 0) * pr->fe_nn[1] + pv * I[1] + cy) *
                                pr->fe_nn[0] + pv * I[0] + cx;
        for (int d = 0; d < pr->dim; ++d) u[d] += pr->fe_u[d * nn + node] * b;
      }
    }
}

void velocity(const orc_problem* pr, const double* x, double t, double* u) {
  double ct = time_factor(pr->vel, t);
  for (int d = 0; d < 3; ++d) u[d] = 0.0;
  for (int k = 0; k < pr->vel.n_terms; ++k) {
    const flsp_vel_term& tm = pr->vel.terms[k];
    double v = tm.coeff;
    for (int a = 0; a < pr->dim; ++a) v *= factor(tm.f[a], x[a]);
    u[tm.comp] += v;
  }
  for (int d = 0; d < pr->dim; ++d) u[d] *= ct;
}

// ---------------------------------------------------------------------
// initial conditions (src/level_set/geometry.cc:17-235, geometry.h:80-160)
// ---------------------------------------------------------------------
double rect_sdf(int dim, const double* lo, const double* hi, const double* x) {
  // outside: distance to the nearest face/edge/corner; inside: max of
  // the signed face distances (HyperRectangle<2/3>::evaluate)
  double out2 = 0.0;
  bool inside = true;
  for (int d = 0; d < dim; ++d) {
    double e = 0.0;
    if (x[d] < lo[d]) { e = x[d] - lo[d]; inside = false; }
    else if (x[d] > hi[d]) { e = x[d] - hi[d]; inside = false; }
    out2 += e * e;
  }
  if (!inside) return std::sqrt(out2);
  double m = -1e300;
  for (int d = 0; d < dim; ++d) {
    m = std::max(m, lo[d] - x[d]);
    m = std::max(m, x[d] - hi[d]);
  }
  return m;
}

double ic_node(const flsp_ic_desc* ic, int dim, int k, const double* x) {
  const flsp_ic_node& nd = ic->nodes[k];
  switch (nd.kind) {
    case FLSP_IC_SPHERE: {
      double s = 0.0;
      for (int d = 0; d < dim; ++d) { double e = x[d] - nd.p[d]; s += e * e; }
      return std::sqrt(s) - nd.p[3];
    }
    case FLSP_IC_RECT: {
      double lo[3] = {nd.p[0], nd.p[1], nd.p[2]}, hi[3] = {nd.p[3], nd.p[4], nd.p[5]};
      return rect_sdf(dim, lo, hi, x);
    }
    case FLSP_IC_HEIGHT: {
      int ax = (int)nd.p[0];
      int u = -1, v = -1;
      for (int a = 0; a < dim; ++a)
        if (a != ax) { if (u < 0) u = a; else v = a; }
      double hgt = nd.p[1];
      for (int m = 0; m < ic->n_waves; ++m) {
        double arg = ic->waves[m][1] * x[u];
        if (v >= 0) arg += ic->waves[m][2] * x[v];
        hgt += ic->waves[m][0] * std::cos(2.0 * kPi * arg + ic->waves[m][3]);
      }
      return x[ax] - hgt;
    }
    case FLSP_IC_UNION:
      return std::min(ic_node(ic, dim, nd.a, x), ic_node(ic, dim, nd.b, x));
    case FLSP_IC_DIFF:
      return std::max(ic_node(ic, dim, nd.a, x), -ic_node(ic, dim, nd.b, x));
    case FLSP_IC_INTERSECT:
      return std::max(ic_node(ic, dim, nd.a, x), ic_node(ic, dim, nd.b, x));
  }
  return 0.0;
}

// deal.II Vector of a cell: phi + c*nb
inline double eval_at(const double* pc, const std::vector<double>& tab, int nb,
                      int np, int q) {
  double s = 0.0;
  for (int j = 0; j < nb; ++j) s += pc[j] * tab[(size_t)j * np + q];
  return s;
}

// smooth sign, reinit.cc:121-133 (USE_TANH_SMOOTHING off)
inline double smooth_signum(double phi0, double gnorm, double cd) {
  return phi0 / std::sqrt(phi0 * phi0 + cd * cd * gnorm * gnorm);
}

// Lax-Friedrichs HJ flux, reinit.cc:136-191 (USE_LF_FLUX on)
inline double lf_flux(int dim, double S, const double* l, const double* r) {
  double avg2 = 0.0;
  double avg[3];
  for (int d = 0; d < dim; ++d) avg[d] = 0.5 * (l[d] + r[d]);
  for (int d = 0; d < dim; ++d) avg2 += avg[d] * avg[d];
  double hj = S * (std::sqrt(avg2) - 1.0);
  for (int d = 0; d < dim; ++d) hj += 0.5 * std::fabs(S) * (l[d] - r[d]);
  return hj;
}

// characteristic velocity, reinit.cc:235-264 -> returns its norm
inline double char_speed(int dim, double S, const double* l, const double* r) {
  double g[3];
  for (int d = 0; d < dim; ++d) {
    if (S >= 0) {
      double lp = std::max(l[d], 0.0), rm = -std::min(r[d], 0.0);
      g[d] = std::fabs(lp) > std::fabs(rm) ? lp : rm;
    } else {
      double lm = -std::min(l[d], 0.0), rp = std::max(r[d], 0.0);
      g[d] = std::fabs(lm) > std::fabs(rp) ? lm : rp;
    }
  }
  double n2 = 0.0;
  for (int d = 0; d < dim; ++d) n2 += g[d] * g[d];
  double nrm = std::sqrt(n2);
  if (!(std::fabs(nrm) <= kEps)) {
    double inv = 1.0 / nrm;
    for (int d = 0; d < dim; ++d) g[d] *= inv;
    for (int d = 0; d < dim; ++d) g[d] *= S;
  }
  double s2 = 0.0;
  for (int d = 0; d < dim; ++d) s2 += g[d] * g[d];
  return std::sqrt(s2);
}

// advection CFL scaling, advection.cc:487-496
inline double adv_cfl_scaling(int p) {
  double pp = p;
  double c = 4.0 / (2.0 + pp) / (2.0 + pp) + 1.0;
  c *= (2.0 * pp + 1.0);
  return c;
}

inline bool is_zero(double x) { return std::fabs(x) <= kEps; }

}  // namespace

// =====================================================================
extern "C" {

void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

void orc_gauss(int n, double* x, double* w) { gauss(n, x, w); }
void orc_legendre(int n, double x, double* v, double* d, double* dd) {
  legendre(n, x, v, d, dd);
}

int orc_set_dirichlet(orc_problem* pr, int boundary_id, double value) {
  if (!pr || boundary_id <= 0 || !std::isfinite(value)) return FLSP_ERR_BAD_ARG;
  pr->dirichlet[boundary_id] = value;
  return FLSP_OK;
}

void orc_clear_dirichlet(orc_problem* pr) {
  if (pr) pr->dirichlet.clear();
}

int orc_create(const flsp_mesh_desc* mesh, int degree, int basis,
               orc_problem** out) {
  if (!mesh || !out || mesh->dim < 2 || mesh->dim > 3 || degree < 0 || degree > 4)
    return FLSP_ERR_BAD_ARG;
  orc_problem* pr = new orc_problem();
  pr->dim = mesh->dim;
  pr->p = degree;
  pr->basis = basis;
  pr->ncell = 1;
  double d2 = 0.0;
  pr->vol = 1.0;
  for (int d = 0; d < 3; ++d) {
    pr->n[d] = d < pr->dim ? mesh->n[d] : 1;
    pr->lo[d] = d < pr->dim ? mesh->lo[d] : 0.0;
    pr->hi[d] = d < pr->dim ? mesh->hi[d] : 1.0;
    if (d < pr->dim) {
      if (pr->n[d] < 1) { delete pr; return FLSP_ERR_BAD_MESH; }
      pr->h[d] = (pr->hi[d] - pr->lo[d]) / pr->n[d];
      pr->ncell *= pr->n[d];
      d2 += pr->h[d] * pr->h[d];
      pr->vol *= pr->h[d];
    } else {
      pr->h[d] = 1.0;
    }
  }
  if (mesh->boundary_ids) {
    long nbf = 0;
    for (int e = 0; e < pr->dim; ++e) nbf += 2 * pr->side_faces(e);
    pr->bid.assign(mesh->boundary_ids, mesh->boundary_ids + nbf);
  }
  // cell diameter = longest diagonal (mesh/src/mesh.implement.h:60-71)
  pr->diam = std::sqrt(d2);
  pr->min_diam = pr->diam;
  // DoF order of FE_DGQLegendre / FE_DGP (PolynomialSpace) inside a cell
  int p = degree;
  int cz = pr->dim > 2 ? p : 0;
  for (int c = 0; c <= cz; ++c)
    for (int b = 0; b <= p; ++b)
      for (int a = 0; a <= p; ++a) {
        if (basis == FLSP_BASIS_P && a + b + c > p) continue;
        pr->modes.push_back({a, b, c});
      }
  if (basis == FLSP_BASIS_P) {
    // PolynomialSpace ordering: c outer, b middle (b <= p - c), a inner
    pr->modes.clear();
    for (int c = 0; c <= cz; ++c)
      for (int b = 0; b <= p - c; ++b)
        for (int a = 0; a <= p - b - c; ++a) pr->modes.push_back({a, b, c});
  }
  pr->nb = (int)pr->modes.size();
  pr->qc = make_quad(pr->dim, p + 2);
  pr->ql = make_quad(pr->dim, p + 1);
  table(pr, pr->qc.xi, pr->vc, &pr->gc);
  table(pr, pr->ql.xi, pr->vl, &pr->gl);
  for (int f = 0; f < 2 * pr->dim; ++f) {
    pr->fc[f] = make_face_quad(pr->dim, p + 2, f);
    pr->fl[f] = make_face_quad(pr->dim, p + 1, f);
    table(pr, pr->fc[f].xi, pr->vfc[f], nullptr);
    table(pr, pr->fl[f].xi, pr->vfl[f], &pr->gfl[f]);
  }
  std::vector<std::array<double, 3>> verts;
  pr->nvert = 1 << pr->dim;
  for (int v = 0; v < pr->nvert; ++v)
    verts.push_back({(double)(v & 1), (double)((v >> 1) & 1), (double)((v >> 2) & 1)});
  table(pr, verts, pr->vvert, &pr->gvert);
  std::memset(&pr->vel, 0, sizeof(pr->vel));
  *out = pr;
  return FLSP_OK;
}

void orc_destroy(orc_problem* pr) { delete pr; }
long orc_n_dofs(const orc_problem* pr) { return pr->ncell * pr->nb; }
int orc_dofs_per_cell(const orc_problem* pr) { return pr->nb; }

void orc_shape(const orc_problem* pr, int npts, const double* xi, double* val,
               double* grad) {
  std::vector<double> v(pr->nb), g(pr->nb * 3);
  for (int q = 0; q < npts; ++q) {
    shape_eval(pr, xi + 3 * q, v.data(), g.data(), nullptr);
    for (int i = 0; i < pr->nb; ++i) {
      val[(size_t)i * npts + q] = v[i];
      if (grad)
        for (int d = 0; d < pr->dim; ++d)
          grad[((size_t)i * npts + q) * pr->dim + d] = g[i * 3 + d];
    }
  }
}

int orc_set_velocity(orc_problem* pr, const flsp_velocity_desc* v) {
  if (!v || v->n_terms < 0 || v->n_terms > FLSP_MAX_VEL_TERMS) return FLSP_ERR_BAD_ARG;
  for (int k = 0; k < v->n_terms; ++k)
    if (v->terms[k].comp < 0 || v->terms[k].comp >= pr->dim) return FLSP_ERR_BAD_ARG;
  pr->vel = *v;
  pr->fe_pv = 0;
  pr->fe_u.clear();
  pr->has_vel = true;
  return FLSP_OK;
}

int orc_set_velocity_fe(orc_problem* pr, int degree, const double* values, long n) {
  if (!values || degree < 1 || degree > 3) return FLSP_ERR_BAD_ARG;
  long nn = 1;
  for (int d = 0; d < 3; ++d) pr->fe_nn[d] = d < pr->dim ? degree * pr->n[d] + 1 : 1;
  for (int d = 0; d < pr->dim; ++d) nn *= pr->fe_nn[d];
  if (n != pr->dim * nn) return FLSP_ERR_BAD_ARG;
  pr->fe_pv = degree;
  // Gauss-Lobatto points of degree 1..3 on [0, 1]
  pr->fe_x[0] = 0.0;
  pr->fe_x[degree] = 1.0;
  if (degree == 2) pr->fe_x[1] = 0.5;
  if (degree == 3) {
    pr->fe_x[1] = 0.5 - 0.5 / std::sqrt(5.0);
    pr->fe_x[2] = 0.5 + 0.5 / std::sqrt(5.0);
  }
  pr->fe_u.assign(values, values + n);
  std::memset(&pr->vel, 0, sizeof(pr->vel));   // constant in time
  pr->has_vel = true;
  return FLSP_OK;
}

void orc_eval_velocity(const orc_problem* pr, const double* x, double t, double* u) {
  velocity(pr, x, t, u);
}

double orc_eval_ic(const flsp_ic_desc* ic, int dim, const double* x) {
  return ic_node(ic, dim, ic->root, x);
}

// L2 projection with QGauss(p+2) (advection.cc:145-161 -> VectorTools::project;
// the DG mass matrix is |K| I for the orthonormal basis)
int orc_project_ic(orc_problem* pr, const flsp_ic_desc* ic, double* phi) {
  if (!ic || ic->n_nodes < 1 || ic->root < 0 || ic->root >= ic->n_nodes) return FLSP_ERR_BAD_ARG;
  const int nb = pr->nb, np = pr->qc.np;
#pragma omp parallel for schedule(static)
  for (long c = 0; c < pr->ncell; ++c) {
    double X0[3];
    pr->x0(c, X0);
    double rhs[128] = {0};
    for (int q = 0; q < np; ++q) {
      double x[3];
      for (int d = 0; d < 3; ++d) x[d] = X0[d] + pr->h[d] * pr->qc.xi[q][d];
      double f = ic_node(ic, pr->dim, ic->root, x);
      double jxw = pr->qc.w[q] * pr->vol;
      for (int i = 0; i < nb; ++i) rhs[i] += f * pr->vc[(size_t)i * np + q] * jxw;
    }
    for (int i = 0; i < nb; ++i) phi[c * nb + i] = rhs[i] / pr->vol;
  }
  return FLSP_OK;
}

// ---------------------------------------------------------------------
// advection RHS: AdvectAssembler<workstream> cell/face/boundary assembly
// (include/felspa/pde/src/advection.implement.h:617-744) + mass solve
// (linear_systems.implement.h:30-47).  Each cell integrates all of its
// faces itself; the reference integrates an interior face once from the
// lower-id side (:568) and scatters the same two contributions.
// ---------------------------------------------------------------------
int orc_advect_rhs(orc_problem* pr, const double* phi, double t, double* phidot) {
  if (!pr->has_vel) return FLSP_ERR_BAD_ARG;
  const int nb = pr->nb, np = pr->qc.np, dim = pr->dim;
#pragma omp parallel for schedule(static)
  for (long c = 0; c < pr->ncell; ++c) {
    double X0[3];
    pr->x0(c, X0);
    const double* pc = phi + c * nb;
    double R[128] = {0};
    // cell term (:617-643), dof-outer / qpt-inner
    double sq[256], uq[256][3];
    for (int q = 0; q < np; ++q) {
      sq[q] = eval_at(pc, pr->vc, nb, np, q);
      double x[3];
      for (int d = 0; d < 3; ++d) x[d] = X0[d] + pr->h[d] * pr->qc.xi[q][d];
      if (pr->fe_pv) fe_velocity(pr, c, pr->qc.xi[q].data(), uq[q]);
      else velocity(pr, x, t, uq[q]);
    }
    for (int i = 0; i < nb; ++i)
      for (int q = 0; q < np; ++q) {
        double ug = 0.0;
        for (int d = 0; d < dim; ++d)
          ug += uq[q][d] * (pr->gc[((size_t)i * np + q) * 3 + d] / pr->h[d]);
        R[i] += ug * sq[q] * (pr->qc.w[q] * pr->vol);
      }
    // faces (:646-744)
    for (int f = 0; f < 2 * dim; ++f) {
      int ax = f / 2, s = f % 2;
      long nbc = pr->neighbor(c, f);
      const double gbc = nbc < 0 ? pr->bc_value(c, f) : std::nan("");
      const FaceQuad& fq = pr->fc[f];
      const std::vector<double>& vin = pr->vfc[f];
      const std::vector<double>& vex = pr->vfc[f ^ 1];
      double area = pr->vol / pr->h[ax];
      for (int q = 0; q < fq.np; ++q) {
        double pin = eval_at(pc, vin, nb, fq.np, q);
        // boundary: the face's Dirichlet value, or without one zero-Neumann
        // (interior trace) (:719-741)
        double pex = nbc >= 0 ? eval_at(phi + nbc * nb, vex, nb, fq.np, q) : (std::isnan(gbc) ? pin : gbc);
        double x[3], u[3];
        for (int d = 0; d < 3; ++d) x[d] = X0[d] + pr->h[d] * fq.xi[q][d];
        // FE field: continuous, so the face value is the same from either cell
        if (pr->fe_pv) fe_velocity(pr, c, fq.xi[q].data(), u);
        else velocity(pr, x, t, u);
        double vn = s ? u[ax] : -u[ax];
        double up = vn > 0.0 ? pin : pex;
        double jxw = fq.w[q] * area;
        for (int i = 0; i < nb; ++i) R[i] -= vn * vin[(size_t)i * fq.np + q] * up * jxw;
      }
    }
    for (int i = 0; i < nb; ++i) phidot[c * nb + i] = R[i] / pr->vol;
  }
  return FLSP_OK;
}

// CFLEstimator::do_estimate/local_estimate (pde_tools.implement.h:18-67):
// max over cells of (max vertex |u|) / diameter
double orc_advect_cfl(orc_problem* pr, double t) {
  double vd = 0.0;
#pragma omp parallel for reduction(max : vd) schedule(static)
  for (long c = 0; c < pr->ncell; ++c) {
    double X0[3];
    pr->x0(c, X0);
    double m = 0.0;
    for (int v = 0; v < pr->nvert; ++v) {
      double x[3] = {X0[0], X0[1], X0[2]}, u[3];
      for (int d = 0; d < pr->dim; ++d) if ((v >> d) & 1) x[d] += pr->h[d];
      const double xi[3] = {(double)(v & 1), (double)((v >> 1) & 1), (double)((v >> 2) & 1)};
      if (pr->fe_pv) fe_velocity(pr, c, xi, u);
      else velocity(pr, x, t, u);
      double s = 0.0;
      for (int d = 0; d < pr->dim; ++d) s += u[d] * u[d];
      m = std::max(m, std::sqrt(s));
    }
    vd = std::max(vd, m / pr->diam);
  }
  return vd;
}

// RungeKuttaTVD<k>::integrate_explicit (time_integration.implement.h:141-234)
static void rk_step(orc_problem* pr, double* phi, int order, double t, double dt) {
  long N = orc_n_dofs(pr);
  std::vector<double> s(phi, phi + N), L(N);
  if (order == 1) {
    orc_advect_rhs(pr, phi, t, L.data());
    for (long i = 0; i < N; ++i) { L[i] *= dt; L[i] += phi[i]; }
    std::copy(L.begin(), L.end(), phi);
    return;
  }
  orc_advect_rhs(pr, s.data(), t, L.data());
  for (long i = 0; i < N; ++i) s[i] += dt * L[i];
  if (order == 2) {
    orc_advect_rhs(pr, s.data(), t + dt, L.data());
    for (long i = 0; i < N; ++i) s[i] += dt * L[i];
    for (long i = 0; i < N; ++i) { s[i] += phi[i]; s[i] *= 0.5; }
    std::copy(s.begin(), s.end(), phi);
    return;
  }
  orc_advect_rhs(pr, s.data(), t + dt, L.data());
  for (long i = 0; i < N; ++i) s[i] += dt * L[i];
  for (long i = 0; i < N; ++i) { s[i] += 3.0 * phi[i]; s[i] *= 0.25; }
  orc_advect_rhs(pr, s.data(), t + 0.5 * dt, L.data());
  for (long i = 0; i < N; ++i) s[i] += dt * L[i];
  const double third = 1.0 / 3.0;
  for (long i = 0; i < N; ++i) { s[i] *= 2.0; s[i] += phi[i]; s[i] *= third; }
  std::copy(s.begin(), s.end(), phi);
}

// AdvectSimulator::advance_time(time_step, single) (advection.cc:359-426)
int orc_advance(orc_problem* pr, double* phi, orc_clock* clk, int rk_order,
                double cfl_max, double time_step, int single_cycle,
                double* advanced) {
  if (!pr->has_vel) return FLSP_ERR_BAD_ARG;
  double cum = 0.0;
  do {
    double vd = orc_advect_cfl(pr, clk->t);
    clk->vd_run = std::max(clk->vd_run, vd);
    double suggest = cfl_max / (clk->vd_run * adv_cfl_scaling(pr->p));
    double sub = std::min(suggest, time_step - cum);
    if (!is_zero(sub)) {  // TempoIntegrator::advance_time_step (:14-41)
      rk_step(pr, phi, rk_order, clk->t, sub);
      clk->t += sub;
      clk->n_substeps++;
    }
    cum += sub;
    if (single_cycle) break;
  } while (!is_zero(cum - time_step));
  if (advanced) *advanced = cum;
  return FLSP_OK;
}

// ---------------------------------------------------------------------
// LDG left/right gradients (hamilton_jacobi.cc:462-511; ldg.cc:355-376 cell,
// :510-621 left, :628-740 right); QGauss(p+1) (system_assembler.implement.h:100-113)
// gl/gr: dim blocks of n_dofs
// ---------------------------------------------------------------------
int orc_hj_gradients(orc_problem* pr, const double* phi, double* gl, double* gr) {
  const int nb = pr->nb, np = pr->ql.np, dim = pr->dim;
  const long N = orc_n_dofs(pr);
#pragma omp parallel for schedule(static)
  for (long c = 0; c < pr->ncell; ++c) {
    const double* pc = phi + c * nb;
    double sq[256];
    for (int q = 0; q < np; ++q) sq[q] = eval_at(pc, pr->vl, nb, np, q);
    for (int e = 0; e < dim; ++e) {
      double RL[128] = {0}, RR[128] = {0};
      for (int q = 0; q < np; ++q)
        for (int i = 0; i < nb; ++i) {
          double v = (pr->gl[((size_t)i * np + q) * 3 + e] / pr->h[e]) * sq[q] *
                     (pr->ql.w[q] * pr->vol);
          RL[i] -= v;
          RR[i] -= v;
        }
      double area = pr->vol / pr->h[e];
      for (int s = 0; s < 2; ++s) {
        int f = 2 * e + s;
        long nbc = pr->neighbor(c, f);
        const double gbc = nbc < 0 ? pr->bc_value(c, f) : std::nan("");
        const FaceQuad& fq = pr->fl[f];
        const std::vector<double>& vin = pr->vfl[f];
        const std::vector<double>& vex = pr->vfl[f ^ 1];
        double nrm = s ? 1.0 : -1.0;
        for (int q = 0; q < fq.np; ++q) {
          double pin = eval_at(pc, vin, nb, fq.np, q);
          double pex = nbc >= 0 ? eval_at(phi + nbc * nb, vex, nb, fq.np, q) : (std::isnan(gbc) ? pin : gbc);
          double jxw = fq.w[q] * area;
          // left flux: trace of the lower cell; right: of the upper cell;
          // boundary: the face's Dirichlet value on the side the flux takes
          // (left: lower faces, n_d < 0, ldg.cc:574-601; right: upper faces,
          // n_d >= 0, :711-735), else the interior trace
          double hl = (nrm < 0.0) ? pex : pin;
          double hr = (nrm < 0.0) ? pin : pex;
          for (int i = 0; i < nb; ++i) {
            double psi = vin[(size_t)i * fq.np + q];
            RL[i] += nrm * psi * hl * jxw;
            RR[i] += nrm * psi * hr * jxw;
          }
        }
      }
      for (int i = 0; i < nb; ++i) {
        gl[e * N + c * nb + i] = RL[i] / pr->vol;
        gr[e * N + c * nb + i] = RR[i] / pr->vol;
      }
    }
  }
  return FLSP_OK;
}

// LDGDiffusionTerm::compute_diffusion_term (ldg.cc:249-298) alternating
// gradient (:383-504) then diffusion RHS (:750-838); beta = (1..1)/sqrt(dim)
static void ldg_diffusion(orc_problem* pr, const double* phi, double nu, double* R_all) {
  const int nb = pr->nb, np = pr->ql.np, dim = pr->dim;
  const long N = orc_n_dofs(pr);
  const double beta = 1.0 / std::sqrt((double)dim);
  std::vector<double> q(dim * N);
#pragma omp parallel for schedule(static)
  for (long c = 0; c < pr->ncell; ++c) {
    const double* pc = phi + c * nb;
    double Rq[3][128] = {{0}};
    for (int iq = 0; iq < np; ++iq) {
      double s = eval_at(pc, pr->vl, nb, np, iq);
      for (int i = 0; i < nb; ++i)
        for (int d = 0; d < dim; ++d)
          Rq[d][i] -= (pr->gl[((size_t)i * np + iq) * 3 + d] / pr->h[d]) * s *
                      (pr->ql.w[iq] * pr->vol);
    }
    for (int f = 0; f < 2 * dim; ++f) {
      int e = f / 2, sd = f % 2;
      long nbc = pr->neighbor(c, f);
      const FaceQuad& fq = pr->fl[f];
      const std::vector<double>& vin = pr->vfl[f];
      const std::vector<double>& vex = pr->vfl[f ^ 1];
      double nrm = sd ? 1.0 : -1.0, area = pr->vol / pr->h[e];
      for (int iq = 0; iq < fq.np; ++iq) {
        double pin = eval_at(pc, vin, nb, fq.np, iq);
        double jxw = fq.w[iq] * area;
        double flux;
        if (nbc >= 0) {
          double pex = eval_at(phi + nbc * nb, vex, nb, fq.np, iq);
          double central = 0.5 * (pin + pex);
          double bflux = (beta * nrm) * (pex - pin);
          flux = central + bflux;
        } else {
          flux = pin;
        }
        for (int i = 0; i < nb; ++i) Rq[e][i] += vin[(size_t)i * fq.np + iq] * nrm * flux * jxw;
      }
    }
    for (int d = 0; d < dim; ++d)
      for (int i = 0; i < nb; ++i) q[d * N + c * nb + i] = Rq[d][i] / pr->vol;
  }
#pragma omp parallel for schedule(static)
  for (long c = 0; c < pr->ncell; ++c) {
    double R[128] = {0};
    for (int iq = 0; iq < np; ++iq) {
      double g[3];
      for (int d = 0; d < dim; ++d) g[d] = eval_at(q.data() + d * N + c * nb, pr->vl, nb, np, iq);
      for (int i = 0; i < nb; ++i) {
        double dot = 0.0;
        for (int d = 0; d < dim; ++d) dot += (pr->gl[((size_t)i * np + iq) * 3 + d] / pr->h[d]) * g[d];
        R[i] -= nu * dot * (pr->ql.w[iq] * pr->vol);
      }
    }
    for (int f = 0; f < 2 * dim; ++f) {
      int e = f / 2, sd = f % 2;
      long nbc = pr->neighbor(c, f);
      if (nbc < 0) continue;  // no boundary term (ldg.cc:843-850)
      const FaceQuad& fq = pr->fl[f];
      const std::vector<double>& vin = pr->vfl[f];
      const std::vector<double>& vex = pr->vfl[f ^ 1];
      double nrm = sd ? 1.0 : -1.0, area = pr->vol / pr->h[e];
      for (int iq = 0; iq < fq.np; ++iq) {
        double qin = eval_at(q.data() + e * N + c * nb, vin, nb, fq.np, iq);
        double qex = eval_at(q.data() + e * N + nbc * nb, vex, nb, fq.np, iq);
        double central = 0.5 * (qin + qex);
        double bflux = (nrm * beta) * (qex - qin);
        double flux = (central - bflux) * nrm;
        double jxw = fq.w[iq] * area;
        for (int i = 0; i < nb; ++i) R[i] += nu * vin[(size_t)i * fq.np + iq] * flux * jxw;
      }
    }
    for (int i = 0; i < nb; ++i) R_all[c * nb + i] += R[i];
  }
}

// HJ RHS: HJAssemblerWorkStream::local_assembly (hamilton_jacobi.cc:730-745)
// with ReinitOperator::cell_values (reinit.cc:267-301), QGauss(p+2); then the
// diffusion term and the mass solve (hamilton_jacobi.cc:514-551)
int orc_hj_rhs(orc_problem* pr, const double* phi, const double* phi0,
               double viscosity, double* phidot) {
  const int nb = pr->nb, np = pr->qc.np, dim = pr->dim;
  const long N = orc_n_dofs(pr);
  std::vector<double> gl(dim * N), gr(dim * N), R(N, 0.0);
  orc_hj_gradients(pr, phi, gl.data(), gr.data());
  const double cd = pr->min_diam;
#pragma omp parallel for schedule(static)
  for (long c = 0; c < pr->ncell; ++c) {
    const double* p0 = phi0 + c * nb;
    double Rc[128] = {0};
    for (int q = 0; q < np; ++q) {
      double v0 = eval_at(p0, pr->vc, nb, np, q);
      double g2 = 0.0;
      for (int d = 0; d < dim; ++d) {
        double g = 0.0;
        for (int j = 0; j < nb; ++j) g += p0[j] * (pr->gc[((size_t)j * np + q) * 3 + d] / pr->h[d]);
        g2 += g * g;
      }
      double S = smooth_signum(v0, std::sqrt(g2), cd);
      double l[3], r[3];
      for (int d = 0; d < dim; ++d) {
        l[d] = eval_at(gl.data() + d * N + c * nb, pr->vc, nb, np, q);
        r[d] = eval_at(gr.data() + d * N + c * nb, pr->vc, nb, np, q);
      }
      double H = lf_flux(dim, S, l, r);
      double jxw = pr->qc.w[q] * pr->vol;
      for (int i = 0; i < nb; ++i) Rc[i] -= pr->vc[(size_t)i * np + q] * H * jxw;
    }
    for (int i = 0; i < nb; ++i) R[c * nb + i] = Rc[i];
  }
  if (viscosity != 0.0) ldg_diffusion(pr, phi, viscosity, R.data());
  for (long i = 0; i < N; ++i) phidot[i] = R[i] / pr->vol;
  return FLSP_OK;
}

// HJSimulator::max_velocity_over_diameter before scaling (hamilton_jacobi.cc:431-447;
// CFLEstimator over ReinitOperator::cell_velocities, reinit.cc:304-328)
double orc_hj_cfl(orc_problem* pr, const double* phi_grad_src, const double* phi0) {
  const int nb = pr->nb, dim = pr->dim, nv = pr->nvert;
  const long N = orc_n_dofs(pr);
  std::vector<double> gl(dim * N), gr(dim * N);
  orc_hj_gradients(pr, phi_grad_src, gl.data(), gr.data());
  const double cd = pr->min_diam;
  double vd = 0.0;
#pragma omp parallel for reduction(max : vd) schedule(static)
  for (long c = 0; c < pr->ncell; ++c) {
    const double* p0 = phi0 + c * nb;
    double m = 0.0;
    for (int v = 0; v < nv; ++v) {
      double v0 = eval_at(p0, pr->vvert, nb, nv, v);
      double g2 = 0.0;
      for (int d = 0; d < dim; ++d) {
        double g = 0.0;
        for (int j = 0; j < nb; ++j) g += p0[j] * (pr->gvert[((size_t)j * nv + v) * 3 + d] / pr->h[d]);
        g2 += g * g;
      }
      double S = smooth_signum(v0, std::sqrt(g2), cd);
      double l[3], r[3];
      for (int d = 0; d < dim; ++d) {
        l[d] = eval_at(gl.data() + d * N + c * nb, pr->vvert, nb, nv, v);
        r[d] = eval_at(gr.data() + d * N + c * nb, pr->vvert, nb, nv, v);
      }
      m = std::max(m, char_speed(dim, S, l, r));
    }
    vd = std::max(vd, m / pr->diam);
  }
  return vd;
}

// ---------------------------------------------------------------------
// 2D minmod troubled-cell detector (pde_tools.implement.h:277-376) and
// WENO limiter (:441-734), beta = 1 + dim, gamma_nb = 0.001, eps = 1e-6,
// smoothness derivatives up to min(2, p).  QGauss(p+2).
// ---------------------------------------------------------------------
static double cell_avg(const orc_problem* pr, const double* pc) {
  double s = 0.0;
  for (int q = 0; q < pr->qc.np; ++q)
    s += eval_at(pc, pr->vc, pr->nb, pr->qc.np, q) * (pr->qc.w[q] * pr->vol);
  return s / pr->vol;
}

int orc_minmod_flags(orc_problem* pr, const double* phi, int* flags) {
  if (pr->dim != 2) return FLSP_ERR_UNSUPPORTED;
  const int nb = pr->nb;
  static const int faces_around_vertex[4][2] = {{0, 2}, {2, 1}, {0, 3}, {1, 3}};
  const double beta = 1.0 + pr->dim;
#pragma omp parallel for schedule(static)
  for (long c = 0; c < pr->ncell; ++c) {
    const double* pc = phi + c * nb;
    double avg = cell_avg(pr, pc);
    double X0[3];
    pr->x0(c, X0);
    double cc[2] = {X0[0] + 0.5 * pr->h[0], X0[1] + 0.5 * pr->h[1]};
    int flag = 0;
    for (int v = 0; v < 4 && !flag; ++v) {
      bool skip = false;
      for (int k = 0; k < 2; ++k)
        if (pr->neighbor(c, faces_around_vertex[v][k]) < 0) skip = true;
      if (skip) continue;
      double vx[2] = {X0[0] + ((v & 1) ? pr->h[0] : 0.0), X0[1] + ((v & 2) ? pr->h[1] : 0.0)};
      double cv[2] = {vx[0] - cc[0], vx[1] - cc[1]};
      double interp = 0.0;
      for (int k = 0; k < 2; ++k) {
        long nbc = pr->neighbor(c, faces_around_vertex[v][k]);
        double N0[3];
        pr->x0(nbc, N0);
        double cn[2] = {N0[0] + 0.5 * pr->h[0] - cc[0], N0[1] + 0.5 * pr->h[1] - cc[1]};
        double coeff = (cn[0] * cv[0] + cn[1] * cv[1]) / (cn[0] * cn[0] + cn[1] * cn[1]);
        double navg = cell_avg(pr, phi + nbc * nb);
        interp += (navg - avg) * coeff;
      }
      double vval = eval_at(pc, pr->vvert, nb, pr->nvert, v);
      double a = vval - avg;
      double b = beta * interp;
      // minmod(a, b) (pde_tools.h:370-389) with util::sign
      int sa = (a > 0) - (a < 0), sb = (b > 0) - (b < 0);
      double mm = (sa == sb) ? (double)sa * std::min(std::fabs(a), std::fabs(b)) : 0.0;
      if (a != mm) flag = 1;
    }
    flags[c] = flag;
  }
  return FLSP_OK;
}

int orc_weno(orc_problem* pr, double* phi, int* n_troubled) {
  if (pr->dim != 2) return FLSP_ERR_UNSUPPORTED;
  const int nb = pr->nb, np = pr->qc.np, dim = 2;
  const long N = orc_n_dofs(pr);
  std::vector<int> flags(pr->ncell);
  orc_minmod_flags(pr, phi, flags.data());
  std::vector<double> old(phi, phi + N);
  const int max_deriv = std::min(2, pr->p);
  const double gamma_nb = 0.001, eps = 1.0e-6;
  long cnt = 0;
  for (long c = 0; c < pr->ncell; ++c) cnt += flags[c];
  if (n_troubled) *n_troubled = (int)cnt;
#pragma omp parallel for schedule(dynamic, 16)
  for (long c = 0; c < pr->ncell; ++c) {
    if (!flags[c]) continue;
    const double* ph = old.data() + c * nb;
    double X0[3];
    pr->x0(c, X0);
    std::vector<long> nbs;
    for (int f = 0; f < 4; ++f) {
      long nbc = pr->neighbor(c, f);
      if (nbc >= 0) nbs.push_back(nbc);
    }
    std::vector<double> weights;
    std::vector<std::vector<double>> pq;
    double home_avg = cell_avg(pr, ph);
    // smoothness indicator of one polynomial at the home quadrature points
    auto smooth = [&](const double* coef, const std::array<double, 3>* xi_t, double volume) {
      double beta = 0.0;
      std::vector<double> v(nb), g(nb * 3), hs(nb * 9);
      double gr[256][2], hq[256][2][2];
      for (int q = 0; q < np; ++q) {
        shape_eval(pr, xi_t[q].data(), v.data(), g.data(), hs.data());
        for (int a = 0; a < 2; ++a) {
          gr[q][a] = 0.0;
          for (int j = 0; j < nb; ++j) gr[q][a] += coef[j] * g[j * 3 + a] / pr->h[a];
          for (int b = 0; b < 2; ++b) {
            hq[q][a][b] = 0.0;
            for (int j = 0; j < nb; ++j)
              hq[q][a][b] += coef[j] * hs[(j * 3 + a) * 3 + b] / (pr->h[a] * pr->h[b]);
          }
        }
      }
      if (max_deriv >= 1)
        for (int q = 0; q < np; ++q)
          beta += (gr[q][0] * gr[q][0] + gr[q][1] * gr[q][1]) * (pr->qc.w[q] * pr->vol) * volume;
      if (max_deriv >= 2)
        for (int q = 0; q < np; ++q) {
          // hessians[i][j] with i, j < dim indexes the quadrature point i
          // (pde_tools.implement.h:545-547)
          double ls = 0.0;
          for (int i = 0; i < dim; ++i)
            for (int j = i; j < dim; ++j)
              ls += hq[i][j][0] * hq[i][j][0] + hq[i][j][1] * hq[i][j][1];
          beta += ls * (pr->qc.w[q] * pr->vol) * std::pow(volume, 3);
        }
      return beta;
    };
    // home cell
    {
      double gh = 1.0;
      double acc = 0.0;
      for (size_t k = 0; k < nbs.size(); ++k) acc += gamma_nb;
      gh = 1.0 - acc;
      double den = eps + smooth(ph, pr->qc.xi.data(), pr->vol);
      weights.push_back(gh / den / den);
      std::vector<double> vals(np);
      for (int q = 0; q < np; ++q) vals[q] = eval_at(ph, pr->vc, nb, np, q);
      pq.push_back(vals);
    }
    for (long nbc : nbs) {
      double N0[3];
      pr->x0(nbc, N0);
      std::vector<std::array<double, 3>> xin(np);
      for (int q = 0; q < np; ++q) {
        for (int d = 0; d < 3; ++d) xin[q][d] = 0.0;
        for (int d = 0; d < dim; ++d) {
          double xr = X0[d] + pr->h[d] * pr->qc.xi[q][d];
          xin[q][d] = (xr - N0[d]) / pr->h[d];
        }
      }
      const double* pn = old.data() + nbc * nb;
      double den = eps + smooth(pn, xin.data(), pr->vol);
      weights.push_back(gamma_nb / den / den);
      std::vector<double> v(nb), vals(np);
      double integral = 0.0;
      for (int q = 0; q < np; ++q) {
        shape_eval(pr, xin[q].data(), v.data(), nullptr, nullptr);
        double s = 0.0;
        for (int j = 0; j < nb; ++j) s += pn[j] * v[j];
        vals[q] = s;
        integral += s * (pr->qc.w[q] * pr->vol);
      }
      double this_avg = integral / pr->vol;
      for (int q = 0; q < np; ++q) vals[q] = vals[q] - this_avg + home_avg;
      pq.push_back(vals);
    }
    double wsum = 0.0;
    for (double w : weights) wsum += w;
    for (double& w : weights) w /= wsum;
    std::vector<double> pnew(np, 0.0);
    for (size_t l = 0; l < weights.size(); ++l)
      for (int q = 0; q < np; ++q) pnew[q] += pq[l][q] * weights[l];
    for (int i = 0; i < nb; ++i) {
      double a = 0.0, b = 0.0;
      for (int q = 0; q < np; ++q) {
        double sv = pr->vc[(size_t)i * np + q];
        double jxw = pr->qc.w[q] * pr->vol;
        a += pnew[q] * sv * jxw;
        b += sv * sv * jxw;
      }
      phi[c * nb + i] = a / b;
    }
  }
  return FLSP_OK;
}

// ---------------------------------------------------------------------
// reinitialisation: ReinitSimulatorLDG::initialize / run_iteration*
// (reinit.cc:386-393, 396-480, 529-637)
// ---------------------------------------------------------------------
int orc_reinit(orc_problem* pr, double* phi, const flsp_reinit_opts* o, int* n_iter) {
  const long N = orc_n_dofs(pr);
  const int dim = pr->dim;
  std::vector<double> phi0(phi, phi + N), L(N), s(N);
  const double p1 = pr->p + 1.0;
  // the gradients the next CFL estimate sees: those of the state at the
  // start of the previous pseudo-step (initially of phi0)
  std::vector<double> grad_src(phi, phi + N);
  double vd_run = 0.0, cum = 0.0;
  int it = 0;
  const bool limiter = (o->limiter < 0) ? (dim == 2) : (o->limiter != 0 && dim == 2);
  double horizon;
  if (o->mode == FLSP_REINIT_GLOBAL) {
    double m = 0.0;
    for (long i = 0; i < N; ++i) m = std::max(m, std::fabs(phi[i]));
    horizon = 1.2 * m;
  } else {
    horizon = o->band_width_coeff * pr->min_diam;
  }
  for (;;) {
    if (o->mode == FLSP_REINIT_FIXED) {
      if (it >= o->n_pseudo_steps) break;
    } else if (!(cum < horizon && it <= o->max_iter)) {
      break;
    }
    double vd = orc_hj_cfl(pr, grad_src.data(), phi0.data());
    vd_run = std::max(vd_run, vd);
    double scale = (o->viscosity > 0.0)
                       ? std::pow(p1, 2) * vd_run + o->viscosity * std::pow(p1, 4) / std::pow(pr->min_diam, 2)
                       : adv_cfl_scaling(pr->p) * vd_run;
    double dt = o->cfl_max / scale;
    // explicit_time_derivative ignores its argument and differentiates the
    // current solution (hamilton_jacobi.cc:514-551), so every RK stage sees
    // the same L
    orc_hj_rhs(pr, phi, phi0.data(), o->viscosity, L.data());
    std::copy(phi, phi + N, grad_src.begin());
    int order = o->rk_order < 1 ? 1 : o->rk_order;
    if (order == 1) {
      for (long i = 0; i < N; ++i) { s[i] = L[i] * dt; s[i] += phi[i]; }
    } else if (order == 2) {
      for (long i = 0; i < N; ++i) {
        s[i] = phi[i]; s[i] += dt * L[i]; s[i] += dt * L[i];
        s[i] += phi[i]; s[i] *= 0.5;
      }
    } else {
      const double third = 1.0 / 3.0;
      for (long i = 0; i < N; ++i) {
        s[i] = phi[i]; s[i] += dt * L[i]; s[i] += dt * L[i];
        s[i] += 3.0 * phi[i]; s[i] *= 0.25; s[i] += dt * L[i];
        s[i] *= 2.0; s[i] += phi[i]; s[i] *= third;
      }
    }
    std::copy(s.begin(), s.end(), phi);
    if (limiter) orc_weno(pr, phi, nullptr);
    cum += dt;
    ++it;
  }
  if (n_iter) *n_iter = it;
  if (o->mode == FLSP_REINIT_BAND && it == o->max_iter) return FLSP_ERR_BAND_NOT_REACHED;
  return FLSP_OK;
}

// LevelSetSurface::advance_time(dt, single) (level_set.implement.h:180-205)
int orc_ls_advance(orc_problem* pr, double* phi, orc_clock* clk, int rk_order,
                   double cfl_max, const flsp_ls_opts* o, double time_step,
                   int single_step, double* advanced) {
  double cum = 0.0;
  do {
    double sub = 0.0;
    int st = orc_advance(pr, phi, clk, rk_order, cfl_max, time_step, 1, &sub);
    if (st) return st;
    clk->n_since_reinit++;
    if (o->execute_reinit && clk->n_since_reinit == o->reinit_frequency) {
      int nit = 0;
      st = orc_reinit(pr, phi, &o->reinit, &nit);
      if (st) return st;
      if (nit) clk->n_since_reinit = 0;
    }
    cum += sub;
    time_step -= sub;
  } while (!is_zero(time_step) && !single_step);
  if (advanced) *advanced = cum;
  return FLSP_OK;
}

// ---------------------------------------------------------------------
// reductions (level_set.implement.h:215-295, 356-380, 957-993;
// advection.cc:452-484; reinit.cc:491-526)
// ---------------------------------------------------------------------
static double heaviside_sine(double x, double eps) {
  if (x > eps) return 1.0;
  if (x < -eps) return 0.0;
  double val = 0.5 * (1.0 + x / eps + std::sin(x * kPi / eps) / kPi);
  if (std::fabs(val) < kEps) return 0.0;
  if (std::fabs(val - 1.0) < kEps) return 1.0;
  return val;
}
static double heaviside_sharp(double x) { return x > 0.0 ? 1.0 : (x < 0.0 ? 0.0 : 0.5); }

// MaterialStack mixing: MaterialAccessor<MaterialStack>::reinit + eval_scalars
// (include/felspa/level_set/src/material_stack.implement.h:320-470) with a
// constant scalar per material.  Per QGauss(nq) point: proportion_sum = 1;
// for each level set in stack order while proportion_sum is not zero,
// heaviside = domain_identity(phi) = H(-phi) (level_set.implement.h:356-380,
// smoothing over 1.5 min_diameter, :957-993); if it is not zero the
// material takes proportion_sum * heaviside, which is subtracted; the
// background takes a non-zero remainder; value = sum of value * proportion.
static double mix_heaviside(double y, double eps, int kind) {
  if (kind == FLSP_HEAVISIDE_NONE) return y > 0.0 ? 1.0 : (y < 0.0 ? 0.0 : 0.5);
  if (kind == FLSP_HEAVISIDE_LINEAR) {
    if (y > eps) return 1.0;
    if (y < -eps) return 0.0;
    return 0.5 * (y / eps + 1.0);
  }
  return heaviside_sine(y, eps);
}

int orc_material_mix(int n, orc_problem* const* prs, const double* const* phis, const double* values, int nq,
                     int smoothing, const int64_t* order, double* out) {
  if (n < 1 || !prs || !phis || !values || !out || nq < 1 || nq > 8) return FLSP_ERR_BAD_ARG;
  const orc_problem* p0 = prs[0];
  const int dim = p0->dim;
  double xg[8], wg[8];
  orc_gauss(nq, xg, wg);
  const int npt = dim == 3 ? nq * nq * nq : nq * nq;
  // shape values of every level set at the reference Gauss points
  std::vector<std::vector<double>> sv(n);
  for (int i = 0; i < n; ++i) {
    sv[i].resize((size_t)prs[i]->nb * npt);
    std::vector<double> gtmp((size_t)prs[i]->nb * 3);
    for (int j = 0; j < npt; ++j) {
      const double xi[3] = {xg[j % nq], xg[(j / nq) % nq], dim == 3 ? xg[j / (nq * nq)] : 0.0};
      std::vector<double> val(prs[i]->nb);
      shape_eval(prs[i], xi, val.data(), gtmp.data(), nullptr);
      for (int b = 0; b < prs[i]->nb; ++b) sv[i][(size_t)b * npt + j] = val[b];
    }
  }
#pragma omp parallel for schedule(static)
  for (long k = 0; k < p0->ncell; ++k) {
    const long c = order ? (long)order[k] : k;
    for (int j = 0; j < npt; ++j) {
      double rest = 1.0, v = 0.0;
      for (int i = 0; i < n && !is_zero(rest); ++i) {
        const orc_problem* pr = prs[i];
        double phi = 0.0;
        for (int b = 0; b < pr->nb; ++b) phi += phis[i][c * pr->nb + b] * sv[i][(size_t)b * npt + j];
        const double H = mix_heaviside(-phi, 1.5 * pr->min_diam, smoothing);
        if (!is_zero(H)) {
          const double share = rest * H;
          v += values[i] * share;
          rest -= share;
        }
      }
      if (!is_zero(rest)) v += values[n] * rest;
      out[k * npt + j] = v;
    }
  }
  return FLSP_OK;
}

int orc_reduce(orc_problem* pr, int which, const double* phi, const double* phi_ref,
               const flsp_ic_desc* ic, double* out) {
  const int nb = pr->nb, dim = pr->dim;
  const long N = orc_n_dofs(pr);
  const double eps = 1.5 * pr->min_diam;
  double acc = 0.0, acc2 = 0.0;
  switch (which) {
    case FLSP_RED_MASS:
    case FLSP_RED_MASS_ERROR: {
      const int np = pr->ql.np;
      if (which == FLSP_RED_MASS_ERROR && !ic) return FLSP_ERR_BAD_ARG;
#pragma omp parallel for reduction(+ : acc, acc2) schedule(static)
      for (long c = 0; c < pr->ncell; ++c) {
        double X0[3];
        pr->x0(c, X0);
        for (int q = 0; q < np; ++q) {
          double jxw = pr->ql.w[q] * pr->vol;
          acc += heaviside_sine(-eval_at(phi + c * nb, pr->vl, nb, np, q), eps) * jxw;
          if (ic) {
            double x[3];
            for (int d = 0; d < 3; ++d) x[d] = X0[d] + pr->h[d] * pr->ql.xi[q][d];
            acc2 += heaviside_sine(-ic_node(ic, dim, ic->root, x), eps) * jxw;
          }
        }
      }
      *out = (which == FLSP_RED_MASS) ? acc : (acc - acc2) / acc2;
      return FLSP_OK;
    }
    case FLSP_RED_MASS_SHARP:
    case FLSP_RED_L1_INTERFACE:
    case FLSP_RED_L1_INTERFACE_IC: {
      const int np = pr->qc.np;
      if (which == FLSP_RED_L1_INTERFACE && !phi_ref) return FLSP_ERR_BAD_ARG;
      if (which == FLSP_RED_L1_INTERFACE_IC && !ic) return FLSP_ERR_BAD_ARG;
#pragma omp parallel for reduction(+ : acc) schedule(static)
      for (long c = 0; c < pr->ncell; ++c) {
        double X0[3];
        pr->x0(c, X0);
        for (int q = 0; q < np; ++q) {
          double jxw = pr->qc.w[q] * pr->vol;
          double a = heaviside_sharp(-eval_at(phi + c * nb, pr->vc, nb, np, q));
          if (which == FLSP_RED_MASS_SHARP) { acc += a * jxw; continue; }
          double b;
          if (which == FLSP_RED_L1_INTERFACE) {
            b = heaviside_sharp(-eval_at(phi_ref + c * nb, pr->vc, nb, np, q));
          } else {
            double x[3];
            for (int d = 0; d < 3; ++d) x[d] = X0[d] + pr->h[d] * pr->qc.xi[q][d];
            b = heaviside_sharp(-ic_node(ic, dim, ic->root, x));
          }
          acc += std::fabs(a - b) * jxw;
        }
      }
      *out = acc;
      return FLSP_OK;
    }
    case FLSP_RED_MEAN_ABS_DIFF: {
      if (!phi_ref) return FLSP_ERR_BAD_ARG;
      for (long i = 0; i < N; ++i) acc += std::fabs(phi[i] - phi_ref[i]);
      *out = acc / N;
      return FLSP_OK;
    }
    case FLSP_RED_GRAD_DEVIATION: {
      const int np = pr->ql.np;
#pragma omp parallel for reduction(+ : acc, acc2) schedule(static)
      for (long c = 0; c < pr->ncell; ++c) {
        double dev = 0.0;
        for (int q = 0; q < np; ++q) {
          double g2 = 0.0;
          for (int d = 0; d < dim; ++d) {
            double g = 0.0;
            for (int j = 0; j < nb; ++j) g += phi[c * nb + j] * (pr->gl[((size_t)j * np + q) * 3 + d] / pr->h[d]);
            g2 += g * g;
          }
          dev += std::fabs(std::sqrt(g2) - 1.0) * (pr->ql.w[q] * pr->vol);
        }
        acc += dev;
        acc2 += pr->vol;
      }
      *out = acc / acc2;
      return FLSP_OK;
    }
    case FLSP_RED_MAX_ABS: {
      double m = 0.0;
      for (long i = 0; i < N; ++i) m = std::max(m, std::fabs(phi[i]));
      *out = m;
      return FLSP_OK;
    }
    case FLSP_RED_L2_ERROR_IC: {
      if (!ic) return FLSP_ERR_BAD_ARG;
      const int np = pr->ql.np;
#pragma omp parallel for reduction(+ : acc) schedule(static)
      for (long c = 0; c < pr->ncell; ++c) {
        double X0[3];
        pr->x0(c, X0);
        double e2 = 0.0;
        for (int q = 0; q < np; ++q) {
          double x[3];
          for (int d = 0; d < 3; ++d) x[d] = X0[d] + pr->h[d] * pr->ql.xi[q][d];
          double diff = eval_at(phi + c * nb, pr->vl, nb, np, q) - ic_node(ic, dim, ic->root, x);
          e2 += diff * diff * (pr->ql.w[q] * pr->vol);
        }
        acc += e2;  // sum of squared cell L2 errors (compute_global_error)
      }
      *out = std::sqrt(acc);
      return FLSP_OK;
    }
  }
  return FLSP_ERR_BAD_ARG;
}

// ---------------------------------------------------------------------
// learned reinitialisation: FP64 reference MLP, GELU(x) = x Phi(x)
// layer l: y = W_l x + b_l, W_l row-major [widths[l+1]][widths[l]]
// ---------------------------------------------------------------------
static inline double gelu(double x) { return 0.5 * x * (1.0 + std::erf(x / std::sqrt(2.0))); }
static inline double gelu_d(double x) {
  double cdf = 0.5 * (1.0 + std::erf(x / std::sqrt(2.0)));
  double pdf = std::exp(-0.5 * x * x) / std::sqrt(2.0 * kPi);
  return cdf + x * pdf;
}

int orc_mlp_forward(int n_layers, const int* widths, const double* const* W,
                    const double* const* b, int batch, const double* x, double* y) {
  int maxw = 0;
  for (int l = 0; l <= n_layers; ++l) maxw = std::max(maxw, widths[l]);
#pragma omp parallel for schedule(static)
  for (int s = 0; s < batch; ++s) {
    std::vector<double> a(x + (size_t)s * widths[0], x + (size_t)(s + 1) * widths[0]), z(maxw);
    for (int l = 0; l < n_layers; ++l) {
      int ni = widths[l], no = widths[l + 1];
      for (int o = 0; o < no; ++o) {
        double acc = b[l][o];
        for (int i = 0; i < ni; ++i) acc += W[l][(size_t)o * ni + i] * a[i];
        z[o] = (l + 1 < n_layers) ? gelu(acc) : acc;
      }
      a.assign(z.begin(), z.begin() + no);
    }
    for (int o = 0; o < widths[n_layers]; ++o) y[(size_t)s * widths[n_layers] + o] = a[o];
  }
  return FLSP_OK;
}

int orc_mlp_backward(int n_layers, const int* widths, const double* const* W,
                     const double* const* b, int batch, const double* x,
                     const double* dy, double* const* dW, double* const* db) {
  for (int l = 0; l < n_layers; ++l) {
    std::fill(dW[l], dW[l] + (size_t)widths[l] * widths[l + 1], 0.0);
    std::fill(db[l], db[l] + widths[l + 1], 0.0);
  }
  for (int s = 0; s < batch; ++s) {
    std::vector<std::vector<double>> acts(n_layers + 1), pre(n_layers);
    acts[0].assign(x + (size_t)s * widths[0], x + (size_t)(s + 1) * widths[0]);
    for (int l = 0; l < n_layers; ++l) {
      int ni = widths[l], no = widths[l + 1];
      pre[l].resize(no);
      acts[l + 1].resize(no);
      for (int o = 0; o < no; ++o) {
        double acc = b[l][o];
        for (int i = 0; i < ni; ++i) acc += W[l][(size_t)o * ni + i] * acts[l][i];
        pre[l][o] = acc;
        acts[l + 1][o] = (l + 1 < n_layers) ? gelu(acc) : acc;
      }
    }
    std::vector<double> g(dy + (size_t)s * widths[n_layers], dy + (size_t)(s + 1) * widths[n_layers]);
    for (int l = n_layers - 1; l >= 0; --l) {
      int ni = widths[l], no = widths[l + 1];
      if (l + 1 < n_layers)
        for (int o = 0; o < no; ++o) g[o] *= gelu_d(pre[l][o]);
      std::vector<double> gi(ni, 0.0);
      for (int o = 0; o < no; ++o) {
        db[l][o] += g[o];
        for (int i = 0; i < ni; ++i) {
          dW[l][(size_t)o * ni + i] += g[o] * acts[l][i];
          gi[i] += W[l][(size_t)o * ni + i] * g[o];
        }
      }
      g = gi;
    }
  }
  return FLSP_OK;
}

// LevelSetSurface::CurvatureEstimator::estimate
// (include/felspa/level_set/src/level_set.implement.h:600-620): RHS by
// local_assembly (:667-742) with QGauss(p+1) cell and face rules, the
// advection system's mass solve (|K| I for the orthonormal basis), then the
// absolute value of every coefficient.  Per cell:
//   cell_assembly (:747-763): R_i -= sum_q grad psi_i . grad phi / |grad phi| JxW;
//   boundary_assembly (:796-811): R_i += (grad phi / |grad phi|) . n psi_i JxW;
//   face_assembly (:766-792) on interior faces, computed by the cell with the
//   lower CellId (:717; `order` gives that order: order[k] = lattice index of
//   the k-th cell, NULL = lexicographic), per component d:
//     s = (n_in[d] - n_ex[d]) / (phi_in - phi_ex)     (n = grad phi / |grad phi|)
//     F[d] = s > 0 ? (normal[d] > 0 ? n_in[d] : n_ex[d])
//          : s < 0 ? (normal[d] > 0 ? n_ex[d] : n_in[d]) : 0    (NaN -> 0)
//   and R_in,i += psi_i^in F.n JxW, R_ex,i -= psi_i^ex F.n JxW, where the
//   exterior copy is bound to the owning cell (copy_ex.reinit(cell), :731),
//   so both terms land in the owner's DoFs (psi^ex: the neighbour's basis
//   function of the same index at the shared points) and the neighbour
//   receives nothing from that face.
// to_neighbour != 0: the exterior term goes to the neighbour's DoFs instead
// (each cell adds psi_i F.n_own JxW on every interior face; F is the same
// from either side), i.e. the weak divergence of grad phi / |grad phi|.
int orc_curvature(orc_problem* pr, const double* phi, const int64_t* order, int to_neighbour,
                  double* kappa) {
  const int nb = pr->nb, dim = pr->dim, np = pr->ql.np;
  std::vector<long> pos(pr->ncell);
  for (long k = 0; k < pr->ncell; ++k) {
    const long c = order ? (long)order[k] : k;
    if (c < 0 || c >= pr->ncell) return FLSP_ERR_BAD_ARG;
    pos[c] = k;
  }
#pragma omp parallel for schedule(static)
  for (long c = 0; c < pr->ncell; ++c) {
    const double* pc = phi + c * nb;
    double R[128] = {0};
    // cell term
    for (int q = 0; q < np; ++q) {
      double g[3] = {0, 0, 0};
      for (int j = 0; j < nb; ++j)
        for (int d = 0; d < dim; ++d) g[d] += pc[j] * (pr->gl[((size_t)j * np + q) * 3 + d] / pr->h[d]);
      double nrm = 0.0;
      for (int d = 0; d < dim; ++d) nrm += g[d] * g[d];
      nrm = std::sqrt(nrm);
      const double jxw = pr->ql.w[q] * pr->vol;
      for (int i = 0; i < nb; ++i) {
        double dot = 0.0;
        for (int d = 0; d < dim; ++d) dot += (pr->gl[((size_t)i * np + q) * 3 + d] / pr->h[d]) * (g[d] / nrm);
        R[i] -= dot * jxw;
      }
    }
    // faces
    for (int f = 0; f < 2 * dim; ++f) {
      const int ax = f / 2, s = f % 2;
      const long nbc = pr->neighbor(c, f);
      if (nbc >= 0 && !to_neighbour && pos[c] > pos[nbc]) continue;   // the neighbour owns this face
      const FaceQuad& fq = pr->fl[f];
      const int nf = fq.np;
      const double area = pr->vol / pr->h[ax];
      double normal[3] = {0, 0, 0};
      normal[ax] = s ? 1.0 : -1.0;
      auto trace = [&](const double* pcc, int ff, int q, double* val, double* g) {
        *val = 0.0;
        g[0] = g[1] = g[2] = 0.0;
        for (int j = 0; j < nb; ++j) {
          *val += pcc[j] * pr->vfl[ff][(size_t)j * nf + q];
          for (int d = 0; d < dim; ++d) g[d] += pcc[j] * (pr->gfl[ff][((size_t)j * nf + q) * 3 + d] / pr->h[d]);
        }
      };
      for (int q = 0; q < nf; ++q) {
        const double jxw = fq.w[q] * area;
        double pin, gin[3];
        trace(pc, f, q, &pin, gin);
        double nin = 0.0;
        for (int d = 0; d < dim; ++d) nin += gin[d] * gin[d];
        nin = std::sqrt(nin);
        if (nbc < 0) {
          double fn = 0.0;
          for (int d = 0; d < dim; ++d) fn += gin[d] / nin * normal[d];
          for (int i = 0; i < nb; ++i) R[i] += fn * pr->vfl[f][(size_t)i * nf + q] * jxw;
          continue;
        }
        double pex, gex[3];
        trace(phi + nbc * nb, f ^ 1, q, &pex, gex);
        double nex = 0.0;
        for (int d = 0; d < dim; ++d) nex += gex[d] * gex[d];
        nex = std::sqrt(nex);
        double F[3] = {0, 0, 0};
        for (int d = 0; d < dim; ++d) {
          const double sh = (gin[d] / nin - gex[d] / nex) / (pin - pex);
          if (sh > 0.0) F[d] = normal[d] > 0 ? gin[d] / nin : gex[d] / nex;
          else if (sh < 0.0) F[d] = normal[d] > 0 ? gex[d] / nex : gin[d] / nin;
          else F[d] = 0.0;
        }
        double fn = 0.0;
        for (int d = 0; d < dim; ++d) fn += F[d] * normal[d];
        for (int i = 0; i < nb; ++i) {
          R[i] += pr->vfl[f][(size_t)i * nf + q] * fn * jxw;
          if (!to_neighbour) R[i] -= pr->vfl[f ^ 1][(size_t)i * nf + q] * fn * jxw;
        }
      }
    }
    for (int i = 0; i < nb; ++i) kappa[c * nb + i] = std::fabs(R[i] / pr->vol);
  }
  return FLSP_OK;
}

}  // extern "C"

// flsp_clock.cuh — the device clocks' updates (shared by the single-problem
// clock kernels and the batched ones).
#pragma once
#include "flsp_device.cuh"

namespace flsp {

constexpr double kClockEps = 2.220446049250313e-16;

// AdvectSimulator::advance_time substep set-up (advection.cc:396-404):
// CFL estimate at the current time (running maximum, the estimator never
// resets), substep = min(cfl_max / estimate, remaining), stage time factors.
__device__ __forceinline__ void adv_clock_begin_body(DevClock* c, const AdvClockArgs& a) {
  const double ctn = time_factor(a.tkind, a.ta, a.tb, c->t);
  const double vd = fabs(ctn) * c->vd_static;
  c->vd_run = fmax(c->vd_run, vd);
  double suggest = a.cfl_max / (c->vd_run * a.scale);
  const double remaining = c->scratch[0] - c->scratch[1];   // time_step - cumulative
  // a velocity whose time factor vanishes (e.g. 1 - exp(-t) at t = 0) gives
  // an infinite CFL substep.  A call for a time step (the reference rule)
  // then takes the remaining time; a step-count run, whose horizon only
  // caps the time, falls back to the estimate of the spatial field alone
  // (|time factor| = 1)
  if (a.step_count && !isfinite(suggest) && c->vd_static > 0.0) suggest = a.cfl_max / (c->vd_static * a.scale);
  double dt = fmin(suggest, remaining);
  if (!isfinite(dt) && c->vd_static > 0.0) dt = a.cfl_max / (c->vd_static * a.scale);
  c->dt = dt;
  c->active = fabs(dt) <= kClockEps ? 0 : 1;   // TempoIntegrator skips zero steps
  c->ct[0] = ctn;
  c->ct[1] = time_factor(a.tkind, a.ta, a.tb, c->t + dt);
  c->ct[2] = time_factor(a.tkind, a.ta, a.tb, c->t + 0.5 * dt);
}

__device__ __forceinline__ void adv_clock_end_body(DevClock* c) {
  if (c->active) {
    c->t += c->dt;
    c->n_substeps += 1;
  }
  c->scratch[1] += c->dt;   // cumulative time of this advance call
}

// start an advance call of length time_step (scratch[0]); +inf = unclamped
__device__ __forceinline__ void adv_clock_horizon_body(DevClock* c, double time_step) {
  c->scratch[0] = time_step;
  c->scratch[1] = 0.0;
}

__device__ __forceinline__ void hj_clock_reset_body(DevClock* c) {
  c->hj_vd_run = 0.0;
  c->hj_dt = 0.0;
  c->hj_cum = 0.0;
  c->hj_vd_bits = 0ull;
  c->hj_iter = 0;
}

// ReinitSimulatorLDG::advance_time step size (reinit.cc:396-408) with
// HJSimulator::cfl_scaling (hamilton_jacobi.cc:554-580)
__device__ __forceinline__ void hj_clock_begin_body(DevClock* c, double cfl_max, int p, double nu, double min_diam,
                                                    double adv_scale) {
  const double vd = __longlong_as_double((long long)c->hj_vd_bits);
  c->hj_vd_bits = 0ull;
  c->hj_vd_run = fmax(c->hj_vd_run, vd);
  double scale;
  if (nu > 0.0)
    scale = pow((double)(p + 1), 2.0) * c->hj_vd_run + nu * pow((double)(p + 1), 4.0) / pow(min_diam, 2.0);
  else
    scale = adv_scale * c->hj_vd_run;
  c->hj_dt = cfl_max / scale;
}

__device__ __forceinline__ void hj_clock_end_body(DevClock* c) {
  c->hj_cum += c->hj_dt;
  c->hj_iter += 1;
}

}  // namespace flsp

// Device-side state of the SSP-RK3 time loop (one per candidate) and the
// per-step device functions shared by the single-context kernels
// (kernels_adjoint.cuh) and the grouped batch kernels (kernels_batch.cuh).
#pragma once

#include "kernels.cuh"

namespace o2f {

struct StepState {
  double t, dt, final_time, cfl, min_h, mu;
  double hist0, drop_tol;
  unsigned long long max_wave_bits;  // max(|u|+c) as the bits of a positive double
  long long step, max_steps;
  int stop;  // 0 running, 1 finished (time, step cap or residual drop), 2 non-finite
  int drop_hit;
};

// Start of a step: evaluate the loop condition, reset the wave-speed maximum.
__device__ __forceinline__ void step_begin_at(StepState* st) {
  if (st->stop) return;
  if (!(st->t < st->final_time) || st->step >= st->max_steps || st->drop_hit) {
    st->stop = 1;
    return;
  }
  st->max_wave_bits = (unsigned long long)__double_as_longlong(1e-8);
}
// |u| + c of one cell state folded into the running maximum m with the
// reference's std::max(max_wave, speed) semantics (src/simulation.cpp:96): a
// NaN speed (a cell whose pressure or density went negative while its
// interface states stayed valid) is skipped, not fatal.  Non-finite states
// and residuals are caught by the residual norm (step_norm_block).
template <typename T>
__device__ __forceinline__ void wave_speed_cell(const Vec4<T>& q, double gamma, double& m) {
  const double rho = q.a, ru = q.b, rv = q.c, E = q.d;
  const double u = ru / rho, v = rv / rho;
  const double kinetic = 0.5 * (ru * ru + rv * rv) / rho;
  const double p = (gamma - 1.0) * (E - kinetic);
  const double cs = sqrt(gamma * p / rho);
  const double speed = hypot(u, v) + cs;
  if (speed > m) m = speed;
}

// Warp-level combination of the per-thread maxima into st.
__device__ __forceinline__ void wave_speed_commit(double m, StepState* st) {
  for (int o = 16; o > 0; o >>= 1) {
    const double other = __shfl_down_sync(0xffffffffu, m, o);
    if (other > m) m = other;
  }
  if ((threadIdx.x & 31) == 0 && m > 0.0)
    atomicMax(&st->max_wave_bits, (unsigned long long)__double_as_longlong(m));
}

// dt = min(CFL*min_h/max_wave, 0.5*min_h^2/mu) (src/simulation.cpp:108-110).
__device__ __forceinline__ void step_dt_at(StepState* st) {
  if (st->stop) return;
  const double max_wave = __longlong_as_double((long long)st->max_wave_bits);
  const double dt_adv = st->cfl * st->min_h / max_wave;
  const double dt_diff = 0.5 * (st->min_h * st->min_h) / st->mu;
  st->dt = smin(dt_adv, dt_diff);
}
// One block: fold the partials, record the norm and the stop conditions.
__device__ __forceinline__ void step_norm_block(const double* part, int nparts, double* hist, StepState* st) {
  __shared__ double sm[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) s += part[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += sm[w];
    const double nrm = sqrt(tot);
    if (hist) hist[st->step] = nrm;
    if (st->step == 0) st->hist0 = nrm;
    if (!(nrm <= 1.7976931348623157e308)) st->stop = 2;  // NaN or +inf
    if (st->drop_tol > 0.0 && st->hist0 > 0.0 && nrm <= st->drop_tol * st->hist0) st->drop_hit = 1;
  }
}

__device__ __forceinline__ void step_end_at(StepState* st) {
  if (st->stop) return;
  st->t += st->dt;
  st->step += 1;
}
}  // namespace o2f

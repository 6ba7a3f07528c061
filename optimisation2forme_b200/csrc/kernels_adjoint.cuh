// Kernels of the time-step control, the forces/objective, the discrete adjoint
// (Jacobian-transpose blocks, matrix-free product, right-hand side), the
// BiCGSTAB vector updates with their fused FP64 reductions, and the shape
// perturbation.  Same conventions as kernels.cuh.
#pragma once

#include "kernels.cuh"
#include "step.cuh"

namespace o2f {

// ---------------------------------------------------------------------------
// Deterministic grid reductions.  Kernels that reduce write one partial per
// block; the last block to finish (atomic ticket) sums the partials in block
// order with a fixed warp tree and runs a scalar epilogue.  Results do not
// depend on scheduling.

constexpr int kRedGrid = 148 * 4;  // fixed grid of the reducing vector kernels

template <int N>
__device__ __forceinline__ void warp_sum(double (&v)[N]) {
#pragma unroll
  for (int i = 0; i < N; ++i)
    for (int o = 16; o > 0; o >>= 1) v[i] += __shfl_down_sync(0xffffffffu, v[i], o);
}

// Block-reduce N values; returns true in thread 0 of the LAST block, with the
// grid totals in tot[].  part: [gridDim.x * N] scratch, ticket: zero-initialised
// counter (reset by the last block).
template <int N>
__device__ bool grid_reduce(double (&v)[N], double* part, unsigned int* ticket, double (&tot)[N]) {
  __shared__ double sm[kBlock / 32][N];
  __shared__ bool last;
  warp_sum<N>(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int i = 0; i < N; ++i) sm[warp][i] = v[i];
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < N; ++i) {
      double s = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sm[w][i];
      part[blockIdx.x * N + i] = s;
    }
    __threadfence();
    const unsigned int t = atomicAdd(ticket, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return false;
  // Last block: the first warp sums the partials in a fixed pattern.
  __threadfence();
  if (warp == 0) {
    double acc[N];
#pragma unroll
    for (int i = 0; i < N; ++i) acc[i] = 0.0;
    for (int b = lane; b < (int)gridDim.x; b += 32)
#pragma unroll
      for (int i = 0; i < N; ++i) acc[i] += ((volatile double*)part)[b * N + i];
    warp_sum<N>(acc);
    if (lane == 0) {
#pragma unroll
      for (int i = 0; i < N; ++i) tot[i] = acc[i];
      *ticket = 0u;
    }
  }
  return threadIdx.x == 0;
}

// ---------------------------------------------------------------------------
// Time-step control of Simulator::time_loop (src/simulation.cpp:68-124); the
// per-step device functions and StepState are in step.cuh.

// Start of a step: evaluate the loop condition, reset the wave-speed maximum.
__global__ void k_step_begin(StepState* st) { step_begin_at(st); }

// max over cells of hypot(u, v) + c (src/simulation.cpp:80-96).  The maximum
// of positive doubles is exact, so the atomic order does not matter.
template <typename T>
__global__ void __launch_bounds__(kBlock) k_wave_speed(int64_t nc, const Vec4<T>* __restrict__ U, double gamma,
                                                       StepState* st) {
  if (st->stop) return;
  double m = 0.0;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += (int64_t)gridDim.x * blockDim.x)
    wave_speed_cell(U[c], gamma, m);
  wave_speed_commit(m, st);
}

// dt = min(CFL*min_h/max_wave, 0.5*min_h^2/mu) (src/simulation.cpp:108-110).
__global__ void k_step_dt(StepState* st) { step_dt_at(st); }

// Residual history: ||R_rho||_2 of the first stage, from the per-block partials.
__global__ void k_step_norm(const double* part, int nparts, double* hist, StepState* st) {
  if (st->stop) return;
  step_norm_block(part, nparts, hist, st);
}

__global__ void k_step_end(StepState* st) { step_end_at(st); }

// ---------------------------------------------------------------------------
// computeLiftDragCoefficients (src/compute.cpp:92-132) and
// computeDirectObjectiveTerm (src/shape_optimization.cpp:893-939): pressure
// from the LEFT interface state of wall edges plus the stored wall stress.
// One block; warp-shuffle reduction in FP64.  out = {C_L, C_D, J}.
template <typename T>
__global__ void __launch_bounds__(kBlock) k_forces(int64_t nwall, const int32_t* __restrict__ wall_edges, Geom<T> g,
                                                   const Vec4<T>* __restrict__ eL, const Vec4<T>* __restrict__ etq,
                                                   Phys ph, double beta, double* out) {
  double acc[4] = {0.0, 0.0, 0.0, 0.0};  // lift-axis / drag-axis sums: all edges, J edges
  const double gm1 = ph.gamma - 1.0;
  for (int64_t i = threadIdx.x; i < nwall; i += blockDim.x) {
    const int e = wall_edges[i];
    const Vec4<T> s = eL[e];
    const Vec4<T> eg = g.egeom[e];
    const Vec4<T> t = etq[e];
    const double nx = eg.a, ny = eg.b, A = eg.c;
    const double rho = s.a, ru = s.b, rv = s.c, E = s.d;
    const double p = gm1 * (E - 0.5 * (ru * ru + rv * rv) / rho);
    const double txx = t.a, tyy = t.b, txy = t.c;
    const double Fy = (-p * ny + txy * nx + tyy * ny) * A;
    const double Fx = (-p * nx + txx * nx + txy * ny) * A;
    acc[0] += Fy;
    acc[1] += Fx;
    if (!((double)g.ectr[e].a > 1.3)) {
      acc[2] += Fy;
      acc[3] += Fx;
    }
  }
  __shared__ double sm[kBlock / 32][4];
  warp_sum<4>(acc);
  if ((threadIdx.x & 31) == 0)
    for (int i = 0; i < 4; ++i) sm[threadIdx.x >> 5][i] = acc[i];
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot[4] = {0.0, 0.0, 0.0, 0.0};
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
      for (int i = 0; i < 4; ++i) tot[i] += sm[w][i];
    const double corde = 1.0;
    const double L = tot[0] * ph.cos_a - tot[1] * ph.sin_a;
    const double D = tot[1] * ph.cos_a + tot[0] * ph.sin_a;
    const double LJ = tot[2] * ph.cos_a - tot[3] * ph.sin_a;
    const double DJ = tot[3] * ph.cos_a + tot[2] * ph.sin_a;
    out[0] = L / (ph.q_inf * corde);
    out[1] = D / (ph.q_inf * corde);
    const double CLJ = LJ / (ph.q_inf * corde), CDJ = DJ / (ph.q_inf * corde);
    out[2] = -CLJ + beta * CDJ;
  }
}

// ---------------------------------------------------------------------------
// Jacobian-transpose blocks (src/shape_optimization.cpp:245-430): per edge the
// 4x4 central differences (absolute eps) of the HLLC flux with respect to the
// left and right interface states, with the ghost state rebuilt from the
// perturbed left state on boundary edges.  The blocks depend only on the
// frozen interface states, so they are built once per adjoint solve instead of
// once per product.  Layout: blk[e*32 + r*4 + c] = F_UL[r][c],
// blk[e*32 + 16 + r*4 + c] = F_UR[r][c].  F_UR of boundary edges is never used
// by the product (:437-453) and is left at zero.
__device__ __forceinline__ double& comp(Vec4<double>& v, int j) {
  return j == 0 ? v.a : j == 1 ? v.b : j == 2 ? v.c : v.d;
}
__device__ __forceinline__ double comp(const Vec4<double>& v, int j) {
  return j == 0 ? v.a : j == 1 ? v.b : j == 2 ? v.c : v.d;
}

__global__ void __launch_bounds__(128) k_jt_blocks(int64_t ne, Geom<double> g, const uint8_t* __restrict__ ebc,
                                                   const Vec4<double>* __restrict__ eL,
                                                   const Vec4<double>* __restrict__ eR, Phys ph, double eps,
                                                   double* __restrict__ blk) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  const Vec4<double> eg = g.egeom[e];
  const double gamma = ph.gamma;
  const uint8_t code = ebc[e];
  const Vec4<double> Ls = eL[e], Rs = eR[e];
  double* out = blk + e * 32;
  for (int j = 0; j < 4; ++j) {
    Vec4<double> Lp = Ls, Lm = Ls, Rp = Rs, Rm = Rs;
    comp(Lp, j) = comp(Ls, j) + eps;
    comp(Lm, j) = comp(Ls, j) - eps;
    if (code != 0) {
      Rp = bc_ghost(code, ph, Lp);
      Rm = bc_ghost(code, ph, Lm);
    }
    const Vec4<double> fp = hllc(Lp, Rp, eg.a, eg.b, gamma);
    const Vec4<double> fm = hllc(Lm, Rm, eg.a, eg.b, gamma);
    out[0 * 4 + j] = (fp.a - fm.a) / (2 * eps);
    out[1 * 4 + j] = (fp.b - fm.b) / (2 * eps);
    out[2 * 4 + j] = (fp.c - fm.c) / (2 * eps);
    out[3 * 4 + j] = (fp.d - fm.d) / (2 * eps);
  }
  for (int j = 0; j < 4; ++j) {
    if (code != 0) {
      out[16 + 0 * 4 + j] = 0.0;
      out[16 + 1 * 4 + j] = 0.0;
      out[16 + 2 * 4 + j] = 0.0;
      out[16 + 3 * 4 + j] = 0.0;
      continue;
    }
    Vec4<double> Rp = Rs, Rm = Rs;
    comp(Rp, j) = comp(Rs, j) + eps;
    comp(Rm, j) = comp(Rs, j) - eps;
    const Vec4<double> fp = hllc(Ls, Rp, eg.a, eg.b, gamma);
    const Vec4<double> fm = hllc(Ls, Rm, eg.a, eg.b, gamma);
    out[16 + 0 * 4 + j] = (fp.a - fm.a) / (2 * eps);
    out[16 + 1 * 4 + j] = (fp.b - fm.b) / (2 * eps);
    out[16 + 2 * 4 + j] = (fp.c - fm.c) / (2 * eps);
    out[16 + 3 * 4 + j] = (fp.d - fm.d) / (2 * eps);
  }
}

// y = J^T x as a per-cell gather (src/shape_optimization.cpp:433-482): for each
// edge of the cell, in ascending reference edge id (the order in which the
// reference's atomic updates land at one thread),
//   Delta = (-x_L/V_L + x_R/V_R) L   (boundary: -x_L/V_L L)
//   y_c  += F_{U_side}^T Delta.
// Deterministic: no atomics.  Optional fused epilogue: dots of y with up to
// two other vectors, reduced over the grid (kDots), for BiCGSTAB.
// One 4x4 Jacobian block into registers: FP64 blocks as stored, FP32 blocks
// (the mixed-precision path) widened to FP64 for the accumulation.
__device__ __forceinline__ void load_block(const double* B, double* b) {
#pragma unroll
  for (int i = 0; i < 16; i += 2) {
    const double2 t = *reinterpret_cast<const double2*>(B + i);
    b[i] = t.x;
    b[i + 1] = t.y;
  }
}
__device__ __forceinline__ void load_block(const float* B, double* b) {
#pragma unroll
  for (int i = 0; i < 16; i += 4) {
    const float4 t = *reinterpret_cast<const float4*>(B + i);
    b[i] = (double)t.x;
    b[i + 1] = (double)t.y;
    b[i + 2] = (double)t.z;
    b[i + 3] = (double)t.w;
  }
}

template <int kDots, typename TB>
__device__ __forceinline__ void jt_cell(int64_t c, int64_t nc, const int32_t* __restrict__ jslot, Geom<double> g,
                                        const int2* __restrict__ ec, const uint8_t* __restrict__ ebc,
                                        const TB* __restrict__ blk, const Vec4<double>* __restrict__ x,
                                        Vec4<double>& y) {
  const Vec4<double> xc = x[c];
  const double invVc = 1.0 / g.cgeom[c].c;
  y = v4<double>(0.0, 0.0, 0.0, 0.0);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int s = jslot[(int64_t)k * nc + c];
    if (s < 0) break;
    const int e = s >> 1;
    const bool left = (s & 1) == 0;
    const double L = g.egeom[e].c;
    double d0, d1, d2, d3;
    const TB* B;
    if (ebc[e] != 0) {
      d0 = (-xc.a * invVc) * L;
      d1 = (-xc.b * invVc) * L;
      d2 = (-xc.c * invVc) * L;
      d3 = (-xc.d * invVc) * L;
      B = blk + (int64_t)e * 32;
    } else {
      const int2 cc = ec[e];
      const Vec4<double> xl = left ? xc : x[cc.x];
      const Vec4<double> xr = left ? x[cc.y] : xc;
      const double invVl = left ? invVc : 1.0 / g.cgeom[cc.x].c;
      const double invVr = left ? 1.0 / g.cgeom[cc.y].c : invVc;
      d0 = (-xl.a * invVl + xr.a * invVr) * L;
      d1 = (-xl.b * invVl + xr.b * invVr) * L;
      d2 = (-xl.c * invVl + xr.c * invVr) * L;
      d3 = (-xl.d * invVl + xr.d * invVr) * L;
      B = blk + (int64_t)e * 32 + (left ? 0 : 16);
    }
    double b[16];
    load_block(B, b);
    y.a += (b[0] * d0 + b[4] * d1 + b[8] * d2 + b[12] * d3);
    y.b += (b[1] * d0 + b[5] * d1 + b[9] * d2 + b[13] * d3);
    y.c += (b[2] * d0 + b[6] * d1 + b[10] * d2 + b[14] * d3);
    y.d += (b[3] * d0 + b[7] * d1 + b[11] * d2 + b[15] * d3);
  }
}

template <typename TB>
__global__ void __launch_bounds__(kBlock) k_jt_apply(int64_t nc, const int32_t* __restrict__ jslot, Geom<double> g,
                                                     const int2* __restrict__ ec, const uint8_t* __restrict__ ebc,
                                                     const TB* __restrict__ blk,
                                                     const Vec4<double>* __restrict__ x, Vec4<double>* __restrict__ y) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  Vec4<double> r;
  jt_cell<0, TB>(c, nc, jslot, g, ec, ebc, blk, x, r);
  y[c] = r;
}

// assembleAdjointRHS (src/shape_optimization.cpp:491-554): b = dJ/dU_L from the
// wall pressure, added to the wall edge's left cell, edges in ascending
// reference id.  One thread per cell owning wall edges; b must be zeroed.
__global__ void k_adjoint_rhs(int64_t nwc, const int32_t* __restrict__ wall_cells,
                              const int32_t* __restrict__ wc_off, const int32_t* __restrict__ wc_edges,
                              Geom<double> g, const Vec4<double>* __restrict__ eL, Phys ph, double beta,
                              Vec4<double>* __restrict__ b) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nwc) return;
  const int c = wall_cells[i];
  const double gamma = ph.gamma;
  const double q_inf = ph.q_inf, corde = 1.0;
  Vec4<double> acc = b[c];
  for (int k = wc_off[i]; k < wc_off[i + 1]; ++k) {
    const int e = wc_edges[k];
    const Vec4<double> eg = g.egeom[e];
    const double A_f = eg.c, nx = eg.a, ny = eg.b;
    const Vec4<double> s = eL[e];
    const double rho_L = s.a, rho_u_L = s.b, rho_v_L = s.c;
    const double dp_drho = 0.5 * (gamma - 1.0) * ((rho_u_L * rho_u_L + rho_v_L * rho_v_L) / (rho_L * rho_L));
    const double dp_dru = -(gamma - 1.0) * (rho_u_L / rho_L);
    const double dp_drv = -(gamma - 1.0) * (rho_v_L / rho_L);
    const double dp_dE = (gamma - 1.0);
    // Lift/drag axes rotated by the angle of attack (cos=1, sin=0 reproduces
    // the reference's +ny and -nx coefficients exactly).
    const double coeff_CL = +(ny * ph.cos_a - nx * ph.sin_a) * A_f / (q_inf * corde);
    acc.a += coeff_CL * dp_drho;
    acc.b += coeff_CL * dp_dru;
    acc.c += coeff_CL * dp_drv;
    acc.d += coeff_CL * dp_dE;
    const double coeff_CD = (-(nx * ph.cos_a) - ny * ph.sin_a) * A_f / (q_inf * corde) * beta;
    acc.a += coeff_CD * dp_drho;
    acc.b += coeff_CD * dp_dru;
    acc.c += coeff_CD * dp_drv;
    acc.d += coeff_CD * dp_dE;
  }
  b[c] = acc;
}

// ---------------------------------------------------------------------------
// BiCGSTAB (van der Vorst 1992) with the restart-on-orthogonality remedy,
// driven from the device: the scalars live in KrylovState, every kernel is a
// no-op once `stop` is set, so chunks of iterations can be launched as a CUDA
// graph without host round trips.
struct KrylovState {
  double rho, alpha, omega, beta;
  double rr, bb, r0r0, tol2;
  long long it, it_chunk, chunk_max;
  int stop;      // 0 running, 1 converged, 2 chunk cap, 3 breakdown, 4 non-finite
  int restart_r0;
  unsigned int ticket;
  int pad;
};

// r = b - t, r0 = r, p = v = 0; totals (r,r), (b,b).
__global__ void __launch_bounds__(kBlock) k_bicg_start(int64_t n4, const double* __restrict__ b,
                                                       const double* __restrict__ t, double* __restrict__ r,
                                                       double* __restrict__ r0, double* __restrict__ p,
                                                       double* __restrict__ v, double* part, KrylovState* ks) {
  double acc[2] = {0.0, 0.0};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += (int64_t)gridDim.x * blockDim.x) {
    const double ri = b[i] - t[i];
    r[i] = ri;
    r0[i] = ri;
    p[i] = 0.0;
    v[i] = 0.0;
    acc[0] += ri * ri;
    acc[1] += b[i] * b[i];
  }
  double tot[2];
  if (grid_reduce<2>(acc, part, &ks->ticket, tot)) {
    ks->rr = tot[0];
    ks->bb = tot[1];
    ks->r0r0 = tot[0];
    ks->alpha = 1.0;
    ks->omega = 1.0;
    ks->rho = 1.0;
    // First iteration: rho_1 = (r0, r) = (r, r); beta multiplies p = 0.
    const double rho_new = tot[0];
    ks->beta = (rho_new / ks->rho) * (ks->alpha / ks->omega);
    ks->rho = rho_new;
    ks->it_chunk = 0;
    ks->restart_r0 = 0;
    ks->stop = 0;
    if (!(tot[0] == tot[0]) || !(tot[1] == tot[1])) ks->stop = 4;
    else if (tot[0] <= ks->tol2) ks->stop = 1;
    else if (ks->chunk_max <= 0) ks->stop = 2;
  }
}

// p = r + beta (p - omega v) (and r0 = r on a restart).
__global__ void __launch_bounds__(kBlock) k_bicg_p(int64_t n4, const double* __restrict__ r, double* __restrict__ r0,
                                                   double* __restrict__ p, const double* __restrict__ v,
                                                   KrylovState* ks) {
  if (ks->stop) return;
  const double beta = ks->beta, omega = ks->omega;
  const int restart = ks->restart_r0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += (int64_t)gridDim.x * blockDim.x) {
    const double ri = r[i];
    if (restart) r0[i] = ri;
    p[i] = ri + beta * (p[i] - omega * v[i]);
  }
}

// v = J^T p with the fused dot (r0, v); epilogue alpha = rho / (r0, v).
template <typename TB>
__global__ void __launch_bounds__(kBlock) k_bicg_jt_v(int64_t nc, const int32_t* __restrict__ jslot, Geom<double> g,
                                                      const int2* __restrict__ ec, const uint8_t* __restrict__ ebc,
                                                      const TB* __restrict__ blk,
                                                      const Vec4<double>* __restrict__ p, Vec4<double>* __restrict__ v,
                                                      const Vec4<double>* __restrict__ r0, double* part,
                                                      KrylovState* ks) {
  if (ks->stop) return;
  double acc[1] = {0.0};
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += (int64_t)gridDim.x * blockDim.x) {
    Vec4<double> y;
    jt_cell<0, TB>(c, nc, jslot, g, ec, ebc, blk, p, y);
    v[c] = y;
    const Vec4<double> q = r0[c];
    acc[0] += q.a * y.a + q.b * y.b + q.c * y.c + q.d * y.d;
  }
  double tot[1];
  if (grid_reduce<1>(acc, part, &ks->ticket, tot)) {
    ks->alpha = ks->rho / tot[0];
    ks->restart_r0 = 0;
    if (!(ks->alpha == ks->alpha) || isinf(ks->alpha)) ks->stop = 3;
  }
}

// s = r - alpha v.
__global__ void __launch_bounds__(kBlock) k_bicg_s(int64_t n4, const double* __restrict__ r,
                                                   const double* __restrict__ v, double* __restrict__ s,
                                                   KrylovState* ks) {
  if (ks->stop) return;
  const double alpha = ks->alpha;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += (int64_t)gridDim.x * blockDim.x)
    s[i] = r[i] - alpha * v[i];
}

// t = J^T shat (shat = M^{-1} s, or s itself without preconditioner) with the
// fused dots (t, t), (t, s); epilogue omega.
template <typename TB>
__global__ void __launch_bounds__(kBlock) k_bicg_jt_t(int64_t nc, const int32_t* __restrict__ jslot, Geom<double> g,
                                                      const int2* __restrict__ ec, const uint8_t* __restrict__ ebc,
                                                      const TB* __restrict__ blk,
                                                      const Vec4<double>* __restrict__ shat,
                                                      const Vec4<double>* __restrict__ s, Vec4<double>* __restrict__ t,
                                                      double* part, KrylovState* ks) {
  if (ks->stop) return;
  double acc[2] = {0.0, 0.0};
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += (int64_t)gridDim.x * blockDim.x) {
    Vec4<double> y;
    jt_cell<0, TB>(c, nc, jslot, g, ec, ebc, blk, shat, y);
    t[c] = y;
    const Vec4<double> q = s[c];
    acc[0] += y.a * y.a + y.b * y.b + y.c * y.c + y.d * y.d;
    acc[1] += y.a * q.a + y.b * q.b + y.c * q.c + y.d * q.d;
  }
  double tot[2];
  if (grid_reduce<2>(acc, part, &ks->ticket, tot)) ks->omega = (tot[0] > 0.0) ? tot[1] / tot[0] : 0.0;
}

// x += alpha phat + omega shat; r = s - omega t; dots (r0, r), (r, r);
// epilogue: convergence test, restart test, next beta.
__global__ void __launch_bounds__(kBlock) k_bicg_xr(int64_t n4, double* __restrict__ x,
                                                    const double* __restrict__ phat, const double* __restrict__ shat,
                                                    const double* __restrict__ s, const double* __restrict__ t,
                                                    double* __restrict__ r, const double* __restrict__ r0,
                                                    double* part, KrylovState* ks) {
  if (ks->stop) return;
  const double alpha = ks->alpha, omega = ks->omega;
  double acc[2] = {0.0, 0.0};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += (int64_t)gridDim.x * blockDim.x) {
    const double si = s[i];
    x[i] = x[i] + alpha * phat[i] + omega * shat[i];
    const double ri = si - omega * t[i];
    r[i] = ri;
    acc[0] += r0[i] * ri;
    acc[1] += ri * ri;
  }
  double tot[2];
  if (grid_reduce<2>(acc, part, &ks->ticket, tot)) {
    ks->it += 1;
    ks->it_chunk += 1;
    ks->rr = tot[1];
    double rho_new = tot[0];
    if (!(tot[1] == tot[1]) || isinf(tot[1])) {
      ks->stop = 4;
    } else if (tot[1] <= ks->tol2) {
      ks->stop = 1;
    } else if (ks->it_chunk >= ks->chunk_max) {
      ks->stop = 2;
    } else {
      if (fabs(rho_new) < kDblEps * kDblEps * ks->r0r0) {
        ks->restart_r0 = 1;
        ks->r0r0 = tot[1];
        rho_new = tot[1];
      }
      if (omega == 0.0) ks->stop = 3;
      ks->beta = (rho_new / ks->rho) * (alpha / omega);
      ks->rho = rho_new;
    }
  }
}

// Grid-reduced dot products of FP64 vectors: out[0] = (a, b), out[1] = (c, d).
__global__ void __launch_bounds__(kBlock) k_dot2(int64_t n, const double* __restrict__ a, const double* __restrict__ b,
                                                 const double* __restrict__ c, const double* __restrict__ d,
                                                 double* part, unsigned int* ticket, double* out) {
  double acc[2] = {0.0, 0.0};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    acc[0] += a[i] * b[i];
    if (c) acc[1] += c[i] * d[i];
  }
  double tot[2];
  if (grid_reduce<2>(acc, part, ticket, tot)) {
    out[0] = tot[0];
    out[1] = tot[1];
  }
}

// out = (lambda, (Rp - Rm) / (2 eps)) -- the lambda^T dR/dtheta term of
// computeShapeGradient (src/shape_optimization.cpp:1004-1014).
template <typename T>
__global__ void __launch_bounds__(kBlock) k_lambda_dR(int64_t nc, const Vec4<double>* __restrict__ lam,
                                                      const Vec4<T>* __restrict__ Rp, const Vec4<T>* __restrict__ Rm,
                                                      double two_eps, double* part, unsigned int* ticket,
                                                      double* out) {
  double acc[1] = {0.0};
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += (int64_t)gridDim.x * blockDim.x) {
    const Vec4<double> l = lam[c];
    const Vec4<T> p = Rp[c], m = Rm[c];
    acc[0] += l.a * (((double)p.a - (double)m.a) / two_eps) + l.b * (((double)p.b - (double)m.b) / two_eps) +
              l.c * (((double)p.c - (double)m.c) / two_eps) + l.d * (((double)p.d - (double)m.d) / two_eps);
  }
  double tot[1];
  if (grid_reduce<1>(acc, part, ticket, tot)) out[0] = tot[0];
}

// ---------------------------------------------------------------------------
// Shape perturbation: applyShapePerturbationNACA12 (src/shape_optimization.cpp:
// 828-890) with yc_naca4 / yt_naca4 (:807-826) and updateDerivedGeometry
// (:748-805).  Wall vertices with xr < 0.9 snap to yc(m',p') + s*yt(t'),
// where s is the side of the camber line of the unperturbed shape.

struct ShapeArgs {
  double pos_x, c, m0, p0, t0;  // unperturbed parameters
  double m1, p1, t1;            // perturbed parameters
};

__device__ __forceinline__ double yc_naca4(double m, double p, double xr) {
  xr = sclamp(xr, 0.0, 1.0);
  if (m == 0.0) return 0.0;
  if (xr <= p) {
    return m / (p * p) * (2.0 * p * xr - xr * xr);
  } else {
    return m / ((1.0 - p) * (1.0 - p)) * ((1.0 - 2.0 * p) + 2.0 * p * xr - xr * xr);
  }
}

__device__ __forceinline__ double yt_naca4(double t, double c, double xr) {
  xr = sclamp(xr, 0.0, 1.0);
  return 5.0 * t * c *
         (0.2969 * sqrt(xr) - 0.1260 * xr - 0.3516 * xr * xr + 0.2843 * xr * xr * xr - 0.1015 * xr * xr * xr * xr);
}

__global__ void k_perturb_vertices(int64_t n, const int32_t* __restrict__ verts, ShapeArgs a,
                                   Vec2<double>* __restrict__ vxy) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int v = verts[i];
  const Vec2<double> pnt = vxy[v];
  const double x_local = pnt.a - a.pos_x;
  const double xr = x_local / a.c;
  if (xr >= 0.9) return;
  const double yc0 = yc_naca4(a.m0, a.p0, xr);
  const double yt1 = yt_naca4(a.t1, a.c, xr);
  const double s = (pnt.b >= yc0) ? +1.0 : -1.0;
  const double yc1 = yc_naca4(a.m1, a.p1, xr);
  Vec2<double> q;
  q.a = a.pos_x + xr * a.c;
  q.b = yc1 + s * yt1;
  vxy[v] = q;
}

// Cell volume and centre from the (moved) vertices (src/shape_optimization.cpp:770-792).
template <typename T>
__global__ void k_perturb_cells(int64_t n, const int32_t* __restrict__ cells, const int32_t* __restrict__ cverts,
                                const uint8_t* __restrict__ ctype, int64_t nc, const Vec2<double>* __restrict__ vxy,
                                double limiter_k, Vec4<T>* __restrict__ cgeom) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = cells[i];
  const Vec2<double> n0 = vxy[cverts[4 * (int64_t)c]], n1 = vxy[cverts[4 * (int64_t)c + 1]],
                     n2 = vxy[cverts[4 * (int64_t)c + 2]];
  double vol, cx, cy;
  if (ctype[c] == 3) {
    const double ax = n1.a - n0.a, ay = n1.b - n0.b, bx = n2.a - n0.a, by = n2.b - n0.b;
    vol = fabs(0.5 * (ax * by - bx * ay));
    cx = 1.0 / 3.0 * (n0.a + n1.a + n2.a);
    cy = 1.0 / 3.0 * (n0.b + n1.b + n2.b);
  } else {
    const Vec2<double> n3 = vxy[cverts[4 * (int64_t)c + 3]];
    const double ax = n1.a - n0.a, ay = n1.b - n0.b, bx = n2.a - n0.a, by = n2.b - n0.b;
    const double qx = n1.a - n2.a, qy = n1.b - n2.b, rx = n3.a - n2.a, ry = n3.b - n2.b;
    vol = 0.5 * (fabs(ax * by - bx * ay) + fabs(qx * ry - rx * qy));
    cx = 0.25 * (n0.a + n1.a + n2.a + n3.a);
    cy = 0.25 * (n0.b + n1.b + n2.b + n3.b);
  }
  const double h = sqrt(vol / 3.14159265358979323846);
  const double k = limiter_k;
  cgeom[c] = v4<T>((T)cx, (T)cy, (T)vol, (T)(k * k * k * h * h * h));
}

// Edge length, normal (toward the left cell's new centre) and centre
// (src/shape_optimization.cpp:760-801).
template <typename T>
__global__ void k_perturb_edges(int64_t n, const int32_t* __restrict__ edges, const int2* __restrict__ ev,
                                const int2* __restrict__ ec, const Vec2<double>* __restrict__ vxy,
                                const Vec4<T>* __restrict__ cgeom, Vec4<T>* __restrict__ egeom,
                                Vec2<T>* __restrict__ ectr) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int e = edges[i];
  const int2 vv = ev[e];
  const Vec2<double> a = vxy[vv.x], b = vxy[vv.y];
  const double tx = a.a - b.a, ty = a.b - b.b, tz = 0.0;
  const double len = sqrt(tx * tx + ty * ty + tz * tz);
  double nx = ty / len, ny = -tx / len;
  const Vec4<T> cl = cgeom[ec[e].x];
  const double ex = 0.5 * (a.a + b.a), ey = 0.5 * (a.b + b.b);
  const double dx = (double)cl.a - ex, dy = (double)cl.b - ey;
  if (dx * nx + dy * ny < 0) {
    nx = -nx;
    ny = -ny;
  }
  egeom[e] = v4<T>((T)nx, (T)ny, (T)len, (T)0);
  Vec2<T> ce;
  ce.a = (T)ex;
  ce.b = (T)ey;
  ectr[e] = ce;
}

// Interpolation weights of the listed vertices, same formulas as the host
// build (valence 3 barycentric in cellIDs order, >= 4 mean value over the
// atan2 order, boundary fans of >= 5 cells inverse distance).
template <typename T>
__global__ void k_vertex_weights(int64_t n, const int32_t* __restrict__ verts, const int32_t* __restrict__ voff,
                                 const int32_t* __restrict__ vcid, const int32_t* __restrict__ vcid_ord,
                                 const uint8_t* __restrict__ vbc, const Vec2<double>* __restrict__ vxy,
                                 const Vec4<T>* __restrict__ cgeom, T* __restrict__ vw) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int v = verts[i];
  const int o = voff[v], nn = voff[v + 1] - o;
  const double px = vxy[v].a, py = vxy[v].b;
  if (nn == 3) {
    const Vec4<T> c0 = cgeom[vcid[o]], c1 = cgeom[vcid[o + 1]], c2 = cgeom[vcid[o + 2]];
    const double c0x = c0.a, c0y = c0.b, c1x = c1.a, c1y = c1.b, c2x = c2.a, c2y = c2.b;
    const double w0_num = (c1x - px) * (c2y - py) - (c2x - px) * (c1y - py);
    const double w0_den = (c1x - c0x) * (c2y - c0y) - (c2x - c0x) * (c1y - c0y);
    const double w0 = (w0_num / w0_den);
    const double w1_num = (c2x - px) * (c0y - py) - (c0x - px) * (c2y - py);
    const double w1 = (w1_num / w0_den);
    vw[o] = (T)w0;
    vw[o + 1] = (T)w1;
    vw[o + 2] = (T)(1 - w0 - w1);
  } else if (nn >= 4) {
    constexpr int kMax = 16;
    if (nn > kMax) return;
    double d[kMax], ux[kMax], uy[kMax], w[kMax];
    for (int k = 0; k < nn; ++k) {
      const Vec4<T> cc = cgeom[vcid_ord[o + k]];
      const double dx = (double)cc.a - px, dy = (double)cc.b - py;
      d[k] = hypot(dx, dy);
      ux[k] = dx / d[k];
      uy[k] = dy / d[k];
    }
    if (nn > 4 && vbc[v] != 0) {
      for (int k = 0; k < nn; ++k) w[k] = 1.0 / d[k];
    } else {
      for (int k = 0; k < nn; ++k) {
        const int km1 = (k + nn - 1) % nn, kp1 = (k + 1) % nn;
        const double cos_prev = sclamp(ux[km1] * ux[k] + uy[km1] * uy[k], -1.0, 1.0);
        const double cos_next = sclamp(ux[k] * ux[kp1] + uy[k] * uy[kp1], -1.0, 1.0);
        w[k] = (tan(0.5 * acos(cos_prev)) + tan(0.5 * acos(cos_next))) / d[k];
      }
    }
    double wsum = 0.0;
    for (int k = 0; k < nn; ++k) wsum += w[k];
    for (int k = 0; k < nn; ++k) vw[o + k] = (T)(w[k] / wsum);
  }
}

// Uniform state fill (init_one_x, src/init.cpp:57-81), on the device.
template <typename T>
__global__ void k_fill_state(int64_t nc, Vec4<T> v, Vec4<T>* __restrict__ U) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c < nc) U[c] = v;
}

// Venkatakrishnan eps = (k h)^3, h = sqrt(V / pi) (src/advection.cpp:214-215).
template <typename T>
__global__ void k_venkat_eps(int64_t nc, double limiter_k, Vec4<T>* __restrict__ cgeom) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  Vec4<T> g = cgeom[c];
  const double h = sqrt((double)g.c / 3.14159265358979323846);
  const double k = limiter_k;
  g.d = (T)(k * k * k * h * h * h);
  cgeom[c] = g;
}

}  // namespace o2f

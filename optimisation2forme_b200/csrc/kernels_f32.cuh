// Kernels of the mixed-precision path (o2f_params.precision = O2F_PREC_F32):
// the residual runs on FP32 copies of the geometry and of the state, while
// the RK3 update accumulates into the FP64 state, and the reductions, forces,
// adjoint Krylov vectors and shape gradient stay FP64.  Compiled in a
// translation unit of its own with multiply-add contraction enabled.
#pragma once

#include "kernels.cuh"

namespace o2f {

// dst[i] = (float)src[i]
__global__ void __launch_bounds__(kBlock) k_narrow(int64_t n, const double* __restrict__ src, float* __restrict__ dst) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = (float)src[i];
}

// dst[i] = (double)src[i]
__global__ void __launch_bounds__(kBlock) k_widen(int64_t n, const float* __restrict__ src, double* __restrict__ dst) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = (double)src[i];
}

// The residual gather of k_cell_residual (src/advection.cpp:439-464 and the
// viscous divergence, src/diffusion.cpp:176-201) in FP32 from the FP32 fluxes.
// Without kRk, R is written widened to FP64.  With kRk, the SSP-RK3 stage
// (src/simulation.cpp:159-167) updates the FP64 state U (and U_old at the
// first stage) with the FP32 residual, refreshes the FP32 shadow U32 and
// writes the block partial sums of R_rho^2 in FP64.  `keep` (may be null)
// receives the FP64 state the stage started from (the last stage's input is
// what the FP64 path linearises about after the loop).
template <bool kRk>
__device__ __forceinline__ double cell_residual_mixed_at(
    int64_t c, int64_t nc, const int32_t* __restrict__ slot, const Geom<float>& g, const Vec4<float>* __restrict__ F,
    const Vec4<float>* __restrict__ etq, const float* __restrict__ etqy, Vec4<float>* __restrict__ U32,
    Vec4<double>* __restrict__ U, Vec4<double>* __restrict__ Uold, Vec4<double>* __restrict__ R, const RkStage& rk,
    const double* dtp, Vec4<double>* __restrict__ keep) {
  double r2 = 0.0;
  const float cv = g.cgeom[c].c;
  int sl[4], nk = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) sl[k] = slot[(int64_t)k * nc + c];
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (sl[k] >= 0 && nk == k) nk = k + 1;
  const Vec4<float> u32 = U32[c];
  const float uu = u32.b / u32.a;
  const float vv = u32.c / u32.a;
  float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (k >= nk) continue;
    const int s = sl[k];
    const int e = s >> 1;
    const float sign = ((s & 1) == 0) ? 1.f : -1.f;
    const Vec4<float> eg = g.egeom[e];
    const Vec4<float> f = F[e];
    a0 += sign * f.a * eg.c;
    a1 += sign * f.b * eg.c;
    a2 += sign * f.c * eg.c;
    a3 += sign * f.d * eg.c;
  }
  const float invV = 1.f / cv;
  a0 *= -invV;
  a1 *= -invV;
  a2 *= -invV;
  a3 *= -invV;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (k >= nk) continue;
    const int s = sl[k];
    const int e = s >> 1;
    const Vec4<float> eg = g.egeom[e];
    const float el = eg.c;
    float enx = eg.a, eny = eg.b;
    if ((s & 1) == 0) {
      enx = -enx;
      eny = -eny;
    }
    const Vec4<float> t = etq[e];
    const float qy = etqy[e];
    a1 += t.a * el * enx / cv + t.c * el * eny / cv;
    a2 += t.c * el * enx / cv + t.b * el * eny / cv;
    a3 += (uu * t.a + vv * t.c - t.d) * el * enx / cv + (uu * t.c + vv * t.b - qy) * el * eny / cv;
  }
  if (!kRk) {
    R[c] = v4<double>(a0, a1, a2, a3);
  } else {
    if (rk.norm_part) r2 = (double)a0 * (double)a0;
    const double dt = *dtp;
    Vec4<double> u = U[c];
    if (keep) keep[c] = u;
    Vec4<double> uo;
    if (rk.snapshot) {
      uo = u;
      Uold[c] = u;
    } else {
      uo = Uold[c];
    }
    u.a = rk.c0 * uo.a + rk.c1 * (u.a + dt * (double)a0);
    u.b = rk.c0 * uo.b + rk.c1 * (u.b + dt * (double)a1);
    u.c = rk.c0 * uo.c + rk.c1 * (u.c + dt * (double)a2);
    u.d = rk.c0 * uo.d + rk.c1 * (u.d + dt * (double)a3);
    U[c] = u;
    U32[c] = v4<float>((float)u.a, (float)u.b, (float)u.c, (float)u.d);
  }
  return r2;
}

template <bool kRk>
__global__ void __launch_bounds__(kBlock) k_cell_residual_mixed(
    int64_t nc, const int32_t* __restrict__ slot, Geom<float> g, const Vec4<float>* __restrict__ F,
    const Vec4<float>* __restrict__ etq, const float* __restrict__ etqy, Vec4<float>* __restrict__ U32,
    Vec4<double>* __restrict__ U, Vec4<double>* __restrict__ Uold, Vec4<double>* __restrict__ R, RkStage rk,
    Vec4<double>* __restrict__ keep, const int* gate) {
  __shared__ double smem[kBlock / 32];
  if (gated(gate)) return;
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double r2 = 0.0;
  if (c < nc) r2 = cell_residual_mixed_at<kRk>(c, nc, slot, g, F, etq, etqy, U32, U, Uold, R, rk, rk.dt, keep);
  if (kRk && rk.norm_part) {
    const double s = block_sum(r2, smem);
    if (threadIdx.x == 0) rk.norm_part[blockIdx.x] = s;
  }
}

}  // namespace o2f

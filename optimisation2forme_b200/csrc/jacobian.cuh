// Consistent adjoint: the Jacobian of the whole residual (reconstruction,
// limiter, HLLC, diffusion, boundary conditions) by coloured central finite
// differences, and the objective's gradient by the same perturbations.  The
// reference linearises only the first-order HLLC flux and the inviscid wall
// pressure (applyJacobianTranspose / assembleAdjointRHS,
// src/shape_optimization.cpp:237-554), so its adjoint is not the adjoint of
// its own residual; this one is, to finite-difference accuracy.
//
// Stencil: R_i depends on U_j for the cells j within two vertex rings of i
// (vertex states, Green-Gauss gradients, limiter, interface states and the
// viscous vertex stresses all reach one vertex ring further), written S(i);
// the relation is symmetric.  Cells are coloured so that no S(i) holds two
// cells of one colour; perturbing every cell of a colour at once then
// leaves, in each R_i, the effect of at most one perturbed cell.
//
// Storage: for every cell j, the blocks J[i][j] = dR_i/dU_j for i in S(j)
// (ascending i), 16 doubles each, row r = component of R, column c =
// component of U.  (J^T x)_j = sum_i J[i][j]^T x_i is a gather over that
// list, in a fixed order.
// Included by solver.cu only (non-template kernels).
#pragma once

#include "kernels_adjoint.cuh"

namespace o2f {

// The gradient phase of the residual with the limiter recorded (kAlpha 1)
// or held (kAlpha 2); the rest of the residual is launched as usual.
template <int kAlpha>
__global__ void __launch_bounds__(kBlock, 3) k_cell_gradient_alpha(
    int64_t nc, const int32_t* __restrict__ slot, Geom<double> g, const int2* __restrict__ ev,
    const int2* __restrict__ ec, const uint8_t* __restrict__ ebc, const Vec4<double>* __restrict__ U,
    const Vec4<double>* __restrict__ vq, Phys ph, Vec4<double>* __restrict__ eL, Vec4<double>* __restrict__ eR,
    Vec4<double>* __restrict__ ctq, double* __restrict__ ctqy, Vec4<double>* __restrict__ alpha) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  cell_gradient_at<double, false, kAlpha>(c, nc, slot, g, ev, ec, ebc, U, vq, ph, eL, eR, ctq, ctqy, nullptr, alpha);
}

struct FjacEps {
  double h;         // relative step
  double floor[4];  // absolute floor per component
};

__device__ __forceinline__ double vcomp(const Vec4<double>& u, int k) {
  return k == 0 ? u.a : k == 1 ? u.b : k == 2 ? u.c : u.d;
}

__device__ __forceinline__ double fjac_eps(const Vec4<double>& u, int k, const FjacEps& e) {
  return e.h * fmax(fabs(vcomp(u, k)), e.floor[k]);
}

// Up[j] = U[j] + sign * eps_jk e_k for the cells of one colour.
__global__ void k_fjac_perturb(int64_t n, const int32_t* __restrict__ cells, const Vec4<double>* __restrict__ U,
                               Vec4<double>* __restrict__ Up, int k, double sign, FjacEps e) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int j = cells[i];
  Vec4<double> u = U[j];
  const double d = sign * fjac_eps(u, k, e);
  if (k == 0) u.a += d;
  else if (k == 1) u.b += d;
  else if (k == 2) u.c += d;
  else u.d += d;
  Up[j] = u;
}

__global__ void k_fjac_restore(int64_t n, const int32_t* __restrict__ cells, const Vec4<double>* __restrict__ U,
                               Vec4<double>* __restrict__ Up) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Up[cells[i]] = U[cells[i]];
}

// Column k of J[i][j] for every i in S(j), j in the colour.
__global__ void k_fjac_extract(int64_t n, const int32_t* __restrict__ cells, const int64_t* __restrict__ off,
                               const int32_t* __restrict__ idx, const Vec4<double>* __restrict__ U,
                               const Vec4<double>* __restrict__ Rp, const Vec4<double>* __restrict__ Rm, int k,
                               FjacEps e, double* __restrict__ blk) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int j = cells[t];
  const double two_eps = 2.0 * fjac_eps(U[j], k, e);
  for (int64_t p = off[j]; p < off[j + 1]; ++p) {
    const int i = idx[p];
    const Vec4<double> a = Rp[i], b = Rm[i];
    double* q = blk + 16 * p + k;
    q[0] = (a.a - b.a) / two_eps;
    q[4] = (a.b - b.b) / two_eps;
    q[8] = (a.c - b.c) / two_eps;
    q[12] = (a.d - b.d) / two_eps;
  }
}

// Per wall edge: its lift and drag coefficients in the objective's sums
// (computeDirectObjectiveTerm, src/shape_optimization.cpp:893-939: pressure
// of the left interface state, wall stresses, edges at x > 1.3 left out).
__global__ void k_fjac_wall_terms(int64_t nwall, const int32_t* __restrict__ wall_edges, Geom<double> g,
                                  const Vec4<double>* __restrict__ eL, const Vec4<double>* __restrict__ etq, Phys ph,
                                  double* __restrict__ tl, double* __restrict__ td) {
  const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= nwall) return;
  const int e = wall_edges[w];
  double l = 0.0, d = 0.0;
  if (!(g.ectr[e].a > 1.3)) {
    const Vec4<double> s = eL[e], eg = g.egeom[e], t = etq[e];
    const double nx = eg.a, ny = eg.b, A = eg.c;
    const double p = (ph.gamma - 1.0) * (s.d - 0.5 * (s.b * s.b + s.c * s.c) / s.a);
    const double Fy = (-p * ny + t.c * nx + t.b * ny) * A;
    const double Fx = (-p * nx + t.a * nx + t.c * ny) * A;
    l = (Fy * ph.cos_a - Fx * ph.sin_a) / ph.q_inf;
    d = (Fx * ph.cos_a + Fy * ph.sin_a) / ph.q_inf;
  }
  tl[w] = l;
  td[w] = d;
}

// Component k of dC_L/dU_j and dC_D/dU_j (objective edges) for the cells of
// the colour: the wall edges whose stencil holds j, in ascending order.
__global__ void k_fjac_grad_extract(int64_t n, const int32_t* __restrict__ cells, const int64_t* __restrict__ woff,
                                    const int32_t* __restrict__ widx, const Vec4<double>* __restrict__ U,
                                    const double* __restrict__ tlp, const double* __restrict__ tdp,
                                    const double* __restrict__ tlm, const double* __restrict__ tdm, int k, FjacEps e,
                                    double* __restrict__ gL, double* __restrict__ gD) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int j = cells[t];
  if (woff[j] == woff[j + 1]) return;
  const double two_eps = 2.0 * fjac_eps(U[j], k, e);
  double sl = 0.0, sd = 0.0;
  for (int64_t q = woff[j]; q < woff[j + 1]; ++q) {
    const int w = widx[q];
    sl += tlp[w] - tlm[w];
    sd += tdp[w] - tdm[w];
  }
  gL[4 * j + k] = sl / two_eps;
  gD[4 * j + k] = sd / two_eps;
}

// b = dJ/dU = -dC_L/dU + beta dC_D/dU.
__global__ void k_fjac_rhs(int64_t n4, const double* __restrict__ gL, const double* __restrict__ gD, double beta,
                           double* __restrict__ b) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n4) b[i] = -gL[i] + beta * gD[i];
}

// ILU(0) input rows of A = J^T from the full Jacobian on the first-order
// pattern: diagonal block J[c][c]^T and, per face neighbour o,
// J[o][c]^T (both in S(c)); the pseudo-time shift as k_ilu_assemble.
__device__ __forceinline__ int64_t fjac_find(const int64_t* __restrict__ off, const int32_t* __restrict__ idx,
                                             int64_t j, int32_t i) {
  int64_t lo = off[j], hi = off[j + 1];
  while (lo < hi) {
    const int64_t mid = (lo + hi) / 2;
    if (idx[mid] < i) lo = mid + 1;
    else hi = mid;
  }
  return (lo < off[j + 1] && idx[lo] == i) ? lo : -1;
}

__global__ void __launch_bounds__(kBlock) k_ilu_assemble_full(int64_t nc, const int64_t* __restrict__ off,
                                                              const int32_t* __restrict__ idx,
                                                              const double* __restrict__ blk, double shift,
                                                              IluDev ilu) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  double* row = ilu.A + c * 80;
  for (int k = 0; k < 5; ++k) {
    double* out = row + 16 * k;
    const int32_t o = k == 0 ? (int32_t)c : ilu.nbr[(int64_t)(k - 1) * nc + c];
    const int64_t p = o >= 0 ? fjac_find(off, idx, c, o) : -1;
    for (int r = 0; r < 4; ++r)
      for (int q = 0; q < 4; ++q) out[r * 4 + q] = p >= 0 ? blk[16 * p + q * 4 + r] : 0.0;
  }
  if (shift > 0.0) {
    double nrm = 0.0;
    for (int r = 0; r < 4; ++r)
      nrm = fmax(nrm, fabs(row[r * 4]) + fabs(row[r * 4 + 1]) + fabs(row[r * 4 + 2]) + fabs(row[r * 4 + 3]));
    for (int r = 0; r < 4; ++r) row[r * 5] += (row[r * 5] < 0.0 ? -shift : shift) * nrm;
  }
}

// y_j = sum over i in S(j) of J[i][j]^T x_i.
__device__ __forceinline__ Vec4<double> fjt_cell(int64_t j, const int64_t* __restrict__ off,
                                                 const int32_t* __restrict__ idx, const double* __restrict__ blk,
                                                 const Vec4<double>* __restrict__ x) {
  double y0 = 0.0, y1 = 0.0, y2 = 0.0, y3 = 0.0;
  for (int64_t p = off[j]; p < off[j + 1]; ++p) {
    const Vec4<double> xi = x[idx[p]];
    const double* q = blk + 16 * p;
    y0 += q[0] * xi.a + q[4] * xi.b + q[8] * xi.c + q[12] * xi.d;
    y1 += q[1] * xi.a + q[5] * xi.b + q[9] * xi.c + q[13] * xi.d;
    y2 += q[2] * xi.a + q[6] * xi.b + q[10] * xi.c + q[14] * xi.d;
    y3 += q[3] * xi.a + q[7] * xi.b + q[11] * xi.c + q[15] * xi.d;
  }
  return v4<double>(y0, y1, y2, y3);
}

__global__ void __launch_bounds__(kBlock) k_fjt_apply(int64_t nc, const int64_t* __restrict__ off,
                                                      const int32_t* __restrict__ idx, const double* __restrict__ blk,
                                                      const Vec4<double>* __restrict__ x, Vec4<double>* __restrict__ y) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j < nc) y[j] = fjt_cell(j, off, idx, blk, x);
}

// The BiCGSTAB steps of k_bicg_jt_v / k_bicg_jt_t with the full operator.
__global__ void __launch_bounds__(kBlock) k_bicg_fjt_v(int64_t nc, const int64_t* __restrict__ off,
                                                       const int32_t* __restrict__ idx, const double* __restrict__ blk,
                                                       const Vec4<double>* __restrict__ p, Vec4<double>* __restrict__ v,
                                                       const Vec4<double>* __restrict__ r0, double* part,
                                                       KrylovState* ks) {
  if (ks->stop) return;
  double acc[1] = {0.0};
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += (int64_t)gridDim.x * blockDim.x) {
    const Vec4<double> y = fjt_cell(c, off, idx, blk, p);
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

__global__ void __launch_bounds__(kBlock) k_bicg_fjt_t(int64_t nc, const int64_t* __restrict__ off,
                                                       const int32_t* __restrict__ idx, const double* __restrict__ blk,
                                                       const Vec4<double>* __restrict__ shat,
                                                       const Vec4<double>* __restrict__ s, Vec4<double>* __restrict__ t,
                                                       double* part, KrylovState* ks) {
  if (ks->stop) return;
  double acc[2] = {0.0, 0.0};
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += (int64_t)gridDim.x * blockDim.x) {
    const Vec4<double> y = fjt_cell(c, off, idx, blk, shat);
    t[c] = y;
    const Vec4<double> q = s[c];
    acc[0] += y.a * y.a + y.b * y.b + y.c * y.c + y.d * y.d;
    acc[1] += y.a * q.a + y.b * q.b + y.c * q.c + y.d * q.d;
  }
  double tot[2];
  if (grid_reduce<2>(acc, part, &ks->ticket, tot)) ks->omega = (tot[0] > 0.0) ? tot[1] / tot[0] : 0.0;
}

}  // namespace o2f

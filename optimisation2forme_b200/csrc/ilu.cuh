// Block ILU(0) preconditioner of the adjoint operator A = J^T, for the
// preconditioned BiCGSTAB (no reference counterpart: the reference runs
// BiCGSTAB with the identity preconditioner, src/shape_optimization.cpp:699,
// which on realistic meshes needs 10^4-10^5 iterations).  The preconditioner
// changes only the convergence path: the solution is the same J^T lambda = b
// at the same true-residual tolerance.
//
// A in block form (4x4 blocks, one row per cell).  From the matrix-free
// product (src/shape_optimization.cpp:433-482), with B_{c,e} the flux
// Jacobian block of edge e on cell c's side and s = -1 for the left cell,
// +1 for the right cell of e:
//   A_cc = sum_e (s_c L_e / V_c) B_{c,e}^T
//   A_co = (s_o L_e / V_o) B_{c,e}^T      (o: the other cell of e)
// Rows are stored as 5 blocks: [0] the diagonal, [1..4] the neighbours in the
// cell's slot order (ilu.nbr[k][c], -1 when absent).
//
// Factorization (IKJ form, rows in a reverse Cuthill-McKee order, each level
// of the dependency DAG processed by one launch): for row i and its lower
// neighbours k in increasing order, L_ik = A_ik D_k^{-1}, then
// A_ij -= L_ik U_kj for every block j of row k above k that row i also holds;
// finally D_i^{-1} is stored.  Solves: forward y_i = r_i - sum_{k<i} L_ik y_k,
// backward z_i = D_i^{-1} (y_i - sum_{j>i} U_ij z_j).
#pragma once

#include "kernels.cuh"

namespace o2f {

__device__ __forceinline__ void mat4_mul(const double* a, const double* b, double* c) {
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int q = 0; q < 4; ++q)
      c[r * 4 + q] = a[r * 4 + 0] * b[0 * 4 + q] + a[r * 4 + 1] * b[1 * 4 + q] + a[r * 4 + 2] * b[2 * 4 + q] +
                     a[r * 4 + 3] * b[3 * 4 + q];
}

// 4x4 inverse by Gauss-Jordan elimination with partial pivoting; returns
// false for a singular block (the inverse is then set to the identity).
__device__ __forceinline__ bool mat4_inv(const double* a_in, double* inv) {
  double a[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    a[i] = a_in[i];
    inv[i] = (i % 5 == 0) ? 1.0 : 0.0;
  }
  for (int col = 0; col < 4; ++col) {
    int piv = col;
    double best = fabs(a[col * 4 + col]);
    for (int r = col + 1; r < 4; ++r) {
      const double v = fabs(a[r * 4 + col]);
      if (v > best) {
        best = v;
        piv = r;
      }
    }
    if (!(best > 0.0)) {
#pragma unroll
      for (int i = 0; i < 16; ++i) inv[i] = (i % 5 == 0) ? 1.0 : 0.0;
      return false;
    }
    if (piv != col) {
      for (int q = 0; q < 4; ++q) {
        double t = a[col * 4 + q];
        a[col * 4 + q] = a[piv * 4 + q];
        a[piv * 4 + q] = t;
        t = inv[col * 4 + q];
        inv[col * 4 + q] = inv[piv * 4 + q];
        inv[piv * 4 + q] = t;
      }
    }
    const double d = 1.0 / a[col * 4 + col];
    for (int q = 0; q < 4; ++q) {
      a[col * 4 + q] *= d;
      inv[col * 4 + q] *= d;
    }
    for (int r = 0; r < 4; ++r) {
      if (r == col) continue;
      const double f = a[r * 4 + col];
      if (f == 0.0) continue;
      for (int q = 0; q < 4; ++q) {
        a[r * 4 + q] -= f * a[col * 4 + q];
        inv[r * 4 + q] -= f * inv[col * 4 + q];
      }
    }
  }
  return true;
}

// Assemble the block rows of A from the Jacobian blocks of k_jt_blocks.
__global__ void __launch_bounds__(kBlock) k_ilu_assemble(int64_t nc, const int32_t* __restrict__ jslot, Geom<double> g,
                                                         const int2* __restrict__ ec,
                                                         const uint8_t* __restrict__ ebc,
                                                         const double* __restrict__ blk, IluDev ilu) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  double* row = ilu.A + c * 80;
  double diag[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) diag[i] = 0.0;
  const double Vc = g.cgeom[c].c;
  for (int k = 0; k < 4; ++k) {
    double* nb = row + 16 * (1 + k);
#pragma unroll
    for (int i = 0; i < 16; ++i) nb[i] = 0.0;
    const int s = jslot[(int64_t)k * nc + c];
    if (s < 0) continue;
    const int e = s >> 1;
    const bool left = (s & 1) == 0;
    const double L = g.egeom[e].c;
    const double* B = blk + (int64_t)e * 32 + (left ? 0 : 16);
    const double sc = (left ? -1.0 : 1.0) * L / Vc;
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int q = 0; q < 4; ++q) diag[r * 4 + q] += sc * B[q * 4 + r];  // B^T
    if (ebc[e] != 0) continue;
    const int2 cc = ec[e];
    const int o = left ? cc.y : cc.x;
    const double so = (left ? 1.0 : -1.0) * L / g.cgeom[o].c;
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int q = 0; q < 4; ++q) nb[r * 4 + q] = so * B[q * 4 + r];
  }
#pragma unroll
  for (int i = 0; i < 16; ++i) row[i] = diag[i];
}

// One level of the factorization.
__global__ void __launch_bounds__(128) k_ilu_factor(const int32_t* __restrict__ cells, int n, IluDev ilu,
                                                    int* status) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int i = cells[t];
  const int64_t nc = ilu.nc;
  double* row = ilu.A + (int64_t)i * 80;
  const int pi = ilu.pos[i];
  int nb[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) nb[k] = ilu.nbr[(int64_t)k * nc + i];
  // lower neighbours in increasing ILU position
  int order[4], nlow = 0;
  for (int k = 0; k < 4; ++k)
    if (nb[k] >= 0 && ilu.pos[nb[k]] < pi) order[nlow++] = k;
  for (int a = 1; a < nlow; ++a)
    for (int b = a; b > 0 && ilu.pos[nb[order[b]]] < ilu.pos[nb[order[b - 1]]]; --b) {
      const int tmp = order[b];
      order[b] = order[b - 1];
      order[b - 1] = tmp;
    }
  double L[16], prod[16];
  for (int a = 0; a < nlow; ++a) {
    const int slot = order[a];
    const int k = nb[slot];
    double* Aik = row + 16 * (1 + slot);
    mat4_mul(Aik, ilu.Dinv + (int64_t)k * 16, L);
#pragma unroll
    for (int q = 0; q < 16; ++q) Aik[q] = L[q];
    // subtract L_ik U_kj for the upper blocks j of row k held by row i
    const double* rowk = ilu.A + (int64_t)k * 80;
    const int pk = ilu.pos[k];
    for (int m = 0; m < 4; ++m) {
      const int j = ilu.nbr[(int64_t)m * nc + k];
      if (j < 0 || ilu.pos[j] <= pk) continue;
      double* dst = nullptr;
      if (j == i) {
        dst = row;
      } else {
        for (int s = 0; s < 4; ++s)
          if (nb[s] == j) dst = row + 16 * (1 + s);
      }
      if (!dst) continue;
      mat4_mul(L, rowk + 16 * (1 + m), prod);
#pragma unroll
      for (int q = 0; q < 16; ++q) dst[q] -= prod[q];
    }
  }
  if (!mat4_inv(row, ilu.Dinv + (int64_t)i * 16)) atomicExch(status, 1);
}

// One forward level: y_i = r_i - sum_{k lower} L_ik y_k.
__global__ void __launch_bounds__(128) k_ilu_lower(const int32_t* __restrict__ cells, int n, IluDev ilu,
                                                   const Vec4<double>* __restrict__ r, Vec4<double>* __restrict__ y,
                                                   const int* gate) {
  if (gated(gate)) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int i = cells[t];
  const int64_t nc = ilu.nc;
  const int pi = ilu.pos[i];
  const double* row = ilu.A + (int64_t)i * 80;
  Vec4<double> acc = r[i];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int o = ilu.nbr[(int64_t)k * nc + i];
    if (o < 0 || ilu.pos[o] > pi) continue;
    const double* Lb = row + 16 * (1 + k);
    const Vec4<double> v = y[o];
    acc.a -= Lb[0] * v.a + Lb[1] * v.b + Lb[2] * v.c + Lb[3] * v.d;
    acc.b -= Lb[4] * v.a + Lb[5] * v.b + Lb[6] * v.c + Lb[7] * v.d;
    acc.c -= Lb[8] * v.a + Lb[9] * v.b + Lb[10] * v.c + Lb[11] * v.d;
    acc.d -= Lb[12] * v.a + Lb[13] * v.b + Lb[14] * v.c + Lb[15] * v.d;
  }
  y[i] = acc;
}

// One backward level: z_i = D_i^{-1} (y_i - sum_{j upper} U_ij z_j); z may alias y.
__global__ void __launch_bounds__(128) k_ilu_upper(const int32_t* __restrict__ cells, int n, IluDev ilu,
                                                   const Vec4<double>* y, Vec4<double>* z, const int* gate) {
  if (gated(gate)) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int i = cells[t];
  const int64_t nc = ilu.nc;
  const int pi = ilu.pos[i];
  const double* row = ilu.A + (int64_t)i * 80;
  Vec4<double> acc = y[i];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int o = ilu.nbr[(int64_t)k * nc + i];
    if (o < 0 || ilu.pos[o] < pi) continue;
    const double* Ub = row + 16 * (1 + k);
    const Vec4<double> v = z[o];
    acc.a -= Ub[0] * v.a + Ub[1] * v.b + Ub[2] * v.c + Ub[3] * v.d;
    acc.b -= Ub[4] * v.a + Ub[5] * v.b + Ub[6] * v.c + Ub[7] * v.d;
    acc.c -= Ub[8] * v.a + Ub[9] * v.b + Ub[10] * v.c + Ub[11] * v.d;
    acc.d -= Ub[12] * v.a + Ub[13] * v.b + Ub[14] * v.c + Ub[15] * v.d;
  }
  const double* D = ilu.Dinv + (int64_t)i * 16;
  Vec4<double> out;
  out.a = D[0] * acc.a + D[1] * acc.b + D[2] * acc.c + D[3] * acc.d;
  out.b = D[4] * acc.a + D[5] * acc.b + D[6] * acc.c + D[7] * acc.d;
  out.c = D[8] * acc.a + D[9] * acc.b + D[10] * acc.c + D[11] * acc.d;
  out.d = D[12] * acc.a + D[13] * acc.b + D[14] * acc.c + D[15] * acc.d;
  z[i] = out;
}

}  // namespace o2f

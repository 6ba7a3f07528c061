// Mesh deformation for a new airfoil shape without re-meshing: the wall
// vertices move by the reference's perturbation formula
// (applyShapePerturbationNACA12, src/shape_optimization.cpp:828-890: the
// k_perturb_vertices kernel), and every interior vertex follows by inverse
// distance weighting of the boundary displacements,
//
//   d(x) = sum_j w_j d_j / sum_j w_j,   w_j = |x - x_j|^-power,
//
// over all boundary vertices j: the wall ones with their displacement and
// the far-field / inlet / outlet ones with zero, so the outer boundary stays
// where it is and the displacement decays away from the wall.  The reference
// has no counterpart (its outer loop re-meshes with Gmsh, run_opti.sh).
//
// Every vertex is one thread; the boundary sources are staged through shared
// memory in tiles of one block, the all-pairs pattern of an N-body step.  The
// sums run over the sources in a fixed order, so the result is deterministic.
// Included by solver.cu only (non-template kernels).
#pragma once

#include "kernels.cuh"

namespace o2f {

constexpr int kIdwTile = 256;  // sources per shared-memory tile == block size

// Positions (old) and displacements (new - old) of the boundary sources.
__global__ void k_idw_sources(int64_t n, const int32_t* __restrict__ src, const Vec2<double>* __restrict__ xy_old,
                              const Vec2<double>* __restrict__ xy_new, Vec2<double>* __restrict__ sxy,
                              Vec2<double>* __restrict__ sd) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int v = src[i];
  const Vec2<double> a = xy_old[v], b = xy_new[v];
  sxy[i] = a;
  Vec2<double> d;
  d.a = b.a - a.a;
  d.b = b.b - a.b;
  sd[i] = d;
}

// |r|^-power from r^2 for an integer power in [1, 8].
__device__ __forceinline__ double idw_weight(double r2, int power) {
  double den = 1.0;
  for (int k = 0; k < power / 2; ++k) den *= r2;
  if (power & 1) den *= sqrt(r2);
  return 1.0 / den;
}

// Interior vertices (vbc == 0): xy_new = xy_old + IDW displacement.  Boundary
// vertices are left as they are in xy_new (the wall already moved).  The
// block size must be kIdwTile; every thread takes part in the tile loads.
__global__ void __launch_bounds__(kIdwTile) k_idw_deform(int64_t nv, const uint8_t* __restrict__ vbc,
                                                         const Vec2<double>* __restrict__ xy_old, int64_t n_src,
                                                         const Vec2<double>* __restrict__ sxy,
                                                         const Vec2<double>* __restrict__ sd, int power,
                                                         Vec2<double>* __restrict__ xy_new) {
  __shared__ Vec2<double> txy[kIdwTile], td[kIdwTile];
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = v < nv && vbc[v] == 0;
  Vec2<double> p;
  p.a = 0.0;
  p.b = 0.0;
  if (active) p = xy_old[v];
  double wsum = 0.0, dx = 0.0, dy = 0.0;
  for (int64_t base = 0; base < n_src; base += kIdwTile) {
    __syncthreads();
    const int64_t j = base + threadIdx.x;
    if (j < n_src) {
      txy[threadIdx.x] = sxy[j];
      td[threadIdx.x] = sd[j];
    }
    __syncthreads();
    const int n = (int)((n_src - base) < kIdwTile ? (n_src - base) : kIdwTile);
    if (active) {
      for (int k = 0; k < n; ++k) {
        const double rx = p.a - txy[k].a, ry = p.b - txy[k].b;
        const double w = idw_weight(rx * rx + ry * ry, power);
        wsum += w;
        dx += w * td[k].a;
        dy += w * td[k].b;
      }
    }
  }
  if (active) {
    Vec2<double> q;
    q.a = p.a + dx / wsum;
    q.b = p.b + dy / wsum;
    xy_new[v] = q;
  }
}

}  // namespace o2f

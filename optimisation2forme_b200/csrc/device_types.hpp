// Device-side data layout shared by the kernels and the host drivers.
//
// Everything on the device is in the Hilbert-renumbered order.  Per entity:
//   cells    U          Vec4<T>  (rho, rho_u, rho_v, E), 32 B (FP64) / 16 B (FP32)
//            cgeom      Vec4<T>  (cx, cy, V, eps_venkat)
//            slot[k]    int32    k < 4, slot-major: 2*edge + side (side 1: the cell
//                                 is the edge's right cell), -1 when unused.  Slot
//                                 order = the reference's Cell::edgeIDs order.
//            jslot[k]   int32    same edges sorted by reference edge id (the
//                                 accumulation order of the reference's
//                                 applyJacobianTranspose at one thread)
//   edges    ev         int2     (v0, v1)
//            ec         int2     (left cell, right cell or -1)
//            ebc        uint8    boundary code
//            egeom      Vec4<T>  (nx, ny, L, unused) -- normal points to the left cell
//            ectr       Vec2<T>  (ex, ey)
//   vertices voff/vcid/vw CSR    interpolation cells and weights (reference order)
//            vbc        uint8
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace o2f {

template <typename T>
struct Vec4;
template <>
struct alignas(32) Vec4<double> {
  double a, b, c, d;
};
template <>
struct alignas(16) Vec4<float> {
  float a, b, c, d;
};

template <typename T>
struct Vec2;
template <>
struct alignas(16) Vec2<double> {
  double a, b;
};
template <>
struct alignas(8) Vec2<float> {
  float a, b;
};

// Viscous quantities are stored as two arrays: (tau_xx, tau_yy, tau_xy, q_x)
// as a Vec4 and q_y alone, which keeps every load aligned and unpadded.

// Geometry that the shape perturbation changes (one copy per perturbed mesh).
template <typename T>
struct Geom {
  Vec4<T>* cgeom;  // [nc] cx, cy, V, eps_venkat
  Vec4<T>* egeom;  // [ne] nx, ny, L, -
  Vec2<T>* ectr;   // [ne] ex, ey
  Vec2<double>* vxy;  // [nv] vertex coordinates (always FP64)
  T* vw;           // [nnz] interpolation weights
};

// Topology (never changes after the build).
struct Topo {
  int64_t nc, ne, nv, nnz;
  int32_t* slot;   // [4*nc]
  int32_t* jslot;  // [4*nc]
  int2* ev;        // [ne]
  int2* ec;        // [ne]
  uint8_t* ebc;    // [ne]
  int32_t* voff;   // [nv+1]
  int32_t* vcid;   // [nnz] (internal cell ids)
  int32_t* vcid_ord;  // [nnz] atan2 order (for weight recomputation)
  uint8_t* vbc;    // [nv]
  int32_t* cverts;   // [4*nc] vertex ids (internal), -1 padded
  uint8_t* ctype;    // [nc] 3 or 4
  int32_t* wall_edges;  // [n_wall] ascending reference edge id
  int64_t n_wall;
  int32_t* wall_cells;  // [n_wall_cells] cells that own wall edges
  int32_t* wall_cell_off;  // [n_wall_cells+1] into wall_cell_edges
  int32_t* wall_cell_edges;  // wall edges of each wall cell, ascending reference id
  int64_t n_wall_cells;
  // shape perturbation sets
  int32_t* pert_verts;  // wall vertices
  int64_t n_pert_verts;
  int32_t* pert_edges;  // edges with a wall code or a wall vertex
  int64_t n_pert_edges;
  int32_t* pert_cells;  // left cells of pert_edges (unique)
  int64_t n_pert_cells;
  int32_t* pert_wverts;  // vertices whose interpolation weights must be recomputed
  int64_t n_pert_wverts;
};

// Freestream and physics constants, computed on the host exactly as the
// reference computes them (src/boundary.cpp:10-17, src/diffusion.cpp:208-210).
struct Phys {
  double gamma, mu, kappa, cp, Pr;
  double fs_rho, fs_rhou, fs_rhov, fs_E;  // freestream conserved state
  double q_inf;                           // 0.5*rho_inf*U_inf^2
  double cos_a, sin_a;                    // lift/drag axes
  double limiter_k;
  int limiter;
};

// Block ILU(0) preconditioner of the adjoint operator (see ilu.cuh).
// State of one sync-free triangular sweep (one per direction): warps take
// 32-row chunks in sweep order from `claim`; the last warp to leave resets
// claim/done for the next launch.
struct SweepSync {
  unsigned int claim;
  unsigned int done;  // warps of the launch that have left
  int err;  // a dependency wait ran past its limit (the sweep's result is invalid)
};

struct IluDev {
  int64_t nc;
  int32_t* nbr;       // [4*nc] neighbour cell of each slot (slot order = jslot order), -1 if none
  int32_t* pos;       // [nc] position of the cell in the ILU order
  int32_t* order;     // [nc] cell at each ILU position (inverse of pos)
  int32_t* sweep;     // [2*nc] processing orders of the forward, then the backward sweep
  int32_t* lev_off;   // [n_lo+1 + n_up+1] level offsets into the forward, then the backward order
  int32_t* rec;       // [2*nc*8] block-sweep records per sweep position (row, dependency positions, slots)
  Vec4<double>* out_f;  // [nc] block sweeps: forward values by forward position
  Vec4<double>* out_b;  // [nc] block sweeps: backward values by backward position
  double* pack;       // block sweeps: factor blocks in sweep order, interleaved over 32 positions (k_ilu_pack)
  double* A;          // [nc*5*16] row blocks (diagonal, then the 4 slots), row-major 4x4
  double* Dinv;       // [nc*16]
  int32_t* lo_cells;  // [nc] factorization levels, concatenated (offsets kept on the host)
  Vec4<double>* tmp;  // [nc] forward sweep's output / backward sweep's input (empty between applications)
  SweepSync* sync;    // [2] forward, backward
  int n_lo;
  int n_up;           // dependency levels of the backward sweep
  long long spin_limit;  // polls a sweep row waits before it gives up (error status)
  int32_t stall_row;     // test hook: this row never releases its forward flag (-1: none)
};

// Buffers written by one residual evaluation.
template <typename T>
struct Work {
  Vec4<T>* vq;      // [nv] vertex states
  Vec4<T>* eL;      // [ne] left interface state
  Vec4<T>* eR;      // [ne] right interface state
  Vec4<T>* ctq;     // [nc] cell tau_xx, tau_yy, tau_xy, q_x
  T* ctqy;          // [nc] cell q_y
  Vec4<T>* vtq;     // [nv] vertex tau/q
  T* vtqy;          // [nv]
  Vec4<T>* F;       // [ne] HLLC flux
  T* etqy;          // [ne]
  Vec4<T>* etq;     // [ne] edge tau/q after the diffusion boundary conditions;
                    // on wall edges this is the stored wall stress of the
                    // reference (src/diffusion.cpp:158-162)
  Vec4<T>* grad;    // [2*nc] (x-gradients, y-gradients), may be null
  Vec4<T>* R;       // [nc]
};

}  // namespace o2f

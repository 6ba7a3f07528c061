// Mixed-precision residual and time loop of the Solver (precision
// O2F_PREC_F32).  The FP32 residual kernels are the FP64 ones instantiated
// for float; this translation unit is compiled with multiply-add contraction.
//
// Data kept in FP32: geometry (cell/edge vectors, interpolation weights), a
// shadow of the state, every per-stage array of the residual, and a copy of
// the adjoint's Jacobian blocks.  Kept in FP64: the state the RK3 stages
// accumulate into, the time-step and norm reductions, and (after a residual)
// the interface states and wall stresses that forces, J, the Jacobian blocks
// and the shape gradient read, widened from FP32.
#include "kernels_f32.cuh"
#include "solver.hpp"

namespace o2f {

namespace {
int grid_of(int64_t n) { return (int)std::min<int64_t>((n + kBlock - 1) / kBlock, 148 * 16); }

template <typename X>
void narrow(const X* src, void* dst, int64_t n_doubles, cudaStream_t s) {
  k_narrow<<<grid_of(n_doubles), kBlock, 0, s>>>(n_doubles, reinterpret_cast<const double*>(src),
                                                 static_cast<float*>(dst));
}

template <typename X>
void widen(const void* src, X* dst, int64_t n, cudaStream_t s) {
  k_widen<<<grid_of(n), kBlock, 0, s>>>(n, static_cast<const float*>(src), reinterpret_cast<double*>(dst));
}
}  // namespace

Work<float> Solver::alloc_work_f32() {
  Work<float> w{};
  w.vq = arena_.alloc<Vec4<float>>(topo_.nv);
  w.eL = arena_.alloc<Vec4<float>>(topo_.ne);
  w.eR = arena_.alloc<Vec4<float>>(topo_.ne);
  w.ctq = arena_.alloc<Vec4<float>>(topo_.nc);
  w.ctqy = arena_.alloc<float>(topo_.nc);
  w.vtq = arena_.alloc<Vec4<float>>(topo_.nv);
  w.vtqy = arena_.alloc<float>(topo_.nv);
  w.F = arena_.alloc<Vec4<float>>(topo_.ne);
  w.etq = arena_.alloc<Vec4<float>>(topo_.ne);
  w.etqy = arena_.alloc<float>(topo_.ne);
  w.grad = nullptr;
  w.R = nullptr;
  return w;
}

// FP32 buffers on first use; the geometry copy is refreshed whenever geom_
// changed (set_params rewrites the limiter eps in cgeom).
void Solver::ensure_f32() {
  const Topo& t = topo_;
  if (!f32_ready_) {
    geom32_.cgeom = arena_.alloc<Vec4<float>>(t.nc);
    geom32_.egeom = arena_.alloc<Vec4<float>>(t.ne);
    geom32_.ectr = arena_.alloc<Vec2<float>>(t.ne);
    geom32_.vxy = geom_.vxy;
    geom32_.vw = arena_.alloc<float>(t.nnz);
    work32_ = alloc_work_f32();
    U32_ = arena_.alloc<Vec4<float>>(t.nc);
    Ukeep_ = arena_.alloc<Vec4<double>>(t.nc);
    f32_ready_ = true;
  }
  if (f32_geom_valid_) return;
  narrow(geom_.cgeom, geom32_.cgeom, 4 * t.nc, stream_);
  narrow(geom_.egeom, geom32_.egeom, 4 * t.ne, stream_);
  narrow(geom_.ectr, geom32_.ectr, 2 * t.ne, stream_);
  narrow(geom_.vw, geom32_.vw, t.nnz, stream_);
  O2F_CUDA(cudaGetLastError());
  f32_geom_valid_ = true;
}

// U32 = (float)U
void Solver::f32_state_sync() {
  narrow(U_, U32_, 4 * topo_.nc, stream_);
  O2F_CUDA(cudaGetLastError());
}

// The FP64 interface states and wall stresses from the FP32 residual's.
void Solver::f32_publish_interfaces() {
  const int64_t ne = topo_.ne;
  widen(work32_.eL, work_.eL, 4 * ne, stream_);
  widen(work32_.eR, work_.eR, 4 * ne, stream_);
  widen(work32_.etq, work_.etq, 4 * ne, stream_);
  widen(work32_.etqy, work_.etqy, ne, stream_);
  O2F_CUDA(cudaGetLastError());
}

void Solver::launch_residual_f32(const int* gate, const void* rkp, Vec4<double>* keep) {
  const Topo& t = topo_;
  const Geom<float>& g = geom32_;
  const Work<float>& w = work32_;
  cudaStream_t s = stream_;
  k_vertex_state<float><<<grid(t.nv), kBlock, 0, s>>>(t.nv, t.voff, t.vcid, g.vw, t.vbc, U32_, phys_, w.vq, gate);
  k_cell_gradient<float, false><<<grid(t.nc), kBlock, 0, s>>>(t.nc, t.slot, g, t.ev, t.ec, t.ebc, U32_, w.vq, phys_,
                                                              w.eL, w.eR, w.ctq, w.ctqy, w.grad, gate);
  k_vertex_visc<float><<<grid(t.nv), kBlock, 0, s>>>(t.nv, t.voff, t.vcid, g.vw, t.vbc, w.ctq, w.ctqy, w.vtq, w.vtqy,
                                                     gate);
  k_edge_flux<float><<<grid(t.ne), kBlock, 0, s>>>(t.ne, g, t.ev, t.ebc, w.eL, w.eR, w.vtq, w.vtqy, phys_, w.F, w.etq,
                                                   w.etqy, gate);
  if (rkp) {
    const RkStage rk = *static_cast<const RkStage*>(rkp);
    k_cell_residual_mixed<true><<<grid(t.nc), kBlock, 0, s>>>(t.nc, t.slot, g, w.F, w.etq, w.etqy, U32_, U_, Uold_,
                                                              work_.R, rk, keep, gate);
  } else {
    k_cell_residual_mixed<false><<<grid(t.nc), kBlock, 0, s>>>(t.nc, t.slot, g, w.F, w.etq, w.etqy, U32_, U_, Uold_,
                                                               work_.R, RkStage{}, nullptr, gate);
  }
  launches_ += 5;
  O2F_CUDA(cudaGetLastError());
}

// FP32 copy of the FP64 Jacobian blocks (the mixed path's J^T products).
void Solver::f32_blocks() {
  if (!blk32_) blk32_ = arena_.alloc<float>(32 * topo_.ne);
  narrow(blk_, blk32_, 32 * topo_.ne, stream_);
  O2F_CUDA(cudaGetLastError());
}

}  // namespace o2f

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
#include "batch.hpp"
#include "batch_device.cuh"
#include "kernels_f32.cuh"
#include "solver.hpp"
#include "step.cuh"

namespace o2f {

// Grouped residual phase of a batch of FP32 contexts (the blocks of a launch
// split into per-candidate ranges by `off`, as kb_phase in
// kernels_batch.cuh), running the same per-entity FP32 functions as
// Solver::launch_residual_f32, so each candidate evolves exactly as in its
// own context.
template <int kPhase, bool kRk>
__global__ void __launch_bounds__(kBatchMaxBlock) kb_phase_mixed(const BatchItem* __restrict__ items, int n,
                                                                 const int* __restrict__ off, int tile, RkStage rk,
                                                                 int keep) {
  __shared__ double smem[kBatchMaxBlock / 32];
  const int i = batch_owner(off, n, blockIdx.x);
  const BatchItem& it = items[i];
  if (*(volatile const int*)&it.st->stop) return;  // uniform over the block: one candidate per block
  const int64_t local = blockIdx.x - off[i];
  const int64_t base = local * blockDim.x * tile + threadIdx.x;
  double r2 = 0.0;
  for (int k = 0; k < tile; ++k) {
    const int64_t x = base + (int64_t)k * blockDim.x;
    if (kPhase == kPhVertexState) {
      if (x < it.t.nv)
        vertex_state_at<float>(x, it.t.nv, it.t.voff, it.t.vcid, it.g32.vw, it.t.vbc, it.U32, it.ph, it.w32.vq);
    } else if (kPhase == kPhCellGradient) {
      if (x < it.t.nc)
        cell_gradient_at<float, false>(x, it.t.nc, it.t.slot, it.g32, it.t.ev, it.t.ec, it.t.ebc, it.U32, it.w32.vq,
                                       it.ph, it.w32.eL, it.w32.eR, it.w32.ctq, it.w32.ctqy, it.w32.grad);
    } else if (kPhase == kPhVertexVisc) {
      if (x < it.t.nv)
        vertex_visc_at<float>(x, it.t.nv, it.t.voff, it.t.vcid, it.g32.vw, it.t.vbc, it.w32.ctq, it.w32.ctqy,
                              it.w32.vtq, it.w32.vtqy);
    } else if (kPhase == kPhEdgeFlux) {
      if (x < it.t.ne)
        edge_flux_at<float>(x, it.t.ne, it.g32, it.t.ev, it.t.ebc, it.w32.eL, it.w32.eR, it.w32.vtq, it.w32.vtqy,
                            it.ph, it.w32.F, it.w32.etq, it.w32.etqy);
    } else if (kPhase == kPhCellResidual) {
      if (x < it.t.nc) {
        RkStage r = rk;
        if (kRk && rk.norm_part) r.norm_part = it.norm_part;
        r2 += cell_residual_mixed_at<kRk>(x, it.t.nc, it.t.slot, it.g32, it.w32.F, it.w32.etq, it.w32.etqy, it.U32,
                                          it.U, it.Uold, it.w.R, r, &it.st->dt, keep ? it.Ukeep : nullptr);
      }
    }
  }
  if (kPhase == kPhCellResidual && kRk && rk.norm_part) {
    const double s = block_sum(r2, smem);
    if (threadIdx.x == 0) it.norm_part[local] = s;
  }
}

void batch_launch_mixed(int phase, bool rk, const RkStage& stage, bool keep, const BatchItem* items, int n,
                        const int* off, int grid, int block, int tile, cudaStream_t s) {
  const int kp = keep ? 1 : 0;
  switch (phase) {
    case kPhVertexState:
      kb_phase_mixed<kPhVertexState, false><<<grid, block, 0, s>>>(items, n, off, tile, stage, kp);
      break;
    case kPhCellGradient:
      kb_phase_mixed<kPhCellGradient, false><<<grid, block, 0, s>>>(items, n, off, tile, stage, kp);
      break;
    case kPhVertexVisc:
      kb_phase_mixed<kPhVertexVisc, false><<<grid, block, 0, s>>>(items, n, off, tile, stage, kp);
      break;
    case kPhEdgeFlux:
      kb_phase_mixed<kPhEdgeFlux, false><<<grid, block, 0, s>>>(items, n, off, tile, stage, kp);
      break;
    case kPhCellResidual:
      if (rk)
        kb_phase_mixed<kPhCellResidual, true><<<grid, block, 0, s>>>(items, n, off, tile, stage, kp);
      else
        kb_phase_mixed<kPhCellResidual, false><<<grid, block, 0, s>>>(items, n, off, tile, stage, kp);
      break;
    default:
      throw Error(O2F_ERR_ARG, "unknown mixed batch phase");
  }
}

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

void Solver::profile_kernel_f32(int k) {
  const Topo& t = topo_;
  const Geom<float>& g = geom32_;
  const Work<float>& w = work32_;
  cudaStream_t s = stream_;
  switch (k) {
    case O2F_K_VERTEX_STATE:
      k_vertex_state<float><<<grid(t.nv), kBlock, 0, s>>>(t.nv, t.voff, t.vcid, g.vw, t.vbc, U32_, phys_, w.vq, nullptr);
      break;
    case O2F_K_CELL_GRADIENT:
      k_cell_gradient<float, false><<<grid(t.nc), kBlock, 0, s>>>(t.nc, t.slot, g, t.ev, t.ec, t.ebc, U32_, w.vq, phys_,
                                                                  w.eL, w.eR, w.ctq, w.ctqy, w.grad, nullptr);
      break;
    case O2F_K_VERTEX_VISC:
      k_vertex_visc<float><<<grid(t.nv), kBlock, 0, s>>>(t.nv, t.voff, t.vcid, g.vw, t.vbc, w.ctq, w.ctqy, w.vtq,
                                                         w.vtqy, nullptr);
      break;
    case O2F_K_EDGE_FLUX:
      k_edge_flux<float><<<grid(t.ne), kBlock, 0, s>>>(t.ne, g, t.ev, t.ebc, w.eL, w.eR, w.vtq, w.vtqy, phys_, w.F,
                                                       w.etq, w.etqy, nullptr);
      break;
    case O2F_K_CELL_RESIDUAL:
      k_cell_residual_mixed<false><<<grid(t.nc), kBlock, 0, s>>>(t.nc, t.slot, g, w.F, w.etq, w.etqy, U32_, U_, Uold_,
                                                                 work_.R, RkStage{}, nullptr, nullptr);
      break;
    default:
      break;
  }
}

// FP32 copy of the FP64 Jacobian blocks (the mixed path's J^T products).
void Solver::f32_blocks() {
  if (!blk32_) blk32_ = arena_.alloc<float>(32 * topo_.ne);
  narrow(blk_, blk32_, 32 * topo_.ne, stream_);
  O2F_CUDA(cudaGetLastError());
}

}  // namespace o2f

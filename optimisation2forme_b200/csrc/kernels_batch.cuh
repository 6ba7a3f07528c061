// Grouped kernels of the batched time loop: one launch per phase advances
// every candidate of a batch.  The blocks of a launch are split into
// per-candidate ranges by an offset table (off[i] .. off[i+1] belong to
// candidate i); inside its range a block covers block * tile consecutive
// entities, each thread `tile` of them, with the same per-entity device
// functions as the single-candidate kernels -- so a candidate's FP64 state
// evolves bit for bit as in its own context.
#pragma once

#include "batch.hpp"
#include "batch_device.cuh"
#include "step.cuh"

namespace o2f {

// Residual phases.  kRk only matters for the cell phase.
template <int kPhase, bool kRk>
__global__ void __launch_bounds__(kBatchMaxBlock) kb_phase(const BatchItem* __restrict__ items, int n,
                                                           const int* __restrict__ off, int tile, RkStage rk) {
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
      if (x < it.t.nv) vertex_state_at<double>(x, it.t.nv, it.t.voff, it.t.vcid, it.g.vw, it.t.vbc, it.U, it.ph, it.w.vq);
    } else if (kPhase == kPhCellGradient) {
      if (x < it.t.nc)
        cell_gradient_at<double, false>(x, it.t.nc, it.t.slot, it.g, it.t.ev, it.t.ec, it.t.ebc, it.U, it.w.vq, it.ph,
                                        it.w.eL, it.w.eR, it.w.ctq, it.w.ctqy, it.w.grad);
    } else if (kPhase == kPhVertexVisc) {
      if (x < it.t.nv)
        vertex_visc_at<double>(x, it.t.nv, it.t.voff, it.t.vcid, it.g.vw, it.t.vbc, it.w.ctq, it.w.ctqy, it.w.vtq,
                               it.w.vtqy);
    } else if (kPhase == kPhEdgeFlux) {
      if (x < it.t.ne)
        edge_flux_at<double>(x, it.t.ne, it.g, it.t.ev, it.t.ebc, it.w.eL, it.w.eR, it.w.vtq, it.w.vtqy, it.ph, it.w.F,
                             it.w.etq, it.w.etqy);
    } else if (kPhase == kPhCellResidual) {
      if (x < it.t.nc) {
        // rk.norm_part only flags the first stage: the partials go to the
        // candidate's own array, the step to the candidate's own dt.
        RkStage r = rk;
        if (kRk && rk.norm_part) r.norm_part = it.norm_part;
        if (kRk) r.dt = &it.st->dt;
        r2 += cell_residual_at<double, kRk>(x, it.t.nc, it.t.slot, it.g, it.w.F, it.w.etq, it.w.etqy, it.U, it.Uold,
                                            it.w.R, r);
      }
    }
  }
  if (kPhase == kPhCellResidual && kRk && rk.norm_part) {
    const double s = block_sum(r2, smem);
    if (threadIdx.x == 0) it.norm_part[local] = s;
  }
}

// Max wave speed of every candidate.
__global__ void __launch_bounds__(kBatchMaxBlock) kb_wave_speed(const BatchItem* __restrict__ items, int n,
                                                                const int* __restrict__ off, int tile) {
  const int i = batch_owner(off, n, blockIdx.x);
  const BatchItem& it = items[i];
  if (*(volatile const int*)&it.st->stop) return;
  const int64_t base = (int64_t)(blockIdx.x - off[i]) * blockDim.x * tile + threadIdx.x;
  double m = 0.0;
  for (int k = 0; k < tile; ++k) {
    const int64_t c = base + (int64_t)k * blockDim.x;
    if (c < it.t.nc) wave_speed_cell(it.U[c], it.ph.gamma, m);
  }
  wave_speed_commit(m, it.st);
}

// Scalar steps: one thread per candidate.
__global__ void kb_step_begin(const BatchItem* __restrict__ items, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) step_begin_at(items[i].st);
}
__global__ void kb_step_dt(const BatchItem* __restrict__ items, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) step_dt_at(items[i].st);
}
__global__ void kb_step_end(const BatchItem* __restrict__ items, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) step_end_at(items[i].st);
}
// One block per candidate.
__global__ void __launch_bounds__(1024) kb_step_norm(const BatchItem* __restrict__ items, int n) {
  const BatchItem& it = items[blockIdx.x];
  if (*(volatile const int*)&it.st->stop) return;
  step_norm_block(it.norm_part, it.nparts, it.hist, it.st);
}

}  // namespace o2f

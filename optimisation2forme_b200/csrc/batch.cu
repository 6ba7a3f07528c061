// Batched time loop: many candidates (each an o2f context with its own mesh
// and flow parameters) advanced together, one grouped launch per phase of an
// SSP-RK3 step for the whole batch, captured in a CUDA graph.  Each
// candidate keeps its own dt, residual history and stop condition, and its
// FP64 state evolves exactly as in its own context's o2f_rk3_run.
//
// Autotuner: for each phase, block size (128/256/512) and entities per
// thread (1/2/4) are timed on the batch itself with CUDA events, and the
// winner is cached per mesh-size bucket (log2 of the batch's cells) for the
// rest of the process.
#include <algorithm>
#include <array>
#include <map>
#include <mutex>

#include "kernels_batch.cuh"

namespace o2f {

namespace {

std::mutex g_tune_mu;
std::map<int, std::array<BatchCfg, kBatchPhases>> g_tuned;  // bucket -> configuration

int bucket_of(int64_t cells) {
  int b = 0;
  while (cells > 1) {
    cells >>= 1;
    ++b;
  }
  return b;
}

}  // namespace

int64_t Batch::entities(int i, int phase) const {
  const Topo& t = s_[i]->topo_;
  switch (phase) {
    case kPhVertexState:
    case kPhVertexVisc:
      return t.nv;
    case kPhEdgeFlux:
      return t.ne;
    default:
      return t.nc;
  }
}

Batch::Batch(std::vector<Solver*> solvers) : s_(std::move(solvers)) {
  if (s_.empty()) throw Error(O2F_ERR_ARG, "empty batch");
  if (s_.size() > 4096) throw Error(O2F_ERR_ARG, "at most 4096 candidates per batch");
  stream_ = s_[0]->stream_;
  for (Solver* s : s_)
    if (!s) throw Error(O2F_ERR_ARG, "null context in the batch");
  f32_ = s_[0]->params_.precision == O2F_PREC_F32;
  for (Solver* s : s_) {
    if (s->params_.precision != s_[0]->params_.precision)
      throw Error(O2F_ERR_ARG, "batched contexts must all use the same precision");
    if (f32_) s->ensure_f32();  // the FP32 buffers the grouped kernels write
    total_cells_ += s->topo_.nc;
  }
  const int n = (int)s_.size();
  items_h_.resize(n);
  for (int i = 0; i < n; ++i) {
    Solver& s = *s_[i];
    BatchItem& it = items_h_[i];
    it.t = s.topo_;
    it.g = s.geom_;
    it.w = s.work_;
    it.U = s.U_;
    it.Uold = s.Uold_;
    it.st = s.step_;
    it.norm_part = arena_.alloc<double>((s.topo_.nc + 127) / 128);  // enough for any block >= 128
    it.hist = nullptr;
    if (f32_) {
      it.g32 = s.geom32_;
      it.w32 = s.work32_;
      it.U32 = s.U32_;
      it.Ukeep = s.Ukeep_;
    }
  }
  items_dev_ = arena_.alloc<BatchItem>(n);
  for (int p = 0; p < kBatchPhases; ++p) off_dev_[p] = arena_.alloc<int>(n + 1);
  std::lock_guard<std::mutex> lock(g_tune_mu);
  auto hit = g_tuned.find(2 * bucket_of(total_cells_) + (f32_ ? 1 : 0));
  for (int p = 0; p < kBatchPhases; ++p) cfg_[p] = hit != g_tuned.end() ? hit->second[p] : BatchCfg{256, 1};
  layout();
}

// Offsets of every phase and the per-candidate partial counts, uploaded.
void Batch::layout() {
  const int n = (int)s_.size();
  for (int p = 0; p < kBatchPhases; ++p) {
    std::vector<int> off(n + 1, 0);
    const int64_t per_block = (int64_t)cfg_[p].block * cfg_[p].tile;
    for (int i = 0; i < n; ++i) {
      const int64_t b = (entities(i, p) + per_block - 1) / per_block;
      if (p == kPhCellResidual) items_h_[i].nparts = (int)b;
      off[i + 1] = off[i] + (int)b;
    }
    blocks_[p] = off[n];
    O2F_CUDA(cudaMemcpyAsync(off_dev_[p], off.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice, stream_));
  }
  upload_items();
}

void Batch::upload_items() {
  for (size_t i = 0; i < s_.size(); ++i) {
    if (s_[i]->params_.precision != (f32_ ? O2F_PREC_F32 : O2F_PREC_F64))
      throw Error(O2F_ERR_ARG, "a batched context changed its precision");
    items_h_[i].ph = s_[i]->phys_;
  }
  O2F_CUDA(cudaMemcpyAsync(items_dev_, items_h_.data(), items_h_.size() * sizeof(BatchItem), cudaMemcpyHostToDevice,
                           stream_));
  O2F_CUDA(cudaStreamSynchronize(stream_));
}

void Batch::launch_phase(int p, bool rk, const RkStage& stage, bool keep) {
  const int n = (int)s_.size();
  const int B = cfg_[p].block, T = cfg_[p].tile, G = blocks_[p];
  if (G == 0) return;
  if (f32_ && p != kPhWave) {
    batch_launch_mixed(p, rk, stage, keep, items_dev_, n, off_dev_[p], G, B, T, stream_);
    ++launches_;
    return;
  }
  switch (p) {
    case kPhVertexState:
      kb_phase<kPhVertexState, false><<<G, B, 0, stream_>>>(items_dev_, n, off_dev_[p], T, stage);
      break;
    case kPhCellGradient:
      kb_phase<kPhCellGradient, false><<<G, B, 0, stream_>>>(items_dev_, n, off_dev_[p], T, stage);
      break;
    case kPhVertexVisc:
      kb_phase<kPhVertexVisc, false><<<G, B, 0, stream_>>>(items_dev_, n, off_dev_[p], T, stage);
      break;
    case kPhEdgeFlux:
      kb_phase<kPhEdgeFlux, false><<<G, B, 0, stream_>>>(items_dev_, n, off_dev_[p], T, stage);
      break;
    case kPhCellResidual:
      if (rk)
        kb_phase<kPhCellResidual, true><<<G, B, 0, stream_>>>(items_dev_, n, off_dev_[p], T, stage);
      else
        kb_phase<kPhCellResidual, false><<<G, B, 0, stream_>>>(items_dev_, n, off_dev_[p], T, stage);
      break;
    case kPhWave:
      kb_wave_speed<<<G, B, 0, stream_>>>(items_dev_, n, off_dev_[p], T);
      break;
    default:
      throw Error(O2F_ERR_ARG, "unknown batch phase");
  }
  ++launches_;
}

void Batch::launch_residual(const RkStage* rk, bool keep) {
  for (int p = kPhVertexState; p <= kPhCellResidual; ++p)
    launch_phase(p, rk != nullptr, rk ? *rk : RkStage{}, keep);
}

// StepState of every candidate for a new loop, as Solver::rk3_run sets it.
void Batch::init_steps(int64_t max_steps, double drop_tol) {
  for (Solver* s : s_) {
    StepState st{};
    st.t = 0.0;
    st.final_time = s->params_.final_time;
    st.cfl = s->params_.cfl_number;
    st.min_h = s->min_h_;
    st.mu = s->params_.viscosity;
    if (s->params_.dt_mode == O2F_DT_THERMAL)
      st.mu = std::max(s->params_.viscosity, s->params_.viscosity * s->params_.cp / s->params_.Pr * (s->params_.gamma - 1.0));
    st.drop_tol = drop_tol;
    st.max_steps = max_steps;
    O2F_CUDA(cudaMemcpyAsync(s->step_, &st, sizeof(st), cudaMemcpyHostToDevice, stream_));
  }
}

void Batch::tune(int reps, int* cfg_out) {
  if (reps <= 0) throw Error(O2F_ERR_ARG, "reps must be positive");
  // Valid inputs for every phase: one residual of each candidate's state,
  // with running step states (the grouped kernels skip stopped candidates).
  init_steps(1, 0.0);
  for (Solver* s : s_) {
    if (f32_) {
      s->ensure_f32();
      s->f32_state_sync();
      s->launch_residual_f32(nullptr, nullptr);
    } else {
      s->launch_residual(s->geom_, s->work_, s->U_, nullptr, false, nullptr);
    }
  }
  static const int kBlocks[] = {128, 256, 512};
  static const int kTiles[] = {1, 2, 4};
  cudaEvent_t e0, e1;
  O2F_CUDA(cudaEventCreate(&e0));
  O2F_CUDA(cudaEventCreate(&e1));
  std::array<BatchCfg, kBatchPhases> best{};
  for (int p = 0; p < kBatchPhases; ++p) {
    float best_ms = 1e30f;
    for (int B : kBlocks)
      for (int T : kTiles) {
        cfg_[p] = BatchCfg{B, T};
        layout();
        launch_phase(p, false, RkStage{});  // warm-up
        O2F_CUDA(cudaEventRecord(e0, stream_));
        for (int r = 0; r < reps; ++r) launch_phase(p, false, RkStage{});
        O2F_CUDA(cudaEventRecord(e1, stream_));
        O2F_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        O2F_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best_ms) {
          best_ms = ms;
          best[p] = cfg_[p];
        }
      }
    cfg_[p] = best[p];
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  layout();
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tuned[2 * bucket_of(total_cells_) + (f32_ ? 1 : 0)] = best;
  }
  for (Solver* s : s_) {
    s->have_residual_ = true;
    s->invalidate_linearisation();
  }
  if (cfg_out)
    for (int p = 0; p < kBatchPhases; ++p) {
      cfg_out[2 * p] = cfg_[p].block;
      cfg_out[2 * p + 1] = cfg_[p].tile;
    }
}

void Batch::rk3_run(int64_t max_steps, double drop_tol, int64_t* steps_done, double* t_out, int* status) {
  NvtxRange nvtx_("o2f batch_rk3_run");
  if (max_steps < 0) throw Error(O2F_ERR_ARG, "max_steps < 0");
  const int n = (int)s_.size();
  if (hist_cap_ < std::max<int64_t>(max_steps, 1)) {
    hist_cap_ = std::max<int64_t>(max_steps, 1);
    for (int i = 0; i < n; ++i) items_h_[i].hist = arena_.alloc<double>(hist_cap_);
  }
  upload_items();  // flow parameters may have changed since the batch was made
  init_steps(max_steps, drop_tol);
  if (f32_)  // FP32 geometry (refreshed if the parameters changed) and state shadow
    for (Solver* s : s_) {
      s->ensure_f32();
      s->f32_state_sync();
    }
  const RkStage s1{0.0, 1.0, nullptr, 1, items_h_[0].norm_part};  // norm_part: flag only
  const RkStage s2{3.0 / 4.0, 1.0 / 4.0, nullptr, 0, nullptr};
  const RkStage s3{1.0 / 3.0, 2.0 / 3.0, nullptr, 0, nullptr};
  const int sgrid = (n + 127) / 128;
  const int kStepsPerGraph = total_cells_ < 200000 ? 16 : 4;
  cudaGraph_t graph;
  cudaGraphExec_t exec;
  O2F_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
  for (int k = 0; k < kStepsPerGraph; ++k) {
    kb_step_begin<<<sgrid, 128, 0, stream_>>>(items_dev_, n);
    launch_phase(kPhWave, false, RkStage{});
    kb_step_dt<<<sgrid, 128, 0, stream_>>>(items_dev_, n);
    launch_residual(&s1);
    kb_step_norm<<<n, 1024, 0, stream_>>>(items_dev_, n);
    launch_residual(&s2);
    launch_residual(&s3, true);
    kb_step_end<<<sgrid, 128, 0, stream_>>>(items_dev_, n);
    launches_ += 4;
  }
  O2F_CUDA(cudaStreamEndCapture(stream_, &graph));
  O2F_CUDA(cudaGraphInstantiate(&exec, graph, 0));
  std::vector<StepState> host(n);
  int64_t launched = 0;
  try {
    while (true) {
      O2F_CUDA(cudaGraphLaunch(exec, stream_));
      launched += kStepsPerGraph;
      if (launched % (kStepsPerGraph * 4) == 0 || launched >= max_steps) {
        for (int i = 0; i < n; ++i)
          O2F_CUDA(cudaMemcpyAsync(&host[i], s_[i]->step_, sizeof(StepState), cudaMemcpyDeviceToHost, stream_));
        O2F_CUDA(cudaStreamSynchronize(stream_));
        bool all = true;
        for (int i = 0; i < n; ++i) all = all && host[i].stop != 0;
        if (all) break;
      }
    }
  } catch (...) {
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    throw;
  }
  cudaGraphExecDestroy(exec);
  cudaGraphDestroy(graph);
  for (int i = 0; i < n; ++i) {
    Solver& s = *s_[i];
    if (steps_done) steps_done[i] = host[i].step;
    if (t_out) t_out[i] = host[i].t;
    if (status) status[i] = host[i].stop == 2 ? O2F_ERR_NONFINITE : O2F_OK;
    // FP32 contexts: the linearisation's FP64 interface states about the
    // last stage's input state, as Solver::rk3_run leaves them.
    if (f32_ && host[i].step > 0) s.launch_residual(s.geom_, s.work_, s.Ukeep_, nullptr, false, nullptr);
    s.have_residual_ = host[i].step > 0;
    s.invalidate_linearisation();
  }
  if (f32_) O2F_CUDA(cudaStreamSynchronize(stream_));
}

void Batch::history(int i, double* out, int64_t count) {
  if (i < 0 || i >= (int)s_.size()) throw Error(O2F_ERR_ARG, "candidate index out of range");
  if (count < 0 || count > hist_cap_ || !items_h_[i].hist) throw Error(O2F_ERR_ARG, "history count out of range");
  if (count == 0) return;
  O2F_CUDA(cudaMemcpyAsync(out, items_h_[i].hist, count * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  O2F_CUDA(cudaStreamSynchronize(stream_));
}

}  // namespace o2f

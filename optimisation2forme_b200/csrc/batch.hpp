// Batched time loop over several contexts (batch.cu).
#pragma once

#include <vector>

#include "solver.hpp"

namespace o2f {

struct StepState;
struct RkStage;

// Device view of one candidate (one Solver context) for the grouped kernels.
struct BatchItem {
  Topo t;
  Geom<double> g;
  Work<double> w;
  Phys ph;
  Vec4<double>* U;
  Vec4<double>* Uold;
  StepState* st;
  double* norm_part;  // per-block partial sums of R_rho^2 (the batch's own array)
  double* hist;       // residual history (the batch's own array)
  int nparts;         // blocks of this candidate in the stage-1 cell phase
  // FP32 contexts (mixed precision): FP32 geometry, residual buffers and
  // state shadow, and the FP64 input state of the last RK3 stage
  Geom<float> g32;
  Work<float> w32;
  Vec4<float>* U32;
  Vec4<double>* Ukeep;
};

// Phases of one RK3 stage plus the wave-speed reduction, each one grouped
// launch over the batch.
enum BatchPhase { kPhVertexState = 0, kPhCellGradient, kPhVertexVisc, kPhEdgeFlux, kPhCellResidual, kPhWave };
constexpr int kBatchPhases = 6;

// One grouped launch of a residual phase (kPhVertexState .. kPhCellResidual)
// over a batch of FP32 contexts: the FP32 per-entity functions of their own
// Solver::rk3_run, in a translation unit compiled like theirs (solver_f32.cu).
// keep: the cell phase stores each candidate's FP64 input state in Ukeep.
struct RkStage;
void batch_launch_mixed(int phase, bool rk, const RkStage& stage, bool keep, const BatchItem* items, int n,
                        const int* off, int grid, int block, int tile, cudaStream_t stream);

struct BatchCfg {
  int block;  // threads per block: 128, 256 or 512
  int tile;   // entities per thread: 1, 2 or 4
};

class Batch {
 public:
  explicit Batch(std::vector<Solver*> solvers);
  void tune(int reps, int* cfg_out);
  void rk3_run(int64_t max_steps, double drop_tol, int64_t* steps_done, double* t_out, int* status);
  void history(int i, double* out, int64_t count);
  int size() const { return (int)s_.size(); }
  int64_t launches() const { return launches_; }

 private:
  int64_t entities(int i, int phase) const;
  void layout();
  void upload_items();
  void init_steps(int64_t max_steps, double drop_tol);
  void launch_phase(int phase, bool rk, const RkStage& stage, bool keep = false);
  void launch_residual(const RkStage* rk, bool keep = false);

  std::vector<Solver*> s_;
  cudaStream_t stream_ = nullptr;
  DeviceArena arena_;
  std::vector<BatchItem> items_h_;
  BatchItem* items_dev_ = nullptr;
  BatchCfg cfg_[kBatchPhases]{};
  int* off_dev_[kBatchPhases]{};
  int blocks_[kBatchPhases]{};
  int64_t total_cells_ = 0;
  bool f32_ = false;  // the contexts run the mixed-precision residual
  int64_t hist_cap_ = 0;
  int64_t launches_ = 0;
};

}  // namespace o2f

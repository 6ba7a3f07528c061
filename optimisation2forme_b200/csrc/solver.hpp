// The solver context behind the C ABI: device-resident renumbered mesh, state,
// interface states of the last residual, adjoint vectors and all scratch.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "device_types.hpp"
#include "mesh_host.hpp"
#include "o2f.h"

namespace o2f {

struct KrylovState;
struct StepState;

// NVTX range over a host stage (residual, time loop, adjoint, gradient,
// Jacobian builds, mesh updates, images): named spans for Nsight tools; a
// no-op when no tool is attached (NVTX v3 is header-only).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// A mesh beyond what the GPU topology build handles (a vertex with more
// cells than the set emulation); the host build takes it.
struct TopologyLimit : Error {
  using Error::Error;
};

// Meshes from this many cells up build their topology on the GPU.
constexpr int64_t kGpuTopologyCells = 100000;

void cuda_check(cudaError_t e, const char* what);

// Physical constants of the kernels from the parameters: freestream (rotated
// by the angle of attack), diffusivities, limiter.
Phys phys_of(const o2f_params& p);

// Array forms of the reference's per-edge / per-state functions (pointwise.cu).
void hllc_points(int64_t n, const double* LR_host, const double* normal_host, double gamma, double* flux_host);
void bc_points(int kind, const o2f_params& p, int64_t n, const uint8_t* codes_host, double* inout_host,
               double* out_host);
#define O2F_CUDA(x) ::o2f::cuda_check((x), #x)

// Owning device allocation list.
class DeviceArena {
 public:
  ~DeviceArena();
  template <typename X>
  X* alloc(size_t n) {
    return static_cast<X*>(raw(n * sizeof(X)));
  }
  void* raw(size_t bytes);
  size_t bytes() const { return bytes_; }

 private:
  std::vector<void*> ptrs_;
  size_t bytes_ = 0;
};

class Batch;

class Solver {
  friend class Batch;  // the batched time loop drives the context's device state (batch.cu)

 public:
  Solver(const o2f_mesh_desc& desc, const o2f_params& p, cudaStream_t stream);
  ~Solver();

  void set_params(const o2f_params& p);
  o2f_mesh_info info() const;
  int64_t export_array(const std::string& which, void* out) const;

  void state_set(const double* U_ref);
  void state_get(double* U_ref);
  void state_freestream();
  double* state_device() { return reinterpret_cast<double*>(U_); }
  void cell_permutation(int64_t* new_of_old) const;

  void residual(double* R_ref);
  void debug_get(const std::string& which, double* out);
  void rk3_run(int64_t max_steps, double drop_tol, double* history, int64_t* steps_done, double* t_out);
  void forces(double beta, double* out3);
  void jt_apply(const double* x_ref, double* y_ref);
  void adjoint_rhs(double beta, double* b_ref);
  void adjoint_solve(double beta, double tol, int64_t max_iter, int64_t restart, double* lambda_ref,
                     int64_t* iters, double* relres, const double* guess_ref = nullptr,
                     const double* rhs_ref = nullptr);
  void shape_gradient(const o2f_shape_params& sp, const int* ids, int n, double beta, double eps,
                      const double* lambda_ref, double* grad);
  void debug_perturbed(const o2f_shape_params& sp, int id, double eps, const std::string& which, double* out);
  void profile_kernels(int reps, double* ms_out);
  void residual_norm_noalloc(double* norm_out);  // noalloc.cu
  // New vertex coordinates (reference order) for the same topology: the
  // geometry is rebuilt as for a fresh context on those coordinates.
  void set_vertex_coords(const double* xy_ref);
  // Wall to the shape `to` by the perturbation formula, interior by inverse
  // distance weighting of the boundary displacements (deform.cuh).
  void deform_shape(const o2f_shape_params& from, const o2f_shape_params& to, int power);
  // Headless image of a cell field (render.cuh); rgb: nx*ny*3 bytes, top row first.
  void render_field(const std::string& field, int nx, int ny, const std::string& cmap, const double* range_in,
                    unsigned char* rgb, double* range_out);
  double last_residual_ms() const { return last_residual_ms_; }
  int64_t launches() const { return launches_; }

 private:
  void upload_mesh();
  void upload_geometry();
  void compute_phys();
  // alpha_mode 1 / 2: record / hold the limiter values in fjac_alpha_
  // (the frozen-limiter linearisation); 0 everywhere else.
  void launch_residual(const Geom<double>& g, const Work<double>& w, Vec4<double>* U, const int* gate,
                       bool write_grad, const void* rk, int alpha_mode = 0);
  void build_jt_blocks();
  // Both linearisations (first-order blocks, full Jacobian) belong to the
  // state, geometry and parameters they were built for.
  void invalidate_linearisation() {
    blk_valid_ = false;
    fjac_valid_ = false;
  }
  // consistent adjoint (jacobian.cuh)
  bool full_jac() const { return params_.adjoint_jacobian != O2F_JAC_REFERENCE; }
  void setup_full_jacobian();
  void build_full_jacobian();
  void jt_apply_dev(const Vec4<double>* x, Vec4<double>* y);
  void perturbed_geometry(const o2f_shape_params& sp, int id, double eps);
  void ensure_pert_buffers();
  Work<double> alloc_work();
  // mixed precision (solver_f32.cu)
  bool f32() const { return params_.precision == O2F_PREC_F32; }
  // FP32 Jacobian blocks in the Krylov products (FP64 true residuals)
  bool mixed_adjoint() const { return f32() || params_.adjoint_precision == O2F_PREC_F32; }
  Work<float> alloc_work_f32();
  void ensure_f32();
  void f32_state_sync();
  void f32_publish_interfaces();
  void launch_residual_f32(const int* gate, const void* rk, Vec4<double>* keep = nullptr);
  void profile_kernel_f32(int k);  // one launch of residual kernel class k (O2F_K_*) in FP32
  void f32_blocks();
  void to_internal(const double* ref, Vec4<double>* dev);
  void to_reference(const Vec4<double>* dev, double* ref);
  void sync();
  int grid(int64_t n) const { return (int)((n + 255) / 256); }

  cudaStream_t stream_ = nullptr;
  bool own_stream_ = false;
  o2f_params params_{};
  Phys phys_{};
  HostMesh hm_;
  double min_h_ = 0.0;
  std::vector<int64_t> cperm_, cinv_, eperm_, einv_, vperm_, vinv_;
  std::vector<int32_t> wall_edges_host_;
  DeviceArena arena_;
  Topo topo_{};
  Geom<double> geom_{};
  Work<double> work_{};
  Vec4<double>* U_ = nullptr;
  Vec4<double>* Uold_ = nullptr;
  bool f32_ready_ = false;
  bool f32_geom_valid_ = false;
  Geom<float> geom32_{};
  Work<float> work32_{};
  Vec4<float>* U32_ = nullptr;
  Vec4<double>* Ukeep_ = nullptr;  // mixed path: input state of the last RK3 stage
  float* blk32_ = nullptr;
  double* norm_part_ = nullptr;
  StepState* step_ = nullptr;
  double* hist_dev_ = nullptr;
  int64_t hist_cap_ = 0;
  // adjoint
  double* blk_ = nullptr;
  bool blk_valid_ = false;
  bool have_residual_ = false;
  bool have_lambda_ = false;
  Vec4<double>*lam_ = nullptr, *b_ = nullptr, *r_ = nullptr, *r0_ = nullptr, *p_ = nullptr, *v_ = nullptr,
  *s_ = nullptr, *t_ = nullptr, *tmp_ = nullptr;
  KrylovState* ks_ = nullptr;
  double* part_ = nullptr;
  unsigned int* ticket_ = nullptr;
  double* scal_ = nullptr;  // small device scalars
  // block ILU(0) preconditioner of the adjoint
  void setup_ilu_host(const std::vector<int32_t>& jslot, const std::vector<int2>& ec,
                      const std::vector<uint8_t>& ebc);
  void ilu_factor();
  void ilu_apply(const Vec4<double>* r, Vec4<double>* z, const int* gate);
  void ilu_check_sweeps();

 public:
  void debug_ilu_stall(int stall, long long spin_limit);

 private:
  std::vector<int32_t> ilu_nbr_h_, ilu_pos_h_, ilu_order_h_, lo_off_h_, lo_cells_h_, ilu_sweep_h_;
  int ilu_n_up_ = 0;  // levels of the backward sweep's dependencies
  std::vector<int32_t> ilu_lev_off_h_, ilu_rec_h_;
  bool ilu_waiting_ = false;  // test hook: use the sweeps that wait on other rows
  IluDev ilu_{};
  bool ilu_alloc_ = false;
  int* ilu_status_ = nullptr;
  Vec4<double>*phat_ = nullptr, *shat_ = nullptr;
  // shape perturbation
  Geom<double> pgeom_{};
  Work<double> pwork_{};
  Vec4<double>* Rp_ = nullptr;
  bool pert_alloc_ = false;
  // consistent adjoint: stencil S(j) (device order), colours, blocks, dC/dU
  bool fjac_setup_ = false, fjac_valid_ = false;
  int64_t fjac_nnzb_ = 0;
  int64_t *fjac_off_ = nullptr, *fjac_woff_ = nullptr;
  int32_t *fjac_idx_ = nullptr, *fjac_ccells_ = nullptr, *fjac_widx_ = nullptr;
  std::vector<int64_t> fjac_coff_h_;
  double *fjac_blk_ = nullptr, *fjac_gL_ = nullptr, *fjac_gD_ = nullptr;
  double *fjac_tlp_ = nullptr, *fjac_tdp_ = nullptr, *fjac_tlm_ = nullptr, *fjac_tdm_ = nullptr;
  Vec4<double>*fjac_Up_ = nullptr, *fjac_Rp_ = nullptr, *fjac_alpha_ = nullptr;
  // mesh deformation
  bool deform_alloc_ = false;
  int64_t n_idw_src_ = 0;
  int32_t* idw_src_ = nullptr;
  Vec2<double>*idw_sxy_ = nullptr, *idw_sd_ = nullptr, *dvxy_ = nullptr;
  // field images
  int32_t* render_ref_id_ = nullptr;
  double *render_scalar_ = nullptr, *render_part_ = nullptr;
  double last_residual_ms_ = 0.0;
  int64_t launches_ = 0;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
  void* mailbox_ = nullptr;  // pinned host copy of StepState / KrylovState
};

}  // namespace o2f

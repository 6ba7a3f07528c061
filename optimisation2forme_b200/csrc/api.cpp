// extern "C" entry points of include/o2f.h.  Every call translates C++
// exceptions into an o2f_status and a per-thread message (the reference
// reports errors as std::invalid_argument / std::runtime_error,
// src/boundary.cpp:90, src/shape_optimization.cpp:724-731, src/utils.cpp:35-105).
#include <cstring>
#include <exception>
#include <ios>
#include <memory>
#include <string>
#include <vector>

#include "batch.hpp"
#include "checkpoint.hpp"
#include "mesh_host.hpp"
#include "mlp.hpp"
#include "o2f.h"
#include "solver.hpp"

struct o2f_ctx {
  std::unique_ptr<o2f::Solver> solver;
};

struct o2f_host_mesh {
  o2f::HostMesh mesh;
};

struct o2f_batch {
  std::unique_ptr<o2f::Batch> batch;
};

struct o2f_mlp {
  std::unique_ptr<o2f::mlp::Mlp> net;
};

namespace {

thread_local std::string g_last_error;

template <typename F>
int guarded(F&& f) {
  try {
    f();
    g_last_error.clear();
    return O2F_OK;
  } catch (const o2f::Error& e) {
    g_last_error = e.what();
    return e.code;
  } catch (const std::ios_base::failure& e) {
    g_last_error = e.what();
    return O2F_ERR_IO;
  } catch (const std::invalid_argument& e) {
    g_last_error = e.what();
    return O2F_ERR_ARG;
  } catch (const std::bad_alloc&) {
    g_last_error = "host out of memory";
    return O2F_ERR_INTERNAL;
  } catch (const std::exception& e) {
    g_last_error = std::string("internal error: ") + e.what();
    return O2F_ERR_INTERNAL;
  } catch (...) {
    g_last_error = "unknown internal error";
    return O2F_ERR_INTERNAL;
  }
}

o2f::Solver& S(o2f_ctx* c) {
  if (!c || !c->solver) throw o2f::Error(O2F_ERR_ARG, "null context");
  return *c->solver;
}

const o2f::Solver& S(const o2f_ctx* c) {
  if (!c || !c->solver) throw o2f::Error(O2F_ERR_ARG, "null context");
  return *c->solver;
}

void need(const void* p, const char* what) {
  if (!p) throw o2f::Error(O2F_ERR_ARG, std::string("null ") + what);
}

}  // namespace

extern "C" {

const char* o2f_last_error(void) { return g_last_error.c_str(); }

const char* o2f_version(void) { return "o2f-b200 0.1 (sm_100a)"; }

void o2f_params_default(o2f_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  // SimulationParams defaults (include/params.hpp:24-53) after finalize().
  p->gamma = 1.4;
  p->viscosity = 1e-6;
  p->Pr = 0.71;
  p->cp = 1005.0;
  p->cfl_number = 0.1;
  p->final_time = 5.0;
  p->inflow_velocity = 1.0;
  p->rho_ref = 1.225;
  p->p_ref = 101325.0;
  p->aoa_deg = 0.0;
  p->limiter_k = 1e-2;  // k_eps of computeVenkatAlpha (src/advection.cpp:209)
  p->adjoint_shift = 0.0;
  p->limiter = O2F_LIMITER_VENKAT;
  p->precision = O2F_PREC_F64;
  p->adjoint_precond = O2F_PRECOND_ILU0;
  p->dt_mode = O2F_DT_REFERENCE;
  p->verbosity = 0;
  p->adjoint_jacobian = O2F_JAC_REFERENCE;
  p->adjoint_fd_step = 1e-9;
  p->adjoint_precision = O2F_PREC_F64;
  p->adjoint_sweeps = O2F_SWEEPS_AUTO;
}

int o2f_host_mesh_create(const o2f_mesh_desc* mesh, o2f_host_mesh** out) {
  return guarded([&] {
    need(mesh, "mesh");
    need(out, "out");
    *out = nullptr;
    auto m = std::make_unique<o2f_host_mesh>();
    try {
      m->mesh = o2f::build_mesh(*mesh);
    } catch (const std::invalid_argument&) {
      throw;
    } catch (const std::runtime_error& e) {
      throw o2f::Error(O2F_ERR_MESH, e.what());
    }
    *out = m.release();
  });
}

int o2f_host_mesh_from_msh(const char* path, o2f_host_mesh** out) {
  return guarded([&] {
    need(path, "path");
    need(out, "out");
    *out = nullptr;
    o2f::MshData d = o2f::read_msh2(path);
    o2f_mesh_desc desc = d.desc();
    auto m = std::make_unique<o2f_host_mesh>();
    try {
      m->mesh = o2f::build_mesh(desc);
    } catch (const std::invalid_argument&) {
      throw;
    } catch (const std::ios_base::failure&) {
      throw;
    } catch (const std::runtime_error& e) {
      throw o2f::Error(O2F_ERR_MESH, e.what());
    }
    *out = m.release();
  });
}

int o2f_host_mesh_create_gpu(const o2f_mesh_desc* mesh, void* stream, o2f_host_mesh** out) {
  return guarded([&] {
    need(mesh, "mesh");
    need(out, "out");
    *out = nullptr;
    auto m = std::make_unique<o2f_host_mesh>();
    try {
      m->mesh = o2f::build_mesh_gpu(*mesh, stream);
    } catch (const std::invalid_argument&) {
      throw;
    } catch (const o2f::Error&) {
      throw;
    } catch (const std::runtime_error& e) {
      throw o2f::Error(O2F_ERR_MESH, e.what());
    }
    *out = m.release();
  });
}

int o2f_host_mesh_export(const o2f_host_mesh* mesh, const char* which, void* out, int64_t* count) {
  return guarded([&] {
    need(mesh, "mesh");
    need(which, "which");
    const int64_t n = o2f::export_mesh_array(mesh->mesh, which, out);
    if (count) *count = n;
  });
}

int o2f_host_mesh_destroy(o2f_host_mesh* mesh) {
  return guarded([&] { delete mesh; });
}

int o2f_host_mesh_set_coords(o2f_host_mesh* mesh, const double* node_xy) {
  return guarded([&] {
    need(mesh, "mesh");
    need(node_xy, "node_xy");
    try {
      o2f::set_coordinates(mesh->mesh, node_xy);
    } catch (const std::invalid_argument&) {
      throw;
    } catch (const std::runtime_error& e) {
      throw o2f::Error(O2F_ERR_MESH, e.what());
    }
  });
}

int o2f_checkpoint_write(const char* path, int64_t n_cells, const double* U_host, double time, int64_t steps) {
  return guarded([&] {
    need(path, "path");
    need(U_host, "U");
    o2f::checkpoint_write(path, n_cells, U_host, time, steps);
  });
}

int o2f_checkpoint_read(const char* path, int64_t n_cells, double* U_host, double* time, int64_t* steps) {
  return guarded([&] {
    need(path, "path");
    need(U_host, "U");
    o2f::checkpoint_read(path, n_cells, U_host, time, steps);
  });
}

int o2f_create(const o2f_mesh_desc* mesh, const o2f_params* params, void* stream, o2f_ctx** out) {
  return guarded([&] {
    need(mesh, "mesh");
    need(params, "params");
    need(out, "out");
    *out = nullptr;
    auto ctx = std::make_unique<o2f_ctx>();
    ctx->solver = std::make_unique<o2f::Solver>(*mesh, *params, static_cast<cudaStream_t>(stream));
    *out = ctx.release();
  });
}

int o2f_create_from_msh(const char* path, const o2f_params* params, void* stream, o2f_ctx** out) {
  return guarded([&] {
    need(path, "path");
    need(params, "params");
    need(out, "out");
    *out = nullptr;
    o2f::MshData d = o2f::read_msh2(path);
    o2f_mesh_desc desc = d.desc();
    auto ctx = std::make_unique<o2f_ctx>();
    ctx->solver = std::make_unique<o2f::Solver>(desc, *params, static_cast<cudaStream_t>(stream));
    *out = ctx.release();
  });
}

int o2f_destroy(o2f_ctx* ctx) {
  return guarded([&] { delete ctx; });
}

int o2f_set_params(o2f_ctx* ctx, const o2f_params* params) {
  return guarded([&] {
    need(params, "params");
    S(ctx).set_params(*params);
  });
}

int o2f_get_info(const o2f_ctx* ctx, o2f_mesh_info* info) {
  return guarded([&] {
    need(info, "info");
    *info = S(ctx).info();
  });
}

int o2f_mesh_export(const o2f_ctx* ctx, const char* which, void* out, int64_t* count) {
  return guarded([&] {
    need(which, "which");
    const int64_t n = S(ctx).export_array(which, out);
    if (count) *count = n;
  });
}

int o2f_state_set(o2f_ctx* ctx, const double* U_host) {
  return guarded([&] {
    need(U_host, "U");
    S(ctx).state_set(U_host);
  });
}

int o2f_state_get(o2f_ctx* ctx, double* U_host) {
  return guarded([&] {
    need(U_host, "U");
    S(ctx).state_get(U_host);
  });
}

int o2f_state_freestream(o2f_ctx* ctx) {
  return guarded([&] { S(ctx).state_freestream(); });
}

int o2f_residual(o2f_ctx* ctx, double* R_host) {
  return guarded([&] { S(ctx).residual(R_host); });
}

int o2f_debug_get(o2f_ctx* ctx, const char* which, double* out_host) {
  return guarded([&] {
    need(which, "which");
    need(out_host, "out");
    S(ctx).debug_get(which, out_host);
  });
}

int o2f_rk3_run(o2f_ctx* ctx, int64_t max_steps, double drop_tol, double* history_host, int64_t* steps_done,
                double* t_out) {
  return guarded([&] { S(ctx).rk3_run(max_steps, drop_tol, history_host, steps_done, t_out); });
}

int o2f_forces(o2f_ctx* ctx, double beta, double* forces_out) {
  return guarded([&] {
    need(forces_out, "forces_out");
    S(ctx).forces(beta, forces_out);
  });
}

int o2f_jt_apply(o2f_ctx* ctx, const double* x_host, double* y_host) {
  return guarded([&] {
    need(x_host, "x");
    need(y_host, "y");
    S(ctx).jt_apply(x_host, y_host);
  });
}

int o2f_adjoint_rhs(o2f_ctx* ctx, double beta, double* b_host) {
  return guarded([&] {
    need(b_host, "b");
    S(ctx).adjoint_rhs(beta, b_host);
  });
}

int o2f_adjoint_solve(o2f_ctx* ctx, double beta, double tol, int64_t max_iter, int64_t restart, double* lambda_host,
                      int64_t* iters, double* relres) {
  return guarded([&] { S(ctx).adjoint_solve(beta, tol, max_iter, restart, lambda_host, iters, relres); });
}

int o2f_adjoint_solve_guess(o2f_ctx* ctx, double beta, double tol, int64_t max_iter, int64_t restart,
                            const double* lambda0_host, double* lambda_host, int64_t* iters, double* relres) {
  return guarded([&] {
    need(lambda0_host, "lambda0");
    S(ctx).adjoint_solve(beta, tol, max_iter, restart, lambda_host, iters, relres, lambda0_host);
  });
}

int o2f_adjoint_solve_rhs(o2f_ctx* ctx, const double* rhs_host, double tol, int64_t max_iter, int64_t restart,
                          const double* lambda0_host, double* lambda_host, int64_t* iters, double* relres) {
  return guarded([&] {
    need(rhs_host, "rhs");
    S(ctx).adjoint_solve(0.0, tol, max_iter, restart, lambda_host, iters, relres, lambda0_host, rhs_host);
  });
}

int o2f_shape_gradient(o2f_ctx* ctx, const o2f_shape_params* shape, const int* param_ids, int n_params, double beta,
                       double eps, const double* lambda_host, double* grad_out) {
  return guarded([&] {
    need(shape, "shape");
    S(ctx).shape_gradient(*shape, param_ids, n_params, beta, eps, lambda_host, grad_out);
  });
}

int o2f_optimize_shape(o2f_ctx* ctx, const o2f_shape_params* shape, const int* param_ids, int n_params, double beta,
                       double eps, double tol, double* grad_out, double* out) {
  return guarded([&] {
    need(shape, "shape");
    need(out, "out");
    o2f::Solver& s = S(ctx);
    double f[3];
    s.forces(beta, f);  // J from the interface states left by the last residual (:1039)
    int64_t iters = 0;
    double relres = 0.0;
    s.adjoint_solve(beta, tol, 100000, 500, nullptr, &iters, &relres);
    s.shape_gradient(*shape, param_ids, n_params, beta, eps, nullptr, grad_out);
    out[0] = f[2];
    out[1] = (double)iters;
    out[2] = relres;
  });
}

int o2f_debug_perturbed(o2f_ctx* ctx, const o2f_shape_params* shape, int param_id, double eps, const char* which,
                        double* out_host) {
  return guarded([&] {
    need(shape, "shape");
    need(which, "which");
    need(out_host, "out");
    S(ctx).debug_perturbed(*shape, param_id, eps, which, out_host);
  });
}

int o2f_state_device(o2f_ctx* ctx, double** U_dev) {
  return guarded([&] {
    need(U_dev, "U_dev");
    *U_dev = S(ctx).state_device();
  });
}

int o2f_cell_permutation(const o2f_ctx* ctx, int64_t* new_of_old_host) {
  return guarded([&] {
    need(new_of_old_host, "out");
    S(ctx).cell_permutation(new_of_old_host);
  });
}

int o2f_profile_kernels(o2f_ctx* ctx, int reps, double* ms_out) {
  return guarded([&] {
    need(ms_out, "ms_out");
    S(ctx).profile_kernels(reps, ms_out);
  });
}

int o2f_batch_create(o2f_ctx* const* ctxs, int n, o2f_batch** out) {
  return guarded([&] {
    need(ctxs, "ctxs");
    need(out, "out");
    *out = nullptr;
    if (n <= 0) throw o2f::Error(O2F_ERR_ARG, "a batch needs at least one context");
    std::vector<o2f::Solver*> v;
    for (int i = 0; i < n; ++i) v.push_back(&S(ctxs[i]));
    auto b = std::make_unique<o2f_batch>();
    b->batch = std::make_unique<o2f::Batch>(std::move(v));
    *out = b.release();
  });
}

int o2f_batch_destroy(o2f_batch* batch) {
  return guarded([&] { delete batch; });
}

namespace {
o2f::Batch& B(o2f_batch* b) {
  if (!b || !b->batch) throw o2f::Error(O2F_ERR_ARG, "null batch");
  return *b->batch;
}
}  // namespace

int o2f_batch_tune(o2f_batch* batch, int reps, int* config_out) {
  return guarded([&] { B(batch).tune(reps, config_out); });
}

int o2f_batch_rk3_run(o2f_batch* batch, int64_t max_steps, double drop_tol, int64_t* steps_done, double* t_out,
                      int* status_out) {
  return guarded([&] { B(batch).rk3_run(max_steps, drop_tol, steps_done, t_out, status_out); });
}

int o2f_batch_launches(o2f_batch* batch, int64_t* launches) {
  return guarded([&] {
    need(launches, "launches");
    *launches = B(batch).launches();
  });
}

int o2f_batch_history(o2f_batch* batch, int index, double* history_host, int64_t count) {
  return guarded([&] {
    need(history_host, "history");
    B(batch).history(index, history_host, count);
  });
}

namespace {
o2f::mlp::Mlp& N(o2f_mlp* m) {
  if (!m || !m->net) throw o2f::Error(O2F_ERR_ARG, "null network");
  return *m->net;
}
}  // namespace

int o2f_mlp_create(int max_batch, float freq_scale, uint64_t seed, void* stream, o2f_mlp** out) {
  return guarded([&] {
    need(out, "out");
    *out = nullptr;
    auto m = std::make_unique<o2f_mlp>();
    m->net = std::make_unique<o2f::mlp::Mlp>(max_batch, freq_scale, seed, static_cast<cudaStream_t>(stream));
    *out = m.release();
  });
}

int o2f_mlp_destroy(o2f_mlp* net) {
  return guarded([&] { delete net; });
}

int o2f_mlp_n_params(o2f_mlp* net, int64_t* n) {
  return guarded([&] {
    need(n, "n");
    *n = N(net).n_params();
  });
}

int o2f_mlp_set_data(o2f_mlp* net, const float* inputs, const float* targets, int64_t n) {
  return guarded([&] {
    need(inputs, "inputs");
    need(targets, "targets");
    N(net).set_data(inputs, targets, n);
  });
}

int o2f_mlp_train(o2f_mlp* net, int steps, int batch, float lr, uint64_t seed, float* loss_history) {
  return guarded([&] { N(net).train(steps, batch, lr, seed, loss_history); });
}

int o2f_mlp_predict(o2f_mlp* net, const float* inputs, int64_t n, float* outputs) {
  return guarded([&] {
    need(inputs, "inputs");
    need(outputs, "outputs");
    N(net).predict(inputs, n, outputs);
  });
}

int o2f_mlp_gradients(o2f_mlp* net, const float* inputs, const float* targets, int n, float* grads, float* loss) {
  return guarded([&] {
    need(inputs, "inputs");
    need(targets, "targets");
    need(grads, "grads");
    N(net).gradients(inputs, targets, n, grads, loss);
  });
}

int o2f_mlp_get_params(o2f_mlp* net, float* params, float* freq) {
  return guarded([&] {
    need(params, "params");
    N(net).get_params(params, freq);
  });
}

int o2f_mlp_set_params(o2f_mlp* net, const float* params) {
  return guarded([&] {
    need(params, "params");
    N(net).set_params(params);
  });
}

int o2f_hllc_flux(int64_t n, const double* LR_host, const double* normal_host, double gamma, double* flux_host) {
  return guarded([&] {
    if (n > 0) {
      need(LR_host, "LR_host");
      need(normal_host, "normal_host");
      need(flux_host, "flux_host");
    }
    o2f::hllc_points(n, LR_host, normal_host, gamma, flux_host);
  });
}

int o2f_bc_states(const o2f_params* params, int64_t n, const uint8_t* codes, double* U_host) {
  return guarded([&] {
    need(params, "params");
    if (n > 0) {
      need(codes, "codes");
      need(U_host, "U_host");
    }
    o2f::bc_points(0, *params, n, codes, U_host, nullptr);
  });
}

int o2f_bc_ghosts(const o2f_params* params, int64_t n, const uint8_t* codes, const double* L_host, double* R_host) {
  return guarded([&] {
    need(params, "params");
    if (n > 0) {
      need(codes, "codes");
      need(L_host, "L_host");
      need(R_host, "R_host");
    }
    std::vector<double> L(L_host, L_host + 4 * std::max<int64_t>(n, 0));
    o2f::bc_points(1, *params, n, codes, L.data(), R_host);
  });
}

int o2f_bc_diffusion(int64_t n, const uint8_t* codes, double* tq_host) {
  return guarded([&] {
    if (n > 0) {
      need(codes, "codes");
      need(tq_host, "tq_host");
    }
    o2f_params p;
    o2f_params_default(&p);
    o2f::bc_points(2, p, n, codes, tq_host, nullptr);
  });
}

int o2f_debug_ilu_stall(o2f_ctx* ctx, int stall, int64_t spin_limit) {
  return guarded([&] { S(ctx).debug_ilu_stall(stall, (long long)spin_limit); });
}

int o2f_residual_norm_noalloc(o2f_ctx* ctx, double* norm_out) {
  return guarded([&] {
    need(norm_out, "norm_out");
    S(ctx).residual_norm_noalloc(norm_out);
  });
}

int o2f_set_vertex_coords(o2f_ctx* ctx, const double* node_xy) {
  return guarded([&] {
    need(node_xy, "node_xy");
    S(ctx).set_vertex_coords(node_xy);
  });
}

int o2f_deform_shape(o2f_ctx* ctx, const o2f_shape_params* from, const o2f_shape_params* to, int power) {
  return guarded([&] {
    need(from, "from");
    need(to, "to");
    S(ctx).deform_shape(*from, *to, power);
  });
}

int o2f_render_field(o2f_ctx* ctx, const char* field, int nx, int ny, const char* cmap, const double* range_in,
                     uint8_t* rgb_out, double* range_out) {
  return guarded([&] {
    need(field, "field");
    need(rgb_out, "rgb_out");
    S(ctx).render_field(field, nx, ny, cmap ? cmap : "", range_in, rgb_out, range_out);
  });
}

int o2f_get_timing(const o2f_ctx* ctx, o2f_timing* t) {
  return guarded([&] {
    need(t, "timing");
    t->residual_ms = S(ctx).last_residual_ms();
    t->kernel_launches = S(ctx).launches();
  });
}

}  // extern "C"

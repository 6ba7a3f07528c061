// Array entry points of the reference's per-edge and per-state functions:
// the HLLC flux of edges given their interface states, and the three
// boundary-condition functions.  The reference calls them one edge or one
// state at a time from its loops; here a call takes n of them and evaluates
// them on the GPU with the same device functions as the residual kernels
// (compiled without multiply-add contraction, so each value has the
// reference's bits).
#include "kernels.cuh"
#include "solver.hpp"

namespace o2f {
namespace {

__global__ void k_hllc_points(int64_t n, const double* __restrict__ LR, const double* __restrict__ nrm, double gamma,
                              double* __restrict__ F) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* q = LR + 8 * i;
  const Vec4<double> L = v4<double>(q[0], q[1], q[2], q[3]), R = v4<double>(q[4], q[5], q[6], q[7]);
  const Vec4<double> f = hllc(L, R, nrm[2 * i], nrm[2 * i + 1], gamma);
  F[4 * i] = f.a;
  F[4 * i + 1] = f.b;
  F[4 * i + 2] = f.c;
  F[4 * i + 3] = f.d;
}

// kind 0: apply_boundary_conditions on U in place; 1: the ghost right state
// of apply_InterfaceStates_boundary_conditions from the left state in U,
// written to out; 2: apply_diffusion_bc on 5 values per entry in place.
__global__ void k_bc_points(int kind, int64_t n, const uint8_t* __restrict__ codes, Phys ph, double* __restrict__ U,
                            double* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint8_t code = codes[i];
  if (kind == 0) {
    double* q = U + 4 * i;
    bc_state(code, ph, q[0], q[1], q[2], q[3]);
  } else if (kind == 1) {
    const double* q = U + 4 * i;
    const Vec4<double> r = bc_ghost(code, ph, v4<double>(q[0], q[1], q[2], q[3]));
    out[4 * i] = r.a;
    out[4 * i + 1] = r.b;
    out[4 * i + 2] = r.c;
    out[4 * i + 3] = r.d;
  } else {
    if (code == 'f' || code == 'w')
      for (int k = 0; k < 5; ++k) U[5 * i + k] = 0.0;
  }
}

// Device copies of the call's arrays, freed on every exit path.
struct DevBuf {
  void* p = nullptr;
  explicit DevBuf(size_t bytes) {
    if (bytes) O2F_CUDA(cudaMalloc(&p, bytes));
  }
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  template <typename X>
  X* as() const {
    return static_cast<X*>(p);
  }
};

int grid_of(int64_t n) { return (int)((n + 255) / 256); }

}  // namespace

void hllc_points(int64_t n, const double* LR_host, const double* normal_host, double gamma, double* flux_host) {
  if (n < 0) throw Error(O2F_ERR_ARG, "n < 0");
  if (n == 0) return;
  DevBuf lr(8 * n * sizeof(double)), nr(2 * n * sizeof(double)), f(4 * n * sizeof(double));
  O2F_CUDA(cudaMemcpy(lr.p, LR_host, 8 * n * sizeof(double), cudaMemcpyHostToDevice));
  O2F_CUDA(cudaMemcpy(nr.p, normal_host, 2 * n * sizeof(double), cudaMemcpyHostToDevice));
  k_hllc_points<<<grid_of(n), 256>>>(n, lr.as<double>(), nr.as<double>(), gamma, f.as<double>());
  O2F_CUDA(cudaGetLastError());
  O2F_CUDA(cudaMemcpy(flux_host, f.p, 4 * n * sizeof(double), cudaMemcpyDeviceToHost));
}

void bc_points(int kind, const o2f_params& p, int64_t n, const uint8_t* codes_host, double* inout_host,
               double* out_host) {
  if (n < 0) throw Error(O2F_ERR_ARG, "n < 0");
  if (n == 0) return;
  const int w = kind == 2 ? 5 : 4;
  DevBuf c(n), u(w * n * sizeof(double)), o(kind == 1 ? 4 * n * sizeof(double) : 0);
  O2F_CUDA(cudaMemcpy(c.p, codes_host, n, cudaMemcpyHostToDevice));
  O2F_CUDA(cudaMemcpy(u.p, inout_host, w * n * sizeof(double), cudaMemcpyHostToDevice));
  k_bc_points<<<grid_of(n), 256>>>(kind, n, c.as<uint8_t>(), phys_of(p), u.as<double>(), o.as<double>());
  O2F_CUDA(cudaGetLastError());
  if (kind == 1)
    O2F_CUDA(cudaMemcpy(out_host, o.p, 4 * n * sizeof(double), cudaMemcpyDeviceToHost));
  else
    O2F_CUDA(cudaMemcpy(inout_host, u.p, w * n * sizeof(double), cudaMemcpyDeviceToHost));
}

}  // namespace o2f

// o2f_residual_norm_noalloc: the residual of the current state and
// ||R_rho||_2, with no device allocation on the call path.
//
// Who needs it: a host that drives the residual every step of its own
// time loop cannot afford cudaMalloc there (it synchronises the whole
// device and can stall on the allocator), and a host that hands this
// library a fixed device-memory budget, or owns all device memory through
// its own pool, cannot let a call allocate at all.
//
// This is a variant of the time loop's norm reduction (k_cell_residual's
// per-block partial sums of R_rho^2, folded by k_step_norm), whose partial
// sums live in context memory.  Here the reduction's scratch -- a completion
// ticket, the result slot and the per-block partial sums -- is one file-scope
// static device array of kNormScratchBytes (33,280 bytes), so the call needs
// neither cudaMalloc nor any allocating library routine; the residual itself
// runs in the context's buffers, allocated when the context was created.
//
// What must start at zero: the ticket.  A static device array is zeroed when
// the module is loaded, and the last block of every launch resets the ticket
// to zero before it exits.  The partial sums and the result are written
// before they are read and need no initial value.
//
// The scratch is shared by every context on the same device: calls that
// overlap on one device (two host threads, or two streams) race on it and
// give wrong results.  Serialise them.
//
// Set-up: the scratch address is looked up with cudaGetSymbolAddress once
// per device, on the first call made with that device current, and cached.
// That first call therefore does set-up work; make it before any stream
// capture.  The cached address belongs to the device's context at that
// time: after a cudaDeviceReset (or any reset of the primary context) it is
// stale, so a process that resets a device must not call this entry point
// on that device again.
//
// Precision: the residual is the one o2f_residual computes for the context
// (FP64, or in an FP32 context the FP32 residual with FP64 R); the norm is
// always reduced in FP64.
#include <cmath>
#include <mutex>
#include <string>

#include "solver.hpp"

namespace o2f {
namespace {

constexpr int kNormBlock = 256;
constexpr int kNormCellsPerThread = 16;
constexpr int64_t kNormCellsPerBlock = (int64_t)kNormBlock * kNormCellsPerThread;
constexpr int kNormMaxParts = 4096;
constexpr int64_t kNormMaxCells = kNormCellsPerBlock * kNormMaxParts;  // 16,777,216
// Layout: [0, 4) ticket, [256, 264) result, [512, 512 + 8 * kNormMaxParts) partial sums.
constexpr size_t kNormTicketOff = 0, kNormResultOff = 256, kNormPartOff = 512;
constexpr size_t kNormScratchBytes = kNormPartOff + sizeof(double) * kNormMaxParts;

static __device__ __align__(256) unsigned char g_norm_scratch[kNormScratchBytes];

struct NormScratch {
  unsigned int* ticket;
  double* result;
  double* part;
};

// One partial sum of R_rho^2 per block over kNormCellsPerBlock consecutive
// cells; the last block to finish folds the partials in block order, writes
// sqrt of the total and resets the ticket.
__global__ void __launch_bounds__(kNormBlock) k_rrho_norm_noalloc(const Vec4<double>* __restrict__ R, int64_t nc,
                                                                  NormScratch sc) {
  __shared__ double sm[kNormBlock / 32];
  __shared__ bool last;
  const int64_t base = (int64_t)blockIdx.x * kNormCellsPerBlock;
  double s = 0.0;
  for (int k = 0; k < kNormCellsPerThread; ++k) {
    const int64_t c = base + (int64_t)k * kNormBlock + threadIdx.x;
    if (c < nc) {
      const double a = R[c].a;
      s += a * a;
    }
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = 0.0;
    for (int w = 0; w < kNormBlock / 32; ++w) b += sm[w];
    sc.part[blockIdx.x] = b;
    __threadfence();
    last = atomicAdd(sc.ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double v = 0.0;
  for (unsigned int i = threadIdx.x; i < gridDim.x; i += kNormBlock) v += __ldcg(sc.part + i);
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int w = 0; w < kNormBlock / 32; ++w) tot += sm[w];
    *sc.result = sqrt(tot);
    *sc.ticket = 0u;
  }
}

constexpr int kMaxDevices = 64;
std::mutex g_norm_mu;
unsigned char* g_norm_addr[kMaxDevices] = {};

// Address of g_norm_scratch on the current device (looked up once per device).
NormScratch norm_scratch() {
  int dev = -1;
  O2F_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) throw Error(O2F_ERR_CUDA, "o2f_residual_norm_noalloc: device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_norm_mu);
  if (!g_norm_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_norm_scratch);
    if (e != cudaSuccess || p == nullptr)
      throw Error(O2F_ERR_CUDA, std::string("o2f_residual_norm_noalloc: cudaGetSymbolAddress failed: ") +
                                    cudaGetErrorString(e));
    g_norm_addr[dev] = static_cast<unsigned char*>(p);
  }
  unsigned char* b = g_norm_addr[dev];
  return NormScratch{reinterpret_cast<unsigned int*>(b + kNormTicketOff), reinterpret_cast<double*>(b + kNormResultOff),
                     reinterpret_cast<double*>(b + kNormPartOff)};
}

}  // namespace

void Solver::residual_norm_noalloc(double* norm_out) {
  const int64_t nc = topo_.nc;
  if (nc > kNormMaxCells)
    throw Error(O2F_ERR_ARG, "o2f_residual_norm_noalloc: " + std::to_string(nc) +
                                 " cells exceed the static scratch limit of 16777216 cells");
  const NormScratch sc = norm_scratch();
  if (f32()) {
    // As o2f_residual in an FP32 context: FP32 residual, FP64 R and the
    // widened interface states.  Its buffers come from the context's first
    // FP32 residual or time loop, which this call may not allocate.
    if (!f32_ready_)
      throw Error(O2F_ERR_STATE,
                  "o2f_residual_norm_noalloc: an FP32 context needs one o2f_residual or o2f_rk3_run first "
                  "(it allocates the FP32 buffers)");
    ensure_f32();
    f32_state_sync();
    launch_residual_f32(nullptr, nullptr);
    f32_publish_interfaces();
  } else {
    launch_residual(geom_, work_, U_, nullptr, true, nullptr);
  }
  have_residual_ = true;
  invalidate_linearisation();
  const int blocks = (int)((nc + kNormCellsPerBlock - 1) / kNormCellsPerBlock);
  k_rrho_norm_noalloc<<<blocks, kNormBlock, 0, stream_>>>(work_.R, nc, sc);
  O2F_CUDA(cudaGetLastError());
  launches_ += 1;
  O2F_CUDA(cudaMemcpyAsync(norm_out, sc.result, sizeof(double), cudaMemcpyDeviceToHost, stream_));
  sync();
}

}  // namespace o2f

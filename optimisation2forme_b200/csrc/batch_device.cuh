// Device helpers shared by the grouped batch kernels of both precisions
// (kernels_batch.cuh: FP64 contexts; solver_f32.cu: FP32 contexts).
#pragma once

namespace o2f {

constexpr int kBatchMaxBlock = 512;

// Candidate owning block b: the last i with off[i] <= b.
__device__ __forceinline__ int batch_owner(const int* __restrict__ off, int n, int b) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= b) lo = mid; else hi = mid - 1;
  }
  return lo;
}

}  // namespace o2f

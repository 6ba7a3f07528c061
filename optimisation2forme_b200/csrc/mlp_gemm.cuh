// BF16 GEMM on the 5th-generation tensor cores (tcgen05) for the warm-start
// network: D[M x N] = sum_k A(m, k) B(n, k), BF16 operands staged in shared
// memory, FP32 accumulators in tensor memory (TMEM), fused epilogues.
//
// One CTA of 128 threads computes a 128 x NT tile (NT = 256 or 16).  Warp 0
// allocates NT TMEM columns; every K chunk of 64 is copied from global memory
// into the K-major canonical layout without swizzle (8 x 16-byte core
// matrices: element (r, k) of a chunk at ((k/8)*(rows/8) + r/8)*128 +
// (r%8)*16 + (k%8)*2 bytes), one elected thread issues four
// tcgen05.mma.kind::f16 (M = 128, N = NT, K = 16) and commits them to an
// mbarrier, and all threads wait (bounded) before the next chunk reuses the
// buffers.  The epilogue reads the accumulator rows of each warp's TMEM lane
// quarter with tcgen05.ld.  A and B are read through (row, k) element strides,
// so transposed operands (the weight gradients) need no extra copy.
//
// Descriptor bit layouts come from CUTLASS's cute/arch/mma_sm100_desc.hpp.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

#include <cute/arch/mma_sm100_desc.hpp>

namespace o2f {
namespace mlp {

using bf16 = __nv_bfloat16;

constexpr int kTileM = 128;
constexpr int kKC = 64;          // K elements per shared-memory chunk
constexpr int kGemmThreads = 128;
constexpr long long kWaitLimit = 1ll << 26;  // mbarrier polls before giving up

enum Epilogue : int {
  kEpiHidden = 0,   // z = acc + bias -> pre (bf16), act = silu(z) (bf16)
  kEpiLinear = 1,   // out32 = acc + bias (fp32)
  kEpiBackAct = 2,  // out = bf16(acc * silu'(zprev))
  kEpiAtomic = 3,   // out32 += acc (fp32 atomics; split-K weight gradients)
};

struct GemmArgs {
  int M, N, K;
  const bf16* A;
  int64_t sam, sak;  // A(m, k) = A[m*sam + k*sak]
  const bf16* B;
  int64_t sbn, sbk;  // B(n, k) = B[n*sbn + k*sbk]
  int k_split;       // K elements per blockIdx.z slice (multiple of kKC)
  int epi;
  const float* bias;  // [N] or null
  bf16* out;          // kEpiHidden: activation; kEpiBackAct: gradient
  bf16* pre;          // kEpiHidden: pre-activation
  const bf16* zprev;  // kEpiBackAct: pre-activation of the layer below
  int64_t ldo;        // row stride of out / pre / zprev / out32
  float* out32;       // kEpiLinear / kEpiAtomic
  int* err;           // set when a wait exceeds its limit
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ float silu(float z) { return z / (1.f + expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
  const float s = 1.f / (1.f + expf(-z));
  return s * (1.f + z * (1.f - s));
}

// Shared-memory matrix descriptor of one K=16 slice of a chunk with `rows`
// rows (K-major, no swizzle): leading byte offset = the distance between the
// two 8-element K groups, stride byte offset = the distance between 8-row
// groups.
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t chunk_addr, int rows, int kk) {
  cute::UMMA::SmemDescriptor d;
  d.version_ = 1;
  d.lbo_mode_ = 0;
  d.base_offset_ = 0;
  d.layout_type_ = uint8_t(cute::UMMA::LayoutType::SWIZZLE_NONE);
  const uint32_t group_bytes = (uint32_t)(rows / 8) * 128u;  // one 8-element K group of all rows
  d.start_address_ = (uint16_t)((chunk_addr + (uint32_t)(2 * kk) * group_bytes) >> 4);
  d.leading_byte_offset_ = (uint16_t)(group_bytes >> 4);
  d.stride_byte_offset_ = (uint16_t)(128u >> 4);
  return d.desc_;
}

// Copy rows [r0, r0 + rows) x K chunk [k0, k0 + kKC) of X(r, k) into the
// canonical layout; out-of-range elements are zero.  Row-contiguous operands
// (k stride 1) go through cp.async, 16 bytes per copy, all in flight at once
// (the caller waits with cp.async.wait_all); transposed operands are gathered
// element by element, four 16-byte pieces per thread in flight.
__device__ __forceinline__ void cp_async16(uint8_t* dst, const void* src, bool valid) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src),
               "r"(valid ? 16 : 0)
               : "memory");
}

__device__ __forceinline__ void fill_chunk(uint8_t* dst, int rows, const bf16* __restrict__ X, int64_t sr, int64_t sk,
                                           int r0, int rmax, int k0, int kmax) {
  const int groups = kKC / 8;
  const int items = rows * groups;
  const bool contiguous = (sk == 1) && ((sr & 7) == 0) && ((reinterpret_cast<uintptr_t>(X) & 15) == 0);
  if (contiguous) {
    for (int idx = threadIdx.x; idx < items; idx += blockDim.x) {
      const int r = idx / groups, g = idx % groups;  // consecutive threads: consecutive pieces of a row
      const int gr = r0 + r, gk = k0 + g * 8;
      uint8_t* p = dst + ((size_t)g * (rows / 8) + (r >> 3)) * 128 + (r & 7) * 16;
      if (gk + 8 <= kmax || gk >= kmax) {
        const bool valid = gr < rmax && gk < kmax;
        cp_async16(p, valid ? (const void*)(X + (int64_t)gr * sr + gk) : (const void*)X, valid);
      } else {  // a K edge inside the 8-element piece
        bf16 e[8];
#pragma unroll
        for (int j = 0; j < 8; ++j)
          e[j] = (gr < rmax && gk + j < kmax) ? X[(int64_t)gr * sr + gk + j] : __float2bfloat16_rn(0.f);
        *reinterpret_cast<uint4*>(p) = *reinterpret_cast<const uint4*>(e);
      }
    }
    return;
  }
  constexpr int kBatch = 4;
  for (int base = threadIdx.x; base < items; base += blockDim.x * kBatch) {
    uint4 v[kBatch];
#pragma unroll
    for (int u = 0; u < kBatch; ++u) {  // loads of kBatch pieces first
      const int idx = base + u * blockDim.x;
      const int r = idx % rows, g = idx / rows;  // consecutive threads: consecutive rows (coalesced)
      const int gr = r0 + r, gk = k0 + g * 8;
      bf16 e[8];
#pragma unroll
      for (int j = 0; j < 8; ++j)
        e[j] = (idx < items && gr < rmax && gk + j < kmax) ? X[(int64_t)gr * sr + (int64_t)(gk + j) * sk]
                                                          : __float2bfloat16_rn(0.f);
      v[u] = *reinterpret_cast<const uint4*>(e);
    }
#pragma unroll
    for (int u = 0; u < kBatch; ++u) {
      const int idx = base + u * blockDim.x;
      if (idx >= items) continue;
      const int r = idx % rows, g = idx / rows;
      *reinterpret_cast<uint4*>(dst + ((size_t)g * (rows / 8) + (r >> 3)) * 128 + (r & 7) * 16) = v[u];
    }
  }
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
  for (long long it = 0; it < kWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

template <int NT>
__global__ void __launch_bounds__(kGemmThreads) k_gemm_tc(GemmArgs a) {
  static_assert(NT == 256 || NT == 16, "tile N");
  constexpr int kCols = NT < 32 ? 32 : NT;  // TMEM allocation: power of two >= 32
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* sA = smem;                         // 128 x 64 bf16 = 16 KB
  uint8_t* sB = smem + kTileM * kKC * 2;      // NT x 64 bf16
  uint64_t* bar = reinterpret_cast<uint64_t*>(sB + NT * kKC * 2);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 1);
  __shared__ int s_fail;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * kTileM, n0 = blockIdx.y * NT;
  const int kb = blockIdx.z * a.k_split;
  const int ke = min(a.K, kb + a.k_split);

  if (threadIdx.x == 0) {
    s_fail = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const uint32_t idesc = static_cast<uint32_t>(
      cute::UMMA::make_instr_desc<cute::bfloat16_t, cute::bfloat16_t, float, kTileM, NT, cute::UMMA::Major::K,
                                  cute::UMMA::Major::K>());
  const uint32_t aA = smem_u32(sA), aB = smem_u32(sB), aBar = smem_u32(bar);

  uint32_t phase = 0;
  bool ok = true;
  for (int k0 = kb; k0 < ke; k0 += kKC) {
    fill_chunk(sA, kTileM, a.A, a.sam, a.sak, m0, a.M, k0, ke);
    fill_chunk(sB, NT, a.B, a.sbn, a.sbk, n0, a.N, k0, ke);
    asm volatile("cp.async.wait_all;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // smem writes -> tensor core
    __syncthreads();
    if (threadIdx.x == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int kk = 0; kk < kKC / 16; ++kk) {
        const uint64_t da = kmajor_desc(aA, kTileM, kk), db = kmajor_desc(aB, NT, kk);
        const uint32_t acc = (k0 > kb || kk > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
            "l"(da), "l"(db), "r"(idesc), "r"(acc)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(aBar)
                   : "memory");
    }
    if (!mbar_wait(aBar, phase)) {
      s_fail = 1;
      ok = false;
    }
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    __syncthreads();
    if (s_fail) {
      ok = false;
      break;
    }
  }
  if (!ok) {
    if (threadIdx.x == 0) atomicExch(a.err, 1);
    // the MMAs of the failed chunk may still be in flight: one more bounded wait
    mbar_wait(aBar, phase ^ 1u);
  } else if (ke > kb) {
    // Epilogue: warp w owns TMEM lanes (tile rows) 32w .. 32w+31.
    const int row = m0 + warp * 32 + lane;
    for (int c0 = 0; c0 < NT; c0 += 16) {
      uint32_t r[16];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
          "%15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (row >= a.M) continue;
      const int nb = n0 + c0;
      const int64_t o0 = (int64_t)row * a.ldo + nb;
      // The thread's 16 consecutive outputs of its row go out as 16-byte
      // vectors when the slice is whole and aligned (ldo a multiple of 8).
      const bool whole = nb + 16 <= a.N && (a.ldo & 7) == 0;
      if (a.epi == kEpiHidden && whole) {
        alignas(16) bf16 zb[16], yb[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const float z = __uint_as_float(r[j]) + (a.bias ? a.bias[nb + j] : 0.f);
          zb[j] = __float2bfloat16_rn(z);
          yb[j] = __float2bfloat16_rn(silu(z));
        }
        uint4* pz = reinterpret_cast<uint4*>(a.pre + o0);
        uint4* py = reinterpret_cast<uint4*>(a.out + o0);
        pz[0] = reinterpret_cast<const uint4*>(zb)[0];
        pz[1] = reinterpret_cast<const uint4*>(zb)[1];
        py[0] = reinterpret_cast<const uint4*>(yb)[0];
        py[1] = reinterpret_cast<const uint4*>(yb)[1];
        continue;
      }
      if (a.epi == kEpiBackAct && whole) {
        alignas(16) bf16 zp[16], gb[16];
        reinterpret_cast<uint4*>(zp)[0] = reinterpret_cast<const uint4*>(a.zprev + o0)[0];
        reinterpret_cast<uint4*>(zp)[1] = reinterpret_cast<const uint4*>(a.zprev + o0)[1];
#pragma unroll
        for (int j = 0; j < 16; ++j)
          gb[j] = __float2bfloat16_rn(__uint_as_float(r[j]) * silu_grad(__bfloat162float(zp[j])));
        uint4* pg = reinterpret_cast<uint4*>(a.out + o0);
        pg[0] = reinterpret_cast<const uint4*>(gb)[0];
        pg[1] = reinterpret_cast<const uint4*>(gb)[1];
        continue;
      }
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int n = nb + j;
        if (n >= a.N) continue;
        const float acc = __uint_as_float(r[j]);
        const int64_t o = (int64_t)row * a.ldo + n;
        if (a.epi == kEpiHidden) {
          const float z = acc + (a.bias ? a.bias[n] : 0.f);
          a.pre[o] = __float2bfloat16_rn(z);
          a.out[o] = __float2bfloat16_rn(silu(z));
        } else if (a.epi == kEpiLinear) {
          a.out32[o] = acc + (a.bias ? a.bias[n] : 0.f);
        } else if (a.epi == kEpiBackAct) {
          a.out[o] = __float2bfloat16_rn(acc * silu_grad(__bfloat162float(a.zprev[o])));
        } else {
          atomicAdd(a.out32 + o, acc);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
}

template <int NT>
constexpr int gemm_smem_bytes() {
  return kTileM * kKC * 2 + NT * kKC * 2 + 16;
}

}  // namespace mlp
}  // namespace o2f

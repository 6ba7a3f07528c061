// Block ILU(0) preconditioner of the adjoint operator A = J^T, for the
// preconditioned BiCGSTAB (no reference counterpart: the reference runs
// BiCGSTAB with the identity preconditioner, src/shape_optimization.cpp:699,
// which on realistic meshes needs 10^4-10^5 iterations).  The preconditioner
// changes only the convergence path: the solution is the same J^T lambda = b
// at the same true-residual tolerance.
//
// A in block form (4x4 blocks, one row per cell).  From the matrix-free
// product (src/shape_optimization.cpp:433-482), with B_{c,e} the flux
// Jacobian block of edge e on cell c's side and s = -1 for the left cell,
// +1 for the right cell of e:
//   A_cc = sum_e (s_c L_e / V_c) B_{c,e}^T
//   A_co = (s_o L_e / V_o) B_{c,e}^T      (o: the other cell of e)
// Rows are stored as 5 blocks: [0] the diagonal, [1..4] the neighbours in the
// cell's slot order (ilu.nbr[k][c], -1 when absent).
//
// Factorization (IKJ form, rows in a reverse Cuthill-McKee order, each level
// of the dependency DAG processed by one launch): for row i and its lower
// neighbours k in increasing order, L_ik = A_ik D_k^{-1}, then
// A_ij -= L_ik U_kj for every block j of row k above k that row i also holds;
// finally D_i^{-1} is stored.  Solves: forward y_i = r_i - sum_{k<i} L_ik y_k,
// backward z_i = D_i^{-1} (y_i - sum_{j>i} U_ij z_j).
#pragma once

#include "kernels.cuh"

namespace o2f {

__device__ __forceinline__ void mat4_mul(const double* a, const double* b, double* c) {
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int q = 0; q < 4; ++q)
      c[r * 4 + q] = a[r * 4 + 0] * b[0 * 4 + q] + a[r * 4 + 1] * b[1 * 4 + q] + a[r * 4 + 2] * b[2 * 4 + q] +
                     a[r * 4 + 3] * b[3 * 4 + q];
}

// 4x4 inverse by Gauss-Jordan elimination with partial pivoting; returns
// false for a singular block (the inverse is then set to the identity).
__device__ __forceinline__ bool mat4_inv(const double* a_in, double* inv) {
  double a[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    a[i] = a_in[i];
    inv[i] = (i % 5 == 0) ? 1.0 : 0.0;
  }
  for (int col = 0; col < 4; ++col) {
    int piv = col;
    double best = fabs(a[col * 4 + col]);
    for (int r = col + 1; r < 4; ++r) {
      const double v = fabs(a[r * 4 + col]);
      if (v > best) {
        best = v;
        piv = r;
      }
    }
    if (!(best > 0.0)) {
#pragma unroll
      for (int i = 0; i < 16; ++i) inv[i] = (i % 5 == 0) ? 1.0 : 0.0;
      return false;
    }
    if (piv != col) {
      for (int q = 0; q < 4; ++q) {
        double t = a[col * 4 + q];
        a[col * 4 + q] = a[piv * 4 + q];
        a[piv * 4 + q] = t;
        t = inv[col * 4 + q];
        inv[col * 4 + q] = inv[piv * 4 + q];
        inv[piv * 4 + q] = t;
      }
    }
    const double d = 1.0 / a[col * 4 + col];
    for (int q = 0; q < 4; ++q) {
      a[col * 4 + q] *= d;
      inv[col * 4 + q] *= d;
    }
    for (int r = 0; r < 4; ++r) {
      if (r == col) continue;
      const double f = a[r * 4 + col];
      if (f == 0.0) continue;
      for (int q = 0; q < 4; ++q) {
        a[r * 4 + q] -= f * a[col * 4 + q];
        inv[r * 4 + q] -= f * inv[col * 4 + q];
      }
    }
  }
  return true;
}

// Assemble the block rows of A from the Jacobian blocks of k_jt_blocks.
__global__ void __launch_bounds__(kBlock) k_ilu_assemble(int64_t nc, const int32_t* __restrict__ jslot, Geom<double> g,
                                                         const int2* __restrict__ ec,
                                                         const uint8_t* __restrict__ ebc,
                                                         const double* __restrict__ blk, double shift,
                                                         IluDev ilu) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  double* row = ilu.A + c * 80;
  double diag[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) diag[i] = 0.0;
  const double Vc = g.cgeom[c].c;
  for (int k = 0; k < 4; ++k) {
    double* nb = row + 16 * (1 + k);
#pragma unroll
    for (int i = 0; i < 16; ++i) nb[i] = 0.0;
    const int s = jslot[(int64_t)k * nc + c];
    if (s < 0) continue;
    const int e = s >> 1;
    const bool left = (s & 1) == 0;
    const double L = g.egeom[e].c;
    const double* B = blk + (int64_t)e * 32 + (left ? 0 : 16);
    const double sc = (left ? -1.0 : 1.0) * L / Vc;
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int q = 0; q < 4; ++q) diag[r * 4 + q] += sc * B[q * 4 + r];  // B^T
    if (ebc[e] != 0) continue;
    const int2 cc = ec[e];
    const int o = left ? cc.y : cc.x;
    const double so = (left ? 1.0 : -1.0) * L / g.cgeom[o].c;
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int q = 0; q < 4; ++q) nb[r * 4 + q] = so * B[q * 4 + r];
  }
  if (shift > 0.0) {  // pseudo-time shift: s times the block's max row sum
    double nrm = 0.0;
#pragma unroll
    for (int r = 0; r < 4; ++r)
      nrm = fmax(nrm, fabs(diag[r * 4]) + fabs(diag[r * 4 + 1]) + fabs(diag[r * 4 + 2]) + fabs(diag[r * 4 + 3]));
#pragma unroll
    for (int r = 0; r < 4; ++r) diag[r * 5] += (diag[r * 5] < 0.0 ? -shift : shift) * nrm;
  }
#pragma unroll
  for (int i = 0; i < 16; ++i) row[i] = diag[i];
}

// One level of the factorization.
__global__ void __launch_bounds__(128) k_ilu_factor(const int32_t* __restrict__ cells, int n, IluDev ilu,
                                                    int* status) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int i = cells[t];
  const int64_t nc = ilu.nc;
  double* row = ilu.A + (int64_t)i * 80;
  const int pi = ilu.pos[i];
  int nb[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) nb[k] = ilu.nbr[(int64_t)k * nc + i];
  // lower neighbours in increasing ILU position
  int order[4], nlow = 0;
  for (int k = 0; k < 4; ++k)
    if (nb[k] >= 0 && ilu.pos[nb[k]] < pi) order[nlow++] = k;
  for (int a = 1; a < nlow; ++a)
    for (int b = a; b > 0 && ilu.pos[nb[order[b]]] < ilu.pos[nb[order[b - 1]]]; --b) {
      const int tmp = order[b];
      order[b] = order[b - 1];
      order[b - 1] = tmp;
    }
  double L[16], prod[16];
  for (int a = 0; a < nlow; ++a) {
    const int slot = order[a];
    const int k = nb[slot];
    double* Aik = row + 16 * (1 + slot);
    mat4_mul(Aik, ilu.Dinv + (int64_t)k * 16, L);
#pragma unroll
    for (int q = 0; q < 16; ++q) Aik[q] = L[q];
    // subtract L_ik U_kj for the upper blocks j of row k held by row i
    const double* rowk = ilu.A + (int64_t)k * 80;
    const int pk = ilu.pos[k];
    for (int m = 0; m < 4; ++m) {
      const int j = ilu.nbr[(int64_t)m * nc + k];
      if (j < 0 || ilu.pos[j] <= pk) continue;
      double* dst = nullptr;
      if (j == i) {
        dst = row;
      } else {
        for (int s = 0; s < 4; ++s)
          if (nb[s] == j) dst = row + 16 * (1 + s);
      }
      if (!dst) continue;
      mat4_mul(L, rowk + 16 * (1 + m), prod);
#pragma unroll
      for (int q = 0; q < 16; ++q) dst[q] -= prod[q];
    }
  }
  if (!mat4_inv(row, ilu.Dinv + (int64_t)i * 16)) atomicExch(status, 1);
}

// Sync-free triangular sweeps (one launch per triangle).  Rows are processed
// in a level order of the triangle's dependency graph (ilu.sweep: forward
// levels, then backward levels), a topological order, so the rows of one
// 32-row chunk are mostly independent.  Warps take chunks from a counter
// (see k_ilu_sweep for why the waits cannot deadlock).
//
// The solved values are their own ready signals: every output slot holds
// the sentinel bit pattern kSweepEmpty until its row writes the solution,
// and a waiting row polls the 8-byte words of its dependencies' slots
// (relaxed loads at GPU scope, single-copy atomic per word) until none is
// the sentinel, so a level costs one L2 round trip and no fence.  The
// forward sweep writes into ilu.tmp and resets the backward sweep's output
// to the sentinel; the backward sweep reads ilu.tmp and resets it after
// reading, so both buffers are empty again for the next application.  A
// computed NaN is stored as the canonical NaN, never as the sentinel.
//
// Waits are bounded: past ilu.spin_limit polls (default kSweepSpinLimit) the
// warp records sync->err and stops waiting, and every other waiting row
// gives up once it sees the error; the host turns it into an error status.
constexpr int kSweepBlock = 128;
constexpr long long kSweepSpinLimit = 1ll << 22;
constexpr unsigned long long kSweepEmpty = 0x7ff4f11ed5eed000ull;  // a NaN no arithmetic produces

__device__ __forceinline__ void prefetch_l1(const void* p) {
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const void* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_relaxed_u64(void* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned long long sweep_bits(double x) {
  return x != x ? 0x7ff8000000000000ull : (unsigned long long)__double_as_longlong(x);
}

__device__ __forceinline__ void store_empty(Vec4<double>* p) {
  unsigned long long* q = reinterpret_cast<unsigned long long*>(p);
#pragma unroll
  for (int k = 0; k < 4; ++k) st_relaxed_u64(q + k, kSweepEmpty);
}

// Fill a sweep buffer with the sentinel (set-up of ilu.tmp).
__global__ void k_ilu_empty(int64_t n, Vec4<double>* y) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) store_empty(y + i);
}

// kForward: tmp_i = r_i - sum_{k lower} L_ik tmp_k; z_i <- empty.
// backward: z_i = D_i^{-1} (tmp_i - sum_{j upper} U_ij z_j); tmp_i <- empty.
// A small grid of persistent warps (ilu_sweep_blocks): each warp claims the
// next 32-row chunk, solves it, and claims again, so only the warps near the
// front of the dependency levels poll -- a launch of one warp per chunk kept
// thousands of warps polling and saturated the load path.  Claims are in
// order and a warp claims again only after finishing its chunk, so every
// claimed chunk belongs to a running warp and the earliest unfinished row
// has its dependencies done: no deadlock for any grid size.  The last warp
// to leave resets the counters for the next launch (all its claims, failing
// ones included, come before it leaves).
template <bool kForward>
__global__ void __launch_bounds__(kSweepBlock) k_ilu_sweep(int n, IluDev ilu, const Vec4<double>* r,
                                                           Vec4<double>* z, const int* gate) {
  if (gated(gate)) return;
  constexpr unsigned int kFull = 0xffffffffu;
  SweepSync* sync = ilu.sync + (kForward ? 0 : 1);
  Vec4<double>* out = kForward ? ilu.tmp : z;  // slots this sweep fills (empty on entry)
  const int lane = threadIdx.x & 31;
  const unsigned int nchunks = (unsigned int)(n + 31) / 32u;
  const unsigned int nwarps = gridDim.x * (unsigned int)(kSweepBlock / 32);
  const int64_t nc = ilu.nc;
  while (true) {
    unsigned int chunk = 0;
    if (lane == 0) chunk = atomicAdd(&sync->claim, 1u);
    chunk = __shfl_sync(kFull, chunk, 0);
    if (chunk >= nchunks) break;
    const int p = (int)chunk * 32 + lane;
    const bool active = p < n;
    int i = 0, dep[4], ndep = 0, slot[4];
    Vec4<double> own{};
    if (active) {
      i = ilu.sweep[kForward ? p : (int64_t)n + p];
      const int pi = ilu.pos[i];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int o = ilu.nbr[k * nc + i];
        if (o < 0) continue;
        const int po = ilu.pos[o];
        if (kForward ? po < pi : po > pi) {
          dep[ndep] = o;
          slot[ndep] = k;
          ++ndep;
        }
      }
      // The row's blocks (and D^-1 backward) do not depend on the waits:
      // bring them towards L1 first.
      const char* rowp = reinterpret_cast<const char*>(ilu.A + (int64_t)i * 80);
#pragma unroll
      for (int b = 0; b < 5; ++b) prefetch_l1(rowp + 128 * b);
      if (!kForward) prefetch_l1(ilu.Dinv + (int64_t)i * 16);
      if (kForward) {
        own = r[i];
        store_empty(z + i);  // the backward sweep's slot
      } else {
        const double2* t = reinterpret_cast<const double2*>(ilu.tmp + i);
        const double2 a = __ldcg(t), b = __ldcg(t + 1);
        own = Vec4<double>{a.x, a.y, b.x, b.y};
        store_empty(ilu.tmp + i);  // empty again for the next forward sweep
      }
    }
    bool done = !active;
    long long spins = 0;
    while (__any_sync(kFull, !done)) {
      if (done) continue;
      // the last word first (cheap while waiting), then all four
      bool ready = true;
      for (int d = 0; d < ndep; ++d)
        if (ld_relaxed_u64(reinterpret_cast<const unsigned long long*>(out + dep[d]) + 3) == kSweepEmpty)
          ready = false;
      unsigned long long w[4][4];
      if (ready) {
        for (int d = 0; d < ndep; ++d) {
          const unsigned long long* q = reinterpret_cast<const unsigned long long*>(out + dep[d]);
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            w[d][k] = ld_relaxed_u64(q + k);
            if (w[d][k] == kSweepEmpty) ready = false;
          }
        }
      }
      if (ready) {
        const double* row = ilu.A + (int64_t)i * 80;
        Vec4<double> acc = own;
        for (int d = 0; d < ndep; ++d) {
          const double* Bk = row + 16 * (1 + slot[d]);
          const Vec4<double> v{__longlong_as_double((long long)w[d][0]), __longlong_as_double((long long)w[d][1]),
                               __longlong_as_double((long long)w[d][2]), __longlong_as_double((long long)w[d][3])};
          acc.a -= Bk[0] * v.a + Bk[1] * v.b + Bk[2] * v.c + Bk[3] * v.d;
          acc.b -= Bk[4] * v.a + Bk[5] * v.b + Bk[6] * v.c + Bk[7] * v.d;
          acc.c -= Bk[8] * v.a + Bk[9] * v.b + Bk[10] * v.c + Bk[11] * v.d;
          acc.d -= Bk[12] * v.a + Bk[13] * v.b + Bk[14] * v.c + Bk[15] * v.d;
        }
        if (!kForward) {
          const double* D = ilu.Dinv + (int64_t)i * 16;
          Vec4<double> o4;
          o4.a = D[0] * acc.a + D[1] * acc.b + D[2] * acc.c + D[3] * acc.d;
          o4.b = D[4] * acc.a + D[5] * acc.b + D[6] * acc.c + D[7] * acc.d;
          o4.c = D[8] * acc.a + D[9] * acc.b + D[10] * acc.c + D[11] * acc.d;
          o4.d = D[12] * acc.a + D[13] * acc.b + D[14] * acc.c + D[15] * acc.d;
          acc = o4;
        }
        if (!kForward || i != ilu.stall_row) {
          unsigned long long* q = reinterpret_cast<unsigned long long*>(out + i);
          st_relaxed_u64(q, sweep_bits(acc.a));
          st_relaxed_u64(q + 1, sweep_bits(acc.b));
          st_relaxed_u64(q + 2, sweep_bits(acc.c));
          st_relaxed_u64(q + 3, sweep_bits(acc.d));
        }
        done = true;
      } else {
        __nanosleep(32);
        if ((++spins & 63) == 0) {
          if (spins > ilu.spin_limit) {
            atomicExch(&sync->err, 1);
            done = true;
          } else if (*reinterpret_cast<volatile int*>(&sync->err)) {
            done = true;
          }
        }
      }
    }
  }
  __syncwarp();
  if (lane == 0) {
    __threadfence();
    const unsigned int f = atomicAdd(&sync->done, 1u);  // warps that have left
    if (f == nwarps - 1) {
      sync->claim = 0;
      sync->done = 0;
      __threadfence();
    }
  }
}

// One thread block solves a whole triangle, level after level: the rows of a
// level are independent and a __syncthreads separates the levels, so no row
// ever waits on a flag.  Each sweep position has a record (row, the sweep
// positions of its dependencies, their slots); values are kept by sweep
// position, and the last kSweepWindow of them also in shared memory, where
// a row finds its dependencies -- they lie mostly a few levels back.  A
// dependency q is read from shared memory when q >= e - kSweepWindow (e:
// end of the current level): its slot is not overwritten by this level's
// writes, which reuse the slots of positions [b - W, e - W).
// The arithmetic of a row (dependencies in slot order) is that of
// k_ilu_sweep: both give the same bits.  One SM per sweep, so the sweeps of
// many contexts run side by side.
constexpr int kSweepCtaThreads = 512;
constexpr int kSweepWindow = 2048;  // values kept in shared memory (64 KiB; ~96 % of the dependencies)
// Factor blocks of the next level staged in shared memory (two buffers,
// alternating by level): dependency slots 0 and 1 of each position (on
// triangles a forward row has at most 2 dependencies, a backward row rarely
// 3) for the first 10 chunks of 32 positions forward (8 KiB each), the first
// 6 backward with their D^-1 (4 KiB each) after them.
constexpr int kStageSlots = 2;
constexpr int kStageChunkDoubles = kStageSlots * 512;
constexpr int kStageChunksFwd = 10;
constexpr int kStageChunksBwd = 6;
constexpr int kStageBwdD = kStageChunksBwd * kStageChunkDoubles;  // offset of the staged D^-1, doubles
constexpr int kStageDoubles = kStageChunksFwd * kStageChunkDoubles;  // one buffer (backward: 6*1024 + 6*512)
constexpr size_t kSweepSmem = sizeof(Vec4<double>) * kSweepWindow + 2 * kStageDoubles * sizeof(double);
static_assert(kSweepSmem <= 227 * 1024, "block sweep shared memory above the per-block limit");
static_assert(kStageBwdD + kStageChunksBwd * 512 <= kStageDoubles, "backward staging overflows its buffer");

// Factor blocks of the block sweeps, repacked in sweep order after every
// factorization and interleaved over 32 consecutive positions, so that the
// 32 lanes of a warp (consecutive positions of a level) read 32 consecutive
// doubles per element: element e of dependency d of position p of direction
// dir is pk[dir*n*64 + (p>>5)*2048 + d*512 + e*32 + (p&31)] (n rounded up to
// 32), D^-1 of backward position p is pk[2*n*64 + (p>>5)*512 + e*32 + (p&31)].
__device__ __forceinline__ int64_t sweep_pack_base(int64_t n32, int dir, int p) {
  return (int64_t)dir * n32 * 64 + (int64_t)(p >> 5) * 2048 + (p & 31);
}

__global__ void k_ilu_pack(int n, IluDev ilu) {
  const int64_t n32 = ((int64_t)n + 31) / 32 * 32;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;  // (dir, p, d) with d = 4 for D^-1
  if (t >= (int64_t)2 * n * 5) return;
  const int dir = (int)(t / ((int64_t)n * 5));
  const int64_t rest = t % ((int64_t)n * 5);
  const int p = (int)(rest / 5), d = (int)(rest % 5);
  const int* rec = ilu.rec + 8 * ((int64_t)dir * n + p);
  const int row = rec[0];
  if (d == 4) {
    if (dir == 0) return;
    const double* D = ilu.Dinv + (int64_t)row * 16;
    double* dst = ilu.pack + 2 * n32 * 64 + (int64_t)(p >> 5) * 512 + (p & 31);
#pragma unroll
    for (int e = 0; e < 16; ++e) dst[e * 32] = D[e];
    return;
  }
  if (rec[1 + d] < 0) return;
  const int slot = (int)(((unsigned int)rec[5] >> (8 * d)) & 0xff);
  const double* B = ilu.A + (int64_t)row * 80 + 16 * (1 + slot);
  double* dst = ilu.pack + sweep_pack_base(n32, dir, p) + d * 512;
#pragma unroll
  for (int e = 0; e < 16; ++e) dst[e * 32] = B[e];
}

// One row of a block sweep: own value minus the dependencies' products
// (slot order), times D^-1 backward; stored in the window, by position, and
// (backward) into z by row.  Factor blocks of the level's first `nch` chunks
// (from chunk c0) are read from the staged copy `stage`, the rest from the
// packed copy in global memory: same layout, same values.
template <bool kForward>
__device__ __forceinline__ void sweep_cta_row(const IluDev& ilu, int p, int e, const int4& a, const int4& c,
                                              Vec4<double> acc, const Vec4<double>* win_r, Vec4<double>* win,
                                              Vec4<double>* out, Vec4<double>* z, const double* stage, int c0,
                                              int nch) {
  const int i = a.x;
  const int dq[4] = {a.y, a.z, a.w, c.x};
  const int64_t n32 = ((int64_t)ilu.nc + 31) / 32 * 32;
  const int k = (p >> 5) - c0;  // >= 0: p lies in the level that starts in chunk c0
  const bool staged = k < nch;
  const double* P = ilu.pack + sweep_pack_base(n32, kForward ? 0 : 1, p);
  const double* S = stage + k * kStageChunkDoubles + (p & 31);
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    const int q = dq[d];
    if (q < 0) break;
    const double* Bk = (staged && d < kStageSlots ? S : P) + d * 512;  // element k at Bk[32 k]
    const Vec4<double> v = q >= e - kSweepWindow ? win_r[q % kSweepWindow] : out[q];
    acc.a -= Bk[0] * v.a + Bk[32] * v.b + Bk[64] * v.c + Bk[96] * v.d;
    acc.b -= Bk[128] * v.a + Bk[160] * v.b + Bk[192] * v.c + Bk[224] * v.d;
    acc.c -= Bk[256] * v.a + Bk[288] * v.b + Bk[320] * v.c + Bk[352] * v.d;
    acc.d -= Bk[384] * v.a + Bk[416] * v.b + Bk[448] * v.c + Bk[480] * v.d;
  }
  if (!kForward) {
    const double* D = staged ? stage + kStageBwdD + k * 512 + (p & 31)
                             : ilu.pack + 2 * n32 * 64 + (int64_t)(p >> 5) * 512 + (p & 31);
    Vec4<double> o4;
    o4.a = D[0] * acc.a + D[32] * acc.b + D[64] * acc.c + D[96] * acc.d;
    o4.b = D[128] * acc.a + D[160] * acc.b + D[192] * acc.c + D[224] * acc.d;
    o4.c = D[256] * acc.a + D[288] * acc.b + D[320] * acc.c + D[352] * acc.d;
    o4.d = D[384] * acc.a + D[416] * acc.b + D[448] * acc.c + D[480] * acc.d;
    acc = o4;
  }
  const Vec4<double> v{__longlong_as_double((long long)sweep_bits(acc.a)),
                       __longlong_as_double((long long)sweep_bits(acc.b)),
                       __longlong_as_double((long long)sweep_bits(acc.c)),
                       __longlong_as_double((long long)sweep_bits(acc.d))};
  win[p % kSweepWindow] = v;
  out[p] = v;
  if (!kForward) z[i] = v;
}

// Bulk prefetch of [p, p + bytes) into L2 (a hint: no data is returned and
// no completion is awaited); p 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void prefetch_l2_bulk(const void* p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// The L2 prefetch of one level [b, e) of a block sweep, by one warp: the
// 32-position chunks of packed factor blocks that hold it (16 KiB each, plus
// 4 KiB of D^-1 backward) and its records (32 B per position).  The chunks
// lie inside the packed copy (n rounded up to 32 positions), the records
// inside the 2n records of the two directions.
template <bool kForward>
__device__ __forceinline__ void sweep_prefetch_level(const IluDev& ilu, const int* rec, int b, int e, int lane) {
  if (b >= e) return;
  const int64_t n32 = ((int64_t)ilu.nc + 31) / 32 * 32;
  for (int c = (b >> 5) + lane; c <= ((e - 1) >> 5); c += 32) {
    prefetch_l2_bulk(ilu.pack + (kForward ? 0 : n32 * 64) + (int64_t)c * 2048, 2048 * sizeof(double));
    if (!kForward) prefetch_l2_bulk(ilu.pack + 2 * n32 * 64 + (int64_t)c * 512, 512 * sizeof(double));
  }
  const char* r0 = reinterpret_cast<const char*>(rec + 8 * (int64_t)b);
  const int64_t bytes = (int64_t)(e - b) * 8 * sizeof(int);
  for (int64_t o = (int64_t)lane * 4096; o < bytes; o += 32 * 4096)
    prefetch_l2_bulk(r0 + o, (uint32_t)(bytes - o < 4096 ? bytes - o : 4096));
}

// Asynchronous 16-byte global -> shared copy (completes at cp_async_wait_all).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Chunks of 32 positions of the level [b, e) that are staged.
template <bool kForward>
__device__ __forceinline__ int sweep_stage_chunks(int b, int e) {
  if (b >= e) return 0;
  const int n = ((e - 1) >> 5) - (b >> 5) + 1;
  const int cap = kForward ? kStageChunksFwd : kStageChunksBwd;
  return n < cap ? n : cap;
}

// Stage the factor blocks of level [b, e) into `buf`, by the whole block:
// dependency slots 0 .. kStageSlots-1 of the level's first chunks (the
// leading kStageChunkDoubles of each 2048-double chunk), and D^-1 backward.
// Each copied chunk lies inside the packed copy (chunk indices up to
// (e - 1) >> 5 < n32 / 32); addresses and sizes are multiples of 16 bytes.
template <bool kForward>
__device__ __forceinline__ void sweep_stage_level(const IluDev& ilu, int b, int e, double* buf, int t, int T) {
  const int nch = sweep_stage_chunks<kForward>(b, e);
  if (nch == 0) return;
  const int64_t n32 = ((int64_t)ilu.nc + 31) / 32 * 32;
  const double* src = ilu.pack + (kForward ? 0 : n32 * 64) + (int64_t)(b >> 5) * 2048;
  constexpr int kPieces = kStageChunkDoubles / 2;  // 16-byte pieces per staged chunk
  for (int k = t; k < nch * kPieces; k += T) {
    const int ch = k / kPieces, pc = k - ch * kPieces;
    cp_async16(buf + ch * kStageChunkDoubles + 2 * pc, src + (int64_t)ch * 2048 + 2 * pc);
  }
  if (!kForward) {
    const double* srcD = ilu.pack + 2 * n32 * 64 + (int64_t)(b >> 5) * 512;
    for (int k = t; k < nch * 256; k += T) cp_async16(buf + kStageBwdD + 2 * k, srcD + 2 * k);
  }
}

// The first two rows of each thread in a level are software-pipelined: their
// records are loaded during the level before and their own values (r, or the
// forward value) requested at its end, so a level starts with its operands
// in flight; further rows load at use.  Factor blocks come from the packed
// copy (k_ilu_pack), coalesced across the warp: the first chunks of each
// level staged in shared memory by asynchronous copies issued during the
// level before (two buffers), the rest read from global memory.  The first
// warp also requests the blocks and records of the level two ahead into L2
// as each level starts, for when other contexts' sweeps and products have
// evicted them.  One block per SM is declared so that the compiler keeps the
// rows' loads in registers (about 100 per thread) instead of capping them.
template <bool kForward>
__global__ void __launch_bounds__(kSweepCtaThreads, 1) k_ilu_sweep_cta(int n, IluDev ilu, const Vec4<double>* r,
                                                                    Vec4<double>* z, const int* gate) {
  if (gated(gate)) return;
  extern __shared__ Vec4<double> win[];
  const int* rec = ilu.rec + (kForward ? 0 : (int64_t)8 * n);
  const int32_t* off = ilu.lev_off + (kForward ? 0 : ilu.n_lo + 1);
  const int nlev = kForward ? ilu.n_lo : ilu.n_up;
  Vec4<double>* out = kForward ? ilu.out_f : ilu.out_b;  // by sweep position
  const int T = blockDim.x, t = threadIdx.x;
  auto rec_a = [&](int p) { return *reinterpret_cast<const int4*>(rec + 8 * (int64_t)p); };
  auto rec_c = [&](int p) { return *reinterpret_cast<const int4*>(rec + 8 * (int64_t)p + 4); };
  auto own_of = [&](const int4& a, const int4& c) { return kForward ? r[a.x] : ilu.out_f[c.z]; };
  double* stg = reinterpret_cast<double*>(win + kSweepWindow);  // 2 x kStageDoubles
  int4 ra[2], rc[2];
  Vec4<double> own[2];
  if (t < 32)
    for (int l = 0; l < 2 && l < nlev; ++l) sweep_prefetch_level<kForward>(ilu, rec, off[l], off[l + 1], t);
  if (nlev > 0) {
    sweep_stage_level<kForward>(ilu, off[0], off[1], stg, t, T);
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int p = off[0] + t + k * T;
      if (p < off[1]) {
        ra[k] = rec_a(p);
        rc[k] = rec_c(p);
        own[k] = own_of(ra[k], rc[k]);
      }
    }
    cp_async_wait_all();
    __syncthreads();
  }
  for (int l = 0; l < nlev; ++l) {
    const int b = off[l], e = off[l + 1];
    const int ne = l + 1 < nlev ? off[l + 2] : e;
    if (t < 32 && l + 2 < nlev) sweep_prefetch_level<kForward>(ilu, rec, ne, off[l + 3], t);
    // this level's staged blocks (filled during the level before); the next
    // level's into the other buffer, whose last readers passed the barrier
    const double* cur = stg + (l & 1) * kStageDoubles;
    const int c0 = b >> 5, nch = sweep_stage_chunks<kForward>(b, e);
    if (l + 1 < nlev) sweep_stage_level<kForward>(ilu, e, ne, stg + ((l + 1) & 1) * kStageDoubles, t, T);
    int4 na[2], nc[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {  // the next level's records, in flight during this one
      const int q = e + t + k * T;
      if (q < ne) {
        na[k] = rec_a(q);
        nc[k] = rec_c(q);
      }
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int p = b + t + k * T;
      if (p < e) sweep_cta_row<kForward>(ilu, p, e, ra[k], rc[k], own[k], win, win, out, z, cur, c0, nch);
    }
    for (int p = b + t + 2 * T; p < e; p += T) {
      const int4 a = rec_a(p), c = rec_c(p);
      sweep_cta_row<kForward>(ilu, p, e, a, c, own_of(a, c), win, win, out, z, cur, c0, nch);
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {  // the next level's operands, requested before the barrier
      const int q = e + t + k * T;
      if (q < ne) {
        ra[k] = na[k];
        rc[k] = nc[k];
        own[k] = own_of(ra[k], rc[k]);
      }
    }
    cp_async_wait_all();  // this thread's copies of the next level, visible to all after the barrier
    __syncthreads();
  }
}

// Blocks of one sweep launch: enough warps to cover several dependency
// levels ahead of the front, few enough that waiting warps do not crowd the
// load path, and that the sweeps of other contexts can run beside them.
inline int ilu_sweep_blocks(int n) {
  const int chunks = (n + 31) / 32;
  const int blocks = (chunks + kSweepBlock / 32 - 1) / (kSweepBlock / 32);
  return blocks < 64 ? blocks : 64;
}

}  // namespace o2f

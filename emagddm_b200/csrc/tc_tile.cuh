// tc_tile.cuh -- C -= A B^T for one 128 x 128 tile on the 5th-generation
// tensor cores (tcgen05.mma kind::tf32), for the mixed-precision factor of
// the FETI-DP and direct solvers.
//
// Operands stay FP64 in global memory (column-major, as the fronts store
// them).  Each value is split into two TF32 terms, a = a_hi + a_lo
// (a_hi = tf32(a), a_lo = tf32(a - a_hi)), while it is staged into shared
// memory, and the tile is accumulated in FP32 in tensor memory as
//   a_lo b_hi + a_hi b_lo + a_hi b_hi,
// about 22 significant bits per product (the a_lo b_lo term, ~2^-22
// relative, is dropped): FP32-level contractions whose loss the FP64
// refinement loop of the caller absorbs.
//
// One CTA of 256 threads per tile.  The k dimension runs in stages of 16,
// double-buffered: all threads convert and store a stage (shared memory in
// the canonical K-major, no-swizzle layout: 8-row x 16-byte core matrices),
// one thread issues the 6 MMAs of the stage (two k-steps of 8, three terms)
// and commits them to the stage's mbarrier; a stage is refilled only after
// that mbarrier has completed.  The epilogue reads the 128 x 128 FP32
// accumulator with tcgen05.ld (warp w: lanes 32 (w % 4) .., columns
// 64 (w / 4) ..) and subtracts it from C in FP64.
//
// Every mbarrier wait is bounded (kMaxWait polls); a wait that runs out makes
// the tile return false without writing C, after a bounded wait for the MMAs
// already committed, and the tensor memory is freed on every path.
#pragma once

#include <cstdint>

namespace emg {
namespace tc {

constexpr int kM = 128;                     // tile rows = tensor-memory lanes
constexpr int kN = 128;                     // tile columns = tensor-memory columns (FP32)
constexpr int kKS = 16;                     // k per pipeline stage
constexpr int kThreads = 256;
constexpr int kStages = 2;
constexpr int kOpBytes = kM * kKS * 4;      // one operand term of one stage: 8 KB
constexpr int kStageBytes = 4 * kOpBytes;   // A hi, A lo, B hi, B lo
constexpr int kLBO = 128;                   // bytes between the two 4-wide k halves of one MMA's k = 8
constexpr int kSBO = (kKS / 4) * 128;       // bytes between consecutive 8-row core-matrix groups
constexpr size_t kSmemBytes = static_cast<size_t>(kStages) * kStageBytes + 1024;  // + alignment slack
constexpr int kMaxWait = 1 << 22;           // polls of an mbarrier before giving up
// Instruction descriptor: FP32 accumulator (bits 4-5 = 1), A and B TF32
// (bits 7-9, 10-12 = 2), both K-major (bits 15, 16 = 0), N >> 3 at bit 17,
// M >> 4 at bit 24.
constexpr uint32_t kIdesc =
    (1u << 4) | (2u << 7) | (2u << 10) | (static_cast<uint32_t>(kN >> 3) << 17) | (static_cast<uint32_t>(kM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor, no swizzle, K-major: start address,
// leading byte offset (between the k halves), stride byte offset (between
// 8-row groups), descriptor version 1 (bits 46-47).
__device__ __forceinline__ uint64_t sdesc(uint32_t addr) {
  return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) | (static_cast<uint64_t>(kLBO >> 4) << 16) |
         (static_cast<uint64_t>(kSBO >> 4) << 32) | (static_cast<uint64_t>(1) << 46);
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void split_tf32(double a, uint32_t& hi, uint32_t& lo) {
  hi = to_tf32(static_cast<float>(a));
  lo = to_tf32(static_cast<float>(a - static_cast<double>(__uint_as_float(hi))));
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate));
}

__device__ __forceinline__ void commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ bool wait_parity(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (int i = 0; i < kMaxWait; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Rows [0, rows) x k [k0, k0 + 16) of X (column-major, leading dimension
// ldx, k < K valid) as TF32 hi / lo terms in the core-matrix layout:
// byte (r, k) = (r / 8) SBO + (k / 4) LBO + (r % 8) 16 + (k % 4) 4.
// Rows >= rows and k >= K are zero.
__device__ __forceinline__ void stage_operand(uint8_t* hi, uint8_t* lo, const double* __restrict__ X, int64_t ldx,
                                              int rows, int k0, int K) {
  for (int e = threadIdx.x; e < kM * (kKS / 4); e += kThreads) {
    const int r = e & (kM - 1), q = e >> 7;
    uint32_t h[4], l[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int k = k0 + 4 * q + i;
      const double v = (r < rows && k < K) ? X[r + static_cast<int64_t>(k) * ldx] : 0.0;
      split_tf32(v, h[i], l[i]);
    }
    const int off = (r >> 3) * kSBO + q * kLBO + (r & 7) * 16;
    *reinterpret_cast<uint4*>(hi + off) = make_uint4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<uint4*>(lo + off) = make_uint4(l[0], l[1], l[2], l[3]);
  }
}

// C[0:mr, 0:mc] -= A[0:mr, 0:K] B[0:mc, 0:K]^T (column-major; mr, mc <= 128).
// Call with all kThreads threads of the CTA and kSmemBytes of dynamic shared
// memory; returns false (C untouched) if a wait ran out.
__device__ __forceinline__ bool tile_update(double* __restrict__ C, int64_t ldc, int mr, int mc,
                                            const double* __restrict__ A, int64_t lda,
                                            const double* __restrict__ B, int64_t ldb, int K, uint8_t* dyn) {
  __shared__ __align__(8) uint64_t bar[kStages];
  __shared__ uint32_t tmem_sh;
  __shared__ int sh_ok;
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(dyn) + 1023) & ~static_cast<uintptr_t>(1023));
  const int tid = threadIdx.x, warp = tid >> 5;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_sh)),
                 "r"(kN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int s = 0; s < kStages; ++s)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar[s])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    sh_ok = 1;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_sh;
  const int nk = (K + kKS - 1) / kKS;
  int committed = 0;  // stages committed (thread 0's count; the others track it too)
  for (int c = 0; c < nk; ++c) {
    const int s = c & 1;
    if (c >= kStages) {  // stage s was last read by the MMAs of chunk c - 2
      if (tid == 0 && !wait_parity(&bar[s], static_cast<uint32_t>((c - kStages) >> 1) & 1u)) sh_ok = 0;
      __syncthreads();
      if (!sh_ok) break;
    }
    uint8_t* st = sm + s * kStageBytes;
    stage_operand(st, st + kOpBytes, A, lda, mr, c * kKS, K);
    stage_operand(st + 2 * kOpBytes, st + 3 * kOpBytes, B, ldb, mc, c * kKS, K);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t base = smem_u32(st);
#pragma unroll
      for (int j = 0; j < kKS / 8; ++j) {
        const uint32_t o = static_cast<uint32_t>(j * 2 * kLBO);
        const uint64_t ahi = sdesc(base + o), alo = sdesc(base + kOpBytes + o);
        const uint64_t bhi = sdesc(base + 2 * kOpBytes + o), blo = sdesc(base + 3 * kOpBytes + o);
        mma_tf32(tmem, alo, bhi, (c | j) != 0 ? 1u : 0u);
        mma_tf32(tmem, ahi, blo, 1u);
        mma_tf32(tmem, ahi, bhi, 1u);
      }
      commit(&bar[s]);
    }
    committed = c + 1;
  }
  // The last commit of each mbarrier: afterwards every MMA has completed and
  // no arrive is still on its way to this CTA's shared memory.
  if (tid == 0) {
    for (int b = 0; b < kStages; ++b) {
      const int n_b = (committed - b + kStages - 1) / kStages;  // commits made on bar[b]
      if (n_b > 0 && !wait_parity(&bar[b], static_cast<uint32_t>(n_b - 1) & 1u)) sh_ok = 0;
    }
  }
  __syncthreads();
  const bool ok = sh_ok != 0;
  if (ok && committed > 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int q = warp & 3, h = warp >> 2;
    const int row = 32 * q + (tid & 31);
#pragma unroll 1
    for (int cb = 0; cb < kN / 2; cb += 16) {
      const int col0 = (kN / 2) * h + cb;
      uint32_t v[16];
      tmem_ld16(tmem + (static_cast<uint32_t>(32 * q) << 16) + static_cast<uint32_t>(col0), v);
      if (row < mr) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int col = col0 + j;
          if (col < mc) C[row + static_cast<int64_t>(col) * ldc] -= static_cast<double>(__uint_as_float(v[j]));
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kN));
  return ok;
}

}  // namespace tc
}  // namespace emg

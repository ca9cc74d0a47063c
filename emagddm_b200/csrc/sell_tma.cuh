// sell_tma.cuh -- SELL-32 SpMV fed by bulk asynchronous copies (TMA engine,
// cp.async.bulk global -> shared, completion on mbarriers).
//
// A tile is 8 consecutive slices (256 rows); its column indices and values
// are two contiguous byte ranges, copied into one of kStages shared-memory
// stages by a single thread while the 8 warps of the block compute earlier
// tiles from shared memory.  Each warp owns one slice of the tile and each
// lane one row, so the inner loop reads shared memory conflict-free and
// gathers x from L2.  Blocks are persistent (one per SM) and walk tiles
// round-robin.  Every mbarrier wait is bounded; a wait that runs out sets
// `*err` and the block stops issuing work.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace emg {
namespace tma {

constexpr int kWarps = 8;               // warps per block = slices per tile
constexpr int kStages = 2;              // double buffering; two blocks per SM
constexpr int kBlocksPerSm = 2;
constexpr uint32_t kSpinLimit = 1u << 22;  // try_wait polls before giving up

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// Global -> shared bulk copy completing on `bar`; addresses 16-byte aligned,
// size a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar,
                                         uint64_t policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
      " [%0], [%1], %2, [%3], %4;" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Bounded wait: false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (uint32_t i = 0; i < kSpinLimit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

struct Layout {
  // per stage: values [cap] doubles, then columns [cap] ints
  uint32_t cap;          // slots per stage
  uint32_t stage_bytes;  // 12 * cap, rounded to 128
};

__host__ __device__ inline Layout layout_for(uint32_t max_tile_slots) {
  Layout L;
  L.cap = max_tile_slots;
  L.stage_bytes = ((12u * max_tile_slots + 127u) / 128u) * 128u;
  return L;
}

__host__ __device__ inline size_t smem_bytes(const Layout& L) {
  return static_cast<size_t>(kStages) * L.stage_bytes + 128;  // + barriers
}

}  // namespace tma
}  // namespace emg

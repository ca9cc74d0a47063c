// common.cuh -- device helpers shared by the assembly and Krylov kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace emg {

constexpr int kWarp = 32;

// Deterministic warp sum (fixed butterfly).
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Warp reduce-scatter of K values a lane (K a power of two, 1 <= K <= 32):
// returns in every lane the warp sum of v[j] for j = reduce_scatter_index<K>
// (lane).  Each halving exchange keeps half of the values (lanes with the
// exchange's bit set keep the upper half), the rest are full exchanges: K - 1
// + 5 - log2 K shuffles instead of the 5 K of K separate warp sums.  The
// order of the additions is fixed, so the sums are deterministic; the lanes
// whose low 5 - log2 K bits are zero hold distinct j.
template <int K>
__device__ __forceinline__ double warp_reduce_scatter(double (&v)[K], int lane) {
  static_assert(K >= 1 && K <= 32 && (K & (K - 1)) == 0, "K must be a power of two up to 32");
  int o = 16;
#pragma unroll
  for (int h = K / 2; h >= 1; h >>= 1, o >>= 1) {
    const bool up = (lane & o) != 0;
#pragma unroll
    for (int i = 0; i < h; ++i) {
      const double send = up ? v[i] : v[i + h], keep = up ? v[i + h] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
    }
  }
#pragma unroll
  for (; o >= 1; o >>= 1) v[0] += __shfl_xor_sync(0xffffffffu, v[0], o);
  return v[0];
}
template <int K>
__device__ __forceinline__ int reduce_scatter_index(int lane) {
  int j = 0, o = 16;
#pragma unroll
  for (int h = K / 2; h >= 1; h >>= 1, o >>= 1)
    if (lane & o) j += h;
  return j;
}
template <int K>
__device__ __forceinline__ bool reduce_scatter_writer(int lane) {
  return (lane & (32 / K - 1)) == 0;
}

// Deterministic block sum of one value per thread; result valid in every
// thread.  `scratch` holds blockDim.x / 32 doubles.
__device__ __forceinline__ double block_sum(double v, double* scratch) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) scratch[wid] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < nw; ++w) t += scratch[w];
  return t;
}

// Streaming loads for matrix entries: read once per SpMV, so they carry an
// L2 evict-first policy and skip L1, leaving L2 to the vectors (x, p, r, ...)
// that are re-read every iteration.
__device__ __forceinline__ uint64_t evict_first_policy() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
// EMG_LD_PREFETCH: 1 asks L2 to fetch 256-byte blocks for these loads.
#ifndef EMG_LD_PREFETCH
#define EMG_LD_PREFETCH 0
#endif
__device__ __forceinline__ double ld_stream(const double* p, uint64_t pol) {
  double v;
#if EMG_LD_PREFETCH
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.L2::256B.f64 %0, [%1], %2;"
               : "=d"(v) : "l"(p), "l"(pol));
#else
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;"
               : "=d"(v) : "l"(p), "l"(pol));
#endif
  return v;
}
__device__ __forceinline__ int ld_stream(const int* p, uint64_t pol) {
  int v;
#if EMG_LD_PREFETCH
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.L2::256B.s32 %0, [%1], %2;"
               : "=r"(v) : "l"(p), "l"(pol));
#else
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.s32 %0, [%1], %2;"
               : "=r"(v) : "l"(p), "l"(pol));
#endif
  return v;
}
// 16-bit signed load, sign-extended to int.
__device__ __forceinline__ int ld_stream(const int16_t* p, uint64_t pol) {
  int v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.s16 %0, [%1], %2;"
      : "=r"(v) : "l"(p), "l"(pol));
  return v;
}
// Coherent-at-L2 load for values written by other blocks of the same kernel.
__device__ __forceinline__ double ld_l2(const double* p) { return __ldcg(p); }

}  // namespace emg

// batch.cu -- many independent curl-curl systems solved together: Jacobi/plain
// CG in lockstep over a block-diagonal matrix whose diagonal blocks are the
// systems (the union of disjoint meshes assembles to exactly that).  Every
// block keeps its own alpha, beta, residual, iteration count and status
// (the rules of CGSolver::solve_with_jacobi, src/numeric/iterative_solvers.cpp
// :424-503), blocks that finish stop consuming bandwidth, and the whole batch
// runs as one CUDA graph: a device while-loop that ends when every block is
// done (or a body bound independent of the solver state is reached).
//
// Layout: SELL-32 per block.  Rows of each block are sorted by length inside
// windows of 4096 rows that never cross a block boundary, and each block is
// padded to a multiple of 32 rows, so every 32-row slice belongs to exactly
// one block.  A CTA owns a contiguous range of slices (balanced by stored
// slots, at most kMaxLocal blocks per CTA); per-block dot products are summed
// per CTA in a fixed order, written as one partial per (CTA, block) segment,
// and the last CTA to finish (atomic ticket) sums each block's segments in
// order -- deterministic results for a fixed partition.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "device.h"
#include "trace.h"

namespace emg {

namespace {

constexpr int kBThreads = 512;
constexpr int kBWarps = kBThreads / 32;
constexpr int kMaxLocal = 64;   // blocks touched by one CTA
constexpr int kWindowB = 4096;  // length-sort window (inside a block)
constexpr int kBodyB = 4;       // iterations per while-loop body
// CTAs per SM the slices are split into (each CTA ~ the same number of
// slots).  A CTA whose blocks have all converged returns at once, so more,
// smaller CTAs let the block scheduler spread the blocks still iterating
// over the whole GPU.
#ifndef EMG_BATCH_CTAS_PER_SM
#define EMG_BATCH_CTAS_PER_SM 4
#endif

}  // namespace

struct BatchPlan {
  int64_t n = 0, N = 0, nslices = 0, slots = 0;
  int32_t nb = 0, nctas = 0, nsegs = 0;
  std::vector<int64_t> blocks;   // host copy of the block row partition
  uint64_t version = ~uint64_t(0);
  // device arrays
  int32_t* perm = nullptr;        // new row -> old row, -1 = padding (N)
  int64_t* slice_ptr = nullptr;   // nslices + 1
  int32_t* slice_inst = nullptr;  // block of every slice
  int32_t* cta_slice = nullptr;   // nctas + 1 slice ranges
  int32_t* cta_seg = nullptr;     // first segment id of every CTA
  int32_t* inst_seg = nullptr;    // nb + 1 segment ranges per block
  int32_t* col = nullptr;
  int32_t* src = nullptr;
  double* val = nullptr;
  // workspace
  double *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr, *dinv = nullptr;
  double* partial = nullptr;      // 2 * nsegs
  // per-block state (structure of arrays)
  double *bnorm = nullptr, *rz = nullptr, *alpha = nullptr, *beta = nullptr, *res = nullptr,
         *prev = nullptr;
  int32_t *iter = nullptr, *status = nullptr, *done = nullptr;
  int32_t* ctl = nullptr;         // [0] ticket, [1] active, [2] loops, [3] loop limit, [4] max_iter
  double* tol = nullptr;          // [0]
  cudaStream_t cap = nullptr;
  cudaGraphExec_t loop = nullptr;
  ~BatchPlan();
};

namespace {

struct View {
  int64_t N;
  int32_t nb;
  const int32_t* perm;
  const int64_t* slice_ptr;
  const int32_t* slice_inst;
  const int32_t* cta_slice;
  const int32_t* cta_seg;
  const int32_t* inst_seg;
  const int32_t* col;
  const double* val;
  double *x, *r, *z, *p, *q, *dinv, *partial;
  double *bnorm, *rz, *alpha, *beta, *res, *prev;
  int32_t *iter, *status, *done, *ctl;
  const double* tol;
};

View view_of(const BatchPlan& P) {
  View v;
  v.N = P.N; v.nb = P.nb; v.perm = P.perm; v.slice_ptr = P.slice_ptr; v.slice_inst = P.slice_inst;
  v.cta_slice = P.cta_slice; v.cta_seg = P.cta_seg; v.inst_seg = P.inst_seg; v.col = P.col; v.val = P.val;
  v.x = P.x; v.r = P.r; v.z = P.z; v.p = P.p; v.q = P.q; v.dinv = P.dinv; v.partial = P.partial;
  v.bnorm = P.bnorm; v.rz = P.rz; v.alpha = P.alpha; v.beta = P.beta; v.res = P.res; v.prev = P.prev;
  v.iter = P.iter; v.status = P.status; v.done = P.done; v.ctl = P.ctl; v.tol = P.tol;
  return v;
}

// Per-CTA accumulation of per-block sums: acc[warp][local][k] in shared memory.
template <int K>
struct Acc {
  double (*a)[kMaxLocal][K];
  int first;  // first block of this CTA
};

// Runs body(slice, block, local, lane) -> contributions[K] for every slice of
// this CTA whose block is still active (or every slice when all_blocks), adds
// the warp-reduced contributions per block, and on the last CTA calls
// fin(block, totals) for every block.  Returns after fin has run.
template <int K, bool kAll, class Body, class Fin>
__device__ __forceinline__ void sweep(const View& B, Body body, Fin fin) {
  __shared__ double acc[kBWarps][kMaxLocal][K];
  __shared__ bool last;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = blockIdx.x;
  const int s0 = B.cta_slice[c], s1 = B.cta_slice[c + 1];
  const int first = s0 < s1 ? B.slice_inst[s0] : 0;
  const int nlocal = s0 < s1 ? B.slice_inst[s1 - 1] - first + 1 : 0;
  for (int i = threadIdx.x; i < kBWarps * kMaxLocal * K; i += blockDim.x) (&acc[0][0][0])[i] = 0.0;
  __syncthreads();
  for (int s = s0 + w; s < s1; s += kBWarps) {
    const int inst = B.slice_inst[s];
    if (!kAll && B.done[inst]) continue;
    double v[K];
    body(s, inst, lane, v);
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0)
#pragma unroll
      for (int k = 0; k < K; ++k) acc[w][inst - first][k] += v[k];
  }
  __syncthreads();
  for (int t = threadIdx.x; t < nlocal * K; t += blockDim.x) {
    const int l = t / K, k = t % K;
    double s = 0.0;
    for (int ww = 0; ww < kBWarps; ++ww) s += acc[ww][l][k];
    B.partial[(B.cta_seg[c] + l) * K + k] = s;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(reinterpret_cast<unsigned*>(&B.ctl[0]), 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int i = threadIdx.x; i < B.nb; i += blockDim.x) {
    if (!kAll && B.done[i]) continue;
    double tot[K];
#pragma unroll
    for (int k = 0; k < K; ++k) tot[k] = 0.0;
    for (int sg = B.inst_seg[i]; sg < B.inst_seg[i + 1]; ++sg)
#pragma unroll
      for (int k = 0; k < K; ++k) tot[k] += ld_l2(B.partial + sg * K + k);
    fin(i, tot);
  }
  __syncthreads();
  if (threadIdx.x == 0) B.ctl[0] = 0;
}

__global__ void k_b_jacobi(View B, const int32_t* __restrict__ rp, const int32_t* __restrict__ col,
                           const double* __restrict__ val, int precond) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < B.N;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double d = 1.0;
    const int32_t o = B.perm[i];
    if (precond && o >= 0) {
      int32_t lo = rp[o], hi = rp[o + 1];
      while (lo < hi) {
        const int32_t mid = (lo + hi) >> 1;
        if (col[mid] < o) lo = mid + 1; else hi = mid;
      }
      const double a = (lo < rp[o + 1] && col[lo] == o) ? val[lo] : 0.0;
      d = fabs(a) > 1e-15 ? 1.0 / a : 1.0;
    }
    B.dinv[i] = d;
  }
}

__global__ void __launch_bounds__(kBThreads) k_b_init(View B, const double* __restrict__ b) {
  sweep<2, true>(
      B,
      [&](int s, int, int lane, double* v) {
        const int64_t row = static_cast<int64_t>(s) * 32 + lane;
        const int32_t o = B.perm[row];
        const double bi = o >= 0 ? b[o] : 0.0, zi = B.dinv[row] * bi;
        B.x[row] = 0.0; B.r[row] = bi; B.z[row] = zi; B.p[row] = zi; B.q[row] = 0.0;
        v[0] = bi * bi;
        v[1] = bi * zi;
      },
      [&](int i, const double* tot) {
        const double bn = sqrt(tot[0]);
        const int32_t max_iter = B.ctl[4];
        B.bnorm[i] = bn;
        B.rz[i] = tot[1];
        B.iter[i] = 1;
        B.status[i] = EMG_MAX_ITER_REACHED;
        B.done[i] = 0;
        if (bn < 1e-15) {  // iterative_solvers.cpp:440-446
          B.status[i] = EMG_SUCCESS; B.iter[i] = 0; B.res[i] = 0.0; B.done[i] = 1;
        } else {
          B.res[i] = sqrt(tot[0]) / bn;
          B.prev[i] = B.res[i];
          if (max_iter < 1) { B.iter[i] = max_iter; B.done[i] = 1; }
        }
      });
}

// q = A p and p.q per block -> alpha (or breakdown)
// 1: the batched SpMV keeps the next batch of loads in flight (as the
// single-system SELL kernel does); 0: one batch at a time.
#ifndef EMG_BATCH_PIPE
#define EMG_BATCH_PIPE 1
#endif

__global__ void __launch_bounds__(kBThreads) k_b_spmv_dot(View B) {
  if (B.ctl[1] == 0) return;
  const uint64_t pol = evict_first_policy();
  sweep<1, false>(
      B,
      [&](int s, int, int lane, double* v) {
        const int64_t b0 = B.slice_ptr[s];
        const int len = static_cast<int>((B.slice_ptr[s + 1] - b0) >> 5);
        const int64_t base = b0 + lane;
        double sum = 0.0;
#if !EMG_BATCH_PIPE
        int j = 0;
        for (; j + 4 <= len; j += 4) {
          const int64_t k = base + 32 * j;
          int cc[4];
          double vv[4], xx[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            cc[u] = ld_stream(B.col + k + 32 * u, pol);
            vv[u] = ld_stream(B.val + k + 32 * u, pol);
          }
#pragma unroll
          for (int u = 0; u < 4; ++u) xx[u] = B.p[cc[u]];
#pragma unroll
          for (int u = 0; u < 4; ++u) sum += vv[u] * xx[u];
        }
        for (; j < len; ++j) {
          const int64_t k = base + 32 * j;
          sum += ld_stream(B.val + k, pol) * B.p[ld_stream(B.col + k, pol)];
        }
#else
        // the next batch of 4 columns / values is in flight while this batch
        // gathers p; entries past the row length are masked and add +0 last
        const int nbt = (len + 3) >> 2;
        int cn[4];
        double vn[4];
        auto fetch = [&](int jb) {
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const bool in = jb + u < len;
            const int64_t k = base + 32 * static_cast<int64_t>(jb + u);
            cn[u] = in ? ld_stream(B.col + k, pol) : 0;
            vn[u] = in ? ld_stream(B.val + k, pol) : 0.0;
          }
        };
        if (nbt > 0) fetch(0);
        for (int bt = 0; bt < nbt; ++bt) {
          int cc[4];
          double vv[4], xx[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) { cc[u] = cn[u]; vv[u] = vn[u]; }
          if (bt + 1 < nbt) fetch(4 * (bt + 1));
#pragma unroll
          for (int u = 0; u < 4; ++u) xx[u] = B.p[cc[u]];
#pragma unroll
          for (int u = 0; u < 4; ++u) sum += vv[u] * xx[u];
        }
#endif
        const int64_t row = static_cast<int64_t>(s) * 32 + lane;
        B.q[row] = sum;
        v[0] = B.p[row] * sum;
      },
      [&](int i, const double* tot) {
        if (fabs(tot[0]) < 1e-30) {  // :453-457
          B.status[i] = EMG_NUMERICAL_ERROR;
          B.done[i] = 1;
        } else {
          B.alpha[i] = B.rz[i] / tot[0];
        }
      });
}

__global__ void __launch_bounds__(kBThreads) k_b_update(View B) {
  if (B.ctl[1] == 0) return;
  sweep<2, false>(
      B,
      [&](int s, int inst, int lane, double* v) {
        const int64_t row = static_cast<int64_t>(s) * 32 + lane;
        const double a = B.alpha[inst];
        B.x[row] += a * B.p[row];
        const double ri = B.r[row] - a * B.q[row];
        const double zi = B.dinv[row] * ri;
        B.r[row] = ri;
        B.z[row] = zi;
        v[0] = ri * zi;
        v[1] = ri * ri;
      },
      [&](int i, const double* tot) {
        const int it = B.iter[i];
        const double res = sqrt(tot[1]) / B.bnorm[i];
        B.res[i] = res;
        if (res < B.tol[0]) {
          B.status[i] = EMG_SUCCESS; B.done[i] = 1;
        } else if (it > 10 && res > B.prev[i] * 1000.0) {  // :477-483
          B.status[i] = EMG_DIVERGED; B.done[i] = 1;
        } else {
          B.beta[i] = tot[0] / B.rz[i];
          B.rz[i] = tot[0];
          B.prev[i] = res;
          if (it >= B.ctl[4]) { B.status[i] = EMG_MAX_ITER_REACHED; B.done[i] = 1; }
          else B.iter[i] = it + 1;
        }
      });
}

__global__ void __launch_bounds__(kBThreads) k_b_direction(View B) {
  if (B.ctl[1] == 0) return;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = blockIdx.x;
  for (int s = B.cta_slice[c] + w; s < B.cta_slice[c + 1]; s += kBWarps) {
    const int inst = B.slice_inst[s];
    if (B.done[inst]) continue;
    const int64_t row = static_cast<int64_t>(s) * 32 + lane;
    B.p[row] = B.z[row] + B.beta[inst] * B.p[row];
  }
}

// Counts active blocks and steers the device while-loop.
__global__ void k_b_control(View B, cudaGraphConditionalHandle handle) {
  __shared__ int cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  int mine = 0;
  for (int i = threadIdx.x; i < B.nb; i += blockDim.x) mine += B.done[i] ? 0 : 1;
  atomicAdd(&cnt, mine);
  __syncthreads();
  if (threadIdx.x == 0) {
    B.ctl[1] = cnt;
    const int loops = B.ctl[2] + 1;
    B.ctl[2] = loops;
    cudaGraphSetConditional(handle, (cnt > 0 && loops < B.ctl[3]) ? 1u : 0u);
  }
}

__global__ void k_b_active(View B) {
  __shared__ int cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  int mine = 0;
  for (int i = threadIdx.x; i < B.nb; i += blockDim.x) mine += B.done[i] ? 0 : 1;
  atomicAdd(&cnt, mine);
  __syncthreads();
  if (threadIdx.x == 0) B.ctl[1] = cnt;
}

// Warp per slice: permuted column (via iperm) and CSR source per slot.
__global__ void k_b_fill(int64_t nslices, const int64_t* __restrict__ sp, const int32_t* __restrict__ perm,
                         const int32_t* __restrict__ iperm, const int32_t* __restrict__ rp,
                         const int32_t* __restrict__ ccol, int32_t* __restrict__ col,
                         int32_t* __restrict__ src) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5;
  const int64_t nwarps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t s = warp; s < nslices; s += nwarps) {
    const int64_t b0 = sp[s];
    const int len = static_cast<int>((sp[s + 1] - b0) >> 5);
    const int64_t row = s * 32 + lane;
    const int32_t o = perm[row];
    int32_t a = 0, rl = 0;
    if (o >= 0) { a = rp[o]; rl = rp[o + 1] - a; }
    for (int j = 0; j < len; ++j) {
      const int64_t k = b0 + 32 * j + lane;
      if (j < rl) { col[k] = iperm[ccol[a + j]]; src[k] = a + j; }
      else { col[k] = static_cast<int32_t>(row); src[k] = -1; }
    }
  }
}

__global__ void k_b_values(int64_t slots, const int32_t* __restrict__ src, const double* __restrict__ cval,
                           double* __restrict__ val) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < slots;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    val[i] = src[i] >= 0 ? cval[src[i]] : 0.0;
}

// Every column of a row lies inside the row's block.
// *bad = 1 if a row has a column outside its block (blocks: nb + 1 row
// offsets; the block of row i is the last k with blocks[k] <= i).
__global__ void k_b_check(int64_t n, const int32_t* __restrict__ rp, const int32_t* __restrict__ col,
                          int32_t nb, const int64_t* __restrict__ blocks, int32_t* __restrict__ bad) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int32_t a = 0, b = nb;  // blocks[a] <= i < blocks[b]
    while (b - a > 1) {
      const int32_t m = (a + b) >> 1;
      if (blocks[m] <= i) a = m; else b = m;
    }
    const int64_t lo = blocks[a], hi = blocks[a + 1];
    for (int32_t e = rp[i]; e < rp[i + 1]; ++e)
      if (col[e] < lo || col[e] >= hi) { atomicOr(bad, 1); break; }
  }
}

__global__ void k_b_scatter(int64_t N, const int32_t* __restrict__ perm, const double* __restrict__ in,
                            double* __restrict__ out) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < N;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    if (perm[i] >= 0) out[perm[i]] = in[i];
}

// Plan on the device.  Window w holds rows [row0[w], row0[w] + nrows[w]) of
// one block (at most kWindowB); a warp sorts them by descending length,
// stably (lengths of kLenCapB - 1 and more share the last bucket: the order
// only decides the padding), into perm[out0[w] ...].
constexpr int kLenCapB = 1024;
__global__ void __launch_bounds__(32) k_b_window_perm(const int64_t* __restrict__ row0,
                                                      const int32_t* __restrict__ nrows,
                                                      const int64_t* __restrict__ out0,
                                                      const int32_t* __restrict__ rp, int32_t* __restrict__ perm) {
  __shared__ int32_t cur[kLenCapB];  // bucket 0 = longest rows
  const int lane = threadIdx.x;
  const int64_t w0 = row0[blockIdx.x], w1 = w0 + nrows[blockIdx.x], o0 = out0[blockIdx.x];
  for (int b = lane; b < kLenCapB; b += 32) cur[b] = 0;
  __syncwarp();
  for (int64_t i = w0 + lane; i < w1; i += 32) {
    const int len = rp[i + 1] - rp[i];
    atomicAdd(&cur[kLenCapB - 1 - (len < kLenCapB - 1 ? len : kLenCapB - 1)], 1);
  }
  __syncwarp();
  constexpr int kPer = kLenCapB / 32;  // lane l owns buckets [l kPer, (l + 1) kPer)
  int local = 0;
  for (int k = 0; k < kPer; ++k) local += cur[lane * kPer + k];
  int incl = local;
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  int run = incl - local;
  for (int k = 0; k < kPer; ++k) {
    const int c = cur[lane * kPer + k];
    cur[lane * kPer + k] = run;
    run += c;
  }
  __syncwarp();
  for (int64_t base = w0; base < w1; base += 32) {  // 32 rows a round, ties ranked by lane
    const int64_t i = base + lane;
    const bool valid = i < w1;
    int b = -1 - lane;
    if (valid) {
      const int len = rp[i + 1] - rp[i];
      b = kLenCapB - 1 - (len < kLenCapB - 1 ? len : kLenCapB - 1);
    }
    const unsigned grp = __match_any_sync(0xffffffffu, b);
    const int rank = __popc(grp & ((1u << lane) - 1u));
    const int pos = valid ? cur[b] + rank : 0;
    __syncwarp();
    if (valid && rank == 0) cur[b] += __popc(grp);
    __syncwarp();
    if (valid) perm[o0 + pos] = static_cast<int32_t>(i);
  }
}

// Warp per slice: slots = 32 x the longest row of the slice (padding rows,
// perm -1, count 0).
__global__ void k_b_slice_slots(int64_t ns, const int32_t* __restrict__ perm, const int32_t* __restrict__ rp,
                                int32_t* __restrict__ slots) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t s = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5; s < ns; s += nw) {
    const int32_t o = perm[s * 32 + lane];
    const int len = o >= 0 ? rp[o + 1] - rp[o] : 0;
    const int mx = __reduce_max_sync(0xffffffffu, len);
    if (lane == 0) slots[s] = 32 * mx;
  }
}

__global__ void k_b_widen_iperm(int64_t ns, const int32_t* __restrict__ off, int64_t* __restrict__ sp,
                                int64_t N, const int32_t* __restrict__ perm, int32_t* __restrict__ iperm) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t t0 = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  for (int64_t i = t0; i <= ns; i += stride) sp[i] = off[i];
  for (int64_t i = t0; i < N; i += stride)
    if (perm[i] >= 0) iperm[perm[i]] = static_cast<int32_t>(i);
}

int launch_grid(int64_t work) {
  int64_t b = (work + 255) / 256;
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(b, 148 * 8)));
}

template <class T>
int dalloc(T** p, int64_t count, cudaStream_t st) {
  EMG_CK(cudaMallocAsync(reinterpret_cast<void**>(p), sizeof(T) * std::max<int64_t>(count, 1), st));
  return EMG_SUCCESS;
}

// Host plan: per-block length sort, padding, slices, CTA ranges, segments.
int build_plan(DevCsr& A, const std::vector<int64_t>& blocks, cudaStream_t st, BatchPlan& P) {
  const int64_t n = A.n;
  const int32_t nb = static_cast<int32_t>(blocks.size()) - 1;
  // new numbering: every block padded to a multiple of 32 rows
  std::vector<int64_t> nstart(nb + 1, 0);
  for (int32_t k = 0; k < nb; ++k) nstart[k + 1] = nstart[k] + ((blocks[k + 1] - blocks[k] + 31) / 32) * 32;
  const int64_t N = nstart[nb];
  const int64_t ns = N / 32;
  if (N >= (int64_t(1) << 31)) {
    set_error("batch too large for the solver format");
    return EMG_INVALID_INPUT;
  }
  // length-sort windows inside the blocks
  std::vector<int64_t> wrow, wout;
  std::vector<int32_t> wlen;
  for (int32_t k = 0; k < nb; ++k)
    for (int64_t w0 = blocks[k]; w0 < blocks[k + 1]; w0 += kWindowB) {
      wrow.push_back(w0);
      wlen.push_back(static_cast<int32_t>(std::min<int64_t>(blocks[k + 1] - w0, kWindowB)));
      wout.push_back(nstart[k] + (w0 - blocks[k]));
    }
  const int64_t nwin = static_cast<int64_t>(wrow.size());
  int32_t *d_iperm = nullptr, *d_slots = nullptr, *d_off = nullptr, *d_wlen = nullptr;
  int64_t *d_wrow = nullptr, *d_wout = nullptr;
  int rc = dalloc(&P.perm, N, st);
  if (!rc) rc = dalloc(&d_iperm, n, st);
  if (!rc) rc = dalloc(&P.slice_ptr, ns + 1, st);
  if (!rc) rc = dalloc(&d_slots, ns, st);
  if (!rc) rc = dalloc(&d_off, ns + 1, st);
  if (!rc) rc = dalloc(&d_wrow, nwin, st);
  if (!rc) rc = dalloc(&d_wout, nwin, st);
  if (!rc) rc = dalloc(&d_wlen, nwin, st);
  if (rc) return rc;
  EMG_CK(cudaMemsetAsync(P.perm, 0xff, sizeof(int32_t) * std::max<int64_t>(N, 1), st));
  if (nwin > 0) {
    EMG_CK(cudaMemcpyAsync(d_wrow, wrow.data(), sizeof(int64_t) * nwin, cudaMemcpyHostToDevice, st));
    EMG_CK(cudaMemcpyAsync(d_wout, wout.data(), sizeof(int64_t) * nwin, cudaMemcpyHostToDevice, st));
    EMG_CK(cudaMemcpyAsync(d_wlen, wlen.data(), sizeof(int32_t) * nwin, cudaMemcpyHostToDevice, st));
    k_b_window_perm<<<static_cast<unsigned>(nwin), 32, 0, st>>>(d_wrow, d_wlen, d_wout, A.row_ptr, P.perm);
  }
  if (ns > 0) k_b_slice_slots<<<launch_grid(ns * 32), 256, 0, st>>>(ns, P.perm, A.row_ptr, d_slots);
  EMG_CK(cudaGetLastError());
  int64_t total = 0;
  rc = scan_counts(d_slots, d_off, ns, &total, st);
  if (!rc && total >= (int64_t(1) << 31)) {
    set_error("batch too large for the solver format");
    rc = EMG_INVALID_INPUT;
  }
  if (!rc) {
    k_b_widen_iperm<<<launch_grid(N), 256, 0, st>>>(ns, d_off, P.slice_ptr, N, P.perm, d_iperm);
    if (cudaGetLastError() != cudaSuccess) { set_error("batch plan launch failed"); rc = EMG_ERR_CUDA; }
  }
  std::vector<int64_t> sp(ns + 1, 0);
  if (!rc && cudaMemcpyAsync(sp.data(), P.slice_ptr, sizeof(int64_t) * (ns + 1), cudaMemcpyDeviceToHost, st) !=
                 cudaSuccess) {
    set_error("batch plan copy failed");
    rc = EMG_ERR_CUDA;
  }
  for (void* p : {static_cast<void*>(d_slots), static_cast<void*>(d_off), static_cast<void*>(d_wrow),
                  static_cast<void*>(d_wout), static_cast<void*>(d_wlen)})
    cudaFreeAsync(p, st);
  if (cudaStreamSynchronize(st) != cudaSuccess && !rc) { set_error("batch plan failed"); rc = EMG_ERR_CUDA; }
  if (rc) { cudaFreeAsync(d_iperm, st); return rc; }
  std::vector<int32_t> sinst(ns);
  {
    int32_t k = 0;
    for (int64_t s2 = 0; s2 < ns; ++s2) {
      while (s2 * 32 >= nstart[k + 1]) ++k;
      sinst[s2] = k;
    }
  }
  // CTA ranges: contiguous slices, ~equal slots, at most kMaxLocal blocks each
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t parts = static_cast<int64_t>(EMG_BATCH_CTAS_PER_SM) * sms;
  const int64_t target = std::max<int64_t>(1, (sp[ns] + parts - 1) / parts);
  std::vector<int32_t> cs{0}, cseg;
  std::vector<int32_t> iseg_cnt(nb, 0);
  {
    int64_t acc = 0;
    int32_t first = ns > 0 ? sinst[0] : 0;
    for (int64_t s = 0; s < ns; ++s) {
      const bool split = s > cs.back() && (acc >= target || sinst[s] - first >= kMaxLocal);
      if (split) { cs.push_back(static_cast<int32_t>(s)); acc = 0; first = sinst[s]; }
      acc += sp[s + 1] - sp[s];
    }
    if (ns > 0) cs.push_back(static_cast<int32_t>(ns));
  }
  const int32_t nctas = static_cast<int32_t>(cs.size()) - 1;
  int32_t nsegs = 0;
  for (int32_t c = 0; c < nctas; ++c) {
    cseg.push_back(nsegs);
    const int32_t f = sinst[cs[c]], l = sinst[cs[c + 1] - 1];
    for (int32_t k = f; k <= l; ++k) iseg_cnt[k]++;
    nsegs += l - f + 1;
  }
  std::vector<int32_t> iseg(nb + 1, 0);
  for (int32_t k = 0; k < nb; ++k) iseg[k + 1] = iseg[k] + iseg_cnt[k];
  // a block without rows has no segments; its sums are 0 and it finishes at once
  P.n = n; P.N = N; P.nslices = ns; P.slots = sp[ns]; P.nb = nb; P.nctas = nctas; P.nsegs = nsegs;
  P.blocks = blocks;
  if (!rc) rc = dalloc(&P.slice_inst, ns, st);
  if (!rc) rc = dalloc(&P.cta_slice, nctas + 1, st);
  if (!rc) rc = dalloc(&P.cta_seg, nctas, st);
  if (!rc) rc = dalloc(&P.inst_seg, nb + 1, st);
  if (!rc) rc = dalloc(&P.col, P.slots, st);
  if (!rc) rc = dalloc(&P.src, P.slots, st);
  if (!rc) rc = dalloc(&P.val, P.slots, st);
  for (double** v : {&P.x, &P.r, &P.z, &P.p, &P.q, &P.dinv})
    if (!rc) rc = dalloc(v, N, st);
  if (!rc) rc = dalloc(&P.partial, 2 * static_cast<int64_t>(std::max(nsegs, 1)), st);
  for (double** v : {&P.bnorm, &P.rz, &P.alpha, &P.beta, &P.res, &P.prev})
    if (!rc) rc = dalloc(v, nb, st);
  for (int32_t** v : {&P.iter, &P.status, &P.done})
    if (!rc) rc = dalloc(v, nb, st);
  if (!rc) rc = dalloc(&P.ctl, 8, st);
  if (!rc) rc = dalloc(&P.tol, 1, st);
  if (rc) { cudaFreeAsync(d_iperm, st); return rc; }
  if (ns > 0) EMG_CK(cudaMemcpyAsync(P.slice_inst, sinst.data(), sizeof(int32_t) * ns, cudaMemcpyHostToDevice, st));
  EMG_CK(cudaMemcpyAsync(P.cta_slice, cs.data(), sizeof(int32_t) * (nctas + 1), cudaMemcpyHostToDevice, st));
  if (nctas > 0) EMG_CK(cudaMemcpyAsync(P.cta_seg, cseg.data(), sizeof(int32_t) * nctas, cudaMemcpyHostToDevice, st));
  EMG_CK(cudaMemcpyAsync(P.inst_seg, iseg.data(), sizeof(int32_t) * (nb + 1), cudaMemcpyHostToDevice, st));
  EMG_CK(cudaMemsetAsync(P.ctl, 0, sizeof(int32_t) * 8, st));
  if (ns > 0)
    k_b_fill<<<launch_grid(ns * 32), 256, 0, st>>>(ns, P.slice_ptr, P.perm, d_iperm, A.row_ptr, A.col, P.col, P.src);
  EMG_CK(cudaGetLastError());
  EMG_CK(cudaFreeAsync(d_iperm, st));
  EMG_CK(cudaStreamSynchronize(st));
  EMG_CK(cudaStreamCreate(&P.cap));
  P.version = ~uint64_t(0);
  return EMG_SUCCESS;
}

int capture_batch_loop(BatchPlan& P) {
  cudaGraph_t graph = nullptr;
  EMG_CK(cudaGraphCreate(&graph, 0));
  cudaGraphConditionalHandle handle;
  cudaError_t e = cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault);
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = handle;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  if (e == cudaSuccess) e = cudaGraphAddNode(&node, graph, nullptr, 0, &cp);
  if (e == cudaSuccess) {
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph(P.cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      const View v = view_of(P);
      for (int k = 0; k < kBodyB; ++k) {
        k_b_spmv_dot<<<P.nctas, kBThreads, 0, P.cap>>>(v);
        k_b_update<<<P.nctas, kBThreads, 0, P.cap>>>(v);
        k_b_direction<<<P.nctas, kBThreads, 0, P.cap>>>(v);
      }
      k_b_control<<<1, 256, 0, P.cap>>>(v, handle);
      e = cudaStreamEndCapture(P.cap, &body);
    }
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&P.loop, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error(std::string("batch while-loop graph: ") + cudaGetErrorString(e));
    return EMG_ERR_CUDA;
  }
  return EMG_SUCCESS;
}

}  // namespace

BatchPlan::~BatchPlan() {
  if (loop) cudaGraphExecDestroy(loop);
  for (void* p : {static_cast<void*>(perm), static_cast<void*>(slice_ptr), static_cast<void*>(slice_inst),
                  static_cast<void*>(cta_slice), static_cast<void*>(cta_seg), static_cast<void*>(inst_seg),
                  static_cast<void*>(col), static_cast<void*>(src), static_cast<void*>(val),
                  static_cast<void*>(x), static_cast<void*>(r), static_cast<void*>(z), static_cast<void*>(p),
                  static_cast<void*>(q), static_cast<void*>(dinv), static_cast<void*>(partial),
                  static_cast<void*>(bnorm), static_cast<void*>(rz), static_cast<void*>(alpha),
                  static_cast<void*>(beta), static_cast<void*>(res), static_cast<void*>(prev),
                  static_cast<void*>(iter), static_cast<void*>(status), static_cast<void*>(done),
                  static_cast<void*>(ctl), static_cast<void*>(tol)})
    if (p) cudaFreeAsync(p, 0);
  if (cap) cudaStreamDestroy(cap);
}

void free_batch(BatchPlan* p) { delete p; }

int batch_cg_solve(DevCsr& A, int32_t nb, const int64_t* blocks_in, const double* b, double* x,
                   const emg_krylov_config& cfg, cudaStream_t user, emg_result* results) {
  if (nb <= 0 || !blocks_in || !b || !x || !results) {
    set_error("batch solve: bad arguments");
    return EMG_INVALID_INPUT;
  }
  if (check_krylov_precond(cfg.preconditioner)) return EMG_INVALID_INPUT;
  std::vector<int64_t> blocks(blocks_in, blocks_in + nb + 1);
  if (blocks[0] != 0 || blocks[nb] != A.n) {
    set_error("batch solve: block partition must start at 0 and end at n");
    return EMG_INVALID_INPUT;
  }
  for (int32_t k = 0; k < nb; ++k)
    if (blocks[k + 1] < blocks[k]) { set_error("batch solve: block partition not monotone"); return EMG_INVALID_INPUT; }
  cudaStream_t st = user;
  if (!A.batch || A.batch->blocks != blocks) {
    TraceScope trace_setup("batch.setup");
    // block-diagonal check on the device
    int32_t* d_bad = nullptr;
    int64_t* d_blocks = nullptr;
    EMG_CK(cudaMallocAsync(&d_blocks, sizeof(int64_t) * (nb + 1), st));
    EMG_CK(cudaMallocAsync(&d_bad, sizeof(int32_t), st));
    EMG_CK(cudaMemcpyAsync(d_blocks, blocks.data(), sizeof(int64_t) * (nb + 1), cudaMemcpyHostToDevice, st));
    EMG_CK(cudaMemsetAsync(d_bad, 0, sizeof(int32_t), st));
    k_b_check<<<launch_grid(A.n), 256, 0, st>>>(A.n, A.row_ptr, A.col, nb, d_blocks, d_bad);
    int32_t bad = 0;
    EMG_CK(cudaMemcpyAsync(&bad, d_bad, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    EMG_CK(cudaStreamSynchronize(st));
    for (void* p : {static_cast<void*>(d_blocks), static_cast<void*>(d_bad)}) EMG_CK(cudaFreeAsync(p, st));
    if (bad) { set_error("batch solve: the matrix couples different blocks"); return EMG_INVALID_INPUT; }
    free_batch(A.batch);
    A.batch = new BatchPlan();
    TraceScope trace_plan("batch.plan");
    int rc = build_plan(A, blocks, st, *A.batch);
    if (rc) { free_batch(A.batch); A.batch = nullptr; return rc; }
  }
  BatchPlan& P = *A.batch;
  if (P.version != A.version) {
    if (P.slots > 0) k_b_values<<<launch_grid(P.slots), 256, 0, st>>>(P.slots, P.src, A.val, P.val);
    EMG_CK(cudaGetLastError());
    P.version = A.version;
  }
  if (!P.loop) {
    TraceScope trace_capture("batch.capture");
    int rc = capture_batch_loop(P);
    if (rc) return rc;
  }
  const int32_t max_iter = cfg.max_iterations;
  const int32_t ctl[8] = {0, 1, 0, (max_iter > 0 ? max_iter : 0) / kBodyB + 2, max_iter, 0, 0, 0};
  const auto t0 = std::chrono::steady_clock::now();
  cudaEvent_t e0, e1;
  EMG_CK(cudaEventCreate(&e0));
  EMG_CK(cudaEventCreate(&e1));
  EMG_CK(cudaEventRecord(e0, st));
  EMG_CK(cudaMemcpyAsync(P.ctl, ctl, sizeof(ctl), cudaMemcpyHostToDevice, st));
  EMG_CK(cudaMemcpyAsync(P.tol, &cfg.tolerance, sizeof(double), cudaMemcpyHostToDevice, st));
  const View v = view_of(P);
  k_b_jacobi<<<launch_grid(P.N), 256, 0, st>>>(v, A.row_ptr, A.col, A.val, cfg.preconditioner);
  if (P.nctas > 0) k_b_init<<<P.nctas, kBThreads, 0, st>>>(v, b);
  k_b_active<<<1, 256, 0, st>>>(v);
  EMG_CK(cudaGetLastError());
  EMG_CK(cudaGraphLaunch(P.loop, st));
  k_b_scatter<<<launch_grid(P.N), 256, 0, st>>>(P.N, P.perm, P.x, x);
  EMG_CK(cudaEventRecord(e1, st));
  std::vector<int32_t> it(nb), stt(nb), dn(nb);
  std::vector<double> rs(nb);
  int32_t hctl[8];
  EMG_CK(cudaMemcpyAsync(it.data(), P.iter, sizeof(int32_t) * nb, cudaMemcpyDeviceToHost, st));
  EMG_CK(cudaMemcpyAsync(stt.data(), P.status, sizeof(int32_t) * nb, cudaMemcpyDeviceToHost, st));
  EMG_CK(cudaMemcpyAsync(dn.data(), P.done, sizeof(int32_t) * nb, cudaMemcpyDeviceToHost, st));
  EMG_CK(cudaMemcpyAsync(rs.data(), P.res, sizeof(double) * nb, cudaMemcpyDeviceToHost, st));
  EMG_CK(cudaMemcpyAsync(hctl, P.ctl, sizeof(hctl), cudaMemcpyDeviceToHost, st));
  EMG_CK(cudaStreamSynchronize(st));
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  (void)t0;
  int worst = EMG_SUCCESS;
  for (int32_t k = 0; k < nb; ++k) {
    results[k].status = dn[k] ? stt[k] : EMG_ERR_INTERNAL;
    results[k].iterations = it[k];
    results[k].residual_norm = rs[k];
    results[k].solve_time_ms = ms;
    if (results[k].status != EMG_SUCCESS && worst == EMG_SUCCESS) worst = results[k].status;
  }
  if (hctl[1] != 0) {
    set_error("batch solve: the device loop stopped at its bound with unfinished blocks");
    return EMG_ERR_INTERNAL;
  }
  return worst;
}

}  // namespace emg

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
// one block.  The blocks still iterating are listed once per loop body (a
// block that finishes inside a body is skipped until the next list); the
// slices of the listed blocks are split into equal contiguous shares, one
// per warp of a one-wave grid, so the remaining work always spreads over the
// whole GPU.  Every slice writes its own dot-product partials; a warp per
// block then adds them in slice order -- results do not depend on the grid
// or on which blocks are still iterating.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "device.h"
#include "tune.h"
#include "trace.h"

namespace emg {

namespace {

constexpr int kBT = 256;        // threads of the slice kernels
constexpr int kWindowB = 4096;  // length-sort window (inside a block)
constexpr int kBodyB = 4;       // iterations per while-loop body

}  // namespace

struct BatchPlan {
  int64_t n = 0, N = 0, nslices = 0, slots = 0;
  int32_t nb = 0;
  int grid_spmv = 0, grid_vec = 0;  // one-wave grids of the slice kernels
  bool tuned = false;               // grid_spmv chosen by the autotuner (first solve)
  std::vector<int64_t> blocks;      // host copy of the block row partition
  uint64_t version = ~uint64_t(0);
  // device arrays
  int32_t* perm = nullptr;        // new row -> old row, -1 = padding (N)
  int64_t* slice_ptr = nullptr;   // nslices + 1
  int32_t* inst_slice = nullptr;  // nb + 1: slices of block k are [inst_slice[k], inst_slice[k + 1])
  int32_t* act_inst = nullptr;    // nb: blocks still iterating, ascending
  int32_t* act_start = nullptr;   // nb + 1: their first slice in the active-slice numbering
  int32_t* col = nullptr;
  int32_t* src = nullptr;
  double* val = nullptr;
  // workspace
  double *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr, *dinv = nullptr;
  double* partial = nullptr;      // 2 * nslices: per-slice sums
  // per-block state (structure of arrays)
  double *bnorm = nullptr, *rz = nullptr, *alpha = nullptr, *beta = nullptr, *res = nullptr,
         *prev = nullptr;
  int32_t *iter = nullptr, *status = nullptr, *done = nullptr;
  // [1] active blocks, [2] loops, [3] loop limit, [4] max_iter, [5] listed blocks, [6] listed slices
  int32_t* ctl = nullptr;
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
  const int32_t* inst_slice;
  int32_t* act_inst;
  int32_t* act_start;
  const int32_t* col;
  const double* val;
  double *x, *r, *z, *p, *q, *dinv, *partial;
  double *bnorm, *rz, *alpha, *beta, *res, *prev;
  int32_t *iter, *status, *done, *ctl;
  const double* tol;
};

View view_of(const BatchPlan& P) {
  View v;
  v.N = P.N; v.nb = P.nb; v.perm = P.perm; v.slice_ptr = P.slice_ptr; v.inst_slice = P.inst_slice;
  v.act_inst = P.act_inst; v.act_start = P.act_start; v.col = P.col; v.val = P.val;
  v.x = P.x; v.r = P.r; v.z = P.z; v.p = P.p; v.q = P.q; v.dinv = P.dinv; v.partial = P.partial;
  v.bnorm = P.bnorm; v.rz = P.rz; v.alpha = P.alpha; v.beta = P.beta; v.res = P.res; v.prev = P.prev;
  v.iter = P.iter; v.status = P.status; v.done = P.done; v.ctl = P.ctl; v.tol = P.tol;
  return v;
}

// The slices of the listed blocks (ctl[6] of them, numbered block after
// block) are split into equal contiguous shares, one per warp of the grid,
// so the work of the blocks still iterating spreads over the whole GPU
// however few they are.  body(slice, block, lane) runs for every slice of a
// block that is not done (blocks finish only between launches).
template <class Body>
__device__ __forceinline__ void active_slices(const View& B, Body body) {
  const int64_t total = B.ctl[6];
  const int nact = B.ctl[5];
  const int lane = threadIdx.x & 31;
  const int64_t nw = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  const int64_t gw = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5;
  const int64_t a = total * gw / nw, b = total * (gw + 1) / nw;
  if (a >= b) return;
  int lo = 0, hi = nact;  // act_start[lo] <= a < act_start[hi]
  while (hi - lo > 1) {
    const int m = (lo + hi) >> 1;
    if (B.act_start[m] <= a) lo = m; else hi = m;
  }
  int j = lo;
  int inst = B.act_inst[j];
  int64_t next = B.act_start[j + 1];
  int64_t s = B.inst_slice[inst] + (a - B.act_start[j]);
  bool live = !B.done[inst];
  for (int64_t t = a; t < b; ++t, ++s) {
    while (t == next) {  // a listed block without rows is passed over
      ++j;
      inst = B.act_inst[j];
      next = B.act_start[j + 1];
      s = B.inst_slice[inst];
      live = !B.done[inst];
    }
    if (live) body(s, inst, lane);
  }
}

// Warp per listed block that is not done: the block's per-slice sums added
// in slice order (lane-strided, then a fixed butterfly), then fin(block, tot).
template <int K, bool kAll, class Fin>
__device__ __forceinline__ void finish_blocks(const View& B, Fin fin) {
  const int lane = threadIdx.x & 31;
  const int nact = B.ctl[5];
  const int64_t nw = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t j = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5; j < nact; j += nw) {
    const int inst = B.act_inst[j];
    if (!kAll && B.done[inst]) continue;
    double t[K];
#pragma unroll
    for (int k = 0; k < K; ++k) t[k] = 0.0;
    // 8 slices a lane in flight, added in slice order
    constexpr int kU = 8;
    const int64_t s1 = B.inst_slice[inst + 1];
    for (int64_t s0 = B.inst_slice[inst] + lane; s0 < s1; s0 += 32 * kU) {
      double v[kU][K];
#pragma unroll
      for (int u = 0; u < kU; ++u)
#pragma unroll
        for (int k = 0; k < K; ++k) v[u][k] = s0 + 32 * u < s1 ? B.partial[(s0 + 32 * u) * K + k] : 0.0;
#pragma unroll
      for (int u = 0; u < kU; ++u)
#pragma unroll
        for (int k = 0; k < K; ++k) t[k] += v[u][k];
    }
#pragma unroll
    for (int k = 0; k < K; ++k) t[k] = warp_sum(t[k]);
    if (lane == 0) fin(inst, t);
  }
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

// Lists the blocks that are not done (act_inst, act_start, ctl[5], ctl[6]),
// sets ctl[1] = their count and, with kSteer, counts a loop body and steers
// the device while-loop.  One CTA of 1024 threads, blocks in chunks of 1024.
template <bool kSteer>
__global__ void __launch_bounds__(1024) k_b_list(View B, cudaGraphConditionalHandle handle) {
  __shared__ int32_t wc[32], ws[32];
  __shared__ int32_t carry_c, carry_s;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (threadIdx.x == 0) { carry_c = 0; carry_s = 0; }
  __syncthreads();
  for (int base = 0; base < B.nb; base += 1024) {
    const int i = base + static_cast<int>(threadIdx.x);
    const int f = (i < B.nb && !B.done[i]) ? 1 : 0;
    const int sl = f ? B.inst_slice[i + 1] - B.inst_slice[i] : 0;
    int ic = f, is = sl;  // warp inclusive scans
    for (int o = 1; o < 32; o <<= 1) {
      const int vc = __shfl_up_sync(0xffffffffu, ic, o), vs = __shfl_up_sync(0xffffffffu, is, o);
      if (lane >= o) { ic += vc; is += vs; }
    }
    if (lane == 31) { wc[w] = ic; ws[w] = is; }
    __syncthreads();
    if (w == 0) {
      int c = wc[lane], t = ws[lane];
      for (int o = 1; o < 32; o <<= 1) {
        const int vc = __shfl_up_sync(0xffffffffu, c, o), vs = __shfl_up_sync(0xffffffffu, t, o);
        if (lane >= o) { c += vc; t += vs; }
      }
      wc[lane] = c - wc[lane];  // exclusive warp offsets
      ws[lane] = t - ws[lane];
    }
    __syncthreads();
    if (f) {
      const int pc = carry_c + wc[w] + ic - f;
      B.act_inst[pc] = i;
      B.act_start[pc] = carry_s + ws[w] + is - sl;
    }
    __syncthreads();
    if (threadIdx.x == 1023) { carry_c += wc[w] + ic; carry_s += ws[w] + is; }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    B.act_start[carry_c] = carry_s;
    B.ctl[5] = carry_c;
    B.ctl[6] = carry_s;
    B.ctl[1] = carry_c;
    if constexpr (kSteer) {
      const int loops = B.ctl[2] + 1;
      B.ctl[2] = loops;
      cudaGraphSetConditional(handle, (carry_c > 0 && loops < B.ctl[3]) ? 1u : 0u);
    }
  }
}

// x = 0, r = b, z = p = D^-1 b; per-slice b.b and b.z
__global__ void __launch_bounds__(kBT) k_b_init(View B, const double* __restrict__ b) {
  active_slices(B, [&](int64_t s, int, int lane) {
    const int64_t row = s * 32 + lane;
    const int32_t o = B.perm[row];
    const double bi = o >= 0 ? b[o] : 0.0, zi = B.dinv[row] * bi;
    B.x[row] = 0.0; B.r[row] = bi; B.z[row] = zi; B.p[row] = zi; B.q[row] = 0.0;
    const double bb = warp_sum(bi * bi), bz = warp_sum(bi * zi);
    if (lane == 0) { B.partial[2 * s] = bb; B.partial[2 * s + 1] = bz; }
  });
}

__global__ void __launch_bounds__(kBT) k_b_fin_init(View B) {
  finish_blocks<2, true>(B, [&](int i, const double* tot) {
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

// Walks the warp's share of the listed slices (as active_slices), stopping
// only at slices of blocks that are not done.
struct SliceCursor {
  int64_t t, end, next, s;
  int j, inst;
  __device__ __forceinline__ bool init(const View& B) {
    const int64_t total = B.ctl[6];
    const int nact = B.ctl[5];
    const int64_t nw = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    const int64_t gw = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5;
    t = total * gw / nw;
    end = total * (gw + 1) / nw;
    if (t >= end) return false;
    int lo = 0, hi = nact;
    while (hi - lo > 1) {
      const int m = (lo + hi) >> 1;
      if (B.act_start[m] <= t) lo = m; else hi = m;
    }
    j = lo;
    inst = B.act_inst[j];
    next = B.act_start[j + 1];
    s = B.inst_slice[inst] + (t - B.act_start[j]);
    return live(B);
  }
  // moves to the next slice of a live block; false past the end
  __device__ __forceinline__ bool live(const View& B) {
    while (t < end) {
      if (!B.done[inst]) return true;
      t = next;  // skip the rest of this block
      if (t >= end) break;
      ++j;
      inst = B.act_inst[j];
      next = B.act_start[j + 1];
      s = B.inst_slice[inst];
    }
    return false;
  }
  __device__ __forceinline__ bool step(const View& B) {
    ++t;
    ++s;
    while (t < end && t == next) {  // a listed block without rows is passed over
      ++j;
      inst = B.act_inst[j];
      next = B.act_start[j + 1];
      s = B.inst_slice[inst];
    }
    return live(B);
  }
};

// q = A p and the slice's p.q for every live slice of the warp's share: one
// software pipeline over the share -- the next batch of kBatchB columns /
// values, possibly of the next slice, is in flight while the current batch
// gathers p (entries of a row summed in CSR order; masked entries add +0
// after the real ones).
#ifndef EMG_BATCH_ENTRIES
#define EMG_BATCH_ENTRIES 4
#endif
constexpr int kBatchB = EMG_BATCH_ENTRIES;
__global__ void __launch_bounds__(kBT) k_b_spmv_dot(View B) {
  const uint64_t pol = evict_first_policy();
  const int lane = threadIdx.x & 31;
  SliceCursor F;  // fetch cursor
  bool more = F.init(B);
  if (!more) return;
  int64_t fbase = B.slice_ptr[F.s];
  int flen = static_cast<int>((B.slice_ptr[F.s + 1] - fbase) >> 5);
  fbase += lane;
  int fj = 0;
  auto fetch = [&](int (&c)[kBatchB], double (&v)[kBatchB], bool& last, int64_t& sl) {
#pragma unroll
    for (int u = 0; u < kBatchB; ++u) {
      const bool in = fj + u < flen;
      const int64_t k = fbase + 32 * static_cast<int64_t>(fj + u);
      c[u] = in ? ld_stream(B.col + k, pol) : 0;
      v[u] = in ? ld_stream(B.val + k, pol) : 0.0;
    }
    sl = F.s;
    fj += kBatchB;
    last = fj >= flen;
    if (last) {
      more = F.step(B);
      if (more) {
        fbase = B.slice_ptr[F.s];
        flen = static_cast<int>((B.slice_ptr[F.s + 1] - fbase) >> 5);
        fbase += lane;
        fj = 0;
      }
    }
  };
  int cn[kBatchB];
  double vn[kBatchB];
  bool lastn;
  int64_t sn;
  fetch(cn, vn, lastn, sn);
  double sum = 0.0;
  for (;;) {
    int c[kBatchB];
    double v[kBatchB], xv[kBatchB];
#pragma unroll
    for (int u = 0; u < kBatchB; ++u) { c[u] = cn[u]; v[u] = vn[u]; }
    const bool last = lastn;
    const int64_t sl = sn;
    const bool had_more = more;
    if (more) fetch(cn, vn, lastn, sn);
#pragma unroll
    for (int u = 0; u < kBatchB; ++u) xv[u] = B.p[c[u]];
#pragma unroll
    for (int u = 0; u < kBatchB; ++u) sum += v[u] * xv[u];
    if (last) {
      const int64_t row = sl * 32 + lane;
      B.q[row] = sum;
      const double pq = warp_sum(B.p[row] * sum);
      if (lane == 0) B.partial[sl] = pq;
      sum = 0.0;
      if (!had_more) break;
    }
  }
}

// alpha (or breakdown) per block
__global__ void __launch_bounds__(kBT) k_b_fin_alpha(View B) {
  finish_blocks<1, false>(B, [&](int i, const double* tot) {
    if (fabs(tot[0]) < 1e-30) {  // :453-457
      B.status[i] = EMG_NUMERICAL_ERROR;
      B.done[i] = 1;
    } else {
      B.alpha[i] = B.rz[i] / tot[0];
    }
  });
}

// x += alpha p, r -= alpha q, z = D^-1 r; per-slice r.z and r.r
__global__ void __launch_bounds__(kBT) k_b_update(View B) {
  active_slices(B, [&](int64_t s, int inst, int lane) {
    const int64_t row = s * 32 + lane;
    const double a = B.alpha[inst];
    B.x[row] += a * B.p[row];
    const double ri = B.r[row] - a * B.q[row];
    const double zi = B.dinv[row] * ri;
    B.r[row] = ri;
    B.z[row] = zi;
    const double rz = warp_sum(ri * zi), rr = warp_sum(ri * ri);
    if (lane == 0) { B.partial[2 * s] = rz; B.partial[2 * s + 1] = rr; }
  });
}

// residual test and beta per block (CGSolver::solve_with_jacobi, :459-495)
__global__ void __launch_bounds__(kBT) k_b_fin_beta(View B) {
  finish_blocks<2, false>(B, [&](int i, const double* tot) {
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

__global__ void __launch_bounds__(kBT) k_b_direction(View B) {
  active_slices(B, [&](int64_t s, int inst, int lane) {
    const int64_t row = s * 32 + lane;
    B.p[row] = B.z[row] + B.beta[inst] * B.p[row];
  });
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
  // scratch goes back on every exit (the plan's own arrays go with the plan)
  auto release = [&](bool with_iperm) {
    for (void* q : {static_cast<void*>(d_slots), static_cast<void*>(d_off), static_cast<void*>(d_wrow),
                    static_cast<void*>(d_wout), static_cast<void*>(d_wlen)})
      if (q) cudaFreeAsync(q, st);
    d_slots = d_off = d_wlen = nullptr;
    d_wrow = d_wout = nullptr;
    if (with_iperm && d_iperm) cudaFreeAsync(d_iperm, st);
  };
  if (rc) { release(true); return rc; }
  cudaError_t e = cudaMemsetAsync(P.perm, 0xff, sizeof(int32_t) * std::max<int64_t>(N, 1), st);
  if (e == cudaSuccess && nwin > 0) {
    e = cudaMemcpyAsync(d_wrow, wrow.data(), sizeof(int64_t) * nwin, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_wout, wout.data(), sizeof(int64_t) * nwin, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_wlen, wlen.data(), sizeof(int32_t) * nwin, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      k_b_window_perm<<<static_cast<unsigned>(nwin), 32, 0, st>>>(d_wrow, d_wlen, d_wout, A.row_ptr, P.perm);
  }
  if (e == cudaSuccess && ns > 0) k_b_slice_slots<<<launch_grid(ns * 32), 256, 0, st>>>(ns, P.perm, A.row_ptr, d_slots);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) {
    release(true);
    set_error(std::string("batch plan: ") + cudaGetErrorString(e));
    return EMG_ERR_CUDA;
  }
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
  release(rc != EMG_SUCCESS);
  if (rc) return rc;
  // slices of every block; a block without rows has none, sums 0 and
  // finishes at once
  std::vector<int32_t> islice(nb + 1);
  for (int32_t k = 0; k <= nb; ++k) islice[k] = static_cast<int32_t>(nstart[k] / 32);
  P.n = n; P.N = N; P.nslices = ns; P.slots = total; P.nb = nb;
  P.blocks = blocks;
  {
    int dev = 0, sms = 148, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_b_spmv_dot, kBT, 0) != cudaSuccess || per < 1) per = 4;
    P.grid_spmv = per * sms;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_b_update, kBT, 0) != cudaSuccess || per < 1) per = 4;
    P.grid_vec = per * sms;
    cudaGetLastError();
  }
  if (!rc) rc = dalloc(&P.inst_slice, nb + 1, st);
  if (!rc) rc = dalloc(&P.act_inst, nb, st);
  if (!rc) rc = dalloc(&P.act_start, nb + 1, st);
  if (!rc) rc = dalloc(&P.col, P.slots, st);
  if (!rc) rc = dalloc(&P.src, P.slots, st);
  if (!rc) rc = dalloc(&P.val, P.slots, st);
  for (double** v : {&P.x, &P.r, &P.z, &P.p, &P.q, &P.dinv})
    if (!rc) rc = dalloc(v, N, st);
  if (!rc) rc = dalloc(&P.partial, 2 * ns, st);
  for (double** v : {&P.bnorm, &P.rz, &P.alpha, &P.beta, &P.res, &P.prev})
    if (!rc) rc = dalloc(v, nb, st);
  for (int32_t** v : {&P.iter, &P.status, &P.done})
    if (!rc) rc = dalloc(v, nb, st);
  if (!rc) rc = dalloc(&P.ctl, 8, st);
  if (!rc) rc = dalloc(&P.tol, 1, st);
  if (rc) { cudaFreeAsync(d_iperm, st); return rc; }
  e = cudaMemcpyAsync(P.inst_slice, islice.data(), sizeof(int32_t) * (nb + 1), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(P.ctl, 0, sizeof(int32_t) * 8, st);
  if (e == cudaSuccess && ns > 0) {
    k_b_fill<<<launch_grid(ns * 32), 256, 0, st>>>(ns, P.slice_ptr, P.perm, d_iperm, A.row_ptr, A.col, P.col, P.src);
    e = cudaGetLastError();
  }
  cudaFreeAsync(d_iperm, st);  // the plan's own arrays go with the plan
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    set_error(std::string("batch plan: ") + cudaGetErrorString(e));
    return EMG_ERR_CUDA;
  }
  EMG_CK(cudaStreamCreate(&P.cap));
  P.version = ~uint64_t(0);
  return EMG_SUCCESS;
}

// Warp per block for the per-block sums.
int fin_grid(int32_t nb) {
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((nb + kBT / 32 - 1) / (kBT / 32), 148 * 8)));
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
      const int gf = fin_grid(P.nb);
      for (int k = 0; k < kBodyB; ++k) {
        k_b_spmv_dot<<<P.grid_spmv, kBT, 0, P.cap>>>(v);
        k_b_fin_alpha<<<gf, kBT, 0, P.cap>>>(v);
        k_b_update<<<P.grid_vec, kBT, 0, P.cap>>>(v);
        k_b_fin_beta<<<gf, kBT, 0, P.cap>>>(v);
        k_b_direction<<<P.grid_vec, kBT, 0, P.cap>>>(v);
      }
      k_b_list<true><<<1, 1024, 0, P.cap>>>(v, handle);
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
  for (void* p : {static_cast<void*>(perm), static_cast<void*>(slice_ptr), static_cast<void*>(inst_slice),
                  static_cast<void*>(act_inst), static_cast<void*>(act_start), static_cast<void*>(col), static_cast<void*>(src), static_cast<void*>(val),
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
    int32_t bad = 0;
    cudaError_t e = cudaMallocAsync(&d_blocks, sizeof(int64_t) * (nb + 1), st);
    if (e == cudaSuccess) e = cudaMallocAsync(&d_bad, sizeof(int32_t), st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_blocks, blocks.data(), sizeof(int64_t) * (nb + 1), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_bad, 0, sizeof(int32_t), st);
    if (e == cudaSuccess) {
      k_b_check<<<launch_grid(A.n), 256, 0, st>>>(A.n, A.row_ptr, A.col, nb, d_blocks, d_bad);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, d_bad, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
    for (void* p : {static_cast<void*>(d_blocks), static_cast<void*>(d_bad)})
      if (p) cudaFreeAsync(p, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
      set_error(std::string("batch solve: block check: ") + cudaGetErrorString(e));
      return EMG_ERR_CUDA;
    }
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
  EMG_CK(cudaMemsetAsync(P.done, 0, sizeof(int32_t) * nb, st));
  k_b_list<false><<<1, 1024, 0, st>>>(v, cudaGraphConditionalHandle{});  // every block
  k_b_init<<<P.grid_vec, kBT, 0, st>>>(v, b);
  k_b_fin_init<<<fin_grid(nb), kBT, 0, st>>>(v);
  k_b_list<false><<<1, 1024, 0, st>>>(v, cudaGraphConditionalHandle{});  // blocks with b != 0
  EMG_CK(cudaGetLastError());
  if (!P.tuned) {
    // Warps sharing the slices of the SpMV: one resident wave (default) or
    // one or two blocks per SM fewer, timed on this batch's first SpMV (its
    // q and partials are overwritten by the loop's own first SpMV).
    P.tuned = true;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int per = std::max(1, P.grid_spmv / std::max(sms, 1));
    std::vector<int> cand{P.grid_spmv};
    for (int d = 1; d <= 2; ++d)
      if (per - d >= 1) cand.push_back((per - d) * sms);
    const std::string key = "nb" + std::to_string(nb) + "N" + std::to_string(P.N) + "slots" + std::to_string(P.slots);
    const int g = tune::pick("batch.spmv_grid", key, cand, [&](int gv, cudaStream_t s2) {
      k_b_spmv_dot<<<gv, kBT, 0, s2>>>(v);
    }, st);
    cudaGetLastError();
    if (g != P.grid_spmv) {
      P.grid_spmv = g;
      cudaGraphExecDestroy(P.loop);
      P.loop = nullptr;
      int rc = capture_batch_loop(P);
      if (rc) return rc;
    }
  }
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

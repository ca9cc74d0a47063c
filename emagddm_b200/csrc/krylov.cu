// krylov.cu -- FP64 sparse matrix-vector product and the Jacobi-preconditioned
// CG / BiCGSTAB solvers of the reference (src/numeric/iterative_solvers.cpp:
// 343-503 and :869-1118), with the same iteration, stopping and failure rules.
//
// Matrix format inside the solvers: SELL-32-sigma.  Rows are sorted by length
// (descending) inside windows of 4096 rows and cut into slices of 32 rows; the
// 8 slices of a 256-row group are padded to the group's longest row and
// stored entry-interleaved (entry j of the 8 slices is one 2 KB run of
// values), so one warp reads a slice with 256-byte coalesced loads, every lane
// has a whole row (no shuffles, many independent loads in flight), and the 8
// warps of a block stream one contiguous run together.  The solvers run in the
// permuted numbering (P A P^T, P b): all vector kernels stay contiguous; b is
// permuted on entry and x on exit.  The CSR handed in stays the exported form.
//
// One CG iteration:
//   k_cg_spmv_dot   q = A p and p.q        (last block: alpha / breakdown)
//   k_cg_update     x += a p, r -= a q, z = D^-1 r, r.z and r.r
//                   (last block: residual, convergence, divergence, beta)
//   k_cg_direction  p = z + b p
// Reductions are deterministic: a fixed grid, one partial per block, and the
// last block to finish (atomic ticket) sums the partials in a fixed order and
// updates the solver state on the device.  The host never reads a scalar
// inside the loop: iterations run as CUDA-graph chunks and every kernel of a
// finished solve returns at once; the host polls the state between chunks.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "device.h"
#include "tune.h"
#include "sell_tma.cuh"
#include "trace.h"

namespace emg {

struct SolverState {
  double tol;
  double bnorm;
  double rz;      // CG: r.z of the current iteration
  double rho;     // BiCGSTAB: rho of the current iteration
  double alpha, beta, omega;
  double res;     // last relative residual
  double prev;    // previous relative residual
  int32_t max_iter;
  int32_t iter;   // current iteration (1-based)
  int32_t status;
  int32_t done;
  int32_t early;  // BiCGSTAB early exit on ||s|| pending
  int32_t dcount; // BiCGSTAB growth counter
  uint32_t ticket;
  int32_t loops;       // device-loop bodies executed in this solve
  int32_t loop_limit;  // hard bound on loop bodies (stops the loop without `done`)
  int32_t copy_err;    // a bounded wait (bulk copy, grid barrier) ran out
  uint32_t gen;        // grid-barrier generation of the fused CG update
};

// SELL-32-sigma copy of a DevCsr in the permuted numbering, slices in
// interleaved groups of kGroup.
struct Sell {
  int64_t n = 0, nslices = 0, ngroups = 0, slots = 0;
  int64_t max_tile_slots = 0;    // largest 8-slice tile (bulk-copy stage size)
  bool tma = false;              // stages of the bulk-copy kernels fit in shared memory
  bool ws = false;               // warp-specialized bulk-copy SpMV in use
  uint32_t ws_stage_bytes = 0;   // one slice (largest) of values + columns, 128-byte multiple
  int ws_grid = 0;
  size_t ws_smem = 0;
  int32_t* perm = nullptr;       // new row -> old row
  int64_t* slice_ptr = nullptr;  // ngroups + 1 slot offsets of the slice groups (multiples of 32 kGroup)
  int16_t* dcol = nullptr;       // column - row of every slot, when all fit in 16 bits
  bool narrow = false;           // dcol in use (col freed): 10 bytes per slot instead of 12
  int32_t* col = nullptr;        // permuted column of every slot
  int32_t* src = nullptr;        // CSR index of every slot, -1 = padding
  double* val = nullptr;
  uint64_t version = ~uint64_t(0);
  int grid = 0;                  // autotuned grid of the register-pipeline SpMV kernels (0: one resident wave)
};

struct KrylovWorkspace {
  int64_t n = 0;
  int grid = 0;
  double *dinv = nullptr, *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr;
  double *rh = nullptr, *v = nullptr, *s = nullptr, *t = nullptr;
  double* partial = nullptr;
  double* hist = nullptr;
  int32_t hist_cap = 0;
  int32_t hist_len = 0;
  SolverState* state = nullptr;
  SolverState* state_h = nullptr;  // pinned
  cudaStream_t cap = nullptr;
  cudaGraphExec_t cg_exec = nullptr;  // chunk of kChunk iterations (host-polled)
  cudaGraphExec_t bi_exec = nullptr;
  cudaGraphExec_t cg_loop = nullptr;  // whole solve as a device while-loop
  cudaGraphExec_t bi_loop = nullptr;
  bool loop_unavailable = false;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int dev = -1;  // device of cap / ev0 / ev1
  // fused CG update + direction (one cooperative launch per iteration)
  bool fuse = false;
  int fuse_grid = 0;
  size_t fuse_smem = 0;
  int64_t fuse_stash = 0;  // entry pairs of a block kept in shared memory
};

namespace {

constexpr int kThreads = 256;
constexpr int kChunk = 16;      // iterations per host-polled graph launch
constexpr int kBody = 4;        // iterations per body of the device while-loop
constexpr int kSliceRows = 32;  // SELL slice height = warp width
#ifndef EMG_SELL_WINDOW
#define EMG_SELL_WINDOW 4096
#endif
constexpr int kWindow = EMG_SELL_WINDOW;  // sigma: rows sorted by length inside a window

__device__ __forceinline__ int64_t gtid() {
  return static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
}
__device__ __forceinline__ int64_t gstride() {
  return static_cast<int64_t>(gridDim.x) * blockDim.x;
}

// Bulk-copy (TMA) pipeline for the SpMV: built and tested, but on the 64^3
// curl-curl matrix it measured slower than the plain SELL loop, so it is a
// build-time option (-DEMG_SELL_TMA=1) rather than the default.
#ifndef EMG_SELL_TMA
#define EMG_SELL_TMA 0
#endif
// Warp-specialized bulk-copy SpMV (-DEMG_SELL_WS=1): warp 0 of a block
// streams the slices of the other warps into per-warp rings of kWsStages
// shared-memory stages; those warps only gather x.
#ifndef EMG_SELL_WS
#define EMG_SELL_WS 0
#endif
#ifndef EMG_SELL_WS_CONTIG
#define EMG_SELL_WS_CONTIG 0
#endif
#ifndef EMG_SELL_WS_STAGES
#define EMG_SELL_WS_STAGES 2
#endif
// 16-bit column offsets (10 instead of 12 bytes per slot) when the matrix
// bandwidth allows: fewer bytes, but measured slower than 32-bit columns on
// B200 for the 64^3 curl-curl matrix, so off by default.
#ifndef EMG_SELL_NARROW
#define EMG_SELL_NARROW 0
#endif
#ifndef EMG_SELL_UNROLL
#define EMG_SELL_UNROLL 4  // row entries per batch of loads in the plain SELL loop
#endif
// Load pipeline of the plain SELL loop.  0: one batch of EMG_SELL_UNROLL
// loads at a time; 1: the next batch of the same slice is loaded while the
// current batch's x entries are gathered; 2: one pipeline across all slices
// of a warp, batches of EMG_SELL_BATCH entries (51.7 vs 60.3 us for 1 with
// 8 entries, 63.6 us with 4, for the 64^3 CG matrix on B200, each with the
// one-wave grid of EMG_SPMV_RESIDENT).
#ifndef EMG_SELL_PIPE
#define EMG_SELL_PIPE 2
#endif
#ifndef EMG_SELL_BATCH
#define EMG_SELL_BATCH 8
#endif
// Slices per group: the kGroup slices of a group share one length and are
// interleaved entry by entry (slot of entry j, slice w, lane l at
// group_base + 32 kGroup j + 32 w + l), so the kGroup warps of a block that
// work on one group read one contiguous 32 kGroup-slot run per entry.
#ifndef EMG_SELL_GROUP
#define EMG_SELL_GROUP 1
#endif
// Slice order over the warps: 0 = the warps of a block take adjacent slices
// (slice = global warp id + k * warps); 1 = they take slices gridDim.x apart,
// which spreads the concurrent streams of an SM over memory (64.1 vs 65.6 us
// for the 64^3 CG matrix on B200; interleaving the slices of a block instead,
// EMG_SELL_GROUP=8, was slower: 75.5 us).
#ifndef EMG_SELL_SPREAD
#define EMG_SELL_SPREAD 1
#endif
constexpr int kGroup = EMG_SELL_GROUP;
constexpr int kGroupStride = 32 * kGroup;

// Packed slots: every 32-slot chunk (one warp's entry) is stored as 256 B of
// values followed by 128 B of columns, one stream per warp instead of two.
#ifndef EMG_SELL_PACKED
#define EMG_SELL_PACKED 0
#endif
constexpr int kChunkBytes = 384;
__host__ __device__ __forceinline__ int64_t packed_val_index(int64_t k) { return (k >> 5) * (kChunkBytes / 8) + (k & 31); }
__host__ __device__ __forceinline__ int64_t packed_col_index(int64_t k) {
  return (k >> 5) * (kChunkBytes / 4) + 64 + (k & 31);
}

// Base slot (entry 0, lane 0) and entry count of slice s.
__device__ __forceinline__ void slice_span(const int64_t* __restrict__ gp, int64_t s, int64_t& base, int& len) {
  const int64_t g = s / kGroup;
  const int64_t b0 = gp[g];
  len = static_cast<int>((gp[g + 1] - b0) / kGroupStride);
  base = b0 + 32 * (s - g * kGroup);
}

// Warp per slice, lane per row, as one software pipeline over all slices of
// the warp: the batch of EMG_SELL_BATCH entries after the current one --
// possibly the first batch of the warp's next slice -- is in flight while
// the current batch's x entries are gathered, and the span of the slice
// after the one being fetched is read one slice ahead, so no slice starts
// with an exposed load.  A slice without entries takes one batch of masked
// loads; entries past a row's length are masked (value 0, column 0) and add
// +0 after the real ones, so every row is summed in CSR order.  Calls
// out(row, y_row) for every real row.  Unpacked slots; kNarrow: columns as
// 16-bit offsets from the row (A.dcol).
template <bool kNarrow, class Out>
__device__ __forceinline__ void sell_rows_stream(const Sell& A, const double* __restrict__ x, Out out) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = gstride() >> 5;
  const int64_t warp = EMG_SELL_SPREAD ? static_cast<int64_t>(threadIdx.x >> 5) * gridDim.x + blockIdx.x
                                       : gtid() >> 5;
  const uint64_t pol = evict_first_policy();
  const int64_t* __restrict__ sp = A.slice_ptr;
  const int32_t* __restrict__ col = A.col;
  const int16_t* __restrict__ dcol = A.dcol;
  const double* __restrict__ val = A.val;
  constexpr int U = EMG_SELL_BATCH;
#if EMG_SELL_SPREAD == 2
  // contiguous share of slices per warp
  const int64_t gwc = gtid() >> 5;
  const int64_t s_end = A.nslices * (gwc + 1) / nwarps;
  const int64_t step = 1;
  int64_t cs = A.nslices * gwc / nwarps;
  if (cs >= s_end) return;
#else
  const int64_t s_end = A.nslices;
  const int64_t step = nwarps;
  int64_t cs = warp;  // slice whose batch is being summed
  if (cs >= A.nslices) return;
#endif
  int64_t fs = cs;  // slice being fetched, its lane base, length, next entry
  int64_t fbase;
  int flen;
  slice_span(sp, fs, fbase, flen);
  fbase += lane;
  int fj = 0;
  int64_t nbase = 0;  // span of slice fs + step
  int nlen = 0;
  if (fs + step < s_end) slice_span(sp, fs + step, nbase, nlen);
  bool more = true;
  auto fetch = [&](int (&c)[U], double (&v)[U], bool& last) {
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const bool in = fj + u < flen;
      const int64_t k = fbase + static_cast<int64_t>(kGroupStride) * (fj + u);
      if constexpr (kNarrow) c[u] = in ? static_cast<int>(fs * kSliceRows + lane) + ld_stream(dcol + k, pol) : 0;
      else if constexpr (EMG_SELL_PACKED) c[u] = in ? ld_stream(col + packed_col_index(k), pol) : 0;
      else c[u] = in ? ld_stream(col + k, pol) : 0;
      v[u] = in ? ld_stream(val + (EMG_SELL_PACKED ? packed_val_index(k) : k), pol) : 0.0;
    }
    fj += U;
    last = fj >= flen;
    if (last) {
      fs += step;
      more = fs < s_end;
      fbase = nbase + lane;
      flen = nlen;
      fj = 0;
      if (fs + step < s_end) slice_span(sp, fs + step, nbase, nlen);
    }
  };
  int cn[U];
  double vn[U];
  bool lastn;
  fetch(cn, vn, lastn);
  double sum = 0.0;
  for (;;) {
    int c[U];
    double v[U], xv[U];
#pragma unroll
    for (int u = 0; u < U; ++u) { c[u] = cn[u]; v[u] = vn[u]; }
    const bool last = lastn;
    if (more) fetch(cn, vn, lastn);
#pragma unroll
    for (int u = 0; u < U; ++u) xv[u] = x[c[u]];
#pragma unroll
    for (int u = 0; u < U; ++u) sum += v[u] * xv[u];
    if (last) {
      const int64_t row = cs * kSliceRows + lane;
      if (row < A.n) out(row, sum);
      sum = 0.0;
      cs += step;
      if (cs >= s_end) break;
    }
  }
}

// Warp per slice, lane per row: y_row = sum_j val * x[col].  Calls
// out(row, y_row) for every real row.  Entries of a row are summed in CSR
// order, EMG_SELL_UNROLL loads in flight per lane at a time (with
// EMG_SELL_PIPE=1 the next batch of the same slice as well).
// kNarrow: columns are stored as 16-bit offsets from the row (A.dcol).
template <bool kNarrow, class Out>
__device__ __forceinline__ void sell_rows_sliced(const Sell& A, const double* __restrict__ x, Out out) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = gstride() >> 5;
  const int64_t warp = EMG_SELL_SPREAD ? static_cast<int64_t>(threadIdx.x >> 5) * gridDim.x + blockIdx.x
                                       : gtid() >> 5;
  const uint64_t pol = evict_first_policy();
  const int64_t* __restrict__ sp = A.slice_ptr;
  const int32_t* __restrict__ col = A.col;
  const int16_t* __restrict__ dcol = A.dcol;
  const double* __restrict__ val = A.val;
  auto column = [&](int64_t k, int row) -> int {
    if constexpr (kNarrow) return row + ld_stream(dcol + k, pol);
    else if constexpr (EMG_SELL_PACKED) return ld_stream(col + packed_col_index(k), pol);
    else return ld_stream(col + k, pol);
  };
  auto value = [&](int64_t k) -> double {
    if constexpr (EMG_SELL_PACKED) return ld_stream(val + packed_val_index(k), pol);
    else return ld_stream(val + k, pol);
  };
  for (int64_t s = warp; s < A.nslices; s += nwarps) {
    int64_t base;
    int len;
    slice_span(sp, s, base, len);
    base += lane;
    const int row32 = static_cast<int>(s * kSliceRows + lane);
    double sum = 0.0;
    int j = 0;
#if EMG_SELL_PIPE == 1
    // software pipeline: the next batch's columns and values are in flight
    // while this batch's x entries are gathered; entries past the row length
    // are masked (value 0, column 0) and add +0 after the real ones
    {
      constexpr int U = EMG_SELL_UNROLL;
      const int nb = (len + U - 1) / U;
      int cn[U];
      double vn[U];
      auto fetch = [&](int jb, int (&c)[U], double (&v)[U]) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const bool in = jb + u < len;
          const int64_t k = base + static_cast<int64_t>(kGroupStride) * (jb + u);
          c[u] = in ? column(k, row32) : 0;
          v[u] = in ? value(k) : 0.0;
        }
      };
      if (nb > 0) fetch(0, cn, vn);
      for (int bt = 0; bt < nb; ++bt) {
        int c[U];
        double v[U], xv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) { c[u] = cn[u]; v[u] = vn[u]; }
        if (bt + 1 < nb) fetch((bt + 1) * U, cn, vn);
#pragma unroll
        for (int u = 0; u < U; ++u) xv[u] = x[c[u]];
#pragma unroll
        for (int u = 0; u < U; ++u) sum += v[u] * xv[u];
      }
      j = len;
    }
#endif
    for (; j + EMG_SELL_UNROLL <= len; j += EMG_SELL_UNROLL) {
      const int64_t k = base + static_cast<int64_t>(kGroupStride) * j;
      int c[EMG_SELL_UNROLL];
      double v[EMG_SELL_UNROLL], xv[EMG_SELL_UNROLL];
#pragma unroll
      for (int u = 0; u < EMG_SELL_UNROLL; ++u) {
        c[u] = column(k + kGroupStride * u, row32);
        v[u] = value(k + kGroupStride * u);
      }
#pragma unroll
      for (int u = 0; u < EMG_SELL_UNROLL; ++u) xv[u] = x[c[u]];
#pragma unroll
      for (int u = 0; u < EMG_SELL_UNROLL; ++u) sum += v[u] * xv[u];
    }
    for (; j < len; ++j) {
      const int64_t k = base + static_cast<int64_t>(kGroupStride) * j;
      sum += value(k) * x[column(k, row32)];
    }
    const int64_t row = s * kSliceRows + lane;
    if (row < A.n) out(row, sum);
  }
}

template <bool kNarrow, class Out>
__device__ __forceinline__ void sell_rows(const Sell& A, const double* __restrict__ x, Out out) {
  if constexpr (EMG_SELL_PIPE == 2) sell_rows_stream<kNarrow>(A, x, out);
  else sell_rows_sliced<kNarrow>(A, x, out);
}

// Same product with the slices streamed through shared memory by bulk
// asynchronous copies (see sell_tma.cuh).  Launch: persistent grid, 256
// threads, tma::smem_bytes() of dynamic shared memory.  A bounded wait that
// runs out raises *err and the block drains its copies and stops.
template <class Out>
__device__ __forceinline__ void sell_rows_tma(const Sell& A, const double* __restrict__ x, Out out,
                                              int32_t* err) {
  extern __shared__ __align__(128) unsigned char smem[];
  const tma::Layout Ly = tma::layout_for(static_cast<uint32_t>(A.max_tile_slots));
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + tma::kStages * Ly.stage_bytes);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t* __restrict__ sp = A.slice_ptr;
  const int64_t ns = A.nslices;
  const int64_t ntiles = (ns + tma::kWarps - 1) / tma::kWarps;
  const int64_t stride = gridDim.x;
  const uint64_t pol = evict_first_policy();
  auto tile_range = [&](int64_t t, int64_t& a, int64_t& b) {
    const int64_t s0 = t * tma::kWarps;
    const int64_t s1 = s0 + tma::kWarps < ns ? s0 + tma::kWarps : ns;
    a = sp[s0];
    b = sp[s1];
  };
  auto issue = [&](int64_t t, int stage) {
    int64_t a, b;
    tile_range(t, a, b);
    const uint32_t slots = static_cast<uint32_t>(b - a);
    unsigned char* base = smem + stage * Ly.stage_bytes;
    tma::mbar_expect_tx(&bars[stage], slots * 12u);  // 0 bytes: the arrival alone completes it
    if (slots > 0) {
      tma::bulk_g2s(base, A.val + a, slots * 8u, &bars[stage], pol);
      tma::bulk_g2s(base + slots * 8u, A.col + a, slots * 4u, &bars[stage], pol);
    }
  };
  if (threadIdx.x == 0) {
    for (int s = 0; s < tma::kStages; ++s) tma::mbar_init(&bars[s], 1);
    tma::fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0)
    for (int k = 0; k < tma::kStages; ++k) {
      const int64_t t = blockIdx.x + k * stride;
      if (t < ntiles) issue(t, k);
    }
  bool ok = true;
  int k = 0;
  int64_t t = blockIdx.x;
  for (; t < ntiles; t += stride, ++k) {
    const int stage = k % tma::kStages;
    const uint32_t parity = static_cast<uint32_t>(k / tma::kStages) & 1u;
    ok = __syncthreads_and(tma::mbar_wait(&bars[stage], parity) ? 1 : 0) != 0;
    if (!ok) break;
    const int64_t s = t * tma::kWarps + warp;
    if (s < ns) {
      int64_t a, b;
      tile_range(t, a, b);
      const int64_t b0 = sp[s];
      const int len = static_cast<int>((sp[s + 1] - b0) >> 5);
      const unsigned char* base = smem + stage * Ly.stage_bytes;
      const double* sv = reinterpret_cast<const double*>(base) + (b0 - a) + lane;
      const int32_t* sc =
          reinterpret_cast<const int32_t*>(base + static_cast<uint32_t>(b - a) * 8u) + (b0 - a) + lane;
      // up to 16 gathers of x in flight per lane; summed in row order
      double sum = 0.0;
      for (int j0 = 0; j0 < len; j0 += 16) {
        double xv[16];
#pragma unroll
        for (int u = 0; u < 16; ++u) xv[u] = j0 + u < len ? x[sc[32 * (j0 + u)]] : 0.0;
#pragma unroll
        for (int u = 0; u < 16; ++u)
          if (j0 + u < len) sum += sv[32 * (j0 + u)] * xv[u];
      }
      const int64_t row = s * kSliceRows + lane;
      if (row < A.n) out(row, sum);
    }
    __syncthreads();  // every warp is done with this stage
    if (threadIdx.x == 0) {
      const int64_t tn = t + tma::kStages * stride;
      if (tn < ntiles) {
        tma::fence_proxy_async();
        issue(tn, stage);
      }
    }
  }
  if (!ok) {
    // drain the copies this block still has in flight (bounded), then stop
    if (threadIdx.x == 0) {
      atomicOr(err, 1);
      for (int q = 0; q < tma::kStages; ++q, ++k, t += stride) {
        if (t >= ntiles) break;
        tma::mbar_wait(&bars[k % tma::kStages], static_cast<uint32_t>(k / tma::kStages) & 1u);
      }
    }
    __syncthreads();
  }
}

// Warp-specialized bulk-copy SpMV.  Block = 1 producer warp + kWsC
// consumer warps; consumer c of block b takes slices b kWsC + c + k (kWsC
// gridDim.x), k = 0, 1, ...; producer lane c copies consumer c's next
// slices (values, then columns, one byte range each) into c's ring of
// kWsS stages and the consumer, once a stage's full barrier completes, sums
// its rows from shared memory (entries in CSR order, kWsU gathers of x in
// flight per lane) and releases the stage on its empty barrier.  Every wait
// is bounded: a producer that gives up raises *err and waits (bounded) for
// the copies it already issued; a consumer that gives up raises *err and
// stops.
constexpr int kWsC = kThreads / 32 - 1;
constexpr int kWsS = EMG_SELL_WS_STAGES;
constexpr int kWsU = 16;
__host__ __device__ inline size_t ws_smem_bytes(uint32_t stage_bytes) {
  return static_cast<size_t>(kWsC) * kWsS * stage_bytes + sizeof(uint64_t) * 2 * kWsC * kWsS +
         sizeof(uint32_t) * kWsC * kWsS;
}
template <class Out>
__device__ __forceinline__ void sell_rows_ws(const Sell& A, const double* __restrict__ x, Out out,
                                             int32_t* err) {
  extern __shared__ __align__(128) unsigned char smem[];
  const uint32_t sb = A.ws_stage_bytes;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + static_cast<size_t>(kWsC) * kWsS * sb);
  uint64_t* empty = full + kWsC * kWsS;
  uint32_t* slots_of = reinterpret_cast<uint32_t*>(empty + kWsC * kWsS);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x < kWsC * kWsS) {
    tma::mbar_init(&full[threadIdx.x], 1);
    tma::mbar_init(&empty[threadIdx.x], 1);
  }
  tma::fence_mbar_init();
  __syncthreads();
  const int64_t nc = static_cast<int64_t>(gridDim.x) * kWsC;
  const int64_t* __restrict__ sp = A.slice_ptr;
  if (warp == 0) {
    if (lane < kWsC) {
      const uint64_t pol = evict_first_policy();
      int k = 0;
      bool ok = true;
#if EMG_SELL_WS_CONTIG
      const int64_t gc = static_cast<int64_t>(blockIdx.x) * kWsC + lane;
      const int64_t s_end = A.nslices * (gc + 1) / nc;
      for (int64_t s = A.nslices * gc / nc; s < s_end; ++s, ++k) {
#else
      for (int64_t s = static_cast<int64_t>(blockIdx.x) * kWsC + lane; s < A.nslices; s += nc, ++k) {
#endif
        const int q = lane * kWsS + k % kWsS;
        if (k >= kWsS && !tma::mbar_wait(&empty[q], ((k / kWsS) & 1u) ^ 1u)) { ok = false; break; }
        const int64_t b0 = sp[s];
        const uint32_t slots = static_cast<uint32_t>(sp[s + 1] - b0);
        unsigned char* base = smem + static_cast<size_t>(q) * sb;
        slots_of[q] = slots;
        tma::fence_proxy_async();
        tma::mbar_expect_tx(&full[q], slots * 12u);
        if (slots > 0) {
          tma::bulk_g2s(base, A.val + b0, slots * 8u, &full[q], pol);
          tma::bulk_g2s(base + slots * 8u, A.col + b0, slots * 4u, &full[q], pol);
        }
      }
      if (!ok) {
        atomicOr(err, 1);
        // the copies issued for the last kWsS slices may still be in flight
        for (int j = k - kWsS; j < k; ++j)
          if (j >= 0) tma::mbar_wait(&full[lane * kWsS + j % kWsS], (j / kWsS) & 1u);
      }
    }
    return;
  }
  const int c = warp - 1;
  int k = 0;
#if EMG_SELL_WS_CONTIG
  const int64_t gcc = static_cast<int64_t>(blockIdx.x) * kWsC + c;
  const int64_t c_end = A.nslices * (gcc + 1) / nc;
  for (int64_t s = A.nslices * gcc / nc; s < c_end; ++s, ++k) {
#else
  for (int64_t s = static_cast<int64_t>(blockIdx.x) * kWsC + c; s < A.nslices; s += nc, ++k) {
#endif
    const int q = c * kWsS + k % kWsS;
    if (!tma::mbar_wait(&full[q], (k / kWsS) & 1u)) {
      if (lane == 0) atomicOr(err, 1);
      break;
    }
    const int len = static_cast<int>(slots_of[q] >> 5);
    const double* sv = reinterpret_cast<const double*>(smem + static_cast<size_t>(q) * sb) + lane;
    const int32_t* sc =
        reinterpret_cast<const int32_t*>(smem + static_cast<size_t>(q) * sb + static_cast<size_t>(len) * 256) + lane;
    double sum = 0.0;
    for (int j0 = 0; j0 < len; j0 += kWsU) {
      double xv[kWsU];
#pragma unroll
      for (int u = 0; u < kWsU; ++u) xv[u] = j0 + u < len ? x[sc[32 * (j0 + u)]] : 0.0;
#pragma unroll
      for (int u = 0; u < kWsU; ++u)
        if (j0 + u < len) sum += sv[32 * (j0 + u)] * xv[u];
    }
    __syncwarp();
    if (lane == 0) tma::mbar_arrive(&empty[q]);
    const int64_t row = s * kSliceRows + lane;
    if (row < A.n) out(row, sum);
  }
}

// Row kernels: kMode 0 = SELL with 32-bit columns, 1 = SELL with 16-bit
// column offsets, 2 = bulk-copy pipeline (32-bit columns), 3 = warp-
// specialized bulk-copy pipeline.
template <int kMode, class Out>
__device__ __forceinline__ void spmv_rows(const Sell& A, const double* __restrict__ x, Out out,
                                          int32_t* err) {
  if constexpr (kMode == 2) sell_rows_tma(A, x, out, err);
  else if constexpr (kMode == 3) sell_rows_ws(A, x, out, err);
  else sell_rows<kMode == 1>(A, x, out);
}

// One partial per block; true in the block that finished last (all partials
// visible).  `vals` has kVals entries per thread.
template <int kVals>
__device__ __forceinline__ bool reduce_partials(const double (&vals)[kVals], double* partial,
                                                SolverState* st, double (&tot)[kVals]) {
  __shared__ double red[kThreads / 32];
  __shared__ bool last;
  for (int k = 0; k < kVals; ++k) {
    double b = block_sum(vals[k], red);
    if (threadIdx.x == 0) partial[k * gridDim.x + blockIdx.x] = b;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(&st->ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return false;
  __threadfence();
  for (int k = 0; k < kVals; ++k) {
    double a = 0.0;
    for (int i = threadIdx.x; i < static_cast<int>(gridDim.x); i += blockDim.x)
      a += ld_l2(partial + k * gridDim.x + i);
    tot[k] = block_sum(a, red);
  }
  if (threadIdx.x == 0) st->ticket = 0;
  return true;
}

// ------------------------------------------------------------ SELL build ----
// Warp per slice: column index (permuted) and CSR source of every slot; rows
// at or past n are all padding.
__global__ void k_sell_fill(int64_t n, int64_t nslices, const int64_t* __restrict__ sp,
                            const int32_t* __restrict__ perm, const int32_t* __restrict__ iperm,
                            const int32_t* __restrict__ rp, const int32_t* __restrict__ ccol,
                            int32_t* __restrict__ col, int32_t* __restrict__ src) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = gtid() >> 5, nwarps = gstride() >> 5;
  for (int64_t s = warp; s < nslices; s += nwarps) {
    int64_t b0;
    int len;
    slice_span(sp, s, b0, len);
    const int64_t row = s * kSliceRows + lane;
    int32_t a = 0, rl = 0;
    const int32_t self = static_cast<int32_t>(row < n ? row : n - 1);
    if (row < n) {
      const int32_t old = perm[row];
      a = rp[old];
      rl = rp[old + 1] - a;
    }
    for (int j = 0; j < len; ++j) {
      const int64_t k = b0 + static_cast<int64_t>(kGroupStride) * j + lane;
      const int64_t kc = EMG_SELL_PACKED ? packed_col_index(k) : k;
      if (j < rl) {
        col[kc] = iperm[ccol[a + j]];
        src[k] = a + j;
      } else {
        col[kc] = self;  // padding reads a valid entry and multiplies it by 0
        src[k] = -1;
      }
    }
  }
}

// Warp per slice: dcol = col - row; *overflow = 1 if any offset leaves int16.
__global__ void k_sell_narrow(int64_t nslices, const int64_t* __restrict__ sp,
                              const int32_t* __restrict__ col, int16_t* __restrict__ dcol,
                              int32_t* __restrict__ overflow) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = gtid() >> 5, nwarps = gstride() >> 5;
  for (int64_t s = warp; s < nslices; s += nwarps) {
    int64_t b0;
    int len;
    slice_span(sp, s, b0, len);
    const int64_t row = s * kSliceRows + lane;
    bool bad = false;
    for (int j = 0; j < len; ++j) {
      const int64_t k = b0 + static_cast<int64_t>(kGroupStride) * j + lane;
      const int64_t d = static_cast<int64_t>(col[k]) - row;
      bad |= d < -32768 || d > 32767;
      dcol[k] = static_cast<int16_t>(d);
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(overflow, 1);
  }
}

__global__ void k_sell_values(int64_t slots, const int32_t* __restrict__ src,
                              const double* __restrict__ cval, double* __restrict__ val) {
  for (int64_t i = gtid(); i < slots; i += gstride()) {
    const int32_t s = src[i];
    val[EMG_SELL_PACKED ? packed_val_index(i) : i] = s >= 0 ? cval[s] : 0.0;
  }
}

// Warp per window of kWindow rows: the stable counting sort of the rows by
// descending length.  Lengths of kLenCap - 1 and more share the last bucket
// (kept in row order): the order only decides the padding, never the result.
constexpr int kLenCap = 1024;
__global__ void __launch_bounds__(32) k_sell_window_perm(int64_t n, const int32_t* __restrict__ rp,
                                                         int32_t* __restrict__ perm) {
  __shared__ int32_t cur[kLenCap];  // bucket 0 = longest rows
  const int lane = threadIdx.x;
  const int64_t w0 = static_cast<int64_t>(blockIdx.x) * kWindow;
  const int64_t w1 = w0 + kWindow < n ? w0 + kWindow : n;
  for (int b = lane; b < kLenCap; b += 32) cur[b] = 0;
  __syncwarp();
  for (int64_t i = w0 + lane; i < w1; i += 32) {
    const int len = rp[i + 1] - rp[i];
    atomicAdd(&cur[kLenCap - 1 - (len < kLenCap - 1 ? len : kLenCap - 1)], 1);
  }
  __syncwarp();
  // exclusive scan: lane l owns buckets [l * 32, l * 32 + 32)
  constexpr int kPer = kLenCap / 32;
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
  // 32 rows a round in ascending order; equal buckets ranked by lane
  for (int64_t base = w0; base < w1; base += 32) {
    const int64_t i = base + lane;
    const bool valid = i < w1;
    int b = -1 - lane;  // unique key for lanes past the window
    if (valid) {
      const int len = rp[i + 1] - rp[i];
      b = kLenCap - 1 - (len < kLenCap - 1 ? len : kLenCap - 1);
    }
    const unsigned grp = __match_any_sync(0xffffffffu, b);
    const int rank = __popc(grp & ((1u << lane) - 1u));
    const int pos = valid ? cur[b] + rank : 0;
    __syncwarp();
    if (valid && rank == 0) cur[b] += __popc(grp);
    __syncwarp();
    if (valid) perm[w0 + pos] = static_cast<int32_t>(i);
  }
}

// Slots of every group: 32 kGroup x the longest row it holds.
__global__ void k_sell_group_slots(int64_t n, int64_t ngroups, const int32_t* __restrict__ rp,
                                   const int32_t* __restrict__ perm, int32_t* __restrict__ slots) {
  for (int64_t g = gtid(); g < ngroups; g += gstride()) {
    int32_t len = 0;
    const int64_t r0 = g * kGroupStride;
    const int64_t r1 = r0 + kGroupStride < n ? r0 + kGroupStride : n;
    for (int64_t r = r0; r < r1; ++r) {
      const int32_t o = perm[r];
      len = max(len, rp[o + 1] - rp[o]);
    }
    slots[g] = kGroupStride * len;
  }
}

__global__ void k_widen(int64_t n, const int32_t* __restrict__ in, int64_t* __restrict__ out) {
  for (int64_t i = gtid(); i < n; i += gstride()) out[i] = in[i];
}

__global__ void k_invert_perm(int64_t n, const int32_t* __restrict__ perm, int32_t* __restrict__ iperm) {
  for (int64_t i = gtid(); i < n; i += gstride()) iperm[perm[i]] = static_cast<int32_t>(i);
}

// ------------------------------------------------------------- Jacobi ----
// CGSolver::setup_preconditioner (iterative_solvers.cpp:261-292):
// 1/A(i,i), or 1 where |A(i,i)| <= 1e-15.  precond == 0 gives D^-1 = I.
// Written in the permuted numbering.
__global__ void k_jacobi(int64_t n, const int32_t* __restrict__ rp, const int32_t* __restrict__ col,
                         const double* __restrict__ val, const int32_t* __restrict__ perm,
                         int precond, double* __restrict__ dinv) {
  for (int64_t i = gtid(); i < n; i += gstride()) {
    double d = 1.0;
    if (precond) {
      const int32_t o = perm[i];
      int32_t lo = rp[o], hi = rp[o + 1];
      while (lo < hi) {
        int32_t mid = (lo + hi) >> 1;
        if (col[mid] < o) lo = mid + 1; else hi = mid;
      }
      const double a = (lo < rp[o + 1] && col[lo] == o) ? val[lo] : 0.0;
      d = fabs(a) > 1e-15 ? 1.0 / a : 1.0;
    }
    dinv[i] = d;
  }
}

__global__ void k_gather(int64_t n, const int32_t* __restrict__ perm, const double* __restrict__ in,
                         double* __restrict__ out) {
  for (int64_t i = gtid(); i < n; i += gstride()) out[i] = in[perm[i]];
}

__global__ void k_scatter(int64_t n, const int32_t* __restrict__ perm, const double* __restrict__ in,
                          double* __restrict__ out) {
  for (int64_t i = gtid(); i < n; i += gstride()) out[perm[i]] = in[i];
}

template <int kMode>
__global__ void __launch_bounds__(kThreads) k_spmv(Sell A, const double* __restrict__ x,
                                                   double* __restrict__ y, int32_t* err) {
  spmv_rows<kMode>(A, x, [&](int64_t row, double s) { y[row] = s; }, err);
}

// ----------------------------------------------------------------- CG ----
__global__ void __launch_bounds__(kThreads) k_cg_init(int64_t n, const double* __restrict__ b,
                                                      const int32_t* __restrict__ perm,
                                                      const double* __restrict__ dinv,
                                                      double* __restrict__ x, double* __restrict__ r,
                                                      double* __restrict__ z, double* __restrict__ p,
                                                      double* partial, SolverState* st) {
  double acc[2] = {0.0, 0.0};
  for (int64_t i = gtid(); i < n; i += gstride()) {
    const double bi = b[perm[i]], zi = dinv[i] * bi;
    x[i] = 0.0; r[i] = bi; z[i] = zi; p[i] = zi;
    acc[0] += bi * bi;
    acc[1] += bi * zi;
  }
  double tot[2];
  if (!reduce_partials<2>(acc, partial, st, tot)) return;
  if (threadIdx.x == 0) {
    const double bn = sqrt(tot[0]);
    st->bnorm = bn;
    st->rz = tot[1];
    st->iter = 1;
    st->done = 0;
    st->status = EMG_MAX_ITER_REACHED;
    if (bn < 1e-15) {  // iterative_solvers.cpp:440-446
      st->status = EMG_SUCCESS; st->iter = 0; st->res = 0.0; st->done = 1;
      return;
    }
    st->res = sqrt(tot[0]) / bn;
    st->prev = st->res;
    if (st->max_iter < 1) { st->iter = st->max_iter; st->done = 1; }
  }
}

// Minimum resident blocks per SM asked of the compiler for the CG SpMV
// kernel (0 = no register cap).
#ifndef EMG_SPMV_MINB
#define EMG_SPMV_MINB 0
#endif
#if EMG_SPMV_MINB
#define EMG_SPMV_BOUNDS __launch_bounds__(kThreads, EMG_SPMV_MINB)
#else
#define EMG_SPMV_BOUNDS __launch_bounds__(kThreads)
#endif

template <int kMode>
__global__ void EMG_SPMV_BOUNDS k_cg_spmv_dot(Sell A, const double* __restrict__ p,
                                                          double* __restrict__ q, double* partial,
                                                          SolverState* st) {
  if (st->done) return;
  double dot = 0.0;
  spmv_rows<kMode>(A, p, [&](int64_t row, double s) {
    q[row] = s;
    dot += p[row] * s;
  }, &st->copy_err);
  double acc[1] = {dot};
  double tot[1];
  if (!reduce_partials<1>(acc, partial, st, tot)) return;
  if (threadIdx.x == 0) {
    const double pq = tot[0];
    if (st->copy_err) {
      st->status = EMG_ERR_TIMEOUT;
      st->done = 1;
    } else if (fabs(pq) < 1e-30) {  // :453-457
      st->status = EMG_NUMERICAL_ERROR;
      st->done = 1;
    } else {
      st->alpha = st->rz / pq;
    }
  }
}

__global__ void __launch_bounds__(kThreads) k_cg_update(int64_t n, double* __restrict__ x,
                                                        double* __restrict__ r,
                                                        double* __restrict__ z,
                                                        const double* __restrict__ p,
                                                        const double* __restrict__ q,
                                                        const double* __restrict__ dinv,
                                                        double* partial, SolverState* st,
                                                        double* hist, int32_t hist_cap) {
  if (st->done) return;
  const double a = st->alpha;
  double acc[2] = {0.0, 0.0};
  // pairs of entries per 16-byte access, the odd last entry by thread 0
  const int64_t n2 = n >> 1;
  double2* __restrict__ x2 = reinterpret_cast<double2*>(x);
  double2* __restrict__ r2 = reinterpret_cast<double2*>(r);
  double2* __restrict__ z2 = reinterpret_cast<double2*>(z);
  const double2* __restrict__ p2 = reinterpret_cast<const double2*>(p);
  const double2* __restrict__ q2 = reinterpret_cast<const double2*>(q);
  const double2* __restrict__ d2 = reinterpret_cast<const double2*>(dinv);
  for (int64_t i = gtid(); i < n2; i += gstride()) {
    const double2 pv = p2[i], qv = q2[i], dv = d2[i];
    double2 xv = x2[i], rv = r2[i], zv;
    xv.x += a * pv.x;
    xv.y += a * pv.y;
    rv.x -= a * qv.x;
    rv.y -= a * qv.y;
    zv.x = dv.x * rv.x;
    zv.y = dv.y * rv.y;
    x2[i] = xv;
    r2[i] = rv;
    z2[i] = zv;
    acc[0] += rv.x * zv.x + rv.y * zv.y;
    acc[1] += rv.x * rv.x + rv.y * rv.y;
  }
  if ((n & 1) && gtid() == 0) {
    const int64_t i = n - 1;
    x[i] += a * p[i];
    const double ri = r[i] - a * q[i];
    const double zi = dinv[i] * ri;
    r[i] = ri;
    z[i] = zi;
    acc[0] += ri * zi;
    acc[1] += ri * ri;
  }
  double tot[2];
  if (!reduce_partials<2>(acc, partial, st, tot)) return;
  if (threadIdx.x == 0) {
    const int it = st->iter;
    const double res = sqrt(tot[1]) / st->bnorm;
    st->res = res;
    if (it - 1 < hist_cap) hist[it - 1] = res;
    if (res < st->tol) {
      st->status = EMG_SUCCESS; st->done = 1;
    } else if (it > 10 && res > st->prev * 1000.0) {  // :477-483
      st->status = EMG_DIVERGED; st->done = 1;
    } else {
      st->beta = tot[0] / st->rz;
      st->rz = tot[0];
      st->prev = res;
      if (it >= st->max_iter) { st->status = EMG_MAX_ITER_REACHED; st->done = 1; }
      else st->iter = it + 1;
    }
  }
}

__global__ void __launch_bounds__(kThreads) k_cg_direction(int64_t n, double* __restrict__ p,
                                                           const double* __restrict__ z,
                                                           const SolverState* st) {
  if (st->done) return;
  const double b = st->beta;
  const int64_t n2 = n >> 1;
  double2* __restrict__ p2 = reinterpret_cast<double2*>(p);
  const double2* __restrict__ z2 = reinterpret_cast<const double2*>(z);
  for (int64_t i = gtid(); i < n2; i += gstride()) {
    const double2 zv = z2[i];
    double2 pv = p2[i];
    pv.x = zv.x + b * pv.x;
    pv.y = zv.y + b * pv.y;
    p2[i] = pv;
  }
  if ((n & 1) && gtid() == 0) p[n - 1] = z[n - 1] + b * p[n - 1];
}

// CG update and direction in one cooperative launch (one block of
// kFuseThreads per SM, all resident):
//   x += alpha p,  r -= alpha q,  z = D^-1 r,  partial sums of r.z and r.r;
//   grid barrier: the block that arrives last forms the sums, the residual
//   test and beta (as k_cg_update) and then releases the others;
//   p = z + beta p.
// Every block owns a contiguous run of entry pairs and keeps z and the old p
// of the first `stash` pairs of its run in shared memory, so z is neither
// written nor read back and p is read once (8 vector passes per iteration
// instead of the 11 of k_cg_update + k_cg_direction).  Pairs past the stash
// go through z in global memory.  The barrier wait is bounded: a block that
// gives up raises st->copy_err and skips the direction step; the next SpMV
// then ends the solve with EMG_ERR_TIMEOUT.
constexpr int kFuseThreads = 1024;
constexpr int kBarrierSpins = 1 << 21;  // x >= 100 ns per poll: well over 0.2 s
// Polls a waiting block makes before it gives up; kBarrierSpins unless a
// test lowers it (emg_test_set_barrier_spins) to make the wait run out.
__device__ int32_t g_barrier_spins = kBarrierSpins;

__device__ __forceinline__ uint32_t ld_volatile(const uint32_t* p) { return *reinterpret_cast<const volatile uint32_t*>(p); }

__global__ void __launch_bounds__(kFuseThreads, 1) k_cg_update_dir(
    int64_t n, double* __restrict__ x, double* __restrict__ r, double* __restrict__ z,
    double* __restrict__ p, const double* __restrict__ q, const double* __restrict__ dinv,
    double* partial, SolverState* st, double* hist, int32_t hist_cap, int64_t stash) {
  extern __shared__ __align__(16) double2 keep[];  // [stash] z, then [stash] old p
  __shared__ double red[kFuseThreads / 32];
  __shared__ double sh_beta;
  __shared__ int sh_go;
  __shared__ int sh_last;
  __shared__ uint32_t sh_gen;
  if (st->done) return;
  const double a = st->alpha;
  const int64_t n2 = n >> 1;
  const int64_t per = (n2 + gridDim.x - 1) / gridDim.x;
  const int64_t lo = min(n2, static_cast<int64_t>(blockIdx.x) * per);
  const int64_t hi = min(n2, lo + per);
  double2* __restrict__ x2 = reinterpret_cast<double2*>(x);
  double2* __restrict__ r2 = reinterpret_cast<double2*>(r);
  double2* __restrict__ z2 = reinterpret_cast<double2*>(z);
  double2* __restrict__ p2 = reinterpret_cast<double2*>(p);
  const double2* __restrict__ q2 = reinterpret_cast<const double2*>(q);
  const double2* __restrict__ d2 = reinterpret_cast<const double2*>(dinv);
  double rz = 0.0, rr = 0.0;
  for (int64_t i = lo + threadIdx.x; i < hi; i += kFuseThreads) {
    const double2 pv = p2[i], qv = q2[i], dv = d2[i];
    double2 xv = x2[i], rv = r2[i], zv;
    xv.x += a * pv.x;
    xv.y += a * pv.y;
    rv.x -= a * qv.x;
    rv.y -= a * qv.y;
    zv.x = dv.x * rv.x;
    zv.y = dv.y * rv.y;
    x2[i] = xv;
    r2[i] = rv;
    const int64_t li = i - lo;
    if (li < stash) {
      keep[li] = zv;
      keep[stash + li] = pv;
    } else {
      z2[i] = zv;
    }
    rz += rv.x * zv.x + rv.y * zv.y;
    rr += rv.x * rv.x + rv.y * rv.y;
  }
  const bool odd = (n & 1) && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0;
  if (odd) {
    const int64_t i = n - 1;
    x[i] += a * p[i];
    const double ri = r[i] - a * q[i];
    const double zi = dinv[i] * ri;
    r[i] = ri;
    z[i] = zi;
    rz += ri * zi;
    rr += ri * ri;
  }
  const double brz = block_sum(rz, red);
  const double brr = block_sum(rr, red);
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = brz;
    partial[gridDim.x + blockIdx.x] = brr;
    sh_gen = ld_volatile(&st->gen);  // read before this block's ticket
    __threadfence();
    sh_last = atomicAdd(&st->ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (sh_last) {
    __threadfence();
    double t0 = 0.0, t1 = 0.0;
    for (int i = threadIdx.x; i < static_cast<int>(gridDim.x); i += kFuseThreads) {
      t0 += ld_l2(partial + i);
      t1 += ld_l2(partial + gridDim.x + i);
    }
    const double tot0 = block_sum(t0, red);
    const double tot1 = block_sum(t1, red);
    if (threadIdx.x == 0) {
      const int it = st->iter;
      const double res = sqrt(tot1) / st->bnorm;
      st->res = res;
      if (it - 1 < hist_cap) hist[it - 1] = res;
      if (res < st->tol) {
        st->status = EMG_SUCCESS; st->done = 1;
      } else if (it > 10 && res > st->prev * 1000.0) {  // iterative_solvers.cpp:477-483
        st->status = EMG_DIVERGED; st->done = 1;
      } else {
        st->beta = tot0 / st->rz;
        st->rz = tot0;
        st->prev = res;
        if (it >= st->max_iter) { st->status = EMG_MAX_ITER_REACHED; st->done = 1; }
        else st->iter = it + 1;
      }
      sh_beta = st->beta;
      sh_go = !st->done;
      st->ticket = 0;
      __threadfence();
      atomicAdd(&st->gen, 1u);  // release the other blocks
    }
  } else if (threadIdx.x == 0) {
    bool ok = false;
    const int32_t spins = g_barrier_spins;
    for (int k = 0; k < spins; ++k) {
      if (ld_volatile(&st->gen) != sh_gen) { ok = true; break; }
      __nanosleep(100);
    }
    __threadfence();
    if (ok) {
      sh_beta = *reinterpret_cast<const volatile double*>(&st->beta);
      sh_go = !*reinterpret_cast<const volatile int32_t*>(&st->done);
    } else {
      atomicOr(&st->copy_err, 1);
      sh_go = 0;
    }
  }
  __syncthreads();
  if (!sh_go) return;
  const double b = sh_beta;
  for (int64_t i = lo + threadIdx.x; i < hi; i += kFuseThreads) {
    const int64_t li = i - lo;
    double2 zv, pv;
    if (li < stash) {
      zv = keep[li];
      pv = keep[stash + li];
    } else {
      zv = z2[i];
      pv = p2[i];
    }
    pv.x = zv.x + b * pv.x;
    pv.y = zv.y + b * pv.y;
    p2[i] = pv;
  }
  if (odd) p[n - 1] = z[n - 1] + b * p[n - 1];
}

// ----------------------------------------------------------- BiCGSTAB ----
// Start of iteration `next` (= it + 1) from rho_n = r.r_hat: max-iteration
// stop, rho breakdown, else beta and rho.
__device__ void bi_next_iteration(SolverState* st, int next, double rho_n) {
  if (next > st->max_iter) {
    st->status = EMG_MAX_ITER_REACHED; st->iter = st->max_iter; st->done = 1;
  } else if (fabs(rho_n) < 1e-30) {  // :1031-1035
    st->status = EMG_NUMERICAL_ERROR; st->iter = next; st->done = 1;
  } else {
    st->beta = (rho_n / st->rho) * (st->alpha / st->omega);
    st->rho = rho_n;
    st->iter = next;
  }
}

__global__ void __launch_bounds__(kThreads) k_bi_init(int64_t n, const double* __restrict__ b,
                                                      const int32_t* __restrict__ perm,
                                                      double* __restrict__ x, double* __restrict__ r,
                                                      double* __restrict__ rh, double* __restrict__ p,
                                                      double* __restrict__ v, double* partial,
                                                      SolverState* st) {
  double acc[1] = {0.0};
  for (int64_t i = gtid(); i < n; i += gstride()) {
    const double bi = b[perm[i]];
    x[i] = 0.0; r[i] = bi; rh[i] = bi; p[i] = bi; v[i] = 0.0;
    acc[0] += bi * bi;
  }
  double tot[1];
  if (!reduce_partials<1>(acc, partial, st, tot)) return;
  if (threadIdx.x == 0) {
    const double bn = sqrt(tot[0]);
    st->bnorm = bn;
    st->rho = tot[0];
    st->alpha = 1.0; st->omega = 1.0;
    st->done = 0; st->early = 0; st->dcount = 0;
    st->status = EMG_MAX_ITER_REACHED;
    if (bn < 1e-15) {
      st->status = EMG_SUCCESS; st->iter = 0; st->res = 0.0; st->done = 1;
      return;
    }
    st->res = sqrt(tot[0]) / bn;
    st->prev = st->res;
    bi_next_iteration(st, 1, tot[0]);  // rho of iteration 1 = r.r_hat = b.b
  }
}

// p = r + beta (p - omega v)
__global__ void __launch_bounds__(kThreads) k_bi_p(int64_t n, double* __restrict__ p,
                                                   const double* __restrict__ r,
                                                   const double* __restrict__ v,
                                                   const SolverState* st) {
  if (st->done) return;
  const double b = st->beta, w = st->omega;
  for (int64_t i = gtid(); i < n; i += gstride()) p[i] = r[i] + b * (p[i] - w * v[i]);
}

// v = A p, r_hat . v -> alpha
template <int kMode>
__global__ void __launch_bounds__(kThreads) k_bi_v(Sell A, const double* __restrict__ p,
                                                   double* __restrict__ v,
                                                   const double* __restrict__ rh, double* partial,
                                                   SolverState* st) {
  if (st->done) return;
  double dot = 0.0;
  spmv_rows<kMode>(A, p, [&](int64_t row, double s) {
    v[row] = s;
    dot += rh[row] * s;
  }, &st->copy_err);
  double acc[1] = {dot};
  double tot[1];
  if (!reduce_partials<1>(acc, partial, st, tot)) return;
  if (threadIdx.x == 0) {
    if (st->copy_err) {
      st->status = EMG_ERR_TIMEOUT; st->done = 1;
    } else if (fabs(tot[0]) < 1e-30) {  // :1043-1047
      st->status = EMG_NUMERICAL_ERROR; st->done = 1;
    } else {
      st->alpha = st->rho / tot[0];
    }
  }
}

// s = r - alpha v, z = D^-1 s, ||s|| -> early exit
__global__ void __launch_bounds__(kThreads) k_bi_s(int64_t n, const double* __restrict__ r,
                                                   const double* __restrict__ v,
                                                   const double* __restrict__ dinv,
                                                   double* __restrict__ s, double* __restrict__ z,
                                                   double* partial, SolverState* st) {
  if (st->done) return;
  const double a = st->alpha;
  double acc[1] = {0.0};
  for (int64_t i = gtid(); i < n; i += gstride()) {
    const double si = r[i] - a * v[i];
    s[i] = si;
    z[i] = dinv[i] * si;
    acc[0] += si * si;
  }
  double tot[1];
  if (!reduce_partials<1>(acc, partial, st, tot)) return;
  if (threadIdx.x == 0) {
    const double rs = sqrt(tot[0]) / st->bnorm;
    if (rs < st->tol) {  // :1050-1058
      st->res = rs;
      st->early = 1;
    }
  }
}

// t = A z, t.t and z.t -> omega
template <int kMode>
__global__ void __launch_bounds__(kThreads) k_bi_t(Sell A, const double* __restrict__ z,
                                                   double* __restrict__ t, double* partial,
                                                   SolverState* st) {
  if (st->done || st->early) return;
  double tt = 0.0, zt = 0.0;
  spmv_rows<kMode>(A, z, [&](int64_t row, double s) {
    t[row] = s;
    tt += s * s;
    zt += z[row] * s;
  }, &st->copy_err);
  double acc[2] = {tt, zt};
  double tot[2];
  if (!reduce_partials<2>(acc, partial, st, tot)) return;
  if (threadIdx.x == 0) {
    st->omega = fabs(tot[0]) < 1e-30 ? 0.0 : tot[1] / tot[0];
    if (st->copy_err) { st->status = EMG_ERR_TIMEOUT; st->done = 1; }
  }
}

// x += alpha p + omega z, r = s - omega t; residual checks; next rho
__global__ void __launch_bounds__(kThreads) k_bi_x(int64_t n, double* __restrict__ x,
                                                   double* __restrict__ r,
                                                   const double* __restrict__ p,
                                                   const double* __restrict__ z,
                                                   const double* __restrict__ s,
                                                   const double* __restrict__ t,
                                                   const double* __restrict__ rh, double* partial,
                                                   SolverState* st, double* hist,
                                                   int32_t hist_cap) {
  if (st->done) return;
  const double a = st->alpha;
  if (st->early) {
    for (int64_t i = gtid(); i < n; i += gstride()) x[i] += a * p[i];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      st->status = EMG_SUCCESS;
      const int it = st->iter;
      if (it - 1 < hist_cap) hist[it - 1] = st->res;
    }
    // `done` is raised by the last block so that every block has read
    // `early` before it changes.
    double acc0[1] = {0.0}, tot0[1];
    if (reduce_partials<1>(acc0, partial, st, tot0) && threadIdx.x == 0) st->done = 1;
    return;
  }
  const double w = st->omega;
  double acc[2] = {0.0, 0.0};
  for (int64_t i = gtid(); i < n; i += gstride()) {
    x[i] += a * p[i] + w * z[i];
    const double ri = s[i] - w * t[i];
    r[i] = ri;
    acc[0] += ri * ri;
    acc[1] += ri * rh[i];
  }
  double tot[2];
  if (!reduce_partials<2>(acc, partial, st, tot)) return;
  if (threadIdx.x == 0) {
    const int it = st->iter;
    const double res = sqrt(tot[0]) / st->bnorm;
    st->res = res;
    if (it - 1 < hist_cap) hist[it - 1] = res;
    if (res < st->tol) { st->status = EMG_SUCCESS; st->done = 1; return; }
    if (res > st->prev * 1.5 && it > 20) {  // :1083-1093
      if (++st->dcount >= 3) { st->status = EMG_DIVERGED; st->done = 1; return; }
    } else {
      st->dcount = 0;
    }
    if (it > 10 && res > st->prev * 1000.0) { st->status = EMG_DIVERGED; st->done = 1; return; }
    st->prev = res;
    bi_next_iteration(st, it + 1, tot[1]);
  }
}

// Last node of every while-loop body: keep looping while the solve is not
// done and the body count is below its bound.  The bound is independent of
// the solver state, so the loop ends even if that state were wrong.
__global__ void k_loop_control(SolverState* st, cudaGraphConditionalHandle handle) {
  if (threadIdx.x != 0) return;
  const int loops = st->loops + 1;
  st->loops = loops;
  const bool go = !st->done && loops < st->loop_limit;
  cudaGraphSetConditional(handle, go ? 1u : 0u);
}

int num_sms() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

// Launch shape of the SpMV kernels: the bulk-copy pipeline runs one
// persistent block per SM with its stages in dynamic shared memory.
struct SpmvShape {
  int grid;
  size_t smem;
};
SpmvShape spmv_shape(const Sell& S, int plain_grid) {
  if (S.tma)
    return {tma::kBlocksPerSm * num_sms(),
            tma::smem_bytes(tma::layout_for(static_cast<uint32_t>(S.max_tile_slots)))};
  return {plain_grid, 0};
}

// Grid of a grid-stride solver kernel (SELL SpMV, CG / BiCGSTAB vector
// updates): with EMG_SPMV_RESIDENT, as many blocks as fit on the GPU at once
// (occupancy x SMs, at most `g`), so the loop runs in one wave; otherwise
// `g` (8 blocks per SM, of which 4-5 of the SpMV fit: a second partial wave,
// 63.6 instead of 54.4 us for the 64^3 CG matrix on B200 with the same loop).
#ifndef EMG_SPMV_RESIDENT
#define EMG_SPMV_RESIDENT 1
#endif
template <auto Kernel>
int resident_grid(int g) {
#if EMG_SPMV_RESIDENT
  static int resident = 0;
  if (!resident) {
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, Kernel, kThreads, 0) != cudaSuccess ||
        per_sm < 1 || sms < 1)
      return g;
    resident = per_sm * sms;
  }
  return resident < g ? resident : g;
#else
  return g;
#endif
}

// The SpMV grid: one resident wave, or the autotuned grid of the matrix when
// it is smaller (tune_sell_grid).
template <auto Kernel>
int sell_grid(const Sell& S, int g) {
  const int r = resident_grid<Kernel>(g);
  return S.grid > 0 && S.grid < r ? S.grid : r;
}

int grid_size() {
  static int g = 0;
  if (!g) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    g = sms * 8;  // 8 blocks of 256 threads per SM: 64 resident warps
  }
  return g;
}

// Host: permutation sorting rows by length inside windows (stable), slice
// offsets; device: slots.
int build_sell(DevCsr& A, cudaStream_t st) {
  if (!A.sell) A.sell = new Sell();
  Sell& S = *A.sell;
  const int64_t n = A.n;
  S.n = n;
  // Permutation and slice offsets on the device: a warp per window sorts
  // its rows, a thread per slice takes the longest row, a scan gives offsets.
  const int g = grid_size();
  S.nslices = (n + kSliceRows - 1) / kSliceRows;
  S.ngroups = (S.nslices + kGroup - 1) / kGroup;
  EMG_CK(cudaMallocAsync(&S.perm, sizeof(int32_t) * n, st));
  EMG_CK(cudaMallocAsync(&S.slice_ptr, sizeof(int64_t) * (S.ngroups + 1), st));
  int32_t *slice_slots = nullptr, *slice_off = nullptr;
  EMG_CK(cudaMallocAsync(&slice_slots, sizeof(int32_t) * S.ngroups, st));
  EMG_CK(cudaMallocAsync(&slice_off, sizeof(int32_t) * (S.ngroups + 1), st));
  const int64_t windows = (n + kWindow - 1) / kWindow;
  k_sell_window_perm<<<static_cast<unsigned>(windows), 32, 0, st>>>(n, A.row_ptr, S.perm);
  k_sell_group_slots<<<g, kThreads, 0, st>>>(n, S.ngroups, A.row_ptr, S.perm, slice_slots);
  EMG_CK(cudaGetLastError());
  int64_t total = 0;
  int rc = scan_counts(slice_slots, slice_off, S.ngroups, &total, st);
  if (rc) return rc;
  if (total >= (int64_t(1) << 31)) {
    cudaFreeAsync(slice_slots, st);
    cudaFreeAsync(slice_off, st);
    set_error("matrix too large for the solver format");
    return EMG_INVALID_INPUT;
  }
  k_widen<<<g, kThreads, 0, st>>>(S.ngroups + 1, slice_off, S.slice_ptr);
  EMG_CK(cudaFreeAsync(slice_slots, st));
  EMG_CK(cudaFreeAsync(slice_off, st));
  S.slots = total;
  int32_t* iperm = nullptr;
  const size_t ns = static_cast<size_t>(std::max<int64_t>(S.slots, 1));
  EMG_CK(cudaMallocAsync(&iperm, sizeof(int32_t) * n, st));
  EMG_CK(cudaMallocAsync(&S.src, sizeof(int32_t) * ns, st));
  if (EMG_SELL_PACKED) {  // one buffer: 32-slot chunks of values then columns
    EMG_CK(cudaMallocAsync(&S.val, (sizeof(double) + sizeof(int32_t)) * ns, st));
    S.col = reinterpret_cast<int32_t*>(S.val);
  } else {
    EMG_CK(cudaMallocAsync(&S.col, sizeof(int32_t) * ns, st));
    EMG_CK(cudaMallocAsync(&S.val, sizeof(double) * ns, st));
  }
  k_invert_perm<<<g, kThreads, 0, st>>>(n, S.perm, iperm);
  // every slot of every group is written: slices past the last row are padding
  k_sell_fill<<<g, kThreads, 0, st>>>(n, S.ngroups * kGroup, S.slice_ptr, S.perm, iperm, A.row_ptr, A.col, S.col,
                                      S.src);
  EMG_CK(cudaGetLastError());
  EMG_CK(cudaFreeAsync(iperm, st));
  S.version = ~uint64_t(0);
  S.max_tile_slots = 0;
  S.tma = false;
#if EMG_SELL_TMA
  static_assert(kGroup == 1 && !EMG_SELL_PACKED,
                "the bulk-copy pipeline reads contiguous per-slice runs of separate arrays");
  {
    // bulk-copy pipeline: tiles of 8 slices, kStages stages in shared memory
    std::vector<int64_t> sp(S.nslices + 1);
    EMG_CK(cudaMemcpyAsync(sp.data(), S.slice_ptr, sizeof(int64_t) * (S.nslices + 1), cudaMemcpyDeviceToHost, st));
    EMG_CK(cudaStreamSynchronize(st));
    for (int64_t s0 = 0; s0 < S.nslices; s0 += tma::kWarps) {
      const int64_t s1 = std::min<int64_t>(S.nslices, s0 + tma::kWarps);
      S.max_tile_slots = std::max<int64_t>(S.max_tile_slots, sp[s1] - sp[s0]);
    }
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const size_t need = tma::smem_bytes(tma::layout_for(static_cast<uint32_t>(S.max_tile_slots)));
    if (S.max_tile_slots > 0 && need <= static_cast<size_t>(optin)) {
      const int b = static_cast<int>(need);
      EMG_CK(cudaFuncSetAttribute(k_cg_spmv_dot<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
      EMG_CK(cudaFuncSetAttribute(k_bi_v<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
      EMG_CK(cudaFuncSetAttribute(k_bi_t<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
      EMG_CK(cudaFuncSetAttribute(k_spmv<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
      S.tma = true;
    }
  }
#endif
  S.ws = false;
#if EMG_SELL_WS
  static_assert(kGroup == 1 && !EMG_SELL_PACKED, "the warp-specialized SpMV copies per-slice runs");
  if (!S.tma && S.nslices > 0) {
    std::vector<int64_t> sp(S.nslices + 1);
    EMG_CK(cudaMemcpyAsync(sp.data(), S.slice_ptr, sizeof(int64_t) * (S.nslices + 1), cudaMemcpyDeviceToHost, st));
    EMG_CK(cudaStreamSynchronize(st));
    int64_t mx = 0;
    for (int64_t s = 0; s < S.nslices; ++s) mx = std::max<int64_t>(mx, sp[s + 1] - sp[s]);
    const uint32_t sb = static_cast<uint32_t>(((12 * mx + 127) / 128) * 128);
    const size_t need = ws_smem_bytes(sb);
    int dev = 0, optin = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (mx > 0 && need <= static_cast<size_t>(optin)) {
      const int b = static_cast<int>(need);
      EMG_CK(cudaFuncSetAttribute(k_cg_spmv_dot<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
      EMG_CK(cudaFuncSetAttribute(k_bi_v<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
      EMG_CK(cudaFuncSetAttribute(k_bi_t<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
      EMG_CK(cudaFuncSetAttribute(k_spmv<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
      EMG_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_cg_spmv_dot<3>, kThreads, need));
      if (per > 0) {
        S.ws = true;
        S.ws_stage_bytes = sb;
        S.ws_smem = need;
        S.ws_grid = std::min(per * sms, grid_size());
      }
    }
  }
#endif
  // 16-bit column offsets when every |column - row| fits (banded numberings,
  // e.g. first-appearance edge IDs of structured meshes): 10 bytes per slot.
  S.narrow = false;
  if (EMG_SELL_NARROW && !EMG_SELL_PACKED && !S.tma && !S.ws && S.slots > 0) {
    int32_t* overflow = nullptr;
    EMG_CK(cudaMallocAsync(&S.dcol, sizeof(int16_t) * S.slots, st));
    EMG_CK(cudaMallocAsync(&overflow, sizeof(int32_t), st));
    EMG_CK(cudaMemsetAsync(overflow, 0, sizeof(int32_t), st));
    k_sell_narrow<<<g, kThreads, 0, st>>>(S.nslices, S.slice_ptr, S.col, S.dcol, overflow);
    int32_t h_over = 0;
    EMG_CK(cudaMemcpyAsync(&h_over, overflow, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    EMG_CK(cudaStreamSynchronize(st));
    EMG_CK(cudaFreeAsync(overflow, st));
    if (h_over) {
      EMG_CK(cudaFreeAsync(S.dcol, st));
      S.dcol = nullptr;
    } else {
      EMG_CK(cudaFreeAsync(S.col, st));
      S.col = nullptr;
      S.narrow = true;
    }
  }
  return EMG_SUCCESS;
}

void tune_sell_grid(DevCsr& A, cudaStream_t st);

int ensure_sell(DevCsr& A, cudaStream_t st) {
  bool fresh = false;
  if (!A.sell) {
    int rc = build_sell(A, st);
    if (rc) return rc;
    fresh = true;
  }
  Sell& S = *A.sell;
  if (S.version != A.version) {
    k_sell_values<<<grid_size(), kThreads, 0, st>>>(S.slots, S.src, A.val, S.val);
    EMG_CK(cudaGetLastError());
    S.version = A.version;
  }
  if (fresh && A.ws) tune_sell_grid(A, st);
  return EMG_SUCCESS;
}

void free_sell(Sell* s) {
  if (!s) return;
  void* col = static_cast<void*>(s->col) == static_cast<void*>(s->val) ? nullptr : static_cast<void*>(s->col);
  for (void* p : {static_cast<void*>(s->perm), static_cast<void*>(s->slice_ptr), col,
                  static_cast<void*>(s->dcol), static_cast<void*>(s->src), static_cast<void*>(s->val)})
    if (p) cudaFreeAsync(p, 0);
  delete s;
}

// Pinned host blocks for the solver-state read-back, recycled for the life of
// the process: page-locking and releasing a block per solver
// (cudaMallocHost / cudaFreeHost) costs about a millisecond per solve and,
// measured on B200 boxes, occasionally 50-500 ms inside cudaFreeHost.
// The pool is never destroyed, so workspaces released during process exit
// still find it.
constexpr size_t kPinnedBlock = 256;
static_assert(sizeof(SolverState) <= kPinnedBlock, "solver state must fit a pinned block");
struct PinnedPool {
  std::mutex mu;
  std::vector<void*> free;
};
PinnedPool& pinned_pool() {
  static PinnedPool* p = new PinnedPool();
  return *p;
}

int pinned_state_alloc(SolverState** out) {
  PinnedPool& pool = pinned_pool();
  std::lock_guard<std::mutex> lock(pool.mu);
  if (pool.free.empty()) {
    constexpr int kBlocks = 64;
    char* chunk = nullptr;
    EMG_CK(cudaMallocHost(&chunk, kPinnedBlock * kBlocks));
    for (int b = kBlocks - 1; b >= 0; --b) pool.free.push_back(chunk + kPinnedBlock * b);
  }
  *out = static_cast<SolverState*>(pool.free.back());
  pool.free.pop_back();
  return EMG_SUCCESS;
}

void pinned_state_free(SolverState* p) {
  if (!p) return;
  PinnedPool& pool = pinned_pool();
  std::lock_guard<std::mutex> lock(pool.mu);
  pool.free.push_back(p);
}

// Capture streams and timing events of released workspaces, kept per device
// and handed to the next workspace instead of being destroyed and created
// for every solve (never destroyed, like the pinned blocks above).
struct HandlePool {
  std::mutex mu;
  std::vector<std::pair<int, cudaStream_t>> streams;
  std::vector<std::pair<int, cudaEvent_t>> events;
};
HandlePool& handle_pool() {
  static HandlePool* p = new HandlePool();
  return *p;
}

int take_stream(cudaStream_t* out) {
  int dev = 0;
  EMG_CK(cudaGetDevice(&dev));
  {
    HandlePool& hp = handle_pool();
    std::lock_guard<std::mutex> lock(hp.mu);
    for (size_t i = 0; i < hp.streams.size(); ++i)
      if (hp.streams[i].first == dev) {
        *out = hp.streams[i].second;
        hp.streams.erase(hp.streams.begin() + static_cast<int64_t>(i));
        return EMG_SUCCESS;
      }
  }
  EMG_CK(cudaStreamCreate(out));
  return EMG_SUCCESS;
}

int take_event(cudaEvent_t* out) {
  int dev = 0;
  EMG_CK(cudaGetDevice(&dev));
  {
    HandlePool& hp = handle_pool();
    std::lock_guard<std::mutex> lock(hp.mu);
    for (size_t i = 0; i < hp.events.size(); ++i)
      if (hp.events[i].first == dev) {
        *out = hp.events[i].second;
        hp.events.erase(hp.events.begin() + static_cast<int64_t>(i));
        return EMG_SUCCESS;
      }
  }
  EMG_CK(cudaEventCreate(out));
  return EMG_SUCCESS;
}

// Returns a stream / events of device `dev` to the pool; the stream is first
// drained so that the next owner starts on an idle stream.
void give_back(int dev, cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1) {
  if (dev < 0) return;
  if (s) cudaStreamSynchronize(s);
  HandlePool& hp = handle_pool();
  std::lock_guard<std::mutex> lock(hp.mu);
  if (s) hp.streams.emplace_back(dev, s);
  for (cudaEvent_t e : {e0, e1})
    if (e) hp.events.emplace_back(dev, e);
}

// Workspace vectors come from the stream-ordered pool (allocated on `st`,
// returned with cudaFreeAsync once the device is idle).
// Fused CG update + direction: used when the device takes cooperative
// launches and one block of kFuseThreads with its shared-memory stash fits
// on every SM; otherwise the two-kernel update stays.
#ifndef EMG_CG_FUSE
#define EMG_CG_FUSE 1
#endif
void setup_fuse(KrylovWorkspace& w) {
  w.fuse = false;
  if (!EMG_CG_FUSE || w.n < 2) return;
  int dev = 0, coop = 0, sms = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
      !coop || sms < 1) {
    cudaGetLastError();
    return;
  }
  cudaFuncAttributes fa;
  if (cudaFuncGetAttributes(&fa, k_cg_update_dir) != cudaSuccess) { cudaGetLastError(); return; }
  const int64_t room = (static_cast<int64_t>(optin) - static_cast<int64_t>(fa.sharedSizeBytes)) / 32;
  if (room < 1) return;
  const int64_t n2 = w.n / 2;
  const int64_t per = (n2 + sms - 1) / sms;
  const int64_t stash = per < room ? per : room;
  const size_t smem = static_cast<size_t>(stash) * 32;
  int per_sm = 0;
  if (cudaFuncSetAttribute(k_cg_update_dir, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(room * 32)) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cg_update_dir, kFuseThreads, smem) != cudaSuccess ||
      per_sm < 1) {
    cudaGetLastError();
    return;
  }
  w.fuse_grid = sms;  // one block per SM: at most the co-resident count
  w.fuse_smem = smem;
  w.fuse_stash = stash;
  w.fuse = w.fuse_grid <= 4 * w.grid;  // the partial sums fit w.partial
}

// One fused CG update + direction (cooperative: all blocks co-resident).
void launch_update_dir(KrylovWorkspace& w, int64_t n, cudaStream_t st) {
  cudaLaunchConfig_t c = {};
  c.gridDim = dim3(static_cast<unsigned>(w.fuse_grid));
  c.blockDim = dim3(kFuseThreads);
  c.dynamicSmemBytes = w.fuse_smem;
  c.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  c.attrs = at;
  c.numAttrs = 1;
  cudaLaunchKernelEx(&c, k_cg_update_dir, n, w.x, w.r, w.z, w.p, static_cast<const double*>(w.q),
                     static_cast<const double*>(w.dinv), w.partial, w.state, w.hist, w.hist_cap,
                     w.fuse_stash);
}

int ensure_ws(DevCsr& A, bool bicg, int32_t max_iter, cudaStream_t st) {
  if (!A.ws) {
    A.ws = new KrylovWorkspace();
    KrylovWorkspace& w = *A.ws;
    w.n = A.n;
    w.grid = grid_size();
    const size_t vb = sizeof(double) * (A.n > 0 ? A.n : 1);
    for (double** v : {&w.dinv, &w.x, &w.r, &w.z, &w.p, &w.q})
      EMG_CK(cudaMallocAsync(v, vb, st));
    EMG_CK(cudaMallocAsync(&w.partial, sizeof(double) * 4 * w.grid, st));
    EMG_CK(cudaMallocAsync(&w.state, sizeof(SolverState), st));
    EMG_CK(cudaStreamSynchronize(st));
    EMG_CK(cudaMemset(w.state, 0, sizeof(SolverState)));
    if (int rc = pinned_state_alloc(&w.state_h)) return rc;
    EMG_CK(cudaGetDevice(&w.dev));
    setup_fuse(w);
    if (int rc = take_stream(&w.cap)) return rc;
    if (int rc = take_event(&w.ev0)) return rc;
    if (int rc = take_event(&w.ev1)) return rc;
  }
  KrylovWorkspace& w = *A.ws;
  if (bicg && !w.rh) {
    const size_t vb = sizeof(double) * (A.n > 0 ? A.n : 1);
    for (double** v : {&w.rh, &w.v, &w.s, &w.t}) EMG_CK(cudaMallocAsync(v, vb, st));
    EMG_CK(cudaStreamSynchronize(st));
  }
  if (max_iter > w.hist_cap) {
    if (w.hist) EMG_CK(cudaFreeAsync(w.hist, st));
    w.hist_cap = max_iter;
    EMG_CK(cudaMallocAsync(&w.hist, sizeof(double) * w.hist_cap, st));
    EMG_CK(cudaStreamSynchronize(st));
    // the chunk graphs hold the old pointer
    for (cudaGraphExec_t* g : {&w.cg_exec, &w.bi_exec, &w.cg_loop, &w.bi_loop})
      if (*g) { cudaGraphExecDestroy(*g); *g = nullptr; }
  }
  return EMG_SUCCESS;
}

void launch_iterations(DevCsr& A, bool bicg, int count);

// The whole solve as one graph: a conditional while-node whose body runs
// kBody iterations and then k_loop_control.
int capture_loop(DevCsr& A, bool bicg, cudaGraphExec_t* out) {
  KrylovWorkspace& w = *A.ws;
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
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    cudaGetLastError();
    set_error(std::string("conditional graph node: ") + cudaGetErrorString(e));
    return EMG_ERR_CUDA;
  }
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  e = cudaStreamBeginCaptureToGraph(w.cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    launch_iterations(A, bicg, kBody);
    k_loop_control<<<1, 32, 0, w.cap>>>(w.state, handle);
    e = cudaStreamEndCapture(w.cap, &body);
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(out, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error(std::string("while-loop graph: ") + cudaGetErrorString(e));
    return EMG_ERR_CUDA;
  }
  return EMG_SUCCESS;
}

// Launches KERNEL<mode> for the storage format of S: the bulk-copy pipeline
// (mode 2, persistent grid + dynamic shared memory), 16-bit column offsets
// (mode 1) or 32-bit columns (mode 0).
#define EMG_LAUNCH_SPMV(KERNEL, S, g, st, ...)                                        \
  do {                                                                                \
    if ((S).tma) {                                                                    \
      const SpmvShape sh_ = spmv_shape(S, g);                                         \
      KERNEL<2><<<sh_.grid, kThreads, sh_.smem, st>>>(__VA_ARGS__);                   \
    } else if (EMG_WS_LAUNCH(KERNEL, S, st, __VA_ARGS__)) {                           \
    } else if ((S).narrow) {                                                          \
      KERNEL<1><<<sell_grid<KERNEL<1>>(S, g), kThreads, 0, st>>>(__VA_ARGS__);         \
    } else {                                                                          \
      KERNEL<0><<<sell_grid<KERNEL<0>>(S, g), kThreads, 0, st>>>(__VA_ARGS__);         \
    }                                                                                 \
  } while (0)

#if EMG_SELL_WS
#define EMG_WS_LAUNCH(KERNEL, S, st, ...) \
  ((S).ws ? (KERNEL<3><<<(S).ws_grid, kThreads, (S).ws_smem, st>>>(__VA_ARGS__), true) : false)
#else
#define EMG_WS_LAUNCH(KERNEL, S, st, ...) false
#endif

// Blocks per SM of the register-pipeline SpMV (the SELL kernel without the
// solver's dot product, whose loads and occupancy are the same), chosen by
// the autotuner for this matrix shape: one resident wave (the default) or
// one or two blocks per SM fewer, timed on the matrix itself.
void tune_sell_grid(DevCsr& A, cudaStream_t st) {
  Sell& S = *A.sell;
  if (S.tma || S.ws) return;
  const int g = grid_size(), sms = num_sms();
  const int r = S.narrow ? resident_grid<k_spmv<1>>(g) : resident_grid<k_spmv<0>>(g);
  std::vector<int> cand{r};
  for (int d = 1; d <= 2; ++d)
    if (r - d * sms >= sms) cand.push_back(r - d * sms);
  int32_t* err = &A.ws->state->copy_err;
  const std::string key = "n" + std::to_string(A.n) + "slots" + std::to_string(S.slots);
  S.grid = tune::pick("sell.spmv_grid", key, cand, [&](int v, cudaStream_t s) {
    if (S.narrow) k_spmv<1><<<v, kThreads, 0, s>>>(S, A.ws->p, A.ws->q, err);
    else k_spmv<0><<<v, kThreads, 0, s>>>(S, A.ws->p, A.ws->q, err);
  }, st);
  cudaGetLastError();
}

void launch_iterations(DevCsr& A, bool bicg, int count) {
  KrylovWorkspace& w = *A.ws;
  const Sell S = *A.sell;
  const int g = w.grid;
  for (int c = 0; c < count; ++c) {
    if (!bicg) {
      EMG_LAUNCH_SPMV(k_cg_spmv_dot, S, g, w.cap, S, w.p, w.q, w.partial, w.state);
      if (w.fuse) {
        launch_update_dir(w, A.n, w.cap);
      } else {
        k_cg_update<<<resident_grid<k_cg_update>(g), kThreads, 0, w.cap>>>(
            A.n, w.x, w.r, w.z, w.p, w.q, w.dinv, w.partial, w.state, w.hist, w.hist_cap);
        k_cg_direction<<<resident_grid<k_cg_direction>(g), kThreads, 0, w.cap>>>(A.n, w.p, w.z, w.state);
      }
    } else {
      k_bi_p<<<resident_grid<k_bi_p>(g), kThreads, 0, w.cap>>>(A.n, w.p, w.r, w.v, w.state);
      EMG_LAUNCH_SPMV(k_bi_v, S, g, w.cap, S, w.p, w.v, w.rh, w.partial, w.state);
      k_bi_s<<<resident_grid<k_bi_s>(g), kThreads, 0, w.cap>>>(A.n, w.r, w.v, w.dinv, w.s, w.z, w.partial, w.state);
      EMG_LAUNCH_SPMV(k_bi_t, S, g, w.cap, S, w.z, w.t, w.partial, w.state);
      k_bi_x<<<resident_grid<k_bi_x>(g), kThreads, 0, w.cap>>>(A.n, w.x, w.r, w.p, w.z, w.s, w.t, w.rh, w.partial, w.state,
                                        w.hist, w.hist_cap);
    }
  }
}

int capture_chunk(DevCsr& A, bool bicg, cudaGraphExec_t* out) {
  KrylovWorkspace& w = *A.ws;
  cudaGraph_t graph = nullptr;
  EMG_CK(cudaStreamBeginCapture(w.cap, cudaStreamCaptureModeThreadLocal));
  launch_iterations(A, bicg, kChunk);
  cudaError_t e = cudaStreamEndCapture(w.cap, &graph);
  if (e != cudaSuccess) { set_error(std::string("graph capture: ") + cudaGetErrorString(e)); return EMG_ERR_CUDA; }
  e = cudaGraphInstantiate(out, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) { set_error(std::string("graph instantiate: ") + cudaGetErrorString(e)); return EMG_ERR_CUDA; }
  return EMG_SUCCESS;
}

int run_solver(DevCsr& A, const double* b, double* x, const emg_krylov_config& cfg,
               cudaStream_t user, emg_result* res, bool bicg) {
  std::memset(res, 0, sizeof(*res));
  res->status = EMG_INVALID_INPUT;
  if (!b || !x) { set_error("null vector"); return EMG_INVALID_INPUT; }
  if (A.n <= 0) { set_error("empty matrix"); return EMG_INVALID_INPUT; }
  if (check_krylov_precond(cfg.preconditioner, true)) return EMG_INVALID_INPUT;
  const int32_t max_iter = cfg.max_iterations;
  int rc;
  {
    TraceScope t("solve.workspace");
    rc = ensure_ws(A, bicg, max_iter > 0 ? max_iter : 1, user);
  }
  if (rc) { res->status = rc; return rc; }
  KrylovWorkspace& w = *A.ws;
  cudaStream_t st = user ? user : w.cap;
  {
    trace_pool("solve.sell.begin");
    TraceScope t("solve.sell");
    rc = ensure_sell(A, st);
  }
  trace_pool("solve.sell.end");
  if (rc) { res->status = rc; return rc; }
  // Preferred: the whole solve as one graph with a device while-loop; else
  // host-polled chunks of kChunk iterations.
  cudaGraphExec_t* loop = bicg ? &w.bi_loop : &w.cg_loop;
  if (!*loop && !w.loop_unavailable) {
    TraceScope t("solve.capture_loop");
    int crc = capture_loop(A, bicg, loop);
    if (crc != EMG_SUCCESS && w.fuse && !bicg) {  // retry with the two-kernel update
      w.fuse = false;
      *loop = nullptr;
      crc = capture_loop(A, bicg, loop);
    }
    if (crc != EMG_SUCCESS) {
      w.loop_unavailable = true;
      *loop = nullptr;
    }
  }
  cudaGraphExec_t* exec = bicg ? &w.bi_exec : &w.cg_exec;
  if (!*loop && !*exec) {
    rc = capture_chunk(A, bicg, exec);
    if (rc && w.fuse && !bicg) {
      w.fuse = false;
      *exec = nullptr;
      rc = capture_chunk(A, bicg, exec);
    }
    if (rc) { res->status = rc; return rc; }
  }
  const Sell& S = *A.sell;
  SolverState init;
  std::memset(&init, 0, sizeof(init));
  init.tol = cfg.tolerance;
  init.max_iter = max_iter;
  init.loop_limit = (max_iter > 0 ? max_iter : 0) / kBody + 2;
  *w.state_h = init;
  EMG_CK(cudaEventRecord(w.ev0, st));
  EMG_CK(cudaMemcpyAsync(w.state, w.state_h, sizeof(SolverState), cudaMemcpyHostToDevice, st));
  const int g = w.grid;
  k_jacobi<<<g, kThreads, 0, st>>>(A.n, A.row_ptr, A.col, A.val, S.perm, cfg.preconditioner, w.dinv);
  if (!bicg)
    k_cg_init<<<g, kThreads, 0, st>>>(A.n, b, S.perm, w.dinv, w.x, w.r, w.z, w.p, w.partial, w.state);
  else
    k_bi_init<<<g, kThreads, 0, st>>>(A.n, b, S.perm, w.x, w.r, w.rh, w.p, w.v, w.partial, w.state);
  EMG_CK(cudaGetLastError());
  // Graph chunks until the device state says done; bounded by max_iter.
  const int64_t max_chunks = (static_cast<int64_t>(max_iter > 0 ? max_iter : 0) + kChunk - 1) / kChunk + 1;
  bool done = false;
  if (*loop) {
    EMG_CK(cudaGraphLaunch(*loop, st));
    k_scatter<<<g, kThreads, 0, st>>>(A.n, S.perm, w.x, x);
    EMG_CK(cudaEventRecord(w.ev1, st));
    EMG_CK(cudaMemcpyAsync(w.state_h, w.state, sizeof(SolverState), cudaMemcpyDeviceToHost, st));
    EMG_CK(cudaStreamSynchronize(st));
    done = w.state_h->done != 0;
  } else {
    for (int64_t c = 0; c <= max_chunks; ++c) {
      EMG_CK(cudaMemcpyAsync(w.state_h, w.state, sizeof(SolverState), cudaMemcpyDeviceToHost, st));
      EMG_CK(cudaStreamSynchronize(st));
      if (w.state_h->done) { done = true; break; }
      EMG_CK(cudaGraphLaunch(*exec, st));
    }
    k_scatter<<<g, kThreads, 0, st>>>(A.n, S.perm, w.x, x);
    EMG_CK(cudaEventRecord(w.ev1, st));
    EMG_CK(cudaStreamSynchronize(st));
  }
  float ms = 0.0f;
  EMG_CK(cudaEventElapsedTime(&ms, w.ev0, w.ev1));
  if (!done) {
    set_error("solver state did not finish within the iteration bound");
    res->status = EMG_ERR_INTERNAL;
    return EMG_ERR_INTERNAL;
  }
  const SolverState& s = *w.state_h;
  res->status = s.status;
  res->iterations = s.iter;
  res->residual_norm = s.res;
  res->solve_time_ms = ms;
  w.hist_len = s.iter < w.hist_cap ? s.iter : w.hist_cap;
  if (w.hist_len < 0) w.hist_len = 0;
  return s.status;
}

}  // namespace

int csr_spmv(DevCsr& A, const double* x, double* y, cudaStream_t st) {
  if (!x || !y) { set_error("null vector"); return EMG_INVALID_INPUT; }
  int rc = ensure_ws(A, false, 1, st);
  if (rc) return rc;
  rc = ensure_sell(A, st);
  if (rc) return rc;
  const int g = grid_size();
  const Sell& S = *A.sell;
  // the workspace vectors hold the permuted operands
  k_gather<<<g, kThreads, 0, st>>>(A.n, S.perm, x, A.ws->p);
  int32_t* err = &A.ws->state->copy_err;
  EMG_CK(cudaMemsetAsync(err, 0, sizeof(int32_t), st));
  EMG_LAUNCH_SPMV(k_spmv, S, g, st, S, A.ws->p, A.ws->q, err);
  k_scatter<<<g, kThreads, 0, st>>>(A.n, S.perm, A.ws->q, y);
  EMG_CK(cudaGetLastError());
  return EMG_SUCCESS;
}

int cg_solve(DevCsr& A, const double* b, double* x, const emg_krylov_config& cfg, cudaStream_t st,
             emg_result* res) {
  if (cfg.preconditioner == EMG_PRECOND_ILU0) return ilu_solve(A, b, x, cfg, st, res, false);
  return run_solver(A, b, x, cfg, st, res, false);
}

int bicgstab_solve(DevCsr& A, const double* b, double* x, const emg_krylov_config& cfg,
                   cudaStream_t st, emg_result* res) {
  if (cfg.preconditioner == EMG_PRECOND_ILU0) return ilu_solve(A, b, x, cfg, st, res, true);
  return run_solver(A, b, x, cfg, st, res, true);
}

int set_barrier_spins(int32_t spins) {
  const int32_t v = spins < 0 ? kBarrierSpins : spins;
  EMG_CK(cudaMemcpyToSymbol(g_barrier_spins, &v, sizeof(v)));
  return EMG_SUCCESS;
}

int cg_kernel_times(DevCsr& A, int32_t iterations, cudaStream_t user, double* ms) {
  if (iterations <= 0 || !ms) { set_error("bad arguments"); return EMG_INVALID_INPUT; }
  int rc = ensure_ws(A, false, 1, user);
  if (rc) return rc;
  KrylovWorkspace& w = *A.ws;
  cudaStream_t st = user ? user : w.cap;
  rc = ensure_sell(A, st);
  if (rc) return rc;
  const Sell S = *A.sell;
  const int g = w.grid;
  double* ones = nullptr;
  EMG_CK(cudaMallocAsync(&ones, sizeof(double) * A.n, st));
  std::vector<double> h(A.n, 1.0);
  EMG_CK(cudaMemcpyAsync(ones, h.data(), sizeof(double) * A.n, cudaMemcpyHostToDevice, st));
  SolverState init;
  std::memset(&init, 0, sizeof(init));
  init.tol = 0.0;
  init.max_iter = 1 << 30;
  *w.state_h = init;
  EMG_CK(cudaMemcpyAsync(w.state, w.state_h, sizeof(SolverState), cudaMemcpyHostToDevice, st));
  k_jacobi<<<g, kThreads, 0, st>>>(A.n, A.row_ptr, A.col, A.val, S.perm, 1, w.dinv);
  k_cg_init<<<g, kThreads, 0, st>>>(A.n, ones, S.perm, w.dinv, w.x, w.r, w.z, w.p, w.partial, w.state);
  std::vector<cudaEvent_t> ev(4 * iterations);
  for (auto& e : ev) EMG_CK(cudaEventCreate(&e));
  for (int i = 0; i < iterations; ++i) {
    EMG_CK(cudaEventRecord(ev[4 * i], st));
    EMG_LAUNCH_SPMV(k_cg_spmv_dot, S, g, st, S, w.p, w.q, w.partial, w.state);
    EMG_CK(cudaEventRecord(ev[4 * i + 1], st));
    if (w.fuse) {  // the fused update + direction counts as the update
      launch_update_dir(w, A.n, st);
      EMG_CK(cudaEventRecord(ev[4 * i + 2], st));
    } else {
      k_cg_update<<<resident_grid<k_cg_update>(g), kThreads, 0, st>>>(
          A.n, w.x, w.r, w.z, w.p, w.q, w.dinv, w.partial, w.state, w.hist, w.hist_cap);
      EMG_CK(cudaEventRecord(ev[4 * i + 2], st));
      k_cg_direction<<<resident_grid<k_cg_direction>(g), kThreads, 0, st>>>(A.n, w.p, w.z, w.state);
    }
    EMG_CK(cudaEventRecord(ev[4 * i + 3], st));
  }
  EMG_CK(cudaGetLastError());
  EMG_CK(cudaStreamSynchronize(st));
  EMG_CK(cudaMemcpy(w.state_h, w.state, sizeof(SolverState), cudaMemcpyDeviceToHost));
  double acc[3] = {0, 0, 0};
  for (int i = 0; i < iterations; ++i)
    for (int k = 0; k < 3; ++k) {
      float t = 0.0f;
      EMG_CK(cudaEventElapsedTime(&t, ev[4 * i + k], ev[4 * i + k + 1]));
      acc[k] += t;
    }
  for (auto& e : ev) cudaEventDestroy(e);
  EMG_CK(cudaFreeAsync(ones, st));
  EMG_CK(cudaStreamSynchronize(st));
  if (w.state_h->done) {
    set_error("solver state finished during kernel timing (breakdown)");
    return EMG_NUMERICAL_ERROR;
  }
  for (int k = 0; k < 3; ++k) ms[k] = acc[k] / iterations;
  return EMG_SUCCESS;
}

int csr_history(DevCsr& A, double* out, int32_t cap) {
  if (!A.ws || !A.ws->hist || A.ws->hist_len <= 0) return 0;
  int32_t n = A.ws->hist_len < cap ? A.ws->hist_len : cap;
  if (n <= 0) return 0;
  EMG_CK(cudaMemcpy(out, A.ws->hist, sizeof(double) * n, cudaMemcpyDeviceToHost));
  return n;
}

int64_t sell_slots(DevCsr& A) { return A.sell ? A.sell->slots : -1; }
int64_t sell_slices(DevCsr& A) { return A.sell ? A.sell->nslices : -1; }

void free_workspace(KrylovWorkspace* w) {
  if (!w) return;
  {
    TraceScope t("free_workspace.graphs");
    for (cudaGraphExec_t g : {w->cg_exec, w->bi_exec, w->cg_loop, w->bi_loop})
      if (g) cudaGraphExecDestroy(g);
  }
  {
    TraceScope t("free_workspace.vectors");
    for (double* p : {w->dinv, w->x, w->r, w->z, w->p, w->q, w->rh, w->v, w->s, w->t, w->partial, w->hist})
      if (p) cudaFreeAsync(p, 0);
    if (w->state) cudaFreeAsync(w->state, 0);
  }
  {
    TraceScope t("free_workspace.host_state");
    pinned_state_free(w->state_h);
  }
  {
    TraceScope t("free_workspace.stream_events");
    give_back(w->dev, w->cap, w->ev0, w->ev1);
  }
  delete w;
}

// Pattern and values come from the stream-ordered pool (cudaMallocAsync).
DevCsr::~DevCsr() {
  free_ilu(ilu);
  free_workspace(ws);
  free_sell(sell);
  free_batch(batch);
  if (owns_pattern) {
    if (row_ptr) cudaFreeAsync(row_ptr, 0);
    if (col) cudaFreeAsync(col, 0);
  }
  if (owns_values && val) cudaFreeAsync(val, 0);
}

}  // namespace emg

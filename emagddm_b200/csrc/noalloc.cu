// noalloc.cu -- Jacobi/plain CG on a caller-owned device CSR without any
// device allocation (emg_cg_solve_noalloc).
//
// Who needs it: callers that cannot let a library allocate GPU memory -- a
// host application that reserves and budgets all device memory itself (a
// larger simulation embedding this solver next to its own buffers), and
// latency-bound loops that must not call the CUDA allocator after start-up,
// because cudaMalloc / cudaFree synchronize the device and take unbounded
// time.  emg_cg_solve_device allocates its workspace (vectors, reduction
// partials, the solver format, graphs) on first use; this entry point uses a
// fixed scratch array compiled into the library instead.
//
// The scratch is a file-scope __device__ array sized for kMaxRows rows: five
// work vectors plus reduction partials and the solver state, about 10 MiB.
// Every GPU that loads the library holds it until the process exits.  All
// calls share it and it keeps the last call's contents, so every call clears
// what must start at zero (the solver state and its reduction ticket) before
// use, and two calls whose work overlaps on the GPU (different streams or
// host threads) race on it.
//
// Host code cannot use the array's name as a device address: the first call
// on each device (with that device current) looks the address up with
// cudaGetSymbolAddress and caches it; that first call should come before any
// stream capture.
//
// Every call blocks the calling host thread until the solve has finished: it
// synchronizes the stream after the input check and then reads the solver
// state back every kPollEvery iterations to decide whether to launch more.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "common.cuh"
#include "device.h"

namespace emg {
namespace {

constexpr int64_t kMaxRows = int64_t(1) << 18;  // 262,144 equations
constexpr int kThreads = 256;
constexpr int kGrid = 592;          // 4 blocks per SM on a 148-SM B200
constexpr int kLanes = 8;           // lanes per CSR row
constexpr int kPollEvery = 16;      // iterations between host polls of the state
constexpr int kMaxDevices = 64;

struct NaState {  // solver state at the end of the scratch array
  double tol, bnorm, rz, alpha, beta, res, prev;
  int32_t max_iter, iter, status, done;
  uint32_t ticket;
  int32_t pad[3];
};

constexpr int64_t kVecDoubles = 5 * kMaxRows;                 // dinv, r, z, p, q
constexpr int64_t kPartialDoubles = 2 * kGrid;
constexpr int64_t kStateDoubles = (sizeof(NaState) + 7) / 8;
constexpr int64_t kScratchDoubles = kVecDoubles + kPartialDoubles + kStateDoubles;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

struct Scratch {
  double *dinv, *r, *z, *p, *q, *partial;
  NaState* st;
};

Scratch carve(double* base) {
  Scratch s;
  s.dinv = base;
  s.r = base + kMaxRows;
  s.z = base + 2 * kMaxRows;
  s.p = base + 3 * kMaxRows;
  s.q = base + 4 * kMaxRows;
  s.partial = base + kVecDoubles;
  s.st = reinterpret_cast<NaState*>(base + kVecDoubles + kPartialDoubles);
  return s;
}

__device__ __forceinline__ int64_t tid() { return static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; }
__device__ __forceinline__ int64_t nthreads() { return static_cast<int64_t>(gridDim.x) * blockDim.x; }

// Deterministic block partial + last-block total (ticket in the state).
template <int K>
__device__ __forceinline__ bool reduce(const double (&v)[K], double* partial, NaState* st, double (&tot)[K]) {
  __shared__ double red[kThreads / 32];
  __shared__ bool last;
  for (int k = 0; k < K; ++k) {
    const double b = block_sum(v[k], red);
    if (threadIdx.x == 0) partial[k * gridDim.x + blockIdx.x] = b;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(&st->ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return false;
  __threadfence();
  for (int k = 0; k < K; ++k) {
    double a = 0.0;
    for (int i = threadIdx.x; i < static_cast<int>(gridDim.x); i += blockDim.x) a += ld_l2(partial + k * gridDim.x + i);
    tot[k] = block_sum(a, red);
  }
  if (threadIdx.x == 0) st->ticket = 0;
  return true;
}

// Clears the solver state: the scratch keeps the previous call's contents.
__global__ void k_na_reset(NaState* st, double tol, int32_t max_iter) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    NaState z;
    memset(&z, 0, sizeof(z));
    z.tol = tol;
    z.max_iter = max_iter;
    *st = z;
  }
}

// Input check before any indexed access: offsets monotone and inside
// [0, nnz], columns inside [0, n) and strictly ascending within each row (a
// merged CSR, the form emg_csr_create_device takes; with it the Jacobi
// diagonal below is the row's single diagonal entry, as in
// emg_cg_solve_device).  Flags land in st->pad[0].
__global__ void k_na_check(int64_t n, int64_t nnz, const int32_t* __restrict__ rp,
                           const int32_t* __restrict__ col, NaState* st) {
  for (int64_t i = tid(); i < n; i += nthreads()) {
    const int32_t a = rp[i], b = rp[i + 1];
    if (a < 0 || b < a || b > nnz || (i == 0 && a != 0)) {
      atomicOr(&st->pad[0], 1);
      continue;
    }
    for (int32_t k = a; k < b; ++k) {
      if (col[k] < 0 || col[k] >= n) { atomicOr(&st->pad[0], 2); break; }
      if (k > a && col[k] <= col[k - 1]) { atomicOr(&st->pad[0], 4); break; }
    }
  }
}

__global__ void k_na_init(int64_t n, const int32_t* __restrict__ rp, const int32_t* __restrict__ col,
                          const double* __restrict__ val, const double* __restrict__ b, int precond,
                          double* __restrict__ x, Scratch s) {
  double acc[2] = {0.0, 0.0};
  for (int64_t i = tid(); i < n; i += nthreads()) {
    double d = 1.0;
    if (precond) {  // 1 / A(i,i), or 1 where |A(i,i)| <= 1e-15
      double a = 0.0;
      for (int32_t k = rp[i]; k < rp[i + 1]; ++k)
        if (col[k] == i) a += val[k];
      d = fabs(a) > 1e-15 ? 1.0 / a : 1.0;
    }
    const double bi = b[i], zi = d * bi;
    s.dinv[i] = d;
    x[i] = 0.0; s.r[i] = bi; s.z[i] = zi; s.p[i] = zi;
    acc[0] += bi * bi;
    acc[1] += bi * zi;
  }
  double tot[2];
  if (!reduce<2>(acc, s.partial, s.st, tot)) return;
  if (threadIdx.x == 0) {
    NaState* st = s.st;
    const double bn = sqrt(tot[0]);
    st->bnorm = bn;
    st->rz = tot[1];
    st->iter = 1;
    st->status = EMG_MAX_ITER_REACHED;
    if (bn < 1e-15) { st->status = EMG_SUCCESS; st->iter = 0; st->res = 0.0; st->done = 1; return; }
    st->res = sqrt(tot[0]) / bn;
    st->prev = st->res;
    if (st->max_iter < 1) { st->iter = st->max_iter; st->done = 1; }
  }
}

// q = A p (CSR, kLanes lanes per row) and p.q -> alpha
__global__ void k_na_spmv_dot(int64_t n, const int32_t* __restrict__ rp, const int32_t* __restrict__ col,
                              const double* __restrict__ val, Scratch s) {
  if (s.st->done) return;
  const int lane = threadIdx.x & 31, sub = lane & (kLanes - 1);
  const int64_t warp = tid() >> 5, nwarps = nthreads() >> 5;
  constexpr int G = 32 / kLanes;
  double dot = 0.0;
  for (int64_t base = warp * G; base < n; base += nwarps * G) {
    const int64_t row = base + lane / kLanes;
    double sum = 0.0;
    if (row < n)
      for (int32_t k = rp[row] + sub; k < rp[row + 1]; k += kLanes) sum += val[k] * s.p[col[k]];
#pragma unroll
    for (int o = kLanes / 2; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (row < n && sub == 0) {
      s.q[row] = sum;
      dot += s.p[row] * sum;
    }
  }
  double acc[1] = {dot}, tot[1];
  if (!reduce<1>(acc, s.partial, s.st, tot)) return;
  if (threadIdx.x == 0) {
    if (fabs(tot[0]) < 1e-30) { s.st->status = EMG_NUMERICAL_ERROR; s.st->done = 1; }
    else s.st->alpha = s.st->rz / tot[0];
  }
}

__global__ void k_na_update(int64_t n, double* __restrict__ x, Scratch s) {
  NaState* st = s.st;
  if (st->done) return;
  const double a = st->alpha;
  double acc[2] = {0.0, 0.0};
  for (int64_t i = tid(); i < n; i += nthreads()) {
    x[i] += a * s.p[i];
    const double ri = s.r[i] - a * s.q[i];
    const double zi = s.dinv[i] * ri;
    s.r[i] = ri;
    s.z[i] = zi;
    acc[0] += ri * zi;
    acc[1] += ri * ri;
  }
  double tot[2];
  if (!reduce<2>(acc, s.partial, st, tot)) return;
  if (threadIdx.x == 0) {
    const int it = st->iter;
    const double res = sqrt(tot[1]) / st->bnorm;
    st->res = res;
    if (res < st->tol) { st->status = EMG_SUCCESS; st->done = 1; }
    else if (it > 10 && res > st->prev * 1000.0) { st->status = EMG_DIVERGED; st->done = 1; }
    else {
      st->beta = tot[0] / st->rz;
      st->rz = tot[0];
      st->prev = res;
      if (it >= st->max_iter) { st->status = EMG_MAX_ITER_REACHED; st->done = 1; }
      else st->iter = it + 1;
    }
  }
}

__global__ void k_na_direction(int64_t n, Scratch s) {
  if (s.st->done) return;
  const double b = s.st->beta;
  for (int64_t i = tid(); i < n; i += nthreads()) s.p[i] = s.z[i] + b * s.p[i];
}

std::mutex g_mu;
double* g_base[kMaxDevices] = {nullptr};

// Once per device, with that device current: the device address of the
// scratch array (the host-side symbol is not a device address).
int scratch_base(double** out) {
  int dev = 0;
  EMG_CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) { set_error("device index out of range"); return EMG_INVALID_INPUT; }
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_base[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      set_error(std::string("cudaGetSymbolAddress(no-allocation scratch): ") + cudaGetErrorString(e));
      return EMG_ERR_CUDA;
    }
    g_base[dev] = static_cast<double*>(p);
  }
  *out = g_base[dev];
  return EMG_SUCCESS;
}

}  // namespace

int cg_solve_noalloc(int64_t n, int64_t nnz, const int32_t* rp, const int32_t* col, const double* val,
                     const double* b, double* x, const emg_krylov_config& cfg, cudaStream_t st,
                     emg_result* res) {
  std::memset(res, 0, sizeof(*res));
  res->status = EMG_INVALID_INPUT;
  if (n <= 0 || nnz < 0 || !rp || !col || !val || !b || !x) {
    set_error("emg_cg_solve_noalloc: null array or empty matrix");
    return EMG_INVALID_INPUT;
  }
  if (check_krylov_precond(cfg.preconditioner)) return EMG_INVALID_INPUT;
  if (n > kMaxRows) {
    set_error("emg_cg_solve_noalloc: n = " + std::to_string(n) + " exceeds the no-allocation scratch limit of " +
              std::to_string(kMaxRows) + " rows; use emg_cg_solve_device");
    return EMG_INVALID_INPUT;
  }
  double* base = nullptr;
  int rc = scratch_base(&base);
  if (rc) { res->status = rc; return rc; }
  // From here every early return through EMG_CK is a CUDA error; the paths
  // that end otherwise overwrite the status.
  res->status = EMG_ERR_CUDA;
  const Scratch s = carve(base);
  const auto t0 = std::chrono::steady_clock::now();
  k_na_reset<<<1, 32, 0, st>>>(s.st, cfg.tolerance, cfg.max_iterations);
  k_na_check<<<kGrid, kThreads, 0, st>>>(n, nnz, rp, col, s.st);
  EMG_CK(cudaGetLastError());
  NaState h;
  EMG_CK(cudaMemcpyAsync(&h, s.st, sizeof(NaState), cudaMemcpyDeviceToHost, st));
  EMG_CK(cudaStreamSynchronize(st));
  if (h.pad[0]) {
    set_error(h.pad[0] & 1   ? "emg_cg_solve_noalloc: row_ptr is not a valid offset array"
              : h.pad[0] & 2 ? "emg_cg_solve_noalloc: column index out of range"
                             : "emg_cg_solve_noalloc: columns of a row are not strictly ascending (unmerged CSR)");
    res->status = EMG_INVALID_INPUT;
    return EMG_INVALID_INPUT;
  }
  k_na_init<<<kGrid, kThreads, 0, st>>>(n, rp, col, val, b, cfg.preconditioner, x, s);
  EMG_CK(cudaGetLastError());
  const int64_t max_it = cfg.max_iterations > 0 ? cfg.max_iterations : 0;
  bool done = false;
  for (int64_t it = 0; it <= max_it + kPollEvery; it += kPollEvery) {
    EMG_CK(cudaMemcpyAsync(&h, s.st, sizeof(NaState), cudaMemcpyDeviceToHost, st));
    EMG_CK(cudaStreamSynchronize(st));
    if (h.done) { done = true; break; }
    for (int k = 0; k < kPollEvery; ++k) {
      k_na_spmv_dot<<<kGrid, kThreads, 0, st>>>(n, rp, col, val, s);
      k_na_update<<<kGrid, kThreads, 0, st>>>(n, x, s);
      k_na_direction<<<kGrid, kThreads, 0, st>>>(n, s);
    }
    EMG_CK(cudaGetLastError());
  }
  const auto t1 = std::chrono::steady_clock::now();
  if (!done) {
    set_error("emg_cg_solve_noalloc: solver state did not finish within the iteration bound");
    res->status = EMG_ERR_INTERNAL;
    return EMG_ERR_INTERNAL;
  }
  res->status = h.status;
  res->iterations = h.iter;
  res->residual_norm = h.res;
  res->solve_time_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  return h.status;
}

}  // namespace emg

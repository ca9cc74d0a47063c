// ilu.cu -- the ILU0 preconditioner option of CGSolver / BiCGSTABSolver on
// the device (CGConfig / BiCGSTABConfig::PreconditionerType::ILU0,
// iterative_solvers.h:59-76).
//
// The reference computes Eigen::IncompleteLUT (iterative_solvers.cpp:277-286)
// in set_matrix and, if that fails, drops to no preconditioner
// (:279-282, :805-810).  Here the preconditioner is ILU(0): L (unit, strictly
// lower) and U (upper with the diagonal) on A's own sparsity pattern, the
// classic row-by-row (IKJ) elimination restricted to that pattern.  Rows are
// grouped into levels (a row's level is one more than the highest level of
// the rows its lower part depends on), so the factorization and the two
// triangular solves run as one kernel launch per level, warps or 8-lane
// groups per row; a zero or non-finite pivot counts as a failed
// factorization and, as in the reference, the solve then runs without a
// preconditioner.  Different fill than IncompleteLUT's gives different
// iteration counts; the converged solution is the same.
//
// The Krylov iterations follow the reference's solve_with_ilu0 text step by
// step (CG :505-585; BiCGSTAB :1121-1243, whose omega is z.t / t.t with
// z = M^-1 s and whose p is not preconditioned), every scalar through a
// device state, and run as one CUDA graph: a conditional while-node whose
// body is one iteration (SpMV, dots, the level kernels of M^-1) and a control
// kernel.  Where conditional nodes are unavailable the same body runs from a
// host loop.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "device.h"

namespace emg {

namespace {

constexpr int kIlThreads = 256;
constexpr int kIlGrid = 592;   // vector kernels: 4 blocks of 256 threads per SM of a 148-SM B200
constexpr int kIlLanes = 8;    // lanes per row in the SpMV and the triangular solves

struct IlState {
  double bnorm, rz, rho, alpha, beta, omega, res, prev;
  double tol;
  int32_t iter, max_iter, status, done, early, div_count, loops, loop_limit;
};

enum Step : int32_t {
  kCgPq = 0,     // alpha = rz / p.q, breakdown test
  kCgRr = 1,     // residual of x, r
  kCgRz = 2,     // convergence, divergence, beta
  kBiRho = 3,    // rho, breakdown, beta
  kBiRv = 4,     // alpha = rho / r_hat.v
  kBiSs = 5,     // ||s||: early exit
  kBiTt = 6,     // omega = z.t / t.t
  kBiRr = 7,     // ||r||: convergence, divergence tests, next iteration
  kInitB = 8,    // ||b||
  kInitCg = 9,   // r.z of the start
  kInitBi = 10,  // rho of the start
};

__device__ __forceinline__ int64_t gtid() { return static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; }
__device__ __forceinline__ int64_t gsize() { return static_cast<int64_t>(gridDim.x) * blockDim.x; }

// ----------------------------------------------------------- factorization

// One level of the IKJ elimination, a warp per row i:
//   for k in row i with k < i (ascending): a_ik /= a_kk;
//     for j in row k with j > k and j in row i: a_ij -= a_ik a_kj.
__global__ void __launch_bounds__(kIlThreads) k_ilu_factor(const int32_t* __restrict__ rows, int32_t nrows,
                                                           const int32_t* __restrict__ rp,
                                                           const int32_t* __restrict__ col,
                                                           const int32_t* __restrict__ diag, double* lu,
                                                           int32_t* __restrict__ fail) {
  const int64_t w = gtid() >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= nrows) return;
  const int32_t i = rows[w];
  const int32_t b = rp[i + 1], d = diag[i];
  for (int32_t p = rp[i]; p < d; ++p) {
    const int32_t k = col[p];
    const double l = lu[p] / lu[diag[k]];
    __syncwarp();
    if (lane == 0) lu[p] = l;
    for (int32_t q = diag[k] + 1 + lane; q < rp[k + 1]; q += 32) {
      const int32_t j = col[q];
      int32_t lo = p + 1, hi = b;  // row i's columns after k
      while (lo < hi) {
        const int32_t mid = (lo + hi) >> 1;
        if (col[mid] < j) lo = mid + 1;
        else hi = mid;
      }
      if (lo < b && col[lo] == j) lu[lo] -= l * lu[q];
    }
    __syncwarp();
  }
  if (lane == 0) {
    const double u = lu[d];
    if (!(fabs(u) > 0.0) || !isfinite(u)) atomicOr(fail, 1);
  }
}

// ------------------------------------------------------ triangular solves

// y_i = r_i - sum_{k<i} l_ik y_k for the rows of one level (unit lower L).
__global__ void __launch_bounds__(kIlThreads) k_ilu_lower(const int32_t* __restrict__ rows, int32_t nrows,
                                                          const int32_t* __restrict__ rp,
                                                          const int32_t* __restrict__ col,
                                                          const int32_t* __restrict__ diag,
                                                          const double* __restrict__ lu, const double* __restrict__ r,
                                                          double* y, const IlState* __restrict__ st) {
  if (st->done) return;
  const int64_t g = gtid() / kIlLanes;
  const int sub = threadIdx.x & (kIlLanes - 1);
  double s = 0.0;
  int32_t i = -1;
  if (g < nrows) {
    i = rows[g];
    for (int32_t p = rp[i] + sub; p < diag[i]; p += kIlLanes) s += lu[p] * y[col[p]];
  }
#pragma unroll
  for (int o = kIlLanes / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (i >= 0 && sub == 0) y[i] = r[i] - s;
}

// z_i = (y_i - sum_{j>i} u_ij z_j) / u_ii for the rows of one level.
__global__ void __launch_bounds__(kIlThreads) k_ilu_upper(const int32_t* __restrict__ rows, int32_t nrows,
                                                          const int32_t* __restrict__ rp,
                                                          const int32_t* __restrict__ col,
                                                          const int32_t* __restrict__ diag,
                                                          const double* __restrict__ lu, const double* __restrict__ y,
                                                          double* z, const IlState* __restrict__ st) {
  if (st->done) return;
  const int64_t g = gtid() / kIlLanes;
  const int sub = threadIdx.x & (kIlLanes - 1);
  double s = 0.0;
  int32_t i = -1;
  if (g < nrows) {
    i = rows[g];
    for (int32_t p = diag[i] + 1 + sub; p < rp[i + 1]; p += kIlLanes) s += lu[p] * z[col[p]];
  }
#pragma unroll
  for (int o = kIlLanes / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (i >= 0 && sub == 0) z[i] = (y[i] - s) / lu[diag[i]];
}

// ------------------------------------------------------- vector kernels

// Per-block partial sums of up to two products, partial[k * gridDim + block].
__device__ __forceinline__ void write_partials(double a0, double a1, double* partial) {
  __shared__ double red[kIlThreads / 32];
  const double b0 = block_sum(a0, red);
  const double b1 = block_sum(a1, red);
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = b0;
    partial[gridDim.x + blockIdx.x] = b1;
  }
}

// y = A x (CSR, kIlLanes lanes a row); partials w0.y (w0 null: y.y) and w1.y.
__global__ void __launch_bounds__(kIlThreads) k_il_spmv(int64_t n, const int32_t* __restrict__ rp,
                                                        const int32_t* __restrict__ col,
                                                        const double* __restrict__ val,
                                                        const double* __restrict__ x, double* __restrict__ y,
                                                        const double* __restrict__ w0, const double* __restrict__ w1,
                                                        double* partial, const IlState* __restrict__ st) {
  if (st->done) return;
  const int sub = threadIdx.x & (kIlLanes - 1);
  double a0 = 0.0, a1 = 0.0;
  const int64_t groups = gsize() / kIlLanes;
  const int64_t rounds = (n + groups - 1) / groups;  // the same for every lane: the shuffles stay converged
  for (int64_t k = 0; k < rounds; ++k) {
    const int64_t row = gtid() / kIlLanes + k * groups;
    double s = 0.0;
    if (row < n)
      for (int32_t k = rp[row] + sub; k < rp[row + 1]; k += kIlLanes) s += val[k] * x[col[k]];
#pragma unroll
    for (int o = kIlLanes / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (row < n && sub == 0) {
      y[row] = s;
      a0 += (w0 ? w0[row] : s) * s;
      if (w1) a1 += w1[row] * s;
    }
  }
  write_partials(a0, a1, partial);
}

// partials of a.b
__global__ void __launch_bounds__(kIlThreads) k_il_dot(int64_t n, const double* __restrict__ a,
                                                       const double* __restrict__ b, double* partial,
                                                       const IlState* __restrict__ st) {
  if (st->done) return;
  double acc = 0.0;
  for (int64_t i = gtid(); i < n; i += gsize()) acc += a[i] * b[i];
  write_partials(acc, 0.0, partial);
}

// CG: x += alpha p, r -= alpha q; partials r.r
__global__ void __launch_bounds__(kIlThreads) k_il_cg_xr(int64_t n, double* __restrict__ x, double* __restrict__ r,
                                                         const double* __restrict__ p, const double* __restrict__ q,
                                                         double* partial, const IlState* __restrict__ st) {
  if (st->done) return;
  const double a = st->alpha;
  double acc = 0.0;
  for (int64_t i = gtid(); i < n; i += gsize()) {
    x[i] += a * p[i];
    const double ri = r[i] - a * q[i];
    r[i] = ri;
    acc += ri * ri;
  }
  write_partials(acc, 0.0, partial);
}

// CG: p = z + beta p
__global__ void k_il_cg_dir(int64_t n, double* __restrict__ p, const double* __restrict__ z,
                            const IlState* __restrict__ st) {
  if (st->done) return;
  const double b = st->beta;
  for (int64_t i = gtid(); i < n; i += gsize()) p[i] = z[i] + b * p[i];
}

// BiCGSTAB: p = r + beta (p - omega v)
__global__ void k_il_bi_p(int64_t n, double* __restrict__ p, const double* __restrict__ r,
                          const double* __restrict__ v, const IlState* __restrict__ st) {
  if (st->done) return;
  const double b = st->beta, w = st->omega;
  for (int64_t i = gtid(); i < n; i += gsize()) p[i] = r[i] + b * (p[i] - w * v[i]);
}

// BiCGSTAB: s = r - alpha v; partials s.s
__global__ void __launch_bounds__(kIlThreads) k_il_bi_s(int64_t n, double* __restrict__ s,
                                                        const double* __restrict__ r, const double* __restrict__ v,
                                                        double* partial, const IlState* __restrict__ st) {
  if (st->done) return;
  const double a = st->alpha;
  double acc = 0.0;
  for (int64_t i = gtid(); i < n; i += gsize()) {
    const double si = r[i] - a * v[i];
    s[i] = si;
    acc += si * si;
  }
  write_partials(acc, 0.0, partial);
}

// BiCGSTAB early exit on ||s||: x += alpha p (:1174-1182)
__global__ void k_il_bi_early(int64_t n, double* __restrict__ x, const double* __restrict__ p,
                              const IlState* __restrict__ st) {
  if (st->early != 1) return;
  const double a = st->alpha;
  for (int64_t i = gtid(); i < n; i += gsize()) x[i] += a * p[i];
}

// BiCGSTAB: x += alpha p + omega z, r = s - omega t; partials r.r
__global__ void __launch_bounds__(kIlThreads) k_il_bi_xr(int64_t n, double* __restrict__ x, double* __restrict__ r,
                                                         const double* __restrict__ p, const double* __restrict__ z,
                                                         const double* __restrict__ s, const double* __restrict__ t,
                                                         double* partial, const IlState* __restrict__ st) {
  if (st->done) return;
  const double a = st->alpha, w = st->omega;
  double acc = 0.0;
  for (int64_t i = gtid(); i < n; i += gsize()) {
    x[i] += a * p[i] + w * z[i];
    const double ri = s[i] - w * t[i];
    r[i] = ri;
    acc += ri * ri;
  }
  write_partials(acc, 0.0, partial);
}

// One step of the scalar recurrence from the partials of the last kernel.
__global__ void __launch_bounds__(kIlThreads) k_il_step(const double* __restrict__ partial, int32_t np, IlState* st,
                                                        int32_t step) {
  __shared__ double red[kIlThreads / 32];
  if (step != kInitB && step != kInitCg && step != kInitBi && st->done) return;
  double a0 = 0.0, a1 = 0.0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) {
    a0 += partial[i];
    a1 += partial[np + i];
  }
  const double s0 = block_sum(a0, red);
  const double s1 = block_sum(a1, red);
  if (threadIdx.x != 0) return;
  const int32_t it = st->iter;
  switch (step) {
    case kInitB: st->bnorm = sqrt(s0); break;
    case kInitCg: st->rz = s0; break;
    case kInitBi: st->rho = s0; break;
    case kCgPq:
      if (fabs(s0) < 1e-30) { st->status = EMG_NUMERICAL_ERROR; st->done = 1; }
      else st->alpha = st->rz / s0;
      break;
    case kCgRr: st->res = sqrt(s0) / st->bnorm; break;
    case kCgRz: {
      const double res = st->res;
      if (res < st->tol) { st->status = EMG_SUCCESS; st->done = 1; break; }
      if (it > 10 && res > st->prev * 1000.0) { st->status = EMG_DIVERGED; st->done = 1; break; }
      st->beta = s0 / st->rz;
      st->rz = s0;
      st->prev = res;
      if (it >= st->max_iter) { st->status = EMG_MAX_ITER_REACHED; st->done = 1; }
      else st->iter = it + 1;
      break;
    }
    case kBiRho: {
      const double rho_old = st->rho;
      st->rho = s0;
      if (fabs(s0) < 1e-30) { st->status = EMG_NUMERICAL_ERROR; st->done = 1; break; }
      st->beta = (s0 / rho_old) * (st->alpha / st->omega);
      break;
    }
    case kBiRv:
      if (fabs(s0) < 1e-30) { st->status = EMG_NUMERICAL_ERROR; st->done = 1; }
      else st->alpha = st->rho / s0;
      break;
    case kBiSs: {
      const double res = sqrt(s0) / st->bnorm;
      st->res = res;
      if (res < st->tol) { st->status = EMG_SUCCESS; st->done = 1; st->early = 1; }
      break;
    }
    case kBiTt: st->omega = fabs(s0) < 1e-30 ? 0.0 : s1 / s0; break;
    case kBiRr: {
      const double res = sqrt(s0) / st->bnorm;
      st->res = res;
      if (res < st->tol) { st->status = EMG_SUCCESS; st->done = 1; break; }
      if (res > st->prev * 1.5 && it > 20) {
        if (++st->div_count >= 3) { st->status = EMG_DIVERGED; st->done = 1; break; }
      } else {
        st->div_count = 0;
      }
      if (it > 10 && res > st->prev * 1000.0) { st->status = EMG_DIVERGED; st->done = 1; break; }
      st->prev = res;
      if (it >= st->max_iter) { st->status = EMG_MAX_ITER_REACHED; st->done = 1; }
      else st->iter = it + 1;
      break;
    }
    default: break;
  }
}

// Last node of the loop body: keep looping while not done and below the
// body-count bound (independent of the scalars, so the loop always ends).
__global__ void k_il_control(IlState* st, cudaGraphConditionalHandle handle) {
  if (threadIdx.x != 0) return;
  st->early = 0;
  const int32_t loops = st->loops + 1;
  st->loops = loops;
  cudaGraphSetConditional(handle, (!st->done && loops < st->loop_limit) ? 1u : 0u);
}

__global__ void k_il_host_control(IlState* st) {
  if (threadIdx.x != 0) return;
  st->early = 0;
  st->loops = st->loops + 1;
}

__global__ void k_il_start(int64_t n, const double* __restrict__ b, double* __restrict__ x, double* __restrict__ r,
                           double* __restrict__ rh, double* __restrict__ p, double* __restrict__ v, double* partial,
                           int bicg) {
  double acc = 0.0;
  for (int64_t i = gtid(); i < n; i += gsize()) {
    const double bi = b[i];
    x[i] = 0.0;
    r[i] = bi;
    if (bicg) { rh[i] = bi; p[i] = bi; v[i] = 0.0; }
    acc += bi * bi;
  }
  write_partials(acc, 0.0, partial);
}

__global__ void k_il_copy(int64_t n, const double* __restrict__ a, double* __restrict__ b) {
  for (int64_t i = gtid(); i < n; i += gsize()) b[i] = a[i];
}

unsigned level_grid(int32_t rows, int lanes) {
  const int64_t threads = static_cast<int64_t>(rows) * lanes;
  return static_cast<unsigned>(std::max<int64_t>(1, (threads + kIlThreads - 1) / kIlThreads));
}

}  // namespace

struct IluState {
  int64_t n = 0, nnz = 0;
  uint64_t version = ~0ull;  // A.version the factor was computed from
  bool failed = false;       // no diagonal, or a zero / non-finite pivot
  double* lu = nullptr;
  int32_t *diag = nullptr, *lrows = nullptr, *urows = nullptr, *flag = nullptr;
  std::vector<int32_t> lptr, uptr;  // level offsets into lrows / urows
  double *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr, *y = nullptr;
  double *rh = nullptr, *v = nullptr, *s = nullptr, *t = nullptr, *part = nullptr;
  IlState* st = nullptr;
  cudaStream_t cap = nullptr;
  cudaGraphExec_t loop[2] = {nullptr, nullptr};  // CG, BiCGSTAB
  bool loop_failed = false;
  std::vector<void*> mem;
};

void free_ilu(IluState* s) {
  if (!s) return;
  cudaDeviceSynchronize();
  for (cudaGraphExec_t g : s->loop)
    if (g) cudaGraphExecDestroy(g);
  if (s->cap) cudaStreamDestroy(s->cap);
  for (void* m : s->mem) cudaFree(m);
  delete s;
}

namespace {

template <class T>
int ilu_alloc(IluState& s, T** p, int64_t count) {
  void* m = nullptr;
  EMG_CK(cudaMalloc(&m, sizeof(T) * static_cast<size_t>(std::max<int64_t>(count, 1))));
  s.mem.push_back(m);
  *p = static_cast<T*>(m);
  return EMG_SUCCESS;
}

// Symbolic phase (host integer work on the pattern): diagonal positions and
// the forward / backward level schedules.
int ilu_symbolic(DevCsr& A, IluState& s, cudaStream_t st) {
  const int64_t n = A.n, nnz = A.nnz;
  std::vector<int32_t> rp(n + 1), col(std::max<int64_t>(nnz, 1));
  EMG_CK(cudaMemcpyAsync(rp.data(), A.row_ptr, sizeof(int32_t) * (n + 1), cudaMemcpyDeviceToHost, st));
  if (nnz > 0) EMG_CK(cudaMemcpyAsync(col.data(), A.col, sizeof(int32_t) * nnz, cudaMemcpyDeviceToHost, st));
  EMG_CK(cudaStreamSynchronize(st));
  std::vector<int32_t> diag(n, -1), lo(n), up(n);
  int32_t nl = 0, nu = 0;
  for (int64_t i = 0; i < n; ++i) {
    const int32_t* b = col.data() + rp[i];
    const int32_t* e = col.data() + rp[i + 1];
    const int32_t* d = std::lower_bound(b, e, static_cast<int32_t>(i));
    if (d == e || *d != i) { s.failed = true; continue; }
    diag[i] = static_cast<int32_t>(d - col.data());
    int32_t m = -1;
    for (const int32_t* c = b; c < d; ++c) m = std::max(m, lo[*c]);
    lo[i] = m + 1;
    nl = std::max(nl, lo[i] + 1);
  }
  if (s.failed) return EMG_SUCCESS;
  for (int64_t i = n - 1; i >= 0; --i) {
    int32_t m = -1;
    for (int32_t q = diag[i] + 1; q < rp[i + 1]; ++q) m = std::max(m, up[col[q]]);
    up[i] = m + 1;
    nu = std::max(nu, up[i] + 1);
  }
  auto group = [&](const std::vector<int32_t>& lev, int32_t nlev, std::vector<int32_t>& ptr,
                   std::vector<int32_t>& rows) {
    ptr.assign(nlev + 1, 0);
    for (int64_t i = 0; i < n; ++i) ++ptr[lev[i] + 1];
    for (int32_t k = 0; k < nlev; ++k) ptr[k + 1] += ptr[k];
    rows.resize(n);
    std::vector<int32_t> fill(ptr.begin(), ptr.end() - 1);
    for (int64_t i = 0; i < n; ++i) rows[fill[lev[i]]++] = static_cast<int32_t>(i);
  };
  std::vector<int32_t> lrows, urows;
  group(lo, nl, s.lptr, lrows);
  group(up, nu, s.uptr, urows);
  int rc = EMG_SUCCESS;
  if ((rc = ilu_alloc(s, &s.diag, n)) || (rc = ilu_alloc(s, &s.lrows, n)) || (rc = ilu_alloc(s, &s.urows, n)) ||
      (rc = ilu_alloc(s, &s.lu, nnz)) || (rc = ilu_alloc(s, &s.flag, 1)))
    return rc;
  EMG_CK(cudaMemcpyAsync(s.diag, diag.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
  EMG_CK(cudaMemcpyAsync(s.lrows, lrows.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
  EMG_CK(cudaMemcpyAsync(s.urows, urows.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
  EMG_CK(cudaStreamSynchronize(st));
  return EMG_SUCCESS;
}

int ilu_numeric(DevCsr& A, IluState& s, cudaStream_t st) {
  EMG_CK(cudaMemcpyAsync(s.lu, A.val, sizeof(double) * std::max<int64_t>(A.nnz, 1), cudaMemcpyDeviceToDevice, st));
  EMG_CK(cudaMemsetAsync(s.flag, 0, sizeof(int32_t), st));
  for (size_t k = 0; k + 1 < s.lptr.size(); ++k) {
    const int32_t cnt = s.lptr[k + 1] - s.lptr[k];
    k_ilu_factor<<<level_grid(cnt, 32), kIlThreads, 0, st>>>(s.lrows + s.lptr[k], cnt, A.row_ptr, A.col, s.diag,
                                                              s.lu, s.flag);
  }
  EMG_CK(cudaGetLastError());
  int32_t f = 0;
  EMG_CK(cudaMemcpyAsync(&f, s.flag, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  EMG_CK(cudaStreamSynchronize(st));
  s.failed = f != 0;
  return EMG_SUCCESS;
}

// out = U^-1 L^-1 in (out and s.y are work vectors; in is left unchanged)
void ilu_apply(DevCsr& A, IluState& s, const double* in, double* out, cudaStream_t st) {
  for (size_t k = 0; k + 1 < s.lptr.size(); ++k) {
    const int32_t cnt = s.lptr[k + 1] - s.lptr[k];
    k_ilu_lower<<<level_grid(cnt, kIlLanes), kIlThreads, 0, st>>>(s.lrows + s.lptr[k], cnt, A.row_ptr, A.col, s.diag,
                                                                   s.lu, in, s.y, s.st);
  }
  for (size_t k = 0; k + 1 < s.uptr.size(); ++k) {
    const int32_t cnt = s.uptr[k + 1] - s.uptr[k];
    k_ilu_upper<<<level_grid(cnt, kIlLanes), kIlThreads, 0, st>>>(s.urows + s.uptr[k], cnt, A.row_ptr, A.col, s.diag,
                                                                   s.lu, s.y, out, s.st);
  }
}

// One iteration of the reference's solve_with_ilu0 (CG or BiCGSTAB).
void ilu_body(DevCsr& A, IluState& s, bool bicg, cudaStream_t st) {
  const int64_t n = A.n;
  if (!bicg) {
    k_il_spmv<<<kIlGrid, kIlThreads, 0, st>>>(n, A.row_ptr, A.col, A.val, s.p, s.q, s.p, nullptr, s.part, s.st);
    k_il_step<<<1, kIlThreads, 0, st>>>(s.part, kIlGrid, s.st, kCgPq);
    k_il_cg_xr<<<kIlGrid, kIlThreads, 0, st>>>(n, s.x, s.r, s.p, s.q, s.part, s.st);
    k_il_step<<<1, kIlThreads, 0, st>>>(s.part, kIlGrid, s.st, kCgRr);
    ilu_apply(A, s, s.r, s.z, st);
    k_il_dot<<<kIlGrid, kIlThreads, 0, st>>>(n, s.r, s.z, s.part, s.st);
    k_il_step<<<1, kIlThreads, 0, st>>>(s.part, kIlGrid, s.st, kCgRz);
    k_il_cg_dir<<<kIlGrid, kIlThreads, 0, st>>>(n, s.p, s.z, s.st);
  } else {
    k_il_dot<<<kIlGrid, kIlThreads, 0, st>>>(n, s.r, s.rh, s.part, s.st);
    k_il_step<<<1, kIlThreads, 0, st>>>(s.part, kIlGrid, s.st, kBiRho);
    k_il_bi_p<<<kIlGrid, kIlThreads, 0, st>>>(n, s.p, s.r, s.v, s.st);
    k_il_spmv<<<kIlGrid, kIlThreads, 0, st>>>(n, A.row_ptr, A.col, A.val, s.p, s.v, s.rh, nullptr, s.part, s.st);
    k_il_step<<<1, kIlThreads, 0, st>>>(s.part, kIlGrid, s.st, kBiRv);
    k_il_bi_s<<<kIlGrid, kIlThreads, 0, st>>>(n, s.s, s.r, s.v, s.part, s.st);
    k_il_step<<<1, kIlThreads, 0, st>>>(s.part, kIlGrid, s.st, kBiSs);
    k_il_bi_early<<<kIlGrid, kIlThreads, 0, st>>>(n, s.x, s.p, s.st);
    ilu_apply(A, s, s.s, s.z, st);
    k_il_spmv<<<kIlGrid, kIlThreads, 0, st>>>(n, A.row_ptr, A.col, A.val, s.z, s.t, nullptr, s.z, s.part, s.st);
    k_il_step<<<1, kIlThreads, 0, st>>>(s.part, kIlGrid, s.st, kBiTt);
    k_il_bi_xr<<<kIlGrid, kIlThreads, 0, st>>>(n, s.x, s.r, s.p, s.z, s.s, s.t, s.part, s.st);
    k_il_step<<<1, kIlThreads, 0, st>>>(s.part, kIlGrid, s.st, kBiRr);
  }
}

cudaGraphExec_t ilu_loop_graph(DevCsr& A, IluState& s, bool bicg) {
  if (s.loop[bicg]) return s.loop[bicg];
  if (s.loop_failed) return nullptr;
  if (!s.cap && cudaStreamCreateWithFlags(&s.cap, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    s.loop_failed = true;
    return nullptr;
  }
  cudaGraph_t graph = nullptr;
  if (cudaGraphCreate(&graph, 0) != cudaSuccess) { cudaGetLastError(); s.loop_failed = true; return nullptr; }
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
    e = cudaStreamBeginCaptureToGraph(s.cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      ilu_body(A, s, bicg, s.cap);
      k_il_control<<<1, 32, 0, s.cap>>>(s.st, handle);
      e = cudaStreamEndCapture(s.cap, &body);
    }
  }
  cudaGraphExec_t exec = nullptr;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    cudaGetLastError();
    s.loop_failed = true;
    return nullptr;
  }
  s.loop[bicg] = exec;
  return exec;
}

int ilu_prepare(DevCsr& A, cudaStream_t st) {
  if (!A.ilu) {
    A.ilu = new IluState();
    IluState& s = *A.ilu;
    s.n = A.n;
    s.nnz = A.nnz;
    int rc = ilu_symbolic(A, s, st);
    if (rc) return rc;
    if (!s.failed) {
      const int64_t n = A.n;
      for (double** v : {&s.x, &s.r, &s.z, &s.p, &s.q, &s.y, &s.rh, &s.v, &s.s, &s.t})
        if ((rc = ilu_alloc(s, v, n))) return rc;
      if ((rc = ilu_alloc(s, &s.part, 2 * kIlGrid)) || (rc = ilu_alloc(s, &s.st, 1))) return rc;
    }
  }
  IluState& s = *A.ilu;
  if (s.lu && s.version != A.version) {
    int rc = ilu_numeric(A, s, st);
    if (rc) return rc;
    s.version = A.version;
  }
  return EMG_SUCCESS;
}

}  // namespace

int ilu_solve(DevCsr& A, const double* b, double* x, const emg_krylov_config& cfg, cudaStream_t st,
              emg_result* res, bool bicg) {
  std::memset(res, 0, sizeof(*res));
  res->status = EMG_INVALID_INPUT;
  if (!b || !x) { set_error("null vector"); return EMG_INVALID_INPUT; }
  if (A.n <= 0) { set_error("empty matrix"); return EMG_INVALID_INPUT; }
  const auto t0 = std::chrono::steady_clock::now();
  int rc = ilu_prepare(A, st);
  if (rc) { res->status = rc; return rc; }
  IluState& s = *A.ilu;
  if (s.failed) {
    // as the reference's setup_preconditioner: a failed factorization leaves
    // the solver without a preconditioner
    emg_krylov_config none = cfg;
    none.preconditioner = EMG_PRECOND_NONE;
    return bicg ? bicgstab_solve(A, b, x, none, st, res) : cg_solve(A, b, x, none, st, res);
  }
  const int64_t n = A.n;
  IlState init;
  std::memset(&init, 0, sizeof(init));
  init.tol = cfg.tolerance;
  init.max_iter = cfg.max_iterations;
  init.iter = 1;
  init.status = EMG_MAX_ITER_REACHED;
  init.alpha = 1.0;
  init.omega = 1.0;
  init.res = 1.0;
  init.prev = 1.0;
  init.loop_limit = std::max(cfg.max_iterations, 0) + 2;
  EMG_CK(cudaMemcpyAsync(s.st, &init, sizeof(IlState), cudaMemcpyHostToDevice, st));
  k_il_start<<<kIlGrid, kIlThreads, 0, st>>>(n, b, s.x, s.r, s.rh, s.p, s.v, s.part, bicg ? 1 : 0);
  k_il_step<<<1, kIlThreads, 0, st>>>(s.part, kIlGrid, s.st, kInitB);
  if (!bicg) {  // z = M^-1 r, p = z, rz = r.z
    ilu_apply(A, s, s.r, s.z, st);
    k_il_copy<<<kIlGrid, kIlThreads, 0, st>>>(n, s.z, s.p);
    k_il_dot<<<kIlGrid, kIlThreads, 0, st>>>(n, s.r, s.z, s.part, s.st);
    k_il_step<<<1, kIlThreads, 0, st>>>(s.part, kIlGrid, s.st, kInitCg);
  } else {
    k_il_dot<<<kIlGrid, kIlThreads, 0, st>>>(n, s.r, s.rh, s.part, s.st);
    k_il_step<<<1, kIlThreads, 0, st>>>(s.part, kIlGrid, s.st, kInitBi);
  }
  EMG_CK(cudaGetLastError());
  IlState h;
  EMG_CK(cudaMemcpyAsync(&h, s.st, sizeof(IlState), cudaMemcpyDeviceToHost, st));
  EMG_CK(cudaStreamSynchronize(st));
  if (h.bnorm < 1e-15) {  // :520-526 / :1137-1143
    EMG_CK(cudaMemsetAsync(x, 0, sizeof(double) * n, st));
    EMG_CK(cudaStreamSynchronize(st));
    res->status = EMG_SUCCESS;
    res->iterations = 0;
    res->residual_norm = 0.0;
    res->solve_time_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return EMG_SUCCESS;
  }
  if (cfg.max_iterations > 0) {
    cudaGraphExec_t loop = ilu_loop_graph(A, s, bicg);
    if (loop) {
      EMG_CK(cudaGraphLaunch(loop, st));
    } else {
      for (int32_t k = 0; k <= cfg.max_iterations; ++k) {
        ilu_body(A, s, bicg, st);
        k_il_host_control<<<1, 32, 0, st>>>(s.st);
        EMG_CK(cudaMemcpyAsync(&h, s.st, sizeof(IlState), cudaMemcpyDeviceToHost, st));
        EMG_CK(cudaStreamSynchronize(st));
        if (h.done) break;
      }
    }
    EMG_CK(cudaGetLastError());
  }
  k_il_copy<<<kIlGrid, kIlThreads, 0, st>>>(n, s.x, x);
  EMG_CK(cudaMemcpyAsync(&h, s.st, sizeof(IlState), cudaMemcpyDeviceToHost, st));
  EMG_CK(cudaStreamSynchronize(st));
  EMG_CK(cudaGetLastError());
  res->status = cfg.max_iterations > 0 ? (h.done ? h.status : EMG_ERR_INTERNAL) : EMG_MAX_ITER_REACHED;
  res->iterations = cfg.max_iterations > 0 ? std::min(h.iter, cfg.max_iterations) : 0;
  res->residual_norm = h.res;
  res->solve_time_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (res->status == EMG_ERR_INTERNAL) set_error("ILU0 solve: the loop ended before the solver state did");
  return res->status;
}

}  // namespace emg

// learned.cu -- learned interface preconditioner for FETI-DP: one 3-layer MLP
// per subdomain (width 256, BF16 weights, FP32 accumulation) that maps the
// subdomain's normalised dual residual to a correction of the Dirichlet
// preconditioner, z = M_D r + L(r), inside flexible CG.  No reference
// counterpart (the reference's FETI-DP layer is a context stub).
//
// Per subdomain s with n = nD_s dual entries, for one residual r:
//   x   = (sign_e r[lambda_e])_e / ||.||        (normalised local residual)
//   h1  = relu(W1 x + b1),  h2 = relu(W2 h1 + b2),  y = W3 h2 + b3
//   c_e = ||.|| y_e,   L(r)[lambda] = (sign_a c_a + sign_b c_b) / 2
// Parameters of subdomain s, FP32 master copy (training) and BF16 copy
// (forward passes), in one array at off[s]:
//   W1 [256][n] | b1 [256] | W2 [256][256] | b2 [256] | W3^T [256][n] | b3 [n]
// Training: mean squared error against targets t (the wanted correction,
// e.g. F^-1 r - M_D r) gathered and normalised the same way; backward and
// Adam in hand-written kernels, every reduction in a fixed order.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <random>
#include <string>
#include <vector>

#include "common.cuh"
#include "device.h"
#include "fetidp_dev.h"

namespace emg {
namespace {

constexpr int kH = 256;  // hidden width

__device__ __forceinline__ int64_t p_w1(int32_t n) { return 0; }
__device__ __forceinline__ int64_t p_b1(int32_t n) { return static_cast<int64_t>(kH) * n; }
__device__ __forceinline__ int64_t p_w2(int32_t n) { return p_b1(n) + kH; }
__device__ __forceinline__ int64_t p_b2(int32_t n) { return p_w2(n) + kH * kH; }
__device__ __forceinline__ int64_t p_w3(int32_t n) { return p_b2(n) + kH; }
__device__ __forceinline__ int64_t p_b3(int32_t n) { return p_w3(n) + static_cast<int64_t>(kH) * n; }

struct LearnDev {
  int32_t S;
  const int64_t* dual_off;  // S + 1
  const int32_t* dual_lam;
  const int32_t* dual_sign;
  const int64_t* poff;      // S + 1 parameter offsets
  int64_t nde;              // dual entries
  int64_t nl;               // multipliers
};

// x[b][e] = sign r[b][lambda_e] / ||.||_s, norm[b][s]; tx likewise for t (optional).
__global__ void __launch_bounds__(256) k_l_gather(LearnDev D, const double* __restrict__ r,
                                                  const double* __restrict__ t, float* __restrict__ x,
                                                  float* __restrict__ tx, double* __restrict__ norm) {
  __shared__ double red[8];
  const int32_t s = blockIdx.x, b = blockIdx.y;
  const int64_t e0 = D.dual_off[s], e1 = D.dual_off[s + 1];
  const double* rb = r + static_cast<int64_t>(b) * D.nl;
  double acc = 0.0;
  for (int64_t e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
    const double v = D.dual_sign[e] * rb[D.dual_lam[e]];
    acc = fma(v, v, acc);
  }
  acc = block_sum(acc, red);
  const double nm = acc > 0.0 ? sqrt(acc) : 1.0;
  if (threadIdx.x == 0) norm[static_cast<int64_t>(b) * D.S + s] = nm;
  const double inv = 1.0 / nm;
  float* xb = x + static_cast<int64_t>(b) * D.nde;
  for (int64_t e = e0 + threadIdx.x; e < e1; e += blockDim.x)
    xb[e] = static_cast<float>(D.dual_sign[e] * rb[D.dual_lam[e]] * inv);
  if (t) {
    const double* tb = t + static_cast<int64_t>(b) * D.nl;
    float* txb = tx + static_cast<int64_t>(b) * D.nde;
    for (int64_t e = e0 + threadIdx.x; e < e1; e += blockDim.x)
      txb[e] = static_cast<float>(D.dual_sign[e] * tb[D.dual_lam[e]] * inv);
  }
}

// Forward pass, one CTA (256 threads) per (subdomain, sample); h1, h2 stored
// when non-null (training).  y[b][e] (normalised output).
__global__ void __launch_bounds__(256) k_l_forward(LearnDev D, const __nv_bfloat16* __restrict__ W,
                                                   const float* __restrict__ x, float* __restrict__ h1g,
                                                   float* __restrict__ h2g, float* __restrict__ y) {
  extern __shared__ float xs[];
  __shared__ float h1[kH], h2[kH];
  const int32_t s = blockIdx.x, b = blockIdx.y;
  const int64_t e0 = D.dual_off[s];
  const int32_t n = static_cast<int32_t>(D.dual_off[s + 1] - e0);
  const __nv_bfloat16* P = W + D.poff[s];
  const float* xb = x + static_cast<int64_t>(b) * D.nde + e0;
  for (int32_t i = threadIdx.x; i < n; i += blockDim.x) xs[i] = xb[i];
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int32_t j = wid; j < kH; j += nw) {
    const __nv_bfloat16* row = P + p_w1(n) + static_cast<int64_t>(j) * n;
    float acc = 0.f;
    for (int32_t i = lane; i < n; i += 32) acc = fmaf(__bfloat162float(row[i]), xs[i], acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) h1[j] = fmaxf(acc + __bfloat162float(P[p_b1(n) + j]), 0.f);
  }
  __syncthreads();
  for (int32_t j = wid; j < kH; j += nw) {
    const __nv_bfloat16* row = P + p_w2(n) + static_cast<int64_t>(j) * kH;
    float acc = 0.f;
    for (int32_t k = lane; k < kH; k += 32) acc = fmaf(__bfloat162float(row[k]), h1[k], acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) h2[j] = fmaxf(acc + __bfloat162float(P[p_b2(n) + j]), 0.f);
  }
  __syncthreads();
  if (h1g) {
    const int64_t o = (static_cast<int64_t>(b) * D.S + s) * kH;
    for (int32_t j = threadIdx.x; j < kH; j += blockDim.x) { h1g[o + j] = h1[j]; h2g[o + j] = h2[j]; }
  }
  float* yb = y + static_cast<int64_t>(b) * D.nde + e0;
  for (int32_t i = threadIdx.x; i < n; i += blockDim.x) {
    float acc = __bfloat162float(P[p_b3(n) + i]);
    const __nv_bfloat16* col = P + p_w3(n) + i;
    for (int32_t j = 0; j < kH; ++j) acc = fmaf(__bfloat162float(col[static_cast<int64_t>(j) * n]), h2[j], acc);
    yb[i] = acc;
  }
}

// out[l] = add[l] + (sign_a c_a + sign_b c_b) / 2 with c_e = norm_s y_e (sample 0).
__global__ void k_l_combine(LearnDev D, const int32_t* __restrict__ lam_entry, const int32_t* __restrict__ dual_sub,
                            const float* __restrict__ y, const double* __restrict__ norm,
                            const double* __restrict__ add, double* __restrict__ out) {
  for (int64_t l = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; l < D.nl;
       l += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t ea = lam_entry[2 * l], eb = lam_entry[2 * l + 1];
    const double ca = norm[dual_sub[ea]] * y[ea], cb = norm[dual_sub[eb]] * y[eb];
    out[l] = (add ? add[l] : 0.0) + 0.5 * (ca - cb);  // sign_a = +1, sign_b = -1
  }
}

// Backward for the activations, one CTA per (subdomain, sample):
// dy = 2 (y - t) / count, dh2 = relu'(h2) W3 dy, dh1 = relu'(h1) W2^T dh2;
// loss partial per CTA.
__global__ void __launch_bounds__(256) k_l_backward(LearnDev D, const float* __restrict__ W, const float* __restrict__ y,
                                                    const float* __restrict__ tx, const float* __restrict__ h1g,
                                                    const float* __restrict__ h2g, float* __restrict__ dy,
                                                    float* __restrict__ dh1g, float* __restrict__ dh2g,
                                                    double* __restrict__ loss_part, double inv_count) {
  __shared__ float dh2[kH];
  __shared__ double red[8];
  const int32_t s = blockIdx.x, b = blockIdx.y;
  const int64_t e0 = D.dual_off[s];
  const int32_t n = static_cast<int32_t>(D.dual_off[s + 1] - e0);
  const float* P = W + D.poff[s];
  const int64_t ob = static_cast<int64_t>(b) * D.nde + e0;
  double l2 = 0.0;
  for (int32_t i = threadIdx.x; i < n; i += blockDim.x) {
    const float d = y[ob + i] - tx[ob + i];
    l2 += static_cast<double>(d) * d;
    dy[ob + i] = static_cast<float>(2.0 * inv_count) * d;
  }
  l2 = block_sum(l2, red);
  if (threadIdx.x == 0) loss_part[static_cast<int64_t>(b) * D.S + s] = l2;
  __syncthreads();
  const int64_t oh = (static_cast<int64_t>(b) * D.S + s) * kH;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int32_t j = wid; j < kH; j += nw) {
    const float* row = P + p_w3(n) + static_cast<int64_t>(j) * n;  // W3^T row j = column j of W3
    float acc = 0.f;
    for (int32_t i = lane; i < n; i += 32) acc = fmaf(row[i], dy[ob + i], acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) dh2[j] = h2g[oh + j] > 0.f ? acc : 0.f;
  }
  __syncthreads();
  for (int32_t k = threadIdx.x; k < kH; k += blockDim.x) {
    float acc = 0.f;
    for (int32_t j = 0; j < kH; ++j) acc = fmaf(P[p_w2(n) + static_cast<int64_t>(j) * kH + k], dh2[j], acc);
    dh1g[oh + k] = h1g[oh + k] > 0.f ? acc : 0.f;
    dh2g[oh + k] = dh2[k];
  }
}

// Gradient of every parameter (sum over the batch, fixed order) and the Adam
// step, one thread per parameter of subdomain blockIdx.y; refreshes the BF16 copy.
__global__ void __launch_bounds__(256) k_l_grad_adam(LearnDev D, int32_t B, const float* __restrict__ x,
                                                     const float* __restrict__ h1g, const float* __restrict__ h2g,
                                                     const float* __restrict__ dy, const float* __restrict__ dh1g,
                                                     const float* __restrict__ dh2g, float* __restrict__ W,
                                                     float* __restrict__ m1, float* __restrict__ m2,
                                                     __nv_bfloat16* __restrict__ Wb, float lr, float c1, float c2) {
  const int32_t s = blockIdx.y;
  const int64_t e0 = D.dual_off[s];
  const int32_t n = static_cast<int32_t>(D.dual_off[s + 1] - e0);
  const int64_t np = D.poff[s + 1] - D.poff[s];
  for (int64_t q = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; q < np;
       q += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double g = 0.0;
    if (q < p_b1(n)) {                       // W1[j][i]
      const int32_t j = static_cast<int32_t>(q / n), i = static_cast<int32_t>(q % n);
      for (int32_t b = 0; b < B; ++b)
        g += static_cast<double>(dh1g[(static_cast<int64_t>(b) * D.S + s) * kH + j]) *
             x[static_cast<int64_t>(b) * D.nde + e0 + i];
    } else if (q < p_w2(n)) {                // b1[j]
      const int32_t j = static_cast<int32_t>(q - p_b1(n));
      for (int32_t b = 0; b < B; ++b) g += dh1g[(static_cast<int64_t>(b) * D.S + s) * kH + j];
    } else if (q < p_b2(n)) {                // W2[j][k]
      const int32_t j = static_cast<int32_t>((q - p_w2(n)) / kH), k = static_cast<int32_t>((q - p_w2(n)) % kH);
      for (int32_t b = 0; b < B; ++b) {
        const int64_t o = (static_cast<int64_t>(b) * D.S + s) * kH;
        g += static_cast<double>(dh2g[o + j]) * h1g[o + k];
      }
    } else if (q < p_w3(n)) {                // b2[j]
      const int32_t j = static_cast<int32_t>(q - p_b2(n));
      for (int32_t b = 0; b < B; ++b) g += dh2g[(static_cast<int64_t>(b) * D.S + s) * kH + j];
    } else if (q < p_b3(n)) {                // W3^T[j][i]
      const int32_t j = static_cast<int32_t>((q - p_w3(n)) / n), i = static_cast<int32_t>((q - p_w3(n)) % n);
      for (int32_t b = 0; b < B; ++b)
        g += static_cast<double>(h2g[(static_cast<int64_t>(b) * D.S + s) * kH + j]) *
             dy[static_cast<int64_t>(b) * D.nde + e0 + i];
    } else {                                 // b3[i]
      const int32_t i = static_cast<int32_t>(q - p_b3(n));
      for (int32_t b = 0; b < B; ++b) g += dy[static_cast<int64_t>(b) * D.nde + e0 + i];
    }
    const int64_t k = D.poff[s] + q;
    const float gf = static_cast<float>(g);
    const float a = 0.9f * m1[k] + 0.1f * gf, v = 0.999f * m2[k] + 0.001f * gf * gf;
    m1[k] = a;
    m2[k] = v;
    const float w = W[k] - lr * (a * c1) / (sqrtf(v * c2) + 1e-8f);
    W[k] = w;
    Wb[k] = __float2bfloat16(w);
  }
}

__global__ void k_l_sum(int64_t n, const double* __restrict__ part, double* __restrict__ out) {
  __shared__ double red[32];
  double acc = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) acc += part[i];
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) *out = acc;
}

__global__ void k_l_to_bf16(int64_t n, const float* __restrict__ w, __nv_bfloat16* __restrict__ wb) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    wb[i] = __float2bfloat16(w[i]);
}

}  // namespace

struct LearnState {
  int32_t S = 0, max_n = 0, cap = 0;  // cap: training batch capacity
  int64_t n_params = 0;
  std::vector<int64_t> poff;
  int64_t* d_poff = nullptr;
  float *W = nullptr, *m1 = nullptr, *m2 = nullptr;
  __nv_bfloat16* Wb = nullptr;
  float *x = nullptr, *tx = nullptr, *y = nullptr, *h1 = nullptr, *h2 = nullptr;
  float *dy = nullptr, *dh1 = nullptr, *dh2 = nullptr;
  double *norm = nullptr, *loss_part = nullptr, *loss = nullptr;
  int32_t steps = 0;
  std::vector<void*> mem;
  ~LearnState() {
    for (void* p : mem) cudaFree(p);
  }
};

void free_learn(LearnState* L) { delete L; }

namespace {
LearnDev learn_dev(const FetiDP& F, const LearnState& L) {
  return LearnDev{F.plan.n_parts, F.d_dual_off, F.d_dual_lam, F.d_dual_sign, L.d_poff,
                  F.plan.dual_off[F.plan.n_parts], F.plan.n_lambda};
}

template <class T>
int lalloc(LearnState& L, T** p, int64_t n) {
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, sizeof(T) * std::max<int64_t>(n, 1));
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error(std::string("learned preconditioner: allocation failed: ") + cudaGetErrorString(e));
    return EMG_ERR_NOMEM;
  }
  L.mem.push_back(q);
  *p = static_cast<T*>(q);
  return EMG_SUCCESS;
}

size_t fwd_smem(const LearnState& L) { return sizeof(float) * static_cast<size_t>(std::max(L.max_n, 1)); }

int ensure_batch(FetiDP& F, LearnState& L, int32_t B) {
  if (B <= L.cap) return EMG_SUCCESS;
  const int64_t nde = F.plan.dual_off[F.plan.n_parts];
  const int64_t S = L.S;
  int rc;
  if ((rc = lalloc(L, &L.x, B * nde)) || (rc = lalloc(L, &L.tx, B * nde)) || (rc = lalloc(L, &L.y, B * nde)) ||
      (rc = lalloc(L, &L.dy, B * nde)) || (rc = lalloc(L, &L.h1, B * S * kH)) || (rc = lalloc(L, &L.h2, B * S * kH)) ||
      (rc = lalloc(L, &L.dh1, B * S * kH)) || (rc = lalloc(L, &L.dh2, B * S * kH)) ||
      (rc = lalloc(L, &L.norm, B * S)) || (rc = lalloc(L, &L.loss_part, B * S)))
    return rc;
  L.cap = B;
  return EMG_SUCCESS;
}
}  // namespace

int learned_init(FetiDP& F, uint64_t seed) {
  delete F.learn;
  F.learn = nullptr;
  const FetiPlan& P = F.plan;
  auto* L = new LearnState();
  L->S = P.n_parts;
  L->poff.assign(static_cast<size_t>(P.n_parts) + 1, 0);
  for (int32_t s = 0; s < P.n_parts; ++s) {
    const int64_t n = P.nD[s];
    L->poff[s + 1] = L->poff[s] + 2 * kH * n + 2 * kH + kH * kH + n;
    L->max_n = std::max<int32_t>(L->max_n, P.nD[s]);
  }
  L->n_params = L->poff.back();
  // He initialisation for W1, W2; W3 and all biases zero, so an untrained
  // network adds nothing to the Dirichlet preconditioner
  std::vector<float> w(L->n_params, 0.f);
  std::mt19937_64 rng(seed);
  for (int32_t s = 0; s < P.n_parts; ++s) {
    const int64_t n = P.nD[s], o = L->poff[s];
    std::normal_distribution<float> n1(0.f, std::sqrt(2.f / std::max<int64_t>(n, 1)));
    std::normal_distribution<float> n2(0.f, std::sqrt(2.f / kH));
    for (int64_t q = 0; q < kH * n; ++q) w[o + q] = n1(rng);
    for (int64_t q = 0; q < kH * kH; ++q) w[o + kH * n + kH + q] = n2(rng);
  }
  int rc;
  if ((rc = lalloc(*L, &L->d_poff, P.n_parts + 1)) || (rc = lalloc(*L, &L->W, L->n_params)) ||
      (rc = lalloc(*L, &L->m1, L->n_params)) || (rc = lalloc(*L, &L->m2, L->n_params)) ||
      (rc = lalloc(*L, &L->Wb, L->n_params))) {
    delete L;
    return rc;
  }
  cudaStream_t st = F.st;
  EMG_CK(cudaMemcpyAsync(L->d_poff, L->poff.data(), sizeof(int64_t) * L->poff.size(), cudaMemcpyHostToDevice, st));
  EMG_CK(cudaMemcpyAsync(L->W, w.data(), sizeof(float) * w.size(), cudaMemcpyHostToDevice, st));
  EMG_CK(cudaMemsetAsync(L->m1, 0, sizeof(float) * L->n_params, st));
  EMG_CK(cudaMemsetAsync(L->m2, 0, sizeof(float) * L->n_params, st));
  k_l_to_bf16<<<1184, 256, 0, st>>>(L->n_params, L->W, L->Wb);
  const size_t sm = fwd_smem(*L);
  if (sm > 48 * 1024)
    EMG_CK(cudaFuncSetAttribute(k_l_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sm)));
  EMG_CK(cudaStreamSynchronize(st));
  F.learn = L;
  return ensure_batch(F, *L, 1);
}

// out = add + L(r) for one multiplier vector r (device).
int learned_apply(FetiDP& F, const double* r, const double* add, double* out) {
  LearnState* L = F.learn;
  if (!L) { set_error("learned preconditioner not initialised"); return EMG_INVALID_INPUT; }
  const LearnDev D = learn_dev(F, *L);
  cudaStream_t st = F.st;
  k_l_gather<<<dim3(L->S, 1), 256, 0, st>>>(D, r, nullptr, L->x, nullptr, L->norm);
  k_l_forward<<<dim3(L->S, 1), 256, fwd_smem(*L), st>>>(D, L->Wb, L->x, nullptr, nullptr, L->y);
  k_l_combine<<<256, 256, 0, st>>>(D, F.d_lam_entry, F.d_dual_sub, L->y, L->norm, add, out);
  EMG_CK(cudaGetLastError());
  return EMG_SUCCESS;
}

// One Adam step on a batch of B (residual, target) pairs (B x n_lambda each, device).
int learned_train(FetiDP& F, int32_t B, const double* r, const double* t, float lr, double* loss) {
  LearnState* L = F.learn;
  if (!L) { set_error("learned preconditioner not initialised"); return EMG_INVALID_INPUT; }
  if (B < 1) { set_error("batch must be >= 1"); return EMG_INVALID_INPUT; }
  int rc = ensure_batch(F, *L, B);
  if (rc) return rc;
  const LearnDev D = learn_dev(F, *L);
  cudaStream_t st = F.st;
  const dim3 g(static_cast<unsigned>(L->S), static_cast<unsigned>(B));
  k_l_gather<<<g, 256, 0, st>>>(D, r, t, L->x, L->tx, L->norm);
  k_l_forward<<<g, 256, fwd_smem(*L), st>>>(D, L->Wb, L->x, L->h1, L->h2, L->y);
  const double inv_count = 1.0 / (static_cast<double>(B) * std::max<int64_t>(D.nde, 1));
  k_l_backward<<<g, 256, 0, st>>>(D, L->W, L->y, L->tx, L->h1, L->h2, L->dy, L->dh1, L->dh2, L->loss_part, inv_count);
  ++L->steps;
  const float c1 = 1.f / (1.f - std::pow(0.9f, static_cast<float>(L->steps)));
  const float c2 = 1.f / (1.f - std::pow(0.999f, static_cast<float>(L->steps)));
  int64_t max_np = 0;
  for (int32_t s = 0; s < L->S; ++s) max_np = std::max(max_np, L->poff[s + 1] - L->poff[s]);
  k_l_grad_adam<<<dim3(static_cast<unsigned>(std::min<int64_t>((max_np + 255) / 256, 4096)), L->S), 256, 0, st>>>(
      D, B, L->x, L->h1, L->h2, L->dy, L->dh1, L->dh2, L->W, L->m1, L->m2, L->Wb, lr, c1, c2);
  if (!L->loss) { rc = lalloc(*L, &L->loss, 1); if (rc) return rc; }
  k_l_sum<<<1, 1024, 0, st>>>(static_cast<int64_t>(B) * L->S, L->loss_part, L->loss);
  EMG_CK(cudaGetLastError());
  if (loss) {
    EMG_CK(cudaMemcpyAsync(loss, L->loss, sizeof(double), cudaMemcpyDeviceToHost, st));
    EMG_CK(cudaStreamSynchronize(st));
    *loss *= inv_count;
  }
  return EMG_SUCCESS;
}

int learned_params(FetiDP& F, float* host, int64_t* n, int32_t load) {
  LearnState* L = F.learn;
  if (!L) { set_error("learned preconditioner not initialised"); return EMG_INVALID_INPUT; }
  if (n) *n = L->n_params;
  if (!host) return EMG_SUCCESS;
  if (load) {
    EMG_CK(cudaMemcpyAsync(L->W, host, sizeof(float) * L->n_params, cudaMemcpyHostToDevice, F.st));
    k_l_to_bf16<<<1184, 256, 0, F.st>>>(L->n_params, L->W, L->Wb);
  } else {
    EMG_CK(cudaMemcpyAsync(host, L->W, sizeof(float) * L->n_params, cudaMemcpyDeviceToHost, F.st));
  }
  EMG_CK(cudaStreamSynchronize(F.st));
  return EMG_SUCCESS;
}

}  // namespace emg

// assembly.cu -- EMAssembly::assemble on the GPU for TET4_EDGE and HEX8_EDGE
// elements (reference: src/numeric/em_assembly.cpp:144-420 with the intended
// MagneticVector3DIntegrator formulas, magnetic_vector_3d_integrator.cpp:139-364).
//
// Symbolic phase (once per mesh + DOF map):
//   k_count_rows / scan / k_fill_incidence / k_sort_incidence build, for every
//   equation row r, the sorted list of (element, local edge) slots that map to r;
//   k_row_unique (sorted distinct columns of each row into scratch, counts),
//   a scan and k_row_columns turn those lists into the merged CSR pattern with
//   ascending columns -- the pattern SparseConverter::to_eigen produces from
//   the reference's unmerged CSR (sparse_converter.cpp:19-80).
// Numeric phase:
//   k_assemble_rows (tets) / k_assemble_rows_hex gather, for each row, the
//   contributions of its incident elements in ascending element order and
//   write the row's values once: no atomics,
//   deterministic, and every sum is formed in the same order as an element
//   loop would form it.
#include <cuda_runtime.h>

#include <cstdio>
#include <vector>

#include "common.cuh"
#include "device.h"
#include "internal.h"
#include "trace.h"

namespace emg {

namespace {

constexpr int kMaxSources = 16;
constexpr int kPatternCap = 256;  // candidate columns per row (warp-shared)

__constant__ emg_source c_src[kMaxSources];

enum : int32_t {
  kErrIndex = 1,     // l2g entry >= n
  kErrRowCap = 2,    // more candidate columns than kPatternCap
  kErrSlot = 4,      // column missing from the pattern (internal)
  kErrNode = 8,      // node index out of range
};

// ---------------------------------------------------------------- scan ----
constexpr int kScanTile = 2048;  // elements per block (256 threads x 8)

__global__ void k_scan_tile_sums(const int32_t* __restrict__ in, int64_t n,
                                 int64_t* __restrict__ tile_sums) {
  __shared__ double red[8];
  int64_t base = static_cast<int64_t>(blockIdx.x) * kScanTile;
  int64_t s = 0;
  for (int i = threadIdx.x; i < kScanTile; i += blockDim.x) {
    int64_t g = base + i;
    if (g < n) s += in[g];
  }
  double t = block_sum(static_cast<double>(s), red);  // exact below 2^53
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = static_cast<int64_t>(t);
}

__global__ void k_scan_tiles(int64_t* __restrict__ tile_sums, int64_t n_tiles,
                             int64_t* __restrict__ total) {
  // single block, sequential chunks of blockDim.x
  __shared__ int64_t buf[1024];
  __shared__ int64_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int64_t base = 0; base < n_tiles; base += blockDim.x) {
    int64_t g = base + threadIdx.x;
    int64_t v = g < n_tiles ? tile_sums[g] : 0;
    buf[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < blockDim.x; o <<= 1) {  // Hillis-Steele inclusive
      int64_t a = threadIdx.x >= o ? buf[threadIdx.x - o] : 0;
      __syncthreads();
      buf[threadIdx.x] += a;
      __syncthreads();
    }
    if (g < n_tiles) tile_sums[g] = carry + buf[threadIdx.x] - v;  // exclusive
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry += buf[threadIdx.x];
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void k_scan_apply(const int32_t* __restrict__ in, int64_t n,
                             const int64_t* __restrict__ tile_off, int32_t* __restrict__ out) {
  // 256 threads x 8 consecutive elements
  __shared__ int64_t part[256];
  int64_t base = static_cast<int64_t>(blockIdx.x) * kScanTile + threadIdx.x * 8;
  int64_t loc[8];
  int64_t s = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    int64_t g = base + i;
    loc[i] = s;
    s += g < n ? in[g] : 0;
  }
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < 256; o <<= 1) {
    int64_t a = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += a;
    __syncthreads();
  }
  int64_t off = tile_off[blockIdx.x] + part[threadIdx.x] - s;
  if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = static_cast<int32_t>(tile_off[gridDim.x]);
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    int64_t g = base + i;
    if (g < n) out[g] = static_cast<int32_t>(off + loc[i]);
  }
}

// ----------------------------------------------------------- incidence ----
__global__ void k_count_rows(const int32_t* __restrict__ l2g, int64_t m, int64_t n,
                             int32_t* __restrict__ cnt, int32_t* __restrict__ err) {
  for (int64_t p = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; p < m;
       p += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int32_t r = l2g[p];
    if (r >= n || r < -1) { atomicOr(err, kErrIndex); continue; }
    if (r >= 0) atomicAdd(&cnt[r], 1);
  }
}

__global__ void k_fill_incidence(const int32_t* __restrict__ l2g, int64_t m,
                                 const int32_t* __restrict__ inc_ptr, int32_t* __restrict__ cursor,
                                 int32_t* __restrict__ inc) {
  for (int64_t p = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; p < m;
       p += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int32_t r = l2g[p];
    if (r < 0) continue;
    int32_t s = inc_ptr[r] + atomicAdd(&cursor[r], 1);
    inc[s] = static_cast<int32_t>(p);
  }
}

__global__ void k_sort_incidence(const int32_t* __restrict__ inc_ptr, int32_t* __restrict__ inc,
                                 int64_t n) {
  for (int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; r < n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int32_t a = inc_ptr[r], b = inc_ptr[r + 1];
    for (int32_t i = a + 1; i < b; ++i) {
      int32_t v = inc[i];
      int32_t j = i - 1;
      while (j >= a && inc[j] > v) { inc[j + 1] = inc[j]; --j; }
      inc[j + 1] = v;
    }
  }
}

// Sorts the 64 values v0 (index lane) and v1 (index lane + 32) of a warp
// ascending with a bitonic network in registers.
__device__ __forceinline__ void warp_sort64(int32_t& v0, int32_t& v1) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 2; k <= 64; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      if (j == 32) {  // pairs (lane, lane + 32), k == 64: ascending
        const int32_t lo = min(v0, v1), hi = max(v0, v1);
        v0 = lo;
        v1 = hi;
      } else {
        const int32_t p0 = __shfl_xor_sync(0xffffffffu, v0, j);
        const int32_t p1 = __shfl_xor_sync(0xffffffffu, v1, j);
        const bool lower = (lane & j) == 0;
        const bool up0 = (lane & k) == 0, up1 = ((lane + 32) & k) == 0;
        v0 = (lower == up0) ? min(v0, p0) : max(v0, p0);
        v1 = (lower == up1) ? min(v1, p1) : max(v1, p1);
      }
    }
  }
}

// Warp per row: the distinct columns of all incident elements (slot = epe *
// element + local edge), ascending, into tmp[inc_ptr[r] * epe ...] (room for
// every candidate of the row), and their count into counts[r].  Rows of up to
// 64 candidates are sorted in registers; longer rows (up to kPatternCap) go
// through shared memory.
__global__ void __launch_bounds__(128) k_row_unique(int64_t n, int epe, const int32_t* __restrict__ inc_ptr,
                                                    const int32_t* __restrict__ inc,
                                                    const int32_t* __restrict__ l2g,
                                                    int32_t* __restrict__ counts, int32_t* __restrict__ tmp,
                                                    int32_t* __restrict__ err) {
  __shared__ int32_t cand_all[4][kPatternCap];
  __shared__ uint8_t first_all[4][kPatternCap];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  int32_t* cand = cand_all[wib];
  uint8_t* first = first_all[wib];
  const unsigned lt = (1u << lane) - 1u;
  const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + wib; r < n; r += warps) {
    const int32_t a = inc_ptr[r], b = inc_ptr[r + 1];
    const int m = epe * (b - a);
    int32_t* out = tmp + static_cast<int64_t>(a) * epe;
    if (m <= 64) {
      int32_t v0 = INT32_MAX, v1 = INT32_MAX;
      if (lane < m) {
        const int32_t slot = inc[a + lane / epe];
        v0 = l2g[epe * (slot / epe) + (lane % epe)];
      }
      if (lane + 32 < m) {
        const int32_t slot = inc[a + (lane + 32) / epe];
        v1 = l2g[epe * (slot / epe) + ((lane + 32) % epe)];
      }
      if (v0 < 0) v0 = INT32_MAX;  // constrained / gauged-out local edges
      if (v1 < 0) v1 = INT32_MAX;
      warp_sort64(v0, v1);
      // every lane takes part in each shuffle; lane 0 then swaps in v0 of lane 31
      const int32_t prev0 = __shfl_up_sync(0xffffffffu, v0, 1);
      const int32_t last0 = __shfl_sync(0xffffffffu, v0, 31);
      const int32_t up1 = __shfl_up_sync(0xffffffffu, v1, 1);
      const int32_t prev1 = lane ? up1 : last0;
      const bool keep0 = v0 != INT32_MAX && (lane == 0 || v0 != prev0);
      const bool keep1 = v1 != INT32_MAX && v1 != prev1;
      const unsigned b0 = __ballot_sync(0xffffffffu, keep0), b1 = __ballot_sync(0xffffffffu, keep1);
      if (keep0) out[__popc(b0 & lt)] = v0;
      if (keep1) out[__popc(b0) + __popc(b1 & lt)] = v1;
      if (lane == 0) counts[r] = __popc(b0) + __popc(b1);
      continue;
    }
    if (m > kPatternCap) {
      if (lane == 0) {
        atomicOr(err, kErrRowCap);
        counts[r] = 0;
      }
      continue;
    }
    for (int idx = lane; idx < m; idx += 32) {
      const int32_t slot = inc[a + idx / epe];
      cand[idx] = l2g[epe * (slot / epe) + (idx % epe)];
    }
    __syncwarp();
    for (int idx = lane; idx < m; idx += 32) {  // first occurrence of each valid column
      const int32_t c = cand[idx];
      bool f = c >= 0;
      for (int j = 0; j < idx && f; ++j) f = cand[j] != c;
      first[idx] = f ? 1 : 0;
    }
    __syncwarp();
    int kept = 0;
    for (int base = 0; base < m; base += 32) {
      const int idx = base + lane;
      const bool keep = idx < m && first[idx];
      kept += __popc(__ballot_sync(0xffffffffu, keep));
      if (keep) {
        const int32_t c = cand[idx];
        int rank = 0;  // distinct columns smaller than c
        for (int j = 0; j < m; ++j) rank += (first[j] && cand[j] < c) ? 1 : 0;
        out[rank] = c;
      }
    }
    if (lane == 0) counts[r] = kept;
    __syncwarp();
  }
}

// Warp per row: the row's columns from the scratch rows into the CSR.
__global__ void __launch_bounds__(128) k_row_columns(int64_t n, int epe, const int32_t* __restrict__ inc_ptr,
                                                     const int32_t* __restrict__ tmp,
                                                     const int32_t* __restrict__ row_ptr,
                                                     int32_t* __restrict__ col) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  for (int64_t r = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; r < n; r += warps) {
    const int32_t* src = tmp + static_cast<int64_t>(inc_ptr[r]) * epe;
    const int32_t c0 = row_ptr[r], len = row_ptr[r + 1] - c0;
    for (int k = lane; k < len; k += 32) col[c0 + k] = src[k];
  }
}

// --------------------------------------------------------------- numeric ----
// Nedelec TET4_EDGE edge table (nedelec_element.cpp:54-60): basis k is
// lambda_b grad(lambda_a) - lambda_a grad(lambda_b) for (a, b) = (ned_a(k), ned_b(k)).
// Closed forms of kNed = {(0,1),(1,2),(2,0),(0,3),(1,3),(2,3)}: with k unrolled
// they fold to constants, so no per-thread array is indexed at run time.
__host__ __device__ constexpr int ned_a(int k) { return k < 3 ? k : k - 3; }
__host__ __device__ constexpr int ned_b(int k) { return k < 3 ? (k + 1) % 3 : 3; }
static_assert(ned_a(2) == 2 && ned_b(2) == 0 && ned_a(4) == 1 && ned_b(4) == 3, "nedelec_element.cpp:54-60");

struct Tet {
  double d[3][3];  // d[c] = x_c - x_3 (Jacobian columns)
  double det;
  double g[4][3];  // physical gradients of the barycentric coordinates
  double c[6][3];  // physical curls (J curl_ref / det)
  double x3[3];
  int32_t node[4];
};

__device__ __forceinline__ void cross(const double* a, const double* b, double* o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

__device__ __forceinline__ bool load_tet(const int32_t* __restrict__ tets,
                                         const double* __restrict__ xyz, int64_t n_nodes,
                                         int64_t t, Tet& T) {
  int4 nd = reinterpret_cast<const int4*>(tets)[t];
  T.node[0] = nd.x; T.node[1] = nd.y; T.node[2] = nd.z; T.node[3] = nd.w;
  double x[4][3];
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    int32_t g = T.node[a];
    if (g < 0 || g >= n_nodes) return false;
    x[a][0] = xyz[3 * g]; x[a][1] = xyz[3 * g + 1]; x[a][2] = xyz[3 * g + 2];
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
#pragma unroll
    for (int r = 0; r < 3; ++r) T.d[c][r] = x[c][r] - x[3][r];
  }
#pragma unroll
  for (int r = 0; r < 3; ++r) T.x3[r] = x[3][r];
  double c12[3], c20[3], c01[3];
  cross(T.d[1], T.d[2], c12);
  cross(T.d[2], T.d[0], c20);
  cross(T.d[0], T.d[1], c01);
  T.det = T.d[0][0] * c12[0] + T.d[0][1] * c12[1] + T.d[0][2] * c12[2];
  const double inv = 1.0 / T.det;
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    T.g[0][r] = c12[r] * inv;  // rows of J^-1 = physical gradients
    T.g[1][r] = c20[r] * inv;
    T.g[2][r] = c01[r] * inv;
    T.g[3][r] = -(T.g[0][r] + T.g[1][r] + T.g[2][r]);
  }
  // J * curl_ref / det with curl_ref from curlTet4Edge (nedelec_element.cpp:461-505)
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const double a0 = T.d[0][r] * inv, a1 = T.d[1][r] * inv, a2 = T.d[2][r] * inv;
    T.c[0][r] = -2.0 * a2;
    T.c[1][r] = -2.0 * a0;
    T.c[2][r] = -2.0 * a1;
    T.c[3][r] = -2.0 * a1 + 2.0 * a2;
    T.c[4][r] = 2.0 * a0 - 2.0 * a2;
    T.c[5][r] = -2.0 * a0 + 2.0 * a1;
  }
  return true;
}

// Sum of the current densities of the regions tab[first .. first+count) that
// contain x (open regions).
__device__ __forceinline__ void source_at(const double* x, const emg_source* tab, int first, int count,
                                          double* js) {
  js[0] = js[1] = js[2] = 0.0;
  for (int s = first; s < first + count; ++s) {
    const double* p = tab[s].p;
    bool in = false;
    if (tab[s].kind == EMG_SRC_BOX) {
      in = x[0] > p[0] && x[0] < p[1] && x[1] > p[2] && x[1] < p[3] && x[2] > p[4] && x[2] < p[5];
    } else if (tab[s].kind == EMG_SRC_ANNULUS_Z) {
      const double dx = x[0] - p[0], dy = x[1] - p[1];
      const double rr = sqrt(dx * dx + dy * dy);
      in = rr > p[2] && rr < p[3] && x[2] > p[4] && x[2] < p[5];
    }
    if (in) { js[0] += tab[s].j[0]; js[1] += tab[s].j[1]; js[2] += tab[s].j[2]; }
  }
}

__device__ __forceinline__ int find_slot(const int32_t* __restrict__ col, int32_t lo, int32_t hi,
                                         int32_t c) {
  while (lo < hi) {
    int32_t mid = (lo + hi) >> 1;
    if (col[mid] < c) lo = mid + 1; else hi = mid;
  }
  return lo;
}

struct AsmArgs {
  int64_t n, n_nodes;
  const int32_t* row_ptr;
  const int32_t* col;
  const int32_t* inc_ptr;
  const int32_t* inc;
  const int32_t* elems;
  const double* xyz;
  const int32_t* material;
  const int32_t* l2g;
  const double* nu;
  const double* sigma;
  int32_t n_mat, n_src, flags;
  const emg_source* src_tab;  // global source table when src_map is set
  const int32_t* src_map;     // per-tet source index (-1 = none) or null
  double* kval;
  double* mval;
  double* rhs;
  int32_t* err;
};

// Thread per row: K(r, c) = sum over incident tets of
//   nu |det| wsum s_i s_j curl_i . curl_j
// where curl_k = J curl_ref_k / det is constant per tet, so the quadrature
// sum collapses to the weight sum (1/6 for the Hammer rule, 1/8 for the
// reference's 3-point rule).  M and F are integrated at the quadrature points.
__global__ void __launch_bounds__(128) k_assemble_rows(AsmArgs A) {
  const double qa = 0.13819660112501051517954131656343619;   // (5 - sqrt 5) / 20
  const double qb = 0.58541019662496845446137605030969143;   // (5 + 3 sqrt 5) / 20
  const bool quad3 = (A.flags & EMG_FLAG_QUAD3_LITERAL) != 0;
  const int nq = quad3 ? 3 : 4;
  const double w = 1.0 / 24.0;
  const bool want_mass = (A.flags & EMG_FLAG_MASS) != 0 && A.mval != nullptr;
  const bool signs = (A.flags & EMG_FLAG_NO_EDGE_SIGNS) == 0;
  const bool literal = (A.flags & EMG_FLAG_PIOLA_LITERAL) != 0;
  for (int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; r < A.n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t s0 = A.row_ptr[r], s1 = A.row_ptr[r + 1];
    for (int32_t k = s0; k < s1; ++k) {
      A.kval[k] = 0.0;
      if (want_mass) A.mval[k] = 0.0;
    }
    double f = 0.0;
    for (int32_t q = A.inc_ptr[r]; q < A.inc_ptr[r + 1]; ++q) {
      const int32_t slot = A.inc[q];
      const int64_t t = slot / 6;
      const int i = slot - 6 * static_cast<int>(t);
      const int32_t mid = A.material ? A.material[t] : 0;
      if (mid < 0 || mid >= A.n_mat) continue;  // em_assembly.cpp:270-276 skips the element
      Tet T;
      if (!load_tet(A.elems, A.xyz, A.n_nodes, t, T)) { atomicOr(A.err, kErrNode); continue; }
      const double adet = fabs(T.det);
      if (adet < 1e-15) continue;  // every quadrature point skipped (:169)
      // the row's own local edge, picked out with compile-time indices
      int sgi = 1;
      double ci[3] = {0, 0, 0};
#pragma unroll
      for (int k = 0; k < 6; ++k)
        if (k == i) {
          if (signs) sgi = T.node[ned_b(k)] < T.node[ned_a(k)] ? 1 : -1;
          ci[0] = T.c[k][0]; ci[1] = T.c[k][1]; ci[2] = T.c[k][2];
        }
      const double kf = nq * w * adet * A.nu[mid];
      const double sig = A.sigma ? A.sigma[mid] : 0.0;
      const bool do_mass = want_mass && sig > 0.0;
      const emg_source* tab = c_src;
      int src_first = 0, src_count = A.n_src;
      if (A.src_map) {
        tab = A.src_tab;
        const int32_t sid = A.src_map[t];
        src_first = sid;
        src_count = (sid >= 0 && sid < A.n_src) ? 1 : 0;
      }
      const bool do_src = src_count > 0;
      int32_t pos[6];
#pragma unroll
      for (int j = 0; j < 6; ++j) {
        const int32_t cj = A.l2g[6 * t + j];
        pos[j] = cj >= 0 ? find_slot(A.col, s0, s1, cj) : -1;
        if (cj >= 0 && (pos[j] >= s1 || A.col[pos[j]] != cj)) {
          atomicOr(A.err, kErrSlot);
          pos[j] = -1;
        }
      }
#pragma unroll
      for (int j = 0; j < 6; ++j) {
        if (pos[j] < 0) continue;
        const int sgj = signs ? (T.node[ned_b(j)] < T.node[ned_a(j)] ? 1 : -1) : 1;
        const double d = ci[0] * T.c[j][0] + ci[1] * T.c[j][1] + ci[2] * T.c[j][2];
        A.kval[pos[j]] += static_cast<double>(sgi * sgj) * (kf * d);
      }
      if (do_mass || do_src) {
        double mrow[6] = {0, 0, 0, 0, 0, 0};
        double fi = 0.0;
        for (int qq = 0; qq < nq; ++qq) {
          double lam[4];
          if (qq == 0) { lam[0] = qa; lam[1] = qa; lam[2] = qb; }
          else if (qq == 1) { lam[0] = qa; lam[1] = qb; lam[2] = qa; }
          else if (qq == 2 && !quad3) { lam[0] = qb; lam[1] = qa; lam[2] = qa; }
          else { lam[0] = qa; lam[1] = qa; lam[2] = qa; }
          lam[3] = 1.0 - lam[0] - lam[1] - lam[2];
          double W[6][3], Wi[3] = {0, 0, 0};
#pragma unroll
          for (int k = 0; k < 6; ++k) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              W[k][c] = lam[ned_b(k)] * T.g[ned_a(k)][c] - lam[ned_a(k)] * T.g[ned_b(k)][c];
              if (literal) W[k][c] /= T.det;
            }
            if (k == i) { Wi[0] = W[k][0]; Wi[1] = W[k][1]; Wi[2] = W[k][2]; }
          }
          if (do_mass) {
#pragma unroll
            for (int j = 0; j < 6; ++j)
              mrow[j] += w * adet * sig * (Wi[0] * W[j][0] + Wi[1] * W[j][1] + Wi[2] * W[j][2]);
          }
          if (do_src) {
            double x[3], js[3];
#pragma unroll
            for (int c = 0; c < 3; ++c)
              x[c] = T.x3[c] + lam[0] * T.d[0][c] + lam[1] * T.d[1][c] + lam[2] * T.d[2][c];
            source_at(x, tab, src_first, src_count, js);
            fi += w * adet * (Wi[0] * js[0] + Wi[1] * js[1] + Wi[2] * js[2]);
          }
        }
        if (do_mass) {
#pragma unroll
          for (int j = 0; j < 6; ++j)
            if (pos[j] >= 0) {
              const int sgj = signs ? (T.node[ned_b(j)] < T.node[ned_a(j)] ? 1 : -1) : 1;
              A.mval[pos[j]] += static_cast<double>(sgi * sgj) * mrow[j];
            }
        }
        f += sgi * fi;
      }
    }
    A.rhs[r] = f;
  }
}

// ----------------------------------------------------------- HEX8_EDGE ----
// Reference hexahedron [-1,1]^3, nodes 0-3 on zeta = -1 (counter-clockwise
// from (-1,-1)), 4-7 above them (nedelec_element.cpp:506-517).  Edge k runs
// from local node A to B (ElementGeometry's table, element_geometry.cpp:165-171)
// along reference axis d; with (p, q) = (d+1, d+2) mod 3 and c_p, c_q the
// edge's fixed coordinates, its basis (evalHex8Edge, nedelec_element.cpp:519-615) is
//   W_k = 1/2 s_k (1 + c_p x_p)(1 + c_q x_q) e_d,   s_k = (x_d(B) - x_d(A)) / 2,
// with curl
//   curl W_k = 1/2 s_k [c_q (1 + c_p x_p) e_p - c_p (1 + c_q x_q) e_q].
// (curlHex8Edge, :618-720, has sign / component errors in edges 2, 3, 6, 7;
// the curl here is the derivative of the reference's own W_k.)  The tables
// are closed forms, so with k unrolled they fold to compile-time constants.
__host__ __device__ constexpr int hex_node_coord(int a, int axis) {  // reference coordinate of node a
  return axis == 0 ? (((a & 3) == 1 || (a & 3) == 2) ? 1 : -1) : axis == 1 ? ((a & 2) ? 1 : -1) : ((a & 4) ? 1 : -1);
}
__host__ __device__ constexpr int hex_edge_a(int k) { return k < 8 ? k : k - 8; }
__host__ __device__ constexpr int hex_edge_b(int k) { return k < 4 ? ((k + 1) & 3) : k < 8 ? 4 + ((k + 1) & 3) : k - 4; }
__host__ __device__ constexpr int hex_dir(int k) { return k < 8 ? (k & 1) : 2; }
__host__ __device__ constexpr int hex_sgn(int k) {
  return (hex_node_coord(hex_edge_b(k), hex_dir(k)) - hex_node_coord(hex_edge_a(k), hex_dir(k))) / 2;
}
__host__ __device__ constexpr int hex_cp(int k) { return hex_node_coord(hex_edge_a(k), (hex_dir(k) + 1) % 3); }
__host__ __device__ constexpr int hex_cq(int k) { return hex_node_coord(hex_edge_a(k), (hex_dir(k) + 2) % 3); }
static_assert(hex_edge_a(2) == 2 && hex_edge_b(2) == 3 && hex_edge_b(3) == 0 && hex_edge_b(7) == 4 &&
                  hex_edge_b(11) == 7,
              "edge table of element_geometry.cpp:165-171");
static_assert(hex_sgn(2) == -1 && hex_sgn(3) == -1 && hex_sgn(6) == -1 && hex_sgn(7) == -1 && hex_sgn(8) == 1,
              "basis orientation of nedelec_element.cpp:519-615");
static_assert(hex_cp(0) == -1 && hex_cq(0) == -1 && hex_cp(1) == -1 && hex_cq(1) == 1 && hex_cp(9) == 1 &&
                  hex_cq(9) == -1,
              "edge positions");

// Thread per row, 2x2x2 Gauss-Legendre (points +-1/sqrt 3, weights 1):
//   K(r, c) = sum_q nu / |det J| (curl_ref_i)^T (J^T J) (curl_ref_j)
//   M(r, c) = sum_q sigma |det J| f_i f_j [(J^T J)^-1]_{d_i d_j}
//   F(r)    = sum_q |det J| f_i [J^-1 J_s(x_q)]_{d_i}
// (curl_phys = J curl_ref / det J, W_phys = J^-T W_ref; EMG_FLAG_PIOLA_LITERAL
// divides W_phys by det J once more), incident elements in ascending order.
template <bool kMass>
__global__ void __launch_bounds__(128) k_assemble_rows_hex(AsmArgs A) {
  const double g = 0.57735026918962576450914878050195746;  // 1 / sqrt 3
  const bool want_mass = kMass && A.mval != nullptr;
  const bool signs = (A.flags & EMG_FLAG_NO_EDGE_SIGNS) == 0;
  const bool literal = (A.flags & EMG_FLAG_PIOLA_LITERAL) != 0;
  for (int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; r < A.n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t s0 = A.row_ptr[r], s1 = A.row_ptr[r + 1];
    for (int32_t k = s0; k < s1; ++k) {
      A.kval[k] = 0.0;
      if (want_mass) A.mval[k] = 0.0;
    }
    double f = 0.0;
    for (int32_t u = A.inc_ptr[r]; u < A.inc_ptr[r + 1]; ++u) {
      const int32_t slot = A.inc[u];
      const int64_t t = slot / 12;
      const int i = slot - 12 * static_cast<int>(t);
      const int32_t mid = A.material ? A.material[t] : 0;
      if (mid < 0 || mid >= A.n_mat) continue;  // em_assembly.cpp:270-276 skips the element
      const int4 n0 = reinterpret_cast<const int4*>(A.elems)[2 * t];
      const int4 n1 = reinterpret_cast<const int4*>(A.elems)[2 * t + 1];
      const int32_t node[8] = {n0.x, n0.y, n0.z, n0.w, n1.x, n1.y, n1.z, n1.w};
      double x[8][3];
      bool ok = true;
#pragma unroll
      for (int a = 0; a < 8; ++a) {
        const int32_t gn = node[a];
        if (gn < 0 || gn >= A.n_nodes) { ok = false; break; }
        x[a][0] = A.xyz[3 * gn]; x[a][1] = A.xyz[3 * gn + 1]; x[a][2] = A.xyz[3 * gn + 2];
      }
      if (!ok) { atomicOr(A.err, kErrNode); continue; }
      int sgi = 1;
#pragma unroll
      for (int k = 0; k < 12; ++k)
        if (k == i && signs) sgi = node[hex_edge_a(k)] < node[hex_edge_b(k)] ? 1 : -1;
      const double nu = A.nu[mid];
      const double sig = A.sigma ? A.sigma[mid] : 0.0;
      const bool do_mass = want_mass && sig > 0.0;
      const emg_source* tab = c_src;
      int src_first = 0, src_count = A.n_src;
      if (A.src_map) {
        tab = A.src_tab;
        const int32_t sid = A.src_map[t];
        src_first = sid;
        src_count = (sid >= 0 && sid < A.n_src) ? 1 : 0;
      }
      const bool do_src = src_count > 0;
      int32_t pos[12];
#pragma unroll
      for (int j = 0; j < 12; ++j) {
        const int32_t c = A.l2g[12 * t + j];
        pos[j] = c >= 0 ? find_slot(A.col, s0, s1, c) : -1;
        if (c >= 0 && (pos[j] >= s1 || A.col[pos[j]] != c)) {
          atomicOr(A.err, kErrSlot);
          pos[j] = -1;
        }
      }
      double krow[12], mrow[kMass ? 12 : 1];
#pragma unroll
      for (int j = 0; j < 12; ++j) krow[j] = 0.0;
#pragma unroll
      for (int j = 0; j < (kMass ? 12 : 1); ++j) mrow[j] = 0.0;
      double fi = 0.0;
      const int di = hex_dir(i);
      for (int q = 0; q < 8; ++q) {
        const double xi[3] = {(q & 1) ? g : -g, (q & 2) ? g : -g, (q & 4) ? g : -g};
        // J[r][c] = dx_r / dxi_c of the trilinear map
        double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
        for (int a = 0; a < 8; ++a) {
          const double s0 = hex_node_coord(a, 0), s1 = hex_node_coord(a, 1), s2 = hex_node_coord(a, 2);
          const double l0 = 1.0 + s0 * xi[0], l1 = 1.0 + s1 * xi[1], l2 = 1.0 + s2 * xi[2];
          const double dn[3] = {0.125 * s0 * l1 * l2, 0.125 * s1 * l0 * l2, 0.125 * s2 * l0 * l1};
#pragma unroll
          for (int rr = 0; rr < 3; ++rr)
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) J[rr][cc] += x[a][rr] * dn[cc];
        }
        // adjugate rows: inv(J) = adj / det
        double adj[3][3];
        adj[0][0] = J[1][1] * J[2][2] - J[1][2] * J[2][1];
        adj[0][1] = J[0][2] * J[2][1] - J[0][1] * J[2][2];
        adj[0][2] = J[0][1] * J[1][2] - J[0][2] * J[1][1];
        adj[1][0] = J[1][2] * J[2][0] - J[1][0] * J[2][2];
        adj[1][1] = J[0][0] * J[2][2] - J[0][2] * J[2][0];
        adj[1][2] = J[0][2] * J[1][0] - J[0][0] * J[1][2];
        adj[2][0] = J[1][0] * J[2][1] - J[1][1] * J[2][0];
        adj[2][1] = J[0][1] * J[2][0] - J[0][0] * J[2][1];
        adj[2][2] = J[0][0] * J[1][1] - J[0][1] * J[1][0];
        const double det = J[0][0] * adj[0][0] + J[0][1] * adj[1][0] + J[0][2] * adj[2][0];
        // row d_i of adj (J^-1 = adj / det)
        const double ad[3] = {di == 0 ? adj[0][0] : di == 1 ? adj[1][0] : adj[2][0],
                              di == 0 ? adj[0][1] : di == 1 ? adj[1][1] : adj[2][1],
                              di == 0 ? adj[0][2] : di == 1 ? adj[1][2] : adj[2][2]};
        const double adet = fabs(det);
        if (adet < 1e-15) continue;  // quadrature point skipped (magnetic_vector_3d_integrator.cpp:169)
        // Physical curls (without the 1/det) u_k = J curl_ref_k and the
        // reference basis magnitudes f_k for all 12 edges, the row's own
        // picked out of the same arrays: every product below is formed from
        // the same values in row i and row j, so K and M come out exactly
        // symmetric whatever the contraction into FMAs.
        double u[12][3], fk[12];
#pragma unroll
        for (int k = 0; k < 12; ++k) {
          const int dk = hex_dir(k), pk = (dk + 1) % 3, qk = (dk + 2) % 3;
          const double hk = 0.5 * hex_sgn(k);
          const double lp = 1.0 + hex_cp(k) * xi[pk], lq = 1.0 + hex_cq(k) * xi[qk];
          const double cp = hk * hex_cq(k) * lp, cq = -hk * hex_cp(k) * lq;
#pragma unroll
          for (int rr = 0; rr < 3; ++rr) u[k][rr] = J[rr][pk] * cp + J[rr][qk] * cq;
          fk[k] = hk * lp * lq;  // W_ref_k = f_k e_{d_k}
        }
        double ui[3] = {0, 0, 0}, fi_q = 0.0;
#pragma unroll
        for (int k = 0; k < 12; ++k)
          if (k == i) { ui[0] = u[k][0]; ui[1] = u[k][1]; ui[2] = u[k][2]; fi_q = fk[k]; }
        const double kq = nu / adet;
#pragma unroll
        for (int j = 0; j < 12; ++j) krow[j] += kq * (ui[0] * u[j][0] + ui[1] * u[j][1] + ui[2] * u[j][2]);
        if (do_mass || do_src) {
          const double wscale = literal ? 1.0 / det : 1.0;
          if (kMass && do_mass) {
            // W_i . W_j = f_i f_j [adj adj^T]_{d_i d_j} / det^2, the 3x3 Gram
            // matrix of the adjugate rows formed symmetrically
            double H[3][3];
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
              for (int b = 0; b < 3; ++b) H[a][b] = adj[a][0] * adj[b][0] + adj[a][1] * adj[b][1] + adj[a][2] * adj[b][2];
            const double Hi[3] = {di == 0 ? H[0][0] : di == 1 ? H[1][0] : H[2][0],
                                  di == 0 ? H[0][1] : di == 1 ? H[1][1] : H[2][1],
                                  di == 0 ? H[0][2] : di == 1 ? H[1][2] : H[2][2]};
            const double mq = sig * adet * wscale * wscale / (det * det);
#pragma unroll
            for (int j = 0; j < (kMass ? 12 : 1); ++j) mrow[j] += (mq * (fi_q * fk[j])) * Hi[hex_dir(j)];
          }
          if (do_src) {
            double xq[3] = {0, 0, 0};
#pragma unroll
            for (int a = 0; a < 8; ++a) {
              const double na = 0.125 * (1.0 + hex_node_coord(a, 0) * xi[0]) * (1.0 + hex_node_coord(a, 1) * xi[1]) *
                                (1.0 + hex_node_coord(a, 2) * xi[2]);
#pragma unroll
              for (int c = 0; c < 3; ++c) xq[c] += na * x[a][c];
            }
            double js[3];
            source_at(xq, tab, src_first, src_count, js);
            const double ji = (ad[0] * js[0] + ad[1] * js[1] + ad[2] * js[2]) / det;
            fi += adet * wscale * fi_q * ji;
          }
        }
      }
#pragma unroll
      for (int j = 0; j < 12; ++j) {
        if (pos[j] < 0) continue;
        const int sgj = signs ? (node[hex_edge_a(j)] < node[hex_edge_b(j)] ? 1 : -1) : 1;
        A.kval[pos[j]] += static_cast<double>(sgi * sgj) * krow[j];
        if (kMass && do_mass) A.mval[pos[j]] += static_cast<double>(sgi * sgj) * mrow[kMass ? j : 0];
      }
      f += sgi * fi;
    }
    A.rhs[r] = f;
  }
}

int grid_for(int64_t work, int threads, int max_blocks = 148 * 16) {
  int64_t b = (work + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > max_blocks) b = max_blocks;
  return static_cast<int>(b);
}

std::string err_text(int32_t e) {
  std::string s;
  if (e & kErrIndex) s += " l2g index outside [-1, n_dofs);";
  if (e & kErrRowCap) s += " a row has more than 256 candidate columns;";
  if (e & kErrSlot) s += " pattern lookup failed;";
  if (e & kErrNode) s += " node index outside [0, n_nodes);";
  return s;
}

}  // namespace

int scan_counts(const int32_t* counts, int32_t* out, int64_t n, int64_t* total, cudaStream_t st) {
  int64_t tiles = (n + kScanTile - 1) / kScanTile;
  if (tiles < 1) tiles = 1;
  int64_t* tile = nullptr;
  EMG_CK(cudaMallocAsync(&tile, sizeof(int64_t) * (tiles + 1), st));
  k_scan_tile_sums<<<static_cast<unsigned>(tiles), 256, 0, st>>>(counts, n, tile);
  k_scan_tiles<<<1, 1024, 0, st>>>(tile, tiles, tile + tiles);
  k_scan_apply<<<static_cast<unsigned>(tiles), 256, 0, st>>>(counts, n, tile, out);
  int64_t tot = 0;
  EMG_CK(cudaMemcpyAsync(&tot, tile + tiles, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  EMG_CK(cudaStreamSynchronize(st));
  EMG_CK(cudaFreeAsync(tile, st));
  EMG_CK(cudaGetLastError());
  *total = tot;
  return EMG_SUCCESS;
}

int system_build(System& s, cudaStream_t st) {
  trace_pool("system_build.begin");
  trace_mark(st, "build.begin");
  const int epe = edges_per_elem(s.elem_type);
  const int64_t m = epe * s.n_elems, n = s.n;
  int32_t* cnt = nullptr;
  EMG_CK(cudaMallocAsync(&cnt, sizeof(int32_t) * (n + 1), st));
  EMG_CK(cudaMemsetAsync(cnt, 0, sizeof(int32_t) * (n + 1), st));
  EMG_CK(cudaMemsetAsync(s.err, 0, sizeof(int32_t), st));
  k_count_rows<<<grid_for(m, 256), 256, 0, st>>>(s.l2g, m, n, cnt, s.err);
  EMG_CK(cudaGetLastError());
  EMG_CK(cudaMallocAsync(&s.inc_ptr, sizeof(int32_t) * (n + 1), st));
  int64_t inc_total = 0;
  int rc = scan_counts(cnt, s.inc_ptr, n, &inc_total, st);
  if (rc) return rc;
  trace_mark(st, "build.count_scan");
  int32_t herr = 0;
  EMG_CK(cudaMemcpyAsync(&herr, s.err, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  EMG_CK(cudaStreamSynchronize(st));
  if (herr) { set_error("system build:" + err_text(herr)); return EMG_INVALID_INPUT; }
  EMG_CK(cudaMallocAsync(&s.inc, sizeof(int32_t) * (inc_total > 0 ? inc_total : 1), st));
  EMG_CK(cudaMemsetAsync(cnt, 0, sizeof(int32_t) * (n + 1), st));
  k_fill_incidence<<<grid_for(m, 256), 256, 0, st>>>(s.l2g, m, s.inc_ptr, cnt, s.inc);
  k_sort_incidence<<<grid_for(n, 128), 128, 0, st>>>(s.inc_ptr, s.inc, n);
  trace_mark(st, "build.fill_sort");
  int32_t* tmp = nullptr;  // every row's candidates: epe per incident slot
  {
    TraceScope t("build.tmp_malloc_call");
    EMG_CK(cudaMallocAsync(&tmp, sizeof(int32_t) * (inc_total > 0 ? inc_total * epe : 1), st));
  }
  {
    TraceScope t("build.row_unique_launch_call");
    k_row_unique<<<grid_for(n * 32, 128), 128, 0, st>>>(n, epe, s.inc_ptr, s.inc, s.l2g, cnt, tmp, s.err);
  }
  EMG_CK(cudaGetLastError());
  trace_mark(st, "build.row_unique");
  EMG_CK(cudaMallocAsync(&s.K.row_ptr, sizeof(int32_t) * (n + 1), st));
  int64_t nnz = 0;
  rc = scan_counts(cnt, s.K.row_ptr, n, &nnz, st);
  trace_mark(st, "build.scan2");
  if (!rc) {
    EMG_CK(cudaMemcpyAsync(&herr, s.err, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    EMG_CK(cudaStreamSynchronize(st));
    if (herr) {
      set_error("system build:" + err_text(herr));
      rc = EMG_INVALID_INPUT;
    } else if (nnz >= (int64_t(1) << 31)) {
      set_error("nnz exceeds int32 range");
      rc = EMG_INVALID_INPUT;
    }
  }
  if (rc) {
    cudaFreeAsync(tmp, st);
    cudaFreeAsync(cnt, st);
    return rc;
  }
  s.K.n = n;
  s.K.nnz = nnz;
  {
    TraceScope t("build.colval_malloc_call");
    EMG_CK(cudaMallocAsync(&s.K.col, sizeof(int32_t) * (nnz > 0 ? nnz : 1), st));
    EMG_CK(cudaMallocAsync(&s.K.val, sizeof(double) * (nnz > 0 ? nnz : 1), st));
  }
  k_row_columns<<<grid_for(n * 32, 128), 128, 0, st>>>(n, epe, s.inc_ptr, tmp, s.K.row_ptr, s.K.col);
  EMG_CK(cudaGetLastError());
  EMG_CK(cudaFreeAsync(tmp, st));
  EMG_CK(cudaMallocAsync(&s.rhs, sizeof(double) * (n > 0 ? n : 1), st));
  EMG_CK(cudaMemsetAsync(s.rhs, 0, sizeof(double) * (n > 0 ? n : 1), st));
  EMG_CK(cudaMemsetAsync(s.K.val, 0, sizeof(double) * (nnz > 0 ? nnz : 1), st));
  EMG_CK(cudaFreeAsync(cnt, st));
  EMG_CK(cudaStreamSynchronize(st));
  trace_mark(st, "build.end");
  // M shares the pattern of K
  s.M.n = n;
  s.M.nnz = nnz;
  s.M.row_ptr = s.K.row_ptr;
  s.M.col = s.K.col;
  s.M.owns_pattern = false;
  return EMG_SUCCESS;
}

int system_assemble(System& s, const double* nu, const double* sigma, int32_t n_mat,
                    const emg_source* src, int32_t n_src, int32_t flags, cudaStream_t st) {
  if (n_mat <= 0 || !nu) { set_error("materials list is empty"); return EMG_INVALID_INPUT; }
  if (n_src < 0 || (n_src > 0 && !src) || (!s.src_map && n_src > kMaxSources)) {
    set_error("between 0 and 16 source regions are supported without a per-tet source map");
    return EMG_INVALID_INPUT;
  }
  for (int32_t k = 0; k < n_mat; ++k)
    if (!(nu[k] > 0.0) || (sigma && sigma[k] < 0.0)) {
      // MaterialProperties rejects mu <= 0 and sigma < 0
      set_error("material " + std::to_string(k) + ": nu must be > 0 and sigma >= 0");
      return EMG_INVALID_INPUT;
    }
  const bool mass = (flags & EMG_FLAG_MASS) != 0;
  if (mass && !s.M.val) EMG_CK(cudaMallocAsync(&s.M.val, sizeof(double) * (s.K.nnz > 0 ? s.K.nnz : 1), st));
  s.has_mass = s.has_mass || mass;
  double* mat = nullptr;
  EMG_CK(cudaMallocAsync(&mat, sizeof(double) * 2 * n_mat, st));
  std::vector<double> h(2 * n_mat, 0.0);
  for (int32_t k = 0; k < n_mat; ++k) { h[k] = nu[k]; h[n_mat + k] = sigma ? sigma[k] : 0.0; }
  EMG_CK(cudaMemcpyAsync(mat, h.data(), sizeof(double) * 2 * n_mat, cudaMemcpyHostToDevice, st));
  emg_source* src_tab = nullptr;
  if (n_src > 0 && !s.src_map)
    EMG_CK(cudaMemcpyToSymbolAsync(c_src, src, sizeof(emg_source) * n_src, 0,
                                   cudaMemcpyHostToDevice, st));
  if (n_src > 0 && s.src_map) {
    EMG_CK(cudaMallocAsync(&src_tab, sizeof(emg_source) * n_src, st));
    EMG_CK(cudaMemcpyAsync(src_tab, src, sizeof(emg_source) * n_src, cudaMemcpyHostToDevice, st));
  }
  EMG_CK(cudaMemsetAsync(s.err, 0, sizeof(int32_t), st));
  AsmArgs a;
  a.n = s.n; a.n_nodes = s.n_nodes;
  a.row_ptr = s.K.row_ptr; a.col = s.K.col; a.inc_ptr = s.inc_ptr; a.inc = s.inc;
  a.elems = s.elems; a.xyz = s.xyz; a.material = s.material; a.l2g = s.l2g;
  a.nu = mat; a.sigma = mat + n_mat; a.n_mat = n_mat; a.n_src = n_src; a.flags = flags;
  a.src_tab = src_tab; a.src_map = s.src_map;
  a.kval = s.K.val; a.mval = mass ? s.M.val : nullptr; a.rhs = s.rhs; a.err = s.err;
  if (s.elem_type == EMG_ELEM_HEX8_EDGE && mass)
    k_assemble_rows_hex<true><<<grid_for(s.n, 128, 148 * 32), 128, 0, st>>>(a);
  else if (s.elem_type == EMG_ELEM_HEX8_EDGE)
    k_assemble_rows_hex<false><<<grid_for(s.n, 128, 148 * 32), 128, 0, st>>>(a);
  else
    k_assemble_rows<<<grid_for(s.n, 128, 148 * 32), 128, 0, st>>>(a);
  EMG_CK(cudaGetLastError());
  ++s.K.version;
  if (mass) ++s.M.version;
  int32_t herr = 0;
  EMG_CK(cudaMemcpyAsync(&herr, s.err, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  EMG_CK(cudaFreeAsync(mat, st));
  if (src_tab) EMG_CK(cudaFreeAsync(src_tab, st));
  EMG_CK(cudaStreamSynchronize(st));
  if (herr) { set_error("assembly:" + err_text(herr)); return EMG_INVALID_INPUT; }
  return EMG_SUCCESS;
}

// Buffers of a System come from the stream-ordered pool (cudaMallocAsync);
// the owner synchronizes the device before destruction.
System::~System() {
  for (void* p : {static_cast<void*>(xyz), static_cast<void*>(elems), static_cast<void*>(material),
                  static_cast<void*>(l2g), static_cast<void*>(inc_ptr), static_cast<void*>(inc),
                  static_cast<void*>(err), static_cast<void*>(rhs), static_cast<void*>(src_map)})
    if (p) cudaFreeAsync(p, 0);
}

namespace {
__global__ void k_check_csr(int64_t n, const int32_t* __restrict__ rp, const int32_t* __restrict__ col,
                            int64_t nnz, int32_t* __restrict__ bad) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t a = rp[i], b = rp[i + 1];
    if (a < 0 || b < a || b > nnz || (i == 0 && a != 0) || (i == n - 1 && b != nnz)) {
      atomicOr(bad, 1);
      continue;
    }
    for (int32_t k = a; k < b; ++k) {
      const int32_t c = col[k];
      if (c < 0 || c >= n || (k > a && col[k - 1] >= c)) { atomicOr(bad, 2); break; }
    }
  }
}
}  // namespace

int check_csr(int64_t n, const int32_t* rp, const int32_t* col, int64_t nnz, cudaStream_t st) {
  int32_t* bad = nullptr;
  EMG_CK(cudaMallocAsync(&bad, sizeof(int32_t), st));
  EMG_CK(cudaMemsetAsync(bad, 0, sizeof(int32_t), st));
  k_check_csr<<<grid_for(n, 256), 256, 0, st>>>(n, rp, col, nnz, bad);
  int32_t h = 0;
  EMG_CK(cudaMemcpyAsync(&h, bad, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  EMG_CK(cudaStreamSynchronize(st));
  EMG_CK(cudaFreeAsync(bad, st));
  if (h & 1) { set_error("row_ptr is not a valid offset array"); return EMG_INVALID_INPUT; }
  if (h & 2) { set_error("columns out of range or not strictly ascending in a row"); return EMG_INVALID_INPUT; }
  return EMG_SUCCESS;
}

void trace_pool(const char* where) {
  if (!trace_enabled()) return;
  int dev = 0;
  cudaMemPool_t pool;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess) return;
  uint64_t reserved = 0, used = 0;
  cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
  cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used);
  std::fprintf(stderr, "emg-trace-pool %s %llu %llu\n", where, static_cast<unsigned long long>(reserved),
               static_cast<unsigned long long>(used));
}

void trace_mark(void* stream, const char* label) {
  if (!trace_enabled()) return;
  static thread_local std::chrono::steady_clock::time_point last = std::chrono::steady_clock::now();
  cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
  const auto now = std::chrono::steady_clock::now();
  std::fprintf(stderr, "emg-trace-mark %s %.3f\n", label,
               std::chrono::duration<double, std::milli>(now - last).count());
  last = now;
}

void keep_pool_memory() {
  // Keep freed stream-ordered memory in the pool instead of returning it to
  // the driver at every synchronization (per-process setting).
  static int done_for = -1;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev == done_for) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  done_for = dev;
}

}  // namespace emg

// assembly.cu -- EMAssembly::assemble on the GPU for TET4_EDGE, HEX8_EDGE,
// PRISM6_EDGE and PYRAMID5_EDGE elements (reference: src/numeric/em_assembly.cpp:144-420 with the intended
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
//   tets: k_tet_terms forms every tet's element terms once (the packed 6x6
//   stiffness and mass blocks, the source vector, signs folded in) and
//   k_rows_gather sums, for each row, the terms of its incident tets in
//   ascending element order at column positions k_slot_positions recorded
//   in the symbolic phase (k_rows_from_terms for rows longer than 64);
//   hexahedra, prisms, pyramids: k_elem_terms runs the quadrature loop once
//   per element (elem_shapes.cuh) and k_rows_from_terms gathers the rows.
//   Every row's values are written once: no atomics, deterministic, and
//   every sum is formed in the same order as an element loop would form it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <vector>

#include "common.cuh"
#include "device.h"
#include "internal.h"
#include "elem_shapes.cuh"
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

// Thread per row (TET4_EDGE): for every incidence slot q of the row, element t,
// the positions of the element's columns l2g[6 t + j] inside the row, as bytes
// pos[8 q + j] (0xFF for a constrained edge or a row longer than 254), byte
// pos[8 q + 6] = 1 when two of them coincide (a DOF map that sends two local
// edges of one tet to one DOF), and the longest row into *max_len.
__global__ void k_slot_positions(int64_t n, const int32_t* __restrict__ inc_ptr, const int32_t* __restrict__ inc,
                                 const int32_t* __restrict__ l2g, const int32_t* __restrict__ row_ptr,
                                 const int32_t* __restrict__ col, uint8_t* __restrict__ pos,
                                 int32_t* __restrict__ max_len) {
  int32_t longest = 0;
  for (int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; r < n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t s0 = row_ptr[r], s1 = row_ptr[r + 1];
    longest = max(longest, s1 - s0);
    for (int32_t q = inc_ptr[r]; q < inc_ptr[r + 1]; ++q) {
      const int64_t t = inc[q] / 6;
      uint8_t b[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) b[j] = 0xFF;
#pragma unroll
      for (int j = 0; j < 6; ++j) {
        const int32_t c = l2g[6 * t + j];
        if (c < 0) continue;
        int32_t lo = s0, hi = s1;
        while (lo < hi) {
          const int32_t mid = (lo + hi) >> 1;
          if (col[mid] < c) lo = mid + 1; else hi = mid;
        }
        if (lo < s1 && col[lo] == c && lo - s0 < 0xFF) b[j] = static_cast<uint8_t>(lo - s0);
      }
      uint8_t dup = 0;
#pragma unroll
      for (int j = 0; j < 6; ++j)
#pragma unroll
        for (int k = j + 1; k < 6; ++k) dup |= (b[j] != 0xFF && b[j] == b[k]) ? 1 : 0;
      b[6] = dup;
      uint2 w;
      w.x = b[0] | (b[1] << 8) | (b[2] << 16) | (static_cast<uint32_t>(b[3]) << 24);
      w.y = b[4] | (b[5] << 8) | (b[6] << 16) | (static_cast<uint32_t>(b[7]) << 24);
      reinterpret_cast<uint2*>(pos)[q] = w;
    }
  }
  longest = __reduce_max_sync(0xffffffffu, longest);
  if ((threadIdx.x & 31) == 0) atomicMax(max_len, longest);
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

// Packed upper triangle of a symmetric 6x6 element matrix: entry (i, j),
// i <= j, at i (11 - i) / 2 + j.
__host__ __device__ constexpr int ke_index(int i, int j) { return i * (11 - i) / 2 + j; }
static_assert(ke_index(0, 5) == 5 && ke_index(1, 1) == 6 && ke_index(2, 2) == 11 && ke_index(4, 5) == 19 &&
                  ke_index(5, 5) == 20,
              "packed 6x6 upper triangle");
constexpr int kKe = 21;
constexpr int kTermTile = 128;  // tets per block pass of k_tet_terms

// Copies a block's staged per-tet terms (cnt tets x width doubles, in shared
// memory) to out[t0 * width ...] with consecutive threads on consecutive
// doubles.
__device__ __forceinline__ void store_staged(const double* stage, double* __restrict__ out, int64_t t0, int cnt,
                                             int width) {
  __syncthreads();
  for (int x = threadIdx.x; x < cnt * width; x += blockDim.x) out[t0 * width + x] = stage[x];
  __syncthreads();
}

// Thread per tet, once per tet, the element loop of em_assembly.cpp:144-420:
//   ke[21 t + (i, j)] = s_i s_j nu |det| wsum curl_i . curl_j
// where curl_k = J curl_ref_k / det is constant per tet, so the quadrature
// sum collapses to the weight sum (1/6 for the Hammer rule, 1/8 for the
// reference's 3-point rule);
//   me[21 t + (i, j)] = s_i s_j sum_q w |det| sigma W_i(x_q) . W_j(x_q)
//   fe[6 t + i]       = s_i sum_q w |det| W_i(x_q) . J_s(x_q)
// (s_k the edge sign).  Tets the element loop skips (material id out of
// range, |det| < 1e-15) get zeros, which leave every sum they join unchanged.
// The terms are staged in shared memory and written coalesced.
// kK selects the stiffness terms, kMass / kSrc the quadrature terms: the two
// groups run as separate launches, which keeps each one's registers low.
template <bool kK, bool kMass, bool kSrc>
__global__ void __launch_bounds__(kTermTile, 4) k_tet_terms(AsmArgs A, int64_t n_tets, double* __restrict__ ke,
                                                            double* __restrict__ me, double* __restrict__ fe) {
  __shared__ double stage[kTermTile * kKe];
  const double qa = 0.13819660112501051517954131656343619;   // (5 - sqrt 5) / 20
  const double qb = 0.58541019662496845446137605030969143;   // (5 + 3 sqrt 5) / 20
  const bool quad3 = (A.flags & EMG_FLAG_QUAD3_LITERAL) != 0;
  const int nq = quad3 ? 3 : 4;
  const double w = 1.0 / 24.0;
  const bool signs = (A.flags & EMG_FLAG_NO_EDGE_SIGNS) == 0;
  const bool literal = (A.flags & EMG_FLAG_PIOLA_LITERAL) != 0;
  for (int64_t t0 = static_cast<int64_t>(blockIdx.x) * kTermTile; t0 < n_tets;
       t0 += static_cast<int64_t>(gridDim.x) * kTermTile) {
    const int cnt = static_cast<int>(n_tets - t0 < kTermTile ? n_tets - t0 : kTermTile);
    const int64_t t = t0 + threadIdx.x;
    const int32_t mid = t < n_tets ? (A.material ? A.material[t] : 0) : -1;
    Tet T;
    bool use = mid >= 0 && mid < A.n_mat;  // em_assembly.cpp:270-276 skips the element
    if (use && !load_tet(A.elems, A.xyz, A.n_nodes, t, T)) {
      atomicOr(A.err, kErrNode);
      use = false;
    }
    use = use && !(fabs(T.det) < 1e-15);  // every quadrature point skipped (:169)
    double sg[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) sg[k] = (!use || !signs || T.node[ned_b(k)] < T.node[ned_a(k)]) ? 1.0 : -1.0;
    const double adet = use ? fabs(T.det) : 0.0;
    if (kK) {
      const double kf = use ? nq * w * adet * A.nu[mid] : 0.0;
      double* st = stage + threadIdx.x * kKe;
#pragma unroll
      for (int i = 0; i < 6; ++i) {
#pragma unroll
        for (int j = i; j < 6; ++j) {
          const double d = use ? T.c[i][0] * T.c[j][0] + T.c[i][1] * T.c[j][1] + T.c[i][2] * T.c[j][2] : 0.0;
          st[ke_index(i, j)] = (sg[i] * sg[j]) * (kf * d);
        }
      }
    }
    double mt[kMass ? kKe : 1], ft[kSrc ? 6 : 1];
#pragma unroll
    for (int e = 0; e < (kMass ? kKe : 1); ++e) mt[e] = 0.0;
#pragma unroll
    for (int e = 0; e < (kSrc ? 6 : 1); ++e) ft[e] = 0.0;
    const double sig = use && A.sigma ? A.sigma[mid] : 0.0;
    const bool do_mass = kMass && sig > 0.0;
    const emg_source* tab = c_src;
    int src_first = 0, src_count = use ? A.n_src : 0;
    if (use && A.src_map) {
      tab = A.src_tab;
      const int32_t sid = A.src_map[t];
      src_first = sid;
      src_count = (sid >= 0 && sid < A.n_src) ? 1 : 0;
    }
    const bool do_src = kSrc && src_count > 0;
    if (do_mass || do_src) {
      for (int qq = 0; qq < nq; ++qq) {
        double lam[4];
        if (qq == 0) { lam[0] = qa; lam[1] = qa; lam[2] = qb; }
        else if (qq == 1) { lam[0] = qa; lam[1] = qb; lam[2] = qa; }
        else if (qq == 2 && !quad3) { lam[0] = qb; lam[1] = qa; lam[2] = qa; }
        else { lam[0] = qa; lam[1] = qa; lam[2] = qa; }
        lam[3] = 1.0 - lam[0] - lam[1] - lam[2];
        double js[3] = {0.0, 0.0, 0.0};
        if (kSrc && do_src) {
          double x[3];
#pragma unroll
          for (int c = 0; c < 3; ++c)
            x[c] = T.x3[c] + lam[0] * T.d[0][c] + lam[1] * T.d[1][c] + lam[2] * T.d[2][c];
          source_at(x, tab, src_first, src_count, js);
        }
        // a point outside every source region adds nothing to F
        if (!(kMass && do_mass) && js[0] == 0.0 && js[1] == 0.0 && js[2] == 0.0) continue;
        double W[6][3];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            W[k][c] = lam[ned_b(k)] * T.g[ned_a(k)][c] - lam[ned_a(k)] * T.g[ned_b(k)][c];
            if (literal) W[k][c] /= T.det;
          }
        }
        if (kMass && do_mass) {
#pragma unroll
          for (int i = 0; i < 6; ++i) {
#pragma unroll
            for (int j = i; j < 6; ++j)
              mt[kMass ? ke_index(i, j) : 0] +=
                  w * adet * sig * (W[i][0] * W[j][0] + W[i][1] * W[j][1] + W[i][2] * W[j][2]);
          }
        }
        if (kSrc && do_src) {
#pragma unroll
          for (int k = 0; k < 6; ++k)
            ft[kSrc ? k : 0] += w * adet * (W[k][0] * js[0] + W[k][1] * js[1] + W[k][2] * js[2]);
        }
      }
    }
    if (kK) store_staged(stage, ke, t0, cnt, kKe);
    if (kMass) {
      double* st = stage + threadIdx.x * kKe;
#pragma unroll
      for (int i = 0; i < 6; ++i) {
#pragma unroll
        for (int j = i; j < 6; ++j) st[ke_index(i, j)] = (sg[i] * sg[j]) * mt[kMass ? ke_index(i, j) : 0];
      }
      store_staged(stage, me, t0, cnt, kKe);
    }
    if (kSrc) {
#pragma unroll
      for (int k = 0; k < 6; ++k) stage[threadIdx.x * 6 + k] = sg[k] * ft[kSrc ? k : 0];
      store_staged(stage, fe, t0, cnt, 6);
    }
  }
}

// Packed upper triangle of a symmetric E x E element matrix: entry (i, j),
// i <= j, at i (2E - 1 - i) / 2 + j.
__host__ __device__ constexpr int packed_index(int e, int i, int j) { return i * (2 * e - 1 - i) / 2 + j; }
static_assert(packed_index(6, 2, 3) == ke_index(2, 3) && packed_index(12, 11, 11) == 77 &&
                  packed_index(9, 8, 8) == 44 && packed_index(8, 0, 7) == 7,
              "packed upper triangle");

// Sixteen lanes per row, lane k owning the row's column col[s0 + k] (longer
// rows in passes of sixteen columns), for elements of kEpe edges.  For every
// incident slot (t, i) of the row, in ascending element order, a lane adds
// the entries (i, j) of element t whose column l2g[kEpe t + j] is its own, in
// ascending j: the order in which the element loop forms every sum.  Each
// value is written once, coalesced, without atomics, and K(r, c) and
// K(c, r) add the same terms in the same order, so K is exactly symmetric.
template <int kEpe, bool kMass, bool kSrc>
__global__ void __launch_bounds__(256, 4) k_rows_from_terms(AsmArgs A, const double* __restrict__ ke,
                                                            const double* __restrict__ me,
                                                            const double* __restrict__ fe) {
  constexpr int kP = kEpe * (kEpe + 1) / 2;
  const int sub = threadIdx.x & 15;
  const unsigned half = (threadIdx.x & 16) ? 0xffff0000u : 0x0000ffffu;
  const int64_t stride = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 4;
  for (int64_t r = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 4; r < A.n; r += stride) {
    const int32_t s0 = A.row_ptr[r], s1 = A.row_ptr[r + 1];
    const int32_t a = A.inc_ptr[r], m = A.inc_ptr[r + 1] - a;
    double f = 0.0;
    for (int32_t cb = s0; cb < s1; cb += 16) {
      const int32_t k = cb + sub;
      const int32_t c = k < s1 ? A.col[k] : -2;  // -2 matches no l2g entry
      double acc = 0.0, accm = 0.0;
      for (int32_t qb = 0; qb < m; qb += 16) {
        const int32_t mine = qb + sub < m ? A.inc[a + qb + sub] : 0;
        const int nu = min(16, m - qb);
        for (int u = 0; u < nu; ++u) {
          const int32_t slot = __shfl_sync(half, mine, u, 16);
          const int32_t t = slot / kEpe;
          const int i = slot - kEpe * t;
          const int32_t* lg = A.l2g + static_cast<int64_t>(kEpe) * t;
          unsigned hit = 0;
#pragma unroll
          for (int j = 0; j < kEpe; ++j) hit |= (lg[j] == c ? 1u : 0u) << j;
          const int64_t base = static_cast<int64_t>(kP) * t;
          while (hit) {
            const int j = __ffs(hit) - 1;
            hit &= hit - 1;
            const int e = i <= j ? packed_index(kEpe, i, j) : packed_index(kEpe, j, i);
            acc += ke[base + e];
            if (kMass) accm += me[base + e];
          }
          if (kSrc && cb == s0) f += fe[static_cast<int64_t>(kEpe) * t + i];
        }
      }
      if (k < s1) {
        A.kval[k] = acc;
        if (kMass) A.mval[k] = accm;
      }
    }
    if (sub == 0) A.rhs[r] = f;
  }
}

constexpr int kGatherRows = 5;  // rows per warp, six lanes (local columns j) each
constexpr int kGatherCap = 64;  // longest row k_rows_gather takes

// Five rows per warp, lane (rho, j) handling local column j of row r0 + rho.
// Step q visits the q-th incident slot (t, i) of every row at once (slots
// ascend in element order): the lane adds the tet's entry (i, j) into the
// row's accumulator at the column position the symbolic phase recorded,
// pos[8 q + j].  Within a step the six columns of one tet are distinct, so
// lanes never collide (a DOF map that sends two local edges of one tet to
// the same column is detected and handled one lane at a time); across steps
// each position receives its terms in ascending element order, the order of
// the element loop.  Rows are then written once from shared memory.
template <bool kMass, bool kSrc>
__global__ void __launch_bounds__(256) k_rows_gather(AsmArgs A, const uint8_t* __restrict__ pos,
                                                     const double* __restrict__ ke, const double* __restrict__ me,
                                                     const double* __restrict__ fe) {
  // rows kGatherCap + 1 doubles apart: the rows of a warp start in different banks
  constexpr int kStride = kGatherCap + 1;
  __shared__ double acc_k[8][kGatherRows * kStride];
  __shared__ double acc_m[kMass ? 8 : 1][kMass ? kGatherRows * kStride : 1];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int rho = lane / 6, j = lane - 6 * rho;  // rho == 5: lanes 30, 31 idle
  double* rk = acc_k[wib] + (rho < kGatherRows ? rho : 0) * kStride;
  double* rm = kMass ? acc_m[kMass ? wib : 0] + (rho < kGatherRows ? rho : 0) * kStride : nullptr;
  const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  for (int64_t r0 = (static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + wib) * kGatherRows; r0 < A.n;
       r0 += warps * kGatherRows) {
    const int64_t r = r0 + rho;
    const bool live = rho < kGatherRows && r < A.n;
    int32_t s0 = 0, len = 0, a = 0, m = 0;
    if (live) {
      s0 = A.row_ptr[r];
      len = A.row_ptr[r + 1] - s0;
      a = A.inc_ptr[r];
      m = A.inc_ptr[r + 1] - a;
      for (int k = j; k < len; k += 6) {
        rk[k] = 0.0;
        if (kMass) rm[k] = 0.0;
      }
    }
    const int steps = __reduce_max_sync(0xffffffffu, m);
    __syncwarp();
    double f = 0.0;
    const int src0 = (rho < kGatherRows ? rho : 0) * 6;
    for (int q0 = 0; q0 < steps; q0 += 12) {
      // the row's next twelve incidence slots, two per lane of its group
      const int32_t lo = live && q0 + j < m ? A.inc[a + q0 + j] : 0;
      const int32_t hi = live && q0 + 6 + j < m ? A.inc[a + q0 + 6 + j] : 0;
      const int nq = min(12, steps - q0);
      for (int u = 0; u < nq; ++u) {
        const int q = q0 + u;
        const int32_t slot = __shfl_sync(0xffffffffu, u < 6 ? lo : hi, src0 + (u < 6 ? u : u - 6));
        const bool act = live && q < m;
        const int64_t t = slot / 6;
        const int i = slot - 6 * static_cast<int>(t);
        const uint8_t* pq = pos + 8 * static_cast<int64_t>(a + q);
        const int p = act ? pq[j] : 0xFF;
        const bool clash = __any_sync(0xffffffffu, act && j == 0 && pq[6] != 0);
        const bool add = p != 0xFF;
        const int e = i <= j ? ke_index(i, j) : ke_index(j, i);
        double vk = 0.0, vm = 0.0;
        if (add) {
          vk = ke[kKe * t + e];
          if (kMass) vm = me[kKe * t + e];
        }
        if (kSrc && act && j == 0) f += fe[6 * t + i];
        if (!clash) {
          if (add) {
            rk[p] += vk;
            if (kMass) rm[p] += vm;
          }
        } else {  // two local edges of one tet on one column: add one lane at a time, ascending j
          for (int jj = 0; jj < 6; ++jj) {
            if (add && j == jj) {
              rk[p] += vk;
              if (kMass) rm[p] += vm;
            }
            __syncwarp();
          }
        }
        __syncwarp();
      }
    }
    if (live) {
      for (int k = j; k < len; k += 6) {
        A.kval[s0 + k] = rk[k];
        if (kMass) A.mval[s0 + k] = rm[k];
      }
      if (j == 0) A.rhs[r] = f;
    }
    __syncwarp();
  }
}

template <bool kMass, bool kSrc>
void launch_tet_assembly(const AsmArgs& a, int64_t n_tets, const uint8_t* slot_pos, int32_t max_row_len,
                         double* ke, double* me, double* fe, cudaStream_t st) {
  const int64_t tiles = (n_tets + kTermTile - 1) / kTermTile;
  const unsigned gt = static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(tiles, 148 * 16)));
  k_tet_terms<true, false, false><<<gt, kTermTile, 0, st>>>(a, n_tets, ke, me, fe);
  if (kMass || kSrc) k_tet_terms<false, kMass, kSrc><<<gt, kTermTile, 0, st>>>(a, n_tets, ke, me, fe);
  if (slot_pos && max_row_len <= kGatherCap) {
    const int64_t rb = (a.n + 8 * kGatherRows - 1) / (8 * kGatherRows);  // 8 warps of 5 rows per block
    const unsigned gr = static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(rb, 148 * 64)));
    k_rows_gather<kMass, kSrc><<<gr, 256, 0, st>>>(a, slot_pos, ke, me, fe);
  } else {  // rows longer than the gather kernel's shared-memory rows
    const int64_t rb = (a.n * 16 + 255) / 256;
    const unsigned gr = static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(rb, 148 * 64)));
    k_rows_from_terms<6, kMass, kSrc><<<gr, 256, 0, st>>>(a, ke, me, fe);
  }
}

// ------------------------------------------ HEX8 / PRISM6 / PYRAMID5 ----
constexpr int kElemTile = 64;  // elements per block pass of k_elem_terms

// Thread per element of shape S (elem_shapes.cuh), once per element, the
// quadrature loop of MagneticVector3DIntegrator (computeStiffnessMatrix /
// computeMassMatrix / computeSourceVector, magnetic_vector_3d_integrator.cpp:
// 139-364) with curl_phys = J curl_ref / det J and W_phys = J^-T W_ref
// (divided by det J once more under EMG_FLAG_PIOLA_LITERAL):
//   kK:    ke[P t + (i, j)] = s_i s_j sum_q w_q |det J| nu curl_i . curl_j
//   kMass: me[P t + (i, j)] = s_i s_j sum_q w_q |det J| sigma W_i . W_j
//   kSrc:  fe[E t + i]      = s_i sum_q w_q |det J| W_i . J_s(x_q)
// (P = E (E + 1) / 2 packed upper-triangle entries, s_k the edge sign;
// quadrature points with |det J| < 1e-15 are skipped, elements with a
// material id out of range get zeros).  The stiffness and the quadrature
// terms run as separate launches; the packed sums accumulate in shared
// memory, entry-major so that a warp's lanes touch consecutive words, and are
// written coalesced.
//
// kMixed: a mixed mesh (rows of 9 ints, the type in slot 8): the launch
// integrates the rows of type S only, writes them in the 12-edge layout
// (packed_index(12, i, j), 78 entries; F 12) that one gather reads for every
// type, and scales the hexahedron's terms to its unit-circulation basis (1/4
// of the reference's edge functions: K, M by 1/16, F by 1/4).
template <class S, bool kK, bool kMass, bool kSrc, bool kMixed>
__global__ void __launch_bounds__(kElemTile) k_elem_terms(AsmArgs A, int64_t n_el, double* __restrict__ ke,
                                                          double* __restrict__ me, double* __restrict__ fe) {
  constexpr int E = S::kEdges, N = S::kNodes, P = E * (E + 1) / 2;
  constexpr int kRow = kMixed ? 9 : N;                 // ints per element row
  constexpr int kEOut = kMixed ? 12 : E, kPOut = kEOut * (kEOut + 1) / 2;
  constexpr double kScale = (kMixed && S::kType == 1) ? 0.25 : 1.0;
  constexpr int W = (kK || kMass) ? P : E;  // entries staged per element
  __shared__ double acc[W * kElemTile];
  __shared__ bool mine[kElemTile];
  const bool signs = (A.flags & EMG_FLAG_NO_EDGE_SIGNS) == 0;
  const bool literal = (A.flags & EMG_FLAG_PIOLA_LITERAL) != 0;
  const int tid = threadIdx.x;
  for (int64_t t0 = static_cast<int64_t>(blockIdx.x) * kElemTile; t0 < n_el;
       t0 += static_cast<int64_t>(gridDim.x) * kElemTile) {
    const int cnt = static_cast<int>(n_el - t0 < kElemTile ? n_el - t0 : kElemTile);
    const int64_t t = t0 + tid;
#pragma unroll 1
    for (int e = 0; e < W; ++e) acc[e * kElemTile + tid] = 0.0;
    double ft[kSrc ? E : 1];
#pragma unroll
    for (int k = 0; k < (kSrc ? E : 1); ++k) ft[k] = 0.0;
    bool is_mine = t < n_el;
    if (kMixed && is_mine) {
      const int32_t rt = A.elems[static_cast<int64_t>(kRow) * t + 8];
      is_mine = rt == S::kType;
      // the TET4 launch (the first) flags rows of no known type
      if (S::kType == 0 && (rt < 0 || rt > 3)) atomicOr(A.err, kErrNode);
    }
    mine[tid] = is_mine;
    const int32_t mid = is_mine ? (A.material ? A.material[t] : 0) : -1;
    bool use = mid >= 0 && mid < A.n_mat;  // em_assembly.cpp:270-276 skips the element
    int32_t node[N];
    double X[N][3];
    if (use) {
#pragma unroll
      for (int a = 0; a < N; ++a) {
        node[a] = A.elems[static_cast<int64_t>(kRow) * t + a];
        if (node[a] < 0 || node[a] >= A.n_nodes) use = false;
      }
      if (!use) atomicOr(A.err, kErrNode);
    }
    if (use) {
#pragma unroll
      for (int a = 0; a < N; ++a)
#pragma unroll
        for (int r = 0; r < 3; ++r) X[a][r] = A.xyz[3 * static_cast<int64_t>(node[a]) + r];
    }
    const double nu = use ? A.nu[mid] : 0.0;
    const double sig = use && A.sigma ? A.sigma[mid] : 0.0;
    const emg_source* tab = c_src;
    int src_first = 0, src_count = use ? A.n_src : 0;
    if (use && A.src_map) {
      tab = A.src_tab;
      const int32_t sid = A.src_map[t];
      src_first = sid;
      src_count = (sid >= 0 && sid < A.n_src) ? 1 : 0;
    }
    const bool run = use && (kK || (kMass && sig > 0.0) || (kSrc && src_count > 0));
    if (run) {
#pragma unroll 1
      for (int q = 0; q < S::kPoints; ++q) {
        double x[3], wq, J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        S::point(q, x, &wq);
#pragma unroll
        for (int a = 0; a < N; ++a) {
          double d[3];
          S::dn(a, x, d);
#pragma unroll
          for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) J[r][c] += X[a][r] * d[c];
        }
        const double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                           J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                           J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
        const double adet = fabs(det);
        if (adet < 1e-15) continue;  // magnetic_vector_3d_integrator.cpp:169-176
        if (kK) {
          double c[E][3];
#pragma unroll
          for (int k = 0; k < E; ++k) {
            double cr[3];
            S::curl(k, x, cr);
#pragma unroll
            for (int r = 0; r < 3; ++r) c[k][r] = (J[r][0] * cr[0] + J[r][1] * cr[1] + J[r][2] * cr[2]) / det;
          }
          const double wk = wq * adet * nu;
          int e = 0;
#pragma unroll
          for (int i = 0; i < E; ++i)
#pragma unroll
            for (int j = i; j < E; ++j, ++e)
              acc[e * kElemTile + tid] += wk * (c[i][0] * c[j][0] + c[i][1] * c[j][1] + c[i][2] * c[j][2]);
        } else {
          double inv[3][3];
          inv[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
          inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
          inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
          inv[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / det;
          inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
          inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
          inv[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
          inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
          inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
          double Wp[E][3];
#pragma unroll
          for (int k = 0; k < E; ++k) {
            double wr[3];
            S::basis(k, x, wr);
#pragma unroll
            for (int r = 0; r < 3; ++r) {
              Wp[k][r] = inv[0][r] * wr[0] + inv[1][r] * wr[1] + inv[2][r] * wr[2];
              if (literal) Wp[k][r] /= det;
            }
          }
          if (kMass && sig > 0.0) {
            const double wm = wq * adet * sig;
            int e = 0;
#pragma unroll
            for (int i = 0; i < E; ++i)
#pragma unroll
              for (int j = i; j < E; ++j, ++e)
                acc[e * kElemTile + tid] += wm * (Wp[i][0] * Wp[j][0] + Wp[i][1] * Wp[j][1] + Wp[i][2] * Wp[j][2]);
          }
          if (kSrc && src_count > 0) {
            double p[3] = {0.0, 0.0, 0.0}, js[3];
#pragma unroll
            for (int a = 0; a < N; ++a) {
              const double na = S::n(a, x);
#pragma unroll
              for (int r = 0; r < 3; ++r) p[r] += na * X[a][r];
            }
            source_at(p, tab, src_first, src_count, js);
#pragma unroll
            for (int k = 0; k < (kSrc ? E : 1); ++k)
              ft[k] += wq * adet * (Wp[k][0] * js[0] + Wp[k][1] * js[1] + Wp[k][2] * js[2]);
          }
        }
      }
    }
    double sg[E];
#pragma unroll
    for (int k = 0; k < E; ++k) sg[k] = (!use || !signs || node[S::edge_a(k)] < node[S::edge_b(k)]) ? 1.0 : -1.0;
    if (kK || kMass) {
      int e = 0;
#pragma unroll
      for (int i = 0; i < E; ++i)
#pragma unroll
        for (int j = i; j < E; ++j, ++e) acc[e * kElemTile + tid] *= (kScale * kScale) * (sg[i] * sg[j]);
      __syncthreads();
      double* out = kK ? ke : me;
      if (!kMixed) {
        for (int x = tid; x < cnt * P; x += kElemTile) out[t0 * P + x] = acc[(x % P) * kElemTile + x / P];
      } else {
        for (int x = tid; x < cnt * P; x += kElemTile) {
          const int el = x / P;
          if (!mine[el]) continue;
          int e2 = x - el * P, i = 0;
          while (e2 >= E - i) { e2 -= E - i; ++i; }  // entry e2 of row i of the packed triangle
          out[(t0 + el) * kPOut + packed_index(kEOut, i, i + e2)] = acc[(x - el * P) * kElemTile + el];
        }
      }
      __syncthreads();
    }
    if (kSrc && !kK) {
#pragma unroll
      for (int k = 0; k < (kSrc ? E : 1); ++k) acc[k * kElemTile + tid] = kScale * sg[k] * ft[k];
      __syncthreads();
      for (int x = tid; x < cnt * E; x += kElemTile) {
        const int el = x / E;
        if (kMixed && !mine[el]) continue;
        fe[(t0 + el) * kEOut + (x - el * E)] = acc[(x % E) * kElemTile + el];
      }
      __syncthreads();
    }
  }
}

template <class S, bool kMass, bool kSrc, bool kMixed>
void launch_elem_terms(const AsmArgs& a, int64_t n_el, double* ke, double* me, double* fe, cudaStream_t st) {
  const int64_t tiles = (n_el + kElemTile - 1) / kElemTile;
  const unsigned g = static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(tiles, 148 * 32)));
  k_elem_terms<S, true, false, false, kMixed><<<g, kElemTile, 0, st>>>(a, n_el, ke, me, fe);
  if (kMass || kSrc) k_elem_terms<S, false, kMass, kSrc, kMixed><<<g, kElemTile, 0, st>>>(a, n_el, ke, me, fe);
}

template <int kEpe, bool kMass, bool kSrc>
void launch_rows(const AsmArgs& a, const double* ke, const double* me, const double* fe, cudaStream_t st) {
  const int64_t rb = (a.n * 16 + 255) / 256;
  const unsigned gr = static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(rb, 148 * 64)));
  k_rows_from_terms<kEpe, kMass, kSrc><<<gr, 256, 0, st>>>(a, ke, me, fe);
}

template <class S, bool kMass, bool kSrc>
void launch_elem_assembly(const AsmArgs& a, int64_t n_el, double* ke, double* me, double* fe, cudaStream_t st) {
  launch_elem_terms<S, kMass, kSrc, false>(a, n_el, ke, me, fe, st);
  launch_rows<S::kEdges, kMass, kSrc>(a, ke, me, fe, st);
}

// A mixed mesh: one terms launch per element type, one 12-edge gather.
template <bool kMass, bool kSrc>
void launch_mixed_assembly(const AsmArgs& a, int64_t n_el, double* ke, double* me, double* fe, cudaStream_t st) {
  launch_elem_terms<shape::Tet, kMass, kSrc, true>(a, n_el, ke, me, fe, st);
  launch_elem_terms<shape::Hex, kMass, kSrc, true>(a, n_el, ke, me, fe, st);
  launch_elem_terms<shape::Prism, kMass, kSrc, true>(a, n_el, ke, me, fe, st);
  launch_elem_terms<shape::Pyramid, kMass, kSrc, true>(a, n_el, ke, me, fe, st);
  launch_rows<12, kMass, kSrc>(a, ke, me, fe, st);
}

template <class S>
void launch_elem_assembly(const AsmArgs& a, int64_t n_el, bool mass, bool srcs, double* ke, double* me, double* fe,
                          cudaStream_t st) {
  if (mass && srcs) launch_elem_assembly<S, true, true>(a, n_el, ke, me, fe, st);
  else if (mass) launch_elem_assembly<S, true, false>(a, n_el, ke, me, fe, st);
  else if (srcs) launch_elem_assembly<S, false, true>(a, n_el, ke, me, fe, st);
  else launch_elem_assembly<S, false, false>(a, n_el, ke, me, fe, st);
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
  if (epe == 6) {  // TET4_EDGE: column positions of every incidence slot, for the numeric gather
    int32_t* dmax = nullptr;
    EMG_CK(cudaMallocAsync(&dmax, sizeof(int32_t), st));
    EMG_CK(cudaMemsetAsync(dmax, 0, sizeof(int32_t), st));
    EMG_CK(cudaMallocAsync(&s.slot_pos, 8 * std::max<int64_t>(inc_total, 1), st));
    k_slot_positions<<<grid_for(n, 128), 128, 0, st>>>(n, s.inc_ptr, s.inc, s.l2g, s.K.row_ptr, s.K.col,
                                                       s.slot_pos, dmax);
    EMG_CK(cudaGetLastError());
    EMG_CK(cudaMemcpyAsync(&s.max_row_len, dmax, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    EMG_CK(cudaFreeAsync(dmax, st));
  }
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
  if (s.elem_type == EMG_ELEM_MIXED && (flags & EMG_FLAG_QUAD3_LITERAL)) {
    set_error("EMG_FLAG_QUAD3_LITERAL is a TET4_EDGE-mesh flag (a mixed mesh integrates its tets with the 4-point rule)");
    return EMG_INVALID_INPUT;
  }
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
  // per-element terms: packed K and M (P = E (E + 1) / 2 each, M with the
  // mass matrix) and F (E, with sources)
  double* terms = nullptr;
  const bool srcs = n_src > 0;
  if (s.elem_type != EMG_ELEM_TET4_EDGE) {
    const int64_t T = s.n_elems, E = edges_per_elem(s.elem_type), P = E * (E + 1) / 2;
    const int64_t width = P + (mass ? P : 0) + (srcs ? E : 0);
    EMG_CK(cudaMallocAsync(&terms, sizeof(double) * std::max<int64_t>(width * T, 1), st));
    double* ke = terms;
    double* me = mass ? terms + P * T : nullptr;
    double* fe = srcs ? terms + (mass ? 2 * P : P) * T : nullptr;
    if (s.elem_type == EMG_ELEM_HEX8_EDGE) launch_elem_assembly<shape::Hex>(a, T, mass, srcs, ke, me, fe, st);
    else if (s.elem_type == EMG_ELEM_PRISM6_EDGE) launch_elem_assembly<shape::Prism>(a, T, mass, srcs, ke, me, fe, st);
    else if (s.elem_type == EMG_ELEM_PYRAMID5_EDGE) launch_elem_assembly<shape::Pyramid>(a, T, mass, srcs, ke, me, fe, st);
    else if (mass && srcs) launch_mixed_assembly<true, true>(a, T, ke, me, fe, st);
    else if (mass) launch_mixed_assembly<true, false>(a, T, ke, me, fe, st);
    else if (srcs) launch_mixed_assembly<false, true>(a, T, ke, me, fe, st);
    else launch_mixed_assembly<false, false>(a, T, ke, me, fe, st);
  } else {
    if (reinterpret_cast<uintptr_t>(s.l2g) % 8 != 0) {
      cudaFreeAsync(mat, st);
      if (src_tab) cudaFreeAsync(src_tab, st);
      set_error("assembly: the DOF map must be 8-byte aligned");
      return EMG_INVALID_INPUT;
    }
    const int64_t T = s.n_elems;
    const int64_t width = kKe + (mass ? kKe : 0) + (srcs ? 6 : 0);
    EMG_CK(cudaMallocAsync(&terms, sizeof(double) * std::max<int64_t>(width * T, 1), st));
    double* ke = terms;
    double* me = mass ? terms + kKe * T : nullptr;
    double* fe = srcs ? terms + (mass ? 2 * kKe : kKe) * T : nullptr;
    const uint8_t* sp = s.slot_pos;
    const int32_t ml = s.max_row_len;
    if (mass && srcs) launch_tet_assembly<true, true>(a, T, sp, ml, ke, me, fe, st);
    else if (mass) launch_tet_assembly<true, false>(a, T, sp, ml, ke, me, fe, st);
    else if (srcs) launch_tet_assembly<false, true>(a, T, sp, ml, ke, me, fe, st);
    else launch_tet_assembly<false, false>(a, T, sp, ml, ke, me, fe, st);
  }
  EMG_CK(cudaGetLastError());
  if (terms) EMG_CK(cudaFreeAsync(terms, st));
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
                  static_cast<void*>(err), static_cast<void*>(rhs), static_cast<void*>(src_map),
                  static_cast<void*>(slot_pos)})
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

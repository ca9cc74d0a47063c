// numbering_gpu.cu -- the DOF numbering of numbering.cpp on the device, bit for
// bit: global edge IDs by first appearance (GlobalEdgeIDGenerator,
// src/fe_em/global_edge_id_generator.cpp:30-110), the free numbering
// (EMDOFManager, src/fe_em/em_dof_manager.cpp:29-393) and the tree-cotree
// gauge of the `ref` mode (SpanningTreeBuilder::buildBFSTreeWithBoundaryPriority
// and the remaining-component BFS, spanning_tree.cpp:295-598; circulation
// picks, multi_connected_domain.cpp:190-232; TreeGauge, tree_gauge.cpp:37-290;
// renumberVectorDOFsWithTreeGauge, em_dof_manager.cpp:501-626).
//
// Edge IDs: the element-edge slots p = E t + k, keyed (lower node, higher
// node), go through a stable radix sort; the first slot of each key is its
// leader, and the leaders in slot order receive consecutive IDs -- the order
// in which the reference's hash map hands them out.
//
// Tree: the reference's breadth-first search pops a FIFO queue, and for each
// popped node appends its undiscovered neighbours across Dirichlet edges in
// ascending order, then the others in ascending order.  Level by level that
// order is determined: a node of level L + 1 is discovered by the earliest
// (in queue order) node of level L adjacent to it, and within one
// discovering node by its rank in that node's discovery order.  Each level
// is therefore one atomicMin per undiscovered neighbour over the key
// (queue position of the discoverer << 32 | rank), a count of every
// discoverer's wins, a scan of the counts, and a pass in which each
// discoverer places its wins in discovery order -- no sort.  The host reads
// one count per level.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <vector>

#include "device.h"
#include "internal.h"

namespace emg {
namespace {

constexpr int kT = 256;

unsigned grid_of(int64_t work) {
  int64_t b = (work + kT - 1) / kT;
  return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(b, 148 * 32)));
}

#define GTID (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x)
#define GSTRIDE (static_cast<int64_t>(gridDim.x) * blockDim.x)

// Stream-ordered scratch, freed (in stream order) when the arena goes away.
struct Arena {
  cudaStream_t st;
  std::vector<void*> ptrs;
  bool failed = false;
  explicit Arena(cudaStream_t s) : st(s) {}
  template <class T>
  T* get(int64_t n) {
    void* p = nullptr;
    if (cudaMallocAsync(&p, sizeof(T) * static_cast<size_t>(std::max<int64_t>(n, 1)), st) != cudaSuccess) {
      failed = true;
      return nullptr;
    }
    ptrs.push_back(p);
    return static_cast<T*>(p);
  }
  ~Arena() {
    for (void* p : ptrs) cudaFreeAsync(p, st);
  }
};

// Local edge tables of the four element types (row t of a mixed mesh names
// its type in slot 8).
struct EdgeTables {
  int a[4][12], b[4][12], ne[4];
};

// ------------------------------------------------------------ edge IDs ----
// Key of every element-edge slot; slots past an element's own edges get the
// largest key (they sort last and are left out) and count into *valid the
// others.
__global__ void k_edge_keys(int64_t m, int32_t elem_type, int npe, int epe, EdgeTables le,
                            const int32_t* __restrict__ elems, int64_t n_nodes, uint64_t* __restrict__ key,
                            int32_t* __restrict__ slot, int32_t* __restrict__ err, int32_t* __restrict__ valid) {
  int32_t mine = 0;
  for (int64_t p = GTID; p < m; p += GSTRIDE) {
    const int64_t t = p / epe;
    const int k = static_cast<int>(p - t * epe);
    const int32_t et = elem_type == EMG_ELEM_MIXED ? elems[npe * t + 8] : elem_type;
    slot[p] = static_cast<int32_t>(p);
    if (et < 0 || et > 3) {
      atomicOr(err, 1);
      key[p] = ~0ull;
      continue;
    }
    if (k >= le.ne[et]) {
      key[p] = ~0ull;
      continue;
    }
    const int32_t u = elems[npe * t + le.a[et][k]], w = elems[npe * t + le.b[et][k]];
    if (u < 0 || w < 0 || u >= n_nodes || w >= n_nodes) {
      atomicOr(err, 1);
      key[p] = 0;
    } else {
      key[p] = (static_cast<uint64_t>(min(u, w)) << 32) | static_cast<uint32_t>(max(u, w));
    }
    ++mine;
  }
  if (mine) atomicAdd(valid, mine);
}

// head[i] = i where a run of equal keys starts, else 0 (a max-scan then gives
// every entry its run start); leader[slot] = 1 for the first slot of a run.
__global__ void k_runs(int64_t m, const uint64_t* __restrict__ key, const int32_t* __restrict__ slot,
                       int32_t* __restrict__ head, int32_t* __restrict__ leader) {
  for (int64_t i = GTID; i < m; i += GSTRIDE) {
    const bool h = i == 0 || key[i] != key[i - 1];
    head[i] = h ? static_cast<int32_t>(i) : 0;
    leader[slot[i]] = h ? 1 : 0;
  }
}

__global__ void k_edge_ids(int64_t m, const uint64_t* __restrict__ key, const int32_t* __restrict__ slot,
                           const int32_t* __restrict__ run, const int32_t* __restrict__ id_at,
                           int32_t* __restrict__ elem_edge, int32_t* __restrict__ edge_nodes) {
  for (int64_t i = GTID; i < m; i += GSTRIDE) {
    const int32_t id = id_at[slot[run[i]]];
    elem_edge[slot[i]] = id;
    if (run[i] == i) {
      edge_nodes[2 * static_cast<int64_t>(id)] = static_cast<int32_t>(key[i] >> 32);
      edge_nodes[2 * static_cast<int64_t>(id) + 1] = static_cast<int32_t>(key[i] & 0xffffffffu);
    }
  }
}

// markConstrainedDOFs: every Dirichlet pair that is a mesh edge.
__global__ void k_mark_constrained(int64_t n_dir, const int32_t* __restrict__ pairs, int64_t n_nodes,
                                   int64_t m, const uint64_t* __restrict__ key, const int32_t* __restrict__ slot,
                                   const int32_t* __restrict__ elem_edge, int32_t* __restrict__ constrained) {
  for (int64_t d = GTID; d < n_dir; d += GSTRIDE) {
    const int32_t a = pairs[2 * d], b = pairs[2 * d + 1];
    if (a < 0 || b < 0 || a >= n_nodes || b >= n_nodes) continue;
    const uint64_t k = (static_cast<uint64_t>(min(a, b)) << 32) | static_cast<uint32_t>(max(a, b));
    int64_t lo = 0, hi = m;
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (key[mid] < k) lo = mid + 1; else hi = mid;
    }
    if (lo < m && key[lo] == k) constrained[elem_edge[slot[lo]]] = 1;
  }
}

__global__ void k_not(int64_t n, const int32_t* __restrict__ in, int32_t* __restrict__ out) {
  for (int64_t i = GTID; i < n; i += GSTRIDE) out[i] = in[i] ? 0 : 1;
}

// ------------------------------------------------------------ the graph ----
__global__ void k_adj_keys(int64_t n_edges, const int32_t* __restrict__ edge_nodes, uint64_t* __restrict__ key,
                           int32_t* __restrict__ eid, int32_t* __restrict__ deg) {
  for (int64_t e = GTID; e < n_edges; e += GSTRIDE) {
    const uint32_t u = static_cast<uint32_t>(edge_nodes[2 * e]), w = static_cast<uint32_t>(edge_nodes[2 * e + 1]);
    key[2 * e] = (static_cast<uint64_t>(u) << 32) | w;
    key[2 * e + 1] = (static_cast<uint64_t>(w) << 32) | u;
    eid[2 * e] = eid[2 * e + 1] = static_cast<int32_t>(e);
    atomicAdd(&deg[u], 1);
    atomicAdd(&deg[w], 1);
  }
}

__global__ void k_adj_nb(int64_t n2, const uint64_t* __restrict__ key, int32_t* __restrict__ nb) {
  for (int64_t i = GTID; i < n2; i += GSTRIDE) nb[i] = static_cast<int32_t>(key[i] & 0xffffffffu);
}

// Rank of every adjacency entry in its node's discovery order: with
// `priority`, the entries across constrained edges first (ascending), then
// the others; without, ascending.
__global__ void k_ranks(int64_t n_nodes, const int32_t* __restrict__ ptr, const int32_t* __restrict__ eid,
                        const int32_t* __restrict__ constrained, int priority, int32_t* __restrict__ rank) {
  for (int64_t u = GTID; u < n_nodes; u += GSTRIDE) {
    const int32_t a = ptr[u], b = ptr[u + 1];
    int32_t nc = 0;
    if (priority)
      for (int32_t s = a; s < b; ++s) nc += constrained[eid[s]] ? 1 : 0;
    int32_t rc = 0, ru = 0;
    for (int32_t s = a; s < b; ++s)
      rank[s] = (priority && constrained[eid[s]]) ? rc++ : nc + ru++;
  }
}

// ----------------------------------------------------------- tree (BFS) ----
// Discovery order of entry s of node u: rank[s] with the Dirichlet-first
// rule, s - ptr[u] without it (rank == nullptr).
__device__ __forceinline__ int32_t rank_of(const int32_t* rank, const int32_t* ptr, int32_t u, int32_t s) {
  return rank ? rank[s] : s - ptr[u];
}

// One level, the queue positions [p0, p1): every undiscovered neighbour keeps
// the smallest (discoverer position, rank) key.
__global__ void k_bfs_expand(int32_t p0, int32_t p1, const int32_t* __restrict__ queue,
                             const int32_t* __restrict__ ptr, const int32_t* __restrict__ nb,
                             const int32_t* __restrict__ rank, const int32_t* __restrict__ pos,
                             unsigned long long* __restrict__ key) {
  for (int64_t i = p0 + GTID; i < p1; i += GSTRIDE) {
    const int32_t u = queue[i];
    for (int32_t s = ptr[u]; s < ptr[u + 1]; ++s) {
      const int32_t v = nb[s];
      if (pos[v] >= 0) continue;
      atomicMin(&key[v], (static_cast<unsigned long long>(i) << 32) | static_cast<uint32_t>(rank_of(rank, ptr, u, s)));
    }
  }
}

// Wins of every discoverer of the level (neighbours whose kept key is its own).
__global__ void k_bfs_count(int32_t p0, int32_t p1, const int32_t* __restrict__ queue,
                            const int32_t* __restrict__ ptr, const int32_t* __restrict__ nb,
                            const int32_t* __restrict__ rank, const int32_t* __restrict__ pos,
                            const unsigned long long* __restrict__ key, int32_t* __restrict__ cnt) {
  for (int64_t i = p0 + GTID; i < p1; i += GSTRIDE) {
    const int32_t u = queue[i];
    int32_t c = 0;
    for (int32_t s = ptr[u]; s < ptr[u + 1]; ++s) {
      const int32_t v = nb[s];
      c += (pos[v] < 0 && key[v] == ((static_cast<unsigned long long>(i) << 32) |
                                     static_cast<uint32_t>(rank_of(rank, ptr, u, s))))
               ? 1 : 0;
    }
    cnt[i - p0] = c;
  }
}

// Every discoverer appends its wins at its offset, in its discovery order
// (with the Dirichlet-first rule: entries across constrained edges, then the
// others), and marks the edges it discovered them through as tree edges.
__global__ void k_bfs_place(int32_t p0, int32_t p1, int32_t* __restrict__ queue, const int32_t* __restrict__ ptr,
                            const int32_t* __restrict__ nb, const int32_t* __restrict__ eid,
                            const int32_t* __restrict__ rank, const int32_t* __restrict__ constrained,
                            int32_t* __restrict__ pos, const unsigned long long* __restrict__ key,
                            const int32_t* __restrict__ off, int32_t* __restrict__ tree) {
  for (int64_t i = p0 + GTID; i < p1; i += GSTRIDE) {
    const int32_t u = queue[i];
    int32_t j = p1 + off[i - p0];
    for (int pass = 0; pass < (rank ? 2 : 1); ++pass) {
      for (int32_t s = ptr[u]; s < ptr[u + 1]; ++s) {
        if (rank && (constrained[eid[s]] != 0) != (pass == 0)) continue;
        const int32_t v = nb[s];
        if (pos[v] >= 0) continue;
        if (key[v] != ((static_cast<unsigned long long>(i) << 32) | static_cast<uint32_t>(rank_of(rank, ptr, u, s))))
          continue;
        queue[j] = v;
        pos[v] = j;
        tree[eid[s]] = 1;
        ++j;
      }
    }
  }
}

// Smallest index i < n with flag-test true, into *out (initialised to n).
__global__ void k_first_constrained(int64_t n, const int32_t* __restrict__ constrained, int32_t* __restrict__ out) {
  int32_t best = INT32_MAX;
  for (int64_t e = GTID; e < n; e += GSTRIDE)
    if (constrained[e]) { best = static_cast<int32_t>(e); break; }
  if (best != INT32_MAX) atomicMin(out, best);
}
__global__ void k_first_unseen(int64_t n, const int32_t* __restrict__ deg, const int32_t* __restrict__ pos,
                               int32_t* __restrict__ out) {
  int32_t best = INT32_MAX;
  for (int64_t v = GTID; v < n; v += GSTRIDE)
    if (deg[v] > 0 && pos[v] < 0) { best = static_cast<int32_t>(v); break; }
  if (best != INT32_MAX) atomicMin(out, best);
}
__global__ void k_seed(int32_t v, int32_t at, int32_t* __restrict__ queue, int32_t* __restrict__ pos) {
  queue[at] = v;
  pos[v] = at;
}

// --------------------------------------------------------- the DOF map ----
// flags of the reduced numbering: kept = not tree, not constrained, not a
// circulation pick; circ = a pick (cotree rank in picks[0..n_picks)).
__global__ void k_reduced_flags(int64_t n, const int32_t* __restrict__ tree, const int32_t* __restrict__ constrained,
                                const int32_t* __restrict__ cot_rank, const int32_t* __restrict__ picks,
                                int32_t n_picks, int32_t* __restrict__ kept, int32_t* __restrict__ circ) {
  for (int64_t e = GTID; e < n; e += GSTRIDE) {
    bool c = false;
    if (!tree[e])
      for (int32_t i = 0; i < n_picks; ++i) c |= cot_rank[e] == picks[i];
    circ[e] = c ? 1 : 0;
    kept[e] = (!tree[e] && !constrained[e] && !c) ? 1 : 0;
  }
}

__global__ void k_edge_dof(int64_t n, const int32_t* __restrict__ constrained, const int32_t* __restrict__ kept,
                           const int32_t* __restrict__ kept_rank, const int32_t* __restrict__ circ,
                           const int32_t* __restrict__ circ_rank, int32_t n_kept, int32_t* __restrict__ edge_dof) {
  for (int64_t e = GTID; e < n; e += GSTRIDE)
    edge_dof[e] = constrained[e] ? -1 : kept[e] ? kept_rank[e] : circ[e] ? n_kept + circ_rank[e] : -1;
}

__global__ void k_free_dof(int64_t n, const int32_t* __restrict__ constrained, const int32_t* __restrict__ free_rank,
                           int32_t* __restrict__ edge_dof) {
  for (int64_t e = GTID; e < n; e += GSTRIDE) edge_dof[e] = constrained[e] ? -1 : free_rank[e];
}

__global__ void k_l2g(int64_t m, const int32_t* __restrict__ elem_edge, const int32_t* __restrict__ edge_dof,
                      int32_t* __restrict__ l2g) {
  for (int64_t p = GTID; p < m; p += GSTRIDE) l2g[p] = elem_edge[p] < 0 ? -1 : edge_dof[elem_edge[p]];
}

struct MaxOp {
  __host__ __device__ int32_t operator()(int32_t a, int32_t b) const { return a > b ? a : b; }
};

}  // namespace

// Device DOF numbering of a mesh of one element type; elems (nodes_per_elem *
// n_elems) and dir_pairs (2 * n_dir) are device arrays, l2g_out a device
// array of edges_per_elem * n_elems.  gauge: EMG_GAUGE_NONE or EMG_GAUGE_REF.
int dof_build_gpu(int32_t elem_type, int64_t n_nodes, int64_t n_elems, const int32_t* elems, int64_t n_dir,
                  const int32_t* dir_pairs, int32_t n_hole_markers, int32_t gauge, int32_t* l2g_out,
                  int64_t* n_edges_out, int64_t* n_free_out, int64_t* n_dofs_out, cudaStream_t st) {
  if (!valid_elem_type(elem_type) || n_nodes < 0 || n_elems < 0 || n_dir < 0 || n_hole_markers < 0 ||
      (n_elems > 0 && (!elems || !l2g_out)) || (n_dir > 0 && !dir_pairs)) {
    set_error("emg_dof_build_device: invalid arguments");
    return EMG_INVALID_INPUT;
  }
  if (gauge != EMG_GAUGE_NONE && gauge != EMG_GAUGE_REF) {
    set_error("emg_dof_build_device: gauge must be EMG_GAUGE_NONE or EMG_GAUGE_REF (EMG_GAUGE_BOUNDARY_FIRST: emg_dof_build)");
    return EMG_INVALID_INPUT;
  }
  const int npe = nodes_per_elem(elem_type), epe = edges_per_elem(elem_type);
  const int64_t m = epe * n_elems;
  if (m >= (int64_t(1) << 31) - 1 || n_nodes >= (int64_t(1) << 31) - 1) {
    set_error("emg_dof_build_device: more than 2^31 element edges or nodes");
    return EMG_INVALID_INPUT;
  }
  EdgeTables le{};
  for (int32_t et = 0; et < 4; ++et) {
    const int (*tab)[2] = local_edges(et);
    le.ne[et] = edges_per_elem(et);
    for (int k = 0; k < le.ne[et]; ++k) { le.a[et][k] = tab[k][0]; le.b[et][k] = tab[k][1]; }
  }
  Arena A(st);
  int32_t* err = A.get<int32_t>(2);  // error flag, valid slot count
  uint64_t* key = A.get<uint64_t>(m);
  uint64_t* key_s = A.get<uint64_t>(m);
  int32_t* slot = A.get<int32_t>(m);
  int32_t* slot_s = A.get<int32_t>(m);
  int32_t* head = A.get<int32_t>(m);
  int32_t* run = A.get<int32_t>(m);
  int32_t* leader = A.get<int32_t>(m);
  int32_t* id_at = A.get<int32_t>(m);
  int32_t* elem_edge = A.get<int32_t>(m);
  if (A.failed) { set_error("emg_dof_build_device: out of device memory"); return EMG_ERR_NOMEM; }
  const int mi = static_cast<int>(m);
  int bits = 1;
  while ((int64_t(1) << bits) < std::max<int64_t>(n_nodes, 2)) ++bits;
  size_t tb = 0, tb2 = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tb, key, key_s, slot, slot_s, mi, 0, 32 + bits, st);
  cub::DeviceScan::InclusiveScan(nullptr, tb2, head, run, MaxOp(), mi, st);
  tb = std::max(tb, tb2);
  cub::DeviceScan::ExclusiveSum(nullptr, tb2, leader, id_at, mi, st);
  tb = std::max(tb, tb2);
  const int64_t ne_cap = m + 2;  // edges never exceed the slots
  // scans over edges and nodes use the same temporary storage
  cub::DeviceScan::ExclusiveSum(nullptr, tb2, leader, id_at, static_cast<int>(std::max<int64_t>(ne_cap, n_nodes + 1)), st);
  tb = std::max(tb, tb2);
  cub::DeviceRadixSort::SortPairs(nullptr, tb2, key, key_s, slot, slot_s, static_cast<int>(2 * m), 0, 32 + bits, st);
  tb = std::max(tb, tb2);
  void* tmp = A.get<char>(static_cast<int64_t>(tb));
  if (A.failed) { set_error("emg_dof_build_device: out of device memory"); return EMG_ERR_NOMEM; }
  EMG_CK(cudaMemsetAsync(err, 0, 2 * sizeof(int32_t), st));
  k_edge_keys<<<grid_of(m), kT, 0, st>>>(m, elem_type, npe, epe, le, elems, n_nodes, key, slot, err, err + 1);
  // slots past an element's edges carry the largest key: all 64 bits sorted
  EMG_CK(cub::DeviceRadixSort::SortPairs(tmp, tb, key, key_s, slot, slot_s, mi, 0,
                                         elem_type == EMG_ELEM_MIXED ? 64 : 32 + bits, st));
  int32_t h[4] = {0, 0, 0, 0};  // error flag, valid slots, last id_at, last leader flag
  EMG_CK(cudaMemcpyAsync(h, err, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  EMG_CK(cudaStreamSynchronize(st));
  if (h[0]) {
    set_error("emg_dof_build_device: element node index outside [0, n_nodes) or unknown element type");
    return EMG_INVALID_INPUT;
  }
  const int64_t mv = h[1];  // sorted entries [0, mv) are element edges
  EMG_CK(cudaMemsetAsync(leader, 0, sizeof(int32_t) * std::max<int64_t>(m, 1), st));
  k_runs<<<grid_of(mv), kT, 0, st>>>(mv, key_s, slot_s, head, leader);
  EMG_CK(cub::DeviceScan::InclusiveScan(tmp, tb, head, run, MaxOp(), static_cast<int>(mv), st));
  EMG_CK(cub::DeviceScan::ExclusiveSum(tmp, tb, leader, id_at, mi, st));
  if (m > 0) {
    EMG_CK(cudaMemcpyAsync(&h[2], id_at + m - 1, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    EMG_CK(cudaMemcpyAsync(&h[3], leader + m - 1, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  }
  EMG_CK(cudaStreamSynchronize(st));
  const int64_t E = m > 0 ? static_cast<int64_t>(h[2]) + h[3] : 0;
  int32_t* edge_nodes = A.get<int32_t>(2 * E);
  int32_t* constrained = A.get<int32_t>(E);
  int32_t* ones = A.get<int32_t>(E);
  int32_t* free_rank = A.get<int32_t>(E + 1);
  int32_t* edge_dof = A.get<int32_t>(E);
  if (A.failed) { set_error("emg_dof_build_device: out of device memory"); return EMG_ERR_NOMEM; }
  EMG_CK(cudaMemsetAsync(elem_edge, 0xff, sizeof(int32_t) * std::max<int64_t>(m, 1), st));
  k_edge_ids<<<grid_of(mv), kT, 0, st>>>(mv, key_s, slot_s, run, id_at, elem_edge, edge_nodes);
  EMG_CK(cudaMemsetAsync(constrained, 0, sizeof(int32_t) * std::max<int64_t>(E, 1), st));
  if (n_dir > 0)
    k_mark_constrained<<<grid_of(n_dir), kT, 0, st>>>(n_dir, dir_pairs, n_nodes, mv, key_s, slot_s, elem_edge,
                                                      constrained);
  k_not<<<grid_of(E), kT, 0, st>>>(E, constrained, ones);
  const int ei = static_cast<int>(E);
  EMG_CK(cub::DeviceScan::ExclusiveSum(tmp, tb, ones, free_rank, ei + 1, st));  // free_rank[E] = n_free
  int32_t nf = 0;
  EMG_CK(cudaMemcpyAsync(&nf, free_rank + E, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  EMG_CK(cudaStreamSynchronize(st));
  int64_t n_dofs = nf;
  if (gauge == EMG_GAUGE_NONE) {
    k_free_dof<<<grid_of(E), kT, 0, st>>>(E, constrained, free_rank, edge_dof);
  } else {
    // graph of the mesh edges: adjacency sorted by (node, neighbour)
    const int64_t n2 = 2 * E;
    uint64_t* akey = A.get<uint64_t>(n2);
    uint64_t* akey_s = A.get<uint64_t>(n2);
    int32_t* aeid = A.get<int32_t>(n2);
    int32_t* aeid_s = A.get<int32_t>(n2);
    int32_t* deg = A.get<int32_t>(n_nodes + 1);
    int32_t* ptr = A.get<int32_t>(n_nodes + 1);
    int32_t* nb = A.get<int32_t>(n2);
    int32_t* rank = A.get<int32_t>(n2);
    int32_t* pos = A.get<int32_t>(n_nodes);
    int32_t* queue = A.get<int32_t>(n_nodes);
    unsigned long long* bkey = A.get<unsigned long long>(n_nodes);
    int32_t* tree = A.get<int32_t>(E);
    int32_t* cnt = A.get<int32_t>(n_nodes + 1);
    int32_t* off = A.get<int32_t>(n_nodes + 1);
    int32_t* first = A.get<int32_t>(1);
    if (A.failed) { set_error("emg_dof_build_device: out of device memory"); return EMG_ERR_NOMEM; }
    EMG_CK(cudaMemsetAsync(deg, 0, sizeof(int32_t) * (n_nodes + 1), st));
    k_adj_keys<<<grid_of(E), kT, 0, st>>>(E, edge_nodes, akey, aeid, deg);
    EMG_CK(cub::DeviceRadixSort::SortPairs(tmp, tb, akey, akey_s, aeid, aeid_s, static_cast<int>(n2), 0, 32 + bits, st));
    EMG_CK(cub::DeviceScan::ExclusiveSum(tmp, tb, deg, ptr, static_cast<int>(n_nodes + 1), st));
    k_adj_nb<<<grid_of(n2), kT, 0, st>>>(n2, akey_s, nb);
    k_ranks<<<grid_of(n_nodes), kT, 0, st>>>(n_nodes, ptr, aeid_s, constrained, 1, rank);
    EMG_CK(cudaMemsetAsync(pos, 0xff, sizeof(int32_t) * std::max<int64_t>(n_nodes, 1), st));
    EMG_CK(cudaMemsetAsync(bkey, 0xff, sizeof(unsigned long long) * std::max<int64_t>(n_nodes, 1), st));
    EMG_CK(cudaMemsetAsync(tree, 0, sizeof(int32_t) * std::max<int64_t>(E, 1), st));
    // root: lower node of the lowest constrained edge ID, else the lowest
    // referenced node (SpanningTreeBuilder::selectRootNode, spanning_tree.cpp:517-540)
    int32_t fe = INT32_MAX, root = -1;
    EMG_CK(cudaMemcpyAsync(first, &fe, sizeof(int32_t), cudaMemcpyHostToDevice, st));
    k_first_constrained<<<grid_of(E), kT, 0, st>>>(E, constrained, first);
    EMG_CK(cudaMemcpyAsync(&fe, first, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    EMG_CK(cudaStreamSynchronize(st));
    if (fe != INT32_MAX) {
      EMG_CK(cudaMemcpyAsync(&root, edge_nodes + 2 * static_cast<int64_t>(fe), sizeof(int32_t),
                             cudaMemcpyDeviceToHost, st));
      EMG_CK(cudaStreamSynchronize(st));
    }
    int32_t placed = 0;
    for (int component = 0;; ++component) {
      if (component > 0 || root < 0) {  // lowest referenced node not yet reached
        int32_t v = INT32_MAX;
        EMG_CK(cudaMemcpyAsync(first, &v, sizeof(int32_t), cudaMemcpyHostToDevice, st));
        k_first_unseen<<<grid_of(n_nodes), kT, 0, st>>>(n_nodes, deg, pos, first);
        EMG_CK(cudaMemcpyAsync(&v, first, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        EMG_CK(cudaStreamSynchronize(st));
        if (v == INT32_MAX) break;
        root = v;
      }
      // the first component grows with the Dirichlet-first rule, the others
      // by plain BFS (spanning_tree.cpp:418-445)
      const int32_t* rk = component == 0 ? rank : nullptr;
      k_seed<<<1, 1, 0, st>>>(root, placed, queue, pos);
      int32_t p0 = placed, p1 = placed + 1;
      while (p1 > p0) {
        const int32_t w = p1 - p0;
        k_bfs_expand<<<grid_of(w), kT, 0, st>>>(p0, p1, queue, ptr, nb, rk, pos, bkey);
        k_bfs_count<<<grid_of(w), kT, 0, st>>>(p0, p1, queue, ptr, nb, rk, pos, bkey, cnt);
        EMG_CK(cudaMemsetAsync(cnt + w, 0, sizeof(int32_t), st));
        EMG_CK(cub::DeviceScan::ExclusiveSum(tmp, tb, cnt, off, w + 1, st));
        k_bfs_place<<<grid_of(w), kT, 0, st>>>(p0, p1, queue, ptr, nb, aeid_s, rk, constrained, pos, bkey, off, tree);
        int32_t found = 0;
        EMG_CK(cudaMemcpyAsync(&found, off + w, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        EMG_CK(cudaStreamSynchronize(st));
        p0 = p1;
        p1 += found;
      }
      placed = p1;
      if (component > 100000) { set_error("emg_dof_build_device: too many components"); return EMG_ERR_INTERNAL; }
    }
    // circulation picks: evenly spaced cotree ranks, one per hole marker
    // (selectCirculationDOFs, multi_connected_domain.cpp:190-232)
    int32_t* not_tree = ones;
    k_not<<<grid_of(E), kT, 0, st>>>(E, tree, not_tree);
    int32_t* cot_rank = A.get<int32_t>(E + 1);
    int32_t* kept = A.get<int32_t>(E + 1);
    int32_t* kept_rank = A.get<int32_t>(E + 1);
    int32_t* circ = A.get<int32_t>(E + 1);
    int32_t* circ_rank = A.get<int32_t>(E + 1);
    int32_t* picks = A.get<int32_t>(std::max<int32_t>(n_hole_markers, 1));
    if (A.failed) { set_error("emg_dof_build_device: out of device memory"); return EMG_ERR_NOMEM; }
    EMG_CK(cub::DeviceScan::ExclusiveSum(tmp, tb, not_tree, cot_rank, ei + 1, st));
    int32_t ncot = 0;
    EMG_CK(cudaMemcpyAsync(&ncot, cot_rank + E, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    EMG_CK(cudaStreamSynchronize(st));
    std::vector<int32_t> hp;
    if (n_hole_markers > 0 && ncot > 0) {
      const int64_t pick = std::min<int64_t>(n_hole_markers, ncot);
      for (int64_t i = 0; i < pick; ++i)
        hp.push_back(static_cast<int32_t>(std::min<int64_t>((i * ncot) / pick, ncot - 1)));
      EMG_CK(cudaMemcpyAsync(picks, hp.data(), sizeof(int32_t) * hp.size(), cudaMemcpyHostToDevice, st));
    }
    k_reduced_flags<<<grid_of(E), kT, 0, st>>>(E, tree, constrained, cot_rank, picks, static_cast<int32_t>(hp.size()),
                                               kept, circ);
    EMG_CK(cudaMemsetAsync(kept + E, 0, sizeof(int32_t), st));
    EMG_CK(cudaMemsetAsync(circ + E, 0, sizeof(int32_t), st));
    EMG_CK(cub::DeviceScan::ExclusiveSum(tmp, tb, kept, kept_rank, ei + 1, st));
    EMG_CK(cub::DeviceScan::ExclusiveSum(tmp, tb, circ, circ_rank, ei + 1, st));
    int32_t nk = 0, nc = 0;
    EMG_CK(cudaMemcpyAsync(&nk, kept_rank + E, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    EMG_CK(cudaMemcpyAsync(&nc, circ_rank + E, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    EMG_CK(cudaStreamSynchronize(st));
    k_edge_dof<<<grid_of(E), kT, 0, st>>>(E, constrained, kept, kept_rank, circ, circ_rank, nk, edge_dof);
    n_dofs = static_cast<int64_t>(nk) + nc;
  }
  k_l2g<<<grid_of(m), kT, 0, st>>>(m, elem_edge, edge_dof, l2g_out);
  EMG_CK(cudaGetLastError());
  EMG_CK(cudaStreamSynchronize(st));
  if (n_edges_out) *n_edges_out = E;
  if (n_free_out) *n_free_out = nf;
  if (n_dofs_out) *n_dofs_out = n_dofs;
  return EMG_SUCCESS;
}

}  // namespace emg

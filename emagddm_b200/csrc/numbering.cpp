// numbering.cpp -- host integer work of the solve path: global edge IDs, the
// free-DOF numbering and the tree-cotree gauge.  The results are bit-exact to
// the reference classes
//   GlobalEdgeIDGenerator  (src/fe_em/global_edge_id_generator.cpp:30-110)
//   EMDOFManager           (src/fe_em/em_dof_manager.cpp:29-393, :448-626)
//   MeshGraphExtractor     (src/fe_em/mesh_graph_extractor.cpp:29-176)
//   SpanningTreeBuilder    (src/fe_em/spanning_tree.cpp:295-598)
//   MultiConnectedDomainDetector (src/fe_em/multi_connected_domain.cpp:21-250)
//   TreeGauge              (src/fe_em/tree_gauge.cpp:37-290)
// but run in O(E) / O(E log d) with flat arrays instead of hash maps and
// std::set, and without the O(N^2) renumbering scan of em_dof_manager.cpp:245-286.
#include <algorithm>
#include <cstring>
#include <numeric>

#include "internal.h"

namespace emg {
namespace {

// Compressed adjacency: for every bucket a contiguous run of entries.
struct Buckets {
  std::vector<int64_t> ptr;
  std::vector<int32_t> a;  // first payload
  std::vector<int32_t> b;  // second payload
};

}  // namespace

// Edge IDs by first appearance.  Each element edge (lo, hi, position) is
// bucketed by its lower node; buckets are filled in position order, so the
// leader of a (lo, hi) key is the first entry of the bucket with that hi.  The
// leaders in position order receive consecutive IDs -- exactly the order in
// which the reference's hash map assigns new IDs.
int build_edge_ids(Mesh& m) {
  if (m.edges_built) return EMG_SUCCESS;
  const int npe = m.npe(), epe = m.epe();
  const int64_t T = m.n_elems, V = m.n_nodes, M = epe * T;
  // local edges of element t (a mixed mesh's rows name their own type)
  auto edges_of = [&](int64_t t, const int (**le)[2]) {
    const int32_t et = row_type(m.elem_type, &m.elems[npe * t]);
    *le = local_edges(et);
    return edges_per_elem(et);
  };
  Buckets bk;
  bk.ptr.assign(V + 1, 0);
  for (int64_t t = 0; t < T; ++t) {
    const int (*le)[2];
    const int ne = edges_of(t, &le);
    for (int k = 0; k < ne; ++k) {
      int32_t u = m.elems[npe * t + le[k][0]], w = m.elems[npe * t + le[k][1]];
      bk.ptr[std::min(u, w) + 1]++;
    }
  }
  for (int64_t v = 0; v < V; ++v) bk.ptr[v + 1] += bk.ptr[v];
  bk.a.resize(bk.ptr[V]);  // hi node
  bk.b.resize(bk.ptr[V]);  // position
  std::vector<int64_t> cur(bk.ptr.begin(), bk.ptr.end() - 1);
  for (int64_t t = 0; t < T; ++t) {
    const int (*le)[2];
    const int ne = edges_of(t, &le);
    for (int k = 0; k < ne; ++k) {
      int32_t u = m.elems[npe * t + le[k][0]], w = m.elems[npe * t + le[k][1]];
      int64_t s = cur[std::min(u, w)]++;
      bk.a[s] = std::max(u, w);
      bk.b[s] = static_cast<int32_t>(epe * t + k);
    }
  }
  // leader position of every entry: the bucket's distinct hi nodes so far
  // (a handful per node) are searched instead of all its earlier entries
  std::vector<int32_t> leader(M, -1);  // -1: slot past its element's edges
  std::vector<uint8_t> is_leader(M, 0);
  std::vector<int32_t> seen_hi, seen_pos;
  for (int64_t v = 0; v < V; ++v) {
    seen_hi.clear();
    seen_pos.clear();
    for (int64_t s = bk.ptr[v]; s < bk.ptr[v + 1]; ++s) {
      size_t f = 0;
      while (f < seen_hi.size() && seen_hi[f] != bk.a[s]) ++f;
      if (f == seen_hi.size()) {  // first entry with this hi
        seen_hi.push_back(bk.a[s]);
        seen_pos.push_back(bk.b[s]);
        is_leader[bk.b[s]] = 1;
      }
      leader[bk.b[s]] = seen_pos[f];
    }
  }
  std::vector<int32_t> id_at(M, -1);
  int64_t next = 0;
  for (int64_t p = 0; p < M; ++p)
    if (is_leader[p]) id_at[p] = static_cast<int32_t>(next++);
  m.n_edges = next;
  m.elem_edge.resize(M);
  m.edge_nodes.resize(2 * next);
  for (int64_t p = 0; p < M; ++p) {
    int32_t id = leader[p] < 0 ? -1 : id_at[leader[p]];
    m.elem_edge[p] = id;
    if (is_leader[p]) {
      int64_t t = p / epe;
      int k = static_cast<int>(p % epe);
      const int (*le)[2];
      edges_of(t, &le);
      int32_t u = m.elems[npe * t + le[k][0]], w = m.elems[npe * t + le[k][1]];
      m.edge_nodes[2 * id] = std::min(u, w);
      m.edge_nodes[2 * id + 1] = std::max(u, w);
    }
  }
  m.edges_built = true;
  return EMG_SUCCESS;
}

namespace {

// Graph of the mesh edges over compact node indices (rank of the global node
// ID among referenced nodes), neighbours ascending -- MeshGraphExtractor.
struct EdgeGraph {
  int32_t n_nodes = 0;
  std::vector<int32_t> compact;  // global node -> compact index or -1
  std::vector<int64_t> ptr;
  std::vector<int32_t> nb;       // neighbour compact index
  std::vector<int32_t> edge;     // global edge ID of the entry
};

EdgeGraph make_graph(const Mesh& m) {
  EdgeGraph g;
  g.compact.assign(m.n_nodes, -1);
  const int npe = m.npe();
  for (int64_t t = 0; t < m.n_elems; ++t) {  // nodes referenced by the elements
    const int nn = nodes_per_elem(row_type(m.elem_type, &m.elems[npe * t]));
    for (int a = 0; a < nn; ++a) g.compact[m.elems[npe * t + a]] = 0;
  }
  int32_t c = 0;
  for (int64_t v = 0; v < m.n_nodes; ++v)
    if (g.compact[v] == 0) g.compact[v] = c++;
  g.n_nodes = c;
  g.ptr.assign(static_cast<size_t>(c) + 1, 0);
  const int64_t E = m.n_edges;
  for (int64_t e = 0; e < E; ++e) {
    g.ptr[g.compact[m.edge_nodes[2 * e]] + 1]++;
    g.ptr[g.compact[m.edge_nodes[2 * e + 1]] + 1]++;
  }
  for (int32_t v = 0; v < c; ++v) g.ptr[v + 1] += g.ptr[v];
  g.nb.resize(2 * E);
  g.edge.resize(2 * E);
  std::vector<int64_t> cur(g.ptr.begin(), g.ptr.end() - 1);
  for (int64_t e = 0; e < E; ++e) {
    int32_t u = g.compact[m.edge_nodes[2 * e]], w = g.compact[m.edge_nodes[2 * e + 1]];
    g.nb[cur[u]] = w; g.edge[cur[u]++] = static_cast<int32_t>(e);
    g.nb[cur[w]] = u; g.edge[cur[w]++] = static_cast<int32_t>(e);
  }
  std::vector<std::pair<int32_t, int32_t>> tmp;
  for (int32_t v = 0; v < c; ++v) {
    tmp.clear();
    for (int64_t s = g.ptr[v]; s < g.ptr[v + 1]; ++s) tmp.emplace_back(g.nb[s], g.edge[s]);
    std::sort(tmp.begin(), tmp.end());
    for (size_t i = 0; i < tmp.size(); ++i) {
      g.nb[g.ptr[v] + i] = tmp[i].first;
      g.edge[g.ptr[v] + i] = tmp[i].second;
    }
  }
  return g;
}

// Plain BFS over all edges from the nodes already queued (queue[head..tail)).
void bfs_all(const EdgeGraph& g, std::vector<int32_t>& queue, size_t head,
             std::vector<uint8_t>& seen, std::vector<uint8_t>& tree) {
  for (size_t h = head; h < queue.size(); ++h) {
    int32_t u = queue[h];
    for (int64_t s = g.ptr[u]; s < g.ptr[u + 1]; ++s) {
      int32_t v = g.nb[s];
      if (seen[v]) continue;
      seen[v] = 1;
      tree[g.edge[s]] = 1;
      queue.push_back(v);
    }
  }
}

// Spanning tree; tree[e] = 1 for tree edges.  Returns the root.
int32_t spanning_tree(const Mesh& m, const EdgeGraph& g, const std::vector<uint8_t>& constrained,
                      int32_t gauge_mode, std::vector<uint8_t>& tree) {
  const int64_t E = m.n_edges;
  tree.assign(E, 0);
  std::vector<uint8_t> seen(g.n_nodes, 0);
  std::vector<int32_t> queue;
  queue.reserve(g.n_nodes);
  // Root: smaller compact endpoint of the lowest constrained edge ID, else 0
  // (SpanningTreeBuilder::selectRootNode, DIRICHLET_BOUNDARY, spanning_tree.cpp:517-540).
  int32_t root = 0;
  for (int64_t e = 0; e < E; ++e)
    if (constrained[e]) { root = g.compact[m.edge_nodes[2 * e]]; break; }
  if (g.n_nodes == 0) return -1;
  seen[root] = 1;
  queue.push_back(root);
  if (gauge_mode == EMG_GAUGE_REF) {
    // buildBFSTreeWithBoundaryPriority (spanning_tree.cpp:353-416): for each
    // dequeued node, its unseen neighbours across constrained edges join the
    // tree first, then the others; both groups in ascending neighbour order.
    std::vector<int64_t> later;
    for (size_t h = 0; h < queue.size(); ++h) {
      int32_t u = queue[h];
      later.clear();
      for (int64_t s = g.ptr[u]; s < g.ptr[u + 1]; ++s) {
        int32_t v = g.nb[s];
        if (seen[v]) continue;
        if (constrained[g.edge[s]]) {
          seen[v] = 1;
          tree[g.edge[s]] = 1;
          queue.push_back(v);
        } else {
          later.push_back(s);
        }
      }
      for (int64_t s : later) {
        int32_t v = g.nb[s];
        if (seen[v]) continue;
        seen[v] = 1;
        tree[g.edge[s]] = 1;
        queue.push_back(v);
      }
    }
  } else {
    // Boundary-first: span the constrained-edge subgraph before anything else
    // (every constrained component, lowest edge first), then grow the tree
    // into the interior by plain BFS in visit order.  Every node off the
    // constrained subgraph then owns exactly one tree edge, so the kept
    // unknowns are E_free - V_interior (a complete, not over-constrained,
    // gauge for a connected Dirichlet boundary).
    auto span_constrained = [&](size_t head) {
      for (size_t h = head; h < queue.size(); ++h) {
        int32_t u = queue[h];
        for (int64_t s = g.ptr[u]; s < g.ptr[u + 1]; ++s) {
          int32_t v = g.nb[s];
          if (seen[v] || !constrained[g.edge[s]]) continue;
          seen[v] = 1;
          tree[g.edge[s]] = 1;
          queue.push_back(v);
        }
      }
    };
    span_constrained(0);
    for (int64_t e = 0; e < E; ++e) {
      if (!constrained[e]) continue;
      int32_t s0 = g.compact[m.edge_nodes[2 * e]];
      if (seen[s0]) continue;
      seen[s0] = 1;
      size_t head = queue.size();
      queue.push_back(s0);
      span_constrained(head);
    }
    bfs_all(g, queue, 0, seen, tree);
  }
  // Remaining components, lowest unseen index first (spanning_tree.cpp:418-445).
  for (int32_t s = 0; s < g.n_nodes; ++s) {
    if (seen[s]) continue;
    seen[s] = 1;
    size_t head = queue.size();
    queue.push_back(s);
    bfs_all(g, queue, head, seen, tree);
  }
  return root;
}

// markConstrainedDOFs (em_dof_manager.cpp:152-243): constrained[e] = 1 for
// every mesh edge listed as a Dirichlet node pair; pairs that are not mesh
// edges are skipped.
void mark_constrained(const Mesh& m, std::vector<uint8_t>& constrained) {
  const int64_t E = m.n_edges;
  // Edge lookup by node pair: edges bucketed by lower node.
  std::vector<int64_t> lptr(m.n_nodes + 1, 0);
  for (int64_t e = 0; e < E; ++e) lptr[m.edge_nodes[2 * e] + 1]++;
  for (int64_t v = 0; v < m.n_nodes; ++v) lptr[v + 1] += lptr[v];
  std::vector<int32_t> lid(E);
  {
    std::vector<int64_t> cur(lptr.begin(), lptr.end() - 1);
    for (int64_t e = 0; e < E; ++e) lid[cur[m.edge_nodes[2 * e]]++] = static_cast<int32_t>(e);
  }
  constrained.assign(E, 0);
  const int64_t D = static_cast<int64_t>(m.dirichlet.size() / 2);
  for (int64_t d = 0; d < D; ++d) {
    int32_t a = m.dirichlet[2 * d], b = m.dirichlet[2 * d + 1];
    if (a < 0 || b < 0 || a >= m.n_nodes || b >= m.n_nodes) continue;
    int32_t lo = std::min(a, b), hi = std::max(a, b);
    for (int64_t s = lptr[lo]; s < lptr[lo + 1]; ++s)
      if (m.edge_nodes[2 * lid[s] + 1] == hi) { constrained[lid[s]] = 1; break; }
  }
}

}  // namespace

int build_dofmap(Mesh& m, int32_t gauge_mode, DofMap& out) {
  int rc = build_edge_ids(m);
  if (rc) return rc;
  const int64_t E = m.n_edges, T = m.n_elems;
  out = DofMap{};
  out.elem_type = m.elem_type;
  out.n_elems = T;
  out.n_edges = E;
  std::vector<uint8_t> constrained;
  mark_constrained(m, constrained);
  // Prenumber of an edge in an all-vector mesh = its global ID
  // (assignPrenumbering, :91-150); free index = rank among the unconstrained
  // (renumberFreeDOFs, :245-286).
  std::vector<int32_t> free_of(E);
  int64_t nf = 0;
  for (int64_t e = 0; e < E; ++e) free_of[e] = constrained[e] ? -1 : static_cast<int32_t>(nf++);
  out.n_free = nf;
  out.edge_dof.assign(E, -1);
  if (gauge_mode == EMG_GAUGE_NONE) {
    out.edge_dof = free_of;
    out.n_dofs = nf;
  } else if (gauge_mode == EMG_GAUGE_REF || gauge_mode == EMG_GAUGE_BOUNDARY_FIRST) {
    EdgeGraph g = make_graph(m);
    std::vector<uint8_t> tree;
    out.root = spanning_tree(m, g, constrained, gauge_mode, tree);
    // Circulation DOFs (selectCirculationDOFs, multi_connected_domain.cpp:190-232):
    // one evenly spaced pick per hole marker from the ascending cotree list,
    // taken before constrained edges are promoted to the tree.
    std::vector<uint8_t> circ(E, 0);
    std::vector<int32_t> cot;
    for (int64_t e = 0; e < E; ++e) if (!tree[e]) cot.push_back(static_cast<int32_t>(e));
    if (m.n_hole_markers > 0 && !cot.empty()) {
      int64_t pick = std::min<int64_t>(m.n_hole_markers, static_cast<int64_t>(cot.size()));
      for (int64_t i = 0; i < pick; ++i) {
        int64_t idx = std::min<int64_t>((i * static_cast<int64_t>(cot.size())) / pick,
                                        static_cast<int64_t>(cot.size()) - 1);
        circ[cot[idx]] = 1;
      }
    }
    // classifyEdges / buildReducedMapping (tree_gauge.cpp:159-212) and
    // renumberVectorDOFsWithTreeGauge (em_dof_manager.cpp:501-626).
    std::vector<int32_t> reduced(E, -1);
    int64_t nr = 0;
    for (int64_t e = 0; e < E; ++e)
      if (!tree[e] && !constrained[e] && !circ[e]) reduced[e] = static_cast<int32_t>(nr++);
    for (int64_t e = 0; e < E; ++e)
      if (circ[e] && reduced[e] < 0) reduced[e] = static_cast<int32_t>(nr++);
    for (int64_t e = 0; e < E; ++e) out.edge_dof[e] = free_of[e] < 0 ? -1 : reduced[e];
    out.n_dofs = nr;
  } else {
    set_error("unknown gauge mode");
    return EMG_INVALID_INPUT;
  }
  out.l2g.resize(m.elem_edge.size());
  for (size_t p = 0; p < m.elem_edge.size(); ++p) out.l2g[p] = m.elem_edge[p] < 0 ? -1 : out.edge_dof[m.elem_edge[p]];
  return EMG_SUCCESS;
}

// Per-element DOF types (Element::dof_type, include/fe_em/em_mesh_data.hpp:45-49).
// Scalar unknowns: the nodes of SCALAR_ONLY / MIXED_AV elements, prenumbered
// in ascending node ID (assignPrenumbering, em_dof_manager.cpp:91-150),
// constrained by the scalar Dirichlet node list (markConstrainedDOFs,
// :152-243) and ranked first among the free DOFs (renumberFreeDOFs,
// :245-286).  Edge unknowns: GlobalEdgeIDGenerator and the tree gauge see
// only VECTOR_EDGE_ONLY / MIXED_AV elements (global_edge_id_generator.cpp:44-53,
// mesh_graph_extractor.cpp:78), so they are the edge numbering of that
// sub-mesh (same node IDs, Dirichlet pairs and hole markers) shifted past
// the free scalars, both before the gauge and after it
// (renumberVectorDOFsWithTreeGauge, :501-626).  Element rows follow
// buildScalar/Vector/MixedAVElementMapping (:318-446).
int build_dofmap_av(const Mesh& m, const int32_t* dof_type, int64_t n_sdir, const int32_t* sdir,
                    int32_t gauge_mode, std::vector<int32_t>& l2g, int64_t& n_scalar_free, int64_t& n_free,
                    int64_t& n_dofs) {
  const int npe = m.npe(), epe = m.epe(), w = npe + epe;
  const int64_t T = m.n_elems;
  if (gauge_mode != EMG_GAUGE_NONE && gauge_mode != EMG_GAUGE_REF && gauge_mode != EMG_GAUGE_BOUNDARY_FIRST) {
    set_error("unknown gauge mode");
    return EMG_INVALID_INPUT;
  }
  if (n_sdir < 0 || (n_sdir > 0 && !sdir)) {
    set_error("scalar Dirichlet list: negative count or null pointer");
    return EMG_INVALID_INPUT;
  }
  auto type_of = [&](int64_t e) { return dof_type ? dof_type[e] : static_cast<int32_t>(EMG_DOF_MIXED_AV); };
  Mesh sub;
  sub.elem_type = m.elem_type;
  sub.n_nodes = m.n_nodes;
  sub.dirichlet = m.dirichlet;
  sub.n_hole_markers = m.n_hole_markers;
  std::vector<uint8_t> scalar_node(static_cast<size_t>(m.n_nodes), 0);
  for (int64_t e = 0; e < T; ++e) {
    const int32_t t = type_of(e);
    if (t != EMG_DOF_SCALAR_ONLY && t != EMG_DOF_VECTOR_EDGE_ONLY && t != EMG_DOF_MIXED_AV) {
      set_error("dof_type of element " + std::to_string(e) + " is not SCALAR_ONLY, VECTOR_EDGE_ONLY or MIXED_AV");
      return EMG_INVALID_INPUT;
    }
    const int32_t* nodes = m.elems.data() + static_cast<size_t>(npe) * e;
    if (t != EMG_DOF_VECTOR_EDGE_ONLY)
      for (int i = 0; i < npe; ++i) scalar_node[nodes[i]] = 1;
    if (t != EMG_DOF_SCALAR_ONLY) {
      sub.elems.insert(sub.elems.end(), nodes, nodes + npe);
      sub.n_elems++;
    }
  }
  // Node IDs outside the mesh or on no scalar element constrain nothing, as
  // in the reference (the marker's node is not among the prenumbers).
  for (int64_t i = 0; i < n_sdir; ++i)
    if (sdir[i] >= 0 && sdir[i] < m.n_nodes && scalar_node[sdir[i]]) scalar_node[sdir[i]] = 2;
  std::vector<int32_t> sfree(static_cast<size_t>(m.n_nodes), -1);
  int64_t ns = 0;
  for (int64_t v = 0; v < m.n_nodes; ++v)
    if (scalar_node[v] == 1) sfree[v] = static_cast<int32_t>(ns++);
  DofMap vm;
  if (sub.n_elems > 0) {
    if (int rc = build_dofmap(sub, gauge_mode, vm)) return rc;
  }
  if (ns + vm.n_free > INT32_MAX) {
    set_error("too many DOFs for 32-bit indices");
    return EMG_INVALID_INPUT;
  }
  l2g.assign(static_cast<size_t>(w) * T, EMG_DOF_ABSENT);
  int64_t se = 0;
  for (int64_t e = 0; e < T; ++e) {
    const int32_t t = type_of(e);
    int32_t* row = l2g.data() + static_cast<size_t>(w) * e;
    int c = 0;
    if (t != EMG_DOF_VECTOR_EDGE_ONLY)
      for (int i = 0; i < npe; ++i) row[c++] = sfree[m.elems[static_cast<size_t>(npe) * e + i]];
    if (t != EMG_DOF_SCALAR_ONLY) {
      for (int j = 0; j < epe; ++j) {
        const int32_t d = vm.l2g[static_cast<size_t>(epe) * se + j];
        row[c++] = d < 0 ? -1 : static_cast<int32_t>(d + ns);
      }
      ++se;
    }
  }
  n_scalar_free = ns;
  n_free = ns + vm.n_free;
  n_dofs = ns + vm.n_dofs;
  return EMG_SUCCESS;
}

// Tree-cotree gauge for a non-overlapping partition of the elements (no
// counterpart in the reference, whose FETI-DP context is a stub:
// include/fetidp/fetidp_context.hpp:20-66).  Edges are ranked by class:
//   0 Dirichlet, 1 wire basket (shared by >= 3 subdomains),
//   2 subdomain face (shared by 2), 3 subdomain interior,
// and the spanning tree is grown Prim-style, always through the lowest class
// available (FIFO inside a class).  The Dirichlet surface is spanned first,
// then the wire basket, then every face from its rim, then every interior
// from its boundary, so the tree restricted to one subdomain hangs off that
// subdomain's wire basket.  Primal (coarse) DOFs are the cotree wire-basket
// edges; with the tree and the Dirichlet edges they keep every wire basket
// continuous.  A subdomain whose tree + Dirichlet + primal edges still fall
// apart into several node components gets, in ascending edge-ID order, the
// cotree edges that join two components as extra primal DOFs
// (n_primal_fix) -- that is what makes every local K_rr nonsingular: a local
// gradient field vanishing on a connected edge set is zero.  Reduced DOFs
// are the unconstrained cotree edges in ascending edge ID.
int build_dofmap_partitioned(Mesh& m, const int32_t* tet_part, int32_t n_parts, DofMap& out) {
  if (n_parts < 1 || (m.n_elems > 0 && tet_part == nullptr)) {
    set_error("partitioned gauge: need n_parts >= 1 and a tet_part array");
    return EMG_INVALID_INPUT;
  }
  if (m.n_hole_markers > 0) {
    set_error("partitioned gauge: hole markers (circulation DOFs) are not supported");
    return EMG_INVALID_INPUT;
  }
  const int64_t T = m.n_elems;
  for (int64_t t = 0; t < T; ++t)
    if (tet_part[t] < 0 || tet_part[t] >= n_parts) {
      set_error("partitioned gauge: tet_part[" + std::to_string(t) + "] outside [0, n_parts)");
      return EMG_INVALID_INPUT;
    }
  int rc = build_edge_ids(m);
  if (rc) return rc;
  const int64_t E = m.n_edges;
  const int npe = m.npe(), epe = m.epe();
  out = DofMap{};
  out.elem_type = m.elem_type;
  out.n_elems = T;
  out.n_edges = E;
  out.n_parts = n_parts;
  out.tet_part.assign(tet_part, tet_part + T);
  std::vector<uint8_t> constrained;
  mark_constrained(m, constrained);
  // subdomain multiplicity of every edge: 1, 2 or "3 or more"
  std::vector<int32_t> p1(E, -1), p2(E, -1);
  std::vector<uint8_t> many(E, 0);
  for (int64_t t = 0; t < T; ++t) {
    const int32_t p = tet_part[t];
    for (int k = 0; k < epe; ++k) {
      const int32_t e = m.elem_edge[epe * t + k];
      if (e < 0) continue;  // slot past a mixed-mesh element's edges
      if (p1[e] < 0) p1[e] = p;
      else if (p1[e] != p) {
        if (p2[e] < 0) p2[e] = p;
        else if (p2[e] != p) many[e] = 1;
      }
    }
  }
  std::vector<uint8_t> cls(E);
  for (int64_t e = 0; e < E; ++e)
    cls[e] = constrained[e] ? 0 : many[e] ? 1 : (p2[e] >= 0 ? 2 : 3);

  EdgeGraph g = make_graph(m);
  std::vector<uint8_t> seen(g.n_nodes, 0), tree(E, 0);
  std::vector<int64_t> bucket[4];
  size_t head[4] = {0, 0, 0, 0};
  auto visit = [&](int32_t v) {
    seen[v] = 1;
    for (int64_t s = g.ptr[v]; s < g.ptr[v + 1]; ++s)
      if (!seen[g.nb[s]]) bucket[cls[g.edge[s]]].push_back(s);
  };
  int32_t root = 0;
  for (int64_t e = 0; e < E; ++e)
    if (constrained[e]) { root = g.compact[m.edge_nodes[2 * e]]; break; }
  int32_t cursor = 0;
  if (g.n_nodes > 0) visit(root);
  out.root = g.n_nodes > 0 ? root : -1;
  for (;;) {
    int c = 0;
    while (c < 4 && head[c] >= bucket[c].size()) ++c;
    if (c == 4) {
      // next component: lowest unseen node
      while (cursor < g.n_nodes && seen[cursor]) ++cursor;
      if (cursor >= g.n_nodes) break;
      visit(cursor);
      continue;
    }
    const int64_t s = bucket[c][head[c]++];
    const int32_t v = g.nb[s];
    if (seen[v]) continue;
    tree[g.edge[s]] = 1;
    visit(v);
  }

  std::vector<uint8_t> primal(E, 0);
  for (int64_t e = 0; e < E; ++e)
    if (!tree[e] && !constrained[e] && cls[e] == 1) primal[e] = 1;

  // Connect every subdomain: union-find over its nodes through its tree,
  // Dirichlet and primal edges, then promote joining cotree edges.
  std::vector<int64_t> tptr(static_cast<size_t>(n_parts) + 1, 0);
  for (int64_t t = 0; t < T; ++t) tptr[tet_part[t] + 1]++;
  for (int32_t p = 0; p < n_parts; ++p) tptr[p + 1] += tptr[p];
  std::vector<int32_t> tlist(T);
  {
    std::vector<int64_t> cur(tptr.begin(), tptr.end() - 1);
    for (int64_t t = 0; t < T; ++t) tlist[cur[tet_part[t]]++] = static_cast<int32_t>(t);
  }
  std::vector<int32_t> node_loc(m.n_nodes, -1), uf;
  std::vector<int32_t> nodes, edges;
  auto find = [&](int32_t a) {
    while (uf[a] != a) { uf[a] = uf[uf[a]]; a = uf[a]; }
    return a;
  };
  int64_t fixes = 0;
  for (int32_t p = 0; p < n_parts; ++p) {
    nodes.clear();
    edges.clear();
    for (int64_t q = tptr[p]; q < tptr[p + 1]; ++q) {
      const int64_t t = tlist[q];
      const int nn = nodes_per_elem(row_type(m.elem_type, &m.elems[npe * t]));
      for (int a = 0; a < nn; ++a) {
        const int32_t v = m.elems[npe * t + a];
        if (node_loc[v] < 0) { node_loc[v] = static_cast<int32_t>(nodes.size()); nodes.push_back(v); }
      }
      for (int k = 0; k < epe; ++k)
        if (m.elem_edge[epe * t + k] >= 0) edges.push_back(m.elem_edge[epe * t + k]);
    }
    std::sort(edges.begin(), edges.end());
    edges.erase(std::unique(edges.begin(), edges.end()), edges.end());
    uf.resize(nodes.size());
    std::iota(uf.begin(), uf.end(), 0);
    for (int32_t e : edges) {
      if (!(tree[e] || constrained[e] || primal[e])) continue;
      int32_t a = find(node_loc[m.edge_nodes[2 * e]]), b = find(node_loc[m.edge_nodes[2 * e + 1]]);
      if (a != b) uf[a] = b;
    }
    for (int32_t e : edges) {
      if (tree[e] || constrained[e] || primal[e]) continue;
      int32_t a = find(node_loc[m.edge_nodes[2 * e]]), b = find(node_loc[m.edge_nodes[2 * e + 1]]);
      if (a != b) { uf[a] = b; primal[e] = 1; ++fixes; }
    }
    for (int32_t v : nodes) node_loc[v] = -1;
  }

  std::vector<int32_t> free_of(E);
  int64_t nf = 0;
  for (int64_t e = 0; e < E; ++e) free_of[e] = constrained[e] ? -1 : static_cast<int32_t>(nf++);
  out.n_free = nf;
  out.edge_dof.assign(E, -1);
  int64_t nr = 0;
  for (int64_t e = 0; e < E; ++e)
    if (!tree[e] && !constrained[e]) {
      out.edge_dof[e] = static_cast<int32_t>(nr++);
      out.dof_primal.push_back(primal[e]);
    }
  out.n_dofs = nr;
  out.n_primal_fix = fixes;
  out.l2g.resize(m.elem_edge.size());
  for (size_t p = 0; p < m.elem_edge.size(); ++p) out.l2g[p] = m.elem_edge[p] < 0 ? -1 : out.edge_dof[m.elem_edge[p]];
  return EMG_SUCCESS;
}

}  // namespace emg

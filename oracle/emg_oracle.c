/*
 * emg_oracle.c -- CPU oracle (test infrastructure only) for the TET4 / HEX8
 * Nedelec curl-curl solve path of Poofee/emagddm.  See emg_oracle.h for how each part
 * is pinned.  Only tests/, __graft_entry__.smoke() and bench.py (CPU baseline
 * and the reference arm) load this file's library.
 *
 * Deliberate deviations from the reference's literal element output, each
 * switchable by a flag for element-level comparison:
 *   1. edge signs: the reference scatters unsigned element matrices
 *      (src/numeric/em_assembly.cpp:654-718); a conforming H(curl) assembly
 *      needs s_k = +-1 per local edge.  Convention: global edge oriented from
 *      the lower to the higher global node ID.  ORC_FLAG_NO_EDGE_SIGNS turns
 *      signs off.
 *   2. covariant map W_phys = J^-T W_ref; the reference text divides by detJ as
 *      well (src/numeric/magnetic_vector_3d_integrator.cpp:429-430);
 *      ORC_FLAG_PIOLA_LITERAL restores that.
 *   3. Hammer 4-point rule with weights summing to 1/6; the reference pops the
 *      third point (src/numeric/gauss_quadrature.cpp:205-219) and, called with
 *      TET4_EDGE, returns no points at all (:36-60), so its K_e is zero.
 *      ORC_FLAG_QUAD3_LITERAL restores the 3-point rule.
 *   4. F_i = int W_i . J_s is computed; the reference returns zero
 *      (magnetic_vector_3d_integrator.cpp:343-364, formula at :353).
 */
#include "emg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* TET4 geometry edge table, ElementGeometry::get_local_edges(TET4)
 * (src/fe_em/element_geometry.cpp:115-126). */
static const int GEO_EDGE[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
/* Nedelec TET4_EDGE edge table (src/numeric/nedelec_element.cpp:54-60). */
static const int NED_EDGE[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 3}, {1, 3}, {2, 3}};
/* HEX8 geometry edge table (element_geometry.cpp:161-181); HEX8_EDGE basis k
 * runs from node [k][0] to node [k][1] (nedelec_element.cpp:506-517). */
static const int HEX_EDGE[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                    {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
/* PRISM6 and PYRAMID5 geometry edge tables (element_geometry.cpp:214-237,
 * :268-289); the basis of edge k runs from node [k][0] to node [k][1]. */
static const int PRISM_EDGE[9][2] = {{0, 1}, {1, 2}, {0, 2}, {3, 4}, {4, 5}, {3, 5}, {0, 3}, {1, 4}, {2, 5}};
static const int PYR_EDGE[8][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {0, 4}, {1, 4}, {2, 4}, {3, 4}};
/* HEX8 reference node coordinates (lagrange_element.cpp:765-772). */
static const double HEX_NODE[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                      {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
/* Constant reference curls, curlTet4Edge (nedelec_element.cpp:461-505). */
static const double CURL_REF[6][3] = {{0, 0, -2}, {-2, 0, 0}, {0, -2, 0},
                                      {0, -2, 2}, {2, 0, -2}, {-2, 2, 0}};

/* ---------------------------------------------------------------------------
 * Stable LSD radix sort of (key, payload) pairs, 11-bit digits.
 * ------------------------------------------------------------------------- */
static int radix_sort_u64(int64_t n, uint64_t* key, int64_t* pay, uint64_t max_key) {
  if (n <= 1) return 0;
  int bits = 0;
  while (bits < 64 && (max_key >> bits) != 0) bits++;
  if (bits == 0) return 0;
  uint64_t* k2 = (uint64_t*)malloc((size_t)n * sizeof(uint64_t));
  int64_t* p2 = (int64_t*)malloc((size_t)n * sizeof(int64_t));
  if (!k2 || !p2) { free(k2); free(p2); return -1; }
  const int D = 11, B = 1 << D;
  int64_t cnt[1 << 11];
  uint64_t *ks = key, *kd = k2;
  int64_t *ps = pay, *pd = p2;
  for (int shift = 0; shift < bits; shift += D) {
    memset(cnt, 0, sizeof(cnt));
    for (int64_t i = 0; i < n; i++) cnt[(ks[i] >> shift) & (B - 1)]++;
    int64_t s = 0;
    for (int b = 0; b < B; b++) { int64_t c = cnt[b]; cnt[b] = s; s += c; }
    for (int64_t i = 0; i < n; i++) {
      int64_t d = cnt[(ks[i] >> shift) & (B - 1)]++;
      kd[d] = ks[i];
      pd[d] = ps[i];
    }
    uint64_t* tk = ks; ks = kd; kd = tk;
    int64_t* tp = ps; ps = pd; pd = tp;
  }
  if (ks != key) {
    memcpy(key, ks, (size_t)n * sizeof(uint64_t));
    memcpy(pay, ps, (size_t)n * sizeof(int64_t));
  }
  free(k2);
  free(p2);
  return 0;
}

/* ---------------------------------------------------------------------------
 * Global edge IDs: key = sorted global node pair, ID = order of first
 * appearance over elements in order and local edges in order
 * (global_edge_id_generator.cpp:44-97).  Sort-based restatement of the hash
 * map: a stable sort groups equal keys with the first appearance leading its
 * group, and IDs are the prefix count of group leaders by position.
 * ------------------------------------------------------------------------- */
static int elem_shape(int32_t elem_type, int* npe, int* epe, const int (**tab)[2]) {
  if (elem_type == ORC_ELEM_TET4_EDGE) { *npe = 4; *epe = 6; *tab = GEO_EDGE; return 0; }
  if (elem_type == ORC_ELEM_HEX8_EDGE) { *npe = 8; *epe = 12; *tab = HEX_EDGE; return 0; }
  if (elem_type == ORC_ELEM_PRISM6_EDGE) { *npe = 6; *epe = 9; *tab = PRISM_EDGE; return 0; }
  if (elem_type == ORC_ELEM_PYRAMID5_EDGE) { *npe = 5; *epe = 8; *tab = PYR_EDGE; return 0; }
  if (elem_type == ORC_ELEM_MIXED) { *npe = 9; *epe = 12; *tab = NULL; return 0; }
  return ORC_INVALID_INPUT;
}

/* Nodes, edges, edge table and type of one element row (rows of a mixed mesh
 * carry their type in slot 8). */
static int row_shape(int32_t elem_type, const int32_t* row, int* nn, int* ne, const int (**tab)[2],
                     int32_t* et) {
  *et = elem_type == ORC_ELEM_MIXED ? row[8] : elem_type;
  if (*et == ORC_ELEM_MIXED) return ORC_INVALID_INPUT;
  return elem_shape(*et, nn, ne, tab);
}

int orc_edge_ids(int64_t n_tets, const int32_t* tets, int32_t* elem_edge,
                 int32_t* edge_nodes, int64_t* n_edges) {
  return orc_edge_ids_typed(ORC_ELEM_TET4_EDGE, n_tets, tets, elem_edge, edge_nodes, n_edges);
}

int orc_edge_ids_typed(int32_t elem_type, int64_t n_tets, const int32_t* tets, int32_t* elem_edge,
                       int32_t* edge_nodes, int64_t* n_edges) {
  int npe, epe;
  const int (*tab)[2];
  *n_edges = 0;
  if (elem_shape(elem_type, &npe, &epe, &tab)) return ORC_INVALID_INPUT;
  const int64_t slots = epe * n_tets;
  if (n_tets <= 0) return 0;
  int32_t maxg = 0;
  int64_t m = 0; /* element edges (slots past an element's edges excluded) */
  for (int64_t t = 0; t < n_tets; t++) {
    int nn, ne;
    const int (*rt)[2];
    int32_t et;
    if (row_shape(elem_type, tets + npe * t, &nn, &ne, &rt, &et)) return ORC_INVALID_INPUT;
    for (int a = 0; a < nn; a++) {
      if (tets[npe * t + a] < 0) return ORC_INVALID_INPUT;
      if (tets[npe * t + a] > maxg) maxg = tets[npe * t + a];
    }
    m += ne;
  }
  for (int64_t p = 0; p < slots; p++) elem_edge[p] = -1;
  uint64_t span = (uint64_t)maxg + 1;
  uint64_t* key = (uint64_t*)malloc((size_t)(m > 0 ? m : 1) * sizeof(uint64_t));
  int64_t* pos = (int64_t*)malloc((size_t)(m > 0 ? m : 1) * sizeof(int64_t));
  int64_t* id_at = (int64_t*)malloc((size_t)slots * sizeof(int64_t));
  if (!key || !pos || !id_at) { free(key); free(pos); free(id_at); return -1; }
  {
    int64_t i = 0;
    for (int64_t t = 0; t < n_tets; t++) {
      int nn = 0, ne = 0;
      const int (*rt)[2] = NULL;
      int32_t et;
      if (row_shape(elem_type, tets + npe * t, &nn, &ne, &rt, &et)) ne = 0;
      for (int k = 0; k < ne; k++) {
        uint64_t a = (uint64_t)tets[npe * t + rt[k][0]];
        uint64_t b = (uint64_t)tets[npe * t + rt[k][1]];
        uint64_t lo = a < b ? a : b, hi = a < b ? b : a;
        key[i] = lo * span + hi;
        pos[i++] = epe * t + k;
      }
    }
  }
  if (radix_sort_u64(m, key, pos, span * span - 1)) { free(key); free(pos); free(id_at); return -1; }
  /* leader flags by position */
  for (int64_t i = 0; i < slots; i++) id_at[i] = 0;
  for (int64_t i = 0; i < m; i++)
    if (i == 0 || key[i] != key[i - 1]) id_at[pos[i]] = 1;
  int64_t run = 0;
  for (int64_t i = 0; i < slots; i++) {
    int64_t f = id_at[i];
    id_at[i] = f ? run : -1;
    run += f;
  }
  *n_edges = run;
  int64_t lead = 0;
  for (int64_t i = 0; i < m; i++) {
    if (i == 0 || key[i] != key[i - 1]) lead = pos[i];
    int64_t id = id_at[lead];
    elem_edge[pos[i]] = (int32_t)id;
    if (edge_nodes) {
      edge_nodes[2 * id] = (int32_t)(key[i] / span);
      edge_nodes[2 * id + 1] = (int32_t)(key[i] % span);
    }
  }
  free(key);
  free(pos);
  free(id_at);
  return 0;
}

/* ---------------------------------------------------------------------------
 * DOF numbering and tree gauge.
 * ------------------------------------------------------------------------- */
static int64_t find_edge(const uint64_t* skey, const int32_t* sid, int64_t ne, uint64_t k) {
  int64_t lo = 0, hi = ne;
  while (lo < hi) {
    int64_t mid = (lo + hi) / 2;
    if (skey[mid] < k) lo = mid + 1; else hi = mid;
  }
  if (lo < ne && skey[lo] == k) return sid[lo];
  return -1;
}

int orc_dof_build(int64_t n_tets, const int32_t* tets, const int32_t* elem_edge,
                  const int32_t* edge_nodes, int64_t n_edges, int64_t n_dir,
                  const int32_t* dir_pairs, int32_t n_hole_markers, int32_t gauge,
                  int32_t* l2g, int32_t* edge_dof, int64_t* n_free,
                  int64_t* n_dofs, int32_t* root_node) {
  return orc_dof_build_typed(ORC_ELEM_TET4_EDGE, n_tets, tets, elem_edge, edge_nodes, n_edges, n_dir,
                             dir_pairs, n_hole_markers, gauge, l2g, edge_dof, n_free, n_dofs, root_node);
}

int orc_dof_build_typed(int32_t elem_type, int64_t n_tets, const int32_t* tets, const int32_t* elem_edge,
                        const int32_t* edge_nodes, int64_t n_edges, int64_t n_dir,
                        const int32_t* dir_pairs, int32_t n_hole_markers, int32_t gauge,
                        int32_t* l2g, int32_t* edge_dof, int64_t* n_free,
                        int64_t* n_dofs, int32_t* root_node) {
  int64_t E = n_edges;
  int npe, epe;
  const int (*tab)[2];
  *n_free = 0; *n_dofs = 0;
  if (root_node) *root_node = -1;
  if (elem_shape(elem_type, &npe, &epe, &tab)) return ORC_INVALID_INPUT;
  if (n_tets <= 0 || E <= 0) return ORC_INVALID_INPUT;
  int32_t maxg = 0;
  for (int64_t i = 0; i < 2 * E; i++) if (edge_nodes[i] > maxg) maxg = edge_nodes[i];
  for (int64_t i = 0; i < npe * n_tets; i++)
    if (tets[i] > maxg && (elem_type != ORC_ELEM_MIXED || i % 9 != 8)) maxg = tets[i];
  uint64_t span = (uint64_t)maxg + 1;

  /* Edge lookup by sorted node pair (GlobalEdgeIDGenerator::getGlobalEdgeID,
   * global_edge_id_generator.cpp:124-140). */
  uint64_t* skey = (uint64_t*)malloc((size_t)E * sizeof(uint64_t));
  int64_t* spay = (int64_t*)malloc((size_t)E * sizeof(int64_t));
  int32_t* sid = (int32_t*)malloc((size_t)E * sizeof(int32_t));
  char* constrained = (char*)calloc((size_t)E, 1);
  int32_t* free_of = (int32_t*)malloc((size_t)E * sizeof(int32_t));
  if (!skey || !spay || !sid || !constrained || !free_of) return -1;
  for (int64_t e = 0; e < E; e++) {
    skey[e] = (uint64_t)edge_nodes[2 * e] * span + (uint64_t)edge_nodes[2 * e + 1];
    spay[e] = e;
  }
  radix_sort_u64(E, skey, spay, span * span - 1);
  for (int64_t e = 0; e < E; e++) sid[e] = (int32_t)spay[e];
  free(spay);

  /* markConstrainedDOFs (em_dof_manager.cpp:152-243): Dirichlet node pairs
   * -> global edge IDs; pairs that are not mesh edges are skipped. */
  for (int64_t d = 0; d < n_dir; d++) {
    int32_t a = dir_pairs[2 * d], b = dir_pairs[2 * d + 1];
    if (a < 0 || b < 0 || (uint64_t)a >= span || (uint64_t)b >= span) continue;
    uint64_t lo = a < b ? a : b, hi = a < b ? b : a;
    int64_t id = find_edge(skey, sid, E, lo * span + hi);
    if (id >= 0) constrained[id] = 1;
  }
  /* assignPrenumbering + renumberFreeDOFs (em_dof_manager.cpp:91-150,
   * :245-286): for an all-vector mesh the prenumber of an edge is its global
   * ID, and the free index is the rank among unconstrained prenumbers. */
  int64_t nf = 0;
  for (int64_t e = 0; e < E; e++) free_of[e] = constrained[e] ? -1 : (int32_t)nf++;
  *n_free = nf;

  if (gauge < 0) {
    for (int64_t e = 0; e < E; e++) edge_dof[e] = free_of[e];
    *n_dofs = nf;
  } else {
    /* ---- TreeGauge::build (src/fe_em/tree_gauge.cpp:37-212) ---- */
    /* MeshGraphExtractor (mesh_graph_extractor.cpp:29-176): compact node
     * index = rank of the global node ID among referenced nodes. */
    int32_t* cidx = (int32_t*)malloc((size_t)span * sizeof(int32_t));
    for (uint64_t g = 0; g < span; g++) cidx[g] = -1;
    for (int64_t t = 0; t < n_tets; t++) {  /* nodes referenced by the elements */
      int nn = 0, ne = 0;
      const int (*rt)[2] = NULL;
      int32_t et;
      if (row_shape(elem_type, tets + npe * t, &nn, &ne, &rt, &et)) nn = 0;
      for (int a = 0; a < nn; a++)
        if (tets[npe * t + a] >= 0 && tets[npe * t + a] <= maxg) cidx[tets[npe * t + a]] = 1;
    }
    int32_t V = 0;
    for (uint64_t g = 0; g < span; g++) if (cidx[g] == 1) cidx[g] = V++;
    /* sorted adjacency with the edge of each entry */
    int64_t* aptr = (int64_t*)calloc((size_t)V + 1, sizeof(int64_t));
    int32_t* anb = (int32_t*)malloc((size_t)(2 * E) * sizeof(int32_t));
    int32_t* aed = (int32_t*)malloc((size_t)(2 * E) * sizeof(int32_t));
    for (int64_t e = 0; e < E; e++) {
      aptr[cidx[edge_nodes[2 * e]] + 1]++;
      aptr[cidx[edge_nodes[2 * e + 1]] + 1]++;
    }
    for (int32_t v = 0; v < V; v++) aptr[v + 1] += aptr[v];
    int64_t* fill = (int64_t*)malloc((size_t)V * sizeof(int64_t));
    for (int32_t v = 0; v < V; v++) fill[v] = aptr[v];
    for (int64_t e = 0; e < E; e++) {
      int32_t u = cidx[edge_nodes[2 * e]], w = cidx[edge_nodes[2 * e + 1]];
      anb[fill[u]] = w; aed[fill[u]++] = (int32_t)e;
      anb[fill[w]] = u; aed[fill[w]++] = (int32_t)e;
    }
    free(fill);
    for (int32_t v = 0; v < V; v++) { /* insertion sort by neighbour */
      for (int64_t i = aptr[v] + 1; i < aptr[v + 1]; i++) {
        int32_t nb = anb[i], ed = aed[i];
        int64_t j = i - 1;
        while (j >= aptr[v] && anb[j] > nb) { anb[j + 1] = anb[j]; aed[j + 1] = aed[j]; j--; }
        anb[j + 1] = nb; aed[j + 1] = ed;
      }
    }
    /* selectRootNode DIRICHLET_BOUNDARY (spanning_tree.cpp:517-540): smaller
     * compact endpoint of the smallest constrained edge ID, else node 0. */
    int32_t root = 0;
    for (int64_t e = 0; e < E; e++)
      if (constrained[e]) { root = cidx[edge_nodes[2 * e]]; break; }
    if (root_node) *root_node = root;

    char* tree = (char*)calloc((size_t)E, 1);
    char* visited = (char*)calloc((size_t)V, 1);
    int32_t* queue = (int32_t*)malloc((size_t)V * sizeof(int32_t));
    int32_t* dn = (int32_t*)malloc(64 * sizeof(int32_t));
    int32_t* de = (int32_t*)malloc(64 * sizeof(int32_t));
    int32_t* nn = (int32_t*)malloc(64 * sizeof(int32_t));
    int32_t* ne_ = (int32_t*)malloc(64 * sizeof(int32_t));
    int64_t cap = 64;
    int64_t qh = 0, qt = 0;
    visited[root] = 1;
    queue[qt++] = root;
    if (gauge == ORC_GAUGE_REF) {
      /* buildBFSTreeWithBoundaryPriority (spanning_tree.cpp:295-416): per
       * dequeued node, unvisited neighbours over constrained edges are
       * enqueued first, then the others, each in ascending index order. */
      while (qh < qt) {
        int32_t u = queue[qh++];
        int64_t deg = aptr[u + 1] - aptr[u];
        if (deg > cap) {
          cap = deg;
          dn = (int32_t*)realloc(dn, cap * sizeof(int32_t));
          de = (int32_t*)realloc(de, cap * sizeof(int32_t));
          nn = (int32_t*)realloc(nn, cap * sizeof(int32_t));
          ne_ = (int32_t*)realloc(ne_, cap * sizeof(int32_t));
        }
        int64_t nd = 0, nnn = 0;
        for (int64_t i = aptr[u]; i < aptr[u + 1]; i++) {
          int32_t v = anb[i];
          if (visited[v]) continue;
          if (constrained[aed[i]]) { dn[nd] = v; de[nd++] = aed[i]; }
          else { nn[nnn] = v; ne_[nnn++] = aed[i]; }
        }
        for (int64_t i = 0; i < nd; i++)
          if (!visited[dn[i]]) { visited[dn[i]] = 1; tree[de[i]] = 1; queue[qt++] = dn[i]; }
        for (int64_t i = 0; i < nnn; i++)
          if (!visited[nn[i]]) { visited[nn[i]] = 1; tree[ne_[i]] = 1; queue[qt++] = nn[i]; }
      }
    } else {
      /* boundary_first (this build's corrected gauge): phase 1 spans the
       * constrained-edge subgraph by BFS from the root; phase 2 continues a
       * plain BFS over all edges from every node reached so far, in visit
       * order.  Each unconstrained node then owns exactly one tree edge. */
      while (qh < qt) {
        int32_t u = queue[qh++];
        for (int64_t i = aptr[u]; i < aptr[u + 1]; i++) {
          int32_t v = anb[i];
          if (!visited[v] && constrained[aed[i]]) { visited[v] = 1; tree[aed[i]] = 1; queue[qt++] = v; }
        }
      }
      /* constrained subgraph components not reached from the root */
      for (int64_t e = 0; e < E; e++) {
        if (!constrained[e]) continue;
        int32_t s0 = cidx[edge_nodes[2 * e]];
        if (visited[s0]) continue;
        visited[s0] = 1; queue[qt++] = s0;
        while (qh < qt) {
          int32_t u = queue[qh++];
          for (int64_t i = aptr[u]; i < aptr[u + 1]; i++) {
            int32_t v = anb[i];
            if (!visited[v] && constrained[aed[i]]) { visited[v] = 1; tree[aed[i]] = 1; queue[qt++] = v; }
          }
        }
      }
      qh = 0;
      while (qh < qt) {
        int32_t u = queue[qh++];
        for (int64_t i = aptr[u]; i < aptr[u + 1]; i++) {
          int32_t v = anb[i];
          if (!visited[v]) { visited[v] = 1; tree[aed[i]] = 1; queue[qt++] = v; }
        }
      }
    }
    /* remaining components: plain BFS from the lowest unvisited index
     * (spanning_tree.cpp:418-445) */
    for (int32_t s = 0; s < V; s++) {
      if (visited[s]) continue;
      visited[s] = 1;
      qh = qt = 0;
      queue[qt++] = s;
      while (qh < qt) {
        int32_t u = queue[qh++];
        for (int64_t i = aptr[u]; i < aptr[u + 1]; i++) {
          int32_t v = anb[i];
          if (!visited[v]) { visited[v] = 1; tree[aed[i]] = 1; queue[qt++] = v; }
        }
      }
    }
    /* MultiConnectedDomainDetector::selectCirculationDOFs
     * (multi_connected_domain.cpp:190-232): evenly spaced picks from the
     * ascending cotree list (before constrained edges are promoted). */
    char* circ = (char*)calloc((size_t)E, 1);
    int64_t n_cot = 0;
    for (int64_t e = 0; e < E; e++) if (!tree[e]) n_cot++;
    if (n_hole_markers > 0 && n_cot > 0) {
      int64_t pick = n_hole_markers < n_cot ? n_hole_markers : n_cot;
      int32_t* cot = (int32_t*)malloc((size_t)n_cot * sizeof(int32_t));
      int64_t c = 0;
      for (int64_t e = 0; e < E; e++) if (!tree[e]) cot[c++] = (int32_t)e;
      for (int64_t i = 0; i < pick; i++) {
        int64_t idx = (i * n_cot) / pick;
        if (idx > n_cot - 1) idx = n_cot - 1;
        circ[cot[idx]] = 1;
      }
      free(cot);
    }
    /* classifyEdges + buildReducedMapping (tree_gauge.cpp:159-212): final
     * cotree = cotree minus constrained minus circulation; reduced index =
     * ascending edge ID rank, then circulation edges not yet numbered. */
    int32_t* red = (int32_t*)malloc((size_t)E * sizeof(int32_t));
    int64_t nr = 0;
    for (int64_t e = 0; e < E; e++) {
      red[e] = -1;
      if (!tree[e] && !constrained[e] && !circ[e]) red[e] = (int32_t)nr++;
    }
    for (int64_t e = 0; e < E; e++)
      if (circ[e] && red[e] < 0) red[e] = (int32_t)nr++;
    /* renumberVectorDOFsWithTreeGauge (em_dof_manager.cpp:501-626): only
     * free entries are rewritten; cotree or circulation edges take their
     * reduced index, the rest become -1. */
    for (int64_t e = 0; e < E; e++) {
      if (free_of[e] < 0) { edge_dof[e] = -1; continue; }
      int cot_or_circ = (!tree[e] && !constrained[e] && !circ[e]) || circ[e];
      edge_dof[e] = cot_or_circ ? red[e] : -1;
    }
    *n_dofs = nr;
    free(red); free(circ); free(tree); free(visited); free(queue);
    free(dn); free(de); free(nn); free(ne_);
    free(aptr); free(anb); free(aed); free(cidx);
  }
  /* buildVectorElementMapping (em_dof_manager.cpp:353-393) */
  for (int64_t i = 0; i < epe * n_tets; i++) l2g[i] = elem_edge[i] < 0 ? -1 : edge_dof[elem_edge[i]];
  free(skey); free(sid); free(constrained); free(free_of);
  return 0;
}

/* ---------------------------------------------------------------------------
 * Element integration (MagneticVector3DIntegrator, intended formulas).
 * ------------------------------------------------------------------------- */
static void ref_basis(int k, const double* xi, double* w) {
  /* evalTet4Edge (nedelec_element.cpp:411-459) */
  double l1 = xi[0], l2 = xi[1], l3 = xi[2], l4 = 1.0 - xi[0] - xi[1] - xi[2];
  switch (k) {
    case 0: w[0] = l2; w[1] = -l1; w[2] = 0.0; break;
    case 1: w[0] = 0.0; w[1] = l3; w[2] = -l2; break;
    case 2: w[0] = -l3; w[1] = 0.0; w[2] = l1; break;
    case 3: w[0] = l4 + l1; w[1] = l1; w[2] = l1; break;
    case 4: w[0] = l2; w[1] = l4 + l2; w[2] = l2; break;
    default: w[0] = l3; w[1] = l3; w[2] = l4 + l3; break;
  }
}

static void source_at(const orc_source* src, int32_t n_src, const double* x, double* js) {
  js[0] = js[1] = js[2] = 0.0;
  for (int32_t s = 0; s < n_src; s++) {
    const double* p = src[s].p;
    int in = 0;
    if (src[s].kind == ORC_SRC_BOX) {
      in = x[0] > p[0] && x[0] < p[1] && x[1] > p[2] && x[1] < p[3] && x[2] > p[4] && x[2] < p[5];
    } else if (src[s].kind == ORC_SRC_ANNULUS_Z) {
      double dx = x[0] - p[0], dy = x[1] - p[1];
      double r = sqrt(dx * dx + dy * dy);
      in = r > p[2] && r < p[3] && x[2] > p[4] && x[2] < p[5];
    }
    if (in) { js[0] += src[s].j[0]; js[1] += src[s].j[1]; js[2] += src[s].j[2]; }
  }
}

void orc_element(const double* X, double nu, double sigma, const orc_source* src,
                 int32_t n_src, int32_t flags, double* Ke, double* Me, double* Fe) {
  /* GaussQuadrature::getTet4Points(4) intended points (gauss_quadrature.cpp:
   * 198-219), weight 1/24 each. */
  const double a = (5.0 - sqrt(5.0)) / 20.0, b = (5.0 + 3.0 * sqrt(5.0)) / 20.0;
  double qp[4][3] = {{a, a, b}, {a, b, a}, {b, a, a}, {a, a, a}};
  int nq = 4;
  if (flags & ORC_FLAG_QUAD3_LITERAL) { qp[2][0] = a; qp[2][1] = a; qp[2][2] = a; nq = 3; }
  const double w = 1.0 / 24.0;
  for (int i = 0; i < 36; i++) { Ke[i] = 0.0; if (Me) Me[i] = 0.0; }
  for (int i = 0; i < 6; i++) if (Fe) Fe[i] = 0.0;
  /* calcJacobian with the TET4 Lagrange gradients (shape_function_base.hpp:
   * 335-364, lagrange_element.cpp:658-683): columns x0-x3, x1-x3, x2-x3. */
  double J[3][3];
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) J[r][c] = X[3 * c + r] - X[9 + r];
  double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
               J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
               J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
  double adet = fabs(det);
  if (adet < 1e-15) return; /* magnetic_vector_3d_integrator.cpp:169 */
  double inv[3][3]; /* J^-1 */
  inv[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
  inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
  inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
  inv[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / det;
  inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
  inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
  inv[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
  inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
  inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
  /* physical curls: J curl_ref / detJ (nedelec_element.cpp:246-247) */
  double c[6][3];
  for (int k = 0; k < 6; k++)
    for (int r = 0; r < 3; r++)
      c[k][r] = (J[r][0] * CURL_REF[k][0] + J[r][1] * CURL_REF[k][1] + J[r][2] * CURL_REF[k][2]) / det;
  for (int q = 0; q < nq; q++) {
    /* computeStiffnessMatrix (magnetic_vector_3d_integrator.cpp:139-229) */
    double wf = w * adet * nu;
    for (int i = 0; i < 6; i++)
      for (int j = i; j < 6; j++) {
        double d = c[i][0] * c[j][0] + c[i][1] * c[j][1] + c[i][2] * c[j][2];
        Ke[6 * i + j] += wf * d;
        if (j != i) Ke[6 * j + i] = Ke[6 * i + j];
      }
    /* basis values for M and F: covariant map J^-T W_ref */
    double W[6][3];
    for (int k = 0; k < 6; k++) {
      double wr[3];
      ref_basis(k, qp[q], wr);
      for (int r = 0; r < 3; r++) {
        W[k][r] = inv[0][r] * wr[0] + inv[1][r] * wr[1] + inv[2][r] * wr[2];
        if (flags & ORC_FLAG_PIOLA_LITERAL) W[k][r] /= det;
      }
    }
    if (Me && (flags & ORC_FLAG_MASS) && sigma > 0.0) {
      /* computeMassMatrix (:233-323) */
      double wm = w * adet * sigma;
      for (int i = 0; i < 6; i++)
        for (int j = i; j < 6; j++) {
          double d = W[i][0] * W[j][0] + W[i][1] * W[j][1] + W[i][2] * W[j][2];
          Me[6 * i + j] += wm * d;
          if (j != i) Me[6 * j + i] = Me[6 * i + j];
        }
    }
    if (Fe && n_src > 0) {
      /* F_i = int W_i . J_s (theory formula at :353), physical position by
       * the TET4 map N0=xi, N1=eta, N2=zeta, N3=1-xi-eta-zeta (:437-483). */
      double N[4] = {qp[q][0], qp[q][1], qp[q][2], 1.0 - qp[q][0] - qp[q][1] - qp[q][2]};
      double x[3];
      for (int r = 0; r < 3; r++) x[r] = N[0] * X[r] + N[1] * X[3 + r] + N[2] * X[6 + r] + N[3] * X[9 + r];
      double js[3];
      source_at(src, n_src, x, js);
      double wfj = w * adet;
      for (int i = 0; i < 6; i++) Fe[i] += wfj * (W[i][0] * js[0] + W[i][1] * js[1] + W[i][2] * js[2]);
    }
  }
}

void orc_edge_signs(const int32_t* tet, int32_t* s) {
  for (int k = 0; k < 6; k++) {
    int32_t ga = tet[NED_EDGE[k][0]], gb = tet[NED_EDGE[k][1]];
    s[k] = gb < ga ? 1 : -1;
  }
}

/* ---------------------------------------------------------------------------
 * HEX8_EDGE element (MagneticVector3DIntegrator with HEX8_EDGE, intended
 * formulas: 2x2x2 Gauss-Legendre, GaussQuadrature::getHex8Points,
 * gauss_quadrature.cpp:247-276; the reference calls getPoints(HEX8_EDGE),
 * which returns no points (:36-60), so its literal K_e is zero as for tets).
 * ------------------------------------------------------------------------- */
void orc_hex_basis(int k, const double* x, double* w) {
  /* evalHex8Edge (nedelec_element.cpp:519-615) */
  const double xi = x[0], eta = x[1], zeta = x[2];
  w[0] = w[1] = w[2] = 0.0;
  switch (k) {
    case 0: w[0] = 0.5 * (1.0 - eta) * (1.0 - zeta); break;
    case 1: w[1] = 0.5 * (1.0 + xi) * (1.0 - zeta); break;
    case 2: w[0] = -0.5 * (1.0 + eta) * (1.0 - zeta); break;
    case 3: w[1] = -0.5 * (1.0 - xi) * (1.0 - zeta); break;
    case 4: w[0] = 0.5 * (1.0 - eta) * (1.0 + zeta); break;
    case 5: w[1] = 0.5 * (1.0 + xi) * (1.0 + zeta); break;
    case 6: w[0] = -0.5 * (1.0 + eta) * (1.0 + zeta); break;
    case 7: w[1] = -0.5 * (1.0 - xi) * (1.0 + zeta); break;
    case 8: w[2] = 0.5 * (1.0 - xi) * (1.0 - eta); break;
    case 9: w[2] = 0.5 * (1.0 + xi) * (1.0 - eta); break;
    case 10: w[2] = 0.5 * (1.0 + xi) * (1.0 + eta); break;
    default: w[2] = 0.5 * (1.0 - xi) * (1.0 + eta); break;
  }
}

void orc_hex_curl(int k, const double* x, double* c) {
  /* Reference-domain curl of orc_hex_basis, differentiated by hand:
   * curl(f e_xi) = (0, df/dzeta, -df/deta), curl(f e_eta) = (-df/dzeta, 0, df/dxi),
   * curl(f e_zeta) = (df/deta, -df/dxi, 0).  Equals curlHex8Edge
   * (nedelec_element.cpp:618-720) except at edges 2, 3, 6, 7, where that
   * function has sign and component errors. */
  const double xi = x[0], eta = x[1], zeta = x[2];
  c[0] = c[1] = c[2] = 0.0;
  switch (k) {
    case 0: c[1] = -0.5 * (1.0 - eta); c[2] = 0.5 * (1.0 - zeta); break;
    case 1: c[0] = 0.5 * (1.0 + xi); c[2] = 0.5 * (1.0 - zeta); break;
    case 2: c[1] = 0.5 * (1.0 + eta); c[2] = 0.5 * (1.0 - zeta); break;
    case 3: c[0] = -0.5 * (1.0 - xi); c[2] = 0.5 * (1.0 - zeta); break;
    case 4: c[1] = 0.5 * (1.0 - eta); c[2] = 0.5 * (1.0 + zeta); break;
    case 5: c[0] = -0.5 * (1.0 + xi); c[2] = 0.5 * (1.0 + zeta); break;
    case 6: c[1] = -0.5 * (1.0 + eta); c[2] = 0.5 * (1.0 + zeta); break;
    case 7: c[0] = 0.5 * (1.0 - xi); c[2] = 0.5 * (1.0 + zeta); break;
    case 8: c[0] = -0.5 * (1.0 - xi); c[1] = 0.5 * (1.0 - eta); break;
    case 9: c[0] = -0.5 * (1.0 + xi); c[1] = -0.5 * (1.0 - eta); break;
    case 10: c[0] = 0.5 * (1.0 + xi); c[1] = -0.5 * (1.0 + eta); break;
    default: c[0] = 0.5 * (1.0 - xi); c[1] = 0.5 * (1.0 + eta); break;
  }
}

void orc_hex_jacobian(const double* X, const double* x, double* J, double* det) {
  /* calcJacobian with the HEX8 gradients (evalHex8GradN, lagrange_element.cpp:
   * 787-846): J[r][c] = sum_a X_a[r] dN_a/dx_c. */
  for (int i = 0; i < 9; i++) J[i] = 0.0;
  for (int a = 0; a < 8; a++) {
    double l[3], dn[3];
    for (int c = 0; c < 3; c++) l[c] = 1.0 + HEX_NODE[a][c] * x[c];
    dn[0] = 0.125 * HEX_NODE[a][0] * l[1] * l[2];
    dn[1] = 0.125 * HEX_NODE[a][1] * l[0] * l[2];
    dn[2] = 0.125 * HEX_NODE[a][2] * l[0] * l[1];
    for (int r = 0; r < 3; r++)
      for (int c = 0; c < 3; c++) J[3 * r + c] += X[3 * a + r] * dn[c];
  }
  *det = J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) +
         J[2] * (J[3] * J[7] - J[4] * J[6]);
}

void orc_element_hex(const double* X, double nu, double sigma, const orc_source* src,
                     int32_t n_src, int32_t flags, double* Ke, double* Me, double* Fe) {
  const double g = 1.0 / sqrt(3.0);
  for (int i = 0; i < 144; i++) { Ke[i] = 0.0; if (Me) Me[i] = 0.0; }
  if (Fe) for (int i = 0; i < 12; i++) Fe[i] = 0.0;
  for (int q = 0; q < 8; q++) {
    /* getHex8Points order: i (xi) outermost, then eta, then zeta; weight 1 */
    const double x[3] = {(q & 4) ? g : -g, (q & 2) ? g : -g, (q & 1) ? g : -g};
    double J[9], det;
    orc_hex_jacobian(X, x, J, &det);
    const double adet = fabs(det);
    if (adet < 1e-15) continue; /* magnetic_vector_3d_integrator.cpp:169-176 */
    double inv[3][3];
    inv[0][0] = (J[4] * J[8] - J[5] * J[7]) / det;
    inv[0][1] = (J[2] * J[7] - J[1] * J[8]) / det;
    inv[0][2] = (J[1] * J[5] - J[2] * J[4]) / det;
    inv[1][0] = (J[5] * J[6] - J[3] * J[8]) / det;
    inv[1][1] = (J[0] * J[8] - J[2] * J[6]) / det;
    inv[1][2] = (J[2] * J[3] - J[0] * J[5]) / det;
    inv[2][0] = (J[3] * J[7] - J[4] * J[6]) / det;
    inv[2][1] = (J[1] * J[6] - J[0] * J[7]) / det;
    inv[2][2] = (J[0] * J[4] - J[1] * J[3]) / det;
    double c[12][3], W[12][3];
    for (int k = 0; k < 12; k++) {
      double cr[3], wr[3];
      orc_hex_curl(k, x, cr);
      orc_hex_basis(k, x, wr);
      for (int r = 0; r < 3; r++) {
        /* J curl_ref / detJ (nedelec_element.cpp:242-247); J^-T W_ref */
        c[k][r] = (J[3 * r] * cr[0] + J[3 * r + 1] * cr[1] + J[3 * r + 2] * cr[2]) / det;
        W[k][r] = inv[0][r] * wr[0] + inv[1][r] * wr[1] + inv[2][r] * wr[2];
        if (flags & ORC_FLAG_PIOLA_LITERAL) W[k][r] /= det;
      }
    }
    const double wf = adet * nu;
    for (int i = 0; i < 12; i++)
      for (int j = i; j < 12; j++) {
        Ke[12 * i + j] += wf * (c[i][0] * c[j][0] + c[i][1] * c[j][1] + c[i][2] * c[j][2]);
        if (j != i) Ke[12 * j + i] = Ke[12 * i + j];
      }
    if (Me && (flags & ORC_FLAG_MASS) && sigma > 0.0) {
      const double wm = adet * sigma;
      for (int i = 0; i < 12; i++)
        for (int j = i; j < 12; j++) {
          Me[12 * i + j] += wm * (W[i][0] * W[j][0] + W[i][1] * W[j][1] + W[i][2] * W[j][2]);
          if (j != i) Me[12 * j + i] = Me[12 * i + j];
        }
    }
    if (Fe && n_src > 0) {
      /* physical position by the HEX8 map (computePhysicalPosition, :437-483) */
      double p[3] = {0.0, 0.0, 0.0};
      for (int a = 0; a < 8; a++) {
        double N = 0.125 * (1.0 + HEX_NODE[a][0] * x[0]) * (1.0 + HEX_NODE[a][1] * x[1]) *
                   (1.0 + HEX_NODE[a][2] * x[2]);
        for (int r = 0; r < 3; r++) p[r] += N * X[3 * a + r];
      }
      double js[3];
      source_at(src, n_src, p, js);
      for (int i = 0; i < 12; i++) Fe[i] += adet * (W[i][0] * js[0] + W[i][1] * js[1] + W[i][2] * js[2]);
    }
  }
}

void orc_edge_signs_hex(const int32_t* hex, int32_t* s) {
  for (int k = 0; k < 12; k++) s[k] = hex[HEX_EDGE[k][0]] < hex[HEX_EDGE[k][1]] ? 1 : -1;
}

/* ---------------------------------------------------------------------------
 * PRISM6_EDGE and PYRAMID5_EDGE elements.  The reference calls
 * getPoints(PRISM6_EDGE / PYRAMID5_EDGE), which returns no points
 * (gauss_quadrature.cpp:36-60): its literal K_e is zero.  Intended
 * formulas, restated here independently of the library's kernels:
 *  - prism: PRISM6 Lagrange map (lagrange_element.cpp:458-522: node a < 3
 *    has area coordinate L_a, L_0 = xi, L_1 = eta, L_2 = 1 - xi - eta, at
 *    zeta = -1, node a + 3 the same at zeta = +1), the basis forms of
 *    evalPrism6Edge (nedelec_element.cpp:744-792) placed on their own edges
 *    with unit circulation, the reference's 6-point rule
 *    (gauss_quadrature.cpp:304-345);
 *  - pyramid: PYRAMID5 Lagrange map (lagrange_element.cpp:51-135: base
 *    corners N_a = (1 - zeta) P_a(xi, eta), apex N_4 = zeta, zeta in
 *    [0, 1]), a conforming basis (base edges 1/4 (1 +- x_perp)(1 - zeta)^2
 *    along the edge, slant edges N_a grad N_4 - N_4 grad N_a), 2 x 2 x 3
 *    Gauss-Legendre points on [-1, 1]^2 x [0, 1].
 * ------------------------------------------------------------------------- */
typedef struct {
  int npe, epe, nq;
  void (*point)(int q, double* x, double* w);
  void (*grad)(int a, const double* x, double* d);     /* dN_a / d(xi, eta, zeta) */
  double (*value)(int a, const double* x);              /* N_a */
  void (*basis)(int k, const double* x, double* w);    /* W_k, reference components */
  void (*curl)(int k, const double* x, double* c);     /* reference curl of W_k */
} orc_shape;

static const double PR_DL[3][2] = {{1.0, 0.0}, {0.0, 1.0}, {-1.0, -1.0}};
static double pr_l(int a, const double* x) { return a == 0 ? x[0] : a == 1 ? x[1] : 1.0 - x[0] - x[1]; }
static void pr_point(int q, double* x, double* w) {
  static const double tri[3][2] = {{1.0 / 6.0, 1.0 / 6.0}, {2.0 / 3.0, 1.0 / 6.0}, {1.0 / 6.0, 2.0 / 3.0}};
  const double g = 1.0 / sqrt(3.0);
  x[0] = tri[q % 3][0];
  x[1] = tri[q % 3][1];
  x[2] = q < 3 ? -g : g; /* zeta outer loop, triangle points inner */
  *w = 1.0 / 6.0;
}
static double pr_value(int a, const double* x) {
  return pr_l(a % 3, x) * (a < 3 ? 0.5 * (1.0 - x[2]) : 0.5 * (1.0 + x[2]));
}
static void pr_grad(int a, const double* x, double* d) {
  const double h = a < 3 ? 0.5 * (1.0 - x[2]) : 0.5 * (1.0 + x[2]);
  d[0] = h * PR_DL[a % 3][0];
  d[1] = h * PR_DL[a % 3][1];
  d[2] = (a < 3 ? -0.5 : 0.5) * pr_l(a % 3, x);
}
static void pr_basis(int k, const double* x, double* w) {
  if (k >= 6) { w[0] = 0.0; w[1] = 0.0; w[2] = 0.5 * pr_l(k - 6, x); return; }
  const int a = PRISM_EDGE[k][0] % 3, b = PRISM_EDGE[k][1] % 3;
  const double h = k < 3 ? 0.5 * (1.0 - x[2]) : 0.5 * (1.0 + x[2]);
  for (int c = 0; c < 2; c++) w[c] = h * (pr_l(a, x) * PR_DL[b][c] - pr_l(b, x) * PR_DL[a][c]);
  w[2] = 0.0;
}
static void pr_curl(int k, const double* x, double* c) {
  if (k >= 6) { c[0] = 0.5 * PR_DL[k - 6][1]; c[1] = -0.5 * PR_DL[k - 6][0]; c[2] = 0.0; return; }
  const int a = PRISM_EDGE[k][0] % 3, b = PRISM_EDGE[k][1] % 3;
  const double h = k < 3 ? 0.5 * (1.0 - x[2]) : 0.5 * (1.0 + x[2]), dh = k < 3 ? -0.5 : 0.5;
  double wv[2];
  for (int i = 0; i < 2; i++) wv[i] = pr_l(a, x) * PR_DL[b][i] - pr_l(b, x) * PR_DL[a][i];
  /* grad(h) x w + h curl(w), curl(w) = 2 grad L_a x grad L_b */
  c[0] = -dh * wv[1];
  c[1] = dh * wv[0];
  c[2] = 2.0 * h * (PR_DL[a][0] * PR_DL[b][1] - PR_DL[a][1] * PR_DL[b][0]);
}

static const double PY_C[4][2] = {{-1.0, -1.0}, {1.0, -1.0}, {1.0, 1.0}, {-1.0, 1.0}};
static void py_point(int q, double* x, double* w) {
  const double g = 1.0 / sqrt(3.0), s = sqrt(0.6);
  const double zt[3] = {-s, 0.0, s}, zw[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
  x[0] = (q / 6) ? g : -g;
  x[1] = ((q / 3) % 2) ? g : -g;
  x[2] = 0.5 * (1.0 + zt[q % 3]);
  *w = 0.5 * zw[q % 3];
}
static double py_p(int a, const double* x) { return 0.25 * (1.0 + PY_C[a][0] * x[0]) * (1.0 + PY_C[a][1] * x[1]); }
static double py_value(int a, const double* x) { return a == 4 ? x[2] : (1.0 - x[2]) * py_p(a, x); }
static void py_grad(int a, const double* x, double* d) {
  if (a == 4) { d[0] = 0.0; d[1] = 0.0; d[2] = 1.0; return; }
  d[0] = (1.0 - x[2]) * 0.25 * PY_C[a][0] * (1.0 + PY_C[a][1] * x[1]);
  d[1] = (1.0 - x[2]) * 0.25 * PY_C[a][1] * (1.0 + PY_C[a][0] * x[0]);
  d[2] = -py_p(a, x);
}
static void py_basis(int k, const double* x, double* w) {
  const double r2 = (1.0 - x[2]) * (1.0 - x[2]);
  w[0] = w[1] = w[2] = 0.0;
  if (k < 4) {
    /* along +-e_xi (edges 0, 2) or +-e_eta (1, 3), vanishing on the opposite side */
    const int axis = k & 1;
    const double dir = PY_C[PYR_EDGE[k][1]][axis] - PY_C[PYR_EDGE[k][0]][axis]; /* +-2 */
    const double side = PY_C[PYR_EDGE[k][0]][1 - axis];                           /* fixed coordinate */
    w[axis] = 0.125 * dir * (1.0 + side * x[1 - axis]) * r2;
    return;
  }
  const int a = k - 4;
  double d[3];
  py_grad(a, x, d);
  /* N_a grad N_4 - N_4 grad N_a */
  const double na = py_value(a, x), n4 = x[2];
  w[0] = -n4 * d[0];
  w[1] = -n4 * d[1];
  w[2] = na - n4 * d[2];
}
static void py_curl(int k, const double* x, double* c) {
  const double r = 1.0 - x[2];
  if (k < 4) {
    const int axis = k & 1;
    const double dir = PY_C[PYR_EDGE[k][1]][axis] - PY_C[PYR_EDGE[k][0]][axis];
    const double side = PY_C[PYR_EDGE[k][0]][1 - axis];
    const double f = 0.125 * dir * (1.0 + side * x[1 - axis]); /* W_axis = f r^2 */
    const double df = 0.125 * dir * side;                      /* d f / d x_other */
    /* curl (0-form components): axis 0: (0, dW0/dz, -dW0/dy); axis 1: (-dW1/dz, 0, dW1/dx) */
    if (axis == 0) { c[0] = 0.0; c[1] = -2.0 * f * r; c[2] = -df * r * r; }
    else { c[0] = 2.0 * f * r; c[1] = 0.0; c[2] = df * r * r; }
    return;
  }
  /* 2 grad N_a x grad N_4 */
  double d[3];
  py_grad(k - 4, x, d);
  c[0] = 2.0 * d[1];
  c[1] = -2.0 * d[0];
  c[2] = 0.0;
}

static const orc_shape ORC_PRISM = {6, 9, 6, pr_point, pr_grad, pr_value, pr_basis, pr_curl};
static const orc_shape ORC_PYRAMID = {5, 8, 12, py_point, py_grad, py_value, py_basis, py_curl};

/* K_e, M_e, F_e of a quadrature element (the HEX8_EDGE transforms above):
 * curl_phys = J curl_ref / det, W_phys = J^-T W_ref (divided by det once
 * more under ORC_FLAG_PIOLA_LITERAL), weights w_q |det J|. */
static void orc_element_shape(const orc_shape* S, const double* X, double nu, double sigma,
                              const orc_source* src, int32_t n_src, int32_t flags, double* Ke, double* Me,
                              double* Fe) {
  const int E = S->epe;
  for (int i = 0; i < E * E; i++) { Ke[i] = 0.0; Me[i] = 0.0; }
  for (int i = 0; i < E; i++) Fe[i] = 0.0;
  for (int q = 0; q < S->nq; q++) {
    double x[3], wq, J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    S->point(q, x, &wq);
    for (int a = 0; a < S->npe; a++) {
      double d[3];
      S->grad(a, x, d);
      for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) J[3 * r + c] += X[3 * a + r] * d[c];
    }
    const double det = J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) +
                       J[2] * (J[3] * J[7] - J[4] * J[6]);
    const double adet = fabs(det);
    if (adet < 1e-15) continue;
    double inv[3][3];
    inv[0][0] = (J[4] * J[8] - J[5] * J[7]) / det;
    inv[0][1] = (J[2] * J[7] - J[1] * J[8]) / det;
    inv[0][2] = (J[1] * J[5] - J[2] * J[4]) / det;
    inv[1][0] = (J[5] * J[6] - J[3] * J[8]) / det;
    inv[1][1] = (J[0] * J[8] - J[2] * J[6]) / det;
    inv[1][2] = (J[2] * J[3] - J[0] * J[5]) / det;
    inv[2][0] = (J[3] * J[7] - J[4] * J[6]) / det;
    inv[2][1] = (J[1] * J[6] - J[0] * J[7]) / det;
    inv[2][2] = (J[0] * J[4] - J[1] * J[3]) / det;
    double c[12][3], W[12][3];
    for (int k = 0; k < E; k++) {
      double cr[3], wr[3];
      S->curl(k, x, cr);
      S->basis(k, x, wr);
      for (int r = 0; r < 3; r++) {
        c[k][r] = (J[3 * r] * cr[0] + J[3 * r + 1] * cr[1] + J[3 * r + 2] * cr[2]) / det;
        W[k][r] = inv[0][r] * wr[0] + inv[1][r] * wr[1] + inv[2][r] * wr[2];
        if (flags & ORC_FLAG_PIOLA_LITERAL) W[k][r] /= det;
      }
    }
    for (int i = 0; i < E; i++)
      for (int j = 0; j < E; j++) {
        Ke[E * i + j] += wq * adet * nu * (c[i][0] * c[j][0] + c[i][1] * c[j][1] + c[i][2] * c[j][2]);
        if ((flags & ORC_FLAG_MASS) && sigma > 0.0)
          Me[E * i + j] += wq * adet * sigma * (W[i][0] * W[j][0] + W[i][1] * W[j][1] + W[i][2] * W[j][2]);
      }
    if (n_src > 0) {
      double p[3] = {0.0, 0.0, 0.0}, js[3];
      for (int a = 0; a < S->npe; a++) {
        const double N = S->value(a, x);
        for (int r = 0; r < 3; r++) p[r] += N * X[3 * a + r];
      }
      source_at(src, n_src, p, js);
      for (int i = 0; i < E; i++) Fe[i] += wq * adet * (W[i][0] * js[0] + W[i][1] * js[1] + W[i][2] * js[2]);
    }
  }
}

/* Reference-element checks for the tests: circulation of W_k along edge e
 * (midpoint rule, n segments, reference coordinates; the pyramid's slant
 * edges are the collapsed cube's vertical edges) and the largest difference
 * between grad N_a and the edge-basis combination sum_k (N_a(b_k) -
 * N_a(a_k)) W_k at point x. */
static void shape_node(int32_t elem_type, int a, double* x) {
  if (elem_type == ORC_ELEM_PRISM6_EDGE) {
    const double v[3][2] = {{1.0, 0.0}, {0.0, 1.0}, {0.0, 0.0}};
    x[0] = v[a % 3][0]; x[1] = v[a % 3][1]; x[2] = a < 3 ? -1.0 : 1.0;
  } else {
    x[0] = a == 4 ? 0.0 : PY_C[a][0]; x[1] = a == 4 ? 0.0 : PY_C[a][1]; x[2] = a == 4 ? 1.0 : 0.0;
  }
}
double orc_shape_circulation(int32_t elem_type, int k, int e, int n) {
  const orc_shape* S = elem_type == ORC_ELEM_PRISM6_EDGE ? &ORC_PRISM : &ORC_PYRAMID;
  const int (*tab)[2] = elem_type == ORC_ELEM_PRISM6_EDGE ? PRISM_EDGE : PYR_EDGE;
  double xa[3], xb[3], s = 0.0;
  shape_node(elem_type, tab[e][0], xa);
  shape_node(elem_type, tab[e][1], xb);
  if (elem_type == ORC_ELEM_PYRAMID5_EDGE && tab[e][1] == 4) { xb[0] = xa[0]; xb[1] = xa[1]; }
  (void)S;
  for (int i = 0; i < n; i++) {
    double x[3], w[3];
    const double t = (i + 0.5) / n;
    for (int c = 0; c < 3; c++) x[c] = xa[c] + t * (xb[c] - xa[c]);
    S->basis(k, x, w);
    for (int c = 0; c < 3; c++) s += w[c] * (xb[c] - xa[c]) / n;
  }
  return s;
}
double orc_shape_grad_residual(int32_t elem_type, const double* x) {
  const orc_shape* S = elem_type == ORC_ELEM_PRISM6_EDGE ? &ORC_PRISM : &ORC_PYRAMID;
  const int (*tab)[2] = elem_type == ORC_ELEM_PRISM6_EDGE ? PRISM_EDGE : PYR_EDGE;
  double worst = 0.0;
  for (int a = 0; a < S->npe; a++) {
    double g[3], sum[3] = {0.0, 0.0, 0.0};
    S->grad(a, x, g);
    for (int k = 0; k < S->epe; k++) {
      double w[3];
      const double coef = (tab[k][1] == a) - (tab[k][0] == a);
      S->basis(k, x, w);
      for (int r = 0; r < 3; r++) sum[r] += coef * w[r];
    }
    for (int r = 0; r < 3; r++) worst = fmax(worst, fabs(g[r] - sum[r]));
  }
  return worst;
}

/* ---------------------------------------------------------------------------
 * CSR pattern and numeric assembly (EMAssembly::assemble,
 * src/numeric/em_assembly.cpp:144-420, scatter :654-765; duplicates summed
 * as SparseConverter::to_eigen does, sparse_converter.cpp:19-80).
 * ------------------------------------------------------------------------- */
static int build_incidence(int epe, int64_t n_tets, const int32_t* l2g, int64_t n, int64_t** iptr_o,
                           int64_t** ilist_o) {
  int64_t* iptr = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
  if (!iptr) return -1;
  for (int64_t i = 0; i < epe * n_tets; i++) {
    int32_t r = l2g[i];
    if (r >= n) { free(iptr); return ORC_INVALID_INPUT; }
    if (r >= 0) iptr[r + 1]++;
  }
  for (int64_t r = 0; r < n; r++) iptr[r + 1] += iptr[r];
  int64_t* ilist = (int64_t*)malloc((size_t)(iptr[n] > 0 ? iptr[n] : 1) * sizeof(int64_t));
  int64_t* fill = (int64_t*)malloc((size_t)(n > 0 ? n : 1) * sizeof(int64_t));
  for (int64_t r = 0; r < n; r++) fill[r] = iptr[r];
  for (int64_t i = 0; i < epe * n_tets; i++)
    if (l2g[i] >= 0) ilist[fill[l2g[i]]++] = i;
  free(fill);
  *iptr_o = iptr;
  *ilist_o = ilist;
  return 0;
}

int orc_pattern(int64_t n_tets, const int32_t* l2g, int64_t n, int64_t* row_ptr,
                int32_t* col, int64_t* nnz) {
  return orc_pattern_typed(ORC_ELEM_TET4_EDGE, n_tets, l2g, n, row_ptr, col, nnz);
}

int orc_pattern_typed(int32_t elem_type, int64_t n_tets, const int32_t* l2g, int64_t n, int64_t* row_ptr,
                      int32_t* col, int64_t* nnz) {
  int npe, epe;
  const int (*tab)[2];
  if (elem_shape(elem_type, &npe, &epe, &tab)) return ORC_INVALID_INPUT;
  int64_t *iptr, *ilist;
  int rc = build_incidence(epe, n_tets, l2g, n, &iptr, &ilist);
  if (rc) return rc;
  row_ptr[0] = 0;
  int64_t total = 0;
  int32_t buf[1024];
  for (int64_t r = 0; r < n; r++) {
    int m = 0;
    for (int64_t q = iptr[r]; q < iptr[r + 1]; q++) {
      int64_t t = ilist[q] / epe;
      for (int k = 0; k < epe; k++) {
        int32_t c = l2g[epe * t + k];
        if (c < 0) continue;
        int found = 0;
        for (int z = 0; z < m; z++) if (buf[z] == c) { found = 1; break; }
        if (!found && m < 1024) buf[m++] = c;
      }
    }
    for (int i = 1; i < m; i++) { /* sort the row */
      int32_t v = buf[i];
      int j = i - 1;
      while (j >= 0 && buf[j] > v) { buf[j + 1] = buf[j]; j--; }
      buf[j + 1] = v;
    }
    if (col) memcpy(col + total, buf, (size_t)m * sizeof(int32_t));
    total += m;
    row_ptr[r + 1] = total;
  }
  *nnz = total;
  free(iptr);
  free(ilist);
  return 0;
}

static int64_t slot_of(const int64_t* row_ptr, const int32_t* col, int32_t r, int32_t c) {
  int64_t lo = row_ptr[r], hi = row_ptr[r + 1];
  while (lo < hi) {
    int64_t mid = (lo + hi) / 2;
    if (col[mid] < c) lo = mid + 1; else hi = mid;
  }
  return (lo < row_ptr[r + 1] && col[lo] == c) ? lo : -1;
}

int orc_assemble(int64_t n_nodes, const double* xyz, int64_t n_tets,
                 const int32_t* tets, const int32_t* material, const int32_t* l2g,
                 const double* nu_mat, const double* sigma_mat, int32_t n_mat,
                 const orc_source* src, int32_t n_src, int32_t flags, int64_t n,
                 const int64_t* row_ptr, const int32_t* col, double* kval,
                 double* mval, double* rhs) {
  return orc_assemble_typed(ORC_ELEM_TET4_EDGE, n_nodes, xyz, n_tets, tets, material, l2g, nu_mat, sigma_mat,
                            n_mat, src, n_src, flags, n, row_ptr, col, kval, mval, rhs);
}

int orc_assemble_typed(int32_t elem_type, int64_t n_nodes, const double* xyz, int64_t n_tets,
                       const int32_t* tets, const int32_t* material, const int32_t* l2g,
                       const double* nu_mat, const double* sigma_mat, int32_t n_mat,
                       const orc_source* src, int32_t n_src, int32_t flags, int64_t n,
                       const int64_t* row_ptr, const int32_t* col, double* kval,
                       double* mval, double* rhs) {
  int npe, epe;
  const int (*tab)[2];
  if (elem_shape(elem_type, &npe, &epe, &tab)) return ORC_INVALID_INPUT;
  int64_t nnz = row_ptr[n];
  for (int64_t i = 0; i < nnz; i++) { kval[i] = 0.0; if (mval) mval[i] = 0.0; }
  if (rhs) for (int64_t i = 0; i < n; i++) rhs[i] = 0.0;
  for (int64_t t = 0; t < n_tets; t++) {
    int32_t mid = material ? material[t] : 0;
    if (mid < 0 || mid >= n_mat) continue; /* em_assembly.cpp:270-276 */
    int nn, ne;
    const int (*rt)[2];
    int32_t et;
    if (row_shape(elem_type, tets + npe * t, &nn, &ne, &rt, &et)) return ORC_INVALID_INPUT;
    double X[24];
    for (int a = 0; a < nn; a++) {
      int32_t g = tets[npe * t + a];
      if (g < 0 || g >= n_nodes) return ORC_INVALID_INPUT;
      X[3 * a] = xyz[3 * g]; X[3 * a + 1] = xyz[3 * g + 1]; X[3 * a + 2] = xyz[3 * g + 2];
    }
    double Ke[144], Me[144], Fe[12];
    int32_t s[12];
    const double sg = sigma_mat ? sigma_mat[mid] : 0.0;
    if (et == ORC_ELEM_HEX8_EDGE) {
      orc_element_hex(X, nu_mat[mid], sg, src, n_src, flags, Ke, Me, Fe);
      orc_edge_signs_hex(tets + npe * t, s);
      if (elem_type == ORC_ELEM_MIXED) {
        /* in a mixed mesh the hex basis is scaled to unit circulation (1/4)
         * so that it agrees with the other elements on shared edges */
        for (int i = 0; i < 144; i++) { Ke[i] *= 0.0625; Me[i] *= 0.0625; }
        for (int i = 0; i < 12; i++) Fe[i] *= 0.25;
      }
    } else if (et == ORC_ELEM_PRISM6_EDGE || et == ORC_ELEM_PYRAMID5_EDGE) {
      orc_element_shape(et == ORC_ELEM_PRISM6_EDGE ? &ORC_PRISM : &ORC_PYRAMID, X, nu_mat[mid], sg, src, n_src,
                        flags, Ke, Me, Fe);
      for (int k = 0; k < ne; k++) s[k] = tets[npe * t + rt[k][0]] < tets[npe * t + rt[k][1]] ? 1 : -1;
    } else {
      orc_element(X, nu_mat[mid], sg, src, n_src, flags, Ke, Me, Fe);
      orc_edge_signs(tets + npe * t, s);
    }
    if (flags & ORC_FLAG_NO_EDGE_SIGNS) for (int k = 0; k < ne; k++) s[k] = 1;
    const int32_t* L = l2g + epe * t;
    for (int i = 0; i < ne; i++) {
      if (L[i] < 0) continue;
      if (rhs) rhs[L[i]] += s[i] * Fe[i];
      for (int j = 0; j < ne; j++) {
        if (L[j] < 0) continue;
        int64_t p = slot_of(row_ptr, col, L[i], L[j]);
        if (p < 0) return ORC_INVALID_INPUT;
        kval[p] += (double)(s[i] * s[j]) * Ke[ne * i + j];
        if (mval && (flags & ORC_FLAG_MASS)) mval[p] += (double)(s[i] * s[j]) * Me[ne * i + j];
      }
    }
  }
  return 0;
}

/* ---------------------------------------------------------------------------
 * Krylov solvers.
 * ------------------------------------------------------------------------- */
void orc_spmv(int64_t n, const int64_t* rp, const int32_t* col, const double* val,
              const double* x, double* y) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) {
    double s = 0.0;
    for (int64_t k = rp[i]; k < rp[i + 1]; k++) s += val[k] * x[col[k]];
    y[i] = s;
  }
}

/* Deterministic dot product: fixed 64 chunks summed in order, independent of
 * the thread count. */
static double vdot(int64_t n, const double* a, const double* b) {
  enum { NCH = 64 };
  double part[NCH];
#pragma omp parallel for schedule(static)
  for (int c = 0; c < NCH; c++) {
    int64_t lo = n * c / NCH, hi = n * (c + 1) / NCH;
    double s = 0.0;
    for (int64_t i = lo; i < hi; i++) s += a[i] * b[i];
    part[c] = s;
  }
  double s = 0.0;
  for (int c = 0; c < NCH; c++) s += part[c];
  return s;
}

static void jacobi_inverse(int64_t n, const int64_t* rp, const int32_t* col,
                           const double* val, double* dinv) {
  /* CGSolver::setup_preconditioner (iterative_solvers.cpp:261-292) */
  for (int64_t i = 0; i < n; i++) {
    double d = 0.0;
    for (int64_t k = rp[i]; k < rp[i + 1]; k++) if (col[k] == i) d += val[k];
    dinv[i] = fabs(d) > 1e-15 ? 1.0 / d : 1.0;
  }
}

/* Preconditioners of CGSolver / BiCGSTABSolver: 0 none, 1 Jacobi
 * (setup_preconditioner, iterative_solvers.cpp:261-292), 2 ILU0.  The
 * reference's ILU0 is Eigen's IncompleteLUT (:277-286); this restatement
 * uses ILU(0) on the matrix's own pattern -- the IKJ elimination (Saad,
 * Iterative Methods for Sparse Linear Systems, 2nd ed., Algorithm 10.4)
 * restricted to that pattern, as the GPU solver does -- and, like the
 * reference, runs without a preconditioner when the factorization fails
 * (:279-282): a row without a diagonal entry, columns not ascending, or a
 * zero / non-finite pivot. */
typedef struct {
  int kind;        /* 0 none, 1 Jacobi, 2 ILU(0) */
  double* dinv;    /* Jacobi */
  double* lu;      /* ILU(0): unit L below, U on and above the diagonal */
  int64_t* diag;
  double* y;
} OrcPrec;

static void prec_free(OrcPrec* P) {
  free(P->dinv); free(P->lu); free(P->diag); free(P->y);
  P->dinv = P->lu = P->y = NULL;
  P->diag = NULL;
}

static int ilu0_factor(int64_t n, const int64_t* rp, const int32_t* col, const double* val, OrcPrec* P) {
  P->lu = (double*)malloc((size_t)(rp[n] > 0 ? rp[n] : 1) * sizeof(double));
  P->diag = (int64_t*)malloc((size_t)n * sizeof(int64_t));
  P->y = (double*)malloc((size_t)n * sizeof(double));
  int64_t* where = (int64_t*)malloc((size_t)n * sizeof(int64_t));
  if (!P->lu || !P->diag || !P->y || !where) { free(where); return 0; }
  memcpy(P->lu, val, (size_t)rp[n] * sizeof(double));
  for (int64_t i = 0; i < n; i++) where[i] = -1;
  int ok = 1;
  for (int64_t i = 0; i < n && ok; i++) {
    P->diag[i] = -1;
    for (int64_t q = rp[i]; q < rp[i + 1]; q++) {
      if (q > rp[i] && col[q] <= col[q - 1]) ok = 0;
      if (col[q] == i) P->diag[i] = q;
    }
    if (P->diag[i] < 0) ok = 0;
  }
  for (int64_t i = 0; i < n && ok; i++) {
    for (int64_t q = rp[i]; q < rp[i + 1]; q++) where[col[q]] = q;
    for (int64_t p = rp[i]; p < P->diag[i]; p++) {
      const int64_t k = col[p];
      const double l = P->lu[p] / P->lu[P->diag[k]];
      P->lu[p] = l;
      for (int64_t q = P->diag[k] + 1; q < rp[k + 1]; q++) {
        const int64_t w = where[col[q]];
        if (w >= 0) P->lu[w] -= l * P->lu[q];
      }
    }
    for (int64_t q = rp[i]; q < rp[i + 1]; q++) where[col[q]] = -1;
    const double u = P->lu[P->diag[i]];
    if (!(fabs(u) > 0.0) || !isfinite(u)) ok = 0;
  }
  free(where);
  return ok;
}

static int prec_setup(OrcPrec* P, int64_t n, const int64_t* rp, const int32_t* col, const double* val,
                      int32_t precond) {
  memset(P, 0, sizeof(*P));
  P->kind = precond == 1 ? 1 : precond == 2 ? 2 : 0;
  if (P->kind == 1) {
    P->dinv = (double*)malloc((size_t)n * sizeof(double));
    if (!P->dinv) return -1;
    jacobi_inverse(n, rp, col, val, P->dinv);
  } else if (P->kind == 2 && !ilu0_factor(n, rp, col, val, P)) {
    prec_free(P);
    P->kind = 0;  /* the reference falls back to no preconditioner */
  }
  return 0;
}

/* out = M^-1 in */
static void prec_apply(const OrcPrec* P, int64_t n, const int64_t* rp, const int32_t* col, const double* in,
                       double* out) {
  if (P->kind == 1) {
    for (int64_t i = 0; i < n; i++) out[i] = P->dinv[i] * in[i];
  } else if (P->kind == 2) {
    for (int64_t i = 0; i < n; i++) {
      double s = 0.0;
      for (int64_t p = rp[i]; p < P->diag[i]; p++) s += P->lu[p] * P->y[col[p]];
      P->y[i] = in[i] - s;
    }
    for (int64_t i = n - 1; i >= 0; i--) {
      double s = 0.0;
      for (int64_t p = P->diag[i] + 1; p < rp[i + 1]; p++) s += P->lu[p] * out[col[p]];
      out[i] = (P->y[i] - s) / P->lu[P->diag[i]];
    }
  } else {
    for (int64_t i = 0; i < n; i++) out[i] = in[i];
  }
}

int orc_pcg(int64_t n, const int64_t* rp, const int32_t* col, const double* val,
            const double* b, double* x, double tol, int32_t max_iter, int32_t precond,
            int32_t* iterations, double* residual_norm) {
  return orc_pcg_snap(n, rp, col, val, b, x, tol, max_iter, precond, iterations, residual_norm,
                      0.0, NULL, NULL);
}

/* orc_pcg with a snapshot: the first iterate whose relative residual is
 * below snap_tol is copied to x_snap (its iteration to *snap_iter, -1 if
 * never), so one run to a tight tolerance also gives the iterate at which a
 * solve to snap_tol stops (same sequence of iterates). */
int orc_pcg_snap(int64_t n, const int64_t* rp, const int32_t* col, const double* val,
                 const double* b, double* x, double tol, int32_t max_iter, int32_t precond,
                 int32_t* iterations, double* residual_norm, double snap_tol, double* x_snap,
                 int32_t* snap_iter) {
  *iterations = 0;
  *residual_norm = 0.0;
  if (snap_iter) *snap_iter = -1;
  if (n <= 0) return ORC_INVALID_INPUT;
  double* r = (double*)malloc((size_t)n * sizeof(double));
  double* z = (double*)malloc((size_t)n * sizeof(double));
  double* p = (double*)malloc((size_t)n * sizeof(double));
  double* q = (double*)malloc((size_t)n * sizeof(double));
  OrcPrec M;
  if (!r || !z || !p || !q || prec_setup(&M, n, rp, col, val, precond)) return -1;
  for (int64_t i = 0; i < n; i++) { x[i] = 0.0; r[i] = b[i]; }
  prec_apply(&M, n, rp, col, r, z);
  for (int64_t i = 0; i < n; i++) p[i] = z[i];
  double rz = vdot(n, r, z);
  double bnorm = sqrt(vdot(n, b, b));
  int status = ORC_MAX_ITER_REACHED;
  if (bnorm < 1e-15) { /* :361-367 / :440-446 */
    free(r); free(z); free(p); free(q); prec_free(&M);
    return ORC_SUCCESS;
  }
  double res = sqrt(vdot(n, r, r)) / bnorm, prev = res;
  int32_t it;
  for (it = 1; it <= max_iter; it++) {
    orc_spmv(n, rp, col, val, p, q);
    double pq = vdot(n, p, q);
    if (fabs(pq) < 1e-30) { status = ORC_NUMERICAL_ERROR; break; }
    double alpha = rz / pq;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
      x[i] += alpha * p[i];
      r[i] -= alpha * q[i];
    }
    prec_apply(&M, n, rp, col, r, z);
    double rz_new = vdot(n, r, z);
    res = sqrt(vdot(n, r, r)) / bnorm;
    if (x_snap && snap_iter && *snap_iter < 0 && res < snap_tol) {
      memcpy(x_snap, x, (size_t)n * sizeof(double));
      *snap_iter = it;
    }
    if (res < tol) { status = ORC_SUCCESS; break; }
    if (it > 10 && res > prev * 1000.0) { status = ORC_DIVERGED; break; }
    double beta = rz_new / rz;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
    rz = rz_new;
    prev = res;
  }
  *iterations = it <= max_iter ? it : max_iter;
  *residual_norm = res;
  free(r); free(z); free(p); free(q); prec_free(&M);
  return status;
}

int orc_bicgstab(int64_t n, const int64_t* rp, const int32_t* col, const double* val,
                 const double* b, double* x, double tol, int32_t max_iter, int32_t precond,
                 int32_t* iterations, double* residual_norm) {
  *iterations = 0;
  *residual_norm = 0.0;
  if (n <= 0) return ORC_INVALID_INPUT;
  size_t sz = (size_t)n * sizeof(double);
  double *r = malloc(sz), *rh = malloc(sz), *p = malloc(sz), *v = malloc(sz);
  double *s = malloc(sz), *z = malloc(sz), *t = malloc(sz);
  OrcPrec M;
  if (!r || !rh || !p || !v || !s || !z || !t || prec_setup(&M, n, rp, col, val, precond)) return -1;
  for (int64_t i = 0; i < n; i++) { x[i] = 0.0; r[i] = b[i]; rh[i] = b[i]; p[i] = b[i]; v[i] = 0.0; }
  double rho = vdot(n, r, rh), alpha = 1.0, omega = 1.0;
  double bnorm = sqrt(vdot(n, b, b));
  int status = ORC_MAX_ITER_REACHED;
  if (bnorm < 1e-15) { free(r); free(rh); free(p); free(v); free(s); free(z); free(t); prec_free(&M); return ORC_SUCCESS; }
  double res = sqrt(vdot(n, r, r)) / bnorm, prev = res;
  int dcount = 0;
  int32_t it;
  for (it = 1; it <= max_iter; it++) {
    double rho_old = rho;
    rho = vdot(n, r, rh);
    if (fabs(rho) < 1e-30) { status = ORC_NUMERICAL_ERROR; break; }
    double beta = (rho / rho_old) * (alpha / omega);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) p[i] = r[i] + beta * (p[i] - omega * v[i]);
    orc_spmv(n, rp, col, val, p, v);
    double rv = vdot(n, rh, v);
    if (fabs(rv) < 1e-30) { status = ORC_NUMERICAL_ERROR; break; }
    alpha = rho / rv;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) s[i] = r[i] - alpha * v[i];
    res = sqrt(vdot(n, s, s)) / bnorm;
    if (res < tol) { /* early exit on ||s|| (:1050-1058) */
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < n; i++) x[i] += alpha * p[i];
      *iterations = it;
      *residual_norm = res;
      free(r); free(rh); free(p); free(v); free(s); free(z); free(t); prec_free(&M);
      return ORC_SUCCESS;
    }
    /* precondition s only (:1061, :1186) */
    prec_apply(&M, n, rp, col, s, z);
    orc_spmv(n, rp, col, val, z, t);
    double tt = vdot(n, t, t);
    omega = fabs(tt) < 1e-30 ? 0.0 : vdot(n, z, t) / tt;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
      x[i] += alpha * p[i] + omega * z[i];
      r[i] = s[i] - omega * t[i];
    }
    res = sqrt(vdot(n, r, r)) / bnorm;
    if (res < tol) { status = ORC_SUCCESS; break; }
    if (res > prev * 1.5 && it > 20) {
      if (++dcount >= 3) { status = ORC_DIVERGED; break; }
    } else {
      dcount = 0;
    }
    if (it > 10 && res > prev * 1000.0) { status = ORC_DIVERGED; break; }
    prev = res;
  }
  *iterations = it <= max_iter ? it : max_iter;
  *residual_norm = res;
  free(r); free(rh); free(p); free(v); free(s); free(z); free(t); prec_free(&M);
  return status;
}

/* ------------------------------------------------------------------------
 * Per-element DOF types (MIXED_AV): see emg_oracle.h.  The scalar part is
 * restated here; the edge part runs the edge-ID and DOF/gauge restatement
 * above on the vector-carrying elements in their order, which is the mesh
 * GlobalEdgeIDGenerator and MeshGraphExtractor see
 * (mesh_graph_extractor.cpp:78, :182). */
int orc_dof_build_av(int32_t elem_type, int64_t n_nodes, int64_t n_elems, const int32_t* elems,
                     const int32_t* dof_type, int64_t n_dir, const int32_t* dir_pairs, int64_t n_sdir,
                     const int32_t* sdir_nodes, int32_t n_hole_markers, int32_t gauge, int32_t* l2g,
                     int64_t* n_scalar_free, int64_t* n_free, int64_t* n_dofs) {
  int npe, epe;
  const int (*tab)[2];
  if (elem_type == ORC_ELEM_MIXED || elem_shape(elem_type, &npe, &epe, &tab)) return ORC_INVALID_INPUT;
  const int w = npe + epe;
  int64_t i, e, nv = 0, nsf = 0, ne = 0, vf = 0, vd = 0, k = 0;
  int32_t root = -1;
  int rc = 0;
  for (e = 0; e < n_elems; ++e) {
    if (dof_type[e] < 0 || dof_type[e] > 2) return -1;
    if (dof_type[e] != ORC_DOF_SCALAR_ONLY) nv++;
  }
  /* scalar prenumbers: nodes of SCALAR_ONLY / MIXED_AV elements, ascending */
  uint8_t* ref = calloc((size_t)(n_nodes > 0 ? n_nodes : 1), 1);
  uint8_t* con = calloc((size_t)(n_nodes > 0 ? n_nodes : 1), 1);
  int32_t* sfree = malloc(sizeof(int32_t) * (size_t)(n_nodes > 0 ? n_nodes : 1));
  int32_t* vel = malloc(sizeof(int32_t) * (size_t)(npe * (nv > 0 ? nv : 1)));
  int32_t* vee = malloc(sizeof(int32_t) * (size_t)(epe * (nv > 0 ? nv : 1)));
  int32_t* vl2g = malloc(sizeof(int32_t) * (size_t)(epe * (nv > 0 ? nv : 1)));
  int32_t* ven = malloc(sizeof(int32_t) * (size_t)(2 * epe * (nv > 0 ? nv : 1)));
  int32_t* vdof = malloc(sizeof(int32_t) * (size_t)(epe * (nv > 0 ? nv : 1)));
  if (!ref || !con || !sfree || !vel || !vee || !vl2g || !ven || !vdof) { rc = -2; goto done; }
  for (e = 0; e < n_elems; ++e)
    if (dof_type[e] != ORC_DOF_VECTOR_EDGE_ONLY)
      for (i = 0; i < npe; ++i) {
        const int32_t v = elems[npe * e + i];
        if (v < 0 || v >= n_nodes) { rc = -1; goto done; }
        ref[v] = 1;
      }
  for (i = 0; i < n_sdir; ++i)
    if (sdir_nodes[i] >= 0 && sdir_nodes[i] < n_nodes) con[sdir_nodes[i]] = 1;
  for (i = 0; i < n_nodes; ++i) sfree[i] = (ref[i] && !con[i]) ? (int32_t)nsf++ : -1;
  /* edge part on the vector-carrying elements */
  for (e = 0; e < n_elems; ++e)
    if (dof_type[e] != ORC_DOF_SCALAR_ONLY) {
      memcpy(vel + npe * k, elems + npe * e, sizeof(int32_t) * (size_t)npe);
      k++;
    }
  if (nv > 0) {
    rc = orc_edge_ids_typed(elem_type, nv, vel, vee, ven, &ne);
    if (!rc)
      rc = orc_dof_build_typed(elem_type, nv, vel, vee, ven, ne, n_dir, dir_pairs, n_hole_markers, gauge, vl2g,
                               vdof, &vf, &vd, &root);
    if (rc) goto done;
  }
  /* rows: node DOFs, then edge DOFs offset by the free scalars, then -2 */
  k = 0;
  for (e = 0; e < n_elems; ++e) {
    int32_t* row = l2g + (int64_t)w * e;
    int c = 0;
    for (i = 0; i < w; ++i) row[i] = -2;
    if (dof_type[e] != ORC_DOF_VECTOR_EDGE_ONLY)
      for (i = 0; i < npe; ++i) row[c++] = sfree[elems[npe * e + i]];
    if (dof_type[e] != ORC_DOF_SCALAR_ONLY) {
      for (i = 0; i < epe; ++i) {
        const int32_t d = vl2g[epe * k + i];
        row[c++] = d < 0 ? -1 : (int32_t)(d + nsf);
      }
      k++;
    }
  }
  *n_scalar_free = nsf;
  *n_free = nsf + vf;
  *n_dofs = nsf + vd;
done:
  free(ref); free(con); free(sfree); free(vel); free(vee); free(vl2g); free(ven); free(vdof);
  return rc;
}

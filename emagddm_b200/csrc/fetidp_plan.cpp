// fetidp_plan.cpp -- symbolic phase of the FETI-DP solver (host, integer work).
//
// For every subdomain: its local DOFs split into I / D / P, a geometric
// nested-dissection ordering of I (edge midpoints, median split along the
// longest extent, vertex separator = the smaller of the two boundary layers),
// and the multifrontal front structure of A_rr with the D DOFs eliminated
// last as one dense "root" front -- so the root front, once its children are
// added in, is the subdomain's Dirichlet Schur complement S_DD.  Globally: the
// union numbering of all subdomain blocks, one Lagrange multiplier per dual
// DOF, the coarse numbering of the primal DOFs and the gather lists that
// assemble the coarse matrix deterministically.
#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>
#include <string>

#include "fetidp.h"

namespace emg {
namespace {

constexpr int kLeaf = 128;      // largest ND leaf (pivots)
constexpr int64_t kAlign = 32;  // doubles (256 B) between blocks

int64_t pad(int64_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

struct NdNode {
  std::vector<int32_t> piv;   // initial local indices, ascending
  std::vector<int32_t> kids;  // node ids
  int32_t p0 = 0;
};

struct Sub {
  int32_t nI = 0, nD = 0, nP = 0;
  std::vector<int32_t> gdof;  // initial local index -> global DOF: I, D, P (each ascending)
  std::vector<int64_t> aptr;  // adjacency over r DOFs (initial local indices)
  std::vector<int32_t> adj;
  std::vector<double> coord;  // 3 * nI edge midpoints
  std::vector<int8_t> side;
  std::vector<NdNode> nodes;
  std::vector<int32_t> roots;
  std::vector<int32_t> pos;   // initial local index -> position
};

void nd(Sub& w, std::vector<int32_t> set, std::vector<int32_t>& roots) {
  if (set.empty()) return;
  auto leaf = [&]() {
    NdNode n;
    n.piv = std::move(set);
    std::sort(n.piv.begin(), n.piv.end());
    w.nodes.push_back(std::move(n));
    roots.push_back(static_cast<int32_t>(w.nodes.size() - 1));
  };
  if (static_cast<int>(set.size()) <= kLeaf) { leaf(); return; }
  double lo[3], hi[3];
  for (int a = 0; a < 3; ++a) { lo[a] = std::numeric_limits<double>::infinity(); hi[a] = -lo[a]; }
  for (int32_t v : set)
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], w.coord[3 * v + a]);
      hi[a] = std::max(hi[a], w.coord[3 * v + a]);
    }
  int order[3] = {0, 1, 2};
  std::stable_sort(order, order + 3, [&](int a, int b) { return hi[a] - lo[a] > hi[b] - lo[b]; });
  std::vector<int32_t> left, right;
  bool ok = false;
  for (int ai = 0; ai < 3 && !ok; ++ai) {
    const int a = order[ai];
    if (!(hi[a] > lo[a])) continue;
    std::vector<double> cs(set.size());
    for (size_t i = 0; i < set.size(); ++i) cs[i] = w.coord[3 * set[i] + a];
    const size_t mid = cs.size() / 2;
    std::nth_element(cs.begin(), cs.begin() + mid, cs.end());
    double split = cs[mid];
    if (!(split > lo[a])) {
      split = std::numeric_limits<double>::infinity();
      for (double c : cs)
        if (c > lo[a] && c < split) split = c;
    }
    left.clear();
    right.clear();
    for (int32_t v : set) (w.coord[3 * v + a] < split ? left : right).push_back(v);
    ok = !left.empty() && !right.empty();
  }
  if (!ok) { leaf(); return; }
  for (int32_t v : left) w.side[v] = 0;
  for (int32_t v : right) w.side[v] = 1;
  std::vector<int32_t> sepL, sepR;
  for (int32_t v : left)
    for (int64_t q = w.aptr[v]; q < w.aptr[v + 1]; ++q)
      if (w.side[w.adj[q]] == 1) { sepL.push_back(v); break; }
  for (int32_t v : right)
    for (int64_t q = w.aptr[v]; q < w.aptr[v + 1]; ++q)
      if (w.side[w.adj[q]] == 0) { sepR.push_back(v); break; }
  const bool take_left = sepL.size() <= sepR.size();
  std::vector<int32_t>& sep = take_left ? sepL : sepR;
  std::vector<int32_t>& from = take_left ? left : right;
  for (int32_t v : sep) w.side[v] = 2;
  from.erase(std::remove_if(from.begin(), from.end(), [&](int32_t v) { return w.side[v] == 2; }),
             from.end());
  for (int32_t v : set) w.side[v] = -1;
  std::vector<int32_t>().swap(set);
  std::vector<int32_t> kids;
  nd(w, std::move(left), kids);
  nd(w, std::move(right), kids);
  if (sep.empty()) {
    roots.insert(roots.end(), kids.begin(), kids.end());
    return;
  }
  NdNode n;
  n.piv = std::move(sep);
  std::sort(n.piv.begin(), n.piv.end());
  n.kids = std::move(kids);
  w.nodes.push_back(std::move(n));
  roots.push_back(static_cast<int32_t>(w.nodes.size() - 1));
}

void assign_positions(Sub& w, int32_t node, int32_t& next) {
  for (int32_t k : w.nodes[node].kids) assign_positions(w, k, next);
  NdNode& n = w.nodes[node];
  n.p0 = next;
  for (int32_t v : n.piv) w.pos[v] = next++;
}

struct LocalFront {
  int32_t p0 = 0, npiv = 0, height = 0;
  std::vector<int32_t> border;
  std::vector<int32_t> kids;  // local front ids
  bool root = false;
};

// Second postorder pass: border sets and heights; appends fronts in postorder.
int32_t make_fronts(Sub& w, int32_t node, std::vector<LocalFront>& out) {
  std::vector<int32_t> kid_fronts;
  for (int32_t k : w.nodes[node].kids) kid_fronts.push_back(make_fronts(w, k, out));
  const NdNode& n = w.nodes[node];
  LocalFront f;
  f.p0 = n.p0;
  f.npiv = static_cast<int32_t>(n.piv.size());
  const int32_t last = f.p0 + f.npiv - 1;
  std::vector<int32_t> b;
  int32_t h = 0;
  for (int32_t kf : kid_fronts) {
    for (int32_t r : out[kf].border)
      if (r > last) b.push_back(r);
    h = std::max(h, out[kf].height + 1);
  }
  for (int32_t v : n.piv)
    for (int64_t q = w.aptr[v]; q < w.aptr[v + 1]; ++q) {
      const int32_t r = w.pos[w.adj[q]];
      if (r > last) b.push_back(r);
    }
  std::sort(b.begin(), b.end());
  b.erase(std::unique(b.begin(), b.end()), b.end());
  f.border = std::move(b);
  f.height = h;
  f.kids = std::move(kid_fronts);
  out.push_back(std::move(f));
  return static_cast<int32_t>(out.size() - 1);
}

struct FreeList {
  std::vector<std::pair<int64_t, int64_t>> free;  // (offset, size), ascending offset
  int64_t top = 0;
  int64_t alloc(int64_t n) {
    for (size_t i = 0; i < free.size(); ++i)
      if (free[i].second >= n) {
        const int64_t off = free[i].first;
        free[i].first += n;
        free[i].second -= n;
        if (free[i].second == 0) free.erase(free.begin() + static_cast<long>(i));
        return off;
      }
    const int64_t off = top;
    top += n;
    return off;
  }
  void release(int64_t off, int64_t n) {
    auto it = std::lower_bound(free.begin(), free.end(), std::make_pair(off, int64_t(0)));
    it = free.insert(it, {off, n});
    size_t i = static_cast<size_t>(it - free.begin());
    if (i + 1 < free.size() && free[i].first + free[i].second == free[i + 1].first) {
      free[i].second += free[i + 1].second;
      free.erase(free.begin() + static_cast<long>(i + 1));
    }
    if (i > 0 && free[i - 1].first + free[i - 1].second == free[i].first) {
      free[i - 1].second += free[i].second;
      free.erase(free.begin() + static_cast<long>(i));
    }
  }
};

}  // namespace

int build_feti_plan(const Mesh& m, const DofMap& d, FetiPlan& p) {
  if (d.n_parts < 1 || static_cast<int64_t>(d.dof_primal.size()) != d.n_dofs) {
    set_error("FETI-DP needs a DOF map from emg_dof_build_partitioned");
    return EMG_INVALID_INPUT;
  }
  if (!m.edges_built || d.n_elems != m.n_elems || d.elem_type != m.elem_type || d.n_edges != m.n_edges) {
    set_error("FETI-DP: DOF map does not belong to this mesh");
    return EMG_INVALID_INPUT;
  }
  p = FetiPlan{};
  const int32_t S = d.n_parts;
  const int64_t T = m.n_elems, N = d.n_dofs;
  const int epe = m.epe();
  p.n_parts = S;
  p.n_dofs = N;
  // subdomains touching every DOF
  std::vector<int32_t> q1(N, -1), q2(N, -1);
  std::vector<uint8_t> many(N, 0);
  for (int64_t t = 0; t < T; ++t) {
    const int32_t s = d.tet_part[t];
    for (int k = 0; k < epe; ++k) {
      const int32_t g = d.l2g[epe * t + k];
      if (g < 0) continue;
      if (q1[g] < 0) q1[g] = s;
      else if (q1[g] != s) {
        if (q2[g] < 0) q2[g] = s;
        else if (q2[g] != s) many[g] = 1;
      }
    }
  }
  for (int64_t g = 0; g < N; ++g) {
    if (q1[g] < 0) { set_error("FETI-DP: a DOF is used by no element"); return EMG_INVALID_INPUT; }
    if (many[g] && !d.dof_primal[g]) {
      set_error("FETI-DP: a DOF shared by 3 or more subdomains is not primal");
      return EMG_ERR_INTERNAL;
    }
  }
  std::vector<int32_t> edge_of(N, -1);
  for (int64_t e = 0; e < m.n_edges; ++e)
    if (d.edge_dof[e] >= 0) edge_of[d.edge_dof[e]] = static_cast<int32_t>(e);
  // tets per subdomain
  std::vector<int64_t> tptr(static_cast<size_t>(S) + 1, 0);
  for (int64_t t = 0; t < T; ++t) tptr[d.tet_part[t] + 1]++;
  for (int32_t s = 0; s < S; ++s) tptr[s + 1] += tptr[s];
  std::vector<int32_t> tlist(T);
  {
    std::vector<int64_t> cur(tptr.begin(), tptr.end() - 1);
    for (int64_t t = 0; t < T; ++t) tlist[cur[d.tet_part[t]]++] = static_cast<int32_t>(t);
  }
  // multiplier and coarse numbering (ascending global DOF)
  std::vector<int32_t> lam_of(N, -1), coarse_of(N, -1);
  for (int64_t g = 0; g < N; ++g) {
    if (d.dof_primal[g]) coarse_of[g] = p.n_coarse++;
    else if (q2[g] >= 0) lam_of[g] = static_cast<int32_t>(p.n_lambda++);
  }
  p.lam_entry.assign(2 * p.n_lambda, -1);
  p.loc_off.assign(static_cast<size_t>(S) + 1, 0);
  p.dual_off.assign(static_cast<size_t>(S) + 1, 0);
  p.pri_off.assign(static_cast<size_t>(S) + 1, 0);
  p.cblk_off.assign(static_cast<size_t>(S) + 1, 0);
  p.root_off.assign(static_cast<size_t>(S) + 1, 0);
  p.nI.assign(S, 0);
  p.nD.assign(S, 0);
  p.nP.assign(S, 0);
  p.l2g_union.assign(epe * T, -1);
  p.root_front.assign(S, -1);

  std::vector<int32_t> stamp(N, -1);
  std::vector<std::vector<LocalFront>> subf(S);
  std::vector<std::vector<int32_t>> sub_gdof_pos(S);  // position -> global DOF
  for (int32_t s = 0; s < S; ++s) {
    Sub w;
    std::vector<int32_t> I, D, P;
    for (int64_t q = tptr[s]; q < tptr[s + 1]; ++q) {
      const int64_t t = tlist[q];
      for (int k = 0; k < epe; ++k) {
        const int32_t g = d.l2g[epe * t + k];
        if (g < 0 || stamp[g] == -2) continue;
        stamp[g] = -2;
        (d.dof_primal[g] ? P : (q2[g] >= 0 ? D : I)).push_back(g);
      }
    }
    std::sort(I.begin(), I.end());
    std::sort(D.begin(), D.end());
    std::sort(P.begin(), P.end());
    w.nI = static_cast<int32_t>(I.size());
    w.nD = static_cast<int32_t>(D.size());
    w.nP = static_cast<int32_t>(P.size());
    const int32_t nr = w.nI + w.nD;
    w.gdof = I;
    w.gdof.insert(w.gdof.end(), D.begin(), D.end());
    w.gdof.insert(w.gdof.end(), P.begin(), P.end());
    for (size_t i = 0; i < w.gdof.size(); ++i) stamp[w.gdof[i]] = static_cast<int32_t>(i);
    // adjacency over r DOFs through the subdomain's tets
    w.aptr.assign(static_cast<size_t>(nr) + 1, 0);
    std::vector<std::pair<int32_t, int32_t>> pairs;
    pairs.reserve(static_cast<size_t>(tptr[s + 1] - tptr[s]) * epe * (epe - 1));
    for (int64_t q = tptr[s]; q < tptr[s + 1]; ++q) {
      const int64_t t = tlist[q];
      int32_t loc[12];
      for (int k = 0; k < epe; ++k) {
        const int32_t g = d.l2g[epe * t + k];
        loc[k] = (g >= 0 && stamp[g] < nr) ? stamp[g] : -1;
      }
      for (int a = 0; a < epe; ++a)
        for (int b = 0; b < epe; ++b)
          if (a != b && loc[a] >= 0 && loc[b] >= 0 && loc[a] != loc[b]) pairs.emplace_back(loc[a], loc[b]);
    }
    std::sort(pairs.begin(), pairs.end());
    pairs.erase(std::unique(pairs.begin(), pairs.end()), pairs.end());
    for (auto& pr : pairs) w.aptr[pr.first + 1]++;
    for (int32_t v = 0; v < nr; ++v) w.aptr[v + 1] += w.aptr[v];
    w.adj.resize(pairs.size());
    for (size_t i = 0; i < pairs.size(); ++i) w.adj[i] = pairs[i].second;
    std::vector<std::pair<int32_t, int32_t>>().swap(pairs);
    w.coord.resize(3 * static_cast<size_t>(w.nI));
    for (int32_t v = 0; v < w.nI; ++v) {
      const int32_t e = edge_of[w.gdof[v]];
      const int32_t a = m.edge_nodes[2 * e], b = m.edge_nodes[2 * e + 1];
      for (int c = 0; c < 3; ++c) w.coord[3 * v + c] = 0.5 * (m.xyz[3 * a + c] + m.xyz[3 * b + c]);
    }
    w.side.assign(nr, -1);
    {
      std::vector<int32_t> all(w.nI);
      std::iota(all.begin(), all.end(), 0);
      nd(w, std::move(all), w.roots);
    }
    w.pos.assign(nr, -1);
    int32_t next = 0;
    for (int32_t r : w.roots) assign_positions(w, r, next);
    if (next != w.nI) { set_error("FETI-DP: nested dissection lost DOFs"); return EMG_ERR_INTERNAL; }
    for (int32_t v = w.nI; v < nr; ++v) w.pos[v] = v;
    std::vector<LocalFront>& lf = subf[s];
    std::vector<int32_t> top;
    for (int32_t r : w.roots) top.push_back(make_fronts(w, r, lf));
    if (w.nD > 0) {
      LocalFront rf;
      rf.p0 = w.nI;
      rf.npiv = w.nD;
      rf.root = true;
      rf.kids = top;
      for (int32_t k : top) rf.height = std::max(rf.height, lf[k].height + 1);
      lf.push_back(std::move(rf));
    } else {
      for (int32_t k : top)
        if (!lf[k].border.empty()) { set_error("FETI-DP: border without dual DOFs"); return EMG_ERR_INTERNAL; }
    }
    // position -> global DOF; union block of the subdomain's tets
    std::vector<int32_t>& pg = sub_gdof_pos[s];
    pg.assign(w.gdof.size(), -1);
    for (int32_t v = 0; v < nr; ++v) pg[w.pos[v]] = w.gdof[v];
    for (int32_t v = nr; v < static_cast<int32_t>(w.gdof.size()); ++v) pg[v] = w.gdof[v];
    p.nI[s] = w.nI;
    p.nD[s] = w.nD;
    p.nP[s] = w.nP;
    p.loc_off[s + 1] = p.loc_off[s] + static_cast<int64_t>(w.gdof.size());
    p.dual_off[s + 1] = p.dual_off[s] + w.nD;
    p.pri_off[s + 1] = p.pri_off[s] + w.nP;
    p.cblk_off[s + 1] = p.cblk_off[s] + static_cast<int64_t>(w.nP) * w.nP;
    p.root_off[s + 1] = p.root_off[s] + pad(static_cast<int64_t>(w.nD) * w.nD);
    for (size_t i = 0; i < w.gdof.size(); ++i) stamp[w.gdof[i]] = -1;
    for (size_t i = 0; i < pg.size(); ++i) stamp[pg[i]] = static_cast<int32_t>(i);  // global -> position
    for (int64_t q = tptr[s]; q < tptr[s + 1]; ++q) {
      const int64_t t = tlist[q];
      for (int k = 0; k < epe; ++k) {
        const int32_t g = d.l2g[epe * t + k];
        if (g >= 0) p.l2g_union[epe * t + k] = static_cast<int32_t>(p.loc_off[s] + stamp[g]);
      }
    }
    for (size_t i = 0; i < pg.size(); ++i) stamp[pg[i]] = -1;
  }
  p.n_union = p.loc_off[S];
  if (p.n_union >= (int64_t(1) << 31)) { set_error("FETI-DP: union system too large"); return EMG_INVALID_INPUT; }
  // union -> global, global -> union copies
  p.union_gdof.resize(p.n_union);
  for (int32_t s = 0; s < S; ++s)
    for (size_t i = 0; i < sub_gdof_pos[s].size(); ++i) p.union_gdof[p.loc_off[s] + i] = sub_gdof_pos[s][i];
  p.gptr.assign(N + 1, 0);
  for (int64_t u = 0; u < p.n_union; ++u) p.gptr[p.union_gdof[u] + 1]++;
  for (int64_t g = 0; g < N; ++g) p.gptr[g + 1] += p.gptr[g];
  p.glist.resize(p.n_union);
  {
    std::vector<int64_t> cur(p.gptr.begin(), p.gptr.end() - 1);
    for (int64_t u = 0; u < p.n_union; ++u) p.glist[cur[p.union_gdof[u]]++] = static_cast<int32_t>(u);
  }
  // dual entries: sign +1 on the lower-numbered subdomain
  p.dual_lam.resize(p.dual_off[S]);
  p.dual_sign.resize(p.dual_off[S]);
  for (int32_t s = 0; s < S; ++s)
    for (int32_t i = 0; i < p.nD[s]; ++i) {
      const int64_t e = p.dual_off[s] + i;
      const int32_t g = sub_gdof_pos[s][p.nI[s] + i];
      const int32_t lam = lam_of[g];
      const bool plus = s == std::min(q1[g], q2[g]);
      p.dual_lam[e] = lam;
      p.dual_sign[e] = plus ? 1 : -1;
      p.lam_entry[2 * static_cast<int64_t>(lam) + (plus ? 0 : 1)] = static_cast<int32_t>(e);
    }
  // faces: multipliers grouped by (plus-side subdomain, minus-side subdomain)
  {
    std::vector<int32_t> dsub(p.dual_off[S]);
    for (int32_t s = 0; s < S; ++s)
      for (int64_t e = p.dual_off[s]; e < p.dual_off[s + 1]; ++e) dsub[e] = s;
    std::vector<std::pair<int64_t, int32_t>> key(p.n_lambda);
    for (int64_t l = 0; l < p.n_lambda; ++l)
      key[l] = {static_cast<int64_t>(dsub[p.lam_entry[2 * l]]) * S + dsub[p.lam_entry[2 * l + 1]],
                static_cast<int32_t>(l)};
    std::sort(key.begin(), key.end());
    p.face_ptr.push_back(0);
    p.face_off.push_back(0);
    for (int64_t i = 0; i < p.n_lambda; ++i) {
      if (i == 0 || key[i].first != key[i - 1].first) {
        if (i > 0) {
          p.face_ptr.push_back(i);
          const int64_t f = i - p.face_ptr[p.face_ptr.size() - 2];
          p.face_off.push_back(p.face_off.back() + pad(f * f));
        }
        p.face_a.push_back(static_cast<int32_t>(key[i].first / S));
        p.face_b.push_back(static_cast<int32_t>(key[i].first % S));
      }
      p.face_lam.push_back(key[i].second);
    }
    if (p.n_lambda > 0) {
      p.face_ptr.push_back(p.n_lambda);
      const int64_t f = p.n_lambda - p.face_ptr[p.face_ptr.size() - 2];
      p.face_off.push_back(p.face_off.back() + pad(f * f));
    }
    p.n_faces = static_cast<int32_t>(p.face_a.size());
  }
  // primal entries and coarse gather lists
  p.pri_coarse.resize(p.pri_off[S]);
  p.coarse_ptr.assign(static_cast<size_t>(p.n_coarse) + 1, 0);
  for (int32_t s = 0; s < S; ++s)
    for (int32_t i = 0; i < p.nP[s]; ++i) {
      const int32_t g = sub_gdof_pos[s][p.nI[s] + p.nD[s] + i];
      p.pri_coarse[p.pri_off[s] + i] = coarse_of[g];
      p.coarse_ptr[coarse_of[g] + 1]++;
    }
  for (int32_t c = 0; c < p.n_coarse; ++c) p.coarse_ptr[c + 1] += p.coarse_ptr[c];
  p.coarse_list.resize(p.pri_off[S]);
  {
    std::vector<int64_t> cur(p.coarse_ptr.begin(), p.coarse_ptr.end() - 1);
    for (int64_t e = 0; e < p.pri_off[S]; ++e) p.coarse_list[cur[p.pri_coarse[e]]++] = static_cast<int32_t>(e);
  }
  {
    const int64_t nc = p.n_coarse;
    std::vector<std::pair<int64_t, int64_t>> tg;  // (target, coarse-block entry), s ascending
    for (int32_t s = 0; s < S; ++s)
      for (int32_t b = 0; b < p.nP[s]; ++b)
        for (int32_t a = 0; a < p.nP[s]; ++a) {
          const int64_t A = p.pri_coarse[p.pri_off[s] + a], B = p.pri_coarse[p.pri_off[s] + b];
          tg.emplace_back(A + B * nc, p.cblk_off[s] + a + static_cast<int64_t>(b) * p.nP[s]);
        }
    std::stable_sort(tg.begin(), tg.end(),
                     [](const std::pair<int64_t, int64_t>& x, const std::pair<int64_t, int64_t>& y) {
                       return x.first < y.first;
                     });
    p.sc_ptr.assign(nc * nc + 1, 0);
    for (auto& x : tg) p.sc_ptr[x.first + 1]++;
    for (int64_t i = 0; i < nc * nc; ++i) p.sc_ptr[i + 1] += p.sc_ptr[i];
    p.sc_list.resize(tg.size());
    for (size_t i = 0; i < tg.size(); ++i) p.sc_list[i] = tg[i].second;
  }
  // global front table in level order; inside a level by pivot count and
  // front size, descending, so that each panel step of the factorization can
  // launch only the prefix of fronts that still have pivots left
  struct Key { int32_t h, np, f, s, i; };
  std::vector<Key> keys;
  for (int32_t s = 0; s < S; ++s)
    for (int32_t i = 0; i < static_cast<int32_t>(subf[s].size()); ++i) {
      const LocalFront& lf = subf[s][i];
      keys.push_back({lf.height, lf.npiv, lf.npiv + static_cast<int32_t>(lf.border.size()), s, i});
    }
  std::stable_sort(keys.begin(), keys.end(), [](const Key& a, const Key& b) {
    if (a.h != b.h) return a.h < b.h;
    if (a.np != b.np) return a.np > b.np;
    if (a.f != b.f) return a.f > b.f;
    if (a.s != b.s) return a.s < b.s;
    return a.i < b.i;
  });
  std::vector<std::vector<int32_t>> gid(S);
  for (int32_t s = 0; s < S; ++s) gid[s].assign(subf[s].size(), -1);
  for (size_t k = 0; k < keys.size(); ++k) gid[keys[k].s][keys[k].i] = static_cast<int32_t>(k);
  const int32_t F = static_cast<int32_t>(keys.size());
  p.fronts.resize(F);
  int32_t max_h = -1;
  for (int32_t k = 0; k < F; ++k) {
    const LocalFront& lf = subf[keys[k].s][keys[k].i];
    FetiFront& fr = p.fronts[k];
    fr.sub = keys[k].s;
    fr.p0 = lf.p0;
    fr.npiv = lf.npiv;
    fr.f = lf.npiv + static_cast<int32_t>(lf.border.size());
    fr.height = lf.height;
    fr.is_root = lf.root ? 1 : 0;
    fr.rows = static_cast<int64_t>(p.rows.size());
    for (int32_t i = 0; i < lf.npiv; ++i) p.rows.push_back(lf.p0 + i);
    p.rows.insert(p.rows.end(), lf.border.begin(), lf.border.end());
    fr.child0 = static_cast<int32_t>(p.child_list.size());
    fr.nchild = static_cast<int32_t>(lf.kids.size());
    for (int32_t c : lf.kids) p.child_list.push_back(gid[keys[k].s][c]);
    if (lf.root) p.root_front[fr.sub] = k;
    max_h = std::max(max_h, lf.height);
    p.max_front = std::max(p.max_front, fr.f);
    p.max_npiv = std::max(p.max_npiv, fr.npiv);
    p.max_children = std::max(p.max_children, fr.nchild);
  }
  for (int32_t k = 0; k < F; ++k)
    for (int32_t c = 0; c < p.fronts[k].nchild; ++c) p.fronts[p.child_list[p.fronts[k].child0 + c]].parent = k;
  p.level_ptr.assign(static_cast<size_t>(max_h) + 2, 0);
  for (int32_t k = 0; k < F; ++k) p.level_ptr[p.fronts[k].height + 1]++;
  for (int32_t h = 0; h <= max_h; ++h) p.level_ptr[h + 1] += p.level_ptr[h];
  // child -> parent row positions
  for (int32_t k = 0; k < F; ++k) {
    FetiFront& fr = p.fronts[k];
    fr.cpos = static_cast<int64_t>(p.cpos.size());
    if (fr.f == fr.npiv) continue;
    if (fr.parent < 0) { set_error("FETI-DP: front with an update but no parent"); return EMG_ERR_INTERNAL; }
    const FetiFront& pa = p.fronts[fr.parent];
    const int32_t* pr = p.rows.data() + pa.rows;
    for (int32_t i = fr.npiv; i < fr.f; ++i) {
      const int32_t r = p.rows[fr.rows + i];
      const int32_t* it = std::lower_bound(pr, pr + pa.f, r);
      if (it == pr + pa.f || *it != r) {
        set_error("FETI-DP: update row missing in the parent front");
        return EMG_ERR_INTERNAL;
      }
      p.cpos.push_back(static_cast<int32_t>(it - pr));
    }
  }
  // storage: factor blocks, update-vector rows, update pool (first fit over lifetimes)
  for (int32_t k = 0; k < F; ++k) {
    FetiFront& fr = p.fronts[k];
    fr.fac = p.fac_size;
    p.fac_size += pad(static_cast<int64_t>(fr.f) * fr.npiv);
    fr.vec = p.vec_rows;
    p.vec_rows += fr.f - fr.npiv;
  }
  {
    FreeList fl;
    for (int32_t h = 0; h <= max_h; ++h) {
      for (int32_t k = p.level_ptr[h]; k < p.level_ptr[h + 1]; ++k) {
        FetiFront& fr = p.fronts[k];
        const int64_t nupd = fr.f - fr.npiv;
        if (nupd > 0) fr.upd = fl.alloc(pad(nupd * nupd));
      }
      for (int32_t k = p.level_ptr[h]; k < p.level_ptr[h + 1]; ++k) {
        const FetiFront& fr = p.fronts[k];
        for (int32_t c = 0; c < fr.nchild; ++c) {
          const FetiFront& ch = p.fronts[p.child_list[fr.child0 + c]];
          const int64_t nupd = ch.f - ch.npiv;
          if (nupd > 0) fl.release(ch.upd, pad(nupd * nupd));
        }
      }
    }
    p.upd_pool = fl.top;
  }
  return validate_feti_plan(p);
}

int validate_feti_plan(const FetiPlan& p) {
  auto fail = [](const char* what) {
    set_error(std::string("FETI-DP plan check failed: ") + what);
    return EMG_ERR_INTERNAL;
  };
  const int32_t S = p.n_parts;
  for (int32_t s = 0; s < S; ++s) {
    const int64_t n = p.loc_off[s + 1] - p.loc_off[s];
    if (n != static_cast<int64_t>(p.nI[s]) + p.nD[s] + p.nP[s]) return fail("subdomain size");
    if (p.dual_off[s + 1] - p.dual_off[s] != p.nD[s]) return fail("dual offsets");
    if (p.pri_off[s + 1] - p.pri_off[s] != p.nP[s]) return fail("primal offsets");
  }
  for (int32_t u : p.l2g_union)
    if (u < -1 || u >= p.n_union) return fail("union l2g");
  for (int32_t g : p.union_gdof)
    if (g < 0 || g >= p.n_dofs) return fail("union -> global");
  for (int32_t u : p.glist)
    if (u < 0 || u >= p.n_union) return fail("global -> union");
  for (int64_t l = 0; l < p.n_lambda; ++l) {
    const int32_t a = p.lam_entry[2 * l], b = p.lam_entry[2 * l + 1];
    if (a < 0 || b < 0 || a >= p.dual_off[S] || b >= p.dual_off[S]) return fail("multiplier sides");
    if (p.dual_lam[a] != l || p.dual_lam[b] != l || p.dual_sign[a] != 1 || p.dual_sign[b] != -1)
      return fail("multiplier signs");
  }
  for (int32_t c : p.pri_coarse)
    if (c < 0 || c >= p.n_coarse) return fail("coarse index");
  if (static_cast<int64_t>(p.face_ptr.size()) != p.n_faces + 1 ||
      static_cast<int64_t>(p.face_off.size()) != p.n_faces + 1 ||
      static_cast<int64_t>(p.face_lam.size()) != p.n_lambda || p.face_ptr.back() != p.n_lambda)
    return fail("face tables");
  for (int32_t f = 0; f < p.n_faces; ++f) {
    const int64_t n = p.face_ptr[f + 1] - p.face_ptr[f];
    if (n < 1 || p.face_off[f + 1] - p.face_off[f] < n * n) return fail("face block");
    if (p.face_a[f] < 0 || p.face_a[f] >= p.face_b[f] || p.face_b[f] >= S) return fail("face sides");
    for (int64_t i = p.face_ptr[f]; i < p.face_ptr[f + 1]; ++i) {
      const int32_t l = p.face_lam[i];
      if (l < 0 || l >= p.n_lambda || (i > p.face_ptr[f] && l <= p.face_lam[i - 1])) return fail("face multipliers");
      const int32_t ea = p.lam_entry[2 * l], eb = p.lam_entry[2 * l + 1];
      if (ea < p.dual_off[p.face_a[f]] || ea >= p.dual_off[p.face_a[f] + 1] || eb < p.dual_off[p.face_b[f]] ||
          eb >= p.dual_off[p.face_b[f] + 1])
        return fail("face entries");
    }
  }
  for (int64_t e : p.sc_list)
    if (e < 0 || e >= p.cblk_off[S]) return fail("coarse block entry");
  const int32_t F = static_cast<int32_t>(p.fronts.size());
  for (int32_t k = 0; k < F; ++k) {
    const FetiFront& fr = p.fronts[k];
    const int32_t nr = p.nI[fr.sub] + p.nD[fr.sub];
    if (fr.npiv < 1 || fr.f < fr.npiv) return fail("front sizes");
    if (fr.p0 < 0 || fr.p0 + fr.npiv > nr) return fail("pivot range");
    if (fr.rows < 0 || fr.rows + fr.f > static_cast<int64_t>(p.rows.size())) return fail("front rows range");
    for (int32_t i = 0; i < fr.f; ++i) {
      const int32_t r = p.rows[fr.rows + i];
      if (r < 0 || r >= nr) return fail("front row outside the subdomain");
      if (i > 0 && r <= p.rows[fr.rows + i - 1]) return fail("front rows not ascending");
      if (i < fr.npiv && r != fr.p0 + i) return fail("pivot rows");
    }
    if (fr.fac < 0 || fr.fac + static_cast<int64_t>(fr.f) * fr.npiv > p.fac_size) return fail("factor block");
    const int64_t nupd = fr.f - fr.npiv;
    if (nupd > 0) {
      if (fr.upd < 0 || fr.upd + nupd * nupd > p.upd_pool) return fail("update block");
      if (fr.parent <= k) return fail("parent order");
      if (fr.cpos < 0 || fr.cpos + nupd > static_cast<int64_t>(p.cpos.size())) return fail("cpos range");
      const FetiFront& pa = p.fronts[fr.parent];
      if (pa.height <= fr.height || pa.sub != fr.sub) return fail("parent height");
      for (int64_t i = 0; i < nupd; ++i) {
        const int32_t c = p.cpos[fr.cpos + i];
        if (c < 0 || c >= pa.f) return fail("cpos value");
        if (p.rows[pa.rows + c] != p.rows[fr.rows + fr.npiv + i]) return fail("cpos row");
      }
    }
    if (fr.vec < 0 || fr.vec + nupd > p.vec_rows) return fail("update vector range");
    if (fr.child0 < 0 || fr.child0 + fr.nchild > static_cast<int32_t>(p.child_list.size())) return fail("children");
    for (int32_t c = 0; c < fr.nchild; ++c) {
      const int32_t ch = p.child_list[fr.child0 + c];
      if (ch < 0 || ch >= k || p.fronts[ch].parent != k) return fail("child link");
    }
    if (fr.is_root && (fr.npiv != p.nD[fr.sub] || fr.p0 != p.nI[fr.sub] || fr.f != fr.npiv))
      return fail("root front");
  }
  for (int32_t s = 0; s < S; ++s) {
    const int32_t r = p.root_front[s];
    if ((r < 0) != (p.nD[s] == 0)) return fail("root front presence");
    if (r >= F) return fail("root front index");
    if (p.root_off[s + 1] - p.root_off[s] < static_cast<int64_t>(p.nD[s]) * p.nD[s]) return fail("root block");
  }
  return EMG_SUCCESS;
}

}  // namespace emg

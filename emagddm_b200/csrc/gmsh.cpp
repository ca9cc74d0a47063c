// gmsh.cpp -- Gmsh ASCII mesh input (MSH 2.2 and 4.1) for the solve path.
//
// The reference plans Gmsh .msh files as its mesh format (mesh/README.md) and
// consumes meshes as fe_em::EMMeshData (include/fe_em/em_mesh_data.hpp:90-230):
// nodes, TET4 elements with a material id, and a DIRICHLET / VECTOR_EDGE_ONLY
// boundary marker whose targets are edge node pairs.  This reader produces
// exactly those arrays:
//   * nodes in ascending Gmsh tag order (index = rank of the tag);
//   * 4-node tetrahedra (element type 4) in file order; material id = rank of
//     the element's physical tag among the distinct physical tags of the
//     tetrahedra (ascending); higher-order tetrahedra are rejected;
//   * Dirichlet node pairs = the edges of the triangles (type 2) whose
//     physical tag is listed, or, with no list, the edges of every boundary
//     face (a face of exactly one tetrahedron).
#include <algorithm>
#include <array>
#include <cstdio>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "internal.h"

namespace emg {
namespace {

struct Raw {
  std::vector<int64_t> node_tag;
  std::vector<double> xyz;
  std::vector<int64_t> tet_nodes;  // 4 per tet, Gmsh node tags
  std::vector<int32_t> tet_phys;
  std::vector<int64_t> tri_nodes;  // 3 per triangle
  std::vector<int32_t> tri_phys;
};

bool seek(std::istream& in, const std::string& section) {
  std::string line;
  while (std::getline(in, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (line == section) return true;
  }
  return false;
}

int fail(const std::string& what) {
  set_error("gmsh: " + what);
  return EMG_INVALID_INPUT;
}

int parse_v2(std::istream& in, Raw& r) {
  std::streampos start = in.tellg();
  if (!seek(in, "$Nodes")) return fail("no $Nodes section");
  int64_t n = 0;
  in >> n;
  if (!in || n <= 0) return fail("bad node count");
  r.node_tag.resize(n);
  r.xyz.resize(3 * n);
  for (int64_t i = 0; i < n; ++i) in >> r.node_tag[i] >> r.xyz[3 * i] >> r.xyz[3 * i + 1] >> r.xyz[3 * i + 2];
  if (!in) return fail("truncated $Nodes");
  in.clear();
  in.seekg(start);
  if (!seek(in, "$Elements")) return fail("no $Elements section");
  int64_t m = 0;
  in >> m;
  if (!in || m < 0) return fail("bad element count");
  std::string line;
  std::getline(in, line);
  for (int64_t e = 0; e < m; ++e) {
    if (!std::getline(in, line)) return fail("truncated $Elements");
    std::istringstream ls(line);
    int64_t id = 0, type = 0, ntags = 0;
    ls >> id >> type >> ntags;
    std::vector<int64_t> tags(ntags);
    for (auto& t : tags) ls >> t;
    const int32_t phys = ntags > 0 ? static_cast<int32_t>(tags[0]) : 0;
    if (type == 4) {
      int64_t v[4];
      ls >> v[0] >> v[1] >> v[2] >> v[3];
      if (!ls) return fail("bad tetrahedron line");
      r.tet_nodes.insert(r.tet_nodes.end(), v, v + 4);
      r.tet_phys.push_back(phys);
    } else if (type == 2) {
      int64_t v[3];
      ls >> v[0] >> v[1] >> v[2];
      if (!ls) return fail("bad triangle line");
      r.tri_nodes.insert(r.tri_nodes.end(), v, v + 3);
      r.tri_phys.push_back(phys);
    } else if (type == 11 || type == 29 || type == 30 || type == 31) {
      return fail("higher-order tetrahedra are not TET4_EDGE meshes");
    }
  }
  return EMG_SUCCESS;
}

int parse_v4(std::istream& in, Raw& r) {
  std::streampos start = in.tellg();
  // entity -> first physical tag, for surfaces (dim 2) and volumes (dim 3)
  std::map<std::pair<int, int>, int32_t> phys;
  if (seek(in, "$Entities")) {
    int64_t np = 0, nc = 0, ns = 0, nv = 0;
    in >> np >> nc >> ns >> nv;
    std::string line;
    std::getline(in, line);
    for (int64_t i = 0; i < np; ++i) std::getline(in, line);
    for (int64_t i = 0; i < nc; ++i) std::getline(in, line);
    for (int dim = 2; dim <= 3; ++dim) {
      const int64_t cnt = dim == 2 ? ns : nv;
      for (int64_t i = 0; i < cnt; ++i) {
        if (!std::getline(in, line)) return fail("truncated $Entities");
        std::istringstream ls(line);
        int tag = 0;
        double bb[6];
        int64_t nph = 0;
        ls >> tag;
        for (double& b : bb) ls >> b;
        ls >> nph;
        int32_t p = 0;
        if (nph > 0) ls >> p;
        phys[{dim, tag}] = p;
      }
    }
  }
  in.clear();
  in.seekg(start);
  if (!seek(in, "$Nodes")) return fail("no $Nodes section");
  int64_t nblocks = 0, nnodes = 0, mn = 0, mx = 0;
  in >> nblocks >> nnodes >> mn >> mx;
  if (!in || nnodes <= 0) return fail("bad $Nodes header");
  r.node_tag.reserve(nnodes);
  r.xyz.reserve(3 * nnodes);
  for (int64_t b = 0; b < nblocks; ++b) {
    int dim = 0, tag = 0, param = 0;
    int64_t cnt = 0;
    in >> dim >> tag >> param >> cnt;
    if (param) return fail("parametric nodes are not supported");
    const size_t base = r.node_tag.size();
    for (int64_t i = 0; i < cnt; ++i) {
      int64_t t = 0;
      in >> t;
      r.node_tag.push_back(t);
    }
    for (int64_t i = 0; i < cnt; ++i) {
      double x, y, z;
      in >> x >> y >> z;
      r.xyz.push_back(x);
      r.xyz.push_back(y);
      r.xyz.push_back(z);
    }
    (void)base;
  }
  if (!in) return fail("truncated $Nodes");
  in.clear();
  in.seekg(start);
  if (!seek(in, "$Elements")) return fail("no $Elements section");
  in >> nblocks >> nnodes >> mn >> mx;
  if (!in) return fail("bad $Elements header");
  for (int64_t b = 0; b < nblocks; ++b) {
    int dim = 0, tag = 0, type = 0;
    int64_t cnt = 0;
    in >> dim >> tag >> type >> cnt;
    const auto it = phys.find({dim, tag});
    const int32_t p = it == phys.end() ? 0 : it->second;
    const int nv = type == 4 ? 4 : type == 2 ? 3 : type == 1 ? 2 : type == 15 ? 1 : type == 3 ? 4 : type == 5 ? 8 :
                   type == 6 ? 6 : type == 7 ? 5 : type == 11 ? 10 : type == 9 ? 6 : type == 8 ? 3 : -1;
    if (nv < 0) return fail("unsupported element type " + std::to_string(type));
    if (type == 11) return fail("higher-order tetrahedra are not TET4_EDGE meshes");
    for (int64_t i = 0; i < cnt; ++i) {
      int64_t id = 0, v[10];
      in >> id;
      for (int k = 0; k < nv; ++k) in >> v[k];
      if (type == 4) {
        r.tet_nodes.insert(r.tet_nodes.end(), v, v + 4);
        r.tet_phys.push_back(p);
      } else if (type == 2) {
        r.tri_nodes.insert(r.tri_nodes.end(), v, v + 3);
        r.tri_phys.push_back(p);
      }
    }
  }
  if (!in) return fail("truncated $Elements");
  return EMG_SUCCESS;
}

}  // namespace

int read_gmsh(const std::string& path, const int32_t* dirichlet_tags, int32_t n_tags, Mesh& m,
              std::vector<int32_t>& material_tags) {
  std::ifstream in(path);
  if (!in) return fail("cannot open " + path);
  if (!seek(in, "$MeshFormat")) return fail("no $MeshFormat section");
  double version = 0.0;
  int file_type = 0, dsize = 0;
  in >> version >> file_type >> dsize;
  if (!in) return fail("bad $MeshFormat line");
  if (file_type != 0) return fail("binary .msh files are not supported (ASCII only)");
  in.seekg(0);
  Raw r;
  int rc = version >= 4.0 ? parse_v4(in, r) : version >= 2.0 ? parse_v2(in, r) : fail("unsupported version");
  if (rc) return rc;
  if (r.tet_phys.empty()) return fail("no 4-node tetrahedra");
  // node index = rank of the tag
  std::vector<int64_t> order(r.node_tag.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = static_cast<int64_t>(i);
  std::sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return r.node_tag[a] < r.node_tag[b]; });
  std::unordered_map<int64_t, int32_t> index;
  index.reserve(order.size() * 2);
  m = Mesh{};
  m.n_nodes = static_cast<int64_t>(order.size());
  m.xyz.resize(3 * order.size());
  for (size_t k = 0; k < order.size(); ++k) {
    const int64_t i = order[k];
    if (!index.emplace(r.node_tag[i], static_cast<int32_t>(k)).second) return fail("duplicate node tag");
    for (int c = 0; c < 3; ++c) m.xyz[3 * k + c] = r.xyz[3 * i + c];
  }
  auto idx = [&](int64_t tag, int32_t& out) {
    const auto it = index.find(tag);
    if (it == index.end()) return false;
    out = it->second;
    return true;
  };
  m.n_elems = static_cast<int64_t>(r.tet_phys.size());
  m.elems.resize(4 * m.n_elems);
  for (size_t i = 0; i < r.tet_nodes.size(); ++i)
    if (!idx(r.tet_nodes[i], m.elems[i])) return fail("element references an unknown node");
  material_tags = r.tet_phys;
  std::sort(material_tags.begin(), material_tags.end());
  material_tags.erase(std::unique(material_tags.begin(), material_tags.end()), material_tags.end());
  m.material.resize(m.n_elems);
  for (int64_t t = 0; t < m.n_elems; ++t)
    m.material[t] = static_cast<int32_t>(std::lower_bound(material_tags.begin(), material_tags.end(), r.tet_phys[t]) -
                                         material_tags.begin());
  // Dirichlet node pairs
  auto add_face = [&](const int32_t* v) {
    const int e[3][2] = {{0, 1}, {1, 2}, {0, 2}};
    for (auto& p : e) {
      m.dirichlet.push_back(v[p[0]]);
      m.dirichlet.push_back(v[p[1]]);
    }
  };
  if (n_tags > 0) {
    std::vector<int32_t> want(dirichlet_tags, dirichlet_tags + n_tags);
    std::sort(want.begin(), want.end());
    for (size_t f = 0; f < r.tri_phys.size(); ++f) {
      if (!std::binary_search(want.begin(), want.end(), r.tri_phys[f])) continue;
      int32_t v[3];
      for (int k = 0; k < 3; ++k)
        if (!idx(r.tri_nodes[3 * f + k], v[k])) return fail("triangle references an unknown node");
      add_face(v);
    }
  } else {
    // faces of exactly one tetrahedron
    std::vector<std::pair<std::array<int32_t, 3>, int64_t>> faces;
    faces.reserve(4 * m.n_elems);
    const int tf[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
    for (int64_t t = 0; t < m.n_elems; ++t)
      for (auto& f : tf) {
        std::array<int32_t, 3> k = {m.elems[4 * t + f[0]], m.elems[4 * t + f[1]], m.elems[4 * t + f[2]]};
        std::sort(k.begin(), k.end());
        faces.push_back({k, t});
      }
    std::sort(faces.begin(), faces.end(),
              [](const auto& x, const auto& y) { return x.first < y.first; });
    for (size_t i = 0; i < faces.size();) {
      size_t j = i;
      while (j < faces.size() && faces[j].first == faces[i].first) ++j;
      if (j - i == 1) add_face(faces[i].first.data());
      i = j;
    }
  }
  return EMG_SUCCESS;
}

}  // namespace emg

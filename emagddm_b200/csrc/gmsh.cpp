// gmsh.cpp -- Gmsh ASCII mesh input (MSH 2.2 and 4.1) for the solve path.
//
// The reference plans Gmsh .msh files as its mesh format (mesh/README.md) and
// consumes meshes as fe_em::EMMeshData (include/fe_em/em_mesh_data.hpp:90-230):
// nodes, TET4 / HEX8 elements with a material id, and a DIRICHLET /
// VECTOR_EDGE_ONLY boundary marker whose targets are edge node pairs.  This
// reader produces exactly those arrays:
//   * nodes in ascending Gmsh tag order (index = rank of the tag);
//   * 4-node tetrahedra (element type 4) or 8-node hexahedra (type 5, Gmsh's
//     vertex order = ElementGeometry's HEX8 order) in file order, one type per
//     file; material id = rank of the element's physical tag among the
//     distinct physical tags of the volume elements (ascending); higher-order,
//     prism and pyramid volumes are rejected;
//   * Dirichlet node pairs = the edges of the triangles (type 2) and
//     quadrangles (type 3) whose physical tag is listed, or, with no list, the
//     edges of every boundary face (a face of exactly one volume element).
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
  int vol_type = 0;                // Gmsh type of the volume elements: 4 or 5
  std::vector<int64_t> vol_nodes;  // 4 or 8 per element, Gmsh node tags
  std::vector<int32_t> vol_phys;
  std::vector<int64_t> tri_nodes;  // 3 per triangle
  std::vector<int32_t> tri_phys;
  std::vector<int64_t> quad_nodes;  // 4 per quadrangle
  std::vector<int32_t> quad_phys;
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

// One element of Gmsh type `type` with nodes v: kept, skipped, or rejected.
int take(Raw& r, int64_t type, const int64_t* v, int32_t phys) {
  if (type == 4 || type == 5) {
    if (r.vol_type && r.vol_type != type) return fail("tetrahedra and hexahedra in one mesh are not supported");
    r.vol_type = static_cast<int>(type);
    r.vol_nodes.insert(r.vol_nodes.end(), v, v + (type == 4 ? 4 : 8));
    r.vol_phys.push_back(phys);
  } else if (type == 2) {
    r.tri_nodes.insert(r.tri_nodes.end(), v, v + 3);
    r.tri_phys.push_back(phys);
  } else if (type == 3) {
    r.quad_nodes.insert(r.quad_nodes.end(), v, v + 4);
    r.quad_phys.push_back(phys);
  } else if (type == 11 || type == 29 || type == 30 || type == 31) {
    return fail("higher-order tetrahedra are not TET4_EDGE meshes");
  } else if (type == 12 || type == 17 || type == 92 || type == 93) {
    return fail("higher-order hexahedra are not HEX8_EDGE meshes");
  } else if (type == 6 || type == 7 || type == 13 || type == 14 || type == 18 || type == 19) {
    return fail("prism and pyramid elements are not supported");
  }
  return EMG_SUCCESS;
}

// Nodes of Gmsh element types the reader has to step over.
int node_count(int64_t type) {
  switch (type) {
    case 15: return 1;
    case 1: return 2;
    case 2: case 8: return 3;
    case 3: case 4: return 4;
    case 7: return 5;
    case 6: case 9: return 6;
    case 5: return 8;
    case 16: return 8;
    case 10: return 9;
    case 11: return 10;
    default: return -1;
  }
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
    if (type == 2 || type == 3 || type == 4 || type == 5) {
      const int nv = node_count(type);
      int64_t v[8];
      for (int k = 0; k < nv; ++k) ls >> v[k];
      if (!ls) return fail("bad element line");
      if (int rc = take(r, type, v, phys)) return rc;
    } else if (int rc = take(r, type, nullptr, phys)) {
      return rc;
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
    if (int rc = take(r, type == 2 || type == 3 || type == 4 || type == 5 ? 0 : type, nullptr, p)) return rc;
    const int nv = node_count(type);
    if (nv < 0) return fail("unsupported element type " + std::to_string(type));
    for (int64_t i = 0; i < cnt; ++i) {
      int64_t id = 0, v[10];
      in >> id;
      for (int k = 0; k < nv; ++k) in >> v[k];
      if (type == 2 || type == 3 || type == 4 || type == 5)
        if (int rc = take(r, type, v, p)) return rc;
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
  if (r.vol_phys.empty()) return fail("no 4-node tetrahedra or 8-node hexahedra");
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
  const bool hex = r.vol_type == 5;
  m.elem_type = hex ? EMG_ELEM_HEX8_EDGE : EMG_ELEM_TET4_EDGE;
  const int npe = m.npe();
  m.n_elems = static_cast<int64_t>(r.vol_phys.size());
  m.elems.resize(npe * m.n_elems);
  for (size_t i = 0; i < r.vol_nodes.size(); ++i)
    if (!idx(r.vol_nodes[i], m.elems[i])) return fail("element references an unknown node");
  material_tags = r.vol_phys;
  std::sort(material_tags.begin(), material_tags.end());
  material_tags.erase(std::unique(material_tags.begin(), material_tags.end()), material_tags.end());
  m.material.resize(m.n_elems);
  for (int64_t t = 0; t < m.n_elems; ++t)
    m.material[t] = static_cast<int32_t>(std::lower_bound(material_tags.begin(), material_tags.end(), r.vol_phys[t]) -
                                         material_tags.begin());
  // Dirichlet node pairs: a triangle's 3 corner pairs (0,1), (1,2), (0,2);
  // a quadrangle's 4 sides from its corners in cyclic order (no diagonals)
  auto add_face = [&](const int32_t* v, int nv) {
    const int tri[3][2] = {{0, 1}, {1, 2}, {0, 2}};
    for (int k = 0; k < nv; ++k) {
      m.dirichlet.push_back(nv == 3 ? v[tri[k][0]] : v[k]);
      m.dirichlet.push_back(nv == 3 ? v[tri[k][1]] : v[(k + 1) % nv]);
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
      add_face(v, 3);
    }
    for (size_t f = 0; f < r.quad_phys.size(); ++f) {
      if (!std::binary_search(want.begin(), want.end(), r.quad_phys[f])) continue;
      int32_t v[4];
      for (int k = 0; k < 4; ++k)
        if (!idx(r.quad_nodes[4 * f + k], v[k])) return fail("quadrangle references an unknown node");
      add_face(v, 4);
    }
  } else {
    // faces of exactly one volume element, corners in cyclic order
    // (ElementGeometry's TET4 / HEX8 faces, element_geometry.cpp:112-181)
    const int tf[4][4] = {{0, 1, 2, -1}, {0, 1, 3, -1}, {0, 2, 3, -1}, {1, 2, 3, -1}};
    const int hf[6][4] = {{0, 1, 2, 3}, {4, 5, 6, 7}, {0, 1, 5, 4}, {2, 3, 7, 6}, {0, 3, 7, 4}, {1, 2, 6, 5}};
    const int nf = hex ? 6 : 4, nv = hex ? 4 : 3;
    struct Face {
      std::array<int32_t, 4> key;  // sorted corners (-1 padded)
      std::array<int32_t, 4> cyc;  // corners in cyclic order
    };
    std::vector<Face> faces;
    faces.reserve(static_cast<size_t>(nf) * m.n_elems);
    for (int64_t t = 0; t < m.n_elems; ++t)
      for (int f = 0; f < nf; ++f) {
        Face fc;
        fc.cyc = {-1, -1, -1, -1};
        for (int k = 0; k < nv; ++k) fc.cyc[k] = m.elems[npe * t + (hex ? hf[f][k] : tf[f][k])];
        fc.key = fc.cyc;
        std::sort(fc.key.begin(), fc.key.begin() + nv);
        faces.push_back(fc);
      }
    std::sort(faces.begin(), faces.end(), [](const Face& x, const Face& y) { return x.key < y.key; });
    for (size_t i = 0; i < faces.size();) {
      size_t j = i;
      while (j < faces.size() && faces[j].key == faces[i].key) ++j;
      if (j - i == 1) add_face(nv == 3 ? faces[i].key.data() : faces[i].cyc.data(), nv);
      i = j;
    }
  }
  return EMG_SUCCESS;
}

}  // namespace emg

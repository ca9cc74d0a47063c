// internal.h -- shared host-side declarations of libemagddm_b200.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "emagddm_b200.h"

namespace emg {

// Thread-local error message behind emg_last_error().
void set_error(const std::string& msg);

// Local node pairs of the element edges, ElementGeometry::get_local_edges
// (src/fe_em/element_geometry.cpp:115-126 TET4, :161-181 HEX8, :214-237
// PRISM6, :268-289 PYRAMID5).
constexpr int kTetEdge[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
constexpr int kHexEdge[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                 {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
constexpr int kPrismEdge[9][2] = {{0, 1}, {1, 2}, {0, 2}, {3, 4}, {4, 5}, {3, 5}, {0, 3}, {1, 4}, {2, 5}};
constexpr int kPyramidEdge[8][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {0, 4}, {1, 4}, {2, 4}, {3, 4}};

inline bool valid_single_type(int32_t t) {
  return t == EMG_ELEM_TET4_EDGE || t == EMG_ELEM_HEX8_EDGE || t == EMG_ELEM_PRISM6_EDGE ||
         t == EMG_ELEM_PYRAMID5_EDGE;
}
inline bool valid_elem_type(int32_t t) { return valid_single_type(t) || t == EMG_ELEM_MIXED; }
// Row width and edge slots of an element array (EMG_ELEM_MIXED: 9 and 12).
inline int nodes_per_elem(int32_t t) {
  return t == EMG_ELEM_HEX8_EDGE       ? 8
         : t == EMG_ELEM_PRISM6_EDGE   ? 6
         : t == EMG_ELEM_PYRAMID5_EDGE ? 5
         : t == EMG_ELEM_MIXED         ? 9
                                       : 4;
}
inline int edges_per_elem(int32_t t) {
  return t == EMG_ELEM_HEX8_EDGE || t == EMG_ELEM_MIXED ? 12
         : t == EMG_ELEM_PRISM6_EDGE                    ? 9
         : t == EMG_ELEM_PYRAMID5_EDGE                  ? 8
                                                        : 6;
}
inline const int (*local_edges(int32_t t))[2] {
  return t == EMG_ELEM_HEX8_EDGE       ? kHexEdge
         : t == EMG_ELEM_PRISM6_EDGE   ? kPrismEdge
         : t == EMG_ELEM_PYRAMID5_EDGE ? kPyramidEdge
                                       : kTetEdge;
}
// Type of one element row (a mixed mesh's rows carry it in slot 8).
inline int32_t row_type(int32_t elem_type, const int32_t* row) { return elem_type == EMG_ELEM_MIXED ? row[8] : elem_type; }
// Validates one row: its type and its node indices (-1 in the unused slots
// of a mixed row).
inline bool valid_row(int32_t elem_type, const int32_t* row, int64_t n_nodes) {
  const int32_t et = row_type(elem_type, row);
  if (!valid_single_type(et)) return false;
  const int nn = nodes_per_elem(et);
  for (int a = 0; a < nn; ++a)
    if (row[a] < 0 || row[a] >= n_nodes) return false;
  if (elem_type == EMG_ELEM_MIXED)
    for (int a = nn; a < 8; ++a)
      if (row[a] != -1) return false;
  return true;
}

struct Mesh {
  int32_t elem_type = EMG_ELEM_TET4_EDGE;
  int64_t n_nodes = 0;
  int64_t n_elems = 0;
  std::vector<double> xyz;        // 3 * n_nodes
  std::vector<int32_t> elems;     // npe() * n_elems
  std::vector<int32_t> material;  // n_elems
  std::vector<int32_t> dirichlet; // 2 * n_dirichlet
  int32_t n_hole_markers = 0;
  // lazily built edge table
  bool edges_built = false;
  int64_t n_edges = 0;
  std::vector<int32_t> elem_edge;   // epe() * n_elems
  std::vector<int32_t> edge_nodes;  // 2 * n_edges, (lo, hi) global node IDs
  int npe() const { return nodes_per_elem(elem_type); }
  int epe() const { return edges_per_elem(elem_type); }
};

struct DofMap {
  int32_t elem_type = EMG_ELEM_TET4_EDGE;
  int64_t n_elems = 0;
  int64_t n_edges = 0;
  int64_t n_free = 0;
  int64_t n_dofs = 0;
  int32_t root = -1;
  std::vector<int32_t> l2g;       // edges_per_elem * n_elems
  std::vector<int32_t> edge_dof;  // n_edges
  // Set by the partitioned gauge only.
  int32_t n_parts = 0;
  std::vector<int32_t> tet_part;    // n_elems, subdomain of every element
  std::vector<uint8_t> dof_primal;  // n_dofs, 1 = primal (coarse) DOF
  int64_t n_primal_fix = 0;         // primal DOFs added to connect a subdomain
};

// Host integer numbering (numbering.cpp).
int build_edge_ids(Mesh& m);
int build_dofmap(Mesh& m, int32_t gauge_mode, DofMap& out);
int build_dofmap_partitioned(Mesh& m, const int32_t* tet_part, int32_t n_parts, DofMap& out);
// EMDOFManager with per-element DOF types (SCALAR_ONLY / VECTOR_EDGE_ONLY /
// MIXED_AV); l2g rows of npe + epe entries padded with EMG_DOF_ABSENT.
int build_dofmap_av(const Mesh& m, const int32_t* dof_type, int64_t n_sdir, const int32_t* sdir,
                    int32_t gauge_mode, std::vector<int32_t>& l2g, int64_t& n_scalar_free, int64_t& n_free,
                    int64_t& n_dofs);
// Gmsh ASCII reader (gmsh.cpp); material_tags[i] = physical tag of material i.
int read_gmsh(const std::string& path, const int32_t* dirichlet_tags, int32_t n_tags, Mesh& m,
              std::vector<int32_t>& material_tags);

// Materials, objects and boundaries of an Ansys Maxwell project file
// (aedt.cpp).
struct AedtProject {
  struct Material {
    std::string name;
    double mu_r = 1.0, sigma = 0.0;
    int32_t flags = 0;  // 1 nonlinear (BH curve), 2 permeability not a number, 4 conductivity not a number
    std::vector<double> h, b;  // BH curve of a nonlinear material
  };
  struct Object {
    std::string name, material;
    int32_t solve_inside = 1;
  };
  struct Boundary {
    std::string name, type, value;
  };
  std::vector<Material> materials;
  std::vector<Object> objects;
  std::vector<Boundary> boundaries;
};
int aedt_read(const std::string& path, AedtProject& out);

}  // namespace emg

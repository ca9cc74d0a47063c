// internal.h -- shared host-side declarations of libemagddm_b200.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "emagddm_b200.h"

namespace emg {

// Thread-local error message behind emg_last_error().
void set_error(const std::string& msg);

struct Mesh {
  int64_t n_nodes = 0;
  int64_t n_tets = 0;
  std::vector<double> xyz;        // 3 * n_nodes
  std::vector<int32_t> tets;      // 4 * n_tets
  std::vector<int32_t> material;  // n_tets
  std::vector<int32_t> dirichlet; // 2 * n_dirichlet
  int32_t n_hole_markers = 0;
  // lazily built edge table
  bool edges_built = false;
  int64_t n_edges = 0;
  std::vector<int32_t> elem_edge;   // 6 * n_tets
  std::vector<int32_t> edge_nodes;  // 2 * n_edges, (lo, hi) global node IDs
};

struct DofMap {
  int64_t n_tets = 0;
  int64_t n_edges = 0;
  int64_t n_free = 0;
  int64_t n_dofs = 0;
  int32_t root = -1;
  std::vector<int32_t> l2g;       // 6 * n_tets
  std::vector<int32_t> edge_dof;  // n_edges
  // Set by the partitioned gauge only.
  int32_t n_parts = 0;
  std::vector<int32_t> tet_part;    // n_tets, subdomain of every tet
  std::vector<uint8_t> dof_primal;  // n_dofs, 1 = primal (coarse) DOF
  int64_t n_primal_fix = 0;         // primal DOFs added to connect a subdomain
};

// Host integer numbering (numbering.cpp).
int build_edge_ids(Mesh& m);
int build_dofmap(Mesh& m, int32_t gauge_mode, DofMap& out);
int build_dofmap_partitioned(Mesh& m, const int32_t* tet_part, int32_t n_parts, DofMap& out);
// Gmsh ASCII reader (gmsh.cpp); material_tags[i] = physical tag of material i.
int read_gmsh(const std::string& path, const int32_t* dirichlet_tags, int32_t n_tags, Mesh& m,
              std::vector<int32_t>& material_tags);

}  // namespace emg

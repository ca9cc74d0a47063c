// fetidp.h -- FETI-DP for the partitioned, gauged TET4_EDGE system: host plan
// (symbolic phase) and the device solver built on it.
//
// Notation (per subdomain s): I = interior DOFs (one subdomain), D = dual
// DOFs (shared by two subdomains, glued by one Lagrange multiplier each),
// P = primal DOFs (coarse, assembled), r = I u D.  Local DOF positions are the
// elimination order: I in nested-dissection postorder, then D (ascending
// global DOF), then P (ascending global DOF).  The union ("block-diagonal")
// numbering places subdomain s at loc_off[s] .. loc_off[s+1].
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "internal.h"

namespace emg {

struct FetiFront {
  int32_t sub = 0;      // subdomain
  int32_t p0 = 0;       // first pivot (local position)
  int32_t npiv = 0;
  int32_t f = 0;        // front size = npiv + nupd
  int32_t height = 0;
  int32_t parent = -1;  // front index or -1
  int32_t child0 = 0, nchild = 0;  // children: child_list[child0 .. child0 + nchild)
  int32_t is_root = 0;  // the D front of its subdomain
  int64_t rows = 0;     // offset into rows[]: f local positions, ascending
  int64_t fac = 0;      // offset of the f x npiv factor block (column-major, ld f)
  int64_t upd = -1;     // offset of the nupd x nupd update block in the update pool
  int64_t cpos = 0;     // offset into cpos[]: nupd positions in the parent front
  int64_t vec = 0;      // offset of the update-vector rows (nupd) in the solve pool
};

struct FetiPlan {
  int32_t n_parts = 0;
  int64_t n_dofs = 0, n_union = 0;
  std::vector<int64_t> loc_off;           // n_parts + 1
  std::vector<int32_t> nI, nD, nP;        // per subdomain
  std::vector<int32_t> l2g_union;         // edges_per_elem * n_elems
  std::vector<int32_t> union_gdof;        // n_union
  std::vector<int64_t> gptr;              // n_dofs + 1
  std::vector<int32_t> glist;             // union positions of each global DOF
  // multipliers
  int64_t n_lambda = 0;
  std::vector<int64_t> dual_off;          // n_parts + 1 (dual entry = (s, D position))
  std::vector<int32_t> dual_lam, dual_sign;
  std::vector<int32_t> lam_entry;         // 2 * n_lambda: (+) and (-) dual entries
  // coarse
  int32_t n_coarse = 0;
  std::vector<int64_t> pri_off;           // n_parts + 1 (primal entry = (s, P position))
  std::vector<int32_t> pri_coarse;        // per primal entry
  std::vector<int64_t> coarse_ptr;        // n_coarse + 1
  std::vector<int32_t> coarse_list;       // primal entries of each coarse DOF (ascending s)
  std::vector<int64_t> cblk_off;          // n_parts + 1: nP x nP coarse blocks
  std::vector<int64_t> sc_ptr;            // n_coarse^2 + 1 (column-major targets)
  std::vector<int64_t> sc_list;           // coarse-block entries per target
  // faces (deluxe scaling): the multipliers grouped by their subdomain pair
  int32_t n_faces = 0;
  std::vector<int32_t> face_a, face_b;    // subdomains, face_a < face_b
  std::vector<int64_t> face_ptr;          // n_faces + 1 into face_lam
  std::vector<int32_t> face_lam;          // multipliers of each face, ascending
  std::vector<int64_t> face_off;          // n_faces + 1: f x f dense blocks (padded)
  // fronts (level order: by height, then subdomain, then postorder)
  std::vector<FetiFront> fronts;
  std::vector<int32_t> level_ptr;         // n_levels + 1
  std::vector<int32_t> rows, child_list, cpos;
  std::vector<int32_t> root_front;        // per subdomain, -1 without D
  std::vector<int64_t> root_off;          // n_parts + 1: nD x nD blocks (S, L^-1)
  int64_t fac_size = 0;                   // doubles
  int64_t upd_pool = 0;                   // doubles (first-fit over front lifetimes)
  int64_t vec_rows = 0;                   // update-vector rows over all fronts
  int32_t max_front = 0, max_npiv = 0, max_children = 0;
};

// Builds the plan from a partitioned DOF map (emg_dof_build_partitioned).
int build_feti_plan(const Mesh& m, const DofMap& d, FetiPlan& p);
// Checks every index of the plan against the sizes it addresses.
int validate_feti_plan(const FetiPlan& p);
// One 128 x 128 tensor-core tile C -= A B^T (device arrays; test hook).
int tc_tile_test(int32_t mr, int32_t mc, int32_t K, const double* A, int64_t lda, const double* B, int64_t ldb,
                 double* C, int64_t ldc, cudaStream_t st);

}  // namespace emg

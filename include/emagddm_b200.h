/*
 * emagddm_b200.h -- C ABI of the B200-native TET4 Nedelec curl-curl solve path.
 *
 * The entry points replace the CPU chain of Poofee/emagddm
 *   GlobalEdgeIDGenerator -> EMDOFManager (+ TreeGauge) -> EMAssembly
 *   -> CsrMatrix -> CGSolver / BiCGSTABSolver
 * with host C++ integer numbering and hand-written sm_100a CUDA kernels.  Each
 * declaration cites the reference interface it replaces (paths inside the
 * reference project).
 *
 * Conventions
 *   - Every function returns an int status; 0 (EMG_SUCCESS) means the call
 *     ran.  Solver entry points return the solver outcome (the values of
 *     numeric::SolverStatus, include/numeric/em_linear_solver.h:26-32) and
 *     also store it in emg_result.status.  Nothing throws across the ABI.
 *   - emg_last_error() returns a message for the last failing call of the
 *     calling thread.
 *   - Pointers are host pointers unless the name ends in _d (device).
 *   - Handles own their device memory; arrays passed in are copied; arrays
 *     passed out are caller-allocated.  One handle per thread / stream.
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default).
 *   - Indices are 0-based int32 (the reference uses int throughout).
 */
#ifndef EMAGDDM_B200_H
#define EMAGDDM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EMG_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------- */
enum {
  EMG_SUCCESS = 0,          /* SolverStatus::SUCCESS           */
  EMG_NUMERICAL_ERROR = 1,  /* SolverStatus::NUMERICAL_ERROR   */
  EMG_DIVERGED = 2,         /* SolverStatus::DIVERGED          */
  EMG_MAX_ITER_REACHED = 3, /* SolverStatus::MAX_ITER_REACHED  */
  EMG_INVALID_INPUT = 4,    /* SolverStatus::INVALID_INPUT     */
  EMG_ERR_CUDA = 5,         /* a CUDA runtime call failed      */
  EMG_ERR_TIMEOUT = 6,      /* a bounded device wait ran out   */
  EMG_ERR_NOMEM = 7,        /* host or device allocation failed */
  EMG_ERR_INTERNAL = 8      /* device-side consistency check failed */
};

/* ---- gauge modes (EMDOFManager::applyTreeGauge) -------------------------- */
enum {
  EMG_GAUGE_NONE = -1,          /* EMDOFManager::build only                   */
  EMG_GAUGE_REF = 0,            /* reference tree gauge, bit-exact numbering  */
  EMG_GAUGE_BOUNDARY_FIRST = 1  /* tree spans the Dirichlet boundary first    */
};

/* ---- element types (numeric::ElementType, include/numeric/shape_function_base.hpp:51-57)
 * One type per mesh.  Local node and edge order follow ElementGeometry
 * (src/fe_em/element_geometry.cpp:112-126 TET4, :158-181 HEX8, :214-237
 * PRISM6, :268-289 PYRAMID5). */
enum {
  EMG_ELEM_TET4_EDGE = 0,    /* 4 nodes, 6 edges                                     */
  EMG_ELEM_HEX8_EDGE = 1,    /* 8 nodes (bottom face 0-3, top face 4-7 above them), 12 edges */
  EMG_ELEM_PRISM6_EDGE = 2,  /* 6 nodes (bottom triangle 0-2, top 3-5 above them), 9 edges */
  EMG_ELEM_PYRAMID5_EDGE = 3, /* 5 nodes (base quadrilateral 0-3, apex 4), 8 edges    */
  /* A mesh of several of the types above (per element, as fe_em::Element::
   * elem_type): every element is a row of 9 ints -- its nodes in the order of
   * its own type, -1 in the unused node slots, and its type (EMG_ELEM_TET4_EDGE
   * .. EMG_ELEM_PYRAMID5_EDGE) in slot 8 -- and has 12 entries in l2g (-1 past
   * its own edges).  Numbering, assembly and the Krylov solvers take it; in
   * such a mesh the hexahedron's edge functions are scaled to unit
   * circulation (1/4 of the reference's) to agree with the other elements on
   * shared edges. */
  EMG_ELEM_MIXED = 4
};

/* ---- assembly flags ------------------------------------------------------ */
enum {
  EMG_FLAG_MASS = 1,           /* also assemble M_ij = int sigma W_i . W_j      */
  EMG_FLAG_NO_EDGE_SIGNS = 2,  /* scatter unsigned element matrices            */
  EMG_FLAG_PIOLA_LITERAL = 4,  /* W_phys = J^-T W_ref / detJ (reference text)   */
  EMG_FLAG_QUAD3_LITERAL = 8,  /* the reference's 3-point TET4 rule             */
  EMG_FLAG_FACTOR_TF32 = 16    /* FETI-DP / direct factor: subdomain contractions
                                  on the TF32 tensor cores (two-term split, FP32
                                  accumulation); FP64 refinement on the true
                                  residual restores full accuracy */
};

/* ---- source regions: J evaluated at quadrature points ------------------- */
enum { EMG_SRC_BOX = 1, EMG_SRC_ANNULUS_Z = 2 };
typedef struct {
  int32_t kind;   /* EMG_SRC_*                                                  */
  double j[3];    /* current density inside the region                          */
  double p[6];    /* BOX: xmin,xmax,ymin,ymax,zmin,zmax (open intervals)        */
                  /* ANNULUS_Z: cx,cy,rmin,rmax,zmin,zmax (r from (cx,cy), open) */
} emg_source;

/* ---- solver configuration and result ------------------------------------ */
/* CGConfig / BiCGSTABConfig::PreconditionerType (iterative_solvers.h:59-76).
 * ILU0: the reference factors Eigen::IncompleteLUT (fill factor 10, drop
 * tolerance 1e-12; iterative_solvers.h:324, .cpp:277-286); the GPU solvers
 * factor ILU(0) on the matrix's own pattern (level-scheduled kernels, the
 * factor kept with the matrix until its values change) and run the
 * reference's CG / BiCGSTAB ILU0 iterations (.cpp:505-585, :1121-1243).  The
 * fill differs, so iteration counts differ; a factorization that breaks down
 * (missing diagonal, zero or non-finite pivot) leaves the solve without a
 * preconditioner, as the reference's does.  Any other value is rejected with
 * EMG_INVALID_INPUT; the batched and allocation-free solvers take NONE and
 * JACOBI only. */
enum { EMG_PRECOND_NONE = 0, EMG_PRECOND_JACOBI = 1, EMG_PRECOND_ILU0 = 2 };
typedef struct {
  double tolerance;          /* ||r||/||b|| stop threshold (IterativeSolverConfig, default 1e-8) */
  int32_t max_iterations;    /* default 1000                                          */
  int32_t preconditioner;    /* EMG_PRECOND_*                                          */
} emg_krylov_config;

typedef struct {
  int32_t status;            /* SolverStatus value                           */
  int32_t iterations;        /* iterations performed                         */
  double residual_norm;      /* relative residual ||r||/||b||                */
  double solve_time_ms;      /* device time of the solve (CUDA events)       */
} emg_result;                /* numeric::SolverResult, em_linear_solver.h:53-61 */

typedef struct emg_mesh_t* emg_mesh;
typedef struct emg_dofmap_t* emg_dofmap;
typedef struct emg_system_t* emg_system;
typedef struct emg_csr_t* emg_csr;

/* ---- library ------------------------------------------------------------ */
int32_t emg_abi_version(void);
const char* emg_last_error(void);

/* ---- mesh: fe_em::EMMeshData (include/fe_em/em_mesh_data.hpp:90-230) ----
 * xyz: 3*n_nodes; tets: 4*n_tets (TET4_EDGE, VECTOR_EDGE_ONLY); material_id:
 * n_tets or NULL; dirichlet_pairs: 2*n_dirichlet node pairs of the
 * DIRICHLET / VECTOR_EDGE_ONLY marker; n_hole_markers: number of boundary
 * markers the reference's name heuristic counts as holes
 * (src/fe_em/multi_connected_domain.cpp:126-188). */
int emg_mesh_create(int64_t n_nodes, const double* xyz, int64_t n_tets, const int32_t* tets,
                    const int32_t* material_id, int64_t n_dirichlet,
                    const int32_t* dirichlet_pairs, int32_t n_hole_markers, emg_mesh* out);
/* Same for a mesh of one element type (EMG_ELEM_*): elems holds
 * nodes_per_elem * n_elems node indices (4 TET4_EDGE, 8 HEX8_EDGE, 6 PRISM6_EDGE,
 * 5 PYRAMID5_EDGE);
 * emg_mesh_create is elem_type = EMG_ELEM_TET4_EDGE.  Everything downstream
 * (edge IDs, DOF maps, gauges, systems, the FETI-DP and direct solvers) then
 * works per element with edges_per_elem (6, 12, 9 or 8) local edges; arrays
 * documented below as 4*n_tets / 6*n_tets hold nodes_per_elem*n_elems /
 * edges_per_elem*n_elems entries for such a mesh. */
int emg_mesh_create_typed(int32_t elem_type, int64_t n_nodes, const double* xyz, int64_t n_elems,
                          const int32_t* elems, const int32_t* material_id, int64_t n_dirichlet,
                          const int32_t* dirichlet_pairs, int32_t n_hole_markers, emg_mesh* out);
/* Element type, nodes and edges per element of a mesh; any pointer may be NULL. */
int emg_mesh_elem_type(emg_mesh mesh, int32_t* elem_type, int32_t* nodes_per_elem,
                       int32_t* edges_per_elem);
void emg_mesh_destroy(emg_mesh mesh);
/* Gmsh ASCII mesh (format 2.2 or 4.1; the reference's planned mesh format,
 * mesh/README.md) as an EMMeshData (include/fe_em/em_mesh_data.hpp:90-230):
 * nodes in ascending Gmsh tag order, the 4-node tetrahedra (type 4) or the
 * 8-node hexahedra (type 5; one volume type per file; emg_mesh_elem_type
 * tells which) in file order with material id = rank of their physical tag
 * among the volume elements' distinct physical tags, Dirichlet node pairs =
 * edges of the triangles / quadrangles (types 2 / 3) whose physical tag is in
 * dirichlet_tags, or of every boundary face (a face of one volume element)
 * when n_tags == 0.  Binary files, mixed tetrahedra and hexahedra,
 * higher-order, prism and pyramid volumes are rejected with
 * EMG_INVALID_INPUT. */
int emg_mesh_read_gmsh(const char* path, const int32_t* dirichlet_tags, int32_t n_tags, emg_mesh* out);
/* Sizes of a mesh handle; any pointer may be NULL. */
int emg_mesh_info(emg_mesh mesh, int64_t* n_nodes, int64_t* n_tets, int64_t* n_dirichlet_pairs,
                  int32_t* n_materials);
/* Copies out 3*n_nodes coordinates, 4*n_tets nodes, n_tets material ids and
 * 2*n_dirichlet_pairs nodes; any pointer may be NULL. */
int emg_mesh_export(emg_mesh mesh, double* xyz, int32_t* tets, int32_t* material, int32_t* dirichlet_pairs);
/* Physical tag of each material id (n_materials values) of a Gmsh mesh. */
int emg_mesh_material_tags(emg_mesh mesh, int32_t* tags);

/* ---- GlobalEdgeIDGenerator::generate (src/fe_em/global_edge_id_generator.cpp:30-110)
 * elem_edge: 6*n_tets output or NULL; edge_nodes: 2*n_edges sorted node pair
 * per edge or NULL (size the buffer with a first call passing NULL). */
int emg_edge_ids(emg_mesh mesh, int32_t* elem_edge, int32_t* edge_nodes, int64_t* n_edges);

/* ---- EMDOFManager::build (src/fe_em/em_dof_manager.cpp:29-65) and, for
 * gauge_mode >= 0, EMDOFManager::applyTreeGauge (:448-495) with TreeGauge::build
 * (src/fe_em/tree_gauge.cpp:37-212). */
int emg_dof_build(emg_mesh mesh, int32_t gauge_mode, emg_dofmap* out);
int emg_dofmap_info(emg_dofmap map, int64_t* n_edges, int64_t* n_free, int64_t* n_dofs);
/* l2g: 6*n_tets Local2Global::indices (-1 = constrained or tree edge);
 * edge_dof: n_edges (equation index of each global edge or -1). */
int emg_dofmap_export(emg_dofmap map, int32_t* l2g, int32_t* edge_dof);
/* TreeGauge::mapReducedSolutionToFull (src/fe_em/tree_gauge.cpp:261-290):
 * full[e] = reduced[edge_dof[e]] or 0. */
int emg_dofmap_expand(emg_dofmap map, const double* reduced, double* full);
void emg_dofmap_destroy(emg_dofmap map);
/* emg_dof_build on the device: the same edge IDs, free numbering and `ref`
 * tree-cotree gauge, bit for bit, computed by GPU kernels from DEVICE arrays
 * (elems: nodes_per_elem * n_elems node indices, or the 9-int rows of an
 * EMG_ELEM_MIXED mesh; dir_pairs: 2 * n_dir
 * Dirichlet node pairs) into the device array l2g (edges_per_elem * n_elems
 * Local2Global::indices, -1 = constrained or tree edge), ready for
 * emg_system_create_typed with on_device = 1.  gauge_mode: EMG_GAUGE_NONE or
 * EMG_GAUGE_REF (EMG_GAUGE_BOUNDARY_FIRST is host-only: emg_dof_build).
 * Returns the edge, free and equation counts; blocks the calling host thread
 * (one read-back per tree level). */
int emg_dof_build_device(int32_t elem_type, int64_t n_nodes, int64_t n_elems, const int32_t* elems,
                         int64_t n_dir, const int32_t* dir_pairs, int32_t n_hole_markers, int32_t gauge_mode,
                         int32_t* l2g, int64_t* n_edges, int64_t* n_free, int64_t* n_dofs, void* stream);

/* ---- Per-element DOF types: EMDOFManager::build with Element::dof_type
 * (include/fe_em/em_mesh_data.hpp:45-49).  SCALAR_ONLY elements carry nodal
 * DOFs, VECTOR_EDGE_ONLY edge DOFs, MIXED_AV both (the A-V formulation):
 * assignPrenumbering (src/fe_em/em_dof_manager.cpp:91-150) numbers the nodes
 * of the scalar-carrying elements in ascending ID, then the edges of the
 * vector-carrying elements by first appearance; markConstrainedDOFs
 * (:152-243) takes the scalar_dirichlet node IDs and the mesh's Dirichlet
 * edge pairs; renumberFreeDOFs (:245-286) ranks the unconstrained, scalars
 * first; the element maps (:288-446) list node DOFs, edge DOFs, or node then
 * edge DOFs.  For gauge_mode >= 0, applyTreeGauge (:448-626) gauges the edge
 * DOFs with the tree of the vector-carrying elements; they keep following
 * the free scalar DOFs.
 * dof_type: n_elems values, or NULL for all MIXED_AV.
 * l2g: (nodes_per_elem + edges_per_elem) * n_elems or NULL; row e holds
 *   Local2Global::indices of element e, padded with EMG_DOF_ABSENT
 *   (-1 = constrained DOF or tree edge, as everywhere).
 * n_scalar_free: free scalar DOFs, equations 0 .. n_scalar_free - 1;
 * n_free: free DOFs before the gauge; n_dofs: equations.  Any output may be
 * NULL.  EMG_INVALID_INPUT for a dof_type value outside the enum. */
enum { EMG_DOF_SCALAR_ONLY = 0, EMG_DOF_VECTOR_EDGE_ONLY = 1, EMG_DOF_MIXED_AV = 2, EMG_DOF_ABSENT = -2 };
int emg_dof_build_av(emg_mesh mesh, const int32_t* dof_type, int64_t n_scalar_dirichlet,
                     const int32_t* scalar_dirichlet, int32_t gauge_mode, int32_t* l2g,
                     int64_t* n_scalar_free, int64_t* n_free, int64_t* n_dofs);

/* ---- Tree-cotree gauge for a non-overlapping partition of the tets, the
 * numbering the FETI-DP solver below works on.  No reference counterpart:
 * the reference's FETI-DP layer is a stub (include/fetidp/fetidp_context.hpp:20-66,
 * src/fetidp/fetidp_context.cpp:15-45).  tet_part[t] in [0, n_parts).  The
 * tree spans the Dirichlet surface, then the subdomain wire baskets (edges
 * shared by >= 3 subdomains), then each face, then each interior; reduced DOFs
 * are the unconstrained cotree edges in ascending edge ID (as in the `ref`
 * gauge's reduced map).  Primal DOFs: the cotree wire-basket edges, plus any
 * cotree edge needed to connect a subdomain's tree.  Hole markers are
 * rejected. */
int emg_dof_build_partitioned(emg_mesh mesh, const int32_t* tet_part, int32_t n_parts,
                              emg_dofmap* out);
/* Partition data of a map from emg_dof_build_partitioned: primal: n_dofs flags
 * (1 = primal) or NULL; n_parts / n_primal / n_primal_fix may be NULL.
 * EMG_INVALID_INPUT for a map without a partition. */
int emg_dofmap_partition_info(emg_dofmap map, int32_t* n_parts, int64_t* n_primal,
                              int64_t* n_primal_fix, int32_t* primal);

/* ---- FETI-DP (dual-primal domain decomposition) of the gauged curl-curl
 * system on one GPU.  The reference has only the FETI-DP context
 * (include/fetidp/fetidp_context.hpp:20-66: subdomain count and zeroed
 * SubdomainData); the operators it leaves out are built here:
 *   - local Neumann matrices K^(s) of every subdomain (one block-diagonal
 *     GPU assembly), K_rr^(s) factored by a batched multifrontal Cholesky
 *     (nested dissection inside the subdomain, dual DOFs last);
 *   - the jump operator B (one multiplier per dual DOF, +1 on the lower
 *     subdomain id) and its transpose;
 *   - the primal coarse Schur complement S_cc, factored on the GPU;
 *   - the Dirichlet preconditioner, scaled per face by "deluxe" weights
 *     (S_a,F + S_b,F)^-1 S_b,F built from the two sides' Schur complements,
 *     which keeps the iteration count flat across coefficient jumps that cut
 *     through subdomains, or by diagonal stiffness weights.
 * The interface problem is solved by FP64 PCG; x is the global solution in
 * the partitioned map's numbering (n_dofs), out->residual_norm the true
 * ||F - K x|| / ||F|| of the global system and cfg->tolerance the bound on
 * it: multiplier PCG passes with defect correction on the true residual
 * (each pass's multiplier tolerance from the measured amplification of the
 * dual jump) until it holds or cfg->max_iterations multiplier iterations are
 * spent in total.  cfg->preconditioner: EMG_FETI_PRECOND_NONE, _STIFFNESS,
 * _DELUXE or _DELUXE_FP32.  map must come from emg_dof_build_partitioned on
 * the same mesh. */
enum {
  EMG_FETI_PRECOND_NONE = 0,
  EMG_FETI_PRECOND_STIFFNESS = 1,
  EMG_FETI_PRECOND_DELUXE = 2,
  EMG_FETI_PRECOND_DELUXE_FP32 = 3  /* deluxe, S_DD and face weights stored in FP32 (mixed precision) */
};
typedef struct emg_fetidp_t* emg_fetidp;
int emg_fetidp_create(emg_mesh mesh, emg_dofmap map, void* stream, emg_fetidp* out);
/* Numeric phase (materials and sources as emg_system_assemble; EMG_FLAG_MASS
 * is ignored).  EMG_NUMERICAL_ERROR when a subdomain matrix is not positive
 * definite. */
int emg_fetidp_factor(emg_fetidp fd, const double* nu, const double* sigma, int32_t n_materials,
                      const emg_source* sources, int32_t n_sources, int32_t flags);
int emg_fetidp_solve(emg_fetidp fd, const emg_krylov_config* cfg, double* x, int32_t x_on_device,
                     emg_result* out);
/* Same for a caller's global right-hand side b (n_dofs, the partitioned map's
 * numbering) instead of the assembled F; b and x are both host or both device
 * arrays.  The factorization is reused, so many right-hand sides cost one
 * emg_fetidp_factor. */
int emg_fetidp_solve_rhs(emg_fetidp fd, const emg_krylov_config* cfg, const double* b, double* x,
                         int32_t on_device, emg_result* out);
/* ---- Learned interface preconditioner (no reference counterpart): one
 * 3-layer MLP per subdomain (width 256, BF16 weights, FP32 accumulation)
 * mapping the subdomain's normalised dual residual to a correction of the
 * deluxe Dirichlet step; preconditioner EMG_FETI_PRECOND_LEARNED solves with
 * flexible CG and z = M_D r + L(r), falling back to M_D r where that is not
 * a descent direction; the true FP64 residual still decides convergence.
 * Initialised with W3 = 0 (adds nothing until trained). */
enum { EMG_FETI_PRECOND_LEARNED = 4 };
int emg_fetidp_learned_init(emg_fetidp fd, uint64_t seed);
/* One Adam step on `batch` (residual, wanted correction) pairs: r_d, t_d are
 * device arrays of batch x n_lambda; loss (may be NULL) gets the mean squared
 * error of the normalised outputs before the step. */
int emg_fetidp_learned_train(emg_fetidp fd, int32_t batch, const double* r_d, const double* t_d, float lr,
                             double* loss);
/* FP32 master parameters (host array of *n floats): load != 0 copies in. */
int emg_fetidp_learned_params(emg_fetidp fd, float* params, int64_t* n, int32_t load);
/* Multiplier space, device vectors of n_lambda (emg_fetidp_info[3]):
 * op 0 F, 1 deluxe Dirichlet M_D, 2 learned correction L, 3 M_D + L. */
int emg_fetidp_apply(emg_fetidp fd, int32_t op, const double* in_d, double* out_d);
/* Right-hand side d - G S_cc^-1 g_c of the multiplier system for a global b
 * (device, n_dofs; NULL = the assembled F) into rhs_d (device, n_lambda). */
int emg_fetidp_lambda_rhs(emg_fetidp fd, const double* b_d, double* rhs_d);
/* Dual layout: dual_off (n_parts + 1) over the dual entries (subdomain,
 * dual DOF), each entry's multiplier and sign (+1 on the lower subdomain),
 * and lam_entry (2 per multiplier: its + and - entries).  NULL skips. */
int emg_fetidp_duals(emg_fetidp fd, int64_t* dual_off, int32_t* dual_lam, int32_t* dual_sign, int32_t* lam_entry);

/* info[0..21]: n_parts, n_dofs, n_union, n_lambda, n_coarse, n_fronts,
 * n_levels, max_front, max_pivots, factor doubles, update-pool doubles,
 * dual-block doubles, sum nI, sum nD, sum nP, max nD, max children, the
 * flops of the numeric phase (front panels, front update blocks, inverse
 * factors + deluxe weights), the S_DD entries the preconditioner reads a
 * multiplier iteration (64 x 64 tiles on and below the diagonal) and the
 * entries of one of each face's four deluxe blocks.  A shorter n_info
 * returns the first n_info values. */
int emg_fetidp_info(emg_fetidp fd, int64_t* info, int32_t n_info);
/* stats[0..7]: factor ms, solve ms, iterations, multiplier residual, true
 * residual, FETI-DP passes, and the solve's device ms split into the
 * multiplier iterations and the right-hand-side / recovery front solves. */
int emg_fetidp_stats(emg_fetidp fd, double* stats, int32_t n_stats);
void emg_fetidp_destroy(emg_fetidp fd);
/* Host-only symbolic analysis (no GPU needed): the info[] of the plan; a map
 * without a partition is analysed as one subdomain (the direct solver's plan). */
int emg_fetidp_plan_info(emg_mesh mesh, emg_dofmap map, int64_t* info, int32_t n_info);

/* ---- GPU sparse direct solver for the gauged system: the SolverBackend
 * role of MUMPSBackend / EigenLLTBackend (include/numeric/solver_backend.h:81-244,
 * include/numeric/mumps_solver_backend.h:96-140, eigen_solver_backends.h:338-420).
 * Nested dissection of the edge DOFs (edge midpoints), multifrontal Cholesky
 * on the GPU (fronts of one height factored together, FP64), then forward /
 * backward solves with iterative refinement on the true residual until
 * ||F - K x|| / ||F|| < cfg->tolerance (cfg->max_iterations bounds the
 * refinement passes; cfg->preconditioner is ignored).  map: any map of the
 * mesh (emg_dof_build with any gauge, or emg_dof_build_partitioned); the
 * system must be symmetric positive definite (a gauged curl-curl system is).
 * EMG_NUMERICAL_ERROR from emg_direct_factor when it is not. */
typedef struct emg_direct_t* emg_direct;
int emg_direct_create(emg_mesh mesh, emg_dofmap map, void* stream, emg_direct* out);
int emg_direct_factor(emg_direct d, const double* nu, const double* sigma, int32_t n_materials,
                      const emg_source* sources, int32_t n_sources, int32_t flags);
/* b: right-hand side (n_dofs) or NULL for the assembled F; b and x both host
 * or both device arrays. */
int emg_direct_solve(emg_direct d, const emg_krylov_config* cfg, const double* b, double* x,
                     int32_t on_device, emg_result* out);
/* info as emg_fetidp_info (one subdomain, no multipliers). */
int emg_direct_info(emg_direct d, int64_t* info, int32_t n_info);
void emg_direct_destroy(emg_direct d);

/* ---- EMAssembly::assemble on the GPU (src/numeric/em_assembly.cpp:144-420)
 * A system owns the device copy of the geometry and DOF map, the CSR pattern
 * (merged, rows sorted: what SparseConverter::to_eigen yields), the stiffness
 * values K, optional mass values M and the source vector F.
 * Geometry arrays: xyz 3*n_nodes, tets 4*n_tets, material n_tets (NULL = 0),
 * l2g 6*n_tets; n_dofs <= 0 means max index + 1 (em_assembly.cpp:190-215).
 * emg_system_create reads host arrays; emg_system_create_device reads device
 * arrays (resident inputs) and copies nothing back.  Both build the pattern
 * on the device. */
int emg_system_create(int64_t n_nodes, const double* xyz, int64_t n_tets, const int32_t* tets,
                      const int32_t* material, const int32_t* l2g, int64_t n_dofs, void* stream,
                      emg_system* out);
int emg_system_create_device(int64_t n_nodes, const double* xyz_d, int64_t n_tets,
                             const int32_t* tets_d, const int32_t* material_d,
                             const int32_t* l2g_d, int64_t n_dofs, void* stream, emg_system* out);
/* Either of the above for elements of type elem_type (EMG_ELEM_*): elems
 * nodes_per_elem*n_elems, material n_elems, l2g edges_per_elem*n_elems;
 * on_device selects device (1) or host (0) arrays.  HEX8_EDGE elements are
 * integrated with the 2x2x2 Gauss-Legendre rule (GaussQuadrature::getHex8Points,
 * src/numeric/gauss_quadrature.cpp:232-276) on the trilinear map. */
int emg_system_create_typed(int32_t elem_type, int64_t n_nodes, const double* xyz, int64_t n_elems,
                            const int32_t* elems, const int32_t* material, const int32_t* l2g,
                            int64_t n_dofs, int32_t on_device, void* stream, emg_system* out);
/* Numeric assembly: nu (1/mu) and sigma per material; sources; EMG_FLAG_*. */
int emg_system_assemble(emg_system sys, const double* nu_per_material,
                        const double* sigma_per_material, int32_t n_materials,
                        const emg_source* sources, int32_t n_sources, int32_t flags, void* stream);
/* Per-tet source selection (host array of n_tets; NULL clears): with a map
 * set, tet t evaluates only sources[tet_source[t]] (none when < 0) and the
 * source table passed to emg_system_assemble may have any length.  Used to
 * give every instance of a batched (block-diagonal) system its own source. */
int emg_system_set_source_map(emg_system sys, const int32_t* tet_source);
int emg_system_info(emg_system sys, int64_t* n_rows, int64_t* nnz);
/* Copies to host; any pointer may be NULL.  row_ptr n+1, col/kval/mval nnz, rhs n. */
int emg_system_export(emg_system sys, int32_t* row_ptr, int32_t* col, double* kval,
                      double* mval, double* rhs);
/* Transient / eddy-current operator alpha*K + beta*M (e.g. K + M/dt for the
 * sigma dA/dt term, magnetic_vector_3d_integrator.cpp:233-339) as a new,
 * caller-owned device matrix on K's pattern (destroy with emg_csr_destroy).
 * Needs a system assembled with EMG_FLAG_MASS. */
int emg_system_combine(emg_system sys, double alpha, double beta, emg_csr* out);
/* Borrowed handles / pointers, valid while the system lives. which: 0 K, 1 M. */
emg_csr emg_system_matrix(emg_system sys, int32_t which);
const double* emg_system_rhs_device(emg_system sys);
void emg_system_destroy(emg_system sys);

/* ---- CsrMatrix<double> + CGSolver::set_matrix (include/numeric/csr_matrix.hpp:31-259,
 * src/numeric/iterative_solvers.cpp:83-97).  Host CSR, duplicates allowed and
 * summed, columns in any order (CsrMatrix::build_from_coo keeps duplicates,
 * SparseConverter::to_eigen sums them).  The device variant expects a merged
 * CSR with sorted rows. */
int emg_csr_create(int64_t n, const int32_t* row_ptr, const int32_t* col, const double* val,
                   void* stream, emg_csr* out);
int emg_csr_create_device(int64_t n, int64_t nnz, const int32_t* row_ptr_d,
                          const int32_t* col_d, const double* val_d, void* stream,
                          emg_csr* out);
int emg_csr_info(emg_csr A, int64_t* n, int64_t* nnz);
void emg_csr_destroy(emg_csr A);

/* ---- CsrMatrix::mat_vec (include/numeric/csr_matrix_impl.hpp:131-147): y_d = A x_d */
int emg_spmv(emg_csr A, const double* x_d, double* y_d, void* stream);

/* ---- CGSolver::solve (src/numeric/iterative_solvers.cpp:294-503) and
 * BiCGSTABSolver::solve (:820-1118), same iteration, stopping and failure
 * rules.  Host b/x or device b_d/x_d; x starts at zero. */
int emg_cg_solve(emg_csr A, const double* b, double* x, const emg_krylov_config* cfg,
                 emg_result* out);
int emg_cg_solve_device(emg_csr A, const double* b_d, double* x_d,
                        const emg_krylov_config* cfg, void* stream, emg_result* out);
int emg_bicgstab_solve(emg_csr A, const double* b, double* x, const emg_krylov_config* cfg,
                       emg_result* out);
int emg_bicgstab_solve_device(emg_csr A, const double* b_d, double* x_d,
                              const emg_krylov_config* cfg, void* stream, emg_result* out);

/* Assemble-and-solve convenience for a system: K x = F with the system's own
 * source vector (CGSolver / BiCGSTABSolver after EMAssembly::assemble).
 * kind: 0 CG, 1 BiCGSTAB.  x is a host array, or a device array when
 * x_on_device != 0. */
int emg_system_solve(emg_system sys, int32_t kind, const emg_krylov_config* cfg, double* x,
                     int32_t x_on_device, void* stream, emg_result* out);

/* Profiling hook: device time of each CG kernel (SpMV + p.q, update, direction;
 * ms[0..2]) averaged over `iterations` plain launches from a fresh start with
 * b = ones, each launch bracketed by CUDA events on `stream`. */
int emg_cg_kernel_times(emg_csr A, int32_t iterations, void* stream, double* ms);

/* ---- Ansys Maxwell project input (MaxwellParserImpl / AedtProjectLoader,
 * src/tool/maxwell_parser_impl.cpp, src/tool/aedt_project_loader.cpp:60-130)
 * The materials, geometry parts (objects) and boundaries of an .aedt text
 * project.  The mesh is not stored in .aedt files: a mesh read with
 * emg_mesh_read_gmsh whose physical volumes carry the objects' names takes
 * nu / sigma from here (Python: emagddm_b200.aedt). */
typedef struct emg_aedt_t* emg_aedt;
int emg_aedt_read(const char* path, emg_aedt* out);
int emg_aedt_info(emg_aedt a, int32_t* n_materials, int32_t* n_objects, int32_t* n_boundaries);
/* Material k: name (NUL-terminated, at most cap bytes), relative permeability
 * (a nonlinear material: its initial permeability, the first BH point with
 * H > 0 as B / (mu0 H)), conductivity [S/m], flags (1 nonlinear, 2
 * permeability not a number, 4 conductivity not a number) and the number of
 * BH-curve points. */
int emg_aedt_material(emg_aedt a, int32_t k, char* name, int32_t cap, double* mu_r, double* sigma,
                      int32_t* flags, int32_t* n_bh);
/* BH curve of material k: H [A/m] and B [T], at most cap points. */
int emg_aedt_bh_curve(emg_aedt a, int32_t k, double* h, double* b, int32_t cap);
/* Object k: name, material name, solve-inside flag. */
int emg_aedt_object(emg_aedt a, int32_t k, char* name, int32_t cap, char* material, int32_t mcap,
                    int32_t* solve_inside);
/* Boundary k: name, type ('Vector Potential', 'Coil', ...), value. */
int emg_aedt_boundary(emg_aedt a, int32_t k, char* name, int32_t cap, char* type, int32_t tcap, char* value,
                      int32_t vcap);
void emg_aedt_destroy(emg_aedt a);

/* ---- Launch-configuration autotuner (no counterpart in the reference) ----
 * The library times candidate launch configurations of some kernels on the
 * device the first time it meets a problem shape and keeps the fastest:
 * the grid of the SELL SpMV of each matrix, and the CTA widths of the
 * FETI-DP / direct solve kernels after a solver's first factorization.
 * Tuning is on by default (EMG_TUNE=0 in the environment turns it off:
 * built-in defaults); EMG_TUNE_CACHE=<file> keeps the decisions between
 * processes.  emg_tune_enable switches it for the rest of the process. */
int emg_tune_enable(int32_t on);
/* The decisions so far as JSON ({"family|shape": {"value": v,
 * "candidates_ms": {...}}}) into buf (cap bytes, NUL-terminated); returns the
 * length needed including the NUL. */
int32_t emg_tune_report(char* buf, int32_t cap);

/* Test hook (no counterpart in the reference): polls a block of the fused
 * CG update makes at its grid barrier before giving up (default 2^21, about
 * 0.2 s or more; a negative value restores it) on the current device.  A
 * block that gives up ends the solve with EMG_ERR_TIMEOUT instead of
 * waiting on; tests lower the limit to make that wait run out. */
int emg_test_set_barrier_spins(int32_t spins);

/* Test hook (no counterpart in the reference): one tile of the
 * mixed-precision factor's tensor-core contraction, C -= A B^T with A
 * (mr x k, leading dimension lda), B (mc x k, ldb), C (mr x mc, ldc), all
 * column-major FP64 device arrays, 1 <= mr, mc <= 128; the tile splits each
 * value into two TF32 terms and accumulates in FP32 (EMG_FLAG_FACTOR_TF32). */
int emg_test_tc_tile(int32_t mr, int32_t mc, int32_t k, const double* a_d, int64_t lda, const double* b_d,
                     int64_t ldb, double* c_d, int64_t ldc, void* stream);

/* Solver storage of A (SELL-32-sigma copy built at the first solve or SpMV):
 * stored slots including padding and number of 32-row slices; -1 before the
 * first solve. */
int emg_csr_solver_format(emg_csr A, int64_t* slots, int64_t* slices);

/* ---- Batched solves: many independent systems in one device loop ---------
 * A is block diagonal: rows [block_row_ptr[k], block_row_ptr[k+1]) form
 * system k and couple to no other block (checked; the union of disjoint
 * meshes assembled as one system has exactly this form).  Every block runs
 * CGSolver's Jacobi/plain CG (iterative_solvers.cpp:424-503) with its own
 * scalars, statuses and iteration counts, in lockstep, as one CUDA graph.
 * block_row_ptr is a host array of n_blocks+1; b_d/x_d are device vectors of
 * A's size; results[k] (host, n_blocks) receives each block's outcome, with
 * solve_time_ms = device time of the whole batch.  Returns EMG_SUCCESS when
 * every block converged, else the first non-success block status. */
int emg_batch_cg_solve_device(emg_csr A, int32_t n_blocks, const int64_t* block_row_ptr,
                              const double* b_d, double* x_d, const emg_krylov_config* cfg,
                              void* stream, emg_result* results);

/* ---- Allocation-free CG (no counterpart in the reference) --------------
 * For callers that must not let a library allocate GPU memory: applications
 * that budget all device memory themselves, and loops that may not call the
 * CUDA allocator after start-up (cudaMalloc/cudaFree synchronize the device
 * and take unbounded time).  Same iteration, stopping and failure rules as
 * emg_cg_solve_device, on a caller-owned merged CSR in device memory
 * (row_ptr_d n+1, col_d/val_d nnz, columns strictly ascending within each
 * row; b_d, x_d n; an unmerged CSR returns EMG_INVALID_INPUT).  Allocates
 * nothing: the work
 * vectors live in a fixed scratch array inside the library (about 10 MiB,
 * held by every GPU that loads the library until exit), so n is limited to
 * 262,144 rows; larger n returns EMG_INVALID_INPUT.  The first call on a
 * device looks up the scratch address and should come before any stream
 * capture.  Every call blocks the host until the solve ends: it synchronizes
 * the stream and reads the solver state back every 16 iterations.  Calls
 * share the scratch: calls that overlap on the GPU (other streams or
 * threads) race.  solve_time_ms is host wall time. */
int emg_cg_solve_noalloc(int64_t n, int64_t nnz, const int32_t* row_ptr_d, const int32_t* col_d,
                         const double* val_d, const double* b_d, double* x_d,
                         const emg_krylov_config* cfg, void* stream, emg_result* out);

/* Residual monitor of the last solve on A (ConvergenceHistory,
 * iterative_solvers.cpp:24-60): relative residual after every iteration, up
 * to cap entries; returns the number written. */
int emg_last_history(emg_csr A, double* residuals, int32_t cap);

#ifdef __cplusplus
}
#endif
#endif /* EMAGDDM_B200_H */

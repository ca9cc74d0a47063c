/*
 * emg_oracle.h -- CPU oracle for the TET4 / HEX8 Nedelec curl-curl solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithm (Poofee/emagddm): the tests compare the CUDA product path with it,
 * and bench.py times it as the CPU baseline.  Nothing in the product library links,
 * loads or calls it.
 *
 * Parity anchors:
 *   - integer outputs (edge IDs, free-DOF map, tree gauge, CSR pattern) are
 *     pinned against the reference's own C++ sources compiled under
 *     oracle/_ref (ref_bridge.cpp) and against the count fixtures in
 *     tests/golden;
 *   - element matrices follow the reference's intended formulas (the
 *     reference integrator returns zero matrices for TET4_EDGE, see
 *     emg_oracle.c header), pinned against the reference-domain curls of
 *     test/test_shape_function.cpp:290-330 and against closed forms;
 *   - solvers restate CGSolver / BiCGSTABSolver and are cross-checked against
 *     the reference solvers compiled under oracle/_ref.
 */
#ifndef EMG_ORACLE_H
#define EMG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes: same values as numeric::SolverStatus
 * (include/numeric/em_linear_solver.h:26-32). */
enum {
  ORC_SUCCESS = 0,
  ORC_NUMERICAL_ERROR = 1,
  ORC_DIVERGED = 2,
  ORC_MAX_ITER_REACHED = 3,
  ORC_INVALID_INPUT = 4
};

/* Element types (same values as the C ABI's EMG_ELEM_*). */
enum { ORC_ELEM_TET4_EDGE = 0, ORC_ELEM_HEX8_EDGE = 1, ORC_ELEM_PRISM6_EDGE = 2, ORC_ELEM_PYRAMID5_EDGE = 3,
       /* mixed mesh: 9 ints per element (8 node slots, -1 past the element's
        * nodes, then its type), 12 edge slots per element (-1 past its edges) */
       ORC_ELEM_MIXED = 4 };

/* Gauge modes. */
enum { ORC_GAUGE_NONE = -1, ORC_GAUGE_REF = 0, ORC_GAUGE_BOUNDARY_FIRST = 1 };

/* Assembly flags. */
enum {
  ORC_FLAG_MASS = 1,           /* also assemble M (sigma W_i . W_j)           */
  ORC_FLAG_NO_EDGE_SIGNS = 2,  /* scatter unsigned, as the reference does     */
  ORC_FLAG_PIOLA_LITERAL = 4,  /* W_phys = J^-T W_ref / detJ (reference text) */
  ORC_FLAG_QUAD3_LITERAL = 8   /* 3-point rule left by the pop_back quirk      */
};

/* Source region kinds (current density J evaluated at quadrature points). */
enum { ORC_SRC_BOX = 1, ORC_SRC_ANNULUS_Z = 2 };

typedef struct {
  int32_t kind;
  double j[3];   /* current density vector inside the region            */
  double p[6];   /* BOX: xmin,xmax,ymin,ymax,zmin,zmax (open intervals)  */
                 /* ANNULUS_Z: cx,cy,rmin,rmax,zmin,zmax (open)          */
} orc_source;

/* GlobalEdgeIDGenerator::generate (src/fe_em/global_edge_id_generator.cpp:30-110).
 * elem_edge: T*6 global edge IDs by first appearance; edge_nodes (optional,
 * 2*E): sorted node pair of each edge.  Returns 0 on success. */
int orc_edge_ids(int64_t n_tets, const int32_t* tets, int32_t* elem_edge,
                 int32_t* edge_nodes, int64_t* n_edges);

/* EMDOFManager::build (+ applyTreeGauge when gauge >= 0).
 * l2g: T*6 output (-1 = constrained / tree edge); edge_dof: E output. */
int orc_dof_build(int64_t n_tets, const int32_t* tets, const int32_t* elem_edge,
                  const int32_t* edge_nodes, int64_t n_edges, int64_t n_dir,
                  const int32_t* dir_pairs, int32_t n_hole_markers, int32_t gauge,
                  int32_t* l2g, int32_t* edge_dof, int64_t* n_free,
                  int64_t* n_dofs, int32_t* root_node);

/* Element matrices of one TET4_EDGE element (reference-local basis order,
 * unsigned).  xyz: 4 nodes x 3.  Ke, Me: 36 (row-major), Fe: 6. */
void orc_element(const double* xyz, double nu, double sigma,
                 const orc_source* src, int32_t n_src, int32_t flags,
                 double* Ke, double* Me, double* Fe);

/* Edge signs s_k of one element (+1 when the reference basis orientation
 * agrees with the global low->high node-ID orientation). */
void orc_edge_signs(const int32_t* tet, int32_t* s);

/* Pattern of the merged CSR (what SparseConverter::to_eigen produces):
 * row_ptr (n+1) always written; col written when not NULL.  nnz returned. */
int orc_pattern(int64_t n_tets, const int32_t* l2g, int64_t n_dofs,
                int64_t* row_ptr, int32_t* col, int64_t* nnz);

/* Numeric assembly into a pattern from orc_pattern. */
int orc_assemble(int64_t n_nodes, const double* xyz, int64_t n_tets,
                 const int32_t* tets, const int32_t* material, const int32_t* l2g,
                 const double* nu_mat, const double* sigma_mat, int32_t n_mat,
                 const orc_source* src, int32_t n_src, int32_t flags,
                 int64_t n_dofs, const int64_t* row_ptr, const int32_t* col,
                 double* kval, double* mval, double* rhs);

/* y = A x */
void orc_spmv(int64_t n, const int64_t* row_ptr, const int32_t* col,
              const double* val, const double* x, double* y);

/* CGSolver::solve_no_preconditioner / solve_with_jacobi / solve_with_ilu0
 * (src/numeric/iterative_solvers.cpp:343-585).  precond: 0 none, 1 jacobi,
 * 2 ILU0 (restated as ILU(0) on the matrix's pattern; the reference's is
 * Eigen's IncompleteLUT). */
int orc_pcg(int64_t n, const int64_t* row_ptr, const int32_t* col,
            const double* val, const double* b, double* x, double tol,
            int32_t max_iter, int32_t precond, int32_t* iterations,
            double* residual_norm);

/* orc_pcg that also copies the first iterate whose relative residual is
 * below snap_tol into x_snap (its iteration into *snap_iter, -1 if none). */
int orc_pcg_snap(int64_t n, const int64_t* row_ptr, const int32_t* col,
                 const double* val, const double* b, double* x, double tol,
                 int32_t max_iter, int32_t precond, int32_t* iterations,
                 double* residual_norm, double snap_tol, double* x_snap,
                 int32_t* snap_iter);

/* BiCGSTABSolver::solve_no_preconditioner / solve_with_jacobi
 * (src/numeric/iterative_solvers.cpp:869-1118). */
int orc_bicgstab(int64_t n, const int64_t* row_ptr, const int32_t* col,
                 const double* val, const double* b, double* x, double tol,
                 int32_t max_iter, int32_t precond, int32_t* iterations,
                 double* residual_norm);

/* ---- element-typed variants: elems holds 4 (TET4_EDGE), 8 (HEX8_EDGE),
 * 6 (PRISM6_EDGE) or 5 (PYRAMID5_EDGE) nodes per element, elem_edge / l2g
 * 6, 12, 9 or 8 entries per element; the
 * untyped functions above are elem_type = ORC_ELEM_TET4_EDGE. */
int orc_edge_ids_typed(int32_t elem_type, int64_t n_elems, const int32_t* elems, int32_t* elem_edge,
                       int32_t* edge_nodes, int64_t* n_edges);
int orc_dof_build_typed(int32_t elem_type, int64_t n_elems, const int32_t* elems, const int32_t* elem_edge,
                        const int32_t* edge_nodes, int64_t n_edges, int64_t n_dir,
                        const int32_t* dir_pairs, int32_t n_hole_markers, int32_t gauge,
                        int32_t* l2g, int32_t* edge_dof, int64_t* n_free,
                        int64_t* n_dofs, int32_t* root_node);
int orc_pattern_typed(int32_t elem_type, int64_t n_elems, const int32_t* l2g, int64_t n_dofs,
                      int64_t* row_ptr, int32_t* col, int64_t* nnz);

/* EMDOFManager::build (+ applyTreeGauge when gauge >= 0) with per-element
 * Element::dof_type (ORC_DOF_SCALAR_ONLY / VECTOR_EDGE_ONLY / MIXED_AV,
 * include/fe_em/em_mesh_data.hpp:45-49):
 *   assignPrenumbering  (src/fe_em/em_dof_manager.cpp:91-150): nodes of the
 *     scalar-carrying elements in ascending node ID, then the edges of the
 *     vector-carrying elements by first appearance (GlobalEdgeIDGenerator
 *     skips scalar-only elements, global_edge_id_generator.cpp:44-53);
 *   markConstrainedDOFs (:152-243): scalar_dirichlet node IDs, dir_pairs edges;
 *   renumberFreeDOFs    (:245-286): free index = rank among the unconstrained
 *     prenumbers (scalars first);
 *   buildMappingTables  (:288-446): node DOFs, edge DOFs, or node then edge
 *     DOFs per element;
 *   renumberVectorDOFsWithTreeGauge (:501-626): the tree gauge of the
 *     vector-carrying elements, edge DOF = n_scalar_free + reduced index.
 * l2g: (npe + epe) * n_elems, each row Local2Global::indices padded with -2. */
#define ORC_DOF_SCALAR_ONLY 0
#define ORC_DOF_VECTOR_EDGE_ONLY 1
#define ORC_DOF_MIXED_AV 2
int orc_dof_build_av(int32_t elem_type, int64_t n_nodes, int64_t n_elems, const int32_t* elems,
                     const int32_t* dof_type, int64_t n_dir, const int32_t* dir_pairs, int64_t n_sdir,
                     const int32_t* sdir_nodes, int32_t n_hole_markers, int32_t gauge, int32_t* l2g,
                     int64_t* n_scalar_free, int64_t* n_free, int64_t* n_dofs);
int orc_assemble_typed(int32_t elem_type, int64_t n_nodes, const double* xyz, int64_t n_elems,
                       const int32_t* elems, const int32_t* material, const int32_t* l2g,
                       const double* nu_mat, const double* sigma_mat, int32_t n_mat,
                       const orc_source* src, int32_t n_src, int32_t flags,
                       int64_t n_dofs, const int64_t* row_ptr, const int32_t* col,
                       double* kval, double* mval, double* rhs);

/* HEX8_EDGE: reference-domain basis value and curl of edge k at x (3),
 * Jacobian (row-major dx_r/dxi_c) and determinant of the trilinear map of
 * the 8 nodes X (8 x 3), element matrices (144 row-major, Fe 12) and the
 * edge signs of one element. */
void orc_hex_basis(int k, const double* x, double* w);
void orc_hex_curl(int k, const double* x, double* c);
void orc_hex_jacobian(const double* X, const double* x, double* J, double* det);
void orc_element_hex(const double* xyz, double nu, double sigma,
                     const orc_source* src, int32_t n_src, int32_t flags,
                     double* Ke, double* Me, double* Fe);
void orc_edge_signs_hex(const int32_t* hex, int32_t* s);
/* PRISM6_EDGE / PYRAMID5_EDGE reference-element checks: circulation of basis
 * k along edge e (n midpoint segments), and max |grad N_a - sum_k (N_a(b_k) -
 * N_a(a_k)) W_k| over the nodes a at reference point x. */
double orc_shape_circulation(int32_t elem_type, int k, int e, int n);
double orc_shape_grad_residual(int32_t elem_type, const double* x);

/* Thread count used by the parallel loops (OpenMP when compiled with it). */
int orc_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif

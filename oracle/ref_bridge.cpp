// ref_bridge.cpp -- TEST INFRASTRUCTURE: a thin extern "C" wrapper that links
// the reference's own C++ sources (compiled in place by Makefile.ref, outputs
// only into oracle/_ref/) so tests can compare this library's integer outputs
// and solver behaviour with the reference itself, and so bench.py can time the
// reference's CPU solver.  It calls only the reference's public API:
//   GlobalEdgeIDGenerator::generate      (src/fe_em/global_edge_id_generator.cpp:30)
//   EMDOFManager::build / applyTreeGauge (src/fe_em/em_dof_manager.cpp:29, :448)
//   EMAssembly::assemble                 (src/numeric/em_assembly.cpp:144)
//   SparseConverter::to_eigen            (src/numeric/sparse_converter.cpp:19)
//   CGSolver / BiCGSTABSolver            (src/numeric/iterative_solvers.cpp)
//   NedelecElement<3> (TET4_EDGE, HEX8_EDGE), GaussQuadrature, MagneticVector3DIntegrator.
#include <Eigen/Sparse>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <vector>

#include "em_assembly.hpp"
#include "em_dof_manager.hpp"
#include "em_mesh_data.hpp"
#include "gauss_quadrature.hpp"
#include "global_edge_id_generator.hpp"
#include "iterative_solvers.h"
#include "logger.hpp"
#include "logger_factory.hpp"
#include "magnetic_vector_3d_integrator.hpp"
#include "nedelec_element.hpp"
#include "shape_function_factory.hpp"
#include "sparse_converter.h"

namespace {

// Element types of the C ABI (EMG_ELEM_*) as the reference's ElementType.
// Type 4 is a mixed mesh: rows of 9 ints (8 node slots, -1 past the
// element's nodes, then its type) and 12 edge slots per element.
static int bridge_npe(int32_t t) { return t == 1 ? 8 : t == 2 ? 6 : t == 3 ? 5 : t == 4 ? 9 : 4; }
static int bridge_epe(int32_t t) { return t == 1 ? 12 : t == 2 ? 9 : t == 3 ? 8 : t == 4 ? 12 : 6; }
static int32_t row_type(int32_t elem_type, const int32_t* row) { return elem_type == 4 ? row[8] : elem_type; }
static numeric::ElementType bridge_type(int32_t t) {
  return t == 1   ? numeric::ElementType::HEX8_EDGE
         : t == 2 ? numeric::ElementType::PRISM6_EDGE
         : t == 3 ? numeric::ElementType::PYRAMID5_EDGE
                  : numeric::ElementType::TET4_EDGE;
}

fe_em::EMMeshData make_mesh(int64_t n_nodes, const double* xyz, int64_t n_tets, const int32_t* tets,
                            int64_t n_dir, const int32_t* dir_pairs, int32_t n_hole_markers,
                            int32_t elem_type = 0) {
  const int npe = bridge_npe(elem_type);
  fe_em::EMMeshData m;
  m.nodes.resize(n_nodes);
  for (int64_t i = 0; i < n_nodes; ++i) {
    m.nodes[i] = fe_em::Node{static_cast<int>(i), xyz ? xyz[3 * i] : 0.0, xyz ? xyz[3 * i + 1] : 0.0,
                             xyz ? xyz[3 * i + 2] : 0.0, 0};
  }
  m.elements.resize(n_tets);
  for (int64_t t = 0; t < n_tets; ++t) {
    auto& e = m.elements[t];
    e.id = static_cast<int>(t);
    const int32_t et = row_type(elem_type, tets + npe * t);
    e.node_ids.assign(tets + npe * t, tets + npe * t + bridge_npe(et));
    e.elem_type = bridge_type(et);
    e.dof_type = fe_em::DOFType::VECTOR_EDGE_ONLY;
    e.material_id = 0;
    e.region_id = 0;
  }
  fe_em::EMBoundaryMarker bm;
  bm.id = 0;
  bm.bnd_type = tool::BndType::DIRICHLET;
  bm.dof_type = fe_em::DOFType::VECTOR_EDGE_ONLY;
  std::vector<std::vector<int>> pairs(n_dir);
  for (int64_t d = 0; d < n_dir; ++d) pairs[d] = {dir_pairs[2 * d], dir_pairs[2 * d + 1]};
  bm.target_ids = pairs;
  bm.value = 0.0;
  bm.name = "outer_faces";
  m.boundary_markers.push_back(bm);
  // Extra markers whose names trigger the hole heuristic of
  // MultiConnectedDomainDetector::analyzeBoundaryMarkers
  // (src/fe_em/multi_connected_domain.cpp:126-188).
  for (int32_t h = 0; h < n_hole_markers; ++h) {
    fe_em::EMBoundaryMarker hm;
    hm.id = 1 + h;
    hm.bnd_type = tool::BndType::NEUMANN;
    hm.dof_type = fe_em::DOFType::VECTOR_EDGE_ONLY;
    hm.target_ids = std::vector<std::vector<int>>{};
    hm.value = 0.0;
    hm.name = "hole_" + std::to_string(h);
    m.boundary_markers.push_back(hm);
  }
  return m;
}

numeric::CsrMatrix<double> make_csr(int64_t n, const int64_t* rp, const int32_t* col, const double* val) {
  numeric::CooMatrix<double> coo(static_cast<int>(n), static_cast<int>(n), static_cast<int>(rp[n]));
  for (int64_t i = 0; i < n; ++i)
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k) coo.add_value(static_cast<int>(i), col[k], val[k]);
  numeric::CsrMatrix<double> A(static_cast<int>(n), static_cast<int>(n));
  A.build_from_coo(coo);
  return A;
}

int status_code(numeric::SolverStatus s) { return static_cast<int>(s); }

}  // namespace

extern "C" {

void refb_quiet(int quiet) {
  FEEM_SET_LEVEL(quiet ? tool::LogLevel::CRITICAL : tool::LogLevel::INFO);
}

// Edge IDs + DOF map (+ tree gauge when apply_gauge != 0); elem_type 0 =
// TET4_EDGE (4 nodes, 6 edges per element), 1 = HEX8_EDGE (8 nodes, 12 edges).
int refb_dof_build_typed(int32_t elem_type, int64_t n_nodes, int64_t n_tets, const int32_t* tets, int64_t n_dir,
                         const int32_t* dir_pairs, int32_t n_hole_markers, int32_t apply_gauge,
                         int32_t* elem_edge_out, int32_t* l2g_out, int64_t* n_edges, int64_t* n_free,
                         int64_t* n_dofs);

int refb_dof_build(int64_t n_nodes, int64_t n_tets, const int32_t* tets, int64_t n_dir,
                   const int32_t* dir_pairs, int32_t n_hole_markers, int32_t apply_gauge,
                   int32_t* elem_edge_out, int32_t* l2g_out, int64_t* n_edges, int64_t* n_free,
                   int64_t* n_dofs) {
  return refb_dof_build_typed(0, n_nodes, n_tets, tets, n_dir, dir_pairs, n_hole_markers, apply_gauge,
                              elem_edge_out, l2g_out, n_edges, n_free, n_dofs);
}

int refb_dof_build_typed(int32_t elem_type, int64_t n_nodes, int64_t n_tets, const int32_t* tets, int64_t n_dir,
                         const int32_t* dir_pairs, int32_t n_hole_markers, int32_t apply_gauge,
                         int32_t* elem_edge_out, int32_t* l2g_out, int64_t* n_edges, int64_t* n_free,
                         int64_t* n_dofs) {
  const int epe = bridge_epe(elem_type);
  try {
    auto mesh = make_mesh(n_nodes, nullptr, n_tets, tets, n_dir, dir_pairs, n_hole_markers, elem_type);
    fe_em::GlobalEdgeIDGenerator gen(mesh);
    gen.generate();
    const auto& l2e = gen.getElemLocalToGlobalEdge();
    for (int64_t t = 0; t < n_tets; ++t) {
      const int ne = bridge_epe(row_type(elem_type, tets + bridge_npe(elem_type) * t));
      if (static_cast<int>(l2e[t].size()) != ne) return -3;
      for (int k = 0; k < epe; ++k) elem_edge_out[epe * t + k] = k < ne ? l2e[t][k] : -1;
    }
    *n_edges = gen.getNumGlobalEdges();
    fe_em::EMDOFManager dm(mesh, l2e, &gen);
    dm.build();
    *n_free = dm.getNumFreeDOFs();
    if (apply_gauge) dm.applyTreeGauge();
    *n_dofs = dm.getNumFreeDOFs();
    const auto& l2g = dm.getElemLocalToGlobal();
    for (int64_t t = 0; t < n_tets; ++t) {
      const int ne = bridge_epe(row_type(elem_type, tets + bridge_npe(elem_type) * t));
      if (static_cast<int>(l2g[t].indices.size()) != ne) return -3;
      for (int k = 0; k < epe; ++k) l2g_out[epe * t + k] = k < ne ? l2g[t].indices[k] : -1;
    }
    return 0;
  } catch (const std::exception&) {
    return -1;
  }
}

// EMDOFManager::build (+ applyTreeGauge) on elements with per-element
// Element::dof_type (0 SCALAR_ONLY, 1 VECTOR_EDGE_ONLY, 2 MIXED_AV) and a
// DIRICHLET marker on scalar DOFs (node IDs) next to the one on edges.
// l2g_out rows hold npe + epe entries: Local2Global::indices, the rest -2.
int refb_dof_build_av(int32_t elem_type, int64_t n_nodes, int64_t n_elems, const int32_t* elems,
                      const int32_t* dof_type, int64_t n_dir, const int32_t* dir_pairs, int64_t n_sdir,
                      const int32_t* sdir_nodes, int32_t n_hole_markers, int32_t apply_gauge,
                      int32_t* l2g_out, int64_t* n_free, int64_t* n_dofs) {
  const int npe = bridge_npe(elem_type), epe = bridge_epe(elem_type);
  try {
    auto mesh = make_mesh(n_nodes, nullptr, n_elems, elems, n_dir, dir_pairs, n_hole_markers, elem_type);
    for (int64_t t = 0; t < n_elems; ++t)
      mesh.elements[t].dof_type = dof_type[t] == 0   ? fe_em::DOFType::SCALAR_ONLY
                                  : dof_type[t] == 1 ? fe_em::DOFType::VECTOR_EDGE_ONLY
                                                     : fe_em::DOFType::MIXED_AV;
    fe_em::EMBoundaryMarker sm;
    sm.id = 100;
    sm.bnd_type = tool::BndType::DIRICHLET;
    sm.dof_type = fe_em::DOFType::SCALAR_ONLY;
    sm.target_ids = std::vector<int>(sdir_nodes, sdir_nodes + n_sdir);
    sm.value = 0.0;
    sm.name = "outer_potential";
    mesh.boundary_markers.push_back(sm);
    fe_em::GlobalEdgeIDGenerator gen(mesh);
    gen.generate();
    fe_em::EMDOFManager dm(mesh, gen.getElemLocalToGlobalEdge(), &gen);
    dm.build();
    *n_free = dm.getNumFreeDOFs();
    if (apply_gauge) dm.applyTreeGauge();
    *n_dofs = dm.getNumFreeDOFs();
    const auto& l2g = dm.getElemLocalToGlobal();
    for (int64_t t = 0; t < n_elems; ++t) {
      const auto& ix = l2g[t].indices;
      if (static_cast<int>(ix.size()) > npe + epe) return -3;
      for (int k = 0; k < npe + epe; ++k) l2g_out[(npe + epe) * t + k] = k < static_cast<int>(ix.size()) ? ix[k] : -2;
    }
    return 0;
  } catch (const std::exception&) {
    return -1;
  }
}

// Merged CSR pattern via EMAssembly (placeholder integrator) + to_eigen.
// col_out may be NULL (count only).  raw_nnz = entries before merging.
int refb_pattern_typed(int32_t elem_type, int64_t n_nodes, const double* xyz, int64_t n_tets,
                       const int32_t* tets, const int32_t* l2g, int64_t* row_ptr_out, int32_t* col_out,
                       int64_t* nnz, int64_t* raw_nnz, int64_t* n_rows);

int refb_pattern(int64_t n_nodes, const double* xyz, int64_t n_tets, const int32_t* tets,
                 const int32_t* l2g, int64_t* row_ptr_out, int32_t* col_out, int64_t* nnz,
                 int64_t* raw_nnz, int64_t* n_rows) {
  return refb_pattern_typed(0, n_nodes, xyz, n_tets, tets, l2g, row_ptr_out, col_out, nnz, raw_nnz, n_rows);
}

int refb_pattern_typed(int32_t elem_type, int64_t n_nodes, const double* xyz, int64_t n_tets,
                       const int32_t* tets, const int32_t* l2g, int64_t* row_ptr_out, int32_t* col_out,
                       int64_t* nnz, int64_t* raw_nnz, int64_t* n_rows) {
  const int epe = bridge_epe(elem_type);
  try {
    auto mesh = make_mesh(n_nodes, xyz, n_tets, tets, 0, nullptr, 0, elem_type);
    std::vector<fe_em::Local2Global> maps(n_tets);
    for (int64_t t = 0; t < n_tets; ++t) {
      maps[t] = fe_em::Local2Global(epe);
      for (int k = 0; k < epe; ++k) maps[t].indices[k] = l2g[epe * t + k];
      maps[t].element_id = static_cast<int>(t);
      maps[t].num_vector_dofs = epe;
      maps[t].elem_type = bridge_type(elem_type);
    }
    std::vector<numeric::MaterialProperties> mats(1);
    numeric::EMAssembly as;
    if (!as.assemble(mesh, maps, mats, false)) return -2;
    const auto& K = as.getStiffnessMatrix();
    *raw_nnz = K.nnz();
    *n_rows = K.rows();
    Eigen::SparseMatrix<double> E = numeric::SparseConverter::to_eigen(K);
    Eigen::SparseMatrix<double, Eigen::RowMajor> R = E;
    R.makeCompressed();
    *nnz = R.nonZeros();
    if (row_ptr_out)
      for (int64_t i = 0; i <= R.rows(); ++i) row_ptr_out[i] = R.outerIndexPtr()[i];
    if (col_out)
      for (int64_t k = 0; k < R.nonZeros(); ++k) col_out[k] = R.innerIndexPtr()[k];
    return 0;
  } catch (const std::exception&) {
    return -1;
  }
}

// CGSolver / BiCGSTABSolver on a host CSR.  kind: 0 = CG, 1 = BiCGSTAB.
// precond: 0 none, 1 jacobi, 2 ILU0 (Eigen IncompleteLUT inside the
// reference).  Returns SolverStatus; times set_matrix and solve.
int refb_krylov(int32_t kind, int64_t n, const int64_t* rp, const int32_t* col, const double* val,
                const double* b, double* x, double tol, int32_t max_iter, int32_t precond,
                int32_t* iterations, double* residual, double* setup_ms, double* solve_ms) {
  try {
    auto A = make_csr(n, rp, col, val);
    Eigen::VectorXd bb = Eigen::Map<const Eigen::VectorXd>(b, n);
    numeric::SolverResult res;
    auto t0 = std::chrono::steady_clock::now();
    if (kind == 0) {
      numeric::CGConfig cfg;
      cfg.tolerance = tol;
      cfg.max_iterations = max_iter;
      cfg.preconditioner = precond == 2   ? numeric::CGConfig::PreconditionerType::ILU0
                           : precond == 1 ? numeric::CGConfig::PreconditionerType::JACOBI
                                          : numeric::CGConfig::PreconditionerType::NONE;
      numeric::CGSolver s(cfg);
      s.set_matrix(A);
      auto t1 = std::chrono::steady_clock::now();
      res = s.solve(bb);
      auto t2 = std::chrono::steady_clock::now();
      *setup_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
      *solve_ms = std::chrono::duration<double, std::milli>(t2 - t1).count();
    } else {
      numeric::BiCGSTABConfig cfg;
      cfg.tolerance = tol;
      cfg.max_iterations = max_iter;
      cfg.preconditioner = precond == 2   ? numeric::BiCGSTABConfig::PreconditionerType::ILU0
                           : precond == 1 ? numeric::BiCGSTABConfig::PreconditionerType::JACOBI
                                          : numeric::BiCGSTABConfig::PreconditionerType::NONE;
      numeric::BiCGSTABSolver s(cfg);
      s.set_matrix(A);
      auto t1 = std::chrono::steady_clock::now();
      res = s.solve(bb);
      auto t2 = std::chrono::steady_clock::now();
      *setup_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
      *solve_ms = std::chrono::duration<double, std::milli>(t2 - t1).count();
    }
    *iterations = res.iterations;
    *residual = res.residual_norm;
    if (res.x.size() == n) std::memcpy(x, res.x.data(), sizeof(double) * n);
    return status_code(res.status);
  } catch (const std::exception&) {
    return -1;
  }
}

// Reference-domain Nedelec values and curls at one point: w_out[6*3], c_out[6*3].
void refb_nedelec_tet4(double xi, double eta, double zeta, double* w_out, double* c_out) {
  numeric::NedelecElement<3> ned(numeric::ElementType::TET4_EDGE);
  numeric::LocalPoint p(xi, eta, zeta);
  for (int k = 0; k < 6; ++k) {
    Eigen::Vector3d w = ned.evalEdgeFunction(k, p);
    Eigen::Vector3d c = ned.evalCurlEdge(k, p);
    for (int r = 0; r < 3; ++r) { w_out[3 * k + r] = w[r]; c_out[3 * k + r] = c[r]; }
  }
}

// GaussQuadrature::getPoints(type, order): 0 = TET4, 1 = TET4_EDGE.
int refb_quadrature(int32_t edge_type, int32_t order, double* pts_out /*4*4*/) {
  auto pts = numeric::GaussQuadrature::getPoints(
      edge_type ? numeric::ElementType::TET4_EDGE : numeric::ElementType::TET4, order);
  int n = static_cast<int>(pts.size());
  for (int i = 0; i < n && i < 4; ++i) {
    pts_out[4 * i] = pts[i].coords[0];
    pts_out[4 * i + 1] = pts[i].coords[1];
    pts_out[4 * i + 2] = pts[i].coords[2];
    pts_out[4 * i + 3] = pts[i].weight;
  }
  return n;
}

// The reference's own MagneticVector3DIntegrator K for one TET4_EDGE element.
int refb_integrator_k(const double* xyz /*4 nodes x 3*/, double mu, double* K_out /*36*/) {
  try {
    numeric::MagneticVector3DIntegrator it(numeric::ElementType::TET4_EDGE);
    numeric::MaterialProperties mp;
    mp.mu = mu;
    it.setMaterialProperties(mp);
    Eigen::MatrixXd X(3, 4);
    for (int a = 0; a < 4; ++a)
      for (int r = 0; r < 3; ++r) X(r, a) = xyz[3 * a + r];
    Eigen::MatrixXd K = it.computeStiffnessMatrix(X);
    if (K.rows() != 6 || K.cols() != 6) return -2;
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 6; ++j) K_out[6 * i + j] = K(i, j);
    return 0;
  } catch (const std::exception&) {
    return -1;
  }
}

// HEX8_EDGE reference-domain values and curls at one point: w_out[12*3], c_out[12*3].
void refb_nedelec_hex8(double xi, double eta, double zeta, double* w_out, double* c_out) {
  numeric::NedelecElement<3> ned(numeric::ElementType::HEX8_EDGE);
  numeric::LocalPoint p(xi, eta, zeta);
  for (int k = 0; k < 12; ++k) {
    Eigen::Vector3d w = ned.evalEdgeFunction(k, p);
    Eigen::Vector3d c = ned.evalCurlEdge(k, p);
    for (int r = 0; r < 3; ++r) { w_out[3 * k + r] = w[r]; c_out[3 * k + r] = c[r]; }
  }
}

// Jacobian (row-major dx_r/dxi_c) and determinant of the HEX8 Lagrange map
// of the 8 nodes X (node a at X[3a..3a+2]) at one point, through
// ShapeFunctionFactory::create("HEX8")->calcJacobian -- the geometry map the
// integrator uses for positions (computePhysicalPosition).  (NedelecElement's
// own calcJacobian multiplies the 3 x 8 node matrix by its zero 12 x 3
// evalGradN, a dimension mismatch, and is not called here.)
int refb_hex8_jacobian(const double* X, double xi, double eta, double zeta, double* J_out, double* det_out) {
  try {
    auto sf = numeric::ShapeFunctionFactory::create("HEX8");
    if (!sf) return -2;
    numeric::LocalPoint p(xi, eta, zeta);
    Eigen::MatrixXd N(3, 8);
    for (int a = 0; a < 8; ++a)
      for (int r = 0; r < 3; ++r) N(r, a) = X[3 * a + r];
    numeric::JacobianResult jr = sf->calcJacobian(p, N);
    if (jr.jacobian.rows() != 3 || jr.jacobian.cols() != 3) return -3;
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) J_out[3 * r + c] = jr.jacobian(r, c);
    *det_out = jr.det_j;
    return 0;
  } catch (const std::exception&) {
    return -1;
  }
}

// GaussQuadrature::getPoints(type, order) for HEX8 (edge_type 0) or
// HEX8_EDGE (edge_type 1): up to 8 points (x, y, z, w) into pts_out.
int refb_quadrature_hex(int32_t edge_type, int32_t order, double* pts_out /*8*4*/) {
  auto pts = numeric::GaussQuadrature::getPoints(
      edge_type ? numeric::ElementType::HEX8_EDGE : numeric::ElementType::HEX8, order);
  int n = static_cast<int>(pts.size());
  for (int i = 0; i < n && i < 8; ++i) {
    pts_out[4 * i] = pts[i].coords[0];
    pts_out[4 * i + 1] = pts[i].coords[1];
    pts_out[4 * i + 2] = pts[i].coords[2];
    pts_out[4 * i + 3] = pts[i].weight;
  }
  return n;
}

// The reference's own MagneticVector3DIntegrator K for one HEX8_EDGE element.
int refb_integrator_k_hex(const double* xyz /*8 nodes x 3*/, double mu, double* K_out /*144*/) {
  try {
    numeric::MagneticVector3DIntegrator it(numeric::ElementType::HEX8_EDGE);
    numeric::MaterialProperties mp;
    mp.mu = mu;
    it.setMaterialProperties(mp);
    Eigen::MatrixXd X(3, 8);
    for (int a = 0; a < 8; ++a)
      for (int r = 0; r < 3; ++r) X(r, a) = xyz[3 * a + r];
    Eigen::MatrixXd K = it.computeStiffnessMatrix(X);
    if (K.rows() != 12 || K.cols() != 12) return -2;
    for (int i = 0; i < 12; ++i)
      for (int j = 0; j < 12; ++j) K_out[12 * i + j] = K(i, j);
    return 0;
  } catch (const std::exception&) {
    return -1;
  }
}

}  // extern "C"

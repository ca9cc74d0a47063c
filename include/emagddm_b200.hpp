// emagddm_b200.hpp -- header-only C++ adapters over the C ABI that mirror the
// reference's classes on the TET4_EDGE solve path, so a C++ caller of
//   fe_em::GlobalEdgeIDGenerator / fe_em::EMDOFManager   (src/fe_em/)
//   numeric::EMAssembly                                  (src/numeric/em_assembly.cpp)
//   numeric::CGSolver / numeric::BiCGSTABSolver          (src/numeric/iterative_solvers.cpp)
// switches by type.  Same method names and argument meaning; errors follow
// the reference: numbering misuse throws std::invalid_argument /
// std::runtime_error, assemble() returns false with a message, solve()
// never throws and reports through SolverResult::status.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "emagddm_b200.h"

namespace emg {

enum class SolverStatus : int {
  SUCCESS = EMG_SUCCESS,
  NUMERICAL_ERROR = EMG_NUMERICAL_ERROR,
  DIVERGED = EMG_DIVERGED,
  MAX_ITER_REACHED = EMG_MAX_ITER_REACHED,
  INVALID_INPUT = EMG_INVALID_INPUT
};

// numeric::SolverResult (include/numeric/em_linear_solver.h:53-61)
struct SolverResult {
  std::vector<double> x;
  SolverStatus status = SolverStatus::INVALID_INPUT;
  int iterations = 0;
  double residual_norm = 0.0;
  double solve_time_ms = 0.0;
  std::string error_msg;
};

inline std::string last_error() { return emg_last_error(); }

// fe_em::EMMeshData restricted to the edge path: nodes (id = index), elements
// of one type (TET4_EDGE: 4 nodes each, HEX8_EDGE: 8, PRISM6_EDGE: 6,
// PYRAMID5_EDGE: 5) with material ids,
// Dirichlet edge node pairs, hole-marker count.
class Mesh {
 public:
  Mesh(std::vector<double> xyz, std::vector<int32_t> elems, std::vector<int32_t> material,
       std::vector<int32_t> dirichlet_pairs, int32_t n_hole_markers = 0,
       int32_t elem_type = EMG_ELEM_TET4_EDGE)
      : xyz_(std::move(xyz)), elems_(std::move(elems)), material_(std::move(material)), type_(elem_type) {
    const int rc = emg_mesh_create_typed(type_, static_cast<int64_t>(xyz_.size() / 3), xyz_.data(),
                                         getElementCount(), elems_.data(),
                                         material_.empty() ? nullptr : material_.data(),
                                         static_cast<int64_t>(dirichlet_pairs.size() / 2),
                                         dirichlet_pairs.empty() ? nullptr : dirichlet_pairs.data(),
                                         n_hole_markers, &h_);
    if (rc != EMG_SUCCESS) throw std::invalid_argument("emg_mesh_create_typed: " + last_error());
  }
  ~Mesh() { emg_mesh_destroy(h_); }
  Mesh(const Mesh&) = delete;
  Mesh& operator=(const Mesh&) = delete;
  emg_mesh handle() const { return h_; }
  int32_t elementType() const { return type_; }
  int nodesPerElement() const {
    return type_ == EMG_ELEM_HEX8_EDGE ? 8 : type_ == EMG_ELEM_PRISM6_EDGE ? 6 : type_ == EMG_ELEM_PYRAMID5_EDGE ? 5 : 4;
  }
  int edgesPerElement() const {
    return type_ == EMG_ELEM_HEX8_EDGE ? 12 : type_ == EMG_ELEM_PRISM6_EDGE ? 9 : type_ == EMG_ELEM_PYRAMID5_EDGE ? 8 : 6;
  }
  int64_t getNodeCount() const { return static_cast<int64_t>(xyz_.size() / 3); }
  int64_t getElementCount() const { return static_cast<int64_t>(elems_.size() / nodesPerElement()); }
  const std::vector<double>& xyz() const { return xyz_; }
  const std::vector<int32_t>& elements() const { return elems_; }
  const std::vector<int32_t>& tets() const { return elems_; }  // TET4_EDGE meshes
  const std::vector<int32_t>& material() const { return material_; }

 private:
  std::vector<double> xyz_;
  std::vector<int32_t> elems_, material_;
  int32_t type_ = EMG_ELEM_TET4_EDGE;
  emg_mesh h_ = nullptr;
};

// fe_em::GlobalEdgeIDGenerator (src/fe_em/global_edge_id_generator.cpp:30-140)
class GlobalEdgeIDGenerator {
 public:
  explicit GlobalEdgeIDGenerator(const Mesh& mesh) : mesh_(mesh) {}
  void generate() {
    int64_t n = 0;
    if (emg_edge_ids(mesh_.handle(), nullptr, nullptr, &n) != EMG_SUCCESS)
      throw std::invalid_argument("GlobalEdgeIDGenerator::generate: " + last_error());
    elem_edge_.resize(mesh_.edgesPerElement() * mesh_.getElementCount());
    edge_nodes_.resize(2 * n);
    emg_edge_ids(mesh_.handle(), elem_edge_.data(), edge_nodes_.data(), &n);
  }
  int getNumGlobalEdges() const { return static_cast<int>(edge_nodes_.size() / 2); }
  // element-major, 6 (TET4), 12 (HEX8), 9 (PRISM6) or 8 (PYRAMID5) local edges per element in
  // ElementGeometry's order
  const std::vector<int32_t>& getElemLocalToGlobalEdge() const { return elem_edge_; }
  const std::vector<int32_t>& getEdgeNodes() const { return edge_nodes_; }

 private:
  const Mesh& mesh_;
  std::vector<int32_t> elem_edge_, edge_nodes_;
};

// fe_em::EMDOFManager (src/fe_em/em_dof_manager.cpp:29-626)
class EMDOFManager {
 public:
  explicit EMDOFManager(const Mesh& mesh) : mesh_(mesh) {}
  ~EMDOFManager() { emg_dofmap_destroy(map_); }
  EMDOFManager(const EMDOFManager&) = delete;
  EMDOFManager& operator=(const EMDOFManager&) = delete;
  void build() { run(EMG_GAUGE_NONE); gauged_ = false; }
  // Tree gauge for a partition of the elements (FETI-DP); replaces any gauge.
  void applyPartitionedGauge(const std::vector<int32_t>& tet_part, int32_t n_parts) {
    emg_dofmap m = nullptr;
    if (emg_dof_build_partitioned(mesh_.handle(), tet_part.data(), n_parts, &m) != EMG_SUCCESS)
      throw std::invalid_argument("EMDOFManager: " + last_error());
    adopt(m);
    gauged_ = true;
  }
  emg_dofmap handle() const { return map_; }
  void applyTreeGauge(int32_t mode = EMG_GAUGE_REF) {
    if (!map_) throw std::runtime_error("build() must be called before applyTreeGauge()");
    if (gauged_) return;  // repeated calls are ignored, as in the reference
    run(mode);
    gauged_ = true;
  }
  // Elements with Element::dof_type SCALAR_ONLY / VECTOR_EDGE_ONLY / MIXED_AV
  // (EMG_DOF_*), scalar Dirichlet node IDs: EMDOFManager::build (+
  // applyTreeGauge for mode >= 0).  Returns Local2Global::indices per
  // element (node DOFs, edge DOFs, or node then edge DOFs).
  std::vector<std::vector<int32_t>> buildWithDofTypes(const std::vector<int32_t>& dof_type,
                                                      const std::vector<int32_t>& scalar_dirichlet,
                                                      int32_t mode = EMG_GAUGE_REF) {
    int32_t et = 0, npe = 0, epe = 0;
    emg_mesh_elem_type(mesh_.handle(), &et, &npe, &epe);
    if (static_cast<int64_t>(dof_type.size()) != static_cast<int64_t>(mesh_.getElementCount()))
      throw std::invalid_argument("EMDOFManager: dof_type needs one entry per element");
    const size_t ne = dof_type.size(), w = static_cast<size_t>(npe + epe);
    std::vector<int32_t> rows(w * ne);
    int64_t ns = 0, nf = 0, nd = 0;
    if (emg_dof_build_av(mesh_.handle(), dof_type.data(), static_cast<int64_t>(scalar_dirichlet.size()),
                         scalar_dirichlet.data(), mode, rows.data(), &ns, &nf, &nd) != EMG_SUCCESS)
      throw std::invalid_argument("EMDOFManager: " + last_error());
    std::vector<std::vector<int32_t>> out(ne);
    for (size_t e = 0; e < ne; ++e)
      for (size_t k = 0; k < w && rows[w * e + k] != EMG_DOF_ABSENT; ++k) out[e].push_back(rows[w * e + k]);
    n_dofs_ = nd;
    n_scalar_free_ = ns;
    return out;
  }
  int getNumScalarFreeDOFs() const { return static_cast<int>(n_scalar_free_); }
  int getNumFreeDOFs() const { return static_cast<int>(n_dofs_); }
  const std::vector<int32_t>& getElemLocalToGlobal() const { return l2g_; }
  const std::vector<int32_t>& getEdgeToDOF() const { return edge_dof_; }
  std::vector<double> mapReducedSolutionToFull(const std::vector<double>& reduced) const {
    std::vector<double> full(edge_dof_.size());
    if (emg_dofmap_expand(map_, reduced.data(), full.data()) != EMG_SUCCESS)
      throw std::invalid_argument("mapReducedSolutionToFull: " + last_error());
    return full;
  }

 private:
  void run(int32_t mode) {
    emg_dofmap m = nullptr;
    if (emg_dof_build(mesh_.handle(), mode, &m) != EMG_SUCCESS)
      throw std::invalid_argument("EMDOFManager: " + last_error());
    adopt(m);
  }
  void adopt(emg_dofmap m) {
    if (map_) emg_dofmap_destroy(map_);
    map_ = m;
    int64_t ne = 0, nf = 0;
    emg_dofmap_info(map_, &ne, &nf, &n_dofs_);
    l2g_.resize(mesh_.edgesPerElement() * mesh_.getElementCount());
    edge_dof_.resize(ne);
    emg_dofmap_export(map_, l2g_.data(), edge_dof_.data());
  }
  const Mesh& mesh_;
  emg_dofmap map_ = nullptr;
  int64_t n_dofs_ = 0;
  int64_t n_scalar_free_ = 0;
  bool gauged_ = false;
  std::vector<int32_t> l2g_, edge_dof_;
};

// numeric::EMAssembly for TET4_EDGE / HEX8_EDGE / PRISM6_EDGE / PYRAMID5_EDGE on the GPU
// (src/numeric/em_assembly.cpp:144-420).
// Materials are reluctivity nu = 1/mu and conductivity sigma per material id.
class GpuEMAssembly {
 public:
  ~GpuEMAssembly() { clear(); }
  bool assemble(const Mesh& mesh, const std::vector<int32_t>& elem_local_to_global,
                const std::vector<double>& nu, const std::vector<double>& sigma,
                const std::vector<emg_source>& sources = {}, bool is_transient = false,
                int32_t flags = 0) {
    clear();
    int rc = emg_system_create_typed(mesh.elementType(), mesh.getNodeCount(), mesh.xyz().data(),
                                     mesh.getElementCount(), mesh.elements().data(),
                                     mesh.material().empty() ? nullptr : mesh.material().data(),
                                     elem_local_to_global.data(), 0, 0, nullptr, &sys_);
    if (rc == EMG_SUCCESS)
      rc = emg_system_assemble(sys_, nu.data(), sigma.empty() ? nullptr : sigma.data(),
                               static_cast<int32_t>(nu.size()), sources.empty() ? nullptr : sources.data(),
                               static_cast<int32_t>(sources.size()),
                               flags | (is_transient ? EMG_FLAG_MASS : 0), nullptr);
    if (rc != EMG_SUCCESS) {
      error_ = last_error();
      return false;
    }
    return true;
  }
  // Borrowed device matrix handles (valid while this object lives).
  emg_csr getStiffnessMatrix() const { return emg_system_matrix(sys_, 0); }
  emg_csr getMassMatrix() const { return emg_system_matrix(sys_, 1); }
  std::vector<double> getSourceVector() const {
    int64_t n = 0, nnz = 0;
    emg_system_info(sys_, &n, &nnz);
    std::vector<double> f(n);
    emg_system_export(sys_, nullptr, nullptr, nullptr, nullptr, f.data());
    return f;
  }
  int64_t rows() const {
    int64_t n = 0, nnz = 0;
    emg_system_info(sys_, &n, &nnz);
    return n;
  }
  emg_system handle() const { return sys_; }
  const std::string& error_message() const { return error_; }
  void clear() {
    emg_system_destroy(sys_);
    sys_ = nullptr;
  }

 private:
  emg_system sys_ = nullptr;
  std::string error_;
};

// numeric::CGSolver / numeric::BiCGSTABSolver (iterative_solvers.cpp:64-503, :820-1118)
template <bool kBiCG>
class GpuKrylovSolver {
 public:
  // preconditioner: EMG_PRECOND_NONE (0), _JACOBI (1) or _ILU0 (2), the
  // values of PreconditionerType (a bool `jacobi` converts to 0 / 1)
  explicit GpuKrylovSolver(double tolerance = 1e-8, int32_t max_iterations = 1000,
                           int32_t preconditioner = EMG_PRECOND_NONE)
      : cfg_{tolerance, max_iterations, preconditioner} {}
  ~GpuKrylovSolver() { clear(); }
  // CsrMatrix<double> from host arrays (duplicates summed, as to_eigen does).
  void set_matrix(int64_t n, const std::vector<int32_t>& row_ptr, const std::vector<int32_t>& col,
                  const std::vector<double>& val) {
    clear();
    if (emg_csr_create(n, row_ptr.data(), col.data(), val.data(), nullptr, &owned_) != EMG_SUCCESS)
      throw std::invalid_argument("set_matrix: " + last_error());
    A_ = owned_;
  }
  // Device matrix of a GpuEMAssembly (borrowed).
  void set_matrix(emg_csr device_matrix) {
    clear();
    A_ = device_matrix;
  }
  SolverResult solve(const std::vector<double>& b) {
    SolverResult r;
    if (!A_) {
      r.error_msg = "matrix not set";
      return r;
    }
    r.x.resize(b.size());
    emg_result out{};
    const int rc = kBiCG ? emg_bicgstab_solve(A_, b.data(), r.x.data(), &cfg_, &out)
                         : emg_cg_solve(A_, b.data(), r.x.data(), &cfg_, &out);
    r.status = static_cast<SolverStatus>(out.status <= EMG_INVALID_INPUT ? out.status : EMG_NUMERICAL_ERROR);
    r.iterations = out.iterations;
    r.residual_norm = out.residual_norm;
    r.solve_time_ms = out.solve_time_ms;
    if (rc > EMG_INVALID_INPUT) r.error_msg = last_error();
    return r;
  }
  std::string get_solver_name() const {
    return std::string(kBiCG ? "BiCGSTABSolver" : "CGSolver") +
           (cfg_.preconditioner == EMG_PRECOND_JACOBI ? "_Jacobi"
            : cfg_.preconditioner == EMG_PRECOND_ILU0 ? "_ILU0"
                                                      : "_None");
  }
  void clear() {
    if (owned_) emg_csr_destroy(owned_);
    owned_ = nullptr;
    A_ = nullptr;
  }

 private:
  emg_krylov_config cfg_;
  emg_csr A_ = nullptr;
  emg_csr owned_ = nullptr;
};

using GpuCGSolver = GpuKrylovSolver<false>;
using GpuBiCGSTABSolver = GpuKrylovSolver<true>;

// Mesh-level GPU solvers that own their factorization: kind false = the
// direct backend (SolverBackend / MUMPSBackend role, mumps_solver_backend.h:96-140),
// kind true = FETI-DP (fetidp_context.hpp:20-66 has no operators).
template <bool kFeti>
class GpuMeshSolver {
 public:
  GpuMeshSolver(const Mesh& mesh, const EMDOFManager& dofs) {
    const int rc = kFeti ? emg_fetidp_create(mesh.handle(), dofs.handle(), nullptr,
                                             reinterpret_cast<emg_fetidp*>(&h_))
                         : emg_direct_create(mesh.handle(), dofs.handle(), nullptr,
                                             reinterpret_cast<emg_direct*>(&h_));
    if (rc != EMG_SUCCESS) throw std::runtime_error(std::string(name()) + ": " + last_error());
  }
  ~GpuMeshSolver() {
    if (kFeti) emg_fetidp_destroy(static_cast<emg_fetidp>(h_));
    else emg_direct_destroy(static_cast<emg_direct>(h_));
  }
  GpuMeshSolver(const GpuMeshSolver&) = delete;
  GpuMeshSolver& operator=(const GpuMeshSolver&) = delete;
  // Numeric factorization for the materials (nu = 1/mu per material id) and sources.
  bool factor(const std::vector<double>& nu, const std::vector<double>& sigma = {},
              const std::vector<emg_source>& sources = {}) {
    const int32_t nm = static_cast<int32_t>(nu.size()), ns = static_cast<int32_t>(sources.size());
    const double* sg = sigma.empty() ? nullptr : sigma.data();
    const emg_source* src = sources.empty() ? nullptr : sources.data();
    const int rc = kFeti ? emg_fetidp_factor(static_cast<emg_fetidp>(h_), nu.data(), sg, nm, src, ns, 0)
                         : emg_direct_factor(static_cast<emg_direct>(h_), nu.data(), sg, nm, src, ns, 0);
    error_ = rc == EMG_SUCCESS ? "" : last_error();
    return rc == EMG_SUCCESS;
  }
  // K x = b (b empty: the assembled F) to a true relative residual `tolerance`.
  SolverResult solve(const std::vector<double>& b = {}, double tolerance = 1e-8, int32_t max_iterations = 1000) {
    SolverResult r;
    r.x.resize(n_dofs());
    emg_krylov_config cfg{tolerance, max_iterations, kFeti ? EMG_FETI_PRECOND_DELUXE : 0};
    emg_result out{};
    const double* bp = b.empty() ? nullptr : b.data();
    int rc;
    if (kFeti)
      rc = bp ? emg_fetidp_solve_rhs(static_cast<emg_fetidp>(h_), &cfg, bp, r.x.data(), 0, &out)
              : emg_fetidp_solve(static_cast<emg_fetidp>(h_), &cfg, r.x.data(), 0, &out);
    else
      rc = emg_direct_solve(static_cast<emg_direct>(h_), &cfg, bp, r.x.data(), 0, &out);
    r.status = static_cast<SolverStatus>(out.status <= EMG_INVALID_INPUT ? out.status : EMG_NUMERICAL_ERROR);
    if (rc > EMG_INVALID_INPUT) r.status = SolverStatus::NUMERICAL_ERROR;
    r.iterations = out.iterations;
    r.residual_norm = out.residual_norm;
    r.solve_time_ms = out.solve_time_ms;
    if (rc != EMG_SUCCESS) r.error_msg = last_error();
    return r;
  }
  int64_t n_dofs() const {
    int64_t info[2] = {0, 0};
    if (kFeti) emg_fetidp_info(static_cast<emg_fetidp>(h_), info, 2);
    else emg_direct_info(static_cast<emg_direct>(h_), info, 2);
    return info[1];
  }
  static const char* name() { return kFeti ? "GpuFetiDpSolver" : "GpuDirectBackend"; }
  const std::string& error_message() const { return error_; }

 private:
  void* h_ = nullptr;
  std::string error_;
};

using GpuDirectBackend = GpuMeshSolver<false>;
using GpuFetiDpSolver = GpuMeshSolver<true>;

}  // namespace emg

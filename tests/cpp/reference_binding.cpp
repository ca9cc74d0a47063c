// The reference-side binding of the GPU Krylov solvers, compiled against the
// reference's own headers: numeric::GpuCGSolver derives from the reference's
// EMLinearSolverBase (include/numeric/em_linear_solver.h:76-236) and takes the
// reference's CsrMatrix<double> (include/numeric/csr_matrix.hpp) and CGConfig
// (include/numeric/iterative_solvers.h:59-76), exactly as a maintainer would
// add it next to CGSolver.  main() reads a system written by the test
// (tests/test_reference_binding.py), solves it through the binding and through
// the reference's own CGSolver / BiCGSTABSolver (from the reference sources,
// linked from oracle/_ref), and prints one line per solve:
//   <solver> <precond> <status> <iterations> <residual> <rel. diff to the reference's x>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "em_linear_solver.h"
#include "emagddm_b200.h"
#include "iterative_solvers.h"

namespace numeric {

class GpuCGSolver : public EMLinearSolverBase {
 public:
  explicit GpuCGSolver(const CGConfig& c, bool bicgstab = false) : c_(c), bicg_(bicgstab) {}
  ~GpuCGSolver() override { clear(); }
  void set_matrix(const CsrMatrix<double>& A) override {
    clear();  // duplicates are summed, as SparseConverter::to_eigen does
    emg_csr_create(A.rows(), A.get_row_ptr().data(), A.get_col_indices().data(), A.get_values().data(), nullptr,
                   &A_);
  }
  void set_matrix(const CsrMatrix<std::complex<double>>&) override {}  // real systems only
  SolverResult solve(const Eigen::VectorXd& b) override {
    SolverResult r;
    r.x.resize(b.size());
    const int32_t pc = c_.preconditioner == CGConfig::PreconditionerType::JACOBI ? EMG_PRECOND_JACOBI
                       : c_.preconditioner == CGConfig::PreconditionerType::ILU0 ? EMG_PRECOND_ILU0
                                                                                 : EMG_PRECOND_NONE;
    emg_krylov_config cfg{c_.tolerance, c_.max_iterations, pc};
    emg_result o{};
    const int rc = bicg_ ? emg_bicgstab_solve(A_, b.data(), r.x.data(), &cfg, &o)
                         : emg_cg_solve(A_, b.data(), r.x.data(), &cfg, &o);
    r.status = static_cast<SolverStatus>(o.status <= 4 ? o.status : 1);
    r.iterations = o.iterations;
    r.residual_norm = o.residual_norm;
    r.solve_time_ms = o.solve_time_ms;
    if (rc > 4) r.error_msg = emg_last_error();
    return r;
  }
  SolverResult solve(const Eigen::VectorXcd&) override { return {}; }
  std::string get_solver_name() const override { return bicg_ ? "GpuBiCGSTAB" : "GpuCG"; }
  void clear() override {
    if (A_) emg_csr_destroy(A_);
    A_ = nullptr;
  }

 private:
  CGConfig c_;
  bool bicg_;
  emg_csr A_ = nullptr;
};

}  // namespace numeric

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: %s system.txt\n", argv[0]);
    return 2;
  }
  // system.txt: n nnz / row col value (nnz lines, COO, duplicates allowed) / b (n lines)
  std::ifstream f(argv[1]);
  int n = 0, nnz = 0;
  f >> n >> nnz;
  numeric::CooMatrix<double> coo(n, n);
  for (int k = 0; k < nnz; ++k) {
    int i, j;
    double v;
    f >> i >> j >> v;
    coo.add_value(i, j, v);
  }
  Eigen::VectorXd b(n);
  for (int i = 0; i < n; ++i) f >> b[i];
  numeric::CsrMatrix<double> A(n, n);
  A.build_from_coo(coo);
  const std::pair<numeric::CGConfig::PreconditionerType, const char*> pcs[] = {
      {numeric::CGConfig::PreconditionerType::NONE, "none"},
      {numeric::CGConfig::PreconditionerType::JACOBI, "jacobi"},
      {numeric::CGConfig::PreconditionerType::ILU0, "ilu0"}};
  for (const auto& [pc, name] : pcs) {
    numeric::CGConfig cfg;
    cfg.tolerance = 1e-10;
    cfg.max_iterations = 5000;
    cfg.preconditioner = pc;
    std::unique_ptr<numeric::EMLinearSolverBase> gpu = std::make_unique<numeric::GpuCGSolver>(cfg);
    numeric::CGSolver ref(cfg);
    gpu->set_matrix(A);
    ref.set_matrix(A);
    const numeric::SolverResult rg = gpu->solve(b), rr = ref.solve(b);
    const double diff = (rg.x - rr.x).norm() / std::max(rr.x.norm(), 1e-300);
    std::printf("%s %s %d %d %.6e %.6e\n", gpu->get_solver_name().c_str(), name, static_cast<int>(rg.status),
                rg.iterations, rg.residual_norm, diff);
    std::printf("CGSolver %s %d %d %.6e 0\n", name, static_cast<int>(rr.status), rr.iterations, rr.residual_norm);
  }
  return 0;
}

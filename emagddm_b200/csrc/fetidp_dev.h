// fetidp_dev.h -- device state of the FETI-DP solver (fetidp.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "device.h"
#include "fetidp.h"

namespace emg {

// Front table in structure-of-arrays form (front index F = the coarse matrix).
struct FrontsDev {
  const int32_t* sub;
  const int32_t* p0;
  const int32_t* npiv;
  const int32_t* f;
  const int32_t* nchild;
  const int32_t* child0;
  const int32_t* is_root;
  const int64_t* rows;
  const int64_t* fac;
  const int64_t* upd;
  const int64_t* cpos;
  const int64_t* vec;
  const int32_t* rows_v;
  const int32_t* child_v;
  const int32_t* cpos_v;
};

// Right-hand-side blocks of the multifrontal solves: subdomain s holds
// ncol[s] columns of n_r values at x[off[s] + pos + col * n_r].
struct RhsDev {
  double* x;
  const int64_t* off;
  const int32_t* ncol;
  const int64_t* voff;  // per front: offset of its nupd x ncol update vectors
  double* v;
};

// Faces of the deluxe scaling (multipliers grouped by subdomain pair).
struct FacesDev {
  int32_t n;
  const int32_t* a;
  const int32_t* b;
  const int32_t* dim;
  const int64_t* ptr;
  const int32_t* lam;
  const int64_t* off;  // f x f block offset of every face
  const int64_t* fac;  // offset of the face's Sa + Sb factor block in fac
};

struct FetiStats {
  int32_t iterations = 0;         // multiplier iterations over all correction passes
  int32_t refinements = 0;        // FETI-DP passes (1 + defect corrections)
  double lambda_residual = 0.0;   // ||r_lambda|| / ||r_lambda,0||
  double residual = 0.0;          // true ||b - A x|| / ||b|| of the global system
  double factor_ms = 0.0, solve_ms = 0.0;
  double lambda_ms = 0.0;  // device time of the multiplier iterations
  double fronts_ms = 0.0;  // device time of the right-hand sides and recoveries (front and coarse solves)
};

struct LearnState;
void free_learn(LearnState* L);

struct FetiDP {
  FetiPlan plan;
  LearnState* learn = nullptr;  // learned interface preconditioner (learned.cu), optional
  System un;  // block-diagonal union of the subdomain matrices
  cudaStream_t st = nullptr;
  std::vector<void*> dev;
  FrontsDev fd{};
  FacesDev fc{};
  bool factored = false;
  bool tc_factor = false;  // factor contractions on the TF32 tensor cores (EMG_FLAG_FACTOR_TF32)
  // CTA widths of the solve kernels (autotuned after the first factorization)
  int32_t piv_threads = 512, upd_rows = 256, gemv_warps = 8;
  bool mid_fronts = true;  // fused CTA-per-front solve kernels on the levels of medium fronts
  bool tuned = false;
  int32_t precond = 2;  // 0 none, 1 Dirichlet stiffness-scaled, 2 deluxe-scaled, 3 deluxe with FP32 blocks,
                        // 4 deluxe + learned correction (flexible CG)
  FetiStats stats;
  // plan tables
  int64_t* d_loc_off = nullptr;
  int32_t *d_nI = nullptr, *d_nD = nullptr, *d_nP = nullptr;
  int64_t* d_dual_off = nullptr;
  int32_t *d_dual_lam = nullptr, *d_dual_sign = nullptr, *d_lam_entry = nullptr, *d_dual_sub = nullptr;
  int64_t* d_pri_off = nullptr;
  int32_t *d_pri_coarse = nullptr, *d_pri_sub = nullptr;
  int64_t* d_coarse_ptr = nullptr;
  int32_t* d_coarse_list = nullptr;
  int64_t *d_cblk_off = nullptr, *d_sc_ptr = nullptr, *d_sc_list = nullptr;
  int64_t* d_gptr = nullptr;
  int32_t *d_glist = nullptr, *d_union_gdof = nullptr;
  int64_t* d_root_off = nullptr;
  // dense blocks
  int32_t n_roots = 0, max_nD = 0, max_ncol = 1;
  int32_t* d_rdim = nullptr;
  int32_t *d_root_k = nullptr, *d_root_sub = nullptr;
  int64_t *d_rfac = nullptr, *d_roff = nullptr, *d_rvoff = nullptr;
  int64_t* d_pcoff = nullptr;  // per root: offset of its column-sum slots in pc_d
  double* pc_d = nullptr;       // column sums of the tiles below the diagonal (symmetric S_DD products)
  int32_t* d_cdim = nullptr;
  int64_t *d_cfac = nullptr, *d_czero = nullptr;
  int64_t coarse_fac = 0;
  // extra fronts after the plan's: [0] the coarse matrix, [1 + f] face f's S_a + S_b
  std::vector<int32_t> xnp;
  std::vector<int32_t> lvl_max_np, lvl_max_nu, lvl_max_f;  // per level, non-root fronts: largest pivot / update
                                                         // counts and front size
  int32_t max_fdim = 0;
  // solve layouts
  int64_t *d_roff_s = nullptr, *d_roff1 = nullptr, *d_voff_s = nullptr, *d_voff1 = nullptr;
  int32_t *d_ncol_s = nullptr, *d_ncol1 = nullptr;
  int64_t phi_size = 0, vs_size = 0;
  // numeric storage
  double *fac_d = nullptr, *upd_d = nullptr, *S_d = nullptr, *Linv_d = nullptr, *Lcc_d = nullptr;
  double *phi_d = nullptr, *vs_d = nullptr, *v1_d = nullptr, *cblk_d = nullptr, *h_d = nullptr;
  double *gc_d = nullptr, *uc_d = nullptr, *t_d = nullptr, *t2_d = nullptr;
  double* cdots_d = nullptr;  // per primal entry of each coarse DOF: its Phi_D column dot
  double *rho_d = nullptr, *wt_d = nullptr, *w_d = nullptr, *y_d = nullptr, *y2_d = nullptr;
  double *xu_d = nullptr, *ru_d = nullptr, *xg_d = nullptr, *rg_d = nullptr, *bg_d = nullptr;
  double *lam_d = nullptr, *r_d = nullptr, *z_d = nullptr, *p_d = nullptr, *q_d = nullptr, *rhs_d = nullptr;
  double* part_d = nullptr;
  double *fSa_d = nullptr, *fSb_d = nullptr, *fX_d = nullptr, *fXt_d = nullptr, *fZ_d = nullptr;
  double *fDa_d = nullptr, *fDb_d = nullptr, *c_d = nullptr;
  double *fu_d = nullptr, *xacc_d = nullptr, *rglob_d = nullptr, *root_tmp_d = nullptr;
  double *rold_d = nullptr, *zm_d = nullptr;  // flexible CG
  double *fp_d = nullptr, *fq_d = nullptr, *fr0_d = nullptr;  // global flexible CG (mixed factor)
  double* diag0_d = nullptr;  // original diagonal of the subdomain matrices (union numbering), pivot scale
  // FP32 copies of the preconditioner blocks (mixed-precision mode)
  float *S32_d = nullptr, *fDa32_d = nullptr, *fDb32_d = nullptr, *fDaT32_d = nullptr, *fDbT32_d = nullptr;
  void* state_d = nullptr;
  int32_t* err_d = nullptr;
  // device-side multiplier loop: one while-loop graph per preconditioner 0..3
  cudaGraphExec_t lam_exec[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaStream_t cap_st = nullptr;
  // second stream of the captured factorization: the deluxe face set-up
  // (which needs only the assembled S_DD blocks) beside the root inverse
  // factors and the coarse basis
  cudaStream_t side_st = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  bool graph_failed = false;
  // the numeric factorization as one graph per factor mode (FP64, mixed)
  cudaGraphExec_t fac_exec[2] = {nullptr, nullptr};
  bool fac_eager[2] = {false, false};  // a factorization of this kind (FP64 / TF32) has run eagerly
  bool fac_graph_failed = false;
  bool capturing = false;  // a capture is recording: defer checks, no attribute calls
  static constexpr int kParts = 592;

  ~FetiDP();
  void release();
  // Symbolic phase: plan, union system pattern, device tables and storage.
  int create(const Mesh& m, const DofMap& d, cudaStream_t stream);
  // Numeric phase for the given materials / sources.
  int factor(const double* nu, const double* sigma, int32_t n_mat, const emg_source* src, int32_t n_src,
             int32_t flags);
  // K x = b for the global right-hand side b_d (device, n_dofs; null = the
  // assembled F) to the true relative residual cfg.tolerance: FETI-DP passes
  // (lambda-PCG, recovery) with defect correction on the true residual.
  int solve(const emg_krylov_config& cfg, const double* b_d, double* x_d, emg_result* res);
  // Multiplier-space pieces for training and tests: op 0 F, 1 deluxe M_D,
  // 2 learned correction L, 3 M_D + L (device vectors of n_lambda).
  int apply_op(int32_t op, const double* in, double* out);
  // Right-hand side of the multiplier system for a global b (null = F).
  int lambda_rhs(const double* b, double* out);

 private:
  template <class T>
  int up(T** dst, const std::vector<T>& src);
  int zalloc(double** dst, int64_t n);
  int zallocf(float** dst, int64_t n);
  int setup_device();
  int check_err(const char* where);
  int factor_range(int32_t f0, int32_t f1);
  int factor_device();
  int solve_fronts(const RhsDev& R, int32_t ncol);
  void coarse_solve(const double* t, double* u);
  void coarse_apply_t(const RhsDev& R, const double* w, const double* add, double* t);
  template <class T>
  void symv_roots(const T* M, const double* w, double* y);
  void apply_F(const double* p, double* q, double* part);
  void apply_M(const double* r, double* z, double* part);
  int dot(const double* a, const double* b, int64_t n, int which);
  int setup_deluxe();
  void tune_solve_kernels();
  int trtri(int32_t n_mat, int32_t max_n, const int32_t* dim, const int64_t* l_off, const int64_t* x_off, double* X);
  int prepare_rhs(const double* fu);
  int lambda_pcg(double tol, int32_t max_it, int32_t* iters, double* rel);
  void lambda_body(void* state);
  cudaGraphExec_t lambda_loop_graph();
  int lambda_fcg(double tol, int32_t max_it, int32_t* iters, double* rel);
  double dot_host(const double* a, const double* b, int64_t n);
  int recover(const double* fu);
  int global_residual(const double* b, const double* x, double* rr);
  int fcg(const emg_krylov_config& cfg, double bb, int* status, int32_t* total, int32_t* outer, double* rel,
          double* lam_rel, double* lambda_ms, double* fronts_ms);
};

// learned.cu
int learned_init(FetiDP& F, uint64_t seed);
int learned_apply(FetiDP& F, const double* r, const double* add, double* out);
int learned_train(FetiDP& F, int32_t B, const double* r, const double* t, float lr, double* loss);
int learned_params(FetiDP& F, float* host, int64_t* n, int32_t load);

}  // namespace emg

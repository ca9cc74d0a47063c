// device.h -- host-side interface of the CUDA parts of libemagddm_b200.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "emagddm_b200.h"

namespace emg {

void set_error(const std::string& msg);

#define EMG_CK(call)                                                              \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess) {                                                      \
      ::emg::set_error(std::string(#call) + ": " + cudaGetErrorString(e_));       \
      return EMG_ERR_CUDA;                                                        \
    }                                                                             \
  } while (0)

struct KrylovWorkspace;
struct Sell;
struct BatchPlan;
struct IluState;

// Device CSR matrix (int32 row_ptr / col, fp64 values, rows sorted, merged).
// `version` changes whenever the values change (re-assembly), so derived
// solver formats know when to refresh.
struct DevCsr {
  int64_t n = 0;
  int64_t nnz = 0;
  int32_t* row_ptr = nullptr;
  int32_t* col = nullptr;
  double* val = nullptr;
  bool owns_pattern = true;
  bool owns_values = true;
  uint64_t version = 0;
  KrylovWorkspace* ws = nullptr;
  Sell* sell = nullptr;
  BatchPlan* batch = nullptr;  // lockstep batch layout (batch.cu)
  IluState* ilu = nullptr;     // ILU(0) factor, level schedules and Krylov state (ilu.cu)
  ~DevCsr();
};

// Assembled system on the device (EMAssembly state).
struct System {
  int32_t elem_type = EMG_ELEM_TET4_EDGE;
  int64_t n_nodes = 0, n_elems = 0, n = 0;
  double* xyz = nullptr;       // 3 * n_nodes
  int32_t* elems = nullptr;    // nodes_per_elem * n_elems
  int32_t* material = nullptr; // n_elems
  int32_t* l2g = nullptr;      // edges_per_elem * n_elems
  int32_t* inc_ptr = nullptr;  // n + 1: incidence of every row (element-edge slots)
  int32_t* inc = nullptr;      // sorted slots edges_per_elem * t + k per row
  int32_t* err = nullptr;      // device error word
  double* rhs = nullptr;       // n
  int32_t* src_map = nullptr;  // optional per-element source index (n_elems)
  // TET4_EDGE: for every incidence slot (8 bytes each), the position of the
  // slot's element columns 0..5 inside the row (0xFF: constrained edge)
  uint8_t* slot_pos = nullptr;
  int32_t max_row_len = 0;     // longest CSR row
  DevCsr K, M;                 // M shares K's pattern
  bool has_mass = false;
  ~System();
};

// DOF numbering of a one-type mesh on the device (numbering_gpu.cu), bit-exact
// to build_dofmap for EMG_GAUGE_NONE / EMG_GAUGE_REF.
int dof_build_gpu(int32_t elem_type, int64_t n_nodes, int64_t n_elems, const int32_t* elems, int64_t n_dir,
                  const int32_t* dir_pairs, int32_t n_hole_markers, int32_t gauge, int32_t* l2g_out,
                  int64_t* n_edges_out, int64_t* n_free_out, int64_t* n_dofs_out, cudaStream_t st);

// Symbolic phase: incidence lists and the merged CSR pattern, all on the device.
int system_build(System& s, cudaStream_t st);
// Numeric phase: K (and M), F.
int system_assemble(System& s, const double* nu, const double* sigma, int32_t n_mat,
                    const emg_source* src, int32_t n_src, int32_t flags, cudaStream_t st);

// EMG_PRECOND_NONE / _JACOBI (and _ILU0 where the solver has it), else
// EMG_INVALID_INPUT with a message (no silent substitution).
inline int check_krylov_precond(int32_t p, bool ilu0_allowed = false) {
  if (p == EMG_PRECOND_NONE || p == EMG_PRECOND_JACOBI || (ilu0_allowed && p == EMG_PRECOND_ILU0)) return EMG_SUCCESS;
  set_error("preconditioner " + std::to_string(p) +
            (ilu0_allowed ? ": use EMG_PRECOND_NONE (0), EMG_PRECOND_JACOBI (1) or EMG_PRECOND_ILU0 (2)"
                          : ": this solver takes EMG_PRECOND_NONE (0) or EMG_PRECOND_JACOBI (1)"));
  return EMG_INVALID_INPUT;
}

// Exclusive scan of n int32 counts into out[0..n]; returns the total.
int scan_counts(const int32_t* counts, int32_t* out, int64_t n, int64_t* total, cudaStream_t st);

// Validates a device CSR (offsets, column range, ascending columns).
int check_csr(int64_t n, const int32_t* rp, const int32_t* col, int64_t nnz, cudaStream_t st);
// out = a x + b y (n values; ops.cu).
int axpby_values(double* out, double a, const double* x, double b, const double* y, int64_t n,
                 cudaStream_t st);
// Keeps the default memory pool's freed blocks cached (once per device).
void keep_pool_memory();

int csr_spmv(DevCsr& A, const double* x, double* y, cudaStream_t st);
int cg_solve(DevCsr& A, const double* b, double* x, const emg_krylov_config& cfg,
             cudaStream_t st, emg_result* res);
int bicgstab_solve(DevCsr& A, const double* b, double* x, const emg_krylov_config& cfg,
                   cudaStream_t st, emg_result* res);
int csr_history(DevCsr& A, double* out, int32_t cap);
int cg_kernel_times(DevCsr& A, int32_t iterations, cudaStream_t st, double* ms);
int set_barrier_spins(int32_t spins);
void free_workspace(KrylovWorkspace* ws);
void free_batch(BatchPlan* p);
void free_ilu(IluState* s);
// CG / BiCGSTAB with the ILU(0) preconditioner (ilu.cu).
int ilu_solve(DevCsr& A, const double* b, double* x, const emg_krylov_config& cfg, cudaStream_t st,
              emg_result* res, bool bicg);
// Lockstep CG over the diagonal blocks [blocks[k], blocks[k+1]) of A (batch.cu).
int batch_cg_solve(DevCsr& A, int32_t nb, const int64_t* blocks, const double* b, double* x,
                   const emg_krylov_config& cfg, cudaStream_t st, emg_result* results);
// Allocation-free CG on a caller-owned device CSR (noalloc.cu).
int cg_solve_noalloc(int64_t n, int64_t nnz, const int32_t* rp, const int32_t* col, const double* val,
                     const double* b, double* x, const emg_krylov_config& cfg, cudaStream_t st,
                     emg_result* res);
int64_t sell_slots(DevCsr& A);
int64_t sell_slices(DevCsr& A);

}  // namespace emg

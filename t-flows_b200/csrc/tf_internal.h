// tf_internal.h -- host-side structures shared by the library's .cu files.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/tf_krylov.h"
#include "tf_common.cuh"

#include "tf_tile.cuh"

// Every int-returning C-ABI entry point runs its body between TF_API_BEGIN
// and TF_API_END, so no C++ exception crosses the C ABI: a failed host
// allocation returns TF_ERR_OOM, any other exception TF_ERR_HOST.
#define TF_API_BEGIN try {
#define TF_API_END                                              \
  }                                                             \
  catch (const std::bad_alloc&) { return TF_ERR_OOM; }          \
  catch (const std::length_error&) { return TF_ERR_OOM; }       \
  catch (...) { return TF_ERR_HOST; }

// The same for work done on the library's own threads (pool workers, the
// server loop): f's status, or the status of the exception it threw.
template <class F>
int tf_guarded(F&& f) {
  try {
    return f();
  } catch (const std::bad_alloc&) {
    return TF_ERR_OOM;
  } catch (const std::length_error&) {
    return TF_ERR_OOM;
  } catch (...) {
    return TF_ERR_HOST;
  }
}

#define TF_CUDA_TRY(expr)                                       \
  do {                                                          \
    cudaError_t _e = (expr);                                    \
    if (_e != cudaSuccess) {                                    \
      tf_set_last_cuda_error(_e, #expr, __FILE__, __LINE__);    \
      return (_e == cudaErrorMemoryAllocation) ? TF_ERR_OOM     \
                                               : TF_ERR_CUDA;   \
    }                                                           \
  } while (0)

void tf_set_last_cuda_error(cudaError_t e, const char* what, const char* file,
                            int line);
void tf_set_last_message(const char* msg);

struct tf_ctx_s {
  int device = 0;
  int sm_count = 148;
  size_t l2_bytes = 0;
  cudaStream_t stream = nullptr;
  int history = 0;
  unsigned long long wait_ns = 0;   // bounded-wait limit of this context's solves (0: default)
  double* d_vec_scratch = nullptr;  // partial sums of the tf_vec_* reductions (tf_vec.cu)
  std::vector<double> last_hist;
  int last_count = 0;
  // Stream-ordered allocation (cudaMallocAsync / cudaFreeAsync on `stream`)
  // for matrices registered on this context: set by the request pool so a
  // worker never synchronises the device when it registers or releases.
  int async_alloc = 0;
  tf::SolveState* h_state = nullptr;    // pinned, lent to async matrices
  tf::SolveParams* h_params = nullptr;
};

// Right-hand sides 2..nrhs of a multi-RHS solve (tf_solve_multi): their own
// Krylov vectors, reduction partials and solve state over the matrix's
// structure and values.
struct tf_slice_s {
  double* d_x = nullptr;
  double* d_b = nullptr;
  double* d_r = nullptr;
  double* d_p = nullptr;
  double* d_q = nullptr;
  double* d_adiag = nullptr;
  double* d_part = nullptr;
  tf::SolveState* d_state = nullptr;
};
constexpr int kMaxRhs = 4;

// Device mirror of one Matrix_Type plus the Krylov workspace of its solves.
struct tf_matrix_s {
  tf_ctx_s* ctx = nullptr;
  int nt = 0, ni = 0;
  int64_t nnz = 0;
  int max_row_len = 0;
  int diag_first = 1;
  // structure, 0-based, padded for 16-byte bulk copies
  int* d_row = nullptr;
  int* d_col = nullptr;
  int* d_dia = nullptr;
  // FP64 values and vectors (nt entries, padded)
  double* d_val = nullptr;
  double* d_x = nullptr;
  double* d_b = nullptr;
  double* d_r = nullptr;
  double* d_p = nullptr;
  double* d_q = nullptr;
  double* d_z = nullptr;      // preconditioned residual (ICC only)
  double* d_adiag = nullptr;  // diagonal of the scaled matrix
  double* d_part = nullptr;   // grid-reduction partials
  double* d_hist = nullptr;
  int hist_cap = 0;
  tf::SolveState* d_state = nullptr;
  tf::SolveParams* d_params = nullptr;
  tf::SolveState* h_state = nullptr;    // pinned
  tf::SolveParams* h_params = nullptr;  // pinned
  // Row-pattern column layout (structured meshes): one pattern byte per
  // own row and the pattern table; npat = 0 when the rows do not fit it.
  unsigned char* d_pat = nullptr;
  int* d_pat_tab = nullptr;
  int npat = 0;
  // SpMV tiling picked at registration; variable tiles (tile_cfg 4-7):
  // ntiles + 1 row boundaries
  int tile_cfg = tf::kTileNone;
  int* d_tiles = nullptr;
  int ntiles = 0;
  // SpMV layouts timed at registration (configuration, median us per launch)
  std::vector<std::pair<int, double>> tune;
  int spmv_grid = 1;
  int vec_grid = 1;
  int vec_dir = 0;       // walking direction of the vector kernels (see tf_fp64.cu)
  // ICC level schedule (built at registration for diagonal-first matrices)
  int icc_ready = 0;
  int* d_levf_rows = nullptr;  // forward-sweep rows grouped by level
  int* d_levb_rows = nullptr;  // backward-sweep rows grouped by level
  std::vector<int> h_levf_ptr, h_levb_ptr;
  double* d_icc_d = nullptr;     // Prec_Form's d
  double* d_icc_dinv = nullptr;  // Prec_Form's d_inv
  // Persistent sweeps (k_icc_sweep): the level pointers on the device.
  int* d_icc_levf_ptr = nullptr;
  int* d_icc_levb_ptr = nullptr;
  int icc_sweep_grid = 0;        // 0: per-level kernels
  // cached graphs, one per (preconditioner, x update deferred or not)
  cudaGraphExec_t graph[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  // The same graphs bound to a caller's device val/x/b (tf_solve_device in
  // place): d_val, d_x, d_b point at the caller's arrays while such a solve
  // runs (ext_bound), and ext_key names the arrays ext_graph was built on.
  cudaGraphExec_t ext_graph[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  const void* ext_key[3] = {nullptr, nullptr, nullptr};
  int ext_bound = 0;
  std::mutex mu;
  int async_alloc = 0;   // device arrays from cudaMallocAsync on ctx->stream
  int host_lent = 0;     // h_state / h_params belong to the context
  size_t dev_bytes = 0;  // device bytes this matrix holds (with `ren`)
  // Renumbered copy for the Jacobi / none solves (tf_renumber.cu): row i'
  // of `ren` is row perm[i'] here, entry j' of `ren` is entry src[j'].
  tf_matrix_s* ren = nullptr;
  int* d_perm = nullptr;
  int* d_src = nullptr;
  tf_matrix_s* active = nullptr;  // the matrix the last solve ran on
  // Face topology for device-side assembly (tf_assemble.cu): per face the
  // two cells (0-based, -1 on a boundary) and pos(1:2) (0-based entries),
  // per cell its faces in ascending order (bit 0: the cell is the face's c2).
  int n_faces = 0;
  int* d_face_cell = nullptr;
  int* d_face_pos = nullptr;
  int* d_cf_ptr = nullptr;
  int* d_cf = nullptr;
  // Multi-RHS solves: slices for right-hand sides 2..kMaxRhs (allocated on
  // first use), pinned states of all right-hand sides, cached graphs per
  // (rhs count, preconditioner, x update deferred).
  tf_slice_s* slices[kMaxRhs - 1] = {nullptr, nullptr, nullptr};
  tf::SolveState* h_mstate = nullptr;
  cudaGraphExec_t mgraph[kMaxRhs + 1][2][2] = {};
};
// Multi-RHS drop-in (tf_fp64.cu): slice allocation and the solve on
// device-resident val / x_i / b_i (x and b slices of nt doubles each).
int tf_fp64_run_multi(tf_matrix_s* m, int prec, int nrhs);
int tf_slices_ensure(tf_matrix_s* m, int nrhs);   // allocate slices 1..nrhs-1
void tf_slices_free(tf_matrix_s* m);

// FP64 drop-in entry points implemented in tf_fp64.cu
int tf_fp64_prepare(tf_matrix_s* m);
// Picks the SpMV layout of a freshly registered matrix (tf_fp64.cu): the
// TF_TILE_CFG override when valid, else the fastest of the candidate
// layouts timed on the device (cached per matrix class), else a rule for
// small matrices; then prepares the kernels.  fit_mask bit c: fixed tile
// configuration c (0-2) holds every tile of the matrix.
int tf_choose_tiles(tf_matrix_s* m, unsigned fit_mask);
void tf_tune_cache_clear();
int tf_fp64_run(tf_matrix_s* m, int prec);   // runs on m->ctx->stream
int tf_fp64_spmv(tf_matrix_s* m, const double* val, const double* p,
                 double* q, double* pq);
int tf_fp64_residual(tf_matrix_s* m, const double* val, const double* b,
                     const double* x, double* r);
int tf_fp64_nrms(tf_matrix_s* m, const double* val, const double* r,
                 const double* x, int has_norm, double norm, double* out);
int tf_icc_build(tf_matrix_s* m, const int* h_row0, const int* h_col0);
// Grid of the persistent ICC sweeps (tf_fp64.cu), which run only when
// TF_ICC_PERSISTENT is set at registration (and the device launches
// cooperatively): one kernel per level measured faster (a 120^3 hex: 4.8
// against 5.3 ms per iteration).  icc_sweep_grid = 0 selects the per-level
// kernels.
int tf_icc_prepare_sweeps(tf_matrix_s* m);
// Registration behind tf_matrix_register; want_icc = 0 skips the ICC level
// schedule.  Device bytes the matrix will hold, for budgeting.
int tf_matrix_create(tf_ctx_s* ctx, int n_cells, int n_own, int64_t nnz, const int* row,
                     const int* col, const int* dia, int want_icc, tf_matrix_s** out);
void tf_matrix_free(tf_matrix_s* m);
size_t tf_matrix_bytes(int n_cells, int64_t nnz);
// Solve on a registered matrix with val/x/b already in its device buffers.
int tf_solve_resident(tf_matrix_s* m, int prec, int miter, double tol, const double* norm,
                      int* niter, double* fin_res);
int tf_dev_alloc_bytes(tf_ctx_s* ctx, void** p, size_t bytes);
// Renumbering (tf_renumber.cu)
double tf_gather_lines_per_warp(const int* row, const int* col, int n, int base);
// Row patterns of the first ni rows of a 0-based CSR: pat[i] (ni + 32
// bytes) names row i's offset sequence (col_j - i over its entries, in
// storage order), tab holds the sequences ([npat][kPatMaxLen], then the
// npat lengths).  Returns npat, or 0 when more than kPatMax patterns or a
// row longer than kPatMaxLen would be needed.
int tf_find_row_patterns(const std::vector<int>& row0, const std::vector<int>& col0, int ni,
                         std::vector<unsigned char>& pat, std::vector<int>& tab);
void tf_rcm_order(const std::vector<int>& row0, const std::vector<int>& col0, int n,
                  std::vector<int>& order);
int tf_renumber_in(tf_matrix_s* m);
int tf_renumber_out(tf_matrix_s* m);
// Matrices of at least this many rows whose sampled warp gathers touch more
// than kRenumberLines lines get a renumbered copy when RCM cuts that by 20 %.
constexpr int kRenumberMinRows = 10000;
constexpr double kRenumberLines = 6.0;
// Device bytes registration may take, renumbered copy included, for
// budgeting before the matrix exists (Matrix_Type 1-based row/col).
size_t tf_matrix_bytes_for(int n_cells, int64_t nnz, const int* row, const int* col);


/* ==========================================================================
 *  tf_krylov.h -- C ABI of the B200 native Krylov solvers for T-Flows.
 *
 *  Drop-in replacement for the body of Native_Type % Solve_Native
 *  (Sources/Process/Cpu/Native_Mod/Solve_Native.f90:2-46) and the solvers it
 *  dispatches to (Native_Mod/Cg.f90, Native_Mod/Bicg.f90) with the
 *  preconditioners of Native_Mod/Prec_Form.f90 and Prec_Solve.f90.
 *
 *  Conventions (those of Matrix_Type, Sources/Process/Cpu/Matrix_Mod.f90:57-76):
 *    - row(1..n+1), col(1..nnz), dia(1..n) hold 1-based indices, exactly as
 *      Create_Matrix builds them; the diagonal is the first entry of a row;
 *    - every real is double (the REAL=double build);
 *    - x points at x(1) of the Fortran array x(-nb:n); boundary entries
 *      x(-nb:0) are never referenced because col >= 1.
 *  Every function returns an int status (TF_OK = 0).  Non-convergence is not
 *  an error: it is reported as niter == miter with fin_res >= tol, as the
 *  reference does.
 *
 *  Threading: one CUDA stream per context; calls on one context must not
 *  overlap.  Different contexts may be used from different threads.
 * ========================================================================== */
#ifndef TF_KRYLOV_H
#define TF_KRYLOV_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  64 is the code the reference passes to Message % Error for
 * an unknown solver (Solve_Native.f90:38); 72 the one its control reader uses
 * for an unknown preconditioner keyword
 * (Shared/Control_Mod/Native/Preconditioner_For_System_Matrix.f90:36), here
 * returned for a preconditioner code outside enum tf_prec.  A preconditioner
 * NAME that is not known runs unpreconditioned, as Solve_Native does. */
enum tf_status {
  TF_OK = 0,
  TF_ERR_CUDA = 1,           /* a CUDA runtime call failed                       */
  TF_ERR_OOM = 2,            /* device (or host) allocation failed, or over the
                                memory budget                                  */
  TF_ERR_ARG = 3,            /* bad argument (null pointer, size, index range)   */
  TF_ERR_TIMEOUT = 4,        /* a bounded device-side wait gave up               */
  TF_ERR_LAYOUT = 5,         /* CSR layout violates Matrix_Type's contract       */
  TF_ERR_NO_DEVICE = 6,      /* no CUDA device / driver                          */
  TF_ERR_BUSY = 7,           /* serving queue full or handle in use              */
  TF_ERR_CANCELLED = 8,      /* request cancelled before it finished             */
  TF_ERR_HOST = 9,           /* host-side failure (no entry point lets a C++
                                exception escape; host out-of-memory is OOM)  */
  TF_ERR_UNKNOWN_SOLVER = 64,
  TF_ERR_UNKNOWN_PREC = 72
};

enum tf_solver { TF_SOLVER_CG = 0, TF_SOLVER_BICG = 1 };
enum tf_prec { TF_PREC_NONE = 0, TF_PREC_JACOBI = 1, TF_PREC_ICC = 2 };

typedef struct tf_ctx_s* tf_ctx;        /* device, stream, Krylov workspace   */
typedef struct tf_matrix_s* tf_matrix;  /* device-resident CSR structure      */

/* Human-readable text for a status code (static storage). */
const char* tf_status_string(int status);

/* Library version, e.g. "tfkrylov 0.1 sm_100a". */
const char* tf_version(void);

/* Text of the last CUDA failure or argument rejection seen by the library
 * (process-wide, static storage until the next failure). */
const char* tf_last_error_message(void);

/* Context on CUDA device `device` (-1: current device).  Replaces the
 * Work_Mod scratch arrays that Cg/Bicg connect (Cg.f90:44, Bicg.f90:45)
 * and the Nat object made by Create_Native (Native_Mod/Create_Native.f90:2-25). */
int tf_ctx_create(int device, tf_ctx* out);
int tf_ctx_destroy(tf_ctx ctx);

/* Upload the structure of one Matrix_Type (row, col, dia) once; values are
 * passed per solve because Process assembles them on the host each time.
 * Replaces Matrix_Mod/Create_Matrix.f90's result being visible to the
 * solver.  n_cells = Grid % n_cells (nt), n_own = nt - n_buff_cells (ni),
 * nnz = row(n_cells+1) - 1.  The arrays are copied; the caller keeps them. */
int tf_matrix_register(tf_ctx ctx, int n_cells, int n_own, int64_t nnz,
                       const int* row, const int* col, const int* dia,
                       tf_matrix* out);
int tf_matrix_release(tf_matrix m);
int tf_matrix_info(tf_matrix m, int* n_cells, int* n_own, int64_t* nnz,
                   int* max_row_len);
/* SpMV layout chosen at registration: 0/1/2 = fixed tiles of 512/256/128
 * rows staged in shared memory (row-pattern or CSR columns), 3 = rows read
 * straight from global memory, 4/5/6/7 = CSR tiles of variable length (at
 * most 512 rows and 4096 entries) whose rows are summed by groups of
 * 1/2/4/8 lanes.  Every layout gives the same row sums bit for bit.  The
 * layout is chosen by timing the candidates on the device when the matrix
 * is registered (tf_matrix_tuning), once per class of matrix (size, mean
 * and longest row, row patterns or not) per process; the environment
 * variable TF_TILE_CFG forces one, TF_NO_TUNE skips the timing. */
int tf_matrix_tile_config(tf_matrix m);
/* The candidates timed when m was registered: cfg[i] (as
 * tf_matrix_tile_config) and us[i], the median microseconds of one q = A p
 * launch, for i < min(cap, *count).  *count = 0 when the layout came from
 * the cache of an earlier registration of the same class, from
 * TF_TILE_CFG, or from the rule used for small matrices (under 16,384 rows)
 * and row-pattern matrices.  No reference counterpart (the reference has a
 * single loop order). */
int tf_matrix_tuning(tf_matrix m, int* cfg, double* us, int cap, int* count);
/* Forget the layouts chosen for earlier registrations, so the next matrix
 * of each class is timed again. */
int tf_tuning_cache_clear(void);
/* Levels of the incomplete-Cholesky sweeps built at registration (rows of
 * one level depend only on rows of earlier levels in Prec_Form.f90:69-78 /
 * Prec_Solve.f90:67-92's recurrences): forward and backward counts, 0 when
 * ICC is unavailable (diagonal not first).  No reference counterpart. */
int tf_matrix_icc_levels(tf_matrix m, int* forward, int* backward);
/* Number of row patterns of the compressed column layout chosen at
 * registration (rows whose column offsets relative to the row index repeat,
 * as on structured hex blocks: one byte per row instead of four per entry;
 * same entries, same order, same sums), 0 when the CSR columns are used.
 * No reference counterpart: a property of this library's device layout. */
int tf_matrix_row_patterns(tf_matrix m);
/* 1 when registration also built a renumbered copy of the matrix (reverse
 * Cuthill-McKee, applied symmetrically) because the given cell numbering
 * scatters the SpMV's gathers; Jacobi / none solves then run on that copy
 * (inputs permuted in and results back on the device; every row keeps its
 * entries in storage order, so row sums are unchanged).  0 otherwise.
 * No reference counterpart: a property of this library's device layout. */
int tf_matrix_renumbered(tf_matrix m);

/* Solve A x = b.  Replaces Native_Type % Solve_Native (Solve_Native.f90:2-46)
 * and so Cg.f90:2-257 / Bicg.f90:2-269.  val, x and b are host arrays of
 * nnz, n_cells and n_cells doubles and are updated exactly as the reference
 * updates them: x is overwritten with the solution, val and b come back as
 * (v*fn)/fn where fn = 1/mean(diag) (Cg.f90:62-84, 245-250).  norm == NULL
 * means the optional argument `norm` is absent (Fortran bind(C) passes NULL
 * for an absent OPTIONAL).  niter/fin_res follow Cg.f90:101-123, 220-228. */
int tf_solve(tf_ctx ctx, tf_matrix m, int solver, int prec, double* val,
             double* x, double* b, int miter, int* niter, double tol,
             double* fin_res, const double* norm);

/* Same, with the solver and preconditioner given by name as in
 * Solve_Native.f90:33-44 ('cg', 'bicg') and Prec_Form.f90:47-89 ('jacobi',
 * 'icc', anything else = none: the else branches of Prec_Form and
 * Prec_Solve, so an unknown name is not an error, as in the reference).
 * The control-file spellings 'diagonal' and 'incomplete_cholesky' are
 * mapped as Preconditioner_For_System_Matrix.f90:43-44 maps them.  Trailing
 * blanks are ignored.  Unknown solver -> TF_ERR_UNKNOWN_SOLVER (the
 * reference's 64). */
int tf_solve_native(tf_ctx ctx, tf_matrix m, const char* solver,
                    const char* prec, double* val, double* x, double* b,
                    int miter, int* niter, double tol, double* fin_res,
                    const double* norm);

/* Same as tf_solve with val, x and b already in device memory (e.g. an
 * OpenACC `host_data use_device` region).  Nothing crosses PCIe except the
 * two result scalars.  When all three are 16-byte aligned (as cudaMalloc'd
 * arrays are) the solve runs on them in place: the first call with a new
 * set of arrays builds the solve's CUDA graph on them, later calls with the
 * same arrays reuse it.  val is then read in 16-byte units, so up to 8
 * bytes past its last entry are read (inside any cudaMalloc allocation).
 * Arrays off a 16-byte boundary are copied into the matrix's own buffers
 * and back (same results). */
int tf_solve_device(tf_ctx ctx, tf_matrix m, int solver, int prec,
                    double* d_val, double* d_x, double* d_b, int miter,
                    int* niter, double tol, double* fin_res,
                    const double* norm);

/* Several right-hand sides with one matrix: nrhs (1..4) solves of
 * Solve_Native's kind (Jacobi or none; Bicg = Cg as in tf_solve) on the same
 * val, x and b holding nrhs vectors of n_cells doubles one after another
 * (the velocity components of Compute_Momentum.f90:153-399 when their
 * matrices are equal).  Each right-hand side runs its own recurrence --
 * niter[i], fin_res[i], x_i and b_i are those of tf_solve on (val, x_i,
 * b_i), bit for bit on row-pattern matrices (on other matrices to the
 * rounding of the dot products) -- while one SpMV per iteration reads the
 * matrix once for all of them.  val is scaled and returned once.  ICC is
 * not offered here (TF_ERR_ARG).  No reference counterpart. */
int tf_solve_multi(tf_ctx ctx, tf_matrix m, int solver, int prec, int nrhs,
                   double* val, double* x, double* b, int miter, int* niter,
                   double tol, double* fin_res, const double* norm);
int tf_solve_multi_device(tf_ctx ctx, tf_matrix m, int solver, int prec, int nrhs,
                          double* d_val, double* d_x, double* d_b, int miter,
                          int* niter, double tol, double* fin_res, const double* norm);

/* Per-iteration residual history of the last solve on ctx: hist[0] is the
 * residual before the loop, hist[k] after iteration k, for k <= niter.
 * Enabled by tf_ctx_set_history(ctx, 1) (off by default: it costs nothing
 * on the device, one extra copy on the host). */
int tf_ctx_set_history(tf_ctx ctx, int enable);
int tf_last_history(tf_ctx ctx, double* hist, int cap, int* count);

/* Watchdog of this context's solves, in seconds (0 restores the default of
 * 2 s): a streaming kernel of the solve (the SpMV and residual passes) stops
 * at its first wait for a tile's copies or a free pipeline stage after this
 * much time since its start -- or once such a wait has been blocked that
 * long -- and the solve ends with TF_ERR_TIMEOUT.  Before a stopped CTA
 * exits it still waits for the copies it started (with the default limit),
 * and the context stays usable.  The reference has no counterpart (its
 * failures stop the run, Shared/Message_Mod/Error.f90:74). */
int tf_ctx_set_wait_limit(tf_ctx ctx, double seconds);

/* Pin (page-lock) a host array the caller will pass to tf_solve on every
 * call, e.g. A % val, so its copies run at full PCIe/C2C bandwidth.
 * Wraps cudaHostRegister / cudaHostUnregister. */
int tf_host_pin(void* ptr, size_t bytes);
int tf_host_unpin(void* ptr);

/* ---------------------------------------------------------------------------
 *  Batched and served solves (C++ engine behind a C ABI).
 *
 *  No single reference counterpart: T-Flows solves its systems one at a
 *  time through Solve_Native.  A batch holds many independent systems of
 *  uneven size (Matrix_Type layout, 1-based); all of them iterate together
 *  on the device, each with its own scalars, until each reaches
 *  ||b - A x||_2 <= tol ||b||_2 (FP64) or its iteration limit.  The Krylov
 *  recurrence is Cg's (Cg.f90:139-224, which Bicg.f90 also computes) with
 *  Jacobi preconditioning (Prec_Form.f90:47-53), Krylov vectors in FP32 or
 *  FP64, FP64 reductions, and FP64 reliable updates (iterative refinement).
 * ------------------------------------------------------------------------- */
typedef struct tf_batch_opts {
  int vec_fp32;       /* 1: Krylov vectors stored in FP32; 0: FP64            */
  int val_fp32;       /* 1: the SpMV streams an FP32 copy of the values       */
  int sweep_iters;    /* iterations per captured graph launch (default 8)     */
  int max_systems;    /* system slots (default 1024)                          */
  double ru_delta;    /* refinement when |r| fell by this factor (0.1)        */
  size_t mem_budget;  /* device bytes for all systems' data (default 4 GiB)   */
  int two_phase_rows; /* SpMV consumers: 0 (default) = warp groups of 1/2/4
                         lanes per row by each tile's mean row length, no
                         barrier between warps; 1 = two phases (products
                         staged in shared memory, a barrier, then one thread
                         per row).  The same row sums bit for bit           */
} tf_batch_opts;

typedef struct tf_batch_s* tf_batch;
typedef struct tf_server_s* tf_server;

/* Status of a system in a batch / request in a server. */
enum tf_sys_status {
  TF_SYS_FREE = 0, TF_SYS_INIT = 1, TF_SYS_ACTIVE = 2, TF_SYS_CONVERGED = 3,
  TF_SYS_MAXITER = 4, TF_SYS_BREAKDOWN = 5
};

int tf_batch_create(tf_ctx ctx, const tf_batch_opts* opts, tf_batch* out);
int tf_batch_destroy(tf_batch b);
/* Copy one system in (host arrays; x0 may be NULL for zeros).  Returns
 * TF_ERR_BUSY when the memory budget or the slots are exhausted.
 * Systems with the same structure share one device copy of it (as a CFD
 * time loop solves one mesh's matrix again and again with new values): the
 * engine keeps a prepared structure (0-based CSR, renumbering, tiles) keyed
 * by the row/col/dia addresses, n, nnz and a hash of row, dia and every
 * 16th column index; its device copy stays resident after its systems
 * retire and is dropped, least recently used first, when a new system
 * needs the space.  Arrays changed in place between calls must change in
 * those hashed entries, or be passed at other addresses.  A structure whose
 * rows fit at most 64 column-offset patterns (structured hex blocks) is
 * stored as one pattern byte per row instead of its columns (the
 * environment variable TF_NO_ROW_PATTERNS keeps the columns; the same bits
 * either way).  The values are read in place until the call returns. */
int tf_batch_add(tf_batch b, int n, int64_t nnz, const int* row, const int* col,
                 const int* dia, const double* val, const double* rhs,
                 const double* x0, double tol, int maxit, int* sys);
/* Several systems at once (array i holds system i's arguments of
 * tf_batch_add; x0 may be NULL, or x0[i] NULL for zeros).  The host
 * preparation and the copies to the device run on `threads` threads (0:
 * one per hardware thread, at most 64; each copies on a stream of its own),
 * holding at most 2 x threads prepared host copies at a time; slots and
 * space are reserved in order, so sys[] and the results equal count calls
 * of tf_batch_add.  On an error the systems before the failing one stay
 * added (sys[i] >= 0), the rest get sys[i] = -1.  No reference counterpart
 * (the reference solves one system per call). */
int tf_batch_add_many(tf_batch b, int count, const int* n, const int64_t* nnz,
                      const int* const* row, const int* const* col, const int* const* dia,
                      const double* const* val, const double* const* rhs,
                      const double* const* x0, const double* tol, const int* maxit,
                      int threads, int* sys);
/* Iterate until every system has converged or stopped. */
int tf_batch_run(tf_batch b);
/* x (host, n doubles) may be NULL; true_rel_res = ||b-Ax||_2/||b||_2 in FP64;
 * n_updates counts FP64 residual evaluations (initial one included);
 * done_ms = wall time from the start of tf_batch_run to the sweep in which
 * the system finished (-1 if it has not). */
int tf_batch_result(tf_batch b, int sys, double* x, int* iters,
                    double* true_rel_res, int* status, int* n_updates,
                    double* done_ms);
int tf_batch_remove(tf_batch b, int sys);
/* Timeline of the last tf_batch_run, one record per sweep; *count = sweeps,
 * at most cap records are written. */
typedef struct tf_batch_sweep {
  int active;            /* systems iterating when the sweep was launched */
  int items;             /* work items (row tiles) in its list */
  int64_t rows, nnz;     /* rows and entries of those systems */
  double iter_bytes;     /* their inner iteration's algorithmic bytes: 12 per
                            entry (8 per entry and 1 per row with row
                            patterns), 4 per row pointer, 13 iterate vectors */
  double ms;             /* wall time, launch to the state read back */
  double kernel_ms[8];   /* TF_BATCH_PROFILE only (else 0): the sweep's time in
                            the eight kernels of tf_batch_kernel_ms */
} tf_batch_sweep;
int tf_batch_trace(tf_batch b, tf_batch_sweep* out, int cap, int* count);
/* With TF_BATCH_PROFILE set when the batch was created, sweeps run as direct
 * launches with CUDA events around every kernel: ms8 receives the time spent
 * in the eight kernels of an iteration over all runs so far, in launch
 * order: p update, SpMV (tile totals of p.q), alpha per system, x/r update
 * (tile totals of rho and |r|^2), beta per system, refinement fold,
 * refinement residual, refinement test per system.  TF_ERR_ARG when the
 * batch was not created for profiling. */
int tf_batch_kernel_ms(tf_batch b, double* ms8);
int tf_batch_info(tf_batch b, int* sweeps, int* work_items, size_t* free_bytes);
/* Where the time of tf_batch_add / tf_batch_add_many went, in milliseconds
 * over all adds so far: host preparation (conversion, checks, renumbering,
 * tiling) summed over the systems -- on worker threads for add_many, so it
 * can exceed the wall time --, the reserving thread's wait for prepared
 * systems, and admission (reservations, and the copies to the device summed
 * over the threads that make them).
 * Any pointer may be NULL. */
int tf_batch_upload_ms(tf_batch b, double* prep_ms, double* wait_ms, double* admit_ms);

/* Continuous batching: queued requests are admitted in arrival order
 * whenever the memory budget and slots allow, their copies made on a
 * stream of their own while the sweeps run; every sweep iterates all
 * admitted systems; finished systems leave at the end of their sweep and
 * their results are copied out on a third stream.  Requests arriving while
 * others run join at the next sweep after their copies land.  Submit
 * copies the system (its values and right-hand side; the structure is
 * prepared once and shared by every request with the same row/col/dia
 * arrays -- same addresses, sizes and contents, see tf_batch_add); wait
 * blocks until done and reports end-to-end and queueing latency in
 * milliseconds. */
int tf_server_create(tf_ctx ctx, const tf_batch_opts* opts, tf_server* out);
int tf_server_submit(tf_server s, int n, int64_t nnz, const int* row,
                     const int* col, const int* dia, const double* val,
                     const double* rhs, const double* x0, double tol, int maxit,
                     int64_t* req);
int tf_server_wait(tf_server s, int64_t req, double* x, int* iters,
                   double* true_rel_res, int* status, double* latency_ms,
                   double* queue_ms);
int tf_server_stats(tf_server s, long long* admitted, long long* completed,
                    int* peak_running, int* sweeps);
/* Cancel a request: a queued one is dropped at once, an admitted one is
 * retired at the end of the current sweep (its Krylov state and slot are
 * freed); tf_server_wait then returns TF_ERR_CANCELLED.  Returns TF_OK,
 * TF_ERR_BUSY when the request had already finished (its result stands),
 * or TF_ERR_ARG for an unknown or collected id.  No reference counterpart. */
int tf_server_cancel(tf_server s, int64_t req);
/* Where the server's time went, in milliseconds since it was created, by
 * thread: ms5[0] host preparation of submitted systems (summed over the
 * submitting threads; a structure already prepared for an earlier request
 * is not prepared again), ms5[1] the admission thread (reservations and
 * uploads on its own stream), ms5[2] and ms5[3] the worker thread (host
 * work: commits, building and uploading the next work list, launching the
 * next sweep behind the one in flight; waits for the sweep in flight), and
 * ms5[4] the collector thread (results copied out, retirements). */
int tf_server_timing(tf_server s, double* ms5);
int tf_server_destroy(tf_server s);

/* ---------------------------------------------------------------------------
 *  Request pool: concurrent Solve_Native calls on a pool of CUDA streams.
 *
 *  Each request is exactly one Solve_Native call (Solve_Native.f90:33-44,
 *  same arguments and results as tf_solve; x is the initial guess on entry
 *  and receives the solution; val and b are read, not modified).  The
 *  caller's arrays are used in place and must stay valid until tf_pool_wait
 *  returns.  `workers` threads each own a context (stream); a request is
 *  registered with stream-ordered allocation, solved by the FP64 drop-in
 *  and released, so independent solves overlap on the GPU.  Requests are
 *  admitted in arrival order while the device bytes in flight stay within
 *  mem_budget (0: 20 GiB); one larger than the budget fails with
 *  TF_ERR_OOM.  Submit returns at once; wait blocks
 *  until the request finished and reports end-to-end and queueing latency
 *  in milliseconds.  All pool functions are thread-safe.
 * ------------------------------------------------------------------------- */
typedef struct tf_pool_s* tf_pool;
int tf_pool_create(int device, int workers, size_t mem_budget, tf_pool* out);
int tf_pool_submit(tf_pool p, int solver, int prec, int n, int64_t nnz,
                   const int* row, const int* col, const int* dia,
                   const double* val, const double* rhs, double* x,
                   int miter, double tol, const double* norm, int64_t* req);
int tf_pool_wait(tf_pool p, int64_t req, int* niter, double* fin_res,
                 double* latency_ms, double* queue_ms);
int tf_pool_stats(tf_pool p, long long* submitted, long long* completed,
                  long long* rejected, size_t* peak_bytes);
/* Cancel a request not yet taken by a worker (tf_pool_wait then returns
 * TF_ERR_CANCELLED and x is left untouched).  A request already running
 * is one Solve_Native graph on the device and runs to its end: TF_ERR_BUSY,
 * as for a finished one.  TF_ERR_ARG for an unknown or collected id.  No
 * reference counterpart. */
int tf_pool_cancel(tf_pool p, int64_t req);
/* Resident structures: requests reusing a held registration (`reused`),
 * registrations currently held and their budgeted bytes.  A request whose
 * row/col/dia arrays (same addresses, same sampled contents, same sizes)
 * were registered by an earlier request runs on that registration when the
 * worker holding it takes it.  No reference counterpart. */
int tf_pool_resident(tf_pool p, long long* reused, int* held, size_t* held_bytes);
int tf_pool_destroy(tf_pool p);

/* ---------------------------------------------------------------------------
 *  Building blocks exposed for testing and for callers that keep their own
 *  Krylov loop.  All pointers are device pointers; vectors have n_cells
 *  entries; val has nnz entries.  Each call is asynchronous on ctx's stream;
 *  tf_ctx_sync waits for it.
 * ------------------------------------------------------------------------- */
/* Device-side assembly through Matrix_Type's pos map (no counterpart in the
 * C ABI of the reference: replaces the host face loops that fill A % val).
 *
 * tf_faces_register: the face topology of a registered matrix, once:
 *   faces_c[2*s], faces_c[2*s+1] = c1, c2 of face s (1-based; c2 <= 0 on a
 *   boundary face, Grid % faces_c), pos[2*s], pos[2*s+1] = the 1-based
 *   entries of (c1, c2) and (c2, c1) (Create_Matrix.f90:124-139).
 * tf_assemble_pressure: d_val (device, nnz) = the pressure-correction
 *   matrix of Rhie_And_Chow.f90:183-205 (a12 = fc (fs v_m(c1) + (1 - fs)
 *   v_m(c2)); off-diagonals -a12, diagonals sum a12 in face order) plus
 *   Compute_Pressure.f90:140-160's boundary faces flagged in d_bnd_open
 *   (fc v_m(c1) added to the diagonal; may be NULL).  d_fc, d_fw per face,
 *   d_vm per cell (NULL: 1).
 * tf_assemble_momentum: d_val = the upwind-blended momentum matrix of
 *   Compute_Momentum.f90:270-297 (m0 = vis fc, m12 = m0 - min(F,0) rho,
 *   m21 = m0 + max(F,0) rho; wall faces flagged in d_bnd_wall add m12 to
 *   the diagonal) plus Inertial_Term.f90's rho vol / dt.
 * Both zero d_val first and give the reference's face loops' values bit for
 * bit; they run on the context's stream (d_val is then ready for
 * tf_solve_device on the same stream). */
int tf_faces_register(tf_ctx ctx, tf_matrix m, int n_faces, const int* faces_c, const int* pos);
int tf_assemble_pressure(tf_ctx ctx, tf_matrix m, const double* d_fc, const double* d_fw,
                         const double* d_vm, const int* d_bnd_open, double* d_val);
int tf_assemble_momentum(tf_ctx ctx, tf_matrix m, const double* d_fc, const double* d_flux,
                         const int* d_bnd_wall, double vis, double rho, const double* d_vol,
                         double dt, double* d_val);

/* q = A p over rows 1..n_own, in the row order and summation order of
 * Cg.f90:177-185.  If pq != NULL, *pq (device) receives sum_i p_i q_i. */
int tf_spmv(tf_ctx ctx, tf_matrix m, const double* d_val, const double* d_p,
            double* d_q, double* d_pq);
/* r = b - A x (Residual_Vector.f90:34-42). */
int tf_residual(tf_ctx ctx, tf_matrix m, const double* d_val,
                const double* d_b, const double* d_x, double* d_r);
/* Normalized_Root_Mean_Square.f90:33-63 of r, on device; result to *d_out. */
int tf_nrms(tf_ctx ctx, tf_matrix m, const double* d_val, const double* d_r,
            const double* d_x, const double* norm, double* d_out);
int tf_ctx_sync(tf_ctx ctx);

/* Vector kernels for callers that run their own Krylov loop around tf_spmv,
 * e.g. one system split by rows over several GPUs (the reference's MPI
 * sub-domains: Cg.f90 with Exchange_Cells_Real before each SpMV and the
 * Global % Sum_Real of every dot product), where the caller exchanges the
 * buffer cells and sums the partial results over processes between these
 * calls.  Device pointers, n entries, asynchronous on ctx's stream; every
 * expression is rounded as the reference's loop rounds it, and every sum is
 * deterministic (fixed grid, partials combined in block order), written to
 * device memory (d_out).
 *   tf_vec_axpby:  y = a x + b y (first != 0: y = a x; a == 0: y = b y) --
 *                  p = z + beta p, x + alfa p, r - alfa q (Cg.f90:166-209);
 *   tf_vec_gather / tf_vec_scatter: out[k] = src[idx[k]] / dst[idx[k]] =
 *                  vals[k] (packing and unpacking buffer cells);
 *   tf_vec_recip:  out = 1 / x (Prec_Form.f90:51);
 *   tf_vec_dot:    d_out[0] = sum a_i b_i (b NULL: sum a_i);
 *   tf_vec_nrms_sum: d_out[0] = sum r_i^2 / d_i^2
 *                  (Normalized_Root_Mean_Square.f90:33-36, before the sum
 *                  over processes, the root and the scaling);
 *   tf_vec_jacobi: z = r d_inv and d_out[0] = sum z_i r_i (Prec_Solve.f90:
 *                  44-49, Cg.f90:151-155);
 *   tf_vec_minmax: d_out[0], d_out[1] = min and max of x
 *                  (Normalized_Root_Mean_Square.f90:42-48). */
int tf_vec_axpby(tf_ctx ctx, int n, double a, const double* d_x, double b, double* d_y,
                 int first);
int tf_vec_gather(tf_ctx ctx, int n, const double* d_src, const int64_t* d_idx, double* d_out);
int tf_vec_scatter(tf_ctx ctx, int n, double* d_dst, const int64_t* d_idx,
                   const double* d_vals);
int tf_vec_recip(tf_ctx ctx, int n, const double* d_x, double* d_out);
int tf_vec_dot(tf_ctx ctx, int n, const double* d_a, const double* d_b, double* d_out);
int tf_vec_nrms_sum(tf_ctx ctx, int n, const double* d_r, const double* d_diag, double* d_out);
int tf_vec_jacobi(tf_ctx ctx, int n, const double* d_r, const double* d_dinv, double* d_z,
                  double* d_out);
int tf_vec_minmax(tf_ctx ctx, int n, const double* d_x, double* d_out2);
/* The CUDA stream of ctx (a cudaStream_t), for callers that order their
 * own work with it. */
void* tf_ctx_stream(tf_ctx ctx);

/* ---------------------------------------------------------------------------
 *  q = A p and p.q for callers that cannot allocate device memory.
 *  No counterpart in the reference: T-Flows has no device code of its own.
 *
 *  Meant for code whose device memory belongs to someone else -- an OpenACC
 *  data region (T-Flows' GPU layer), a caching or pooled allocator, a
 *  process held to a fixed device-memory budget -- or that cannot pay for
 *  the device synchronisation cudaFree brings.  Nothing is allocated: no
 *  context, no registration, no cudaMalloc/cudaFree.  All arguments are
 *  device pointers the caller owns: row (n+1) and col (nnz) are 1-based as
 *  Matrix_Type stores them, val (nnz), p and q (n), and *d_pq receives
 *  sum_i p_i q_i.  q's rows are summed in storage order, as tf_spmv does.
 *
 *  The kernel's only scratch, one partial sum per 256-row tile and a
 *  counter, is a fixed 512 KiB array inside the library that every GPU which
 *  loads the library keeps until exit.  It bounds n to
 *  TF_SPMV_NOALLOC_MAX_ROWS; larger n returns TF_ERR_ARG (the reason is in
 *  tf_last_error_message).  The first call on a device looks up the array's
 *  device address (cudaGetSymbolAddress, with that device current) and keeps
 *  it for the life of the process; make that first call before any stream
 *  capture.  A cudaDeviceReset of a device the entry point was used on is
 *  not supported (the kept address would be stale): do not call it on that
 *  device afterwards.  Work is queued on `stream`
 *  (a cudaStream_t, NULL = legacy default stream) and the call returns
 *  without waiting.  Every call shares the one array: calls that can
 *  overlap on the GPU (different streams, or different host threads on one
 *  device) race and must be serialised by the caller.
 * ------------------------------------------------------------------------- */
#define TF_SPMV_NOALLOC_MAX_ROWS 16777216
int tf_spmv_noalloc(int n, const int* d_row, const int* d_col,
                    const double* d_val, const double* d_p, double* d_q,
                    double* d_pq, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* TF_KRYLOV_H */

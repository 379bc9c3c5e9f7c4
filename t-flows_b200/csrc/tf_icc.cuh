// tf_icc.cuh -- incomplete-Cholesky preconditioning by level scheduling.
//
// Prec_Form.f90:68-78 and Prec_Solve.f90:64-92 are sequential recurrences
// over rows.  Row i depends only on its lower neighbours k < i (forward
// sweep, and the d(k) of Prec_Form) or on its upper neighbours k > i
// (backward sweep).  Rows are grouped into levels such that every
// dependency of a row lies in an earlier level; one kernel per level then
// computes all of its rows in parallel, each row with exactly the
// reference's arithmetic in exactly its order, so d, d_inv and z are the
// reference's bits given the same inputs.  Requires the diagonal-first,
// ascending-column layout Create_Matrix produces (the reference's ICC
// relies on it too, Prec_Form.f90:55-66).
#pragma once
#include "../../include/tf_krylov.h"
#include "tf_common.cuh"

namespace tf {

struct IccArgs {
  const int* row;      // 0-based CSR
  const int* col;
  const double* val;   // scaled matrix
  const int* rows;     // rows of this level
  int count;           // rows in this level
  int ni;
  double* d;           // Prec_Form's d (1/pivot)
  double* d_inv;       // Prec_Form's d_inv (pivot)
  const double* r;     // right-hand side of the solve (r1)
  double* y;           // forward-sweep values
  double* z;           // result
  const SolveState* st;
};

// Prec_Form.f90:69-78 for the rows of one level.
__global__ void __launch_bounds__(256) k_icc_form_level(IccArgs a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.count) return;
  const int i = a.rows[t];
  const int js = a.row[i], je = a.row[i + 1];
  double sum = a.val[js];                       // diagonal entry (first)
  for (int j = js + 1; j < je; ++j) {
    const int k = a.col[j];
    if (k > i) break;
    const double v = a.val[j];
    sum = __dsub_rn(sum, __dmul_rn(__dmul_rn(a.d[k], v), v));
  }
  a.d_inv[i] = sum;
  a.d[i] = __ddiv_rn(1.0, sum);
}

// Forward substitution (Prec_Solve.f90:67-75) for one level; also applies
// the diagonal scaling of :77-81 into z, keeping the unscaled y for the
// rows of later levels.
__global__ void __launch_bounds__(256) k_icc_fwd_level(IccArgs a) {
  if (a.st && a.st->done) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.count) return;
  const int i = a.rows[t];
  const int js = a.row[i], je = a.row[i + 1];
  double sum = a.r[i];
  for (int j = js + 1; j < je; ++j) {
    const int k = a.col[j];
    if (k > i) break;
    sum = __dsub_rn(sum, __dmul_rn(a.val[j], a.y[k]));
  }
  const double yi = __dmul_rn(sum, a.d[i]);
  a.y[i] = yi;
  a.z[i] = __dmul_rn(yi, a.d_inv[i]);
}

// Backward substitution (Prec_Solve.f90:84-92) for one level.
__global__ void __launch_bounds__(256) k_icc_bwd_level(IccArgs a) {
  if (a.st && a.st->done) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.count) return;
  const int i = a.rows[t];
  const int js = a.row[i], je = a.row[i + 1];
  double sum = a.z[i];
  for (int j = je - 1; j >= js + 1; --j) {
    const int k = a.col[j];
    if (k < i) break;
    if (k < a.ni) sum = __dsub_rn(sum, __dmul_rn(a.val[j], a.z[k]));
  }
  a.z[i] = __dmul_rn(sum, a.d[i]);
}

// ---------------------------------------------------------------------------
// The same three recurrences as single persistent kernels, level by level:
// one kernel per sweep instead of one per level.  Every thread of the grid
// takes rows t, t + T, ... of the current level (T threads in all), then
// all CTAs meet at a grid barrier before the next level, so the rows of a
// level read only values written before the barrier (read from L2, since
// other SMs wrote them).  The arithmetic of every row is the per-level
// kernels' (and so the reference's) in the same order: the same bits.
// The barrier needs every CTA resident: the kernel is launched
// cooperatively with no more CTAs than fit at once.  It is a counter and a
// generation word in the solve state; its waits are bounded by the solve's
// deadline, and a timeout is recorded in the solve status (the other CTAs
// then time out at the next barrier too).
// ---------------------------------------------------------------------------
enum IccSweepKind { kSweepForm = 0, kSweepFwd = 1, kSweepBwd = 2 };

struct IccSweepArgs {
  IccArgs a;             // arrays; a.rows = rows in this sweep's level order
  const int* lev_ptr;    // level l is a.rows[lev_ptr[l] .. lev_ptr[l+1])
  int nlev;
  SolveState* st;        // solve state (barrier, status); never null here
  const SolveParams* prm;
};

// Grid barrier: every CTA's thread 0 arrives on bar_count; the last one
// resets it and advances bar_gen, which the others wait for.  Writes before the barrier are visible after it (fences at
// GPU scope around the arrival).  Returns false, CTA-uniformly, on timeout.
__device__ __forceinline__ bool icc_grid_barrier(SolveState* st, unsigned long long deadline) {
  __syncthreads();
  int ok = 1;
  if (threadIdx.x == 0) {
    const unsigned g = ld_acquire_gpu(&st->bar_gen);
    __threadfence();
    if (atomicAdd(&st->bar_count, 1u) == gridDim.x - 1) {
      st->bar_count = 0u;
      __threadfence();
      st_release_gpu(&st->bar_gen, g + 1u);
    } else {
      // One poller per CTA, polling at full rate: a sleep's wake-up
      // granularity would add to every level of the sweep.
      while (ld_acquire_gpu(&st->bar_gen) == g) {
        if (globaltimer_ns() > deadline) {
          ok = 0;
          break;
        }
      }
    }
  }
  return __syncthreads_and(ok) != 0;
}

template <int KIND>
__device__ __forceinline__ void icc_sweep_row(const IccArgs& a, int i) {
  const int js = a.row[i], je = a.row[i + 1];
  if (KIND == kSweepForm) {             // Prec_Form.f90:69-78
    double sum = a.val[js];
    for (int j = js + 1; j < je; ++j) {
      const int k = a.col[j];
      if (k > i) break;
      const double v = a.val[j];
      sum = __dsub_rn(sum, __dmul_rn(__dmul_rn(__ldcg(a.d + k), v), v));
    }
    a.d_inv[i] = sum;
    a.d[i] = __ddiv_rn(1.0, sum);
  } else if (KIND == kSweepFwd) {       // Prec_Solve.f90:67-81
    double sum = a.r[i];
    for (int j = js + 1; j < je; ++j) {
      const int k = a.col[j];
      if (k > i) break;
      sum = __dsub_rn(sum, __dmul_rn(a.val[j], __ldcg(a.y + k)));
    }
    const double yi = __dmul_rn(sum, a.d[i]);
    a.y[i] = yi;
    a.z[i] = __dmul_rn(yi, a.d_inv[i]);
  } else {                              // Prec_Solve.f90:84-92
    double sum = __ldcg(a.z + i);
    for (int j = je - 1; j >= js + 1; --j) {
      const int k = a.col[j];
      if (k < i) break;
      if (k < a.ni) sum = __dsub_rn(sum, __dmul_rn(a.val[j], __ldcg(a.z + k)));
    }
    a.z[i] = __dmul_rn(sum, a.d[i]);
  }
}

template <int KIND>
__global__ void __launch_bounds__(256) k_icc_sweep(IccSweepArgs s) {
  SolveState* st = s.st;
  if (KIND != kSweepForm && st->done) return;   // the same for every CTA
  const unsigned long long deadline = deadline_after(wait_limit(s.prm));
  const int T = (int)(gridDim.x * blockDim.x);
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  // The next level's first row of this thread is looked up before the
  // barrier, so after it only the neighbours' values are waited for.
  int b = __ldg(s.lev_ptr), e = __ldg(s.lev_ptr + 1);
  int i0 = (b + t < e) ? __ldg(s.a.rows + b + t) : -1;
  for (int l = 0; l < s.nlev; ++l) {
    if (i0 >= 0) icc_sweep_row<KIND>(s.a, i0);
    for (int q = b + t + T; q < e; q += T) icc_sweep_row<KIND>(s.a, __ldg(s.a.rows + q));
    if (l + 1 < s.nlev) {
      b = __ldg(s.lev_ptr + l + 1);
      e = __ldg(s.lev_ptr + l + 2);
      i0 = (b + t < e) ? __ldg(s.a.rows + b + t) : -1;
      if (!icc_grid_barrier(st, deadline)) {
        if (threadIdx.x == 0) atomicExch(&st->status, (int)TF_ERR_TIMEOUT);
        return;
      }
    }
  }
}

// rho = z.r (Cg.f90:150-156) after an ICC solve.  At iteration 1 it is the
// first rho; later it shifts rho into rho_old first (Cg.f90:222).
__global__ void __launch_bounds__(256) k_icc_rho(int ni, const double* z, const double* r,
                                                 double* part, SolveState* st) {
  __shared__ double scratch[32];
  if (st->done) return;
  double s = 0.0;
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ni; i += stride)
    s = __dadd_rn(s, __dmul_rn(z[i], r[i]));
  double v[1] = {block_red<kSum>(s, scratch)};
  const int ops[1] = {kSum};
  if (grid_reduce_last<1>(v, ops, part, &st->counter[kCntZ], scratch) && threadIdx.x == 0) {
    if (st->iter > 1) st->rho_old = st->rho;
    st->rho = v[0];
  }
}

}  // namespace tf

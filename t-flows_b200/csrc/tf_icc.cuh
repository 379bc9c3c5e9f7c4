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
// The same three recurrences as single persistent kernels.  One kernel
// per sweep instead of one per level: its warps walk units of at most 32
// rows of one level, in level order (warp w takes units w, w + W, ...).
// Before reading a row k's value a lane waits until flag[k] holds this
// sweep's epoch; after writing row i's value it publishes flag[i] = epoch
// with release semantics, and readers acquire it, reading the value from
// L2.  The arithmetic of every row is the per-level kernels' (and so the
// reference's) in the same order, so the bits are the same.  A unit waits
// only on rows of earlier levels, i.e. of earlier units, and every warp
// walks its units in order, so the lowest unfinished unit can always
// proceed -- provided every CTA is resident: the kernel is launched
// cooperatively, with no more CTAs than fit at once.  Waits are bounded by
// the solve's deadline (a timeout is recorded in the solve status).  The
// kernel's last CTA advances the epoch for the next sweep.
// ---------------------------------------------------------------------------
enum IccSweepKind { kSweepForm = 0, kSweepFwd = 1, kSweepBwd = 2 };

struct IccSweepArgs {
  IccArgs a;             // arrays; a.rows = rows in this sweep's level order
  const int2* units;     // (first index into rows, count <= 32), level order
  int nunits;
  unsigned* flag;        // per row: epoch of the last sweep that computed it
  SolveState* st;        // solve state (epoch, status); never null here
  const SolveParams* prm;
};

__device__ __forceinline__ bool icc_wait(const unsigned* f, unsigned epoch,
                                         unsigned long long deadline) {
  while ((int)(epoch - ld_acquire_gpu(f)) > 0)
    if (globaltimer_ns() > deadline) return false;
  return true;
}

template <int KIND>
__global__ void __launch_bounds__(256) k_icc_sweep(IccSweepArgs s) {
  SolveState* st = s.st;
  if (KIND != kSweepForm && st->done) return;
  const IccArgs& a = s.a;
  const unsigned epoch = st->icc_epoch + 1u;
  const unsigned long long deadline = deadline_after(wait_limit(s.prm));
  const int lane = threadIdx.x & 31;
  const int nw = (int)((gridDim.x * blockDim.x) >> 5);
  bool ok = true;
  for (int u = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); u < s.nunits; u += nw) {
    const int2 un = s.units[u];
    if (lane < un.y && ok) {
      const int i = a.rows[un.x + lane];
      const int js = a.row[i], je = a.row[i + 1];
      if (KIND == kSweepForm) {           // Prec_Form.f90:69-78
        double sum = a.val[js];
        for (int j = js + 1; j < je; ++j) {
          const int k = a.col[j];
          if (k > i) break;
          if (!icc_wait(s.flag + k, epoch, deadline)) { ok = false; break; }
          const double v = a.val[j];
          sum = __dsub_rn(sum, __dmul_rn(__dmul_rn(__ldcg(a.d + k), v), v));
        }
        a.d_inv[i] = sum;
        a.d[i] = __ddiv_rn(1.0, sum);
      } else if (KIND == kSweepFwd) {     // Prec_Solve.f90:67-81
        double sum = a.r[i];
        for (int j = js + 1; j < je; ++j) {
          const int k = a.col[j];
          if (k > i) break;
          if (!icc_wait(s.flag + k, epoch, deadline)) { ok = false; break; }
          sum = __dsub_rn(sum, __dmul_rn(a.val[j], __ldcg(a.y + k)));
        }
        const double yi = __dmul_rn(sum, a.d[i]);
        a.y[i] = yi;
        a.z[i] = __dmul_rn(yi, a.d_inv[i]);
      } else {                            // Prec_Solve.f90:84-92
        double sum = __ldcg(a.z + i);
        for (int j = je - 1; j >= js + 1; --j) {
          const int k = a.col[j];
          if (k < i) break;
          if (k < a.ni) {
            if (!icc_wait(s.flag + k, epoch, deadline)) { ok = false; break; }
            sum = __dsub_rn(sum, __dmul_rn(a.val[j], __ldcg(a.z + k)));
          }
        }
        a.z[i] = __dmul_rn(sum, a.d[i]);
      }
      st_release_gpu(s.flag + i, epoch);
    }
  }
  if (!ok) atomicExch(&st->status, (int)TF_ERR_TIMEOUT);
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&st->counter[kCntSweep], 1u) == gridDim.x - 1) {
      st->counter[kCntSweep] = 0u;
      st->icc_epoch = epoch;
      __threadfence();
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

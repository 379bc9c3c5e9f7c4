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

// tf_icc.cu -- incomplete-Cholesky preconditioned solves (placeholder until
// the level-scheduled triangular sweeps land).
#include "tf_internal.h"

int tf_icc_build(tf_matrix_s*, const int*, const int*) { return TF_ERR_ARG; }
int tf_icc_run_solve(tf_matrix_s*) { return TF_ERR_ARG; }

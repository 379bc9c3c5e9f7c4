// tf_icc.cu -- host side of the level-scheduled incomplete Cholesky:
// level sets of the forward and backward sweeps, computed once per matrix
// from its structure.
#include <algorithm>
#include <vector>

#include "tf_internal.h"

namespace {

// Counting sort of rows by level: rows[ptr[l] .. ptr[l+1]) are level l.
void bucket(const std::vector<int>& lev, int nlev, std::vector<int>& ptr,
            std::vector<int>& rows) {
  ptr.assign(nlev + 1, 0);
  for (int v : lev) ptr[v + 1]++;
  for (int l = 0; l < nlev; ++l) ptr[l + 1] += ptr[l];
  rows.resize(lev.size());
  std::vector<int> fill(ptr.begin(), ptr.end() - 1);
  for (int i = 0; i < (int)lev.size(); ++i) rows[fill[lev[i]]++] = i;
}

}  // namespace

// Levels of the sweeps in Prec_Form.f90:69-78 / Prec_Solve.f90:67-92.
// Forward: row i waits for the lower entries visited by `do j = a_row(i)+1,
// ...; if(k > i) exit`; backward: for the upper entries visited from the
// row's end down to `if(k < i) exit`, owned rows only (k <= ni).
int tf_icc_build(tf_matrix_s* m, const int* row0, const int* col0) {
  const int ni = m->ni;
  std::vector<int> levf(ni, 0), levb(ni, 0);
  int nf = 0, nb = 0;
  for (int i = 0; i < ni; ++i) {
    int l = 0;
    for (int j = row0[i] + 1; j < row0[i + 1]; ++j) {
      const int k = col0[j];
      if (k > i) break;
      l = std::max(l, levf[k] + 1);
    }
    levf[i] = l;
    nf = std::max(nf, l + 1);
  }
  for (int i = ni - 1; i >= 0; --i) {
    int l = 0;
    for (int j = row0[i + 1] - 1; j >= row0[i] + 1; --j) {
      const int k = col0[j];
      if (k < i) break;
      if (k < ni) l = std::max(l, levb[k] + 1);
    }
    levb[i] = l;
    nb = std::max(nb, l + 1);
  }
  std::vector<int> rf, rb;
  bucket(levf, nf, m->h_levf_ptr, rf);
  bucket(levb, nb, m->h_levb_ptr, rb);
  const size_t nv = (size_t)m->nt + 8;
  void* p = nullptr;
  int st = tf_dev_alloc_bytes(m->ctx, &p, std::max<size_t>(rf.size(), 1) * sizeof(int));
  m->d_levf_rows = (int*)p;
  if (st == TF_OK) st = tf_dev_alloc_bytes(m->ctx, &p, std::max<size_t>(rb.size(), 1) * sizeof(int));
  m->d_levb_rows = (int*)p;
  if (st == TF_OK) st = tf_dev_alloc_bytes(m->ctx, &p, nv * sizeof(double));
  m->d_z = (double*)p;
  if (st == TF_OK) st = tf_dev_alloc_bytes(m->ctx, &p, nv * sizeof(double));
  m->d_icc_d = (double*)p;
  if (st == TF_OK) st = tf_dev_alloc_bytes(m->ctx, &p, nv * sizeof(double));
  m->d_icc_dinv = (double*)p;
  if (st != TF_OK) return st;
  // Level pointers of the persistent sweeps.
  void* q = nullptr;
  st = tf_dev_alloc_bytes(m->ctx, &q, m->h_levf_ptr.size() * sizeof(int));
  if (st != TF_OK) return st;
  m->d_icc_levf_ptr = (int*)q;
  st = tf_dev_alloc_bytes(m->ctx, &q, m->h_levb_ptr.size() * sizeof(int));
  if (st != TF_OK) return st;
  m->d_icc_levb_ptr = (int*)q;
  // From pageable memory these return once the source has been staged.
  TF_CUDA_TRY(cudaMemcpyAsync(m->d_levf_rows, rf.data(), rf.size() * sizeof(int),
                              cudaMemcpyHostToDevice, m->ctx->stream));
  TF_CUDA_TRY(cudaMemcpyAsync(m->d_levb_rows, rb.data(), rb.size() * sizeof(int),
                              cudaMemcpyHostToDevice, m->ctx->stream));
  TF_CUDA_TRY(cudaMemcpyAsync(m->d_icc_levf_ptr, m->h_levf_ptr.data(),
                              m->h_levf_ptr.size() * sizeof(int), cudaMemcpyHostToDevice,
                              m->ctx->stream));
  TF_CUDA_TRY(cudaMemcpyAsync(m->d_icc_levb_ptr, m->h_levb_ptr.data(),
                              m->h_levb_ptr.size() * sizeof(int), cudaMemcpyHostToDevice,
                              m->ctx->stream));
  if (!m->ctx->async_alloc) TF_CUDA_TRY(cudaStreamSynchronize(m->ctx->stream));
  m->icc_ready = 1;
  return tf_icc_prepare_sweeps(m);
}

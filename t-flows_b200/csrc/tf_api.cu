// tf_api.cu -- the C ABI (include/tf_krylov.h): contexts, matrix
// registration, the Solve_Native drop-in and the building blocks.
#include <cuda_runtime.h>
#include <limits.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "tf_internal.h"
#include "tf_tile.cuh"

namespace {
std::mutex g_err_mu;
std::string g_last_err;
}  // namespace

void tf_set_last_cuda_error(cudaError_t e, const char* what, const char* file,
                            int line) {
  std::lock_guard<std::mutex> lk(g_err_mu);
  char buf[512];
  snprintf(buf, sizeof buf, "%s failed: %s (%s:%d)", what, cudaGetErrorString(e),
           file, line);
  g_last_err = buf;
}

void tf_set_last_message(const char* msg) {
  std::lock_guard<std::mutex> lk(g_err_mu);
  g_last_err = msg;
}

extern "C" const char* tf_last_error_message(void) {
  std::lock_guard<std::mutex> lk(g_err_mu);
  return g_last_err.c_str();
}

extern "C" const char* tf_status_string(int status) {
  switch (status) {
    case TF_OK: return "ok";
    case TF_ERR_CUDA: return "CUDA runtime error";
    case TF_ERR_OOM: return "out of memory";
    case TF_ERR_ARG: return "invalid argument";
    case TF_ERR_TIMEOUT: return "bounded device wait timed out";
    case TF_ERR_LAYOUT: return "CSR layout violates Matrix_Type contract";
    case TF_ERR_NO_DEVICE: return "no CUDA device";
    case TF_ERR_BUSY: return "busy";
    case TF_ERR_CANCELLED: return "cancelled";
    case TF_ERR_HOST: return "host-side failure";
    case TF_ERR_UNKNOWN_SOLVER: return "unknown native solver";
    case TF_ERR_UNKNOWN_PREC: return "unknown preconditioner";
    default: return "unknown status";
  }
}

extern "C" const char* tf_version(void) { return "tfkrylov 0.1 sm_100a"; }

// ---------------------------------------------------------------------------
// Contexts
// ---------------------------------------------------------------------------
extern "C" int tf_ctx_create(int device, tf_ctx* out) {
  TF_API_BEGIN
  if (!out) return TF_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return TF_ERR_NO_DEVICE;
  }
  if (device < 0) TF_CUDA_TRY(cudaGetDevice(&device));
  if (device >= ndev) return TF_ERR_ARG;
  TF_CUDA_TRY(cudaSetDevice(device));
  tf_ctx_s* c = new tf_ctx_s();
  c->device = device;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) {
    c->sm_count = prop.multiProcessorCount;
    c->l2_bytes = prop.l2CacheSize;
  }
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    TF_CUDA_TRY(e);
  }
  *out = c;
  return TF_OK;
  TF_API_END
}

extern "C" int tf_ctx_destroy(tf_ctx ctx) {
  TF_API_BEGIN
  if (!ctx) return TF_ERR_ARG;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  if (ctx->d_vec_scratch) {
    if (ctx->async_alloc) cudaFreeAsync(ctx->d_vec_scratch, ctx->stream);
    else cudaFree(ctx->d_vec_scratch);
    cudaStreamSynchronize(ctx->stream);
  }
  cudaStreamDestroy(ctx->stream);
  delete ctx;
  return TF_OK;
  TF_API_END
}

extern "C" int tf_ctx_sync(tf_ctx ctx) {
  TF_API_BEGIN
  if (!ctx) return TF_ERR_ARG;
  TF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return TF_OK;
  TF_API_END
}

extern "C" void* tf_ctx_stream(tf_ctx ctx) { return ctx ? (void*)ctx->stream : nullptr; }

extern "C" int tf_ctx_set_history(tf_ctx ctx, int enable) {
  TF_API_BEGIN
  if (!ctx) return TF_ERR_ARG;
  ctx->history = enable ? 1 : 0;
  return TF_OK;
  TF_API_END
}

extern "C" int tf_ctx_set_wait_limit(tf_ctx ctx, double seconds) {
  TF_API_BEGIN
  if (!ctx || !(seconds >= 0.0) || seconds > 3600.0) return TF_ERR_ARG;
  ctx->wait_ns = (unsigned long long)(seconds * 1e9);
  if (seconds > 0.0 && ctx->wait_ns == 0) ctx->wait_ns = 1;
  return TF_OK;
  TF_API_END
}

extern "C" int tf_last_history(tf_ctx ctx, double* hist, int cap, int* count) {
  TF_API_BEGIN
  if (!ctx || !count || (cap > 0 && !hist)) return TF_ERR_ARG;
  const int n = std::min(cap, ctx->last_count);
  for (int i = 0; i < n; ++i) hist[i] = ctx->last_hist[i];
  *count = ctx->last_count;
  return TF_OK;
  TF_API_END
}

extern "C" int tf_host_pin(void* ptr, size_t bytes) {
  TF_API_BEGIN
  if (!ptr || bytes == 0) return TF_ERR_ARG;
  TF_CUDA_TRY(cudaHostRegister(ptr, bytes, cudaHostRegisterDefault));
  return TF_OK;
  TF_API_END
}

extern "C" int tf_host_unpin(void* ptr) {
  TF_API_BEGIN
  if (!ptr) return TF_ERR_ARG;
  TF_CUDA_TRY(cudaHostUnregister(ptr));
  return TF_OK;
  TF_API_END
}

// ---------------------------------------------------------------------------
// Matrices
// ---------------------------------------------------------------------------
namespace {

template <class T>
int dev_alloc(tf_ctx_s* ctx, T** p, size_t count) {
  void* v = nullptr;
  const int st = tf_dev_alloc_bytes(ctx, &v, std::max<size_t>(count, 1) * sizeof(T));
  *p = static_cast<T*>(v);
  return st;
}

}  // namespace

// Zeroed device memory; stream-ordered on the context's stream when the
// context asks for it (no device-wide synchronisation).
int tf_dev_alloc_bytes(tf_ctx_s* ctx, void** p, size_t bytes) {
  *p = nullptr;
  if (ctx->async_alloc) {
    TF_CUDA_TRY(cudaMallocAsync(p, bytes, ctx->stream));
    TF_CUDA_TRY(cudaMemsetAsync(*p, 0, bytes, ctx->stream));
  } else {
    TF_CUDA_TRY(cudaMalloc(p, bytes));
    TF_CUDA_TRY(cudaMemset(*p, 0, bytes));
  }
  return TF_OK;
}

void tf_matrix_free(tf_matrix_s* m) {
  if (!m) return;
  cudaSetDevice(m->ctx->device);
  tf_matrix_free(m->ren);
  for (auto& g : m->graph)
    if (g) cudaGraphExecDestroy(g);
  for (auto& g : m->ext_graph)
    if (g) cudaGraphExecDestroy(g);
  tf_slices_free(m);
  void* ptrs[] = {m->d_row, m->d_col, m->d_dia, m->d_tiles, m->d_val, m->d_x, m->d_b,
                  m->d_r, m->d_p, m->d_q, m->d_z, m->d_adiag, m->d_part,
                  m->d_hist, m->d_state, m->d_params, m->d_levf_rows, m->d_levb_rows,
                  m->d_icc_d, m->d_icc_dinv, m->d_icc_levf_ptr, m->d_icc_levb_ptr,
                  m->d_pat, m->d_pat_tab, m->d_perm, m->d_src,
                  m->d_face_cell, m->d_face_pos, m->d_cf_ptr, m->d_cf};
  for (void* p : ptrs)
    if (p) {
      if (m->async_alloc) cudaFreeAsync(p, m->ctx->stream);
      else cudaFree(p);
    }
  if (!m->host_lent) {
    if (m->h_state) cudaFreeHost(m->h_state);
    if (m->h_params) cudaFreeHost(m->h_params);
  }
  delete m;
}

size_t tf_matrix_bytes_for(int n_cells, int64_t nnz, const int* row, const int* col) {
  size_t b = tf_matrix_bytes(n_cells, nnz);
  if (n_cells >= kRenumberMinRows && row && col && !getenv("TF_NO_RENUMBER") &&
      tf_gather_lines_per_warp(row, col, n_cells, 1) > kRenumberLines)
    b += tf_matrix_bytes(n_cells, nnz) + 4 * ((size_t)n_cells + (size_t)nnz) + 1024;
  return b;
}

size_t tf_matrix_bytes(int n_cells, int64_t nnz) {
  auto up = [](size_t b) { return (b + 511) & ~size_t(511); };
  const size_t nv = (size_t)n_cells + 8, nz = (size_t)nnz + 8;
  return up(((size_t)n_cells + 9) * 4) + up(nz * 4) + up(nv * 4) + up(nz * 8) +
         6 * up(nv * 8) + up(((size_t)8 * tf::kMaxBlocks + 16) * 8) + up((size_t)n_cells + 32) +
         up((size_t)tf::kPatMax * (tf::kPatMaxLen + 1) * 4) + 2048;
}

// Row patterns of the first ni rows: pat[i] names the offset sequence
// (col_j - i over the row's entries, in storage order).  Returns the number
// of patterns, or 0 when there are more than kPatMax of them or a row is
// longer than kPatMaxLen (then the CSR columns are used).
int tf_find_row_patterns(const std::vector<int>& row0, const std::vector<int>& col0, int ni,
                         std::vector<unsigned char>& pat, std::vector<int>& tab) {
  using tf::kPatMax;
  using tf::kPatMaxLen;
  std::vector<int> offs((size_t)kPatMax * kPatMaxLen, 0), lens;
  std::vector<uint64_t> keys;
  pat.assign((size_t)ni + 32, 0);
  int last = -1;
  for (int i = 0; i < ni; ++i) {
    const int js = row0[i], len = row0[i + 1] - js;
    if (len > kPatMaxLen) return 0;
    uint64_t h = 1469598103934665603ull ^ (uint64_t)len;
    for (int k = 0; k < len; ++k)
      h = (h ^ (uint64_t)(uint32_t)(col0[js + k] - i)) * 1099511628211ull;
    auto same = [&](int p) {
      if (keys[p] != h || lens[p] != len) return false;
      for (int k = 0; k < len; ++k)
        if (offs[(size_t)p * kPatMaxLen + k] != col0[js + k] - i) return false;
      return true;
    };
    int id = -1;
    if (last >= 0 && same(last)) id = last;   // runs of equal rows are the norm
    for (int p = 0; id < 0 && p < (int)keys.size(); ++p)
      if (same(p)) id = p;
    if (id < 0) {
      if ((int)keys.size() == kPatMax) return 0;
      id = (int)keys.size();
      keys.push_back(h);
      lens.push_back(len);
      for (int k = 0; k < len; ++k) offs[(size_t)id * kPatMaxLen + k] = col0[js + k] - i;
    }
    pat[i] = (unsigned char)id;
    last = id;
  }
  const int np = (int)keys.size();
  tab.assign((size_t)np * (kPatMaxLen + 1), 0);
  std::copy(offs.begin(), offs.begin() + (size_t)np * kPatMaxLen, tab.begin());
  std::copy(lens.begin(), lens.end(), tab.begin() + (size_t)np * kPatMaxLen);
  return np;
}

namespace {


// Largest nnz of any tile of `rows` consecutive rows among the first ni.
// Variable tiles: consecutive rows, at most kTileRows / kTileNnzCap of the
// var configurations each.  False when one row alone exceeds the entry cap.
bool var_tiles(const std::vector<int>& row0, int ni, std::vector<int>& tiles) {
  const int rows = tf::kTileRows[tf::kTileVar1], cap = tf::kTileNnzCap[tf::kTileVar1];
  tiles.clear();
  tiles.push_back(0);
  int r0 = 0;
  while (r0 < ni) {
    if (row0[r0 + 1] - row0[r0] > cap) return false;
    int r1 = r0 + 1;
    while (r1 < ni && r1 - r0 < rows && row0[r1 + 1] - row0[r0] <= cap) ++r1;
    tiles.push_back(r1);
    r0 = r1;
  }
  return ni > 0;
}

int64_t max_tile_nnz(const std::vector<int>& row0, int ni, int rows) {
  int64_t mx = 0;
  for (int r0 = 0; r0 < ni; r0 += rows) {
    const int r1 = std::min(r0 + rows, ni);
    mx = std::max<int64_t>(mx, (int64_t)row0[r1] - row0[r0]);
  }
  return mx;
}

}  // namespace

extern "C" int tf_matrix_register(tf_ctx ctx, int n_cells, int n_own,
                                  int64_t nnz, const int* row, const int* col,
                                  const int* dia, tf_matrix* out) {
  TF_API_BEGIN
  if (!ctx || !out) return TF_ERR_ARG;
  return tf_matrix_create(ctx, n_cells, n_own, nnz, row, col, dia, 1, out);
  TF_API_END
}

namespace {
int matrix_create_impl(tf_ctx_s* ctx, int n_cells, int n_own, int64_t nnz, const int* row,
                       const int* col, const int* dia, int want_icc, int allow_renumber,
                       tf_matrix_s** out);

// Renumbered copy of m for the Jacobi / none solves, when the gathers of the
// given numbering are scattered and reverse Cuthill-McKee gathers better.
int attach_renumbered(tf_matrix_s* m, const std::vector<int>& row0,
                      const std::vector<int>& col0, const std::vector<int>& dia0) {
  const int n = m->nt;
  if (n < kRenumberMinRows || m->ni != n || getenv("TF_NO_RENUMBER")) return TF_OK;
  const double before = tf_gather_lines_per_warp(row0.data(), col0.data(), n, 0);
  if (before <= kRenumberLines) return TF_OK;
  std::vector<int> order;
  tf_rcm_order(row0, col0, n, order);
  std::vector<int> inv(n);
  for (int i = 0; i < n; ++i) inv[order[i]] = i;
  const int64_t nnz = m->nnz;
  std::vector<int> row_r((size_t)n + 1), col_r((size_t)nnz), dia_r(n), src((size_t)nnz),
      row_r0((size_t)n + 1), col_r0((size_t)nnz);
  row_r[0] = 1;
  for (int i = 0; i < n; ++i) {
    const int o = order[i], js = row0[o], len = row0[o + 1] - js;
    const int base = row_r[i] - 1;
    for (int k = 0; k < len; ++k) {
      src[base + k] = js + k;
      col_r0[base + k] = inv[col0[js + k]];
      col_r[base + k] = col_r0[base + k] + 1;
    }
    row_r[i + 1] = row_r[i] + len;
    dia_r[i] = row_r[i] + (dia0[o] - js);
  }
  for (int i = 0; i <= n; ++i) row_r0[i] = row_r[i] - 1;
  const double after = tf_gather_lines_per_warp(row_r0.data(), col_r0.data(), n, 0);
  if (after > 0.8 * before) return TF_OK;
  tf_matrix_s* r = nullptr;
  int st = matrix_create_impl(m->ctx, n, n, nnz, row_r.data(), col_r.data(), dia_r.data(), 0,
                              0, &r);
  if (st != TF_OK) return st;
  m->ren = r;
  st = tf_dev_alloc_bytes(m->ctx, (void**)&m->d_perm, (size_t)n * sizeof(int));
  if (st == TF_OK) st = tf_dev_alloc_bytes(m->ctx, (void**)&m->d_src, (size_t)nnz * sizeof(int));
  if (st != TF_OK) return st;
  cudaError_t e = cudaMemcpyAsync(m->d_perm, order.data(), (size_t)n * sizeof(int),
                                  cudaMemcpyHostToDevice, m->ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(m->d_src, src.data(), (size_t)nnz * sizeof(int),
                        cudaMemcpyHostToDevice, m->ctx->stream);
  if (e == cudaSuccess && !m->ctx->async_alloc) e = cudaStreamSynchronize(m->ctx->stream);
  if (e != cudaSuccess) {
    tf_set_last_cuda_error(e, "cudaMemcpy(renumbering)", __FILE__, __LINE__);
    return TF_ERR_CUDA;
  }
  m->dev_bytes += r->dev_bytes + 4 * ((size_t)n + (size_t)nnz);
  return TF_OK;
}
}  // namespace

int tf_matrix_create(tf_ctx_s* ctx, int n_cells, int n_own, int64_t nnz, const int* row,
                     const int* col, const int* dia, int want_icc, tf_matrix_s** out) {
  return matrix_create_impl(ctx, n_cells, n_own, nnz, row, col, dia, want_icc, 1, out);
}

namespace {
int matrix_create_impl(tf_ctx_s* ctx, int n_cells, int n_own, int64_t nnz, const int* row,
                       const int* col, const int* dia, int want_icc, int allow_renumber,
                       tf_matrix_s** out) {
  if (!ctx || !out) return TF_ERR_ARG;
  *out = nullptr;
  if (n_cells < 0 || n_own < 0 || n_own > n_cells || nnz < 0) return TF_ERR_ARG;
  if (n_cells > 0 && (n_own < 1 || !row || !col || !dia)) return TF_ERR_ARG;
  if (nnz > (int64_t)INT_MAX - 64) return TF_ERR_ARG;

  // Validate the Matrix_Type contract (Create_Matrix.f90:87-119).
  int max_len = 0, diag_first = 1;
  if (n_cells > 0) {
    if (row[0] != 1 || (int64_t)row[n_cells] - 1 != nnz) return TF_ERR_LAYOUT;
    for (int i = 0; i < n_cells; ++i) {
      if (row[i + 1] < row[i]) return TF_ERR_LAYOUT;
      max_len = std::max(max_len, row[i + 1] - row[i]);
      const int d = dia[i];
      if (d < row[i] || d >= row[i + 1] || col[d - 1] != i + 1) return TF_ERR_LAYOUT;
      if (col[row[i] - 1] != i + 1) diag_first = 0;
    }
    for (int64_t j = 0; j < nnz; ++j)
      if (col[j] < 1 || col[j] > n_cells) return TF_ERR_LAYOUT;
  }

  TF_CUDA_TRY(cudaSetDevice(ctx->device));
  tf_matrix_s* m = new tf_matrix_s();
  m->ctx = ctx;
  m->nt = n_cells;
  m->ni = n_own;
  m->nnz = nnz;
  m->max_row_len = max_len;
  m->diag_first = diag_first;
  m->async_alloc = ctx->async_alloc;
  m->dev_bytes = tf_matrix_bytes(n_cells, nnz);

  std::vector<int> row0((size_t)n_cells + 1 + 8, 0), col0((size_t)nnz + 8, 0),
      dia0((size_t)n_cells + 8, 0);
  if (n_cells > 0) {
    for (int i = 0; i <= n_cells; ++i) row0[i] = row[i] - 1;
    for (int i = n_cells + 1; i < (int)row0.size(); ++i) row0[i] = row0[n_cells];
    for (int64_t j = 0; j < nnz; ++j) col0[j] = col[j] - 1;
    for (int i = 0; i < n_cells; ++i) dia0[i] = dia[i] - 1;
  }

  const size_t nv = (size_t)n_cells + 8, nz = (size_t)nnz + 8;
  int st = TF_OK;
#define TRY_ALLOC(p, n)                          \
  if (st == TF_OK) st = dev_alloc(ctx, &(p), (n));
  TRY_ALLOC(m->d_row, row0.size());
  TRY_ALLOC(m->d_col, nz);
  TRY_ALLOC(m->d_dia, nv);
  TRY_ALLOC(m->d_val, nz);
  TRY_ALLOC(m->d_x, nv);
  TRY_ALLOC(m->d_b, nv);
  TRY_ALLOC(m->d_r, nv);
  TRY_ALLOC(m->d_p, nv);
  TRY_ALLOC(m->d_q, nv);
  TRY_ALLOC(m->d_adiag, nv);
  TRY_ALLOC(m->d_part, (size_t)8 * tf::kMaxBlocks + 16);
  TRY_ALLOC(m->d_state, 1);
  TRY_ALLOC(m->d_params, 1);
#undef TRY_ALLOC
  if (st == TF_OK && ctx->async_alloc && ctx->h_state) {   // lent by the context
    m->h_state = ctx->h_state;
    m->h_params = ctx->h_params;
    m->host_lent = 1;
  } else if (st == TF_OK) {
    cudaError_t e = cudaMallocHost((void**)&m->h_state, sizeof(tf::SolveState));
    if (e == cudaSuccess) e = cudaMallocHost((void**)&m->h_params, sizeof(tf::SolveParams));
    if (e != cudaSuccess) {
      tf_set_last_cuda_error(e, "cudaMallocHost", __FILE__, __LINE__);
      st = TF_ERR_OOM;
    }
  }
  if (st == TF_OK) {
    // From pageable memory these return once the source has been staged.
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaMemcpyAsync(m->d_row, row0.data(), row0.size() * sizeof(int),
                                    cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(m->d_col, col0.data(), col0.size() * sizeof(int),
                          cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(m->d_dia, dia0.data(), dia0.size() * sizeof(int),
                          cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && !ctx->async_alloc) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      tf_set_last_cuda_error(e, "cudaMemcpy(structure)", __FILE__, __LINE__);
      st = TF_ERR_CUDA;
    }
  }
  if (st == TF_OK && n_cells > 0) {
    // Fixed tiles whose entries fit their stage.
    unsigned fit_mask = 0;
    int fixed = tf::kTileNone;
    for (int c = 2; c >= 0; --c)
      if (max_tile_nnz(row0, n_own, tf::kTileRows[c]) <= tf::kTileNnzCap[c]) {
        fit_mask |= 1u << c;
        fixed = c;
      }
    // Row-pattern columns for tiled matrices (TF_NO_ROW_PATTERNS keeps CSR).
    if (fixed != tf::kTileNone && !getenv("TF_NO_ROW_PATTERNS")) {
      std::vector<unsigned char> pat;
      std::vector<int> tab;
      const int np = tf_find_row_patterns(row0, col0, n_own, pat, tab);
      if (np > 0) {
        st = dev_alloc(ctx, &m->d_pat, pat.size());
        if (st == TF_OK) st = dev_alloc(ctx, &m->d_pat_tab, tab.size());
        if (st == TF_OK) {
          cudaError_t e = cudaMemcpyAsync(m->d_pat, pat.data(), pat.size(),
                                          cudaMemcpyHostToDevice, ctx->stream);
          if (e == cudaSuccess)
            e = cudaMemcpyAsync(m->d_pat_tab, tab.data(), tab.size() * sizeof(int),
                                cudaMemcpyHostToDevice, ctx->stream);
          if (e == cudaSuccess && !ctx->async_alloc) e = cudaStreamSynchronize(ctx->stream);
          if (e != cudaSuccess) {
            tf_set_last_cuda_error(e, "cudaMemcpy(row patterns)", __FILE__, __LINE__);
            st = TF_ERR_CUDA;
          }
        }
        if (st == TF_OK) m->npat = np;
      }
    }
    // Variable-length CSR tiles (every row fits a stage).
    std::vector<int> tiles;
    if (st == TF_OK && var_tiles(row0, n_own, tiles)) {
      st = dev_alloc(ctx, &m->d_tiles, tiles.size() + 8);
      if (st == TF_OK) {
        cudaError_t e = cudaMemcpyAsync(m->d_tiles, tiles.data(), tiles.size() * sizeof(int),
                                        cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess && !ctx->async_alloc) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) {
          tf_set_last_cuda_error(e, "cudaMemcpy(tiles)", __FILE__, __LINE__);
          st = TF_ERR_CUDA;
        }
        m->ntiles = (int)tiles.size() - 1;
      }
    }
    if (st == TF_OK) st = tf_choose_tiles(m, fit_mask);
  }  if (st == TF_OK && n_cells > 0 && diag_first && want_icc)
    st = tf_icc_build(m, row0.data(), col0.data());
  if (st == TF_OK && allow_renumber) st = attach_renumbered(m, row0, col0, dia0);
  if (st != TF_OK) {
    tf_matrix_free(m);
    return st;
  }
  *out = m;
  return TF_OK;
}
}  // namespace

extern "C" int tf_matrix_release(tf_matrix m) {
  TF_API_BEGIN
  if (!m) return TF_ERR_ARG;
  cudaSetDevice(m->ctx->device);
  cudaStreamSynchronize(m->ctx->stream);
  tf_matrix_free(m);
  return TF_OK;
  TF_API_END
}

extern "C" int tf_matrix_row_patterns(tf_matrix m) {
  TF_API_BEGIN
  return m ? m->npat : TF_ERR_ARG;
  TF_API_END
}

extern "C" int tf_matrix_renumbered(tf_matrix m) {
  TF_API_BEGIN
  return m ? (m->ren != nullptr) : TF_ERR_ARG;
  TF_API_END
}

extern "C" int tf_matrix_info(tf_matrix m, int* n_cells, int* n_own,
                              int64_t* nnz, int* max_row_len) {
  TF_API_BEGIN
  if (!m) return TF_ERR_ARG;
  if (n_cells) *n_cells = m->nt;
  if (n_own) *n_own = m->ni;
  if (nnz) *nnz = m->nnz;
  if (max_row_len) *max_row_len = m->max_row_len;
  return TF_OK;
  TF_API_END
}

extern "C" int tf_matrix_tile_config(tf_matrix m) { return m ? m->tile_cfg : -1; }

extern "C" int tf_matrix_tuning(tf_matrix m, int* cfg, double* us, int cap, int* count) {
  TF_API_BEGIN
  if (!m || !count || (cap > 0 && (!cfg || !us))) return TF_ERR_ARG;
  const int n = std::min<int>(cap, (int)m->tune.size());
  for (int i = 0; i < n; ++i) {
    cfg[i] = m->tune[i].first;
    us[i] = m->tune[i].second;
  }
  *count = (int)m->tune.size();
  return TF_OK;
  TF_API_END
}

extern "C" int tf_matrix_icc_levels(tf_matrix m, int* forward, int* backward) {
  TF_API_BEGIN
  if (!m || !forward || !backward) return TF_ERR_ARG;
  *forward = m->icc_ready ? (int)m->h_levf_ptr.size() - 1 : 0;
  *backward = m->icc_ready ? (int)m->h_levb_ptr.size() - 1 : 0;
  return TF_OK;
  TF_API_END
}

extern "C" int tf_tuning_cache_clear(void) {
  TF_API_BEGIN
  tf_tune_cache_clear();
  return TF_OK;
  TF_API_END
}

// ---------------------------------------------------------------------------
// Solves
// ---------------------------------------------------------------------------
namespace {

int ensure_hist(tf_matrix_s* m, int need) {
  if (m->hist_cap >= need) return TF_OK;
  if (m->d_hist) cudaFree(m->d_hist);
  m->d_hist = nullptr;
  m->hist_cap = 0;
  TF_CUDA_TRY(cudaMalloc((void**)&m->d_hist, (size_t)need * sizeof(double)));
  m->hist_cap = need;
  return TF_OK;
}

int run_solve_core(tf_matrix_s* m, int prec, int miter, double tol,
                   const double* norm) {
  tf_ctx_s* c = m->ctx;
  // Jacobi / none run on the renumbered copy when there is one.
  tf_matrix_s* a = (m->ren && prec != tf::kPrecIcc) ? m->ren : m;
  m->active = a;
  tf::SolveParams* hp = a->h_params;
  hp->tol = tol;
  hp->norm = norm ? *norm : 0.0;
  hp->has_norm = norm ? 1 : 0;
  hp->miter = miter;
  hp->hist = nullptr;
  hp->hist_cap = 0;
  hp->wait_ns = c->wait_ns;
  if (c->history && miter >= 0) {
    int st = ensure_hist(a, miter + 1);
    if (st != TF_OK) return st;
    hp->hist = a->d_hist;
    hp->hist_cap = miter + 1;
  }
  TF_CUDA_TRY(cudaMemcpyAsync(a->d_params, hp, sizeof(*hp), cudaMemcpyHostToDevice, c->stream));
  if (prec == tf::kPrecIcc && !m->icc_ready) return TF_ERR_LAYOUT;  // needs diagonal first
  int st = TF_OK;
  if (a != m) st = tf_renumber_in(m);
  if (st == TF_OK) st = tf_fp64_run(a, prec);
  if (st == TF_OK && a != m) st = tf_renumber_out(m);
  if (st != TF_OK) return st;
  TF_CUDA_TRY(cudaMemcpyAsync(m->h_state, a->d_state, sizeof(tf::SolveState),
                              cudaMemcpyDeviceToHost, c->stream));
  return TF_OK;
}

int finish_solve(tf_matrix_s* m, int* niter, double* fin_res) {
  tf_ctx_s* c = m->ctx;
  TF_CUDA_TRY(cudaStreamSynchronize(c->stream));
  const tf::SolveState& s = *m->h_state;
  if (s.status != 0) return s.status;
  *niter = s.niter;
  *fin_res = s.res;
  c->last_count = 0;
  const tf_matrix_s* a = m->active ? m->active : m;
  if (c->history && a->hist_cap > 0) {
    const bool early_b = s.bnrm2 < a->h_params->tol;
    const int cnt = early_b ? 0 : std::min(s.niter + 1, a->hist_cap);
    c->last_hist.resize(std::max(cnt, 1));
    if (cnt > 0)
      TF_CUDA_TRY(cudaMemcpy(c->last_hist.data(), a->d_hist, cnt * sizeof(double),
                             cudaMemcpyDeviceToHost));
    c->last_count = cnt;
  }
  return TF_OK;
}

}  // namespace

int tf_solve_resident(tf_matrix_s* m, int prec, int miter, double tol, const double* norm,
                      int* niter, double* fin_res) {
  const int st = run_solve_core(m, prec, miter, tol, norm);
  if (st != TF_OK) {
    cudaStreamSynchronize(m->ctx->stream);
    return st;
  }
  return finish_solve(m, niter, fin_res);
}

namespace {

// tf_solve_device on the caller's own arrays: the matrix's val/x/b pointers
// are bound to them for the length of the solve, and the graphs built on
// them are kept while the caller passes the same arrays (one rebuild when
// the arrays change).  A renumbered matrix gathers from and scatters to
// them directly.  Called with m->mu held.
int solve_in_place(tf_matrix_s* m, int prec, double* d_val, double* d_x, double* d_b,
                   int miter, int* niter, double tol, double* fin_res, const double* norm) {
  if (m->ext_key[0] != d_val || m->ext_key[1] != d_x || m->ext_key[2] != d_b) {
    for (auto& g : m->ext_graph)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
    m->ext_key[0] = d_val;
    m->ext_key[1] = d_x;
    m->ext_key[2] = d_b;
  }
  double* own[3] = {m->d_val, m->d_x, m->d_b};
  m->d_val = d_val;
  m->d_x = d_x;
  m->d_b = d_b;
  m->ext_bound = 1;
  const int st = run_solve_core(m, prec, miter, tol, norm);
  m->d_val = own[0];
  m->d_x = own[1];
  m->d_b = own[2];
  m->ext_bound = 0;
  if (st != TF_OK) {
    cudaStreamSynchronize(m->ctx->stream);
    return st;
  }
  return finish_solve(m, niter, fin_res);
}

int check_solve_args(tf_ctx ctx, tf_matrix m, int solver, int prec, int* niter,
                     double* fin_res) {
  if (!ctx || !m || m->ctx != ctx || !niter || !fin_res) return TF_ERR_ARG;
  if (solver != TF_SOLVER_CG && solver != TF_SOLVER_BICG) return TF_ERR_UNKNOWN_SOLVER;
  if (prec < TF_PREC_NONE || prec > TF_PREC_ICC) return TF_ERR_UNKNOWN_PREC;
  return TF_OK;
}

}  // namespace

extern "C" int tf_solve(tf_ctx ctx, tf_matrix m, int solver, int prec,
                        double* val, double* x, double* b, int miter,
                        int* niter, double tol, double* fin_res,
                        const double* norm) {
  TF_API_BEGIN
  int st = check_solve_args(ctx, m, solver, prec, niter, fin_res);
  if (st != TF_OK) return st;
  if (m->nt == 0) {
    *niter = 0;
    *fin_res = 0.0;
    return TF_OK;
  }
  if (!val || !x || !b) return TF_ERR_ARG;
  std::lock_guard<std::mutex> lk(m->mu);
  TF_CUDA_TRY(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  const size_t vb = (size_t)m->nnz * sizeof(double), nb = (size_t)m->nt * sizeof(double);
  TF_CUDA_TRY(cudaMemcpyAsync(m->d_val, val, vb, cudaMemcpyHostToDevice, s));
  TF_CUDA_TRY(cudaMemcpyAsync(m->d_x, x, nb, cudaMemcpyHostToDevice, s));
  TF_CUDA_TRY(cudaMemcpyAsync(m->d_b, b, nb, cudaMemcpyHostToDevice, s));
  st = run_solve_core(m, prec, miter, tol, norm);
  if (st != TF_OK) {
    cudaStreamSynchronize(s);
    return st;
  }
  TF_CUDA_TRY(cudaMemcpyAsync(val, m->d_val, vb, cudaMemcpyDeviceToHost, s));
  TF_CUDA_TRY(cudaMemcpyAsync(x, m->d_x, nb, cudaMemcpyDeviceToHost, s));
  TF_CUDA_TRY(cudaMemcpyAsync(b, m->d_b, nb, cudaMemcpyDeviceToHost, s));
  return finish_solve(m, niter, fin_res);
  TF_API_END
}

extern "C" int tf_solve_device(tf_ctx ctx, tf_matrix m, int solver, int prec,
                               double* d_val, double* d_x, double* d_b,
                               int miter, int* niter, double tol,
                               double* fin_res, const double* norm) {
  TF_API_BEGIN
  int st = check_solve_args(ctx, m, solver, prec, niter, fin_res);
  if (st != TF_OK) return st;
  if (m->nt == 0) {
    *niter = 0;
    *fin_res = 0.0;
    return TF_OK;
  }
  if (!d_val || !d_x || !d_b) return TF_ERR_ARG;
  std::lock_guard<std::mutex> lk(m->mu);
  TF_CUDA_TRY(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  if ((((uintptr_t)d_val | (uintptr_t)d_x | (uintptr_t)d_b) & 15) == 0)
    return solve_in_place(m, prec, d_val, d_x, d_b, miter, niter, tol, fin_res, norm);
  // Arrays off a 16-byte boundary: solve on the matrix's own buffers.
  const size_t vb = (size_t)m->nnz * sizeof(double), nb = (size_t)m->nt * sizeof(double);
  TF_CUDA_TRY(cudaMemcpyAsync(m->d_val, d_val, vb, cudaMemcpyDeviceToDevice, s));
  TF_CUDA_TRY(cudaMemcpyAsync(m->d_x, d_x, nb, cudaMemcpyDeviceToDevice, s));
  TF_CUDA_TRY(cudaMemcpyAsync(m->d_b, d_b, nb, cudaMemcpyDeviceToDevice, s));
  st = run_solve_core(m, prec, miter, tol, norm);
  if (st != TF_OK) {
    cudaStreamSynchronize(s);
    return st;
  }
  TF_CUDA_TRY(cudaMemcpyAsync(d_val, m->d_val, vb, cudaMemcpyDeviceToDevice, s));
  TF_CUDA_TRY(cudaMemcpyAsync(d_x, m->d_x, nb, cudaMemcpyDeviceToDevice, s));
  TF_CUDA_TRY(cudaMemcpyAsync(d_b, m->d_b, nb, cudaMemcpyDeviceToDevice, s));
  return finish_solve(m, niter, fin_res);
  TF_API_END
}

// ---------------------------------------------------------------------------
// Multi-RHS solves
// ---------------------------------------------------------------------------
namespace {

// Device pointers of right-hand side i's x and b inside the workspace.
double* rhs_x(tf_matrix_s* m, int i) { return i == 0 ? m->d_x : m->slices[i - 1]->d_x; }
double* rhs_b(tf_matrix_s* m, int i) { return i == 0 ? m->d_b : m->slices[i - 1]->d_b; }
const tf::SolveState* rhs_state(tf_matrix_s* m, int i) {
  return i == 0 ? m->d_state : m->slices[i - 1]->d_state;
}

// Runs the multi-RHS graph on the workspace (val, x_i, b_i already there)
// and fetches the states; the caller copies results and synchronises.
int run_multi_core(tf_matrix_s* m, int prec, int nrhs, int miter, double tol,
                   const double* norm) {
  tf_ctx_s* c = m->ctx;
  tf::SolveParams* hp = m->h_params;
  hp->tol = tol;
  hp->norm = norm ? *norm : 0.0;
  hp->has_norm = norm ? 1 : 0;
  hp->miter = miter;
  hp->hist = nullptr;
  hp->hist_cap = 0;
  hp->wait_ns = c->wait_ns;
  TF_CUDA_TRY(cudaMemcpyAsync(m->d_params, hp, sizeof(*hp), cudaMemcpyHostToDevice, c->stream));
  int st = tf_fp64_run_multi(m, prec, nrhs);
  if (st != TF_OK) return st;
  if (!m->h_mstate) {
    cudaError_t e = cudaMallocHost((void**)&m->h_mstate, kMaxRhs * sizeof(tf::SolveState));
    if (e != cudaSuccess) {
      tf_set_last_cuda_error(e, "cudaMallocHost", __FILE__, __LINE__);
      return TF_ERR_OOM;
    }
  }
  for (int i = 0; i < nrhs; ++i)
    TF_CUDA_TRY(cudaMemcpyAsync(m->h_mstate + i, rhs_state(m, i), sizeof(tf::SolveState),
                                cudaMemcpyDeviceToHost, c->stream));
  return TF_OK;
}

int finish_multi(tf_matrix_s* m, int nrhs, int* niter, double* fin_res) {
  TF_CUDA_TRY(cudaStreamSynchronize(m->ctx->stream));
  for (int i = 0; i < nrhs; ++i)
    if (m->h_mstate[i].status != 0) return m->h_mstate[i].status;
  for (int i = 0; i < nrhs; ++i) {
    niter[i] = m->h_mstate[i].niter;
    fin_res[i] = m->h_mstate[i].res;
  }
  return TF_OK;
}

int check_multi_args(tf_ctx ctx, tf_matrix m, int solver, int prec, int nrhs, int* niter,
                     double* fin_res) {
  int st = check_solve_args(ctx, m, solver, prec, niter, fin_res);
  if (st != TF_OK) return st;
  if (nrhs < 1 || nrhs > kMaxRhs || prec == TF_PREC_ICC) return TF_ERR_ARG;
  return TF_OK;
}

}  // namespace

extern "C" int tf_solve_multi(tf_ctx ctx, tf_matrix m, int solver, int prec, int nrhs,
                              double* val, double* x, double* b, int miter, int* niter,
                              double tol, double* fin_res, const double* norm) {
  TF_API_BEGIN
  int st = check_multi_args(ctx, m, solver, prec, nrhs, niter, fin_res);
  if (st != TF_OK) return st;
  if (m->nt == 0) {
    for (int i = 0; i < nrhs; ++i) niter[i] = 0, fin_res[i] = 0.0;
    return TF_OK;
  }
  if (!val || !x || !b) return TF_ERR_ARG;
  std::lock_guard<std::mutex> lk(m->mu);
  TF_CUDA_TRY(cudaSetDevice(ctx->device));
  st = tf_slices_ensure(m, nrhs);
  if (st != TF_OK) return st;
  cudaStream_t s = ctx->stream;
  const size_t vb = (size_t)m->nnz * sizeof(double), nb = (size_t)m->nt * sizeof(double);
  TF_CUDA_TRY(cudaMemcpyAsync(m->d_val, val, vb, cudaMemcpyHostToDevice, s));
  for (int i = 0; i < nrhs; ++i) {
    TF_CUDA_TRY(cudaMemcpyAsync(rhs_x(m, i), x + (size_t)i * m->nt, nb,
                                cudaMemcpyHostToDevice, s));
    TF_CUDA_TRY(cudaMemcpyAsync(rhs_b(m, i), b + (size_t)i * m->nt, nb,
                                cudaMemcpyHostToDevice, s));
  }
  st = run_multi_core(m, prec, nrhs, miter, tol, norm);
  if (st != TF_OK) {
    cudaStreamSynchronize(s);
    return st;
  }
  TF_CUDA_TRY(cudaMemcpyAsync(val, m->d_val, vb, cudaMemcpyDeviceToHost, s));
  for (int i = 0; i < nrhs; ++i) {
    TF_CUDA_TRY(cudaMemcpyAsync(x + (size_t)i * m->nt, rhs_x(m, i), nb,
                                cudaMemcpyDeviceToHost, s));
    TF_CUDA_TRY(cudaMemcpyAsync(b + (size_t)i * m->nt, rhs_b(m, i), nb,
                                cudaMemcpyDeviceToHost, s));
  }
  return finish_multi(m, nrhs, niter, fin_res);
  TF_API_END
}

extern "C" int tf_solve_multi_device(tf_ctx ctx, tf_matrix m, int solver, int prec, int nrhs,
                                     double* d_val, double* d_x, double* d_b, int miter,
                                     int* niter, double tol, double* fin_res,
                                     const double* norm) {
  TF_API_BEGIN
  int st = check_multi_args(ctx, m, solver, prec, nrhs, niter, fin_res);
  if (st != TF_OK) return st;
  if (m->nt == 0) {
    for (int i = 0; i < nrhs; ++i) niter[i] = 0, fin_res[i] = 0.0;
    return TF_OK;
  }
  if (!d_val || !d_x || !d_b) return TF_ERR_ARG;
  std::lock_guard<std::mutex> lk(m->mu);
  TF_CUDA_TRY(cudaSetDevice(ctx->device));
  st = tf_slices_ensure(m, nrhs);
  if (st != TF_OK) return st;
  cudaStream_t s = ctx->stream;
  const size_t vb = (size_t)m->nnz * sizeof(double), nb = (size_t)m->nt * sizeof(double);
  const cudaMemcpyKind dd = cudaMemcpyDeviceToDevice;
  TF_CUDA_TRY(cudaMemcpyAsync(m->d_val, d_val, vb, dd, s));
  for (int i = 0; i < nrhs; ++i) {
    TF_CUDA_TRY(cudaMemcpyAsync(rhs_x(m, i), d_x + (size_t)i * m->nt, nb, dd, s));
    TF_CUDA_TRY(cudaMemcpyAsync(rhs_b(m, i), d_b + (size_t)i * m->nt, nb, dd, s));
  }
  st = run_multi_core(m, prec, nrhs, miter, tol, norm);
  if (st != TF_OK) {
    cudaStreamSynchronize(s);
    return st;
  }
  TF_CUDA_TRY(cudaMemcpyAsync(d_val, m->d_val, vb, dd, s));
  for (int i = 0; i < nrhs; ++i) {
    TF_CUDA_TRY(cudaMemcpyAsync(d_x + (size_t)i * m->nt, rhs_x(m, i), nb, dd, s));
    TF_CUDA_TRY(cudaMemcpyAsync(d_b + (size_t)i * m->nt, rhs_b(m, i), nb, dd, s));
  }
  return finish_multi(m, nrhs, niter, fin_res);
  TF_API_END
}

namespace {
// Fortran-style comparison: trailing blanks are not significant.
bool name_is(const char* s, const char* want) {
  size_t n = strlen(s);
  while (n > 0 && s[n - 1] == ' ') --n;
  return n == strlen(want) && strncmp(s, want, n) == 0;
}
}  // namespace

extern "C" int tf_solve_native(tf_ctx ctx, tf_matrix m, const char* solver,
                               const char* prec, double* val, double* x,
                               double* b, int miter, int* niter, double tol,
                               double* fin_res, const double* norm) {
  TF_API_BEGIN
  if (!solver || !prec) return TF_ERR_ARG;
  int s;
  if (name_is(solver, "bicg")) s = TF_SOLVER_BICG;        // Solve_Native.f90:33
  else if (name_is(solver, "cg")) s = TF_SOLVER_CG;       // Solve_Native.f90:35
  else return TF_ERR_UNKNOWN_SOLVER;                      // Solve_Native.f90:38
  // Prec_Form.f90:47-89 / Prec_Solve.f90:44-102: 'jacobi', 'icc', and any
  // other name runs unpreconditioned (their else branches).
  int p;
  if (name_is(prec, "jacobi") || name_is(prec, "diagonal")) p = TF_PREC_JACOBI;
  else if (name_is(prec, "icc") || name_is(prec, "incomplete_cholesky")) p = TF_PREC_ICC;
  else p = TF_PREC_NONE;
  return tf_solve(ctx, m, s, p, val, x, b, miter, niter, tol, fin_res, norm);
  TF_API_END
}

// ---------------------------------------------------------------------------
// Building blocks
// ---------------------------------------------------------------------------
extern "C" int tf_spmv(tf_ctx ctx, tf_matrix m, const double* d_val,
                       const double* d_p, double* d_q, double* d_pq) {
  TF_API_BEGIN
  if (!ctx || !m || m->ctx != ctx) return TF_ERR_ARG;
  if (m->nt == 0) return TF_OK;
  if (!d_val || !d_p || !d_q) return TF_ERR_ARG;
  if (((uintptr_t)d_val & 15) != 0) return TF_ERR_ARG;  // bulk copies need 16 B
  TF_CUDA_TRY(cudaSetDevice(ctx->device));
  return tf_fp64_spmv(m, d_val, d_p, d_q, d_pq);
  TF_API_END
}

extern "C" int tf_residual(tf_ctx ctx, tf_matrix m, const double* d_val,
                           const double* d_b, const double* d_x, double* d_r) {
  TF_API_BEGIN
  if (!ctx || !m || m->ctx != ctx) return TF_ERR_ARG;
  if (m->nt == 0) return TF_OK;
  if (!d_val || !d_b || !d_x || !d_r) return TF_ERR_ARG;
  if (((uintptr_t)d_val & 15) != 0) return TF_ERR_ARG;
  TF_CUDA_TRY(cudaSetDevice(ctx->device));
  return tf_fp64_residual(m, d_val, d_b, d_x, d_r);
  TF_API_END
}

extern "C" int tf_nrms(tf_ctx ctx, tf_matrix m, const double* d_val,
                       const double* d_r, const double* d_x,
                       const double* norm, double* d_out) {
  TF_API_BEGIN
  if (!ctx || !m || m->ctx != ctx || !d_val || !d_r || !d_x || !d_out) return TF_ERR_ARG;
  if (m->nt == 0) return TF_ERR_ARG;
  TF_CUDA_TRY(cudaSetDevice(ctx->device));
  return tf_fp64_nrms(m, d_val, d_r, d_x, norm ? 1 : 0, norm ? *norm : 0.0, d_out);
  TF_API_END
}

// tf_vec.cu -- vector kernels for callers that run their own Krylov loop
// (the row-block solve of one system over several GPUs): the updates and
// partial sums of Native_Mod/Cg.f90 on device vectors, each expression
// rounded as the reference's loop rounds it, and deterministic sums (fixed
// grid, per-block partials combined in block order by the last block).
#include <cuda_runtime.h>

#include <algorithm>

#include "tf_internal.h"

namespace tf {

constexpr int kVecThreads = 256;

struct VecRed {
  double* part;        // kVecMaxBlocks * 2 partials
  unsigned* counter;
  double* out;
};

// y = a x + b y (Cg.f90:166-170 p = z + beta p, :204-209 x + alfa p and
// r - alfa q); first: y = a x; a == 0: y = b y.
__global__ void __launch_bounds__(kVecThreads) k_vec_axpby(int n, double a, const double* x,
                                                           double b, double* y, int first) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    if (first) y[i] = __dmul_rn(a, x[i]);
    else if (a == 0.0) y[i] = __dmul_rn(b, y[i]);
    else y[i] = __dadd_rn(__dmul_rn(a, x[i]), __dmul_rn(b, y[i]));
  }
}

__global__ void __launch_bounds__(kVecThreads) k_vec_gather(int n, const double* src,
                                                            const long long* idx, double* out) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) out[i] = src[idx[i]];
}

__global__ void __launch_bounds__(kVecThreads) k_vec_scatter(int n, double* dst,
                                                             const long long* idx,
                                                             const double* vals) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) dst[idx[i]] = vals[i];
}

__global__ void __launch_bounds__(kVecThreads) k_vec_recip(int n, const double* x, double* out) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    out[i] = __ddiv_rn(1.0, x[i]);   // Prec_Form.f90:51 d_inv = 1.0 / d
}

// KIND 0: sum a_i b_i (b null: sum a_i); 1: sum r_i^2 / d_i^2
// (Normalized_Root_Mean_Square.f90:33-36); 2: z = r d_inv (Prec_Solve.f90:
// 44-49) and sum z_i r_i (Cg.f90:151-155); 3: min and max of x.
template <int KIND>
__global__ void __launch_bounds__(kVecThreads) k_vec_reduce(int n, const double* a,
                                                            const double* b, double* z,
                                                            VecRed red) {
  __shared__ double scratch[2 * (kVecThreads / 32)];
  double s0 = KIND == 3 ? red_identity<kMin>() : 0.0;
  double s1 = red_identity<kMax>();
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    if (KIND == 0) s0 = __dadd_rn(s0, b ? __dmul_rn(a[i], b[i]) : a[i]);
    if (KIND == 1) s0 = __dadd_rn(s0, nrms_term(a[i], b[i]));
    if (KIND == 2) {
      const double zi = __dmul_rn(a[i], b[i]);
      z[i] = zi;
      s0 = __dadd_rn(s0, __dmul_rn(zi, a[i]));
    }
    if (KIND == 3) {
      s0 = fmin(s0, a[i]);
      s1 = fmax(s1, a[i]);
    }
  }
  if (KIND == 3) {
    double v[2] = {block_red<kMin>(s0, scratch), block_red<kMax>(s1, scratch)};
    const int ops[2] = {kMin, kMax};
    if (grid_reduce_last<2>(v, ops, red.part, red.counter, scratch) && threadIdx.x == 0) {
      red.out[0] = v[0];
      red.out[1] = v[1];
    }
  } else {
    double v[1] = {block_red<kSum>(s0, scratch)};
    const int ops[1] = {kSum};
    if (grid_reduce_last<1>(v, ops, red.part, red.counter, scratch) && threadIdx.x == 0)
      red.out[0] = v[0];
  }
}

}  // namespace tf

using namespace tf;

namespace {

constexpr int kVecMaxBlocks = 1024;

int vec_grid(tf_ctx_s* c, int n) {
  return std::max(1, std::min({(n + kVecThreads - 1) / kVecThreads, c->sm_count * 4,
                               kVecMaxBlocks}));
}

// The context's scratch for the sums (partials and a counter), on first use.
int vec_scratch(tf_ctx_s* c, VecRed* r, double* out) {
  if (!c->d_vec_scratch) {
    void* p = nullptr;
    const int st = tf_dev_alloc_bytes(c, &p, (2 * kVecMaxBlocks + 16) * sizeof(double));
    if (st != TF_OK) return st;
    c->d_vec_scratch = static_cast<double*>(p);
  }
  r->part = c->d_vec_scratch;
  r->counter = reinterpret_cast<unsigned*>(c->d_vec_scratch + 2 * kVecMaxBlocks);
  r->out = out;
  return TF_OK;
}

template <int KIND>
int vec_reduce(tf_ctx ctx, int n, const double* a, const double* b, double* z, double* out) {
  if (!ctx || n < 0 || !out || (n > 0 && !a) || (KIND >= 1 && KIND <= 2 && n > 0 && !b) ||
      (KIND == 2 && n > 0 && !z))
    return TF_ERR_ARG;
  TF_CUDA_TRY(cudaSetDevice(ctx->device));
  VecRed red;
  int st = vec_scratch(ctx, &red, out);
  if (st != TF_OK) return st;
  k_vec_reduce<KIND><<<vec_grid(ctx, n), kVecThreads, 0, ctx->stream>>>(n, a, b, z, red);
  TF_CUDA_TRY(cudaGetLastError());
  return TF_OK;
}

}  // namespace

extern "C" int tf_vec_axpby(tf_ctx ctx, int n, double a, const double* d_x, double b,
                            double* d_y, int first) {
  TF_API_BEGIN
  if (!ctx || n < 0 || (n > 0 && (!d_x || !d_y))) return TF_ERR_ARG;
  if (n == 0) return TF_OK;
  TF_CUDA_TRY(cudaSetDevice(ctx->device));
  k_vec_axpby<<<vec_grid(ctx, n), kVecThreads, 0, ctx->stream>>>(n, a, d_x, b, d_y, first);
  TF_CUDA_TRY(cudaGetLastError());
  return TF_OK;
  TF_API_END
}

extern "C" int tf_vec_gather(tf_ctx ctx, int n, const double* d_src, const int64_t* d_idx,
                             double* d_out) {
  TF_API_BEGIN
  if (!ctx || n < 0 || (n > 0 && (!d_src || !d_idx || !d_out))) return TF_ERR_ARG;
  if (n == 0) return TF_OK;
  TF_CUDA_TRY(cudaSetDevice(ctx->device));
  k_vec_gather<<<vec_grid(ctx, n), kVecThreads, 0, ctx->stream>>>(
      n, d_src, reinterpret_cast<const long long*>(d_idx), d_out);
  TF_CUDA_TRY(cudaGetLastError());
  return TF_OK;
  TF_API_END
}

extern "C" int tf_vec_scatter(tf_ctx ctx, int n, double* d_dst, const int64_t* d_idx,
                              const double* d_vals) {
  TF_API_BEGIN
  if (!ctx || n < 0 || (n > 0 && (!d_dst || !d_idx || !d_vals))) return TF_ERR_ARG;
  if (n == 0) return TF_OK;
  TF_CUDA_TRY(cudaSetDevice(ctx->device));
  k_vec_scatter<<<vec_grid(ctx, n), kVecThreads, 0, ctx->stream>>>(
      n, d_dst, reinterpret_cast<const long long*>(d_idx), d_vals);
  TF_CUDA_TRY(cudaGetLastError());
  return TF_OK;
  TF_API_END
}

extern "C" int tf_vec_recip(tf_ctx ctx, int n, const double* d_x, double* d_out) {
  TF_API_BEGIN
  if (!ctx || n < 0 || (n > 0 && (!d_x || !d_out))) return TF_ERR_ARG;
  if (n == 0) return TF_OK;
  TF_CUDA_TRY(cudaSetDevice(ctx->device));
  k_vec_recip<<<vec_grid(ctx, n), kVecThreads, 0, ctx->stream>>>(n, d_x, d_out);
  TF_CUDA_TRY(cudaGetLastError());
  return TF_OK;
  TF_API_END
}

extern "C" int tf_vec_dot(tf_ctx ctx, int n, const double* d_a, const double* d_b,
                          double* d_out) {
  TF_API_BEGIN
  return vec_reduce<0>(ctx, n, d_a, d_b, nullptr, d_out);
  TF_API_END
}

extern "C" int tf_vec_nrms_sum(tf_ctx ctx, int n, const double* d_r, const double* d_diag,
                               double* d_out) {
  TF_API_BEGIN
  return vec_reduce<1>(ctx, n, d_r, d_diag, nullptr, d_out);
  TF_API_END
}

extern "C" int tf_vec_jacobi(tf_ctx ctx, int n, const double* d_r, const double* d_dinv,
                             double* d_z, double* d_out) {
  TF_API_BEGIN
  return vec_reduce<2>(ctx, n, d_r, d_dinv, d_z, d_out);
  TF_API_END
}

extern "C" int tf_vec_minmax(tf_ctx ctx, int n, const double* d_x, double* d_out2) {
  TF_API_BEGIN
  return vec_reduce<3>(ctx, n, d_x, nullptr, nullptr, d_out2);
  TF_API_END
}

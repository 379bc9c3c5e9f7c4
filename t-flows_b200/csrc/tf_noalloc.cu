// tf_noalloc.cu -- q = A p and p.q without any device allocation.
//
// Some callers cannot call cudaMalloc: their device memory is owned by
// another runtime or pool (an OpenACC data region such as T-Flows' GPU
// layer, a caching allocator, a serving process held to a fixed memory
// budget), or they run a time-stepping loop that cannot afford the device
// synchronisation a cudaFree implies.  tf_spmv_noalloc serves them: the
// caller passes every input and output in device memory it already owns,
// and the only scratch the kernel needs -- one partial sum per row tile plus
// a completion counter -- lives in a fixed array compiled into this library.
//
// The array is kNoAllocTiles doubles (512 KiB) and every GPU that loads the
// library keeps it until the process exits.  With 256-row tiles that bounds
// the matrix at kNoAllocMaxRows = 16,777,216 rows; larger calls are
// rejected with TF_ERR_ARG and a message.
#include <cuda_runtime.h>
#include <stdio.h>

#include <mutex>

#include "tf_internal.h"

namespace {

constexpr int kNoAllocTileRows = 256;
constexpr int kNoAllocTiles = 65536;
constexpr long long kNoAllocMaxRows = (long long)kNoAllocTileRows * kNoAllocTiles;
static_assert(kNoAllocMaxRows == TF_SPMV_NOALLOC_MAX_ROWS, "header limit out of date");

// [0, 256): completion counter (unsigned, cleared before every launch)
// [256, 256 + 8 * kNoAllocTiles): per-tile partial sums of p_i q_i
constexpr size_t kCounterBytes = 256;
constexpr size_t kScratchBytes = kCounterBytes + sizeof(double) * kNoAllocTiles;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Same row arithmetic as the library's SpMV (entries in storage order,
// products and sums rounded separately), reading a 1-based Matrix_Type CSR
// straight from global memory.  One CTA per 256-row tile; the tile's p.q
// partial goes to scratch[tile]; the last CTA sums the partials in tile
// order, so the result is the same for every launch.
__global__ void __launch_bounds__(kNoAllocTileRows)
k_spmv_dot_noalloc(int n, const int* __restrict__ row, const int* __restrict__ col,
                   const double* __restrict__ val, const double* __restrict__ p,
                   double* __restrict__ q, double* __restrict__ pq_out,
                   unsigned char* scratch) {
  __shared__ double red[32];
  __shared__ int s_last;
  unsigned* counter = reinterpret_cast<unsigned*>(scratch);
  double* part = reinterpret_cast<double*>(scratch + kCounterBytes);

  const int i = blockIdx.x * kNoAllocTileRows + threadIdx.x;
  double mine = 0.0;
  if (i < n) {
    const int js = row[i] - 1, je = row[i + 1] - 1;
    double acc = 0.0;
    for (int j = js; j < je; ++j)
      acc = __dadd_rn(acc, __dmul_rn(val[j], __ldg(p + (col[j] - 1))));
    q[i] = acc;
    mine = __dmul_rn(__ldg(p + i), acc);
  }
  mine = tf::block_red<tf::kSum>(mine, red);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = mine;
    __threadfence();
    s_last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double acc = 0.0;
  for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
    acc = __dadd_rn(acc, __ldcg(part + b));
  acc = tf::block_red<tf::kSum>(acc, red);
  if (threadIdx.x == 0) *pq_out = acc;
}

// Device address of the scratch array, looked up once per device.
constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char* g_ptr[kMaxDevices] = {};

int scratch_for_current_device(unsigned char** out) {
  int dev = 0;
  TF_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    char msg[128];
    snprintf(msg, sizeof msg, "tf_spmv_noalloc: device ordinal %d is not below %d", dev,
             kMaxDevices);
    tf_set_last_message(msg);
    return TF_ERR_ARG;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_ptr[dev]) {
    void* p = nullptr;
    TF_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_ptr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_ptr[dev];
  return TF_OK;
}

}  // namespace

extern "C" int tf_spmv_noalloc(int n, const int* d_row, const int* d_col,
                               const double* d_val, const double* d_p,
                               double* d_q, double* d_pq, void* stream) {
  TF_API_BEGIN
  if (n < 0 || (n > 0 && (!d_row || !d_col || !d_val || !d_p || !d_q || !d_pq)))
    return TF_ERR_ARG;
  if ((long long)n > kNoAllocMaxRows) {
    char msg[160];
    snprintf(msg, sizeof msg,
             "tf_spmv_noalloc: %d rows exceed the fixed scratch limit of %lld rows",
             n, kNoAllocMaxRows);
    tf_set_last_message(msg);
    return TF_ERR_ARG;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (n == 0) {
    TF_CUDA_TRY(cudaMemsetAsync(d_pq, 0, sizeof(double), s));
    return TF_OK;
  }
  unsigned char* scratch = nullptr;
  int st = scratch_for_current_device(&scratch);
  if (st != TF_OK) return st;
  // The counter must start at zero; the partials are all overwritten.
  TF_CUDA_TRY(cudaMemsetAsync(scratch, 0, kCounterBytes, s));
  const int tiles = (n + kNoAllocTileRows - 1) / kNoAllocTileRows;
  k_spmv_dot_noalloc<<<tiles, kNoAllocTileRows, 0, s>>>(n, d_row, d_col, d_val, d_p, d_q,
                                                         d_pq, scratch);
  TF_CUDA_TRY(cudaGetLastError());
  return TF_OK;
  TF_API_END
}

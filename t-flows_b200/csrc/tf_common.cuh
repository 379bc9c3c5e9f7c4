// tf_common.cuh -- shared device helpers of the B200 Krylov library:
// deterministic reductions, mbarrier / bulk-copy (TMA 1D) wrappers with
// bounded waits, and the device-side solve state.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace tf {

// Sources/Shared/Const_Mod.f90:84-93
constexpr double kTiny = 1.0e-15;
constexpr double kHuge = 1.0e+15;
constexpr double kMicro = 1.0e-6;

// Upper bound on CTAs of any grid-reduced kernel (size of partial arrays).
constexpr int kMaxBlocks = 4096;
// A bounded device-side wait gives up after this many nanoseconds; the
// streaming kernels of a solve stop at this deadline past their start
// unless the caller set another limit (tf_ctx_set_wait_limit).  Draining
// the bulk copies a CTA armed before it exits always allows this default:
// a kernel never returns with a copy into its shared memory in flight.
constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // 2 s

enum Prec : int { kPrecNone = 0, kPrecJacobi = 1, kPrecIcc = 2 };

// Per-call parameters, uploaded with each solve so captured graphs stay valid.
struct SolveParams {
  double tol;
  double norm;
  int has_norm;
  int miter;
  int hist_cap;       // entries available in hist
  int pad;
  double* hist;       // per-iteration residuals (may be null)
  unsigned long long wait_ns;   // bounded-wait limit (0: kWaitLimitNs)
};

__host__ __device__ __forceinline__ unsigned long long wait_limit(const SolveParams* p) {
  return (p && p->wait_ns) ? p->wait_ns : kWaitLimitNs;
}

// Device-resident solver state; one per matrix handle.
struct SolveState {
  double fn;          // 1/mean(diag) of Cg.f90:75-76
  double sum_a;
  double bnrm2;
  double res;         // current normalised residual (fin_res at the end)
  double rho;         // rho of the current iteration
  double rho_old;
  double alpha;
  double pq;
  double xmin, xmax;  // x range of the initial x (norm absent)
  int iter;           // iteration being executed (1-based)
  int niter;
  int done;
  int status;         // TF_OK or TF_ERR_TIMEOUT
  int x_pend;         // x still lacks the last alpha * p (deferred update)
  int pad;
  unsigned counter[8];  // last-block-done counters, one per kernel kind
  unsigned bar_count;   // grid barrier of the persistent ICC sweeps: arrivals
  unsigned bar_gen;     // ... and generation
};

enum CounterSlot { kCntDiag = 0, kCntScale, kCntResid, kCntSpmv, kCntUpdate,
                   kCntZ, kCntAux, kCntAux2 };

// Acquire / release accesses at GPU scope: a flag read with ld_acquire_gpu
// that returns the value st_release_gpu stored makes every write the
// storing thread made before it visible to the reader's later loads.
__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_gpu(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// ---------------------------------------------------------------------------
// Deterministic reductions: xor-butterfly in a warp, warps in fixed order.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    v = __dadd_rn(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

enum RedOp { kSum = 0, kMin = 1, kMax = 2 };

template <int OP>
__device__ __forceinline__ double red2(double a, double b) {
  if (OP == kSum) return __dadd_rn(a, b);
  if (OP == kMin) return fmin(a, b);
  return fmax(a, b);
}
template <int OP>
__device__ __forceinline__ double warp_red(double v) {
  if (OP == kSum) return warp_sum(v);
  if (OP == kMin) return warp_min(v);
  return warp_max(v);
}
template <int OP>
__device__ __forceinline__ double red_identity() {
  if (OP == kSum) return 0.0;
  if (OP == kMin) return __longlong_as_double(0x7ff0000000000000LL);  // +inf
  return __longlong_as_double(0xfff0000000000000LL);                 // -inf
}

// Block reduction of one value; every thread gets the result.  `scratch`
// needs blockDim/32 doubles.  Contains __syncthreads.
template <int OP>
__device__ double block_red(double v, double* scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  v = warp_red<OP>(v);
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  double r = red_identity<OP>();
  for (int w = 0; w < nw; ++w) r = red2<OP>(r, scratch[w]);
  return r;
}

// Block reduction of NQ values at once (two __syncthreads instead of two
// per value); every thread gets the results.  `scratch` needs
// NQ * blockDim/32 doubles.  Warp partials are combined in warp order, as
// block_red does, so the result is the same as NQ separate block_red calls.
template <int NQ>
__device__ void block_red_n(double (&v)[NQ], const int (&ops)[NQ], double* scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    if (ops[q] == kSum) v[q] = warp_red<kSum>(v[q]);
    else if (ops[q] == kMin) v[q] = warp_red<kMin>(v[q]);
    else v[q] = warp_red<kMax>(v[q]);
  }
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) scratch[q * 32 + warp] = v[q];
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    double r;
    if (ops[q] == kSum) r = red_identity<kSum>();
    else if (ops[q] == kMin) r = red_identity<kMin>();
    else r = red_identity<kMax>();
    for (int w = 0; w < nw; ++w) {
      const double s = scratch[q * 32 + w];
      if (ops[q] == kSum) r = red2<kSum>(r, s);
      else if (ops[q] == kMin) r = red2<kMin>(r, s);
      else r = red2<kMax>(r, s);
    }
    v[q] = r;
  }
}

// Grid-level "last block done" reduction of NQ values with ops OPS.
// Every block calls it once with its block-reduced values (valid in all
// threads).  Returns true in all threads of the last block, whose `vals`
// then hold the grid results, reduced in blockIdx order (deterministic for
// a fixed grid).  part must hold NQ * gridDim.x doubles.
template <int NQ>
__device__ bool grid_reduce_last(double (&vals)[NQ], const int (&ops)[NQ],
                                 double* part, unsigned* counter,
                                 double* scratch) {
  __shared__ int s_last;
  const unsigned G = gridDim.x;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) part[q * G + blockIdx.x] = vals[q];
    __threadfence();
    unsigned prev = atomicAdd(counter, 1u);
    s_last = (prev == G - 1);
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    double acc;
    if (ops[q] == kSum) acc = 0.0;
    else if (ops[q] == kMin) acc = red_identity<kMin>();
    else acc = red_identity<kMax>();
    for (unsigned b = threadIdx.x; b < G; b += blockDim.x) {
      double v = __ldcg(part + q * G + b);
      if (ops[q] == kSum) acc = __dadd_rn(acc, v);
      else if (ops[q] == kMin) acc = fmin(acc, v);
      else acc = fmax(acc, v);
    }
    if (ops[q] == kSum) acc = block_red<kSum>(acc, scratch);
    else if (ops[q] == kMin) acc = block_red<kMin>(acc, scratch);
    else acc = block_red<kMax>(acc, scratch);
    vals[q] = acc;
  }
  if (threadIdx.x == 0) *counter = 0u;  // ready for the next launch
  return true;
}

// grid_reduce_last with one block_red_n for all NQ values in the last
// block; scratch needs NQ * 32 doubles.  Same combination order, so the
// same results as grid_reduce_last.
template <int NQ>
__device__ bool grid_reduce_last_n(double (&vals)[NQ], const int (&ops)[NQ],
                                   double* part, unsigned* counter, double* scratch) {
  __shared__ int s_last;
  const unsigned G = gridDim.x;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) part[q * G + blockIdx.x] = vals[q];
    __threadfence();
    unsigned prev = atomicAdd(counter, 1u);
    s_last = (prev == G - 1);
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    double acc;
    if (ops[q] == kSum) acc = 0.0;
    else if (ops[q] == kMin) acc = red_identity<kMin>();
    else acc = red_identity<kMax>();
    for (unsigned b = threadIdx.x; b < G; b += blockDim.x) {
      double v = __ldcg(part + q * G + b);
      if (ops[q] == kSum) acc = __dadd_rn(acc, v);
      else if (ops[q] == kMin) acc = fmin(acc, v);
      else acc = fmax(acc, v);
    }
    vals[q] = acc;
  }
  block_red_n<NQ>(vals, ops, scratch);
  if (threadIdx.x == 0) *counter = 0u;  // ready for the next launch
  return true;
}

// Normalised RMS finish (Normalized_Root_Mean_Square.f90:38-63).
__device__ __forceinline__ double nrms_finish(double sum_sq, int has_norm,
                                              double norm, double xmin,
                                              double xmax) {
  double rms = __dsqrt_rn(sum_sq);
  double x_min, x_max;
  if (!has_norm) { x_min = xmin; x_max = xmax; }
  else { x_min = 0.0; x_max = norm; }
  double xmm = __dsub_rn(x_max, x_min);
  xmm = (kTiny > xmm) ? kTiny : xmm;
  return __ddiv_rn(rms, xmm);
}

// r_i^2 / a_ii^2 as Normalized_Root_Mean_Square.f90:35 evaluates it.
__device__ __forceinline__ double nrms_term(double r, double a) {
  return __ddiv_rn(__dmul_rn(r, r), __dmul_rn(a, a));
}

// ---------------------------------------------------------------------------
// mbarrier + cp.async.bulk (1D TMA) wrappers
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar,
                                                      unsigned bytes) {
  asm volatile(
      "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
          smem_u32(bar)),
      "r"(bytes)
      : "memory");
}
// Plain arrival (one of the barrier's expected count), release semantics.
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Wait for `parity` with a time limit.  Returns false on timeout.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = globaltimer_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (globaltimer_ns() - t0 > kWaitLimitNs) return false;
  }
  return true;
}

// Waits of the streaming kernels run against a deadline: the kernel's
// start (globaltimer) plus the limit of the solve (tf_ctx_set_wait_limit,
// 2 s by default).  A wait fails when its barrier has not completed by the
// deadline, and also when it completes after the deadline, so a kernel that
// outlives its limit stops at its next wait whether or not its data keeps
// arriving (mbarrier.try_wait suspends in hardware until the phase
// completes, so a limit on the time spent inside one wait alone would
// rarely be reached).
__device__ __forceinline__ unsigned long long deadline_after(unsigned long long limit_ns) {
  return globaltimer_ns() + limit_ns;
}
__device__ __forceinline__ bool mbar_wait_deadline(uint64_t* bar, unsigned parity,
                                                   unsigned long long deadline) {
  while (!mbar_try_wait(bar, parity))
    if (globaltimer_ns() > deadline) return false;
  return globaltimer_ns() <= deadline;
}
// The same, also ending (false) once *abort_flag is set.
__device__ __forceinline__ bool mbar_wait_or_abort(uint64_t* bar, unsigned parity,
                                                   volatile int* abort_flag,
                                                   unsigned long long deadline) {
  while (!mbar_try_wait(bar, parity))
    if (*abort_flag || globaltimer_ns() > deadline) return false;
  return globaltimer_ns() <= deadline;
}
// Wait for the bulk copies armed on `bar` before the CTA exits: always the
// default limit (never the caller's), so a short caller limit cannot end a
// CTA with copies into its shared memory still in flight.
__device__ __forceinline__ void mbar_drain(uint64_t* bar, unsigned parity) {
  mbar_wait_bounded(bar, parity);
}
// Global -> shared bulk copy completing on `bar`.  dst, src 16-byte aligned,
// bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src,
                                         unsigned bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

}  // namespace tf

// tf_batch.cu -- many independent systems solved together.
//
// Design
// ------
// Every system keeps its own CSR (0-based, tile table) and Krylov state in
// one contiguous segment of a device arena.  A work list names (system,
// row tile) items; persistent CTAs walk it, so all active systems advance
// one Jacobi-CG iteration per kernel sequence, each with its own alpha and
// beta.  The Cg/Bicg recurrence is the reference's (Bicg.f90's shadow
// sequence equals the primary one, see tf_fp64.cu).
//
// Precision: the Krylov vectors (x correction, r, p, q, z, 1/diag) are
// stored in V = float ("mixed") or double; the matrix values are FP64 by
// default (optionally FP32); every SpMV row is accumulated in FP64; all dot
// products, alpha, beta and norms are FP64.  Iterative refinement runs as
// reliable updates: when the recursive residual has fallen by `ru_delta`
// since the last update (or reaches tol, or maxit), the FP32 correction is
// folded into the FP64 solution, and the residual is recomputed in FP64 as
// b - A x with FP64 values, which also decides convergence:
// ||b - A x||_2 <= tol ||b||_2.  Measured on stretched Poisson matrices,
// FP32 iterates with FP64 values need ~1.03x the FP64 iteration count,
// while FP32 values need 1.3-1.75x (the perturbed operator breaks the
// recurrence), so FP64 values are the default.
//
// Per-system reductions in two steps, with no atomics and no fences on the
// tile passes: every tile pass stores its tile's totals (in the elementwise
// kernels one warp owns a tile; in the tile streamers the reducer warp sums
// the consumer warps' partials in warp order), and a finishing kernel, one
// warp per system, sums the system's tile totals in a fixed order and
// updates the system's scalars; the kernel boundary orders the two.  A
// system's arithmetic never depends on which other systems share the
// batch: results are bit-identical alone and in any mix.  The refinement
// kernels walk a compact list of the tiles of the systems due an update,
// appended by the warp that decides it.
//
// Kernels of one iteration (all skip systems with nothing to do):
//   kb_pupdate   z = dinv r, p = z + beta p
//   kb_spmv      q = A p (tile streamer), p.q per tile
//   kb_alpha     alpha per system
//   kb_update    xlo += alpha p, r -= alpha q, rho and |r|^2 per tile
//   kb_beta      rho, beta, RU trigger per system
//   kb_ru_fold   x += xlo, xlo = 0                       (systems due an RU)
//   kb_ru_res    r = b - A x in FP64 (tile streamer), |r|^2, rho per tile;
//                on a new system also forms dinv and |b|^2
//   kb_ru_finish the refinement's test per system
// A sweep of S iterations is captured once as a CUDA graph; the host only
// looks at the state array between sweeps (retire, admit, rebuild the list).
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <tuple>
#include <memory>
#include <mutex>
#include <new>
#include <stdexcept>
#include <system_error>
#include <thread>
#include <vector>

#include "tf_internal.h"
#include "tf_tile.cuh"
#include "tf_tile2.cuh"

namespace tfb {

using namespace tf;

enum SysStatus : int {
  kFree = 0, kInit = 1, kActive = 2, kConverged = 3, kMaxIter = 4, kBreakdown = 5
};

constexpr int kRows = 512;       // rows per tile (max) = threads per tile CTA
constexpr int kWarps = kRows / 32;
constexpr int kNnzCap = 4096;    // entries per tile stage
constexpr int kStages = 2;
constexpr int kPartQ = 4;        // partial sums kept per tile / warp
constexpr int kRuEvery = 50;     // FP32 iterates: refine at least this often
// Kernels of an iteration, in launch order (profiling: tf_batch_kernel_ms).
constexpr int kKernels = 8;

template <typename V>
struct SysDev {
  const int* row;       // n+1, 0-based
  const int* col;       // nnz, 0-based local (null with row patterns)
  const unsigned char* pat;   // row patterns: one byte per row (else null)
  const int* tab;             // their offsets, [npat][kPatMaxLen]
  int npat;
  const double* val;    // FP64 values
  const float* val32;   // FP32 copy (use_val32)
  const int* tiles;     // ntiles+1 row boundaries
  const int* dia;       // n, 0-based
  const double* b;
  double* x;
  V* xlo;
  V* r;
  V* p;
  V* q;
  V* dinv;
  double* tile_tot;     // ntiles * kPartQ: per-tile totals
  double* chunk_tot;    // n_fin_chunks * kPartQ: chunk totals (finishing kernels)
  double* warp_part;    // FP32 values: ntiles * kWarps * kPartQ per-warp partials
  unsigned* tile_cnt;   // FP32 values: ntiles, warps of a tile that have reported
  int n, ntiles;
  int maxit, use_val32;
  double tol;
};

// Bytes of one slot's descriptor staging (either iterate type).
constexpr size_t kDescBytes =
    ((sizeof(SysDev<double>) > sizeof(SysDev<float>) ? sizeof(SysDev<double>)
                                                      : sizeof(SysDev<float>)) + 63) / 64 * 64;

struct SysState {
  double rho, rho_old, beta, alpha;
  double rr, rr_ru, bnorm2, res_true;
  int status, iter, first, need_ru;
  int n_ru, iter_ru;   // refinements so far; iteration of the last one
  unsigned fin_cnt;    // chunks of a finishing kernel that have reported
  int pad;
};

struct Work {
  int sys;
  int tile;
  int r0, r1;             // the tile's rows
  int j0, j1;             // its entries (row[r0], row[r1])
};

// Refinement (reliable-update) work list: the warp that finishes a system in
// kb_update appends that system's tiles when an update is due; the host
// pre-fills it with the tiles of newly admitted systems; the last CTA of
// kb_ru_res empties it.  The refinement kernels touch only these tiles.
struct RuList {
  Work* items;
  int* count;
};

// An item of the finishing kernels: chunk `chunk` (kFinTiles tile totals)
// of system `sys`.
struct FinItem {
  int sys, chunk;
};

struct BatchArgs {
  const void* desc;       // SysDev<V>*
  SysState* st;
  const Work* work;
  const int* nwork;
  double ru_delta2;
  RuList ru;
  const FinItem* fin;     // the finishing kernels' items
  const int* nfin;
  unsigned* gate_cnt;     // CTAs of kb_beta that are done (the last opens the gate)
  cudaGraphConditionalHandle ru_gate;   // the refinement kernels' IF node
  int use_gate;           // 0: launched directly (no graph), the kernels always run
};

__device__ __forceinline__ bool active(const SysState& s) { return s.status == kActive; }

// ---------------------------------------------------------------------------
// Per-system reductions: tile totals, then one warp per system.
// ---------------------------------------------------------------------------
template <int NQ>
__device__ __forceinline__ void put_tile_total(double* tile_tot, int tile,
                                               const double (&v)[NQ]) {
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) tile_tot[(size_t)tile * kPartQ + q] = v[q];
  }
}

// FP32-value SpMV (one CTA of kWarps warps per tile): every warp reports
// its partial; the tile's last warp sums the kWarps partials in warp order
// and returns true with v = the tile's totals.  v: this thread's values.
template <int NQ>
__device__ bool cta_tile_total(double* warp_part, unsigned* tile_cnt, int tile,
                               double (&v)[NQ]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q) v[q] = warp_sum(v[q]);
  unsigned last = 0;
  if (lane == 0) {
    double* wp = warp_part + ((size_t)tile * kWarps + warp) * kPartQ;
#pragma unroll
    for (int q = 0; q < NQ; ++q) wp[q] = v[q];
    __threadfence();
    last = (atomicAdd(tile_cnt + tile, 1u) == (unsigned)kWarps - 1);
  }
  last = __shfl_sync(0xffffffffu, last, 0);
  if (!last) return false;
  __threadfence();
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    const double w = lane < kWarps
                         ? __ldcg(warp_part + ((size_t)tile * kWarps + lane) * kPartQ + q)
                         : 0.0;
    v[q] = warp_sum(w);
  }
  if (lane == 0) tile_cnt[tile] = 0u;
  return true;
}

// ---------------------------------------------------------------------------
// Elementwise kernels: one warp per tile.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int warp_global() {
  return (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
}
__device__ __forceinline__ int warps_total() { return (int)((gridDim.x * blockDim.x) >> 5); }

// A warp takes a whole tile (at most kRows rows): lane l owns rows
// r0 + l + 32 u, u < kPerLane.  Every load of the tile is issued before the
// first result is formed, so a warp keeps kPerLane loads per array in
// flight.  The tile descriptors are software-pipelined: while a warp works
// on item k it already holds the descriptor (system state and array
// pointers) of item k + stride and the work entry of item k + 2 stride, so
// only the data loads' latency is on its path.  Neither kernel changes a
// system's state, so a descriptor read early is still current.
constexpr int kPerLane = kRows / 32;

// The work entries of a warp's items, one stride apart.
struct WorkStream {
  const Work* work;
  int nw, k, stride;
  __device__ Work at(int kk) const { return kk < nw ? work[kk] : Work{0, 0, 0, 0, 0, 0}; }
};

template <typename V>
struct PupdateDesc {
  int r0, r1, go, first;
  double beta;
  const V* r;
  const V* dinv;
  V* p;
  __device__ void load(const Work& w, const SysDev<V>* D, const SysState* st) {
    const SysState& s = st[w.sys];
    const SysDev<V>& d = D[w.sys];
    r0 = w.r0;
    r1 = w.r1;
    go = active(s);
    first = s.first;
    beta = s.beta;
    r = d.r;
    dinv = d.dinv;
    p = d.p;
  }
};

// Resident CTAs per SM asked of the register allocator (FP32 iterates:
// all of a tile's values fit in registers at this occupancy).
template <typename V>
constexpr int ew_min_blocks(int fp32) { return sizeof(V) == 4 ? fp32 : 1; }

template <typename V>
__global__ void __launch_bounds__(256, ew_min_blocks<V>(3)) kb_pupdate(BatchArgs a) {
  const SysDev<V>* D = static_cast<const SysDev<V>*>(a.desc);
  const WorkStream ws{a.work, *a.nwork, warp_global(), warps_total()};
  if (ws.k >= ws.nw) return;
  const int lane = threadIdx.x & 31;
  PupdateDesc<V> cur, nxt;
  cur.load(ws.at(ws.k), D, a.st);
  Work wn = ws.at(ws.k + ws.stride);
  for (int k = ws.k; k < ws.nw; k += ws.stride) {
    const Work wnn = ws.at(k + 2 * ws.stride);
    if (k + ws.stride < ws.nw) nxt.load(wn, D, a.st);
    if (cur.go) {
      const V* __restrict__ r = cur.r;
      const V* __restrict__ dinv = cur.dinv;
      V* __restrict__ p = cur.p;
      const int i0 = cur.r0 + lane, nr = cur.r1 - cur.r0;
      V rv[kPerLane], dv[kPerLane], pv[kPerLane];
#pragma unroll
      for (int u = 0; u < kPerLane; ++u)
        if (lane + 32 * u < nr) {
          rv[u] = r[i0 + 32 * u];
          dv[u] = dinv[i0 + 32 * u];
          pv[u] = cur.first ? (V)0 : p[i0 + 32 * u];
        }
#pragma unroll
      for (int u = 0; u < kPerLane; ++u)
        if (lane + 32 * u < nr) {
          const V z = rv[u] * dv[u];
          p[i0 + 32 * u] = cur.first ? z : (V)((double)z + cur.beta * (double)pv[u]);
        }
    }
    cur = nxt;
    wn = wnn;
  }
}

template <typename V>
struct UpdateDesc {
  int r0, r1, tile, go;
  double alpha;
  const SysDev<V>* d;
  V* xlo;
  V* r;
  const V* p;
  const V* q;
  const V* dinv;
  __device__ void load(const Work& w, const SysDev<V>* D, const SysState* st) {
    const SysState& s = st[w.sys];
    d = D + w.sys;
    r0 = w.r0;
    r1 = w.r1;
    tile = w.tile;
    go = active(s);
    alpha = s.alpha;
    xlo = d->xlo;
    r = d->r;
    p = d->p;
    q = d->q;
    dinv = d->dinv;
  }
};

template <typename V>
__global__ void __launch_bounds__(256, ew_min_blocks<V>(2)) kb_update(BatchArgs a) {
  const SysDev<V>* D = static_cast<const SysDev<V>*>(a.desc);
  const WorkStream ws{a.work, *a.nwork, warp_global(), warps_total()};
  if (ws.k >= ws.nw) return;
  const int lane = threadIdx.x & 31;
  UpdateDesc<V> cur, nxt;
  cur.load(ws.at(ws.k), D, a.st);
  Work wn = ws.at(ws.k + ws.stride);
  for (int k = ws.k; k < ws.nw; k += ws.stride) {
    const Work wnn = ws.at(k + 2 * ws.stride);
    if (k + ws.stride < ws.nw) nxt.load(wn, D, a.st);
    if (cur.go) {   // warp-uniform
      V* __restrict__ xlo = cur.xlo;
      V* __restrict__ r = cur.r;
      const V* __restrict__ p = cur.p;
      const V* __restrict__ q = cur.q;
      const V* __restrict__ dinv = cur.dinv;
      const double al = cur.alpha;
      const int i0 = cur.r0 + lane, nr = cur.r1 - cur.r0;
      V xv[kPerLane], pv[kPerLane], rv[kPerLane], qv[kPerLane], dv[kPerLane];
#pragma unroll
      for (int u = 0; u < kPerLane; ++u)
        if (lane + 32 * u < nr) {
          const int i = i0 + 32 * u;
          xv[u] = xlo[i];
          pv[u] = p[i];
          rv[u] = r[i];
          qv[u] = q[i];
          dv[u] = dinv[i];
        }
      double v[2] = {0.0, 0.0};   // rho, |r|^2
#pragma unroll
      for (int u = 0; u < kPerLane; ++u)
        if (lane + 32 * u < nr) {
          const int i = i0 + 32 * u;
          const V xl = (V)((double)xv[u] + al * (double)pv[u]);
          const V ri = (V)((double)rv[u] - al * (double)qv[u]);
          xlo[i] = xl;
          r[i] = ri;
          const V zi = ri * dv[u];
          v[0] = __dadd_rn(v[0], __dmul_rn((double)zi, (double)ri));
          v[1] = __dadd_rn(v[1], __dmul_rn((double)ri, (double)ri));
        }
      v[0] = warp_sum(v[0]);
      v[1] = warp_sum(v[1]);
      put_tile_total<2>(cur.d->tile_tot, cur.tile, v);
    }
    cur = nxt;
    wn = wnn;
  }
}

// The finishing kernels: one CTA of kFinThreads per item (a grid-stride
// loop over the list), an item being a chunk of kFinTiles tile totals of a
// system; a system of more than one chunk is finished by the CTA of its
// last chunk to report.
constexpr int kFinThreads = 256;
constexpr int kFinPer = 8;                          // tile totals per thread
constexpr int kFinTiles = kFinThreads * kFinPer;    // per item

__host__ __device__ __forceinline__ int fin_chunks(int ntiles) {
  return (ntiles + kFinTiles - 1) / kFinTiles;
}

// v (every thread) = the CTA's sum of w: each warp sums its lanes
// (butterfly), then every warp sums the warps' results in warp order.
template <int NQ>
__device__ __forceinline__ void cta_sum(double (&w)[NQ], double (&v)[NQ]) {
  constexpr int kW = kFinThreads / 32;
  __shared__ double part[NQ][kW];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    const double s = warp_sum(w[q]);
    if (lane == 0) part[q][warp] = s;
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NQ; ++q) v[q] = warp_sum(lane < kW ? part[q][lane] : 0.0);
  __syncthreads();   // part is reused
}

// A system's totals from its tile totals, chunk by chunk: the CTA of item
// (sys, chunk) loads the chunk's tile totals (thread t takes tiles t,
// t + kFinThreads, ..., all loads issued before the first add) and sums
// them with cta_sum; a one-chunk system is done here.  Otherwise the chunk
// total is stored and the chunk's CTA reports on the system's counter; the
// last to report sums the chunk totals in chunk order.  The order depends
// only on the system's tiling.  Returns true (CTA-uniform) in the CTA that
// holds the system's totals in v.
template <int NQ, typename V>
__device__ bool finish_sum(const SysDev<V>& d, unsigned* cnt, int chunk, double (&v)[NQ]) {
  __shared__ int last_sh;
  const int t0 = chunk * kFinTiles, t1 = min(d.ntiles, t0 + kFinTiles);
  double ld[kFinPer][NQ];
#pragma unroll
  for (int k = 0; k < kFinPer; ++k) {
    const int t = t0 + (int)threadIdx.x + k * kFinThreads;
#pragma unroll
    for (int q = 0; q < NQ; ++q)
      ld[k][q] = t < t1 ? __ldcg(d.tile_tot + (size_t)t * kPartQ + q) : 0.0;
  }
  double w[NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    w[q] = 0.0;
#pragma unroll
    for (int k = 0; k < kFinPer; ++k) w[q] = __dadd_rn(w[q], ld[k][q]);
  }
  cta_sum<NQ>(w, v);
  const int nch = fin_chunks(d.ntiles);
  if (nch == 1) return true;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) d.chunk_tot[(size_t)chunk * kPartQ + q] = v[q];
    __threadfence();
    last_sh = atomicAdd(cnt, 1u) == (unsigned)nch - 1;
  }
  __syncthreads();
  const bool last = last_sh;
  __syncthreads();   // last_sh is reused
  if (!last) return false;
  __threadfence();
#pragma unroll
  for (int q = 0; q < NQ; ++q) w[q] = 0.0;
  for (int c = threadIdx.x; c < nch; c += kFinThreads)
#pragma unroll
    for (int q = 0; q < NQ; ++q)
      w[q] = __dadd_rn(w[q], __ldcg(d.chunk_tot + (size_t)c * kPartQ + q));
  cta_sum<NQ>(w, v);
  if (threadIdx.x == 0) *cnt = 0u;   // ready for the next finishing kernel
  return true;
}

// Per system after kb_update: rho, beta, the iteration count and the
// refinement trigger; a system due an update lists its tiles for the
// refinement kernels.
template <typename V>
__global__ void __launch_bounds__(kFinThreads) kb_beta(BatchArgs a) {
  const SysDev<V>* D = static_cast<const SysDev<V>*>(a.desc);
  __shared__ int base_sh;
  const int nf = *a.nfin;
  for (int k = blockIdx.x; k < nf; k += gridDim.x) {
    const FinItem it = a.fin[k];
    const int sys = it.sys;
    SysState& s = a.st[sys];
    if (!active(s)) continue;   // CTA-uniform
    const SysDev<V>& d = D[sys];
    double v[2];
    if (!finish_sum<2>(d, &s.fin_cnt, it.chunk, v)) continue;
    if (threadIdx.x == 0) {
      int base = -1;
      s.rho_old = s.rho;
      s.rho = v[0];
      s.beta = __ddiv_rn(s.rho, s.rho_old);
      s.rr = v[1];
      s.iter += 1;
      s.first = 0;
      const double tb = d.tol * d.tol * s.bnorm2;
      // FP32 iterates drift from the FP64 recurrence as the condition
      // number grows (2M-cell polyhedral Poisson: 4,338 iterations against
      // 1,218 with refinements only on a 10x residual drop); refining at
      // least every kRuEvery iterations keeps them within 1 % of FP64.
      const bool periodic = sizeof(V) == 4 && s.iter - s.iter_ru >= kRuEvery;
      if (s.rr < a.ru_delta2 * s.rr_ru || s.rr <= tb || s.iter >= d.maxit ||
          !(s.rr == s.rr) || periodic) {
        s.need_ru = 1;
        base = atomicAdd(a.ru.count, d.ntiles);
      }
      base_sh = base;
    }
    __syncthreads();
    const int base = base_sh;
    __syncthreads();   // base_sh is reused by the next system
    if (base >= 0)     // list this system's tiles for the refinement kernels
      for (int t = threadIdx.x; t < d.ntiles; t += kFinThreads)
        a.ru.items[base + t] = Work{sys, t, d.tiles[t], d.tiles[t + 1],
                                    d.row[d.tiles[t]], d.row[d.tiles[t + 1]]};
  }
  // The last CTA opens the refinement kernels' gate when any system is due
  // an update (or was admitted and waits for its first residual).
  if (a.use_gate) {
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      if (atomicAdd(a.gate_cnt, 1u) == gridDim.x - 1) {
        *a.gate_cnt = 0u;
        __threadfence();
        const int due = *(volatile int*)a.ru.count;
        cudaGraphSetConditional(a.ru_gate, due > 0 ? 1u : 0u);
      }
    }
  }
}

// Per system after kb_spmv: alpha = rho / p.q (breakdown when p.q <= 0 or
// NaN).
template <typename V>
__global__ void __launch_bounds__(kFinThreads) kb_alpha(BatchArgs a) {
  const SysDev<V>* D = static_cast<const SysDev<V>*>(a.desc);
  const int nf = *a.nfin;
  for (int k = blockIdx.x; k < nf; k += gridDim.x) {
    const FinItem it = a.fin[k];
    SysState& s = a.st[it.sys];
    if (!active(s)) continue;   // CTA-uniform
    double v[1];
    if (!finish_sum<1>(D[it.sys], &s.fin_cnt, it.chunk, v)) continue;
    if (threadIdx.x == 0) {
      if (!(v[0] > 0.0)) s.status = kBreakdown;
      else s.alpha = __ddiv_rn(s.rho, v[0]);
    }
  }
}

template <typename V>
__global__ void __launch_bounds__(256) kb_ru_fold(BatchArgs a) {
  const SysDev<V>* D = static_cast<const SysDev<V>*>(a.desc);
  const int nw = *a.ru.count;
  const int lane = threadIdx.x & 31;
  for (int k = warp_global(); k < nw; k += warps_total()) {
    const Work w = a.ru.items[k];
    const SysState& s = a.st[w.sys];
    if (!(s.status == kActive && s.need_ru)) continue;
    double* __restrict__ x = D[w.sys].x;
    V* __restrict__ xlo = D[w.sys].xlo;
    const int i0 = w.r0 + lane, nr = w.r1 - w.r0;
    double xv[kPerLane];
    V lv[kPerLane];
#pragma unroll
    for (int u = 0; u < kPerLane; ++u)
      if (lane + 32 * u < nr) {
        xv[u] = x[i0 + 32 * u];
        lv[u] = xlo[i0 + 32 * u];
      }
#pragma unroll
    for (int u = 0; u < kPerLane; ++u)
      if (lane + 32 * u < nr) {
        x[i0 + 32 * u] = __dadd_rn(xv[u], (double)lv[u]);
        xlo[i0 + 32 * u] = (V)0;
      }
  }
}

// q = A p with FP64 row sums, p.q per tile, alpha per system.
template <typename V, typename VT>
struct SpmvWork {
  using Item = Work;
  const SysDev<V>* D;
  SysState* st;
  const Work* work;
  int nw;
  double acc;     // this thread's p_i q_i in the current tile
  int ck;         // item whose pointers are cached below
  const V* cp;
  V* cq;
  __device__ int count() const { return nw; }
  __device__ Work item(int k) const { return work[k]; }
  __device__ void resolve(const Work& w, TileRes<VT>& rs) const {
    const SysDev<V>& d = D[w.sys];
    rs.row = d.row;
    rs.col = d.col;
    if constexpr (sizeof(VT) == 4) rs.val = d.val32;
    else rs.val = d.val;
    rs.skip = !active(st[w.sys]);
  }
  __device__ void row(int k, int i, const VT* v, const int* c, int len) {
    if (k != ck) {
      ck = k;
      const SysDev<V>& d = D[work[k].sys];
      cp = d.p;
      cq = d.q;
    }
    const V* __restrict__ p = cp;
    double s = 0.0;
#pragma unroll 1
    for (int j0 = 0; j0 < len; j0 += 8) {
      double pv[8], vv[8];
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (j0 + u < len) {
          vv[u] = (double)v[j0 + u];
          pv[u] = (double)__ldg(p + c[j0 + u]);
        }
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (j0 + u < len) s = __dadd_rn(s, __dmul_rn(vv[u], pv[u]));
    }
    const V qi = (V)s;
    cq[i] = qi;
    acc = __dadd_rn(acc, __dmul_rn((double)__ldg(p + i), (double)qi));
  }
  __device__ void tile_end(int k) {
    const Work w = work[k];
    const SysDev<V>& d = D[w.sys];
    double v[1] = {acc};
    acc = 0.0;
    if (cta_tile_total<1>(d.warp_part, d.tile_cnt, w.tile, v))
      put_tile_total<1>(d.tile_tot, w.tile, v);
  }
};

// Work-list items as tiles of the producer-warp streamer; SKIP decides
// which items have nothing to do in this launch.
template <typename V, int KIND>
struct BatchTiles {
  static constexpr bool kRowPatterns = true;   // structured systems' tiles
  const SysDev<V>* D;
  const SysState* st;
  const Work* work;
  int nw;
  __device__ int count() const { return nw; }
  __device__ TileDesc desc(int k) const {
    const Work w = work[k];
    const SysDev<V>& d = D[w.sys];
    TileDesc t;
    t.row = d.row;
    t.col = d.col;
    t.pat = d.pat;
    t.tab = d.tab;
    t.npat = d.npat;
    t.val = d.val;
    t.r0 = w.r0;
    t.r1 = w.r1;
    t.j0 = w.j0;
    t.j1 = w.j1;
    const SysState& s = st[w.sys];
    t.skip = KIND == 0 ? !active(s) : !(s.status == kInit || (s.status == kActive && s.need_ru));
    t.aux0 = KIND == 0 ? (const void*)d.p : (const void*)&D[w.sys];
    t.aux1 = KIND == 0 ? (void*)d.q : nullptr;
    t.aux2 = w.sys;
    t.aux3 = w.tile;
    return t;
  }
};

// Tile reduction for the producer-warp streamer (tf_tile2.cuh), by its
// reducer warp: every consumer warp sums its lanes and parks the result in
// shared memory (slot it & 1, tile_end), consumer thread 0 adds the tile's
// system and index (tile_id); the reducer warp sums the kWarps partials in
// warp order -- the order cta_tile_total uses -- and stores the tile's
// totals.  The consumers never wait for a report.
__shared__ double g_tile_part[2][kPartQ][kWarps];
struct TileId {
  int sys, tile, skip;
};
__shared__ TileId g_tile_id[2];

template <int NQ>
__device__ __forceinline__ void park_partials(double (&v)[NQ], int it) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q) v[q] = warp_sum(v[q]);
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) g_tile_part[it & 1][q][warp] = v[q];
  }
}

// The reducer warp: the parked tile's totals, in warp order.
template <int NQ>
__device__ __forceinline__ void sum_partials(double (&v)[NQ], int it) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    const double w = lane < kWarps ? g_tile_part[it & 1][q][lane] : 0.0;
    v[q] = warp_sum(w);
  }
}

template <typename V>
struct SpmvOp2 {
  static constexpr bool kReducer = true;
  const SysDev<V>* D;
  SysState* st;
  const Work* work;
  double acc;
  const V* p;
  V* q;
  __device__ void begin(int, TileAux aux) {
    p = static_cast<const V*>(aux.a0);
    q = static_cast<V*>(aux.a1);
  }
  __device__ double gather(int c) const { return (double)__ldg(p + c); }
  __device__ double row_init(int) const { return 0.0; }
  __device__ double combine(double a, double prod) const { return __dadd_rn(a, prod); }
  __device__ void row_done(int i, double sum) {
    const V qi = (V)sum;
    q[i] = qi;
    acc = __dadd_rn(acc, __dmul_rn((double)__ldg(p + i), (double)qi));
  }
  __device__ void tile_end(int it) {
    double v[1] = {acc};
    acc = 0.0;
    park_partials<1>(v, it);
  }
  __device__ void tile_id(int it, int skip, TileAux aux) {
    g_tile_id[it & 1] = TileId{aux.i2, aux.i3, skip};
  }
  __device__ void reduce_tile(int it) {
    const TileId id = g_tile_id[it & 1];
    if (id.skip) return;
    double v[1];
    sum_partials<1>(v, it);
    put_tile_total<1>(D[id.sys].tile_tot, id.tile, v);
  }
};

// G = 0: the two-phase consumers; G = -1: warp groups, width per tile.
template <typename V, typename VT, int G>
__global__ void __launch_bounds__(kCsr2RedThreads, 2) kb_spmv(BatchArgs a) {
  if constexpr (sizeof(VT) == 8) {
    BatchTiles<V, 0> src{static_cast<const SysDev<V>*>(a.desc), a.st, a.work, *a.nwork};
    SpmvOp2<V> op{static_cast<const SysDev<V>*>(a.desc), a.st, a.work, 0.0, nullptr, nullptr};
    stream_csr2<kRows, kNnzCap, kStages, G>(src, op);
  } else {
    // FP32 values: the one-thread-per-row streamer (kRows threads do the
    // work; the extra warp only joins the CTA-wide barriers).
    SpmvWork<V, VT> w{static_cast<const SysDev<V>*>(a.desc), a.st, a.work, *a.nwork, 0.0, -1,
                      nullptr, nullptr};
    stream_items<kRows, kNnzCap, VT, kStages>(w);
  }
}

// A system's refinement step after its FP64 residual: v = {|r|^2, rho,
// |b|^2 (first time)}.  Run by one thread.
template <typename V>
__device__ void res_finish(SysState& s, const SysDev<V>& d, const double (&v)[3]) {
  if (s.status == kInit) {
    s.bnorm2 = v[2];
    s.status = kActive;
    s.first = 1;
    s.iter = 0;
  }
  s.n_ru += 1;
  s.iter_ru = s.iter;
  const double bn = s.bnorm2 > 0.0 ? __dsqrt_rn(s.bnorm2) : 1.0;
  s.res_true = __ddiv_rn(__dsqrt_rn(v[0]), bn);
  s.need_ru = 0;
  if (s.res_true <= d.tol) {
    s.status = kConverged;
  } else if (s.iter >= d.maxit) {
    s.status = kMaxIter;
  } else if (!(v[0] == v[0])) {
    s.status = kBreakdown;
  } else {
    s.rr = v[0];
    s.rr_ru = v[0];
    s.rho = v[1];
    if (!s.first) s.beta = __ddiv_rn(s.rho, s.rho_old);
  }
}

// r = b - A x in FP64 for the producer-warp streamer; new systems also
// form dinv and |b|^2.
template <typename V>
struct ResOp2 {
  static constexpr bool kReducer = true;
  const SysDev<V>* D;
  SysState* st;
  const Work* work;
  double rr, rho, bb;
  const SysDev<V>* d;
  bool init;
  __device__ void begin(int, TileAux aux) {
    d = static_cast<const SysDev<V>*>(aux.a0);
    init = st[aux.i2].status == kInit;
  }
  __device__ double gather(int c) const { return d->x[c]; }
  __device__ double row_init(int i) const { return d->b[i]; }
  __device__ double combine(double a, double prod) const { return __dsub_rn(a, prod); }
  __device__ void row_done(int i, double s) {
    if (init) {
      const double aii = d->val[d->dia[i]];
      d->dinv[i] = (V)__drcp_rn(aii);
      bb = __dadd_rn(bb, __dmul_rn(d->b[i], d->b[i]));
    }
    const V ri = (V)s;
    d->r[i] = ri;
    const V zi = ri * d->dinv[i];
    rr = __dadd_rn(rr, __dmul_rn(s, s));
    rho = __dadd_rn(rho, __dmul_rn((double)zi, (double)ri));
  }
  __device__ void tile_end(int it) {
    double v[3] = {rr, rho, bb};
    rr = rho = bb = 0.0;
    park_partials<3>(v, it);
  }
  __device__ void tile_id(int it, int skip, TileAux aux) {
    g_tile_id[it & 1] = TileId{aux.i2, aux.i3, skip};
  }
  __device__ void reduce_tile(int it) {
    const TileId id = g_tile_id[it & 1];
    if (id.skip) return;
    double v[3];
    sum_partials<3>(v, it);
    put_tile_total<3>(D[id.sys].tile_tot, id.tile, v);
  }
};

template <typename V, int G>
__global__ void __launch_bounds__(kCsr2RedThreads, 2) kb_ru_res(BatchArgs a) {
  BatchTiles<V, 1> src{static_cast<const SysDev<V>*>(a.desc), a.st, a.ru.items, *a.ru.count};
  ResOp2<V> op{static_cast<const SysDev<V>*>(a.desc), a.st, a.ru.items, 0.0, 0.0, 0.0,
               nullptr, false};
  stream_csr2<kRows, kNnzCap, kStages, G>(src, op);
}

// Per system after kb_ru_res: the refinement's convergence test and the
// restarted scalars (res_finish); then the refinement list is emptied for
// the next iteration.
template <typename V>
__global__ void __launch_bounds__(kFinThreads) kb_ru_finish(BatchArgs a) {
  const SysDev<V>* D = static_cast<const SysDev<V>*>(a.desc);
  const int nf = *a.nfin;
  for (int k = blockIdx.x; k < nf; k += gridDim.x) {
    const FinItem it = a.fin[k];
    SysState& s = a.st[it.sys];
    if (!(s.status == kInit || (s.status == kActive && s.need_ru))) continue;   // CTA-uniform
    double v[3];
    if (!finish_sum<3>(D[it.sys], &s.fin_cnt, it.chunk, v)) continue;
    if (threadIdx.x == 0) res_finish(s, D[it.sys], v);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *a.ru.count = 0;
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
struct Arena {
  char* base = nullptr;
  size_t size = 0;
  std::map<size_t, size_t> free_;   // offset -> length
  int init(size_t bytes) {
    size = bytes;
    TF_CUDA_TRY(cudaMalloc((void**)&base, bytes));
    free_.clear();
    free_[0] = bytes;
    return TF_OK;
  }
  static size_t up(size_t v) { return (v + 255) & ~size_t(255); }
  bool alloc(size_t bytes, size_t* off) {
    bytes = up(bytes);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= bytes) {
        *off = it->first;
        const size_t rest = it->second - bytes;
        const size_t o = it->first + bytes;
        free_.erase(it);
        if (rest) free_[o] = rest;
        return true;
      }
    }
    return false;
  }
  void release(size_t off, size_t bytes) {
    bytes = up(bytes);
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  size_t free_bytes() const {
    size_t s = 0;
    for (auto& kv : free_) s += kv.second;
    return s;
  }
};

// ---------------------------------------------------------------------------
// Host preparation
// ---------------------------------------------------------------------------
// A matrix structure as the engine iterates it: 0-based CSR (renumbered by
// reverse Cuthill-McKee when the caller's numbering scatters the gathers;
// every row keeps its entries in storage order, so row sums are those of
// the caller's matrix) and its row tiles.  Once a system using it is
// admitted, one device copy in the arena serves every system with the same
// structure; the engine keeps it resident after they retire (a structure
// cache keyed by the caller's arrays) until the memory is needed.
struct Structure {
  int n = 0;
  long long nnz = 0;
  std::vector<int> row, dia;   // 0-based, n + 1 + 8 and n + 8
  std::vector<int> col;        // 0-based, nnz + 8; freed once on the device
  std::vector<int> tiles;      // row boundaries of the tiles
  std::vector<int> tile_j;     // entry boundaries of the tiles (row[tiles[t]])
  std::vector<int> perm;       // renumbered: row i is the caller's row perm[i]
  // Row patterns (npat > 0): on the device these replace the columns.
  int npat = 0;
  std::vector<unsigned char> pat;
  std::vector<int> tab;
  // engine lock from here on
  int ready = 0;               // 0 being prepared, 1 prepared, < 0 -(its error status)
  bool resident = false;       // a device copy exists (or is being uploaded)
  size_t off = 0, bytes = 0, o_row = 0, o_col = 0, o_dia = 0, o_tiles = 0, o_pat = 0,
         o_tab = 0;
  int users = 0;               // admitted systems reading the device copy
  uint64_t last_use = 0;       // eviction order: least recently used first
  int ntiles() const { return (int)tiles.size() - 1; }
};

// The structure cache's key: the caller's arrays (addresses and sizes) and
// a 64-bit FNV-1a hash of row and dia and of every 16th column index (and
// the last 16).  A structure changed in place at the same addresses in
// those entries is seen as new.
struct StructKey {
  const int* row;
  const int* col;
  const int* dia;
  int n;
  long long nnz;
  uint64_t hash;
  bool operator<(const StructKey& o) const {
    return std::tie(row, col, dia, n, nnz, hash) <
           std::tie(o.row, o.col, o.dia, o.n, o.nnz, o.hash);
  }
};

inline uint64_t fnv1a(uint64_t h, const int* p, long long count, long long step) {
  for (long long i = 0; i < count; i += step) {
    h ^= (uint32_t)p[i];
    h *= 1099511628211ull;
  }
  return h;
}

StructKey struct_key(int n, long long nnz, const int* row, const int* col, const int* dia) {
  uint64_t h = 1469598103934665603ull;
  h = fnv1a(h, row, (long long)n + 1, 1);
  h = fnv1a(h, dia, n, 1);
  h = fnv1a(h, col, nnz, 16);
  const long long tail = std::min<long long>(nnz, 16);
  h = fnv1a(h, col + (nnz - tail), tail, 1);
  return StructKey{row, col, dia, n, nnz, h};
}

// Checks the caller's 1-based Matrix_Type structure, converts it, renumbers
// a scattered numbering, cuts the tiles and, with want_patterns, replaces
// the columns by row patterns where every row fits one of kPatMax patterns
// (structured hex blocks: 1 byte per row instead of 4 per entry).
int prepare_structure(Structure& S, int n, long long nnz, const int* row, const int* col,
                      const int* dia, bool want_patterns) {
  if (n < 1 || nnz < n || !row || !col || !dia) return TF_ERR_ARG;
  if (row[0] != 1 || (long long)row[n] - 1 != nnz) return TF_ERR_LAYOUT;
  S.n = n;
  S.nnz = nnz;
  S.row.resize((size_t)n + 1 + 8);
  S.col.resize((size_t)nnz + 8);
  S.dia.resize((size_t)n + 8);
  for (int i = 0; i <= n; ++i) S.row[i] = row[i] - 1;
  for (size_t i = n + 1; i < S.row.size(); ++i) S.row[i] = S.row[n];
  for (long long j = 0; j < nnz; ++j) {
    if (col[j] < 1 || col[j] > n) return TF_ERR_LAYOUT;
    S.col[j] = col[j] - 1;
  }
  for (int i = 0; i < n; ++i) {
    if (S.row[i + 1] < S.row[i]) return TF_ERR_LAYOUT;
    const int d = dia[i] - 1;
    if (d < S.row[i] || d >= S.row[i + 1] || S.col[d] != i) return TF_ERR_LAYOUT;
    S.dia[i] = d;
  }
  // Scattered numbering: renumber by reverse Cuthill-McKee (see
  // tf_renumber.cu); kept when it cuts the gathered lines by 20 %.
  S.perm.clear();
  if (n >= kRenumberMinRows && !getenv("TF_NO_RENUMBER")) {
    const double before = tf_gather_lines_per_warp(S.row.data(), S.col.data(), n, 0);
    if (before > kRenumberLines) {
      std::vector<int> order, inv(n);
      tf_rcm_order(S.row, S.col, n, order);
      for (int i = 0; i < n; ++i) inv[order[i]] = i;
      std::vector<int> row2(S.row.size()), col2(S.col.size(), 0), dia2(S.dia.size(), 0);
      row2[0] = 0;
      for (int i = 0; i < n; ++i) {
        const int o = order[i], js = S.row[o], len = S.row[o + 1] - js;
        const int r = row2[i];
        for (int k = 0; k < len; ++k) col2[r + k] = inv[S.col[js + k]];
        dia2[i] = r + (S.dia[o] - js);
        row2[i + 1] = r + len;
      }
      for (size_t i = n + 1; i < row2.size(); ++i) row2[i] = row2[n];
      if (tf_gather_lines_per_warp(row2.data(), col2.data(), n, 0) <= 0.8 * before) {
        S.row.swap(row2);
        S.col.swap(col2);
        S.dia.swap(dia2);
        S.perm.swap(order);
      }
    }
  }
  // tiles: <= kRows rows and <= kNnzCap entries each
  S.tiles.clear();
  S.tiles.push_back(0);
  int r0 = 0;
  while (r0 < n) {
    int r1 = r0;
    while (r1 < n && r1 - r0 < kRows && S.row[r1 + 1] - S.row[r0] <= kNnzCap) ++r1;
    if (r1 == r0) return TF_ERR_LAYOUT;   // one row longer than a tile stage
    // A tile cut short by its entry cap between kRows/2 and kRows rows is
    // trimmed to kRows/2, so the streamer can give each row 2 threads;
    // shorter tiles keep their rows (2 or 4 threads per row as they are:
    // halving them would double the per-tile costs).
    if (r1 < n && r1 - r0 > kRows / 2 && r1 - r0 < kRows) r1 = r0 + kRows / 2;
    S.tiles.push_back(r1);
    r0 = r1;
  }
  S.tile_j.resize(S.tiles.size());
  for (size_t t = 0; t < S.tiles.size(); ++t) S.tile_j[t] = S.row[S.tiles[t]];
  S.npat = want_patterns ? tf_find_row_patterns(S.row, S.col, n, S.pat, S.tab) : 0;
  if (S.npat == 0) {
    S.pat.clear();
    S.tab.clear();
  }
  return TF_OK;
}

// One system ready to upload: its structure (shared) and its values,
// right-hand side and start vector in the structure's row order.
struct HostSys {
  std::shared_ptr<Structure> st;
  StructKey key{};
  int n = 0;
  long long nnz = 0;
  std::vector<double> val, b, x0;
  const double* val_in = nullptr;   // the caller's values, used in place (borrowed)
  std::vector<float> val32;
  double tol = 1e-10;
  int maxit = 10000;
  const double* values() const { return val_in ? val_in : val.data(); }
};

// The per-system arrays of h in S's order (val permuted row by row with the
// structure when it was renumbered).  borrow: the caller's values stay
// where they are until the upload (a structure in the caller's numbering
// needs no copy of them).
int prepare_values(HostSys& h, const Structure& S, const int* row, const double* val,
                   const double* b, const double* x0, int use_val32, bool borrow) {
  if (!val || !b) return TF_ERR_ARG;
  const int n = S.n;
  const long long nnz = S.nnz;
  h.n = n;
  h.nnz = nnz;
  h.val_in = nullptr;
  if (S.perm.empty()) {
    if (borrow && !use_val32) {
      h.val_in = val;
    } else {
      h.val.assign(val, val + nnz);
      h.val.resize((size_t)nnz + 8, 0.0);
    }
    h.b.assign(b, b + n);
    if (x0) h.x0.assign(x0, x0 + n);
    else h.x0.assign(n, 0.0);
  } else {
    h.val.assign((size_t)nnz + 8, 0.0);
    h.b.resize(n);
    h.x0.assign(n, 0.0);
    for (int i = 0; i < n; ++i) {
      const int o = S.perm[i];
      const long long js = row[o] - 1, len = row[o + 1] - row[o];
      std::copy(val + js, val + js + len, h.val.begin() + S.row[i]);
      h.b[i] = b[o];
      if (x0) h.x0[i] = x0[o];
    }
  }
  if (use_val32) {
    h.val32.resize((size_t)nnz + 8);
    for (long long j = 0; j < nnz + 8; ++j) h.val32[j] = (float)h.val[j];
  }
  return TF_OK;
}

// Byte layout of one system's own segment (its structure lives in a
// segment of its own, shared).
struct Layout {
  size_t val, val32, b, x, xlo, r, p, q, dinv, tile_tot, chunk_tot, warp_part, tile_cnt, total;
};

Layout layout_for(const HostSys& h, int ntiles, size_t vsz, int use_val32) {
  Layout L{};
  size_t o = 0;
  auto take = [&](size_t bytes) { size_t r = o; o = Arena::up(o + bytes); return r; };
  const size_t n8 = (size_t)h.n + 8;
  L.val = take(((size_t)h.nnz + 8) * 8);
  L.val32 = use_val32 ? take(((size_t)h.nnz + 8) * 4) : 0;
  L.b = take(n8 * 8);
  L.x = take(n8 * 8);
  L.xlo = take(n8 * vsz);
  L.r = take(n8 * vsz);
  L.p = take(n8 * vsz);
  L.q = take(n8 * vsz);
  L.dinv = take(n8 * vsz);
  L.tile_tot = take((size_t)ntiles * kPartQ * 8);
  L.chunk_tot = take((size_t)fin_chunks(ntiles) * kPartQ * 8);
  if (use_val32) {   // the FP32-value SpMV's per-warp partials
    L.warp_part = take((size_t)ntiles * kWarps * kPartQ * 8);
    L.tile_cnt = take((size_t)ntiles * 4);
  }
  L.total = o;
  return L;
}

struct Slot {
  int used = 0;            // 1: admitted; 2: reserved, its copies in flight
  int listed = 0;          // in a work list already (its first residual is queued)
  size_t off = 0, bytes = 0;
  int n = 0, ntiles = 0;
  double done_ms = -1.0;   // wall time from tf_batch_run's start to completion
  Layout L{};
  std::shared_ptr<Structure> st;
};

// Copies from pageable host memory through two pinned buffers in turn: a
// thread fills one while the DMA of the other runs, so host-to-device
// copies run at the DMA rate instead of the driver's staged pageable rate,
// and several threads copying at once do not serialise on its staging.
struct Stager {
  static constexpr size_t kBytes = (size_t)8 << 20;   // per buffer
  unsigned char* buf[2] = {nullptr, nullptr};
  cudaEvent_t done[2] = {nullptr, nullptr};   // the last DMA from each buffer
  int k = 0;
  int init() {
    for (int j = 0; j < 2; ++j) {
      TF_CUDA_TRY(cudaMallocHost((void**)&buf[j], kBytes));
      TF_CUDA_TRY(cudaEventCreateWithFlags(&done[j], cudaEventDisableTiming));
    }
    return TF_OK;
  }
  ~Stager() {
    for (int j = 0; j < 2; ++j) {
      if (done[j]) {
        cudaEventSynchronize(done[j]);
        cudaEventDestroy(done[j]);
      }
      if (buf[j]) cudaFreeHost(buf[j]);
    }
  }
  cudaError_t copy(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    const unsigned char* from = static_cast<const unsigned char*>(src);
    unsigned char* to = static_cast<unsigned char*>(dst);
    while (bytes) {
      const size_t c = std::min(bytes, kBytes);
      cudaError_t e = cudaEventSynchronize(done[k]);   // its last DMA has drained
      if (e != cudaSuccess) return e;
      memcpy(buf[k], from, c);
      e = cudaMemcpyAsync(to, buf[k], c, cudaMemcpyHostToDevice, s);
      if (e == cudaSuccess) e = cudaEventRecord(done[k], s);
      if (e != cudaSuccess) return e;
      k ^= 1;
      from += c;
      to += c;
      bytes -= c;
    }
    return cudaSuccess;
  }
};

// A slot and arena space held for a system whose copies are in flight.
struct Reservation {
  int slot = -1;
  bool new_struct = false;   // this system uploads its structure
  Layout L{};
};

}  // namespace tfb

using namespace tfb;

// ---------------------------------------------------------------------------
// The engine (one per tf_batch / tf_server)
// ---------------------------------------------------------------------------
struct tf_batch_s {
  tf_ctx_s* ctx = nullptr;
  tf_batch_opts opts{};
  size_t vsz = 4;
  Arena arena;
  int max_sys = 0;
  std::vector<Slot> slots;
  void* d_desc = nullptr;           // SysDev<V>[max_sys]
  SysState* d_state = nullptr;
  SysState* h_state = nullptr;      // the latest known state of every slot
  unsigned* d_gate_cnt = nullptr;
  // Staging of the descriptors and initial states of committed systems
  // (pinned, one entry per slot: copies ahead of a running sweep stay
  // asynchronous).
  unsigned char* h_desc_stage = nullptr;
  SysState* h_init_stage = nullptr;

  // A work list -- the (system, tile) items, the refinement items of new
  // systems, the finishing kernels' items -- with its device buffers,
  // pinned host buffers and the sweep graph bound to them.  The batch API
  // uses one; the server alternates two, building and uploading the next
  // sweep's list while the current sweep runs.
  struct ListSet {
    Work* d_work = nullptr;
    Work* d_ru = nullptr;          // refinement work list (same capacity)
    FinItem* d_fin = nullptr;
    int* d_cnt = nullptr;          // work items, refinement items, finishing items
    int work_cap = 0, fin_cap = 0;
    Work* h_work = nullptr;        // pinned staging of the lists
    Work* h_ru = nullptr;
    FinItem* h_fin = nullptr;
    int* h_cnt = nullptr;
    int h_work_cap = 0, h_ru_cap = 0, h_fin_cap = 0;
    SysState* h_state = nullptr;   // pinned: every slot's state after this list's last sweep
    cudaGraphExec_t graph = nullptr;
    cudaEvent_t done = nullptr;    // this list's last sweep, state copy included
    std::vector<int> slots;        // the systems listed
    int nwork = 0, nru = 0, nfin = 0;
    long long rows = 0, nnz = 0;   // rows and entries of the listed systems
    double bytes = 0.0;            // their inner iteration's algorithmic bytes
  };
  ListSet ls[2];
  int nwork = 0;                   // items of the last list built

  // Pinned staging for uploads, kept for later calls (one per copying thread).
  std::mutex stager_mu;
  std::vector<std::unique_ptr<Stager>> stagers;
  std::unique_ptr<Stager> take_stager() {
    {
      std::lock_guard<std::mutex> lk(stager_mu);
      if (!stagers.empty()) {
        std::unique_ptr<Stager> p = std::move(stagers.back());
        stagers.pop_back();
        return p;
      }
    }
    std::unique_ptr<Stager> p(new Stager());
    if (p->init() != TF_OK) return nullptr;   // copies go without staging then
    return p;
  }
  void give_stager(std::unique_ptr<Stager> p) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(stager_mu);
    stagers.push_back(std::move(p));
  }
  int grid_pupdate = 1, grid_update = 1, grid_fold = 1, grid_tile = 1, grid_fin = 1;
  int sweeps = 0;
  long long total_iters = 0;
  // Per sweep of the last tf_batch_run (tf_batch_sweep): systems running at
  // its launch with their rows and entries, work items (tiles) of the list,
  // wall time of the sweep (launch to state read), kernel times (profiling).
  std::vector<tf_batch_sweep> trace;
  double sweep_kms[kKernels] = {};   // the last profiled sweep's kernel times
  // Upload time over all adds (tf_batch_upload_ms): host preparation summed
  // over the systems, the admitting thread's wait for it, and admission.
  double up_prep_ms = 0.0, up_wait_ms = 0.0, up_admit_ms = 0.0;

  ~tf_batch_s() {
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (ListSet& L : ls) {
      if (L.graph) cudaGraphExecDestroy(L.graph);
      if (L.done) cudaEventDestroy(L.done);
      for (void* p : {(void*)L.d_work, (void*)L.d_ru, (void*)L.d_fin, (void*)L.d_cnt})
        if (p) cudaFree(p);
      for (void* p : {(void*)L.h_work, (void*)L.h_ru, (void*)L.h_fin, (void*)L.h_cnt,
                      (void*)L.h_state})
        if (p) cudaFreeHost(p);
    }
    if (arena.base) cudaFree(arena.base);
    for (void* p : {d_desc, (void*)d_state, (void*)d_gate_cnt})
      if (p) cudaFree(p);
    for (void* p : {(void*)h_state, (void*)h_desc_stage, (void*)h_init_stage})
      if (p) cudaFreeHost(p);
  }

  // Shared memory of the tile kernels: the producer-warp streamer (FP64
  // values) and the one-thread-per-row streamer (FP32 values).
  static size_t smem_csr2() { return Csr2Layout<kRows, kNnzCap, kStages>::kSmemBytes; }
  static size_t smem_rows32() { return TileLayout<kRows, kNnzCap, float, kStages>::kSmemBytes; }

  BatchArgs args(const ListSet& L) const {
    return BatchArgs{d_desc,      d_state,       L.d_work, L.d_cnt, opts.ru_delta * opts.ru_delta,
                     RuList{L.d_ru, L.d_cnt + 1}, L.d_fin, L.d_cnt + 2, d_gate_cnt, 0, 0};
  }

  // The kernels of an iteration, in launch order (tf_batch_kernel_ms).
  struct Launch {
    const void* fn;
    int grid, block;
    size_t smem;
  };
  template <typename V>
  std::vector<Launch> iteration_kernels(const ListSet& L) const {
    // The finishing kernels need no more CTAs than the list can hold items
    // (a single large system has a handful).
    const int gf = std::max(1, std::min(grid_fin, L.fin_cap));
    const void* spmv = opts.val_fp32         ? (const void*)kb_spmv<V, float, 0>
                       : opts.two_phase_rows ? (const void*)kb_spmv<V, double, 0>
                                             : (const void*)kb_spmv<V, double, -1>;
    const int spmv_block = opts.val_fp32 ? kRows : kCsr2RedThreads;
    const size_t spmv_smem = opts.val_fp32 ? smem_rows32() : smem_csr2();
    const void* ru_res = opts.two_phase_rows ? (const void*)kb_ru_res<V, 0>
                                             : (const void*)kb_ru_res<V, -1>;
    return {{(const void*)kb_pupdate<V>, grid_pupdate, 256, 0},
            {spmv, grid_tile, spmv_block, spmv_smem},
            {(const void*)kb_alpha<V>, gf, kFinThreads, 0},
            {(const void*)kb_update<V>, grid_update, 256, 0},
            {(const void*)kb_beta<V>, gf, kFinThreads, 0},
            {(const void*)kb_ru_fold<V>, grid_fold, 256, 0},
            {ru_res, grid_tile, kCsr2RedThreads, smem_csr2()},
            {(const void*)kb_ru_finish<V>, gf, kFinThreads, 0}};
  }
  // The last three (fold, FP64 residual, test) run only when a system is
  // due a refinement: in the sweep graph they sit in an IF node that
  // kb_beta's last CTA opens.
  static constexpr int kFirstRuKernel = 5;

  // Direct launches of one iteration (profiling: ev receives an event before
  // each kernel and after the last).
  template <typename V>
  int launch_iteration(cudaStream_t s, const BatchArgs& a, const ListSet& L, cudaEvent_t* ev) {
    const std::vector<Launch> ks = iteration_kernels<V>(L);
    int e = 0;
    for (const Launch& k : ks) {
      if (ev) cudaEventRecord(ev[e++], s);
      void* kp[] = {const_cast<BatchArgs*>(&a)};
      TF_CUDA_TRY(cudaLaunchKernel(k.fn, dim3(k.grid), dim3(k.block), kp, k.smem, s));
    }
    if (ev) cudaEventRecord(ev[e], s);
    return TF_OK;
  }

  // Profiling (TF_BATCH_PROFILE set when the batch was created): sweeps run
  // as direct launches with events around every kernel; kern_ms accumulates
  // each kernel's time over the run.
  bool profile = false;
  double kern_ms[kKernels] = {};
  int run_sweep_profiled() {
    cudaStream_t s = ctx->stream;
    ListSet& L = ls[0];
    const BatchArgs a = args(L);
    constexpr int kEv = kKernels + 1;
    std::vector<cudaEvent_t> ev(kEv * opts.sweep_iters);
    for (auto& e : ev) TF_CUDA_TRY(cudaEventCreate(&e));
    for (int it = 0; it < opts.sweep_iters; ++it) {
      const int st = vsz == 4 ? launch_iteration<float>(s, a, L, &ev[kEv * it])
                              : launch_iteration<double>(s, a, L, &ev[kEv * it]);
      if (st != TF_OK) return st;
    }
    TF_CUDA_TRY(cudaMemcpyAsync(L.h_state, d_state, (size_t)max_sys * sizeof(SysState),
                                cudaMemcpyDeviceToHost, s));
    TF_CUDA_TRY(cudaStreamSynchronize(s));
    merge_state(L);
    for (int k = 0; k < kKernels; ++k) sweep_kms[k] = 0.0;
    for (int it = 0; it < opts.sweep_iters; ++it)
      for (int k = 0; k < kKernels; ++k) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, ev[kEv * it + k], ev[kEv * it + k + 1]);
        kern_ms[k] += ms;
        sweep_kms[k] += ms;
      }
    for (auto& e : ev) cudaEventDestroy(e);
    ++sweeps;
    return TF_OK;
  }

  template <typename V>
  int setup_kernels() {
    for (const void* f : {(const void*)kb_spmv<V, double, 0>, (const void*)kb_spmv<V, double, -1>,
                          (const void*)kb_ru_res<V, 0>, (const void*)kb_ru_res<V, -1>})
      TF_CUDA_TRY(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem_csr2()));
    TF_CUDA_TRY(cudaFuncSetAttribute(kb_spmv<V, float, 0>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem_rows32()));
    int per_sm = 1;
    TF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kb_spmv<V, double, 0>,
                                                              kCsr2RedThreads, smem_csr2()));
    grid_tile = std::max(1, per_sm) * ctx->sm_count;
    // The elementwise kernels keep a whole tile per warp in registers: one
    // resident wave each, so no CTA waits for another to leave.
    auto resident = [&](const void* f, int* grid) -> int {
      int n = 1;
      TF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f, 256, 0));
      *grid = std::max(1, n) * ctx->sm_count;
      return TF_OK;
    };
    int st = resident((const void*)kb_pupdate<V>, &grid_pupdate);
    if (st == TF_OK) st = resident((const void*)kb_update<V>, &grid_update);
    if (st == TF_OK) st = resident((const void*)kb_ru_fold<V>, &grid_fold);
    if (st != TF_OK) return st;
    grid_fin = ctx->sm_count * 4;
    return TF_OK;
  }

  // The sweep graph of list set L (it holds L's buffers), ending with the
  // copy of every slot's state into L.h_state.
  int build_sweep(ListSet& L) {
    if (L.graph) {
      cudaGraphExecDestroy(L.graph);
      L.graph = nullptr;
    }
    cudaGraph_t g = nullptr;
    TF_CUDA_TRY(cudaGraphCreate(&g, 0));
    cudaGraphNode_t last = nullptr;
    int st = vsz == 4 ? add_sweep_nodes<float>(g, L, &last) : add_sweep_nodes<double>(g, L, &last);
    cudaError_t e = cudaSuccess;
    if (st == TF_OK) {
      cudaGraphNode_t cp = nullptr;
      e = cudaGraphAddMemcpyNode1D(&cp, g, &last, 1, L.h_state, d_state,
                                   (size_t)max_sys * sizeof(SysState), cudaMemcpyDeviceToHost);
      if (e == cudaSuccess) e = cudaGraphInstantiate(&L.graph, g, 0);
      if (e != cudaSuccess) {
        tf_set_last_cuda_error(e, "batch sweep graph", __FILE__, __LINE__);
        st = TF_ERR_CUDA;
      }
    }
    cudaGraphDestroy(g);
    return st;
  }

  // A sweep as a graph: per iteration pupdate -> spmv -> alpha -> update ->
  // beta -> IF(gate){ fold -> residual -> test }, each iteration's IF node
  // with a conditional handle of its own (kb_beta of that iteration sets it).
  template <typename V>
  int add_sweep_nodes(cudaGraph_t g, const ListSet& L, cudaGraphNode_t* last) {
    const std::vector<Launch> ks = iteration_kernels<V>(L);
    auto add = [](cudaGraph_t gr, const Launch& k, const BatchArgs* a, cudaGraphNode_t dep,
                  cudaGraphNode_t* out) {
      cudaKernelNodeParams p{};
      p.func = const_cast<void*>(k.fn);
      p.gridDim = dim3(k.grid);
      p.blockDim = dim3(k.block);
      p.sharedMemBytes = (unsigned)k.smem;
      void* kp[] = {const_cast<BatchArgs*>(a)};
      p.kernelParams = kp;
      return cudaGraphAddKernelNode(out, gr, dep ? &dep : nullptr, dep ? 1 : 0, &p);
    };
    cudaGraphNode_t dep = nullptr;
    for (int it = 0; it < opts.sweep_iters; ++it) {
      BatchArgs a = args(L);
      cudaError_t e = cudaGraphConditionalHandleCreate(&a.ru_gate, g, 0,
                                                       cudaGraphCondAssignDefault);
      a.use_gate = 1;
      for (int k = 0; k < kFirstRuKernel && e == cudaSuccess; ++k) e = add(g, ks[k], &a, dep, &dep);
      cudaGraphNodeParams cp{};
      if (e == cudaSuccess) {
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = a.ru_gate;
        cp.conditional.type = cudaGraphCondTypeIf;
        cp.conditional.size = 1;
        e = cudaGraphAddNode(&dep, g, &dep, 1, &cp);
      }
      cudaGraphNode_t bdep = nullptr;
      for (int k = kFirstRuKernel; k < kKernels && e == cudaSuccess; ++k)
        e = add(cp.conditional.phGraph_out[0], ks[k], &a, bdep, &bdep);
      if (e != cudaSuccess) {
        tf_set_last_cuda_error(e, "batch sweep graph", __FILE__, __LINE__);
        return TF_ERR_CUDA;
      }
    }
    *last = dep;
    return TF_OK;
  }

  int init(tf_ctx_s* c, const tf_batch_opts* o) {
    ctx = c;
    opts.vec_fp32 = 1;
    opts.val_fp32 = 0;
    opts.sweep_iters = 8;
    opts.ru_delta = 0.1;
    opts.mem_budget = (size_t)4 << 30;
    opts.max_systems = 1024;
    if (o) {
      opts = *o;
      if (opts.sweep_iters < 1) opts.sweep_iters = 8;
      if (!(opts.ru_delta > 0.0 && opts.ru_delta < 1.0)) opts.ru_delta = 0.1;
      if (opts.max_systems < 1) opts.max_systems = 1024;
      if (opts.mem_budget < ((size_t)1 << 20)) opts.mem_budget = (size_t)1 << 20;
    }
    vsz = opts.vec_fp32 ? 4 : 8;
    max_sys = opts.max_systems;
    profile = getenv("TF_BATCH_PROFILE") != nullptr;
    TF_CUDA_TRY(cudaSetDevice(ctx->device));
    int st = arena.init(opts.mem_budget);
    if (st != TF_OK) return st;
    slots.assign(max_sys, Slot{});
    const size_t desc_bytes = (size_t)max_sys * std::max(sizeof(SysDev<float>),
                                                         sizeof(SysDev<double>));
    TF_CUDA_TRY(cudaMalloc(&d_desc, desc_bytes));
    TF_CUDA_TRY(cudaMemset(d_desc, 0, desc_bytes));
    TF_CUDA_TRY(cudaMalloc((void**)&d_state, (size_t)max_sys * sizeof(SysState)));
    TF_CUDA_TRY(cudaMemset(d_state, 0, (size_t)max_sys * sizeof(SysState)));
    TF_CUDA_TRY(cudaMallocHost((void**)&h_state, (size_t)max_sys * sizeof(SysState)));
    memset(h_state, 0, (size_t)max_sys * sizeof(SysState));
    TF_CUDA_TRY(cudaMallocHost((void**)&h_desc_stage, (size_t)max_sys * kDescBytes));
    TF_CUDA_TRY(cudaMallocHost((void**)&h_init_stage, (size_t)max_sys * sizeof(SysState)));
    for (ListSet& L : ls) {
      TF_CUDA_TRY(cudaMalloc((void**)&L.d_cnt, 4 * sizeof(int)));
      TF_CUDA_TRY(cudaMemset(L.d_cnt, 0, 4 * sizeof(int)));
      TF_CUDA_TRY(cudaMallocHost((void**)&L.h_cnt, 4 * sizeof(int)));
      TF_CUDA_TRY(cudaMallocHost((void**)&L.h_state, (size_t)max_sys * sizeof(SysState)));
      TF_CUDA_TRY(cudaEventCreateWithFlags(&L.done, cudaEventDisableTiming));
    }
    TF_CUDA_TRY(cudaMalloc((void**)&d_gate_cnt, sizeof(unsigned)));
    TF_CUDA_TRY(cudaMemset(d_gate_cnt, 0, sizeof(unsigned)));
    st = (vsz == 4) ? setup_kernels<float>() : setup_kernels<double>();
    if (st != TF_OK) return st;
    for (ListSet& L : ls) {
      st = build_sweep(L);
      if (st != TF_OK) return st;
    }
    return TF_OK;
  }

  // ---- admission: prepare, reserve, upload, commit ----
  // The engine lock guards slots, the arena and the structure cache; the
  // server's admission thread reserves and uploads while its worker thread
  // sweeps, commits and retires.
  std::mutex emu;
  std::map<StructKey, std::shared_ptr<Structure>> scache;
  uint64_t tick = 0;

  std::condition_variable scv;   // a structure's preparation finished

  // Drops cached structures that are prepared but neither on the device
  // nor held by a queued system.  Engine lock held.
  void purge_unused() {
    for (auto it = scache.begin(); it != scache.end();)
      if (it->second->ready != 0 && !it->second->resident && it->second.use_count() == 1)
        it = scache.erase(it);
      else
        ++it;
  }

  // A system's host copy: its structure from the cache (prepared once for
  // all the systems that share it, even while the first of them is still
  // being prepared), else prepared here; then its values.  Host allocation
  // failures are TF_ERR_OOM.
  // borrow: val stays the caller's until the upload (calls that upload
  // before returning).
  int prepare(HostSys& h, int n, long long nnz, const int* row, const int* col, const int* dia,
              const double* val, const double* b, const double* x0, double tol, int maxit,
              bool borrow = false) {
    try {
      if (n < 1 || nnz < n || !row || !col || !dia || !val || !b) return TF_ERR_ARG;
      h.key = struct_key(n, nnz, row, col, dia);
      const bool patterns =
          !opts.two_phase_rows && !opts.val_fp32 && !getenv("TF_NO_ROW_PATTERNS");
      std::shared_ptr<Structure> S;
      bool mine = false;
      {
        std::unique_lock<std::mutex> lk(emu);
        purge_unused();
        auto it = scache.find(h.key);
        if (it != scache.end()) {
          S = it->second;
          scv.wait(lk, [&] { return S->ready != 0; });
          if (S->ready < 0) return -S->ready;
        } else {
          S = std::make_shared<Structure>();
          scache[h.key] = S;
          mine = true;
        }
      }
      if (mine) {
        int st;
        try {
          st = prepare_structure(*S, n, nnz, row, col, dia, patterns);
        } catch (const std::bad_alloc&) {
          st = TF_ERR_OOM;
        } catch (const std::length_error&) {
          st = TF_ERR_OOM;
        }
        std::lock_guard<std::mutex> lk(emu);
        S->ready = st == TF_OK ? 1 : -st;
        if (st != TF_OK) {
          auto it = scache.find(h.key);
          if (it != scache.end() && it->second == S) scache.erase(it);
        }
        scv.notify_all();
        if (st != TF_OK) return st;
      }
      h.st = std::move(S);
      h.tol = tol;
      h.maxit = maxit;
      return prepare_values(h, *h.st, row, val, b, x0, opts.val_fp32, borrow);
    } catch (const std::bad_alloc&) {
      h = HostSys();
      return TF_ERR_OOM;
    } catch (const std::length_error&) {
      h = HostSys();
      return TF_ERR_OOM;
    }
  }

  // Byte layout of a structure's device copy (columns or row patterns).
  static size_t struct_layout(Structure& S) {
    size_t o = 0;
    auto take = [&](size_t bytes) { size_t r = o; o = Arena::up(o + bytes); return r; };
    S.o_row = take(S.row.size() * 4);
    S.o_col = S.npat ? 0 : take(((size_t)S.nnz + 8) * 4);
    S.o_dia = take(S.dia.size() * 4);
    S.o_tiles = take(S.tiles.size() * 4);
    S.o_pat = S.npat ? take(S.pat.size()) : 0;
    S.o_tab = S.npat ? take(S.tab.size() * 4) : 0;
    return o;
  }

  // Evicts the least recently used resident structure that no system and
  // no queued request uses; false when there is none.  Engine lock held.
  bool evict_one() {
    auto victim = scache.end();
    for (auto it = scache.begin(); it != scache.end(); ++it)
      if (it->second->resident && it->second->users == 0 && it->second.use_count() == 1 &&
          (victim == scache.end() || it->second->last_use < victim->second->last_use))
        victim = it;
    if (victim == scache.end()) return false;
    Structure& S = *victim->second;
    arena.release(S.off, S.bytes);
    S.resident = false;
    scache.erase(victim);
    return true;
  }

  // A slot and arena space for h (and for its structure when no device copy
  // is resident); TF_ERR_BUSY when none is free now.  Engine lock held.
  int reserve(HostSys& h, Reservation* rv) {
    int slot = -1;
    for (int i = 0; i < max_sys; ++i)
      if (!slots[i].used) { slot = i; break; }
    if (slot < 0) return TF_ERR_BUSY;
    if (!h.st->resident) {   // uploaded meanwhile by a system with the same structure?
      auto it = scache.find(h.key);
      if (it != scache.end()) h.st = it->second;
    }
    Structure& S = *h.st;
    const int ntiles = S.ntiles();
    const Layout L = layout_for(h, ntiles, vsz, opts.val_fp32);
    size_t soff = 0, sb = 0, off = 0;
    const bool new_struct = !S.resident;
    if (new_struct) sb = struct_layout(S);
    // Both segments, or neither: on failure evict one unused structure and
    // try both again (evicting before the retry, not between the two
    // allocations, keeps the freed space in one piece where it can be).
    for (;;) {
      bool ok = !new_struct || arena.alloc(sb, &soff);
      if (ok && !arena.alloc(L.total, &off)) {
        if (new_struct) arena.release(soff, sb);
        ok = false;
      }
      if (ok) break;
      if (!evict_one()) return TF_ERR_BUSY;
    }
    if (new_struct) {
      S.off = soff;
      S.bytes = sb;
      S.resident = true;
      scache[h.key] = h.st;
    }
    S.users += 1;
    S.last_use = ++tick;
    Slot& sl = slots[slot];
    sl = Slot{};
    sl.used = 2;
    sl.off = off;
    sl.bytes = L.total;
    sl.n = h.n;
    sl.ntiles = ntiles;
    sl.L = L;
    sl.st = h.st;
    rv->slot = slot;
    rv->new_struct = new_struct;
    rv->L = L;
    return TF_OK;
  }

  // Gives a reservation back (its copies failed or its request went away).
  // Engine lock held.
  void unreserve(const Reservation& rv) {
    Slot& sl = slots[rv.slot];
    Structure& S = *sl.st;
    S.users -= 1;
    if (rv.new_struct) {   // the copy never landed: prepared, not resident, again
      arena.release(S.off, S.bytes);
      S.resident = false;
    }
    arena.release(sl.off, sl.bytes);
    sl = Slot{};
  }

  // The copies of a reserved system (and of its structure when new) on
  // stream s, through `stager`'s pinned buffers when given.  No lock: the
  // reservation's slot and segments are this caller's until it commits or
  // gives them back.
  int upload(const HostSys& h, const Reservation& rv, cudaStream_t s,
             Stager* stager = nullptr) {
    const Slot& sl = slots[rv.slot];
    const Structure& S = *sl.st;
    const Layout& L = rv.L;
    char* base = arena.base + sl.off;
    auto up = [&](char* dst, const void* src, size_t bytes) {
      return stager ? stager->copy(dst, src, bytes, s)
                    : cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
    };
    const size_t n8 = (size_t)h.n + 8;
    cudaError_t e = cudaSuccess;
    if (rv.new_struct) {
      char* sbase = arena.base + S.off;
      e = up(sbase + S.o_row, S.row.data(), S.row.size() * 4);
      if (e == cudaSuccess && !S.npat) e = up(sbase + S.o_col, S.col.data(), S.col.size() * 4);
      if (e == cudaSuccess) e = up(sbase + S.o_dia, S.dia.data(), S.dia.size() * 4);
      if (e == cudaSuccess) e = up(sbase + S.o_tiles, S.tiles.data(), S.tiles.size() * 4);
      if (e == cudaSuccess && S.npat) e = up(sbase + S.o_pat, S.pat.data(), S.pat.size());
      if (e == cudaSuccess && S.npat) e = up(sbase + S.o_tab, S.tab.data(), S.tab.size() * 4);
    }
    if (e == cudaSuccess) e = up(base + L.val, h.values(), (size_t)h.nnz * 8);
    if (e == cudaSuccess && opts.val_fp32)
      e = up(base + L.val32, h.val32.data(), (size_t)h.nnz * 4);
    if (e == cudaSuccess) e = up(base + L.b, h.b.data(), (size_t)h.n * 8);
    if (e == cudaSuccess) e = up(base + L.x, h.x0.data(), (size_t)h.n * 8);
    if (e == cudaSuccess) e = cudaMemsetAsync(base + L.xlo, 0, n8 * vsz, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(base + L.p, 0, n8 * vsz, s);
    if (e == cudaSuccess && opts.val_fp32)
      e = cudaMemsetAsync(base + L.tile_cnt, 0, (size_t)sl.ntiles * 4, s);
    if (e != cudaSuccess) {
      tf_set_last_cuda_error(e, "batch admit copies", __FILE__, __LINE__);
      return TF_ERR_CUDA;
    }
    return TF_OK;
  }

  // Makes an uploaded system part of the batch: its descriptor and state
  // (on the engine's stream, asynchronously from the slot's pinned staging,
  // ahead of the next sweep launched there).  The copies of the
  // reservation must have completed.  Engine lock held.
  int commit(const HostSys& h, const Reservation& rv) {
    Slot& sl = slots[rv.slot];
    Structure& S = *sl.st;
    if (rv.new_struct) std::vector<int>().swap(S.col);   // the device copy is complete
    const Layout& L = rv.L;
    char* base = arena.base + sl.off;
    char* sbase = arena.base + S.off;
    cudaStream_t s = ctx->stream;
    auto fill = [&](auto& d) {
      using VV = std::remove_pointer_t<decltype(d.xlo)>;
      d.row = (const int*)(sbase + S.o_row);
      d.col = S.npat ? nullptr : (const int*)(sbase + S.o_col);
      d.pat = S.npat ? (const unsigned char*)(sbase + S.o_pat) : nullptr;
      d.tab = S.npat ? (const int*)(sbase + S.o_tab) : nullptr;
      d.npat = S.npat;
      d.dia = (const int*)(sbase + S.o_dia);
      d.tiles = (const int*)(sbase + S.o_tiles);
      d.val = (const double*)(base + L.val);
      d.val32 = opts.val_fp32 ? (const float*)(base + L.val32) : nullptr;
      d.b = (const double*)(base + L.b);
      d.x = (double*)(base + L.x);
      d.xlo = (VV*)(base + L.xlo);
      d.r = (VV*)(base + L.r);
      d.p = (VV*)(base + L.p);
      d.q = (VV*)(base + L.q);
      d.dinv = (VV*)(base + L.dinv);
      d.tile_tot = (double*)(base + L.tile_tot);
      d.chunk_tot = (double*)(base + L.chunk_tot);
      d.warp_part = opts.val_fp32 ? (double*)(base + L.warp_part) : nullptr;
      d.tile_cnt = opts.val_fp32 ? (unsigned*)(base + L.tile_cnt) : nullptr;
      d.n = h.n;
      d.ntiles = sl.ntiles;
      d.maxit = h.maxit;
      d.use_val32 = opts.val_fp32;
      d.tol = h.tol;
    };
    SysState& ss = h_init_stage[rv.slot];
    ss = SysState{};
    ss.status = kInit;
    cudaError_t e;
    void* stage = h_desc_stage + (size_t)rv.slot * kDescBytes;
    if (vsz == 4) {
      SysDev<float>& d = *static_cast<SysDev<float>*>(stage);
      d = SysDev<float>{};
      fill(d);
      e = cudaMemcpyAsync((SysDev<float>*)d_desc + rv.slot, &d, sizeof d,
                          cudaMemcpyHostToDevice, s);
    } else {
      SysDev<double>& d = *static_cast<SysDev<double>*>(stage);
      d = SysDev<double>{};
      fill(d);
      e = cudaMemcpyAsync((SysDev<double>*)d_desc + rv.slot, &d, sizeof d,
                          cudaMemcpyHostToDevice, s);
    }
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_state + rv.slot, &ss, sizeof ss, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) {
      unreserve(rv);
      tf_set_last_cuda_error(e, "batch admit descriptors", __FILE__, __LINE__);
      return TF_ERR_CUDA;
    }
    sl.used = 1;
    h_state[rv.slot] = ss;
    return TF_OK;
  }

  // Reserve, upload and commit on the engine's stream, synchronously (the
  // batch API); TF_ERR_BUSY if no slot or no arena space.
  int admit(HostSys& h, int* out_slot) {
    Reservation rv;
    int st;
    {
      std::lock_guard<std::mutex> lk(emu);
      st = reserve(h, &rv);
    }
    if (st != TF_OK) return st;
    st = upload(h, rv, ctx->stream);
    if (st == TF_OK) {
      const cudaError_t e = cudaStreamSynchronize(ctx->stream);   // host buffers may go away
      if (e != cudaSuccess) {
        tf_set_last_cuda_error(e, "batch admit copies", __FILE__, __LINE__);
        st = TF_ERR_CUDA;
      }
    }
    std::lock_guard<std::mutex> lk(emu);
    if (st != TF_OK) {
      unreserve(rv);
      return st;
    }
    st = commit(h, rv);
    if (st == TF_OK) {
      const cudaError_t e = cudaStreamSynchronize(ctx->stream);
      if (e != cudaSuccess) {
        tf_set_last_cuda_error(e, "batch admit descriptors", __FILE__, __LINE__);
        return TF_ERR_CUDA;
      }
      *out_slot = rv.slot;
    }
    return st;
  }

  // Grows a pinned buffer (contents dropped) to at least n elements.
  template <typename T>
  static int grow_pinned(T** p, int* cap, int n) {
    if (n <= *cap) return TF_OK;
    if (*p) cudaFreeHost(*p);
    *p = nullptr;
    *cap = std::max(n, 2 * *cap);
    TF_CUDA_TRY(cudaMallocHost((void**)p, (size_t)*cap * sizeof(T)));
    return TF_OK;
  }

  // Fills list set L: every tile of every admitted system that still
  // iterates (skip[slot] != 0 leaves a system out); the refinement list
  // starts with the tiles of systems not yet initialised.  Grows L's
  // buffers (and rebuilds its graph) when needed, which requires L's last
  // sweep to have finished.  Engine lock held when threads share the engine.
  int build_list(ListSet& L, const std::vector<char>* skip = nullptr) {
    int nw = 0, nr = 0, nf = 0;
    L.slots.clear();
    L.rows = L.nnz = 0;
    L.bytes = 0.0;
    for (int i = 0; i < max_sys; ++i) {
      if (slots[i].used != 1 || (skip && (*skip)[i])) continue;
      const int stt = h_state[i].status;
      if (stt != kInit && stt != kActive) continue;
      L.slots.push_back(i);
      nw += slots[i].ntiles;
      if (stt == kInit && !slots[i].listed) nr += slots[i].ntiles;
      nf += fin_chunks(slots[i].ntiles);
      L.rows += slots[i].n;
      const long long e = slots[i].st->tile_j[slots[i].ntiles];
      L.nnz += e;
      // An inner iteration's algorithmic bytes: the matrix (8 per value and
      // 4 per column, or 1 per row with row patterns; 4 per row pointer) and
      // 13 iterate vectors (p gathered and read, q, r, x-correction, 1/d).
      L.bytes += (double)e * (slots[i].st->npat ? 8.0 : 12.0) +
                 (double)slots[i].n * ((slots[i].st->npat ? 1.0 : 0.0) + 4.0 + 13.0 * vsz);
    }
    int st = grow_pinned(&L.h_work, &L.h_work_cap, std::max(nw, 1));
    if (st == TF_OK) st = grow_pinned(&L.h_ru, &L.h_ru_cap, std::max(nr, 1));
    if (st == TF_OK) st = grow_pinned(&L.h_fin, &L.h_fin_cap, std::max(nf, 1));
    if (st != TF_OK) return st;
    if (nw > L.work_cap || nf > L.fin_cap) {
      for (void* p : {(void*)L.d_work, (void*)L.d_ru, (void*)L.d_fin})
        if (p) cudaFree(p);
      L.d_work = nullptr;
      L.d_ru = nullptr;
      L.d_fin = nullptr;
      L.work_cap = std::max(nw, 2 * L.work_cap);
      L.fin_cap = std::max(nf, 2 * L.fin_cap);
      TF_CUDA_TRY(cudaMalloc((void**)&L.d_work, (size_t)L.work_cap * sizeof(Work)));
      TF_CUDA_TRY(cudaMalloc((void**)&L.d_ru, (size_t)L.work_cap * sizeof(Work)));
      TF_CUDA_TRY(cudaMalloc((void**)&L.d_fin, (size_t)L.fin_cap * sizeof(FinItem)));
      st = build_sweep(L);   // the graph holds the lists' pointers
      if (st != TF_OK) return st;
    }
    int w = 0, r = 0, f = 0;
    for (int i : L.slots) {
      const std::vector<int>& tl = slots[i].st->tiles;
      const std::vector<int>& tj = slots[i].st->tile_j;
      // A new system's first residual is queued once, with its first list:
      // a list built while that sweep is still in flight sees the system's
      // state as new too, and must not queue it again (the refinement
      // kernels would then fold and recompute its tiles twice, concurrently).
      const bool init = h_state[i].status == kInit && !slots[i].listed;
      slots[i].listed = 1;
      for (int t = 0; t < slots[i].ntiles; ++t) {
        const Work wk{i, t, tl[t], tl[t + 1], tj[t], tj[t + 1]};
        L.h_work[w++] = wk;
        if (init) L.h_ru[r++] = wk;
      }
      for (int c = 0; c < fin_chunks(slots[i].ntiles); ++c) L.h_fin[f++] = FinItem{i, c};
    }
    L.nwork = nw;
    L.nru = nr;
    L.nfin = nf;
    nwork = nw;
    return TF_OK;
  }

  // Copies L's lists to the device on stream s (asynchronously: from pinned
  // memory, ahead of the sweep launched after them).
  int upload_list(ListSet& L, cudaStream_t s) {
    if (L.nwork)
      TF_CUDA_TRY(cudaMemcpyAsync(L.d_work, L.h_work, (size_t)L.nwork * sizeof(Work),
                                  cudaMemcpyHostToDevice, s));
    if (L.nru)
      TF_CUDA_TRY(cudaMemcpyAsync(L.d_ru, L.h_ru, (size_t)L.nru * sizeof(Work),
                                  cudaMemcpyHostToDevice, s));
    if (L.nfin)
      TF_CUDA_TRY(cudaMemcpyAsync(L.d_fin, L.h_fin, (size_t)L.nfin * sizeof(FinItem),
                                  cudaMemcpyHostToDevice, s));
    L.h_cnt[0] = L.nwork;
    L.h_cnt[1] = L.nru;
    L.h_cnt[2] = L.nfin;
    TF_CUDA_TRY(cudaMemcpyAsync(L.d_cnt, L.h_cnt, 3 * sizeof(int), cudaMemcpyHostToDevice, s));
    return TF_OK;
  }

  // The listed systems' state after L's sweep (slots not in the list keep
  // theirs: they may have been committed since the sweep was launched).
  void merge_state(const ListSet& L) {
    for (int i : L.slots) h_state[i] = L.h_state[i];
  }

  // The batch API's list: set 0, built and uploaded ahead of the next sweep.
  int rebuild_work() {
    int st = build_list(ls[0]);
    if (st == TF_OK) st = upload_list(ls[0], ctx->stream);
    return st;
  }

  // One sweep (sweep_iters iterations) of set 0, then refresh the host state.
  int run_sweep() {
    if (profile) return run_sweep_profiled();
    ListSet& L = ls[0];
    TF_CUDA_TRY(cudaGraphLaunch(L.graph, ctx->stream));
    TF_CUDA_TRY(cudaEventRecord(L.done, ctx->stream));
    TF_CUDA_TRY(cudaEventSynchronize(L.done));
    merge_state(L);
    ++sweeps;
    return TF_OK;
  }

  int n_running() const {
    int c = 0;
    for (int i = 0; i < max_sys; ++i)
      if (slots[i].used == 1 && (h_state[i].status == kInit || h_state[i].status == kActive))
        ++c;
    return c;
  }

  int run_all() {
    const auto t0 = std::chrono::steady_clock::now();
    int st = rebuild_work();
    if (st != TF_OK) return st;
    int running = n_running();
    trace.clear();
    while (running > 0) {
      const auto ts = std::chrono::steady_clock::now();
      st = run_sweep();
      if (st != TF_OK) return st;
      const auto te = std::chrono::steady_clock::now();
      tf_batch_sweep rec{};
      rec.active = running;
      rec.items = nwork;
      rec.rows = ls[0].rows;
      rec.nnz = ls[0].nnz;
      rec.iter_bytes = ls[0].bytes;
      rec.ms = std::chrono::duration<double, std::milli>(te - ts).count();
      if (profile)
        for (int k = 0; k < kKernels; ++k) rec.kernel_ms[k] = sweep_kms[k];
      trace.push_back(rec);
      const double ms = std::chrono::duration<double, std::milli>(te - t0).count();
      for (int i = 0; i < max_sys; ++i)
        if (slots[i].used == 1 && slots[i].done_ms < 0.0 && h_state[i].status != kInit &&
            h_state[i].status != kActive)
          slots[i].done_ms = ms;
      const int now = n_running();
      if (now != running) {
        st = rebuild_work();
        if (st != TF_OK) return st;
      }
      running = now;
    }
    return TF_OK;
  }

  // x of a finished system in the caller's numbering, copied on stream s
  // (the engine's stream by default).
  int fetch_x(int slot, double* x, cudaStream_t s = nullptr) {
    if (!s) s = ctx->stream;
    const Slot& sl = slots[slot];
    const std::vector<int>& perm = sl.st->perm;
    if (perm.empty()) {
      TF_CUDA_TRY(cudaMemcpyAsync(x, arena.base + sl.off + sl.L.x, (size_t)sl.n * 8,
                                  cudaMemcpyDeviceToHost, s));
      TF_CUDA_TRY(cudaStreamSynchronize(s));
      return TF_OK;
    }
    std::vector<double> tmp((size_t)sl.n);
    TF_CUDA_TRY(cudaMemcpyAsync(tmp.data(), arena.base + sl.off + sl.L.x, (size_t)sl.n * 8,
                                cudaMemcpyDeviceToHost, s));
    TF_CUDA_TRY(cudaStreamSynchronize(s));
    for (int i = 0; i < sl.n; ++i) x[perm[i]] = tmp[i];
    return TF_OK;
  }

  // A finished or removed system gives its slot and segment back; its
  // structure stays resident for later systems until the space is needed.
  // Engine lock held by callers that share the engine between threads.
  void retire(int slot) {
    Slot& sl = slots[slot];
    if (sl.used != 1) return;
    sl.st->users -= 1;
    sl.st->last_use = ++tick;
    arena.release(sl.off, sl.bytes);
    sl = Slot{};
    h_state[slot].status = kFree;
  }
};

// ---------------------------------------------------------------------------
// C ABI: batches
// ---------------------------------------------------------------------------
extern "C" int tf_batch_create(tf_ctx ctx, const tf_batch_opts* opts, tf_batch* out) {
  TF_API_BEGIN
  if (!ctx || !out) return TF_ERR_ARG;
  *out = nullptr;
  auto* b = new tf_batch_s();
  const int st = b->init(ctx, opts);
  if (st != TF_OK) {
    delete b;
    return st;
  }
  *out = b;
  return TF_OK;
  TF_API_END
}

extern "C" int tf_batch_destroy(tf_batch b) {
  TF_API_BEGIN
  if (!b) return TF_ERR_ARG;
  delete b;
  return TF_OK;
  TF_API_END
}

extern "C" int tf_batch_add(tf_batch bt, int n, int64_t nnz, const int* row, const int* col,
                            const int* dia, const double* val, const double* b,
                            const double* x0, double tol, int maxit, int* sys) {
  TF_API_BEGIN
  if (!bt || !sys) return TF_ERR_ARG;
  HostSys h;
  const auto t0 = std::chrono::steady_clock::now();
  int st = bt->prepare(h, n, nnz, row, col, dia, val, b, x0, tol, maxit, true);
  const auto t1 = std::chrono::steady_clock::now();
  bt->up_prep_ms += std::chrono::duration<double, std::milli>(t1 - t0).count();
  if (st != TF_OK) return st;
  TF_CUDA_TRY(cudaSetDevice(bt->ctx->device));
  st = bt->admit(h, sys);
  bt->up_admit_ms += std::chrono::duration<double, std::milli>(
                         std::chrono::steady_clock::now() - t1).count();
  return st;
  TF_API_END
}

// Several systems in one call: the host preparation (conversion,
// renumbering, tiling) and the copies to the device run on `threads`
// worker threads (0: one per hardware thread), each copying on a stream of
// its own; this thread reserves slots and space in order, so slots,
// results and errors are those of tf_batch_add called for each system in
// turn.  At most 2 x threads prepared systems wait for their copies.
extern "C" int tf_batch_add_many(tf_batch bt, int count, const int* n, const int64_t* nnz,
                                 const int* const* row, const int* const* col,
                                 const int* const* dia, const double* const* val,
                                 const double* const* rhs, const double* const* x0,
                                 const double* tol, const int* maxit, int threads, int* sys) {
  TF_API_BEGIN
  if (!bt || count < 0) return TF_ERR_ARG;
  if (count == 0) return TF_OK;
  if (!n || !nnz || !row || !col || !dia || !val || !rhs || !tol || !maxit || !sys)
    return TF_ERR_ARG;
  for (int i = 0; i < count; ++i) sys[i] = -1;
  TF_CUDA_TRY(cudaSetDevice(bt->ctx->device));
  int nt = threads > 0 ? threads : (int)std::thread::hardware_concurrency();
  nt = std::max(1, std::min(std::min(nt, count), 64));
  const int window = 2 * nt;
  using clk = std::chrono::steady_clock;
  auto ms_since = [](clk::time_point t0) {
    return std::chrono::duration<double, std::milli>(clk::now() - t0).count();
  };
  std::vector<HostSys> hs(count);
  std::vector<Reservation> rv(count);
  std::vector<int> st(count, TF_OK);
  std::vector<char> ready(count, 0);
  std::deque<int> upq;   // reserved, waiting for their copies
  std::mutex mu;
  std::condition_variable cv;
  int next = 0, reserved = 0, copied = 0;
  bool stop_prep = false, stop_all = false;
  int copy_err = TF_OK;
  double prep_ms = 0.0, wait_ms = 0.0, admit_ms = 0.0;
  auto prepare = [&](int i) {
    const auto t0 = clk::now();
    const int r = tf_guarded([&] {
      return bt->prepare(hs[i], n[i], nnz[i], row[i], col[i], dia[i], val[i], rhs[i],
                         x0 ? x0[i] : nullptr, tol[i], maxit[i], true);
    });
    const double ms = ms_since(t0);
    std::lock_guard<std::mutex> lk(mu);
    st[i] = r;
    ready[i] = 1;
    prep_ms += ms;
  };
  // The copies of reserved system i on stream s, then its commit.
  auto copy_in = [&](int i, cudaStream_t s, Stager* stager) {
    const auto t0 = clk::now();
    int r = tf_guarded([&] { return bt->upload(hs[i], rv[i], s, stager); });
    if (r == TF_OK) {
      const cudaError_t e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) {
        tf_set_last_cuda_error(e, "batch admit copies", __FILE__, __LINE__);
        r = TF_ERR_CUDA;
      }
    }
    {
      std::lock_guard<std::mutex> el(bt->emu);
      if (r == TF_OK) r = tf_guarded([&] { return bt->commit(hs[i], rv[i]); });
      else bt->unreserve(rv[i]);
    }
    hs[i] = HostSys();   // on the device now
    std::lock_guard<std::mutex> lk(mu);
    if (r == TF_OK) sys[i] = rv[i].slot;
    else if (copy_err == TF_OK) copy_err = r;
    ++copied;
    admit_ms += ms_since(t0);
  };
  auto worker = [&]() {
    cudaSetDevice(bt->ctx->device);
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) s = nullptr;
    std::unique_ptr<Stager> stager = bt->take_stager();
    for (;;) {
      int i = -1;
      bool up = false;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] {
          return stop_all || !upq.empty() ||
                 (!stop_prep && next < count && next < copied + window);
        });
        if (!upq.empty()) {
          i = upq.front();
          upq.pop_front();
          up = true;
        } else if (!stop_prep && next < count && next < copied + window) {
          i = next++;
        } else {
          break;   // stop_all
        }
      }
      if (up) copy_in(i, s ? s : bt->ctx->stream, stager.get());
      else prepare(i);
      cv.notify_all();
    }
    if (s) cudaStreamSynchronize(s);
    bt->give_stager(std::move(stager));
    if (s) cudaStreamDestroy(s);
  };
  std::vector<std::thread> pool;
  try {
    for (int t = 0; t < nt; ++t) pool.emplace_back(worker);
  } catch (const std::system_error&) {
    // fewer workers than asked for (none: this thread does everything)
  }
  const bool inline_work = pool.empty();
  int result = TF_OK;
  for (int i = 0; i < count; ++i) {
    const auto t0 = clk::now();
    if (inline_work) {
      prepare(i);
    } else {
      std::unique_lock<std::mutex> lk(mu);
      cv.wait(lk, [&] { return ready[i] != 0; });
    }
    const auto t1 = clk::now();
    int r = st[i];
    if (r == TF_OK) {
      std::lock_guard<std::mutex> el(bt->emu);
      r = tf_guarded([&] { return bt->reserve(hs[i], &rv[i]); });
    }
    {
      std::lock_guard<std::mutex> lk(mu);
      wait_ms += std::chrono::duration<double, std::milli>(t1 - t0).count();
      admit_ms += ms_since(t1);
      if (r == TF_OK) {
        ++reserved;
        if (!inline_work) upq.push_back(i);
      } else {
        stop_prep = true;
      }
    }
    cv.notify_all();
    if (inline_work && r == TF_OK) copy_in(i, bt->ctx->stream, nullptr);
    if (r != TF_OK) {
      hs[i] = HostSys();
      result = r;
      break;
    }
  }
  {
    std::unique_lock<std::mutex> lk(mu);
    stop_prep = true;
    cv.wait(lk, [&] { return copied == reserved; });
    stop_all = true;
  }
  cv.notify_all();
  for (auto& t : pool) t.join();
  TF_CUDA_TRY(cudaStreamSynchronize(bt->ctx->stream));   // the commits' descriptors
  bt->up_prep_ms += prep_ms;
  bt->up_wait_ms += wait_ms;
  bt->up_admit_ms += admit_ms;
  if (result == TF_OK) result = copy_err;
  return result;
  TF_API_END
}

extern "C" int tf_batch_upload_ms(tf_batch bt, double* prep_ms, double* wait_ms,
                                  double* admit_ms) {
  TF_API_BEGIN
  if (!bt) return TF_ERR_ARG;
  if (prep_ms) *prep_ms = bt->up_prep_ms;
  if (wait_ms) *wait_ms = bt->up_wait_ms;
  if (admit_ms) *admit_ms = bt->up_admit_ms;
  return TF_OK;
  TF_API_END
}

extern "C" int tf_batch_run(tf_batch bt) {
  TF_API_BEGIN
  if (!bt) return TF_ERR_ARG;
  TF_CUDA_TRY(cudaSetDevice(bt->ctx->device));
  return bt->run_all();
  TF_API_END
}

extern "C" int tf_batch_result(tf_batch bt, int sys, double* x, int* iters,
                               double* true_rel_res, int* status, int* n_updates,
                               double* done_ms) {
  TF_API_BEGIN
  if (!bt || sys < 0 || sys >= bt->max_sys || bt->slots[sys].used != 1) return TF_ERR_ARG;
  const SysState& s = bt->h_state[sys];
  if (done_ms) *done_ms = bt->slots[sys].done_ms;
  if (iters) *iters = s.iter;
  if (true_rel_res) *true_rel_res = s.res_true;
  if (status) *status = s.status;
  if (n_updates) *n_updates = s.n_ru;
  if (x) return bt->fetch_x(sys, x);
  return TF_OK;
  TF_API_END
}

extern "C" int tf_batch_kernel_ms(tf_batch bt, double* ms8) {
  TF_API_BEGIN
  if (!bt || !ms8) return TF_ERR_ARG;
  for (int k = 0; k < kKernels; ++k) ms8[k] = bt->kern_ms[k];
  return bt->profile ? TF_OK : TF_ERR_ARG;
  TF_API_END
}

extern "C" int tf_batch_trace(tf_batch bt, tf_batch_sweep* out, int cap, int* count) {
  TF_API_BEGIN
  if (!bt || !count || cap < 0 || (cap > 0 && !out)) return TF_ERR_ARG;
  const int n = std::min<int>(cap, (int)bt->trace.size());
  for (int i = 0; i < n; ++i) out[i] = bt->trace[i];
  *count = (int)bt->trace.size();
  return TF_OK;
  TF_API_END
}

extern "C" int tf_batch_remove(tf_batch bt, int sys) {
  TF_API_BEGIN
  if (!bt || sys < 0 || sys >= bt->max_sys || bt->slots[sys].used != 1) return TF_ERR_ARG;
  bt->retire(sys);
  return TF_OK;
  TF_API_END
}

extern "C" int tf_batch_info(tf_batch bt, int* sweeps, int* work_items, size_t* free_bytes) {
  TF_API_BEGIN
  if (!bt) return TF_ERR_ARG;
  if (sweeps) *sweeps = bt->sweeps;
  if (work_items) *work_items = bt->nwork;
  if (free_bytes) *free_bytes = bt->arena.free_bytes();
  return TF_OK;
  TF_API_END
}

// ---------------------------------------------------------------------------
// C ABI: the serving loop (continuous batching)
// ---------------------------------------------------------------------------
namespace {
using Clock = std::chrono::steady_clock;

struct Request {
  int64_t id = 0;
  int n = 0;
  HostSys h;            // host copy until its upload has landed
  Reservation rv;       // slot and arena space once reserved
  cudaEvent_t ev = nullptr;   // the upload's completion (copy stream)
  Clock::time_point t_submit, t_admit, t_done;
  int slot = -1;
  int status = 0;       // SysStatus at completion, or an error code (< 0)
  int iters = 0, n_ru = 0;
  double res = 0.0;
  std::vector<double> x;
  bool done = false;
  bool cancel = false;  // set by tf_server_cancel while the request is staged or runs
};
}  // namespace

// Continuous batching with four kinds of threads:
//   submitting threads  prepare a request's host copy (its structure shared
//                       through the engine's cache) and queue it;
//   the admission thread takes queued requests in arrival order, reserves
//                       a slot and arena space when memory allows and
//                       uploads them on a copy stream of its own, so the
//                       copies overlap the sweeps;
//   the worker thread   commits requests whose copies have landed (their
//                       descriptors go ahead of the next sweep), runs the
//                       sweeps, and takes finished and cancelled requests
//                       out of the work list;
//   the collector       copies their results out on a stream of its own
//                       and retires them, which frees space for the
//                       admission thread.
struct tf_server_s {
  tf_batch_s eng;
  cudaStream_t copy_stream = nullptr, fetch_stream = nullptr;
  std::mutex mu;   // everything below (the engine's own state: eng.emu)
  std::condition_variable cv_work, cv_done, cv_admit, cv_collect;
  std::deque<std::shared_ptr<Request>> queue;    // prepared, waiting for space
  std::deque<std::shared_ptr<Request>> staged;   // reserved, copies in flight
  std::deque<std::shared_ptr<Request>> finishing;   // out of the work list, to collect
  std::map<int64_t, std::shared_ptr<Request>> live;     // submitted, not yet collected
  std::map<int, std::shared_ptr<Request>> by_slot;      // running (worker thread)
  int n_running = 0;        // by_slot.size(), readable by the admission thread
  int n_releasing = 0;      // finished or cancelled, their memory not yet released
  uint64_t retire_gen = 0;  // counts retirements (the admission thread waits on it)
  int64_t next_id = 1;
  bool stop = false;
  int error = TF_OK;
  std::thread worker, admitter, collector;
  // stats
  long long admitted = 0, completed = 0, rejected = 0;
  int peak_running = 0;
  // Wall time (ms) by activity (tf_server_timing): preparation on the
  // submitting threads (summed), the admission thread's reservations and
  // uploads, the worker thread's host work (commits, lists, launches) and
  // its waits for the sweep in flight, and the collector's result copies
  // and retirements.
  double t_ms[5] = {0, 0, 0, 0, 0};
  static double ms_since(Clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
  }

  // Ends a request that never ran (lock mu held).
  void fail(const std::shared_ptr<Request>& r, int status) {
    r->status = -status;
    r->t_done = Clock::now();
    r->done = true;
    r->h = HostSys();
    cv_done.notify_all();
  }

  void admit_loop() {
    cudaSetDevice(eng.ctx->device);
    std::unique_ptr<Stager> stager = eng.take_stager();
    for (;;) {
      std::shared_ptr<Request> r;
      uint64_t gen;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_admit.wait(lk, [&] { return stop || !queue.empty(); });
        if (stop) return;
        r = queue.front();
        gen = retire_gen;
      }
      const auto t0 = Clock::now();
      Reservation rv;
      int st = tf_guarded([&] {
        std::lock_guard<std::mutex> el(eng.emu);
        return eng.reserve(r->h, &rv);
      });
      if (st == TF_ERR_BUSY) {
        std::unique_lock<std::mutex> lk(mu);
        t_ms[1] += ms_since(t0);
        if (n_running == 0 && staged.empty() && n_releasing == 0 && retire_gen == gen) {
          // Nothing runs, lands or is being released that could free space:
          // it never fits.
          if (!queue.empty() && queue.front() == r) {
            queue.pop_front();
            ++rejected;
            fail(r, TF_ERR_OOM);
          }
          continue;
        }
        cv_admit.wait(lk, [&] { return stop || retire_gen != gen; });
        continue;
      }
      cudaEvent_t ev = nullptr;
      if (st == TF_OK)
        st = tf_guarded([&] { return eng.upload(r->h, rv, copy_stream, stager.get()); });
      if (st == TF_OK) {
        cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(ev, copy_stream);
        if (e != cudaSuccess) {
          tf_set_last_cuda_error(e, "server upload event", __FILE__, __LINE__);
          st = TF_ERR_CUDA;
        }
      }
      bool give_back = false;
      {
        std::lock_guard<std::mutex> lk(mu);
        t_ms[1] += ms_since(t0);
        if (queue.empty() || queue.front() != r) {   // cancelled meanwhile
          give_back = (st == TF_OK || rv.slot >= 0);
        } else {
          queue.pop_front();
          if (st != TF_OK) {
            give_back = rv.slot >= 0;
            fail(r, st);
          } else {
            r->rv = rv;
            r->ev = ev;
            ev = nullptr;
            staged.push_back(r);
            cv_work.notify_one();
          }
        }
      }
      if (give_back) {   // after its copies: the space must not be reused under them
        cudaStreamSynchronize(copy_stream);
        std::lock_guard<std::mutex> el(eng.emu);
        eng.unreserve(rv);
      }
      if (ev) cudaEventDestroy(ev);
    }
  }

  // The worker: sweeps back to back, two work lists alternating.  While
  // sweep k runs, the next list is built from the systems admitted so far
  // (committed ones included, finished ones left out), uploaded and sweep
  // k + 1 launched behind it; then the worker waits for sweep k, reads its
  // state and takes the systems it finished (or that were cancelled) out
  // of the lists.  Those are still in sweep k + 1's list (built before they
  // were seen), where they are skipped; they go to the collector once sweep
  // k + 1 has ended, so no sweep in flight refers to their memory when it
  // is released.
  void loop() {
    cudaSetDevice(eng.ctx->device);
    cudaStream_t s = eng.ctx->stream;
    std::vector<char> out(eng.max_sys, 0);          // left out of the lists
    // out of the next list, still in the one in flight
    std::vector<std::shared_ptr<Request>> leaving;
    int cur = 0;
    bool inflight = false;
    for (;;) {
      std::vector<std::shared_ptr<Request>> ready;
      std::shared_ptr<Request> wait_for;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] {
          return stop || !staged.empty() || !by_slot.empty() || inflight || !leaving.empty();
        });
        if (stop) break;
        while (!staged.empty() && cudaEventQuery(staged.front()->ev) == cudaSuccess) {
          ready.push_back(staged.front());
          staged.pop_front();
        }
        if (ready.empty() && by_slot.empty() && !inflight && leaving.empty())
          wait_for = staged.front();
      }
      if (wait_for) {   // nothing to sweep: wait for the next upload to land
        cudaEventSynchronize(wait_for->ev);
        continue;
      }
      auto t0 = Clock::now();
      for (auto& r : ready) {
        cudaEventDestroy(r->ev);
        r->ev = nullptr;
        int st;
        {
          std::lock_guard<std::mutex> el(eng.emu);
          if (r->cancel) {
            eng.unreserve(r->rv);
            st = TF_ERR_CANCELLED;
          } else {
            st = tf_guarded([&] { return eng.commit(r->h, r->rv); });
          }
        }
        std::lock_guard<std::mutex> lk(mu);
        if (st != TF_OK) {   // its reservation was given back
          fail(r, st);
          ++retire_gen;
          cv_admit.notify_all();
          continue;
        }
        r->slot = r->rv.slot;
        r->t_admit = Clock::now();
        r->h = HostSys();   // on the device now
        out[r->slot] = 0;
        by_slot[r->slot] = r;
        n_running = (int)by_slot.size();
        ++admitted;
      }
      peak_running = std::max(peak_running, (int)by_slot.size());
      // Launch the next sweep behind the one in flight.
      const int nxt = inflight ? (cur ^ 1) : cur;
      bool launched = false;
      int st = TF_OK;
      if (!by_slot.empty()) {
        tf_batch_s::ListSet& L = eng.ls[nxt];
        st = tf_guarded([&] {
          std::lock_guard<std::mutex> el(eng.emu);
          return eng.build_list(L, &out);
        });
        if (st == TF_OK && L.nwork > 0) {
          st = eng.upload_list(L, s);
          if (st == TF_OK) {
            cudaError_t e = cudaGraphLaunch(L.graph, s);
            if (e == cudaSuccess) e = cudaEventRecord(L.done, s);
            if (e != cudaSuccess) {
              tf_set_last_cuda_error(e, "server sweep", __FILE__, __LINE__);
              st = TF_ERR_CUDA;
            }
          }
          launched = st == TF_OK;
        }
      }
      const auto t1 = Clock::now();
      // Wait for the sweep in flight and read its state.
      std::vector<int> fin, cancelled;
      if (st == TF_OK && inflight) {
        tf_batch_s::ListSet& L = eng.ls[cur];
        const cudaError_t e = cudaEventSynchronize(L.done);
        if (e != cudaSuccess) {
          tf_set_last_cuda_error(e, "server sweep", __FILE__, __LINE__);
          st = TF_ERR_CUDA;
        } else {
          std::lock_guard<std::mutex> el(eng.emu);
          eng.merge_state(L);
          ++eng.sweeps;
        }
      }
      const auto t2 = Clock::now();
      if (st != TF_OK) {
        std::lock_guard<std::mutex> lk(mu);
        error = st;
        for (auto& kv : by_slot) {
          kv.second->status = -st;
          kv.second->done = true;
        }
        by_slot.clear();
        n_running = 0;
        cv_done.notify_all();
        inflight = false;
        continue;
      }
      std::lock_guard<std::mutex> lk(mu);
      // Systems left out of the list just launched are in no sweep now.
      if (inflight && !leaving.empty()) {
        for (auto& r : leaving) finishing.push_back(r);
        leaving.clear();
        cv_collect.notify_one();
      }
      if (inflight) {
        for (auto& kv : by_slot) {
          const int ss = eng.h_state[kv.first].status;
          if (ss != kInit && ss != kActive) fin.push_back(kv.first);
          else if (kv.second->cancel) cancelled.push_back(kv.first);
        }
        for (int slot : fin) {
          auto r = by_slot[slot];
          const SysState& ss = eng.h_state[slot];
          r->status = ss.status;
          r->iters = ss.iter;
          r->n_ru = ss.n_ru;
          r->res = ss.res_true;
        }
        for (int slot : cancelled) by_slot[slot]->status = -TF_ERR_CANCELLED;
        for (int slot : fin) {
          out[slot] = 1;
          leaving.push_back(by_slot[slot]);
          by_slot.erase(slot);
        }
        for (int slot : cancelled) {
          out[slot] = 1;
          leaving.push_back(by_slot[slot]);
          by_slot.erase(slot);
        }
        n_releasing += (int)(fin.size() + cancelled.size());
        n_running = (int)by_slot.size();
      }
      if (launched) {
        cur = nxt;
        inflight = true;
      } else {
        inflight = false;
        // Nothing in flight: whatever is leaving is in no sweep.
        for (auto& r : leaving) finishing.push_back(r);
        if (!leaving.empty()) cv_collect.notify_one();
        leaving.clear();
      }
      t_ms[2] += std::chrono::duration<double, std::milli>(t1 - t0).count() + ms_since(t2);
      t_ms[3] += std::chrono::duration<double, std::milli>(t2 - t1).count();
    }
    // Stopping: let the sweeps end before the engine goes away.
    cudaStreamSynchronize(s);
  }

  void collect_loop() {
    cudaSetDevice(eng.ctx->device);
    for (;;) {
      std::shared_ptr<Request> r;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_collect.wait(lk, [&] { return stop || !finishing.empty(); });
        if (stop) return;
        r = finishing.front();
        finishing.pop_front();
      }
      const auto t0 = Clock::now();
      int st = TF_OK;
      if (r->status >= 0) {
        r->x.resize(r->n);
        st = tf_guarded([&] { return eng.fetch_x(r->slot, r->x.data(), fetch_stream); });
      }
      {
        std::lock_guard<std::mutex> el(eng.emu);
        eng.retire(r->slot);
      }
      std::lock_guard<std::mutex> lk(mu);
      if (st != TF_OK) r->status = -st;
      r->t_done = Clock::now();
      r->done = true;
      if (r->status >= 0) ++completed;
      --n_releasing;
      ++retire_gen;
      t_ms[4] += ms_since(t0);
      cv_admit.notify_all();
      cv_done.notify_all();
    }
  }
};

extern "C" int tf_server_create(tf_ctx ctx, const tf_batch_opts* opts, tf_server* out) {
  TF_API_BEGIN
  if (!ctx || !out) return TF_ERR_ARG;
  *out = nullptr;
  auto* s = new tf_server_s();
  int st = s->eng.init(ctx, opts);
  if (st == TF_OK) {
    cudaError_t e = cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->fetch_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      tf_set_last_cuda_error(e, "server copy stream", __FILE__, __LINE__);
      st = TF_ERR_CUDA;
    }
  }
  if (st != TF_OK) {
    delete s;
    return st;
  }
  s->worker = std::thread([s] { s->loop(); });
  s->admitter = std::thread([s] { s->admit_loop(); });
  s->collector = std::thread([s] { s->collect_loop(); });
  *out = s;
  return TF_OK;
  TF_API_END
}

extern "C" int tf_server_submit(tf_server sv, int n, int64_t nnz, const int* row,
                                const int* col, const int* dia, const double* val,
                                const double* b, const double* x0, double tol, int maxit,
                                int64_t* req) {
  TF_API_BEGIN
  if (!sv || !req) return TF_ERR_ARG;
  auto r = std::make_shared<Request>();
  const auto t0 = Clock::now();
  const int st = sv->eng.prepare(r->h, n, nnz, row, col, dia, val, b, x0, tol, maxit);
  if (st != TF_OK) return st;
  r->n = n;
  std::lock_guard<std::mutex> lk(sv->mu);
  sv->t_ms[0] += tf_server_s::ms_since(t0);
  if (sv->stop) return TF_ERR_CANCELLED;
  r->id = sv->next_id++;
  r->t_submit = Clock::now();
  sv->queue.push_back(r);
  sv->live[r->id] = r;
  *req = r->id;
  sv->cv_admit.notify_one();
  return TF_OK;
  TF_API_END
}

extern "C" int tf_server_wait(tf_server sv, int64_t req, double* x, int* iters,
                              double* true_rel_res, int* status, double* latency_ms,
                              double* queue_ms) {
  TF_API_BEGIN
  if (!sv) return TF_ERR_ARG;
  std::unique_lock<std::mutex> lk(sv->mu);
  auto it = sv->live.find(req);
  if (it == sv->live.end()) return TF_ERR_ARG;
  auto r = it->second;
  sv->cv_done.wait(lk, [&] { return r->done; });
  sv->live.erase(req);
  if (status) *status = r->status;
  if (iters) *iters = r->iters;
  if (true_rel_res) *true_rel_res = r->res;
  using ms = std::chrono::duration<double, std::milli>;
  if (latency_ms) *latency_ms = ms(r->t_done - r->t_submit).count();
  if (queue_ms)
    *queue_ms = r->slot >= 0 ? ms(r->t_admit - r->t_submit).count()
                             : ms(r->t_done - r->t_submit).count();
  if (r->status < 0) return -r->status;
  if (x && !r->x.empty()) memcpy(x, r->x.data(), r->x.size() * sizeof(double));
  return TF_OK;
  TF_API_END
}

extern "C" int tf_server_cancel(tf_server sv, int64_t req) {
  TF_API_BEGIN
  if (!sv) return TF_ERR_ARG;
  std::lock_guard<std::mutex> lk(sv->mu);
  auto it = sv->live.find(req);
  if (it == sv->live.end()) return TF_ERR_ARG;
  auto r = it->second;
  if (r->done) return TF_ERR_BUSY;            // finished: its result stands
  for (auto q = sv->queue.begin(); q != sv->queue.end(); ++q)
    if (*q == r) {                            // still queued
      sv->queue.erase(q);
      r->status = -TF_ERR_CANCELLED;
      r->t_done = Clock::now();
      r->done = true;
      sv->cv_done.notify_all();
      return TF_OK;
    }
  r->cancel = true;   // staged: given back at commit; running: retired after this sweep
  sv->cv_work.notify_one();
  return TF_OK;
  TF_API_END
}

extern "C" int tf_server_stats(tf_server sv, long long* admitted, long long* completed,
                               int* peak_running, int* sweeps) {
  TF_API_BEGIN
  if (!sv) return TF_ERR_ARG;
  std::lock_guard<std::mutex> lk(sv->mu);
  if (admitted) *admitted = sv->admitted;
  if (completed) *completed = sv->completed;
  if (peak_running) *peak_running = sv->peak_running;
  if (sweeps) *sweeps = sv->eng.sweeps;
  return sv->error;
  TF_API_END
}

extern "C" int tf_server_timing(tf_server sv, double* ms5) {
  TF_API_BEGIN
  if (!sv || !ms5) return TF_ERR_ARG;
  std::lock_guard<std::mutex> lk(sv->mu);
  for (int k = 0; k < 5; ++k) ms5[k] = sv->t_ms[k];
  return TF_OK;
  TF_API_END
}

extern "C" int tf_server_destroy(tf_server sv) {
  TF_API_BEGIN
  if (!sv) return TF_ERR_ARG;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->stop = true;
    for (auto& kv : sv->live)
      if (!kv.second->done) {
        kv.second->status = -TF_ERR_CANCELLED;
        kv.second->done = true;
      }
    sv->cv_work.notify_all();
    sv->cv_admit.notify_all();
    sv->cv_collect.notify_all();
    sv->cv_done.notify_all();
  }
  if (sv->worker.joinable()) sv->worker.join();
  if (sv->admitter.joinable()) sv->admitter.join();
  if (sv->collector.joinable()) sv->collector.join();
  cudaSetDevice(sv->eng.ctx->device);
  for (cudaStream_t st : {sv->copy_stream, sv->fetch_stream})
    if (st) {
      cudaStreamSynchronize(st);
      cudaStreamDestroy(st);
    }
  for (auto& r : sv->staged)
    if (r->ev) cudaEventDestroy(r->ev);
  delete sv;
  return TF_OK;
  TF_API_END
}

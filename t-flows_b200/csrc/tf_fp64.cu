// tf_fp64.cu -- FP64 drop-in for Native_Mod's Cg and Bicg (Jacobi / none /
// ICC preconditioning) on one B200.
//
// One solve is one CUDA graph:
//
//   k_diag -> k_scale -> k_residual -> WHILE(cond) { k_pupdate -> k_spmv_alpha
//                                                     -> k_update [-> ICC z] }
//          -> k_unscale
//
// k_diag/k_scale      normalisation of Cg.f90:62-84 (+ NRMS(b), :95-104)
// k_residual          r = b - A x and NRMS(r) (:109-123), rho of iteration 1
// k_pupdate           z = M^-1 r (Prec_Solve) and p = z + beta p (:145-171)
// k_spmv_alpha        q = A p, p.q, alfa = rho/(p.q)          (:176-198)
// k_update            x += alfa p, r -= alfa q, NRMS(r,x), next rho, the
//                     convergence test (:204-222) and the loop condition
// k_unscale           de-normalisation (:245-250)
//
// Convergence is decided on the device: k_update's last CTA writes the
// WHILE node's condition with cudaGraphSetConditional, so a whole solve is
// one graph launch with no host round trip per iteration.
//
// Bicg (Bicg.f90) is served by the same graph: its shadow sequence starts as
// r2 = r1 (:129-133) and is updated by exactly the operations applied to the
// primary sequence with A in place of A^T (:143-145, 178-181), so r2, z2, p2
// and q2 equal r1, z1, p1 and q1 bit for bit at every iteration, rho = z1.r1
// and alfa's denominator p2.q1 = p1.q1.  Computing the shadow would double
// the vector traffic and change no output.
//
// Rounding: every product and sum that the reference writes as a*b+c is
// issued as __dmul_rn then __dadd_rn (no FMA contraction), matching the
// reference's gnu build (-O3, x86-64 baseline, no FMA).  Row sums of the
// SpMV and of r = b - A x are accumulated in storage order, so q and r agree
// with the reference bit for bit given the same inputs; only the grid-wide
// dot products are summed in a different (fixed, deterministic) order.
#include <cuda_runtime.h>
#include <stdio.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <type_traits>
#include <vector>

#include "tf_icc.cuh"
#include "tf_internal.h"
#include "tf_tile.cuh"
#include "tf_tile2.cuh"

namespace tf {

struct VecArgs {
  int nt, ni;
  long long nnz;
  const int* dia;
  double* val;
  double* x;
  double* b;
  double* r;
  double* p;
  double* q;
  double* z;
  double* adiag;
  double* part;
  SolveState* st;
  const SolveParams* prm;
  cudaGraphConditionalHandle cond;
  int use_cond;
};

__device__ __forceinline__ void set_cond(const VecArgs& a, int v) {
  if (a.use_cond) cudaGraphSetConditional(a.cond, (unsigned)v);
}

// Fortran min/max as the reference's loops evaluate them.
__device__ __forceinline__ double fmin_ref(double a, double b) {
  return (b < a) ? b : a;
}
__device__ __forceinline__ double fmax_ref(double a, double b) {
  return (b > a) ? b : a;
}

// ---------------------------------------------------------------------------
// Normalisation (Cg.f90:62-76): adiag = diagonal, sum_a, fn = 1/(sum_a/ni)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_diag(VecArgs a) {
  __shared__ double scratch[32];
  double s = 0.0;
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.ni; i += stride) {
    const double d = a.val[a.dia[i]];
    a.adiag[i] = d;
    s = __dadd_rn(s, d);
  }
  s = block_red<kSum>(s, scratch);
  double v[1] = {s};
  const int ops[1] = {kSum};
  if (grid_reduce_last<1>(v, ops, a.part, &a.st->counter[kCntDiag], scratch) &&
      threadIdx.x == 0) {
    SolveState* st = a.st;
    st->sum_a = v[0];
    const double mean = __ddiv_rn(v[0], (double)a.ni);
    st->fn = __ddiv_rn(1.0, mean);
    st->done = 0;
    st->iter = 0;
    st->niter = 0;
    st->status = 0;
    st->bar_count = 0u;   // a timed-out ICC sweep may have left arrivals behind
    st->res = 0.0;
    st->rho = 0.0;
    st->rho_old = 0.0;
    st->alpha = 0.0;
    st->x_pend = 0;
  }
}

// val *= fn, b *= fn (Cg.f90:77-84); adiag *= fn; NRMS(b) (Cg.f90:95-104)
__global__ void __launch_bounds__(256) k_scale(VecArgs a) {
  __shared__ double scratch[32];
  const double fn = a.st->fn;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll 4
  for (long long j = tid; j < a.nnz; j += stride) a.val[j] = __dmul_rn(a.val[j], fn);
  const int has_norm = a.prm->has_norm;
  double s = 0.0, mn = kHuge, mx = -kHuge;
  for (long long i = tid; i < a.nt; i += stride) {
    const double bi = __dmul_rn(a.b[i], fn);
    a.b[i] = bi;
    if (i < a.ni) {
      const double ai = __dmul_rn(a.adiag[i], fn);
      a.adiag[i] = ai;
      s = __dadd_rn(s, nrms_term(bi, ai));
      if (!has_norm) {
        const double xi = a.x[i];
        mn = fmin_ref(mn, xi);
        mx = fmax_ref(mx, xi);
      }
    }
  }
  s = block_red<kSum>(s, scratch);
  mn = block_red<kMin>(mn, scratch);
  mx = block_red<kMax>(mx, scratch);
  double v[3] = {s, mn, mx};
  const int ops[3] = {kSum, kMin, kMax};
  if (grid_reduce_last<3>(v, ops, a.part, &a.st->counter[kCntScale], scratch) &&
      threadIdx.x == 0) {
    SolveState* st = a.st;
    st->xmin = v[1];
    st->xmax = v[2];
    const double bnrm2 = nrms_finish(v[0], has_norm, a.prm->norm, v[1], v[2]);
    st->bnrm2 = bnrm2;
    if (bnrm2 < a.prm->tol) {   // Cg.f90:101-104: iter = 0, res stays 0.0
      st->done = 1;
      st->niter = 0;
      st->res = 0.0;
      set_cond(a, 0);
    }
  }
}

// val /= fn, b /= fn (Cg.f90:245-250); the last x += alfa p when the
// update was deferred (k_update with XDEF).
__global__ void __launch_bounds__(256) k_unscale(VecArgs a) {
  const double fn = a.st->fn;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll 4
  for (long long j = tid; j < a.nnz; j += stride) a.val[j] = __ddiv_rn(a.val[j], fn);
  for (long long i = tid; i < a.nt; i += stride) a.b[i] = __ddiv_rn(a.b[i], fn);
  if (a.st->x_pend) {
    const double alpha = a.st->alpha;
    for (long long i = tid; i < a.ni; i += stride)
      a.x[i] = __dadd_rn(a.x[i], __dmul_rn(alpha, a.p[i]));
  }
}

// ---------------------------------------------------------------------------
// Per-row operators for the tile streamer
// ---------------------------------------------------------------------------
// Row sums visit the row's entries in storage order.  COL(k) gives the
// column of entry k: the staged column index (CSR tiles) or i + offset
// (row-pattern tiles); either way the same operands in the same order.

// q_i = sum_j a_ij p_j (Cg.f90:179-183), accumulates p_i q_i (:190-195)
struct OpSpmvDot {
  const double* __restrict__ p;
  double* __restrict__ q;
  double pq;
  template <class COL>
  __device__ __forceinline__ void body(int i, const double* v, COL col, int len) {
    double acc = 0.0;
#pragma unroll 1
    for (int k0 = 0; k0 < len; k0 += 8) {
      double pv[8], vv[8];
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (k0 + u < len) {
          vv[u] = v[k0 + u];
          pv[u] = __ldg(p + col(k0 + u));
        }
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (k0 + u < len) acc = __dadd_rn(acc, __dmul_rn(vv[u], pv[u]));
    }
    q[i] = acc;
    pq = __dadd_rn(pq, __dmul_rn(__ldg(p + i), acc));
  }
  __device__ __forceinline__ void operator()(int i, const double* v, const int* c, int len) {
    body(i, v, [c](int k) { return c[k]; }, len);
  }
  __device__ __forceinline__ void pat(int i, const double* v, const int* o, int len) {
    body(i, v, [i, o](int k) { return i + o[k]; }, len);
  }
  // per-row hooks (row-pattern and CSR streamers)
  static constexpr bool kRowOps = true;
  __device__ __forceinline__ void begin(int, TileAux) {}
  static constexpr bool kReducer = false;
  __device__ __forceinline__ double gather(int c) const { return __ldg(p + c); }
  __device__ __forceinline__ double row_init(int) const { return 0.0; }
  __device__ __forceinline__ double combine(double acc, double prod) const {
    return __dadd_rn(acc, prod);
  }
  __device__ __forceinline__ void row_done(int i, double acc) {
    q[i] = acc;
    pq = __dadd_rn(pq, __dmul_rn(__ldg(p + i), acc));
  }
  __device__ __forceinline__ void tile_end(int) {}
};

// r_i = b_i - sum_j a_ij x_j (Residual_Vector.f90:35-41), accumulates the
// NRMS term and rho = z.r for Jacobi / none.
template <int PREC>
struct OpResidual {
  const double* __restrict__ x;
  const double* __restrict__ b;
  double* __restrict__ r;
  const double* __restrict__ adiag;
  double s, rho;
  template <class COL>
  __device__ __forceinline__ void body(int i, const double* v, COL col, int len) {
    double acc = b[i];
#pragma unroll 1
    for (int k0 = 0; k0 < len; k0 += 8) {
      double xv[8], vv[8];
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (k0 + u < len) {
          vv[u] = v[k0 + u];
          xv[u] = __ldg(x + col(k0 + u));
        }
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (k0 + u < len) acc = __dsub_rn(acc, __dmul_rn(vv[u], xv[u]));
    }
    r[i] = acc;
    const double ai = adiag[i];
    s = __dadd_rn(s, nrms_term(acc, ai));
    if (PREC == kPrecJacobi) {
      const double zi = __dmul_rn(acc, __drcp_rn(ai));
      rho = __dadd_rn(rho, __dmul_rn(zi, acc));
    } else if (PREC == kPrecNone) {
      rho = __dadd_rn(rho, __dmul_rn(acc, acc));
    }
  }
  __device__ __forceinline__ void operator()(int i, const double* v, const int* c, int len) {
    body(i, v, [c](int k) { return c[k]; }, len);
  }
  __device__ __forceinline__ void pat(int i, const double* v, const int* o, int len) {
    body(i, v, [i, o](int k) { return i + o[k]; }, len);
  }
  // per-row hooks (row-pattern and CSR streamers)
  static constexpr bool kRowOps = true;
  __device__ __forceinline__ void begin(int, TileAux) {}
  static constexpr bool kReducer = false;
  __device__ __forceinline__ double gather(int c) const { return __ldg(x + c); }
  __device__ __forceinline__ double row_init(int i) const { return b[i]; }
  __device__ __forceinline__ double combine(double acc, double prod) const {
    return __dsub_rn(acc, prod);
  }
  __device__ __forceinline__ void row_done(int i, double acc) {
    r[i] = acc;
    const double ai = adiag[i];
    s = __dadd_rn(s, nrms_term(acc, ai));
    if (PREC == kPrecJacobi) {
      const double zi = __dmul_rn(acc, __drcp_rn(ai));
      rho = __dadd_rn(rho, __dmul_rn(zi, acc));
    } else if (PREC == kPrecNone) {
      rho = __dadd_rn(rho, __dmul_rn(acc, acc));
    }
  }
  __device__ __forceinline__ void tile_end(int) {}
};

// Fixed tiles of ROWS rows over one matrix (the drop-in's tile source).
template <int ROWS>
struct FixedTiles {
  const int* row;
  const int* col;
  const double* val;
  int nrows;
  __device__ int count() const { return (nrows + ROWS - 1) / ROWS; }
  __device__ TileDesc desc(int k) const {
    TileDesc d;
    d.row = row;
    d.col = col;
    d.val = val;
    d.r0 = k * ROWS;
    d.r1 = min(d.r0 + ROWS, nrows);
    d.j0 = __ldg(row + d.r0);
    d.j1 = __ldg(row + d.r1);
    d.skip = 0;
    d.aux0 = nullptr;
    d.aux1 = nullptr;
    d.aux2 = d.aux3 = 0;
    return d;
  }
};

// Variable-length tiles over one matrix: tile k is rows [tiles[k],
// tiles[k+1]) (the drop-in's tile source for the var configurations).
struct VarTiles {
  const int* row;
  const int* col;
  const double* val;
  const int* tiles;
  int ntiles;
  __device__ int count() const { return ntiles; }
  __device__ TileDesc desc(int k) const {
    TileDesc d;
    d.row = row;
    d.col = col;
    d.val = val;
    d.r0 = __ldg(tiles + k);
    d.r1 = __ldg(tiles + k + 1);
    d.j0 = __ldg(row + d.r0);
    d.j1 = __ldg(row + d.r1);
    d.skip = 0;
    d.aux0 = nullptr;
    d.aux1 = nullptr;
    d.aux2 = d.aux3 = 0;
    return d;
  }
};

struct SpArgs {
  const int* row;
  const int* col;
  const double* val;
  PatTable pt;       // row patterns (pt.npat > 0 when the PAT kernels run)
  const int* tiles;  // variable tiles (var configurations)
  int ntiles;
  int nrows;
  VecArgs v;
  double* out_scalar;  // building-block mode: receives the dot product
};

// Rows through shared-memory tiles (CFG < kTileNone; PAT: row-pattern
// columns) or straight from global memory (kTileNone: rows too long for
// any tile).
template <int CFG, int PAT, class Op>
__device__ __forceinline__ bool run_rows(const SpArgs& a, Op& op) {
  if constexpr (CFG != kTileNone && PAT) {
    return stream_tiles_pat<kTileRows[CFG], kTileNnzCap[CFG], kPatStages>(
        a.row, a.pt, a.val, a.nrows, op, wait_limit(a.v.prm));
  } else if constexpr (CFG == kTileNone) {
    const int stride = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.nrows; i += stride) {
      const int js = a.row[i], je = a.row[i + 1];
      op(i, a.val + js, a.col + js, je - js);
    }
    return true;
  } else if constexpr (tile_is_var(CFG)) {
    VarTiles src{a.row, a.col, a.val, a.tiles, a.ntiles};
    return stream_csr2<kTileRows[CFG], kTileNnzCap[CFG], 2, tile_var_g(CFG)>(
        src, op, wait_limit(a.v.prm));
  } else {
    FixedTiles<kTileRows[CFG]> src{a.row, a.col, a.val, a.nrows};
    return stream_csr2<kTileRows[CFG], kTileNnzCap[CFG], 2>(src, op, wait_limit(a.v.prm));
  }
}

template <int CFG, int PAT = 0>
constexpr int cfg_threads() {
  if constexpr (CFG == kTileNone) return 256;
  else if constexpr (PAT != 0) return pat_threads<kTileRows[CFG]>();
  else return kCsr2Threads;
}
// Two CTAs per SM: caps the tiled kernels (consumers + a producer warp) at
// the registers that two of them can hold.
template <int CFG, int PAT>
constexpr int cfg_min_blocks() { return CFG != kTileNone ? 2 : 1; }

__device__ __forceinline__ void flag_timeout(SolveState* st) {
  if (st) atomicExch(&st->status, (int)TF_ERR_TIMEOUT);
}

// r = b - A x, NRMS(r) (Cg.f90:109-123), rho of iteration 1.
template <int CFG, int PREC, int PAT>
__global__ void __launch_bounds__(cfg_threads<CFG, PAT>(), cfg_min_blocks<CFG, PAT>())
    k_residual(SpArgs a) {
  __shared__ double scratch[32];
  SolveState* st = a.v.st;
  if (st && st->done) return;
  OpResidual<PREC> op{a.v.x, a.v.b, a.v.r, a.v.adiag, 0.0, 0.0};
  if (!run_rows<CFG, PAT>(a, op) && threadIdx.x == 0) flag_timeout(st);
  double v[2] = {block_red<kSum>(op.s, scratch), block_red<kSum>(op.rho, scratch)};
  const int ops[2] = {kSum, kSum};
  unsigned* cnt = st ? &st->counter[kCntResid] : reinterpret_cast<unsigned*>(a.out_scalar + 1);
  if (grid_reduce_last<2>(v, ops, a.v.part, cnt, scratch) && threadIdx.x == 0) {
    if (!st) return;
    const SolveParams* prm = a.v.prm;
    const double res = nrms_finish(v[0], prm->has_norm, prm->norm, st->xmin, st->xmax);
    st->res = res;
    if (prm->hist && prm->hist_cap > 0) prm->hist[0] = res;
    if (st->status != 0 || res < prm->tol || prm->miter < 1) {
      st->done = 1;   // Cg.f90:120-123 (iter = 0), or a zero-trip loop
      st->niter = 0;
      set_cond(a.v, 0);
    } else {
      if (PREC != kPrecIcc) st->rho = v[1];
      st->iter = 1;
      set_cond(a.v, 1);
    }
  }
}

// Vector kernels walk the rows in pairs (16-byte loads) and, per step,
// load kBatch pairs into registers before computing any of them, so each
// thread keeps kBatch x (arrays read) x 16 bytes in flight.  Pair j of
// step t is base + u * stride for u < kBatch (coalesced across a warp).
// DESC walks pairs from the top down: the rows a kernel touches last are
// still in L2 when the next kernel, walking the other way, starts on them.
constexpr int kBatch = 2;

__device__ __forceinline__ int pair_index(int j, int np, bool desc) {
  return desc ? np - 1 - j : j;
}

// z = M^-1 r (Prec_Solve.f90:44-49 / :97-102) and p = z + beta p
// (Cg.f90:158-171).  ICC reads z from the triangular solves.  XDEF: the
// previous iteration's x += alfa p (Cg.f90:204-206) is applied here, just
// before p is overwritten, instead of in k_update -- same operands, same
// rounding, one pass over p fewer.
template <int PREC, int XDEF, int DESC>
__global__ void __launch_bounds__(256) k_pupdate(VecArgs a) {
  const SolveState* st = a.st;
  if (st->done) return;
  const int k = st->iter;
  const bool first = (k == 1);
  const double beta = first ? 0.0 : __ddiv_rn(st->rho, st->rho_old);
  const double alpha = st->alpha;   // alfa of iteration k-1
  const double2* __restrict__ r2 = reinterpret_cast<const double2*>(PREC == kPrecIcc ? a.z : a.r);
  const double2* __restrict__ a2 = reinterpret_cast<const double2*>(a.adiag);
  double2* __restrict__ p2 = reinterpret_cast<double2*>(a.p);
  double2* __restrict__ x2 = reinterpret_cast<double2*>(a.x);
  const int np = a.ni >> 1;
  const int stride = gridDim.x * blockDim.x;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  auto zval = [&](double ri, double ai) {
    if (PREC == kPrecJacobi) return __dmul_rn(ri, __drcp_rn(ai));
    return ri;
  };
  auto pval = [&](double zi, double pi) {
    return first ? zi : __dadd_rn(zi, __dmul_rn(beta, pi));
  };
  for (int base = tid; base < np; base += kBatch * stride) {
    double2 rv[kBatch], av[kBatch], pv[kBatch], xv[kBatch];
#pragma unroll
    for (int u = 0; u < kBatch; ++u) {
      const int j = base + u * stride;
      if (j < np) {
        const int jj = pair_index(j, np, DESC);
        rv[u] = r2[jj];
        if (PREC == kPrecJacobi) av[u] = a2[jj];
        if (!first) pv[u] = p2[jj];
        if (XDEF && !first) xv[u] = x2[jj];
      }
    }
#pragma unroll
    for (int u = 0; u < kBatch; ++u) {
      const int j = base + u * stride;
      if (j < np) {
        const int jj = pair_index(j, np, DESC);
        if (XDEF && !first) {
          xv[u].x = __dadd_rn(xv[u].x, __dmul_rn(alpha, pv[u].x));
          xv[u].y = __dadd_rn(xv[u].y, __dmul_rn(alpha, pv[u].y));
          x2[jj] = xv[u];
        }
        double2 o;
        o.x = pval(zval(rv[u].x, PREC == kPrecJacobi ? av[u].x : 1.0), pv[u].x);
        o.y = pval(zval(rv[u].y, PREC == kPrecJacobi ? av[u].y : 1.0), pv[u].y);
        p2[jj] = o;
      }
    }
  }
  if ((a.ni & 1) && tid == 0) {   // the odd last row
    const int i = a.ni - 1;
    const double ri = (PREC == kPrecIcc) ? a.z[i] : a.r[i];
    const double pi = first ? 0.0 : a.p[i];
    if (XDEF && !first) a.x[i] = __dadd_rn(a.x[i], __dmul_rn(alpha, pi));
    a.p[i] = pval(zval(ri, PREC == kPrecJacobi ? a.adiag[i] : 1.0), pi);
  }
}

// q = A p, p.q, alfa = rho / p.q (Cg.f90:176-198)
template <int CFG, int PAT>
__global__ void __launch_bounds__(cfg_threads<CFG, PAT>(), cfg_min_blocks<CFG, PAT>())
    k_spmv_alpha(SpArgs a) {
  __shared__ double scratch[32];
  SolveState* st = a.v.st;
  if (st && st->done) return;
  OpSpmvDot op{a.v.p, a.v.q, 0.0};
  if (!run_rows<CFG, PAT>(a, op) && threadIdx.x == 0) flag_timeout(st);
  double v[1] = {block_red<kSum>(op.pq, scratch)};
  const int ops[1] = {kSum};
  unsigned* cnt = st ? &st->counter[kCntSpmv] : reinterpret_cast<unsigned*>(a.out_scalar + 1);
  if (grid_reduce_last<1>(v, ops, a.v.part, cnt, scratch) && threadIdx.x == 0) {
    if (a.out_scalar) a.out_scalar[0] = v[0];
    if (st) {
      st->pq = v[0];
      st->alpha = __ddiv_rn(st->rho, v[0]);
    }
  }
}

// r -= alfa q (Cg.f90:207-209) and, unless deferred to the next k_pupdate
// (XDEF), x += alfa p (:204-206); NRMS(r, x) and the test (:214-222); rho
// for the next iteration (Jacobi / none).  XDEF requires norm present (the
// NRMS then does not look at x).
template <int PREC, int XDEF, int DESC>
__global__ void __launch_bounds__(256, 3) k_update(VecArgs a) {
  __shared__ double scratch[4 * 32];
  SolveState* st = a.st;
  if (st->done) {
    if (blockIdx.x == 0 && threadIdx.x == 0) set_cond(a, 0);
    return;
  }
  const double alpha = st->alpha;
  const SolveParams* prm = a.prm;
  const int has_norm = prm->has_norm;
  double s = 0.0, rho = 0.0, mn = kHuge, mx = -kHuge;
  double2* __restrict__ r2 = reinterpret_cast<double2*>(a.r);
  const double2* __restrict__ q2 = reinterpret_cast<const double2*>(a.q);
  const double2* __restrict__ a2 = reinterpret_cast<const double2*>(a.adiag);
  const double2* __restrict__ p2 = reinterpret_cast<const double2*>(a.p);
  double2* __restrict__ x2 = reinterpret_cast<double2*>(a.x);
  const int np = a.ni >> 1;
  const int stride = gridDim.x * blockDim.x;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  // one row: returns the new r; accumulates the NRMS term, rho, x range
  auto row = [&](double ri, double qi, double ai) {
    ri = __dsub_rn(ri, __dmul_rn(alpha, qi));
    s = __dadd_rn(s, nrms_term(ri, ai));
    if (PREC == kPrecJacobi) {
      const double zi = __dmul_rn(ri, __drcp_rn(ai));
      rho = __dadd_rn(rho, __dmul_rn(zi, ri));
    } else if (PREC == kPrecNone) {
      rho = __dadd_rn(rho, __dmul_rn(ri, ri));
    }
    return ri;
  };
  auto xrow = [&](double xi, double pi) {
    xi = __dadd_rn(xi, __dmul_rn(alpha, pi));
    if (!has_norm) {
      mn = fmin_ref(mn, xi);
      mx = fmax_ref(mx, xi);
    }
    return xi;
  };
  for (int base = tid; base < np; base += kBatch * stride) {
    double2 rv[kBatch], qv[kBatch], av[kBatch], pv[kBatch], xv[kBatch];
#pragma unroll
    for (int u = 0; u < kBatch; ++u) {
      const int j = base + u * stride;
      if (j < np) {
        const int jj = pair_index(j, np, DESC);
        rv[u] = r2[jj];
        qv[u] = q2[jj];
        av[u] = a2[jj];
        if (!XDEF) {
          pv[u] = p2[jj];
          xv[u] = x2[jj];
        }
      }
    }
#pragma unroll
    for (int u = 0; u < kBatch; ++u) {
      const int j = base + u * stride;
      if (j < np) {
        const int jj = pair_index(j, np, DESC);
        if (!XDEF) {   // the reference's order: x first (:204-206), then r
          xv[u].x = xrow(xv[u].x, pv[u].x);
          xv[u].y = xrow(xv[u].y, pv[u].y);
          x2[jj] = xv[u];
        }
        double2 o;
        o.x = row(rv[u].x, qv[u].x, av[u].x);
        o.y = row(rv[u].y, qv[u].y, av[u].y);
        r2[jj] = o;
      }
    }
  }
  if ((a.ni & 1) && tid == 0) {   // the odd last row
    const int i = a.ni - 1;
    if (!XDEF) a.x[i] = xrow(a.x[i], a.p[i]);
    a.r[i] = row(a.r[i], a.q[i], a.adiag[i]);
  }
  double v[4] = {s, rho, mn, mx};
  const int ops[4] = {kSum, kSum, kMin, kMax};
  block_red_n<4>(v, ops, scratch);
  if (grid_reduce_last_n<4>(v, ops, a.part, &st->counter[kCntUpdate], scratch) &&
      threadIdx.x == 0) {
    const double res = nrms_finish(v[0], has_norm, prm->norm, v[2], v[3]);
    st->res = res;
    const int k = st->iter;
    if (prm->hist && k < prm->hist_cap) prm->hist[k] = res;
    if (st->status != 0) {
      st->done = 1;
      st->niter = k;
    } else if (res < prm->tol) {         // Cg.f90:220
      st->done = 1;
      st->niter = k;
    } else if (k >= prm->miter) {        // loop exhausted: niter = miter
      st->done = 1;
      st->niter = prm->miter;
    } else {
      if (PREC != kPrecIcc) {            // Cg.f90:222 and :150-156
        st->rho_old = st->rho;
        st->rho = v[1];
      }
      st->iter = k + 1;
    }
    if (XDEF && st->done) st->x_pend = 1;   // k_unscale applies the last alfa p
    set_cond(a, st->done ? 0 : 1);
  }
}

}  // namespace tf

using namespace tf;

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
namespace {

template <int V>
using IC = std::integral_constant<int, V>;

// Calls f(IC<CFG>, IC<PAT>) for the matrix's tile configuration.
template <class F>
auto dispatch_cfg(int cfg, bool pat, F&& f) {
  switch (cfg) {
    case kTile512: return pat ? f(IC<kTile512>{}, IC<1>{}) : f(IC<kTile512>{}, IC<0>{});
    case kTile256: return pat ? f(IC<kTile256>{}, IC<1>{}) : f(IC<kTile256>{}, IC<0>{});
    case kTile128: return pat ? f(IC<kTile128>{}, IC<1>{}) : f(IC<kTile128>{}, IC<0>{});
    case kTileVar1: return f(IC<kTileVar1>{}, IC<0>{});
    case kTileVar2: return f(IC<kTileVar2>{}, IC<0>{});
    case kTileVar4: return f(IC<kTileVar4>{}, IC<0>{});
    case kTileVar8: return f(IC<kTileVar8>{}, IC<0>{});
    default: return f(IC<kTileNone>{}, IC<0>{});
  }
}

template <int CFG, int PAT>
size_t cfg_smem() {
  if constexpr (CFG == kTileNone) return 0;
  else if constexpr (PAT)
    return PatLayout<kTileRows[CFG], kTileNnzCap[CFG], kPatStages>::kSmemBytes;
  else return Csr2Layout<kTileRows[CFG], kTileNnzCap[CFG], 2>::kSmemBytes;
}

template <int CFG, int PREC, int PAT>
int set_attrs_cfg() {
  const size_t sm = cfg_smem<CFG, PAT>();
  if (sm > 48 * 1024) {
    TF_CUDA_TRY(cudaFuncSetAttribute(k_residual<CFG, PREC, PAT>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    TF_CUDA_TRY(cudaFuncSetAttribute(k_spmv_alpha<CFG, PAT>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  }
  return TF_OK;
}

VecArgs make_vec_args(tf_matrix_s* m) {
  VecArgs a{};
  a.nt = m->nt;
  a.ni = m->ni;
  a.nnz = (long long)m->nnz;
  a.dia = m->d_dia;
  a.val = m->d_val;
  a.x = m->d_x;
  a.b = m->d_b;
  a.r = m->d_r;
  a.p = m->d_p;
  a.q = m->d_q;
  a.z = m->d_z;
  a.adiag = m->d_adiag;
  a.part = m->d_part;
  a.st = m->d_state;
  a.prm = m->d_params;
  a.cond = 0;
  a.use_cond = 0;
  return a;
}

SpArgs make_sp_args(tf_matrix_s* m, const VecArgs& v) {
  SpArgs s{};
  s.row = m->d_row;
  s.col = m->d_col;
  s.val = m->d_val;
  s.pt.pat = m->d_pat;
  s.pt.tab = m->d_pat_tab;
  s.pt.npat = m->npat;
  s.tiles = m->d_tiles;
  s.ntiles = m->ntiles;
  s.nrows = m->ni;
  s.v = v;
  s.out_scalar = nullptr;
  return s;
}

struct NodeBuilder {
  cudaGraph_t g;
  int status = TF_OK;
  cudaGraphNode_t add(const void* fn, dim3 grid, dim3 block, size_t smem,
                      void** args, cudaGraphNode_t dep) {
    if (status != TF_OK) return nullptr;
    cudaKernelNodeParams p{};
    p.func = const_cast<void*>(fn);
    p.gridDim = grid;
    p.blockDim = block;
    p.sharedMemBytes = (unsigned)smem;
    p.kernelParams = args;
    p.extra = nullptr;
    cudaGraphNode_t node = nullptr;
    cudaError_t e = cudaGraphAddKernelNode(&node, g, dep ? &dep : nullptr, dep ? 1 : 0, &p);
    if (e != cudaSuccess) {
      tf_set_last_cuda_error(e, "cudaGraphAddKernelNode", __FILE__, __LINE__);
      status = TF_ERR_CUDA;
    }
    return node;
  }
  // A kernel node launched cooperatively (all its CTAs resident at once).
  cudaGraphNode_t add_coop(const void* fn, dim3 grid, dim3 block, void** args,
                           cudaGraphNode_t dep) {
    cudaGraphNode_t node = add(fn, grid, block, 0, args, dep);
    if (status != TF_OK) return nullptr;
    cudaKernelNodeAttrValue v{};
    v.cooperative = 1;
    cudaError_t e = cudaGraphKernelNodeSetAttribute(node, cudaKernelNodeAttributeCooperative, &v);
    if (e != cudaSuccess) {
      tf_set_last_cuda_error(e, "cudaGraphKernelNodeSetAttribute(cooperative)", __FILE__,
                             __LINE__);
      status = TF_ERR_CUDA;
    }
    return node;
  }
};

// Arguments of the persistent ICC sweeps.
struct IccSweeps {
  IccSweepArgs form, fwd, bwd;
};
IccArgs icc_args(tf_matrix_s* m);
IccSweeps icc_sweep_args(tf_matrix_s* m) {
  IccSweeps w{};
  IccArgs a = icc_args(m);
  a.rows = m->d_levf_rows;
  w.fwd = IccSweepArgs{a, m->d_icc_levf_ptr, (int)m->h_levf_ptr.size() - 1, m->d_state,
                       m->d_params};
  w.form = w.fwd;
  w.form.a.st = nullptr;
  a.rows = m->d_levb_rows;
  w.bwd = IccSweepArgs{a, m->d_icc_levb_ptr, (int)m->h_levb_ptr.size() - 1, m->d_state,
                       m->d_params};
  return w;
}

IccArgs icc_args(tf_matrix_s* m) {
  IccArgs a{};
  a.row = m->d_row;
  a.col = m->d_col;
  a.val = m->d_val;
  a.ni = m->ni;
  a.d = m->d_icc_d;
  a.d_inv = m->d_icc_dinv;
  a.r = m->d_r;
  a.y = m->d_q;   // q is free between k_update and the next SpMV
  a.z = m->d_z;
  a.st = m->d_state;
  return a;
}

// Per-level kernel arguments, kept alive while a graph is built.
struct IccLevelArgs {
  std::vector<IccArgs> form, fwd, bwd;
};

IccLevelArgs icc_level_args(tf_matrix_s* m) {
  IccLevelArgs L;
  const IccArgs base = icc_args(m);
  for (size_t l = 0; l + 1 < m->h_levf_ptr.size(); ++l) {
    IccArgs a = base;
    a.rows = m->d_levf_rows + m->h_levf_ptr[l];
    a.count = m->h_levf_ptr[l + 1] - m->h_levf_ptr[l];
    L.fwd.push_back(a);
    a.st = nullptr;
    L.form.push_back(a);
  }
  for (size_t l = 0; l + 1 < m->h_levb_ptr.size(); ++l) {
    IccArgs a = base;
    a.rows = m->d_levb_rows + m->h_levb_ptr[l];
    a.count = m->h_levb_ptr[l + 1] - m->h_levb_ptr[l];
    L.bwd.push_back(a);
  }
  return L;
}

struct RhoArgs {
  int ni;
  const double* z;
  const double* r;
  double* part;
  SolveState* st;
};

// The iteration's vector kernels for this solve: xdef defers x += alfa p
// to the next k_pupdate (norm present; Jacobi / none only).  vec_dir 0
// walks k_update up and k_pupdate down, 1 the reverse.
struct IterFns {
  const void* pupdate;
  const void* update;
};
template <int PREC>
IterFns iter_fns(int xdef, int dir) {
  if (PREC == kPrecIcc) xdef = 0;
  if (xdef) {
    if (dir) return {(const void*)k_pupdate<PREC, 1, 0>, (const void*)k_update<PREC, 1, 1>};
    return {(const void*)k_pupdate<PREC, 1, 1>, (const void*)k_update<PREC, 1, 0>};
  }
  if (dir) return {(const void*)k_pupdate<PREC, 0, 0>, (const void*)k_update<PREC, 0, 1>};
  return {(const void*)k_pupdate<PREC, 0, 1>, (const void*)k_update<PREC, 0, 0>};
}

template <int CFG, int PREC, int PAT>
int build_graph_t(tf_matrix_s* m, int xdef, cudaGraphExec_t* out) {
  int st = set_attrs_cfg<CFG, PREC, PAT>();
  if (st != TF_OK) return st;
  cudaGraph_t g = nullptr;
  TF_CUDA_TRY(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle h = 0;
  cudaError_t e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    TF_CUDA_TRY(e);
  }
  VecArgs va = make_vec_args(m);
  va.cond = h;
  va.use_cond = 1;
  SpArgs sa = make_sp_args(m, va);
  const dim3 vb(256), vg(m->vec_grid);
  const dim3 sb(cfg_threads<CFG, PAT>()), sg(m->spmv_grid);
  const size_t ssm = cfg_smem<CFG, PAT>();

  NodeBuilder nb{g};
  void* vargs[] = {&va};
  void* sargs[] = {&sa};
  IccLevelArgs lv;
  RhoArgs ra{m->ni, m->d_z, m->d_r, m->d_part, m->d_state};
  void* rargs[] = {&ra.ni, &ra.z, &ra.r, &ra.part, &ra.st};
  std::vector<void*> form_args, fwd_args, bwd_args;
  IccSweeps sw{};
  void* sw_form[] = {&sw.form};
  void* sw_fwd[] = {&sw.fwd};
  void* sw_bwd[] = {&sw.bwd};
  const bool sweeps = PREC == kPrecIcc && m->icc_sweep_grid > 0;
  const dim3 swg(std::max(1, m->icc_sweep_grid));
  if (PREC == kPrecIcc) {
    lv = icc_level_args(m);
    sw = icc_sweep_args(m);
    for (auto& a : lv.form) form_args.push_back(&a);
    for (auto& a : lv.fwd) fwd_args.push_back(&a);
    for (auto& a : lv.bwd) bwd_args.push_back(&a);
  }
  auto lgrid = [](int count) { return dim3(std::max(1, (count + 255) / 256)); };
  // z = M^-1 r by the two triangular sweeps (persistent kernels, or one
  // kernel per level), then rho = z.r
  auto add_icc_apply = [&](NodeBuilder& b, cudaGraphNode_t dep) {
    if (sweeps) {
      dep = b.add_coop((const void*)k_icc_sweep<kSweepFwd>, swg, dim3(256), sw_fwd, dep);
      dep = b.add_coop((const void*)k_icc_sweep<kSweepBwd>, swg, dim3(256), sw_bwd, dep);
    } else {
      for (size_t l = 0; l < lv.fwd.size(); ++l)
        dep = b.add((const void*)k_icc_fwd_level, lgrid(lv.fwd[l].count), dim3(256), 0,
                    &fwd_args[l], dep);
      for (size_t l = 0; l < lv.bwd.size(); ++l)
        dep = b.add((const void*)k_icc_bwd_level, lgrid(lv.bwd[l].count), dim3(256), 0,
                    &bwd_args[l], dep);
    }
    return b.add((const void*)k_icc_rho, vg, vb, 0, rargs, dep);
  };
  cudaGraphNode_t n1 = nb.add((const void*)k_diag, vg, vb, 0, vargs, nullptr);
  cudaGraphNode_t n2 = nb.add((const void*)k_scale, vg, vb, 0, vargs, n1);
  if (PREC == kPrecIcc && sweeps)   // Prec_Form (Cg.f90:89) on the scaled matrix
    n2 = nb.add_coop((const void*)k_icc_sweep<kSweepForm>, swg, dim3(256), sw_form, n2);
  else if (PREC == kPrecIcc)
    for (size_t l = 0; l < lv.form.size(); ++l)
      n2 = nb.add((const void*)k_icc_form_level, lgrid(lv.form[l].count), dim3(256), 0,
                  &form_args[l], n2);
  cudaGraphNode_t n3 = nb.add((const void*)k_residual<CFG, PREC, PAT>, sg, sb, ssm, sargs, n2);
  cudaGraphNode_t last = n3;
  if (PREC == kPrecIcc) last = add_icc_apply(nb, last);
  cudaGraphNode_t cnode = nullptr;
  if (nb.status == TF_OK) {
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    e = cudaGraphAddNode(&cnode, g, &last, 1, &cp);
    if (e != cudaSuccess) {
      tf_set_last_cuda_error(e, "cudaGraphAddNode(conditional)", __FILE__, __LINE__);
      nb.status = TF_ERR_CUDA;
    } else {
      NodeBuilder body{cp.conditional.phGraph_out[0]};
      const IterFns fns = iter_fns<PREC>(xdef, m->vec_dir);
      cudaGraphNode_t b1 = body.add(fns.pupdate, vg, vb, 0, vargs, nullptr);
      cudaGraphNode_t b2 = body.add((const void*)k_spmv_alpha<CFG, PAT>, sg, sb, ssm, sargs, b1);
      cudaGraphNode_t b3 = body.add(fns.update, vg, vb, 0, vargs, b2);
      if (PREC == kPrecIcc) add_icc_apply(body, b3);
      if (body.status != TF_OK) nb.status = body.status;
    }
  }
  nb.add((const void*)k_unscale, vg, vb, 0, vargs, cnode);
  if (nb.status != TF_OK) {
    cudaGraphDestroy(g);
    return nb.status;
  }
  e = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  TF_CUDA_TRY(e);
  return TF_OK;
}

template <int PREC>
int build_graph_p(tf_matrix_s* m, int xdef, cudaGraphExec_t* out) {
  return dispatch_cfg(m->tile_cfg, m->npat > 0, [&](auto C, auto P) {
    return build_graph_t<decltype(C)::value, PREC, decltype(P)::value>(m, xdef, out);
  });
}

template <int CFG>
int occupancy_grid(tf_matrix_s* m, const void* fn, int threads, size_t smem,
                   int nrows, int* grid) {
  int per_sm = 0;
  TF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem));
  if (per_sm < 1) per_sm = 1;
  int units = (CFG == kTileNone)     ? (nrows + threads - 1) / threads
              : tile_is_var(CFG)      ? m->ntiles
                                      : (nrows + kTileRows[CFG] - 1) / kTileRows[CFG];
  int g = std::min(units, per_sm * m->ctx->sm_count);
  g = std::max(1, std::min(g, kMaxBlocks));
  *grid = g;
  return TF_OK;
}

template <int CFG, int PAT>
int prepare_cfg(tf_matrix_s* m) {
  int st = set_attrs_cfg<CFG, kPrecJacobi, PAT>();
  if (st != TF_OK) return st;
  st = set_attrs_cfg<CFG, kPrecNone, PAT>();
  if (st != TF_OK) return st;
  st = set_attrs_cfg<CFG, kPrecIcc, PAT>();
  if (st != TF_OK) return st;
  return occupancy_grid<CFG>(m, (const void*)k_spmv_alpha<CFG, PAT>, cfg_threads<CFG, PAT>(),
                             cfg_smem<CFG, PAT>(), m->ni, &m->spmv_grid);
}

}  // namespace

int tf_icc_prepare_sweeps(tf_matrix_s* m) {
  m->icc_sweep_grid = 0;
  if (!getenv("TF_ICC_PERSISTENT")) return TF_OK;
  int coop = 0;
  TF_CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, m->ctx->device));
  if (!coop) return TF_OK;
  int per_sm = 1 << 30;
  for (const void* fn : {(const void*)k_icc_sweep<kSweepForm>, (const void*)k_icc_sweep<kSweepFwd>,
                         (const void*)k_icc_sweep<kSweepBwd>}) {
    int b = 0;
    TF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, 256, 0));
    per_sm = std::min(per_sm, b);
  }
  if (per_sm < 1) return TF_OK;
  // One CTA of 256 threads per SM: a level of a 200^3 hex grid has at most
  // ~30,000 rows (about one per thread), and every CTA joins every barrier.
  int widest = 1;
  for (const auto* ptr : {&m->h_levf_ptr, &m->h_levb_ptr})
    for (size_t l = 0; l + 1 < ptr->size(); ++l) widest = std::max(widest, (*ptr)[l + 1] - (*ptr)[l]);
  m->icc_sweep_grid = std::max(1, std::min(m->ctx->sm_count, (widest + 255) / 256));
  return TF_OK;
}

// ---------------------------------------------------------------------------
// SpMV layout choice: the autotuner
// ---------------------------------------------------------------------------
namespace {

constexpr int kTuneMinRows = 16384;   // below: launch latency dominates, use the rule
constexpr int kTuneReps = 5;

std::mutex g_tune_mu;
std::map<std::vector<long long>, int> g_tune_cache;

// Matrices of one class share a layout: device, row patterns or not, size
// (power of two of the rows), mean entries per row (halves), longest row
// (eighths of 64).
std::vector<long long> tune_key(const tf_matrix_s* m) {
  const double mean = m->ni > 0 ? (double)m->nnz / (double)m->nt : 0.0;
  int lg = 0;
  while ((1 << (lg + 1)) <= m->ni) ++lg;
  return {m->ctx->device, m->npat > 0, lg, (long long)std::lround(2.0 * mean),
          std::min(m->max_row_len, 64) / 8};
}

// Without timing: patterns keep their fixed tile; CSR rows take variable
// tiles, one lane per row unless rows are long (one lane per row measured
// fastest on polyhedral rows of 16.5 entries on average).
int tile_rule(const tf_matrix_s* m, const std::vector<int>& cands) {
  if (m->npat > 0) return cands.front();
  const double mean = m->nt > 0 ? (double)m->nnz / (double)m->nt : 0.0;
  const int want = mean > 48.0 ? kTileVar4 : mean > 24.0 ? kTileVar2 : kTileVar1;
  for (int c : cands)
    if (c == want) return c;
  return cands.front();
}

// Median microseconds of one q = A p launch with configuration cfg, timed
// with CUDA events on the context's stream (values and p are the zeroed
// registration buffers: the same memory traffic as real data).
int time_cfg(tf_matrix_s* m, int cfg, int npat, double* us) {
  m->tile_cfg = cfg;
  m->npat = cfg <= kTile128 ? npat : 0;
  int st = tf_fp64_prepare(m);
  if (st != TF_OK) return st;
  cudaEvent_t ev[kTuneReps + 1];
  for (auto& e : ev) TF_CUDA_TRY(cudaEventCreate(&e));
  for (int w = 0; w < 2 && st == TF_OK; ++w) st = tf_fp64_spmv(m, m->d_val, m->d_p, m->d_q, nullptr);
  for (int k = 0; k < kTuneReps && st == TF_OK; ++k) {
    cudaEventRecord(ev[k], m->ctx->stream);
    st = tf_fp64_spmv(m, m->d_val, m->d_p, m->d_q, nullptr);
  }
  cudaEventRecord(ev[kTuneReps], m->ctx->stream);
  cudaError_t e = cudaEventSynchronize(ev[kTuneReps]);
  std::vector<float> t(kTuneReps, 0.0f);
  for (int k = 0; k < kTuneReps && e == cudaSuccess; ++k)
    e = cudaEventElapsedTime(&t[k], ev[k], ev[k + 1]);
  for (auto& x : ev) cudaEventDestroy(x);
  if (st != TF_OK) return st;
  TF_CUDA_TRY(e);
  std::sort(t.begin(), t.end());
  *us = 1e3 * (double)t[kTuneReps / 2];
  return TF_OK;
}

}  // namespace

void tf_tune_cache_clear() {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_cache.clear();
}

int tf_choose_tiles(tf_matrix_s* m, unsigned fit_mask) {
  const int npat = m->npat;
  std::vector<int> cands;
  for (int c = 0; c <= kTile128; ++c)
    if (fit_mask & (1u << c)) cands.push_back(c);
  if (npat == 0 || cands.empty()) {
    if (m->ntiles > 0)
      for (int c : {kTileVar1, kTileVar2, kTileVar4, kTileVar8}) cands.push_back(c);
    cands.push_back(kTileNone);
  } else {
    cands.resize(1);   // row patterns: the widest fixed tile
  }
  m->tune.clear();
  int choice = -1;
  if (const char* f = getenv("TF_TILE_CFG")) {
    const int c = atoi(f);
    const bool ok = c == kTileNone || (c <= kTile128 && c >= 0 && (fit_mask & (1u << c))) ||
                    (c < kNumTileCfgs && tile_is_var(c) && m->ntiles > 0);
    if (ok) choice = c;
  }
  if (choice < 0 && cands.size() == 1) choice = cands[0];
  if (choice < 0 && (m->ni < kTuneMinRows || getenv("TF_NO_TUNE"))) choice = tile_rule(m, cands);
  const std::vector<long long> key = tune_key(m);
  if (choice < 0) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) choice = it->second;
  }
  if (choice < 0) {
    double best = 0.0;
    for (int c : cands) {
      double us = 0.0;
      const int st = time_cfg(m, c, npat, &us);
      if (st != TF_OK) return st;
      m->tune.emplace_back(c, us);
      if (choice < 0 || us < best) {
        best = us;
        choice = c;
      }
    }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = choice;
  }
  m->tile_cfg = choice;
  m->npat = choice <= kTile128 ? npat : 0;
  return tf_fp64_prepare(m);
}

int tf_fp64_prepare(tf_matrix_s* m) {
  const int n = std::max(m->nt, 1);
  int per_sm = 0;
  TF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, (const void*)k_update<kPrecJacobi, 1, 0>, 256, 0));
  per_sm = std::max(1, per_sm);
  m->vec_grid = std::max(1, std::min({(n + 511) / 512, m->ctx->sm_count * per_sm, kMaxBlocks}));
  if (const char* e = getenv("TF_VEC_DIR")) m->vec_dir = atoi(e) ? 1 : 0;
  if (m->tile_cfg == kTileNone) m->npat = 0;
  return dispatch_cfg(m->tile_cfg, m->npat > 0, [&](auto C, auto P) {
    return prepare_cfg<decltype(C)::value, decltype(P)::value>(m);
  });
}

namespace {
// Host-driven loop: the same kernels launched directly, the loop condition
// read back every kChunk iterations (kernels after convergence return at
// once).  Used when TF_NO_GRAPH is set.
template <int CFG, int PREC, int PAT>
int run_host_loop_t(tf_matrix_s* m, int xdef) {
  int st = set_attrs_cfg<CFG, PREC, PAT>();
  if (st != TF_OK) return st;
  cudaStream_t s = m->ctx->stream;
  VecArgs va = make_vec_args(m);
  SpArgs sa = make_sp_args(m, va);
  const int vg = m->vec_grid, sg = m->spmv_grid;
  const size_t ssm = cfg_smem<CFG, PAT>();
  const IterFns fns = iter_fns<PREC>(xdef, m->vec_dir);
  void* vargs[] = {&va};
  IccLevelArgs lv;
  IccSweeps sw{};
  const bool sweeps = PREC == kPrecIcc && m->icc_sweep_grid > 0;
  if (PREC == kPrecIcc) {
    lv = icc_level_args(m);
    sw = icc_sweep_args(m);
  }
  auto lgrid = [](int count) { return std::max(1, (count + 255) / 256); };
  auto coop = [&](const void* fn, IccSweepArgs* a) {
    void* args[] = {a};
    return cudaLaunchCooperativeKernel(fn, dim3(m->icc_sweep_grid), dim3(256), args, 0, s);
  };
  auto icc_apply = [&]() {
    if (sweeps) {
      coop((const void*)k_icc_sweep<kSweepFwd>, &sw.fwd);
      coop((const void*)k_icc_sweep<kSweepBwd>, &sw.bwd);
    } else {
      for (auto& a : lv.fwd) k_icc_fwd_level<<<lgrid(a.count), 256, 0, s>>>(a);
      for (auto& a : lv.bwd) k_icc_bwd_level<<<lgrid(a.count), 256, 0, s>>>(a);
    }
    k_icc_rho<<<vg, 256, 0, s>>>(m->ni, m->d_z, m->d_r, m->d_part, m->d_state);
  };
  k_diag<<<vg, 256, 0, s>>>(va);
  k_scale<<<vg, 256, 0, s>>>(va);
  if (PREC == kPrecIcc && sweeps)
    TF_CUDA_TRY(coop((const void*)k_icc_sweep<kSweepForm>, &sw.form));
  else if (PREC == kPrecIcc)
    for (auto& a : lv.form) k_icc_form_level<<<lgrid(a.count), 256, 0, s>>>(a);
  k_residual<CFG, PREC, PAT><<<sg, cfg_threads<CFG, PAT>(), ssm, s>>>(sa);
  if (PREC == kPrecIcc) icc_apply();
  TF_CUDA_TRY(cudaGetLastError());
  constexpr int kChunk = 16;
  for (;;) {
    TF_CUDA_TRY(cudaMemcpyAsync(m->h_state, m->d_state, sizeof(SolveState),
                                cudaMemcpyDeviceToHost, s));
    TF_CUDA_TRY(cudaStreamSynchronize(s));
    if (m->h_state->done) break;
    for (int k = 0; k < kChunk; ++k) {
      TF_CUDA_TRY(cudaLaunchKernel(fns.pupdate, dim3(vg), dim3(256), vargs, 0, s));
      k_spmv_alpha<CFG, PAT><<<sg, cfg_threads<CFG, PAT>(), ssm, s>>>(sa);
      TF_CUDA_TRY(cudaLaunchKernel(fns.update, dim3(vg), dim3(256), vargs, 0, s));
      if (PREC == kPrecIcc) icc_apply();
    }
    TF_CUDA_TRY(cudaGetLastError());
  }
  k_unscale<<<vg, 256, 0, s>>>(va);
  TF_CUDA_TRY(cudaGetLastError());
  return TF_OK;
}

template <int PREC>
int run_host_loop_p(tf_matrix_s* m, int xdef) {
  return dispatch_cfg(m->tile_cfg, m->npat > 0, [&](auto C, auto P) {
    return run_host_loop_t<decltype(C)::value, PREC, decltype(P)::value>(m, xdef);
  });
}
}  // namespace

int tf_fp64_run(tf_matrix_s* m, int prec) {
  if (prec < 0 || prec > 2) return TF_ERR_ARG;
  // x += alfa p can wait for the next k_pupdate when the NRMS does not
  // need the range of x (norm present); ICC keeps it in k_update.
  const int xdef = (prec != kPrecIcc && m->h_params->has_norm) ? 1 : 0;
  static const bool no_graph = getenv("TF_NO_GRAPH") != nullptr;
  if (no_graph) {
    if (prec == kPrecJacobi) return run_host_loop_p<kPrecJacobi>(m, xdef);
    if (prec == kPrecNone) return run_host_loop_p<kPrecNone>(m, xdef);
    return run_host_loop_p<kPrecIcc>(m, 0);
  }
  cudaGraphExec_t& g = (m->ext_bound ? m->ext_graph : m->graph)[2 * prec + xdef];
  if (!g) {
    int st;
    if (prec == kPrecJacobi) st = build_graph_p<kPrecJacobi>(m, xdef, &g);
    else if (prec == kPrecNone) st = build_graph_p<kPrecNone>(m, xdef, &g);
    else st = build_graph_p<kPrecIcc>(m, 0, &g);
    if (st != TF_OK) return st;
  }
  TF_CUDA_TRY(cudaGraphLaunch(g, m->ctx->stream));
  return TF_OK;
}

// ---- building blocks (direct launches, no solve state) --------------------
namespace {
template <int CFG, int PAT>
int launch_spmv(tf_matrix_s* m, const double* val, const double* p, double* q,
                double* scal) {
  VecArgs va = make_vec_args(m);
  va.st = nullptr;
  va.p = const_cast<double*>(p);
  va.q = q;
  SpArgs sa = make_sp_args(m, va);
  sa.val = val;
  sa.out_scalar = scal;
  k_spmv_alpha<CFG, PAT><<<m->spmv_grid, cfg_threads<CFG, PAT>(), cfg_smem<CFG, PAT>(),
                          m->ctx->stream>>>(sa);
  TF_CUDA_TRY(cudaGetLastError());
  return TF_OK;
}
template <int CFG, int PAT>
int launch_resid(tf_matrix_s* m, const double* val, const double* b,
                 const double* x, double* r, double* scal) {
  VecArgs va = make_vec_args(m);
  va.st = nullptr;
  va.x = const_cast<double*>(x);
  va.b = const_cast<double*>(b);
  va.r = r;
  SpArgs sa = make_sp_args(m, va);
  sa.val = val;
  sa.out_scalar = scal;
  k_residual<CFG, kPrecNone, PAT><<<m->spmv_grid, cfg_threads<CFG, PAT>(), cfg_smem<CFG, PAT>(),
                                   m->ctx->stream>>>(sa);
  TF_CUDA_TRY(cudaGetLastError());
  return TF_OK;
}
}  // namespace

// The building-block kernels need a scratch scalar pair: [0] result,
// [1] reinterpreted as the last-block counter.  d_part's tail holds it.
static double* bb_scalar(tf_matrix_s* m) { return m->d_part + 8 * kMaxBlocks; }

int tf_fp64_spmv(tf_matrix_s* m, const double* val, const double* p, double* q,
                 double* pq) {
  double* scal = bb_scalar(m);
  const int st = dispatch_cfg(m->tile_cfg, m->npat > 0, [&](auto C, auto P) {
    return launch_spmv<decltype(C)::value, decltype(P)::value>(m, val, p, q, scal);
  });
  if (st == TF_OK && pq)
    TF_CUDA_TRY(cudaMemcpyAsync(pq, scal, sizeof(double), cudaMemcpyDeviceToDevice,
                                m->ctx->stream));
  return st;
}

int tf_fp64_residual(tf_matrix_s* m, const double* val, const double* b,
                     const double* x, double* r) {
  double* scal = bb_scalar(m);
  return dispatch_cfg(m->tile_cfg, m->npat > 0, [&](auto C, auto P) {
    return launch_resid<decltype(C)::value, decltype(P)::value>(m, val, b, x, r, scal);
  });
}

namespace tf {
// NRMS of r with the diagonal of `val` (Normalized_Root_Mean_Square.f90).
__global__ void __launch_bounds__(256) k_nrms(int ni, const int* dia, const double* val,
                                              const double* r, const double* x,
                                              int has_norm, double norm,
                                              double* part, double* out) {
  __shared__ double scratch[32];
  double s = 0.0, mn = kHuge, mx = -kHuge;
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ni; i += stride) {
    s = __dadd_rn(s, nrms_term(r[i], val[dia[i]]));
    if (!has_norm) {
      mn = fmin_ref(mn, x[i]);
      mx = fmax_ref(mx, x[i]);
    }
  }
  double v[3] = {block_red<kSum>(s, scratch), block_red<kMin>(mn, scratch),
                 block_red<kMax>(mx, scratch)};
  const int ops[3] = {kSum, kMin, kMax};
  if (grid_reduce_last<3>(v, ops, part, reinterpret_cast<unsigned*>(out + 1), scratch) &&
      threadIdx.x == 0)
    out[0] = nrms_finish(v[0], has_norm, norm, v[1], v[2]);
}
}  // namespace tf

int tf_fp64_nrms(tf_matrix_s* m, const double* val, const double* r,
                 const double* x, int has_norm, double norm, double* out) {
  double* scal = bb_scalar(m);
  k_nrms<<<m->vec_grid, 256, 0, m->ctx->stream>>>(m->ni, m->d_dia, val, r, x, has_norm,
                                                  norm, m->d_part, scal);
  TF_CUDA_TRY(cudaGetLastError());
  TF_CUDA_TRY(cudaMemcpyAsync(out, scal, sizeof(double), cudaMemcpyDeviceToDevice,
                              m->ctx->stream));
  return TF_OK;
}

// ===========================================================================
// Multi-RHS solves: nrhs right-hand sides with one matrix (the three
// velocity components of Compute_Momentum.f90:153-399 when their matrices
// are equal).  Right-hand side 0 uses the matrix's own workspace, the others
// a slice each (tf_slice_s).  Every right-hand side runs its own Cg/Bicg
// recurrence with the single-RHS kernels -- same arithmetic, same
// reduction order, so each result is bit-identical to its own solve -- and
// one SpMV per iteration reads the matrix once for all of them.  The loop
// ends when every right-hand side is done (k_multi_cond).
// ===========================================================================
namespace tf {

struct MultiArgs {
  SpArgs sa;                   // the matrix (structure, values, patterns)
  int nr;
  const double* p[kMaxRhs];
  double* q[kMaxRhs];
  SolveState* st[kMaxRhs];
  double* part[kMaxRhs];
};

struct MultiCond {
  SolveState* st[kMaxRhs];
  int nr;
  cudaGraphConditionalHandle cond;
};

// q_r = A p_r for every active right-hand side r < NR; row sums in storage
// order, entries taken kMultiChunk at a time (the NR gathers of a group in
// flight together; small enough for two CTAs per SM).
constexpr int kMultiChunk = 2;
template <int NR>
struct OpSpmvMulti {
  static constexpr bool kRowOps = false;
  const double* p[NR];
  double* q[NR];
  double pq[NR];
  unsigned act;
  template <class VAL, class COL>
  __device__ __forceinline__ void body(int i, VAL v, COL col, int len) {
    double acc[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) acc[r] = 0.0;
#pragma unroll 1
    for (int k0 = 0; k0 < len; k0 += kMultiChunk) {
      double vv[kMultiChunk];
      int cc[kMultiChunk];
#pragma unroll
      for (int u = 0; u < kMultiChunk; ++u)
        if (k0 + u < len) {
          vv[u] = v(k0 + u);
          cc[u] = col(k0 + u);
        }
      double pv[NR][kMultiChunk];
#pragma unroll
      for (int r = 0; r < NR; ++r)
#pragma unroll
        for (int u = 0; u < kMultiChunk; ++u)
          if (((act >> r) & 1u) && k0 + u < len) pv[r][u] = __ldg(p[r] + cc[u]);
#pragma unroll
      for (int r = 0; r < NR; ++r)
#pragma unroll
        for (int u = 0; u < kMultiChunk; ++u)
          if (((act >> r) & 1u) && k0 + u < len)
            acc[r] = __dadd_rn(acc[r], __dmul_rn(vv[u], pv[r][u]));
    }
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      if (!((act >> r) & 1u)) continue;
      q[r][i] = acc[r];
      pq[r] = __dadd_rn(pq[r], __dmul_rn(__ldg(p[r] + i), acc[r]));
    }
  }
  __device__ __forceinline__ void operator()(int i, const double* v, const int* c, int len) {
    body(i, [v](int k) { return v[k]; }, [c](int k) { return c[k]; }, len);
  }
  __device__ __forceinline__ void pat(int i, const double* v, const int* o, int len) {
    body(i, [v](int k) { return v[k]; }, [i, o](int k) { return i + o[k]; }, len);
  }
};

// One SpMV for all active right-hand sides: on row-pattern tiles with the
// single-RHS kernel's tiles and grid (so each p.q is reduced exactly as in
// its own solve), otherwise one thread per row straight from global memory.
// Two CTAs per SM, as the single-RHS kernel.
template <int CFG, int PAT, int NR>
__global__ void __launch_bounds__(cfg_threads<CFG, PAT>(), 2) k_spmv_multi(MultiArgs a) {
  __shared__ double scratch[32];
  unsigned act = 0;
  for (int r = 0; r < NR; ++r)
    if (!a.st[r]->done) act |= 1u << r;
  if (!act) return;
  OpSpmvMulti<NR> op;
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    op.p[r] = a.p[r];
    op.q[r] = a.q[r];
    op.pq[r] = 0.0;
  }
  op.act = act;
  bool ok = true;
  if constexpr (CFG != kTileNone && PAT != 0) {
    ok = stream_tiles_pat<kTileRows[CFG], kTileNnzCap[CFG], kPatStages>(a.sa.row, a.sa.pt,
                                                                        a.sa.val, a.sa.nrows, op);
  } else {
    const int stride = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.sa.nrows; i += stride) {
      const int js = a.sa.row[i], je = a.sa.row[i + 1];
      op(i, a.sa.val + js, a.sa.col + js, je - js);
    }
  }
  if (!ok && threadIdx.x == 0)
    for (int r = 0; r < NR; ++r) flag_timeout(a.st[r]);
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    if (!((act >> r) & 1u)) continue;   // the same for every CTA
    double v[1] = {block_red<kSum>(op.pq[r], scratch)};
    const int ops[1] = {kSum};
    if (grid_reduce_last<1>(v, ops, a.part[r], &a.st[r]->counter[kCntSpmv], scratch) &&
        threadIdx.x == 0) {
      a.st[r]->pq = v[0];
      a.st[r]->alpha = __ddiv_rn(a.st[r]->rho, v[0]);
    }
  }
}

// The loop goes on while any right-hand side is not done.
__global__ void k_multi_cond(MultiCond c) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  unsigned any = 0;
  for (int r = 0; r < c.nr; ++r) any |= c.st[r]->done ? 0u : 1u;
  cudaGraphSetConditional(c.cond, any);
}

}  // namespace tf

namespace {

VecArgs slice_vec_args(tf_matrix_s* m, int i) {
  VecArgs a = make_vec_args(m);
  if (i > 0) {
    tf_slice_s* s = m->slices[i - 1];
    a.x = s->d_x;
    a.b = s->d_b;
    a.r = s->d_r;
    a.p = s->d_p;
    a.q = s->d_q;
    a.z = nullptr;
    a.adiag = s->d_adiag;
    a.part = s->d_part;
    a.st = s->d_state;
    a.nnz = 0;   // val is scaled and unscaled once, by right-hand side 0
  }
  return a;
}

template <int CFG, int PAT, int PREC>
int build_multi_graph_t(tf_matrix_s* m, int nr, int xdef, cudaGraphExec_t* out) {
  int st = set_attrs_cfg<CFG, PREC, PAT>();
  if (st != TF_OK) return st;
  const void* kmulti = nr == 1   ? (const void*)k_spmv_multi<CFG, PAT, 1>
                       : nr == 2 ? (const void*)k_spmv_multi<CFG, PAT, 2>
                       : nr == 3 ? (const void*)k_spmv_multi<CFG, PAT, 3>
                                 : (const void*)k_spmv_multi<CFG, PAT, 4>;
  if (cfg_smem<CFG, PAT>() > 48 * 1024 && PAT)
    TF_CUDA_TRY(cudaFuncSetAttribute(kmulti, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)cfg_smem<CFG, PAT>()));
  cudaGraph_t g = nullptr;
  TF_CUDA_TRY(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle h = 0;
  cudaError_t e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    TF_CUDA_TRY(e);
  }
  VecArgs va[kMaxRhs];
  SpArgs sa[kMaxRhs];
  MultiArgs ma{};
  MultiCond mc{};
  for (int i = 0; i < nr; ++i) {
    va[i] = slice_vec_args(m, i);
    sa[i] = make_sp_args(m, va[i]);
    ma.p[i] = va[i].p;
    ma.q[i] = va[i].q;
    ma.st[i] = va[i].st;
    ma.part[i] = va[i].part;
    mc.st[i] = va[i].st;
  }
  ma.sa = sa[0];
  ma.nr = nr;
  mc.nr = nr;
  mc.cond = h;
  const dim3 vb(256), vg(m->vec_grid);
  const dim3 sb(cfg_threads<CFG, PAT>()), sg(m->spmv_grid);
  const size_t ssm = cfg_smem<CFG, PAT>();
  const bool tiled_pat = CFG != kTileNone && PAT;
  const dim3 mb = tiled_pat ? sb : dim3(256), mg = tiled_pat ? sg : vg;
  const size_t msm = tiled_pat ? ssm : 0;
  const IterFns fns = iter_fns<PREC>(xdef, m->vec_dir);
  void* vargs[kMaxRhs][1];
  void* sargs[kMaxRhs][1];
  for (int i = 0; i < nr; ++i) {
    vargs[i][0] = &va[i];
    sargs[i][0] = &sa[i];
  }
  void* margs[] = {&ma};
  void* cargs[] = {&mc};
  NodeBuilder nb{g};
  cudaGraphNode_t prev = nullptr;
  for (int i = 0; i < nr; ++i) prev = nb.add((const void*)k_diag, vg, vb, 0, vargs[i], prev);
  for (int i = 0; i < nr; ++i) prev = nb.add((const void*)k_scale, vg, vb, 0, vargs[i], prev);
  for (int i = 0; i < nr; ++i)
    prev = nb.add((const void*)k_residual<CFG, PREC, PAT>, sg, sb, ssm, sargs[i], prev);
  prev = nb.add((const void*)k_multi_cond, dim3(1), dim3(32), 0, cargs, prev);
  cudaGraphNode_t cnode = nullptr;
  if (nb.status == TF_OK) {
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    e = cudaGraphAddNode(&cnode, g, &prev, 1, &cp);
    if (e != cudaSuccess) {
      tf_set_last_cuda_error(e, "cudaGraphAddNode(conditional)", __FILE__, __LINE__);
      nb.status = TF_ERR_CUDA;
    } else {
      NodeBuilder body{cp.conditional.phGraph_out[0]};
      cudaGraphNode_t b = nullptr;
      for (int i = 0; i < nr; ++i) b = body.add(fns.pupdate, vg, vb, 0, vargs[i], b);
      b = body.add(kmulti, mg, mb, msm, margs, b);
      for (int i = 0; i < nr; ++i) b = body.add(fns.update, vg, vb, 0, vargs[i], b);
      body.add((const void*)k_multi_cond, dim3(1), dim3(32), 0, cargs, b);
      if (body.status != TF_OK) nb.status = body.status;
    }
  }
  prev = cnode;
  for (int i = 0; i < nr; ++i) prev = nb.add((const void*)k_unscale, vg, vb, 0, vargs[i], prev);
  if (nb.status != TF_OK) {
    cudaGraphDestroy(g);
    return nb.status;
  }
  e = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  TF_CUDA_TRY(e);
  return TF_OK;
}

template <int PREC>
int build_multi_graph_p(tf_matrix_s* m, int nr, int xdef, cudaGraphExec_t* out) {
  return dispatch_cfg(m->tile_cfg, m->npat > 0, [&](auto C, auto P) {
    return build_multi_graph_t<decltype(C)::value, decltype(P)::value, PREC>(m, nr, xdef, out);
  });
}

int alloc_slice(tf_matrix_s* m, tf_slice_s** out) {
  auto* s = new tf_slice_s();
  const size_t nv = ((size_t)m->nt + 8) * sizeof(double);
  int st = TF_OK;
  for (double** p : {&s->d_x, &s->d_b, &s->d_r, &s->d_p, &s->d_q, &s->d_adiag})
    if (st == TF_OK) st = tf_dev_alloc_bytes(m->ctx, (void**)p, nv);
  if (st == TF_OK)
    st = tf_dev_alloc_bytes(m->ctx, (void**)&s->d_part,
                            ((size_t)8 * kMaxBlocks + 16) * sizeof(double));
  if (st == TF_OK) st = tf_dev_alloc_bytes(m->ctx, (void**)&s->d_state, sizeof(SolveState));
  *out = s;
  return st;
}

}  // namespace

void tf_slices_free(tf_matrix_s* m) {
  for (auto& s : m->slices) {
    if (!s) continue;
    for (void* p : {(void*)s->d_x, (void*)s->d_b, (void*)s->d_r, (void*)s->d_p, (void*)s->d_q,
                    (void*)s->d_adiag, (void*)s->d_part, (void*)s->d_state})
      if (p) {
        if (m->async_alloc) cudaFreeAsync(p, m->ctx->stream);
        else cudaFree(p);
      }
    delete s;
    s = nullptr;
  }
  for (auto& a : m->mgraph)
    for (auto& b : a)
      for (auto& g : b)
        if (g) {
          cudaGraphExecDestroy(g);
          g = nullptr;
        }
  if (m->h_mstate) {
    cudaFreeHost(m->h_mstate);
    m->h_mstate = nullptr;
  }
}

int tf_slices_ensure(tf_matrix_s* m, int nr) {
  if (nr < 1 || nr > kMaxRhs) return TF_ERR_ARG;
  for (int i = 0; i + 1 < nr; ++i)
    if (!m->slices[i]) {
      const int st = alloc_slice(m, &m->slices[i]);
      if (st != TF_OK) return st;
    }
  return TF_OK;
}

int tf_fp64_run_multi(tf_matrix_s* m, int prec, int nr) {
  if (nr < 1 || nr > kMaxRhs || (prec != kPrecJacobi && prec != kPrecNone)) return TF_ERR_ARG;
  const int st0 = tf_slices_ensure(m, nr);
  if (st0 != TF_OK) return st0;
  const int xdef = m->h_params->has_norm ? 1 : 0;
  cudaGraphExec_t& g = m->mgraph[nr][prec][xdef];
  if (!g) {
    const int st = prec == kPrecJacobi ? build_multi_graph_p<kPrecJacobi>(m, nr, xdef, &g)
                                       : build_multi_graph_p<kPrecNone>(m, nr, xdef, &g);
    if (st != TF_OK) return st;
  }
  TF_CUDA_TRY(cudaGraphLaunch(g, m->ctx->stream));
  return TF_OK;
}

// tf_tile.cuh -- row-tile streaming of a CSR matrix through shared memory.
//
// A tile is a run of consecutive rows.  Its row pointers, column indices
// (or row-pattern bytes) and values are contiguous in the device arrays, so
// one thread issues 1D bulk copies (cp.async.bulk, the TMA's linear mode)
// into a shared-memory stage and arms that stage's mbarrier with the byte
// count.  Stages form a ring: while tile k is computed from stage s, the
// copies of the next tiles are in flight.  Persistent CTAs walk tiles
// blockIdx.x, blockIdx.x + gridDim.x, ... so the tile -> CTA map (and hence
// every partial sum) is fixed for a fixed grid.
//
// Here: the work-list streamer of the batch engine (FP32-value path) and
// the row-pattern streamer with a producer warp; the CSR streamer with a
// producer warp is in tf_tile2.cuh.
//
// Each row is then handed to a per-row operator with pointers into the
// stage: one thread per row, entries visited in storage order, so a row sum
// is accumulated in exactly the order of the reference's loop
// `do j = a_row(i), a_row(i+1)-1` (Native_Mod/Cg.f90:180-183).
//
// Bulk copies need 16-byte aligned addresses and sizes.  Segment starts are
// rounded down and ends rounded up to 16 bytes; the device arrays carry
// enough padding that the rounded-up ends stay inside the allocation.
#pragma once
#include "tf_common.cuh"

namespace tf {

template <int ROWS, int NNZCAP, typename VT, int STAGES>
struct TileLayout {
  static constexpr int kEv = 16 / (int)sizeof(VT);  // values per 16 bytes
  static constexpr int kValCap = NNZCAP + 2 * kEv;
  static constexpr int kColCap = NNZCAP + 8;
  static constexpr int kRowCap = ROWS + 8;
  static constexpr size_t kValBytes = ((kValCap * sizeof(VT) + 127) / 128) * 128;
  static constexpr size_t kColBytes = ((kColCap * 4 + 127) / 128) * 128;
  static constexpr size_t kRowBytes = ((kRowCap * 4 + 127) / 128) * 128;
  static constexpr size_t kStageBytes = kValBytes + kColBytes + kRowBytes;
  static constexpr size_t kBarOffset = STAGES * kStageBytes;
  static constexpr size_t kMetaOffset = kBarOffset + 8 * STAGES;
  static constexpr size_t kSmemBytes = kMetaOffset + 32 * STAGES;
};

// ---------------------------------------------------------------------------
// Work-list streamer with descriptor prefetch.  Items carry their row range
// and entry range (r0, r1, j0, j1) so issuing a tile needs only the owning
// matrix's base pointers.  Thread 0 runs a two-deep prefetch ring: while
// item k is computed, the item that will refill its stage (k + STAGES*G)
// is already resolved (base pointers and skip flag loaded before the wait)
// and the following one (k + G + STAGES*G) is being fetched, so the bulk
// copies of a freed stage go out with no dependent global load on the
// critical path.
//   W::Item, W::count(), W::item(k) -> Item (has r0, r1, j0, j1)
//   W::resolve(const Item&, TileRes<VT>&)   base pointers + skip flag
//   W::row(k, i, vals, cols, len)            one thread per row
//   W::tile_end(k)                           all threads, after the rows
// ---------------------------------------------------------------------------
template <typename VT>
struct TileRes {
  const int* row;
  const int* col;
  const VT* val;
  int skip;
};

template <int ROWS, int NNZCAP, typename VT, int STAGES, class W>
__device__ bool stream_items(W& w) {
  using L = TileLayout<ROWS, NNZCAP, VT, STAGES>;
  using It = typename W::Item;
  constexpr int kEv = L::kEv;
  extern __shared__ __align__(128) unsigned char tf_smem[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(tf_smem + L::kBarOffset);
  int* meta = reinterpret_cast<int*>(tf_smem + L::kMetaOffset);
  auto sval = [&](int s) { return reinterpret_cast<VT*>(tf_smem + s * L::kStageBytes); };
  auto scol = [&](int s) {
    return reinterpret_cast<int*>(tf_smem + s * L::kStageBytes + L::kValBytes);
  };
  auto srow = [&](int s) {
    return reinterpret_cast<int*>(tf_smem + s * L::kStageBytes + L::kValBytes + L::kColBytes);
  };
  const int count = w.count();
  const int G = gridDim.x;
  if ((int)blockIdx.x >= count) return true;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int s = 0; s < STAGES; ++s) mbar_init(&bars[s], 1);
    mbar_fence_init();
  }
  __syncthreads();

  // Copies of a resolved item into stage s (thread 0).
  auto issue = [&](const It& it, const TileRes<VT>& rs, int s) {
    int* m = meta + 8 * s;
    if (rs.skip) {   // nothing to copy: complete the phase at once
      m[5] = 1;
      mbar_arrive_expect_tx(&bars[s], 0);
      return;
    }
    const int r0 = it.r0, r1 = it.r1, j0 = it.j0, j1 = it.j1;
    const int a0 = j0 & ~(kEv - 1), a1 = (j1 + kEv - 1) & ~(kEv - 1);
    const int c0 = j0 & ~3, c1 = (j1 + 3) & ~3;
    const int p0 = r0 & ~3, p1 = (r1 + 1 + 3) & ~3;
    m[0] = a0; m[1] = c0; m[2] = p0; m[3] = r0; m[4] = r1; m[5] = 0;
    const unsigned bv = (unsigned)(a1 - a0) * (unsigned)sizeof(VT);
    const unsigned bc = (unsigned)(c1 - c0) * 4u;
    const unsigned br = (unsigned)(p1 - p0) * 4u;
    mbar_arrive_expect_tx(&bars[s], bv + bc + br);
    if (bv) bulk_g2s(sval(s), rs.val + a0, bv, &bars[s]);
    if (bc) bulk_g2s(scol(s), rs.col + c0, bc, &bars[s]);
    bulk_g2s(srow(s), rs.row + p0, br, &bars[s]);
  };

  // At the iteration of item k: nxt = item k + STAGES*G (refills this
  // stage at the end of the iteration), nxt2 = item k + G + STAGES*G.
  It nxt{}, nxt2{};
  if (threadIdx.x == 0) {
#pragma unroll
    for (int s = 0; s < STAGES; ++s) {
      const int k = blockIdx.x + s * G;
      if (k < count) {
        const It it = w.item(k);
        TileRes<VT> rs;
        w.resolve(it, rs);
        issue(it, rs, s);
      }
    }
    const int k1 = blockIdx.x + STAGES * G;
    if (k1 < count) nxt = w.item(k1);
    if (k1 + G < count) nxt2 = w.item(k1 + G);
  }

  bool ok = true;
  int it_no = 0;
  for (int k = blockIdx.x; k < count; k += G, ++it_no) {
    const int s = it_no % STAGES;
    const unsigned par = (unsigned)(it_no / STAGES) & 1u;
    const int nk = k + STAGES * G;
    TileRes<VT> nres{};
    if (threadIdx.x == 0 && nk < count) w.resolve(nxt, nres);   // loads in flight
    const bool mine = mbar_wait_bounded(&bars[s], par);
    if (__syncthreads_or(!mine)) { ok = false; break; }
    const int* m = meta + 8 * s;
    if (!m[5]) {
      const int a0 = m[0], c0 = m[1], p0 = m[2], r0 = m[3], r1 = m[4];
      const VT* sv = sval(s);
      const int* sc = scol(s);
      const int* sr = srow(s);
      for (int r = r0 + (int)threadIdx.x; r < r1; r += ROWS) {
        const int js = sr[r - p0], je = sr[r + 1 - p0];
        w.row(k, r, sv + (js - a0), sc + (js - c0), je - js);
      }
      w.tile_end(k);
    }
    __syncthreads();   // stage s fully consumed
    if (threadIdx.x == 0 && nk < count) {
      fence_proxy_async_smem();
      issue(nxt, nres, s);
      nxt = nxt2;                        // item nk + G
      if (nk + 2 * G < count) nxt2 = w.item(nk + 2 * G);
    }
  }
  if (!ok && threadIdx.x == 0) {
    for (int d = 0; d < STAGES; ++d) {
      const int itk = it_no + d;
      const int k = blockIdx.x + itk * G;
      if (k >= count) break;
      mbar_drain(&bars[itk % STAGES], (unsigned)(itk / STAGES) & 1u);
    }
  }
  __syncthreads();
  return ok;
}

// ---------------------------------------------------------------------------
// Row-pattern variant.  On structured parts of a mesh most rows have the
// same column offsets relative to their own index (a hex cell's diagonal
// then its six neighbours at -nx*ny, -nx, -1, +1, +nx, +nx*ny), so the
// column array can be replaced by one byte per row naming the row's offset
// pattern, col_j = i + off[pattern(i)][j - row_i].  The values, the order
// of the entries and hence every row sum are those of the CSR arrays; only
// the column bytes (4 per entry) shrink to 1 per row.  A tile stage holds
// the values, the row pointers and the pattern bytes; the pattern table
// (at most kPatMax patterns of at most kPatMaxLen entries) sits in shared
// memory for the whole kernel.
// ---------------------------------------------------------------------------
constexpr int kPatMax = 64;
constexpr int kPatMaxLen = 16;
// Stages of the row-pattern ring.  Two: a third (2 x 109 KB of shared
// memory per SM) measured slower, the smaller L1 left for the x-gather
// costing more than the deeper copy pipeline gains.
constexpr int kPatStages = 2;

template <int ROWS, int NNZCAP, int STAGES>
struct PatLayout {
  static constexpr size_t kValBytes = (((NNZCAP + 4) * 8 + 127) / 128) * 128;
  static constexpr size_t kRowBytes = (((ROWS + 8) * 4 + 127) / 128) * 128;
  static constexpr size_t kPatBytes = ((ROWS + 32 + 127) / 128) * 128;
  static constexpr size_t kStageBytes = kValBytes + kRowBytes + kPatBytes;
  static constexpr size_t kTabOffset = STAGES * kStageBytes;
  static constexpr size_t kTabBytes = (size_t)kPatMax * (kPatMaxLen + 1) * 4;
  static constexpr size_t kBarOffset = kTabOffset + kTabBytes;      // full[S], empty[S]
  static constexpr size_t kMetaOffset = kBarOffset + 16 * STAGES;
  static constexpr size_t kSmemBytes = kMetaOffset + 32 * STAGES + 16;
};

// Pattern table in global memory: npat rows of kPatMaxLen offsets, then
// npat lengths.
struct PatTable {
  const unsigned char* pat;  // one byte per row
  const int* tab;            // [npat][kPatMaxLen] offsets, then [npat] lengths
  int npat;
};

// One row of a row-pattern tile for operators with per-row hooks
// (kRowOps: gather / row_init / combine / row_done): the row's gathers are
// issued eight at a time before their products are added, so a thread
// keeps a hex row's (at most 7) loads in flight together; the sum is the
// one-entry-at-a-time sum in storage order, bit for bit.  Eight slots, not
// kPatMaxLen: every slot costs its instructions even when predicated off,
// and on hex rows this loop is issue-bound.
template <class Op>
__device__ __forceinline__ void pat_row(Op& op, int i, const double* v, const int* off,
                                        int len) {
  double acc = op.row_init(i);
  for (int u0 = 0; u0 < len; u0 += 8) {
    double pr[8];
#pragma unroll
    for (int u = 0; u < 8; ++u)
      pr[u] = (u0 + u < len) ? __dmul_rn(v[u0 + u], op.gather(i + off[u0 + u])) : 0.0;
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (u0 + u < len) acc = op.combine(acc, pr[u]);
  }
  op.row_done(i, acc);
}

// Threads of a row-pattern CTA: ROWS consumer threads (one row each) and
// one producer warp.
template <int ROWS>
constexpr int pat_threads() { return ROWS + 32; }

// Warp-specialised streamer over row-pattern tiles.  The last warp is the
// producer: lane 0 issues the bulk copies of tile k into stage k % STAGES
// once every consumer warp has released that stage (empty[s], one arrival
// per consumer warp) and arms full[s] with the byte count.  Consumer warps
// wait on full[s], run op.pat(i, vals, offs, len) for their rows (thread t
// of the CTA takes row r0 + t; offs are the row pattern's offsets in
// shared memory, col = i + offs[k]) and release the stage -- no CTA-wide
// barrier per tile, so a warp whose rows are done moves on to the next
// staged tile while slower warps finish theirs.
//
// Every wait is bounded.  A consumer that times out raises a shared abort
// flag; the others stop at their next tile, the producer stops issuing, and
// before returning the producer waits (bounded) for the copies of every
// stage it armed.  Returns false on a timeout (the caller records it).
template <int ROWS, int NNZCAP, int STAGES, class Op>
__device__ bool stream_tiles_pat(const int* __restrict__ row, const PatTable& pt,
                                 const double* __restrict__ val, int nrows, Op& op,
                                 unsigned long long wait_ns = kWaitLimitNs) {
  using L = PatLayout<ROWS, NNZCAP, STAGES>;
  constexpr int kConsumerWarps = ROWS / 32;
  extern __shared__ __align__(128) unsigned char tf_smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(tf_smem + L::kBarOffset);
  uint64_t* empty = full + STAGES;
  int* meta = reinterpret_cast<int*>(tf_smem + L::kMetaOffset);
  volatile int* abort_flag = meta + 8 * STAGES;
  int* tab = reinterpret_cast<int*>(tf_smem + L::kTabOffset);
  auto sval = [&](int s) { return reinterpret_cast<double*>(tf_smem + s * L::kStageBytes); };
  auto srow = [&](int s) {
    return reinterpret_cast<int*>(tf_smem + s * L::kStageBytes + L::kValBytes);
  };
  auto spat = [&](int s) {
    return tf_smem + s * L::kStageBytes + L::kValBytes + L::kRowBytes;
  };

  const int ntiles = (nrows + ROWS - 1) / ROWS;
  if ((int)blockIdx.x >= ntiles) return true;
  const int ntab = pt.npat * (kPatMaxLen + 1);
  for (int k = threadIdx.x; k < ntab; k += blockDim.x) tab[k] = __ldg(pt.tab + k);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kConsumerWarps);
    }
    *abort_flag = 0;
    mbar_fence_init();
  }
  __syncthreads();
  const int* tab_len = tab + pt.npat * kPatMaxLen;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned long long deadline = deadline_after(wait_ns);
  bool ok = true;

  if (warp == kConsumerWarps) {
    // ---- producer warp ----
    if (lane == 0) {
      int issued = 0;
      for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++issued) {
        const int s = issued % STAGES;
        if (issued >= STAGES) {
          if (!mbar_wait_deadline(&empty[s], (unsigned)(issued / STAGES - 1) & 1u, deadline)) {
            ok = false;
            *abort_flag = 1;
            break;
          }
          fence_proxy_async_smem();   // consumers' reads before the async overwrite
        }
        if (*abort_flag) break;
        const int r0 = tile * ROWS;
        const int r1 = min(r0 + ROWS, nrows);
        const int j0 = __ldg(row + r0), j1 = __ldg(row + r1);
        const int a0 = j0 & ~1, a1 = (j1 + 1) & ~1;
        const int p0 = r0 & ~3, p1 = (r1 + 1 + 3) & ~3;
        const int b0 = r0 & ~15, b1 = (r1 + 15) & ~15;
        int* m = meta + 8 * s;
        m[0] = a0; m[1] = b0; m[2] = p0; m[3] = r0; m[4] = r1;
        const unsigned bv = (unsigned)(a1 - a0) * 8u;
        const unsigned br = (unsigned)(p1 - p0) * 4u;
        const unsigned bp = (unsigned)(b1 - b0);
        mbar_arrive_expect_tx(&full[s], bv + br + bp);
        if (bv) bulk_g2s(sval(s), val + a0, bv, &full[s]);
        bulk_g2s(srow(s), row + p0, br, &full[s]);
        bulk_g2s(spat(s), pt.pat + b0, bp, &full[s]);
      }
      // Drain: the copies of the last armed phase of every stage.
      for (int k = (issued > STAGES ? issued - STAGES : 0); k < issued; ++k)
        mbar_drain(&full[k % STAGES], (unsigned)(k / STAGES) & 1u);
    }
  } else {
    // ---- consumer warps ----
    int it = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
      const int s = it % STAGES;
      if (!mbar_wait_deadline(&full[s], (unsigned)(it / STAGES) & 1u, deadline)) {
        ok = false;
        *abort_flag = 1;
        break;
      }
      const int* m = meta + 8 * s;
      const int a0 = m[0], b0 = m[1], p0 = m[2], r0 = m[3], r1 = m[4];
      const int r = r0 + (int)threadIdx.x;
      if (r < r1) {
        const int js = srow(s)[r - p0];
        const int pid = spat(s)[r - b0];
        if constexpr (Op::kRowOps)
          pat_row(op, r, sval(s) + (js - a0), tab + pid * kPatMaxLen, tab_len[pid]);
        else
          op.pat(r, sval(s) + (js - a0), tab + pid * kPatMaxLen, tab_len[pid]);
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
      if (*abort_flag) { ok = false; break; }
    }
  }
  __syncthreads();
  return !__syncthreads_or(!ok);
}

// Tile configurations the host may pick.
//   0-2  fixed tiles of 512 / 256 / 128 rows (row patterns, or CSR with the
//        two-phase consumers of tf_tile2.cuh);
//   3    no tiles: one thread per row straight from global memory;
//   4-7  CSR tiles of variable length (at most 512 rows and 4096 entries,
//        boundaries listed at registration) with warp-group consumers of
//        G = 1, 2, 4, 8 lanes per row.
enum TileCfgId { kTile512 = 0, kTile256 = 1, kTile128 = 2, kTileNone = 3,
                 kTileVar1 = 4, kTileVar2 = 5, kTileVar4 = 6, kTileVar8 = 7 };
constexpr int kNumTileCfgs = 8;
constexpr int kTileRows[kNumTileCfgs] = {512, 256, 128, 512, 512, 512, 512, 512};
constexpr int kTileNnzCap[kNumTileCfgs] = {4096, 4096, 2048, 0, 4096, 4096, 4096, 4096};
__host__ __device__ constexpr bool tile_is_var(int c) { return c >= kTileVar1; }
__host__ __device__ constexpr int tile_var_g(int c) {
  return c == kTileVar1 ? 1 : c == kTileVar2 ? 2 : c == kTileVar4 ? 4 : 8;
}

}  // namespace tf

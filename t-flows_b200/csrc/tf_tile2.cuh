// tf_tile2.cuh -- two-phase CSR tile streamer with a producer warp.
//
// A tile holds at most kCons rows and NNZCAP entries.  Tiles of more than
// kCons/2 rows are summed one thread per row.  Shorter tiles (long rows:
// polyhedral cells have 10-18 entries, so a 4096-entry tile has ~270 rows)
// would leave half the threads idle, so they are consumed in two phases:
//
//   A  tpr = 2 or 4 threads per row: thread t forms the products
//      a_j * x(col_j) of every tpr-th entry of row r0 + (t mod kCons/tpr)
//      (a warp gathers for 32 consecutive rows, coalesced when neighbours
//      have nearby indices) and stores them over the staged values;
//   B  one thread per row sums the row's products in storage order,
//      starting from op.row_init (0 for A p, b_i for b - A x).
//
// Every product is rounded once (__dmul_rn) and the row's sum adds them one
// by one in the order of the entries (__dadd_rn / __dsub_rn), exactly the
// sequence of the reference's loop (Native_Mod/Cg.f90:180-183,
// Residual_Vector.f90:35-41), so results are bit-identical to one thread
// walking the row.
//
// Pipeline: the last warp is the producer; its lane 0 issues three 1D bulk
// copies (values, columns, row pointers) per tile into a ring of STAGES
// stages, arming full[s] with the byte count once every consumer warp has
// released the stage (empty[s]).  Consumers meet at a named barrier before
// each tile (to agree on stopping) and between the two phases (the
// products of a row come from other threads) -- the producer never waits
// there.  With Op::kReducer a third role, the reducer warp (after the
// producer), takes each tile's parked partials over two mbarriers (parked:
// every consumer warp has parked the tile; freed: the reducer is done with
// its slot), so no consumer waits for a tile's report.  All waits are
// bounded; on a timeout the CTA stops, the producer drains its armed copies
// and the streamer returns false.
//
// The tile source `S` provides (producer lane only):
//   int count()                    -- tiles (items) to walk
//   TileDesc desc(int k)           -- arrays and row/entry range of item k
// and the operator `Op` (consumer threads):
//   void begin(int k, TileAux aux) -- item k starts (aux: the descriptor's aux)
//   double gather(int c)           -- the vector entry multiplied by column c
//   double row_init(int i)         -- 0.0 or b_i
//   double combine(double acc, double prod)  -- acc + prod or acc - prod
//   void row_done(int i, double acc)
//   void tile_end(int it)          -- after the rows of the tile of consumer
//                                     iteration `it` (no barriers)
//   static constexpr bool kReducer -- true: a reducer warp (one more warp,
//                                     kCsr2RedThreads per CTA) takes over
//                                     the tile reductions:
//   void tile_id(int it, int skip, TileAux aux) -- consumer warp 0, lane 0,
//                                     before the tile's partials are parked
//   void reduce_tile(int it)       -- the reducer warp, once every consumer
//                                     warp has parked tile it (tile_end)
#pragma once
#include "tf_common.cuh"
#include "tf_tile.cuh"   // kPatMaxLen: the row-pattern table's row length

namespace tf {

constexpr int kCons = 512;               // consumer threads per CTA
constexpr int kCsr2Threads = kCons + 32;  // + the producer warp
constexpr int kCsr2RedThreads = kCsr2Threads + 32;   // + a reducer warp

struct TileDesc {
  const int* row;
  const int* col;
  const double* val;
  int r0, r1, j0, j1;
  int skip;
  const void* aux0;   // handed to op.begin through the stage (e.g. x, y vectors)
  void* aux1;
  int aux2, aux3;
  // Row-pattern tile (warp-group consumers of a source with kRowPatterns
  // only): the rows' pattern bytes and the pattern table ([npat][kPatMaxLen]
  // offsets, npat <= kPatMax) are staged instead of the columns,
  // col = i + tab[pat(i)][k].
  const unsigned char* pat = nullptr;
  const int* tab = nullptr;
  int npat = 0;
};

// What op.begin receives about its tile (copied by the producer into the
// stage's metadata, so consumers need no global loads to start a tile).
struct TileAux {
  const void* a0;
  void* a1;
  int i2, i3;
};

// The staged pattern table follows the pattern bytes of a stage's column
// region, at this byte offset (a multiple of 16).
template <int ROWCAP>
__host__ __device__ constexpr int pat_tab_offset() { return ((ROWCAP + 32 + 15) / 16) * 16; }

template <int ROWCAP, int NNZCAP, int STAGES>
struct Csr2Layout {
  static constexpr size_t kValBytes = (((NNZCAP + 4) * 8 + 127) / 128) * 128;
  static constexpr size_t kColBytes = (((NNZCAP + 8) * 4 + 127) / 128) * 128;
  static constexpr size_t kRowBytes = (((ROWCAP + 8) * 4 + 127) / 128) * 128;
  static constexpr size_t kStageBytes = kValBytes + kColBytes + kRowBytes;
  static constexpr size_t kBarOffset = STAGES * kStageBytes;   // full[S], empty[S]
  static constexpr size_t kMetaOffset = kBarOffset + 16 * STAGES;
  // 0-8 tile, 9-10 aux ints, 11 row patterns (their count), 12-15 aux pointers
  static constexpr int kMetaInts = 16;
  static_assert((size_t)pat_tab_offset<ROWCAP>() + kPatMax * kPatMaxLen * 4 <=
                    (size_t)(NNZCAP + 8) * 4,
                "a stage's column region holds the pattern bytes and table");
  // parked[2], freed[2]: the reducer warp's hand-over (after the abort flag)
  static constexpr size_t kRedBarOffset = kMetaOffset + 4 * kMetaInts * STAGES + 16;
  static constexpr size_t kSmemBytes = kRedBarOffset + 4 * 8;
};

// Named barrier 1 over the consumer threads only (the producer warp never
// joins it).
__device__ __forceinline__ void consumer_bar() {
  asm volatile("bar.sync 1, %0;" ::"r"(kCons) : "memory");
}
// The same barrier with an OR-reduction: every consumer gets the same
// answer, so all of them leave a loop at the same tile.
__device__ __forceinline__ bool consumer_bar_or(bool v) {
  unsigned r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, 1, %2, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"((unsigned)v), "r"(kCons)
      : "memory");
  return r != 0;
}

// Warp-group consumers (G = 1, 2, 4 or 8; G = 0 selects the two-phase
// consumers above).  Each warp takes 32/G rows of the staged tile at a
// time, G lanes per row: lane g of a row's group forms the products of
// the row's entries g, g+G, g+2G, ... of a chunk of CHUNK entries (CHUNK/G
// gathers in flight per lane), and the group's first lane adds the
// chunk's products in entry order, fetched by warp shuffles, before the
// next chunk.  The sum is
// the one-thread-per-row sum in storage order, bit for bit; no barrier
// joins the consumer warps, so each warp moves on as soon as its rows are
// done.  Rows of any length up to the tile's entry cap are handled.
// Columns of a staged CSR tile: entry q of the row starting at staged
// entry js.
struct CsrCols {
  const int* cc;
  __device__ __forceinline__ const int* row(int, int js) const { return cc + js; }
  __device__ __forceinline__ int col(const int* rc, int, int q) const { return rc[q]; }
};
// Columns of a staged row-pattern tile: row i's offsets from its pattern
// byte and the pattern table, both staged.
struct PatCols {
  const unsigned char* sp;   // pattern bytes, sp[i - b0]
  int b0;
  const int* tab;            // [npat][kPatMaxLen]
  __device__ __forceinline__ const int* row(int i, int) const {
    return tab + (int)sp[i - b0] * kPatMaxLen;
  }
  __device__ __forceinline__ int col(const int* rc, int i, int q) const { return i + rc[q]; }
};

template <int G, int CHUNK, class Op, class Cols>
__device__ __forceinline__ void wg_rows(Op& op, const double* prod, const Cols& cols,
                                        const int* sr, int p0, int r0, int r1, int j0,
                                        int warp, int lane, int nwarps) {
  constexpr int kRpw = 32 / G;   // rows per warp pass
  constexpr int kChunk = CHUNK;  // entries per chunk (see wg_chunk)
  constexpr int kU = kChunk / G;  // products per lane per chunk
  const int grp = lane / G, g = lane & (G - 1);
  const int gbase = lane & ~(G - 1);
  for (int rb = r0 + warp * kRpw; rb < r1; rb += nwarps * kRpw) {
    const int i = rb + grp;
    int js = 0, len = 0;
    const int* rc = nullptr;
    if (i < r1) {
      js = sr[i - p0] - j0;
      len = sr[i + 1 - p0] - j0 - js;
      rc = cols.row(i, js);
    }
    const int maxlen = __reduce_max_sync(0xffffffffu, len);
    double acc = (i < r1) ? op.row_init(i) : 0.0;
    for (int k0 = 0; k0 < maxlen; k0 += kChunk) {
      double pr[kU];
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const int q = k0 + u * G + g;
        pr[u] = (q < len) ? __dmul_rn(prod[js + q], op.gather(cols.col(rc, i, q))) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        if constexpr (G == 1) {
          if (k0 + u < len) acc = op.combine(acc, pr[u]);
        } else {
#pragma unroll
          for (int gg = 0; gg < G; ++gg) {
            const double v = __shfl_sync(0xffffffffu, pr[u], gbase + gg);
            if (k0 + u * G + gg < len) acc = op.combine(acc, v);
          }
        }
      }
    }
    if (g == 0 && i < r1) op.row_done(i, acc);
  }
}

// Whether a tile source may hand out row-pattern tiles (S::kRowPatterns);
// sources without the member never do, and their streamers carry no
// pattern code.
template <class S, class = void>
struct tile_patterns {
  static constexpr bool value = false;
};
template <class S>
struct tile_patterns<S, decltype((void)S::kRowPatterns)> {
  static constexpr bool value = S::kRowPatterns;
};

// Entries per chunk for one lane per row: every slot of a chunk costs its
// instructions even when predicated off, and on short rows (hex: 7
// entries) this path is issue-bound, so tiles of at most 8 entries per row
// on average take chunks of 8; longer rows keep 16 (their second chunk's
// gathers would otherwise wait for the first chunk's sum).
__device__ __forceinline__ bool wg_short_rows(int rows, int entries) {
  return entries <= 8 * rows;
}

// G = -1: the group width is picked per tile from its mean row length
// (the same for every warp of the CTA), for sources whose tiles mix short
// and long rows (the batch engine's systems).
__device__ __forceinline__ int tile_group_width(int rows, int entries) {
  // One lane per row measured fastest up to polyhedral rows (16.5 entries
  // on average, up to 49); groups pay off only for long rows.
  return entries > 48 * rows ? 4 : entries > 24 * rows ? 2 : 1;
}

template <int ROWCAP, int NNZCAP, int STAGES, int G = 0, class S, class Op>
__device__ bool stream_csr2(S& src, Op& op, unsigned long long wait_ns = kWaitLimitNs) {
  using L = Csr2Layout<ROWCAP, NNZCAP, STAGES>;
  constexpr int kConsWarps = kCons / 32;
  extern __shared__ __align__(128) unsigned char tf_smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(tf_smem + L::kBarOffset);
  uint64_t* empty = full + STAGES;
  // Reducer hand-over, by tile parity: parked (every consumer warp has
  // parked the tile's partials), freed (the reducer is done with them).
  uint64_t* parked = reinterpret_cast<uint64_t*>(tf_smem + L::kRedBarOffset);
  uint64_t* freed = parked + 2;
  constexpr bool kRed = Op::kReducer;
  constexpr bool kPat = G != 0 && tile_patterns<S>::value;
  int* meta = reinterpret_cast<int*>(tf_smem + L::kMetaOffset);
  volatile int* abort_flag = meta + L::kMetaInts * STAGES;
  auto sval = [&](int s) { return reinterpret_cast<double*>(tf_smem + s * L::kStageBytes); };
  auto scol = [&](int s) {
    return reinterpret_cast<int*>(tf_smem + s * L::kStageBytes + L::kValBytes);
  };
  auto srow = [&](int s) {
    return reinterpret_cast<int*>(tf_smem + s * L::kStageBytes + L::kValBytes + L::kColBytes);
  };

  const int count = src.count();
  if ((int)blockIdx.x >= count) return true;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kConsWarps);
    }
    if constexpr (kRed) {
      for (int s = 0; s < 2; ++s) {
        mbar_init(&parked[s], kConsWarps);
        mbar_init(&freed[s], 1);
      }
    }
    *abort_flag = 0;
    mbar_fence_init();
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned long long deadline = deadline_after(wait_ns);
  bool ok = true;

  if (warp == kConsWarps) {
    // ---- producer warp ----
    if (lane == 0) {
      int issued = 0;
      // The next tile's descriptor is loaded a round early, so its (possibly
      // dependent) global loads overlap the wait for a free stage.
      TileDesc nxt = src.desc(blockIdx.x);
      for (int k = blockIdx.x; k < count; k += gridDim.x, ++issued) {
        const int s = issued % STAGES;
        const TileDesc d = nxt;
        if (k + (int)gridDim.x < count) nxt = src.desc(k + gridDim.x);
        if (issued >= STAGES) {
          if (!mbar_wait_deadline(&empty[s], (unsigned)(issued / STAGES - 1) & 1u, deadline)) {
            ok = false;
            *abort_flag = 1;
            break;
          }
          fence_proxy_async_smem();
        }
        if (*abort_flag) break;
        int* m = meta + L::kMetaInts * s;
        m[7] = d.skip;
        m[8] = k;
        m[9] = d.aux2;
        m[10] = d.aux3;
        *reinterpret_cast<const void**>(m + 12) = d.aux0;
        *reinterpret_cast<void**>(m + 14) = d.aux1;
        if (d.skip) {
          mbar_arrive_expect_tx(&full[s], 0);
          continue;
        }
        const bool pat = kPat && d.pat != nullptr && d.npat > 0;
        const int a0 = d.j0 & ~1, a1 = (d.j1 + 1) & ~1;
        // the columns' (or the pattern bytes') first staged element
        const int c0 = pat ? (d.r0 & ~15) : (d.j0 & ~3);
        const int c1 = pat ? ((d.r1 + 15) & ~15) : ((d.j1 + 3) & ~3);
        const int p0 = d.r0 & ~3, p1 = (d.r1 + 1 + 3) & ~3;
        m[0] = a0; m[1] = c0; m[2] = p0; m[3] = d.r0; m[4] = d.r1; m[5] = d.j0; m[6] = d.j1;
        m[11] = pat ? d.npat : 0;
        const unsigned bv = (unsigned)(a1 - a0) * 8u;
        const unsigned bc = (unsigned)(c1 - c0) * (pat ? 1u : 4u);
        const unsigned br = (unsigned)(p1 - p0) * 4u;
        const unsigned bt = pat ? (unsigned)d.npat * kPatMaxLen * 4u : 0u;
        mbar_arrive_expect_tx(&full[s], bv + bc + br + bt);
        if (bv) bulk_g2s(sval(s), d.val + a0, bv, &full[s]);
        if (bc && pat) bulk_g2s(scol(s), d.pat + c0, bc, &full[s]);
        else if (bc) bulk_g2s(scol(s), d.col + c0, bc, &full[s]);
        if (bt)
          bulk_g2s(reinterpret_cast<unsigned char*>(scol(s)) + pat_tab_offset<ROWCAP>(), d.tab,
                   bt, &full[s]);
        bulk_g2s(srow(s), d.row + p0, br, &full[s]);
      }
      for (int k = (issued > STAGES ? issued - STAGES : 0); k < issued; ++k)
        mbar_drain(&full[k % STAGES], (unsigned)(k / STAGES) & 1u);
    }
  } else if (warp > kConsWarps) {
    // ---- reducer warp (Op::kReducer) ----
    if constexpr (kRed) {
      int it = 0;
      for (int k = blockIdx.x; k < count; k += gridDim.x, ++it) {
        if (!mbar_wait_or_abort(&parked[it & 1], (unsigned)(it >> 1) & 1u, abort_flag,
                                deadline)) {
          ok = false;
          *abort_flag = 1;
          break;
        }
        op.reduce_tile(it);
        __syncwarp();
        if (lane == 0) mbar_arrive(&freed[it & 1]);
      }
    }
  } else if constexpr (G != 0) {
    // ---- consumer warps, G lanes per row (wg_rows) ----
    int it = 0;
    for (int k = blockIdx.x; k < count; k += gridDim.x, ++it) {
      const int s = it % STAGES;
      bool stop = !mbar_wait_deadline(&full[s], (unsigned)(it / STAGES) & 1u, deadline);
      stop = __any_sync(0xffffffffu, stop || *abort_flag);   // warp-uniform
      if (stop) {
        ok = false;
        *abort_flag = 1;
        break;
      }
      const int* m = meta + L::kMetaInts * s;
      if (!m[7]) {
        const int a0 = m[0], c0 = m[1], p0 = m[2], r0 = m[3], r1 = m[4], j0 = m[5];
        const TileAux aux{*reinterpret_cast<const void* const*>(m + 12),
                          *reinterpret_cast<void* const*>(m + 14), m[9], m[10]};
        op.begin(k, aux);
        const double* prod = sval(s) + (j0 - a0);
        const bool short_rows = wg_short_rows(r1 - r0, m[6] - j0);
        auto one_lane = [&](const auto& cols) {
          if (short_rows)
            wg_rows<1, 8>(op, prod, cols, srow(s), p0, r0, r1, j0, warp, lane, kConsWarps);
          else
            wg_rows<1, 16>(op, prod, cols, srow(s), p0, r0, r1, j0, warp, lane, kConsWarps);
        };
        auto rows = [&](const auto& cols) {
          if constexpr (G == 1) {
            one_lane(cols);
          } else if constexpr (G > 0) {
            wg_rows<G, 16>(op, prod, cols, srow(s), p0, r0, r1, j0, warp, lane, kConsWarps);
          } else {
            switch (tile_group_width(r1 - r0, m[6] - j0)) {
              case 1: one_lane(cols); break;
              case 2:
                wg_rows<2, 16>(op, prod, cols, srow(s), p0, r0, r1, j0, warp, lane, kConsWarps);
                break;
              default:
                wg_rows<4, 16>(op, prod, cols, srow(s), p0, r0, r1, j0, warp, lane, kConsWarps);
            }
          }
        };
        bool done = false;
        if constexpr (kPat) {
          if (m[11]) {   // rows of at most kPatMaxLen entries: one lane per row
            const unsigned char* sp = reinterpret_cast<const unsigned char*>(scol(s));
            one_lane(PatCols{sp, c0,
                             reinterpret_cast<const int*>(sp + pat_tab_offset<ROWCAP>())});
            done = true;
          }
        }
        if (!done) rows(CsrCols{scol(s) + (j0 - c0)});
        if constexpr (!kRed) op.tile_end(it);
      }
      if constexpr (kRed) {
        const bool slot_free = __all_sync(
            0xffffffffu,
            it < 2 ||
                mbar_wait_or_abort(&freed[it & 1], (unsigned)((it >> 1) - 1) & 1u, abort_flag,
                                   deadline));
        if (!slot_free) {
          ok = false;
          *abort_flag = 1;
        }
        if (!m[7] && slot_free) op.tile_end(it);
        if (threadIdx.x == 0)
          op.tile_id(it, m[7], TileAux{*reinterpret_cast<const void* const*>(m + 12),
                                       *reinterpret_cast<void* const*>(m + 14), m[9], m[10]});
        __syncwarp();
        if (lane == 0) mbar_arrive(&parked[it & 1]);
      }
      __syncwarp();   // the stage is only read here: the producer's proxy fence suffices
      if (lane == 0) mbar_arrive(&empty[s]);
    }
  } else {
    // ---- consumer warps ----
    const int t = threadIdx.x;
    int it = 0;
    for (int k = blockIdx.x; k < count; k += gridDim.x, ++it) {
      const int s = it % STAGES;
      bool stop = !mbar_wait_deadline(&full[s], (unsigned)(it / STAGES) & 1u, deadline);
      stop = stop || *abort_flag;
      // Consumers must pass the named barrier equally often: they decide
      // together whether to stop here.
      if (consumer_bar_or(stop)) {
        ok = false;
        *abort_flag = 1;
        break;
      }
      const int* m = meta + L::kMetaInts * s;
      if (!m[7]) {
        const int a0 = m[0], c0 = m[1], p0 = m[2], r0 = m[3], r1 = m[4], j0 = m[5];
        double* prod = sval(s) + (j0 - a0);
        const int* cc = scol(s) + (j0 - c0);
        const TileAux aux{*reinterpret_cast<const void* const*>(m + 12),
                          *reinterpret_cast<void* const*>(m + 14), m[9], m[10]};
        op.begin(k, aux);
        const int* sr = srow(s);
        const int nr = r1 - r0;
        if (nr > kCons / 2) {
          // One thread per row: the row's gathers are in flight together
          // and its products are summed as they arrive.
          const int i = r0 + t;
          if (i < r1) {
            const int js = sr[i - p0] - j0, je = sr[i + 1 - p0] - j0;
            double acc = op.row_init(i);
            for (int q0 = js; q0 < je; q0 += 8) {
              double g[8];
#pragma unroll
              for (int u = 0; u < 8; ++u)
                if (q0 + u < je) g[u] = op.gather(cc[q0 + u]);
#pragma unroll
              for (int u = 0; u < 8; ++u)
                if (q0 + u < je) acc = op.combine(acc, __dmul_rn(prod[q0 + u], g[u]));
            }
            op.row_done(i, acc);
          }
        } else {
          // tpr = 2 or 4 threads per row: thread t takes row r0 + (t mod R)
          // and every tpr-th entry of it from slot t / R, so a warp's
          // gathers are those of 32 consecutive rows (coalesced for
          // structured column offsets).  Products go over the staged
          // values; then one thread per row sums them in storage order.
          const int lg = (nr > kCons / 4) ? 1 : 2;      // log2(tpr)
          const int tpr = 1 << lg, R = kCons >> lg;
          const int i = r0 + (t & (R - 1)), sl = t >> (__ffs(R) - 1);
          int js = 0, je = 0;
          if (i < r1) {
            js = sr[i - p0] - j0;
            je = sr[i + 1 - p0] - j0;
          }
          for (int q0 = js + sl; q0 < je; q0 += 8 * tpr) {
            double g[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
              const int q = q0 + u * tpr;
              if (q < je) g[u] = op.gather(cc[q]);
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
              const int q = q0 + u * tpr;
              if (q < je) prod[q] = __dmul_rn(prod[q], g[u]);
            }
          }
          consumer_bar();
          if (sl == 0 && i < r1) {
            double acc = op.row_init(i);
            for (int q = js; q < je; ++q) acc = op.combine(acc, prod[q]);
            op.row_done(i, acc);
          }
        }
        if constexpr (!kRed) op.tile_end(it);
      }
      if constexpr (kRed) {
        // Hand the tile to the reducer warp: its parity slot is free once
        // the reducer is done with tile it - 2.  A timeout or an abort here
        // stops the CTA at the next tile (every consumer still passes this
        // tile's barriers; the tile is not parked).
        // (Warp-uniform: tile_end shuffles across the warp.)
        const bool slot_free = __all_sync(
            0xffffffffu,
            it < 2 ||
                mbar_wait_or_abort(&freed[it & 1], (unsigned)((it >> 1) - 1) & 1u, abort_flag,
                                   deadline));
        if (!slot_free) {
          ok = false;
          *abort_flag = 1;
        }
        if (!m[7] && slot_free) op.tile_end(it);
        if (t == 0)
          op.tile_id(it, m[7], TileAux{*reinterpret_cast<const void* const*>(m + 12),
                                       *reinterpret_cast<void* const*>(m + 14), m[9], m[10]});
        __syncwarp();
        if (lane == 0) mbar_arrive(&parked[it & 1]);
      }
      fence_proxy_async_smem();   // product writes before the next bulk copy
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
    }
  }
  __syncthreads();
  return !__syncthreads_or(!ok);
}

}  // namespace tf

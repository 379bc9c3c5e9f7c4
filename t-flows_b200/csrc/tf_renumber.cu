// tf_renumber.cu -- cell renumbering for gather locality.
//
// T-Flows numbers cells by sorting their centres by coordinates
// (Grid_Mod/Sorting/Sort_Cells_By_Coordinates.f90, called by Generate and
// Convert).  On structured blocks that is a lattice order, but on an
// unstructured (e.g. polyhedral) mesh it leaves neighbouring cells far
// apart in index space, and the SpMV's x-gather -- 32 consecutive rows per
// warp -- touches ~26 different 128-byte lines per load instead of ~3.
//
// A matrix whose sampled gathers are that scattered gets a renumbered copy
// for the Jacobi / none solves: reverse Cuthill-McKee on the matrix graph,
// applied symmetrically (P A P^T).  Row i' = perm[i'] keeps its entries in
// the original storage order, only the column labels change, so every row
// sum is the original row's sum to the bit; the inputs are gathered into
// the new order on the device before the solve and scattered back after it.
// ICC keeps the original order (its factor depends on the ordering).
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "tf_internal.h"

// Mean number of distinct 128-byte lines (16 doubles) one warp-wide gather
// touches: slot k of 32 consecutive rows, every 37th warp sampled.  `base`
// is the index base of row/col (1 for Matrix_Type arrays).
double tf_gather_lines_per_warp(const int* row, const int* col, int n, int base) {
  long long lines = 0, loads = 0;
  int buf[32];
  for (int w0 = 0; w0 + 32 <= n; w0 += 32 * 37) {
    int maxlen = 0;
    for (int r = w0; r < w0 + 32; ++r) maxlen = std::max(maxlen, row[r + 1] - row[r]);
    for (int k = 0; k < maxlen; ++k) {
      int m = 0;
      for (int r = w0; r < w0 + 32; ++r)
        if (row[r + 1] - row[r] > k) buf[m++] = (col[row[r] - base + k] - base) >> 4;
      std::sort(buf, buf + m);
      lines += std::unique(buf, buf + m) - buf;
      ++loads;
    }
  }
  return loads ? (double)lines / (double)loads : 0.0;
}

namespace {

// Breadth-first levels from `s` over unvisited-in-this-pass nodes; returns
// the last node of the deepest level with the smallest degree.
int bfs_far(const std::vector<int>& row0, const std::vector<int>& col0, int s,
            std::vector<int>& stamp, int pass, std::vector<int>& queue, int& depth) {
  queue.clear();
  queue.push_back(s);
  stamp[s] = pass;
  size_t head = 0, level_start = 0;
  depth = 0;
  while (head < queue.size()) {
    const size_t level_end = queue.size();
    level_start = head;
    for (; head < level_end; ++head) {
      const int u = queue[head];
      for (int j = row0[u]; j < row0[u + 1]; ++j) {
        const int v = col0[j];
        if (stamp[v] != pass) {
          stamp[v] = pass;
          queue.push_back(v);
        }
      }
    }
    if (queue.size() > level_end) ++depth;
  }
  int best = queue[level_start];
  for (size_t q = level_start; q < queue.size(); ++q) {
    const int u = queue[q];
    if (row0[u + 1] - row0[u] < row0[best + 1] - row0[best]) best = u;
  }
  return best;
}

}  // namespace

// Reverse Cuthill-McKee order (new -> old) of the graph of a CSR pattern
// (0-based), component by component, each started from a pseudo-peripheral
// node (the lowest-degree node of the last level of a sweep from the
// component's first node); neighbours are visited in increasing degree,
// ties by index.
void tf_rcm_order(const std::vector<int>& row0, const std::vector<int>& col0, int n,
                  std::vector<int>& order) {
  order.clear();
  order.reserve(n);
  std::vector<int> stamp(n, -1), queue;
  std::vector<char> placed(n, 0);
  int pass = 0;
  for (int seed = 0; seed < n; ++seed) {
    if (placed[seed]) continue;
    int depth = 0;
    const int s = bfs_far(row0, col0, seed, stamp, pass++, queue, depth);
    const size_t begin = order.size();
    order.push_back(s);
    placed[s] = 1;
    for (size_t head = begin; head < order.size(); ++head) {
      const int u = order[head];
      const size_t first = order.size();
      for (int j = row0[u]; j < row0[u + 1]; ++j) {
        const int v = col0[j];
        if (!placed[v]) {
          placed[v] = 1;
          order.push_back(v);
        }
      }
      // insertion sort of the few new neighbours by (degree, index)
      for (size_t a = first + 1; a < order.size(); ++a) {
        const int v = order[a];
        const int dv = row0[v + 1] - row0[v];
        size_t b = a;
        while (b > first) {
          const int w = order[b - 1];
          const int dw = row0[w + 1] - row0[w];
          if (dw < dv || (dw == dv && w < v)) break;
          order[b] = w;
          --b;
        }
        order[b] = v;
      }
    }
  }
  std::reverse(order.begin(), order.end());
}

// ---------------------------------------------------------------------------
// Device permutations between a matrix and its renumbered copy
// ---------------------------------------------------------------------------
namespace tf {

__global__ void __launch_bounds__(256) k_perm_in(const double* __restrict__ val,
                                                 const double* __restrict__ x,
                                                 const double* __restrict__ b,
                                                 const int* __restrict__ src,
                                                 const int* __restrict__ perm, long long nnz,
                                                 int n, double* __restrict__ rv,
                                                 double* __restrict__ rx,
                                                 double* __restrict__ rb) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  for (long long j = t; j < nnz; j += stride) rv[j] = val[src[j]];
  for (long long i = t; i < n; i += stride) {
    const int o = perm[i];
    rx[i] = x[o];
    rb[i] = b[o];
  }
}

__global__ void __launch_bounds__(256) k_perm_out(const double* __restrict__ rv,
                                                  const double* __restrict__ rx,
                                                  const double* __restrict__ rb,
                                                  const int* __restrict__ src,
                                                  const int* __restrict__ perm, long long nnz,
                                                  int n, double* __restrict__ val,
                                                  double* __restrict__ x,
                                                  double* __restrict__ b) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  for (long long j = t; j < nnz; j += stride) val[src[j]] = rv[j];
  for (long long i = t; i < n; i += stride) {
    const int o = perm[i];
    x[o] = rx[i];
    b[o] = rb[i];
  }
}

}  // namespace tf

int tf_renumber_in(tf_matrix_s* m) {
  tf_matrix_s* r = m->ren;
  const int grid = std::max(1, std::min(m->ctx->sm_count * 8, (int)((m->nnz + 255) / 256)));
  tf::k_perm_in<<<grid, 256, 0, m->ctx->stream>>>(m->d_val, m->d_x, m->d_b, m->d_src, m->d_perm,
                                                  (long long)m->nnz, m->nt, r->d_val, r->d_x,
                                                  r->d_b);
  TF_CUDA_TRY(cudaGetLastError());
  return TF_OK;
}

int tf_renumber_out(tf_matrix_s* m) {
  tf_matrix_s* r = m->ren;
  const int grid = std::max(1, std::min(m->ctx->sm_count * 8, (int)((m->nnz + 255) / 256)));
  tf::k_perm_out<<<grid, 256, 0, m->ctx->stream>>>(r->d_val, r->d_x, r->d_b, m->d_src,
                                                   m->d_perm, (long long)m->nnz, m->nt,
                                                   m->d_val, m->d_x, m->d_b);
  TF_CUDA_TRY(cudaGetLastError());
  return TF_OK;
}

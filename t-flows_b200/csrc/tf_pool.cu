// tf_pool.cu -- a pool of CUDA streams that serves Solve_Native requests.
//
// Independent solves are overlapped rather than fused: each worker thread
// owns a context (one CUDA stream) and runs whole requests through the FP64
// drop-in (one graph launch per solve, convergence decided on the device).
// A request is exactly a Solve_Native call (Solve_Native.f90:33-44) on a
// system the caller hands over: the pool copies it, registers it on the
// worker's stream with stream-ordered allocation (cudaMallocAsync, so no
// registration or release ever synchronises the device or another worker),
// uploads the values, solves, writes x back and releases the memory.  The
// caller's arrays are used in place (no copy on submission), so they must
// stay valid until tf_pool_wait returns; conversion and upload run on the
// workers, in parallel.
//
// Admission: requests are taken in arrival order while the device bytes of
// the requests in flight plus the next one's stay within the memory budget;
// a request larger than the whole budget is rejected (TF_ERR_OOM).  Small
// systems, which a single stream leaves launch-latency bound, thus run many
// at a time, and a large one shares the GPU with whatever fits beside it.
//
// Resident structures: a Process solves the same Matrix_Type over and over
// (Create_Native.f90 builds it once; every outer iteration only refills
// val and b).  A registered matrix therefore stays on the device after its
// request, keyed by the caller's row/col/dia pointers, sizes and a sampled
// fingerprint of their contents; a later request with the same key, taken
// by the worker that holds it, skips validation, tiling, renumbering and
// the structure upload.  Held structures count toward the budget and are
// released, least recently used first, when a new request needs the room.
// A worker looks a few requests down the queue for one whose structure it
// holds before taking the head.
#include <cuda_runtime.h>
#include <string.h>

#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "tf_internal.h"

namespace {
using Clock = std::chrono::steady_clock;

struct PoolReq {
  int64_t id = 0;
  int solver = 0, prec = 1;
  int n = 0;
  int64_t nnz = 0;
  const int* row = nullptr;   // caller's arrays, valid until tf_pool_wait
  const int* col = nullptr;
  const int* dia = nullptr;
  const double* val = nullptr;
  const double* b = nullptr;
  double* x = nullptr;        // initial guess in, solution out
  int miter = 0;
  double tol = 0.0;
  int has_norm = 0;
  double norm = 0.0;
  size_t bytes = 0;
  uint64_t key = 0;           // structure key (pointers, sizes, sampled contents)
  Clock::time_point t_submit, t_start, t_done;
  int status = TF_OK;
  int niter = 0;
  double fin_res = 0.0;
  bool done = false;
};
// Sampled fingerprint of a Matrix_Type structure plus the caller's array
// addresses: equal keys mean "the same arrays, unchanged where sampled".
uint64_t structure_key(int n, int64_t nnz, const int* row, const int* col, const int* dia,
                       int icc) {
  uint64_t h = 1469598103934665603ull;
  auto mix = [&](uint64_t v) { h = (h ^ v) * 1099511628211ull; };
  mix((uint64_t)n);
  mix((uint64_t)nnz);
  mix((uint64_t)(uintptr_t)row);
  mix((uint64_t)(uintptr_t)col);
  mix((uint64_t)(uintptr_t)dia);
  mix((uint64_t)icc);
  for (int k = 0; k <= 64; ++k) mix((uint64_t)(uint32_t)row[(int64_t)n * k / 64]);
  for (int k = 0; k < 256; ++k) mix((uint64_t)(uint32_t)col[nnz * k / 256]);
  for (int k = 0; k < 64; ++k) mix((uint64_t)(uint32_t)dia[(int64_t)(n - 1) * k / 63]);
  return h;
}

constexpr int kLookahead = 16;   // queued requests a worker scans for its own structures
}  // namespace

struct tf_pool_s {
  int device = 0;
  size_t budget = 0, used = 0, peak = 0;
  std::vector<tf_ctx_s*> ctxs;
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<PoolReq>> queue;
  std::map<int64_t, std::shared_ptr<PoolReq>> live;
  int64_t next_id = 1;
  bool stop = false;
  long long submitted = 0, completed = 0, rejected = 0, reused = 0;

  // Resident structures (see the header comment).
  struct Held {
    uint64_t key = 0;
    tf_matrix_s* m = nullptr;
    int owner = 0;
    bool in_use = false;
    size_t bytes = 0;
    uint64_t last = 0;
  };
  std::vector<Held> held;
  uint64_t tick = 0;

  int find_held(uint64_t key, int w) const {
    for (size_t i = 0; i < held.size(); ++i)
      if (held[i].key == key && held[i].owner == w && !held[i].in_use) return (int)i;
    return -1;
  }
  // Release idle held structures, least recently used first, until `need`
  // more bytes fit in the budget.  Caller holds mu.
  bool make_room(size_t need) {
    while (used + need > budget) {
      int victim = -1;
      for (size_t i = 0; i < held.size(); ++i)
        if (!held[i].in_use && (victim < 0 || held[i].last < held[victim].last)) victim = (int)i;
      if (victim < 0) return false;
      tf_matrix_free(held[victim].m);   // stream-ordered on its owner's stream
      used -= held[victim].bytes;
      held.erase(held.begin() + victim);
    }
    return true;
  }
  // Pick worker w's next request: one whose structure it holds among the
  // first kLookahead, else the head if it fits.  Caller holds mu.
  std::shared_ptr<PoolReq> pick(int w, int* slot) {
    *slot = -1;
    const int look = std::min<int>((int)queue.size(), kLookahead);
    for (int q = 0; q < look; ++q) {
      const int h = find_held(queue[q]->key, w);
      if (h >= 0) {
        auto r = queue[q];
        queue.erase(queue.begin() + q);
        *slot = h;
        return r;
      }
    }
    if (queue.empty() || !make_room(queue.front()->bytes)) return nullptr;
    auto r = queue.front();
    queue.pop_front();
    return r;
  }

  // Run one request on worker w's context, on matrix m when it is held.
  int run(tf_ctx_s* ctx, PoolReq& r, tf_matrix_s** pm) {
    tf_matrix_s* m = *pm;
    int st = TF_OK;
    if (!m) {
      st = tf_matrix_create(ctx, r.n, r.n, r.nnz, r.row, r.col, r.dia, r.prec == tf::kPrecIcc,
                            &m);
      if (st != TF_OK) return st;
      *pm = m;
    }
    cudaStream_t s = ctx->stream;
    const size_t vb = (size_t)r.nnz * 8, nb = (size_t)r.n * 8;
    cudaError_t e = cudaMemcpyAsync(m->d_val, r.val, vb, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(m->d_x, r.x, nb, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(m->d_b, r.b, nb, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) {
      tf_set_last_cuda_error(e, "pool upload", __FILE__, __LINE__);
      st = TF_ERR_CUDA;
    }
    if (st == TF_OK)
      st = tf_solve_resident(m, r.prec, r.miter, r.tol, r.has_norm ? &r.norm : nullptr,
                             &r.niter, &r.fin_res);
    if (st == TF_OK) {
      e = cudaMemcpyAsync(r.x, m->d_x, nb, cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) {
        tf_set_last_cuda_error(e, "pool download", __FILE__, __LINE__);
        st = TF_ERR_CUDA;
      }
    }
    return st;
  }

  void loop(int w) {
    tf_ctx_s* ctx = ctxs[w];
    cudaSetDevice(device);
    for (;;) {
      std::shared_ptr<PoolReq> r;
      int h = -1;
      tf_matrix_s* m = nullptr;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] {
          if (stop) return true;
          r = pick(w, &h);
          return r != nullptr;
        });
        if (stop) return;
        if (h >= 0) {
          held[h].in_use = true;
          m = held[h].m;
          ++reused;
        } else {
          used += r->bytes;
          peak = std::max(peak, used);
        }
        r->t_start = Clock::now();
      }
      const int st = tf_guarded([&] { return run(ctx, *r, &m); });
      {
        std::lock_guard<std::mutex> lk(mu);
        if (h >= 0) {
          // the held entry may have moved in the vector: find it again
          for (auto& e : held)
            if (e.m == m) {
              e.in_use = false;
              e.last = ++tick;
            }
        } else if (m && st == TF_OK) {   // keep the structure resident
          Held e;
          e.key = r->key;
          e.m = m;
          e.owner = w;
          e.bytes = r->bytes;
          e.last = ++tick;
          held.push_back(e);
        } else {
          if (m) tf_matrix_free(m);
          used -= r->bytes;
        }
        r->status = st;
        r->t_done = Clock::now();
        r->done = true;
        ++completed;
        cv_done.notify_all();
        cv_work.notify_all();
      }
    }
  }
};

extern "C" int tf_pool_create(int device, int workers, size_t mem_budget, tf_pool* out) {
  TF_API_BEGIN
  if (!out || workers < 1 || workers > 256) return TF_ERR_ARG;
  *out = nullptr;
  auto* p = new tf_pool_s();
  p->budget = mem_budget ? mem_budget : ((size_t)20 << 30);
  for (int w = 0; w < workers; ++w) {
    tf_ctx c = nullptr;
    int st = tf_ctx_create(device, &c);
    if (st == TF_OK) {
      c->async_alloc = 1;
      cudaError_t e = cudaMallocHost((void**)&c->h_state, sizeof(tf::SolveState));
      if (e == cudaSuccess) e = cudaMallocHost((void**)&c->h_params, sizeof(tf::SolveParams));
      if (e != cudaSuccess) st = TF_ERR_OOM;
    }
    if (st != TF_OK) {
      if (c) tf_ctx_destroy(c);
      for (tf_ctx_s* x : p->ctxs) tf_ctx_destroy(x);
      delete p;
      return st;
    }
    p->ctxs.push_back(c);
  }
  p->device = p->ctxs[0]->device;
  // Keep freed stream-ordered memory in the device's pool for reuse.
  cudaMemPool_t mp;
  if (cudaDeviceGetDefaultMemPool(&mp, p->device) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(mp, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  for (int w = 0; w < workers; ++w) p->workers.emplace_back([p, w] { p->loop(w); });
  *out = p;
  return TF_OK;
  TF_API_END
}

extern "C" int tf_pool_submit(tf_pool p, int solver, int prec, int n, int64_t nnz,
                              const int* row, const int* col, const int* dia,
                              const double* val, const double* b, double* x,
                              int miter, double tol, const double* norm, int64_t* req) {
  TF_API_BEGIN
  if (!p || !req || n < 1 || nnz < n || !row || !col || !dia || !val || !b || !x)
    return TF_ERR_ARG;
  if (solver != TF_SOLVER_CG && solver != TF_SOLVER_BICG) return TF_ERR_UNKNOWN_SOLVER;
  if (prec < TF_PREC_NONE || prec > TF_PREC_ICC) return TF_ERR_UNKNOWN_PREC;
  auto r = std::make_shared<PoolReq>();
  r->solver = solver;
  r->prec = prec;
  r->n = n;
  r->nnz = nnz;
  r->row = row;
  r->col = col;
  r->dia = dia;
  r->val = val;
  r->b = b;
  r->x = x;
  r->miter = miter;
  r->tol = tol;
  r->has_norm = norm ? 1 : 0;
  r->norm = norm ? *norm : 0.0;
  r->bytes = tf_matrix_bytes_for(n, nnz, row, col) +
             (prec == TF_PREC_ICC ? (size_t)n * 40 + 4096 : 0);
  r->key = structure_key(n, nnz, row, col, dia, prec == TF_PREC_ICC);
  std::lock_guard<std::mutex> lk(p->mu);
  if (p->stop) return TF_ERR_CANCELLED;
  r->id = p->next_id++;
  r->t_submit = Clock::now();
  p->live[r->id] = r;
  ++p->submitted;
  if (r->bytes > p->budget) {      // can never be admitted
    r->status = TF_ERR_OOM;
    r->done = true;
    r->t_start = r->t_done = r->t_submit;
    ++p->rejected;
  } else {
    p->queue.push_back(r);
    p->cv_work.notify_all();
  }
  *req = r->id;
  return TF_OK;
  TF_API_END
}

extern "C" int tf_pool_wait(tf_pool p, int64_t req, int* niter, double* fin_res,
                            double* latency_ms, double* queue_ms) {
  TF_API_BEGIN
  if (!p) return TF_ERR_ARG;
  std::unique_lock<std::mutex> lk(p->mu);
  auto it = p->live.find(req);
  if (it == p->live.end()) return TF_ERR_ARG;
  auto r = it->second;
  p->cv_done.wait(lk, [&] { return r->done; });
  p->live.erase(it);
  using ms = std::chrono::duration<double, std::milli>;
  if (latency_ms) *latency_ms = ms(r->t_done - r->t_submit).count();
  if (queue_ms) *queue_ms = ms(r->t_start - r->t_submit).count();
  if (r->status != TF_OK) return r->status;
  if (niter) *niter = r->niter;
  if (fin_res) *fin_res = r->fin_res;
  return TF_OK;
  TF_API_END
}

extern "C" int tf_pool_cancel(tf_pool p, int64_t req) {
  TF_API_BEGIN
  if (!p) return TF_ERR_ARG;
  std::lock_guard<std::mutex> lk(p->mu);
  auto it = p->live.find(req);
  if (it == p->live.end()) return TF_ERR_ARG;
  auto r = it->second;
  if (r->done) return TF_ERR_BUSY;            // finished: its result stands
  for (auto q = p->queue.begin(); q != p->queue.end(); ++q)
    if (*q == r) {                            // not yet taken by a worker
      p->queue.erase(q);
      r->status = TF_ERR_CANCELLED;
      r->t_start = r->t_done = Clock::now();
      r->done = true;
      p->cv_done.notify_all();
      p->cv_work.notify_all();
      return TF_OK;
    }
  return TF_ERR_BUSY;                         // running: a solve runs to its end
  TF_API_END
}

extern "C" int tf_pool_stats(tf_pool p, long long* submitted, long long* completed,
                             long long* rejected, size_t* peak_bytes) {
  TF_API_BEGIN
  if (!p) return TF_ERR_ARG;
  std::lock_guard<std::mutex> lk(p->mu);
  if (submitted) *submitted = p->submitted;
  if (completed) *completed = p->completed;
  if (rejected) *rejected = p->rejected;
  if (peak_bytes) *peak_bytes = p->peak;
  return TF_OK;
  TF_API_END
}

extern "C" int tf_pool_resident(tf_pool p, long long* reused, int* held, size_t* held_bytes) {
  TF_API_BEGIN
  if (!p) return TF_ERR_ARG;
  std::lock_guard<std::mutex> lk(p->mu);
  if (reused) *reused = p->reused;
  if (held) *held = (int)p->held.size();
  if (held_bytes) {
    size_t b = 0;
    for (auto& e : p->held) b += e.bytes;
    *held_bytes = b;
  }
  return TF_OK;
  TF_API_END
}

extern "C" int tf_pool_destroy(tf_pool p) {
  TF_API_BEGIN
  if (!p) return TF_ERR_ARG;
  {
    std::lock_guard<std::mutex> lk(p->mu);
    p->stop = true;
    for (auto& kv : p->live)
      if (!kv.second->done) {
        kv.second->status = TF_ERR_CANCELLED;
        kv.second->done = true;
      }
    p->cv_work.notify_all();
    p->cv_done.notify_all();
  }
  for (auto& t : p->workers) t.join();
  for (auto& e : p->held) tf_matrix_free(e.m);
  p->held.clear();
  for (tf_ctx_s* c : p->ctxs) {
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    if (c->h_state) cudaFreeHost(c->h_state);
    if (c->h_params) cudaFreeHost(c->h_params);
    c->h_state = nullptr;
    c->h_params = nullptr;
    tf_ctx_destroy(c);
  }
  delete p;
  return TF_OK;
  TF_API_END
}

// server.cpp -- a serving loop for the AIFMM-LS direct solver on one GPU.
//
// The reference solves one problem with one right-hand side per process run
// (testFMM2D_find_error.cpp:41-176); it has no serving layer.  This one keeps
// factorisations resident on the device and answers two kinds of requests:
//   * factorize(key, desc): tables, tree, assembly and factorisation of a
//     geometry, kept under `key`;
//   * solve(key, b): right-hand sides against the kept factors of `key`.
// Scheduling:
//   * admission by device memory: a factorisation is started only when the
//     estimated footprint fits the budget next to the factors already held;
//     otherwise the least recently used idle factorisation is evicted (its
//     description is kept: a later solve on that key factors it again);
//   * continuous batching: a worker that takes a key's solves takes every
//     solve queued for that key at that moment (up to max_batch_rhs right-hand
//     sides) and runs them as one multi-RHS solve; requests that arrive while it
//     runs form the next batch.  Every column of a multi-RHS solve is computed
//     exactly as it would be alone (the kernels treat columns independently), so
//     a result does not depend on the batch it rode in;
//   * overlap: each worker drives its own handle and CUDA streams, so work on
//     different keys runs concurrently on the GPU; one key is used by one worker
//     at a time (a handle's calls must not overlap);
//   * form (aifmm_server_set_form): plain -- FP64 factors, direct solves -- or
//     mixed -- complex64 factors kept with the complex128 assembly, and every
//     solve refined by GMRES against the compressed product to a relative
//     residual.  A column's refined result does not depend on its batch beyond
//     that tolerance (the columns iterate in lockstep until the worst converges).
//     Complex64 factors serve trees up to depth 3, FP64 factors deeper ones
//     (measured: complex64 factors of a deeper tree do not precondition); when a
//     refinement stagnates all the same, the key is refactored in FP64 from its
//     kept assembly and the batch refined again.
// Failures (bad descriptions, a factorisation that cannot fit, CUDA errors) end
// the request with a status; the server keeps running.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/aifmm_b200.h"

namespace {

using clk = std::chrono::steady_clock;

struct Req {
  long id = 0;
  int kind = 0;  // 0 factorize, 1 solve
  long long key = 0;
  aifmm_desc desc{};
  int nrhs = 0;
  const double* b = nullptr;
  double* x = nullptr;
  clk::time_point t_submit, t_done;
  bool done = false;
  aifmm_status status = AIFMM_OK;
  std::string err;
  int batch_rhs = 0;  // right-hand sides of the batch this solve ran in
};

struct Factor {
  aifmm_desc desc{};
  aifmm_problem* p = nullptr;
  int precision = AIFMM_PRECISION_FP64;  // the precision of its factors
  bool refine = false;                   // mixed form: every solve refined to rtol
  double rtol = 0;
  bool ready = false;     // factors resident
  bool busy = false;      // a worker is using the handle
  bool queued_factor = false;  // a factorize request for it is waiting
  size_t bytes = 0;       // measured device footprint while resident
  size_t reserve = 0;     // admitted estimate while a factorisation runs
  uint64_t last_use = 0;
  std::deque<Req*> solves;
};

double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double pos = q * (v.size() - 1);
  const size_t i = (size_t)pos;
  const double f = pos - i;
  return i + 1 < v.size() ? v[i] * (1 - f) + v[i + 1] * f : v[i];
}

}  // namespace

struct aifmm_server {
  int device = 0;
  size_t budget = 0;
  int max_batch_rhs = 64;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::map<long long, Factor> factors;
  std::deque<Req*> factor_q;
  std::map<long, std::unique_ptr<Req>> reqs;
  std::vector<std::thread> workers;
  bool stopping = false;
  int factoring = 0;    // workers running a factorisation
  int factor_cap = -1;  // at most this many at once (< 0: all workers but one)
  int precision = AIFMM_PRECISION_FP64;  // the form of factorisations admitted from now on
  double rtol = 1e-8;
  long refine_iters = 0;                 // GMRES iterations over all refined batches
  long promotions = 0;                   // mixed-form keys refactored in FP64 (refinement stagnated)
  long next_id = 1;
  uint64_t tick = 0;
  // statistics
  std::vector<double> lat_solve, lat_factor;
  long evictions = 0, batches = 0, batch_rhs_total = 0, rejected = 0;

  // Device bytes a factorisation of this description may hold at its peak: the
  // 6x6-node depth-7 benchmark problem holds its blocks (the pool) plus the
  // assembly's chunked ACA buffers (at most a few GB), scaled by the points per
  // leaf.  Once factored, the measured footprint (the workspaces returned)
  // replaces the estimate.
  // The refined (mixed) form keeps the complex128 assembly next to the factors
  // and holds a second copy of the blocks while it factorises: about 1.7 times
  // the plain peak.
  static size_t estimate(const aifmm_desc& d, bool refine) {
    const double rank = (double)d.n_cheb * d.n_cheb;
    const double N = std::ldexp(1.0, 2 * d.depth) * rank;
    const double per = refine ? 1900.0 : 1100.0;
    return (size_t)(N * rank * per) + (size_t(64) << 20);
  }
  // complex64 factors precondition trees up to this depth (measured: at depth 4
  // the elimination's internal growth times FP32 rounding stalls the refinement)
  static constexpr int kC64MaxDepth = 3;
  size_t in_use() const {
    size_t s = 0;
    for (auto& kv : factors) s += kv.second.ready ? kv.second.bytes : kv.second.reserve;
    return s;
  }
  // evict least recently used idle factors until `need` more bytes fit; false if they cannot
  bool make_room(size_t need, long long except) {
    while (in_use() + need > budget) {
      Factor* lru = nullptr;
      long long lru_key = 0;
      for (auto& kv : factors) {
        Factor& f = kv.second;
        if (kv.first == except || !f.ready || f.busy || !f.solves.empty()) continue;
        if (!lru || f.last_use < lru->last_use) { lru = &f; lru_key = kv.first; }
      }
      if (!lru) return false;
      aifmm_problem_destroy(lru->p);
      lru->p = nullptr;
      lru->ready = false;
      lru->bytes = 0;
      ++evictions;
      (void)lru_key;
    }
    return true;
  }
  // internal requests (a factorisation again after an eviction) have negative ids
  // and no caller waiting for them
  void forget(Req* r) {
    if (r->id < 0) reqs.erase(r->id);
  }
  void finish(Req* r, aifmm_status st, const std::string& err) {
    r->status = st;
    r->err = err;
    r->t_done = clk::now();
    r->done = true;
    const double ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
    if (st == AIFMM_OK) (r->kind == 0 ? lat_factor : lat_solve).push_back(ms);
    else ++rejected;
  }

  // ---- the work a worker does outside the lock
  aifmm_status build(Factor& f, std::string& err, size_t& bytes) {
    aifmm_problem* p = nullptr;
    aifmm_status st = aifmm_problem_create(&f.desc, device, &p);
    if (st != AIFMM_OK) { err = aifmm_status_string(st); return st; }
    auto fail = [&](aifmm_status s) { err = aifmm_last_error(p); aifmm_problem_destroy(p); return s; };
    if ((st = aifmm_tables_compute(p, 1)) != AIFMM_OK) return fail(st);
    if ((st = aifmm_build_tree(p)) != AIFMM_OK) return fail(st);
    if ((st = aifmm_assemble(p)) != AIFMM_OK) return fail(st);
    if ((st = aifmm_autotune(p, nullptr, nullptr)) != AIFMM_OK) return fail(st);  // tile widths for this problem
    if ((st = aifmm_factorize(p, f.precision, f.refine ? AIFMM_KEEP_ASSEMBLY : 0)) != AIFMM_OK) return fail(st);
    // a refined key keeps the complex128 assembly its refinement multiplies with
    if ((st = f.refine ? aifmm_release_workspaces(p) : aifmm_trim(p)) != AIFMM_OK) return fail(st);
    double v[15] = {0};
    aifmm_stats(p, v, 15);
    bytes = (size_t)(v[13] + v[14]);
    f.p = p;
    return AIFMM_OK;
  }

  void worker(int dev) {
    cudaSetDevice(dev);
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
      Req* fr = nullptr;
      long long skey = 0;
      bool have_solve = false;
      // factorisations that fit now come first: they unblock queued solves.  One
      // that does not fit yet stays queued while solves on resident keys run
      // (their completion is what makes idle factors evictable).  With more than
      // one worker, by default one is always left for solves, which take
      // milliseconds where a factorisation takes seconds
      // (aifmm_server_set_factor_workers changes the share).
      const int cap = factor_cap > 0 ? factor_cap : std::max(1, (int)workers.size() - 1);
      const bool may_factor = factoring < cap;
      for (auto it = factor_q.begin(); may_factor && it != factor_q.end();) {
        Req* r = *it;
        Factor& f = factors[r->key];
        if (f.busy) { ++it; continue; }
        const size_t need = estimate(r->desc, precision == AIFMM_PRECISION_C64);
        if (need > budget) {  // can never fit
          it = factor_q.erase(it);
          f.queued_factor = false;
          finish(r, AIFMM_ERR_NOMEM, "factorisation larger than the server's device-memory budget");
          while (!f.solves.empty()) { finish(f.solves.front(), AIFMM_ERR_NOMEM, "factorisation not admitted"); f.solves.pop_front(); }
          forget(r);
          cv_done.notify_all();
          continue;
        }
        if (f.ready) {  // factored again: the new description replaces the old one
          aifmm_problem_destroy(f.p);
          f.p = nullptr;
          f.ready = false;
          f.bytes = 0;
        }
        if (!make_room(need, r->key)) { ++it; continue; }
        fr = r;
        factor_q.erase(it);
        break;
      }
      if (!fr) {  // the idle, resident key whose oldest queued solve is oldest
        clk::time_point best{};
        for (auto& kv : factors) {
          Factor& f = kv.second;
          if (f.busy || f.solves.empty() || f.queued_factor) continue;
          if (!have_solve || f.solves.front()->t_submit < best) {
            best = f.solves.front()->t_submit;
            skey = kv.first;
            have_solve = true;
          }
        }
      }
      if (!fr && !have_solve) {
        if (stopping) return;
        cv_work.wait(lk);
        continue;
      }
      if (fr) {
        Factor& f = factors[fr->key];
        f.desc = fr->desc;
        f.refine = precision == AIFMM_PRECISION_C64;
        f.precision = f.refine && f.desc.depth <= kC64MaxDepth ? AIFMM_PRECISION_C64 : AIFMM_PRECISION_FP64;
        f.rtol = rtol;
        const size_t need = estimate(f.desc, f.refine);
        f.busy = true;
        f.reserve = need;
        ++factoring;
        lk.unlock();
        std::string err;
        size_t bytes = 0;
        const aifmm_status st = build(f, err, bytes);
        lk.lock();
        --factoring;
        f.busy = false;
        f.reserve = 0;
        f.queued_factor = false;
        f.last_use = ++tick;
        if (st == AIFMM_OK) { f.ready = true; f.bytes = bytes; }
        finish(fr, st, err);
        if (st != AIFMM_OK)
          while (!f.solves.empty()) { finish(f.solves.front(), st, "factorisation failed: " + err); f.solves.pop_front(); }
        forget(fr);
        cv_done.notify_all();
        cv_work.notify_all();
        continue;
      }
      // ---- a batch of solves on one key
      Factor& f = factors[skey];
      if (!f.ready) {  // evicted: factor it again from the kept description
        Req* rf = new Req();
        rf->id = -(next_id++);
        rf->kind = 0;
        rf->key = skey;
        rf->desc = f.desc;
        rf->t_submit = clk::now();
        reqs[rf->id].reset(rf);
        f.queued_factor = true;
        factor_q.push_back(rf);
        continue;
      }
      std::vector<Req*> batch;
      int tot = 0;
      while (!f.solves.empty() && (batch.empty() || tot + f.solves.front()->nrhs <= max_batch_rhs)) {
        batch.push_back(f.solves.front());
        tot += f.solves.front()->nrhs;
        f.solves.pop_front();
      }
      f.busy = true;
      aifmm_problem* p = f.p;
      lk.unlock();
      int N = 0;
      aifmm_num_points(p, &N);
      // the batch is padded with zero columns to a power of two, so that each key
      // needs at most log2(max_batch_rhs) + 1 solve graphs; padding changes no
      // other column (every column is computed on its own)
      int width = 1;
      while (width < tot) width <<= 1;
      if (width > max_batch_rhs) width = tot;
      std::vector<double> B((size_t)2 * N * width, 0.0), X((size_t)2 * N * width);
      size_t o = 0;
      for (Req* r : batch) {
        std::memcpy(B.data() + o, r->b, sizeof(double) * 2 * (size_t)N * r->nrhs);
        o += (size_t)2 * N * r->nrhs;
      }
      int iters = 0;
      std::string err;
      const bool refine = f.refine;
      bool promoted = false;
      double relres = 0;
      aifmm_status st =
          refine ? aifmm_solve_refined(p, width, B.data(), N, X.data(), N, f.rtol, 90, &iters, &relres, AIFMM_PTR_HOST)
                 : aifmm_solve(p, width, B.data(), N, X.data(), N, nullptr, AIFMM_PTR_HOST | AIFMM_SOLVE_GRAPH);
      if (refine && st == AIFMM_ERR_NUMERIC && f.precision == AIFMM_PRECISION_C64) {
        // complex64 factors that do not precondition this problem (a deep tree's
        // growth times FP32 rounding): refactor from the kept complex128 assembly in
        // FP64 and refine again; the key keeps the FP64 factors.  The refactoring
        // is admitted like a factorisation (idle factors evicted to make room).
        bool room;
        {
          std::lock_guard<std::mutex> g(mu);
          room = make_room(estimate(f.desc, true), skey);
        }
        if (!room) {
          st = AIFMM_ERR_NOMEM;
          err = "no room to refactor in FP64 after the complex64 refinement stagnated";
        } else {
          st = aifmm_factorize(p, AIFMM_PRECISION_FP64, AIFMM_KEEP_ASSEMBLY);
          if (st == AIFMM_OK)
            st = aifmm_solve_refined(p, width, B.data(), N, X.data(), N, f.rtol, 90, &iters, &relres, AIFMM_PTR_HOST);
          promoted = true;
        }
      }
      if (refine && st == AIFMM_OK && !(relres <= f.rtol)) {  // the form promises rtol: say when it is not met
        st = AIFMM_ERR_NUMERIC;
        err = "refinement reached relative residual " + std::to_string(relres) + " in " + std::to_string(iters) +
              " iterations, above the form's target";
      }
      if (st != AIFMM_OK && err.empty()) err = aifmm_last_error(p);
      double v[15] = {0};
      aifmm_stats(p, v, 15);  // the graphs' buffers count towards the key's footprint
      o = 0;
      if (st == AIFMM_OK)
        for (Req* r : batch) {
          std::memcpy(r->x, X.data() + o, sizeof(double) * 2 * (size_t)N * r->nrhs);
          o += (size_t)2 * N * r->nrhs;
        }
      lk.lock();
      if (promoted) {
        f.precision = AIFMM_PRECISION_FP64;
        ++promotions;
      }
      f.busy = false;
      f.bytes = (size_t)(v[13] + v[14]);
      f.last_use = ++tick;
      ++batches;
      batch_rhs_total += tot;
      refine_iters += iters;
      for (Req* r : batch) { r->batch_rhs = tot; finish(r, st, err); }
      cv_done.notify_all();
      cv_work.notify_all();
    }
  }
};

extern "C" {

aifmm_status aifmm_server_create(int device, double hbm_budget_bytes, int workers, int max_batch_rhs,
                                 aifmm_server** out) {
  if (!out || workers < 1 || workers > 64 || max_batch_rhs < 1) return AIFMM_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return AIFMM_ERR_NODEVICE;
  if (device < 0 || device >= ndev) return AIFMM_ERR_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return AIFMM_ERR_CUDA;
  size_t fr = 0, tot = 0;
  if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return AIFMM_ERR_CUDA;
  auto* s = new aifmm_server();
  s->device = device;
  s->budget = hbm_budget_bytes > 0 ? (size_t)hbm_budget_bytes : (size_t)(0.8 * fr);
  s->max_batch_rhs = max_batch_rhs;
  for (int w = 0; w < workers; ++w) s->workers.emplace_back([s, device] { s->worker(device); });
  *out = s;
  return AIFMM_OK;
}

aifmm_status aifmm_server_destroy(aifmm_server* s) {
  if (!s) return AIFMM_ERR_ARG;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
  }
  s->cv_work.notify_all();
  for (auto& t : s->workers) t.join();
  // requests still queued never ran
  for (auto& kv : s->reqs)
    if (!kv.second->done) s->finish(kv.second.get(), AIFMM_ERR_STATE, "server stopped");
  for (auto& kv : s->factors)
    if (kv.second.p) aifmm_problem_destroy(kv.second.p);
  delete s;
  return AIFMM_OK;
}

aifmm_status aifmm_server_set_factor_workers(aifmm_server* s, int n) {
  if (!s || n < 1) return AIFMM_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  s->factor_cap = std::min(n, (int)s->workers.size());
  s->cv_work.notify_all();
  return AIFMM_OK;
}

aifmm_status aifmm_server_set_form(aifmm_server* s, int precision, double rtol) {
  if (!s || (precision != AIFMM_PRECISION_FP64 && precision != AIFMM_PRECISION_C64)) return AIFMM_ERR_ARG;
  if (precision == AIFMM_PRECISION_C64 && !(rtol > 0 && rtol < 1)) return AIFMM_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  s->precision = precision;
  s->rtol = rtol;
  return AIFMM_OK;
}

aifmm_status aifmm_server_factorize(aifmm_server* s, long long key, const aifmm_desc* desc, long* request) {
  if (!s || !desc || !request) return AIFMM_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stopping) return AIFMM_ERR_STATE;
  auto* r = new Req();
  r->id = s->next_id++;
  r->kind = 0;
  r->key = key;
  r->desc = *desc;
  r->t_submit = clk::now();
  s->reqs[r->id].reset(r);
  Factor& f = s->factors[key];
  if (!f.ready && !f.busy) f.desc = *desc;
  f.queued_factor = true;
  s->factor_q.push_back(r);
  *request = r->id;
  s->cv_work.notify_one();
  return AIFMM_OK;
}

aifmm_status aifmm_server_solve(aifmm_server* s, long long key, int nrhs, const double* b, double* x, long* request) {
  if (!s || !b || !x || !request || nrhs < 1) return AIFMM_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stopping) return AIFMM_ERR_STATE;
  auto it = s->factors.find(key);
  if (it == s->factors.end()) return AIFMM_ERR_STATE;  // never factored
  if (nrhs > s->max_batch_rhs) return AIFMM_ERR_ARG;
  auto* r = new Req();
  r->id = s->next_id++;
  r->kind = 1;
  r->key = key;
  r->nrhs = nrhs;
  r->b = b;
  r->x = x;
  r->t_submit = clk::now();
  s->reqs[r->id].reset(r);
  it->second.solves.push_back(r);
  *request = r->id;
  s->cv_work.notify_one();
  return AIFMM_OK;
}

aifmm_status aifmm_server_wait(aifmm_server* s, long request, double timeout_s, aifmm_status* result,
                               double* latency_ms, int* batch_rhs) {
  if (!s) return AIFMM_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(request);
  if (it == s->reqs.end()) return AIFMM_ERR_ARG;
  Req* r = it->second.get();
  const auto until = clk::now() + std::chrono::duration_cast<clk::duration>(std::chrono::duration<double>(timeout_s));
  while (!r->done)
    if (s->cv_done.wait_until(lk, until) == std::cv_status::timeout && !r->done) return AIFMM_ERR_STATE;
  if (result) *result = r->status;
  if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
  if (batch_rhs) *batch_rhs = r->batch_rhs;
  s->reqs.erase(it);
  return AIFMM_OK;
}

aifmm_status aifmm_server_stats(aifmm_server* s, double* out, int n) {
  if (!s || !out) return AIFMM_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  int resident = 0;
  for (auto& kv : s->factors) resident += kv.second.ready ? 1 : 0;
  const double v[14] = {percentile(s->lat_solve, 0.5), percentile(s->lat_solve, 0.99),
                        percentile(s->lat_factor, 0.5), percentile(s->lat_factor, 0.99),
                        (double)s->lat_solve.size(), (double)s->lat_factor.size(), (double)s->evictions,
                        (double)s->batches, s->batches ? (double)s->batch_rhs_total / s->batches : 0.0,
                        (double)s->in_use(), (double)resident, (double)s->rejected,
                        s->batches ? (double)s->refine_iters / s->batches : 0.0, (double)s->promotions};
  for (int i = 0; i < n && i < 14; ++i) out[i] = v[i];
  return AIFMM_OK;
}

}  // extern "C"

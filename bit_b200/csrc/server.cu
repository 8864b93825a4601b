// Serving: a request loop with continuous batching over one GPU.
//
// Callers submit evaluate requests (potential at every particle of a system) and solve
// requests (the treecode GMRES) of any size at any time.  The server keeps a FIFO of
// pending requests and `slots` worker threads, each owning a context (its own CUDA stream
// and device memory).  A request starts as soon as a slot is free and its reservation fits
// in the HBM budget next to everything else the server's contexts hold: the reservations
// of the running requests and the bytes the idle slots keep (live buffers and cached
// blocks).  A running request's context may allocate at most its reservation (the larger
// of its estimate and what its slot already holds), so the device memory of all slots
// together never exceeds the budget: a request whose estimate proves too small fails with
// BIT_ERR_BUDGET instead of overrunning it.  The head of the queue is never overtaken, so
// no request starves.  Requests in different slots run on
// different streams, so their kernels overlap on the device; a request's tree, moments,
// interaction lists and Krylov basis stay resident in its slot until it finishes.  Every
// request records when it was submitted, started and finished (seconds on the server's
// clock), which is what p50/p99 latencies are computed from.
//
// Results do not depend on what else runs: each request uses only its own context and the
// kernels are deterministic, so a result is bit-identical alone and in the mix.
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "common.cuh"

namespace bit {
namespace {

struct Request {
  long long id = 0;
  int kind = 0;  // 0 evaluate, 1 solve
  int n = 0, nterms = 0, maxmemb = 0;
  std::vector<double> x, y, z, q, f;  // q: charges (evaluate) or weights (solve)
  bit_eval_params p{};
  double diag = 0.0;
  bit_gmres_opts g{};
  size_t est = 0;
  size_t reservation = 0;  // bytes its slot's context may hold while it runs
  std::vector<double> out;
  bit_request_info info{};
  bool done = false;
};

using Clock = std::chrono::steady_clock;

// Device memory a request may need: particles in tree order (coordinates, sources in FP64
// and FP32, permutations), build scratch, interaction lists, moments, outputs, the mixed
// near field's close-pair records (28 B per target); a solve adds its Krylov basis and
// work vectors.  Measured peaks stay below these figures.
size_t estimate_bytes(int kind, int n, int restart) {
  size_t per = 448;
  if (kind == 1) per += 8ull * (restart + 10);
  return (64ull << 20) + per * (size_t)n;
}

}  // namespace
}  // namespace bit

struct bit_server {
  int device = 0;
  int nslots = 0;
  size_t budget = 0, reserved = 0, max_reserved = 0;
  int running = 0, max_running = 0;
  long long next_id = 1, submitted = 0, completed = 0;
  std::vector<bit_ctx*> ctx;
  // device bytes each idle slot's context holds (live + cached), the cached part, and the
  // sum over idle slots; squeeze: idle slots are asked to free their cached blocks
  std::vector<size_t> held, cached;
  std::vector<char> busy;  // the slot runs a request (its held / cached are not current)
  size_t idle_held = 0;
  bool squeeze = false;
  std::deque<std::shared_ptr<bit::Request>> queue;
  std::map<long long, std::shared_ptr<bit::Request>> reqs;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::vector<std::thread> workers;
  bool stopping = false;
  bit::Clock::time_point t0;
  std::string last_error;

  double now() const {
    return std::chrono::duration<double>(bit::Clock::now() - t0).count();
  }

  void run(int slot, bit::Request& r) {
    bit_ctx* c = ctx[slot];
    bit_tree* t = nullptr;
    bit_status st = bit_tree_build(c, r.n, r.x.data(), r.y.data(), r.z.data(), r.maxmemb, &t);
    r.out.assign(r.n, 0.0);
    if (st == BIT_OK && r.kind == 0) {
      st = bit_tree_set_charges(t, r.q.data(), nullptr);
      if (st == BIT_OK) st = bit_tree_moments(t, r.nterms);
      if (st == BIT_OK) st = bit_eval_particles(t, &r.p, r.out.data());
    } else if (st == BIT_OK) {
      st = bit_bie_solve(t, &r.p, r.nterms, r.diag, r.q.data(), r.f.data(), r.out.data(), &r.g,
                         &r.info.gmres);
    }
    if (t) bit_tree_destroy(t);
    size_t in_use = 0, peak = 0;
    bit_ctx_memory(c, &in_use, &peak);
    r.info.peak_bytes = peak;
    r.info.status = st;
  }

  // The head request fits when this slot takes it: everything else held, plus the larger of
  // its estimate and what this slot already holds (its cached blocks are reused).
  bool fits(int slot) const {
    return reserved + idle_held - held[slot] + std::max(queue.front()->est, held[slot]) <= budget;
  }
  // It would fit if the idle slots gave back their cached blocks.
  bool fits_after_squeeze() const {
    size_t live = 0;
    for (size_t i = 0; i < held.size(); i++)
      if (!busy[i]) live += held[i] - cached[i];
    return reserved + live + queue.front()->est <= budget;
  }

  void worker(int slot) {
    for (;;) {
      std::shared_ptr<bit::Request> r;
      {
        std::unique_lock<std::mutex> lock(mu);
        // the head of the queue starts when it fits next to everything else held; if it
        // would fit only after the idle slots free their cached blocks, they free them
        cv_work.wait(lock, [&] {
          if (stopping && queue.empty()) return true;
          if (queue.empty()) return false;
          if (fits(slot)) return true;
          if (!squeeze && fits_after_squeeze()) {
            squeeze = true;
            cv_work.notify_all();
          }
          return squeeze && cached[slot] > 0;
        });
        if (queue.empty()) return;
        if (!fits(slot)) {
          // give this idle slot's cached blocks back, then look again
          lock.unlock();
          ctx_trim(&ctx[slot]->c, 0);
          const size_t h = ctx[slot]->c.in_use + ctx[slot]->c.cached;
          lock.lock();
          idle_held = idle_held - held[slot] + h;
          held[slot] = h;
          cached[slot] = ctx[slot]->c.cached;
          cv_work.notify_all();
          continue;
        }
        squeeze = false;
        busy[slot] = 1;
        r = queue.front();
        queue.pop_front();
        r->reservation = std::max(r->est, held[slot]);
        r->info.bytes_reserved = r->reservation;
        idle_held -= held[slot];
        reserved += r->reservation;
        running++;
        max_reserved = std::max(max_reserved, reserved + idle_held);
        max_running = std::max(max_running, running);
        r->info.t_start = now();
        r->info.slot = slot;
      }
      ctx[slot]->c.peak = ctx[slot]->c.in_use;
      ctx[slot]->c.budget = r->reservation;  // the context may not allocate beyond it
      run(slot, *r);
      // give back cached blocks above this slot's share of the budget
      ctx_trim(&ctx[slot]->c, budget / nslots);
      const size_t h = ctx[slot]->c.in_use + ctx[slot]->c.cached;
      {
        std::lock_guard<std::mutex> lock(mu);
        r->info.t_done = now();
        r->done = true;
        reserved -= r->reservation;
        held[slot] = h;
        cached[slot] = ctx[slot]->c.cached;
        busy[slot] = 0;
        idle_held += h;
        running--;
        completed++;
      }
      cv_work.notify_all();
      cv_done.notify_all();
    }
  }
};

using namespace bit;

extern "C" {

bit_status bit_server_create(bit_server** out, const bit_server_opts* o) {
  if (!out) return BIT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  const int slots = o ? o->slots : 4;
  if (slots < 1 || slots > 64) return BIT_ERR_INVALID_ARGUMENT;
  auto* s = new (std::nothrow) bit_server;
  if (!s) return BIT_ERR_OUT_OF_MEMORY;
  s->device = o ? o->device : 0;
  s->nslots = slots;
  s->t0 = Clock::now();
  size_t budget = o ? o->hbm_budget : 0;
  if (budget == 0) {
    size_t fr = 0, tot = 0;
    if (cudaSetDevice(s->device) != cudaSuccess || cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
      cudaGetLastError();
      delete s;
      return BIT_ERR_NO_DEVICE;
    }
    budget = fr / 10 * 9;
  }
  s->budget = budget;
  for (int i = 0; i < slots; i++) {
    bit_ctx_opts co{s->device, nullptr, 0};
    bit_ctx* c = nullptr;
    bit_status st = bit_ctx_create(&c, &co);
    if (st != BIT_OK) {
      for (bit_ctx* d : s->ctx) bit_ctx_destroy(d);
      delete s;
      return st;
    }
    s->ctx.push_back(c);
    const size_t h = c->c.in_use + c->c.cached;
    s->held.push_back(h);
    s->cached.push_back(c->c.cached);
    s->busy.push_back(0);
    s->idle_held += h;
  }
  for (int i = 0; i < slots; i++) s->workers.emplace_back(&bit_server::worker, s, i);
  *out = s;
  return BIT_OK;
}

bit_status bit_server_destroy(bit_server* s) {
  if (!s) return BIT_ERR_INVALID_ARGUMENT;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->stopping = true;
  }
  s->cv_work.notify_all();
  for (auto& w : s->workers) w.join();
  for (bit_ctx* c : s->ctx) bit_ctx_destroy(c);
  delete s;
  return BIT_OK;
}

static bit_status submit(bit_server* s, std::shared_ptr<Request> r, long long* id) {
  r->est = estimate_bytes(r->kind, r->n, r->kind == 1 ? r->g.restart : 0);
  std::lock_guard<std::mutex> lock(s->mu);
  if (r->est > s->budget) {
    s->last_error = "request needs about " + std::to_string(r->est) +
                    " bytes, more than the whole HBM budget";
    return BIT_ERR_BUDGET;
  }
  r->id = s->next_id++;
  r->info.t_submit = s->now();
  r->info.bytes_reserved = r->est;
  s->reqs[r->id] = r;
  s->queue.push_back(r);
  s->submitted++;
  *id = r->id;
  s->cv_work.notify_all();
  return BIT_OK;
}

bit_status bit_server_submit_eval(bit_server* s, int n, const double* x, const double* y,
                                  const double* z, const double* q, int nterms, int maxmemb,
                                  const bit_eval_params* p, long long* id) {
  if (!s || !x || !y || !z || !q || !p || !id || n < 1 || maxmemb < 1 || nterms < 1 ||
      nterms > kNtermsMax)
    return BIT_ERR_INVALID_ARGUMENT;
  auto r = std::make_shared<Request>();
  r->kind = 0;
  r->n = n;
  r->nterms = nterms;
  r->maxmemb = maxmemb;
  r->x.assign(x, x + n); r->y.assign(y, y + n); r->z.assign(z, z + n); r->q.assign(q, q + n);
  r->p = *p;
  return submit(s, r, id);
}

bit_status bit_server_submit_solve(bit_server* s, int n, const double* x, const double* y,
                                   const double* z, const double* w, const double* f,
                                   int nterms, int maxmemb, const bit_eval_params* p,
                                   double diag, const bit_gmres_opts* g, long long* id) {
  if (!s || !x || !y || !z || !w || !f || !p || !g || !id || n < 1 || maxmemb < 1 ||
      nterms < 1 || nterms > kNtermsMax || g->restart < 1)
    return BIT_ERR_INVALID_ARGUMENT;
  auto r = std::make_shared<Request>();
  r->kind = 1;
  r->n = n;
  r->nterms = nterms;
  r->maxmemb = maxmemb;
  r->x.assign(x, x + n); r->y.assign(y, y + n); r->z.assign(z, z + n);
  r->q.assign(w, w + n); r->f.assign(f, f + n);
  r->p = *p;
  r->diag = diag;
  r->g = *g;
  return submit(s, r, id);
}

bit_status bit_server_wait(bit_server* s, long long id, double* out, bit_request_info* info) {
  if (!s) return BIT_ERR_INVALID_ARGUMENT;
  std::shared_ptr<Request> r;
  {
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return BIT_ERR_INVALID_ARGUMENT;
    r = it->second;
    s->cv_done.wait(lock, [&] { return r->done; });
    s->reqs.erase(it);
  }
  if (out) std::copy(r->out.begin(), r->out.end(), out);
  if (info) *info = r->info;
  return r->info.status;
}

bit_status bit_server_poll(bit_server* s, long long id, int* done) {
  if (!s || !done) return BIT_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return BIT_ERR_INVALID_ARGUMENT;
  *done = it->second->done ? 1 : 0;
  return BIT_OK;
}

bit_status bit_server_stats(bit_server* s, bit_server_info* st) {
  if (!s || !st) return BIT_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(s->mu);
  st->submitted = s->submitted;
  st->completed = s->completed;
  st->queued = (long long)s->queue.size();
  st->running = s->running;
  st->max_running = s->max_running;
  st->budget = s->budget;
  st->reserved = s->reserved + s->idle_held;
  st->max_reserved = s->max_reserved;
  st->slots = s->nslots;
  st->now = s->now();
  return BIT_OK;
}

const char* bit_server_last_error(const bit_server* s) {
  return s ? s->last_error.c_str() : "null server";
}

}  // extern "C"

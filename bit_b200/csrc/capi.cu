// The extern "C" boundary (include/bit_b200.h): argument checking, status codes, device
// memory accounting, and the order of kernel phases for each entry point.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <new>
#include <set>
#include <numeric>
#include <vector>

#include "common.cuh"

namespace bit {

// Device memory: a per-context cache of freed blocks.  All work of a context runs on its
// one stream, so a block freed after a launch can be handed to a later launch on the same
// stream without a device synchronisation (stream order protects it).  The HBM budget
// bounds live + cached bytes; cached blocks are released first when it would be exceeded.
static size_t round_block(size_t b) {
  const size_t g = b < (1u << 20) ? 512 : (size_t)2 << 20;
  return (b + g - 1) / g * g;
}

static void release_cache(Ctx* c) {
  for (auto& kv : c->cache) cudaFree(kv.second);
  c->cache.clear();
  c->cached = 0;
}

void ctx_trim(Ctx* c, size_t keep) {
  if (c->in_use + c->cached <= keep) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  // largest blocks first
  while (!c->cache.empty() && c->in_use + c->cached > keep) {
    auto it = std::prev(c->cache.end());
    cudaFree(it->second);
    c->cached -= it->first;
    c->cache.erase(it);
  }
}

// Over the budget, a request is served from any larger cached block (it costs no memory),
// and otherwise only as many cached blocks are freed, largest first, as the new block needs:
// every cudaFree waits for the device, and freeing the whole cache for one small block
// stalled served requests by hundreds of milliseconds.
static void release_for(Ctx* c, size_t bytes) {
  while (!c->cache.empty() && c->in_use + c->cached + bytes > c->budget) {
    auto it = std::prev(c->cache.end());
    cudaFree(it->second);
    c->cached -= it->first;
    c->cache.erase(it);
  }
}

void* dev_alloc(Ctx* c, size_t bytes) {
  bytes = round_block(bytes);
  auto it = c->cache.lower_bound(bytes);
  const bool tight = c->budget && c->in_use + c->cached + bytes > c->budget;
  if (it != c->cache.end() && (it->first <= 2 * bytes || tight)) {
    void* p = it->second;
    size_t sz = it->first;
    c->cache.erase(it);
    c->cached -= sz;
    c->in_use += sz;
    c->peak = std::max(c->peak, c->in_use);
    c->allocs.push_back({p, sz});
    return p;
  }
  if (tight) release_for(c, bytes);
  if (c->budget && c->in_use + bytes > c->budget)
    fail(BIT_ERR_BUDGET, "allocation of " + std::to_string(bytes) + " bytes exceeds the HBM budget");
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    release_cache(c);
    e = cudaMalloc(&p, bytes);
  }
  BIT_CUDA(e);
  c->in_use += bytes;
  c->peak = std::max(c->peak, c->in_use);
  c->allocs.push_back({p, bytes});
  return p;
}

void dev_free(Ctx* c, void* p) {
  if (!p) return;
  for (size_t i = 0; i < c->allocs.size(); i++)
    if (c->allocs[i].first == p) {
      size_t sz = c->allocs[i].second;
      c->in_use -= sz;
      c->allocs[i] = c->allocs.back();
      c->allocs.pop_back();
      c->cache.insert({sz, p});
      c->cached += sz;
      return;
    }
  cudaFree(p);
}

// Blocking device-to-host copy ordered on the context's stream (the legacy default stream
// does not order against the non-blocking context stream).
void d2h(Ctx* c, void* dst, const void* src, size_t bytes) {
  BIT_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream));
  BIT_CUDA(cudaStreamSynchronize(c->stream));
}

namespace {

__global__ void k_scatter_out(int n, const int* perm, const double* sorted, double* out) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) out[perm[e]] = sorted[e];
}

template <class F>
bit_status guard(Ctx* c, F&& f) {
  try {
    f();
    if (c) c->last_error.clear();
    return BIT_OK;
  } catch (const Error& e) {
    if (c) c->last_error = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    if (c) c->last_error = "host allocation failed";
    return BIT_ERR_OUT_OF_MEMORY;
  } catch (...) {
    if (c) c->last_error = "unexpected internal error";
    return BIT_ERR_CUDA;
  }
}

void check_params(const bit_eval_params* p) {
  if (!p) fail(BIT_ERR_INVALID_ARGUMENT, "params is NULL");
  if (p->kernel < BIT_KERNEL_COULOMB || p->kernel > BIT_KERNEL_SCREENED_REG)
    fail(BIT_ERR_INVALID_ARGUMENT, "unknown kernel");
  if (p->mode != BIT_MODE_REFERENCE && p->mode != BIT_MODE_CONSISTENT)
    fail(BIT_ERR_INVALID_ARGUMENT, "unknown mode");
  if (p->precision != BIT_PREC_FP64 && p->precision != BIT_PREC_MIXED)
    fail(BIT_ERR_INVALID_ARGUMENT, "unknown precision");
  if (!(p->acc >= 0) || !std::isfinite(p->acc)) fail(BIT_ERR_INVALID_ARGUMENT, "acc must be >= 0");
  if (!(p->del >= 0) || !std::isfinite(p->del)) fail(BIT_ERR_INVALID_ARGUMENT, "del must be >= 0");
  if (p->kernel != BIT_KERNEL_COULOMB && !(p->kappa >= 0))
    fail(BIT_ERR_INVALID_ARGUMENT, "kappa must be >= 0");
}

// Phase timers on the context stream.
enum { EV_BUILD = 0, EV_MOM = 2, EV_LIST = 4, EV_FAR = 6, EV_NEAR = 8, EV_ALL = 10 };

void ev_init(Tree* t) {
  for (auto& e : t->ev)
    if (!e) BIT_CUDA(cudaEventCreate(&e));
}
void ev_rec(Tree* t, int i) { BIT_CUDA(cudaEventRecord(t->ev[i], t->ctx->stream)); }
double ev_sec(Tree* t, int i) {
  float ms = 0;
  if (cudaEventElapsedTime(&ms, t->ev[i], t->ev[i + 1]) != cudaSuccess) {
    cudaGetLastError();
    return 0.0;
  }
  return ms * 1e-3;
}

// Errors raised on the device (a bounded wait that gave up) since the last check.
void check_dev_err(Ctx* c) {
  if (!c->err_flag) return;
  int e = 0;
  d2h(c, &e, c->err_flag, sizeof(int));
  if (e) {
    BIT_CUDA(cudaMemsetAsync(c->err_flag, 0, sizeof(int), c->stream));
    fail(BIT_ERR_CUDA, "a device-side wait gave up (error flags " + std::to_string(e) + ")");
  }
}

void eval_particles_sorted(Tree* t, const std::vector<bit_eval_params>& prm) {
  prepare_particles(t, prm, 0);
  t->pot_sorted.ensure(t->ctx, t->n);
  ev_rec(t, EV_FAR);
  eval_far(t, &t->plists, t->pplan, t->sx.p, t->sy.p, t->sz.p, t->pot_sorted.p);
  ev_rec(t, EV_FAR + 1);
  ev_rec(t, EV_NEAR);
  eval_near(t, &t->plists, t->pplan, t->sx.p, t->sy.p, t->sz.p, t->pot_sorted.p);
  ev_rec(t, EV_NEAR + 1);
  t->stats.far_pairs = t->plists.far_pairs;
  t->stats.near_pairs = t->plists.near_pairs;
  t->stats.far_entries = t->plists.nfar;
  t->stats.near_entries = t->plists.nnear;
  t->stats.batches = t->plists.ngroups;
  // several classes run as one work-queue launch each when the context allows it
  const int nfc = (int)t->pplan.far_classes.size(), nnc = (int)t->pplan.near_classes.size();
  t->stats.far_launches = (t->ctx->work_queue && nfc > 1) ? 1 : nfc;
  t->stats.near_launches = (t->ctx->work_queue && nnc > 1) ? 1 : nnc;
  t->stats.list_fallback = t->plists.fallback ? 1 : 0;
  t->stats.lists_shared = t->plists.shared ? 1 : 0;
}

uint64_t spread3(uint64_t v) {
  v &= 0x1fffff;
  v = (v | v << 32) & 0x1f00000000ffffULL;
  v = (v | v << 16) & 0x1f0000ff0000ffULL;
  v = (v | v << 8) & 0x100f00f00f00f00fULL;
  v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
  v = (v | v << 2) & 0x1249249249249249ULL;
  return v;
}

}  // namespace
}  // namespace bit

using namespace bit;

extern "C" {

const char* bit_status_string(bit_status s) {
  switch (s) {
    case BIT_OK: return "ok";
    case BIT_ERR_INVALID_ARGUMENT: return "invalid argument";
    case BIT_ERR_CUDA: return "CUDA error";
    case BIT_ERR_OUT_OF_MEMORY: return "out of memory";
    case BIT_ERR_CAPACITY: return "capacity exceeded";
    case BIT_ERR_DEGENERATE: return "degenerate input (coincident particles)";
    case BIT_ERR_BREAKDOWN: return "GMRES breakdown";
    case BIT_ERR_NOT_CONVERGED: return "not converged";
    case BIT_ERR_NO_DEVICE: return "no CUDA device";
    case BIT_ERR_BUDGET: return "HBM budget exceeded";
    case BIT_ERR_STATE: return "invalid call order";
  }
  return "unknown status";
}

int bit_abi_version(void) { return BIT_ABI_VERSION; }

bit_status bit_ctx_create(bit_ctx** out, const bit_ctx_opts* opts) {
  if (!out) return BIT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return BIT_ERR_NO_DEVICE;
  }
  bit_ctx* h = new (std::nothrow) bit_ctx;
  if (!h) return BIT_ERR_OUT_OF_MEMORY;
  bit_status st = guard(&h->c, [&] {
    Ctx& c = h->c;
    c.device = opts ? opts->device : 0;
    if (c.device < 0 || c.device >= ndev) fail(BIT_ERR_INVALID_ARGUMENT, "bad device ordinal");
    BIT_CUDA(cudaSetDevice(c.device));
    c.budget = opts ? opts->hbm_budget : 0;
    if (opts && opts->stream) {
      c.stream = static_cast<cudaStream_t>(opts->stream);
    } else {
      BIT_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
      c.own_stream = true;
    }
    BIT_CUDA(cudaDeviceGetAttribute(&c.num_sms, cudaDevAttrMultiProcessorCount, c.device));
    BIT_CUDA(cudaMallocHost(&c.h_pinned, 64 * sizeof(long long)));
  });
  if (st != BIT_OK) {
    delete h;
    return st;
  }
  *out = h;
  return BIT_OK;
}

bit_status bit_ctx_destroy(bit_ctx* h) {
  if (!h) return BIT_ERR_INVALID_ARGUMENT;
  Ctx& c = h->c;
  cudaSetDevice(c.device);
  if (c.stream) cudaStreamSynchronize(c.stream);
  // trees still held by the caller lose their device memory and their context; a later
  // bit_tree_destroy on them only frees the handle
  for (Tree* t : c.trees) {
    for (auto& e : t->ev)
      if (e) cudaEventDestroy(e);
    t->~Tree();
    new (t) Tree();
  }
  c.trees.clear();
  c.scratch_ll.release();
  c.close_cnt.release();
  c.close_n.release();
  c.close_rec.release();
  c.close_list.release();
  release_cache(&c);
  if (c.h_pinned) cudaFreeHost(c.h_pinned);
  for (int i = 0; i < 2; i++) {
    if (c.stage_ev[i]) cudaEventSynchronize(c.stage_ev[i]);
    if (c.stage[i]) cudaFreeHost(c.stage[i]);
    if (c.stage_ev[i]) cudaEventDestroy(c.stage_ev[i]);
  }
  if (c.own_stream && c.stream) cudaStreamDestroy(c.stream);
  delete h;
  return BIT_OK;
}

const char* bit_ctx_last_error(const bit_ctx* h) { return h ? h->c.last_error.c_str() : "null context"; }

bit_status bit_ctx_set_group_size(bit_ctx* h, int targets) {
  if (!h || (targets != 0 && (targets < 32 || targets > kGroupMax))) return BIT_ERR_INVALID_ARGUMENT;
  h->c.group_targets = targets;
  return BIT_OK;
}

bit_status bit_ctx_set_near_config(bit_ctx* h, int tile, int threads_per_target) {
  if (!h) return BIT_ERR_INVALID_ARGUMENT;
  if (tile != 0 && (tile < 128 || tile > 2048 || (tile & (tile - 1)))) return BIT_ERR_INVALID_ARGUMENT;
  const int s = threads_per_target;
  if (s != 0 && (s < 1 || s > 32 || (s & (s - 1)))) return BIT_ERR_INVALID_ARGUMENT;
  h->c.near_tile = tile;
  h->c.near_split = s;
  return BIT_OK;
}

bit_status bit_ctx_set_work_queue(bit_ctx* h, int on) {
  if (!h || (on != 0 && on != 1)) return BIT_ERR_INVALID_ARGUMENT;
  h->c.work_queue = on;
  return BIT_OK;
}

bit_status bit_ctx_synchronize(bit_ctx* h) {
  if (!h) return BIT_ERR_INVALID_ARGUMENT;
  return guard(&h->c, [&] { BIT_CUDA(cudaStreamSynchronize(h->c.stream)); });
}

bit_status bit_ctx_stream(const bit_ctx* h, void** stream) {
  if (!h || !stream) return BIT_ERR_INVALID_ARGUMENT;
  *stream = h->c.stream;
  return BIT_OK;
}

bit_status bit_ctx_memory(const bit_ctx* h, size_t* in_use, size_t* peak) {
  if (!h) return BIT_ERR_INVALID_ARGUMENT;
  if (in_use) *in_use = h->c.in_use;
  if (peak) *peak = h->c.peak;
  return BIT_OK;
}

bit_status bit_ctx_trim(bit_ctx* h, size_t keep) {
  if (!h) return BIT_ERR_INVALID_ARGUMENT;
  Ctx* c = &h->c;
  return guard(c, [&] {
    BIT_CUDA(cudaSetDevice(c->device));
    ctx_trim(c, keep);
  });
}

static bit_status build_common(bit_ctx* h, int nsys, const int* ns, const int* mm,
                               const double* x, const double* y, const double* z,
                               bit_tree** out, bool host) {
  if (!h || !out || !x || !y || !z || !ns || !mm || nsys < 1) return BIT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  Ctx* c = &h->c;
  long long total = 0;
  int mmin = INT_MAX;
  for (int s = 0; s < nsys; s++) {
    if (ns[s] < 1 || mm[s] < 1) {
      c->last_error = "n and maxmemb must be >= 1 (every system)";
      return BIT_ERR_INVALID_ARGUMENT;
    }
    total += ns[s];
    mmin = std::min(mmin, mm[s]);
  }
  if (total > INT_MAX / 2) {
    c->last_error = "too many particles";
    return BIT_ERR_INVALID_ARGUMENT;
  }
  const int n = (int)total;
  bit_tree* th = new (std::nothrow) bit_tree;
  if (!th) return BIT_ERR_OUT_OF_MEMORY;
  bit_status st = guard(c, [&] {
    BIT_CUDA(cudaSetDevice(c->device));
    Tree* t = &th->t;
    t->ctx = c;
    t->n = n;
    t->maxmemb = mmin;
    t->nsys = nsys;
    t->h_sys_start.resize(nsys);
    t->h_sys_n.assign(ns, ns + nsys);
    t->h_sys_maxmemb.assign(mm, mm + nsys);
    for (int s = 0, o = 0; s < nsys; o += ns[s], s++) t->h_sys_start[s] = o;
    ev_init(t);
    ev_rec(t, EV_BUILD);
    if (host) {
      DBuf<double> dx, dy, dz;
      dx.ensure(c, n); dy.ensure(c, n); dz.ensure(c, n);
      copy_h2d(c, dx.p, x, n * sizeof(double));
      copy_h2d(c, dy.p, y, n * sizeof(double));
      copy_h2d(c, dz.p, z, n * sizeof(double));
      tree_build(t, dx.p, dy.p, dz.p);
    } else {
      tree_build(t, x, y, z);
    }
    ev_rec(t, EV_BUILD + 1);
    t->stats.numtree = t->numtree;
    t->stats.nleaves = t->nleaves;
    t->stats.depth = t->depth;
  });
  if (st != BIT_OK) {
    for (auto& e : th->t.ev)
      if (e) cudaEventDestroy(e);
    delete th;
    return st;
  }
  c->trees.push_back(&th->t);
  *out = th;
  return BIT_OK;
}

bit_status bit_tree_build(bit_ctx* h, int n, const double* x, const double* y, const double* z,
                          int maxmemb, bit_tree** out) {
  return build_common(h, 1, &n, &maxmemb, x, y, z, out, true);
}

bit_status bit_tree_build_device(bit_ctx* h, int n, const double* x, const double* y,
                                 const double* z, int maxmemb, bit_tree** out) {
  return build_common(h, 1, &n, &maxmemb, x, y, z, out, false);
}

bit_status bit_forest_build(bit_ctx* h, int nsys, const int* n, const int* maxmemb,
                            const double* x, const double* y, const double* z, bit_tree** out) {
  return build_common(h, nsys, n, maxmemb, x, y, z, out, true);
}

bit_status bit_forest_build_device(bit_ctx* h, int nsys, const int* n, const int* maxmemb,
                                   const double* x, const double* y, const double* z,
                                   bit_tree** out) {
  return build_common(h, nsys, n, maxmemb, x, y, z, out, false);
}

bit_status bit_forest_systems(const bit_tree* th, int* nsys) {
  if (!th || !nsys) return BIT_ERR_INVALID_ARGUMENT;
  *nsys = th->t.nsys;
  return BIT_OK;
}

bit_status bit_forest_moments(bit_tree* th, const int* nterms) {
  if (!th || !nterms) return BIT_ERR_INVALID_ARGUMENT;
  Tree* t = &th->t;
  return guard(t->ctx, [&] {
    BIT_CUDA(cudaSetDevice(t->ctx->device));
    ev_rec(t, EV_MOM);
    tree_moments_sys(t, std::vector<int>(nterms, nterms + t->nsys));
    ev_rec(t, EV_MOM + 1);
    t->stats.nterms = t->nterms;
  });
}

static bit_status forest_eval(bit_tree* th, const bit_eval_params* prm, double* pot, bool host) {
  if (!th || !prm || !pot) return BIT_ERR_INVALID_ARGUMENT;
  Tree* t = &th->t;
  Ctx* c = t->ctx;
  return guard(c, [&] {
    for (int s = 0; s < t->nsys; s++) check_params(prm + s);
    BIT_CUDA(cudaSetDevice(c->device));
    DBuf<double> out;
    double* dst = pot;
    if (host) {
      out.ensure(c, t->n);
      dst = out.p;
    }
    ev_rec(t, EV_ALL);
    eval_particles_sorted(t, std::vector<bit_eval_params>(prm, prm + t->nsys));
    count_launch(), k_scatter_out<<<grid_for(t->n, 256), 256, 0, c->stream>>>(t->n, t->perm.p,
                                                                             t->pot_sorted.p, dst);
    BIT_CHECK_LAUNCH();
    ev_rec(t, EV_ALL + 1);
    if (host) {
      copy_d2h(c, pot, out.p, t->n * sizeof(double));
      BIT_CUDA(cudaStreamSynchronize(c->stream));
      check_dev_err(c);
    }
  });
}

bit_status bit_forest_eval(bit_tree* th, const bit_eval_params* prm, double* pot) {
  return forest_eval(th, prm, pot, true);
}
bit_status bit_forest_eval_device(bit_tree* th, const bit_eval_params* prm, double* pot) {
  return forest_eval(th, prm, pot, false);
}

bit_status bit_tree_destroy(bit_tree* th) {
  if (!th) return BIT_ERR_INVALID_ARGUMENT;
  Tree& t = th->t;
  if (t.ctx) {
    cudaSetDevice(t.ctx->device);
    cudaStreamSynchronize(t.ctx->stream);
    auto& v = t.ctx->trees;
    v.erase(std::remove(v.begin(), v.end(), &t), v.end());
  }
  for (auto& e : t.ev)
    if (e) cudaEventDestroy(e);
  delete th;
  return BIT_OK;
}

bit_status bit_tree_info(const bit_tree* th, int* numtree, int* nleaves, int* depth) {
  if (!th) return BIT_ERR_INVALID_ARGUMENT;
  if (numtree) *numtree = th->t.numtree;
  if (nleaves) *nleaves = th->t.nleaves;
  if (depth) *depth = th->t.depth;
  return BIT_OK;
}

static bit_status set_charges(bit_tree* th, const double* q, const double* w, bool host) {
  if (!th || !q) return BIT_ERR_INVALID_ARGUMENT;
  Tree* t = &th->t;
  Ctx* c = t->ctx;
  return guard(c, [&] {
    BIT_CUDA(cudaSetDevice(c->device));
    if (host) {
      DBuf<double> dq, dw;
      dq.ensure(c, t->n);
      copy_h2d(c, dq.p, q, t->n * sizeof(double));
      if (w) {
        dw.ensure(c, t->n);
        copy_h2d(c, dw.p, w, t->n * sizeof(double));
      }
      tree_set_charges(t, dq.p, w ? dw.p : nullptr);
      BIT_CUDA(cudaStreamSynchronize(c->stream));
    } else {
      tree_set_charges(t, q, w);
    }
  });
}

bit_status bit_tree_set_charges(bit_tree* th, const double* q, const double* w) {
  return set_charges(th, q, w, true);
}
bit_status bit_tree_set_charges_device(bit_tree* th, const double* q, const double* w) {
  return set_charges(th, q, w, false);
}

bit_status bit_tree_moments(bit_tree* th, int nterms) {
  if (!th) return BIT_ERR_INVALID_ARGUMENT;
  Tree* t = &th->t;
  return guard(t->ctx, [&] {
    BIT_CUDA(cudaSetDevice(t->ctx->device));
    ev_rec(t, EV_MOM);
    tree_moments(t, nterms);
    ev_rec(t, EV_MOM + 1);
    t->stats.nterms = nterms;
  });
}

bit_status bit_tree_export(const bit_tree* th, int* nummemb, int* children, double* fields,
                           int* members) {
  if (!th) return BIT_ERR_INVALID_ARGUMENT;
  const Tree* t = &th->t;
  return guard(t->ctx, [&] {
    const int b = t->numtree;
    if (nummemb) std::memcpy(nummemb, t->h_nummemb.data(), b * sizeof(int));
    if (children) std::memcpy(children, t->h_children.data(), 8LL * b * sizeof(int));
    if (fields) std::memcpy(fields, t->h_fields.data(), 13LL * b * sizeof(double));
    if (members) {
      std::vector<int> perm(t->n);
      d2h(t->ctx, perm.data(), t->perm.p, t->n * sizeof(int));
      long long off = 0;
      for (int i = 0; i < b; i++) {
        int st = t->h_start[i], cnt = t->h_nummemb[i];
        std::memcpy(members + off, perm.data() + st, cnt * sizeof(int));
        std::sort(members + off, members + off + cnt);
        off += cnt;
      }
    }
  });
}

bit_status bit_tree_export_moments(const bit_tree* th, double* mom) {
  if (!th || !mom) return BIT_ERR_INVALID_ARGUMENT;
  const Tree* t = &th->t;
  if (!t->has_moments) return BIT_ERR_STATE;
  return guard(t->ctx, [&] {
    d2h(t->ctx, mom, t->mom64.p, (size_t)t->mom_total * sizeof(double));
  });
}

bit_status bit_eval_particles_device(bit_tree* th, const bit_eval_params* prm, double* pot) {
  if (!th || !pot) return BIT_ERR_INVALID_ARGUMENT;
  Tree* t = &th->t;
  return guard(t->ctx, [&] {
    check_params(prm);
    BIT_CUDA(cudaSetDevice(t->ctx->device));
    ev_rec(t, EV_ALL);
    eval_particles_sorted(t, {*prm});
    count_launch(), k_scatter_out<<<grid_for(t->n, 256), 256, 0, t->ctx->stream>>>(t->n, t->perm.p,
                                                                   t->pot_sorted.p, pot);
    BIT_CHECK_LAUNCH();
    ev_rec(t, EV_ALL + 1);
  });
}

bit_status bit_eval_particles(bit_tree* th, const bit_eval_params* prm, double* pot) {
  if (!th || !pot) return BIT_ERR_INVALID_ARGUMENT;
  Tree* t = &th->t;
  Ctx* c = t->ctx;
  return guard(c, [&] {
    check_params(prm);
    BIT_CUDA(cudaSetDevice(c->device));
    DBuf<double> out;
    out.ensure(c, t->n);
    ev_rec(t, EV_ALL);
    eval_particles_sorted(t, {*prm});
    count_launch(), k_scatter_out<<<grid_for(t->n, 256), 256, 0, c->stream>>>(t->n, t->perm.p, t->pot_sorted.p, out.p);
    BIT_CHECK_LAUNCH();
    ev_rec(t, EV_ALL + 1);
    copy_d2h(c, pot, out.p, t->n * sizeof(double));
    BIT_CUDA(cudaStreamSynchronize(c->stream));
    check_dev_err(c);
  });
}

bit_status bit_eval_points(bit_tree* th, const bit_eval_params* prm, int m, const double* x,
                           const double* y, const double* z, double* pot) {
  if (!th || !x || !y || !z || !pot || m < 0) return BIT_ERR_INVALID_ARGUMENT;
  if (m == 0) return BIT_OK;
  Tree* t = &th->t;
  Ctx* c = t->ctx;
  return guard(c, [&] {
    check_params(prm);
    if (!t->has_moments) fail(BIT_ERR_STATE, "moments not computed");
    BIT_CUDA(cudaSetDevice(c->device));
    // spatial (Morton) order of the points so that a batch is compact
    double lo[3] = {x[0], y[0], z[0]}, hi[3] = {x[0], y[0], z[0]};
    for (int i = 0; i < m; i++) {
      double v[3] = {x[i], y[i], z[i]};
      for (int a = 0; a < 3; a++) {
        if (std::isnan(v[a])) fail(BIT_ERR_INVALID_ARGUMENT, "point coordinates contain NaN");
        lo[a] = std::min(lo[a], v[a]);
        hi[a] = std::max(hi[a], v[a]);
      }
    }
    std::vector<std::pair<uint64_t, int>> key(m);
    for (int i = 0; i < m; i++) {
      double v[3] = {x[i], y[i], z[i]};
      uint64_t code = 0;
      for (int a = 0; a < 3; a++) {
        double s = hi[a] > lo[a] ? (v[a] - lo[a]) / (hi[a] - lo[a]) : 0.0;
        uint64_t q = (uint64_t)std::min(2097151.0, std::max(0.0, s * 2097151.0));
        code |= spread3(q) << a;
      }
      key[i] = {code, i};
    }
    std::sort(key.begin(), key.end());
    std::vector<double> sx(m), sy(m), sz(m);
    std::vector<int> ord(m);
    for (int i = 0; i < m; i++) {
      ord[i] = key[i].second;
      sx[i] = x[ord[i]]; sy[i] = y[ord[i]]; sz[i] = z[ord[i]];
    }
    DBuf<double> dx, dy, dz, out;
    DBuf<int> dord;
    dx.ensure(c, m); dy.ensure(c, m); dz.ensure(c, m); out.ensure(c, m); dord.ensure(c, m);
    cudaStream_t s = c->stream;
    copy_h2d(c, dx.p, sx.data(), m * sizeof(double));
    copy_h2d(c, dy.p, sy.data(), m * sizeof(double));
    copy_h2d(c, dz.p, sz.data(), m * sizeof(double));
    copy_h2d(c, dord.p, ord.data(), m * sizeof(int));
    Lists L;
    EvalPlan P;
    plan_sys(t, &P, {*prm}, 1, 0);
    build_lists(t, &L, plan_key(t, P, 1), m, dx.p, dy.p, dz.p, P.sys.p);
    plan_classes(t, &L, &P);
    eval_far(t, &L, P, dx.p, dy.p, dz.p, out.p);
    eval_near(t, &L, P, dx.p, dy.p, dz.p, out.p);
    DBuf<double> res;
    res.ensure(c, m);
    count_launch(), k_scatter_out<<<grid_for(m, 256), 256, 0, s>>>(m, dord.p, out.p, res.p);
    BIT_CHECK_LAUNCH();
    copy_d2h(c, pot, res.p, m * sizeof(double));
    BIT_CUDA(cudaStreamSynchronize(s));
    check_dev_err(c);
  });
}

bit_status bit_eval_force(bit_tree* th, double del, double acc, bit_precision prec, double* fx,
                          double* fy, double* fz) {
  bit_field_params f{};
  f.kind = BIT_FIELD_COULOMB;
  f.precision = prec;
  f.del = del;
  f.acc = acc;
  return bit_eval_field(th, &f, fx, fy, fz);
}

bit_status bit_eval_field(bit_tree* th, const bit_field_params* fp, double* fx, double* fy,
                          double* fz) {
  if (!th || !fp || !fx || !fy || !fz) return BIT_ERR_INVALID_ARGUMENT;
  Tree* t = &th->t;
  Ctx* c = t->ctx;
  return guard(c, [&] {
    if (!t->has_moments) fail(BIT_ERR_STATE, "moments not computed");
    if (t->nterms > kNtermsMax) fail(BIT_ERR_INVALID_ARGUMENT, "nterms too large for the force");
    if (fp->kind != BIT_FIELD_COULOMB && fp->kind != BIT_FIELD_SCREENED)
      fail(BIT_ERR_INVALID_ARGUMENT, "unknown field kind");
    if (fp->precision != BIT_PREC_FP64 && fp->precision != BIT_PREC_MIXED)
      fail(BIT_ERR_INVALID_ARGUMENT, "unknown precision");
    if (fp->kernel_order < 0 || fp->kernel_order > BIT_KERNEL_ORDER_MAX)
      fail(BIT_ERR_INVALID_ARGUMENT, "kernel_order out of range");
    if (fp->precision == BIT_PREC_MIXED && (fp->kind == BIT_FIELD_SCREENED || fp->kernel_order > 0))
      fail(BIT_ERR_INVALID_ARGUMENT, "this field is evaluated in FP64 only");
    if (!(fp->acc >= 0.0) || !std::isfinite(fp->del) || !std::isfinite(fp->kappa))
      fail(BIT_ERR_INVALID_ARGUMENT, "acc, del and kappa must be finite, acc >= 0");
    BIT_CUDA(cudaSetDevice(c->device));
    bit_eval_params p{};
    p.kernel = fp->kind == BIT_FIELD_SCREENED ? BIT_KERNEL_SCREENED : BIT_KERNEL_COULOMB;
    p.del = fp->del;
    p.mac_del = fp->mac_del;
    p.kappa = fp->kappa;
    p.acc = fp->acc;
    p.precision = fp->precision;
    prepare_particles(t, {p}, fp->kind == BIT_FIELD_SCREENED ? 2 : 1, fp->kernel_order);
    const int n = t->n;
    t->fx_sorted.ensure(c, n); t->fy_sorted.ensure(c, n); t->fz_sorted.ensure(c, n);
    ev_rec(t, EV_FAR);
    eval_far_force(t, &t->plists, t->pplan, t->fx_sorted.p, t->fy_sorted.p, t->fz_sorted.p);
    ev_rec(t, EV_FAR + 1);
    ev_rec(t, EV_NEAR);
    eval_near_force(t, &t->plists, t->pplan, t->fx_sorted.p, t->fy_sorted.p, t->fz_sorted.p);
    ev_rec(t, EV_NEAR + 1);
    DBuf<double> o;
    o.ensure(c, 3LL * n);
    cudaStream_t s = c->stream;
    count_launch(), k_scatter_out<<<grid_for(n, 256), 256, 0, s>>>(n, t->perm.p, t->fx_sorted.p, o.p);
    count_launch(), k_scatter_out<<<grid_for(n, 256), 256, 0, s>>>(n, t->perm.p, t->fy_sorted.p, o.p + n);
    count_launch(), k_scatter_out<<<grid_for(n, 256), 256, 0, s>>>(n, t->perm.p, t->fz_sorted.p, o.p + 2LL * n);
    BIT_CHECK_LAUNCH();
    copy_d2h(c, fx, o.p, n * sizeof(double));
    copy_d2h(c, fy, o.p + n, n * sizeof(double));
    copy_d2h(c, fz, o.p + 2LL * n, n * sizeof(double));
    BIT_CUDA(cudaStreamSynchronize(s));
    check_dev_err(c);
  });
}

namespace bit {
namespace {
// After the field of step k (tree order): the reference's force scaling and explicit
// update, particle by particle in original order, without contraction so the arithmetic
// is the reference's (src/tree3d.cpp:2330-2332, 4846-4848, 4884-4886):
//   F = f * charge_constant * q;  u += dt * F * invmass;  x += dt * u
__global__ void k_pic_update(int n, const int* perm, const double* fxs, const double* fys,
                             const double* fzs, const double* q, double cc, double invmass,
                             double dt, double* x, double* y, double* z, double* u, double* v,
                             double* w, double* fx_out, double* fy_out, double* fz_out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const int j = perm[e];
  const double qj = q[j];
  const double Fx = dmul(dmul(fxs[e], cc), qj), Fy = dmul(dmul(fys[e], cc), qj),
               Fz = dmul(dmul(fzs[e], cc), qj);
  if (fx_out) { fx_out[j] = Fx; fy_out[j] = Fy; fz_out[j] = Fz; }
  const double uj = dadd(u[j], dmul(dmul(dt, Fx), invmass));
  const double vj = dadd(v[j], dmul(dmul(dt, Fy), invmass));
  const double wj = dadd(w[j], dmul(dmul(dt, Fz), invmass));
  u[j] = uj; v[j] = vj; w[j] = wj;
  x[j] = dadd(x[j], dmul(dt, uj));
  y[j] = dadd(y[j], dmul(dt, vj));
  z[j] = dadd(z[j], dmul(dt, wj));
}
}  // namespace
}  // namespace bit

bit_status bit_pic_steps(bit_ctx* h, int n, double* x, double* y, double* z, double* u,
                         double* v, double* w, const double* q, const bit_pic_opts* o,
                         double* fx, double* fy, double* fz) {
  if (!h || !x || !y || !z || !u || !v || !w || !q || !o || n < 1) return BIT_ERR_INVALID_ARGUMENT;
  if ((fx || fy || fz) && !(fx && fy && fz)) return BIT_ERR_INVALID_ARGUMENT;
  Ctx* c = &h->c;
  if (o->steps < 0 || o->maxmemb < 1 || o->nterms < 1 || o->nterms > kNtermsMax) {
    c->last_error = "steps >= 0, maxmemb >= 1 and 1 <= nterms <= BIT_NTERMS_MAX required";
    return BIT_ERR_INVALID_ARGUMENT;
  }
  for (int k = 0; k < o->steps; k++) {
    bit_tree* th = nullptr;
    bit_status st = bit_tree_build_device(h, n, x, y, z, o->maxmemb, &th);
    if (st == BIT_OK) st = bit_tree_set_charges_device(th, q, nullptr);
    if (st == BIT_OK) st = bit_tree_moments(th, o->nterms);
    if (st == BIT_OK) {
      Tree* t = &th->t;
      st = guard(c, [&] {
        bit_eval_params p{};
        p.kernel = BIT_KERNEL_COULOMB;
        p.del = o->del;
        p.acc = o->acc;
        p.precision = o->precision;
        prepare_particles(t, {p}, 1);
        t->fx_sorted.ensure(c, n); t->fy_sorted.ensure(c, n); t->fz_sorted.ensure(c, n);
        eval_far_force(t, &t->plists, t->pplan, t->fx_sorted.p, t->fy_sorted.p, t->fz_sorted.p);
        eval_near_force(t, &t->plists, t->pplan, t->fx_sorted.p, t->fy_sorted.p, t->fz_sorted.p);
        const bool last = k == o->steps - 1;
        count_launch(), k_pic_update<<<grid_for(n, 256), 256, 0, c->stream>>>(
            n, t->perm.p, t->fx_sorted.p, t->fy_sorted.p, t->fz_sorted.p, q, o->charge_constant,
            o->invmass, o->dt, x, y, z, u, v, w, last ? fx : nullptr, last ? fy : nullptr,
            last ? fz : nullptr);
        BIT_CHECK_LAUNCH();
      });
    }
    if (th) {
      std::string keep = c->last_error;
      bit_tree_destroy(th);
      c->last_error = keep;
    }
    if (st != BIT_OK) return st;
  }
  return guard(c, [&] {
    BIT_CUDA(cudaStreamSynchronize(c->stream));
    check_dev_err(c);
  });
}

bit_status bit_treecode_potential(bit_ctx* h, int n, const double* x, const double* y,
                                  const double* z, const double* q, const double* w, int nterms,
                                  int maxmemb, const bit_eval_params* prm, double* pot) {
  if (!h || !q || !pot || !prm) return BIT_ERR_INVALID_ARGUMENT;
  bit_tree* t = nullptr;
  bit_status st = bit_tree_build(h, n, x, y, z, maxmemb, &t);
  if (st == BIT_OK) st = bit_tree_set_charges(t, q, w);
  if (st == BIT_OK) st = bit_tree_moments(t, nterms);
  if (st == BIT_OK) st = bit_eval_particles(t, prm, pot);
  if (t) {
    std::string keep = h->c.last_error;
    bit_tree_destroy(t);
    h->c.last_error = keep;
  }
  return st;
}

bit_status bit_direct_potential(bit_ctx* h, int n, const double* x, const double* y,
                                const double* z, const double* q, const bit_eval_params* prm,
                                int m, const int* targets, double* pot) {
  if (!h || !x || !y || !z || !q || !prm || !targets || !pot || n < 1 || m < 0)
    return BIT_ERR_INVALID_ARGUMENT;
  if (m == 0) return BIT_OK;
  Ctx* c = &h->c;
  return guard(c, [&] {
    check_params(prm);
    for (int i = 0; i < m; i++)
      if (targets[i] < 0 || targets[i] >= n) fail(BIT_ERR_INVALID_ARGUMENT, "target index out of range");
    BIT_CUDA(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    DBuf<double> dx, dy, dz, dq, out;
    DBuf<int> dt;
    dx.ensure(c, n); dy.ensure(c, n); dz.ensure(c, n); dq.ensure(c, n);
    dt.ensure(c, m); out.ensure(c, m);
    copy_h2d(c, dx.p, x, n * sizeof(double));
    copy_h2d(c, dy.p, y, n * sizeof(double));
    copy_h2d(c, dz.p, z, n * sizeof(double));
    copy_h2d(c, dq.p, q, n * sizeof(double));
    copy_h2d(c, dt.p, targets, m * sizeof(int));
    direct_potential(c, n, dx.p, dy.p, dz.p, dq.p, *prm, m, dt.p, out.p);
    copy_d2h(c, pot, out.p, m * sizeof(double));
    BIT_CUDA(cudaStreamSynchronize(s));
    check_dev_err(c);
  });
}

bit_status bit_direct_potential_device(bit_ctx* h, int n, const double* x, const double* y,
                                       const double* z, const double* q,
                                       const bit_eval_params* prm, int m, const int* targets,
                                       double* pot) {
  if (!h || !x || !y || !z || !q || !prm || !targets || !pot || n < 1 || m < 0)
    return BIT_ERR_INVALID_ARGUMENT;
  if (m == 0) return BIT_OK;
  Ctx* c = &h->c;
  return guard(c, [&] {
    check_params(prm);
    BIT_CUDA(cudaSetDevice(c->device));
    direct_potential(c, n, x, y, z, q, *prm, m, targets, pot);
  });
}

bit_status bit_direct_field(bit_ctx* h, int n, const double* x, const double* y,
                            const double* z, const double* q, int regularised, double del,
                            int kernel_order, int m, const int* targets, double* fx, double* fy,
                            double* fz) {
  if (!h || !x || !y || !z || !q || !targets || !fx || !fy || !fz || n < 1 || m < 0)
    return BIT_ERR_INVALID_ARGUMENT;
  if (m == 0) return BIT_OK;
  Ctx* c = &h->c;
  return guard(c, [&] {
    if (kernel_order < 0 || kernel_order > BIT_KERNEL_ORDER_MAX)
      fail(BIT_ERR_INVALID_ARGUMENT, "kernel_order out of range");
    if (!std::isfinite(del)) fail(BIT_ERR_INVALID_ARGUMENT, "del must be finite");
    for (int i = 0; i < m; i++)
      if (targets[i] < 0 || targets[i] >= n) fail(BIT_ERR_INVALID_ARGUMENT, "target index out of range");
    BIT_CUDA(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    DBuf<double> dx, dy, dz, dq, out;
    DBuf<int> dt;
    dx.ensure(c, n); dy.ensure(c, n); dz.ensure(c, n); dq.ensure(c, n);
    dt.ensure(c, m); out.ensure(c, 3LL * m);
    copy_h2d(c, dx.p, x, n * sizeof(double));
    copy_h2d(c, dy.p, y, n * sizeof(double));
    copy_h2d(c, dz.p, z, n * sizeof(double));
    copy_h2d(c, dq.p, q, n * sizeof(double));
    copy_h2d(c, dt.p, targets, m * sizeof(int));
    direct_field(c, n, dx.p, dy.p, dz.p, dq.p, regularised, del, kernel_order, m, dt.p, out.p);
    copy_d2h(c, fx, out.p, m * sizeof(double));
    copy_d2h(c, fy, out.p + m, m * sizeof(double));
    copy_d2h(c, fz, out.p + 2LL * m, m * sizeof(double));
    BIT_CUDA(cudaStreamSynchronize(s));
    check_dev_err(c);
  });
}

bit_status bit_device_fma_peak(bit_ctx* h, bit_precision prec, double* flops_per_s) {
  if (!h || !flops_per_s || (prec != BIT_PREC_FP64 && prec != BIT_PREC_MIXED))
    return BIT_ERR_INVALID_ARGUMENT;
  Ctx* c = &h->c;
  return guard(c, [&] {
    BIT_CUDA(cudaSetDevice(c->device));
    *flops_per_s = fma_peak(c, prec == BIT_PREC_MIXED);
  });
}

bit_status bit_device_fp64_math_error(bit_ctx* h, long long n, double* exp_ulps,
                                      double* rsqrt_ulps) {
  if (!h || !exp_ulps || !rsqrt_ulps || n < 1) return BIT_ERR_INVALID_ARGUMENT;
  Ctx* c = &h->c;
  return guard(c, [&] {
    BIT_CUDA(cudaSetDevice(c->device));
    fp64_math_error(c, n, exp_ulps, rsqrt_ulps);
  });
}

bit_status bit_device_wait_check(bit_ctx* h, int limit) {
  if (!h || limit < 1) return BIT_ERR_INVALID_ARGUMENT;
  Ctx* c = &h->c;
  return guard(c, [&] {
    BIT_CUDA(cudaSetDevice(c->device));
    device_wait_check(c, limit);
    check_dev_err(c);
  });
}

bit_status bit_tree_stats(const bit_tree* th, bit_stats* st) {
  if (!th || !st) return BIT_ERR_INVALID_ARGUMENT;
  Tree* t = const_cast<Tree*>(&th->t);
  return guard(t->ctx, [&] {
    BIT_CUDA(cudaStreamSynchronize(t->ctx->stream));
    check_dev_err(t->ctx);
    bit_stats s = t->stats;
    s.t_build = ev_sec(t, EV_BUILD);
    s.t_moments = ev_sec(t, EV_MOM);
    s.t_lists = t->lists_built ? ev_sec(t, EV_LIST) : 0.0;  // 0: the lists were reused
    s.t_far = ev_sec(t, EV_FAR);
    s.t_near = ev_sec(t, EV_NEAR);
    s.t_total = ev_sec(t, EV_ALL);
    s.numtree = t->numtree;
    s.nleaves = t->nleaves;
    s.depth = t->depth;
    s.nterms = t->nterms;
    *st = s;
  });
}

bit_status bit_tree_target_lists(bit_tree* th, const bit_eval_params* prm, int p, int* node,
                                 int* kind, int cap, int* n) {
  if (!th || !prm || !n || p < 0 || p >= th->t.n) return BIT_ERR_INVALID_ARGUMENT;
  Tree* t = &th->t;
  return guard(t->ctx, [&] {
    check_params(prm);
    prepare_particles(t, {*prm}, 0);
    Lists& L = t->plists;
    Ctx* c = t->ctx;
    int e = 0;
    d2h(c, &e, t->iperm.p + p, sizeof(int));
    const int ng = L.ngroups;
    std::vector<int> ts(ng), tc(ng);
    d2h(c, ts.data(), L.g_tstart.p, ng * sizeof(int));
    d2h(c, tc.data(), L.g_tcount.p, ng * sizeof(int));
    int g = -1;
    for (int i = 0; i < ng; i++)
      if (e >= ts[i] && e < ts[i] + tc[i]) { g = i; break; }
    if (g < 0) fail(BIT_ERR_STATE, "target not found in the groups");
    const int lane = e - ts[g], W = (tc[g] + 31) / 32;
    std::vector<std::pair<int, int>> all;
    for (int kd = 0; kd < 2; kd++) {
      const DBuf<long long>& off = kd ? L.near_off : L.far_off;
      const DBuf<int>& cntb = kd ? L.near_cnt : L.far_cnt;
      const DBuf<long long>& moff = kd ? L.near_moff : L.far_moff;
      const DBuf<int>& nd = kd ? L.near_node : L.far_node;
      const DBuf<unsigned>& mk = kd ? L.near_mask : L.far_mask;
      long long o[1], mo = 0;
      int ecount = 0;
      d2h(c, o, off.p + g, sizeof(long long));
      d2h(c, &ecount, cntb.p + g, sizeof(int));
      d2h(c, &mo, moff.p + g, sizeof(long long));
      const long long ne = ecount;
      if (!ne) continue;
      std::vector<int> nodes(ne);
      std::vector<unsigned> masks(ne * W);
      d2h(c, nodes.data(), nd.p + o[0], ne * sizeof(int));
      d2h(c, masks.data(), mk.p + mo, ne * W * sizeof(unsigned));
      for (long long k = 0; k < ne; k++)
        if ((masks[k * W + lane / 32] >> (lane % 32)) & 1u) all.push_back({nodes[k], kd});
    }
    // far and near entries were emitted along one depth-first walk: order by preorder rank
    std::vector<int> rank(t->numtree, 0);
    {
      int r = 0;
      std::vector<int> stk;
      for (int sy = t->nsys - 1; sy >= 0; sy--) stk.push_back(sy);
      while (!stk.empty()) {
        int nd = stk.back();
        stk.pop_back();
        rank[nd] = r++;
        for (int k = 7; k >= 0; k--) {
          int ch = t->h_children[8LL * nd + k];
          if (ch != -1) stk.push_back(ch);
        }
      }
    }
    std::sort(all.begin(), all.end(), [&](const std::pair<int, int>& a, const std::pair<int, int>& b2) {
      return rank[a.first] < rank[b2.first];
    });
    for (int i = 0; i < (int)all.size() && i < cap; i++) {
      if (node) node[i] = all[i].first;
      if (kind) kind[i] = all[i].second;
    }
    *n = (int)all.size();
  });
}

}  // extern "C"

namespace bit {
std::atomic<long long>& launch_counter() {
  static std::atomic<long long> n{0};
  return n;
}

void ensure_smem_attr(const void* kernel, int bytes) {
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  int dev = 0;
  BIT_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  const auto key = std::make_pair(kernel, dev);
  if (done.count(key)) return;
  BIT_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  done.insert(key);
}
}  // namespace bit

extern "C" long long bit_kernel_launches(void) { return bit::launch_counter().load(); }

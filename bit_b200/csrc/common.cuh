// Internal definitions shared by the CUDA sources of libbit_b200 (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <map>
#include <string>
#include <vector>

#include "bit_b200.h"

namespace bit {

constexpr int kWarp = 32;
constexpr int kNtermsMax = BIT_NTERMS_MAX;
constexpr int kGroupMax = 1024;   // targets per group (one CTA; 32 mask words)
constexpr int kPointGroup = 256;  // external points per group
constexpr double kEpsNear = 1e-14;  // src/constants.h:35

__host__ __device__ constexpr int num_terms(int n) { return n * (n + 1) * (n + 2) / 6; }

// ---- status plumbing ----------------------------------------------------------------
struct Error {
  bit_status code;
  std::string msg;
};

#define BIT_CUDA(call)                                                                   \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      throw ::bit::Error{e_ == cudaErrorMemoryAllocation ? BIT_ERR_OUT_OF_MEMORY        \
                                                         : BIT_ERR_CUDA,                 \
                         std::string(#call) + ": " + cudaGetErrorString(e_)};            \
  } while (0)

#define BIT_CHECK_LAUNCH() BIT_CUDA(cudaGetLastError())

inline void fail(bit_status c, const std::string& m) { throw Error{c, m}; }

// Kernels launched by this library in this process (every launch site counts itself;
// several host threads may launch at once).
std::atomic<long long>& launch_counter();
inline void count_launch() { launch_counter().fetch_add(1, std::memory_order_relaxed); }

// Set a kernel's dynamic shared-memory limit once per (kernel, current device); safe to
// call from several host threads.
void ensure_smem_attr(const void* kernel, int bytes);

// ---- device memory with budget accounting ------------------------------------------
struct Ctx;
struct Tree;
void* dev_alloc(Ctx* c, size_t bytes);
void dev_free(Ctx* c, void* p);
// Copies between caller (pageable) host arrays and device memory on the context stream;
// large ones are staged through pinned chunks.  copy_h2d returns once the host array may be
// reused (the device copy completes in stream order); copy_d2h returns with the data in
// place.
void copy_h2d(Ctx* c, void* dst, const void* src, size_t bytes);
void copy_d2h(Ctx* c, void* dst, const void* src, size_t bytes);
// Free cached (unused) blocks until live + cached bytes are at most `keep`.
void ctx_trim(Ctx* c, size_t keep);

template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  Ctx* c = nullptr;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  void release() {
    if (p) dev_free(c, p);
    p = nullptr;
    n = 0;
  }
  // (Re)allocate to at least `count` elements; contents are not preserved.
  void ensure(Ctx* ctx, size_t count) {
    if (count <= n && p) return;
    release();
    c = ctx;
    if (count == 0) count = 1;
    p = static_cast<T*>(dev_alloc(ctx, count * sizeof(T)));
    n = count;
  }
  // Grow keeping the first `keep` elements.
  void grow(Ctx* ctx, size_t count, size_t keep, cudaStream_t s);
  T* get() const { return p; }
};

// ---- per-system evaluation parameters (device copy) ------------------------------------
// Everything a kernel needs to know about the system a target group belongs to.
struct SysEval {
  double acc, mac_add, mac_sub;  // MAC: sqradius < acc * ((r^2 + mac_add) - mac_sub)
  double far_add;                // distance^2 fed to the far recurrence: r^2 + far_add
  double far_sign;               // +1, or -1 for the screened potential
  double kappa;
  double near_del;               // added to r^2 in the near field
  double intg;                   // reference-mode screened self term
  int kernel, nterms;
  int near_sign, eps_check, self_term, particles;
  int kernel_order;  // regularised Coulomb field: the reference's KERNEL_ORDER (src/problem.h:13)
  int pad_;
};

// One launch of a far / near kernel: the groups of one (nterms, kernel) class.
struct LaunchClass {
  int nterms, kernel, eps;  // eps: near field skips r^2 <= 1e-14
  int begin, count;         // range in the class-ordered group array
};

struct EvalPlan {
  std::vector<SysEval> h_sys;
  DBuf<SysEval> sys;
  bool f32 = false;
  int force = 0;
  std::vector<LaunchClass> far_classes, near_classes;
  DBuf<int> far_order, near_order;   // used when there is more than one class
  const int* far_ord = nullptr;      // group order of the far / near launches
  const int* near_ord = nullptr;
  long long lists_version = -1;      // lists the classes were planned for
  std::vector<long long> class_key;  // per system: far and near class of the last plan
};

// ---- interaction lists of one target set under one MAC --------------------------------
struct ListKey {
  double acc = -1, add_del = 0, sub_del = 0;
  int points = 0;  // 0: particle targets, 1: external points
  int group = 0;  // particle targets packed per group (0: one leaf per group)
  long long gen = -1;  // tree generation it was built for
  std::vector<double> sysmac;  // forests: (acc, add, sub) of every system
  bool operator==(const ListKey& o) const {
    return acc == o.acc && add_del == o.add_del && sub_del == o.sub_del &&
           points == o.points && group == o.group && gen == o.gen && sysmac == o.sysmac;
  }
  bool same_mac(const ListKey& o) const {
    return acc == o.acc && add_del == o.add_del && sub_del == o.sub_del && sysmac == o.sysmac;
  }
};

// Sizes of a list build, kept to size the next one (by its tree, and by its context for
// the next tree: a step that rebuilds its tree meets the same MAC on similar data).
struct ListSizing {
  int ngroups = 0;                          // 0: no build yet
  double acc = -1;                          // the build's MAC parameter
  int points = 0;
  unsigned long long totals[4] = {0, 0, 0, 0};  // far entries, far words, near entries, near words
  long long stage[2] = {0, 0};              // largest group: far, near staging words
                                            // (entries x (mask words + 1))
};

struct Lists {
  ListKey key;
  bool valid = false;
  int ngroups = 0;
  int ntargets = 0;                         // targets the groups cover
  long long nfar = 0, nnear = 0;            // entries
  long long far_pairs = 0, near_pairs = 0;  // interactions
  DBuf<int> g_tstart, g_tcount;             // group: first target, count
  DBuf<int> g_sys;                          // group: system (its root node)
  std::vector<int> h_g_sys;
  DBuf<long long> far_off, near_off;        // first entry of each group
  DBuf<int> far_cnt, near_cnt;              // entries of each group
  DBuf<long long> far_moff, near_moff;      // first mask word of each group
  DBuf<int> far_node, near_node;            // entry -> node
  DBuf<unsigned> far_mask, near_mask;       // (tcount+31)/32 words per entry
  DBuf<int> order;                          // groups by decreasing work
  DBuf<int> far_cost;                       // far field scratch: targets of each far entry
  std::vector<long long> h_work;            // estimated work of each group
  long long version = 0;                    // bumped by every build
  ListSizing last;                          // the last build's sizes
  bool fallback = false;                    // the last build used count, scan and fill
  DBuf<unsigned> gstage;                    // per resident CTA: staging of one group's entries
  DBuf<int> head;                           // the single-pass build's work counter
  // The lists also serve alt_key when alt_valid: the build checked that MAC at every
  // (target, node) it visited and no decision differed, so that MAC's own traversal
  // would have visited the same nodes and emitted the same entries.
  ListKey alt_key;
  bool alt_valid = false;
  bool shared = false;  // the last evaluation used them through alt_key
};

struct Ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  size_t budget = 0, in_use = 0, peak = 0;
  std::string last_error;
  int num_sms = 148;
  int group_targets = 0;  // leaves packed into groups of up to this many targets (0: off)
  // Plans with several launch classes (forests): 1 runs each field as one persistent
  // kernel over a device work queue of all groups, 0 as one launch per class.
  int work_queue = 1;
  DBuf<int> queue_heads;  // the work queues' counters (far, near)
  // near-field tuning knobs (bit_ctx_set_near_config): source records per tile and the cap
  // on threads per target (0: the defaults)
  int near_tile = 0, near_split = 0;
  ListKey mac_hint;       // MAC of the last particle-target evaluation (acc < 0: none)
  ListSizing list_hint;   // sizes of the last list build of any tree
  // small device scratch for flags / counters
  DBuf<long long> scratch_ll;
  long long* h_pinned = nullptr;  // pinned host staging for small read-backs (64 entries)
  std::vector<std::pair<void*, size_t>> allocs;  // live device allocations and their sizes
  std::multimap<size_t, void*> cache;             // freed blocks kept for reuse, by size
  size_t cached = 0;                              // bytes held in `cache`
  std::vector<Tree*> trees;                       // trees built by this context
  long long launches = 0;                         // kernels launched by this context
  int* err_flag = nullptr;                        // device word kernels raise errors in
  // mixed near field: close pairs left to the FP64 pass, per target
  DBuf<int> close_cnt, close_n;
  DBuf<int2> close_rec, close_list;
  void* stage[2] = {nullptr, nullptr};            // pinned staging chunks for host copies
  cudaEvent_t stage_ev[2] = {nullptr, nullptr};
  int* dev_err() {
    if (!err_flag) {
      err_flag = static_cast<int*>(dev_alloc(this, 64));
      cudaMemsetAsync(err_flag, 0, 64, stream);
    }
    return err_flag;
  }
};

struct Tree {
  Ctx* ctx = nullptr;
  long long gen = 0;
  int n = 0, maxmemb = 0, numtree = 0, nleaves = 0, depth = 0, cap = 0;
  // A tree holds nsys independent systems (a forest): system s owns particles
  // [sys_start[s], sys_start[s] + sys_n[s]) and its root is node s.
  int nsys = 1;
  std::vector<int> h_sys_start, h_sys_n, h_sys_maxmemb, h_sys_nterms, h_node_sys;
  std::vector<double> h_sys_leaf_sqr;  // per system: largest leaf sqradius
  DBuf<int> sys_start, sys_n, sys_maxmemb, node_sys;
  // particles in tree order (sorted position e); perm[e] = original index
  DBuf<int> perm, iperm;
  DBuf<double> sx, sy, sz, sq, sw;
  DBuf<double4> src64;   // (x, y, z, q)
  DBuf<float4> src32;    // leaf-centred (x-c, y-c, z-c, q)
  DBuf<int> leaf_of;     // leaf node of each sorted position
  // nodes
  DBuf<int> nummemb, start, children, level, parent;
  DBuf<double> fields;   // 13 per node
  DBuf<double4> nodec;   // (xmid, ymid, zmid, sqradius)
  DBuf<float4> nodeh;    // half extents of the box about the midpoint (rounded up)
  DBuf<int2> kids;       // children: (first index or -1, count | slot order 3 bits each)
  DBuf<int> leaves;
  // host mirror of the node structure
  std::vector<int> h_nummemb, h_start, h_children, h_level, h_perm;
  std::vector<double> h_fields;
  // charges and moments
  bool has_charges = false, has_weights = false;
  int nterms = 0;
  bool has_moments = false;
  bool lists_built = false;  // the last evaluation built its particle-target lists
  DBuf<double> mom64;
  DBuf<float> mom32;
  std::vector<long long> h_mom_off;  // first moment of each node (systems may differ in nterms)
  DBuf<long long> mom_off;
  // the same moments in the far field's shell order, each node's block padded with zeros to
  // a multiple of 4 (16-byte aligned blocks, copied whole into shared memory by TMA)
  DBuf<double> msh64;
  DBuf<float> msh32;
  DBuf<long long> msh_off;
  // moment work plan: (node, first, last) member chunks and per-chunk partial sums
  long long mplan_gen = -1;
  int mplan_nch = 0;
  long long mom_total = 0, msh_total = 0;
  std::vector<int> mplan_cls;  // chunk range of each nterms class
  DBuf<int4> mplan_chunks;
  DBuf<int> mplan_c0, mplan_c1, mplan_T;
  DBuf<double> mplan_part;
  // lists and outputs
  Lists plists;            // particle targets
  EvalPlan pplan;          // plan of the last particle-target evaluation
  DBuf<double> pot_sorted, fx_sorted, fy_sorted, fz_sorted;
  bit_stats stats{};
  cudaEvent_t ev[12] = {};
};

// ---- exact FP64 helpers (no contraction) for the MAC and the tree fields -----------------
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

// FP32 moments are stored normalised: M_v / h^|v| with h = 2^e the smallest power of two
// above the cluster radius (sqrt(sqradius)), so the scaling is exact (exponent shifts) and
// the FP32 far field works with (h/r)^n, which stays bounded at any scale.  Both the
// moment pass and the far kernels call this on the same FP64 sqradius.
__device__ __forceinline__ int mom32_scale_exp(double sqradius) {
  if (!(sqradius > 0.0) || !(sqradius < 1e300)) return 0;
  const int e = ilogb(sqrt(sqradius)) + 1;
  return e < -100 ? -100 : (e > 100 ? 100 : e);
}

// ---- entry points implemented in the .cu files -----------------------------------------
void tree_build(Tree* t, const double* dx, const double* dy, const double* dz);
void tree_sync_host(Tree* t);
void tree_set_charges(Tree* t, const double* dq, const double* dw);
void tree_moments(Tree* t, int nterms);
void tree_moments_sys(Tree* t, const std::vector<int>& nterms_per_system);
// alt (single-system keys only, or nullptr): a second MAC checked during the traversal.
void build_lists(Tree* t, Lists* L, const ListKey& key, int ntargets, const double* tx,
                 const double* ty, const double* tz, const SysEval* d_sys,
                 const ListKey* alt = nullptr);
// Evaluation plan of one call: per-system parameters on the device and the groups of
// each launch class, ordered by class and then by decreasing work.
void eval_far(Tree* t, Lists* L, const EvalPlan& P, const double* tx, const double* ty,
              const double* tz, double* out_sorted);
void eval_near(Tree* t, Lists* L, const EvalPlan& P, const double* tx, const double* ty,
               const double* tz, double* out_sorted);
void eval_far_force(Tree* t, Lists* L, const EvalPlan& P, double* fx, double* fy, double* fz);
// FP64 direct sum at m particle targets tg (device pointers); out[i] for target i.
void direct_potential(Ctx* c, int n, const double* x, const double* y, const double* z,
                      const double* q, const bit_eval_params& p, int m, const int* tg,
                      double* out);
void eval_near_force(Tree* t, Lists* L, const EvalPlan& P, double* fx, double* fy, double* fz);
// Measured FMA throughput of the context's device, flop/s (2 per FMA), FP32 or FP64.
double fma_peak(Ctx* c, bool f32);
void fp64_math_error(Ctx* c, long long n, double* exp_ulps, double* rsqrt_ulps);
void device_wait_check(Ctx* c, int limit);
// FP64 field direct sum at m particle targets tg (device pointers); out = fx | fy | fz.
void direct_field(Ctx* c, int n, const double* x, const double* y, const double* z,
                  const double* q, int regularised, double del, int korder, int m,
                  const int* tg, double* out);

// Per-system parameters of a potential (force = 0) or field evaluation: force = 1 the
// regularised Coulomb field of treeforce (kernel_order: the reference's KERNEL_ORDER),
// force = 2 the screened 2-D field of shielded_treeforce.
SysEval make_sys_eval(const bit_eval_params& p, int nterms, int points, int force,
                      int kernel_order = 0);
// Fill P->h_sys (one entry per system; prm holds one entry for all or one per system) and
// its device copy.
void plan_sys(Tree* t, EvalPlan* P, const std::vector<bit_eval_params>& prm, int points,
              int force, int kernel_order = 0);
// Key of the lists the plan's MAC needs.
ListKey plan_key(const Tree* t, const EvalPlan& P, int points);
// Launch classes and class-ordered groups of P over the lists L.
void plan_classes(Tree* t, Lists* L, EvalPlan* P);
// Particle-target lists and plan of a tree (t->plists, t->pplan) for these parameters.
void prepare_particles(Tree* t, const std::vector<bit_eval_params>& prm, int force,
                       int kernel_order = 0);

inline unsigned grid_for(long long work, int per_block) {
  long long g = (work + per_block - 1) / per_block;
  return (unsigned)(g < 1 ? 1 : g);
}

}  // namespace bit

struct bit_ctx {
  bit::Ctx c;
};
struct bit_tree {
  bit::Tree t;
};

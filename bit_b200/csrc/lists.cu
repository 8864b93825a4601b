// Interaction lists: the MAC traversal of treepotential / shielded_treepot / treeforce
// (src/tree3d.cpp:4679-4778, 3448-3627, 851-971) for a whole group of targets at once.
//
// A group is up to 1024 consecutive targets (a run of consecutive small leaves, a leaf, or
// a chunk of one; for external points, 256 consecutive points in Morton order).  One CTA walks the tree for the group,
// one thread per target, one 32-bit mask word per warp.  At a node every active target
// evaluates the reference's acceptance test in FP64 without contraction
// (sqradius < acc * ((dx*dx + dy*dy + dz*dz + add) - sub)); the node becomes a far entry
// for the accepting targets, and the others descend into the children in the reference's
// children[] order, or get a near entry at a leaf.  Entries carry the group's bitmask.
// Restricted to one target, the entries are exactly its reference traversal, in order.
// In a forest the walk starts at the root of the group's system, with that system's MAC.
//
// Single pass: a persistent kernel whose CTAs take groups from a device counter; each CTA
// stages a group's entries in its own region of global memory, then reserves room in the
// global lists with one atomic per list and copies them out (a group's entries stay
// contiguous and in order; groups land in completion order, addressed by begin/count).
// The lists are written in place, into arrays sized from an estimate, and the staging
// regions are sized from the largest group of the previous build (of this tree, else the
// context's last build under the same MAC; a first build uses an allowance; no region is
// larger than the tree's worst case, every node a far entry and every leaf a near one).
// A group that overflows its staging region, or a reservation that runs past the arrays,
// makes the whole build fall back to a count pass, a prefix sum and a fill pass; so does
// a context whose memory budget has no room for the staging.
//
// Optionally the walk also evaluates a second MAC (another kernel's parameters, e.g. the
// Coulomb test's (r^2 + del) - del next to the screened r^2 - mac_del) at every (target,
// node) it visits.  If no decision differs, that MAC's own walk would take the same path
// and emit the same entries, so the lists serve both MACs bit for bit; one differing
// decision anywhere and they serve only their own.
#include <algorithm>
#include <numeric>
#include <vector>

#include "common.cuh"

namespace bit {

namespace {

constexpr int LT = 1024;          // threads of the list builder (one per target of a group)
constexpr int LSTK = 256;         // traversal stack entries per group
constexpr size_t STACK_BYTES = 32 * LSTK * sizeof(int);  // per-warp node stacks
constexpr long long STAGE_FIRST[2] = {768 * 33, 192 * 33};  // first build: far, near words

enum { MODE_COUNT = 0, MODE_FILL = 1, MODE_STAGE = 2 };

struct ListArgs {
  const int *g_tstart, *g_tcount;
  const double *tx, *ty, *tz;
  const double4* nodec;
  const int2* kids;  // per node: (first child, count | slot order), a leaf (-1, members)
  const SysEval* sys;  // per system: MAC parameters
  const int* g_sys;    // per group: system (its root is node g_sys[g])
  // per group
  long long *far_off, *near_off, *far_moff, *near_moff;
  int *far_cnt, *near_cnt;
  // lists
  int *far_node, *near_node;
  unsigned *far_mask, *near_mask;
  unsigned long long* totals;  // far entries, far words, near entries, near words
  unsigned long long* pairs;   // far pairs, near pairs
  int* err;                    // 1: stack overflow, 2: staging or arena overflow,
                               // 4: the alternative MAC disagreed somewhere
  unsigned long long cap[4];   // MODE_STAGE: room in the four output arrays
  int has_alt;                 // also evaluate a second MAC and compare its decisions
  double alt_acc, alt_add, alt_sub;
  // MODE_STAGE (k_lists_queue): each resident CTA's own staging region in global memory,
  // stage_far + stage_near words (far nodes | far masks, near nodes | near masks), and the
  // work counter over the ngroups groups
  unsigned* gstage;
  long long stage_far, stage_near;
  int* head;
  int ngroups;
};

// The alternative MAC's decision for squared distance s and node sqradius w.
__device__ __forceinline__ bool alt_ok(const ListArgs& a, double s, double w) {
  return w < dmul(a.alt_acc, dsub(dadd(s, a.alt_add), a.alt_sub));
}

// Barrier `id` (1..15) among the first `nthreads` threads of the CTA (a multiple of 32);
// barrier 0 is __syncthreads.
__device__ __forceinline__ void bar_sync_n(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// The walk of group g by the whole CTA.  MODE_COUNT counts the group's entries, MODE_FILL
// writes them at the offsets a scan gave, MODE_STAGE writes them into the CTA's staging
// region and then copies them into room reserved with one atomic per list.
template <int MODE>
__device__ __forceinline__ void walk_group(const ListArgs& a, int g) {
  __shared__ unsigned s_mask[LSTK][32];  // each warp's mask word of every stack entry
  __shared__ unsigned s_am[2][32], s_rm[2][32];  // accept / reject words, by parity
  __shared__ unsigned long long s_base[4];
  __shared__ int s_flags;  // the walk's overflow (1) / full staging (2), for every warp
  __shared__ long long s_n[2];  // the walk's far and near entry counts, for every warp
  extern __shared__ unsigned dyn[];
  // dynamic shared memory: each warp's own copy of the node stack
  int (*s_node)[LSTK] = reinterpret_cast<int (*)[LSTK]>(dyn);
  unsigned* stage = MODE == MODE_STAGE
                        ? a.gstage + (size_t)blockIdx.x * (size_t)(a.stage_far + a.stage_near)
                        : nullptr;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int t0 = a.g_tstart[g], tc = a.g_tcount[g];
  const int W = (tc + 31) >> 5;
  const int i = threadIdx.x;
  const int root = a.g_sys[g];
  const double macc = a.sys[root].acc, madd = a.sys[root].mac_add, msub = a.sys[root].mac_sub;
  // staging layout: far nodes | far masks, near nodes | near masks
  const long long fcap = MODE == MODE_STAGE ? a.stage_far / (W + 1) : 0;
  const long long ncap = MODE == MODE_STAGE ? a.stage_near / (W + 1) : 0;
  int* sf_node = reinterpret_cast<int*>(stage);
  unsigned* sf_mask = stage + fcap;
  int* sn_node = reinterpret_cast<int*>(stage + a.stage_far);
  unsigned* sn_mask = stage + a.stage_far + ncap;
  double x = 0, y = 0, z = 0;
  if (i < tc) { x = a.tx[t0 + i]; y = a.ty[t0 + i]; z = a.tz[t0 + i]; }
  if (lane == 0) {
    s_node[w][0] = root;
    int live = tc - 32 * w;
    s_mask[0][w] = live >= 32 ? 0xffffffffu : (live > 0 ? (1u << live) - 1u : 0u);
  }
  // warps without targets do not walk: their accept / reject words stay 0
  if (threadIdx.x < 64) {
    s_am[threadIdx.x >> 5][lane] = 0u;
    s_rm[threadIdx.x >> 5][lane] = 0u;
  }
  if (threadIdx.x == 0) s_flags = 0;
  int sp = 1;
  long long nf = 0, nn = 0, fpairs = 0, npairs = 0;
  const long long fo = MODE == MODE_FILL ? a.far_off[g] : 0, no = MODE == MODE_FILL ? a.near_off[g] : 0;
  const long long fmo = MODE == MODE_FILL ? a.far_moff[g] : 0, nmo = MODE == MODE_FILL ? a.near_moff[g] : 0;
  bool overflow = false, full = false, differ = false;
  __syncthreads();
  // One barrier per visited node, after every warp has published its accept / reject
  // words.  Every warp pushes the same children onto its own stack (all threads see the
  // same children and the same CTA-wide decision), so no warp waits for another's push;
  // the words alternate between two buffers, so a fast warp never overwrites words a
  // slow one is still reading (it cannot get two barriers ahead of it).  Only the W warps
  // that hold targets walk, on barrier 1 among their 32 W threads: they pop the same
  // entries and take the same number of steps, while the others wait at the barrier after
  // the walk (a group of 650 targets leaves 11 of the 32 warps idle).
  int par = 0;
  while (w < W && sp > 0) {
    sp--;
    const int node = s_node[w][sp];
    const unsigned word = s_mask[sp][w];
    const int2 kd = a.kids[node];  // loads alongside the centre, needed only to descend
    bool ok = false;
    if ((word >> lane) & 1u) {
      const double4 c = a.nodec[node];
      double dx = dsub(x, c.x), dy = dsub(y, c.y), dz = dsub(z, c.z);
      double s = dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz));
      ok = c.w < dmul(macc, dsub(dadd(s, madd), msub));
      if (a.has_alt) differ |= ok != alt_ok(a, s, c.w);
    }
    const unsigned am = __ballot_sync(0xffffffffu, ok) & word;
    const unsigned rm = word & ~am;
    if (lane == 0) { s_am[par][w] = am; s_rm[par][w] = rm; }
    bar_sync_n(1, 32 * W);
    const bool anyA = __ballot_sync(0xffffffffu, s_am[par][lane] != 0u) != 0u;
    const bool anyR = __ballot_sync(0xffffffffu, s_rm[par][lane] != 0u) != 0u;
    par ^= 1;
    if (anyA) {
      if (MODE == MODE_FILL) {
        if (threadIdx.x == 0) a.far_node[fo + nf] = node;
        if (lane == 0 && w < W) a.far_mask[fmo + nf * W + w] = am;
      } else if (MODE == MODE_STAGE) {
        if (nf >= fcap) { full = true; break; }
        if (threadIdx.x == 0) sf_node[nf] = node;
        if (lane == 0 && w < W) sf_mask[nf * W + w] = am;
      }
      nf++;
      if (lane == 0) fpairs += __popc(am);
    }
    if (anyR) {
      if (kd.x < 0) {
        if (MODE == MODE_FILL) {
          if (threadIdx.x == 0) a.near_node[no + nn] = node;
          if (lane == 0 && w < W) a.near_mask[nmo + nn * W + w] = rm;
        } else if (MODE == MODE_STAGE) {
          if (nn >= ncap) { full = true; break; }
          if (threadIdx.x == 0) sn_node[nn] = node;
          if (lane == 0 && w < W) sn_mask[nn * W + w] = rm;
        }
        nn++;
        if (lane == 0) npairs += (long long)__popc(rm) * kd.y;
      } else {
        const int cnt = kd.y & 15;
        if (sp + cnt > LSTK) { overflow = true; break; }
        // children[k] = kd.x + order[k]; the last slot goes deepest, so children[0] pops first
        if (lane == 0)
          for (int k = cnt - 1, q = sp; k >= 0; k--, q++) {
            s_node[w][q] = kd.x + ((kd.y >> (4 + 3 * k)) & 7);
            s_mask[q][w] = rm;
          }
        sp += cnt;
      }
    }
    __syncwarp();  // this warp's pushes, before its next pop
  }
  // the walk's outcome and entry counts for every warp (thread 0's warp walked)
  if (threadIdx.x == 0) {
    if (overflow || full) s_flags = overflow ? 1 : 2;
    s_n[0] = nf;
    s_n[1] = nn;
  }
  __syncthreads();
  overflow = s_flags == 1;
  full = s_flags == 2;
  nf = s_n[0];
  nn = s_n[1];
  if (threadIdx.x == 0 && (overflow || full)) atomicOr(a.err, overflow ? 1 : 2);
  if (a.has_alt && __any_sync(0xffffffffu, differ) && lane == 0) atomicOr(a.err, 4);
  if (MODE != MODE_FILL && lane == 0 && (fpairs || npairs)) {
    atomicAdd(&a.pairs[0], (unsigned long long)fpairs);
    atomicAdd(&a.pairs[1], (unsigned long long)npairs);
  }
  if (MODE == MODE_COUNT && threadIdx.x == 0) {
    a.far_cnt[g] = (int)nf;
    a.near_cnt[g] = (int)nn;
  }
  if (MODE != MODE_STAGE || overflow || full) return;
  __syncthreads();
  if (threadIdx.x == 0) {
    s_base[0] = atomicAdd(&a.totals[0], (unsigned long long)nf);
    s_base[1] = atomicAdd(&a.totals[1], (unsigned long long)(nf * W));
    s_base[2] = atomicAdd(&a.totals[2], (unsigned long long)nn);
    s_base[3] = atomicAdd(&a.totals[3], (unsigned long long)(nn * W));
    // the arrays were sized from an estimate: past their end, the build falls back
    if (s_base[0] + nf > a.cap[0] || s_base[1] + nf * W > a.cap[1] ||
        s_base[2] + nn > a.cap[2] || s_base[3] + nn * W > a.cap[3]) {
      atomicOr(a.err, 2);
      s_base[0] = ~0ull;
    }
    a.far_off[g] = (long long)s_base[0];
    a.far_moff[g] = (long long)s_base[1];
    a.near_off[g] = (long long)s_base[2];
    a.near_moff[g] = (long long)s_base[3];
    a.far_cnt[g] = (int)nf;
    a.near_cnt[g] = (int)nn;
  }
  __syncthreads();
  if (s_base[0] == ~0ull) return;
  for (int k = threadIdx.x; k < nf; k += LT) a.far_node[s_base[0] + k] = sf_node[k];
  for (int k = threadIdx.x; k < nf * W; k += LT) a.far_mask[s_base[1] + k] = sf_mask[k];
  for (int k = threadIdx.x; k < nn; k += LT) a.near_node[s_base[2] + k] = sn_node[k];
  for (int k = threadIdx.x; k < nn * W; k += LT) a.near_mask[s_base[3] + k] = sn_mask[k];
}

// Count / fill passes: CTA b walks group b.
template <int MODE>
__global__ void __launch_bounds__(LT) k_lists(ListArgs a) {
  walk_group<MODE>(a, blockIdx.x);
}

// The single-pass build: a persistent kernel whose CTAs take groups from a device counter
// and stage each group's entries in their own global-memory region, so that a group is
// walked once.  No CTA waits for another; the counter is the only shared state.
__global__ void __launch_bounds__(LT) k_lists_queue(ListArgs a) {
  __shared__ int s_item;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(a.head, 1);
    __syncthreads();
    const int g = s_item;
    __syncthreads();  // every thread has read s_item before it is overwritten
    if (g >= a.ngroups) return;
    walk_group<MODE_STAGE>(a, g);
    __syncthreads();  // the group's copy-out reads precede the next group's staging writes
  }
}

// Exclusive scan of int counts times a per-group factor (one block); the total goes to
// *total.  tcount == nullptr: factor 1, else (tcount+31)/32 mask words per entry.
__global__ void k_scan_cnt(const int* in, const int* tcount, long long* out, int n,
                           unsigned long long* total) {
  __shared__ long long ws[32];
  __shared__ long long carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int base = 0; base < n; base += blockDim.x) {
    int i = base + threadIdx.x;
    long long v = i < n ? (long long)in[i] * (tcount ? (long long)((tcount[i] + 31) >> 5) : 1LL) : 0;
    long long s = v;
    for (int o = 1; o < 32; o <<= 1) {
      long long t = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += t;
    }
    if (lane == 31) ws[w] = s;
    __syncthreads();
    if (w == 0) {
      long long t = lane < nw ? ws[lane] : 0;
      for (int o = 1; o < 32; o <<= 1) {
        long long u = __shfl_up_sync(0xffffffffu, t, o);
        if (lane >= o) t += u;
      }
      if (lane < nw) ws[lane] = t;
    }
    __syncthreads();
    long long pre = carry + (w ? ws[w - 1] : 0) + s - v;
    if (i < n) out[i] = pre;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = pre + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = (unsigned long long)carry;
}

void set_stage_attr() {
  // static + dynamic shared memory is above the 48 KB default
  ensure_smem_attr(reinterpret_cast<const void*>(k_lists_queue), (int)STACK_BYTES);
  ensure_smem_attr(reinterpret_cast<const void*>(k_lists<MODE_COUNT>), (int)STACK_BYTES);
  ensure_smem_attr(reinterpret_cast<const void*>(k_lists<MODE_FILL>), (int)STACK_BYTES);
}

}  // namespace

// Groups for particle targets.  G = 0: each leaf, in chunks of at most kGroupMax targets.
// G > 0: runs of consecutive leaves (in tree order, which keeps them spatially close:
// siblings and cousins) of one system, up to G targets together; a leaf larger than G is
// cut into chunks of G.  Packed small leaves share one traversal, one set of entries and
// the near field's source tiles, but each near entry then covers fewer targets; which is
// faster depends on the workload (bit_b200.autotune measures it).
static void particle_groups(Tree* t, int G, std::vector<int>& ts, std::vector<int>& tc,
                            std::vector<int>& sys) {
  if (G <= 0) {
    for (int i = 0; i < t->numtree; i++) {
      if (t->h_children[8LL * i] != -1) continue;
      const int st = t->h_start[i], en = st + t->h_nummemb[i];
      for (int e = st; e < en; e += kGroupMax) {
        ts.push_back(e);
        tc.push_back(std::min(kGroupMax, en - e));
        sys.push_back(t->h_node_sys[i]);
      }
    }
    return;
  }
  std::vector<int> leaves;
  for (int i = 0; i < t->numtree; i++)
    if (t->h_children[8LL * i] == -1) leaves.push_back(i);
  std::sort(leaves.begin(), leaves.end(),
            [&](int a, int b) { return t->h_start[a] < t->h_start[b]; });
  int cur0 = -1, curn = 0, cursys = -1;
  auto flush = [&] {
    if (curn > 0) {
      ts.push_back(cur0);
      tc.push_back(curn);
      sys.push_back(cursys);
    }
    curn = 0;
  };
  for (int i : leaves) {
    const int st = t->h_start[i], cnt = t->h_nummemb[i], sy = t->h_node_sys[i];
    if (cnt > G) {
      flush();
      for (int e = st; e < st + cnt; e += G) {
        ts.push_back(e);
        tc.push_back(std::min(G, st + cnt - e));
        sys.push_back(sy);
      }
      continue;
    }
    if (curn > 0 && (sy != cursys || curn + cnt > G || cur0 + curn != st)) flush();
    if (curn == 0) {
      cur0 = st;
      cursys = sy;
    }
    curn += cnt;
  }
  flush();
}

void build_lists(Tree* t, Lists* L, const ListKey& key, int ntargets, const double* tx,
                 const double* ty, const double* tz, const SysEval* d_sys, const ListKey* alt) {
  if (alt && (!alt->sysmac.empty() || !key.sysmac.empty() || t->nsys != 1)) alt = nullptr;
  L->valid = false;  // the arrays are rewritten below; valid again once the build completes
  L->alt_valid = false;
  Ctx* c = t->ctx;
  cudaStream_t s = c->stream;
  std::vector<int> ts, tc, gsys;
  if (key.points) {
    if (t->nsys != 1) fail(BIT_ERR_INVALID_ARGUMENT, "external points need a single-system tree");
    for (int e = 0; e < ntargets; e += kPointGroup) {
      ts.push_back(e);
      tc.push_back(std::min(kPointGroup, ntargets - e));
      gsys.push_back(0);
    }
  } else {
    particle_groups(t, key.group, ts, tc, gsys);
  }
  const int ng = (int)ts.size();
  L->ngroups = ng;
  L->ntargets = ntargets;
  L->g_tstart.ensure(c, ng);
  L->g_tcount.ensure(c, ng);
  BIT_CUDA(cudaMemcpyAsync(L->g_tstart.p, ts.data(), ng * sizeof(int), cudaMemcpyHostToDevice, s));
  BIT_CUDA(cudaMemcpyAsync(L->g_tcount.p, tc.data(), ng * sizeof(int), cudaMemcpyHostToDevice, s));
  L->g_sys.ensure(c, ng);
  BIT_CUDA(cudaMemcpyAsync(L->g_sys.p, gsys.data(), ng * sizeof(int), cudaMemcpyHostToDevice, s));
  L->h_g_sys = gsys;
  L->far_off.ensure(c, ng);
  L->near_off.ensure(c, ng);
  L->far_moff.ensure(c, ng);
  L->near_moff.ensure(c, ng);
  L->far_cnt.ensure(c, ng);
  L->near_cnt.ensure(c, ng);
  DBuf<unsigned long long> cnt;  // totals[4], pairs[2], err (as the 7th word)
  cnt.ensure(c, 8);
  BIT_CUDA(cudaMemsetAsync(cnt.p, 0, 8 * sizeof(unsigned long long), s));
  ListArgs a{};
  a.g_tstart = L->g_tstart.p;
  a.g_tcount = L->g_tcount.p;
  a.tx = tx; a.ty = ty; a.tz = tz;
  a.nodec = t->nodec.p;
  a.kids = t->kids.p;
  a.sys = d_sys;
  a.g_sys = L->g_sys.p;
  a.far_off = L->far_off.p; a.near_off = L->near_off.p;
  a.far_moff = L->far_moff.p; a.near_moff = L->near_moff.p;
  a.far_cnt = L->far_cnt.p; a.near_cnt = L->near_cnt.p;
  a.totals = cnt.p;
  a.pairs = cnt.p + 4;
  a.err = reinterpret_cast<int*>(cnt.p + 6);
  if (alt) {
    a.has_alt = 1;
    a.alt_acc = alt->acc;
    a.alt_add = alt->add_del;
    a.alt_sub = alt->sub_del;
  }
  // Single pass straight into the lists, sized from an estimate: the last build's totals
  // scaled by the group count, else a per-group allowance.  A group that does not fit
  // its staging area or the arrays makes the build fall back to count, scan and fill.
  long long words = 0;
  for (int g = 0; g < ng; g++) words += (tc[g] + 31) / 32;
  // sizes of this tree's last build, else of the context's last build under the same MAC
  const ListSizing* hint = L->last.ngroups > 0 ? &L->last : nullptr;
  if (!hint && c->list_hint.ngroups > 0 && c->list_hint.acc == key.acc &&
      c->list_hint.points == key.points)
    hint = &c->list_hint;
  unsigned long long cap[4];
  if (hint) {
    const double f = 1.25 * (double)ng / hint->ngroups;
    for (int k = 0; k < 4; k++) cap[k] = (unsigned long long)(f * hint->totals[k]) + 1024;
  } else {
    cap[0] = 192ull * ng + 1024;
    cap[1] = 192ull * words + 1024;
    cap[2] = 48ull * ng + 1024;
    cap[3] = 48ull * words + 1024;
  }
  L->far_node.ensure(c, cap[0]);
  L->far_mask.ensure(c, cap[1]);
  L->near_node.ensure(c, cap[2]);
  L->near_mask.ensure(c, cap[3]);
  for (int k = 0; k < 4; k++) a.cap[k] = cap[k];
  a.far_node = L->far_node.p; a.far_mask = L->far_mask.p;
  a.near_node = L->near_node.p; a.near_mask = L->near_mask.p;
  set_stage_attr();
  // staging: one region per resident CTA.  A group's entries number at most the tree's
  // nodes (far) and leaves (near), each with at most 32 mask words.
  int maxw = 1;
  for (int g = 0; g < ng; g++) maxw = std::max(maxw, (tc[g] + 31) / 32);
  int per_sm = 0;
  BIT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_lists_queue, LT, STACK_BYTES));
  const int slots = std::max(1, std::min(ng, c->num_sms * std::max(per_sm, 1)));
  const long long worst[2] = {(maxw + 1LL) * std::max(t->numtree, 1),
                              (maxw + 1LL) * std::max(t->nleaves, 1)};
  long long want[2];
  for (int k = 0; k < 2; k++)
    want[k] = std::min(worst[k], hint && hint->stage[k] > 0
                                     ? hint->stage[k] + hint->stage[k] / 4 + 64
                                     : STAGE_FIRST[k]);
  a.stage_far = want[0];
  a.stage_near = want[1];
  const size_t stage_words = (size_t)slots * (size_t)(want[0] + want[1]);
  const bool staged = L->gstage.n >= stage_words ||
                      !c->budget || c->in_use + stage_words * sizeof(unsigned) <= c->budget;
  unsigned long long h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  std::vector<int> hf(ng), hn(ng);
  int err = 2;  // no single pass: straight to count, scan and fill
  if (staged) {
    L->gstage.ensure(c, stage_words);
    L->head.ensure(c, 1);
    BIT_CUDA(cudaMemsetAsync(L->head.p, 0, sizeof(int), s));
    a.gstage = L->gstage.p;
    a.head = L->head.p;
    a.ngroups = ng;
    count_launch(), k_lists_queue<<<slots, LT, STACK_BYTES, s>>>(a);
    BIT_CHECK_LAUNCH();
    BIT_CUDA(cudaMemcpyAsync(h, cnt.p, 8 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    BIT_CUDA(cudaMemcpyAsync(hf.data(), L->far_cnt.p, ng * sizeof(int), cudaMemcpyDeviceToHost, s));
    BIT_CUDA(cudaMemcpyAsync(hn.data(), L->near_cnt.p, ng * sizeof(int), cudaMemcpyDeviceToHost, s));
    BIT_CUDA(cudaStreamSynchronize(s));
    err = (int)(h[6] & 0xffffffffu);
    if (err & 1) fail(BIT_ERR_CAPACITY, "traversal stack capacity exceeded (tree deeper than supported)");
  }
  L->fallback = (err & 2) != 0;
  if (err & 2) {
    // some group's lists exceed the staging area or the arrays: count, scan, fill
    BIT_CUDA(cudaMemsetAsync(cnt.p, 0, 8 * sizeof(unsigned long long), s));
    count_launch(), k_lists<MODE_COUNT><<<ng, LT, STACK_BYTES, s>>>(a);
    count_launch(), k_scan_cnt<<<1, 1024, 0, s>>>(L->far_cnt.p, nullptr, L->far_off.p, ng, cnt.p + 0);
    count_launch(), k_scan_cnt<<<1, 1024, 0, s>>>(L->far_cnt.p, L->g_tcount.p, L->far_moff.p, ng, cnt.p + 1);
    count_launch(), k_scan_cnt<<<1, 1024, 0, s>>>(L->near_cnt.p, nullptr, L->near_off.p, ng, cnt.p + 2);
    count_launch(), k_scan_cnt<<<1, 1024, 0, s>>>(L->near_cnt.p, L->g_tcount.p, L->near_moff.p, ng, cnt.p + 3);
    BIT_CUDA(cudaMemcpyAsync(h, cnt.p, 8 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    BIT_CUDA(cudaMemcpyAsync(hf.data(), L->far_cnt.p, ng * sizeof(int), cudaMemcpyDeviceToHost, s));
    BIT_CUDA(cudaMemcpyAsync(hn.data(), L->near_cnt.p, ng * sizeof(int), cudaMemcpyDeviceToHost, s));
    BIT_CUDA(cudaStreamSynchronize(s));
    err = (int)(h[6] & 0xffffffffu);  // this pass walked every group to the end
    if (err & 1) fail(BIT_ERR_CAPACITY, "traversal stack capacity exceeded");
    L->far_node.ensure(c, h[0]);
    L->far_mask.ensure(c, h[1]);
    L->near_node.ensure(c, h[2]);
    L->near_mask.ensure(c, h[3]);
    a.far_node = L->far_node.p; a.far_mask = L->far_mask.p;
    a.near_node = L->near_node.p; a.near_mask = L->near_mask.p;
    count_launch(), k_lists<MODE_FILL><<<ng, LT, STACK_BYTES, s>>>(a);
    BIT_CHECK_LAUNCH();
  }
  ListSizing& z = L->last;
  z.ngroups = ng;
  z.acc = key.acc;
  z.points = key.points;
  for (int k = 0; k < 4; k++) z.totals[k] = h[k];
  z.stage[0] = z.stage[1] = 0;
  for (int g = 0; g < ng; g++) {
    const long long w1 = (tc[g] + 31) / 32 + 1;
    z.stage[0] = std::max(z.stage[0], w1 * hf[g]);
    z.stage[1] = std::max(z.stage[1], w1 * hn[g]);
  }
  c->list_hint = z;
  L->nfar = (long long)h[0];
  L->nnear = (long long)h[2];
  L->far_pairs = (long long)h[4];
  L->near_pairs = (long long)h[5];
  // heaviest groups first, so the evaluation kernels' tail is short
  std::vector<int> ord(ng);
  std::iota(ord.begin(), ord.end(), 0);
  std::vector<long long> wk(ng);
  for (int g = 0; g < ng; g++) wk[g] = (40LL * hf[g] + hn[g]) * (long long)tc[g];
  std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return wk[x] > wk[y]; });
  L->h_work = wk;
  L->order.ensure(c, ng);
  BIT_CUDA(cudaMemcpyAsync(L->order.p, ord.data(), ng * sizeof(int), cudaMemcpyHostToDevice, s));
  BIT_CUDA(cudaStreamSynchronize(s));
  L->key = key;
  L->valid = true;
  L->version++;
  L->alt_valid = alt && !(err & 4);
  if (L->alt_valid) {
    L->alt_key = key;
    L->alt_key.acc = alt->acc;
    L->alt_key.add_del = alt->add_del;
    L->alt_key.sub_del = alt->sub_del;
  }
}

}  // namespace bit

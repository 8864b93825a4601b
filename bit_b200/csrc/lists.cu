// Interaction lists: the MAC traversal of treepotential / shielded_treepot / treeforce
// (src/tree3d.cpp:4679-4778, 3448-3627, 851-971) for a whole group of targets at once.
//
// A group is up to 1024 consecutive targets (a leaf, or a chunk of one; for external
// points, 256 consecutive points in Morton order).  One CTA walks the tree for the group,
// one thread per target, 32 mask words per node (one per warp).  At a node every active
// target evaluates the reference's acceptance test in FP64 without contraction
// (sqradius < acc * ((dx*dx + dy*dy + dz*dz + add) - sub)); the node becomes a far entry
// for the accepting targets, and the others descend into the children in the reference's
// children[] order, or get a near entry at a leaf.  Entries carry the group's bitmask.
// Restricted to one target, the entries are exactly its reference traversal, in order.
//
// Two launches: one counts entries and mask words per group, the second writes them at
// the prefix-summed offsets.
#include <algorithm>
#include <numeric>
#include <vector>

#include "common.cuh"

namespace bit {

namespace {

constexpr int LT = 1024;   // threads of the list builder (one per target of a group)
constexpr int LSTK = 256;  // traversal stack entries per group

template <bool FILL>
__global__ void __launch_bounds__(LT)
    k_lists(const int* g_tstart, const int* g_tcount, const double* tx, const double* ty,
            const double* tz, const double4* nodec, const int* children, const int* nummemb,
            double acc, double add, double sub, long long* far_cnt, long long* near_cnt,
            long long* pair_cnt, const long long* far_off, const long long* near_off,
            const long long* far_moff, const long long* near_moff, int* far_node,
            unsigned* far_mask, int* near_node, unsigned* near_mask, int* err) {
  __shared__ int s_node[LSTK];
  __shared__ unsigned s_mask[LSTK][32];
  const int g = blockIdx.x;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int t0 = g_tstart[g], tc = g_tcount[g];
  const int W = (tc + 31) >> 5;
  const int i = threadIdx.x;
  double x = 0, y = 0, z = 0;
  if (i < tc) { x = tx[t0 + i]; y = ty[t0 + i]; z = tz[t0 + i]; }
  if (threadIdx.x == 0) s_node[0] = 0;
  if (lane == 0) {
    int live = tc - 32 * w;
    s_mask[0][w] = live >= 32 ? 0xffffffffu : (live > 0 ? (1u << live) - 1u : 0u);
  }
  int sp = 1;
  long long nf = 0, nn = 0, fpairs = 0, npairs = 0;
  const long long fo = FILL ? far_off[g] : 0, no = FILL ? near_off[g] : 0;
  const long long fmo = FILL ? far_moff[g] : 0, nmo = FILL ? near_moff[g] : 0;
  bool overflow = false;
  __syncthreads();
  while (sp > 0) {
    sp--;
    const int node = s_node[sp];
    const unsigned word = s_mask[sp][w];
    __syncthreads();  // the popped slot may be overwritten below
    bool ok = false;
    if ((word >> lane) & 1u) {
      const double4 c = nodec[node];
      double dx = dsub(x, c.x), dy = dsub(y, c.y), dz = dsub(z, c.z);
      double s = dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz));
      ok = c.w < dmul(acc, dsub(dadd(s, add), sub));
    }
    const unsigned am = __ballot_sync(0xffffffffu, ok) & word;
    const unsigned rm = word & ~am;
    const int anyA = __syncthreads_or(lane == 0 && am != 0u);
    const int anyR = __syncthreads_or(lane == 0 && rm != 0u);
    if (anyA) {
      if (FILL) {
        if (threadIdx.x == 0) far_node[fo + nf] = node;
        if (lane == 0 && w < W) far_mask[fmo + nf * W + w] = am;
      }
      nf++;
      if (lane == 0) fpairs += __popc(am);
    }
    if (anyR) {
      const int* ch = children + 8LL * node;
      if (ch[0] == -1) {
        if (FILL) {
          if (threadIdx.x == 0) near_node[no + nn] = node;
          if (lane == 0 && w < W) near_mask[nmo + nn * W + w] = rm;
        }
        nn++;
        if (lane == 0) npairs += (long long)__popc(rm) * nummemb[node];
      } else {
        int cnt = 0;
        for (int k = 0; k < 8; k++) cnt += ch[k] != -1;
        if (sp + cnt > LSTK) { overflow = true; break; }
        int q = sp;
        for (int k = 7; k >= 0; k--) {
          if (ch[k] == -1) continue;
          if (threadIdx.x == 0) s_node[q] = ch[k];
          if (lane == 0) s_mask[q][w] = rm;
          q++;
        }
        sp += cnt;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (overflow) atomicOr(err, 1);
    if (!FILL) {
      far_cnt[g] = nf;
      near_cnt[g] = nn;
    }
  }
  if (!FILL && lane == 0 && (fpairs || npairs)) {
    atomicAdd((unsigned long long*)&pair_cnt[0], (unsigned long long)fpairs);
    atomicAdd((unsigned long long*)&pair_cnt[1], (unsigned long long)npairs);
  }
}

// Exclusive scan of long long counts times a per-element factor (one block), total in
// out[n].  factor == nullptr: factor 1.
__global__ void k_scan_ll(const long long* in, const int* tcount, long long* out, int n) {
  __shared__ long long ws[32];
  __shared__ long long carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int base = 0; base < n; base += blockDim.x) {
    int i = base + threadIdx.x;
    long long v = i < n ? in[i] * (tcount ? (long long)((tcount[i] + 31) >> 5) : 1LL) : 0;
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
  if (threadIdx.x == 0) out[n] = carry;
}

}  // namespace

// Groups for particle targets: each leaf, in chunks of at most kGroupMax members.
static void particle_groups(Tree* t, std::vector<int>& ts, std::vector<int>& tc,
                            std::vector<int>& own) {
  for (int i = 0; i < t->numtree; i++) {
    if (t->h_children[8LL * i] != -1) continue;
    int st = t->h_start[i], en = st + t->h_nummemb[i];
    for (int e = st; e < en; e += kGroupMax) {
      ts.push_back(e);
      tc.push_back(std::min(kGroupMax, en - e));
      own.push_back(i);
    }
  }
}

void build_lists(Tree* t, Lists* L, const ListKey& key, int ntargets, const double* tx,
                 const double* ty, const double* tz, const int* /*unused*/) {
  Ctx* c = t->ctx;
  cudaStream_t s = c->stream;
  std::vector<int> ts, tc, own;
  if (key.points) {
    for (int e = 0; e < ntargets; e += kPointGroup) {
      ts.push_back(e);
      tc.push_back(std::min(kPointGroup, ntargets - e));
      own.push_back(-1);
    }
  } else {
    particle_groups(t, ts, tc, own);
  }
  const int ng = (int)ts.size();
  L->ngroups = ng;
  L->g_tstart.ensure(c, ng);
  L->g_tcount.ensure(c, ng);
  L->g_own.ensure(c, ng);
  BIT_CUDA(cudaMemcpyAsync(L->g_tstart.p, ts.data(), ng * sizeof(int), cudaMemcpyHostToDevice, s));
  BIT_CUDA(cudaMemcpyAsync(L->g_tcount.p, tc.data(), ng * sizeof(int), cudaMemcpyHostToDevice, s));
  BIT_CUDA(cudaMemcpyAsync(L->g_own.p, own.data(), ng * sizeof(int), cudaMemcpyHostToDevice, s));
  DBuf<long long> fcnt, ncnt, pairs;
  DBuf<int> err;
  fcnt.ensure(c, ng);
  ncnt.ensure(c, ng);
  pairs.ensure(c, 2);
  err.ensure(c, 1);
  L->far_off.ensure(c, ng + 1);
  L->near_off.ensure(c, ng + 1);
  L->far_moff.ensure(c, ng + 1);
  L->near_moff.ensure(c, ng + 1);
  BIT_CUDA(cudaMemsetAsync(pairs.p, 0, 2 * sizeof(long long), s));
  BIT_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), s));
  count_launch(), k_lists<false><<<ng, LT, 0, s>>>(
      L->g_tstart.p, L->g_tcount.p, tx, ty, tz, t->nodec.p, t->children.p, t->nummemb.p,
      key.acc, key.add_del, key.sub_del, fcnt.p, ncnt.p, pairs.p, nullptr, nullptr, nullptr,
      nullptr, nullptr, nullptr, nullptr, nullptr, err.p);
  count_launch(), k_scan_ll<<<1, 1024, 0, s>>>(fcnt.p, nullptr, L->far_off.p, ng);
  count_launch(), k_scan_ll<<<1, 1024, 0, s>>>(ncnt.p, nullptr, L->near_off.p, ng);
  count_launch(), k_scan_ll<<<1, 1024, 0, s>>>(fcnt.p, L->g_tcount.p, L->far_moff.p, ng);
  count_launch(), k_scan_ll<<<1, 1024, 0, s>>>(ncnt.p, L->g_tcount.p, L->near_moff.p, ng);
  std::vector<long long> hf(ng), hn(ng);
  long long* hp = c->h_pinned;
  BIT_CUDA(cudaMemcpyAsync(hp, L->far_off.p + ng, sizeof(long long), cudaMemcpyDeviceToHost, s));
  BIT_CUDA(cudaMemcpyAsync(hp + 1, L->near_off.p + ng, sizeof(long long), cudaMemcpyDeviceToHost, s));
  BIT_CUDA(cudaMemcpyAsync(hp + 2, pairs.p, 2 * sizeof(long long), cudaMemcpyDeviceToHost, s));
  BIT_CUDA(cudaMemcpyAsync(hp + 4, err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  BIT_CUDA(cudaMemcpyAsync(hp + 5, L->far_moff.p + ng, sizeof(long long), cudaMemcpyDeviceToHost, s));
  BIT_CUDA(cudaMemcpyAsync(hp + 6, L->near_moff.p + ng, sizeof(long long), cudaMemcpyDeviceToHost, s));
  BIT_CUDA(cudaMemcpyAsync(hf.data(), fcnt.p, ng * sizeof(long long), cudaMemcpyDeviceToHost, s));
  BIT_CUDA(cudaMemcpyAsync(hn.data(), ncnt.p, ng * sizeof(long long), cudaMemcpyDeviceToHost, s));
  BIT_CUDA(cudaStreamSynchronize(s));
  if (*reinterpret_cast<int*>(hp + 4))
    fail(BIT_ERR_CAPACITY, "traversal stack capacity exceeded (tree deeper than supported)");
  L->nfar = hp[0];
  L->nnear = hp[1];
  L->far_pairs = hp[2];
  L->near_pairs = hp[3];
  L->far_node.ensure(c, L->nfar);
  L->near_node.ensure(c, L->nnear);
  L->far_mask.ensure(c, hp[5]);
  L->near_mask.ensure(c, hp[6]);
  count_launch(), k_lists<true><<<ng, LT, 0, s>>>(
      L->g_tstart.p, L->g_tcount.p, tx, ty, tz, t->nodec.p, t->children.p, t->nummemb.p,
      key.acc, key.add_del, key.sub_del, nullptr, nullptr, nullptr, L->far_off.p,
      L->near_off.p, L->far_moff.p, L->near_moff.p, L->far_node.p, L->far_mask.p,
      L->near_node.p, L->near_mask.p, err.p);
  BIT_CHECK_LAUNCH();
  // heaviest groups first, so the evaluation kernels' tail is short
  std::vector<int> ord(ng);
  std::iota(ord.begin(), ord.end(), 0);
  std::vector<long long> wk(ng);
  for (int g = 0; g < ng; g++) wk[g] = (40 * hf[g] + hn[g]) * (long long)tc[g];
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return wk[a] > wk[b]; });
  L->order.ensure(c, ng);
  BIT_CUDA(cudaMemcpyAsync(L->order.p, ord.data(), ng * sizeof(int), cudaMemcpyHostToDevice, s));
  BIT_CUDA(cudaStreamSynchronize(s));
  L->key = key;
  L->valid = true;
}

}  // namespace bit

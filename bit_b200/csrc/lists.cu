// Interaction lists: the MAC traversal of treepotential / shielded_treepot / treeforce
// (src/tree3d.cpp:4679-4778, 3448-3627, 851-971) for batches of 32 targets.
//
// One warp walks the tree for one batch, one target per lane.  At a node every lane
// still inside evaluates the reference's acceptance test in FP64 without contraction
// (sqradius < acc * ((dx*dx + dy*dy + dz*dz + add) - sub)); lanes that accept get a far
// entry (node, lane mask); the rest descend into the children in the reference's
// children[] order, or get a near entry if the node is a leaf.  Restricted to one lane,
// the entries are exactly that target's reference traversal, in the same order.
//
// Two launches: the first counts entries per batch, the second writes them at the
// prefix-summed offsets.
#include <algorithm>
#include <vector>

#include "common.cuh"

namespace bit {

namespace {

constexpr int LWARPS = 4;  // warps per block

template <bool FILL>
__global__ void __launch_bounds__(32 * LWARPS)
    k_lists(int nbatch, const int* b_tstart, const int* b_tcount, const double* tx,
            const double* ty, const double* tz, const double4* nodec, const int* children,
            const int* nummemb, double acc, double add, double sub, long long* far_cnt,
            long long* near_cnt, long long* pair_cnt, const long long* far_off,
            const long long* near_off, int2* far_ent, int2* near_ent, int* err) {
  __shared__ int2 stk[LWARPS][kStackCap];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int b = blockIdx.x * LWARPS + w;
  if (b >= nbatch) return;
  const int t0 = b_tstart[b], tc = b_tcount[b];
  const bool live = lane < tc;
  double x = 0, y = 0, z = 0;
  if (live) { x = tx[t0 + lane]; y = ty[t0 + lane]; z = tz[t0 + lane]; }
  const unsigned full = tc >= 32 ? 0xffffffffu : ((1u << tc) - 1u);
  int2* S = stk[w];
  int sp = 0;
  if (lane == 0) S[0] = make_int2(0, (int)full);
  sp = 1;
  long long nf = 0, nn = 0, fpairs = 0, npairs = 0;
  long long fo = FILL ? far_off[b] : 0, no = FILL ? near_off[b] : 0;
  bool overflow = false;
  __syncwarp();
  while (sp > 0) {
    const int2 top = S[sp - 1];
    sp--;
    __syncwarp();
    const int node = top.x;
    const unsigned mask = (unsigned)top.y;
    const double4 c = nodec[node];
    bool ok = false;
    if ((mask >> lane) & 1u) {
      double dx = dsub(x, c.x), dy = dsub(y, c.y), dz = dsub(z, c.z);
      double s = dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz));
      double rs = dadd(s, add);
      ok = c.w < dmul(acc, dsub(rs, sub));
    }
    const unsigned am = __ballot_sync(0xffffffffu, ok) & mask;
    if (am) {
      if (FILL && lane == 0) far_ent[fo + nf] = make_int2(node, (int)am);
      nf++;
      fpairs += __popc(am);
    }
    const unsigned rem = mask & ~am;
    if (rem) {
      const int* ch = children + 8LL * node;
      if (ch[0] == -1) {
        if (FILL && lane == 0) near_ent[no + nn] = make_int2(node, (int)rem);
        nn++;
        npairs += (long long)__popc(rem) * nummemb[node];
      } else {
        int cnt = 0;
        for (int k = 0; k < 8; k++) cnt += ch[k] != -1;
        if (sp + cnt > kStackCap) { overflow = true; break; }
        if (lane == 0) {
          int q = sp;
          for (int k = 7; k >= 0; k--)
            if (ch[k] != -1) S[q++] = make_int2(ch[k], (int)rem);
        }
        sp += cnt;
        __syncwarp();
      }
    }
  }
  if (lane == 0) {
    if (overflow) atomicOr(err, 1);
    if (!FILL) {
      far_cnt[b] = nf;
      near_cnt[b] = nn;
      atomicAdd((unsigned long long*)&pair_cnt[0], (unsigned long long)fpairs);
      atomicAdd((unsigned long long*)&pair_cnt[1], (unsigned long long)npairs);
    }
  }
}

// Exclusive scan of long long counts (one block, serial over tiles), total in out[n].
__global__ void k_scan_ll(const long long* in, long long* out, int n) {
  __shared__ long long ws[32];
  __shared__ long long carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int base = 0; base < n; base += blockDim.x) {
    int i = base + threadIdx.x;
    long long v = i < n ? in[i] : 0;
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

// Batches for particle targets: consecutive runs of <= 32 members of one leaf.
static void particle_batches(Tree* t, Lists* L) {
  std::vector<int> ts, tc, sl;
  for (int i = 0; i < t->numtree; i++) {
    if (t->h_children[8LL * i] != -1) continue;
    int st = t->h_start[i], en = st + t->h_nummemb[i];
    for (int e = st; e < en; e += kBatch) {
      ts.push_back(e);
      tc.push_back(std::min(kBatch, en - e));
      sl.push_back(i);
    }
  }
  Ctx* c = t->ctx;
  L->nbatch = (int)ts.size();
  L->b_tstart.ensure(c, ts.size());
  L->b_tcount.ensure(c, ts.size());
  L->b_srcleaf.ensure(c, ts.size());
  BIT_CUDA(cudaMemcpyAsync(L->b_tstart.p, ts.data(), ts.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  BIT_CUDA(cudaMemcpyAsync(L->b_tcount.p, tc.data(), tc.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  BIT_CUDA(cudaMemcpyAsync(L->b_srcleaf.p, sl.data(), sl.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
}

// Batches for m external points already in their evaluation order.
static void point_batches(Tree* t, Lists* L, int m) {
  std::vector<int> ts, tc, sl;
  for (int e = 0; e < m; e += kBatch) {
    ts.push_back(e);
    tc.push_back(std::min(kBatch, m - e));
    sl.push_back(-1);
  }
  Ctx* c = t->ctx;
  L->nbatch = (int)ts.size();
  L->b_tstart.ensure(c, ts.size());
  L->b_tcount.ensure(c, ts.size());
  L->b_srcleaf.ensure(c, ts.size());
  BIT_CUDA(cudaMemcpyAsync(L->b_tstart.p, ts.data(), ts.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  BIT_CUDA(cudaMemcpyAsync(L->b_tcount.p, tc.data(), tc.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  BIT_CUDA(cudaMemcpyAsync(L->b_srcleaf.p, sl.data(), sl.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
}

void build_lists(Tree* t, Lists* L, const ListKey& key, int ntargets, const double* tx,
                 const double* ty, const double* tz, const int* /*t_leaf*/) {
  Ctx* c = t->ctx;
  cudaStream_t s = c->stream;
  if (key.points) point_batches(t, L, ntargets);
  else particle_batches(t, L);
  const int nb = L->nbatch;
  DBuf<long long> fcnt, ncnt, pairs;
  DBuf<int> err;
  fcnt.ensure(c, nb);
  ncnt.ensure(c, nb);
  pairs.ensure(c, 2);
  err.ensure(c, 1);
  L->far_off.ensure(c, nb + 1);
  L->near_off.ensure(c, nb + 1);
  BIT_CUDA(cudaMemsetAsync(pairs.p, 0, 2 * sizeof(long long), s));
  BIT_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), s));
  const unsigned g = grid_for(nb, LWARPS);
  count_launch(), k_lists<false><<<g, 32 * LWARPS, 0, s>>>(nb, L->b_tstart.p, L->b_tcount.p, tx, ty, tz,
                                           t->nodec.p, t->children.p, t->nummemb.p, key.acc,
                                           key.add_del, key.sub_del, fcnt.p, ncnt.p, pairs.p,
                                           nullptr, nullptr, nullptr, nullptr, err.p);
  count_launch(), k_scan_ll<<<1, 1024, 0, s>>>(fcnt.p, L->far_off.p, nb);
  count_launch(), k_scan_ll<<<1, 1024, 0, s>>>(ncnt.p, L->near_off.p, nb);
  long long* hp = c->h_pinned;
  BIT_CUDA(cudaMemcpyAsync(hp, L->far_off.p + nb, sizeof(long long), cudaMemcpyDeviceToHost, s));
  BIT_CUDA(cudaMemcpyAsync(hp + 1, L->near_off.p + nb, sizeof(long long), cudaMemcpyDeviceToHost, s));
  BIT_CUDA(cudaMemcpyAsync(hp + 2, pairs.p, 2 * sizeof(long long), cudaMemcpyDeviceToHost, s));
  BIT_CUDA(cudaMemcpyAsync(hp + 4, err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  BIT_CUDA(cudaStreamSynchronize(s));
  if (*reinterpret_cast<int*>(hp + 4))
    fail(BIT_ERR_CAPACITY, "traversal stack capacity exceeded (tree deeper than supported)");
  L->nfar = hp[0];
  L->nnear = hp[1];
  L->far_pairs = hp[2];
  L->near_pairs = hp[3];
  L->far_ent.ensure(c, L->nfar);
  L->near_ent.ensure(c, L->nnear);
  count_launch(), k_lists<true><<<g, 32 * LWARPS, 0, s>>>(nb, L->b_tstart.p, L->b_tcount.p, tx, ty, tz,
                                          t->nodec.p, t->children.p, t->nummemb.p, key.acc,
                                          key.add_del, key.sub_del, nullptr, nullptr, nullptr,
                                          L->far_off.p, L->near_off.p, L->far_ent.p,
                                          L->near_ent.p, err.p);
  BIT_CHECK_LAUNCH();
  // largest batches first, so the evaluation kernels' tail is short
  {
    std::vector<long long> fo(nb + 1), no(nb + 1);
    BIT_CUDA(cudaMemcpyAsync(fo.data(), L->far_off.p, (nb + 1) * sizeof(long long), cudaMemcpyDeviceToHost, s));
    BIT_CUDA(cudaMemcpyAsync(no.data(), L->near_off.p, (nb + 1) * sizeof(long long), cudaMemcpyDeviceToHost, s));
    BIT_CUDA(cudaStreamSynchronize(s));
    std::vector<int> ord(nb);
    for (int i = 0; i < nb; i++) ord[i] = i;
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) {
      long long wa = 40 * (fo[a + 1] - fo[a]) + (no[a + 1] - no[a]);
      long long wb = 40 * (fo[b + 1] - fo[b]) + (no[b + 1] - no[b]);
      return wa > wb;
    });
    L->order.ensure(c, nb);
    BIT_CUDA(cudaMemcpyAsync(L->order.p, ord.data(), nb * sizeof(int), cudaMemcpyHostToDevice, s));
    BIT_CUDA(cudaStreamSynchronize(s));
  }
  L->key = key;
  L->valid = true;
}

}  // namespace bit

// GPU tree build: the reference's aspect-ratio bisection tree (treemake,
// src/tree3d.cpp:1345-1551), level by level.
//
// Nodes of one level are consecutive indices [a, b); their children become [b, c) in
// parent order, which is the reference's breadth-first numbering.  Inside a node the
// reference runs a short sequential program of up to seven bisections (treedivide,
// src/tree3d.cpp:1163-1304), each needing the member count and bounding box of both
// halves of the slot it splits.  Here every node keeps the results of its completed
// bisections; a one-thread "decide" step replays the program from the start on those
// cached results until it reaches the first bisection it has no result for, and a
// "pass" kernel over all members of the level's nodes computes that bisection's counts
// and bounding boxes (block reduction + atomics; min/max are order independent, so the
// result is exact).  The first decision of a level is a kernel of its own; each later one
// is made inside the pass, by the CTA that finishes the node's last chunk.  Members carry a slot label; a final stable counting scatter
// lays each node's children out contiguously in slot order, members in ascending
// original index (the reference's member order).  Field arithmetic (midpoints, aspect
// ratios, sqradius) is the reference's, with no FMA contraction.
#include <algorithm>
#include <climits>
#include <cstring>

#include "common.cuh"

namespace bit {

namespace {

constexpr int CH = 2048;  // members per chunk (one block)
constexpr int TB = 256;   // threads per block
static_assert(CH % TB == 0, "a chunk is a whole number of block strides");

__device__ __forceinline__ unsigned long long okey(double v) {
  long long b = __double_as_longlong(v);
  if (b == (long long)0x8000000000000000ULL) b = 0;  // -0.0 -> +0.0
  return b >= 0 ? ((unsigned long long)b | 0x8000000000000000ULL) : ~(unsigned long long)b;
}
__device__ __forceinline__ double okey_inv(unsigned long long k) {
  long long b = (k & 0x8000000000000000ULL) ? (long long)(k & 0x7FFFFFFFFFFFFFFFULL)
                                            : (long long)(~k);
  return __longlong_as_double(b);
}

// treeinit (src/tree3d.cpp:1045-1073)
__device__ void box_fields(double* f, double x0, double x1, double y0, double y1, double z0,
                           double z1) {
  double x = dmul(0.5, dadd(x1, x0)), y = dmul(0.5, dadd(y1, y0)), z = dmul(0.5, dadd(z1, z0));
  f[0] = x0; f[1] = x1; f[2] = y0; f[3] = y1; f[4] = z0; f[5] = z1;
  f[6] = x; f[7] = y; f[8] = z;
  f[9] = fabs(__ddiv_rn(dsub(x1, x0), dsub(y1, y0)));
  f[10] = fabs(__ddiv_rn(dsub(x1, x0), dsub(z1, z0)));
  f[11] = fabs(__ddiv_rn(dsub(y1, y0), dsub(z1, z0)));
  x = dsub(x1, x); y = dsub(y1, y); z = dsub(z1, z);
  f[12] = dadd(dadd(dmul(x, x), dmul(y, y)), dmul(z, z));
}

struct Divide {
  int dir, src, c1, c2;  // src -1: the node itself
  double mid;
};

struct SplitState {
  int active, finished, ndone, has_cur, has_prev, nchild, prev_c2eff, pad;
  Divide cur, prev;
  int res_cnt[7][2];
  double res_bb[7][2][6];
  int order[8];
  int slot_n[8];
  double slot_f[8][13];
};

struct SplitAcc {
  int cnt[2];
  unsigned long long mn[2][3], mx[2][3];
};

__device__ void acc_reset(SplitAcc* a) {
  for (int h = 0; h < 2; h++) {
    a->cnt[h] = 0;
    for (int d = 0; d < 3; d++) { a->mn[h][d] = ~0ULL; a->mx[h][d] = 0ULL; }
  }
}

// Replay of the split program on cached bisection results.
struct Replay {
  SplitState* S;
  const double* pf;
  int maxmemb;
  double lim;
  int d;
  bool need;
  int n[8];
  double f[8][13];
};

__device__ int rp_bisect(Replay& r, int dir, int src, int c1, int c2) {
  if (r.need) return 0;
  const double* f = src < 0 ? r.pf : r.f[src];
  if (r.d >= r.S->ndone) {
    r.S->cur.dir = dir; r.S->cur.src = src; r.S->cur.c1 = c1; r.S->cur.c2 = c2;
    r.S->cur.mid = f[6 + dir];
    r.need = true;
    return 0;
  }
  const int* cnt = r.S->res_cnt[r.d];
  int dst[2] = {c1, cnt[0] > 0 ? c2 : c1};
  int made = 0;
  for (int h = 0; h < 2; h++) {
    if (!cnt[h]) continue;
    const double* bb = r.S->res_bb[r.d][h];
    r.n[dst[h]] = cnt[h];
    box_fields(r.f[dst[h]], bb[0], bb[1], bb[2], bb[3], bb[4], bb[5]);
    made++;
  }
  r.d++;
  return made;
}

__device__ __forceinline__ bool zsplit_ok(const Replay& r, int s) {
  return r.f[s][10] < r.lim && r.f[s][11] < r.lim && r.n[s] > r.maxmemb;
}

// treemake's per-node program (src/tree3d.cpp:1412-1545) on slots relative to the first
// free node index.  Returns nchild; order[] receives the children in recorded order.
__device__ int split_program(Replay& r, int* order) {
  const double lim = r.lim;
  const double* P = r.pf;
  int nchild = 0, nchild2 = 0, ind2;
  for (int s = 0; s < 8; s++) r.n[s] = 0;
  if (P[9] > lim && P[10] > lim) {
    int xc = rp_bisect(r, 0, -1, 0, 1);
    ind2 = xc;
    for (int j = 0; j < xc; j++) {
      order[nchild++] = j;
      if (r.f[j][9] < lim && r.f[j][11] > lim && r.n[j] > r.maxmemb) {
        int yc = rp_bisect(r, 1, j, j, ind2);
        if (yc == 2) { order[nchild++] = ind2; ind2++; }
        for (int k = 0; k < yc; k++) {
          // the reference's numtree+j+k*(nchild2+1) (src/tree3d.cpp:1460), as written
          int t = j + k * (nchild2 + 1);
          if (t >= 8 || t >= ind2) continue;  // never-created slot: nummemb == 0
          if (zsplit_ok(r, t)) {
            int zc = rp_bisect(r, 2, t, t, ind2);
            if (zc == 2) { order[nchild++] = ind2; nchild2++; ind2++; }
          }
        }
      } else if (zsplit_ok(r, j)) {
        int zc = rp_bisect(r, 2, j, j, ind2);
        if (zc == 2) { order[nchild++] = ind2; ind2++; }
      }
    }
  } else if (P[9] < lim && P[11] > lim) {
    int yc = rp_bisect(r, 1, -1, 0, 1);
    ind2 = yc;
    for (int j = 0; j < yc; j++) {
      order[nchild++] = j;
      if (zsplit_ok(r, j)) {
        int zc = rp_bisect(r, 2, j, j, ind2);
        if (zc == 2) { order[nchild++] = ind2; ind2++; }
      }
    }
  } else {
    int zc = rp_bisect(r, 2, -1, 0, 1);
    for (int j = 0; j < zc; j++) order[nchild++] = j;
  }
  return nchild;
}

__global__ void k_iota(int* p, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = i;
}

template <class T>
__device__ __forceinline__ T warp_min(T v) {
  for (int o = 16; o; o >>= 1) { T w = __shfl_xor_sync(0xffffffffu, v, o); v = w < v ? w : v; }
  return v;
}
template <class T>
__device__ __forceinline__ T warp_max(T v) {
  for (int o = 16; o; o >>= 1) { T w = __shfl_xor_sync(0xffffffffu, v, o); v = w > v ? w : v; }
  return v;
}
__device__ __forceinline__ int warp_sum(int v) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Bounding box of each system's particles (its root, src/tree3d.cpp:1385-1403); flags
// NaNs.  grid.y = system, grid.x = blocks striding over that system.
__global__ void k_root_bbox(const int* sys_start, const int* sys_n, const double* x,
                            const double* y, const double* z, SplitAcc* acc, int* err) {
  const int sy = blockIdx.y;
  const int i0 = sys_start[sy], i1 = i0 + sys_n[sy];
  unsigned long long mn[3] = {~0ULL, ~0ULL, ~0ULL}, mx[3] = {0, 0, 0};
  int bad = 0;
  for (int i = i0 + blockIdx.x * blockDim.x + threadIdx.x; i < i1; i += gridDim.x * blockDim.x) {
    double v[3] = {x[i], y[i], z[i]};
    for (int d = 0; d < 3; d++) {
      if (isnan(v[d])) bad = 1;
      unsigned long long k = okey(v[d]);
      mn[d] = k < mn[d] ? k : mn[d];
      mx[d] = k > mx[d] ? k : mx[d];
    }
  }
  for (int d = 0; d < 3; d++) {
    mn[d] = warp_min(mn[d]);
    mx[d] = warp_max(mx[d]);
  }
  bad = __any_sync(0xffffffffu, bad);
  if ((threadIdx.x & 31) == 0) {
    for (int d = 0; d < 3; d++) {
      atomicMin(&acc[sy].mn[0][d], mn[d]);
      atomicMax(&acc[sy].mx[0][d], mx[d]);
    }
    if (bad) atomicOr(err, 1);
  }
}

__global__ void k_acc_reset(SplitAcc* acc, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) acc_reset(&acc[i]);
}

__global__ void k_root_init(int nsys, const int* sys_start, const int* sys_n, const SplitAcc* acc,
                            int* nummemb, int* start, int* children, int* level, int* parent,
                            double* fields, int* node_sys) {
  const int sy = blockIdx.x * blockDim.x + threadIdx.x;
  if (sy >= nsys) return;
  double f[13];
  const SplitAcc* A = &acc[sy];
  box_fields(f, okey_inv(A->mn[0][0]), okey_inv(A->mx[0][0]), okey_inv(A->mn[0][1]),
             okey_inv(A->mx[0][1]), okey_inv(A->mn[0][2]), okey_inv(A->mx[0][2]));
  for (int k = 0; k < 13; k++) fields[13LL * sy + k] = f[k];
  nummemb[sy] = sys_n[sy]; start[sy] = sys_start[sy]; level[sy] = 0; parent[sy] = -1;
  node_sys[sy] = sy;
  for (int c = 0; c < 8; c++) children[8LL * sy + c] = -1;
}

// Per level node: active flag and the number of member chunks it needs.
__global__ void k_level_init(int a, int nlev, const int* nummemb, const int* node_sys,
                             const int* sys_maxmemb, SplitState* st, SplitAcc* acc, int* nchunk,
                             int* done) {
  int li = blockIdx.x * blockDim.x + threadIdx.x;
  if (li >= nlev) return;
  SplitState* S = &st[li];
  int cnt = nummemb[a + li];
  S->active = cnt > sys_maxmemb[node_sys[a + li]];
  S->finished = 0; S->ndone = 0; S->has_cur = 0; S->has_prev = 0; S->nchild = 0;
  acc_reset(&acc[li]);
  nchunk[li] = S->active ? (cnt + CH - 1) / CH : 0;
  done[li] = 0;
}

// Exclusive scan of a small int array in one block; total in out[n].
__global__ void k_scan_small(const int* in, int* out, int n) {
  __shared__ int ws[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int base = 0; base < n; base += blockDim.x) {
    int i = base + threadIdx.x;
    int v = i < n ? in[i] : 0;
    int s = v;
    for (int o = 1; o < 32; o <<= 1) {
      int t = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += t;
    }
    if (lane == 31) ws[w] = s;
    __syncthreads();
    if (w == 0) {
      int t = lane < nw ? ws[lane] : 0;
      for (int o = 1; o < 32; o <<= 1) {
        int u = __shfl_up_sync(0xffffffffu, t, o);
        if (lane >= o) t += u;
      }
      if (lane < nw) ws[lane] = t;
    }
    __syncthreads();
    int pre = carry + (w ? ws[w - 1] : 0) + s - v;
    if (i < n) out[i] = pre;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = pre + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) out[n] = carry;
}

__global__ void k_fill_chunks(int a, int nlev, const int* start, const int* nummemb,
                              const int* cbeg, int2* chunks) {
  int li = blockIdx.x * blockDim.x + threadIdx.x;
  if (li >= nlev) return;
  int s = start[a + li];
  for (int c = cbeg[li]; c < cbeg[li + 1]; c++) chunks[c] = make_int2(li, s + (c - cbeg[li]) * CH);
}

// Record the bisection step just reduced for node a + li and plan its next one.
__device__ __noinline__ void decide_node(int a, int li, const double* fields, const int* node_sys,
                                         const int* sys_maxmemb, SplitState* st, SplitAcc* acc,
                                         double lim, int* err) {
  SplitState* S = &st[li];
  if (!S->active) return;
  SplitAcc* A = &acc[li];
  if (S->has_cur) {
    // The sums arrived as atomics in L2 from other CTAs of this launch (when the decision
    // is made inside k_split_pass); __ldcg reads them there, never from a line this SM's
    // L1 may hold from a neighbouring node's decision.
    int d = S->ndone;
    for (int h = 0; h < 2; h++) {
      S->res_cnt[d][h] = __ldcg(&A->cnt[h]);
      for (int q = 0; q < 3; q++) {
        S->res_bb[d][h][2 * q] = okey_inv(__ldcg(&A->mn[h][q]));
        S->res_bb[d][h][2 * q + 1] = okey_inv(__ldcg(&A->mx[h][q]));
      }
    }
    S->ndone = d + 1;
    S->prev = S->cur;
    S->prev_c2eff = S->res_cnt[d][0] > 0 ? S->cur.c2 : S->cur.c1;
    S->has_prev = 1;
    S->has_cur = 0;
    acc_reset(A);
  } else {
    S->has_prev = 0;
  }
  if (S->finished) return;
  Replay r;
  r.S = S; r.pf = fields + 13 * (long long)(a + li); r.lim = lim;
  r.maxmemb = sys_maxmemb[node_sys[a + li]];
  r.d = 0; r.need = false;
  int order[8];
  int nchild = split_program(r, order);
  if (r.need) {
    S->has_cur = 1;
    if (S->ndone >= 7) atomicOr(err, 4);  // cannot happen: at most 7 bisections per node
    return;
  }
  S->finished = 1;
  S->nchild = nchild;
  for (int c = 0; c < 8; c++) S->order[c] = c < nchild ? order[c] : -1;
  for (int s = 0; s < 8; s++) {
    S->slot_n[s] = s < nchild ? r.n[s] : 0;
    if (s < nchild)
      for (int k = 0; k < 13; k++) S->slot_f[s][k] = r.f[s][k];
  }
  if (nchild < 2) atomicOr(err, 2);  // one child == the node itself: never terminates
}

__global__ void k_split_decide(int a, int nlev, const double* fields, const int* node_sys,
                               const int* sys_maxmemb, SplitState* st, SplitAcc* acc, double lim,
                               int* err) {
  int li = blockIdx.x * blockDim.x + threadIdx.x;
  if (li < nlev) decide_node(a, li, fields, node_sys, sys_maxmemb, st, acc, lim, err);
}

__device__ __forceinline__ double coord(int dir, const double* sx, const double* sy,
                                        const double* sz, int e) {
  return dir == 0 ? sx[e] : (dir == 1 ? sy[e] : sz[e]);
}

// Per-level inputs of the decision a split pass makes for each node when its last chunk
// is done (decide = 0: the level's final pass, which only relabels).
struct DecideArgs {
  const int* nchunk;
  int* done;
  const double* fields;
  const int* node_sys;
  const int* sys_maxmemb;
  double lim;
  int* err;
  int decide;
};

// One bisection step for every active node of the level: apply the previous step's
// relabel, then reduce counts / bounding boxes of both halves of the current step.  The
// CTA that finishes a node's last chunk then makes the node's decision for the next step.
// 6 CTAs per SM as without the decision (40 registers); whatever the call to decide_node
// needs beyond that is spilled on the deciding thread's path only
__global__ void __launch_bounds__(TB, 6) k_split_pass(const int2* chunks, const int* nch, int a, const int* start,
                                                   const int* nummemb, const double* __restrict__ sx,
                                                   const double* __restrict__ sy,
                                                   const double* __restrict__ sz,
                                                   signed char* __restrict__ lab, SplitState* st,
                                                   SplitAcc* acc, DecideArgs da) {
  if ((int)blockIdx.x >= *nch) return;  // the grid is sized from a bound
  const int2 ck = chunks[blockIdx.x];
  const SplitState* S = &st[ck.x];
  const int hp = S->has_prev, hc = S->has_cur;
  if (!hp && !hc) return;  // (its decision would change nothing)
  const Divide pv = S->prev, cu = S->cur;
  const int pc2 = S->prev_c2eff;
  const int node = a + ck.x;
  const int e1 = min(ck.y + CH, start[node] + nummemb[node]);
  int cnt[2] = {0, 0};
  unsigned long long mn[2][3], mx[2][3];
  for (int h = 0; h < 2; h++)
    for (int d = 0; d < 3; d++) { mn[h][d] = ~0ULL; mx[h][d] = 0ULL; }
  // this thread's members e = ck.y + tid + k TB: every label first, then the unrolled
  // loop, so the members' loads overlap instead of waiting one after the other
  constexpr int PER = CH / TB;
  signed char lb[PER];
#pragma unroll
  for (int k = 0; k < PER; k++) {
    const int e = ck.y + threadIdx.x + k * TB;
    lb[k] = e < e1 ? lab[e] : (signed char)-128;  // no slot has label -128
  }
#pragma unroll
  for (int k = 0; k < PER; k++) {
    const int e = ck.y + threadIdx.x + k * TB;
    int l = lb[k];
    if (l == -128) continue;
    if (hp && l == pv.src) {
      l = (coord(pv.dir, sx, sy, sz, e) <= pv.mid) ? pv.c1 : pc2;
      lab[e] = (signed char)l;
    }
    if (hc && l == cu.src) {
      int h = (coord(cu.dir, sx, sy, sz, e) <= cu.mid) ? 0 : 1;
      double v[3] = {sx[e], sy[e], sz[e]};
      cnt[h]++;
      for (int d = 0; d < 3; d++) {
        unsigned long long k = okey(v[d]);
        mn[h][d] = k < mn[h][d] ? k : mn[h][d];
        mx[h][d] = k > mx[h][d] ? k : mx[h][d];
      }
    }
  }
  // warp, then CTA reductions; one set of global atomics per CTA (min / max / sum are
  // order-independent, so the result is exact whatever the order)
  constexpr int NW = TB / 32;
  __shared__ int s_c[NW][2];
  __shared__ unsigned long long s_m[NW][2][3], s_M[NW][2][3];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int h = 0; h < 2; h++) {
    const int c = warp_sum(cnt[h]);
    unsigned long long m[3], M[3];
    for (int d = 0; d < 3; d++) { m[d] = warp_min(mn[h][d]); M[d] = warp_max(mx[h][d]); }
    if (lane == 0) {
      s_c[w][h] = c;
      for (int d = 0; d < 3; d++) { s_m[w][h][d] = m[d]; s_M[w][h][d] = M[d]; }
    }
  }
  __syncthreads();
  if (hc && threadIdx.x < 2 * 7) {  // thread (h, v): v = 0..5 min/max of one axis, v = 6 count
    const int h = threadIdx.x / 7, v = threadIdx.x % 7;
    int c = 0;
    for (int q = 0; q < NW; q++) c += s_c[q][h];
    if (c > 0) {
      if (v == 6) {
        atomicAdd(&acc[ck.x].cnt[h], c);
      } else {
        const int d = v >> 1;
        if (v & 1) {
          unsigned long long M = 0;
          for (int q = 0; q < NW; q++) M = s_M[q][h][d] > M ? s_M[q][h][d] : M;
          atomicMax(&acc[ck.x].mx[h][d], M);
        } else {
          unsigned long long m = ~0ULL;
          for (int q = 0; q < NW; q++) m = s_m[q][h][d] < m ? s_m[q][h][d] : m;
          atomicMin(&acc[ck.x].mn[h][d], m);
        }
      }
    }
  }
  if (!da.decide) return;
  // the CTA that completes the node's chunk count decides (its atomics, and every other
  // chunk's, are visible after the fences)
  __shared__ int s_last;
  __threadfence();  // this thread's atomics, before the count that may complete the node
  __syncthreads();
  if (threadIdx.x == 0) {
    s_last = atomicAdd(&da.done[ck.x], 1) == da.nchunk[ck.x] - 1;
    if (s_last) {
      __threadfence();
      decide_node(a, ck.x, da.fields, da.node_sys, da.sys_maxmemb, st, acc, da.lim, da.err);
      da.done[ck.x] = 0;
    }
  }
}

__global__ void k_scatter_count(const int2* chunks, const int* nch, int a, const int* start, const int* nummemb,
                                const signed char* lab, int* cc) {
  if ((int)blockIdx.x >= *nch) return;  // the grid is sized from a bound
  const int2 ck = chunks[blockIdx.x];
  const int node = a + ck.x;
  const int e1 = min(ck.y + CH, start[node] + nummemb[node]);
  __shared__ int s[8];
  if (threadIdx.x < 8) s[threadIdx.x] = 0;
  __syncthreads();
  int c[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int e = ck.y + threadIdx.x; e < e1; e += TB) {
    int l = lab[e];
#pragma unroll
    for (int v = 0; v < 8; v++) c[v] += (l == v);
  }
#pragma unroll
  for (int v = 0; v < 8; v++) {
    int t = warp_sum(c[v]);
    if ((threadIdx.x & 31) == 0 && t) atomicAdd(&s[v], t);
  }
  __syncthreads();
  if (threadIdx.x < 8) cc[blockIdx.x * 8 + threadIdx.x] = s[threadIdx.x];
}

// Per node (one block): destination offset of each chunk's members of each child slot,
// an exclusive scan over the node's chunks of the per-slot counts, 8 slots at once.
__global__ void __launch_bounds__(TB) k_scatter_offsets(int a, const int* start, const int* cbeg,
                                                        const int* cc, int* coff,
                                                        const SplitState* st, int* err) {
  const int li = blockIdx.x;
  const SplitState* S = &st[li];
  if (!S->active) return;
  constexpr int NW = TB / 32;
  __shared__ int s_base[8], s_carry[8], s_warp[NW][8];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  if (tid == 0) {
    int acc = 0;
    for (int v = 0; v < 8; v++) { s_base[v] = start[a + li] + acc; acc += S->slot_n[v]; s_carry[v] = 0; }
  }
  __syncthreads();
  const int c0 = cbeg[li], c1 = cbeg[li + 1];
  for (int cb = c0; cb < c1; cb += TB) {
    const int c = cb + tid;
    int val[8], inc[8];
    for (int v = 0; v < 8; v++) {
      val[v] = c < c1 ? cc[c * 8 + v] : 0;
      inc[v] = val[v];
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, inc[v], o);
        if (lane >= o) inc[v] += t;
      }
    }
    if (lane == 31)
      for (int v = 0; v < 8; v++) s_warp[w][v] = inc[v];
    __syncthreads();
    if (c < c1)
      for (int v = 0; v < 8; v++) {
        int before = s_carry[v];
        for (int q = 0; q < w; q++) before += s_warp[q][v];
        coff[c * 8 + v] = s_base[v] + before + inc[v] - val[v];
      }
    __syncthreads();
    if (tid < 8)
      for (int q = 0; q < NW; q++) s_carry[tid] += s_warp[q][tid];
    __syncthreads();
  }
  if (tid < 8 && s_carry[tid] != S->slot_n[tid]) atomicOr(err, 8);
}

// Stable scatter of each chunk's members to their child's range (order kept).
__global__ void __launch_bounds__(TB) k_scatter(const int2* chunks, const int* nch, int a, const int* start,
                                                const int* nummemb, const signed char* __restrict__ lab,
                                                const int* coff, const int* __restrict__ perm,
                                                const double* __restrict__ sx,
                                                const double* __restrict__ sy,
                                                const double* __restrict__ sz, int* __restrict__ perm2,
                                                double* __restrict__ sx2, double* __restrict__ sy2,
                                                double* __restrict__ sz2) {
  if ((int)blockIdx.x >= *nch) return;  // the grid is sized from a bound
  const int2 ck = chunks[blockIdx.x];
  const int node = a + ck.x;
  const int e1 = min(ck.y + CH, start[node] + nummemb[node]);
  __shared__ int wcnt[TB / 32][8];
  __shared__ int run[8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (threadIdx.x < 8) run[threadIdx.x] = coff[blockIdx.x * 8 + threadIdx.x];
  __syncthreads();
  const unsigned lt = (1u << lane) - 1u;
  for (int t0 = ck.y; t0 < e1; t0 += TB) {
    int e = t0 + threadIdx.x;
    int l = e < e1 ? lab[e] : -2;
    // the member's record loads while its rank among the block's members is formed
    int pv = 0;
    double xv = 0.0, yv = 0.0, zv = 0.0;
    if (l >= 0) { pv = perm[e]; xv = sx[e]; yv = sy[e]; zv = sz[e]; }
    int my_rank = 0;
    for (int v = 0; v < 8; v++) {
      unsigned m = __ballot_sync(0xffffffffu, l == v);
      if (l == v) my_rank = __popc(m & lt);
      if (lane == 0) wcnt[w][v] = __popc(m);
    }
    __syncthreads();
    if (l >= 0) {
      int dst = run[l] + my_rank;
      for (int q = 0; q < w; q++) dst += wcnt[q][l];
      perm2[dst] = pv;
      sx2[dst] = xv;
      sy2[dst] = yv;
      sz2[dst] = zv;
    }
    __syncthreads();
    if (threadIdx.x < 8) {
      int tot = 0;
      for (int q = 0; q < TB / 32; q++) tot += wcnt[q][threadIdx.x];
      run[threadIdx.x] += tot;
    }
    __syncthreads();
  }
}

// (restrict: the two copies never overlap, so a thread's members' loads need not wait
// for its earlier stores)
__global__ void k_copy_back(const int2* chunks, const int* nch, int a, const int* start, const int* nummemb,
                            const int* __restrict__ perm2, const double* __restrict__ sx2,
                            const double* __restrict__ sy2, const double* __restrict__ sz2,
                            int* __restrict__ perm, double* __restrict__ sx,
                            double* __restrict__ sy, double* __restrict__ sz) {
  if ((int)blockIdx.x >= *nch) return;  // the grid is sized from a bound
  const int2 ck = chunks[blockIdx.x];
  const int node = a + ck.x;
  const int e1 = min(ck.y + CH, start[node] + nummemb[node]);
#pragma unroll
  for (int e = ck.y + threadIdx.x; e < e1; e += TB) {
    perm[e] = perm2[e]; sx[e] = sx2[e]; sy[e] = sy2[e]; sz[e] = sz2[e];
  }
}

__global__ void k_child_counts(int nlev, const SplitState* st, int* nch) {
  int li = blockIdx.x * blockDim.x + threadIdx.x;
  if (li < nlev) nch[li] = st[li].active ? st[li].nchild : 0;
}

__global__ void k_make_children(int a, int b, int nlev, const SplitState* st, const int* cscan,
                                int* nummemb, int* start, int* children, int* level,
                                int* parent, double* fields, int* node_sys) {
  int li = blockIdx.x * blockDim.x + threadIdx.x;
  if (li >= nlev) return;
  const SplitState* S = &st[li];
  if (!S->active) return;
  const int p = a + li, base = b + cscan[li];
  int off = start[p];
  for (int s = 0; s < S->nchild; s++) {
    int node = base + s;
    nummemb[node] = S->slot_n[s];
    start[node] = off;
    off += S->slot_n[s];
    level[node] = level[p] + 1;
    parent[node] = p;
    node_sys[node] = node_sys[p];
    for (int k = 0; k < 13; k++) fields[13LL * node + k] = S->slot_f[s][k];
    for (int c = 0; c < 8; c++) children[8LL * node + c] = -1;
  }
  for (int c = 0; c < 8; c++) children[8LL * p + c] = c < S->nchild ? base + S->order[c] : -1;
}

__global__ void k_node_centres(int numtree, const double* fields, const int* children,
                               const int* nummemb, double4* nodec, float4* nodeh, int2* kids) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < numtree) {
    // children[] holds base + order[c] in its first nchild slots (consecutive node
    // indices, in another order), so one int2 gives the traversal all of them:
    // (base, nchild | order[c] << (4 + 3c)); a leaf is (-1, nummemb)
    const int* ch = children + 8LL * i;
    int base = ch[0], cnt = 0;
    for (int c = 0; c < 8 && ch[c] != -1; c++) {
      base = min(base, ch[c]);
      cnt++;
    }
    int code = cnt;
    for (int c = 0; c < cnt; c++) code |= (ch[c] - base) << (4 + 3 * c);
    kids[i] = cnt ? make_int2(base, code) : make_int2(-1, nummemb[i]);
    const double* f = fields + 13LL * i;
    nodec[i] = make_double4(f[6], f[7], f[8], f[12]);
    // half extents about the midpoint, rounded up to FP32 (a box the members are inside of)
    const double hx = fmax(f[1] - f[6], f[6] - f[0]), hy = fmax(f[3] - f[7], f[7] - f[2]),
                 hz = fmax(f[5] - f[8], f[8] - f[4]);
    nodeh[i] = make_float4(__double2float_ru(hx), __double2float_ru(hy), __double2float_ru(hz), 0.f);
  }
}

__global__ void k_leaf_of(int nleaves, const int* leaves, const int* start, const int* nummemb,
                          int* leaf_of) {
  int l = blockIdx.x;
  if (l >= nleaves) return;
  int node = leaves[l];
  for (int e = start[node] + threadIdx.x; e < start[node] + nummemb[node]; e += blockDim.x)
    leaf_of[e] = node;
}

__global__ void k_iperm(int n, const int* perm, int* iperm) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) iperm[perm[e]] = e;
}

}  // namespace

template <class T>
void DBuf<T>::grow(Ctx* ctx, size_t count, size_t keep, cudaStream_t s) {
  if (count <= n && p) return;
  T* q = static_cast<T*>(dev_alloc(ctx, count * sizeof(T)));
  if (p && keep) BIT_CUDA(cudaMemcpyAsync(q, p, keep * sizeof(T), cudaMemcpyDeviceToDevice, s));
  BIT_CUDA(cudaStreamSynchronize(s));
  release();
  p = q;
  n = count;
  c = ctx;
}
template struct DBuf<int>;
template struct DBuf<double>;

void tree_build(Tree* t, const double* x, const double* y, const double* z) {
  Ctx* c = t->ctx;
  cudaStream_t s = c->stream;
  const int n = t->n;
  const int nsys = t->nsys;
  // systems: particle ranges and leaf sizes (one system unless the caller made a forest)
  if ((int)t->h_sys_start.size() != nsys) {
    t->h_sys_start.assign(1, 0);
    t->h_sys_n.assign(1, n);
    t->h_sys_maxmemb.assign(1, t->maxmemb);
  }
  t->sys_start.ensure(c, nsys);
  t->sys_n.ensure(c, nsys);
  t->sys_maxmemb.ensure(c, nsys);
  BIT_CUDA(cudaMemcpyAsync(t->sys_start.p, t->h_sys_start.data(), nsys * sizeof(int), cudaMemcpyHostToDevice, s));
  BIT_CUDA(cudaMemcpyAsync(t->sys_n.p, t->h_sys_n.data(), nsys * sizeof(int), cudaMemcpyHostToDevice, s));
  BIT_CUDA(cudaMemcpyAsync(t->sys_maxmemb.p, t->h_sys_maxmemb.data(), nsys * sizeof(int), cudaMemcpyHostToDevice, s));
  t->perm.ensure(c, n);
  t->sx.ensure(c, n); t->sy.ensure(c, n); t->sz.ensure(c, n);
  DBuf<int> perm2; DBuf<double> sx2, sy2, sz2;
  perm2.ensure(c, n); sx2.ensure(c, n); sy2.ensure(c, n); sz2.ensure(c, n);
  DBuf<signed char> lab;
  lab.ensure(c, n);
  long long capl = 64;
  for (int k = 0; k < nsys; k++)
    capl += 16LL * (t->h_sys_n[k] / std::max(t->h_sys_maxmemb[k], 1) + 1) + 8;
  int cap = (int)std::min<long long>(capl, 1LL << 30);
  t->nummemb.ensure(c, cap); t->start.ensure(c, cap); t->level.ensure(c, cap);
  t->parent.ensure(c, cap); t->children.ensure(c, 8LL * cap); t->fields.ensure(c, 13LL * cap);
  t->node_sys.ensure(c, cap);
  DBuf<int> err;
  err.ensure(c, 4);
  BIT_CUDA(cudaMemsetAsync(err.p, 0, 4 * sizeof(int), s));
  long long* hp = c->h_pinned;

  count_launch(), k_iota<<<grid_for(n, 256), 256, 0, s>>>(t->perm.p, n);
  BIT_CUDA(cudaMemcpyAsync(t->sx.p, x, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  BIT_CUDA(cudaMemcpyAsync(t->sy.p, y, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  BIT_CUDA(cudaMemcpyAsync(t->sz.p, z, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  BIT_CUDA(cudaMemsetAsync(lab.p, -1, n, s));

  DBuf<SplitAcc> acc;
  acc.ensure(c, nsys);
  count_launch(), k_acc_reset<<<grid_for(nsys, 128), 128, 0, s>>>(acc.p, nsys);
  {
    const unsigned per = std::max(1u, std::min<unsigned>(grid_for(n / nsys + 1, 256), 4 * c->num_sms / nsys + 1));
    count_launch(), k_root_bbox<<<dim3(per, nsys), 256, 0, s>>>(t->sys_start.p, t->sys_n.p, t->sx.p,
                                                                t->sy.p, t->sz.p, acc.p, err.p);
  }
  count_launch(), k_root_init<<<grid_for(nsys, 128), 128, 0, s>>>(
      nsys, t->sys_start.p, t->sys_n.p, acc.p, t->nummemb.p, t->start.p, t->children.p,
      t->level.p, t->parent.p, t->fields.p, t->node_sys.p);
  BIT_CHECK_LAUNCH();

  const double lim = 1.0 / std::sqrt(2.0);  // src/tree3d.cpp:1371
  DBuf<SplitState> st;
  DBuf<int> nchunk, cbeg, cc, coff, nch, cscan, done;
  DBuf<int2> chunks;
  int a = 0, b = nsys, depth = 1;
  while (true) {
    const int nlev = b - a;
    st.ensure(c, nlev);
    acc.ensure(c, nlev);
    nchunk.ensure(c, nlev);
    cbeg.ensure(c, nlev + 1);
    nch.ensure(c, nlev);
    cscan.ensure(c, nlev + 1);
    const unsigned gl = grid_for(nlev, 128);
    done.ensure(c, nlev);
    count_launch(), k_level_init<<<gl, 128, 0, s>>>(a, nlev, t->nummemb.p, t->node_sys.p,
                                                    t->sys_maxmemb.p, st.p, acc.p, nchunk.p, done.p);
    count_launch(), k_scan_small<<<1, 1024, 0, s>>>(nchunk.p, cbeg.p, nlev);
    // The level's chunk count stays on the device (cbeg[nlev]): the chunk kernels run on a
    // grid sized from its bound, n / CH + one partial chunk per node, and CTAs past the
    // count return.  A level of leaves only runs empty kernels, and ends the loop below
    // with no children.
    const int* nchk = cbeg.p + nlev;
    const int nch_total = (int)std::min<long long>((long long)n / CH + nlev + 1, INT_MAX);
    chunks.ensure(c, nch_total);
    cc.ensure(c, 8LL * nch_total);
    coff.ensure(c, 8LL * nch_total);
    count_launch(), k_fill_chunks<<<gl, 128, 0, s>>>(a, nlev, t->start.p, t->nummemb.p, cbeg.p, chunks.p);
    count_launch(), k_split_decide<<<gl, 128, 0, s>>>(a, nlev, t->fields.p, t->node_sys.p,
                                                      t->sys_maxmemb.p, st.p, acc.p, lim, err.p);
    DecideArgs da{nchunk.p, done.p, t->fields.p, t->node_sys.p, t->sys_maxmemb.p, lim, err.p, 1};
    for (int step = 0; step < 8; step++) {  // 7 bisection steps at most, then the last relabel
      da.decide = step < 7;
      count_launch(), k_split_pass<<<nch_total, TB, 0, s>>>(chunks.p, nchk, a, t->start.p, t->nummemb.p, t->sx.p,
                                                            t->sy.p, t->sz.p, lab.p, st.p, acc.p, da);
    }
    count_launch(), k_scatter_count<<<nch_total, TB, 0, s>>>(chunks.p, nchk, a, t->start.p, t->nummemb.p, lab.p, cc.p);
    count_launch(), k_scatter_offsets<<<nlev, TB, 0, s>>>(a, t->start.p, cbeg.p, cc.p, coff.p, st.p, err.p);
    count_launch(), k_scatter<<<nch_total, TB, 0, s>>>(chunks.p, nchk, a, t->start.p, t->nummemb.p, lab.p, coff.p,
                                                       t->perm.p, t->sx.p, t->sy.p, t->sz.p, perm2.p, sx2.p,
                                                       sy2.p, sz2.p);
    count_launch(), k_copy_back<<<nch_total, TB, 0, s>>>(chunks.p, nchk, a, t->start.p, t->nummemb.p, perm2.p, sx2.p,
                                                         sy2.p, sz2.p, t->perm.p, t->sx.p, t->sy.p, t->sz.p);
    // the next level's members start unlabelled
    BIT_CUDA(cudaMemsetAsync(lab.p, -1, n, s));
    count_launch(), k_child_counts<<<gl, 128, 0, s>>>(nlev, st.p, nch.p);
    count_launch(), k_scan_small<<<1, 1024, 0, s>>>(nch.p, cscan.p, nlev);
    BIT_CUDA(cudaMemcpyAsync(hp, cscan.p + nlev, sizeof(int), cudaMemcpyDeviceToHost, s));
    BIT_CUDA(cudaMemcpyAsync(hp + 1, err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    BIT_CUDA(cudaStreamSynchronize(s));
    const int total = *reinterpret_cast<int*>(hp);
    const int e = *reinterpret_cast<int*>(hp + 1);
    if (e & 1) fail(BIT_ERR_INVALID_ARGUMENT, "particle coordinates contain NaN");
    if (e & 2)
      fail(BIT_ERR_DEGENERATE,
           "a node with more than maxmemb members cannot be split (coincident particles); "
           "the reference's treemake would not terminate");
    if (e & 12) fail(BIT_ERR_CUDA, "internal tree-build consistency check failed");
    if (total == 0) break;
    if (b + total > cap) {
      int ncap = std::max(2 * cap, b + total + 64);
      t->nummemb.grow(c, ncap, b, s); t->start.grow(c, ncap, b, s);
      t->level.grow(c, ncap, b, s); t->parent.grow(c, ncap, b, s);
      t->children.grow(c, 8LL * ncap, 8LL * b, s); t->fields.grow(c, 13LL * ncap, 13LL * b, s);
      t->node_sys.grow(c, ncap, b, s);
      cap = ncap;
    }
    count_launch(), k_make_children<<<gl, 128, 0, s>>>(a, b, nlev, st.p, cscan.p, t->nummemb.p, t->start.p,
                                                       t->children.p, t->level.p, t->parent.p, t->fields.p,
                                                       t->node_sys.p);
    BIT_CHECK_LAUNCH();
    a = b;
    b += total;
    depth++;
  }
  {
    // roots that are leaves (n <= maxmemb) still have to report NaNs
    BIT_CUDA(cudaMemcpyAsync(hp + 1, err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    BIT_CUDA(cudaStreamSynchronize(s));
    if (*reinterpret_cast<int*>(hp + 1) & 1)
      fail(BIT_ERR_INVALID_ARGUMENT, "particle coordinates contain NaN");
  }
  t->numtree = b;
  t->depth = depth;
  t->cap = cap;
  t->nodec.ensure(c, b);
  t->nodeh.ensure(c, b);
  t->kids.ensure(c, b);
  count_launch(), k_node_centres<<<grid_for(b, 128), 128, 0, s>>>(b, t->fields.p, t->children.p, t->nummemb.p,
                                                                 t->nodec.p, t->nodeh.p, t->kids.p);
  tree_sync_host(t);
  // leaves in node order
  std::vector<int> leaves;
  for (int i = 0; i < b; i++)
    if (t->h_children[8LL * i] == -1) leaves.push_back(i);
  t->nleaves = (int)leaves.size();
  t->leaves.ensure(c, leaves.size());
  BIT_CUDA(cudaMemcpyAsync(t->leaves.p, leaves.data(), leaves.size() * sizeof(int),
                           cudaMemcpyHostToDevice, s));
  t->leaf_of.ensure(c, n);
  count_launch(), k_leaf_of<<<t->nleaves, 256, 0, s>>>(t->nleaves, t->leaves.p, t->start.p, t->nummemb.p,
                                                       t->leaf_of.p);
  t->iperm.ensure(c, n);
  count_launch(), k_iperm<<<grid_for(n, 256), 256, 0, s>>>(n, t->perm.p, t->iperm.p);
  BIT_CHECK_LAUNCH();
  BIT_CUDA(cudaStreamSynchronize(s));
  t->gen++;
  t->has_moments = false;
  t->plists.valid = false;
  t->plists.alt_valid = false;
}

template struct DBuf<signed char>;
template struct DBuf<SplitState>;
template struct DBuf<SplitAcc>;
template struct DBuf<int2>;

void tree_sync_host(Tree* t) {
  cudaStream_t s = t->ctx->stream;
  const int b = t->numtree;
  t->h_nummemb.resize(b); t->h_start.resize(b); t->h_children.resize(8LL * b);
  t->h_level.resize(b); t->h_fields.resize(13LL * b); t->h_node_sys.resize(b);
  BIT_CUDA(cudaMemcpyAsync(t->h_nummemb.data(), t->nummemb.p, b * sizeof(int), cudaMemcpyDeviceToHost, s));
  BIT_CUDA(cudaMemcpyAsync(t->h_start.data(), t->start.p, b * sizeof(int), cudaMemcpyDeviceToHost, s));
  BIT_CUDA(cudaMemcpyAsync(t->h_children.data(), t->children.p, 8LL * b * sizeof(int), cudaMemcpyDeviceToHost, s));
  BIT_CUDA(cudaMemcpyAsync(t->h_level.data(), t->level.p, b * sizeof(int), cudaMemcpyDeviceToHost, s));
  BIT_CUDA(cudaMemcpyAsync(t->h_fields.data(), t->fields.p, 13LL * b * sizeof(double), cudaMemcpyDeviceToHost, s));
  BIT_CUDA(cudaMemcpyAsync(t->h_node_sys.data(), t->node_sys.p, b * sizeof(int), cudaMemcpyDeviceToHost, s));
  BIT_CUDA(cudaStreamSynchronize(s));
  t->h_sys_leaf_sqr.assign(t->nsys, 0.0);
  for (int i = 0; i < b; i++)
    if (t->h_children[8LL * i] == -1) {
      double& m = t->h_sys_leaf_sqr[t->h_node_sys[i]];
      m = std::max(m, t->h_fields[13LL * i + 12]);
    }
}

}  // namespace bit

// Cluster moments (treemoments, src/tree3d.cpp:2631-2711):
//   M_ijk(node) = sum over members q * dx^i dy^j dz^k,  i+j+k < nterms,
// about the node's box midpoint, in FP64 for every node.
//
// Members of every node are contiguous in tree order, so a node is a run of chunks.  One
// block per (node, chunk): each warp keeps one group of terms in registers while its lanes
// run over the chunk's members (powers in registers, no shared-memory traffic per term);
// lanes are combined by shuffles and chunks per node in chunk order, so the result is
// deterministic (no floating-point atomics).
#include <algorithm>
#include <vector>

#include "common.cuh"

namespace bit {

namespace {

constexpr int MCH = 1024;  // members per chunk
constexpr int MTB = 256;   // threads per block: 8 warps = 4 term groups x 2 member halves

// The terms are split into MG groups of consecutive packed indices, cut at (i, j)
// boundaries (a run of k for one (i, j) stays in one group) and balanced by count.
constexpr int MG = 4;
template <int NT>
struct MomPlan {
  // packed index of (i, j, 0)
  static constexpr int start(int i, int j) {
    int s = 0;
    for (int a = 0; a < i; a++) s += (NT - a) * (NT - a + 1) / 2;
    for (int b = 0; b < j; b++) s += NT - i - b;
    return s;
  }
  // first packed index of group g (bound(MG) == T)
  static constexpr int bound(int g) {
    const int T = num_terms(NT);
    if (g <= 0) return 0;
    if (g >= MG) return T;
    for (int i = 0; i < NT; i++)
      for (int j = 0; j < NT - i; j++)
        if (start(i, j) * MG >= g * T) return start(i, j);
    return T;
  }
};

// One warp: the terms of group G for the chunk's members e0 + half*32 + lane + 64 r, with
// powers and accumulators in registers; the 32 lanes are summed by shuffles (fixed order).
template <int NT, int G>
__device__ __forceinline__ void moments_group(const double4* __restrict__ src, int e0, int e1,
                                              double4 c, int lane, int half, double* s_part) {
  constexpr int T0 = MomPlan<NT>::bound(G), T1 = MomPlan<NT>::bound(G + 1);
  constexpr int NG = T1 - T0;
  constexpr int TMAX = num_terms(kNtermsMax);
  if constexpr (NG > 0) {
    double acc[NG];
#pragma unroll
    for (int t = 0; t < NG; t++) acc[t] = 0.0;
    for (int e = e0 + half * 32 + lane; e < e1; e += 64) {
      const double4 s = src[e];
      const double dx = s.x - c.x, dy = s.y - c.y, dz = s.z - c.z;
      double py[NT], pz[NT];
      py[0] = 1.0;
      pz[0] = 1.0;
#pragma unroll
      for (int k = 1; k < NT; k++) {
        py[k] = py[k - 1] * dy;
        pz[k] = pz[k - 1] * dz;
      }
      double px = s.w;  // q dx^i
#pragma unroll
      for (int i = 0; i < NT; i++) {
#pragma unroll
        for (int j = 0; j < NT - i; j++) {
          const int st = MomPlan<NT>::start(i, j);
          if (st >= T0 && st < T1) {
            const double xy = px * py[j];
#pragma unroll
            for (int k = 0; k < NT - i - j; k++) acc[st - T0 + k] = fma(xy, pz[k], acc[st - T0 + k]);
          }
        }
        px *= dx;
      }
    }
#pragma unroll
    for (int t = 0; t < NG; t++) {
      double v = acc[t];
#pragma unroll
      for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) s_part[half * TMAX + T0 + t] = v;
    }
  }
}

// chunks: (node, first member, last member, chunk id); partials at part[id * TMAX + term].
// 8 warps: warp w takes term group w % 4 for the members of half w / 4.
template <int NT>
__global__ void __launch_bounds__(MTB) k_moments_partial(const int4* chunks, const double4* fld,
                                                         const double4* src, double* part) {
  constexpr int T = num_terms(NT);
  constexpr int TMAX = num_terms(kNtermsMax);
  __shared__ double s_part[2 * TMAX];
  const int4 ck = chunks[blockIdx.x];
  const double4 c = fld[ck.x];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = w & (MG - 1), half = w / MG;
  switch (g) {
    case 0: moments_group<NT, 0>(src, ck.y, ck.z, c, lane, half, s_part); break;
    case 1: moments_group<NT, 1>(src, ck.y, ck.z, c, lane, half, s_part); break;
    case 2: moments_group<NT, 2>(src, ck.y, ck.z, c, lane, half, s_part); break;
    default: moments_group<NT, 3>(src, ck.y, ck.z, c, lane, half, s_part); break;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < T; t += MTB)
    part[(long long)ck.w * TMAX + t] = s_part[t] + s_part[TMAX + t];
}

// Degree i + j + k of canonical moment index t (i outer, j, k inner, i + j + k < nt).
__device__ int canon_degree(int t, int nt) {
  int i = 0, j = 0;
  for (; t >= (nt - i) * (nt - i + 1) / 2; i++) t -= (nt - i) * (nt - i + 1) / 2;
  for (; t >= nt - i - j; j++) t -= nt - i - j;
  return i + j + t;
}

// Position of canonical moment index t in the far field's shell order: by degree d, then i
// descending, then j descending (the order gen_farfield.py's recurrences produce their
// coefficients in): the C(d + 2, 3) terms of lower degree, then (d - i)(d - i + 1) / 2 for
// the larger i of degree d, then d - i - j.
__device__ int canon_shell_pos(int t, int nt) {
  int i = 0, j = 0;
  for (; t >= (nt - i) * (nt - i + 1) / 2; i++) t -= (nt - i) * (nt - i + 1) / 2;
  for (; t >= nt - i - j; j++) t -= nt - i - j;
  const int d = i + j + t;
  return d * (d + 1) * (d + 2) / 6 + (d - i) * (d - i + 1) / 2 + (d - i - j);
}

constexpr int kReduceSlices = 4;  // chunk-sum slices per term (a top node has ~n/1024 chunks)

// Per node: the sum of its chunks' partials.  Slice k of term t sums chunks c0 + k,
// c0 + k + 4, ... in order and the slices are added in slice order, so the result is fixed;
// the slices shorten the serial sums of the top nodes, which set the kernel's length.
// The FP32 copy is normalised by h^degree, h = 2^mom32_scale_exp(sqradius) (exact: an
// exponent shift).
__global__ void __launch_bounds__(256 * kReduceSlices)
    k_moments_reduce(const int* node_c0, const int* node_c1, const int* node_T,
                     const long long* mom_off, const long long* msh_off, const double4* nodec,
                     const double* part, double* mom64, float* mom32, double* msh64,
                     float* msh32) {
  constexpr int TMAX = num_terms(kNtermsMax);
  static_assert(TMAX <= 256, "one slice of 256 threads covers every term");
  __shared__ double s_part[kReduceSlices][256];
  const int node = blockIdx.x;
  const int c0 = node_c0[node], c1 = node_c1[node], T = node_T[node];
  const int t = threadIdx.x & 255, slice = threadIdx.x >> 8;
  if (t < T) {
    double s = 0.0;
    for (int c = c0 + slice; c < c1; c += kReduceSlices) s += part[(long long)c * TMAX + t];
    s_part[slice][t] = s;
  }
  __syncthreads();
  if (slice != 0) return;
  const long long so = msh_off[node];
  if (t >= T) {
    if (t < (T + 3) / 4 * 4) { msh64[so + t] = 0.0; msh32[so + t] = 0.f; }  // block padding
    return;
  }
  double s = s_part[0][t];
  for (int k = 1; k < kReduceSlices; k++) s += s_part[k][t];
  int nt = 1;
  while (num_terms(nt) < T) nt++;
  const long long o = mom_off[node];
  const float s32 = (float)ldexp(s, -mom32_scale_exp(nodec[node].w) * canon_degree(t, nt));
  mom64[o + t] = s;
  mom32[o + t] = s32;
  const int p = canon_shell_pos(t, nt);
  msh64[so + p] = s;
  msh32[so + p] = s32;
}

__global__ void k_gather_charges(int n, const int* perm, const double* q, const double* w,
                                 const double* sx, const double* sy, const double* sz,
                                 double* sq, double* sw, double4* src64) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  int j = perm[e];
  double qq = q[j];
  sq[e] = qq;
  if (w) sw[e] = w[j];
  src64[e] = make_double4(sx[e], sy[e], sz[e], qq);
}

// FP32 sources in the coordinates of their own leaf's centre.
__global__ void k_leaf_local(int n, const int* leaf_of, const double4* nodec,
                             const double4* src64, float4* src32) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  double4 s = src64[e];
  double4 c = nodec[leaf_of[e]];
  src32[e] = make_float4((float)(s.x - c.x), (float)(s.y - c.y), (float)(s.z - c.z), (float)s.w);
}

template <int NT>
void launch_partial(int nch, const int4* ck, const double4* fld, const double4* src,
                    double* part, cudaStream_t s) {
  count_launch(), k_moments_partial<NT><<<nch, MTB, 0, s>>>(ck, fld, src, part);
}

}  // namespace

void tree_set_charges(Tree* t, const double* q, const double* w) {
  Ctx* c = t->ctx;
  cudaStream_t s = c->stream;
  const int n = t->n;
  t->sq.ensure(c, n);
  if (w) t->sw.ensure(c, n);
  t->src64.ensure(c, n);
  t->src32.ensure(c, n);
  count_launch(), k_gather_charges<<<grid_for(n, 256), 256, 0, s>>>(n, t->perm.p, q, w, t->sx.p, t->sy.p,
                                                    t->sz.p, t->sq.p, w ? t->sw.p : nullptr,
                                                    t->src64.p);
  count_launch(), k_leaf_local<<<grid_for(n, 256), 256, 0, s>>>(n, t->leaf_of.p, t->nodec.p, t->src64.p,
                                                t->src32.p);
  BIT_CHECK_LAUNCH();
  t->has_charges = true;
  t->has_weights = w != nullptr;
  t->has_moments = false;
}

void tree_moments(Tree* t, int nterms) {
  tree_moments_sys(t, std::vector<int>(t->nsys, nterms));
}

void tree_moments_sys(Tree* t, const std::vector<int>& nt_sys) {
  if ((int)nt_sys.size() != t->nsys) fail(BIT_ERR_INVALID_ARGUMENT, "one nterms per system expected");
  for (int v : nt_sys)
    if (v < 1 || v > kNtermsMax) fail(BIT_ERR_INVALID_ARGUMENT, "nterms out of range");
  if (!t->has_charges) fail(BIT_ERR_STATE, "charges not set");
  Ctx* c = t->ctx;
  cudaStream_t s = c->stream;
  constexpr int TMAX = num_terms(kNtermsMax);
  if (t->mplan_gen != t->gen || t->h_sys_nterms != nt_sys) {
    // chunks of every node, grouped by the node's nterms (one launch per distinct nterms)
    const int nn = t->numtree;
    std::vector<int> c0(nn), c1(nn), nodeT(nn);
    std::vector<long long> off(nn + 1, 0), soff(nn + 1, 0);
    for (int i = 0; i < nn; i++) {
      nodeT[i] = num_terms(nt_sys[t->h_node_sys[i]]);
      off[i + 1] = off[i] + nodeT[i];
      soff[i + 1] = soff[i] + (nodeT[i] + 3) / 4 * 4;
    }
    std::vector<int4> ck;
    std::vector<int> cls_begin(kNtermsMax + 2, 0);
    for (int k = 1; k <= kNtermsMax; k++) {
      cls_begin[k] = (int)ck.size();
      for (int i = 0; i < nn; i++) {
        if (nt_sys[t->h_node_sys[i]] != k) continue;
        c0[i] = (int)ck.size();
        int st = t->h_start[i], en = st + t->h_nummemb[i];
        for (int e = st; e < en; e += MCH) ck.push_back(make_int4(i, e, e + MCH < en ? e + MCH : en, 0));
        c1[i] = (int)ck.size();
      }
    }
    cls_begin[kNtermsMax + 1] = (int)ck.size();
    for (size_t q = 0; q < ck.size(); q++) ck[q].w = (int)q;
    t->mplan_cls = cls_begin;
    t->mplan_nch = (int)ck.size();
    t->h_mom_off.assign(off.begin(), off.end() - 1);
    t->mom_total = off[nn];
    t->msh_total = soff[nn];
    t->mplan_chunks.ensure(c, ck.size());
    t->mplan_c0.ensure(c, nn);
    t->mplan_c1.ensure(c, nn);
    t->mplan_T.ensure(c, nn);
    t->mom_off.ensure(c, nn);
    t->msh_off.ensure(c, nn);
    BIT_CUDA(cudaMemcpyAsync(t->mplan_chunks.p, ck.data(), ck.size() * sizeof(int4), cudaMemcpyHostToDevice, s));
    BIT_CUDA(cudaMemcpyAsync(t->mplan_c0.p, c0.data(), nn * sizeof(int), cudaMemcpyHostToDevice, s));
    BIT_CUDA(cudaMemcpyAsync(t->mplan_c1.p, c1.data(), nn * sizeof(int), cudaMemcpyHostToDevice, s));
    BIT_CUDA(cudaMemcpyAsync(t->mplan_T.p, nodeT.data(), nn * sizeof(int), cudaMemcpyHostToDevice, s));
    BIT_CUDA(cudaMemcpyAsync(t->mom_off.p, t->h_mom_off.data(), nn * sizeof(long long), cudaMemcpyHostToDevice, s));
    BIT_CUDA(cudaMemcpyAsync(t->msh_off.p, soff.data(), nn * sizeof(long long), cudaMemcpyHostToDevice, s));
    BIT_CUDA(cudaStreamSynchronize(s));
    t->mplan_gen = t->gen;
    t->h_sys_nterms = nt_sys;
  }
  t->mplan_part.ensure(c, (size_t)t->mplan_nch * TMAX);
  t->mom64.ensure(c, t->mom_total);
  t->mom32.ensure(c, t->mom_total);
  t->msh64.ensure(c, t->msh_total);
  t->msh32.ensure(c, t->msh_total);
  for (int k = 1; k <= kNtermsMax; k++) {
    const int b0 = t->mplan_cls[k], b1 = t->mplan_cls[k + 1];
    if (b1 == b0) continue;
    const int4* ckp = t->mplan_chunks.p + b0;
    switch (k) {
#define CASE(N) case N: launch_partial<N>(b1 - b0, ckp, t->nodec.p, t->src64.p, t->mplan_part.p, s); break;
      CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7) CASE(8) CASE(9) CASE(10)
#undef CASE
    }
  }
  count_launch(), k_moments_reduce<<<t->numtree, 256 * kReduceSlices, 0, s>>>(t->mplan_c0.p, t->mplan_c1.p, t->mplan_T.p,
                                                              t->mom_off.p, t->msh_off.p, t->nodec.p,
                                                              t->mplan_part.p, t->mom64.p,
                                                              t->mom32.p, t->msh64.p, t->msh32.p);
  BIT_CHECK_LAUNCH();
  int mx = 0;
  for (int v : nt_sys) mx = std::max(mx, v);
  t->nterms = mx;
  t->has_moments = true;
}

}  // namespace bit

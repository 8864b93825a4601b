// Cluster moments (treemoments, src/tree3d.cpp:2631-2711):
//   M_ijk(node) = sum over members q * dx^i dy^j dz^k,  i+j+k < nterms,
// about the node's box midpoint, in FP64 for every node.
//
// Members of every node are contiguous in tree order, so a node is a run of chunks.  One
// block per (node, chunk): members' powers are staged in shared memory and each thread
// owns one (i, j, k) term; per-chunk partial sums are then added per node in chunk order,
// so the result is deterministic (no floating-point atomics).
#include <algorithm>
#include <vector>

#include "common.cuh"

namespace bit {

namespace {

constexpr int MCH = 1024;  // members per chunk
constexpr int SUB = 128;   // members staged in shared memory at a time
constexpr int MTB = 256;   // threads per block (>= num_terms(10) = 220)

// chunks: (node, first member, last member, chunk id); partials at part[id * TMAX + term]
template <int NT>
__global__ void __launch_bounds__(MTB) k_moments_partial(const int4* chunks, const double4* fld,
                                                         const double4* src, double* part) {
  constexpr int T = num_terms(NT);
  constexpr int TMAX = num_terms(kNtermsMax);
  __shared__ double P[SUB][3 * NT];
  const int4 ck = chunks[blockIdx.x];
  const double4 c = fld[ck.x];
  int ti = 0, tj = 0, tk = 0;
  {
    int idx = 0;
    for (int i = 0; i < NT; i++)
      for (int j = 0; j < NT - i; j++)
        for (int k = 0; k < NT - i - j; k++) {
          if (idx == (int)threadIdx.x) { ti = i; tj = j; tk = k; }
          idx++;
        }
  }
  double acc = 0.0;
  for (int e0 = ck.y; e0 < ck.z; e0 += SUB) {
    const int cnt = min(SUB, ck.z - e0);
    if ((int)threadIdx.x < cnt) {
      double4 s = src[e0 + threadIdx.x];
      double dx = s.x - c.x, dy = s.y - c.y, dz = s.z - c.z;
      double px = s.w, py = 1.0, pz = 1.0;
#pragma unroll
      for (int i = 0; i < NT; i++) {
        P[threadIdx.x][i] = px;
        P[threadIdx.x][NT + i] = py;
        P[threadIdx.x][2 * NT + i] = pz;
        px *= dx; py *= dy; pz *= dz;
      }
    }
    __syncthreads();
    if ((int)threadIdx.x < T) {
      for (int e = 0; e < cnt; e++)
        acc = fma(P[e][ti] * P[e][NT + tj], P[e][2 * NT + tk], acc);
    }
    __syncthreads();
  }
  if ((int)threadIdx.x < T) part[(long long)ck.w * TMAX + threadIdx.x] = acc;
}

// Per node: the sum of its chunks' partials, in chunk order.
__global__ void k_moments_reduce(const int* node_c0, const int* node_c1, const int* node_T,
                                 const long long* mom_off, const double* part, double* mom64,
                                 float* mom32) {
  constexpr int TMAX = num_terms(kNtermsMax);
  const int node = blockIdx.x;
  const int c0 = node_c0[node], c1 = node_c1[node], T = node_T[node];
  const long long o = mom_off[node];
  for (int t = threadIdx.x; t < T; t += blockDim.x) {
    double s = 0.0;
    for (int c = c0; c < c1; c++) s += part[(long long)c * TMAX + t];
    mom64[o + t] = s;
    mom32[o + t] = (float)s;
  }
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
    std::vector<long long> off(nn + 1, 0);
    for (int i = 0; i < nn; i++) {
      nodeT[i] = num_terms(nt_sys[t->h_node_sys[i]]);
      off[i + 1] = off[i] + nodeT[i];
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
    t->mplan_chunks.ensure(c, ck.size());
    t->mplan_c0.ensure(c, nn);
    t->mplan_c1.ensure(c, nn);
    t->mplan_T.ensure(c, nn);
    t->mom_off.ensure(c, nn);
    BIT_CUDA(cudaMemcpyAsync(t->mplan_chunks.p, ck.data(), ck.size() * sizeof(int4), cudaMemcpyHostToDevice, s));
    BIT_CUDA(cudaMemcpyAsync(t->mplan_c0.p, c0.data(), nn * sizeof(int), cudaMemcpyHostToDevice, s));
    BIT_CUDA(cudaMemcpyAsync(t->mplan_c1.p, c1.data(), nn * sizeof(int), cudaMemcpyHostToDevice, s));
    BIT_CUDA(cudaMemcpyAsync(t->mplan_T.p, nodeT.data(), nn * sizeof(int), cudaMemcpyHostToDevice, s));
    BIT_CUDA(cudaMemcpyAsync(t->mom_off.p, t->h_mom_off.data(), nn * sizeof(long long), cudaMemcpyHostToDevice, s));
    BIT_CUDA(cudaStreamSynchronize(s));
    t->mplan_gen = t->gen;
    t->h_sys_nterms = nt_sys;
  }
  t->mplan_part.ensure(c, (size_t)t->mplan_nch * TMAX);
  t->mom64.ensure(c, t->mom_total);
  t->mom32.ensure(c, t->mom_total);
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
  count_launch(), k_moments_reduce<<<t->numtree, 256, 0, s>>>(t->mplan_c0.p, t->mplan_c1.p, t->mplan_T.p,
                                                              t->mom_off.p, t->mplan_part.p,
                                                              t->mom64.p, t->mom32.p);
  BIT_CHECK_LAUNCH();
  int mx = 0;
  for (int v : nt_sys) mx = std::max(mx, v);
  t->nterms = mx;
  t->has_moments = true;
}

}  // namespace bit

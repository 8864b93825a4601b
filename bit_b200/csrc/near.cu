// Near field: the leaf direct sums of treepotential / shielded_treepot / treeforce
// (src/tree3d.cpp:4737-4774, 3539-3623, 923-967), one CTA per target group.
//
// For each near entry (source leaf, bitmask over the group's targets) the CTA packs the
// targets that need the leaf into a dense list, and when fewer than half the threads
// would be busy it splits the leaf's sources across 2..32 threads per target (partial
// sums combined by warp shuffles).  Source tiles are staged in shared memory by TMA bulk
// copies (cp.async.bulk with an mbarrier), double buffered so the next tile streams in
// while the current one is consumed; every thread then reads each source from shared
// memory, broadcast across the targets.  Accumulation per target is in shared memory in a
// fixed order, so results are deterministic.
//
// FP64 path: the reference's arithmetic.  Mixed path: sources in FP32 relative to their
// leaf centre, the target's offset from that centre formed in FP64 and rounded once, MUFU
// rsqrt / ex2, and per-target compensated (two-sum) accumulation.
#include <climits>

#include "common.cuh"
#include "tma.cuh"

namespace bit {

namespace {

constexpr int NT = 256;  // threads per CTA

struct NearArgs {
  const int *order, *g_tstart, *g_tcount, *g_own;
  const double *tx, *ty, *tz;
  const long long *off, *moff;
  const int* cnt;
  const int* node;
  const unsigned* mask;
  const int *start, *nummemb;
  const double4* nodec;
  const void* src;  // float4 (mixed) or double4 (FP64) in tree order
  const double4* src64;
  const double* sw;
  const SysEval* sys;  // per system: near_del, kappa, intg, near_sign, self_term, particles
  const int* g_sys;    // per group: system
  double *out, *out_y, *out_z;  // potential, or the three field components
  int* err;
};

__device__ __forceinline__ float rsqrt_approx(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
// Knuth two-sum: s + e accumulates b with the rounding error of each step kept in e.
__device__ __forceinline__ void two_sum(float& s, float& e, float b) {
  float t = s + b;
  float bp = t - s;
  e += (s - (t - bp)) + (b - bp);
  s = t;
}

template <bool F32>
struct Prec;
template <>
struct Prec<true> {
  using S = float4;
  using T = float;
  static constexpr int TILE = 1024;
};
template <>
struct Prec<false> {
  using S = double4;
  using T = double;
  static constexpr int TILE = 512;
};

// One pair's contribution.  Mixed: target and source relative to the source leaf centre.
template <int KER, bool EPS>
__device__ __forceinline__ float pair(float xt, float yt, float zt, float4 s, float del,
                                      float kl2) {
  const float dx = s.x - xt, dy = s.y - yt, dz = s.z - zt;
  const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, del)));
  const float ri = rsqrt_approx(r2);
  float v = KER == BIT_KERNEL_COULOMB ? s.w * ri : s.w * ex2_approx(r2 * ri * kl2) * ri;
  if (EPS && !(r2 > (float)kEpsNear)) v = 0.f;
  return v;
}
template <int KER, bool EPS>
__device__ __forceinline__ double pair(double x, double y, double z, double4 s, double del,
                                       double kappa) {
  const double dx = x - s.x, dy = y - s.y, dz = z - s.z;
  const double r2 = dx * dx + dy * dy + dz * dz + del;
  if (EPS && !(r2 > kEpsNear)) return 0.0;
  if (KER == BIT_KERNEL_COULOMB) return s.w / sqrt(r2);
  const double r = sqrt(r2);
  return s.w * exp(-kappa * r) / r;
}
// Field of eval_grad_kernel_reg (src/tree3d.cpp:73-97), KERNEL_ORDER = 0:
// q * (-(x_j - x) / (r * r^2)).
__device__ __forceinline__ void fpair(float xt, float yt, float zt, float4 s, float del,
                                      float& ax, float& ay, float& az) {
  const float dx = xt - s.x, dy = yt - s.y, dz = zt - s.z;
  const float rs = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, del)));
  const float ri = rsqrt_approx(rs);
  const float tq = s.w * ri * ri * ri;
  ax = fmaf(dx, tq, ax); ay = fmaf(dy, tq, ay); az = fmaf(dz, tq, az);
}
__device__ __forceinline__ void fpair(double x, double y, double z, double4 s, double del,
                                      double& ax, double& ay, double& az) {
  const double dx = s.x - x, dy = s.y - y, dz = s.z - z;
  const double rs = dx * dx + dy * dy + dz * dz + del;
  const double r = sqrt(rs);
  const double t = s.w / (r * rs);
  ax -= dx * t; ay -= dy * t; az -= dz * t;
}

template <class T>
__device__ __forceinline__ T shfl_sum(T v, int tpt) {
  for (int o = tpt >> 1; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Shared-memory layout of one CTA.
template <bool F32, bool FORCE>
struct Smem {
  using S = typename Prec<F32>::S;
  static constexpr int TILE = Prec<F32>::TILE;
  static constexpr int NACC = FORCE ? 3 : 1;
  static constexpr size_t tiles = 2 * TILE * sizeof(S);
  static constexpr size_t coords = 0;  // target coordinates are read through L1
  // mixed: float hi + lo per target; FP64: one double; force: three doubles
  static constexpr size_t acc = (FORCE ? 3 : 1) * kGroupMax * sizeof(double);
  static constexpr size_t self = kGroupMax * sizeof(double);
  static constexpr size_t list = kGroupMax * sizeof(int);
  static constexpr size_t bars = 64;
  static constexpr size_t total = tiles + coords + acc + self + list + bars;
};

// The whole near field of one group.  FORCE: the three field components instead of the
// potential (Coulomb only).
template <int KER, bool EPS, bool F32, bool FORCE>
__global__ void __launch_bounds__(NT) k_near(NearArgs a) {
  using P = Prec<F32>;
  using S = typename P::S;
  using T = typename P::T;
  using L = Smem<F32, FORCE>;
  constexpr int TILE = P::TILE;
  extern __shared__ __align__(128) unsigned char sm[];
  S* tiles = reinterpret_cast<S*>(sm);
  const double* cx = a.tx + 0;  // group targets, indexed t0 + i below
  const double* cy = a.ty + 0;
  const double* cz = a.tz + 0;
  double* accd = reinterpret_cast<double*>(sm + L::tiles + L::coords);
  float* acch = reinterpret_cast<float*>(accd);  // mixed: hi [0,1024), lo [1024,2048)
  double* selfv = reinterpret_cast<double*>(sm + L::tiles + L::coords + L::acc);
  int* tl = reinterpret_cast<int*>(sm + L::tiles + L::coords + L::acc + L::self);
  uint64_t* bar =
      reinterpret_cast<uint64_t*>(sm + L::tiles + L::coords + L::acc + L::self + L::list);
  __shared__ int s_cnt;

  const int g = a.order[blockIdx.x];
  const int t0 = a.g_tstart[g], tc = a.g_tcount[g];
  const SysEval* se = a.sys + a.g_sys[g];
  const double sdel = se->near_del, skappa = se->kappa;
  const int own = se->particles ? a.g_own[g] : -1;
  const int W = (tc + 31) >> 5;
  const long long e0 = a.off[g], e1 = e0 + a.cnt[g];
  const long long m0 = a.moff[g];
  const int tid = threadIdx.x, lane = tid & 31;
  for (int i = tid; i < tc; i += NT) selfv[i] = 0.0;
  // the whole accumulator block (the mixed path views it as float hi / lo rows)
  for (int k = tid; k < L::NACC * kGroupMax; k += NT) accd[k] = 0.0;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (e0 < e1) {
    const S* src = reinterpret_cast<const S*>(a.src);
    const float del = (float)sdel;
    const float kl2 = (float)(-skappa * 1.4426950408889634);  // -kappa*log2(e)
    // job iterator: (entry e, first source of the tile in the entry's leaf)
    long long e = e0;
    int node = a.node[e];
    int j0 = a.start[node], jn = a.nummemb[node];
    int toff = 0;
    if (tid == 0) {
      const int cnt0 = min(TILE, jn);
      fence_proxy_async();
      mbar_expect_tx(&bar[0], cnt0 * (unsigned)sizeof(S));
      tma_load_1d(tiles, src + j0, cnt0 * (unsigned)sizeof(S), &bar[0]);
    }
    int k = 0, tpt = 1, cnt = 0;
    while (true) {
      const int buf = k & 1;
      const int ns = min(TILE, jn - toff);
      if (toff == 0 && tid < 32) {
        // pack the targets of this entry (warp 0)
        unsigned wd = lane < W ? a.mask[m0 + (e - e0) * W + lane] : 0u;
        const int c = __popc(wd);
        int pre = c;
        for (int o = 1; o < 32; o <<= 1) {
          int t = __shfl_up_sync(0xffffffffu, pre, o);
          if (lane >= o) pre += t;
        }
        int base = pre - c;
        while (wd) {
          const int b = __ffs(wd) - 1;
          wd &= wd - 1;
          tl[base++] = 32 * lane + b;
        }
        if (lane == 31) s_cnt = pre;
      }
      // the next job streams into the other buffer while this one is consumed
      long long ne = e;
      int noff = toff + TILE;
      if (noff >= jn) { ne = e + 1; noff = 0; }
      if (tid == 0 && ne < e1) {
        const int nd = a.node[ne];
        const int cntn = min(TILE, a.nummemb[nd] - noff);
        fence_proxy_async();
        mbar_expect_tx(&bar[buf ^ 1], cntn * (unsigned)sizeof(S));
        tma_load_1d(tiles + (buf ^ 1) * TILE, src + a.start[nd] + noff,
                    cntn * (unsigned)sizeof(S), &bar[buf ^ 1]);
      }
      __syncthreads();
      if (toff == 0) {
        cnt = s_cnt;
        tpt = 1;
        while (tpt < 32 && cnt * tpt * 2 <= NT) tpt <<= 1;
      }
      if (!mbar_wait(&bar[buf], (k >> 1) & 1)) {
        if (tid == 0) atomicOr(a.err, 2);
        if (ne < e1) mbar_wait(&bar[buf ^ 1], ((k + 1) >> 1) & 1);  // let the other copy land
        return;
      }
      const S* ts = tiles + buf * TILE;
      const double4 c = a.nodec[node];
      // tile index of target i's own source is i + selfbase (particle targets, own leaf)
      const int selfbase = (node == own) ? (t0 - (j0 + toff)) : INT_MIN;
      const int units = cnt * tpt;
      const int lt = __ffs(tpt) - 1;
      for (int u0 = 0; u0 < units; u0 += NT) {
        const int u = u0 + tid;
        const bool valid = u < units;
        const int slot = u >> lt, slice = u & (tpt - 1);
        const int i = valid ? tl[slot] : 0;
        const int selfj = selfbase == INT_MIN ? -1 : i + selfbase;
        if (!FORCE) {
          T part = 0;
          if (valid) {
            if constexpr (F32) {
              const float4* fs = reinterpret_cast<const float4*>(ts);
              const float xt = (float)(cx[t0 + i] - c.x), yt = (float)(cy[t0 + i] - c.y),
                          zt = (float)(cz[t0 + i] - c.z);
              float p0 = 0.f, p1 = 0.f;
              int j = slice;
              for (; j + tpt < ns; j += 2 * tpt) {
                const float v0 = pair<KER, EPS>(xt, yt, zt, fs[j], del, kl2);
                const float v1 = pair<KER, EPS>(xt, yt, zt, fs[j + tpt], del, kl2);
                p0 += (j == selfj) ? 0.f : v0;
                p1 += (j + tpt == selfj) ? 0.f : v1;
              }
              if (j < ns && j != selfj) p0 += pair<KER, EPS>(xt, yt, zt, fs[j], del, kl2);
              part = p0 + p1;
            } else {
              const double4* ds = reinterpret_cast<const double4*>(ts);
              double p = 0.0;
              const double x = cx[t0 + i], y = cy[t0 + i], z = cz[t0 + i];
              for (int j = slice; j < ns; j += tpt)
                if (j != selfj) p += pair<KER, EPS>(x, y, z, ds[j], sdel, skappa);
              part = p;
            }
            if (se->self_term && selfj >= 0 && selfj < ns && ((selfj - slice) & (tpt - 1)) == 0) {
              const int jg = j0 + toff + selfj;  // added, not subtracted (src/tree3d.cpp:3596)
              selfv[i] = a.src64[jg].w * se->intg / (a.sw ? a.sw[jg] : 1.0);
            }
          }
          part = shfl_sum(part, tpt);
          if (valid && slice == 0) {
            if constexpr (F32) two_sum(acch[i], acch[kGroupMax + i], (float)part);
            else accd[i] += (double)part;
          }
        } else {
          T fx = 0, fy = 0, fz = 0;
          if (valid) {
            if constexpr (F32) {
              const float4* fs = reinterpret_cast<const float4*>(ts);
              const float xt = (float)(cx[t0 + i] - c.x), yt = (float)(cy[t0 + i] - c.y),
                          zt = (float)(cz[t0 + i] - c.z);
              for (int j = slice; j < ns; j += tpt)
                if (j != selfj) fpair(xt, yt, zt, fs[j], del, fx, fy, fz);
            } else {
              const double4* ds = reinterpret_cast<const double4*>(ts);
              const double x = cx[t0 + i], y = cy[t0 + i], z = cz[t0 + i];
              for (int j = slice; j < ns; j += tpt)
                if (j != selfj) fpair(x, y, z, ds[j], sdel, fx, fy, fz);
            }
          }
          fx = shfl_sum(fx, tpt);
          fy = shfl_sum(fy, tpt);
          fz = shfl_sum(fz, tpt);
          if (valid && slice == 0) {
            accd[i] += (double)fx;
            accd[kGroupMax + i] += (double)fy;
            accd[2 * kGroupMax + i] += (double)fz;
          }
        }
      }
      __syncthreads();
      k++;
      if (ne >= e1) break;
      if (ne != e) {
        e = ne;
        node = a.node[e];
        j0 = a.start[node];
        jn = a.nummemb[node];
      }
      toff = noff;
    }
  }
  __syncthreads();
  for (int i = tid; i < tc; i += NT) {
    if (FORCE) {
      a.out[t0 + i] += accd[i];
      a.out_y[t0 + i] += accd[kGroupMax + i];
      a.out_z[t0 + i] += accd[2 * kGroupMax + i];
    } else if (F32) {
      a.out[t0 + i] += se->near_sign * ((double)acch[i] + (double)acch[kGroupMax + i]) + selfv[i];
    } else {
      a.out[t0 + i] += se->near_sign * accd[i] + selfv[i];
    }
  }
}

template <int KER, bool EPS, bool F32, bool FORCE>
void launch(const NearArgs& a, int ngroups, cudaStream_t s) {
  constexpr size_t bytes = Smem<F32, FORCE>::total;
  static int done[64] = {0};  // once per kernel and device
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && !done[dev]) {
    BIT_CUDA(cudaFuncSetAttribute(k_near<KER, EPS, F32, FORCE>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    done[dev] = 1;
  }
  count_launch(), k_near<KER, EPS, F32, FORCE><<<ngroups, NT, bytes, s>>>(a);
}

NearArgs base_args(Tree* t, Lists* L, const EvalPlan& P, const double* tx, const double* ty,
                   const double* tz) {
  NearArgs a{};
  a.g_tstart = L->g_tstart.p;
  a.g_tcount = L->g_tcount.p;
  a.g_own = L->g_own.p;
  a.tx = tx; a.ty = ty; a.tz = tz;
  a.off = L->near_off.p;
  a.cnt = L->near_cnt.p;
  a.moff = L->near_moff.p;
  a.node = L->near_node.p;
  a.mask = L->near_mask.p;
  a.start = t->start.p;
  a.nummemb = t->nummemb.p;
  a.nodec = t->nodec.p;
  a.src = P.f32 ? (const void*)t->src32.p : (const void*)t->src64.p;
  a.src64 = t->src64.p;
  a.sw = t->has_weights ? t->sw.p : nullptr;
  a.sys = P.sys.p;
  a.g_sys = L->g_sys.p;
  a.err = t->ctx->dev_err();
  return a;
}

}  // namespace

// One launch per (kernel, eps check) class, each over its groups (P.near_ord + begin).
void eval_near(Tree* t, Lists* L, const EvalPlan& P, const double* tx, const double* ty,
               const double* tz, double* out) {
  cudaStream_t s = t->ctx->stream;
  NearArgs a = base_args(t, L, P, tx, ty, tz);
  a.out = out;
  const bool f32 = P.f32;
  for (const LaunchClass& k : P.near_classes) {
    a.order = P.near_ord + k.begin;
    const int ng = k.count;
    const bool scr = k.kernel != BIT_KERNEL_COULOMB;
    const bool eps = k.eps != 0;
#define GO(K, E, F) launch<K, E, F, false>(a, ng, s)
    if (f32) {
      if (!scr) { if (eps) GO(BIT_KERNEL_COULOMB, true, true); else GO(BIT_KERNEL_COULOMB, false, true); }
      else { if (eps) GO(BIT_KERNEL_SCREENED, true, true); else GO(BIT_KERNEL_SCREENED, false, true); }
    } else {
      if (!scr) { if (eps) GO(BIT_KERNEL_COULOMB, true, false); else GO(BIT_KERNEL_COULOMB, false, false); }
      else { if (eps) GO(BIT_KERNEL_SCREENED, true, false); else GO(BIT_KERNEL_SCREENED, false, false); }
    }
#undef GO
    BIT_CHECK_LAUNCH();
  }
}

void eval_near_force(Tree* t, Lists* L, const EvalPlan& P, double* fx, double* fy, double* fz) {
  cudaStream_t s = t->ctx->stream;
  NearArgs a = base_args(t, L, P, t->sx.p, t->sy.p, t->sz.p);
  a.out = fx; a.out_y = fy; a.out_z = fz;
  for (const LaunchClass& k : P.near_classes) {
    a.order = P.near_ord + k.begin;
    if (P.f32) launch<BIT_KERNEL_COULOMB, false, true, true>(a, k.count, s);
    else launch<BIT_KERNEL_COULOMB, false, false, true>(a, k.count, s);
    BIT_CHECK_LAUNCH();
  }
}

}  // namespace bit

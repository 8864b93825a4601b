// Near field: the leaf direct sums of treepotential / shielded_treepot / treeforce
// (src/tree3d.cpp:4737-4774, 3539-3623, 923-967), one CTA per target group.
//
// For each near entry (source leaf, bitmask over the group's targets) the CTA packs the
// targets that need the leaf into a dense list and splits the leaf's sources across 1..32
// threads per target, whichever keeps the most threads busy (partial sums combined by
// warp shuffles).  Source tiles are staged in shared memory by TMA bulk
// copies (cp.async.bulk with an mbarrier), double buffered so the next tile streams in
// while the current one is consumed; every thread then reads each source from shared
// memory, broadcast across the targets.  Accumulation per target is in shared memory in a
// fixed order, so results are deterministic.
//
// FP64 path: the reference's arithmetic.  Mixed path: sources in FP32 relative to their
// leaf centre, the target's offset from that centre formed in FP64 and rounded once, MUFU
// rsqrt / ex2, and per-target compensated (two-sum) accumulation; pairs too close for FP32
// coordinates are summed in FP64 (below).  The self pair is skipped by splitting each
// lane's index range around it.
#include <algorithm>
#include <climits>

#include "common.cuh"
#include "fp64math.cuh"
#include "tma.cuh"

namespace bit {

namespace {

constexpr int NT = 256;  // threads per CTA

struct NearArgs {
  const int *order, *g_tstart, *g_tcount;
  const double *tx, *ty, *tz;
  const long long *off, *moff;
  const int* cnt;
  const int* node;
  const unsigned* mask;
  const int *start, *nummemb;
  const double4* nodec;
  const void* src;  // float4 (mixed) or double4 (FP64) in tree order
  const double4* src64;
  const float4* nodeh;  // per node: half extents of the box, rounded up
  const double* sw;
  const SysEval* sys;  // per system: near_del, kappa, intg, near_sign, self_term, particles
  const int* g_sys;    // per group: system
  double *out, *out_y, *out_z;  // potential, or the three field components
  int* err;
  // mixed potentials: close pairs left out of the FP32 sums, per target (k_close)
  int* ccnt;    // tiles recorded for the target
  int2* crec;   // up to kCloseRec (near entry, first source of the tile) per target
  int2* clist;  // (target, group) of every target with a record
  int* cn;      // entries of clist
  int tile;     // sources per tile (Prec<>::TILE_MIN..TILE_MAX)
  int split;    // threads per target: 0 the precision's rule, else at most this many
};

constexpr int kCloseRec = 2;  // record slots per target; beyond them k_close scans them all

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
// Source tile (records per TMA copy): the default, and the range a context may choose
// (bit_ctx_set_near_config); shared memory holds two tiles.
template <>
struct Prec<true> {
  using S = float4;
  using T = float;
  static constexpr int TILE = 1024, TILE_MIN = 256, TILE_MAX = 2048;
};
template <>
struct Prec<false> {
  using S = double4;
  using T = double;
  static constexpr int TILE = 512, TILE_MIN = 128, TILE_MAX = 1024;
};

// One pair's contribution in FP64, added to acc: the reference's q / sqrt(r^2) and
// q e^{-kappa r} / r (src/tree3d.cpp:4765-4769, 3609-3618).  1/r comes from a refined
// reciprocal square root (rsqrt_nr, within an ulp of 1/sqrt) in place of a square root
// and a division, the exponential from a branch-free exp (exp_tang, within an ulp), so
// that the unrolled pairs of a sweep interleave; r^2 + del is one FMA chain, and the
// Coulomb pair folds q and the accumulation into the Newton step's last FMA.  At 2M
// clustered, p = 8, theta = 0.7, the screened FP64 near field takes 21.2 ms against 26.2
// ms with CUDA's exp and rsqrt and the plain forms, the Coulomb one 10.8 against 12.1 ms
// (the same tuned tiles); the results move by about 2e-16 (relative L2).  EPS: a pair with
// r^2 <= 1e-14 adds nothing.  SMALL: kappa r < kSmallExpArg, the exponential's
// small-argument form (no underflow check; the same value).
template <int KER, bool EPS, bool SMALL = false>
__device__ __forceinline__ void pair_acc(double x, double y, double z, double4 s, double del,
                                         double kappa, double& acc) {
  const double dx = x - s.x, dy = y - s.y, dz = z - s.z;
  const double r2 = fma(dx, dx, fma(dy, dy, fma(dz, dz, del)));
  double q = s.w, rr = r2;
  if (EPS) {
    const bool skip = !(r2 > kEpsNear);
    q = skip ? 0.0 : q;
    rr = skip ? 1.0 : rr;
  }
  double y0;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y0) : "d"(rr));
  // one third-order Newton step, as rsqrt_nr: y0 (1 + e c), e = 1 - rr y0^2, c = 1/2 + 3e/8
  const double e = fma(-rr * y0, y0, 1.0);
  const double ec = e * fma(e, 0.375, 0.5);
  if (KER == BIT_KERNEL_COULOMB) {
    const double qy = q * y0;
    acc = fma(qy, ec, acc + qy);
  } else {
    const double ri = fma(y0, ec, y0);
    acc = fma(q * exp_tang<SMALL>(-kappa * (rr * ri)), ri, acc);
  }
}
// Field of eval_grad_kernel_reg (src/tree3d.cpp:73-97), KERNEL_ORDER = 0:
// q * (-(x_j - x) / (r * r^2)).
__device__ __forceinline__ void fpair(double x, double y, double z, double4 s, double del,
                                      double& ax, double& ay, double& az) {
  const double dx = s.x - x, dy = s.y - y, dz = s.z - z;
  const double rs = dx * dx + dy * dy + dz * dz + del;
  const double r = sqrt(rs);
  const double t = s.w / (r * rs);
  ax -= dx * t; ay -= dy * t; az -= dz * t;
}
// The same with the reference's KERNEL_ORDER family (eval_grad_kernel_reg,
// src/tree3d.cpp:80-91): 1/(r rs) plus korder terms, each the previous one times
// (l + 1/2)/l * del/rs.
__device__ __forceinline__ void fpair_order(double x, double y, double z, double4 s, double del,
                                            int korder, double& ax, double& ay, double& az) {
  const double dx = s.x - x, dy = s.y - y, dz = s.z - z;
  const double rs = dx * dx + dy * dy + dz * dz + del;
  const double r = sqrt(rs);
  double temp = 1.0 / (r * rs), f = temp;
  for (int l = 1; l <= korder; l++) {
    f = f * (l + 0.5) / l * del / rs;
    temp += f;
  }
  const double t = s.w * temp;
  ax -= dx * t; ay -= dy * t; az -= dz * t;
}
// Screened 2-D field of one pair (shielded_treeforce's leaf loop, src/tree3d.cpp:3384-3398):
// t = q e^{-kappa r} / r^2 (kappa + 1/r), fx -= dy t, fy += dx t, no del.
__device__ __forceinline__ void cpair(double x, double y, double z, double4 s, double kappa,
                                      double& ax, double& ay) {
  const double dx = x - s.x, dy = y - s.y, dz = z - s.z;
  const double rs = dx * dx + dy * dy + dz * dz;
  const double r = sqrt(rs);
  const double t = s.w * exp(-kappa * r) / rs * (kappa + 1 / r);
  ax -= dy * t; ay += dx * t;
}

template <class T>
__device__ __forceinline__ T shfl_sum(T v, int tpt) {
  for (int o = tpt >> 1; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Close pairs in the mixed path.  FP32 leaf-centred coordinates carry an absolute error of
// about 6e-8 of their magnitude, so a pair much closer than the leaf's size loses relative
// accuracy in its FP32 difference (two particles 1e-4 apart in a leaf of size 0.1 give
// ~1e-5).  Pairs closer than r_t = 1/32 of the source leaf's radius (r^2 below thr) are
// left out of the FP32 sum and summed in FP64 from the FP64 sources instead, with the
// reference's rules (including its r^2 <= 1e-14 skip, which only such pairs can meet:
// thr >= 2e-14).  Every other pair keeps at most ~4e-6 relative error, far below 1e-6 of a
// target's total.  Close pairs can only occur where a target lies within r_t of the source
// leaf's box (its own leaf, or a neighbour's boundary), and only where the kernel's del is
// below thr (FP32 r^2 >= del), so a warp runs the checked loop on those tiles and the plain
// loop, with no test at all, everywhere else.
constexpr float kCloseFrac = 1.0f / 1024.0f;  // (1/32)^2
constexpr float kThrMin = 2e-14f;             // above the 1e-14 skip of src/constants.h:35

// Squared distance from a point (relative to a leaf's centre) to the leaf's box (half
// extents h, rounded up); 0 inside.
__device__ __forceinline__ float box_d2(float x, float y, float z, float4 h) {
  const float dx = fmaxf(fabsf(x) - h.x, 0.f), dy = fmaxf(fabsf(y) - h.y, 0.f),
              dz = fmaxf(fabsf(z) - h.z, 0.f);
  return dx * dx + dy * dy + dz * dz;
}

// FP32 r^2 of a pair (identical wherever it is formed, so the FP32 and FP64 sums split the
// pairs exactly).
__device__ __forceinline__ float r2_32(float xt, float yt, float zt, float4 s, float del) {
  const float dx = s.x - xt, dy = s.y - yt, dz = s.z - zt;
  return fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, del)));
}

// p += q * G(r); CHK: pairs with r^2 < thr are left out and flagged.
template <int KER, bool CHK>
__device__ __forceinline__ void acc_pot(float xt, float yt, float zt, float4 s, float del,
                                        float kl2, float thr, float& p, bool& close) {
  float r2 = r2_32(xt, yt, zt, s, del);
  float q = s.w;
  if (CHK) {
    const bool cl = r2 < thr;
    close |= cl;
    q = cl ? 0.f : q;
    r2 = cl ? 1.f : r2;
  }
  const float ri = rsqrt_approx(r2);
  if (KER == BIT_KERNEL_COULOMB) p = fmaf(q, ri, p);
  else p = fmaf(q * ri, ex2_approx(r2 * ri * kl2), p);
}

// FP64: this lane's pairs j, j + tpt, ... < je (the target's own source excluded by the
// caller's split of the range), eight pairs per iteration into four independent
// accumulators so that consecutive pairs do not wait on one another's additions.  SMALL:
// kappa r < kSmallExpArg for every pair (exp_tang's small-argument form).
template <int KER, bool EPS, bool SMALL = false>
__device__ __forceinline__ void sweep_pot64(const double4* ds, int j, int je, int tpt, double x,
                                            double y, double z, double del, double kappa,
                                            double& p0, double& p1) {
  double p2 = 0.0, p3 = 0.0;
  for (; j + 7 * tpt < je; j += 8 * tpt) {
    pair_acc<KER, EPS, SMALL>(x, y, z, ds[j], del, kappa, p0);
    pair_acc<KER, EPS, SMALL>(x, y, z, ds[j + tpt], del, kappa, p1);
    pair_acc<KER, EPS, SMALL>(x, y, z, ds[j + 2 * tpt], del, kappa, p2);
    pair_acc<KER, EPS, SMALL>(x, y, z, ds[j + 3 * tpt], del, kappa, p3);
    pair_acc<KER, EPS, SMALL>(x, y, z, ds[j + 4 * tpt], del, kappa, p0);
    pair_acc<KER, EPS, SMALL>(x, y, z, ds[j + 5 * tpt], del, kappa, p1);
    pair_acc<KER, EPS, SMALL>(x, y, z, ds[j + 6 * tpt], del, kappa, p2);
    pair_acc<KER, EPS, SMALL>(x, y, z, ds[j + 7 * tpt], del, kappa, p3);
  }
  for (; j < je; j += tpt) pair_acc<KER, EPS, SMALL>(x, y, z, ds[j], del, kappa, p0);
  p0 += p2;
  p1 += p3;
}

// This lane's pairs j = jb, jb + tpt, ... < je, eight per iteration into four independent
// accumulators (against four per iteration: Coulomb 4.13 -> 3.89 ms at 2M).  Both
// exponentials and reciprocal square roots stay on the MUFU: moving 1, 2 or 3 of every 8
// screened exponentials to the FMA pipe (a Cody-Waite / minimax exp2) measured 3-12%
// slower at 2M, since this loop is bound by latency and issue, not by MUFU throughput.
template <int KER, bool CHK>
__device__ __forceinline__ void sweep_pot(const float4* fs, int j, int je, int tpt, float xt,
                                          float yt, float zt, float del, float kl2, float thr,
                                          float& p0, float& p1, bool& close) {
  float p2 = 0.f, p3 = 0.f;
  for (; j + 7 * tpt < je; j += 8 * tpt) {
    acc_pot<KER, CHK>(xt, yt, zt, fs[j], del, kl2, thr, p0, close);
    acc_pot<KER, CHK>(xt, yt, zt, fs[j + tpt], del, kl2, thr, p1, close);
    acc_pot<KER, CHK>(xt, yt, zt, fs[j + 2 * tpt], del, kl2, thr, p2, close);
    acc_pot<KER, CHK>(xt, yt, zt, fs[j + 3 * tpt], del, kl2, thr, p3, close);
    acc_pot<KER, CHK>(xt, yt, zt, fs[j + 4 * tpt], del, kl2, thr, p0, close);
    acc_pot<KER, CHK>(xt, yt, zt, fs[j + 5 * tpt], del, kl2, thr, p1, close);
    acc_pot<KER, CHK>(xt, yt, zt, fs[j + 6 * tpt], del, kl2, thr, p2, close);
    acc_pot<KER, CHK>(xt, yt, zt, fs[j + 7 * tpt], del, kl2, thr, p3, close);
  }
  for (; j < je; j += tpt) acc_pot<KER, CHK>(xt, yt, zt, fs[j], del, kl2, thr, p0, close);
  p1 += p2 + p3;
}

// Target t left close pairs out of this job's FP32 sum (near entry e, tile at toff).  One
// thread handles a target per job, and the CTA's jobs are separated by barriers, so the
// target's records need no atomics and come in job order.
__device__ __forceinline__ void record_close(const NearArgs& a, int t, int g, long long e,
                                             int toff) {
  const int c = a.ccnt[t];
  if (c < kCloseRec) a.crec[(long long)t * kCloseRec + c] = make_int2((int)e, toff);
  a.ccnt[t] = c + 1;
  if (c == 0) a.clist[atomicAdd(a.cn, 1)] = make_int2(t, g);
}

// Field of one pair, q (x - x_j) / r^3 (eval_grad_kernel_reg, src/tree3d.cpp:73-97,
// KERNEL_ORDER = 0); CHK as acc_pot.
template <bool CHK>
__device__ __forceinline__ void acc_force(float xt, float yt, float zt, float4 s, float del,
                                          float thr, float& ax, float& ay, float& az,
                                          bool& close) {
  const float dx = xt - s.x, dy = yt - s.y, dz = zt - s.z;
  float rs = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, del)));
  float q = s.w;
  if (CHK) {
    const bool cl = rs < thr;
    close |= cl;
    q = cl ? 0.f : q;
    rs = cl ? 1.f : rs;
  }
  const float ri = rsqrt_approx(rs);
  const float tq = q * ri * ri * ri;
  ax = fmaf(dx, tq, ax); ay = fmaf(dy, tq, ay); az = fmaf(dz, tq, az);
}

__device__ __forceinline__ void close_force(float xt, float yt, float zt, double x, double y,
                                         double z, const float4* fs, const double4* s64,
                                         int slice, int tpt, int ns, int selfj, float del,
                                         float thr, double del64, double& cx, double& cy,
                                         double& cz) {
  for (int j = slice; j < ns; j += tpt)
    if (j != selfj && r2_32(xt, yt, zt, fs[j], del) < thr) fpair(x, y, z, s64[j], del64, cx, cy, cz);
}

// Threads per target for an entry with cnt targets.  FP64 pairs (slow arithmetic): the
// power of two (1..32) that keeps the most of the CTA's threads busy over the rounds of NT
// units (a larger split must win by 4% to be taken, since it adds a shuffle reduction and
// shortens each thread's run).  FP32 pairs are cheap enough that the per-unit overhead
// weighs more: split only until half the threads are busy (measured: the utilisation rule
// gains 1.5% on 2M clustered screened targets but loses 14% on 82k-node BIE matvecs).
// cap > 0 (a tuned setting): the utilisation rule over 1..cap threads.
template <bool CHEAP>
__device__ __forceinline__ int split_for(int cnt, int cap) {
  if (CHEAP && cap == 0) {
    int tpt = 1;
    while (tpt < 32 && cnt * tpt * 2 <= NT) tpt <<= 1;
    return tpt;
  }
  const int maxtp = cap > 0 ? cap : 32;
  int best = 1;
  float bu = 0.f;
  for (int tp = 1; tp <= maxtp; tp <<= 1) {
    const int units = cnt * tp;
    const int rounds = (units + NT - 1) / NT;
    const float util = (float)units / (float)(rounds * NT);
    if (util > bu + 0.04f) {
      bu = util;
      best = tp;
    }
  }
  return best;
}

// Shared-memory layout of one CTA: two source tiles of `tile` records, then the
// accumulators, the self terms, the packed target list and the mbarriers (target
// coordinates are read through L1).
template <bool F32, bool FORCE>
struct Smem {
  using S = typename Prec<F32>::S;
  static constexpr int NACC = FORCE ? 3 : 1;
  // mixed: float hi + lo per target; FP64: one double; force: three doubles
  static constexpr size_t acc = (FORCE ? 3 : 1) * kGroupMax * sizeof(double);
  static constexpr size_t self = kGroupMax * sizeof(double);
  static constexpr size_t list = kGroupMax * sizeof(int);
  static constexpr size_t bars = 64;
  __host__ __device__ static size_t tiles(int tile) { return 2 * (size_t)tile * sizeof(S); }
  __host__ __device__ static size_t total(int tile) { return tiles(tile) + acc + self + list + bars; }
};

// The whole near field of group g, by the whole CTA.  FORCE: the three field components
// instead of the potential.  Returns false (in every thread) if a bounded wait gave up:
// the error flag is set, and the CTA has waited, bounded again, for its copies in flight.
template <int KER, bool EPS, bool F32, bool FORCE>
__device__ __forceinline__ bool near_group(const NearArgs& a, int g) {
  using P = Prec<F32>;
  using S = typename P::S;
  using T = typename P::T;
  using L = Smem<F32, FORCE>;
  const int TILE = a.tile;
  extern __shared__ __align__(128) unsigned char sm[];
  S* tiles = reinterpret_cast<S*>(sm);
  const double* cx = a.tx + 0;  // group targets, indexed t0 + i below
  const double* cy = a.ty + 0;
  const double* cz = a.tz + 0;
  unsigned char* rest = sm + L::tiles(TILE);
  double* accd = reinterpret_cast<double*>(rest);
  float* acch = reinterpret_cast<float*>(accd);  // mixed: hi [0,1024), lo [1024,2048)
  double* selfv = reinterpret_cast<double*>(rest + L::acc);
  int* tl = reinterpret_cast<int*>(rest + L::acc + L::self);
  uint64_t* bar = reinterpret_cast<uint64_t*>(rest + L::acc + L::self + L::list);
  __shared__ int s_cnt;

  const int t0 = a.g_tstart[g], tc = a.g_tcount[g];
  const SysEval* se = a.sys + a.g_sys[g];
  const double sdel = se->near_del, skappa = se->kappa;
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
      // Every thread waits (bounded) for this job's tile; the barrier then combines the
      // outcomes, so the whole CTA takes the same branch.  On a timeout the CTA waits,
      // bounded again, for both copies it may still have in flight into its shared memory
      // before it returns, and the host reports the error flag.
      const bool landed = mbar_wait(&bar[buf], (k >> 1) & 1);
      if (__syncthreads_or(!landed)) {
        if (tid == 0) {
          atomicOr(a.err, 2);
          mbar_wait(&bar[buf], (k >> 1) & 1);
          if (ne < e1) mbar_wait(&bar[buf ^ 1], ((k + 1) >> 1) & 1);
        }
        __syncthreads();
        return false;
      }
      if (toff == 0) {
        cnt = s_cnt;
        tpt = split_for<F32 && !FORCE>(cnt, a.split);
      }
      const S* ts = tiles + buf * TILE;
      const double4 c = a.nodec[node];
      // Particle targets: target i's own source sits at its sorted position t0 + i, i.e.
      // at tile index i + selfbase, which is inside this tile only if the target is one
      // of the tile's sources.
      const int selfbase = se->particles ? (t0 - (j0 + toff)) : INT_MIN;
      const int units = cnt * tpt;
      const int lt = __ffs(tpt) - 1;
      // close-pair checks are needed only where a target comes within r_t of this leaf's box
      float thr = fmaxf((float)c.w * kCloseFrac, kThrMin);  // r_t^2 = sqradius / 1024
      // the FP32 r^2 is at least del (fmaf of non-negative squares onto del), so where del
      // reaches thr no pair of this tile can be close: thr = 0 keeps every warp on the
      // plain loop (no box distance is below 0), which is then exact
      if (!(del < thr)) thr = 0.f;
      const float4 hb = a.nodeh[node];
      const double4* s64 = a.src64 + j0 + toff;
      for (int u0 = 0; u0 < units; u0 += NT) {
        const int u = u0 + tid;
        const bool valid = u < units;
        const int slot = u >> lt, slice = u & (tpt - 1);
        const int i = valid ? tl[slot] : 0;
        const int selfj = selfbase == INT_MIN ? -1 : i + selfbase;
        // the target's own source in this lane's slice: sum around it
        const bool self_in = selfj >= 0 && selfj < ns && ((selfj - slice) & (tpt - 1)) == 0;
        const int je = self_in ? selfj : ns;
        if (!FORCE) {
          T part = 0;
          bool close = false;  // mixed: a pair of this lane was left for the FP64 pass
          if constexpr (F32) {
            const float4* fs = reinterpret_cast<const float4*>(ts);
            const float xt = (float)(cx[t0 + i] - c.x), yt = (float)(cy[t0 + i] - c.y),
                        zt = (float)(cz[t0 + i] - c.z);
            const bool chk = __any_sync(0xffffffffu, valid && box_d2(xt, yt, zt, hb) < thr);
            if (valid) {
              float p0 = 0.f, p1 = 0.f;
              if (!chk) {
                sweep_pot<KER, false>(fs, slice, je, tpt, xt, yt, zt, del, kl2, thr, p0, p1, close);
                if (self_in)
                  sweep_pot<KER, false>(fs, selfj + tpt, ns, tpt, xt, yt, zt, del, kl2, thr, p0, p1, close);
              } else {
                sweep_pot<KER, true>(fs, slice, je, tpt, xt, yt, zt, del, kl2, thr, p0, p1, close);
                if (self_in)
                  sweep_pot<KER, true>(fs, selfj + tpt, ns, tpt, xt, yt, zt, del, kl2, thr, p0, p1, close);
              }
              part = p0 + p1;
            }
          } else {
            // screened: kappa r stays below kSmallExpArg for every pair of this warp's
            // targets and tile if it does at r^2 = dmax^2 + del, dmax the target's distance
            // to the leaf centre plus the leaf's half diagonal (a warp-uniform choice of
            // the exp form)
            bool small = false;
            if (KER == BIT_KERNEL_SCREENED) {
              const double ox = cx[t0 + i] - c.x, oy = cy[t0 + i] - c.y, oz = cz[t0 + i] - c.z;
              const double dmax = sqrt(fma(ox, ox, fma(oy, oy, oz * oz))) + sqrt(c.w);
              small = __all_sync(0xffffffffu, !valid || skappa * sqrt(fma(dmax, dmax, sdel)) < kSmallExpArg);
            }
            if (valid) {
              const double4* ds = reinterpret_cast<const double4*>(ts);
              double p0 = 0.0, p1 = 0.0;
              const double x = cx[t0 + i], y = cy[t0 + i], z = cz[t0 + i];
              if (small) {
                sweep_pot64<KER, EPS, true>(ds, slice, je, tpt, x, y, z, sdel, skappa, p0, p1);
                if (self_in) sweep_pot64<KER, EPS, true>(ds, selfj + tpt, ns, tpt, x, y, z, sdel, skappa, p0, p1);
              } else {
                sweep_pot64<KER, EPS>(ds, slice, je, tpt, x, y, z, sdel, skappa, p0, p1);
                if (self_in) sweep_pot64<KER, EPS>(ds, selfj + tpt, ns, tpt, x, y, z, sdel, skappa, p0, p1);
              }
              part = p0 + p1;
            }
          }
          if (valid && se->self_term && self_in) {
            const int jg = j0 + toff + selfj;  // added, not subtracted (src/tree3d.cpp:3596)
            selfv[i] = a.src64[jg].w * se->intg / (a.sw ? a.sw[jg] : 1.0);
          }
          part = shfl_sum(part, tpt);
          if (valid && slice == 0) {
            if constexpr (F32) two_sum(acch[i], acch[kGroupMax + i], (float)part);
            else accd[i] += (double)part;
          }
          if constexpr (F32) {
            if (a.ccnt) {  // (null where no pair can be close)
              // a target's tpt slices share a warp: one record per target and tile
              for (int o = tpt >> 1; o; o >>= 1) close |= __shfl_xor_sync(0xffffffffu, (int)close, o) != 0;
              if (valid && slice == 0 && close) record_close(a, t0 + i, g, e, toff);
            }
          }
        } else {
          T fx = 0, fy = 0, fz = 0;
          if constexpr (F32) {
            const float4* fs = reinterpret_cast<const float4*>(ts);
            const float xt = (float)(cx[t0 + i] - c.x), yt = (float)(cy[t0 + i] - c.y),
                        zt = (float)(cz[t0 + i] - c.z);
            const bool chk = __any_sync(0xffffffffu, valid && box_d2(xt, yt, zt, hb) < thr);
            if (valid) {
              bool close = false;
              if (!chk) {
                for (int j = slice; j < je; j += tpt)
                  acc_force<false>(xt, yt, zt, fs[j], del, thr, fx, fy, fz, close);
                if (self_in)
                  for (int j = selfj + tpt; j < ns; j += tpt)
                    acc_force<false>(xt, yt, zt, fs[j], del, thr, fx, fy, fz, close);
              } else {
                for (int j = slice; j < je; j += tpt)
                  acc_force<true>(xt, yt, zt, fs[j], del, thr, fx, fy, fz, close);
                if (self_in)
                  for (int j = selfj + tpt; j < ns; j += tpt)
                    acc_force<true>(xt, yt, zt, fs[j], del, thr, fx, fy, fz, close);
              }
              if (close) {
                double qx = 0.0, qy = 0.0, qz = 0.0;
                close_force(xt, yt, zt, cx[t0 + i], cy[t0 + i], cz[t0 + i], fs, s64, slice, tpt,
                            ns, selfj, del, thr, sdel, qx, qy, qz);
                fx += (float)qx; fy += (float)qy; fz += (float)qz;
              }
            }
          } else {
            if (valid) {
              const double4* ds = reinterpret_cast<const double4*>(ts);
              const double x = cx[t0 + i], y = cy[t0 + i], z = cz[t0 + i];
              const int korder = se->kernel_order;
              if (KER == BIT_KERNEL_SCREENED) {
                for (int j = slice; j < ns; j += tpt)
                  if (j != selfj) cpair(x, y, z, ds[j], skappa, fx, fy);
              } else if (korder > 0) {
                for (int j = slice; j < ns; j += tpt)
                  if (j != selfj) fpair_order(x, y, z, ds[j], sdel, korder, fx, fy, fz);
              } else {
                for (int j = slice; j < ns; j += tpt)
                  if (j != selfj) fpair(x, y, z, ds[j], sdel, fx, fy, fz);
              }
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
  return true;
}

// One launch class: CTA b takes group order[b].  Potential kernels keep four CTAs per SM
// (64 registers; the FP64 one chose 72 and three CTAs unconstrained, 4% slower at 2M),
// except the mixed screened one, which runs three (85 registers): at 2M clustered, p = 8,
// theta = 0.7, 6.43 -> 6.13 ms, while the mixed Coulomb one went 3.92 -> 4.26 ms with three.
template <int KER, bool EPS, bool F32, bool FORCE>
__global__ void __launch_bounds__(NT, FORCE ? 0 : ((F32 && KER == BIT_KERNEL_SCREENED) ? 3 : 4))
    k_near(NearArgs a) {
  near_group<KER, EPS, F32, FORCE>(a, a.order[blockIdx.x]);
}

// Persistent work queue over the groups of every class of a potential evaluation: each CTA
// takes the next item (a group, in the given order) from a device counter until none is
// left and runs near_group for that group's kernel and eps rule -- the same device code as
// k_near, so the results are identical.  A CTA whose bounded wait gave up stops taking
// items (the host reports the error flag).
template <bool F32>
__global__ void __launch_bounds__(NT, 4) k_near_queue(NearArgs a, int count, int* head) {
  __shared__ int s_item;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(head, 1);
    __syncthreads();
    const int item = s_item;
    __syncthreads();  // every thread has read s_item before it is overwritten
    if (item >= count) return;
    const int g = a.order[item];
    const SysEval* se = a.sys + a.g_sys[g];
    bool ok;
    if (se->kernel == BIT_KERNEL_COULOMB) {
      ok = se->eps_check ? near_group<BIT_KERNEL_COULOMB, true, F32, false>(a, g)
                         : near_group<BIT_KERNEL_COULOMB, false, F32, false>(a, g);
    } else {
      ok = se->eps_check ? near_group<BIT_KERNEL_SCREENED, true, F32, false>(a, g)
                         : near_group<BIT_KERNEL_SCREENED, false, F32, false>(a, g);
    }
    if (!ok) return;
    __syncthreads();  // the group's last reads of shared memory precede the next group's writes
  }
}

template <int KER, bool EPS, bool F32, bool FORCE>
void launch(const NearArgs& a, int ngroups, cudaStream_t s) {
  const size_t bytes = Smem<F32, FORCE>::total(a.tile);
  ensure_smem_attr(reinterpret_cast<const void*>(k_near<KER, EPS, F32, FORCE>),
                   (int)Smem<F32, FORCE>::total(Prec<F32>::TILE_MAX));
  count_launch(), k_near<KER, EPS, F32, FORCE><<<ngroups, NT, bytes, s>>>(a);
}

template <bool F32>
void launch_queue(Ctx* c, const NearArgs& a, int count, cudaStream_t s) {
  const size_t bytes = Smem<F32, false>::total(a.tile);
  ensure_smem_attr(reinterpret_cast<const void*>(k_near_queue<F32>),
                   (int)Smem<F32, false>::total(Prec<F32>::TILE_MAX));
  int per_sm = 0;
  BIT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_near_queue<F32>, NT, bytes));
  const int grid = std::max(1, std::min(count, c->num_sms * std::max(per_sm, 1)));
  c->queue_heads.ensure(c, 2);
  BIT_CUDA(cudaMemsetAsync(c->queue_heads.p + 1, 0, sizeof(int), s));
  count_launch(), k_near_queue<F32><<<grid, NT, bytes, s>>>(a, count, c->queue_heads.p + 1);
}

// FP64 sum of the close pairs that the mixed near kernel left out (FP32 r^2 < thr, the
// target's own source excluded), one warp per recorded target: the recorded tiles in job
// order, or, for a target with more tiles than record slots, every near entry of its group
// that covers it (tiles without close pairs add nothing, so the sum is the same).  Lanes
// take the sources in the kernel's order and the warp reduces in a fixed order, so the
// result does not depend on scheduling.
template <int KER, bool EPS>
__device__ double close_sum(const NearArgs& a, const SysEval* se, int t, int g, double x,
                            double y, double z) {
  const int lane = threadIdx.x & 31;
  const double sdel = se->near_del, skappa = se->kappa;
  const float del = (float)sdel;
  const int self = se->particles ? t : -1;  // sorted position of the target's own source
  const float4* fs = reinterpret_cast<const float4*>(a.src);
  double acc = 0.0;
  auto tile = [&](int node, int j0, int j1) {
    const double4 c = a.nodec[node];
    const float xt = (float)(x - c.x), yt = (float)(y - c.y), zt = (float)(z - c.z);
    const float thr = fmaxf((float)c.w * kCloseFrac, kThrMin);
    const int s0 = a.start[node];
    for (int j = s0 + j0 + lane; j < s0 + j1; j += 32)
      if (j != self && r2_32(xt, yt, zt, fs[j], del) < thr)
        pair_acc<KER, EPS>(x, y, z, a.src64[j], sdel, skappa, acc);
  };
  const int nrec = a.ccnt[t];
  if (nrec <= kCloseRec) {
    for (int k = 0; k < nrec; k++) {
      const int2 r = a.crec[(long long)t * kCloseRec + k];
      const int node = a.node[r.x];
      tile(node, r.y, min(r.y + a.tile, a.nummemb[node]));
    }
  } else {
    const int i = t - a.g_tstart[g], W = (a.g_tcount[g] + 31) >> 5;
    const long long e0 = a.off[g], e1 = e0 + a.cnt[g], m0 = a.moff[g];
    for (long long e = e0; e < e1; e++)
      if ((a.mask[m0 + (e - e0) * W + (i >> 5)] >> (i & 31)) & 1u) {
        const int node = a.node[e];
        tile(node, 0, a.nummemb[node]);
      }
  }
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  return acc;
}

__global__ void __launch_bounds__(256) k_close(NearArgs a) {
  const int lane = threadIdx.x & 31;
  const int n = *a.cn;
  for (int w = blockIdx.x * 8 + (threadIdx.x >> 5); w < n; w += gridDim.x * 8) {
    const int2 tg = a.clist[w];
    const int t = tg.x, g = tg.y;
    const SysEval* se = a.sys + a.g_sys[g];
    const double x = a.tx[t], y = a.ty[t], z = a.tz[t];
    double v;
    if (se->kernel == BIT_KERNEL_COULOMB)
      v = se->eps_check ? close_sum<BIT_KERNEL_COULOMB, true>(a, se, t, g, x, y, z)
                        : close_sum<BIT_KERNEL_COULOMB, false>(a, se, t, g, x, y, z);
    else
      v = se->eps_check ? close_sum<BIT_KERNEL_SCREENED, true>(a, se, t, g, x, y, z)
                        : close_sum<BIT_KERNEL_SCREENED, false>(a, se, t, g, x, y, z);
    if (lane == 0) a.out[t] += se->near_sign * v;
  }
}

NearArgs base_args(Tree* t, Lists* L, const EvalPlan& P, const double* tx, const double* ty,
                   const double* tz) {
  NearArgs a{};
  a.g_tstart = L->g_tstart.p;
  a.g_tcount = L->g_tcount.p;
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
  a.nodeh = t->nodeh.p;
  a.sw = t->has_weights ? t->sw.p : nullptr;
  a.sys = P.sys.p;
  a.g_sys = L->g_sys.p;
  a.err = t->ctx->dev_err();
  // the context's tile, clamped to the precision's range (0: the default)
  const int want = t->ctx->near_tile;
  const int lo = P.f32 ? Prec<true>::TILE_MIN : Prec<false>::TILE_MIN;
  const int hi = P.f32 ? Prec<true>::TILE_MAX : Prec<false>::TILE_MAX;
  a.tile = want == 0 ? (P.f32 ? Prec<true>::TILE : Prec<false>::TILE) : std::min(hi, std::max(lo, want));
  a.split = t->ctx->near_split;
  return a;
}

}  // namespace

// One launch per (kernel, eps check) class, each over its groups (P.near_ord + begin).
void eval_near(Tree* t, Lists* L, const EvalPlan& P, const double* tx, const double* ty,
               const double* tz, double* out) {
  Ctx* c = t->ctx;
  cudaStream_t s = c->stream;
  NearArgs a = base_args(t, L, P, tx, ty, tz);
  a.out = out;
  // Mixed: close pairs need r^2 < thr = max(sqradius / 1024, 2e-14) of some leaf, and the
  // FP32 r^2 is at least the system's del (a rounded sum of non-negative terms and del);
  // where del reaches the largest leaf threshold no pair can be close, and the records
  // and the FP64 pass are skipped.
  bool close_possible = false;
  if (P.f32)
    for (size_t sy = 0; sy < P.h_sys.size(); sy++) {
      const float thr_max = fmaxf((float)t->h_sys_leaf_sqr[sy] * kCloseFrac, kThrMin);
      close_possible |= (float)P.h_sys[sy].near_del < thr_max;
    }
  const bool f32 = P.f32;
  if (close_possible) {
    // close-pair records, cleared for this evaluation (k_close consumes them)
    const int nt = L->ntargets;
    if (L->nnear >= INT_MAX) fail(BIT_ERR_CAPACITY, "too many near entries");
    c->close_cnt.ensure(c, nt);
    c->close_rec.ensure(c, (size_t)nt * kCloseRec);
    c->close_list.ensure(c, nt);
    c->close_n.ensure(c, 1);
    BIT_CUDA(cudaMemsetAsync(c->close_cnt.p, 0, (size_t)nt * sizeof(int), s));
    BIT_CUDA(cudaMemsetAsync(c->close_n.p, 0, sizeof(int), s));
    a.ccnt = c->close_cnt.p;
    a.crec = c->close_rec.p;
    a.clist = c->close_list.p;
    a.cn = c->close_n.p;
  }
  // several classes (a forest): one persistent launch over a work queue of all groups
  if (c->work_queue && P.near_classes.size() > 1) {
    int count = 0;
    for (const LaunchClass& k : P.near_classes) count += k.count;
    a.order = L->order.p;
    if (f32) launch_queue<true>(c, a, count, s);
    else launch_queue<false>(c, a, count, s);
    BIT_CHECK_LAUNCH();
  }
  for (const LaunchClass& k : P.near_classes) {
    if (c->work_queue && P.near_classes.size() > 1) break;
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
  if (close_possible) {
    count_launch(), k_close<<<c->num_sms * 4, 256, 0, s>>>(a);
    BIT_CHECK_LAUNCH();
  }
}

void eval_near_force(Tree* t, Lists* L, const EvalPlan& P, double* fx, double* fy, double* fz) {
  cudaStream_t s = t->ctx->stream;
  NearArgs a = base_args(t, L, P, t->sx.p, t->sy.p, t->sz.p);
  a.out = fx; a.out_y = fy; a.out_z = fz;
  // P.force: 1 the regularised Coulomb field (kernel order per system; FP64 beyond order
  // 0), 2 the screened 2-D field of shielded_treeforce (FP64)
  for (const LaunchClass& k : P.near_classes) {
    a.order = P.near_ord + k.begin;
    if (P.force == 2) {
      if (P.f32) fail(BIT_ERR_INVALID_ARGUMENT, "the screened field is FP64 only");
      launch<BIT_KERNEL_SCREENED, false, false, true>(a, k.count, s);
    } else if (P.f32) {
      launch<BIT_KERNEL_COULOMB, false, true, true>(a, k.count, s);
    } else {
      launch<BIT_KERNEL_COULOMB, false, false, true>(a, k.count, s);
    }
    BIT_CHECK_LAUNCH();
  }
}

}  // namespace bit

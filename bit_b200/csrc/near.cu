// Near field: the leaf direct sums of treepotential / shielded_treepot / treeforce
// (src/tree3d.cpp:4737-4774, 3539-3623, 923-967) over each batch's near entries.
//
// One warp per batch, one target per lane; the leaf's sources are contiguous in tree
// order and every active lane reads the same source at the same time (one broadcast
// transaction).  FP64 path: the reference's arithmetic.  Mixed path: sources in FP32
// relative to their leaf centre, the target's offset from that centre formed in FP64 and
// rounded once, MUFU rsqrt / ex2, and per-target compensated (two-sum) accumulation of
// 8-term partial sums.
#include "common.cuh"

namespace bit {

namespace {

constexpr int NWARPS = 4;

struct NearSpec {
  double del;    // added to r^2
  double kappa;
  double intg;   // reference-mode screened self term
  int eps_check; // skip r^2 <= 1e-14
  int self_term; // 1: add q*intg/w for j == p
  int sign;      // +1 / -1
  int particles; // targets are the sources (self excluded by position)
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
// Knuth two-sum: s + e == a + b exactly.
__device__ __forceinline__ void two_sum(float& s, float& e, float b) {
  float t = s + b;
  float bp = t - s;
  e += (s - (t - bp)) + (b - bp);
  s = t;
}

// Self handling of particle targets: the batch's own leaf is the one near entry that
// can contain the target itself; every other entry runs without a per-source check.
template <int KER, bool EPS>
__device__ __forceinline__ double pair64(double x, double y, double z, double4 s, double del,
                                         double kappa) {
  const double dx = x - s.x, dy = y - s.y, dz = z - s.z;
  const double r2 = dx * dx + dy * dy + dz * dz + del;
  if (EPS && !(r2 > kEpsNear)) return 0.0;
  if (KER == BIT_KERNEL_COULOMB) return s.w / sqrt(r2);
  const double r = sqrt(r2);
  return s.w * exp(-kappa * r) / r;
}

template <int KER, bool EPS>
__global__ void __launch_bounds__(32 * NWARPS)
    k_near64(int nbatch, const int* order, const int* b_tstart, const int* b_tcount,
             const int* b_leaf, const double* tx, const double* ty, const double* tz,
             const long long* off, const int2* ent, const int* start, const int* nummemb,
             const double4* src, const double* sw, NearSpec sp, double* out) {
  const int lane = threadIdx.x & 31;
  const int wi = blockIdx.x * NWARPS + (threadIdx.x >> 5);
  if (wi >= nbatch) return;
  const int b = order[wi];
  const int t0 = b_tstart[b], tc = b_tcount[b];
  const int own = sp.particles ? b_leaf[b] : -1;
  const bool live = lane < tc;
  const int tpos = sp.particles ? t0 + lane : -1;
  double x = 0, y = 0, z = 0;
  if (live) { x = tx[t0 + lane]; y = ty[t0 + lane]; z = tz[t0 + lane]; }
  double acc = 0.0, self = 0.0;
  for (long long e = off[b]; e < off[b + 1]; e++) {
    const int2 en = ent[e];
    if (!((unsigned(en.y) >> lane) & 1u)) continue;
    const int j0 = start[en.x], j1 = j0 + nummemb[en.x];
    if (en.x == own) {
      for (int j = j0; j < j1; j++) {
        const double4 s = src[j];
        if (j == tpos) {
          // added, not subtracted, by the reference (src/tree3d.cpp:3596)
          if (sp.self_term) self += s.w * sp.intg / (sw ? sw[j] : 1.0);
          continue;
        }
        acc += pair64<KER, EPS>(x, y, z, s, sp.del, sp.kappa);
      }
      continue;
    }
    int j = j0;
    for (; j + 4 <= j1; j += 4) {
      double4 s[4];
#pragma unroll
      for (int k = 0; k < 4; k++) s[k] = src[j + k];
#pragma unroll
      for (int k = 0; k < 4; k++) acc += pair64<KER, EPS>(x, y, z, s[k], sp.del, sp.kappa);
    }
    for (; j < j1; j++) acc += pair64<KER, EPS>(x, y, z, src[j], sp.del, sp.kappa);
  }
  if (live) out[t0 + lane] += sp.sign * acc + self;
}

template <int KER, bool EPS>
__device__ __forceinline__ float pair32(float xt, float yt, float zt, float4 s, float del,
                                        float kl2) {
  const float dx = s.x - xt, dy = s.y - yt, dz = s.z - zt;
  const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, del)));
  const float ri = rsqrt_approx(r2);
  float v;
  if (KER == BIT_KERNEL_COULOMB) v = s.w * ri;
  else v = s.w * ex2_approx(r2 * ri * kl2) * ri;
  if (EPS && !(r2 > (float)kEpsNear)) v = 0.f;
  return v;
}

template <int KER, bool EPS>
__global__ void __launch_bounds__(32 * NWARPS)
    k_near32(int nbatch, const int* order, const int* b_tstart, const int* b_tcount,
             const int* b_leaf, const double* tx, const double* ty, const double* tz,
             const long long* off, const int2* ent, const int* start, const int* nummemb,
             const double4* nodec, const float4* __restrict__ src, const double4* src64,
             const double* sw, NearSpec sp, double* out) {
  const int lane = threadIdx.x & 31;
  const int wi = blockIdx.x * NWARPS + (threadIdx.x >> 5);
  if (wi >= nbatch) return;
  const int b = order[wi];
  const int t0 = b_tstart[b], tc = b_tcount[b];
  const int own = sp.particles ? b_leaf[b] : -1;
  const bool live = lane < tc;
  const int tpos = sp.particles ? t0 + lane : -1;
  double x = 0, y = 0, z = 0;
  if (live) { x = tx[t0 + lane]; y = ty[t0 + lane]; z = tz[t0 + lane]; }
  const float del = (float)sp.del;
  const float kl2 = (float)(-sp.kappa * 1.4426950408889634);  // -kappa * log2(e)
  float hi = 0.f, lo = 0.f;
  double self = 0.0;
  for (long long e = off[b]; e < off[b + 1]; e++) {
    const int2 en = ent[e];
    if (!((unsigned(en.y) >> lane) & 1u)) continue;
    const double4 c = nodec[en.x];
    const float xt = (float)(x - c.x), yt = (float)(y - c.y), zt = (float)(z - c.z);
    const int j0 = start[en.x], j1 = j0 + nummemb[en.x];
    if (en.x == own) {
      for (int jb = j0; jb < j1; jb += 8) {
        float part = 0.f;
        const int je = min(jb + 8, j1);
        for (int j = jb; j < je; j++) {
          if (j == tpos) {
            if (sp.self_term) self += src64[j].w * sp.intg / (sw ? sw[j] : 1.0);
            continue;
          }
          part += pair32<KER, EPS>(xt, yt, zt, src[j], del, kl2);
        }
        two_sum(hi, lo, part);
      }
      continue;
    }
    int j = j0;
    for (; j + 8 <= j1; j += 8) {
      float4 s[8];
#pragma unroll
      for (int k = 0; k < 8; k++) s[k] = src[j + k];
      float p0 = 0.f, p1 = 0.f;
#pragma unroll
      for (int k = 0; k < 8; k += 2) {
        p0 += pair32<KER, EPS>(xt, yt, zt, s[k], del, kl2);
        p1 += pair32<KER, EPS>(xt, yt, zt, s[k + 1], del, kl2);
      }
      two_sum(hi, lo, p0 + p1);
    }
    float part = 0.f;
    for (; j < j1; j++) part += pair32<KER, EPS>(xt, yt, zt, src[j], del, kl2);
    two_sum(hi, lo, part);
  }
  if (live) out[t0 + lane] += sp.sign * ((double)hi + (double)lo) + self;
}

// Field of the regularised Coulomb kernel, eval_grad_kernel_reg (src/tree3d.cpp:73-97)
// with KERNEL_ORDER = 0: f += q * (-(x_j - x) / (r * r^2)), r^2 = |x_j - x|^2 + del.
__global__ void __launch_bounds__(32 * NWARPS)
    k_near_force64(int nbatch, const int* order, const int* b_tstart, const int* b_tcount,
                   const double* tx, const double* ty, const double* tz, const long long* off,
                   const int2* ent, const int* start, const int* nummemb, const double4* src,
                   double del, int particles, double* fx, double* fy, double* fz) {
  const int lane = threadIdx.x & 31;
  const int wi = blockIdx.x * NWARPS + (threadIdx.x >> 5);
  if (wi >= nbatch) return;
  const int b = order[wi];
  const int t0 = b_tstart[b], tc = b_tcount[b];
  const bool live = lane < tc;
  const int tpos = particles ? t0 + lane : -1;
  double x = 0, y = 0, z = 0;
  if (live) { x = tx[t0 + lane]; y = ty[t0 + lane]; z = tz[t0 + lane]; }
  double ax = 0, ay = 0, az = 0;
  for (long long e = off[b]; e < off[b + 1]; e++) {
    const int2 en = ent[e];
    if (!((unsigned(en.y) >> lane) & 1u)) continue;
    const int j0 = start[en.x], j1 = j0 + nummemb[en.x];
    for (int j = j0; j < j1; j++) {
      if (j == tpos) continue;
      const double4 s = src[j];
      const double dx = s.x - x, dy = s.y - y, dz = s.z - z;
      const double rs = dx * dx + dy * dy + dz * dz + del;
      const double r = sqrt(rs);
      const double temp = s.w / (r * rs);
      ax -= dx * temp;
      ay -= dy * temp;
      az -= dz * temp;
    }
  }
  if (live) { fx[t0 + lane] += ax; fy[t0 + lane] += ay; fz[t0 + lane] += az; }
}

__global__ void __launch_bounds__(32 * NWARPS)
    k_near_force32(int nbatch, const int* order, const int* b_tstart, const int* b_tcount,
                   const double* tx, const double* ty, const double* tz, const long long* off,
                   const int2* ent, const int* start, const int* nummemb, const double4* nodec,
                   const float4* src, double del, int particles, double* fx, double* fy,
                   double* fz) {
  const int lane = threadIdx.x & 31;
  const int wi = blockIdx.x * NWARPS + (threadIdx.x >> 5);
  if (wi >= nbatch) return;
  const int b = order[wi];
  const int t0 = b_tstart[b], tc = b_tcount[b];
  const bool live = lane < tc;
  const int tpos = particles ? t0 + lane : -1;
  double x = 0, y = 0, z = 0;
  if (live) { x = tx[t0 + lane]; y = ty[t0 + lane]; z = tz[t0 + lane]; }
  const float d = (float)del;
  float h[3] = {0, 0, 0}, l[3] = {0, 0, 0};
  for (long long e = off[b]; e < off[b + 1]; e++) {
    const int2 en = ent[e];
    if (!((unsigned(en.y) >> lane) & 1u)) continue;
    const double4 c = nodec[en.x];
    const float xt = (float)(x - c.x), yt = (float)(y - c.y), zt = (float)(z - c.z);
    const int j0 = start[en.x], j1 = j0 + nummemb[en.x];
    for (int jb = j0; jb < j1; jb += 8) {
      float p[3] = {0, 0, 0};
      const int je = min(jb + 8, j1);
      for (int j = jb; j < je; j++) {
        if (j == tpos) continue;
        const float4 s = src[j];
        const float dx = s.x - xt, dy = s.y - yt, dz = s.z - zt;
        const float rs = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, d)));
        const float ri = rsqrt_approx(rs);
        const float tq = s.w * ri * ri * ri;
        p[0] = fmaf(-dx, tq, p[0]);
        p[1] = fmaf(-dy, tq, p[1]);
        p[2] = fmaf(-dz, tq, p[2]);
      }
      for (int a = 0; a < 3; a++) two_sum(h[a], l[a], p[a]);
    }
  }
  if (live) {
    fx[t0 + lane] += (double)h[0] + (double)l[0];
    fy[t0 + lane] += (double)h[1] + (double)l[1];
    fz[t0 + lane] += (double)h[2] + (double)l[2];
  }
}

NearSpec make_spec(const bit_eval_params& p, int points) {
  NearSpec s{};
  const bool ref = p.mode == BIT_MODE_REFERENCE;
  s.kappa = p.kappa;
  s.intg = p.intg;
  s.particles = !points;
  switch (p.kernel) {
    case BIT_KERNEL_COULOMB:
      // src/tree3d.cpp:4744-4772: points use del, particles drop it (reference mode)
      s.del = (points || !ref) ? p.del : 0.0;
      s.eps_check = 1;
      s.sign = 1;
      break;
    case BIT_KERNEL_SCREENED:
      s.del = 0.0;
      s.eps_check = points ? 1 : 0;          // :3557 / :3604-3619
      s.sign = (points && ref) ? 1 : -1;     // :3558 adds, :3619 subtracts
      s.self_term = (!points && ref) ? 1 : 0;  // :3575-3596
      break;
    default:
      s.del = p.del;
      s.eps_check = 1;
      s.sign = 1;
      break;
  }
  return s;
}

}  // namespace

void eval_near(Tree* t, Lists* L, const bit_eval_params& p, int points, const double* tx,
               const double* ty, const double* tz, double* out) {
  cudaStream_t s = t->ctx->stream;
  const NearSpec sp = make_spec(p, points);
  const unsigned g = grid_for(L->nbatch, NWARPS);
  const double* sw = t->has_weights ? t->sw.p : nullptr;
  const bool f32 = p.precision == BIT_PREC_MIXED;
  const bool scr = p.kernel != BIT_KERNEL_COULOMB;
#define ARGS64 L->nbatch, L->order.p, L->b_tstart.p, L->b_tcount.p, L->b_srcleaf.p, tx, ty, tz, \
               L->near_off.p, L->near_ent.p, t->start.p, t->nummemb.p, t->src64.p, sw, sp, out
#define ARGS32 L->nbatch, L->order.p, L->b_tstart.p, L->b_tcount.p, L->b_srcleaf.p, tx, ty, tz, \
               L->near_off.p, L->near_ent.p, t->start.p, t->nummemb.p, t->nodec.p, t->src32.p, \
               t->src64.p, sw, sp, out
#define LAUNCH(K, E)                                                                   \
  do {                                                                                 \
    if (f32) k_near32<K, E><<<g, 32 * NWARPS, 0, s>>>(ARGS32);                         \
    else k_near64<K, E><<<g, 32 * NWARPS, 0, s>>>(ARGS64);                             \
  } while (0)
  if (!scr) {
    if (sp.eps_check) LAUNCH(BIT_KERNEL_COULOMB, true);
    else LAUNCH(BIT_KERNEL_COULOMB, false);
  } else {
    if (sp.eps_check) LAUNCH(BIT_KERNEL_SCREENED, true);
    else LAUNCH(BIT_KERNEL_SCREENED, false);
  }
#undef LAUNCH
#undef ARGS64
#undef ARGS32
  count_launch();
  BIT_CHECK_LAUNCH();
}

void eval_near_force(Tree* t, Lists* L, double del, bit_precision prec, double* fx, double* fy,
                     double* fz) {
  cudaStream_t s = t->ctx->stream;
  const unsigned g = grid_for(L->nbatch, NWARPS);
  if (prec == BIT_PREC_MIXED)
    count_launch(), k_near_force32<<<g, 32 * NWARPS, 0, s>>>(L->nbatch, L->order.p, L->b_tstart.p, L->b_tcount.p,
                                             t->sx.p, t->sy.p, t->sz.p, L->near_off.p,
                                             L->near_ent.p, t->start.p, t->nummemb.p,
                                             t->nodec.p, t->src32.p, del, 1, fx, fy, fz);
  else
    count_launch(), k_near_force64<<<g, 32 * NWARPS, 0, s>>>(L->nbatch, L->order.p, L->b_tstart.p, L->b_tcount.p,
                                             t->sx.p, t->sy.p, t->sz.p, L->near_off.p,
                                             L->near_ent.p, t->start.p, t->nummemb.p,
                                             t->src64.p, del, 1, fx, fy, fz);
  BIT_CHECK_LAUNCH();
}

}  // namespace bit

// Far field: Taylor expansion about every accepted cluster (treetaylorpotential,
// shielded_treetaylorpot, treetaylorforce; src/tree3d.cpp:4468-4640, 3004-3227, 456-810).
//
// One warp per batch, one target per lane, walking the batch's far entries; every lane
// whose bit is set evaluates the unrolled recurrence for its own offset from the cluster
// centre (generated per nterms by gen_farfield.py) against the cluster's moments.  The
// offset is formed in FP64; the mixed path rounds it once to FP32 and runs recurrence and
// dot product in FP32 with compensated accumulation across clusters.
#include "common.cuh"

namespace bit {
// Precision-generic math used by the generated recurrences.
__device__ __forceinline__ double sqrt_t(double x) { return sqrt(x); }
__device__ __forceinline__ float sqrt_t(float x) { return sqrtf(x); }
__device__ __forceinline__ double rsqrt_t(double x) { return rsqrt(x); }
__device__ __forceinline__ float rsqrt_t(float x) { return rsqrtf(x); }
__device__ __forceinline__ double exp_t(double x) { return exp(x); }
__device__ __forceinline__ float exp_t(float x) { return expf(x); }
__device__ __forceinline__ double fma_t(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float fma_t(float a, float b, float c) { return fmaf(a, b, c); }

}  // namespace bit

#include "generated/farfield_gen.cuh"

namespace bit {

namespace {

constexpr int FWARPS = 4;

template <class T>
struct Acc;
template <>
struct Acc<double> {
  double s = 0.0;
  __device__ void add(double v) { s += v; }
  __device__ double value() const { return s; }
};
template <>
struct Acc<float> {
  float s = 0.f, e = 0.f;
  __device__ void add(float v) {
    float t = s + v, bp = t - s;
    e += (s - (t - bp)) + (v - bp);
    s = t;
  }
  __device__ double value() const { return (double)s + (double)e; }
};

template <int NT, int KER, class T>
__global__ void __launch_bounds__(32 * FWARPS)
    k_far(int nbatch, const int* order, const int* b_tstart, const int* b_tcount,
          const double* tx, const double* ty, const double* tz, const long long* off,
          const int2* ent, const double4* nodec, const T* __restrict__ mom, double add,
          double kappa, double sign, double* out) {
  constexpr int TT = num_terms(NT);
  const int lane = threadIdx.x & 31;
  const int wi = blockIdx.x * FWARPS + (threadIdx.x >> 5);
  if (wi >= nbatch) return;
  const int b = order[wi];
  const int t0 = b_tstart[b], tc = b_tcount[b];
  const bool live = lane < tc;
  double x = 0, y = 0, z = 0;
  if (live) { x = tx[t0 + lane]; y = ty[t0 + lane]; z = tz[t0 + lane]; }
  const T tadd = (T)add, tk = (T)kappa;
  Acc<T> acc;
  for (long long e = off[b]; e < off[b + 1]; e++) {
    const int2 en = ent[e];
    if (!((unsigned(en.y) >> lane) & 1u)) continue;
    const double4 c = nodec[en.x];
    const T dx = (T)(x - c.x), dy = (T)(y - c.y), dz = (T)(z - c.z);
    const T r2 = dx * dx + dy * dy + dz * dz + tadd;
    const T* M = mom + (long long)en.x * TT;
    T v;
    if (KER == BIT_KERNEL_COULOMB) v = FarField<NT>::template coulomb<T>(dx, dy, dz, r2, M);
    else v = FarField<NT>::template screened<T>(dx, dy, dz, r2, tk, M);
    acc.add(v);
  }
  if (live) out[t0 + lane] = sign * acc.value();
}

template <int NT, class T>
__global__ void __launch_bounds__(32 * FWARPS)
    k_far_force(int nbatch, const int* order, const int* b_tstart, const int* b_tcount,
                const double* tx, const double* ty, const double* tz, const long long* off,
                const int2* ent, const double4* nodec, const T* __restrict__ mom, double del,
                double* fx, double* fy, double* fz) {
  constexpr int TT = num_terms(NT);
  const int lane = threadIdx.x & 31;
  const int wi = blockIdx.x * FWARPS + (threadIdx.x >> 5);
  if (wi >= nbatch) return;
  const int b = order[wi];
  const int t0 = b_tstart[b], tc = b_tcount[b];
  const bool live = lane < tc;
  double x = 0, y = 0, z = 0;
  if (live) { x = tx[t0 + lane]; y = ty[t0 + lane]; z = tz[t0 + lane]; }
  Acc<T> ax, ay, az;
  for (long long e = off[b]; e < off[b + 1]; e++) {
    const int2 en = ent[e];
    if (!((unsigned(en.y) >> lane) & 1u)) continue;
    const double4 c = nodec[en.x];
    const T dx = (T)(x - c.x), dy = (T)(y - c.y), dz = (T)(z - c.z);
    const T rs = dx * dx + dy * dy + dz * dz + (T)del;
    T fxv = 0, fyv = 0, fzv = 0;
    FarField<NT>::template force<T>(dx, dy, dz, rs, mom + (long long)en.x * TT, fxv, fyv, fzv);
    ax.add(fxv); ay.add(fyv); az.add(fzv);
  }
  if (live) {
    fx[t0 + lane] = ax.value();
    fy[t0 + lane] = ay.value();
    fz[t0 + lane] = az.value();
  }
}

template <int NT, int KER>
void launch_far(Tree* t, Lists* L, bool f32, double add, double kappa, double sign,
                const double* tx, const double* ty, const double* tz, double* out) {
  const unsigned g = grid_for(L->nbatch, FWARPS);
  cudaStream_t s = t->ctx->stream;
  if (f32)
    count_launch(), k_far<NT, KER, float><<<g, 32 * FWARPS, 0, s>>>(L->nbatch, L->order.p, L->b_tstart.p,
                                                    L->b_tcount.p, tx, ty, tz, L->far_off.p,
                                                    L->far_ent.p, t->nodec.p, t->mom32.p, add,
                                                    kappa, sign, out);
  else
    count_launch(), k_far<NT, KER, double><<<g, 32 * FWARPS, 0, s>>>(L->nbatch, L->order.p, L->b_tstart.p,
                                                     L->b_tcount.p, tx, ty, tz, L->far_off.p,
                                                     L->far_ent.p, t->nodec.p, t->mom64.p, add,
                                                     kappa, sign, out);
}

template <int NT>
void launch_far_force(Tree* t, Lists* L, bool f32, double del, double* fx, double* fy,
                      double* fz) {
  const unsigned g = grid_for(L->nbatch, FWARPS);
  cudaStream_t s = t->ctx->stream;
  if (f32)
    count_launch(), k_far_force<NT, float><<<g, 32 * FWARPS, 0, s>>>(L->nbatch, L->order.p, L->b_tstart.p,
                                                     L->b_tcount.p, t->sx.p, t->sy.p, t->sz.p,
                                                     L->far_off.p, L->far_ent.p, t->nodec.p,
                                                     t->mom32.p, del, fx, fy, fz);
  else
    count_launch(), k_far_force<NT, double><<<g, 32 * FWARPS, 0, s>>>(L->nbatch, L->order.p, L->b_tstart.p,
                                                      L->b_tcount.p, t->sx.p, t->sy.p, t->sz.p,
                                                      L->far_off.p, L->far_ent.p, t->nodec.p,
                                                      t->mom64.p, del, fx, fy, fz);
}

}  // namespace

void eval_far(Tree* t, Lists* L, const bit_eval_params& p, int /*points*/, const double* tx,
              const double* ty, const double* tz, double* out) {
  const bool f32 = p.precision == BIT_PREC_MIXED;
  // distance^2 fed to the recurrence: r^2 + del (Coulomb, regularised screened) or r^2
  const double add = p.kernel == BIT_KERNEL_SCREENED ? 0.0 : p.del;
  const double sign = p.kernel == BIT_KERNEL_SCREENED ? -1.0 : 1.0;  // :3222 subtracts
  const bool coul = p.kernel == BIT_KERNEL_COULOMB;
  switch (t->nterms) {
#define CASE(N)                                                                            \
  case N:                                                                                  \
    if (coul) launch_far<N, BIT_KERNEL_COULOMB>(t, L, f32, add, p.kappa, sign, tx, ty, tz, out); \
    else launch_far<N, BIT_KERNEL_SCREENED>(t, L, f32, add, p.kappa, sign, tx, ty, tz, out); \
    break;
    CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7) CASE(8) CASE(9) CASE(10)
#undef CASE
    default:
      fail(BIT_ERR_STATE, "moments not computed");
  }
  BIT_CHECK_LAUNCH();
}

void eval_far_force(Tree* t, Lists* L, double del, bit_precision prec, double* fx, double* fy,
                    double* fz) {
  const bool f32 = prec == BIT_PREC_MIXED;
  switch (t->nterms) {
#define CASE(N) case N: launch_far_force<N>(t, L, f32, del, fx, fy, fz); break;
    CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7) CASE(8) CASE(9) CASE(10)
#undef CASE
    default:
      fail(BIT_ERR_STATE, "moments not computed");
  }
  BIT_CHECK_LAUNCH();
}

}  // namespace bit

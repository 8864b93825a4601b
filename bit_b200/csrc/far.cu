// Far field: Taylor expansion about every accepted cluster (treetaylorpotential,
// shielded_treetaylorpot, treetaylorforce; src/tree3d.cpp:4468-4640, 3004-3227, 456-810),
// one CTA per target group.
//
// The CTA's warps take the group's far entries round-robin.  A warp packs the targets of
// its entry (the set bits of the entry's mask) into a dense list while a TMA bulk copy
// brings the cluster's moments (a padded shell-order block, no multicast) into the warp's
// shared-memory slot, and its lanes run the unrolled recurrence (generated per nterms by
// gen_farfield.py) for one target each, against those moments (warp-uniform loads).  Each warp accumulates into its own
// shared-memory row; rows are summed in warp order at the end, so the result does not
// depend on timing.  The target-centre offset is formed in FP64; the mixed path rounds it
// once to FP32 and runs recurrence and dot product in FP32, accumulating with two-sum.
#include <algorithm>

#include "common.cuh"
#include "tma.cuh"

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
__device__ __forceinline__ double pow_t(double a, double b) { return pow(a, b); }
__device__ __forceinline__ float pow_t(float a, float b) { return powf(a, b); }
template <class T>
struct V4 {
  T x, y, z, w;
};
// Four consecutive moments; M is 16-byte aligned.
__device__ __forceinline__ V4<float> ld4(const float* M, int q) {
  const float4 v = reinterpret_cast<const float4*>(M)[q];
  return {v.x, v.y, v.z, v.w};
}
__device__ __forceinline__ V4<double> ld4(const double* M, int q) {
  const double2 a = reinterpret_cast<const double2*>(M)[2 * q];
  const double2 b = reinterpret_cast<const double2*>(M)[2 * q + 1];
  return {a.x, a.y, b.x, b.y};
}
}  // namespace bit

#include "generated/farfield_gen.cuh"

namespace bit {

namespace {

struct FarArgs {
  const int *order, *g_tstart, *g_tcount;
  const double *tx, *ty, *tz;
  const long long *off, *moff;
  const int* cnt;
  const int* node;
  const unsigned* mask;
  const double4* nodec;
  const void* mom;  // float or double, T(nterms of the node's system) per node
  const long long* mom_off;  // first moment of each node
  const void* msh;           // the same in shell order, padded blocks (potential kernels)
  const long long* msh_off;  // first element of each node's block
  int* err;                  // device error flags (a bounded wait that gave up: 8)
  int* cost;                 // scratch, one int per far entry: its number of targets
  const SysEval* sys;        // per system: far_add, kappa, far_sign
  const int* g_sys;          // per group: system
  double *out, *out_y, *out_z;
};

// Pack the set bits of a group mask (W words, lane l holds word l) into tl; returns count.
__device__ __forceinline__ int warp_pack(unsigned wd, unsigned short* tl) {
  const int lane = threadIdx.x & 31;
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
    tl[base++] = (unsigned short)(32 * lane + b);
  }
  __syncwarp();
  return __shfl_sync(0xffffffffu, pre, 31);
}

template <class T>
struct WarpAcc;  // per-warp accumulator rows in shared memory
template <>
struct WarpAcc<float> {
  static constexpr int words = 2;  // hi, lo
  __device__ static void add(float* row, int i, float v) {
    float& s = row[i];
    float& e = row[kGroupMax + i];
    float t = s + v, bp = t - s;
    e += (s - (t - bp)) + (v - bp);
    s = t;
  }
  __device__ static double get(const float* row, int i) {
    return (double)row[i] + (double)row[kGroupMax + i];
  }
};
template <>
struct WarpAcc<double> {
  static constexpr int words = 1;
  __device__ static void add(double* row, int i, double v) { row[i] += v; }
  __device__ static double get(const double* row, int i) { return row[i]; }
};

template <int NW>
constexpr size_t far_smem(size_t acc_bytes_per_row_target, size_t moment_bytes) {
  return 3 * kGroupMax * sizeof(double) + NW * kGroupMax * sizeof(unsigned short) +
         NW * kGroupMax * acc_bytes_per_row_target + NW * moment_bytes;
}

// Warps per CTA of the potential kernels (NW).  FP32: 8 warps, two CTAs per SM at 128
// registers.  FP64 (254 registers): with many groups, 4 warps, so that two CTAs share an SM
// and one keeps the FP64 pipe busy while the other waits at its group's closing barrier;
// with few, 8 warps, so that each group is spread over more warps (eval_far).  Measured on
// clustered systems, p = 8 (screened, ms, 4 / 8 warps): 378 groups 1.41 / 1.07, 835 groups
// 3.17 / 3.23, 3,091 groups (2M) 17.25 / 18.12.
template <class T>
constexpr int min_blocks(int nw) { return sizeof(T) == 8 && nw == 8 ? 1 : 2; }
constexpr int NWF = 4;  // warps per CTA, force (three accumulators)

// The far field of one target group g (the CTA's whole work for that group).  Shared
// memory: the group's target coordinates, per warp a packed target list, an accumulator row
// and one cluster's moments (NW * TP of them; a kernel running several orders sizes this for
// the largest).  bar: one mbarrier per warp, phase: this warp's count of its completed
// copies.  Returns false (in every thread) if a warp's bounded wait for its moments gave up:
// the error flag is set, the warp has waited (bounded again) for that copy, and the group's
// result is not valid.
template <int NT, int KER, class T, int NW>
__device__ __forceinline__ bool far_group(const FarArgs& a, int g, uint64_t* bar, unsigned& phase) {
  constexpr int TT = num_terms(NT);
  constexpr int TP = FarField<NT>::kPadded;
  extern __shared__ __align__(16) unsigned char sm[];
  double* cx = reinterpret_cast<double*>(sm);
  double* cy = cx + kGroupMax;
  double* cz = cy + kGroupMax;
  unsigned short* tlb = reinterpret_cast<unsigned short*>(cz + kGroupMax);
  T* accb = reinterpret_cast<T*>(tlb + NW * kGroupMax);
  constexpr int ROW = WarpAcc<T>::words * kGroupMax;
  T* msb = accb + NW * ROW;  // one cluster's moments per warp

  const int t0 = a.g_tstart[g], tc = a.g_tcount[g];
  const int W = (tc + 31) >> 5;
  const long long e0 = a.off[g], e1 = e0 + a.cnt[g], m0 = a.moff[g];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  for (int i = tid; i < tc; i += 32 * NW) {
    cx[i] = a.tx[t0 + i]; cy[i] = a.ty[t0 + i]; cz[i] = a.tz[t0 + i];
  }
  for (int i = tid; i < NW * ROW; i += 32 * NW) accb[i] = T(0);
  __syncthreads();
  unsigned short* tl = tlb + w * kGroupMax;
  T* row = accb + w * ROW;
  const T* msh = reinterpret_cast<const T*>(a.msh);
  const SysEval* se = a.sys + a.g_sys[g];
  const T tadd = (T)se->far_add, tk = (T)se->kappa;
  const double sign = se->far_sign;
  bool failed = false;
  // Each warp takes a contiguous run of the group's entries holding about 1/NW of its
  // (target, cluster) pairs: the entries whose exclusive prefix P of target counts has
  // w C <= NW P < (w + 1) C, C the group's total.  The entries' costs vary widely, so the
  // round-robin deal this replaces left warps idle at the group's closing barrier.  The
  // split depends on the lists only, so results stay deterministic.
  for (long long e = e0 + w; e < e1; e += NW) {
    const unsigned wd = lane < W ? a.mask[m0 + (e - e0) * W + lane] : 0u;
    const int c = __reduce_add_sync(0xffffffffu, __popc(wd));
    if (lane == 0) a.cost[e] = c;
  }
  __syncthreads();
  long long tot = 0;
  for (long long b = e0; b < e1; b += 32)
    tot += __reduce_add_sync(0xffffffffu, b + lane < e1 ? __ldcg(a.cost + b + lane) : 0);
  long long run = 0;
  int eb = 0, ee = 0;
  for (long long b = e0; b < e1; b += 32) {
    const bool in = b + lane < e1;
    const int c = in ? __ldcg(a.cost + b + lane) : 0;
    int inc = c;
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += t;
    }
    const long long P = (run + inc - c) * NW;
    eb += __popc(__ballot_sync(0xffffffffu, in && P < w * tot));
    ee += __popc(__ballot_sync(0xffffffffu, in && P < (w + 1) * tot));
    run += __shfl_sync(0xffffffffu, inc, 31);
  }
  for (long long e = e0 + eb; e < e0 + ee; e++) {
    const int node = a.node[e];
    T* M = msb + w * TP;
    // The cluster's moments, its whole padded shell-order block (TP values, 16-byte aligned
    // in global and shared memory), by one TMA bulk copy into the warp's slot while the
    // warp packs the entry's targets.  The previous entry's reads of the slot ended at the
    // __syncwarp closing its loop.
    if (lane == 0) {
      fence_proxy_async();
      mbar_expect_tx(&bar[w], TP * (unsigned)sizeof(T));
      tma_load_1d(M, msh + a.msh_off[node], TP * (unsigned)sizeof(T), &bar[w]);
    }
    const unsigned wd = lane < W ? a.mask[m0 + (e - e0) * W + lane] : 0u;
    const int cnt = warp_pack(wd, tl);
    const double4 c = a.nodec[node];
    const bool landed = __all_sync(0xffffffffu, mbar_wait(&bar[w], phase & 1));
    phase++;
    if (!landed) {
      if (lane == 0) {
        atomicOr(a.err, 8);
        mbar_wait(&bar[w], (phase - 1) & 1);
      }
      __syncwarp();
      failed = true;
      break;
    }
    // Both precisions run the scaled form of the reference's recurrence (fewer operations
    // than the literal one, the same function).  FP32 moments are normalised by h^|v|,
    // h = 2^e; FP64 moments are the plain ones, i.e. h = 1.  The FP32 kernels take the
    // forms with per-pair products hoisted (at nterms 9, screened: 886 fma + 189 mul per
    // pair against 886 + 447, Coulomb: 572 + 68 against 572 + 123; at 2M clustered, p = 8,
    // theta = 0.7: screened 9.77 -> 9.09 ms, Coulomb 6.41 -> 6.07 ms); the FP64
    // ones keep the plain forms, since the hoisted screened one spilled there and ran 1%
    // slower.
    const T h = sizeof(T) == 4 ? (T)ldexpf(1.f, mom32_scale_exp(c.w)) : T(1);
    __syncwarp();
    for (int r = lane; r < cnt; r += 32) {
      const int i = tl[r];
      const T dx = (T)(cx[i] - c.x), dy = (T)(cy[i] - c.y), dz = (T)(cz[i] - c.z);
      const T r2 = dx * dx + dy * dy + dz * dz + tadd;
      T v;
      if (sizeof(T) == 4)
        v = KER == BIT_KERNEL_COULOMB ? FarField<NT>::template coulomb_s<T>(dx, dy, dz, r2, h, M)
                                      : FarField<NT>::template screened_s<T>(dx, dy, dz, r2, tk, h, M);
      else
        v = KER == BIT_KERNEL_COULOMB ? FarField<NT>::template coulomb_sp<T>(dx, dy, dz, r2, h, M)
                                      : FarField<NT>::template screened_sp<T>(dx, dy, dz, r2, tk, h, M);
      WarpAcc<T>::add(row, i, v);
    }
    __syncwarp();
  }
  if (__syncthreads_or(failed)) return false;
  for (int i = tid; i < tc; i += 32 * NW) {
    double s = 0.0;
    for (int q = 0; q < NW; q++) s += WarpAcc<T>::get(accb + q * ROW, i);
    a.out[t0 + i] = sign * s;
  }
  return true;
}

// One mbarrier per warp for the moment copies, initialised before the kernel's first
// __syncthreads.
template <int NW>
__device__ __forceinline__ void far_bars_init(uint64_t* bar) {
  if (threadIdx.x == 0) {
    for (int k = 0; k < NW; k++) mbar_init(&bar[k], 1);
    fence_mbar_init();
  }
}

// One launch class: CTA b takes group order[b].
template <int NT, int KER, class T, int NW>
__global__ void __launch_bounds__(32 * NW, min_blocks<T>(NW)) k_far(FarArgs a) {
  __shared__ uint64_t bar[NW];
  far_bars_init<NW>(bar);
  unsigned phase = 0;
  far_group<NT, KER, T, NW>(a, a.order[blockIdx.x], bar, phase);
}

// Persistent work queue over the groups of every class: each CTA takes the next item
// (a group, in the given order) from a device counter until none is left, and runs the
// far field of that group's system (its nterms and kernel) -- the same device code, in the
// same order within the group, as k_far, so the results are identical.  No CTA waits for
// another; the counter is the only shared state.
template <class T, int NW>
__global__ void __launch_bounds__(32 * NW, min_blocks<T>(NW))
    k_far_queue(FarArgs a, int count, int* head) {
  __shared__ int s_item;
  __shared__ uint64_t bar[NW];
  far_bars_init<NW>(bar);
  unsigned phase = 0;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(head, 1);
    __syncthreads();
    const int item = s_item;
    __syncthreads();  // every thread has read s_item before it is overwritten
    if (item >= count) return;
    const int g = a.order[item];
    const SysEval* se = a.sys + a.g_sys[g];
    const bool coul = se->kernel == BIT_KERNEL_COULOMB;
    bool ok = true;
    switch (se->nterms) {
#define FQ(N)                                                                   \
  case N:                                                                       \
    ok = coul ? far_group<N, BIT_KERNEL_COULOMB, T, NW>(a, g, bar, phase)       \
              : far_group<N, BIT_KERNEL_SCREENED, T, NW>(a, g, bar, phase);     \
    break;
      FQ(1) FQ(2) FQ(3) FQ(4) FQ(5) FQ(6) FQ(7) FQ(8) FQ(9) FQ(10)
#undef FQ
      default:
        break;
    }
    if (!ok) return;  // a bounded wait gave up (every thread saw it): take no more items
    __syncthreads();  // the group's last reads of shared memory precede the next group's writes
  }
}

// Field kinds of k_far_force: the regularised Coulomb field of treetaylorforce with
// KERNEL_ORDER = 0 (FK_COULOMB) or with the system's kernel order (FK_COULOMB_KORDER, FP64),
// and the screened 2-D field of shielded_treetaylorforce (FK_SCREENED_CURL, FP64).
constexpr int FK_COULOMB = 0, FK_COULOMB_KORDER = 1, FK_SCREENED_CURL = 2;

template <int NT, int FK, class T>
__global__ void __launch_bounds__(32 * NWF) k_far_force(FarArgs a) {
  constexpr int TT = num_terms(NT);
  constexpr int TP = FarField<NT>::kPadded;
  constexpr int NW = NWF;
  extern __shared__ __align__(16) unsigned char sm[];
  double* cx = reinterpret_cast<double*>(sm);
  double* cy = cx + kGroupMax;
  double* cz = cy + kGroupMax;
  unsigned short* tlb = reinterpret_cast<unsigned short*>(cz + kGroupMax);
  double* accb = reinterpret_cast<double*>(tlb + NW * kGroupMax);  // [NW][3][kGroupMax]
  T* msb = reinterpret_cast<T*>(accb + NW * 3 * kGroupMax);         // moments, one per warp

  const int g = a.order[blockIdx.x];
  const int t0 = a.g_tstart[g], tc = a.g_tcount[g];
  const int W = (tc + 31) >> 5;
  const long long e0 = a.off[g], e1 = e0 + a.cnt[g], m0 = a.moff[g];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  for (int i = tid; i < tc; i += 32 * NW) {
    cx[i] = a.tx[t0 + i]; cy[i] = a.ty[t0 + i]; cz[i] = a.tz[t0 + i];
  }
  for (int i = tid; i < NW * 3 * kGroupMax; i += 32 * NW) accb[i] = 0.0;
  __syncthreads();
  unsigned short* tl = tlb + w * kGroupMax;
  double* row = accb + w * 3 * kGroupMax;
  const T* mom = reinterpret_cast<const T*>(a.mom);
  const SysEval* se = a.sys + a.g_sys[g];
  const T tadd = (T)se->far_add, tk = (T)se->kappa, tdel = (T)se->near_del;
  const int korder = se->kernel_order;
  for (long long e = e0 + w; e < e1; e += NW) {
    const unsigned wd = lane < W ? a.mask[m0 + (e - e0) * W + lane] : 0u;
    const int cnt = warp_pack(wd, tl);
    const int node = a.node[e];
    const double4 c = a.nodec[node];
    T* M = msb + w * TP;
    const T* mn = mom + a.mom_off[node];
    // FP32 moments are stored normalised by h^|v| (h = 2^e): undo it exactly here, since
    // the force recurrence takes the moments themselves
    const int se = sizeof(T) == 4 ? mom32_scale_exp(c.w) : 0;
    for (int k = lane; k < TP; k += 32) {
      T m = k < TT ? mn[FarField<NT>::canon(k)] : T(0);
      if constexpr (sizeof(T) == 4) {
        int d = 0;  // degree of shell-order index k
        while (num_terms(d + 1) <= k) d++;
        m = ldexpf(m, se * d);
      }
      M[k] = m;
    }
    __syncwarp();
    for (int r = lane; r < cnt; r += 32) {
      const int i = tl[r];
      const T dx = (T)(cx[i] - c.x), dy = (T)(cy[i] - c.y), dz = (T)(cz[i] - c.z);
      const T rs = dx * dx + dy * dy + dz * dz + tadd;
      T fx = 0, fy = 0, fz = 0;
      if constexpr (FK == FK_COULOMB) FarField<NT>::template force<T>(dx, dy, dz, rs, M, fx, fy, fz);
      else if constexpr (FK == FK_COULOMB_KORDER)
        FarField<NT>::template force_korder<T>(dx, dy, dz, rs, tdel, korder, M, fx, fy, fz);
      else FarField<NT>::template screened_curl<T>(dx, dy, dz, rs, tk, M, fx, fy);
      row[i] += (double)fx;
      row[kGroupMax + i] += (double)fy;
      row[2 * kGroupMax + i] += (double)fz;
    }
    __syncwarp();
  }
  __syncthreads();
  for (int i = tid; i < tc; i += 32 * NW) {
    double sx = 0, sy = 0, sz = 0;
    for (int q = 0; q < NW; q++) {
      sx += accb[q * 3 * kGroupMax + i];
      sy += accb[q * 3 * kGroupMax + kGroupMax + i];
      sz += accb[q * 3 * kGroupMax + 2 * kGroupMax + i];
    }
    a.out[t0 + i] = sx;
    a.out_y[t0 + i] = sy;
    a.out_z[t0 + i] = sz;
  }
}

template <class K>
void set_smem(K kernel, size_t bytes) {
  ensure_smem_attr(reinterpret_cast<const void*>(kernel), (int)bytes);
}

template <int NT, int KER, class T, int NW>
void launch_far(const FarArgs& a, int ng, cudaStream_t s) {
  const size_t bytes =
      far_smem<NW>(WarpAcc<T>::words * sizeof(T), FarField<NT>::kPadded * sizeof(T));
  set_smem(k_far<NT, KER, T, NW>, bytes);
  count_launch(), k_far<NT, KER, T, NW><<<ng, 32 * NW, bytes, s>>>(a);
}

template <int NT, int FK, class T>
void launch_force(const FarArgs& a, int ng, cudaStream_t s) {
  const size_t bytes = far_smem<NWF>(3 * sizeof(double), FarField<NT>::kPadded * sizeof(T));
  set_smem(k_far_force<NT, FK, T>, bytes);
  count_launch(), k_far_force<NT, FK, T><<<ng, 32 * NWF, bytes, s>>>(a);
}

FarArgs far_args(Tree* t, Lists* L, const EvalPlan& P, const double* tx, const double* ty,
                 const double* tz) {
  FarArgs a{};
  a.g_tstart = L->g_tstart.p;
  a.g_tcount = L->g_tcount.p;
  a.tx = tx; a.ty = ty; a.tz = tz;
  a.off = L->far_off.p;
  a.cnt = L->far_cnt.p;
  a.moff = L->far_moff.p;
  a.node = L->far_node.p;
  a.mask = L->far_mask.p;
  a.nodec = t->nodec.p;
  a.mom = P.f32 ? (const void*)t->mom32.p : (const void*)t->mom64.p;
  a.mom_off = t->mom_off.p;
  a.msh = P.f32 ? (const void*)t->msh32.p : (const void*)t->msh64.p;
  a.msh_off = t->msh_off.p;
  a.err = t->ctx->dev_err();
  L->far_cost.ensure(t->ctx, std::max(L->nfar, 1LL));
  a.cost = L->far_cost.p;
  a.sys = P.sys.p;
  a.g_sys = L->g_sys.p;
  return a;
}

}  // namespace

// One launch per (nterms, kernel) class, each over its groups (P.far_ord + begin).
template <class T, int NW>
void launch_far_queue(Ctx* c, const FarArgs& a, int count, int max_nterms, int* head,
                      cudaStream_t s) {
  int tp = 0;
  switch (max_nterms) {
#define TPN(N) case N: tp = FarField<N>::kPadded; break;
    TPN(1) TPN(2) TPN(3) TPN(4) TPN(5) TPN(6) TPN(7) TPN(8) TPN(9) TPN(10)
#undef TPN
    default: fail(BIT_ERR_STATE, "moments not computed");
  }
  const size_t bytes = far_smem<NW>(WarpAcc<T>::words * sizeof(T), tp * sizeof(T));
  set_smem(k_far_queue<T, NW>, bytes);
  int per_sm = 0;
  BIT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_far_queue<T, NW>, 32 * NW, bytes));
  const int grid = std::max(1, std::min(count, c->num_sms * std::max(per_sm, 1)));
  count_launch(), k_far_queue<T, NW><<<grid, 32 * NW, bytes, s>>>(a, count, head);
}

// The work-queue form is used for plans of several classes when the context allows it;
// the queue takes every group in decreasing-work order (L->order).
bool use_queue(const Ctx* c, const std::vector<LaunchClass>& classes) {
  return c->work_queue && classes.size() > 1;
}

int* queue_head(Ctx* c, int which, cudaStream_t s) {
  c->queue_heads.ensure(c, 2);
  BIT_CUDA(cudaMemsetAsync(c->queue_heads.p + which, 0, sizeof(int), s));
  return c->queue_heads.p + which;
}

void eval_far(Tree* t, Lists* L, const EvalPlan& P, const double* tx, const double* ty,
              const double* tz, double* out) {
  FarArgs a = far_args(t, L, P, tx, ty, tz);
  a.out = out;
  cudaStream_t s = t->ctx->stream;
  const bool f32 = P.f32;
  // FP64: 4-warp CTAs when the evaluation has at least 4 groups per SM.  The choice
  // follows the whole list (not a launch class), so the queue and the class launches of
  // one evaluation sum in the same order.
  const bool narrow = !f32 && L->ngroups >= 4 * t->ctx->num_sms;
  if (use_queue(t->ctx, P.far_classes)) {
    int nt_max = 0, count = 0;
    for (const LaunchClass& k : P.far_classes) nt_max = std::max(nt_max, k.nterms);
    for (const LaunchClass& k : P.far_classes) count += k.count;
    a.order = L->order.p;
    int* head = queue_head(t->ctx, 0, s);
    if (f32) launch_far_queue<float, 8>(t->ctx, a, count, nt_max, head, s);
    else if (narrow) launch_far_queue<double, 4>(t->ctx, a, count, nt_max, head, s);
    else launch_far_queue<double, 8>(t->ctx, a, count, nt_max, head, s);
    BIT_CHECK_LAUNCH();
    return;
  }
  for (const LaunchClass& k : P.far_classes) {
    a.order = P.far_ord + k.begin;
    const int ng = k.count;
    const bool coul = k.kernel == BIT_KERNEL_COULOMB;
    switch (k.nterms) {
#define CASE(N)                                                                   \
  case N:                                                                         \
    if (f32) {                                                                    \
      if (coul) launch_far<N, BIT_KERNEL_COULOMB, float, 8>(a, ng, s);            \
      else launch_far<N, BIT_KERNEL_SCREENED, float, 8>(a, ng, s);                \
    } else if (narrow) {                                                          \
      if (coul) launch_far<N, BIT_KERNEL_COULOMB, double, 4>(a, ng, s);           \
      else launch_far<N, BIT_KERNEL_SCREENED, double, 4>(a, ng, s);               \
    } else {                                                                      \
      if (coul) launch_far<N, BIT_KERNEL_COULOMB, double, 8>(a, ng, s);           \
      else launch_far<N, BIT_KERNEL_SCREENED, double, 8>(a, ng, s);               \
    }                                                                             \
    break;
      CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7) CASE(8) CASE(9) CASE(10)
#undef CASE
      default:
        fail(BIT_ERR_STATE, "moments not computed");
    }
    BIT_CHECK_LAUNCH();
  }
}

void eval_far_force(Tree* t, Lists* L, const EvalPlan& P, double* fx, double* fy, double* fz) {
  FarArgs a = far_args(t, L, P, t->sx.p, t->sy.p, t->sz.p);
  a.out = fx; a.out_y = fy; a.out_z = fz;
  cudaStream_t s = t->ctx->stream;
  const bool f32 = P.f32;
  // field kind of the plan: 1 Coulomb (kernel order from each system), 2 screened curl
  const bool curl = P.force == 2;
  bool korder = false;
  for (const SysEval& se : P.h_sys) korder |= se.kernel_order > 0;
  if (f32 && (curl || korder)) fail(BIT_ERR_INVALID_ARGUMENT, "this field is FP64 only");
  for (const LaunchClass& k : P.far_classes) {
    a.order = P.far_ord + k.begin;
    const int ng = k.count;
    switch (k.nterms) {
#define CASE(N)                                                            \
  case N:                                                                  \
    if (f32) launch_force<N, FK_COULOMB, float>(a, ng, s);                 \
    else if (curl) launch_force<N, FK_SCREENED_CURL, double>(a, ng, s);    \
    else if (korder) launch_force<N, FK_COULOMB_KORDER, double>(a, ng, s); \
    else launch_force<N, FK_COULOMB, double>(a, ng, s);                    \
    break;
      CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7) CASE(8) CASE(9) CASE(10)
#undef CASE
      default:
        fail(BIT_ERR_STATE, "moments not computed");
    }
    BIT_CHECK_LAUNCH();
  }
}

}  // namespace bit

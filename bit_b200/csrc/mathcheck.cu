// Agreement of the near field's own FP64 exp and rsqrt (fp64math.cuh) with CUDA's exp and
// rsqrt on the device: the largest difference, in units in the last place of CUDA's
// result, over n seeded arguments (exp: t uniform in [-707, 0] for the full form and in
// (-8, 0] for the small-argument form, the larger of the two; rsqrt: x log-uniform in
// [1e-12, 1e6]).  A test holds both to a bound.
#include "common.cuh"
#include "fp64math.cuh"
#include "tma.cuh"

namespace bit {

namespace {

// uniform in [0, 1) from a 64-bit mix of the index (splitmix64's finaliser)
__device__ __forceinline__ double unit(unsigned long long i) {
  unsigned long long z = i * 0x9e3779b97f4a7c15ull + 0x632be59bd9b4e019ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  z ^= z >> 31;
  return (double)(z >> 11) * 0x1p-53;
}

// |a - b| in ulps of b (b finite, non-zero)
__device__ __forceinline__ double ulp_diff(double a, double b) {
  int e;
  frexp(b, &e);
  return fabs(a - b) / ldexp(1.0, e - 53);
}

__global__ void k_math_check(long long n, unsigned long long* worst) {
  double we = 0.0, wr = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double t = -707.0 * unit(2 * i);
    const double x = exp10(-12.0 + 18.0 * unit(2 * i + 1));
    const double ts = -kSmallExpArg * unit(2 * i + 1);
    we = fmax(we, ulp_diff(exp_tang(t), exp(t)));
    we = fmax(we, ulp_diff(exp_tang<true>(ts), exp(ts)));
    wr = fmax(wr, ulp_diff(rsqrt_nr(x), rsqrt(x)));
  }
  // non-negative doubles order as their bit patterns
  atomicMax(worst, (unsigned long long)__double_as_longlong(we));
  atomicMax(worst + 1, (unsigned long long)__double_as_longlong(wr));
}

// The kernels' give-up path, exercised where no copy is in flight: an mbarrier that no
// copy and no thread ever arrives at, waited on by every thread with the kernels' bounded
// wait (at most `limit` attempts), the outcome combined for the CTA as the near field does,
// and the error flag raised (16) when the wait gives up.
__global__ void k_wait_check(int limit, int* err) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  const bool landed = mbar_wait(&bar, 0, limit);
  if (__syncthreads_or(!landed) && threadIdx.x == 0) atomicOr(err, 16);
}

}  // namespace

void device_wait_check(Ctx* c, int limit) {
  count_launch(), k_wait_check<<<1, 128, 0, c->stream>>>(limit, c->dev_err());
  BIT_CHECK_LAUNCH();
  BIT_CUDA(cudaStreamSynchronize(c->stream));
}

void fp64_math_error(Ctx* c, long long n, double* exp_ulps, double* rsqrt_ulps) {
  cudaStream_t s = c->stream;
  DBuf<unsigned long long> w;
  w.ensure(c, 2);
  BIT_CUDA(cudaMemsetAsync(w.p, 0, 2 * sizeof(unsigned long long), s));
  count_launch(), k_math_check<<<c->num_sms * 8, 256, 0, s>>>(n, w.p);
  BIT_CHECK_LAUNCH();
  unsigned long long h[2];
  BIT_CUDA(cudaMemcpyAsync(h, w.p, sizeof(h), cudaMemcpyDeviceToHost, s));
  BIT_CUDA(cudaStreamSynchronize(s));
  *exp_ulps = __builtin_bit_cast(double, h[0]);
  *rsqrt_ulps = __builtin_bit_cast(double, h[1]);
}

}  // namespace bit

// CUDA-core FMA throughput of the device, measured: the denominator of the FP32 / FP64
// rooflines of the near- and far-field kernels (a dense FMA chain workload timed with
// CUDA events, the way a STREAM copy measures HBM bandwidth).
//
// Every thread runs kChains independent FMA chains for `iters` rounds; there are enough
// resident warps and independent chains per warp to cover the pipe latency, so the
// kernel issues FMAs at the pipe's rate.  Each chain's result feeds a final sum that is
// stored only if it equals a value no input can produce, so no chain is dead code.
#include <algorithm>

#include "common.cuh"

namespace bit {

namespace {

constexpr int kChains = 8;
constexpr int kThreads = 512;

template <class T>
__global__ void __launch_bounds__(kThreads) k_fma_peak(int iters, T a, T b, T* sink) {
  T v[kChains];
  for (int c = 0; c < kChains; c++) v[c] = (T)(threadIdx.x + c);
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int c = 0; c < kChains; c++) v[c] = fma(v[c], a, b);
  }
  T s = 0;
  for (int c = 0; c < kChains; c++) s += v[c];
  if (s == (T)-1.2345e30) sink[0] = s;
}

template <class T>
double run_peak(Ctx* c) {
  cudaStream_t s = c->stream;
  DBuf<T> sink;
  sink.ensure(c, 1);
  int per_sm = 0;
  BIT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fma_peak<T>, kThreads, 0));
  const int blocks = c->num_sms * (per_sm > 0 ? per_sm : 1);
  const int iters = sizeof(T) == 4 ? 1 << 16 : 1 << 15;
  // a, b keep every chain finite: v -> v * a + b converges to b / (1 - a)
  const T a = (T)0.999, b = (T)0.001;
  cudaEvent_t e0, e1;
  BIT_CUDA(cudaEventCreate(&e0));
  BIT_CUDA(cudaEventCreate(&e1));
  count_launch(), k_fma_peak<T><<<blocks, kThreads, 0, s>>>(iters / 16, a, b, sink.p);  // warm-up
  BIT_CHECK_LAUNCH();
  double best = 0.0;
  for (int rep = 0; rep < 3; rep++) {
    BIT_CUDA(cudaEventRecord(e0, s));
    count_launch(), k_fma_peak<T><<<blocks, kThreads, 0, s>>>(iters, a, b, sink.p);
    BIT_CHECK_LAUNCH();
    BIT_CUDA(cudaEventRecord(e1, s));
    BIT_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    BIT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    const double flops = 2.0 * kChains * (double)iters * kThreads * blocks;
    if (ms > 0.f) best = std::max(best, flops / (ms * 1e-3));
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return best;
}

}  // namespace

double fma_peak(Ctx* c, bool f32) { return f32 ? run_peak<float>(c) : run_peak<double>(c); }

}  // namespace bit

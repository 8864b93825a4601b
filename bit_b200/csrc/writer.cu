// output_potential (src/tree3d.cpp:4918-4937): one ASCII line per particle,
// "i<TAB>x<TAB>y<TAB>z<TAB>pot" with 14 significant digits (an ostream at precision 14 in
// its default float format, which is printf's %.14g).
//
// The device variant streams: particles go to the file in chunks; while one chunk is
// formatted and written, the next chunk's device-to-host copies run into the other half of
// a double-buffered pinned staging area.
#include <cstdio>
#include <vector>

#include "common.cuh"

namespace bit {
namespace {

constexpr int kChunk = 1 << 16;  // particles per streamed chunk

void format_chunk(std::FILE* f, int i0, int cnt, const double* x, const double* y,
                  const double* z, const double* pot, std::vector<char>& line) {
  for (int k = 0; k < cnt; k++) {
    const int len = std::snprintf(line.data(), line.size(), "%d\t%.14g\t%.14g\t%.14g\t%.14g\n",
                                  i0 + k, x[k], y[k], z[k], pot[k]);
    std::fwrite(line.data(), 1, (size_t)len, f);
  }
}

}  // namespace
}  // namespace bit

using namespace bit;

extern "C" {

bit_status bit_write_potential(const char* path, int n, const double* x, const double* y,
                               const double* z, const double* pot) {
  if (!path || n < 0 || (n > 0 && (!x || !y || !z || !pot))) return BIT_ERR_INVALID_ARGUMENT;
  std::FILE* f = std::fopen(path, "w");
  if (!f) return BIT_ERR_INVALID_ARGUMENT;
  std::vector<char> line(256);
  format_chunk(f, 0, n, x, y, z, pot, line);
  const bool ok = std::fclose(f) == 0;
  return ok ? BIT_OK : BIT_ERR_INVALID_ARGUMENT;
}

bit_status bit_write_potential_device(bit_ctx* h, const char* path, int n, const double* x,
                                      const double* y, const double* z, const double* pot) {
  if (!h || !path || n < 0 || (n > 0 && (!x || !y || !z || !pot))) return BIT_ERR_INVALID_ARGUMENT;
  Ctx* c = &h->c;
  std::FILE* f = std::fopen(path, "w");
  if (!f) {
    c->last_error = std::string("cannot open ") + path;
    return BIT_ERR_INVALID_ARGUMENT;
  }
  double* stage = nullptr;  // 2 halves x 4 arrays x kChunk
  cudaEvent_t ev[2] = {nullptr, nullptr};
  bit_status st = BIT_OK;
  try {
    BIT_CUDA(cudaSetDevice(c->device));
    BIT_CUDA(cudaMallocHost(&stage, 8ull * kChunk * sizeof(double)));
    BIT_CUDA(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
    BIT_CUDA(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
    const double* src[4] = {x, y, z, pot};
    auto issue = [&](int chunk) {
      const int i0 = chunk * kChunk, cnt = std::min(kChunk, n - i0);
      double* half = stage + 4ull * kChunk * (chunk & 1);
      for (int a = 0; a < 4; a++)
        BIT_CUDA(cudaMemcpyAsync(half + (size_t)a * kChunk, src[a] + i0, cnt * sizeof(double),
                                 cudaMemcpyDeviceToHost, c->stream));
      BIT_CUDA(cudaEventRecord(ev[chunk & 1], c->stream));
    };
    const int nch = (n + kChunk - 1) / kChunk;
    std::vector<char> line(256);
    if (nch > 0) issue(0);
    for (int k = 0; k < nch; k++) {
      if (k + 1 < nch) issue(k + 1);  // the other half is free: chunk k-1 was written
      BIT_CUDA(cudaEventSynchronize(ev[k & 1]));
      const double* half = stage + 4ull * kChunk * (k & 1);
      format_chunk(f, k * kChunk, std::min(kChunk, n - k * kChunk), half, half + kChunk,
                   half + 2ull * kChunk, half + 3ull * kChunk, line);
    }
  } catch (const Error& e) {
    c->last_error = e.msg;
    st = e.code;
  }
  if (ev[0]) cudaEventDestroy(ev[0]);
  if (ev[1]) cudaEventDestroy(ev[1]);
  if (stage) cudaFreeHost(stage);
  if (std::fclose(f) != 0 && st == BIT_OK) st = BIT_ERR_INVALID_ARGUMENT;
  return st;
}

}  // extern "C"

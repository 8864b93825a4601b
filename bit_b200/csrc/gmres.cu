// GMRES on the device.
//
// bit_bie_solve: restarted GMRES(m) for (diag*I + K) s = f where K is the treecode with
// charges w*s (no reference counterpart: the reference's solver::gmres takes a dense
// matrix, src/solver.h:157-260).  Vectors live in tree order on the device; each matvec
// rewrites the charges, recomputes the moments (FP64) and runs the far and near kernels
// over the interaction lists built once for the tree.  A whole GMRES iteration runs on the
// device -- the matvec, classical Gram-Schmidt applied twice (FP64), the normalisation and
// the FP64 Givens rotation of the new Hessenberg column -- and every iteration after the
// first of each precision replays it as one CUDA graph; the host reads back the residual
// estimate once per iteration and solves the small triangular system once per cycle.
// Mixed precision: FP32 matvecs inside an FP64 iterative refinement whose residual
// f - A s is always recomputed with the FP64 treecode (those matvecs replay a graph too).
//
// bit_gmres_dense: solver::gmres itself (src/solver.h:157-310) for a dense matrix:
// full GMRES from zero, modified Gram-Schmidt, least squares by Gram-Schmidt QR of the
// Hessenberg re-done every step (minimize, :266-310), stop when the max relative change
// of x is below 1e-5 on odd steps (:243-255), breakdown at h < 1e-14 (:220-225).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "common.cuh"

namespace bit {

namespace {

constexpr int RB = 256;

__global__ void k_gather(int n, const int* perm, const double* src, double* dst) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) dst[e] = src[perm[e]];
}
__global__ void k_scatter(int n, const int* perm, const double* src, double* dst) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) dst[perm[e]] = src[e];
}

// charges q = w * s in tree order, written into every source representation
__global__ void k_charges(int n, const double* w, const double* s, double* sq, double4* src64,
                          float4* src32) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  double q = w[e] * s[e];
  sq[e] = q;
  src64[e].w = q;
  src32[e].w = (float)q;
}

// y = a x + b y; with b == 0, y is written without being read (it may be uninitialised,
// e.g. a reused block holding NaN patterns).
__global__ void k_axpby(int n, double a, const double* x, double b, double* y) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) y[e] = b == 0.0 ? a * x[e] : a * x[e] + b * y[e];
}

// Sum over the block, returned to every thread.
__device__ double block_sum(double v) {
  __shared__ double sh[33];
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    v = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) sh[32] = v;
  }
  __syncthreads();
  v = sh[32];
  __syncthreads();
  return v;
}

// partial[j * nblk + b] = sum over block b's elements of V[j] . w, j < k
__global__ void k_dots(int n, int k, const double* V, const double* w, double* partial) {
  const int per = (n + gridDim.x - 1) / gridDim.x;
  const int i0 = blockIdx.x * per, i1 = min(n, i0 + per);
  for (int j = 0; j < k; j++) {
    double a = 0.0;
    const double* v = V + (long long)j * n;
    for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) a += v[i] * w[i];
    a = block_sum(a);
    if (threadIdx.x == 0) partial[j * gridDim.x + blockIdx.x] = a;
  }
}
__global__ void k_dots_finish(int k, int nblk, const double* partial, double* h) {
  int j = blockIdx.x;
  if (j >= k) return;
  double a = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) a += partial[j * nblk + b];
  a = block_sum(a);
  if (threadIdx.x == 0) h[j] = a;
}
// w -= sum_j h[j] V[j]
__global__ void k_orth_update(int n, int k, const double* V, const double* h, double* w) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double a = w[i];
  for (int j = 0; j < k; j++) a -= h[j] * V[(long long)j * n + i];
  w[i] = a;
}
// x += sum_j y[j] V[j]
__global__ void k_combine(int n, int k, const double* V, const double* y, double* x) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double a = x[i];
  for (int j = 0; j < k; j++) a += y[j] * V[(long long)j * n + i];
  x[i] = a;
}

// ---- one GMRES(m) iteration on the device ------------------------------------------------
// Every kernel below reads the iteration's column k from device memory (*dk), and
// k_givens advances it, so the same launch sequence -- and one CUDA graph of it -- serves
// every iteration of a cycle.  The arithmetic is the host loop's: classical Gram-Schmidt
// applied twice, normalisation, the previous Givens rotations applied to the new column, a
// new rotation, and the rotated right-hand side g whose last entry is the residual norm.

// x = V[k]
__global__ void k_basis_in(int n, const double* V, const int* dk, double* x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] = V[(long long)(*dk) * n + i];
}
// V[k + 1] = y
__global__ void k_basis_out(int n, const double* y, double* V, const int* dk) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) V[(long long)(*dk + 1) * n + i] = y[i];
}
// partial[j * nblk + b] = block b's share of V[j] . V[k + 1], j <= k
__global__ void k_dots_k(int n, const double* V, const int* dk, double* partial) {
  const int k = *dk + 1;
  const double* w = V + (long long)k * n;
  const int per = (n + gridDim.x - 1) / gridDim.x;
  const int i0 = blockIdx.x * per, i1 = min(n, i0 + per);
  for (int j = 0; j < k; j++) {
    double a = 0.0;
    const double* v = V + (long long)j * n;
    for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) a += v[i] * w[i];
    a = block_sum(a);
    if (threadIdx.x == 0) partial[j * gridDim.x + blockIdx.x] = a;
  }
}
// htmp[j] = V[j] . V[k + 1] (this pass), hcol[j] += htmp[j]
__global__ void k_dots_k_finish(int nblk, const double* partial, const int* dk, double* htmp,
                                double* hcol) {
  const int j = blockIdx.x;
  if (j > *dk) return;
  double a = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) a += partial[j * nblk + b];
  a = block_sum(a);
  if (threadIdx.x == 0) {
    htmp[j] = a;
    hcol[j] += a;
  }
}
// V[k + 1] -= sum_{j <= k} htmp[j] V[j]
__global__ void k_orth_k(int n, const double* V, const int* dk, const double* htmp, double* Vw) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int k = *dk;
  double* w = Vw + (long long)(k + 1) * n;
  double a = w[i];
  for (int j = 0; j <= k; j++) a -= htmp[j] * V[(long long)j * n + i];
  w[i] = a;
}
// partial[b] = block b's share of |V[k + 1]|^2
__global__ void k_sqnorm_k(int n, const double* V, const int* dk, double* partial) {
  const double* w = V + (long long)(*dk + 1) * n;
  const int per = (n + gridDim.x - 1) / gridDim.x;
  const int i0 = blockIdx.x * per, i1 = min(n, i0 + per);
  double a = 0.0;
  for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) a += w[i] * w[i];
  a = block_sum(a);
  if (threadIdx.x == 0) partial[blockIdx.x] = a;
}
// scal[0] = |V[k + 1]|
__global__ void k_norm_finish(int nblk, const double* partial, double* scal) {
  double a = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) a += partial[b];
  a = block_sum(a);
  if (threadIdx.x == 0) scal[0] = sqrt(a);
}
// V[k + 1] /= |V[k + 1]| (left as it is when the norm is 0)
__global__ void k_scale_k(int n, double* V, const int* dk, const double* scal) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const double hn = scal[0];
  if (i >= n || !(hn > 0)) return;
  double* w = V + (long long)(*dk + 1) * n;
  w[i] = (1.0 / hn) * w[i];
}
// One thread: the rotations of column k (H ld m), scal[1] = |g[k + 1]|, the column
// cleared for the next iteration, k advanced.
__global__ void k_givens(int m, int* dk, double* H, double* cs, double* sn, double* g,
                         double* hcol, double* scal) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int k = *dk;
  hcol[k + 1] = scal[0];
  for (int j = 0; j < k; j++) {
    const double a = hcol[j], b = hcol[j + 1];
    hcol[j] = cs[j] * a + sn[j] * b;
    hcol[j + 1] = -sn[j] * a + cs[j] * b;
  }
  const double den = hypot(hcol[k], hcol[k + 1]);
  cs[k] = den > 0 ? hcol[k] / den : 1.0;
  sn[k] = den > 0 ? hcol[k + 1] / den : 0.0;
  hcol[k] = den;
  hcol[k + 1] = 0.0;
  for (int j = 0; j <= k; j++) H[(long long)j * m + k] = hcol[j];
  g[k + 1] = -sn[k] * g[k];
  g[k] = cs[k] * g[k];
  scal[1] = fabs(g[k + 1]);
  for (int j = 0; j <= k + 1; j++) hcol[j] = 0.0;
  *dk = k + 1;
}

struct Krylov {
  Ctx* c;
  int n;
  int nblk;
  DBuf<double> partial, hdev;
  double* hh;  // pinned
  Krylov(Ctx* ctx, int n_, int maxk) : c(ctx), n(n_) {
    nblk = std::min(2 * c->num_sms, std::max(1, n / 2048));
    partial.ensure(c, (size_t)nblk * (maxk + 2));
    hdev.ensure(c, maxk + 2);
    BIT_CUDA(cudaMallocHost(&hh, (maxk + 2) * sizeof(double)));
  }
  ~Krylov() { cudaFreeHost(hh); }
  // h[0..k) = V[0..k) . w on the host
  void dots(const double* V, int k, const double* w) {
    cudaStream_t s = c->stream;
    count_launch(), k_dots<<<nblk, RB, 0, s>>>(n, k, V, w, partial.p);
    count_launch(), k_dots_finish<<<k, RB, 0, s>>>(k, nblk, partial.p, hdev.p);
    BIT_CUDA(cudaMemcpyAsync(hh, hdev.p, k * sizeof(double), cudaMemcpyDeviceToHost, s));
    BIT_CUDA(cudaStreamSynchronize(s));
  }
  double norm(const double* w) {
    dots(w, 1, w);
    return std::sqrt(hh[0]);
  }
};

struct BieOp {
  Tree* t;
  bit_eval_params prm;
  int nterms;
  double diag;
  DBuf<double> w_s;
  int mv64 = 0, mv32 = 0;
  // One CUDA graph per precision holds a whole matvec (charges, moments, far and near
  // launches, axpby) on fixed buffers; a matvec then copies x in, replays the graph and
  // copies y out.  It is captured on the second matvec of a precision, after the first
  // (eager) one has made every allocation and plan.  Capture failures fall back to eager
  // launches.
  DBuf<double> gin, gout;
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  long long glaunches[2] = {0, 0};  // kernels in each graph
  int eager[2] = {0, 0};
  bool graphs = true;

  ~BieOp() {
    for (auto& g : gexec)
      if (g) cudaGraphExecDestroy(g);
  }

  // y = diag*x + K(w*x), everything in tree order
  void apply_eager(const double* x, double* y, bit_precision prec) {
    Ctx* c = t->ctx;
    cudaStream_t s = c->stream;
    const int n = t->n;
    count_launch(), k_charges<<<grid_for(n, 256), 256, 0, s>>>(n, w_s.p, x, t->sq.p, t->src64.p, t->src32.p);
    tree_moments(t, nterms);
    bit_eval_params p = prm;
    p.precision = prec;
    prepare_particles(t, {p}, 0);
    eval_far(t, &t->plists, t->pplan, t->sx.p, t->sy.p, t->sz.p, y);
    eval_near(t, &t->plists, t->pplan, t->sx.p, t->sy.p, t->sz.p, y);
    count_launch(), k_axpby<<<grid_for(n, 256), 256, 0, s>>>(n, diag, x, 1.0, y);
    BIT_CHECK_LAUNCH();
  }

  bool capture(int pi, bit_precision prec) {
    Ctx* c = t->ctx;
    cudaStream_t s = c->stream;
    gin.ensure(c, t->n);
    gout.ensure(c, t->n);
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    bool ok = true;
    try {
      apply_eager(gin.p, gout.p, prec);
    } catch (const Error&) {
      ok = false;
    }
    const cudaError_t e = cudaStreamEndCapture(s, &g);
    if (!ok || e != cudaSuccess || !g) {
      cudaGetLastError();
      if (g) cudaGraphDestroy(g);
      return false;
    }
    size_t nodes = 0;
    cudaGraphGetNodes(g, nullptr, &nodes);
    std::vector<cudaGraphNode_t> nv(nodes);
    if (nodes) cudaGraphGetNodes(g, nv.data(), &nodes);
    long long kernels = 0;
    for (auto& nd : nv) {
      cudaGraphNodeType ty;
      if (cudaGraphNodeGetType(nd, &ty) == cudaSuccess && ty == cudaGraphNodeTypeKernel) kernels++;
    }
    launch_counter().fetch_sub(kernels);  // counted while capturing, but nothing ran
    const cudaError_t ie = cudaGraphInstantiate(&gexec[pi], g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
      cudaGetLastError();
      gexec[pi] = nullptr;
      return false;
    }
    glaunches[pi] = kernels;
    return true;
  }

  void apply(const double* x, double* y, bit_precision prec) {
    const int pi = prec == BIT_PREC_MIXED ? 1 : 0;
    (prec == BIT_PREC_FP64 ? mv64 : mv32)++;
    if (graphs && !gexec[pi] && eager[pi] >= 1 && !capture(pi, prec)) graphs = false;
    if (!graphs || !gexec[pi]) {
      eager[pi]++;
      apply_eager(x, y, prec);
      return;
    }
    Ctx* c = t->ctx;
    cudaStream_t s = c->stream;
    const size_t bytes = (size_t)t->n * sizeof(double);
    BIT_CUDA(cudaMemcpyAsync(gin.p, x, bytes, cudaMemcpyDeviceToDevice, s));
    BIT_CUDA(cudaGraphLaunch(gexec[pi], s));
    BIT_CUDA(cudaMemcpyAsync(y, gout.p, bytes, cudaMemcpyDeviceToDevice, s));
    launch_counter().fetch_add(glaunches[pi]);
  }
};

// Restarted GMRES(m) on A x = b from x (device, tree order) with matvecs in `prec`; stops
// when the recurrence residual reaches tol*||b|| or after maxit iterations.  Returns the
// iterations used.
// Device state of GMRES(m) for one solve: the Krylov basis and the Arnoldi / Givens
// arrays, on fixed buffers so that one CUDA graph per precision holds a whole iteration
// (the matvec of BieOp on its fixed input / output, the two Gram-Schmidt passes, the
// normalisation and the rotation) and is replayed by every iteration of every cycle.  It
// is captured on a precision's second iteration, after the first (eager) one has made
// every allocation and plan; capture failures fall back to eager launches.
struct GmresState {
  Ctx* c;
  int n, m, nblk;
  DBuf<double> V, w, H, cs, sn, g, hcol, htmp, scal, partial;
  DBuf<int> dk;
  double* hpin = nullptr;  // pinned: scal[0..1] read back each iteration
  cudaGraphExec_t iexec[2] = {nullptr, nullptr};
  long long ilaunches[2] = {0, 0};
  int eager[2] = {0, 0};
  bool graphs = true;
  GmresState(Ctx* ctx, int n_, int m_) : c(ctx), n(n_), m(m_) {
    nblk = std::min(2 * c->num_sms, std::max(1, n / 2048));
    V.ensure(c, (size_t)(m + 1) * n);
    w.ensure(c, n);
    H.ensure(c, (size_t)(m + 1) * m);
    cs.ensure(c, m); sn.ensure(c, m); g.ensure(c, m + 1);
    hcol.ensure(c, m + 2); htmp.ensure(c, m + 2); scal.ensure(c, 4);
    partial.ensure(c, (size_t)nblk * (m + 2));
    dk.ensure(c, 1);
    BIT_CUDA(cudaMallocHost(&hpin, 4 * sizeof(double)));
  }
  ~GmresState() {
    for (auto& g_ : iexec)
      if (g_) cudaGraphExecDestroy(g_);
    if (hpin) cudaFreeHost(hpin);
  }

  // One iteration on column *dk (eager launches).
  void step_eager(BieOp& A, bit_precision prec) {
    cudaStream_t s = c->stream;
    A.gin.ensure(c, n);
    A.gout.ensure(c, n);
    count_launch(), k_basis_in<<<grid_for(n, 256), 256, 0, s>>>(n, V.p, dk.p, A.gin.p);
    A.apply_eager(A.gin.p, A.gout.p, prec);
    count_launch(), k_basis_out<<<grid_for(n, 256), 256, 0, s>>>(n, A.gout.p, V.p, dk.p);
    for (int pass = 0; pass < 2; pass++) {
      count_launch(), k_dots_k<<<nblk, RB, 0, s>>>(n, V.p, dk.p, partial.p);
      count_launch(), k_dots_k_finish<<<m + 1, RB, 0, s>>>(nblk, partial.p, dk.p, htmp.p, hcol.p);
      count_launch(), k_orth_k<<<grid_for(n, 256), 256, 0, s>>>(n, V.p, dk.p, htmp.p, V.p);
    }
    count_launch(), k_sqnorm_k<<<nblk, RB, 0, s>>>(n, V.p, dk.p, partial.p);
    count_launch(), k_norm_finish<<<1, RB, 0, s>>>(nblk, partial.p, scal.p);
    count_launch(), k_scale_k<<<grid_for(n, 256), 256, 0, s>>>(n, V.p, dk.p, scal.p);
    count_launch(), k_givens<<<1, 32, 0, s>>>(m, dk.p, H.p, cs.p, sn.p, g.p, hcol.p, scal.p);
    BIT_CHECK_LAUNCH();
  }

  bool capture(BieOp& A, int pi, bit_precision prec) {
    cudaStream_t s = c->stream;
    cudaGraph_t gr = nullptr;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    const long long l0 = launch_counter().load();
    bool ok = true;
    try {
      step_eager(A, prec);
    } catch (const Error&) {
      ok = false;
    }
    const long long kernels = launch_counter().load() - l0;
    launch_counter().fetch_sub(kernels);  // counted while capturing, but nothing ran
    const cudaError_t e = cudaStreamEndCapture(s, &gr);
    if (!ok || e != cudaSuccess || !gr) {
      cudaGetLastError();
      if (gr) cudaGraphDestroy(gr);
      return false;
    }
    const cudaError_t ie = cudaGraphInstantiate(&iexec[pi], gr, 0);
    cudaGraphDestroy(gr);
    if (ie != cudaSuccess) {
      cudaGetLastError();
      iexec[pi] = nullptr;
      return false;
    }
    ilaunches[pi] = kernels;
    return true;
  }

  // One iteration (graph replay when available); returns (|v|, |g[k+1]|) read back.
  void step(BieOp& A, bit_precision prec, double& hn, double& res) {
    const int pi = prec == BIT_PREC_MIXED ? 1 : 0;
    (prec == BIT_PREC_FP64 ? A.mv64 : A.mv32)++;
    cudaStream_t s = c->stream;
    if (graphs && !iexec[pi] && eager[pi] >= 1 && !capture(A, pi, prec)) graphs = false;
    if (graphs && iexec[pi]) {
      BIT_CUDA(cudaGraphLaunch(iexec[pi], s));
      launch_counter().fetch_add(ilaunches[pi]);
    } else {
      eager[pi]++;
      step_eager(A, prec);
    }
    BIT_CUDA(cudaMemcpyAsync(hpin, scal.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    BIT_CUDA(cudaStreamSynchronize(s));
    hn = hpin[0];
    res = hpin[1];
  }
};

// Restarted GMRES(m) on A x = b from x (device, tree order) with matvecs in `prec`; stops
// when the recurrence residual reaches tol*||b|| or after maxit iterations.  Returns the
// iterations used.  Each iteration runs on the device (GmresState); the host reads two
// numbers per iteration and solves the small triangular system once per cycle.
int gmres_m(BieOp& A, Krylov& K, GmresState& G, const double* b, double* x, int m, double tol,
            int maxit, bit_precision prec, double bnorm, bool x_is_zero) {
  Ctx* c = A.t->ctx;
  cudaStream_t s = c->stream;
  const int n = A.t->n;
  double* w = G.w.p;
  std::vector<double> H((size_t)(m + 1) * m), g(m + 1), y(m);
  int it = 0;
  while (it < maxit) {
    // r = b - A x
    if (x_is_zero) {
      BIT_CUDA(cudaMemcpyAsync(w, b, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    } else {
      A.apply(x, w, prec);
      count_launch(), k_axpby<<<grid_for(n, 256), 256, 0, s>>>(n, 1.0, b, -1.0, w);
    }
    x_is_zero = false;
    double beta = K.norm(w);
    if (beta <= tol * bnorm || beta == 0.0) break;
    count_launch(), k_axpby<<<grid_for(n, 256), 256, 0, s>>>(n, 1.0 / beta, w, 0.0, G.V.p);
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    BIT_CUDA(cudaMemcpyAsync(G.g.p, g.data(), (m + 1) * sizeof(double), cudaMemcpyHostToDevice, s));
    BIT_CUDA(cudaMemsetAsync(G.hcol.p, 0, (m + 2) * sizeof(double), s));
    BIT_CUDA(cudaMemsetAsync(G.dk.p, 0, sizeof(int), s));
    int k = 0;
    bool done = false;
    for (; k < m && it < maxit; k++) {
      it++;
      double hn = 0.0, res = 0.0;
      G.step(A, prec, hn, res);
      if (res <= tol * bnorm || hn == 0.0) {
        k++;
        done = true;
        break;
      }
    }
    // y = R^-1 g on the host (k x k upper triangle of the rotated Hessenberg)
    BIT_CUDA(cudaMemcpyAsync(H.data(), G.H.p, (size_t)k * m * sizeof(double), cudaMemcpyDeviceToHost, s));
    BIT_CUDA(cudaMemcpyAsync(g.data(), G.g.p, k * sizeof(double), cudaMemcpyDeviceToHost, s));
    BIT_CUDA(cudaStreamSynchronize(s));
    for (int i = k - 1; i >= 0; i--) {
      double a = g[i];
      for (int j = i + 1; j < k; j++) a -= H[(size_t)i * m + j] * y[j];
      y[i] = a / H[(size_t)i * m + i];
    }
    BIT_CUDA(cudaMemcpyAsync(K.hdev.p, y.data(), k * sizeof(double), cudaMemcpyHostToDevice, s));
    count_launch(), k_combine<<<grid_for(n, 256), 256, 0, s>>>(n, k, G.V.p, K.hdev.p, x);
    BIT_CHECK_LAUNCH();
    BIT_CUDA(cudaStreamSynchronize(s));  // y (pageable host memory) has been read
    if (done) break;
  }
  BIT_CUDA(cudaStreamSynchronize(s));
  return it;
}

// ---- dense solver::gmres ---------------------------------------------------------------
// v = A q (row-major n x n), one warp per row
__global__ void k_dense_gemv(int n, const double* A, const double* q, double* v) {
  const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  const double* a = A + (long long)row * n;
  double s = 0.0;
  for (int j = lane; j < n; j += 32) s += a[j] * q[j];
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) v[row] = s;
}

// Modified Gram-Schmidt of v against Q[0..k) in one block; h[0..k) and h[k] = ||v||,
// then Q[k] = v / h[k].  (src/solver.h:203-230)
__global__ void k_dense_mgs(int n, int k, const double* Q, double* v, double* h, double* qk) {
  for (int j = 0; j < k; j++) {
    const double* q = Q + (long long)j * n;
    double a = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) a += q[i] * v[i];
    a = block_sum(a);
    if (threadIdx.x == 0) h[j] = a;
    for (int i = threadIdx.x; i < n; i += blockDim.x) v[i] -= a * q[i];
    __syncthreads();
  }
  double t = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) t += v[i] * v[i];
  t = block_sum(t);
  const double hn = sqrt(t);
  if (threadIdx.x == 0) h[k] = hn;
  for (int i = threadIdx.x; i < n; i += blockDim.x) qk[i] = v[i] / hn;
}

// x = Q y and max_i |(old_i - x_i) / old_i|  (src/solver.h:243-255), one block
__global__ void k_dense_update(int n, int k, const double* Q, const double* y, double* x,
                               double* maxerr) {
  __shared__ double sh[32];
  double m = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double old = x[i], a = 0.0;
    for (int j = 0; j < k; j++) a += Q[(long long)j * n + i] * y[j];
    x[i] = a;
    double e = fabs((old - a) / old);
    if (e > m) m = e;
  }
  for (int o = 16; o; o >>= 1) {
    double u = __shfl_xor_sync(0xffffffffu, m, o);
    m = u > m ? u : m;
  }
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) r = sh[w] > r ? sh[w] : r;
    *maxerr = r;
  }
}

}  // namespace

}  // namespace bit

using namespace bit;

namespace {
template <class F>
bit_status guard2(Ctx* c, F&& f) {
  try {
    f();
    c->last_error.clear();
    return BIT_OK;
  } catch (const Error& e) {
    c->last_error = e.msg;
    return e.code;
  } catch (...) {
    c->last_error = "unexpected internal error";
    return BIT_ERR_CUDA;
  }
}
}  // namespace

extern "C" bit_status bit_bie_solve(bit_tree* th, const bit_eval_params* prm, int nterms,
                                    double diag, const double* w, const double* f, double* sol,
                                    const bit_gmres_opts* opts, bit_gmres_info* info) {
  if (!th || !prm || !w || !f || !sol || !opts) return BIT_ERR_INVALID_ARGUMENT;
  Tree* t = &th->t;
  Ctx* c = t->ctx;
  bit_status result = BIT_OK;
  bit_status st = guard2(c, [&] {
    if (opts->restart < 1 || opts->maxit < 1 || !(opts->tol > 0))
      fail(BIT_ERR_INVALID_ARGUMENT, "restart, maxit and tol must be positive");
    if (nterms < 1 || nterms > kNtermsMax) fail(BIT_ERR_INVALID_ARGUMENT, "nterms out of range");
    BIT_CUDA(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    const int n = t->n;
    cudaEvent_t e0, e1;
    BIT_CUDA(cudaEventCreate(&e0));
    BIT_CUDA(cudaEventCreate(&e1));
    BIT_CUDA(cudaEventRecord(e0, s));
    DBuf<double> tmp, b, x, r, d;
    tmp.ensure(c, n); b.ensure(c, n); x.ensure(c, n); r.ensure(c, n); d.ensure(c, n);
    BieOp A;
    A.t = t;
    A.prm = *prm;
    A.nterms = nterms;
    A.diag = diag;
    A.w_s.ensure(c, n);
    copy_h2d(c, tmp.p, w, n * sizeof(double));
    count_launch(), k_gather<<<grid_for(n, 256), 256, 0, s>>>(n, t->perm.p, tmp.p, A.w_s.p);
    copy_h2d(c, tmp.p, f, n * sizeof(double));
    count_launch(), k_gather<<<grid_for(n, 256), 256, 0, s>>>(n, t->perm.p, tmp.p, b.p);
    BIT_CUDA(cudaMemsetAsync(x.p, 0, n * sizeof(double), s));
    if (!t->has_charges) {
      // first use of this tree for a solve: create the source arrays
      tree_set_charges(t, tmp.p, nullptr);
    }
    Krylov K(c, n, opts->restart + 1);
    GmresState G(c, n, opts->restart);
    const double bnorm = K.norm(b.p);
    int iters = 0, refine = 0;
    double relres = 0.0;
    if (bnorm == 0.0) {
      relres = 0.0;
    } else if (opts->precision == BIT_PREC_FP64) {
      iters = gmres_m(A, K, G, b.p, x.p, opts->restart, opts->tol, opts->maxit, BIT_PREC_FP64,
                      bnorm, true);
      A.apply(x.p, r.p, BIT_PREC_FP64);
      count_launch(), k_axpby<<<grid_for(n, 256), 256, 0, s>>>(n, 1.0, b.p, -1.0, r.p);
      relres = K.norm(r.p) / bnorm;
    } else {
      const double itol = opts->inner_tol > 0 ? opts->inner_tol : 1e-4;
      const int maxref = opts->max_refinements > 0 ? opts->max_refinements : 10;
      BIT_CUDA(cudaMemcpyAsync(r.p, b.p, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
      relres = 1.0;
      while (refine < maxref && iters < opts->maxit) {
        // inner: A32 d = r to itol relative to ||r||
        const double rn = K.norm(r.p);
        BIT_CUDA(cudaMemsetAsync(d.p, 0, n * sizeof(double), s));
        iters += gmres_m(A, K, G, r.p, d.p, opts->restart, itol, opts->maxit - iters,
                         BIT_PREC_MIXED, rn, true);
        count_launch(), k_axpby<<<grid_for(n, 256), 256, 0, s>>>(n, 1.0, d.p, 1.0, x.p);
        refine++;
        // true residual with the FP64 treecode
        A.apply(x.p, r.p, BIT_PREC_FP64);
        count_launch(), k_axpby<<<grid_for(n, 256), 256, 0, s>>>(n, 1.0, b.p, -1.0, r.p);
        relres = K.norm(r.p) / bnorm;
        if (relres <= opts->tol) break;
      }
    }
    count_launch(), k_scatter<<<grid_for(n, 256), 256, 0, s>>>(n, t->perm.p, x.p, tmp.p);
    copy_d2h(c, sol, tmp.p, n * sizeof(double));
    BIT_CUDA(cudaEventRecord(e1, s));
    BIT_CUDA(cudaStreamSynchronize(s));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (info) {
      info->iterations = iters;
      info->refinements = refine;
      info->matvecs_fp64 = A.mv64;
      info->matvecs_fp32 = A.mv32;
      info->relres = relres;
      info->seconds = ms * 1e-3;
    }
    if (!(relres <= opts->tol)) result = BIT_ERR_NOT_CONVERGED;
  });
  return st != BIT_OK ? st : result;
}

namespace bit {
namespace {
bool rhs_is_zero(int n, const double* b) {
  for (int i = 0; i < n; i++)
    if (b[i] != 0.0) return false;
  return true;
}
}  // namespace
}  // namespace bit

extern "C" bit_status bit_gmres_dense(bit_ctx* h, int n, const double* a, const double* b,
                                      double* x, int* iterations) {
  if (!h || !a || !b || !x || n < 1) return BIT_ERR_INVALID_ARGUMENT;
  Ctx* c = &h->c;
  // b = 0: x = 0 solves A x = b exactly (the reference would divide by |b| = 0 and fill
  // its Krylov basis with NaN)
  if (rhs_is_zero(n, b)) {
    for (int i = 0; i < n; i++) x[i] = 0.0;
    if (iterations) *iterations = 0;
    return BIT_OK;
  }
  bit_status result = BIT_OK;
  bit_status st = guard2(c, [&] {
    BIT_CUDA(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    DBuf<double> A, Q, v, hd, y, xd, me;
    A.ensure(c, (size_t)n * n);
    Q.ensure(c, (size_t)(n + 1) * n);
    v.ensure(c, n);
    hd.ensure(c, n + 2);
    y.ensure(c, n + 1);
    xd.ensure(c, n);
    me.ensure(c, 1);
    copy_h2d(c, A.p, a, (size_t)n * n * sizeof(double));
    BIT_CUDA(cudaMemcpyAsync(xd.p, x, n * sizeof(double), cudaMemcpyHostToDevice, s));
    double bnorm = 0.0;
    for (int i = 0; i < n; i++) bnorm += b[i] * b[i];
    bnorm = std::sqrt(bnorm);
    std::vector<double> q0(n);
    for (int i = 0; i < n; i++) q0[i] = b[i] / bnorm;
    BIT_CUDA(cudaMemcpyAsync(Q.p, q0.data(), n * sizeof(double), cudaMemcpyHostToDevice, s));
    // Hessenberg, host, h[i][j] with ld n+1
    const int ld = n + 1;
    std::vector<double> H((size_t)(n + 2) * ld, 0.0), V2, Q2, R2, yv(n + 1), hc(n + 2);
    int go = 1, nn = 0;
    while (go) {
      const int n1 = nn + 1;
      count_launch(), k_dense_gemv<<<grid_for(n, 8), 256, 0, s>>>(n, A.p, Q.p + (long long)nn * n, v.p);
      count_launch(), k_dense_mgs<<<1, 1024, 0, s>>>(n, n1, Q.p, v.p, hd.p, Q.p + (long long)n1 * n);
      BIT_CUDA(cudaMemcpyAsync(hc.data(), hd.p, (n1 + 1) * sizeof(double), cudaMemcpyDeviceToHost, s));
      BIT_CUDA(cudaStreamSynchronize(s));
      for (int j = 0; j <= n1; j++) H[(size_t)j * ld + nn] = hc[j];
      if (n1 < n && hc[n1] < 1e-14) {
        go = 0;
        result = BIT_ERR_BREAKDOWN;
      }
      // minimize(n1): Gram-Schmidt QR of the (n1+1) x n1 Hessenberg, back substitution
      const int m = n1;
      V2.assign((size_t)(m + 1) * m, 0.0);
      Q2.assign((size_t)(m + 1) * m, 0.0);
      R2.assign((size_t)m * m, 0.0);
      for (int j = 0; j < m; j++)
        for (int i = 0; i < j + 2; i++) V2[(size_t)i * m + j] = H[(size_t)i * ld + j];
      for (int i = 0; i < m; i++) {
        const int ind = i + 2;
        double rr = 0.0;
        for (int k = 0; k < ind; k++) rr += V2[(size_t)k * m + i] * V2[(size_t)k * m + i];
        rr = std::sqrt(rr);
        R2[(size_t)i * m + i] = rr;
        for (int k = 0; k < ind; k++) Q2[(size_t)k * m + i] = V2[(size_t)k * m + i] / rr;
        for (int j = i + 1; j < m; j++) {
          double r = 0.0;
          for (int k = 0; k < ind; k++) r += Q2[(size_t)k * m + i] * V2[(size_t)k * m + j];
          R2[(size_t)i * m + j] = r;
          for (int k = 0; k < ind; k++) V2[(size_t)k * m + j] -= r * Q2[(size_t)k * m + i];
        }
      }
      for (int i = m - 1; i > -1; i--) {
        double t = bnorm * Q2[i];
        for (int j = i + 1; j < m; j++) t -= R2[(size_t)i * m + j] * yv[j];
        yv[i] = t / R2[(size_t)i * m + i];
      }
      if (n1 == n) go = 0;
      if (n1 % 2 || !go) {
        BIT_CUDA(cudaMemcpyAsync(y.p, yv.data(), n1 * sizeof(double), cudaMemcpyHostToDevice, s));
        count_launch(), k_dense_update<<<1, 1024, 0, s>>>(n, n1, Q.p, y.p, xd.p, me.p);
        double maxerr = 0.0;
        BIT_CUDA(cudaMemcpyAsync(&maxerr, me.p, sizeof(double), cudaMemcpyDeviceToHost, s));
        BIT_CUDA(cudaStreamSynchronize(s));
        if (maxerr < 1e-5 && nn > 1) go = 0;
      }
      nn++;
    }
    BIT_CUDA(cudaMemcpyAsync(x, xd.p, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    BIT_CUDA(cudaStreamSynchronize(s));
    if (iterations) *iterations = nn;
  });
  return st != BIT_OK ? st : result;
}

// ---- bit_gmres_dense_static: the dense GMRES above with no allocation at call time ------
// Device scratch is one file-scope array sized for n <= BIT_GMRES_STATIC_MAX; host scratch
// (Hessenberg and the least-squares work arrays) is file-scope too.  Every call looks up the
// array's address in the CUDA context current on the calling thread (cudaGetSymbolAddress:
// no allocation once the module is loaded).  The address is not cached: after
// cudaDeviceReset, or with another context current on the same device, the module is
// loaded anew and the array lives elsewhere.  The first call in a context may load the
// module (CUDA's lazy loading), which creates the array: make it once as a warm-up outside
// any region that must not allocate, and before any stream capture.  Calls that overlap in
// time (two host threads, or two streams of one device) share this scratch and race.
namespace bit {
namespace {

constexpr int kStaticMax = BIT_GMRES_STATIC_MAX;
constexpr size_t rup32(size_t v) { return (v + 31) / 32 * 32; }
// segments, in doubles, each a multiple of 256 bytes
constexpr size_t kSegA = rup32((size_t)kStaticMax * kStaticMax);
constexpr size_t kSegQ = rup32((size_t)(kStaticMax + 1) * kStaticMax);
constexpr size_t kSegV = rup32(kStaticMax);
constexpr size_t kSegH = rup32(kStaticMax + 2);
constexpr size_t kSegY = rup32(kStaticMax + 1);
constexpr size_t kSegX = rup32(kStaticMax);
constexpr size_t kSegE = 32;
constexpr size_t kStaticDoubles = kSegA + kSegQ + kSegV + kSegH + kSegY + kSegX + kSegE;

static __device__ __align__(256) double g_dense_static[kStaticDoubles];

constexpr size_t kLd = kStaticMax + 1;
double s_H[(kStaticMax + 2) * kLd];
double s_V2[(kStaticMax + 1) * kStaticMax];
double s_Q2[(kStaticMax + 1) * kStaticMax];
double s_R2[kStaticMax * kStaticMax];
double s_yv[kStaticMax + 1];
double s_hc[kStaticMax + 2];
double s_q0[kStaticMax];

void put_err(char* err, int len, const char* what, const char* detail) {
  if (err && len > 0) std::snprintf(err, (size_t)len, "%s%s%s", what, detail ? ": " : "", detail ? detail : "");
}

}  // namespace
}  // namespace bit

#define BIT_STATIC_CK(call)                                                    \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) {                                                   \
      bit::put_err(err, errlen, #call, cudaGetErrorString(e_));                \
      return BIT_ERR_CUDA;                                                     \
    }                                                                          \
  } while (0)

extern "C" bit_status bit_gmres_dense_static(void* stream, int n, const double* a,
                                             const double* b, double* x, int* iterations,
                                             char* err, int errlen) {
  using namespace bit;
  if (err && errlen > 0) err[0] = '\0';
  if (!a || !b || !x || n < 1) {
    put_err(err, errlen, "a, b and x must be non-NULL and n >= 1", nullptr);
    return BIT_ERR_INVALID_ARGUMENT;
  }
  if (n > kStaticMax) {
    char d[96];
    std::snprintf(d, sizeof d, "n = %d exceeds the static scratch limit %d", n, kStaticMax);
    put_err(err, errlen, "bit_gmres_dense_static", d);
    return BIT_ERR_CAPACITY;
  }
  if (rhs_is_zero(n, b)) {  // as bit_gmres_dense: x = 0, no device work
    for (int i = 0; i < n; i++) x[i] = 0.0;
    if (iterations) *iterations = 0;
    return BIT_OK;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  void* sym = nullptr;
  BIT_STATIC_CK(cudaGetSymbolAddress(&sym, g_dense_static));
  double* base = static_cast<double*>(sym);
  double* A = base;
  double* Q = A + kSegA;
  double* v = Q + kSegQ;
  double* hd = v + kSegV;
  double* y = hd + kSegH;
  double* xd = y + kSegY;
  double* me = xd + kSegX;
  // the reductions' outputs start from zero on every call
  BIT_STATIC_CK(cudaMemsetAsync(hd, 0, kSegH * sizeof(double), s));
  BIT_STATIC_CK(cudaMemsetAsync(me, 0, kSegE * sizeof(double), s));
  BIT_STATIC_CK(cudaMemcpyAsync(A, a, (size_t)n * n * sizeof(double), cudaMemcpyHostToDevice, s));
  BIT_STATIC_CK(cudaMemcpyAsync(xd, x, n * sizeof(double), cudaMemcpyHostToDevice, s));
  double bnorm = 0.0;
  for (int i = 0; i < n; i++) bnorm += b[i] * b[i];
  bnorm = std::sqrt(bnorm);
  for (int i = 0; i < n; i++) s_q0[i] = b[i] / bnorm;
  BIT_STATIC_CK(cudaMemcpyAsync(Q, s_q0, n * sizeof(double), cudaMemcpyHostToDevice, s));
  // the copies above read host scratch asynchronously: finish them before it is reused
  BIT_STATIC_CK(cudaStreamSynchronize(s));
  const int ld = n + 1;
  std::memset(s_H, 0, (size_t)(n + 2) * ld * sizeof(double));
  bit_status result = BIT_OK;
  int go = 1, nn = 0;
  while (go) {
    const int n1 = nn + 1;
    count_launch(), k_dense_gemv<<<grid_for(n, 8), 256, 0, s>>>(n, A, Q + (long long)nn * n, v);
    count_launch(), k_dense_mgs<<<1, 1024, 0, s>>>(n, n1, Q, v, hd, Q + (long long)n1 * n);
    BIT_STATIC_CK(cudaGetLastError());
    BIT_STATIC_CK(cudaMemcpyAsync(s_hc, hd, (n1 + 1) * sizeof(double), cudaMemcpyDeviceToHost, s));
    BIT_STATIC_CK(cudaStreamSynchronize(s));
    for (int j = 0; j <= n1; j++) s_H[(size_t)j * ld + nn] = s_hc[j];
    if (n1 < n && s_hc[n1] < 1e-14) {
      go = 0;
      result = BIT_ERR_BREAKDOWN;
    }
    // minimize(n1): Gram-Schmidt QR of the (n1+1) x n1 Hessenberg, back substitution
    const int m = n1;
    std::memset(s_V2, 0, (size_t)(m + 1) * m * sizeof(double));
    std::memset(s_Q2, 0, (size_t)(m + 1) * m * sizeof(double));
    std::memset(s_R2, 0, (size_t)m * m * sizeof(double));
    for (int j = 0; j < m; j++)
      for (int i = 0; i < j + 2; i++) s_V2[(size_t)i * m + j] = s_H[(size_t)i * ld + j];
    for (int i = 0; i < m; i++) {
      const int ind = i + 2;
      double rr = 0.0;
      for (int k = 0; k < ind; k++) rr += s_V2[(size_t)k * m + i] * s_V2[(size_t)k * m + i];
      rr = std::sqrt(rr);
      s_R2[(size_t)i * m + i] = rr;
      for (int k = 0; k < ind; k++) s_Q2[(size_t)k * m + i] = s_V2[(size_t)k * m + i] / rr;
      for (int j = i + 1; j < m; j++) {
        double r = 0.0;
        for (int k = 0; k < ind; k++) r += s_Q2[(size_t)k * m + i] * s_V2[(size_t)k * m + j];
        s_R2[(size_t)i * m + j] = r;
        for (int k = 0; k < ind; k++) s_V2[(size_t)k * m + j] -= r * s_Q2[(size_t)k * m + i];
      }
    }
    for (int i = m - 1; i > -1; i--) {
      double t = bnorm * s_Q2[i];
      for (int j = i + 1; j < m; j++) t -= s_R2[(size_t)i * m + j] * s_yv[j];
      s_yv[i] = t / s_R2[(size_t)i * m + i];
    }
    if (n1 == n) go = 0;
    if (n1 % 2 || !go) {
      BIT_STATIC_CK(cudaMemcpyAsync(y, s_yv, n1 * sizeof(double), cudaMemcpyHostToDevice, s));
      count_launch(), k_dense_update<<<1, 1024, 0, s>>>(n, n1, Q, y, xd, me);
      BIT_STATIC_CK(cudaGetLastError());
      double maxerr = 0.0;
      BIT_STATIC_CK(cudaMemcpyAsync(&maxerr, me, sizeof(double), cudaMemcpyDeviceToHost, s));
      BIT_STATIC_CK(cudaStreamSynchronize(s));
      if (maxerr < 1e-5 && nn > 1) go = 0;
    }
    nn++;
  }
  BIT_STATIC_CK(cudaMemcpyAsync(x, xd, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  BIT_STATIC_CK(cudaStreamSynchronize(s));
  if (iterations) *iterations = nn;
  if (result == BIT_ERR_BREAKDOWN) put_err(err, errlen, "GMRES breakdown (h < 1e-14)", nullptr);
  return result;
}
#undef BIT_STATIC_CK

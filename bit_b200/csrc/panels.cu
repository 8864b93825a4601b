// Boundary panels of a box and the panel (boundary-integral) solve.
//
// bit_panels_box restates setboundaries / panelinit (src/tree3d.cpp:3764-3934,
// 3984-4018): the six faces of a box centred at the origin cut into xpanels x ypanels
// x zpanels rectangles, Dirichlet, with the reference's hard-coded reference potentials
// (-50 on the xy faces; on the other faces -50, or 0 where the panel lies in 4 < z < 5).
// The panel order, coordinates, midpoints and areas are the reference's, so a caller's
// panel indices carry over.
//
// bit_panel_matrix is panelconstantsreal (src/tree3d.cpp:4054-4078) on the device:
// A[i][j] = -1 / sqrt(|m_i - m_j|^2 + del) / 2 * inv2pi * area_j, midpoint quadrature,
// formed without contraction in the reference's operation order (bit-exact).
//
// bit_panel_solve is the panel solve the reference left commented out (panel_solve_tree,
// src/tree3d.cpp:4351-4438), revived on the treecode: b_i = refpot_i + 0.5 sum_j q_j / r_ij
// (particles at the panel midpoints, FP64 direct sum), then A sigma = b.  With panel
// charges tau_j = area_j sigma_j the dense system is
//   tau_i / sqrt(del) + sum_{j != i} tau_j / sqrt(r_ij^2 + del) = -4 pi b_i,
// i.e. (diag I + K) tau = f with the regularised Coulomb treecode K over the midpoints,
// which bit_bie_solve solves with GMRES(m); sigma_i = tau_i / area_i.
#include <cmath>
#include <vector>

#include "common.cuh"

namespace bit {
namespace {

constexpr double kPi = 3.14159265359;  // src/constants.h:12
constexpr double kInv2Pi = 0.5 / kPi;  // src/constants.h:13

void panel_init(bit_panel* p, double x0, double x1, double y0, double y1, double z0,
                double z1, double refpot, double xn, double yn, double zn, int type,
                int orientation) {
  *p = bit_panel{};
  p->x0 = x0; p->x1 = x1; p->y0 = y0; p->y1 = y1; p->z0 = z0; p->z1 = z1;
  p->midx = 0.5 * (x1 + x0);
  p->midy = 0.5 * (y1 + y0);
  p->midz = 0.5 * (z1 + z0);
  p->refpot = refpot;
  p->xnrm = xn; p->ynrm = yn; p->znrm = zn;
  p->type = type;
  p->orientation = orientation;
  switch (orientation) {
    case 1: p->area = (x1 - x0) * (y1 - y0); break;
    case 2: p->area = (x1 - x0) * (z1 - z0); break;
    case 3: p->area = (z1 - z0) * (y1 - y0); break;
  }
}

// Cut points of one side: -half, step - half, ..., half.
std::vector<double> cuts(int n, double len) {
  std::vector<double> c(n + 1);
  const double half = len / 2.0, step = len / n;
  c[0] = 0.0 - half;
  for (int i = 1; i < n; i++) c[i] = i * step - half;
  c[n] = half;
  return c;
}

__global__ void k_panel_matrix(int n, const double* mx, const double* my, const double* mz,
                               const double* area, double del, double* A) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (long long)n * n) return;
  const int i = (int)(k / n), j = (int)(k % n);
  const double dx = dsub(mx[i], mx[j]), dy = dsub(my[i], my[j]), dz = dsub(mz[i], mz[j]);
  const double r = __dsqrt_rn(dadd(dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz)), del));
  A[k] = dmul(dmul(__ddiv_rn(__ddiv_rn(-1.0, r), 2.0), kInv2Pi), area[j]);
}

// f_i = -4 pi (refpot_i + 0.5 sum_j q_j / r_ij): one block per panel, fixed order.
__global__ void k_panel_rhs(int npan, const double* mx, const double* my, const double* mz,
                            const double* refpot, int np, const double* x, const double* y,
                            const double* z, const double* q, double* f) {
  __shared__ double sh[256];
  const int i = blockIdx.x;
  double acc = 0.0;
  for (int j = threadIdx.x; j < np; j += blockDim.x) {
    const double dx = mx[i] - x[j], dy = my[i] - y[j], dz = mz[i] - z[j];
    acc += 0.5 / sqrt(dx * dx + dy * dy + dz * dz) * q[j];
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) f[i] = -4.0 * kPi * (refpot[i] + sh[0]);
}

}  // namespace
}  // namespace bit

using namespace bit;

extern "C" {

bit_status bit_panels_box(int xp, int yp, int zp, double dl, double dh, double dd,
                          bit_panel* pan, int* numpan) {
  if (!numpan || xp < 1 || yp < 1 || zp < 1) return BIT_ERR_INVALID_ARGUMENT;
  *numpan = 2 * (xp * yp + zp * yp + xp * zp);
  if (!pan) return BIT_OK;
  const int dir = 0;  // Dirichlet, the only kind the reference codes
  const double xy_top = -50.0, xy_bot = -50.0, in_band = 0.0, out_band = -50.0;
  const std::vector<double> x = cuts(xp, dl), y = cuts(yp, dh), z = cuts(zp, dd);
  const double hl = dl / 2.0, hh = dh / 2.0, hd = dd / 2.0;
  int tot = 0;
  auto band = [](double a, double b) { return a > 4 && b < 5; };
  for (int i = 0; i < xp; i++, tot += yp)  // bottom, normal +z
    for (int j = 0; j < yp; j++)
      panel_init(&pan[tot + j], x[i], x[i + 1], y[j], y[j + 1], -hd, -hd, xy_bot, 0, 0, 1, dir, 1);
  for (int i = 0; i < xp; i++, tot += yp)  // top, normal -z
    for (int j = 0; j < yp; j++)
      panel_init(&pan[tot + j], x[i], x[i + 1], y[j], y[j + 1], hd, hd, xy_top, 0, 0, -1, dir, 1);
  for (int i = 0; i < zp; i++, tot += yp)  // left, normal +x
    for (int j = 0; j < yp; j++)
      panel_init(&pan[tot + j], -hl, -hl, y[j], y[j + 1], z[i], z[i + 1],
                 band(z[i], z[i + 1]) ? in_band : out_band, 1, 0, 0, dir, 3);
  for (int i = 0; i < zp; i++, tot += yp)  // right, normal -x
    for (int j = 0; j < yp; j++)
      panel_init(&pan[tot + j], hl, hl, y[j], y[j + 1], z[i], z[i + 1],
                 band(z[i], z[i + 1]) ? in_band : out_band, -1, 0, 0, dir, 3);
  for (int i = 0; i < xp; i++, tot += zp)  // front, normal +y
    for (int j = 0; j < zp; j++)
      panel_init(&pan[tot + j], x[i], x[i + 1], -hh, -hh, z[j], z[j + 1],
                 band(z[j], z[j + 1]) ? in_band : out_band, 0, 1, 0, dir, 2);
  for (int i = 0; i < xp; i++, tot += zp)  // back, normal -y
    for (int j = 0; j < zp; j++)
      panel_init(&pan[tot + j], x[i], x[i + 1], hh, hh, z[j], z[j + 1],
                 band(z[j], z[j + 1]) ? in_band : out_band, 0, -1, 0, dir, 2);
  return BIT_OK;
}

bit_status bit_panel_matrix(bit_ctx* h, int n, const bit_panel* pan, double del, double* A) {
  if (!h || !pan || !A || n < 1) return BIT_ERR_INVALID_ARGUMENT;
  Ctx* c = &h->c;
  try {
    BIT_CUDA(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    std::vector<double> m(4LL * n);
    for (int i = 0; i < n; i++) {
      m[i] = pan[i].midx; m[n + i] = pan[i].midy; m[2LL * n + i] = pan[i].midz;
      m[3LL * n + i] = pan[i].area;
    }
    DBuf<double> dm, dA;
    dm.ensure(c, 4LL * n);
    dA.ensure(c, (size_t)n * n);
    BIT_CUDA(cudaMemcpyAsync(dm.p, m.data(), 4LL * n * sizeof(double), cudaMemcpyHostToDevice, s));
    count_launch(), k_panel_matrix<<<grid_for((long long)n * n, 256), 256, 0, s>>>(
        n, dm.p, dm.p + n, dm.p + 2LL * n, dm.p + 3LL * n, del, dA.p);
    BIT_CHECK_LAUNCH();
    BIT_CUDA(cudaMemcpyAsync(A, dA.p, (size_t)n * n * sizeof(double), cudaMemcpyDeviceToHost, s));
    BIT_CUDA(cudaStreamSynchronize(s));
  } catch (const Error& e) {
    c->last_error = e.msg;
    return e.code;
  }
  c->last_error.clear();
  return BIT_OK;
}

bit_status bit_panel_solve(bit_ctx* h, int npan, bit_panel* pan, int np, const double* x,
                           const double* y, const double* z, const double* q, double del,
                           int nterms, double acc, int maxmemb, const bit_gmres_opts* opts,
                           bit_gmres_info* info) {
  if (!h || !pan || npan < 1 || np < 0 || (np > 0 && (!x || !y || !z || !q)) || !opts ||
      !(del > 0))
    return BIT_ERR_INVALID_ARGUMENT;
  Ctx* c = &h->c;
  std::vector<double> mx(npan), my(npan), mz(npan), rp(npan), f(npan), ones(npan, 1.0),
      tau(npan);
  for (int i = 0; i < npan; i++) {
    mx[i] = pan[i].midx; my[i] = pan[i].midy; mz[i] = pan[i].midz; rp[i] = pan[i].refpot;
  }
  try {
    BIT_CUDA(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    DBuf<double> dm, dp, df;
    dm.ensure(c, 4LL * npan);
    BIT_CUDA(cudaMemcpyAsync(dm.p, mx.data(), npan * sizeof(double), cudaMemcpyHostToDevice, s));
    BIT_CUDA(cudaMemcpyAsync(dm.p + npan, my.data(), npan * sizeof(double), cudaMemcpyHostToDevice, s));
    BIT_CUDA(cudaMemcpyAsync(dm.p + 2LL * npan, mz.data(), npan * sizeof(double), cudaMemcpyHostToDevice, s));
    BIT_CUDA(cudaMemcpyAsync(dm.p + 3LL * npan, rp.data(), npan * sizeof(double), cudaMemcpyHostToDevice, s));
    const int npp = np > 0 ? np : 1;
    dp.ensure(c, 4LL * npp);
    if (np > 0) {
      BIT_CUDA(cudaMemcpyAsync(dp.p, x, np * sizeof(double), cudaMemcpyHostToDevice, s));
      BIT_CUDA(cudaMemcpyAsync(dp.p + np, y, np * sizeof(double), cudaMemcpyHostToDevice, s));
      BIT_CUDA(cudaMemcpyAsync(dp.p + 2LL * np, z, np * sizeof(double), cudaMemcpyHostToDevice, s));
      BIT_CUDA(cudaMemcpyAsync(dp.p + 3LL * np, q, np * sizeof(double), cudaMemcpyHostToDevice, s));
    }
    df.ensure(c, npan);
    count_launch(), k_panel_rhs<<<npan, 256, 0, s>>>(npan, dm.p, dm.p + npan, dm.p + 2LL * npan,
                                                   dm.p + 3LL * npan, np, dp.p, dp.p + npp,
                                                   dp.p + 2LL * npp, dp.p + 3LL * npp, df.p);
    BIT_CHECK_LAUNCH();
    BIT_CUDA(cudaMemcpyAsync(f.data(), df.p, npan * sizeof(double), cudaMemcpyDeviceToHost, s));
    BIT_CUDA(cudaStreamSynchronize(s));
  } catch (const Error& e) {
    c->last_error = e.msg;
    return e.code;
  }
  bit_tree* t = nullptr;
  bit_status st = bit_tree_build(h, npan, mx.data(), my.data(), mz.data(), maxmemb, &t);
  if (st != BIT_OK) return st;
  bit_eval_params p{};
  p.kernel = BIT_KERNEL_COULOMB;
  p.mode = BIT_MODE_CONSISTENT;
  p.precision = BIT_PREC_FP64;
  p.del = del;
  p.acc = acc;
  st = bit_bie_solve(t, &p, nterms, 1.0 / std::sqrt(del), ones.data(), f.data(), tau.data(),
                     opts, info);
  std::string keep = c->last_error;
  bit_tree_destroy(t);
  c->last_error = keep;
  if (st == BIT_OK || st == BIT_ERR_NOT_CONVERGED)
    for (int i = 0; i < npan; i++) pan[i].str = tau[i] / pan[i].area;
  return st;
}

}  // extern "C"

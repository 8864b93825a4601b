// FP64 direct sums at selected particle targets: the O(N^2) reference every treecode
// result is measured against (shielded_pot_particle_ds, src/tree3d.cpp:1966-2016, and the
// Coulomb / regularised-screened sums of the same form).  The target itself is skipped by
// index, as in the reference (`if (i != ind)`).
//
// One CTA per (tile of 256 targets, chunk of sources): the chunk's sources are staged in
// shared memory 1024 at a time and every thread sums them for its target in source order.
// Per-chunk partial sums are then added per target in chunk order, so the result is
// deterministic.
#include <vector>

#include "common.cuh"

namespace bit {

namespace {

constexpr int DT = 256;      // targets per CTA
constexpr int DS = 1024;     // sources staged per tile
constexpr int DCH = 16384;   // sources per chunk

template <int KER>
__global__ void __launch_bounds__(DT) k_direct(int n, const double* x, const double* y,
                                               const double* z, const double* q, int m,
                                               const int* tg, double del, double kappa,
                                               double* part, int* err) {
  __shared__ double4 S[DS];
  const int ti = blockIdx.x * DT + threadIdx.x;
  const int j0 = blockIdx.y * DCH, j1 = min(n, j0 + DCH);
  int p = ti < m ? tg[ti] : -1;
  if (p >= n || p < -1) {  // a target index outside the sources: flag it, sum nothing
    if (blockIdx.y == 0) atomicOr(err, 4);
    p = -1;
  }
  double X = 0, Y = 0, Z = 0;
  if (p >= 0) { X = x[p]; Y = y[p]; Z = z[p]; }
  double acc = 0.0;
  for (int s0 = j0; s0 < j1; s0 += DS) {
    const int cnt = min(DS, j1 - s0);
    __syncthreads();
    for (int k = threadIdx.x; k < cnt; k += DT)
      S[k] = make_double4(x[s0 + k], y[s0 + k], z[s0 + k], q[s0 + k]);
    __syncthreads();
    if (p < 0) continue;
    const int self = p - s0;  // tile index of the target itself (skipped)
    for (int k = 0; k < cnt; k++) {
      if (k == self) continue;
      const double4 s = S[k];
      const double dx = X - s.x, dy = Y - s.y, dz = Z - s.z;
      double r2 = dx * dx + dy * dy + dz * dz;
      if (KER == BIT_KERNEL_COULOMB) {
        r2 += del;
        if (r2 > kEpsNear) acc += s.w / sqrt(r2);
      } else if (KER == BIT_KERNEL_SCREENED) {
        const double r = sqrt(r2);
        acc += s.w * exp(-kappa * r) / r;
      } else {
        r2 += del;
        if (r2 > kEpsNear) {
          const double r = sqrt(r2);
          acc += s.w * exp(-kappa * r) / r;
        }
      }
    }
  }
  if (ti < m) part[(long long)blockIdx.y * m + ti] = acc;
}

// Field direct sums, force_particle_ds_reg (src/tree3d.cpp:298-330, with the KERNEL_ORDER
// family of eval_grad_kernel_reg, :73-97) and force_particle_ds_noreg (:182-213):
// sum over j != target of q_j G(x_j - x), G(d) = -d t, t = 1/(r rs) (+ korder terms) with
// rs = |d|^2 + del (REG) or t = 1/(rs sqrt(rs)) with rs = |d|^2.  Three partial sums per
// (chunk, target): part[(c * 3 + axis) * m + ti].
template <bool REG>
__global__ void __launch_bounds__(DT) k_direct_field(int n, const double* x, const double* y,
                                                     const double* z, const double* q, int m,
                                                     const int* tg, double del, int korder,
                                                     double* part, int* err) {
  __shared__ double4 S[DS];
  const int ti = blockIdx.x * DT + threadIdx.x;
  const int j0 = blockIdx.y * DCH, j1 = min(n, j0 + DCH);
  int p = ti < m ? tg[ti] : -1;
  if (p >= n || p < -1) {
    if (blockIdx.y == 0) atomicOr(err, 4);
    p = -1;
  }
  double X = 0, Y = 0, Z = 0;
  if (p >= 0) { X = x[p]; Y = y[p]; Z = z[p]; }
  double ax = 0.0, ay = 0.0, az = 0.0;
  for (int s0 = j0; s0 < j1; s0 += DS) {
    const int cnt = min(DS, j1 - s0);
    __syncthreads();
    for (int k = threadIdx.x; k < cnt; k += DT)
      S[k] = make_double4(x[s0 + k], y[s0 + k], z[s0 + k], q[s0 + k]);
    __syncthreads();
    if (p < 0) continue;
    const int self = p - s0;
    for (int k = 0; k < cnt; k++) {
      if (k == self) continue;
      const double4 s = S[k];
      const double dx = s.x - X, dy = s.y - Y, dz = s.z - Z;
      double t;
      if (REG) {
        const double rs = dx * dx + dy * dy + dz * dz + del;
        const double r = sqrt(rs);
        t = 1.0 / (r * rs);
        double f = t;
        for (int l = 1; l <= korder; l++) {
          f = f * (l + 0.5) / l * del / rs;
          t += f;
        }
      } else {
        const double rs = dx * dx + dy * dy + dz * dz;
        t = 1 / (rs * sqrt(rs));
      }
      ax += s.w * (-dx * t);
      ay += s.w * (-dy * t);
      az += s.w * (-dz * t);
    }
  }
  if (ti < m) {
    const long long b = (long long)blockIdx.y * 3 * m + ti;
    part[b] = ax;
    part[b + m] = ay;
    part[b + 2LL * m] = az;
  }
}

// out[i] = sign * sum over chunks of part[c][i], in chunk order
__global__ void k_direct_sum(int m, int nch, const double* part, double sign, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  double s = 0.0;
  for (int c = 0; c < nch; c++) s += part[(long long)c * m + i];
  out[i] = sign * s;
}

// out[axis * m + i] = sum over chunks of part[(c * 3 + axis) * m + i], in chunk order
__global__ void k_direct_field_sum(int m, int nch, const double* part, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3 * m) return;
  const int axis = i / m, ti = i - axis * m;
  double s = 0.0;
  for (int c = 0; c < nch; c++) s += part[((long long)c * 3 + axis) * m + ti];
  out[i] = s;
}

}  // namespace

// All pointers on the device; out holds fx, fy, fz of the m targets (3 m doubles).
void direct_field(Ctx* c, int n, const double* x, const double* y, const double* z,
                  const double* q, int regularised, double del, int korder, int m,
                  const int* tg, double* out) {
  cudaStream_t s = c->stream;
  const int nch = (n + DCH - 1) / DCH;
  DBuf<double> part;
  part.ensure(c, (size_t)nch * 3 * m);
  const dim3 grid((m + DT - 1) / DT, nch);
  int* err = c->dev_err();
  if (regularised)
    count_launch(), k_direct_field<true><<<grid, DT, 0, s>>>(n, x, y, z, q, m, tg, del, korder, part.p, err);
  else
    count_launch(), k_direct_field<false><<<grid, DT, 0, s>>>(n, x, y, z, q, m, tg, del, korder, part.p, err);
  count_launch(), k_direct_field_sum<<<grid_for(3LL * m, 256), 256, 0, s>>>(m, nch, part.p, out);
  BIT_CHECK_LAUNCH();
}

// All pointers on the device.  The screened sum is negated (src/tree3d.cpp:2014).
void direct_potential(Ctx* c, int n, const double* x, const double* y, const double* z,
                      const double* q, const bit_eval_params& p, int m, const int* tg,
                      double* out) {
  cudaStream_t s = c->stream;
  const int nch = (n + DCH - 1) / DCH;
  DBuf<double> part;
  part.ensure(c, (size_t)nch * m);
  const dim3 grid((m + DT - 1) / DT, nch);
  int* err = c->dev_err();
  switch (p.kernel) {
    case BIT_KERNEL_COULOMB:
      count_launch(), k_direct<BIT_KERNEL_COULOMB><<<grid, DT, 0, s>>>(n, x, y, z, q, m, tg, p.del, p.kappa, part.p, err);
      break;
    case BIT_KERNEL_SCREENED:
      count_launch(), k_direct<BIT_KERNEL_SCREENED><<<grid, DT, 0, s>>>(n, x, y, z, q, m, tg, p.del, p.kappa, part.p, err);
      break;
    default:
      count_launch(), k_direct<BIT_KERNEL_SCREENED_REG><<<grid, DT, 0, s>>>(n, x, y, z, q, m, tg, p.del, p.kappa, part.p, err);
      break;
  }
  const double sign = p.kernel == BIT_KERNEL_SCREENED ? -1.0 : 1.0;
  count_launch(), k_direct_sum<<<grid_for(m, 256), 256, 0, s>>>(m, nch, part.p, sign, out);
  BIT_CHECK_LAUNCH();
}

}  // namespace bit

// Harmonic bond and angle kernels (flexible water), shared by the bonded operators
// (bonded.cu) and the fused system evaluation (fused.cu). Reference: torchff/bond.py:34-43,
// torchff/angle.py:8-34, 103-112 (pure-torch forms); csrc/bond/harmonic_bond_cuda.cu,
// csrc/angle/harmonic_angle_cuda.cu (device kernels).
#pragma once

#include <math.h>

#include "tff_common.cuh"

namespace tff {
namespace {

constexpr int kBondBlock = 256;

struct BondedWs {
  size_t gx, partials, ticket, energy, bytes;
};

inline BondedWs bonded_ws(int64_t natoms, int nblocks) {
  BondedWs w;
  Carver c(nullptr);
  w.gx = c.off; c.take<char>(3 * natoms * 8);
  w.partials = (c.off + 255) & ~size_t(255); c.take<double>(nblocks);
  w.ticket = (c.off + 255) & ~size_t(255); c.take<unsigned>(1);
  w.energy = (c.off + 255) & ~size_t(255); c.take<double>(1);
  w.bytes = c.bytes();
  return w;
}

int bonded_blocks(int64_t nterms) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((nterms + kBondBlock - 1) / kBondBlock, (int64_t)sm_count() * 4));
}

// E = 1/2 k (r - b0)^2, r = |x_j - x_i| (no periodic image, as the reference). Adds
// dE/dx into gx (nullable); writes dE/db0 = -k dr and dE/dk = dr^2 / 2 (nullable); the
// energy through the fixed-order grid reduction into *energy (nullable).
template <class T>
__global__ void __launch_bounds__(kBondBlock) harmonic_bond_kernel(const T *x, const int64_t *bonds, int64_t nb,
                                                                   const T *b0, const T *k, typename Acc<T>::S *gx,
                                                                   T *gb0, T *gk, double *partials, unsigned *ticket,
                                                                   double *energy) {
  pdl_enter();
  double e = 0.0;
  for (int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m < nb; m += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = bonds[2 * m], j = bonds[2 * m + 1];
    const T dx = x[3 * j] - x[3 * i], dy = x[3 * j + 1] - x[3 * i + 1], dz = x[3 * j + 2] - x[3 * i + 2];
    const T r = sqrt(dx * dx + dy * dy + dz * dz);
    const T kk = k[m], dr = r - b0[m];
    e += (double)(T(0.5) * kk * dr * dr);
    if (gx) {
      const T s = kk * dr / r;
      Acc<T>::add(&gx[3 * j], (double)(s * dx));
      Acc<T>::add(&gx[3 * j + 1], (double)(s * dy));
      Acc<T>::add(&gx[3 * j + 2], (double)(s * dz));
      Acc<T>::add(&gx[3 * i], -(double)(s * dx));
      Acc<T>::add(&gx[3 * i + 1], -(double)(s * dy));
      Acc<T>::add(&gx[3 * i + 2], -(double)(s * dz));
    }
    if (gb0) gb0[m] = -kk * dr;
    if (gk) gk[m] = T(0.5) * dr * dr;
  }
  if (energy) grid_sum<kBondBlock>(e, partials, ticket, energy, false);
}

// Angle at the central atom j of (i, j, k) and, with the unit vectors u = v1/|v1|,
// w = v2/|v2| (v1 = x_i - x_j, v2 = x_k - x_j), dtheta/dv1 = -(w - c u) / (|v1| s) and
// dtheta/dv2 = -(u - c w) / (|v2| s), c = cos(theta), s = sin(theta) (floored at 1e-30
// for straight angles, where the derivative is unbounded).
template <class T>
struct AngleGeom {
  T theta, c, n1, n2, s;
  T u[3], w[3];
};

template <class T>
__device__ __forceinline__ AngleGeom<T> angle_geom(const T *x, int64_t i, int64_t j, int64_t k) {
  AngleGeom<T> g;
  T v1[3], v2[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    v1[a] = x[3 * i + a] - x[3 * j + a];
    v2[a] = x[3 * k + a] - x[3 * j + a];
  }
  g.n1 = sqrt(v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2]);
  g.n2 = sqrt(v2[0] * v2[0] + v2[1] * v2[1] + v2[2] * v2[2]);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    g.u[a] = v1[a] / g.n1;
    g.w[a] = v2[a] / g.n2;
  }
  T c = g.u[0] * g.w[0] + g.u[1] * g.w[1] + g.u[2] * g.w[2];
  c = c > T(1) ? T(1) : (c < T(-1) ? T(-1) : c);
  g.c = c;
  g.theta = acos(c);
  g.s = sqrt(fmax(T(1) - c * c, T(1e-30)));
  return g;
}

// Adds f * dtheta/dx of one angle into gx.
template <class T>
__device__ __forceinline__ void angle_grad_add(typename Acc<T>::S *gx, int64_t i, int64_t j, int64_t k,
                                               const AngleGeom<T> &g, T f) {
  const T a1 = -f / (g.n1 * g.s), a3 = -f / (g.n2 * g.s);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const T g1 = a1 * (g.w[a] - g.c * g.u[a]);
    const T g3 = a3 * (g.u[a] - g.c * g.w[a]);
    Acc<T>::add(&gx[3 * i + a], (double)g1);
    Acc<T>::add(&gx[3 * k + a], (double)g3);
    Acc<T>::add(&gx[3 * j + a], -(double)(g1 + g3));
  }
}

// E = 1/2 k (theta - theta0)^2; outputs as harmonic_bond_kernel (dE/dtheta0, dE/dk).
template <class T>
__global__ void __launch_bounds__(kBondBlock) harmonic_angle_kernel(const T *x, const int64_t *ang, int64_t na,
                                                                    const T *th0, const T *k, typename Acc<T>::S *gx,
                                                                    T *gth0, T *gk, double *partials, unsigned *ticket,
                                                                    double *energy) {
  pdl_enter();
  double e = 0.0;
  for (int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m < na; m += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = ang[3 * m], j = ang[3 * m + 1], kk = ang[3 * m + 2];
    const AngleGeom<T> g = angle_geom(x, i, j, kk);
    const T kt = k[m], dth = g.theta - th0[m];
    e += (double)(T(0.5) * kt * dth * dth);
    if (gx) angle_grad_add(gx, i, j, kk, g, kt * dth);
    if (gth0) gth0[m] = -kt * dth;
    if (gk) gk[m] = T(0.5) * dth * dth;
  }
  if (energy) grid_sum<kBondBlock>(e, partials, ticket, energy, false);
}

// theta of every angle; with `gtheta` instead the backward pass: gx += sum gtheta * dtheta/dx.
template <class T>
__global__ void __launch_bounds__(kBondBlock) angles_kernel(const T *x, const int64_t *ang, int64_t na, T *theta,
                                                            const T *gtheta, typename Acc<T>::S *gx) {
  for (int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m < na; m += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = ang[3 * m], j = ang[3 * m + 1], k = ang[3 * m + 2];
    const AngleGeom<T> g = angle_geom(x, i, j, k);
    if (theta) theta[m] = g.theta;
    if (gtheta) angle_grad_add(gx, i, j, k, g, gtheta[m]);
  }
}

// Bonds and angles of a fused system in one launch: threads [0, nb) take bonds, [nb, nb +
// na) angles; dE/dx into acc (caller order, 3N), the two energies into acc[3N] (bonds) and
// acc[3N + 1] (angles). acc is zeroed by the caller.
template <class T>
__global__ void __launch_bounds__(kBondBlock) system_bonded_kernel(const T *x, int64_t natoms, const int64_t *bonds,
                                                                   int64_t nb, const T *b0, const T *kb,
                                                                   const int64_t *ang, int64_t na, const T *th0,
                                                                   const T *kth, typename Acc<T>::S *acc) {
  double eb = 0.0, ea = 0.0;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nb + na; t += (int64_t)gridDim.x * blockDim.x) {
    if (t < nb) {
      const int64_t i = bonds[2 * t], j = bonds[2 * t + 1];
      const T dx = x[3 * j] - x[3 * i], dy = x[3 * j + 1] - x[3 * i + 1], dz = x[3 * j + 2] - x[3 * i + 2];
      const T r = sqrt(dx * dx + dy * dy + dz * dz);
      const T dr = r - b0[t];
      eb += (double)(T(0.5) * kb[t] * dr * dr);
      const T sc = kb[t] * dr / r;
      Acc<T>::add(&acc[3 * j], (double)(sc * dx));
      Acc<T>::add(&acc[3 * j + 1], (double)(sc * dy));
      Acc<T>::add(&acc[3 * j + 2], (double)(sc * dz));
      Acc<T>::add(&acc[3 * i], -(double)(sc * dx));
      Acc<T>::add(&acc[3 * i + 1], -(double)(sc * dy));
      Acc<T>::add(&acc[3 * i + 2], -(double)(sc * dz));
    } else {
      const int64_t m = t - nb;
      const int64_t i = ang[3 * m], j = ang[3 * m + 1], k = ang[3 * m + 2];
      const AngleGeom<T> g = angle_geom(x, i, j, k);
      const T dth = g.theta - th0[m];
      ea += (double)(T(0.5) * kth[m] * dth * dth);
      angle_grad_add(acc, i, j, k, g, kth[m] * dth);
    }
  }
  eb = warp_sum(eb);
  ea = warp_sum(ea);
  if ((threadIdx.x & 31) == 0) {
    Acc<T>::add(&acc[3 * natoms], eb);
    Acc<T>::add(&acc[3 * natoms + 1], ea);
  }
}

}  // namespace
}  // namespace tff

// Rank-0 smooth PME (order-6 B-splines) on a cubic K^3 grid.
//
//   spread   : Q(g) = sum_i q_i M6(u_i,x) M6(u_i,y) M6(u_i,z)   (fixed-point or FP64 atomics)
//   [to_real]: fixed-point grid -> FP32 (mixed precision)
//   R2C FFT  : S(k)                                             (cuFFT)
//   convolve : S(k) *= C(k)/theta(k)^2, E_rec = 1/2 sum_k C |S|^2/theta^2 (FP64, fixed order)
//   C2R FFT  : Phi(g)                                           (cuFFT, unnormalised)
//   gather   : phi_i = sum_g theta_i(g) Phi(g), dE/dx_i = q_i grad phi_i,
//              dE/dq_i = phi_i - 2 a q_i / sqrt(pi), E_self = -(a/sqrt(pi)) sum q^2
//
// Conventions follow the reference (torchff/pme_ref.py:11-469, csrc/pme/kernels.cuh):
// u = K * (box^-T r) per lattice direction, m0 = ceil(u), the 6 stencil points are
// m0-3 .. m0+2 with weights M6((m0 - u) + k), grid index gx*K^2 + gy*K + gz, and
// the signed frequency of FFT index i is i for 2i < K, else i - K.
#pragma once

#include <cufft.h>

#include <type_traits>

#include "cluster.cuh"

namespace tff {

constexpr int kPmeBlock = 256;

// Per-atom stencil: origin index (already wrapped into [0,K)) and the 3x6 weights.
template <class T>
struct Stencil {
  int g0[3];
  T val[3][6];
  T der[3][6];
};

// recip[d*3 + c] = K * inv[c][d]: u_d = sum_c recip[d][c] r_c
template <class T>
__device__ __forceinline__ void make_stencil(double rx, double ry, double rz, const double *recip, int K,
                                             Stencil<T> &s) {
  const double r[3] = {rx, ry, rz};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double u = recip[3 * d] * r[0] + recip[3 * d + 1] * r[1] + recip[3 * d + 2] * r[2];
    const double m0 = ceil(u);
    const T w = (T)(m0 - u);
    bspline6<T>(w, s.val[d], s.der[d]);
    // first stencil point modulo K: one compare for atoms within a box length of the
    // primary cell (the common case), a 64-bit remainder otherwise
    long long g = (long long)m0 - 3;
    if (g >= -K && g < 2 * (long long)K) {
      g += g < 0 ? K : 0;
      g -= g >= K ? K : 0;
    } else {
      g %= K;
      if (g < 0) g += K;
    }
    s.g0[d] = (int)g;
  }
}

struct PmeShared {
  double recip[9];
  double inv[9];
  double vol;
};

template <class T>
__device__ __forceinline__ void load_pme_shared(const T *box, int K, PmeShared &sh) {
  Box b;
  load_box(box, b);
  for (int d = 0; d < 3; ++d)
    for (int c = 0; c < 3; ++c) sh.recip[3 * d + c] = (double)K * b.inv[3 * c + d];
  for (int k = 0; k < 9; ++k) sh.inv[k] = b.inv[k];
  sh.vol = b.vol;
}

// Atom sources: plain (caller arrays) or cluster-sorted (wrapped positions, charge in .w).
template <class T>
struct PlainAtoms {
  const T *x;
  const T *q;
  int64_t n;
  __device__ __forceinline__ bool get(int64_t t, double &rx, double &ry, double &rz, T &qi) const {
    if (t >= n) return false;
    rx = x[3 * t]; ry = x[3 * t + 1]; rz = x[3 * t + 2];
    qi = q[t];
    return true;
  }
};

template <class T>
struct SortedAtoms {
  const typename V4<T>::type *pos;
  const int *sidx;
  int64_t npad;
  __device__ __forceinline__ bool get(int64_t t, double &rx, double &ry, double &rz, T &qi) const {
    if (t >= npad || sidx[t] < 0) return false;
    const auto p = pos[t];
    rx = p.x; ry = p.y; rz = p.z;
    qi = p.w;
    return true;
  }
};

// Atoms in the cluster (Hilbert) order of a cluster build: slot t is caller atom sidx[t]
// (-1: padding). Coordinates and charges come from the caller arrays, so every atom's
// numbers are those of PlainAtoms; only the visiting order changes, and neighbouring
// threads then touch neighbouring grid points.
template <class T>
struct IndexedAtoms {
  const T *x;
  const T *q;
  const int *sidx;
  int64_t n;  // slots
  __device__ __forceinline__ bool get(int64_t t, double &rx, double &ry, double &rz, T &qi) const {
    if (t >= n) return false;
    const int64_t a = sidx[t];
    if (a < 0) return false;
    rx = x[3 * a]; ry = x[3 * a + 1]; rz = x[3 * a + 2];
    qi = q[a];
    return true;
  }
};

// Spread: a group of kLanesPerAtom lanes per atom; lane g of the group takes the stencil
// rows r = g, g + kLanesPerAtom, ... of the 36 (x, y) rows, 6 z points each. Loops run at
// warp granularity so that every lane of a warp takes the same trip count. `bid` and
// `nblk` are the block index and count over which the atoms are distributed.
constexpr int kLanesPerAtom = 8;
constexpr int kAtomsPerWarp = kWarp / kLanesPerAtom;

template <class T, class Atoms>
__device__ __forceinline__ void spread_atoms(const Atoms &atoms, int64_t nthreads, const PmeShared &sh, int K,
                                             typename Acc<T>::S *grid, int64_t bid, int64_t nblk) {
  const int g = threadIdx.x % kLanesPerAtom;
  const int64_t wglob = (bid * blockDim.x + threadIdx.x) / kWarp;
  const int64_t nwarps = nblk * blockDim.x / kWarp;
  for (int64_t wb = wglob * kAtomsPerWarp; wb < nthreads; wb += nwarps * kAtomsPerWarp) {
    const int64_t t = wb + (threadIdx.x % kWarp) / kLanesPerAtom;
    double rx, ry, rz;
    T q;
    if (t >= nthreads || !atoms.get(t, rx, ry, rz, q)) continue;
    Stencil<T> s;
    make_stencil<T>(rx, ry, rz, sh.recip, K, s);
    for (int r = g; r < 36; r += kLanesPerAtom) {
      const int a = r / 6, b = r % 6;
      int gx = s.g0[0] + a, gy = s.g0[1] + b;
      gx -= (gx >= K) ? K : 0;
      gy -= (gy >= K) ? K : 0;
      const T wxy = q * s.val[0][a] * s.val[1][b];
      const int64_t row = ((int64_t)gx * K + gy) * K;
      int gz = s.g0[2];
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        Acc<T>::add(&grid[row + gz], (double)(wxy * s.val[2][c]));
        gz = (gz + 1 == K) ? 0 : gz + 1;
      }
    }
  }
}

// Spread in groups of kSpreadGroup consecutive atoms (FP32 inputs, fixed-point grid). The
// atoms of a molecule are usually consecutive (a water's O, H, H), so their 6x6x6 stencils
// overlap: a warp sums a group's contributions over the union window of its stencils (at
// most kSpreadWin points per axis) and adds each window point to the grid with one atomic,
// where the per-atom spread adds every contribution (3 x 216 for a water, against 7^3 = 343
// window points for a typical one). Every contribution is rounded to fixed point by itself
// and the integers are summed, exactly as the per-atom spread's atomics sum them, so the
// grid is bit-identical to it. A group whose atoms lie too far apart on the grid (or whose
// stencils are taken on a grid of fewer than kSpreadWin points) is spread atom by atom.
constexpr int kSpreadGroup = 3;
constexpr int kGroupsPerPass = 10;  // most groups staged per warp and pass: 30 atoms, one per lane
constexpr int kSpreadWin = 8;

struct GroupStencil {
  int org[3];    // first stencil point per axis, ceil(u) - 3 wrapped into [0, K)
  float w[3][6]; // B-spline weights
  float q;
  int valid;
};

// Grouped spread of atoms [0, n) by the blocks bid of nblk (warp-strided over groups); S is
// the warp's stencil staging (kSpreadGroup * kGroupsPerPass entries in shared memory). Each
// warp stages as many groups per pass as it takes for the groups to fill the warps.
template <class Atoms>
__device__ __forceinline__ void spread_groups(const Atoms &atoms, int64_t n, const PmeShared &sh, int K,
                                              unsigned long long *grid, int64_t bid, int64_t nblk, GroupStencil *S) {
  const int lane = threadIdx.x & 31;
  const int64_t wg = (bid * blockDim.x + threadIdx.x) / kWarp;
  const int64_t nw = nblk * blockDim.x / kWarp;
  const int64_t groups = (n + kSpreadGroup - 1) / kSpreadGroup;
  const int gpp = (int)min((int64_t)kGroupsPerPass, max((int64_t)1, (groups + nw - 1) / nw));
  const int kAtoms = kSpreadGroup * gpp;
  for (int64_t base = wg * kAtoms; base < n; base += nw * kAtoms) {
    __syncwarp();  // every lane is done with the previous pass's stencils
    if (lane < kAtoms) {
      GroupStencil &g = S[lane];
      double rx, ry, rz;
      float qa;
      const int64_t a = base + lane;
      g.valid = a < n && atoms.get(a, rx, ry, rz, qa);
      if (g.valid) {
        const double r[3] = {rx, ry, rz};
        float der[6];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const double u = sh.recip[3 * d] * r[0] + sh.recip[3 * d + 1] * r[1] + sh.recip[3 * d + 2] * r[2];
          const double m0 = ceil(u);
          bspline6<float>((float)(m0 - u), g.w[d], der);
          // first stencil point wrapped into [0, K) (the window code below relies on it):
          // compares within a box length of the primary cell, a 64-bit remainder beyond
          long long o = (long long)m0 - 3;
          if (o >= -K && o < 2 * (long long)K) {
            o += o < 0 ? K : 0;
            o -= o >= K ? K : 0;
          } else {
            o %= K;
            if (o < 0) o += K;
          }
          g.org[d] = (int)o;
        }
        g.q = qa;
      }
    }
    __syncwarp();
#pragma unroll 1
    for (int gi = 0; gi < gpp; ++gi) {
      const GroupStencil *G = S + kSpreadGroup * gi;
      // offsets of the atoms' stencils from the first valid atom's, taken modulo K into
      // (-K/2, K/2], and the window's extent per axis
      int first = -1;
#pragma unroll
      for (int k = kSpreadGroup - 1; k >= 0; --k)
        if (G[k].valid) first = k;
      if (first < 0) continue;
      int rel[kSpreadGroup][3], lo[3], ext[3];
      bool fits = K >= kSpreadWin;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        int mn = 0, mx = 0;
#pragma unroll
        for (int k = 0; k < kSpreadGroup; ++k) {
          int v = G[k].org[d] - G[first].org[d];  // origins lie in [0, K) (wrapped above): |v| < K
          if (v > K / 2) v -= K;
          if (v <= -((K + 1) / 2)) v += K;
          rel[k][d] = v;
          if (G[k].valid) {
            mn = min(mn, v);
            mx = max(mx, v);
          }
        }
        lo[d] = mn;
        ext[d] = mx - mn + 6;
        fits = fits && ext[d] <= kSpreadWin;
      }
      if (fits) {
        // window point (x, y, z) in window coordinates; atom k covers it when
        // 0 <= x - (rel_k - lo) < 6 on every axis
        const int rows = ext[0] * ext[1];
        for (int r = lane; r < rows; r += kWarp) {
          const int ax = r / ext[1], ay = r % ext[1];
          float wxy[kSpreadGroup];
          int oz[kSpreadGroup];
#pragma unroll
          for (int k = 0; k < kSpreadGroup; ++k) {
            const int ix = ax - (rel[k][0] - lo[0]), iy = ay - (rel[k][1] - lo[1]);
            const bool in = G[k].valid && ix >= 0 && ix < 6 && iy >= 0 && iy < 6;
            wxy[k] = in ? G[k].q * G[k].w[0][ix] * G[k].w[1][iy] : 0.f;
            oz[k] = in ? rel[k][2] - lo[2] : 1 << 20;  // outside every z
          }
          // origin in [0, K), lo in (-K/2, 0], ax, ay < 8 <= K: one wrap either way
          int gx = G[first].org[0] + lo[0] + ax, gy = G[first].org[1] + lo[1] + ay;
          gx += gx < 0 ? K : 0;
          gx -= gx >= K ? K : 0;
          gy += gy < 0 ? K : 0;
          gy -= gy >= K ? K : 0;
          const int64_t row = ((int64_t)gx * K + gy) * K;
          int gz = G[first].org[2] + lo[2];
          gz += gz < 0 ? K : 0;
          for (int z = 0; z < ext[2]; ++z) {
            unsigned long long acc = 0ull;
            bool any = false;
#pragma unroll
            for (int k = 0; k < kSpreadGroup; ++k) {
              const int iz = z - oz[k];
              if (iz >= 0 && iz < 6) {
                acc += to_fix_f(wxy[k] * G[k].w[2][iz]);
                any = true;
              }
            }
            if (any) atomicAdd(&grid[row + gz], acc);
            gz = (gz + 1 == K) ? 0 : gz + 1;
          }
        }
      } else {
        // atom by atom: lanes over the 36 (x, y) rows, 6 z points each
#pragma unroll 1
        for (int k = 0; k < kSpreadGroup; ++k) {
          const GroupStencil &g = G[k];
          if (!g.valid) continue;
          for (int r = lane; r < 36; r += kWarp) {
            const int a = r / 6, b = r % 6;
            int gx = (g.org[0] + a) % K, gy = (g.org[1] + b) % K, gz = g.org[2] % K;
            gx += gx < 0 ? K : 0;
            gy += gy < 0 ? K : 0;
            gz += gz < 0 ? K : 0;
            const float wxy = g.q * g.w[0][a] * g.w[1][b];
            const int64_t row = ((int64_t)gx * K + gy) * K;
#pragma unroll
            for (int c = 0; c < 6; ++c) {
              atomicAdd(&grid[row + gz], to_fix_f(wxy * g.w[2][c]));
              gz = (gz + 1 == K) ? 0 : gz + 1;
            }
          }
        }
      }
    }
  }
}

template <class Atoms>
__global__ void __launch_bounds__(kPmeBlock) pme_spread_grouped_kernel(Atoms atoms, int64_t n, const float *box, int K,
                                                                       unsigned long long *grid) {
  __shared__ PmeShared sh;
  __shared__ GroupStencil st[kPmeBlock / kWarp][kSpreadGroup * kGroupsPerPass];
  if (threadIdx.x == 0) load_pme_shared(box, K, sh);
  __syncthreads();
  spread_groups(atoms, n, sh, K, grid, blockIdx.x, gridDim.x, st[threadIdx.x >> 5]);
}

template <class T, class Atoms>
__global__ void __launch_bounds__(kPmeBlock) pme_spread_kernel(Atoms atoms, int64_t nthreads, const T *box, int K,
                                                               typename Acc<T>::S *grid) {
  __shared__ PmeShared sh;
  if (threadIdx.x == 0) load_pme_shared(box, K, sh);
  __syncthreads();
  spread_atoms<T>(atoms, nthreads, sh, K, grid, blockIdx.x, gridDim.x);
}

static __global__ void pme_fix_to_real_kernel(const unsigned long long *gi, float *gf, int64_t n) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    gf[k] = (float)from_fix(gi[k]);
}

template <class T> struct CplxOf;
template <> struct CplxOf<float> { using type = cufftComplex; };
template <> struct CplxOf<double> { using type = cufftDoubleComplex; };

// Convolution of the points bid, bid + nblk, ... (in blocks of blockDim.x); returns this
// thread's share of sum_k w C(k) |S(k)|^2 / theta(k)^2 (the energy is half of the total).
template <class T>
__device__ __forceinline__ double convolve_points(typename CplxOf<T>::type *S, const PmeShared &sh, int K,
                                                  double alpha, const T *xmod, const T *ymod, const T *zmod,
                                                  int64_t bid, int64_t nblk) {
  const int Kz = K / 2 + 1;
  const int64_t total = (int64_t)K * K * Kz;
  const double four_pi_over_v = 4.0 * 3.14159265358979323846 / sh.vol;
  const double two_pi = 2.0 * 3.14159265358979323846;
  const double inv4a2 = 1.0 / (4.0 * alpha * alpha);
  double e = 0.0;
  // 32-bit index arithmetic (a 64-bit division costs several times a 32-bit one) while the
  // grid has fewer than 2^32 points, i.e. for every K below 2048
  const bool narrow = total < (int64_t(1) << 32);
  for (int64_t t = bid * blockDim.x + threadIdx.x; t < total; t += nblk * blockDim.x) {
    int ix, iy, iz;
    if (narrow) {
      const unsigned tt = (unsigned)t, row = tt / (unsigned)Kz, x = row / (unsigned)K;
      iz = (int)(tt - row * (unsigned)Kz);
      iy = (int)(row - x * (unsigned)K);
      ix = (int)x;
    } else {
      iz = (int)(t % Kz);
      iy = (int)((t / Kz) % K);
      ix = (int)(t / ((int64_t)Kz * K));
    }
    const double mx = (2 * ix < K) ? ix : ix - K;
    const double my = (2 * iy < K) ? iy : iy - K;
    const double mz = (2 * iz < K) ? iz : iz - K;
    double factor = 0.0;
    if (t != 0) {
      // k_c = 2 pi sum_d m_d inv[c][d]
      const double kx = two_pi * (mx * sh.inv[0] + my * sh.inv[1] + mz * sh.inv[2]);
      const double ky = two_pi * (mx * sh.inv[3] + my * sh.inv[4] + mz * sh.inv[5]);
      const double kz = two_pi * (mx * sh.inv[6] + my * sh.inv[7] + mz * sh.inv[8]);
      const double ksq = kx * kx + ky * ky + kz * kz;
      const double th = (double)xmod[ix] * (double)ymod[iy] * (double)zmod[iz];
      factor = four_pi_over_v * exp(-ksq * inv4a2) / (ksq * th * th);
    }
    auto v = S[t];
    const double re = v.x, im = v.y;
    const double w = (iz == 0 || 2 * iz == K) ? 1.0 : 2.0;
    e += w * factor * (re * re + im * im);
    v.x = (T)(re * factor);
    v.y = (T)(im * factor);
    S[t] = v;
  }
  return e;
}

template <class T>
__global__ void __launch_bounds__(kPmeBlock) pme_convolve_kernel(typename CplxOf<T>::type *S, const T *box, int K,
                                                                 double alpha, const T *xmod, const T *ymod,
                                                                 const T *zmod, double *partials, unsigned *ticket,
                                                                 double *e_rec) {
  __shared__ PmeShared sh;
  if (threadIdx.x == 0) load_pme_shared(box, K, sh);
  __syncthreads();
  const double e = convolve_points<T>(S, sh, K, alpha, xmod, ymod, zmod, blockIdx.x, gridDim.x);
  grid_sum<kPmeBlock>(0.5 * e, partials, ticket, e_rec, false);
}

// Gather output: caller arrays (caller order), plain stores (one thread per atom).
template <class T>
struct PlainGatherOut {
  T *phi;    // dE/dq (N), nullable
  T *grad;   // dE/dx (N,3), nullable
  __device__ __forceinline__ void put(int64_t t, double phi_t, double gx, double gy, double gz) const {
    if (phi) phi[t] = (T)phi_t;
    if (grad) {
      grad[3 * t] = (T)gx;
      grad[3 * t + 1] = (T)gy;
      grad[3 * t + 2] = (T)gz;
    }
  }
};

// Gather output for IndexedAtoms: slot t's values go to caller atom sidx[t].
template <class T>
struct IndexedGatherOut {
  T *phi;   // dE/dq (N), nullable
  T *grad;  // dE/dx (N,3), nullable
  const int *sidx;
  __device__ __forceinline__ void put(int64_t t, double phi_t, double gx, double gy, double gz) const {
    const int64_t a = sidx[t];
    if (phi) phi[a] = (T)phi_t;
    if (grad) {
      grad[3 * a] = (T)gx;
      grad[3 * a + 1] = (T)gy;
      grad[3 * a + 2] = (T)gz;
    }
  }
};

// Gather: partial sums of the 216 products (FP64 across the stencil rows) reduced with
// shuffles inside each atom's lane group. Returns this thread's share of the self energy
// -(a/sqrt(pi)) sum q^2. An atom takes 6 lanes, lane a the x index a of the stencil, so
// that every other stencil index is a compile-time constant (registers, not local memory);
// a warp holds 5 atoms (lanes 30, 31 idle). With 8 lanes per atom and the (x, y) row taken
// from the lane index, the stencil weights went through local memory.
constexpr int kGatherLanes = 6;
constexpr int kGatherAtomsPerWarp = kWarp / kGatherLanes;

template <class T>
__device__ __forceinline__ T pick6(const T (&v)[6], int i) {
  T r = v[0];
#pragma unroll
  for (int k = 1; k < 6; ++k) r = i == k ? v[k] : r;
  return r;
}

// Sum over the 6 lanes 6k .. 6k + 5 of an atom, valid on lane 6k (fixed order).
__device__ __forceinline__ double gather_lane_sum(double v) {
  v += __shfl_down_sync(kFull, v, 3);
  const double b1 = __shfl_down_sync(kFull, v, 1), b2 = __shfl_down_sync(kFull, v, 2);
  return (v + b1) + b2;
}

template <class T, class Atoms, class Out>
__device__ __forceinline__ double gather_atoms(const Atoms &atoms, int64_t nthreads, const PmeShared &sh, int K,
                                               const T *Phi, double alpha, const Out &out, int64_t bid,
                                               int64_t nblk) {
  const double a_rpi = alpha / 1.7724538509055160273;
  const int lw = threadIdx.x % kWarp;
  const int slot = lw / kGatherLanes;     // atom of the warp (kGatherAtomsPerWarp: idle lane)
  const int a = lw - slot * kGatherLanes;  // x index of the stencil
  const int64_t wglob = (bid * blockDim.x + threadIdx.x) / kWarp;
  const int64_t nwarps = nblk * blockDim.x / kWarp;
  double e = 0.0;
  for (int64_t wb = wglob * kGatherAtomsPerWarp; wb < nthreads; wb += nwarps * kGatherAtomsPerWarp) {
    const int64_t t = wb + slot;
    double rx = 0.0, ry = 0.0, rz = 0.0;
    T q = T(0);
    const bool ok = slot < kGatherAtomsPerWarp && t < nthreads && atoms.get(t, rx, ry, rz, q);
    double phi = 0.0, du0 = 0.0, du1 = 0.0, du2 = 0.0;
    if (ok) {
      Stencil<T> s;
      make_stencil<T>(rx, ry, rz, sh.recip, K, s);
      int gx = s.g0[0] + a;
      gx -= (gx >= K) ? K : 0;
      // sums over the (y, z) plane at x index a: sum vy pz, sum dy pz, sum vy dz
      double svp = 0.0, sdp = 0.0, svd = 0.0;
#pragma unroll
      for (int b = 0; b < 6; ++b) {
        int gy = s.g0[1] + b;
        gy -= (gy >= K) ? K : 0;
        const int64_t row = ((int64_t)gx * K + gy) * K;
        int gz = s.g0[2];
        T pz = T(0), dz = T(0);
#pragma unroll
        for (int c = 0; c < 6; ++c) {
          const T v = Phi[row + gz];
          pz += v * s.val[2][c];
          dz += v * s.der[2][c];
          gz = (gz + 1 == K) ? 0 : gz + 1;
        }
        svp += (double)s.val[1][b] * (double)pz;
        sdp += (double)s.der[1][b] * (double)pz;
        svd += (double)s.val[1][b] * (double)dz;
      }
      const double vx = (double)pick6(s.val[0], a), dx = (double)pick6(s.der[0], a);
      phi = vx * svp;
      du0 = dx * svp;
      du1 = vx * sdp;
      du2 = vx * svd;
    }
    phi = gather_lane_sum(phi);
    du0 = gather_lane_sum(du0);
    du1 = gather_lane_sum(du1);
    du2 = gather_lane_sum(du2);
    if (ok && a == 0) {
      // u_d = m0 - frac_d + const, so d(stencil u)/dr_c = -recip[d][c]
      const double qd = (double)q;
      const double gxv = -qd * (du0 * sh.recip[0] + du1 * sh.recip[3] + du2 * sh.recip[6]);
      const double gyv = -qd * (du0 * sh.recip[1] + du1 * sh.recip[4] + du2 * sh.recip[7]);
      const double gzv = -qd * (du0 * sh.recip[2] + du1 * sh.recip[5] + du2 * sh.recip[8]);
      out.put(t, phi - 2.0 * a_rpi * qd, gxv, gyv, gzv);
      e -= a_rpi * qd * qd;
    }
  }
  return e;
}

template <class T, class Atoms, class Out>
__global__ void __launch_bounds__(kPmeBlock) pme_gather_kernel(Atoms atoms, int64_t nthreads, const T *box, int K,
                                                               const T *Phi, double alpha, Out out, double *partials,
                                                               unsigned *ticket, double *e_self, const double *e_rec,
                                                               double e_scale, T *energy_out) {
  __shared__ PmeShared sh;
  if (threadIdx.x == 0) load_pme_shared(box, K, sh);
  __syncthreads();
  const double e = gather_atoms<T>(atoms, nthreads, sh, K, Phi, alpha, out, blockIdx.x, gridDim.x);
  const bool last = grid_sum<kPmeBlock>(e, partials, ticket, e_self, false);
  if (last && threadIdx.x == 0 && energy_out) energy_out[0] = (T)(e_scale * (*e_rec + *e_self));
}

// ---- second derivatives along a coordinate direction u (force matching)
// With theta_i(g) the stencil weight and w_d = m0_d - u_d its spline argument
// (dw_d/dr_c = -recip[d][c]), v_i = recip u_i, G_d = d theta / d w_d, H_de = d2 theta / dw_d dw_e:
//   P(g)   = sum_i q_i u_i . grad theta_i(g) = -sum_i q_i sum_d v_d G_d(g)
//   psi    = the same influence-function convolution of P as Phi of Q
//   d/dx_i (sum_j u_j . dE/dx_j) = q_i recip^T (A v_i - B),  A_de = sum_g Phi H_de, B_d = sum_g psi G_d
//   d/dq_i (sum_j u_j . dE/dx_j) = -v_i . C + sum_g psi theta_i,  C_d = sum_g Phi G_d
// (the reciprocal energy is 1/2 Q.Phi; the self term has no coordinate dependence).
template <class T>
__global__ void __launch_bounds__(kPmeBlock) pme_spread_dir_kernel(PlainAtoms<T> atoms, const T *dir, int64_t n,
                                                                   const T *box, int K, typename Acc<T>::S *grid) {
  __shared__ PmeShared sh;
  if (threadIdx.x == 0) load_pme_shared(box, K, sh);
  __syncthreads();
  const int g = threadIdx.x % kLanesPerAtom;
  const int64_t wglob = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp;
  const int64_t nwarps = (int64_t)gridDim.x * blockDim.x / kWarp;
  for (int64_t wb = wglob * kAtomsPerWarp; wb < n; wb += nwarps * kAtomsPerWarp) {
    const int64_t t = wb + (threadIdx.x % kWarp) / kLanesPerAtom;
    double rx, ry, rz;
    T q;
    if (t >= n || !atoms.get(t, rx, ry, rz, q)) continue;
    const double ux = dir[3 * t], uy = dir[3 * t + 1], uz = dir[3 * t + 2];
    const double v0 = sh.recip[0] * ux + sh.recip[1] * uy + sh.recip[2] * uz;
    const double v1 = sh.recip[3] * ux + sh.recip[4] * uy + sh.recip[5] * uz;
    const double v2 = sh.recip[6] * ux + sh.recip[7] * uy + sh.recip[8] * uz;
    Stencil<T> s;
    make_stencil<T>(rx, ry, rz, sh.recip, K, s);
    for (int r = g; r < 36; r += kLanesPerAtom) {
      const int a = r / 6, b = r % 6;
      int gx = s.g0[0] + a, gy = s.g0[1] + b;
      gx -= (gx >= K) ? K : 0;
      gy -= (gy >= K) ? K : 0;
      const double wx = s.val[0][a], dx = s.der[0][a], wy = s.val[1][b], dy = s.der[1][b];
      const double c_val = -(double)q * (v0 * dx * wy + v1 * wx * dy);  // times val_z
      const double c_der = -(double)q * v2 * wx * wy;                    // times der_z
      const int64_t row = ((int64_t)gx * K + gy) * K;
      int gz = s.g0[2];
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        Acc<T>::add(&grid[row + gz], c_val * (double)s.val[2][c] + c_der * (double)s.der[2][c]);
        gz = (gz + 1 == K) ? 0 : gz + 1;
      }
    }
  }
}

// Per atom: kc * d/dx_i and kc * d/dq_i of sum_j u_j . dE_rec/dx_j (kLanesPerAtom lanes per atom).
template <class T>
__global__ void __launch_bounds__(kPmeBlock) pme_gather_hvp_kernel(PlainAtoms<T> atoms, const T *dir, int64_t n,
                                                                   const T *box, int K, const T *Phi, const T *Psi,
                                                                   double kc, T *hx, T *hq) {
  __shared__ PmeShared sh;
  if (threadIdx.x == 0) load_pme_shared(box, K, sh);
  __syncthreads();
  const int g = threadIdx.x % kLanesPerAtom;
  const int64_t wglob = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp;
  const int64_t nwarps = (int64_t)gridDim.x * blockDim.x / kWarp;
  for (int64_t wb = wglob * kAtomsPerWarp; wb < n; wb += nwarps * kAtomsPerWarp) {
    const int64_t t = wb + (threadIdx.x % kWarp) / kLanesPerAtom;
    double rx = 0.0, ry = 0.0, rz = 0.0;
    T q = T(0);
    const bool ok = t < n && atoms.get(t, rx, ry, rz, q);
    // A00 A11 A22 A01 A02 A12, B0..2, C0..2, Psi_i
    double acc[13];
#pragma unroll
    for (int k = 0; k < 13; ++k) acc[k] = 0.0;
    T val[3][6], der[3][6], dd[3][6];
    int g0[3];
    if (ok) {
      const double r[3] = {rx, ry, rz};
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const double u = sh.recip[3 * d] * r[0] + sh.recip[3 * d + 1] * r[1] + sh.recip[3 * d + 2] * r[2];
        const double m0 = ceil(u);
        bspline6_d2<T>((T)(m0 - u), val[d], der[d], dd[d]);
        long long gg = (long long)m0 - 3;
        gg %= K;
        if (gg < 0) gg += K;
        g0[d] = (int)gg;
      }
      for (int rr = g; rr < 36; rr += kLanesPerAtom) {
        const int a = rr / 6, b = rr % 6;
        int gx = g0[0] + a, gy = g0[1] + b;
        gx -= (gx >= K) ? K : 0;
        gy -= (gy >= K) ? K : 0;
        const int64_t row = ((int64_t)gx * K + gy) * K;
        int gz = g0[2];
        double pv = 0.0, pd = 0.0, pdd = 0.0, sv = 0.0, sd = 0.0;
#pragma unroll
        for (int c = 0; c < 6; ++c) {
          const double ph = Phi[row + gz], ps = Psi[row + gz];
          pv += ph * (double)val[2][c];
          pd += ph * (double)der[2][c];
          pdd += ph * (double)dd[2][c];
          sv += ps * (double)val[2][c];
          sd += ps * (double)der[2][c];
          gz = (gz + 1 == K) ? 0 : gz + 1;
        }
        const double vx = val[0][a], dx = der[0][a], ddx = dd[0][a];
        const double vy = val[1][b], dy = der[1][b], ddy = dd[1][b];
        acc[0] += ddx * vy * pv;
        acc[1] += vx * ddy * pv;
        acc[2] += vx * vy * pdd;
        acc[3] += dx * dy * pv;
        acc[4] += dx * vy * pd;
        acc[5] += vx * dy * pd;
        acc[6] += dx * vy * sv;
        acc[7] += vx * dy * sv;
        acc[8] += vx * vy * sd;
        acc[9] += dx * vy * pv;
        acc[10] += vx * dy * pv;
        acc[11] += vx * vy * pd;
        acc[12] += vx * vy * sv;
      }
    }
#pragma unroll
    for (int k = 0; k < 13; ++k)
#pragma unroll
      for (int o = kLanesPerAtom / 2; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(kFull, acc[k], o);
    if (ok && g == 0) {
      const double ux = dir[3 * t], uy = dir[3 * t + 1], uz = dir[3 * t + 2];
      double v[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) v[d] = sh.recip[3 * d] * ux + sh.recip[3 * d + 1] * uy + sh.recip[3 * d + 2] * uz;
      const double A[3][3] = {{acc[0], acc[3], acc[4]}, {acc[3], acc[1], acc[5]}, {acc[4], acc[5], acc[2]}};
      double w[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) w[d] = A[d][0] * v[0] + A[d][1] * v[1] + A[d][2] * v[2] - acc[6 + d];
      const double qd = (double)q;
#pragma unroll
      for (int c = 0; c < 3; ++c)
        hx[3 * t + c] = (T)(kc * qd * (sh.recip[c] * w[0] + sh.recip[3 + c] * w[1] + sh.recip[6 + c] * w[2]));
      hq[t] = (T)(kc * (-(v[0] * acc[9] + v[1] * acc[10] + v[2] * acc[11]) + acc[12]));
    }
  }
}

// ---- batched 3-D real DFT of many grids of different sizes (the serving path)
// One launch per axis pass over every system of a batch. The work units are the planes of
// every grid (system s owns units plane_off .. plane_off + K - 1); blocks loop over them.
// A block stages one plane in shared memory as `lines` x `points` with an
// odd row stride (so lanes reading one point of consecutive lines hit distinct banks),
// evaluates each output as a direct sum over the line with a twiddle table
// w[m] = exp(-+2 pi i m / K) (consecutive lanes share the twiddle: a broadcast), stages
// the outputs and writes them back contiguously. Layouts are those of cuFFT's R2C/C2R:
// real grid [x][y][z] (K^3), half spectrum [kx][ky][kz] (K x K x (K/2+1)), the inverse
// unnormalised. The summation order is fixed, so a grid's result does not depend on the
// batch it runs in.
enum BatchDftPass { kDftZR2C = 0, kDftY, kDftX, kDftXInv, kDftYInv, kDftZC2R };
constexpr int kDftThreads = 256;

__host__ __device__ inline int dft_stride(int K) { return K | 1; }

// Shared memory of one block of a pass for grid side K (twiddles + input + output planes).
template <class T>
inline size_t batch_dft_smem(int K) {
  return (size_t)(K + 2 * (size_t)K * dft_stride(K)) * 2 * sizeof(T);
}

// Next work unit of a persistent batched kernel, drawn from a per-launch counter (zeroed
// before the launch) so that blocks that finish early take more: returns the unit, equal
// to `units` or more when none is left. Called by every thread of the block; the first
// barrier also keeps the previous unit's shared memory until every thread is done with it.
__device__ __forceinline__ int next_unit(unsigned *counter) {
  __shared__ int s_unit;
  __syncthreads();
  if (threadIdx.x == 0) s_unit = (int)atomicAdd(counter, 1u);
  __syncthreads();
  return s_unit;
}

// The batch system owning work unit u: the largest s < nsys whose first unit (plane_off for
// DFT planes, conv_off for convolution units, gather_off for gather and spread units) is at
// most u. Every system owns at least one unit of each kind.
enum BatchUnits { kUnitsPlanes = 0, kUnitsConv, kUnitsGather };
template <int KIND>
__device__ __forceinline__ int unit_system(const BatchSys *sys, int nsys, int u) {
  int lo = 0, hi = nsys - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    const int off = KIND == kUnitsPlanes ? sys[mid].plane_off
                    : KIND == kUnitsConv ? sys[mid].conv_off
                                         : sys[mid].gather_off;
    if (off <= u)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// Twiddle table of every grid side 1..kmax: side K at offset K (K - 1) / 2 holds
// exp(-2 pi i m / K), m = 0..K-1, rounded from FP64. Filled once per batch object.
__host__ __device__ inline int64_t twiddle_offset(int K) { return (int64_t)K * (K - 1) / 2; }

template <class T>
__global__ void batch_twiddle_kernel(typename CplxOf<T>::type *tab, int kmax) {
  const int64_t n = twiddle_offset(kmax + 1);
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    int K = (int)((1.0 + sqrt(1.0 + 8.0 * (double)e)) / 2.0);  // twiddle_offset(K) <= e < twiddle_offset(K + 1)
    while (twiddle_offset(K) > e) --K;
    while (twiddle_offset(K + 1) <= e) ++K;
    const int m = (int)(e - twiddle_offset(K));
    double sn, cs;
    sincospi(2.0 * m / K, &sn, &cs);
    tab[e].x = (T)cs;
    tab[e].y = (T)(-sn);
  }
}

// Lines of a plane each thread transforms at once (one twiddle load serves them all).
// Measured on a 256-system serving batch (0.85 M atoms): 1 -> 2 -> 4 lines per thread
// 4.37 -> 4.27 -> 4.25 ms, 8 lines 4.38 ms.
constexpr int kDftLinesPerThread = 4;

// One plane p of one grid (see batch_dft_kernel); twtab: the batch's twiddle table.
template <class T, int PASS>
__device__ __forceinline__ void batch_dft_plane(const BatchSys &b, const int p, T *real, typename CplxOf<T>::type *cplx,
                                                const typename CplxOf<T>::type *twtab) {
  using C = typename CplxOf<T>::type;
  const int K = b.K;
  const int Kz = K / 2 + 1, st = dft_stride(K);
  constexpr bool kInverse = PASS >= kDftXInv;
  extern __shared__ __align__(16) unsigned char dft_smem[];
  C *tw = reinterpret_cast<C *>(dft_smem);
  C *in = tw + K;
  C *out = in + (size_t)K * st;
  for (int m = threadIdx.x; m < K; m += blockDim.x) {
    C v = twtab[twiddle_offset(K) + m];
    if (kInverse) v.y = -v.y;
    tw[m] = v;
  }
  // plane geometry: lines x points in, lines x nout out
  const int lines = (PASS == kDftZR2C || PASS == kDftZC2R) ? K : Kz;
  const int points = PASS == kDftZC2R ? Kz : K;
  const int nout = PASS == kDftZR2C ? Kz : K;
  T *rgrid = real + b.grid_off;
  C *cgrid = cplx + b.cplx_off;
  // load (global-contiguous order)
  for (int e = threadIdx.x; e < lines * points; e += blockDim.x) {
    int line, pt;
    C v;
    if (PASS == kDftZR2C) {  // plane x: [y][z] reals
      line = e / K;
      pt = e % K;
      v.x = rgrid[(int64_t)p * K * K + e];
      v.y = T(0);
    } else if (PASS == kDftZC2R) {  // plane x: [y][kz]
      line = e / Kz;
      pt = e % Kz;
      v = cgrid[(int64_t)p * K * Kz + e];
    } else if (PASS == kDftY || PASS == kDftYInv) {  // plane x: [y][kz], lines = kz
      pt = e / Kz;
      line = e % Kz;
      v = cgrid[(int64_t)p * K * Kz + e];
    } else {  // plane ky: [x][ky][kz], lines = kz
      pt = e / Kz;
      line = e % Kz;
      v = cgrid[((int64_t)pt * K + p) * Kz + line];
    }
    in[line * st + pt] = v;
  }
  __syncthreads();
  // outputs: one frequency (or z) per thread for R lines lg, lg + G, ... (G = ceil(lines / R)):
  // consecutive lanes take consecutive lines (odd row stride: distinct banks) and each
  // twiddle load serves R lines. Per output the sum runs over the line in a fixed order.
  constexpr int R = kDftLinesPerThread;
  const int G = (lines + R - 1) / R;
  for (int o = threadIdx.x; o < G * nout; o += blockDim.x) {
    const int lg = o % G, f = o / G;
    bool has[R];
    const C *row[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      has[r] = lg + r * G < lines;
      row[r] = in + (has[r] ? lg + r * G : lg) * st;
    }
    C acc[R];
    if (PASS == kDftZC2R) {
      // real output of a Hermitian half spectrum: T0 + 2 sum_{0<k<K/2} Re(Tk w^(zk)) [+ T_{K/2} (-1)^z]
      const int kh = (K - 1) / 2;
      T sum[R];
#pragma unroll
      for (int r = 0; r < R; ++r) sum[r] = row[r][0].x;
      int idx = 0;
      for (int k = 1; k <= kh; ++k) {
        idx += f;
        if (idx >= K) idx -= K;
        const C w = tw[idx];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const C a = row[r][k];
          sum[r] += T(2) * (a.x * w.x - a.y * w.y);
        }
      }
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if (!(K & 1)) sum[r] += (f & 1) ? -row[r][K / 2].x : row[r][K / 2].x;
        acc[r].x = sum[r];
        acc[r].y = T(0);
      }
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) acc[r].x = acc[r].y = T(0);
      int idx = 0;
      for (int j = 0; j < points; ++j) {
        const C w = tw[idx];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const C a = row[r][j];
          if (PASS == kDftZR2C) {  // real input
            acc[r].x += a.x * w.x;
            acc[r].y += a.x * w.y;
          } else {
            acc[r].x += a.x * w.x - a.y * w.y;
            acc[r].y += a.x * w.y + a.y * w.x;
          }
        }
        idx += f;
        if (idx >= K) idx -= K;
      }
    }
#pragma unroll
    for (int r = 0; r < R; ++r)
      if (has[r]) out[(lg + r * G) * st + f] = acc[r];
  }
  __syncthreads();
  // store (global-contiguous order)
  for (int e = threadIdx.x; e < lines * nout; e += blockDim.x) {
    if (PASS == kDftZR2C) {  // [y][kz]
      cgrid[(int64_t)p * K * Kz + e] = out[(e / Kz) * st + e % Kz];
    } else if (PASS == kDftZC2R) {  // [y][z] reals
      rgrid[(int64_t)p * K * K + e] = out[(e / K) * st + e % K].x;
    } else if (PASS == kDftY || PASS == kDftYInv) {  // [ky][kz], lines = kz
      cgrid[(int64_t)p * K * Kz + e] = out[(e % Kz) * st + e / Kz];
    } else {  // [kx][ky][kz], lines = kz
      const int f = e / Kz, line = e % Kz;
      cgrid[((int64_t)f * K + p) * Kz + line] = out[line * st + f];
    }
  }
}

template <class T, int PASS>
__global__ void __launch_bounds__(kDftThreads) batch_dft_kernel(const BatchSys *sys, const BatchShape *shape, T *real,
                                                                typename CplxOf<T>::type *cplx,
                                                                const typename CplxOf<T>::type *twtab,
                                                                unsigned *counter) {
  const int nsys = shape->nsys, units = shape->plane_units;
  for (int u = next_unit(counter); u < units; u = next_unit(counter)) {
    const BatchSys &b = sys[unit_system<kUnitsPlanes>(sys, nsys, u)];
    batch_dft_plane<T, PASS>(b, u - b.plane_off, real, cplx, twtab);
  }
}

// ---- batched PME: persistent kernels over work units numbered across the batch. The spread
// and the gather take units of a system's atoms (system s owns gather_off .. gather_off +
// gather_blocks - 1), the convolution units of its grid points (conv_off ..); a unit count
// depends on the system alone, so that its reductions sum in the same order whatever else
// is in the batch. The spread and the convolution keep 4 resident blocks per SM (at most 64
// registers): the loop's extra state had cost them a block per SM and 29 % / 67 % of their
// time at 256 systems.
constexpr int kBatchPmeMaxBlocks = 256;

// Zeroes the batch's accumulation grid (total_grid points of the shape).
template <class S>
__global__ void batch_zero_grid_kernel(const BatchShape *shape, S *grid) {
  const int64_t n = shape->total_grid;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    grid[k] = S(0);
}

static __global__ void batch_fix_to_real_kernel(const BatchShape *shape, const unsigned long long *gi, float *gf) {
  const int64_t n = shape->total_grid;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    gf[k] = (float)from_fix(gi[k]);
}

// One PME block of one system (a separate call: the unit loop's state then does not share
// the inner loops' register allocation).
template <class T>
__device__ __noinline__ void batch_spread_unit(const BatchSys *sys, const T *x, const T *q, const T *boxes,
                                               typename Acc<T>::S *grid, int sy, int bx, PmeShared &sh,
                                               GroupStencil *st) {
  const BatchSys &b = sys[sy];
  if (threadIdx.x == 0) load_pme_shared(boxes + 9 * (int64_t)sy, b.K, sh);
  __syncthreads();
  PlainAtoms<T> atoms{x + 3 * b.atom_off, q + b.atom_off, b.natoms};
  if constexpr (sizeof(T) == 4)
    spread_groups(atoms, b.natoms, sh, b.K, grid + b.grid_off, bx, b.gather_blocks, st);
  else
    spread_atoms<T>(atoms, b.natoms, sh, b.K, grid + b.grid_off, bx, b.gather_blocks);
}

template <class T>
__global__ void __launch_bounds__(kPmeBlock, 4) batch_spread_kernel(const BatchSys *sys, const BatchShape *shape,
                                                                 const T *x, const T *q, const T *boxes,
                                                                 typename Acc<T>::S *grid, unsigned *counter) {
  __shared__ PmeShared sh;
  __shared__ GroupStencil st[sizeof(T) == 4 ? kPmeBlock / kWarp : 1][kSpreadGroup * kGroupsPerPass];
  // the gather's units (a system's atoms never outnumber its sorted slots)
  const int nsys = shape->nsys, units = shape->gather_units;
  for (int u = next_unit(counter); u < units; u = next_unit(counter)) {
    const int sy = unit_system<kUnitsGather>(sys, nsys, u);
    batch_spread_unit<T>(sys, x, q, boxes, grid, sy, u - sys[sy].gather_off, sh,
                         st[sizeof(T) == 4 ? threadIdx.x >> 5 : 0]);
  }
}

// partials: kBatchPmeMaxBlocks per system; tickets and energies: 2 per system
// ([2s] reciprocal, [2s+1] self).
template <class T>
__global__ void __launch_bounds__(kPmeBlock, 4) batch_convolve_kernel(const BatchSys *sys, const BatchShape *shape,
                                                                   typename CplxOf<T>::type *S, const T *boxes,
                                                                   double alpha, const T *moduli, double *partials,
                                                                   unsigned *tickets, double *energies,
                                                                   unsigned *counter) {
  __shared__ PmeShared sh;
  const int nsys = shape->nsys, units = shape->conv_units;
  for (int u = next_unit(counter); u < units; u = next_unit(counter)) {
    const int sy = unit_system<kUnitsConv>(sys, nsys, u);
    const BatchSys &b = sys[sy];
    const int bx = u - b.conv_off;
    if (threadIdx.x == 0) load_pme_shared(boxes + 9 * (int64_t)sy, b.K, sh);
    __syncthreads();
    const T *xm = moduli + b.mod_off, *ym = xm + b.K, *zm = ym + b.K;
    const double e = convolve_points<T>(S + b.cplx_off, sh, b.K, alpha, xm, ym, zm, bx, b.conv_blocks);
    grid_sum_n<kPmeBlock>(0.5 * e, partials + (int64_t)kBatchPmeMaxBlocks * sy, tickets + 2 * sy, energies + 2 * sy,
                          false, bx, b.conv_blocks);
  }
}

template <class T>
// The atoms of a system are visited in the cluster order of the batch's sort (sidx: sorted
// slot -> batch atom index, -1 for padding), so that neighbouring threads read neighbouring
// grid points; each atom's numbers are those of the caller-order visit.
__global__ void __launch_bounds__(kPmeBlock, sizeof(T) == 4 ? 3 : 2) batch_gather_kernel(const BatchSys *sys, const BatchShape *shape,
                                                                 const T *x, const T *q, const int *sidx,
                                                                 const T *boxes, const T *Phi, double alpha, T *phi,
                                                                 T *grad, double *partials, unsigned *tickets,
                                                                 double *energies, unsigned *counter) {
  __shared__ PmeShared sh;
  const int nsys = shape->nsys, units = shape->gather_units;
  for (int u = next_unit(counter); u < units; u = next_unit(counter)) {
    const int sy = unit_system<kUnitsGather>(sys, nsys, u);
    const BatchSys &b = sys[sy];
    const int bx = u - b.gather_off;
    if (threadIdx.x == 0) load_pme_shared(boxes + 9 * (int64_t)sy, b.K, sh);
    __syncthreads();
    const int *slots = sidx + b.cl_off * kWarp;
    const int64_t nslots = b.ncl * kWarp;
    IndexedAtoms<T> atoms{x, q, slots, nslots};
    IndexedGatherOut<T> out{phi, grad, slots};
    const double e = gather_atoms<T>(atoms, nslots, sh, b.K, Phi + b.grid_off, alpha, out, bx, b.gather_blocks);
    grid_sum_n<kPmeBlock>(e, partials + (int64_t)kBatchPmeMaxBlocks * sy, tickets + 2 * sy + 1,
                          energies + 2 * sy + 1, false, bx, b.gather_blocks);
  }
}

// Scratch layout of one PME evaluation.
struct PmeLayout {
  int K;
  int64_t ngrid, ncplx;
  size_t fix, real, cplx, partials, tickets, energies, bytes;
  size_t zero_off, zero_bytes;
};

inline PmeLayout pme_layout(int dtype, int K) {
  PmeLayout L{};
  L.K = K;
  L.ngrid = (int64_t)K * K * K;
  L.ncplx = (int64_t)K * K * (K / 2 + 1);
  const size_t ts = dtype == TFF_F64 ? 8 : 4;
  Carver c(nullptr);
  // zeroed on every evaluation: reduction tickets, energies, the accumulation grid
  L.tickets = c.off; c.take<unsigned>(64);
  L.energies = (c.off + 255) & ~size_t(255); c.take<double>(8);
  L.fix = (c.off + 255) & ~size_t(255); c.take<char>(L.ngrid * 8);  // u64 fixed point (mixed) / double (FP64)
  L.zero_off = 0;
  L.zero_bytes = c.bytes();
  L.real = (c.off + 255) & ~size_t(255); c.take<char>(dtype == TFF_F64 ? 0 : L.ngrid * ts);
  L.cplx = (c.off + 255) & ~size_t(255); c.take<char>(L.ncplx * 2 * ts);
  L.partials = (c.off + 255) & ~size_t(255); c.take<double>(8192);
  L.bytes = c.bytes();
  return L;
}

struct PmePlanImpl {
  int dtype;
  int K;
  int device;
  cufftHandle r2c, c2r;
};

int pme_cufft_fail(cufftResult r, const char *what);

}  // namespace tff

struct tff_pme_plan_s {
  tff::PmePlanImpl impl;
};

namespace tff {

// FFT -> convolve -> FFT of the spread grid in ws (L.fix) on `s`; leaves the potential grid
// Phi in (T*)(ws + L.real) (mixed) or (T*)(ws + L.fix) (FP64), returned through *phi_grid.
template <class T>
int pme_solve_phase(const PmePlanImpl &p, const PmeLayout &L, char *ws, const T *box, double alpha, const T *xmod,
                    const T *ymod, const T *zmod, cudaStream_t s, T **phi_grid) {
  using S = typename Acc<T>::S;
  const int K = p.K;
  const int sms = sm_count();
  S *grid = reinterpret_cast<S *>(ws + L.fix);
  T *real;
  if (sizeof(T) == 4) {
    real = reinterpret_cast<T *>(ws + L.real);
    const int nb = (int)std::max<int64_t>(1, std::min<int64_t>((L.ngrid + 255) / 256, sms * 8));
    pme_fix_to_real_kernel<<<nb, 256, 0, s>>>(reinterpret_cast<unsigned long long *>(grid),
                                              reinterpret_cast<float *>(real), L.ngrid);
    TFF_LAUNCHED();
  } else {
    real = reinterpret_cast<T *>(grid);
  }
  auto *cplx = reinterpret_cast<typename CplxOf<T>::type *>(ws + L.cplx);
  cufftResult r;
  if ((r = cufftSetStream(p.r2c, s)) != CUFFT_SUCCESS) return pme_cufft_fail(r, "cufftSetStream");
  if ((r = cufftSetStream(p.c2r, s)) != CUFFT_SUCCESS) return pme_cufft_fail(r, "cufftSetStream");
  if (sizeof(T) == 4)
    r = cufftExecR2C(p.r2c, reinterpret_cast<cufftReal *>(real), reinterpret_cast<cufftComplex *>(cplx));
  else
    r = cufftExecD2Z(p.r2c, reinterpret_cast<cufftDoubleReal *>(real), reinterpret_cast<cufftDoubleComplex *>(cplx));
  if (r != CUFFT_SUCCESS) return pme_cufft_fail(r, "forward FFT");
  double *partials = reinterpret_cast<double *>(ws + L.partials);
  unsigned *tickets = reinterpret_cast<unsigned *>(ws + L.tickets);
  double *energies = reinterpret_cast<double *>(ws + L.energies);
  {
    const int nb = (int)std::max<int64_t>(1, std::min<int64_t>((L.ncplx + kPmeBlock - 1) / kPmeBlock, sms * 4));
    pme_convolve_kernel<T><<<nb, kPmeBlock, 0, s>>>(cplx, box, K, alpha, xmod, ymod, zmod, partials, tickets,
                                                    energies);
    TFF_LAUNCHED();
  }
  if (sizeof(T) == 4)
    r = cufftExecC2R(p.c2r, reinterpret_cast<cufftComplex *>(cplx), reinterpret_cast<cufftReal *>(real));
  else
    r = cufftExecZ2D(p.c2r, reinterpret_cast<cufftDoubleComplex *>(cplx), reinterpret_cast<cufftDoubleReal *>(real));
  if (r != CUFFT_SUCCESS) return pme_cufft_fail(r, "inverse FFT");
  *phi_grid = real;
  return TFF_OK;
}

// Enqueue spread -> FFT -> convolve -> FFT on `s` (see pme_solve_phase for the result).
template <class T, class Atoms>
int pme_grid_phase(const PmePlanImpl &p, const PmeLayout &L, char *ws, Atoms atoms, int64_t nthreads, const T *box,
                   double alpha, const T *xmod, const T *ymod, const T *zmod, cudaStream_t s, T **phi_grid) {
  using S = typename Acc<T>::S;
  TFF_CUDA(cudaMemsetAsync(ws + L.zero_off, 0, L.zero_bytes, s));
  S *grid = reinterpret_cast<S *>(ws + L.fix);
  if (nthreads > 0) {
    if constexpr (sizeof(T) == 4 && std::is_same<Atoms, PlainAtoms<float>>::value) {
      // FP32 caller-order atoms: groups of consecutive atoms (bit-identical grid), one warp
      // per group up to a few waves of blocks
      const int64_t groups = (nthreads + kSpreadGroup - 1) / kSpreadGroup;
      const int nb = (int)std::max<int64_t>(1, std::min<int64_t>((groups * kWarp + kPmeBlock - 1) / kPmeBlock,
                                                                 sm_count() * 8));
      pme_spread_grouped_kernel<Atoms><<<nb, kPmeBlock, 0, s>>>(atoms, nthreads, box, p.K, grid);
    } else {
      const int64_t lanes = nthreads * kLanesPerAtom;
      const int nb = (int)std::max<int64_t>(1, std::min<int64_t>((lanes + kPmeBlock - 1) / kPmeBlock, sm_count() * 8));
      pme_spread_kernel<T, Atoms><<<nb, kPmeBlock, 0, s>>>(atoms, nthreads, box, p.K, grid);
    }
    TFF_LAUNCHED();
  }
  return pme_solve_phase<T>(p, L, ws, box, alpha, xmod, ymod, zmod, s, phi_grid);
}

template <class T, class Atoms, class Out>
int pme_gather_phase(const PmePlanImpl &p, const PmeLayout &L, char *ws, Atoms atoms, int64_t nthreads, const T *box,
                     double alpha, const T *phi_grid, Out out, double e_scale, T *energy_out, cudaStream_t s) {
  double *partials = reinterpret_cast<double *>(ws + L.partials);
  unsigned *tickets = reinterpret_cast<unsigned *>(ws + L.tickets);
  double *energies = reinterpret_cast<double *>(ws + L.energies);
  const int64_t lanes = (nthreads + kGatherAtomsPerWarp - 1) / kGatherAtomsPerWarp * kWarp;
  const int nb = (int)std::max<int64_t>(1, std::min<int64_t>((lanes + kPmeBlock - 1) / kPmeBlock, sm_count() * 8));
  pme_gather_kernel<T, Atoms, Out><<<nb, kPmeBlock, 0, s>>>(atoms, nthreads, box, p.K, phi_grid, alpha, out,
                                                            partials, tickets + 1, energies + 1, energies, e_scale,
                                                            energy_out);
  TFF_LAUNCHED();
  return TFF_OK;
}

}  // namespace tff

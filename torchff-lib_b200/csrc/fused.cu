// Fused fixed-charge system: one evaluation = cluster build (full neighbour-cluster lists)
// -> fused real-space tile kernel (LJ with Lorentz-Berthelot combining + erfc-screened
// Coulomb, Ewald exclusion correction) || PME on a second stream (spread, FFT, influence
// function, FFT, gather) -> forces in caller order. It evaluates the nonbonded terms of
// examples/tip3p/model.py:100-133 (NeighborList + Vdw + MultipolarInteraction(rank 0) +
// PME) without materialising an int64 pair list.
//
// Tile kernel: one warp per work item = cluster I (lane l owns atom l of I) and up to
// kItemTiles clusters J taken with a stride from I's FULL neighbour list (entries k,
// k + n, k + 2n, ... for n = ceil(count / kItemTiles)), so that each item samples
// neighbours in every direction and the lanes get similar amounts of work.
//   pass 1: the J clusters are staged in shared memory; every lane sweeps the 32 atoms of
//           each with broadcast reads and builds a 32-bit in-cutoff mask per tile;
//   pass 2: each lane walks its own set bits across all tiles of the item and evaluates
//           LJ + erfc Coulomb only there;
//   pass 3: excluded pairs inside the cutoff get the Ewald exclusion correction.
// A cluster pair whose boxes are close enough uses one periodic shift for all its pairs
// (positions are cluster-contiguous images); other pairs use the per-pair minimum image.
// Each pair is evaluated from both sides, which removes j-side atomics: forces / charge
// gradients of atom i are summed in registers and added once per item into int64 fixed
// point accumulators (mixed) or FP64 atomics (FP64 mode); energies likewise, halved. With
// no block barrier a warp that finishes early does not wait for its block.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "pme.cuh"

namespace tff {
namespace {

constexpr int kMaxExcl = 8;       // excluded partners per atom (self excluded)

// Warps per block of the tile kernel: 4 (FP32) or 2 (FP64) so that the staged tiles fit in
// 48 KB of static shared memory.
template <class T> struct TileCfg { static constexpr int NW = sizeof(T) == 8 ? 2 : 4; };

template <class T> struct V2;
template <> struct V2<float> { using type = float2; };
struct __align__(16) D2 { double x, y; };
template <> struct V2<double> { using type = D2; };
__device__ __forceinline__ float2 make_v2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ D2 make_v2(double a, double b) { return D2{a, b}; }

__device__ __forceinline__ float erf_t(float x) { return erff(x); }
__device__ __forceinline__ double erf_t(double x) { return erf(x); }

// erfc(u) and exp(-u^2): A&S 7.1.26 in FP32, libdevice in FP64.
__device__ __forceinline__ void erfc_exp(float u, float &ec, float &ex) { erfc_exp_as(u, ec, ex); }
__device__ __forceinline__ void erfc_exp(double u, double &ec, double &ex) {
  ec = erfc(u);
  ex = exp(-u * u);
}
__device__ __forceinline__ float rsqrt_t(float x) { return rsqrtf(x); }
__device__ __forceinline__ double rsqrt_t(double x) { return rsqrt(x); }

template <class T>
struct TileArgs {
  ClusterData<T> cl;
  const typename V2<T>::type *lj;  // sorted slots: (sigma/2, sqrt(eps))
  const int *exslot;               // (npad, kMaxExcl) sorted slots of excluded partners, -1 padded
  typename Acc<T>::S *gx;          // (npad, 3) sorted slots, dE/dx
  typename Acc<T>::S *gq;          // (npad) sorted slots, dE/dq
  double rc, alpha, kc;
  typename Acc<T>::S *energies;    // [0] pairs (LJ + erfc Coulomb), [1] exclusion correction
};

// LB parameters and excluded-partner slots in sorted order.
template <class T>
__global__ void sorted_params_kernel(ClusterData<T> cl, const T *sigma, const T *eps, const int *excl,
                                     typename V2<T>::type *lj, int *exslot) {
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < cl.npad; s += (int64_t)gridDim.x * blockDim.x) {
    const int a = cl.sidx[s];
    lj[s] = a >= 0 ? make_v2(T(0.5) * sigma[a], (T)sqrt((double)eps[a])) : make_v2(T(0), T(0));
#pragma unroll
    for (int k = 0; k < kMaxExcl; ++k) {
      const int p = a >= 0 ? excl[(int64_t)a * kMaxExcl + k] : -1;
      exslot[s * kMaxExcl + k] = p >= 0 ? cl.inv[p] : -1;
    }
  }
}

template <class T>
__device__ __forceinline__ void pair_min_image(bool ortho, T &dx, T &dy, T &dz, const T *m, const T *inv) {
  if (ortho) {
    dx = wrap1(dx, m[0], inv[0]);
    dy = wrap1(dy, m[4], inv[4]);
    dz = wrap1(dz, m[8], inv[8]);
  } else {
    min_image(dx, dy, dz, m, inv);
  }
}

template <class T>
__global__ void __launch_bounds__(TileCfg<T>::NW * 32) tile_kernel(TileArgs<T> A) {
  using V = typename V4<T>::type;
  using W2 = typename V2<T>::type;
  constexpr int NW = TileCfg<T>::NW;
  __shared__ V s_pos[NW][kItemTiles][kWarp];
  __shared__ W2 s_lj[NW][kItemTiles][kWarp];
  // negated j positions, structure of arrays, for the packed FP32 distance pass
  __shared__ __align__(8) float s_nx[NW][kItemTiles][sizeof(T) == 4 ? kWarp : 2];
  __shared__ __align__(8) float s_ny[NW][kItemTiles][sizeof(T) == 4 ? kWarp : 2];
  __shared__ __align__(8) float s_nz[NW][kItemTiles][sizeof(T) == 4 ? kWarp : 2];
  __shared__ unsigned s_mask[NW][kItemTiles][kWarp];   // in-cutoff, not excluded
  __shared__ unsigned s_xmask[NW][kItemTiles][kWarp];  // in-cutoff, excluded
  __shared__ int s_mi[NW][kItemTiles];                 // 1: tile needs the per-pair minimum image
  __shared__ T s_m[9], s_inv[9];
  const ClusterData<T> &cl = A.cl;
  if (threadIdx.x < 9) {
    s_m[threadIdx.x] = (T)cl.boxinfo[threadIdx.x];
    s_inv[threadIdx.x] = (T)cl.boxinfo[9 + threadIdx.x];
  }
  __syncthreads();
  const bool ortho = cl.boxinfo[18] != 0.0;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const T rc2 = (T)(A.rc * A.rc);
  const T alpha = (T)A.alpha;
  const T kc = (T)A.kc;
  const T two_a_rpi = (T)(2.0 * A.alpha / 1.7724538509055160273);

  const int nitems = cl.itemoff[cl.nclusters];
  const int nwarps = gridDim.x * NW;
  for (int it = blockIdx.x * NW + w; it < nitems; it += nwarps) {
    const int I = cl.items[it];  // owning cluster: itemoff[I] <= it < itemoff[I + 1]
    const int k = it - cl.itemoff[I];
    const int nch = cl.itemoff[I + 1] - cl.itemoff[I];
    const int cnt = cl.ncount[I];
    const int ntile = (cnt - k + nch - 1) / nch;  // this item takes list entries k, k+nch, ...
    const int64_t si = (int64_t)I * kWarp + lane;
    const bool vi = cl.sidx[si] >= 0;
    const V pi = cl.pos[si];
    const W2 lji = A.lj[si];
    const T kqi = kc * pi.w;
    const V ci = cl.bc[I], hi_ = cl.bh[I];

    // stage the tiles and build their cutoff masks (pass 1)
    for (int t = 0; t < ntile; ++t) {
      const int J = cl.nbr[(int64_t)I * cl.cap + k + t * nch];
      const int64_t sj = (int64_t)J * kWarp + lane;
      // one periodic shift for the whole cluster pair when every pair's displacement then
      // lies within half a box length per axis (orthorhombic boxes)
      bool shifted = false;
      T sx = T(0), sy = T(0), sz = T(0);
      if (ortho) {
        const V cj = cl.bc[J], hj = cl.bh[J];
        const T dcx = ci.x - cj.x, dcy = ci.y - cj.y, dcz = ci.z - cj.z;
        const T nx = floor(dcx + T(0.5)), ny = floor(dcy + T(0.5)), nz = floor(dcz + T(0.5));
        shifted = (fabs(dcx - nx) + hi_.x + hj.x < T(0.49)) && (fabs(dcy - ny) + hi_.y + hj.y < T(0.49)) &&
                  (fabs(dcz - nz) + hi_.z + hj.z < T(0.49));
        sx = nx * s_m[0];
        sy = ny * s_m[4];
        sz = nz * s_m[8];
      }
      V pj = cl.pos[sj];
      if (shifted) {
        pj.x += sx;
        pj.y += sy;
        pj.z += sz;
      }
      s_pos[w][t][lane] = pj;
      s_lj[w][t][lane] = A.lj[sj];
      if (sizeof(T) == 4) {
        s_nx[w][t][lane] = -(float)pj.x;
        s_ny[w][t][lane] = -(float)pj.y;
        s_nz[w][t][lane] = -(float)pj.z;
      }
      const unsigned jvalid = __ballot_sync(kFull, cl.sidx[sj] >= 0);
      __syncwarp();
      unsigned mask = 0u;
      if (sizeof(T) == 4 && shifted) {
        // two j atoms per step with paired FP32 instructions (FADD2/FMUL2/FFMA2)
        const float2 px = make_float2((float)pi.x, (float)pi.x), py = make_float2((float)pi.y, (float)pi.y),
                     pz = make_float2((float)pi.z, (float)pi.z);
        const float rc2f = (float)rc2;
#pragma unroll 4
        for (int s = 0; s < kWarp; s += 2) {
          const float2 nx = *reinterpret_cast<const float2 *>(&s_nx[w][t][s]);
          const float2 ny = *reinterpret_cast<const float2 *>(&s_ny[w][t][s]);
          const float2 nz = *reinterpret_cast<const float2 *>(&s_nz[w][t][s]);
          const float2 dx = __fadd2_rn(px, nx), dy = __fadd2_rn(py, ny), dz = __fadd2_rn(pz, nz);
          float2 r2 = __fmul2_rn(dx, dx);
          r2 = __ffma2_rn(dy, dy, r2);
          r2 = __ffma2_rn(dz, dz, r2);
          mask |= (r2.x <= rc2f ? 1u : 0u) << s;
          mask |= (r2.y <= rc2f ? 2u : 0u) << s;
        }
      } else {
#pragma unroll 8
        for (int s = 0; s < kWarp; ++s) {
          const V q = s_pos[w][t][s];
          T dx = pi.x - q.x, dy = pi.y - q.y, dz = pi.z - q.z;
          if (!shifted) pair_min_image(ortho, dx, dy, dz, s_m, s_inv);
          const T r2 = dx * dx + dy * dy + dz * dz;
          mask |= (r2 <= rc2) ? (1u << s) : 0u;
        }
      }
      mask &= jvalid;
      if (J == I) mask &= ~(1u << lane);
      if (!vi) mask = 0u;
      unsigned emask = 0u;
      if (mask) {
#pragma unroll
        for (int x = 0; x < kMaxExcl; ++x) {
          const int xs = A.exslot[si * kMaxExcl + x];
          if (xs >= 0 && (xs >> 5) == J) emask |= 1u << (xs & 31);
        }
      }
      s_mask[w][t][lane] = mask & ~emask;
      s_xmask[w][t][lane] = mask & emask;
      if (lane == 0) s_mi[w][t] = !shifted;
    }
    __syncwarp();

    // pass 2: every lane walks its own in-cutoff pairs across all tiles of the item
    T fx = T(0), fy = T(0), fz = T(0), dq = T(0);
    double ep = 0.0;
    if constexpr (sizeof(T) == 4) {
      // FP32: two pairs per iteration with paired instructions (FADD2/FMUL2/FFMA2); only
      // rsqrt, reciprocal and exp2 stay scalar. A lane with an odd count pads the second
      // slot with a zero-charge, zero-epsilon copy of the first, which contributes nothing.
      const float2 one2 = make_float2(1.f, 1.f), mone2 = make_float2(-1.f, -1.f);
      const float2 al2 = make_float2(alpha, alpha), ta2 = make_float2(two_a_rpi, two_a_rpi);
      const float2 nkq2 = make_float2(-kqi, -kqi), kq2 = make_float2(kqi, kqi);
      const float2 pix = make_float2(pi.x, pi.x), piy = make_float2(pi.y, pi.y), piz = make_float2(pi.z, pi.z);
      const float2 sgi = make_float2(lji.x, lji.x), epi = make_float2(lji.y, lji.y);
      float2 fx2 = make_float2(0.f, 0.f), fy2 = fx2, fz2 = fx2, dq2 = fx2, te2 = fx2;
      int t = 0, iter = 0;
      unsigned m = ntile > 0 ? s_mask[w][0][lane] : 0u;
      while (true) {
        int ta = 0, sa = 0, tb = 0, sb = 0;
        while (m == 0u && ++t < ntile) m = s_mask[w][t][lane];
        const bool ha = m != 0u;
        if (ha) {
          sa = __ffs(m) - 1;
          m &= m - 1u;
          ta = t;
        }
        while (m == 0u && ++t < ntile) m = s_mask[w][t][lane];
        const bool hb = m != 0u;
        if (hb) {
          sb = __ffs(m) - 1;
          m &= m - 1u;
          tb = t;
        }
        if (!__any_sync(kFull, ha)) break;
        if ((++iter & 15) == 0) {
          ep += (double)(te2.x + te2.y);
          te2 = make_float2(0.f, 0.f);
        }
        if (ha) {
          const float4 qa = s_pos[w][ta][sa];
          float4 qb = hb ? s_pos[w][tb][sb] : make_float4(qa.x, qa.y, qa.z, 0.f);
          const float2 la = s_lj[w][ta][sa];
          const float2 lb = hb ? s_lj[w][tb][sb] : make_float2(0.f, 0.f);
          float2 dx = __fadd2_rn(pix, make_float2(-qa.x, -qb.x));
          float2 dy = __fadd2_rn(piy, make_float2(-qa.y, -qb.y));
          float2 dz = __fadd2_rn(piz, make_float2(-qa.z, -qb.z));
          if (s_mi[w][ta]) pair_min_image(ortho, dx.x, dy.x, dz.x, s_m, s_inv);
          if (hb && s_mi[w][tb]) pair_min_image(ortho, dx.y, dy.y, dz.y, s_m, s_inv);
          float2 r2 = __fmul2_rn(dx, dx);
          r2 = __ffma2_rn(dy, dy, r2);
          r2 = __ffma2_rn(dz, dz, r2);
          const float2 rinv = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
          const float2 rinv2 = __fmul2_rn(rinv, rinv);
          const float2 u = __fmul2_rn(__fmul2_rn(r2, rinv), al2);
          // erfc(u) exp(u^2) by Abramowitz & Stegun 7.1.26 (see erfc_exp_as)
          const float2 den = __ffma2_rn(u, make_float2(0.3275911f, 0.3275911f), one2);
          const float2 tt = make_float2(__fdividef(1.f, den.x), __fdividef(1.f, den.y));
          float2 poly = __ffma2_rn(tt, make_float2(1.061405429f, 1.061405429f),
                                   make_float2(-1.453152027f, -1.453152027f));
          poly = __ffma2_rn(tt, poly, make_float2(1.421413741f, 1.421413741f));
          poly = __ffma2_rn(tt, poly, make_float2(-0.284496736f, -0.284496736f));
          poly = __ffma2_rn(tt, poly, make_float2(0.254829592f, 0.254829592f));
          poly = __fmul2_rn(tt, poly);
          const float2 mu2 = __fmul2_rn(u, u);
          const float2 ex = make_float2(__expf(-mu2.x), __expf(-mu2.y));
          const float2 ec = __fmul2_rn(poly, ex);
          const float2 qj = make_float2(qa.w, qb.w);
          const float2 cq = __fmul2_rn(__fmul2_rn(qj, ec), rinv);  // E_coul / (k q_i)
          const float2 g = __ffma2_rn(ta2, __fmul2_rn(ex, rinv), __fmul2_rn(ec, rinv2));
          float2 dedr = __fmul2_rn(__fmul2_rn(g, rinv), __fmul2_rn(qj, nkq2));
          const float2 sig = __fadd2_rn(sgi, make_float2(la.x, lb.x));
          const float2 eps = __fmul2_rn(epi, make_float2(la.y, lb.y));
          const float2 sr2 = __fmul2_rn(__fmul2_rn(sig, sig), rinv2);
          const float2 sr6 = __fmul2_rn(__fmul2_rn(sr2, sr2), sr2);
          const float2 es6 = __fmul2_rn(eps, sr6);
          dedr = __ffma2_rn(__fmul2_rn(es6, make_float2(-24.f, -24.f)),
                            __fmul2_rn(__ffma2_rn(sr6, make_float2(2.f, 2.f), mone2), rinv2), dedr);
          fx2 = __ffma2_rn(dedr, dx, fx2);
          fy2 = __ffma2_rn(dedr, dy, fy2);
          fz2 = __ffma2_rn(dedr, dz, fz2);
          dq2 = __fadd2_rn(dq2, cq);
          te2 = __ffma2_rn(cq, kq2, te2);
          te2 = __ffma2_rn(__fmul2_rn(es6, make_float2(4.f, 4.f)), __fadd2_rn(sr6, mone2), te2);
        }
      }
      ep += (double)(te2.x + te2.y);
      fx = fx2.x + fx2.y;
      fy = fy2.x + fy2.y;
      fz = fz2.x + fz2.y;
      dq = dq2.x + dq2.y;
    } else {
      T te = T(0);  // partial energy, moved into ep every 16 pairs
      int t = 0, iter = 0;
      unsigned m = ntile > 0 ? s_mask[w][0][lane] : 0u;
      while (true) {
        while (m == 0u && ++t < ntile) m = s_mask[w][t][lane];
        const bool have = m != 0u;
        if (!__any_sync(kFull, have)) break;
        if ((++iter & 15) == 0) {
          ep += (double)te;
          te = T(0);
        }
        if (have) {
          const int s = __ffs(m) - 1;
          m &= m - 1u;
          const V q = s_pos[w][t][s];
          const W2 ljj = s_lj[w][t][s];
          T dx = pi.x - q.x, dy = pi.y - q.y, dz = pi.z - q.z;
          if (s_mi[w][t]) pair_min_image(ortho, dx, dy, dz, s_m, s_inv);
          const T r2 = dx * dx + dy * dy + dz * dz;
          const T rinv = rsqrt_t(r2);
          const T rinv2 = rinv * rinv;
          const T u = alpha * (r2 * rinv);
          T ec, ex2;
          erfc_exp(u, ec, ex2);
          const T cq = q.w * ec * rinv;  // E_coul / (k q_i)
          T dedr_r = -kqi * q.w * (ec * rinv2 + two_a_rpi * ex2 * rinv) * rinv;
          const T sig = lji.x + ljj.x;
          const T eps = lji.y * ljj.y;
          const T sr2 = sig * sig * rinv2;
          const T sr6 = sr2 * sr2 * sr2;
          dedr_r -= T(24) * eps * sr6 * (T(2) * sr6 - T(1)) * rinv2;
          fx += dedr_r * dx;
          fy += dedr_r * dy;
          fz += dedr_r * dz;
          dq += cq;
          te += kqi * cq + T(4) * eps * sr6 * (sr6 - T(1));
        }
      }
      ep += (double)te;
    }
    // pass 3: excluded pairs within the cutoff: Ewald exclusion correction
    // k q_i q_j (erfc(u) - 1)/r = -k q_i q_j erf(u)/r, no LJ
    double ex = 0.0;
    int t = 0;
    unsigned m = ntile > 0 ? s_xmask[w][0][lane] : 0u;
    while (true) {
      while (m == 0u && ++t < ntile) m = s_xmask[w][t][lane];
      const bool have = m != 0u;
      if (!__any_sync(kFull, have)) break;
      if (have) {
        const int s = __ffs(m) - 1;
        m &= m - 1u;
        const V q = s_pos[w][t][s];
        T dx = pi.x - q.x, dy = pi.y - q.y, dz = pi.z - q.z;
        if (s_mi[w][t]) pair_min_image(ortho, dx, dy, dz, s_m, s_inv);
        const T r2 = dx * dx + dy * dy + dz * dz;
        const T rinv = rsqrt_t(r2);
        const T u = alpha * (r2 * rinv);
        const T damp = -erf_t(u);
        const T ex2 = exp(-u * u);
        const T cq = q.w * damp * rinv;
        const T dedr_r = -kqi * q.w * (damp * rinv * rinv + two_a_rpi * ex2 * rinv) * rinv;
        fx += dedr_r * dx;
        fy += dedr_r * dy;
        fz += dedr_r * dz;
        dq += cq;
        ex += (double)(kqi * cq);
      }
    }
    if (vi) {
      Acc<T>::add(&A.gx[3 * si], (double)fx);
      Acc<T>::add(&A.gx[3 * si + 1], (double)fy);
      Acc<T>::add(&A.gx[3 * si + 2], (double)fz);
      Acc<T>::add(&A.gq[si], (double)kc * (double)dq);
    }
    // energies: warp sum, then one order-independent accumulation per work item
    ep = warp_sum(ep);
    ex = warp_sum(ex);
    if (lane == 0) {
      Acc<T>::add(&A.energies[0], 0.5 * ep);
      Acc<T>::add(&A.energies[1], 0.5 * ex);
    }
    __syncwarp();
  }
}

// Sorted real-space accumulators + caller-order PME derivatives -> caller order; energies.
template <class T>
__global__ void finalize_kernel(ClusterData<T> cl, const typename Acc<T>::S *gx, const typename Acc<T>::S *gq,
                                const T *pme_grad, const T *pme_phi, T *forces, double *forces64, T *grad_q,
                                const typename Acc<T>::S *e_tile_acc, const double *e_pme, double kc,
                                double *energy, double *terms) {
  for (int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; a < cl.natoms;
       a += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = cl.inv[a];
    double x = Acc<T>::get(&gx[3 * s]), y = Acc<T>::get(&gx[3 * s + 1]), z = Acc<T>::get(&gx[3 * s + 2]);
    double g = Acc<T>::get(&gq[s]);
    if (pme_grad) {
      x += kc * (double)pme_grad[3 * a];
      y += kc * (double)pme_grad[3 * a + 1];
      z += kc * (double)pme_grad[3 * a + 2];
      g += kc * (double)pme_phi[a];
    }
    if (forces) {
      forces[3 * a] = (T)(-x);
      forces[3 * a + 1] = (T)(-y);
      forces[3 * a + 2] = (T)(-z);
    }
    if (forces64) {
      forces64[3 * a] = -x;
      forces64[3 * a + 1] = -y;
      forces64[3 * a + 2] = -z;
    }
    if (grad_q) grad_q[a] = (T)g;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const double e_tile[2] = {Acc<T>::get(&e_tile_acc[0]), Acc<T>::get(&e_tile_acc[1])};
    const double rec = e_pme ? kc * e_pme[0] : 0.0;
    const double self = e_pme ? kc * e_pme[1] : 0.0;
    const double tot = e_tile[0] + e_tile[1] + rec + self;
    if (energy) energy[0] = tot;
    if (terms) {
      terms[0] = e_tile[0];
      terms[1] = e_tile[1];
      terms[2] = rec;
      terms[3] = self;
    }
  }
}

template <class T>
__global__ void cast_inputs_kernel(const double *x64, const double *box64, T *x, T *box, int64_t n3) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n3; k += (int64_t)gridDim.x * blockDim.x)
    x[k] = (T)x64[k];
  if (blockIdx.x == 0 && threadIdx.x < 9) box[threadIdx.x] = (T)box64[threadIdx.x];
}

// Host-side B-spline moduli theta(k) = sum_{m=-3}^{2} M6(m+3) cos(2 pi m k / K)
// (torchff/bsplines.py:20-63), with M6 at the integers from the same recursion as the
// device splines.
void host_bspline6_at_integers(double val[6]) {
  double m[6] = {0, 1, 0, 0, 0, 0};  // M2(0)=0, M2(1)=1
  for (int n = 3; n <= 6; ++n) {
    double nm[6] = {0};
    for (int k = 0; k < n; ++k) {
      const double cur = (k < n - 1) ? m[k] : 0.0;
      const double prev = (k > 0) ? m[k - 1] : 0.0;
      nm[k] = ((double)k * cur + (double)(n - k) * prev) / (double)(n - 1);
    }
    for (int k = 0; k < 6; ++k) m[k] = nm[k];
  }
  for (int k = 0; k < 6; ++k) val[k] = m[k];
}

std::vector<double> host_moduli(int K, int count) {
  double b[6];
  host_bspline6_at_integers(b);
  std::vector<double> out(count);
  for (int k = 0; k < count; ++k) {
    double s = 0.0;
    for (int m = -3; m < 3; ++m) s += b[m + 3] * std::cos(2.0 * M_PI * m * k / K);
    out[k] = s;
  }
  return out;
}

}  // namespace
}  // namespace tff

using namespace tff;

struct tff_timer_s {
  cudaEvent_t ev[TFF_TIMER_EVENTS];
};

struct tff_system_s {
  tff_system_desc desc;
  int cap;
  ClusterLayout cl;
  PmeLayout pl;
  tff_pme_plan pme = nullptr;
  cudaStream_t pme_stream = nullptr;  // PME runs here, forked from / joined to the caller stream
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
  void *cl_ws = nullptr;
  void *pme_ws = nullptr;
  void *acc = nullptr;         // gx (npad*3), gq (npad): zeroed per evaluation
  size_t acc_bytes = 0;
  void *lj = nullptr;          // sorted (sigma/2, sqrt eps)
  int *exslot = nullptr;       // sorted excluded-partner slots (npad, kMaxExcl)
  void *pme_grad = nullptr;    // PME dE/dx (N,3), caller order, e^2/nm units
  void *pme_phi = nullptr;     // PME dE/dq (N), caller order
  void *q = nullptr, *sigma = nullptr, *eps = nullptr;  // per-atom, system dtype
  int *excl = nullptr;         // (N, kMaxExcl)
  void *moduli = nullptr;      // xmod (K), ymod (K), zmod (K/2+1)
  double *scratch = nullptr;   // real-space energy accumulators (8 x 8 bytes)
  void *host_x = nullptr;      // device staging for *_host: coords64 (3N) + box64 (9)
  void *dev_x = nullptr;       // coords/box in system dtype for *_host
  double *dev_f = nullptr;     // forces64 for *_host
  double *dev_e = nullptr;
  cudaGraphExec_t host_graph = nullptr;  // device part of tff_system_eval_host, captured once
  cudaStream_t capture_stream = nullptr;
};

namespace tff {
namespace {

// Records a timing event; inside a stream capture it becomes an event-record node.
int record_event(cudaEvent_t e, cudaStream_t s) {
  if (e == nullptr) return TFF_OK;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  TFF_CUDA(cudaStreamIsCapturing(s, &cs));
  if (cs == cudaStreamCaptureStatusActive)
    TFF_CUDA(cudaEventRecordWithFlags(e, s, cudaEventRecordExternal));
  else
    TFF_CUDA(cudaEventRecord(e, s));
  return TFF_OK;
}

template <class T>
int system_eval_impl(tff_system sys, const T *x, const T *box, double *energy, T *forces, double *forces64, T *grad_q,
                     double *terms, cudaStream_t s, cudaEvent_t *ev = nullptr) {
  using S = typename Acc<T>::S;
  const int64_t n = sys->desc.natoms;
  auto mark = [&](int k, cudaStream_t st) { return ev ? record_event(ev[k], st) : TFF_OK; };
  int st = mark(0, s);
  if (st != TFF_OK) return st;
  const int sms = sm_count();
  S *energies = reinterpret_cast<S *>(sys->scratch);  // real-space energy accumulators
  TFF_CUDA(cudaMemsetAsync(sys->scratch, 0, 8 * sizeof(double), s));

  // --- PME on the side stream: needs only the caller's coordinates and the charges
  const bool use_pme = sys->pme && n > 0;
  const double *e_pme = nullptr;
  if (use_pme) {
    TFF_CUDA(cudaEventRecord(sys->fork_ev, s));
    TFF_CUDA(cudaStreamWaitEvent(sys->pme_stream, sys->fork_ev, 0));
    cudaStream_t ps = sys->pme_stream;
    const int K = sys->desc.pme_grid;
    const T *xm = static_cast<const T *>(sys->moduli);
    const T *ym = xm + K;
    const T *zm = ym + K;
    char *pw = static_cast<char *>(sys->pme_ws);
    PlainAtoms<T> atoms{x, static_cast<const T *>(sys->q), n};
    T *phi_grid = nullptr;
    st = pme_grid_phase<T>(sys->pme->impl, sys->pl, pw, atoms, n, box, sys->desc.ewald_alpha, xm, ym, zm, ps,
                           &phi_grid);
    if (st != TFF_OK) return st;
    if ((st = mark(3, ps)) != TFF_OK) return st;
    PlainGatherOut<T> out{static_cast<T *>(sys->pme_phi), static_cast<T *>(sys->pme_grad)};
    st = pme_gather_phase<T>(sys->pme->impl, sys->pl, pw, atoms, n, box, sys->desc.ewald_alpha, phi_grid, out, 1.0,
                             (T *)nullptr, ps);
    if (st != TFF_OK) return st;
    if ((st = mark(4, ps)) != TFF_OK) return st;
    TFF_CUDA(cudaEventRecord(sys->join_ev, ps));
    e_pme = reinterpret_cast<const double *>(pw + sys->pl.energies);
  }

  // --- real space on the caller stream
  ClusterData<T> cd = cluster_data<T>(sys->cl, sys->cl_ws);
  st = build_clusters<T>(sys->cl, cd, sys->cl_ws, x, static_cast<const T *>(sys->q), box, sys->desc.cutoff,
                         /*half=*/0, s);
  if (st != TFF_OK) return st;
  if ((st = mark(1, s)) != TFF_OK) return st;
  S *gx = static_cast<S *>(sys->acc);
  S *gq = gx + 3 * sys->cl.npad;
  TFF_CUDA(cudaMemsetAsync(sys->acc, 0, sys->acc_bytes, s));
  auto *lj = static_cast<typename V2<T>::type *>(sys->lj);
  if (n > 0) {
    const int nb = (int)std::max<int64_t>(1, std::min<int64_t>((sys->cl.npad + 255) / 256, sms * 8));
    sorted_params_kernel<T><<<nb, 256, 0, s>>>(cd, static_cast<const T *>(sys->sigma),
                                               static_cast<const T *>(sys->eps), sys->excl, lj, sys->exslot);
    TFF_LAUNCHED();
    TileArgs<T> A;
    A.cl = cd;
    A.lj = lj;
    A.exslot = sys->exslot;
    A.gx = gx;
    A.gq = gq;
    A.rc = sys->desc.cutoff;
    A.alpha = sys->desc.ewald_alpha;
    A.kc = sys->desc.coul_constant;
    A.energies = energies;
    // work items are only known on the device: size the grid for the largest possible
    // count (every cluster with a full list), capped at a few waves of the SMs
    const int64_t max_items = sys->cl.nclusters * ((sys->cl.cap + kItemTiles - 1) / kItemTiles);
    constexpr int NW = TileCfg<T>::NW;
    const int nbt = (int)std::max<int64_t>(1, std::min<int64_t>((max_items + NW - 1) / NW, (int64_t)sms * 48 / NW));
    tile_kernel<T><<<nbt, NW * kWarp, 0, s>>>(A);
    TFF_LAUNCHED();
  }
  if ((st = mark(2, s)) != TFF_OK) return st;
  if (use_pme) TFF_CUDA(cudaStreamWaitEvent(s, sys->join_ev, 0));
  const int nbf = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, sms * 8));
  finalize_kernel<T><<<nbf, 256, 0, s>>>(cd, gx, gq, use_pme ? static_cast<const T *>(sys->pme_grad) : nullptr,
                                         use_pme ? static_cast<const T *>(sys->pme_phi) : nullptr, forces, forces64,
                                         grad_q, energies, e_pme, sys->desc.coul_constant, energy, terms);
  TFF_LAUNCHED();
  return mark(5, s);
}

template <class T>
int set_params_impl(tff_system sys, const T *q, const T *sig, const T *eps, cudaStream_t s) {
  const size_t bytes = sizeof(T) * sys->desc.natoms;
  if (q) TFF_CUDA(cudaMemcpyAsync(sys->q, q, bytes, cudaMemcpyDeviceToDevice, s));
  if (sig) TFF_CUDA(cudaMemcpyAsync(sys->sigma, sig, bytes, cudaMemcpyDeviceToDevice, s));
  if (eps) TFF_CUDA(cudaMemcpyAsync(sys->eps, eps, bytes, cudaMemcpyDeviceToDevice, s));
  return TFF_OK;
}

void free_system(tff_system sys) {
  if (!sys) return;
  if (sys->pme) tff_pme_plan_destroy(sys->pme);
  if (sys->pme_stream) cudaStreamDestroy(sys->pme_stream);
  if (sys->fork_ev) cudaEventDestroy(sys->fork_ev);
  if (sys->join_ev) cudaEventDestroy(sys->join_ev);
  if (sys->host_graph) cudaGraphExecDestroy(sys->host_graph);
  if (sys->capture_stream) cudaStreamDestroy(sys->capture_stream);
  void *ptrs[] = {sys->cl_ws, sys->pme_ws, sys->acc, sys->lj, sys->exslot, sys->pme_grad, sys->pme_phi,
                  sys->q, sys->sigma, sys->eps, sys->excl, sys->moduli, sys->scratch, sys->host_x,
                  sys->dev_x, sys->dev_f, sys->dev_e};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  delete sys;
}

}  // namespace
}  // namespace tff

extern "C" {

int tff_system_create(const tff_system_desc *desc, const double *charges, const double *sigma, const double *epsilon,
                      int64_t nexcl, const int64_t *excl_pairs, tff_system *out) {
  TFF_ARG(desc != nullptr && out != nullptr, "desc/out is NULL");
  TFF_ARG(desc->dtype == TFF_F32 || desc->dtype == TFF_F64, "dtype must be TFF_F32 or TFF_F64");
  const int64_t n = desc->natoms;
  TFF_ARG(n >= 0 && n < (int64_t)1 << 30, "natoms out of range");
  TFF_ARG(desc->cutoff > 0.0, "cutoff must be positive");
  TFF_ARG(desc->ewald_alpha > 0.0, "ewald_alpha must be positive");
  TFF_ARG(desc->pme_grid == 0 || desc->pme_grid >= 6, "pme_grid must be 0 or >= 6");
  TFF_ARG(n == 0 || (charges && sigma && epsilon), "parameters are NULL");
  TFF_ARG(nexcl == 0 || excl_pairs != nullptr, "exclusion pairs are NULL");
  // exclusion partners (both directions, deduplicated, self dropped)
  std::vector<std::vector<int>> part(n);
  for (int64_t e = 0; e < nexcl; ++e) {
    const int64_t a = excl_pairs[2 * e], b = excl_pairs[2 * e + 1];
    TFF_ARG(a >= 0 && b >= 0 && a < n && b < n, "exclusion index out of range");
    if (a == b) continue;
    part[a].push_back((int)b);
    part[b].push_back((int)a);
  }
  std::vector<int> ex((size_t)n * kMaxExcl, -1);
  for (int64_t a = 0; a < n; ++a) {
    auto &v = part[a];
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
    TFF_ARG(v.size() <= (size_t)kMaxExcl, "atom %lld has %zu excluded partners; at most %d supported", (long long)a,
            v.size(), kMaxExcl);
    for (size_t k = 0; k < v.size(); ++k) ex[(size_t)a * kMaxExcl + k] = v[k];
  }
  auto *sys = new tff_system_s();
  sys->desc = *desc;
  const int64_t ncl = (n + kWarp - 1) / kWarp;
  sys->cap = desc->max_cluster_neighbors > 0 ? desc->max_cluster_neighbors
                                             : (int)std::max<int64_t>(1, std::min<int64_t>(ncl, 1024));
  sys->cl = cluster_layout(desc->dtype, n, sys->cap);
  const size_t ts = desc->dtype == TFF_F64 ? 8 : 4;
#define TFF_ALLOC(ptr, bytes)                                              \
  do {                                                                     \
    cudaError_t _e = cudaMalloc((void **)&(ptr), (bytes) ? (bytes) : 256); \
    if (_e != cudaSuccess) {                                               \
      free_system(sys);                                                    \
      return cuda_fail(_e, "cudaMalloc", __FILE__, __LINE__);              \
    }                                                                      \
  } while (0)
  TFF_ALLOC(sys->cl_ws, sys->cl.bytes);
  sys->acc_bytes = (size_t)sys->cl.npad * 4 * 8;
  TFF_ALLOC(sys->acc, sys->acc_bytes);
  TFF_ALLOC(sys->lj, (size_t)sys->cl.npad * 2 * ts);
  TFF_ALLOC(sys->exslot, (size_t)sys->cl.npad * kMaxExcl * sizeof(int));
  TFF_ALLOC(sys->pme_grad, 3 * n * ts);
  TFF_ALLOC(sys->pme_phi, n * ts);
  TFF_ALLOC(sys->q, n * ts);
  TFF_ALLOC(sys->sigma, n * ts);
  TFF_ALLOC(sys->eps, n * ts);
  TFF_ALLOC(sys->excl, ex.size() * sizeof(int));
  TFF_ALLOC(sys->scratch, 8192 * sizeof(double) + 256 + 8 * sizeof(double));
  TFF_ALLOC(sys->host_x, (3 * n + 9) * sizeof(double));
  TFF_ALLOC(sys->dev_x, (3 * n + 9) * ts);
  TFF_ALLOC(sys->dev_f, 3 * n * sizeof(double));
  TFF_ALLOC(sys->dev_e, 8 * sizeof(double));
  cudaError_t e = cudaStreamCreateWithFlags(&sys->pme_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sys->fork_ev, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sys->join_ev, cudaEventDisableTiming);
  auto upload = [&](void *dst, const double *src, int64_t cnt) {
    if (cnt == 0 || e != cudaSuccess) return;
    if (ts == 8) {
      e = cudaMemcpy(dst, src, cnt * 8, cudaMemcpyHostToDevice);
    } else {
      std::vector<float> tmp(src, src + cnt);
      e = cudaMemcpy(dst, tmp.data(), cnt * 4, cudaMemcpyHostToDevice);
    }
  };
  upload(sys->q, charges, n);
  upload(sys->sigma, sigma, n);
  upload(sys->eps, epsilon, n);
  if (e == cudaSuccess && n > 0) e = cudaMemcpy(sys->excl, ex.data(), ex.size() * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(sys->scratch, 0, 8192 * sizeof(double) + 256 + 8 * sizeof(double));
  if (e != cudaSuccess) {
    free_system(sys);
    return cuda_fail(e, "system set-up", __FILE__, __LINE__);
  }
  if (desc->pme_grid > 0) {
    const int K = desc->pme_grid;
    int st = tff_pme_plan_create(desc->dtype, K, &sys->pme);
    if (st != TFF_OK) {
      sys->pme = nullptr;
      free_system(sys);
      return st;
    }
    sys->pl = pme_layout(desc->dtype, K);
    TFF_ALLOC(sys->pme_ws, sys->pl.bytes);
    TFF_ALLOC(sys->moduli, (size_t)(2 * K + K / 2 + 1) * ts);
    std::vector<double> mod;
    auto mx = host_moduli(K, K);
    auto mz = host_moduli(K, K / 2 + 1);
    mod.insert(mod.end(), mx.begin(), mx.end());
    mod.insert(mod.end(), mx.begin(), mx.end());
    mod.insert(mod.end(), mz.begin(), mz.end());
    upload(sys->moduli, mod.data(), (int64_t)mod.size());
    if (e == cudaSuccess) e = cudaMemset(sys->pme_ws, 0, sys->pl.bytes);
    if (e != cudaSuccess) {
      free_system(sys);
      return cuda_fail(e, "upload moduli", __FILE__, __LINE__);
    }
  }
#undef TFF_ALLOC
  *out = sys;
  return TFF_OK;
}

int tff_system_destroy(tff_system sys) {
  free_system(sys);
  return TFF_OK;
}

int tff_system_set_parameters(tff_system sys, const void *charges, const void *sigma, const void *epsilon,
                              tff_stream_t stream) {
  TFF_ARG(sys != nullptr, "system is NULL");
  cudaStream_t s = (cudaStream_t)stream;
  if (sys->desc.dtype == TFF_F32)
    return set_params_impl<float>(sys, (const float *)charges, (const float *)sigma, (const float *)epsilon, s);
  return set_params_impl<double>(sys, (const double *)charges, (const double *)sigma, (const double *)epsilon, s);
}

int tff_system_eval(tff_system sys, const void *coords, const void *box, double *energy, void *forces,
                    void *grad_charges, double *energy_terms, tff_stream_t stream) {
  TFF_ARG(sys != nullptr, "system is NULL");
  TFF_ARG(box != nullptr, "box is NULL");
  TFF_ARG(sys->desc.natoms == 0 || coords != nullptr, "coords is NULL");
  cudaStream_t s = (cudaStream_t)stream;
  if (sys->desc.dtype == TFF_F32)
    return system_eval_impl<float>(sys, (const float *)coords, (const float *)box, energy, (float *)forces, nullptr,
                                   (float *)grad_charges, energy_terms, s);
  return system_eval_impl<double>(sys, (const double *)coords, (const double *)box, energy, (double *)forces, nullptr,
                                  (double *)grad_charges, energy_terms, s);
}

int tff_system_eval_host(tff_system sys, const double *coords, const double *box, double *energy, double *forces,
                         tff_stream_t stream) {
  TFF_ARG(sys != nullptr, "system is NULL");
  TFF_ARG(box != nullptr && energy != nullptr, "box/energy is NULL");
  const int64_t n = sys->desc.natoms;
  TFF_ARG(n == 0 || (coords != nullptr && forces != nullptr), "coords/forces is NULL");
  cudaStream_t s = (cudaStream_t)stream;
  double *stage = static_cast<double *>(sys->host_x);
  // The device part (FP64 -> system dtype cast + evaluation into internal buffers) only
  // touches the system's own buffers, so it is captured into a CUDA graph on the first
  // call (on an internal stream) and replayed on `stream` afterwards.
  if (sys->host_graph == nullptr) {
    if (sys->capture_stream == nullptr)
      TFF_CUDA(cudaStreamCreateWithFlags(&sys->capture_stream, cudaStreamNonBlocking));
    cudaStream_t cs = sys->capture_stream;
    TFF_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    int st;
    const int nb = (int)std::max<int64_t>(1, std::min<int64_t>((3 * n + 255) / 256, sm_count() * 8));
    if (sys->desc.dtype == TFF_F32) {
      float *x = static_cast<float *>(sys->dev_x);
      cast_inputs_kernel<float><<<nb, 256, 0, cs>>>(stage, stage + 3 * n, x, x + 3 * n, 3 * n);
      st = system_eval_impl<float>(sys, x, x + 3 * n, sys->dev_e, nullptr, sys->dev_f, nullptr, nullptr, cs);
    } else {
      double *x = static_cast<double *>(sys->dev_x);
      cast_inputs_kernel<double><<<nb, 256, 0, cs>>>(stage, stage + 3 * n, x, x + 3 * n, 3 * n);
      st = system_eval_impl<double>(sys, x, x + 3 * n, sys->dev_e, nullptr, sys->dev_f, nullptr, nullptr, cs);
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(cs, &graph);
    if (st != TFF_OK) {
      if (graph) cudaGraphDestroy(graph);
      return st;
    }
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture", __FILE__, __LINE__);
    const cudaError_t ie = cudaGraphInstantiate(&sys->host_graph, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) {
      sys->host_graph = nullptr;
      return cuda_fail(ie, "cudaGraphInstantiate", __FILE__, __LINE__);
    }
  }
  if (n > 0) TFF_CUDA(cudaMemcpyAsync(stage, coords, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s));
  TFF_CUDA(cudaMemcpyAsync(stage + 3 * n, box, 9 * sizeof(double), cudaMemcpyHostToDevice, s));
  TFF_CUDA(cudaGraphLaunch(sys->host_graph, s));
  if (n > 0) TFF_CUDA(cudaMemcpyAsync(forces, sys->dev_f, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
  TFF_CUDA(cudaMemcpyAsync(energy, sys->dev_e, sizeof(double), cudaMemcpyDeviceToHost, s));
  TFF_CUDA(cudaStreamSynchronize(s));
  return TFF_OK;
}

int tff_timer_create(tff_timer *timer) {
  TFF_ARG(timer != nullptr, "timer is NULL");
  auto *t = new tff_timer_s();
  for (int k = 0; k < TFF_TIMER_EVENTS; ++k) {
    cudaError_t e = cudaEventCreate(&t->ev[k]);
    if (e != cudaSuccess) {
      for (int j = 0; j < k; ++j) cudaEventDestroy(t->ev[j]);
      delete t;
      return cuda_fail(e, "cudaEventCreate", __FILE__, __LINE__);
    }
  }
  *timer = t;
  return TFF_OK;
}

int tff_timer_destroy(tff_timer timer) {
  if (!timer) return TFF_OK;
  for (int k = 0; k < TFF_TIMER_EVENTS; ++k) cudaEventDestroy(timer->ev[k]);
  delete timer;
  return TFF_OK;
}

int tff_timer_elapsed_ms(tff_timer timer, int from, int to, float *ms) {
  TFF_ARG(timer != nullptr && ms != nullptr, "timer/ms is NULL");
  TFF_ARG(from >= 0 && to >= 0 && from < TFF_TIMER_EVENTS && to < TFF_TIMER_EVENTS, "event index out of range");
  TFF_CUDA(cudaEventSynchronize(timer->ev[to]));
  TFF_CUDA(cudaEventElapsedTime(ms, timer->ev[from], timer->ev[to]));
  return TFF_OK;
}

int tff_system_eval_timed(tff_system sys, const void *coords, const void *box, double *energy, void *forces,
                          tff_timer timer, tff_stream_t stream) {
  TFF_ARG(sys != nullptr && timer != nullptr, "system/timer is NULL");
  TFF_ARG(box != nullptr, "box is NULL");
  TFF_ARG(sys->desc.natoms == 0 || coords != nullptr, "coords is NULL");
  cudaStream_t s = (cudaStream_t)stream;
  if (sys->desc.dtype == TFF_F32)
    return system_eval_impl<float>(sys, (const float *)coords, (const float *)box, energy, (float *)forces, nullptr,
                                   nullptr, nullptr, s, timer->ev);
  return system_eval_impl<double>(sys, (const double *)coords, (const double *)box, energy, (double *)forces,
                                  nullptr, nullptr, nullptr, s, timer->ev);
}

int tff_system_kernel_launches(tff_system sys) {
  if (!sys) return 0;
  // cluster build 7 + sorted params 1 + tile 1 + finalize 1; PME: spread, [to_real], convolve, gather
  int k = 10;
  if (sys->pme) k += sys->desc.dtype == TFF_F32 ? 4 : 3;
  return k;
}

int tff_system_status(tff_system sys, tff_stream_t stream, int *status) {
  TFF_ARG(sys != nullptr && status != nullptr, "system/status is NULL");
  unsigned v = 0;
  char *b = static_cast<char *>(sys->cl_ws);
  TFF_CUDA(cudaMemcpyAsync(&v, b + sys->cl.status, sizeof(unsigned), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
  TFF_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
  *status = (int)v;
  return TFF_OK;
}

}  // extern "C"

// Fused real-space kernels shared by the single-system and the batched evaluation.
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
#pragma once

#include <cmath>
#include <vector>

#include "bonded.cuh"
#include "pme.cuh"

namespace tff {
namespace {

constexpr int kMaxExcl = 8;       // excluded partners per atom (self excluded)

// Warps per block of the tile kernel: 4 (FP32) or 2 (FP64) so that the staged tiles fit in
// 48 KB of static shared memory.
// MODE 0: energy, dE/dx, dE/dq. MODE 1: also dE/dsigma and dE/d(sqrt eps). MODE 2: second
// derivatives along a coordinate direction u: d/dx, d/dq, d/dsigma, d/d(sqrt eps) of u . dE/dx.
template <class T, int MODE = 0> struct TileCfg {
  static constexpr int NW = (sizeof(T) == 8 || MODE == 2) ? 2 : 4;
};

template <class T> struct V2;
template <> struct V2<float> { using type = float2; };
struct __align__(16) D2 { double x, y; };
template <> struct V2<double> { using type = D2; };
__device__ __forceinline__ float2 make_v2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ D2 make_v2(double a, double b) { return D2{a, b}; }

__device__ __forceinline__ float erf_t(float x) { return erff(x); }
__device__ __forceinline__ double erf_t(double x) { return erf(x); }

// erfc(u) and exp(-u^2): libdevice in FP64, A&S 7.1.26 in FP32 (the MODE 0 FP32 path inlines
// the same approximation with paired instructions).
__device__ __forceinline__ void erfc_exp(double u, double &ec, double &ex) {
  ec = erfc(u);
  ex = exp(-u * u);
}
__device__ __forceinline__ void erfc_exp(float u, float &ec, float &ex) { erfc_exp_as(u, ec, ex); }
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
  typename Acc<T>::S *energies;    // per system: [2s] pairs (LJ + erfc Coulomb), [2s+1] exclusion correction
  typename Acc<T>::S *gs = nullptr;  // MODE 1/2: (npad) d/dsigma_i
  typename Acc<T>::S *ga = nullptr;  // MODE 1/2: (npad) d/da_i, a = sqrt(eps)
  const typename V4<T>::type *u = nullptr;  // MODE 2: direction per sorted slot
};

// LB parameters and excluded-partner slots in sorted order. Partner indices are counted
// from the first atom of the atom's own system (batch mode), i.e. global for one system.
// With `dir` (caller order (N,3)) also the direction of a second-derivative pass in
// sorted order.
// With `gx` / `gq` also zeroes the tile kernel's accumulators of each slot (3 + 1 values).
// Also fills the tile kernel's item -> cluster table from the item offsets of the
// neighbour search (the lanes of cluster k write its entries).
template <class T>
__global__ void sorted_params_kernel(ClusterData<T> cl, const T *sigma, const T *eps, const int *excl,
                                     typename V2<T>::type *lj, int *exslot, const T *dir = nullptr,
                                     typename V4<T>::type *dir_sorted = nullptr, typename Acc<T>::S *gx = nullptr,
                                     typename Acc<T>::S *gq = nullptr) {
  pdl_enter();
  const int64_t npad = cl.n_pad();
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < npad; s += (int64_t)gridDim.x * blockDim.x) {
    if (gx) {
      gx[3 * s] = 0;
      gx[3 * s + 1] = 0;
      gx[3 * s + 2] = 0;
      gq[s] = 0;
    }
    {
      const int64_t k = s / kWarp;
      const int o = cl.itemoff[k], nk = cl.itemoff[k + 1] - o;
      for (int j = (int)(s % kWarp); j < nk; j += kWarp) cl.items[o + j] = (int)k;
    }
    const int a = cl.sidx[s];
    if (dir)
      dir_sorted[s] = a >= 0 ? make_v4(dir[3 * (int64_t)a], dir[3 * (int64_t)a + 1], dir[3 * (int64_t)a + 2], T(0))
                             : make_v4(T(0), T(0), T(0), T(0));
    const int64_t base = (cl.sys && a >= 0) ? cl.sys[cl.cl_sys[s / kWarp]].atom_off : 0;
    lj[s] = a >= 0 ? make_v2(T(0.5) * sigma[a], (T)sqrt((double)eps[a])) : make_v2(T(0), T(0));
#pragma unroll
    for (int k = 0; k < kMaxExcl; ++k) {
      const int p = a >= 0 ? excl[(int64_t)a * kMaxExcl + k] : -1;
      exslot[s * kMaxExcl + k] = p >= 0 ? cl.inv[base + p] : -1;
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

// Resident 4-warp blocks per SM the register allocation of the energy kernel must allow
// (6 blocks = 24 warps: at most 80 registers per thread).
constexpr int kTileMinBlocks = 6;

template <class T, int MODE = 0, int MIN_BLOCKS = kTileMinBlocks>
__global__ void __launch_bounds__(TileCfg<T, MODE>::NW * 32, MODE == 0 ? MIN_BLOCKS : 1)
    tile_kernel(TileArgs<T> A) {
  pdl_enter();
  using V = typename V4<T>::type;
  using W2 = typename V2<T>::type;
  constexpr int NW = TileCfg<T, MODE>::NW;
  __shared__ V s_pos[NW][kItemTiles][kWarp];
  __shared__ V s_u[NW][kItemTiles][MODE == 2 ? kWarp : 1];  // MODE 2: direction of the j atoms
  __shared__ W2 s_lj[NW][kItemTiles][kWarp];
  // negated j positions, structure of arrays, for the packed FP32 distance pass
  __shared__ __align__(16) float s_nx[NW][kItemTiles][sizeof(T) == 4 ? kWarp : 4];
  __shared__ __align__(16) float s_ny[NW][kItemTiles][sizeof(T) == 4 ? kWarp : 4];
  __shared__ __align__(16) float s_nz[NW][kItemTiles][sizeof(T) == 4 ? kWarp : 4];
  __shared__ unsigned s_mask[NW][kItemTiles][kWarp];   // in-cutoff, not excluded
  __shared__ unsigned s_xmask[NW][kItemTiles][kWarp];  // in-cutoff, excluded
  __shared__ int s_mi[NW][kItemTiles];                 // 1: tile needs the per-pair minimum image
  __shared__ T s_box[NW][2][9];                         // box and inverse of the warp's current system
  __shared__ T s_rpre2[NW];                             // squared j-atom prefilter radius of that system
  const ClusterData<T> &cl = A.cl;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  T *s_m = s_box[w][0], *s_inv = s_box[w][1];
  int cur_sys = -1;
  bool ortho = false;
  const T rc2 = (T)(A.rc * A.rc);
  const float rc2_up = nextafterf((float)(A.rc * A.rc), INFINITY);  // FP32 pass 1: r2 <= rc2 <=> r2 < rc2_up
  const T alpha = (T)A.alpha;
  const T kc = (T)A.kc;
  const T two_a_rpi = (T)(2.0 * A.alpha / 1.7724538509055160273);

  const int nitems = cl.itemoff[cl.n_clusters()];
  const int nwarps = gridDim.x * NW;
  for (int it = blockIdx.x * NW + w; it < nitems; it += nwarps) {
    const int I = cl.items[it];  // owning cluster: itemoff[I] <= it < itemoff[I + 1]
    const int isys = cl.system_of(I);
    if (isys != cur_sys) {
      const double *info = cl.info(isys);
      if (lane < 9) {
        s_m[lane] = (T)info[lane];
        s_inv[lane] = (T)info[9 + lane];
      }
      ortho = info[18] != 0.0;
      cur_sys = isys;
      if (lane == 0) {
        const T rpre = (T)(A.rc + 1e-3 + 1e-5 * (info[0] + info[4] + info[8]));
        s_rpre2[w] = rpre * rpre;
      }
      __syncwarp();
    }
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
    V ui{};
    if constexpr (MODE == 2) ui = A.u[si];
    // Per-atom shift: every j atom is moved to its image nearest the centre c of cluster I.
    // If h + rc < L/2 on every axis (h: I's half extent), another image of j would be at
    // least L - rc away from an i atom while the chosen one is at most h + L/2 away, so every
    // pair within the cutoff gets its minimum-image displacement and no pair outside the
    // cutoff can appear inside it.
    const bool atom_shift = ortho && (hi_.x + (T)A.rc * s_inv[0] < T(0.499)) &&
                            (hi_.y + (T)A.rc * s_inv[4] < T(0.499)) && (hi_.z + (T)A.rc * s_inv[8] < T(0.499));
    const T cx = ci.x * s_m[0], cy = ci.y * s_m[4], cz = ci.z * s_m[8];

    // Excluded partners of atom i are sorted slots (-1: none), read per tile from two 16-byte
    // loads. Only tiles whose cluster J lies in the warp's range of partner clusters
    // [x_lo, x_hi] (warp-uniform) can hold an excluded pair; the others skip the check.
    const int4 *xs_row = reinterpret_cast<const int4 *>(A.exslot + si * kMaxExcl);
    int x_lo, x_hi;
    {
      const int4 a = xs_row[0], b = xs_row[1];
      const int xs[kMaxExcl] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
      int lo = 0x7fffffff, hi = -1;
#pragma unroll
      for (int x = 0; x < kMaxExcl; ++x)
        if (xs[x] >= 0) {
          lo = min(lo, xs[x] >> 5);
          hi = max(hi, xs[x] >> 5);
        }
      x_lo = __reduce_min_sync(kFull, lo);
      x_hi = __reduce_max_sync(kFull, hi);
    }
    bool all_shifted = true;  // warp-uniform: no tile of the item needs the per-pair minimum image

    // stage the tiles and build their cutoff masks (pass 1)
    for (int t = 0; t < ntile; ++t) {
      const int J = cl.nbr[(int64_t)I * cl.cap + k + t * nch];
      const int64_t sj = (int64_t)J * kWarp + lane;
      // one periodic shift for the whole cluster pair when every pair's displacement then
      // lies within half a box length per axis (orthorhombic boxes)
      bool shifted = false;
      T sx = T(0), sy = T(0), sz = T(0);
      if (ortho && !atom_shift) {
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
      if (atom_shift) {
        pj.x += rint((cx - pj.x) * s_inv[0]) * s_m[0];
        pj.y += rint((cy - pj.y) * s_inv[4]) * s_m[4];
        pj.z += rint((cz - pj.z) * s_inv[8]) * s_m[8];
        shifted = true;
      } else if (shifted) {
        pj.x += sx;
        pj.y += sy;
        pj.z += sz;
      }
      bool keep_j = cl.sidx[sj] >= 0;
      if (shifted && J != I) {
        const T ex_ = fmax(fabs(pj.x - cx) - hi_.x * s_m[0], T(0)), ey_ = fmax(fabs(pj.y - cy) - hi_.y * s_m[4], T(0)),
                ez_ = fmax(fabs(pj.z - cz) - hi_.z * s_m[8], T(0));
        keep_j = keep_j && (ex_ * ex_ + ey_ * ey_ + ez_ * ez_ <= s_rpre2[w]);
      }
      const unsigned keep = __ballot_sync(kFull, keep_j);
      const unsigned lt_mask = lanemask_lt();
      const int nkeep = __popc(keep);
      const int n4 = (nkeep + 3) >> 2;
      if (keep_j) {
        const int slot = __popc(keep & lt_mask);
        s_pos[w][t][slot] = pj;
        s_lj[w][t][slot] = A.lj[sj];
        if constexpr (MODE == 2) s_u[w][t][slot] = A.u[sj];
        if (sizeof(T) == 4) {
          s_nx[w][t][slot] = -(float)pj.x;
          s_ny[w][t][slot] = -(float)pj.y;
          s_nz[w][t][slot] = -(float)pj.z;
        }
      }
      if (sizeof(T) == 4 && lane >= nkeep && lane < 4 * n4) {
        s_nx[w][t][lane] = 1e18f;
        s_ny[w][t][lane] = 1e18f;
        s_nz[w][t][lane] = 1e18f;
      }
      __syncwarp();
      unsigned mask = 0u;
      if (sizeof(T) == 4 && shifted) {
        // four j atoms per shared load, two per paired FP32 instruction (FADD2/FFMA2). The
        // FMA chain starts from -rc2' (rc2' = the float just above rc^2), so its result is
        // negative exactly for the pairs inside the cutoff and the sign bit is the mask bit:
        // a funnel shift appends it (first atom ends in bit 31; reversed once per tile).
        const float2 px = make_float2((float)pi.x, (float)pi.x), py = make_float2((float)pi.y, (float)pi.y),
                     pz = make_float2((float)pi.z, (float)pi.z);
        const float2 nrc2 = make_float2(-rc2_up, -rc2_up);
#pragma unroll
        for (int s = 0; s < kWarp; s += 4) {
          if (s >= 4 * n4) break;
          const float4 nx = *reinterpret_cast<const float4 *>(&s_nx[w][t][s]);
          const float4 ny = *reinterpret_cast<const float4 *>(&s_ny[w][t][s]);
          const float4 nz = *reinterpret_cast<const float4 *>(&s_nz[w][t][s]);
          float2 dx = __fadd2_rn(px, make_float2(nx.x, nx.y)), dy = __fadd2_rn(py, make_float2(ny.x, ny.y)),
                 dz = __fadd2_rn(pz, make_float2(nz.x, nz.y));
          float2 d2 = __ffma2_rn(dx, dx, nrc2);
          d2 = __ffma2_rn(dy, dy, d2);
          d2 = __ffma2_rn(dz, dz, d2);
          mask = __funnelshift_l(__float_as_uint(d2.x), mask, 1);
          mask = __funnelshift_l(__float_as_uint(d2.y), mask, 1);
          dx = __fadd2_rn(px, make_float2(nx.z, nx.w));
          dy = __fadd2_rn(py, make_float2(ny.z, ny.w));
          dz = __fadd2_rn(pz, make_float2(nz.z, nz.w));
          d2 = __ffma2_rn(dx, dx, nrc2);
          d2 = __ffma2_rn(dy, dy, d2);
          d2 = __ffma2_rn(dz, dz, d2);
          mask = __funnelshift_l(__float_as_uint(d2.x), mask, 1);
          mask = __funnelshift_l(__float_as_uint(d2.y), mask, 1);
        }
        mask = n4 > 0 ? __brev(mask) >> (kWarp - 4 * n4) : 0u;
      } else {
#pragma unroll 4
        for (int s = 0; s < nkeep; ++s) {
          const V q = s_pos[w][t][s];
          T dx = pi.x - q.x, dy = pi.y - q.y, dz = pi.z - q.z;
          if (!shifted) pair_min_image(ortho, dx, dy, dz, s_m, s_inv);
          const T r2 = dx * dx + dy * dy + dz * dz;
          mask |= (r2 <= rc2) ? (1u << s) : 0u;
        }
      }
      if (nkeep < kWarp) mask &= (1u << nkeep) - 1u;
      if (J == I) mask &= ~(1u << __popc(keep & lt_mask));
      if (!vi) mask = 0u;
      unsigned emask = 0u;
      if (J >= x_lo && J <= x_hi && mask) {
        const int4 a = xs_row[0], b = xs_row[1];
        const int xs[kMaxExcl] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
        for (int x = 0; x < kMaxExcl; ++x) {
          const int o = xs[x] & 31;
          if ((xs[x] >> 5) == J && ((keep >> o) & 1u)) emask |= 1u << __popc(keep & ((1u << o) - 1u));
        }
      }
      s_mask[w][t][lane] = mask & ~emask;
      s_xmask[w][t][lane] = mask & emask;
      if (lane == 0) s_mi[w][t] = !shifted;
      all_shifted = all_shifted && shifted;
    }
    __syncwarp();

    // pass 2: every lane walks its own in-cutoff pairs across all tiles of the item
    T fx = T(0), fy = T(0), fz = T(0), dq = T(0);
    double ep = 0.0;
    T d_sig = T(0), d_a = T(0);  // MODE 1/2: sigma and sqrt(eps) derivatives of atom i
    if constexpr (MODE == 0 && sizeof(T) == 4) {
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
          if (!all_shifted) {
            if (s_mi[w][ta]) pair_min_image(ortho, dx.x, dy.x, dz.x, s_m, s_inv);
            if (hb && s_mi[w][tb]) pair_min_image(ortho, dx.y, dy.y, dz.y, s_m, s_inv);
          }
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
    } else if constexpr (MODE != 0) {
      // one pair per step. With D = (dE/dr)/r of the pair: MODE 1 adds dE/dsigma_i and
      // dE/da_i; MODE 2 accumulates, with delta = u_i - u_j and rd = r_ij . delta,
      // d/dx_i (u . dE/dx) = D delta + (dD/dr / r) rd r_ij and the parameter derivatives
      // (dD/dp) rd (coordinates: fx..fz, charge: dq (times k later), sigma: d_sig, a: d_a)
      T te = T(0);
      int t = 0, iter = 0;
      unsigned m = ntile > 0 ? s_mask[w][0][lane] : 0u;
      while (true) {
        while (m == 0u && ++t < ntile) m = s_mask[w][t][lane];
        const bool have = m != 0u;
        if (!__any_sync(kFull, have)) break;
        if (MODE == 1 && (++iter & 15) == 0) {
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
          const T sig = lji.x + ljj.x, aj = ljj.y, eps = lji.y * aj;
          const T sr = sig * rinv, sr2 = sr * sr, sr6 = sr2 * sr2 * sr2, sr12 = sr6 * sr6, s5 = sr2 * sr2 * sr;
          const T dcq = -q.w * (ec * rinv2 + two_a_rpi * ex2 * rinv) * rinv;  // D_coulomb / (k q_i)
          const T dlj = T(-24) * eps * (T(2) * sr12 - sr6) * rinv2;           // D_lj
          const T D = kqi * dcq + dlj;
          if constexpr (MODE == 1) {
            fx += D * dx;
            fy += D * dy;
            fz += D * dz;
            dq += q.w * ec * rinv;
            te += kqi * q.w * ec * rinv + T(4) * eps * (sr12 - sr6);
            d_sig += T(12) * eps * rinv * s5 * (T(2) * sr6 - T(1));  // 1/2 dE/dsigma_ij
            d_a += T(4) * aj * (sr12 - sr6);                       // dE/da_i
          } else {
            const V uj = s_u[w][t][s];
            const T ddx = ui.x - uj.x, ddy = ui.y - uj.y, ddz = ui.z - uj.z;
            const T rd = dx * ddx + dy * ddy + dz * ddz;
            const T rinv4 = rinv2 * rinv2;
            const T e2 = kqi * q.w * (T(3) * ec * rinv4 * rinv + two_a_rpi * ex2 * (T(3) * rinv4 + T(2) * alpha * alpha * rinv2)) +
                         T(24) * eps * (T(28) * sr12 - T(8) * sr6) * rinv4;  // (dD/dr) / r
            const T e2rd = e2 * rd;
            fx += D * ddx + e2rd * dx;
            fy += D * ddy + e2rd * dy;
            fz += D * ddz + e2rd * dz;
            dq += dcq * rd;
            d_sig += T(-72) * eps * rinv2 * rinv * s5 * (T(4) * sr6 - T(1)) * rd;  // 1/2 dD/dsigma_ij rd
            d_a += T(-24) * aj * (T(2) * sr12 - sr6) * rinv2 * rd;              // dD/da_i rd
          }
        }
      }
      ep += (double)te;
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
        const T dcq = -q.w * (damp * rinv * rinv + two_a_rpi * ex2 * rinv) * rinv;
        const T dedr_r = kqi * dcq;
        if constexpr (MODE == 2) {
          // same form as the erfc term with erfc(u) -> erfc(u) - 1 (equal derivatives)
          const V uj = s_u[w][t][s];
          const T ddx = ui.x - uj.x, ddy = ui.y - uj.y, ddz = ui.z - uj.z;
          const T rd = dx * ddx + dy * ddy + dz * ddz;
          const T rinv2 = rinv * rinv, rinv4 = rinv2 * rinv2;
          const T e2rd = kqi * q.w * (T(3) * damp * rinv4 * rinv + two_a_rpi * ex2 * (T(3) * rinv4 + T(2) * alpha * alpha * rinv2)) * rd;
          fx += dedr_r * ddx + e2rd * dx;
          fy += dedr_r * ddy + e2rd * dy;
          fz += dedr_r * ddz + e2rd * dz;
          dq += dcq * rd;
        } else {
          fx += dedr_r * dx;
          fy += dedr_r * dy;
          fz += dedr_r * dz;
          dq += cq;
          ex += (double)(kqi * cq);
        }
      }
    }
    if (vi) {
      Acc<T>::add(&A.gx[3 * si], (double)fx);
      Acc<T>::add(&A.gx[3 * si + 1], (double)fy);
      Acc<T>::add(&A.gx[3 * si + 2], (double)fz);
      Acc<T>::add(&A.gq[si], (double)kc * (double)dq);
      if constexpr (MODE != 0) {
        Acc<T>::add(&A.gs[si], (double)d_sig);
        Acc<T>::add(&A.ga[si], (double)d_a);
      }
    }
    // energies: warp sum, then one order-independent accumulation per work item
    ep = warp_sum(ep);
    ex = warp_sum(ex);
    if (MODE != 2 && lane == 0) {
      Acc<T>::add(&A.energies[2 * isys], 0.5 * ep);
      Acc<T>::add(&A.energies[2 * isys + 1], 0.5 * ex);
    }
    __syncwarp();
  }
}

// Sorted real-space accumulators + caller-order PME derivatives -> caller order; energies
// of each of the nsys systems (e_tile_acc and e_pme hold two values per system, terms
// gets four: real-space pairs, exclusion correction, reciprocal, self).
// With `bonded` (one system): its caller-order dE/dx (3N) and the bond and angle energies
// (at 3N, 3N + 1) are added too, and terms gets six values (+ bonds, angles).
template <class T>
__global__ void finalize_kernel(ClusterData<T> cl, const typename Acc<T>::S *gx, const typename Acc<T>::S *gq,
                                const T *pme_grad, const T *pme_phi, T *forces, double *forces64, T *grad_q,
                                const typename Acc<T>::S *e_tile_acc, const double *e_pme, double kc,
                                double *energy, double *terms, int nsys,
                                const typename Acc<T>::S *bonded = nullptr, unsigned *status_out = nullptr) {
  pdl_enter();
  // the build's overflow word (bit 0: a cluster's neighbour list was cut at its capacity),
  // copied out for a host caller that reads it together with the energy
  if (status_out && blockIdx.x == 0 && threadIdx.x == 0) *status_out = cl.status[0];
  const int64_t natoms = cl.n_atoms();
  if (cl.shape) nsys = cl.shape->nsys;
  for (int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; a < natoms;
       a += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = cl.inv[a];
    double x = Acc<T>::get(&gx[3 * s]), y = Acc<T>::get(&gx[3 * s + 1]), z = Acc<T>::get(&gx[3 * s + 2]);
    double g = Acc<T>::get(&gq[s]);
    if (bonded) {
      x += Acc<T>::get(&bonded[3 * a]);
      y += Acc<T>::get(&bonded[3 * a + 1]);
      z += Acc<T>::get(&bonded[3 * a + 2]);
    }
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
  for (int sy = blockIdx.x * blockDim.x + threadIdx.x; sy < nsys; sy += gridDim.x * blockDim.x) {
    const double e_tile[2] = {Acc<T>::get(&e_tile_acc[2 * sy]), Acc<T>::get(&e_tile_acc[2 * sy + 1])};
    const double rec = e_pme ? kc * e_pme[2 * sy] : 0.0;
    const double self = e_pme ? kc * e_pme[2 * sy + 1] : 0.0;
    const double eb = bonded ? Acc<T>::get(&bonded[3 * natoms]) : 0.0;
    const double ea = bonded ? Acc<T>::get(&bonded[3 * natoms + 1]) : 0.0;
    const double tot = e_tile[0] + e_tile[1] + rec + self + eb + ea;
    if (energy) energy[sy] = tot;
    if (terms) {
      const int nt = bonded ? 6 : 4;
      terms[nt * sy] = e_tile[0];
      terms[nt * sy + 1] = e_tile[1];
      terms[nt * sy + 2] = rec;
      terms[nt * sy + 3] = self;
      if (bonded) {
        terms[nt * sy + 4] = eb;
        terms[nt * sy + 5] = ea;
      }
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
inline void host_bspline6_at_integers(double val[6]) {
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

inline std::vector<double> host_moduli(int K, int count) {
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

#include "pair_tile.cuh"

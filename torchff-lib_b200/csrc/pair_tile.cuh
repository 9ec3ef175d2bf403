// FP32 real-space energy + forces over HALF cluster lists (each pair evaluated once).
//
// Work item: cluster I (32 atoms, 4 sub-clusters of 8 consecutive atoms along the Hilbert
// curve) and up to kItemTiles clusters J <= I of its half neighbour list (entries k,
// k + n, ...). Lane l = ti + 8 tj (ti = 0..7, tj = 0..3) owns the i atoms 8c + ti of I's
// four sub-clusters c, in registers. For each J:
//   - J's 32 atoms (moved to the periodic image the pair needs) and parameters are staged
//     in per-warp shared memory;
//   - the 16 sub-tiles (I sub-cluster ci, J sub-cluster cj) are screened by the distance
//     between the two sub-clusters' bounding boxes, computed from the same positions with
//     the same rounding steps as the pair distance, so that a screened-out sub-tile provably
//     holds no pair within the cutoff;
//   - for every J sub-cluster with an active sub-tile, lane (ti, tj) takes the two j atoms
//     8cj + tj and 8cj + tj + 4 as one paired operand (FADD2/FMUL2/FFMA2) against its i
//     atom of each active sub-tile: 64 pairs per sub-tile, each evaluated once; a sub-tile
//     none of whose pairs lies within the cutoff is skipped after the distances (warp vote);
//   - the j-side force and charge-gradient sums of the two j atoms are reduce-scattered
//     over the 8 lanes that hold them (warp shuffles), and each of those lanes adds one of
//     the 8 sums into the int64 fixed-point accumulators.
// The i-side sums stay in registers for the whole item and are reduce-scattered over the 4
// lanes of each i atom at its end. Pairs within one cluster (J == I) count j < i; excluded
// pairs are skipped through a per-J bit mask of each i atom's excluded partners, and their
// Ewald exclusion correction -k q_i q_j erf(alpha r)/r (r <= rc) is evaluated in FP64 once
// per excluded pair, by item 0 of the cluster that holds the pair's later slot.
// Integer accumulation is order-independent, so results are bit-identical run to run;
// energies are summed per lane in a fixed order and added once per item.
#pragma once

namespace tff {
namespace {

// Paired arithmetic on two values: FP32 pairs map onto the packed FP32 instructions of
// sm_100a (FP64 pairs, two scalar operations, keep the helpers generic).
template <class T> struct P2T;
template <> struct P2T<float> { using type = float2; };
template <> struct P2T<double> { using type = D2; };

__device__ __forceinline__ float2 p_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 p_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 p_fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 p_splat(float a) { return make_float2(a, a); }
__device__ __forceinline__ D2 p_add(D2 a, D2 b) { return D2{a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ D2 p_mul(D2 a, D2 b) { return D2{a.x * b.x, a.y * b.y}; }
__device__ __forceinline__ D2 p_fma(D2 a, D2 b, D2 c) { return D2{fma(a.x, b.x, c.x), fma(a.y, b.y, c.y)}; }
__device__ __forceinline__ D2 p_splat(double a) { return D2{a, a}; }

// Per-warp staging, laid out as the paired operands the arithmetic takes, so that one
// 16-byte shared load gives two of them:
// - cluster J (moved to the pair's image; padding slots far away): jp[w][k][4 cj + tj]
//   holds the two j atoms j0 = 8 cj + tj and j1 = j0 + 4 of lane column tj,
//   k = 0: (-x0, -x1, -y0, -y1), 1: (-z0, -z1, q0, q1), 2: (s0, s1, e0, e1), with s = sigma/2
//   and e = sqrt(eps);
// - cluster I (padding far the other way), each value doubled: ip[w][k][atom],
//   k = 0: (x, x, y, y), 1: (z, z, q, q), 2: (s, s, e, e), 3: (kq, kq, -kq, -kq);
// - I's four sub-cluster boxes (lo xyz, hi xyz).
// Entries are indexed by atom (I) or lane column (J) innermost, so the 8 (4) distinct
// entries a warp reads at once are contiguous: one shared-memory wavefront.
template <class T, int NW>
struct PairTileSmem {
  typename V4<T>::type jp[NW][3][16];
  typename V4<T>::type ip[NW][4][kWarp];
  T ibox[NW][4][6];
};

// j-side sums of the two j atoms of a lane (paired): dE/dr / r * (r_i - r_j) summed over
// the lane's i atoms (the j force is its negative) and the k-free charge gradient.
template <class T> struct JSums { typename P2T<T>::type fx, fy, fz, dq; };

// Squared distances of two pairs: dx^2, then + dy^2, then + dz^2 by fused multiply-adds
// (the order box_gap2 repeats).
template <class P2>
__device__ __forceinline__ P2 pair2_r2(P2 dx, P2 dy, P2 dz) {
  P2 r2 = p_mul(dx, dx);
  r2 = p_fma(dy, dy, r2);
  return p_fma(dz, dz, r2);
}

// Constants of the pair arithmetic, doubled for the paired instructions and passed as a
// kernel parameter (constant memory) instead of being rebuilt in registers per use.
// erfc(x) exp(x^2) ~ t (a1 + t (a2 + t (a3 + t (a4 + t a5)))), t = 1 / (1 + p x): Abramowitz &
// Stegun 7.1.26, |error| <= 1.5e-7.
template <class T>
struct PairConst {
  using P2 = typename P2T<T>::type;
  P2 one, a1, a2, a3, a4, a5;
  P2 lj_f1, lj_f0;  // -48, 24: (dE/dr) / r of LJ = eps_ij (sr6) (24 - 48 sr6) / r^2
  P2 lj_e1, lj_e0;  // 4, -4: E of LJ = eps_ij (sr6) (4 sr6 - 4)
  P2 alpha_p;       // alpha p
  P2 nalpha2_log2e; // -alpha^2 log2(e): exp(-(alpha r)^2) = 2^(r^2 (-alpha^2 log2 e))
  P2 two_a_rpi;     // 2 alpha / sqrt(pi)
  T alpha;
};

template <class T>
PairConst<T> pair_const(double alpha) {
  using P2 = typename P2T<T>::type;
  auto d = [](double v) { return P2{(T)v, (T)v}; };
  PairConst<T> c;
  c.one = d(1.0);
  c.a1 = d(0.254829592);
  c.a2 = d(-0.284496736);
  c.a3 = d(1.421413741);
  c.a4 = d(-1.453152027);
  c.a5 = d(1.061405429);
  c.lj_f1 = d(-48.0);
  c.lj_f0 = d(24.0);
  c.lj_e1 = d(4.0);
  c.lj_e0 = d(-4.0);
  c.alpha_p = d(alpha * 0.3275911);
  c.nalpha2_log2e = d(-alpha * alpha * 1.4426950408889634074);
  c.two_a_rpi = d(2.0 * alpha / 1.7724538509055160273);
  c.alpha = (T)alpha;
  return c;
}

__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Two pairs (i; j0, j1): LJ + erfc-screened Coulomb. dx, dy, dz = r_i - r_j (paired), r2
// from pair2_r2; in0 / in1: the pair contributes (valid, not excluded, counted by this
// side, r2 <= rc2). Charge gradients are accumulated k-free (times k when added).
// The i-side operands come doubled: qi2 = (q_i, q_i), kqi2 = k q_i, nkqi2 = -k q_i, sgi2, epi2.
__device__ __forceinline__ void pair2_eval(float2 dx, float2 dy, float2 dz, float2 r2, bool in0, bool in1, float2 qi2,
                                           float2 kqi2, float2 nkqi2, float2 sgi2, float2 epi2, float2 qj,
                                           float2 sgj, float2 epj, const PairConst<float> &pc, float &fxi,
                                           float &fyi, float &fzi, float &dqi, JSums<float> &js, float2 &te) {
  // pairs outside the cutoff (or masked) get rinv = 0, which zeroes every term below
  const float2 rinv = make_float2(in0 ? rsqrtf(r2.x) : 0.f, in1 ? rsqrtf(r2.y) : 0.f);
  const float2 rinv2 = p_mul(rinv, rinv);
  const float2 r = p_mul(r2, rinv);
  const float2 den = p_fma(r, pc.alpha_p, pc.one);  // 1 + p alpha r
  const float2 tt = make_float2(rcp_approx(den.x), rcp_approx(den.y));
  float2 poly = p_fma(tt, pc.a5, pc.a4);
  poly = p_fma(tt, poly, pc.a3);
  poly = p_fma(tt, poly, pc.a2);
  poly = p_fma(tt, poly, pc.a1);
  poly = p_mul(tt, poly);
  const float2 xa = p_mul(r2, pc.nalpha2_log2e);
  const float2 ex = make_float2(ex2_approx(xa.x), ex2_approx(xa.y));  // exp(-(alpha r)^2)
  const float2 ec = p_mul(poly, ex);   // erfc(alpha r)
  const float2 ecr = p_mul(ec, rinv);  // erfc(alpha r) / r
  const float2 cq = p_mul(qj, ecr);    // E_coul / (k q_i)
  // (dE/dr) / r of the Coulomb term: -k q_i q_j (erfc(alpha r)/r + 2 alpha/sqrt(pi) exp(-(alpha r)^2)) / r^2
  float2 dedr = p_mul(p_mul(p_fma(pc.two_a_rpi, ex, ecr), rinv2), p_mul(qj, nkqi2));
  const float2 sig = p_add(sgi2, sgj);
  const float2 eps = p_mul(epi2, epj);
  const float2 sr2 = p_mul(p_mul(sig, sig), rinv2);
  const float2 sr6 = p_mul(p_mul(sr2, sr2), sr2);
  const float2 es6 = p_mul(eps, sr6);
  dedr = p_fma(p_mul(es6, p_fma(sr6, pc.lj_f1, pc.lj_f0)), rinv2, dedr);
  fxi = fmaf(dedr.x, dx.x, fmaf(dedr.y, dx.y, fxi));
  fyi = fmaf(dedr.x, dy.x, fmaf(dedr.y, dy.y, fyi));
  fzi = fmaf(dedr.x, dz.x, fmaf(dedr.y, dz.y, fzi));
  dqi += cq.x + cq.y;
  js.fx = p_fma(dedr, dx, js.fx);
  js.fy = p_fma(dedr, dy, js.fy);
  js.fz = p_fma(dedr, dz, js.fz);
  js.dq = p_fma(qi2, ecr, js.dq);
  te = p_fma(cq, kqi2, te);
  te = p_fma(es6, p_fma(sr6, pc.lj_e1, pc.lj_e0), te);
}

// Bounding box of each lane's 8-lane group (lanes 8c .. 8c+7 hold sub-cluster c), over
// valid atoms only; lo > hi for a group without any.
template <class T>
__device__ __forceinline__ void subcluster_box(bool valid, T x, T y, T z, T lo[3], T hi[3]) {
  const T big = sizeof(T) == 4 ? T(3e37) : T(1e300);
  lo[0] = valid ? x : big;
  lo[1] = valid ? y : big;
  lo[2] = valid ? z : big;
  hi[0] = valid ? x : -big;
  hi[1] = valid ? y : -big;
  hi[2] = valid ? z : -big;
#pragma unroll
  for (int o = 1; o < 8; o <<= 1) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      lo[k] = min(lo[k], __shfl_xor_sync(kFull, lo[k], o));
      hi[k] = max(hi[k], __shfl_xor_sync(kFull, hi[k], o));
    }
  }
}

// Squared gap between two boxes with the rounding steps of the pair distance: per axis
// the difference of two coordinates (monotone in each), then x^2, fma y, fma z (monotone in
// each magnitude), so every pair of atoms of the two boxes has r2 >= the result. Empty
// boxes (lo > hi) give a huge gap.
template <class T>
__device__ __forceinline__ T box_gap2(const T alo[3], const T ahi[3], const T blo[3], const T bhi[3]) {
  T g[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) g[k] = max(T(0), max(blo[k] - ahi[k], alo[k] - bhi[k]));
  T r = g[0] * g[0];
  r = fma(g[1], g[1], r);
  r = fma(g[2], g[2], r);
  return r;
}

// One halving step of a reduce-scatter over lanes that differ in lane bit `o`: a lane with
// that bit set keeps the upper half of v[0, n), the other the lower half, each adding the
// partner's copy of the half it keeps (stored in v[0, n/2)).
template <class T, int N, int n>
__device__ __forceinline__ void rs_halve(T (&v)[N], int o, int lane) {
  const bool up = (lane & o) != 0;
#pragma unroll
  for (int q = 0; q < n / 2; ++q) {
    const T keep = up ? v[q + n / 2] : v[q];
    const T send = up ? v[q] : v[q + n / 2];
    v[q] = keep + __shfl_xor_sync(kFull, send, o);
  }
}

// Warps per block, and resident blocks per SM the register allocation must allow: 4 (at
// most 128 registers, no spills). At 5 (96 registers) the kernel spilled 60 bytes inside its
// loops and ran 1.36 against 1.18 ms at 300,000 atoms (63 against 62 us at 9000).
constexpr int kPairTileWarps = 4;
template <class T> struct PairTileOcc { static constexpr int min_blocks = sizeof(T) == 4 ? 4 : 3; };

// FP32 only: FP64 real space runs on full lists and tile_kernel (see launch_real_space).
template <class T, int NW, int MIN_BLOCKS>
__global__ void __launch_bounds__(NW * 32, MIN_BLOCKS) pair_tile_kernel(TileArgs<T> A, PairConst<T> pc) {
  static_assert(sizeof(T) == 4, "the pair kernel is the FP32 real-space kernel");
  pdl_enter();
  using V = typename V4<T>::type;
  using W2 = typename V2<T>::type;
  using P2 = typename P2T<T>::type;
  __shared__ PairTileSmem<T, NW> sm;
  __shared__ T s_box[NW][2][9];  // box and inverse of the warp's current system
  const ClusterData<T> &cl = A.cl;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int ti = lane & 7, tj = lane >> 3;
  T *s_m = s_box[w][0], *s_inv = s_box[w][1];
  int cur_sys = -1;
  bool ortho = false;
  const T rc2 = (T)(A.rc * A.rc);
  const T kc = (T)A.kc;
  const T far = sizeof(T) == 4 ? T(1e18) : T(1e150);  // padding slots: outside every cutoff

  const int nitems = cl.itemoff[cl.n_clusters()];
  const int nwarps = gridDim.x * NW;
  for (int it = blockIdx.x * NW + w; it < nitems; it += nwarps) {
    const int I = cl.items[it];  // owning cluster: itemoff[I] <= it < itemoff[I + 1]
    const int isys = cl.system_of(I);
    const double *info = cl.info(isys);
    if (isys != cur_sys) {
      __syncwarp();
      if (lane < 9) {
        s_m[lane] = (T)info[lane];
        s_inv[lane] = (T)info[9 + lane];
      }
      ortho = info[18] != 0.0;
      cur_sys = isys;
      __syncwarp();
    }
    const int k = it - cl.itemoff[I];
    const int nch = cl.itemoff[I + 1] - cl.itemoff[I];
    const int cnt = cl.ncount[I];
    const int ntile = (cnt - k + nch - 1) / nch;  // this item takes list entries k, k+nch, ...
    const int64_t sI = (int64_t)I * kWarp;

    // lane-as-atom view of I: staging (padding slots far away, never counted), sub-cluster
    // boxes and the excluded-partner row. The lane's own i atoms are 8c + ti, c = 0..3.
    const int64_t sl = sI + lane;
    const bool vl = cl.sidx[sl] >= 0;
    const unsigned ivalid = __ballot_sync(kFull, vl);
    {
      V p = cl.pos[sl];
      T lo[3], hi[3];
      subcluster_box<T>(vl, p.x, p.y, p.z, lo, hi);
      if (!vl) p.x = p.y = p.z = -far;
      const W2 l = A.lj[sl];
      const T kq = kc * p.w;
      __syncwarp();  // every lane is done with the previous item's staging
      sm.ip[w][0][lane] = make_v4(p.x, p.x, p.y, p.y);
      sm.ip[w][1][lane] = make_v4(p.z, p.z, p.w, p.w);
      sm.ip[w][2][lane] = make_v4(l.x, l.x, l.y, l.y);
      sm.ip[w][3][lane] = make_v4(kq, kq, -kq, -kq);
      if (ti == 0) {
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          sm.ibox[w][tj][q] = lo[q];
          sm.ibox[w][tj][3 + q] = hi[q];
        }
      }
    }
    const V ci = cl.bc[I], hi_ = cl.bh[I];
    // every j atom moved to its image nearest I's centre is the minimum image of every
    // in-cutoff pair when I's half extent + rc < L/2 on each axis (orthorhombic boxes)
    const bool atom_shift = ortho && (hi_.x + (T)A.rc * s_inv[0] < T(0.499)) &&
                            (hi_.y + (T)A.rc * s_inv[4] < T(0.499)) && (hi_.z + (T)A.rc * s_inv[8] < T(0.499));
    const T cx = ci.x * s_m[0], cy = ci.y * s_m[4], cz = ci.z * s_m[8];
    const int4 *xs_row = reinterpret_cast<const int4 *>(A.exslot + sl * kMaxExcl);
    int x_lo, x_hi;  // the warp's range of clusters holding an excluded partner
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

    T fx[4] = {T(0), T(0), T(0), T(0)}, fy[4] = {T(0), T(0), T(0), T(0)}, fz[4] = {T(0), T(0), T(0), T(0)};
    T dq[4] = {T(0), T(0), T(0), T(0)};
    double ep = 0.0;

    // J's list entry, position, LJ parameters and slot are loaded one J ahead, so that their
    // global loads overlap the previous J's arithmetic
    int Jn = 0, sidn = -1;
    V pjn{};
    W2 ljn{};
    if (ntile > 0) {
      Jn = cl.nbr[(int64_t)I * cl.cap + k];
      sidn = cl.sidx[(int64_t)Jn * kWarp + lane];
      pjn = cl.pos[(int64_t)Jn * kWarp + lane];
      ljn = A.lj[(int64_t)Jn * kWarp + lane];
    }
    for (int t = 0; t < ntile; ++t) {
      const int J = Jn;
      const int64_t sJ = (int64_t)J * kWarp;
      const bool vj = sidn >= 0;
      V pj = pjn;
      const W2 lj = ljn;
      if (t + 1 < ntile) {
        Jn = cl.nbr[(int64_t)I * cl.cap + k + (t + 1) * nch];
        sidn = cl.sidx[(int64_t)Jn * kWarp + lane];
        pjn = cl.pos[(int64_t)Jn * kWarp + lane];
        ljn = A.lj[(int64_t)Jn * kWarp + lane];
      }
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
      if (!vj) {
        pj.x = far;
        pj.y = far;
        pj.z = far;
        pj.w = T(0);
      }
      const unsigned jvalid = __ballot_sync(kFull, vj);
      __syncwarp();  // every lane is done with the previous J's staging
      {
        // atom lane = 8 cj + tj + 4 h goes to entry 4 cj + tj, slot h of each pair
        T *e0 = reinterpret_cast<T *>(&sm.jp[w][0][4 * (lane >> 3) + (lane & 3)]) + ((lane >> 2) & 1);
        T *e1 = reinterpret_cast<T *>(&sm.jp[w][1][4 * (lane >> 3) + (lane & 3)]) + ((lane >> 2) & 1);
        T *e2 = reinterpret_cast<T *>(&sm.jp[w][2][4 * (lane >> 3) + (lane & 3)]) + ((lane >> 2) & 1);
        e0[0] = -pj.x;
        e0[2] = -pj.y;
        e1[0] = -pj.z;
        e1[2] = pj.w;
        e2[0] = lj.x;
        e2[2] = lj.y;
      }
      // active sub-tiles: bit ci + 4 cj. Without a common shift every sub-tile is taken.
      unsigned act = 0xffffu;
      if (shifted) {
        T jlo[3], jhi[3];
        subcluster_box<T>(vj, pj.x, pj.y, pj.z, jlo, jhi);
        const int a = (lane & 3) * 8, b = ((lane >> 2) & 3) * 8;
        T alo[3], ahi[3], blo[3], bhi[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          alo[q] = sm.ibox[w][a >> 3][q];
          ahi[q] = sm.ibox[w][a >> 3][3 + q];
          blo[q] = __shfl_sync(kFull, jlo[q], b);
          bhi[q] = __shfl_sync(kFull, jhi[q], b);
        }
        act = __ballot_sync(kFull, lane < 16 && box_gap2<T>(alo, ahi, blo, bhi) <= rc2) & 0xffffu;
      }
      // pairs inside one cluster: j < i, i.e. only sub-tiles cj <= ci (per pair when equal)
      const bool diag = J == I;
      if (diag) act &= 0x8cefu;
      // excluded-partner masks of this lane's i atoms over J's slots (bit = j index in J)
      const bool special = diag || (J >= x_lo && J <= x_hi);
      unsigned xm[4] = {0u, 0u, 0u, 0u};
      if (special) {
        const int4 a = xs_row[0], b = xs_row[1];
        const int xs[kMaxExcl] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
        unsigned m = 0u;
#pragma unroll
        for (int x = 0; x < kMaxExcl; ++x)
          if (xs[x] >= 0 && (xs[x] >> 5) == J) m |= 1u << (xs[x] & 31);
#pragma unroll
        for (int c = 0; c < 4; ++c) xm[c] = __shfl_sync(kFull, m, 8 * c + ti);
      }
      __syncwarp();
      P2 te = p_splat(T(0));
#pragma unroll 1
      for (int cj = 0; cj < 4; ++cj) {
        const unsigned col = (act >> (4 * cj)) & 0xfu;  // i sub-clusters active against cj
        if (!col) continue;
        const int j0 = 8 * cj + tj, j1 = j0 + 4;
        const V ja = sm.jp[w][0][4 * cj + tj], jb = sm.jp[w][1][4 * cj + tj], jc = sm.jp[w][2][4 * cj + tj];
        const P2 nxj = P2{ja.x, ja.y}, nyj = P2{ja.z, ja.w}, nzj = P2{jb.x, jb.y};
        const P2 qj = P2{jb.z, jb.w}, sgj = P2{jc.x, jc.y}, epj = P2{jc.z, jc.w};
        const bool vj0 = (jvalid >> j0) & 1u, vj1 = (jvalid >> j1) & 1u;
        JSums<T> js;
        js.fx = js.fy = js.fz = js.dq = p_splat(T(0));
        bool hit = false;  // some sub-tile of cj holds a pair within the cutoff (warp-uniform)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          if (!((col >> c) & 1u)) continue;
          const V ia = sm.ip[w][0][8 * c + ti], ib = sm.ip[w][1][8 * c + ti];
          P2 dx = p_add(P2{ia.x, ia.y}, nxj);
          P2 dy = p_add(P2{ia.z, ia.w}, nyj);
          P2 dz = p_add(P2{ib.x, ib.y}, nzj);
          // with a common shift, padding atoms (I's far one way, J's far the other) lie
          // outside every cutoff
          bool ok0 = true, ok1 = true;
          if (!shifted) {
            // per-pair minimum image; padding atoms must be masked here (their far positions
            // do not survive the wrap)
            pair_min_image(ortho, dx.x, dy.x, dz.x, s_m, s_inv);
            pair_min_image(ortho, dx.y, dy.y, dz.y, s_m, s_inv);
            const bool vi = (ivalid >> (8 * c + ti)) & 1u;
            ok0 = vi && vj0;
            ok1 = vi && vj1;
          }
          if (special) {
            const int il = 8 * c + ti;
            ok0 = ok0 && !((xm[c] >> j0) & 1u) && (!diag || j0 < il);
            ok1 = ok1 && !((xm[c] >> j1) & 1u) && (!diag || j1 < il);
          }
          const P2 r2 = pair2_r2(dx, dy, dz);
          const bool in0 = ok0 && r2.x <= rc2, in1 = ok1 && r2.y <= rc2;
          // a quarter of the screened-in sub-tiles hold no pair within the cutoff (3000-water
          // box): the warp skips their arithmetic together
          if (!__any_sync(kFull, in0 || in1)) continue;
          hit = true;
          const V ic = sm.ip[w][2][8 * c + ti], id = sm.ip[w][3][8 * c + ti];
          pair2_eval(dx, dy, dz, r2, in0, in1, P2{ib.z, ib.w}, P2{id.x, id.y}, P2{id.z, id.w}, P2{ic.x, ic.y},
                     P2{ic.z, ic.w}, qj, sgj, epj, pc, fx[c], fy[c], fz[c], dq[c], js, te);
        }
        if (!hit) continue;  // nothing to add for cj (a sixth of the screened-in cj at 3000 waters)
        // j side (dE/dx_j = -sum over i of (dE/dr)/r (r_i - r_j)): reduce-scatter over the 8
        // lanes ti that hold j0, j1; lane ti ends with value ti (j0: x y z q, j1: x y z q)
        T v[8] = {-js.fx.x, -js.fy.x, -js.fz.x, js.dq.x, -js.fx.y, -js.fy.y, -js.fz.y, js.dq.y};
        rs_halve<T, 8, 8>(v, 4, lane);
        rs_halve<T, 8, 4>(v, 2, lane);
        rs_halve<T, 8, 2>(v, 1, lane);
        const int64_t sj = sJ + (ti < 4 ? j0 : j1);
        const int comp = ti & 3;
        if ((jvalid >> (ti < 4 ? j0 : j1)) & 1u) {
          if (comp < 3)
            Acc<T>::add(&A.gx[3 * sj + comp], (double)v[0]);
          else
            Acc<T>::add(&A.gq[sj], (double)A.kc * (double)v[0]);
        }
      }
      ep += (double)te.x + (double)te.y;
    }
    // i side: reduce-scatter over the 4 lanes tj of each i atom; lane tj ends with the four
    // sums (x, y, z, q) of its atom c = tj
    {
      T v[16];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        v[4 * c] = fx[c];
        v[4 * c + 1] = fy[c];
        v[4 * c + 2] = fz[c];
        v[4 * c + 3] = dq[c];
      }
      rs_halve<T, 16, 16>(v, 16, lane);
      rs_halve<T, 16, 8>(v, 8, lane);
      if (vl) {  // atom 8 tj + ti is this lane's own slot sl
        Acc<T>::add(&A.gx[3 * sl], (double)v[0]);
        Acc<T>::add(&A.gx[3 * sl + 1], (double)v[1]);
        Acc<T>::add(&A.gx[3 * sl + 2], (double)v[2]);
        Acc<T>::add(&A.gq[sl], (double)A.kc * (double)v[3]);
      }
    }
    ep = warp_sum(ep);

    // Ewald exclusion correction, FP64, once per excluded pair (by the later slot's cluster,
    // item 0): -k q_i q_p erf(alpha r)/r for r <= rc, minimum image of the box
    double ex = 0.0;
    if (k == 0) {
      const double *m = info, *inv = info + 9;
      const double kcd = A.kc, ad = A.alpha, ta = 2.0 * A.alpha / 1.7724538509055160273;
      const int4 a = xs_row[0], b = xs_row[1];
      const int xs[kMaxExcl] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
      const V pl = cl.pos[sl];
#pragma unroll 1
      for (int x = 0; x < kMaxExcl; ++x) {
        const int p = xs[x];
        if (!vl || p < 0 || p >= sl) continue;
        const V pp = cl.pos[p];
        double dx = (double)pl.x - (double)pp.x, dy = (double)pl.y - (double)pp.y, dz = (double)pl.z - (double)pp.z;
        min_image(dx, dy, dz, m, inv);
        const double r2 = dx * dx + dy * dy + dz * dz;
        if (!(r2 <= A.rc * A.rc) || r2 == 0.0) continue;
        const double rinv = rsqrt(r2), r = r2 * rinv;
        const double damp = -erf(ad * r);
        const double e2 = exp(-ad * ad * r2);
        const double kq = kcd * (double)pl.w * (double)pp.w;
        const double dedr = -kq * (damp * rinv * rinv + ta * e2 * rinv) * rinv;
        ex += kq * damp * rinv;
        Acc<T>::add(&A.gx[3 * sl], dedr * dx);
        Acc<T>::add(&A.gx[3 * sl + 1], dedr * dy);
        Acc<T>::add(&A.gx[3 * sl + 2], dedr * dz);
        Acc<T>::add(&A.gx[3 * (int64_t)p], -dedr * dx);
        Acc<T>::add(&A.gx[3 * (int64_t)p + 1], -dedr * dy);
        Acc<T>::add(&A.gx[3 * (int64_t)p + 2], -dedr * dz);
        Acc<T>::add(&A.gq[sl], kcd * (double)pp.w * damp * rinv);
        Acc<T>::add(&A.gq[p], kcd * (double)pl.w * damp * rinv);
      }
      ex = warp_sum(ex);
    }
    if (lane == 0) {
      Acc<T>::add(&A.energies[2 * isys], ep);
      if (k == 0) Acc<T>::add(&A.energies[2 * isys + 1], ex);
    }
  }
}

// Real-space energy kernel per precision. FP32: half cluster lists (J <= I) and the pair
// kernel above, each pair evaluated once. FP64: full lists and tile_kernel, each pair
// evaluated from both sides with every sum in registers: there the j-side FP64 global
// atomics of the pair kernel cost more than the second evaluation they replace
// (3000 waters: 2,476 against 4,922 evaluations per second).
template <class T> constexpr int kHalfLists = sizeof(T) == 4 ? 1 : 0;

// Launches the real-space kernel of precision T on the work items of a cluster build made
// with kHalfLists<T>; the grid covers the largest possible item count (max_items), capped
// at a few waves of the SMs.
template <class T>
int launch_real_space(bool pdl, int64_t max_items, int sms, cudaStream_t s, const TileArgs<T> &A) {
  if constexpr (sizeof(T) == 4) {
    constexpr int NW = kPairTileWarps;
    const int nbt = (int)std::max<int64_t>(1, std::min<int64_t>((max_items + NW - 1) / NW, (int64_t)sms * 48 / NW));
    return launch_k(pdl, pair_tile_kernel<T, NW, PairTileOcc<T>::min_blocks>, nbt, NW * kWarp, 0, s, A,
                    pair_const<T>(A.alpha));
  } else {
    constexpr int NW = TileCfg<T>::NW;
    const int nbt = (int)std::max<int64_t>(1, std::min<int64_t>((max_items + NW - 1) / NW, (int64_t)sms * 48 / NW));
    return launch_k(pdl, tile_kernel<T, 0>, nbt, NW * kWarp, 0, s, A);
  }
}

}  // namespace
}  // namespace tff

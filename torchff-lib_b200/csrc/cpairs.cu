// Cluster-pair neighbour format as first-class operators: the kernels behind
// build_cluster_pairs, decode_cluster_pairs and
// compute_nonbonded_{energy,forces}_from_cluster_pairs (interface of torchff/nblist.py:260-344,
// csrc/nblist/nblist_cluster_pairs_cuda.cu:303-716 and the schemas left commented out in
// csrc/nonbonded/nonbonded_interface.cpp:5-8).
//
// Format (int32 unless noted; built from the Hilbert-ordered 32-atom clusters of cluster.cuh):
//   sorted_atoms   (nclusters * 32)     atom at each slot; -1 in the padding after the last atom
//   tiles          (2, tiles_cap)       cluster pairs (x, y), x <= y, whose 32x32 tile holds an
//                                       excluded atom pair, plus every diagonal tile (x, x); -1 padded
//   tile_masks     (tiles_cap, 32) u32  row (t, lane i): bit j set = the pair (slot 32x+i,
//                                       slot 32y+j) is skipped: excluded, padding, or j <= i on
//                                       a diagonal tile
//   entry_cluster  (entries_cap)        cluster x of each interacting entry; -1 padded
//   entry_atoms    (entries_cap, 32)    atoms of lower clusters that may interact with x (within
//                                       the cutoff of x's bounding box); -1 padded
// Every unordered atom pair within the cutoff that is not excluded lies in exactly one tile or
// entry: same-cluster pairs in the diagonal tile, pairs of clusters A < B that hold an
// exclusion in tile (A, B), all others in B's entries (B scans its half neighbour list, J < B).
#include <climits>

#include "cluster.cuh"

namespace tff {
namespace {

// Distinct clusters of excluded partners per cluster (tile-format limit).
constexpr int kMaxExclClusters = 64;
constexpr int kCpBlock = 128;
constexpr int kCpWarps = kCpBlock / kWarp;

struct CpLayout {
  ClusterLayout cl;
  size_t exset, exn, tcount, ecount, cstat, bytes;
};

inline CpLayout cp_layout(int dtype, int64_t natoms, int cap) {
  CpLayout L;
  L.cl = cluster_layout(dtype, natoms, cap);
  Carver c(nullptr);
  c.off = L.cl.bytes;
  L.exset = (c.off + 255) & ~size_t(255); c.take<int>((size_t)L.cl.nclusters * kMaxExclClusters);
  L.exn = (c.off + 255) & ~size_t(255); c.take<int>(L.cl.nclusters);
  L.tcount = (c.off + 255) & ~size_t(255); c.take<unsigned>(L.cl.nclusters + 1);
  L.ecount = (c.off + 255) & ~size_t(255); c.take<unsigned>(L.cl.nclusters + 1);
  L.cstat = (c.off + 255) & ~size_t(255); c.take<unsigned>(4);
  L.bytes = c.bytes();
  return L;
}

__device__ __forceinline__ int warp_min_int(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(kFull, v, o));
  return v;
}

// One warp per cluster x: the ascending distinct clusters of the excluded partners of its
// atoms (either side of x, x itself included when an atom excludes itself or a neighbour
// in x). cstat[0] |= 1 when a cluster has more than kMaxExclClusters of them.
template <class T>
__global__ void __launch_bounds__(kCpBlock) excl_clusters_kernel(ClusterData<T> d, const int64_t *row_ptr,
                                                                 const int64_t *col, int *exset, int *exn,
                                                                 unsigned *cstat) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * kCpWarps;
  for (int64_t x = (int64_t)blockIdx.x * kCpWarps + (threadIdx.x >> 5); x < d.nclusters; x += nw) {
    const int a = d.sidx[x * kWarp + lane];
    int64_t b = 0, e = 0;
    if (a >= 0 && row_ptr) {
      b = row_ptr[a];
      e = row_ptr[a + 1];
    }
    int last = -1, n = 0;
    while (true) {
      int best = INT_MAX;
      for (int64_t p = b; p < e; ++p) {
        const int y = d.inv[col[p]] >> 5;
        if (y > last && y < best) best = y;
      }
      best = warp_min_int(best);
      if (best == INT_MAX) break;
      if (lane == 0 && n < kMaxExclClusters) exset[x * kMaxExclClusters + n] = best;
      ++n;
      last = best;
    }
    if (lane == 0) {
      exn[x] = min(n, kMaxExclClusters);
      if (n > kMaxExclClusters) atomicOr(&cstat[0], 1u);
    }
  }
}

// Per cluster x (one warp): the tiles (x, y), y in {x} u {exclusion clusters > x}, and the
// interacting entries: atoms of the half-list clusters J < x that are not exclusion clusters
// of x and lie within the cutoff of x's box, compacted 32 to an entry. COUNT mode stores the
// numbers in tcount / ecount; write mode writes them at the scanned offsets (below caps).
template <class T, bool COUNT>
__global__ void __launch_bounds__(kCpBlock) cp_emit_kernel(ClusterData<T> d, double rc, const int64_t *row_ptr,
                                                           const int64_t *col, const int *exset, const int *exn,
                                                           unsigned *tcount, unsigned *ecount, int32_t *tiles,
                                                           int64_t tiles_cap, uint32_t *tile_masks,
                                                           int32_t *entry_cluster, int32_t *entry_atoms,
                                                           int64_t entries_cap) {
  __shared__ int s_buf[kCpWarps][2 * kWarp];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const double *info = d.info(0);
  const int64_t nw = (int64_t)gridDim.x * kCpWarps;
  for (int64_t x = (int64_t)blockIdx.x * kCpWarps + w; x < d.nclusters; x += nw) {
    const int ne = exn[x];
    const int ex0 = lane < ne ? exset[x * kMaxExclClusters + lane] : -1;
    const int ex1 = lane + kWarp < ne ? exset[x * kMaxExclClusters + kWarp + lane] : -1;
    // tiles: the diagonal, then the exclusion clusters above x (a suffix of the sorted set)
    const int nbelow = __popc(__ballot_sync(kFull, ex0 >= 0 && ex0 <= x)) +
                       __popc(__ballot_sync(kFull, ex1 >= 0 && ex1 <= x));
    const int ntile = 1 + ne - nbelow;
    if (COUNT) {
      if (lane == 0) tcount[x] = (unsigned)ntile;
    } else {
      const int64_t t0 = tcount[x];
      const int a = d.sidx[x * kWarp + lane];
      int64_t b = 0, e = 0;
      if (a >= 0 && row_ptr) {
        b = row_ptr[a];
        e = row_ptr[a + 1];
      }
      for (int k = 0; k < ntile; ++k) {
        const int64_t t = t0 + k;
        if (t >= tiles_cap) break;
        const int y = k == 0 ? (int)x : exset[x * kMaxExclClusters + nbelow + k - 1];
        unsigned mask = a < 0 ? kFull : 0u;
        mask |= __ballot_sync(kFull, d.sidx[(int64_t)y * kWarp + lane] < 0);
        if (y == (int)x) mask |= (lane == 31) ? kFull : ((2u << lane) - 1u);
        for (int64_t p = b; p < e; ++p) {
          const int sp = d.inv[col[p]];
          if ((sp >> 5) == y) mask |= 1u << (sp & 31);
        }
        if (lane == 0) {
          tiles[t] = (int32_t)x;
          tiles[tiles_cap + t] = y;
        }
        tile_masks[t * kWarp + lane] = mask;
      }
    }
    // interacting entries
    const auto cx = d.bc[x], hx = d.bh[x];
    const typename V4<T>::type zero = make_v4(T(0), T(0), T(0), T(0));
    const int cnt = d.ncount[x];
    int nb = 0;
    int64_t en = COUNT ? 0 : (int64_t)ecount[x];
    int64_t made = 0;
    for (int c = 0; c < cnt; ++c) {
      const int J = d.nbr[x * d.cap + c];
      if (J == (int)x) continue;
      if (__ballot_sync(kFull, ex0 == J || ex1 == J)) continue;
      const int64_t s = (int64_t)J * kWarp + lane;
      const int aj = d.sidx[s];
      bool ok = aj >= 0;
      if (ok) {
        const auto f = d.frac[s];
        ok = clusters_may_interact<T>(cx, hx, f, zero, info, rc);
      }
      const unsigned bal = __ballot_sync(kFull, ok);
      if (!COUNT && ok) s_buf[w][nb + __popc(bal & ((1u << lane) - 1u))] = aj;
      nb += __popc(bal);
      if (nb >= kWarp) {
        __syncwarp();
        if (!COUNT && en < entries_cap) {
          if (lane == 0) entry_cluster[en] = (int32_t)x;
          entry_atoms[en * kWarp + lane] = s_buf[w][lane];
        }
        __syncwarp();
        if (!COUNT) s_buf[w][lane] = s_buf[w][kWarp + lane];
        __syncwarp();
        nb -= kWarp;
        ++en;
        ++made;
      }
    }
    if (nb > 0) {
      __syncwarp();
      if (!COUNT && en < entries_cap) {
        if (lane == 0) entry_cluster[en] = (int32_t)x;
        entry_atoms[en * kWarp + lane] = lane < nb ? s_buf[w][lane] : -1;
      }
      ++made;
    }
    if (COUNT && lane == 0) ecount[x] = (unsigned)made;
    __syncwarp();
  }
}

// Marks an overflowing cluster list (status bit 1 of counts[2]).
__global__ void cluster_overflow_to_counts(const unsigned *status, int64_t *counts) {
  if (threadIdx.x == 0 && blockIdx.x == 0 && (status[0] & 1u)) counts[2] |= 2;
}

__global__ void cp_totals_kernel(const unsigned *tcount, const unsigned *ecount, int64_t n, const unsigned *cstat,
                                 int64_t *counts) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    counts[0] = tcount[n];
    counts[1] = ecount[n];
    counts[2] = cstat[0];
  }
}

// A unit of work over the format: tile u (u < ntiles) or entry u - ntiles.
struct CpView {
  int64_t natoms;
  const int32_t *sorted;
  int64_t nslots;
  const int32_t *tiles;
  int64_t ntiles;
  const uint32_t *masks;
  const int32_t *ecl;
  const int32_t *eat;
  int64_t nentries;
};

// Loads the unit's i atom (lane) and j atom (lane) and the lane's skip mask over j lanes.
// Returns false when the unit is padding.
__device__ __forceinline__ bool cp_unit(const CpView &v, int64_t u, int lane, int &ai, int &aj, unsigned &skip) {
  int x, y = -1;
  if (u < v.ntiles) {
    x = v.tiles[u];
    y = v.tiles[v.ntiles + u];
    if (x < 0 || y < 0) return false;
    skip = v.masks[u * kWarp + lane];
    const int64_t sj = (int64_t)y * kWarp + lane;
    aj = (y < v.nslots / kWarp) ? v.sorted[sj] : -1;
  } else {
    const int64_t e = u - v.ntiles;
    x = v.ecl[e];
    if (x < 0) return false;
    aj = v.eat[e * kWarp + lane];
    skip = 0u;
  }
  const int64_t si = (int64_t)x * kWarp + lane;
  ai = (x < v.nslots / kWarp) ? v.sorted[si] : -1;
  // indices outside [0, natoms) are treated as padding
  if (ai >= v.natoms) ai = -1;
  if (aj >= v.natoms) aj = -1;
  skip |= __ballot_sync(kFull, aj < 0);
  if (ai < 0) skip = kFull;
  return true;
}

__device__ __forceinline__ float cp_rsqrt(float v) { return rsqrtf(v); }
__device__ __forceinline__ double cp_rsqrt(double v) { return rsqrt(v); }

template <class T>
__device__ __forceinline__ void cp_min_image(bool ortho, T &dx, T &dy, T &dz, const T *m, const T *inv) {
  if (ortho) {
    dx = wrap1(dx, m[0], inv[0]);
    dy = wrap1(dy, m[4], inv[4]);
    dz = wrap1(dz, m[8], inv[8]);
  } else {
    min_image(dx, dy, dz, m, inv);
  }
}

// Same decision as the neighbour-list kernels: FP32 distances within 1e-5 relative of the
// cutoff are re-tested in FP64 from the caller's coordinates.
template <class T>
__device__ __forceinline__ bool cp_within(T r2, T rc2t, const T *x, int i, int j, const Box &b, bool ortho,
                                          double rc2) {
  if (sizeof(T) == 8) return r2 <= rc2t;
  if (fabsf((float)r2 - (float)rc2t) > 1e-5f * (float)rc2t) return r2 <= rc2t;
  double dx = (double)x[3 * (int64_t)i] - (double)x[3 * (int64_t)j];
  double dy = (double)x[3 * (int64_t)i + 1] - (double)x[3 * (int64_t)j + 1];
  double dz = (double)x[3 * (int64_t)i + 2] - (double)x[3 * (int64_t)j + 2];
  cp_min_image<double>(ortho, dx, dy, dz, b.m, b.inv);
  return dx * dx + dy * dy + dz * dz <= rc2;
}

template <class T>
__global__ void __launch_bounds__(kCpBlock) cp_decode_kernel(CpView v, const T *x, const T *box, double rc,
                                                             int32_t *pairs, int64_t cap, int32_t *npairs) {
  __shared__ Box s_b;
  __shared__ T s_m[9], s_inv[9];
  __shared__ T s_px[kCpWarps][kWarp], s_py[kCpWarps][kWarp], s_pz[kCpWarps][kWarp];
  __shared__ int s_a[kCpWarps][kWarp];
  if (threadIdx.x == 0) {
    load_box(box, s_b);
    for (int k = 0; k < 9; ++k) {
      s_m[k] = (T)s_b.m[k];
      s_inv[k] = (T)s_b.inv[k];
    }
  }
  __syncthreads();
  const bool ortho = s_b.m[1] == 0.0 && s_b.m[2] == 0.0 && s_b.m[3] == 0.0 && s_b.m[5] == 0.0 && s_b.m[6] == 0.0 &&
                     s_b.m[7] == 0.0;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const double rc2 = rc * rc;
  const T rc2t = (T)rc2;
  const int64_t nunits = v.ntiles + v.nentries;
  const int64_t nw = (int64_t)gridDim.x * kCpWarps;
  for (int64_t u = (int64_t)blockIdx.x * kCpWarps + w; u < nunits; u += nw) {
    int ai = -1, aj = -1;
    unsigned skip = kFull;
    if (!cp_unit(v, u, lane, ai, aj, skip)) continue;
    __syncwarp();
    s_a[w][lane] = aj;
    s_px[w][lane] = aj >= 0 ? x[3 * (int64_t)aj] : T(0);
    s_py[w][lane] = aj >= 0 ? x[3 * (int64_t)aj + 1] : T(0);
    s_pz[w][lane] = aj >= 0 ? x[3 * (int64_t)aj + 2] : T(0);
    __syncwarp();
    T pix = T(0), piy = T(0), piz = T(0);
    if (ai >= 0) {
      pix = x[3 * (int64_t)ai];
      piy = x[3 * (int64_t)ai + 1];
      piz = x[3 * (int64_t)ai + 2];
    }
    for (int k = 0; k < kWarp; ++k) {
      const int jl = (lane + k) & 31;
      bool ok = !((skip >> jl) & 1u);
      const int j = s_a[w][jl];
      if (ok) {
        T dx = pix - s_px[w][jl], dy = piy - s_py[w][jl], dz = piz - s_pz[w][jl];
        cp_min_image<T>(ortho, dx, dy, dz, s_m, s_inv);
        ok = cp_within<T>(dx * dx + dy * dy + dz * dz, rc2t, x, ai, j, s_b, ortho, rc2);
      }
      const unsigned bal = __ballot_sync(kFull, ok);
      if (bal) {
        int base = 0;
        if (lane == 0) base = atomicAdd(npairs, __popc(bal));
        base = __shfl_sync(kFull, base, 0);
        if (ok) {
          const int64_t r = (int64_t)base + __popc(bal & ((1u << lane) - 1u));
          if (r < cap) {
            pairs[2 * r] = max(ai, j);
            pairs[2 * r + 1] = min(ai, j);
          }
        }
      }
    }
  }
}

// Fused shifted/plain Coulomb + Lennard-Jones (Lorentz-Berthelot) over the format. Lane i
// owns atom i of the unit; at step k it meets j lane (i + k) mod 32, so the 32 lanes touch
// 32 different j atoms in every step and the j-side sums ride along in registers that
// rotate one lane per step (back home after 32 steps). Gradients go into Acc<T> (int64
// fixed point for FP32, FP64 atomics for FP64), energies likewise (acc[0] total, acc[1]
// Coulomb part).
template <class T, bool PG>
__global__ void __launch_bounds__(kCpBlock) cp_energy_kernel(CpView v, const T *x, const T *box, const T *q,
                                                             const T *sig, const T *eps, double kc_, double rc_,
                                                             int do_shift, typename Acc<T>::S *gx,
                                                             typename Acc<T>::S *gq, typename Acc<T>::S *gs,
                                                             typename Acc<T>::S *ge, typename Acc<T>::S *eacc) {
  using V = typename V4<T>::type;
  __shared__ T s_m[9], s_inv[9];
  __shared__ int s_ortho;
  __shared__ V s_p[kCpWarps][kWarp];
  __shared__ T s_s[kCpWarps][kWarp], s_e[kCpWarps][kWarp];
  if (threadIdx.x == 0) {
    Box b;
    load_box(box, b);
    for (int k = 0; k < 9; ++k) {
      s_m[k] = (T)b.m[k];
      s_inv[k] = (T)b.inv[k];
    }
    s_ortho = b.m[1] == 0.0 && b.m[2] == 0.0 && b.m[3] == 0.0 && b.m[5] == 0.0 && b.m[6] == 0.0 && b.m[7] == 0.0;
  }
  __syncthreads();
  const bool ortho = s_ortho;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const T rc = (T)rc_, rc2 = rc * rc, kc = (T)kc_;
  const T inv_rc = do_shift ? T(1) / rc : T(0);
  double e_tot = 0.0, e_coul = 0.0;
  const int64_t nunits = v.ntiles + v.nentries;
  const int64_t nw = (int64_t)gridDim.x * kCpWarps;
  for (int64_t u = (int64_t)blockIdx.x * kCpWarps + w; u < nunits; u += nw) {
    int ai = -1, aj = -1;
    unsigned skip = kFull;
    if (!cp_unit(v, u, lane, ai, aj, skip)) continue;
    __syncwarp();
    s_p[w][lane] = aj >= 0 ? make_v4(x[3 * (int64_t)aj], x[3 * (int64_t)aj + 1], x[3 * (int64_t)aj + 2], q[aj])
                           : make_v4(T(0), T(0), T(0), T(0));
    s_s[w][lane] = aj >= 0 ? sig[aj] : T(0);
    s_e[w][lane] = aj >= 0 ? eps[aj] : T(0);
    __syncwarp();
    V pi = make_v4(T(0), T(0), T(0), T(0));
    T si = T(0), ei = T(0);
    if (ai >= 0) {
      pi = make_v4(x[3 * (int64_t)ai], x[3 * (int64_t)ai + 1], x[3 * (int64_t)ai + 2], q[ai]);
      si = sig[ai];
      ei = eps[ai];
    }
    T fix = T(0), fiy = T(0), fiz = T(0), gqi = T(0), gsi = T(0), gei = T(0);
    T fjx = T(0), fjy = T(0), fjz = T(0), gqj = T(0), gsj = T(0), gej = T(0);
    T et = T(0), ec = T(0);
    for (int k = 0; k < kWarp; ++k) {
      const int jl = (lane + k) & 31;
      if (!((skip >> jl) & 1u)) {
        const V pj = s_p[w][jl];
        T dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
        cp_min_image<T>(ortho, dx, dy, dz, s_m, s_inv);
        const T r2 = dx * dx + dy * dy + dz * dz;
        if (r2 <= rc2) {
          const T rinv = cp_rsqrt(r2);
          const T rinv2 = rinv * rinv;
          const T f = rinv - inv_rc;
          const T kqq = kc * pi.w * pj.w;
          const T e_c = kqq * f;
          T dedr_r = -kqq * rinv2 * rinv;
          const T sj = s_s[w][jl], ej = s_e[w][jl];
          const T s = T(0.5) * (si + sj);
          const T ep = sqrt(ei * ej);
          const T sr2 = s * s * rinv2;
          const T sr6 = sr2 * sr2 * sr2;
          const T e_lj = T(4) * ep * sr6 * (sr6 - T(1));
          const T g = T(24) * ep * sr6 * (T(2) * sr6 - T(1));
          dedr_r -= g * rinv2;
          et += e_c + e_lj;
          ec += e_c;
          fix += dedr_r * dx;
          fiy += dedr_r * dy;
          fiz += dedr_r * dz;
          fjx -= dedr_r * dx;
          fjy -= dedr_r * dy;
          fjz -= dedr_r * dz;
          if (PG) {
            gqi += kc * pj.w * f;
            gqj += kc * pi.w * f;
            const T de_ds = T(0.5) * g / s;
            gsi += de_ds;
            gsj += de_ds;
            if (ep > T(0)) {
              const T h = T(4) * sr6 * (sr6 - T(1)) / (T(2) * ep);
              gei += h * ej;
              gej += h * ei;
            }
          }
        }
      }
      const int src = (lane + 1) & 31;
      fjx = __shfl_sync(kFull, fjx, src);
      fjy = __shfl_sync(kFull, fjy, src);
      fjz = __shfl_sync(kFull, fjz, src);
      if (PG) {
        gqj = __shfl_sync(kFull, gqj, src);
        gsj = __shfl_sync(kFull, gsj, src);
        gej = __shfl_sync(kFull, gej, src);
      }
    }
    e_tot += (double)et;
    e_coul += (double)ec;
    if (ai >= 0 && gx) {
      Acc<T>::add(&gx[3 * (int64_t)ai], (double)fix);
      Acc<T>::add(&gx[3 * (int64_t)ai + 1], (double)fiy);
      Acc<T>::add(&gx[3 * (int64_t)ai + 2], (double)fiz);
    }
    if (aj >= 0 && gx) {
      Acc<T>::add(&gx[3 * (int64_t)aj], (double)fjx);
      Acc<T>::add(&gx[3 * (int64_t)aj + 1], (double)fjy);
      Acc<T>::add(&gx[3 * (int64_t)aj + 2], (double)fjz);
    }
    if (PG) {
      if (ai >= 0) {
        Acc<T>::add(&gq[ai], (double)gqi);
        Acc<T>::add(&gs[ai], (double)gsi);
        Acc<T>::add(&ge[ai], (double)gei);
      }
      if (aj >= 0) {
        Acc<T>::add(&gq[aj], (double)gqj);
        Acc<T>::add(&gs[aj], (double)gsj);
        Acc<T>::add(&ge[aj], (double)gej);
      }
    }
  }
  e_tot = warp_sum(e_tot);
  e_coul = warp_sum(e_coul);
  if (lane == 0 && eacc) {
    Acc<T>::add(&eacc[0], e_tot);
    Acc<T>::add(&eacc[1], e_coul);
  }
}

template <class T>
__global__ void cp_acc_out(const typename Acc<T>::S *acc, T *out, int64_t n, double scale, bool add) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const double v = scale * Acc<T>::get(&acc[k]);
    out[k] = add ? (T)((double)out[k] + v) : (T)v;
  }
}

template <class T>
__global__ void cp_energy_out(const typename Acc<T>::S *eacc, T *energy, T *energy_coulomb) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    if (energy) energy[0] = (T)Acc<T>::get(&eacc[0]);
    if (energy_coulomb) energy_coulomb[0] = (T)Acc<T>::get(&eacc[1]);
  }
}

template <class T>
int cp_build_impl(int64_t natoms, const T *x, const T *box, double rc, const int64_t *rp, const int64_t *col,
                  int32_t *sorted, int32_t *tiles, int64_t tiles_cap, uint32_t *masks, int32_t *ecl, int32_t *eat,
                  int64_t entries_cap, int64_t *counts, int ccap, void *ws, size_t ws_bytes, cudaStream_t s) {
  const int dtype = sizeof(T) == 8 ? TFF_F64 : TFF_F32;
  const int64_t ncl = (natoms + kWarp - 1) / kWarp;
  const int cap = ccap > 0 ? ccap : (int)std::max<int64_t>(1, std::min<int64_t>(ncl, 1024));
  CpLayout L = cp_layout(dtype, natoms, cap);
  if (ws == nullptr || ws_bytes < L.bytes) {
    set_error("workspace too small: need %zu bytes, got %zu", L.bytes, ws_bytes);
    return TFF_ERR_WORKSPACE;
  }
  if (tiles_cap > 0) {
    TFF_CUDA(cudaMemsetAsync(tiles, 0xff, sizeof(int32_t) * 2 * tiles_cap, s));
    TFF_CUDA(cudaMemsetAsync(masks, 0xff, sizeof(uint32_t) * kWarp * tiles_cap, s));
  }
  if (entries_cap > 0) {
    TFF_CUDA(cudaMemsetAsync(ecl, 0xff, sizeof(int32_t) * entries_cap, s));
    TFF_CUDA(cudaMemsetAsync(eat, 0xff, sizeof(int32_t) * kWarp * entries_cap, s));
  }
  TFF_CUDA(cudaMemsetAsync(counts, 0, sizeof(int64_t) * 3, s));
  if (natoms == 0) return TFF_OK;
  char *b = static_cast<char *>(ws);
  ClusterData<T> d = cluster_data<T>(L.cl, ws);
  int *exset = reinterpret_cast<int *>(b + L.exset);
  int *exn = reinterpret_cast<int *>(b + L.exn);
  unsigned *tcount = reinterpret_cast<unsigned *>(b + L.tcount);
  unsigned *ecount = reinterpret_cast<unsigned *>(b + L.ecount);
  unsigned *cstat = reinterpret_cast<unsigned *>(b + L.cstat);
  TFF_CUDA(cudaMemsetAsync(cstat, 0, 4 * sizeof(unsigned), s));
  int st = build_clusters<T>(L.cl, d, ws, x, nullptr, box, rc, /*half=*/1, s);
  if (st != TFF_OK) return st;
  const int nb = (int)std::max<int64_t>(1, std::min<int64_t>((ncl + kCpWarps - 1) / kCpWarps, sm_count() * 16));
  excl_clusters_kernel<T><<<nb, kCpBlock, 0, s>>>(d, rp, col, exset, exn, cstat);
  TFF_LAUNCHED();
  cp_emit_kernel<T, true><<<nb, kCpBlock, 0, s>>>(d, rc, rp, col, exset, exn, tcount, ecount, tiles, tiles_cap, masks,
                                                  ecl, eat, entries_cap);
  TFF_LAUNCHED();
  scan_keys_kernel<<<1, 1024, 0, s>>>(tcount, ncl);
  TFF_LAUNCHED();
  scan_keys_kernel<<<1, 1024, 0, s>>>(ecount, ncl);
  TFF_LAUNCHED();
  cp_emit_kernel<T, false><<<nb, kCpBlock, 0, s>>>(d, rc, rp, col, exset, exn, tcount, ecount, tiles, tiles_cap,
                                                   masks, ecl, eat, entries_cap);
  TFF_LAUNCHED();
  // sorted atom of every slot (-1 padding)
  TFF_CUDA(cudaMemcpyAsync(sorted, d.sidx, sizeof(int32_t) * L.cl.npad, cudaMemcpyDeviceToDevice, s));
  // counts: tiles, entries, status (bit 0: too many exclusion clusters, bit 1: list overflow)
  cp_totals_kernel<<<1, 32, 0, s>>>(tcount, ecount, ncl, cstat, counts);
  TFF_LAUNCHED();
  cluster_overflow_to_counts<<<1, 32, 0, s>>>(d.status, counts);
  TFF_LAUNCHED();
  return TFF_OK;
}

}  // namespace
}  // namespace tff

using namespace tff;

namespace {

template <class T>
int cp_energy_impl(int64_t natoms, const T *x, const T *box, const T *sig, const T *eps, const T *q, double kc,
                   double rc, int do_shift, const CpView &v, T *energy, T *energy_coulomb, T *gx, double gx_scale,
                   bool gx_add, T *gs, T *ge, T *gq, void *ws, size_t ws_bytes, cudaStream_t s) {
  using S = typename Acc<T>::S;
  Carver c(ws);
  S *agx = c.take<S>(3 * natoms);
  S *agq = c.take<S>(natoms);
  S *ags = c.take<S>(natoms);
  S *age = c.take<S>(natoms);
  S *eacc = c.take<S>(2);
  if (ws == nullptr || ws_bytes < c.bytes()) {
    set_error("workspace too small: need %zu bytes, got %zu", c.bytes(), ws_bytes);
    return TFF_ERR_WORKSPACE;
  }
  TFF_CUDA(cudaMemsetAsync(ws, 0, c.bytes(), s));
  const bool pg = gq || gs || ge;
  const int64_t nunits = v.ntiles + v.nentries;
  if (nunits > 0 && natoms > 0) {
    const int nb = (int)std::max<int64_t>(1, std::min<int64_t>((nunits + kCpWarps - 1) / kCpWarps, sm_count() * 8));
    if (pg)
      cp_energy_kernel<T, true><<<nb, kCpBlock, 0, s>>>(v, x, box, q, sig, eps, kc, rc, do_shift, agx, agq, ags, age,
                                                        eacc);
    else
      cp_energy_kernel<T, false><<<nb, kCpBlock, 0, s>>>(v, x, box, q, sig, eps, kc, rc, do_shift,
                                                         gx ? agx : nullptr, nullptr, nullptr, nullptr, eacc);
    TFF_LAUNCHED();
  }
  const int nb = (int)std::max<int64_t>(1, std::min<int64_t>((3 * natoms + 255) / 256, sm_count() * 8));
  if (gx && natoms > 0) {
    cp_acc_out<T><<<nb, 256, 0, s>>>(agx, gx, 3 * natoms, gx_scale, gx_add);
    TFF_LAUNCHED();
  }
  T *pout[3] = {gq, gs, ge};
  S *pacc[3] = {agq, ags, age};
  for (int k = 0; k < 3; ++k) {
    if (pout[k] && natoms > 0) {
      cp_acc_out<T><<<nb, 256, 0, s>>>(pacc[k], pout[k], natoms, 1.0, false);
      TFF_LAUNCHED();
    }
  }
  if (energy || energy_coulomb) {
    cp_energy_out<T><<<1, 32, 0, s>>>(eacc, energy, energy_coulomb);
    TFF_LAUNCHED();
  }
  return TFF_OK;
}

int cp_view_check(int64_t natoms, const int32_t *sorted, int64_t nslots, const int32_t *tiles, int64_t ntiles,
                  const uint32_t *masks, const int32_t *ecl, const int32_t *eat, int64_t nentries) {
  TFF_ARG(natoms >= 0 && nslots >= 0 && ntiles >= 0 && nentries >= 0, "negative sizes");
  TFF_ARG(nslots % kWarp == 0, "sorted_atoms length must be a multiple of 32");
  TFF_ARG(sorted != nullptr || nslots == 0, "sorted_atoms is NULL");
  TFF_ARG((tiles != nullptr && masks != nullptr) || ntiles == 0, "tiles / tile_masks are NULL");
  TFF_ARG((ecl != nullptr && eat != nullptr) || nentries == 0, "entry arrays are NULL");
  return TFF_OK;
}

}  // namespace

extern "C" {

size_t tff_cluster_pairs_workspace_bytes(int dtype, int64_t natoms, int max_cluster_neighbors) {
  const int64_t ncl = (natoms + kWarp - 1) / kWarp;
  const int cap = max_cluster_neighbors > 0 ? max_cluster_neighbors
                                            : (int)std::max<int64_t>(1, std::min<int64_t>(ncl, 1024));
  return cp_layout(dtype, natoms, cap).bytes;
}

int tff_cluster_pairs_build(int dtype, int64_t natoms, const void *coords, const void *box, double cutoff,
                            const int64_t *excl_row_ptr, const int64_t *excl_col, int32_t *sorted_atoms,
                            int32_t *tiles, uint32_t *tile_masks, int64_t tiles_cap, int32_t *entry_cluster,
                            int32_t *entry_atoms, int64_t entries_cap, int64_t *counts, int max_cluster_neighbors,
                            void *workspace, size_t workspace_bytes, tff_stream_t stream) {
  TFF_NVTX("tff_cluster_pairs_build");
  TFF_ARG(dtype == TFF_F32 || dtype == TFF_F64, "dtype must be TFF_F32 or TFF_F64");
  TFF_ARG(box != nullptr, "build_cluster_pairs requires a periodic box");
  TFF_ARG(natoms >= 0 && tiles_cap >= 0 && entries_cap >= 0, "negative sizes");
  TFF_ARG(natoms < (int64_t)INT_MAX / 2, "too many atoms");
  TFF_ARG(coords != nullptr || natoms == 0, "coords is NULL");
  TFF_ARG(counts != nullptr, "counts is NULL");
  TFF_ARG(sorted_atoms != nullptr || natoms == 0, "sorted_atoms is NULL");
  TFF_ARG((tiles != nullptr && tile_masks != nullptr) || tiles_cap == 0, "tiles / tile_masks are NULL");
  TFF_ARG((entry_cluster != nullptr && entry_atoms != nullptr) || entries_cap == 0, "entry arrays are NULL");
  TFF_ARG((excl_row_ptr == nullptr) == (excl_col == nullptr), "exclusion CSR needs both arrays");
  TFF_ARG(cutoff >= 0.0, "cutoff must be >= 0");
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == TFF_F32)
    return cp_build_impl<float>(natoms, (const float *)coords, (const float *)box, cutoff, excl_row_ptr, excl_col,
                                sorted_atoms, tiles, tiles_cap, tile_masks, entry_cluster, entry_atoms, entries_cap,
                                counts, max_cluster_neighbors, workspace, workspace_bytes, s);
  return cp_build_impl<double>(natoms, (const double *)coords, (const double *)box, cutoff, excl_row_ptr, excl_col,
                               sorted_atoms, tiles, tiles_cap, tile_masks, entry_cluster, entry_atoms, entries_cap,
                               counts, max_cluster_neighbors, workspace, workspace_bytes, s);
}

int tff_cluster_pairs_decode(int dtype, int64_t natoms, const void *coords, const void *box, double cutoff,
                             const int32_t *sorted_atoms, int64_t nslots, const int32_t *tiles, int64_t ntiles,
                             const uint32_t *tile_masks, const int32_t *entry_cluster, const int32_t *entry_atoms,
                             int64_t nentries, int32_t *pairs, int64_t max_npairs, int32_t *npairs,
                             tff_stream_t stream) {
  TFF_NVTX("tff_cluster_pairs_decode");
  TFF_ARG(dtype == TFF_F32 || dtype == TFF_F64, "dtype must be TFF_F32 or TFF_F64");
  TFF_ARG(box != nullptr, "decode_cluster_pairs requires a periodic box");
  TFF_ARG(coords != nullptr || natoms == 0, "coords is NULL");
  TFF_ARG(npairs != nullptr, "npairs is NULL");
  TFF_ARG(max_npairs >= 0 && (pairs != nullptr || max_npairs == 0), "pairs is NULL");
  TFF_ARG(cutoff >= 0.0, "cutoff must be >= 0");
  int st = cp_view_check(natoms, sorted_atoms, nslots, tiles, ntiles, tile_masks, entry_cluster, entry_atoms, nentries);
  if (st != TFF_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  if (max_npairs > 0) TFF_CUDA(cudaMemsetAsync(pairs, 0xff, sizeof(int32_t) * 2 * max_npairs, s));
  TFF_CUDA(cudaMemsetAsync(npairs, 0, sizeof(int32_t), s));
  const CpView v{natoms, sorted_atoms, nslots, tiles, ntiles, tile_masks, entry_cluster, entry_atoms, nentries};
  const int64_t nunits = ntiles + nentries;
  if (nunits == 0 || natoms == 0) return TFF_OK;
  const int nb = (int)std::max<int64_t>(1, std::min<int64_t>((nunits + kCpWarps - 1) / kCpWarps, sm_count() * 8));
  if (dtype == TFF_F32)
    cp_decode_kernel<float><<<nb, kCpBlock, 0, s>>>(v, (const float *)coords, (const float *)box, cutoff, pairs,
                                                    max_npairs, npairs);
  else
    cp_decode_kernel<double><<<nb, kCpBlock, 0, s>>>(v, (const double *)coords, (const double *)box, cutoff, pairs,
                                                     max_npairs, npairs);
  TFF_LAUNCHED();
  return TFF_OK;
}

size_t tff_nonbonded_cluster_pairs_workspace_bytes(int dtype, int64_t natoms) {
  const size_t e = 8;  // int64 fixed point (FP32) or double (FP64): both 8 bytes
  (void)dtype;
  Carver c(nullptr);
  c.take<char>(3 * natoms * e);
  c.take<char>(natoms * e);
  c.take<char>(natoms * e);
  c.take<char>(natoms * e);
  c.take<char>(2 * e);
  return c.bytes();
}

int tff_nonbonded_cluster_pairs(int dtype, int64_t natoms, const void *coords, const void *box, const void *sigma,
                                const void *epsilon, const void *charges, double coul_constant, double cutoff,
                                int do_shift, const int32_t *sorted_atoms, int64_t nslots, const int32_t *tiles,
                                int64_t ntiles, const uint32_t *tile_masks, const int32_t *entry_cluster,
                                const int32_t *entry_atoms, int64_t nentries, void *energy, void *energy_coulomb,
                                void *grad_coords, void *grad_sigma, void *grad_epsilon, void *grad_charges,
                                void *workspace, size_t workspace_bytes, tff_stream_t stream) {
  TFF_NVTX("tff_nonbonded_cluster_pairs");
  TFF_ARG(dtype == TFF_F32 || dtype == TFF_F64, "dtype must be TFF_F32 or TFF_F64");
  TFF_ARG(box != nullptr, "the cluster-pair nonbonded term requires a periodic box");
  TFF_ARG(natoms == 0 || (coords && sigma && epsilon && charges), "coords / sigma / epsilon / charges is NULL");
  TFF_ARG(cutoff > 0.0, "cutoff must be > 0");
  int st = cp_view_check(natoms, sorted_atoms, nslots, tiles, ntiles, tile_masks, entry_cluster, entry_atoms, nentries);
  if (st != TFF_OK) return st;
  const CpView v{natoms, sorted_atoms, nslots, tiles, ntiles, tile_masks, entry_cluster, entry_atoms, nentries};
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == TFF_F32)
    return cp_energy_impl<float>(natoms, (const float *)coords, (const float *)box, (const float *)sigma,
                                 (const float *)epsilon, (const float *)charges, coul_constant, cutoff, do_shift, v,
                                 (float *)energy, (float *)energy_coulomb, (float *)grad_coords, 1.0, false,
                                 (float *)grad_sigma, (float *)grad_epsilon, (float *)grad_charges, workspace,
                                 workspace_bytes, s);
  return cp_energy_impl<double>(natoms, (const double *)coords, (const double *)box, (const double *)sigma,
                                (const double *)epsilon, (const double *)charges, coul_constant, cutoff, do_shift, v,
                                (double *)energy, (double *)energy_coulomb, (double *)grad_coords, 1.0, false,
                                (double *)grad_sigma, (double *)grad_epsilon, (double *)grad_charges, workspace,
                                workspace_bytes, s);
}

int tff_nonbonded_forces_cluster_pairs(int dtype, int64_t natoms, const void *coords, const void *box,
                                       const void *sigma, const void *epsilon, const void *charges,
                                       double coul_constant, double cutoff, const int32_t *sorted_atoms,
                                       int64_t nslots, const int32_t *tiles, int64_t ntiles,
                                       const uint32_t *tile_masks, const int32_t *entry_cluster,
                                       const int32_t *entry_atoms, int64_t nentries, void *forces, void *workspace,
                                       size_t workspace_bytes, tff_stream_t stream) {
  TFF_NVTX("tff_nonbonded_forces_cluster_pairs");
  TFF_ARG(dtype == TFF_F32 || dtype == TFF_F64, "dtype must be TFF_F32 or TFF_F64");
  TFF_ARG(box != nullptr, "the cluster-pair nonbonded term requires a periodic box");
  TFF_ARG(natoms == 0 || (coords && sigma && epsilon && charges && forces), "an input array is NULL");
  TFF_ARG(cutoff > 0.0, "cutoff must be > 0");
  int st = cp_view_check(natoms, sorted_atoms, nslots, tiles, ntiles, tile_masks, entry_cluster, entry_atoms, nentries);
  if (st != TFF_OK) return st;
  const CpView v{natoms, sorted_atoms, nslots, tiles, ntiles, tile_masks, entry_cluster, entry_atoms, nentries};
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == TFF_F32)
    return cp_energy_impl<float>(natoms, (const float *)coords, (const float *)box, (const float *)sigma,
                                 (const float *)epsilon, (const float *)charges, coul_constant, cutoff, 1, v, nullptr,
                                 nullptr, (float *)forces, -1.0, true, nullptr, nullptr, nullptr, workspace,
                                 workspace_bytes, s);
  return cp_energy_impl<double>(natoms, (const double *)coords, (const double *)box, (const double *)sigma,
                                (const double *)epsilon, (const double *)charges, coul_constant, cutoff, 1, v, nullptr,
                                nullptr, (double *)forces, -1.0, true, nullptr, nullptr, nullptr, workspace,
                                workspace_bytes, s);
}

}  // extern "C"

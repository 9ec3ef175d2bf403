// Cluster build shared by the cell-list neighbour list and the fused real-space kernel.
//
// 1. cell_keys:      fractional coordinates wrapped to [0,1), cell on an nc^3 grid
//                    (about 8 atoms per cell), Hilbert-curve key, per-key histogram.
// 2. scan_keys:      exclusive scan of the histogram (one block, segmented).
// 3. scatter_atoms:  atoms into key buckets (slot order inside a bucket is arbitrary).
// 4. sort_buckets:   one warp per bucket ranks its atoms by index -> deterministic order; writes the
//                    sorted SoA (wrapped position + charge as a 4-vector, original index,
//                    inverse map, fractional position) and pads to a multiple of 32.
// 5. cluster_bounds: one warp per 32-atom cluster: fractional bounding box.
// 6. cluster_neighbors: one warp per cluster scans all clusters in index order and keeps
//                    those whose boxes can hold a pair within the cutoff (order of the
//                    list is deterministic). `half` keeps only J <= I.
//
// Along the Hilbert curve of ~8-atom cells, 32 consecutive atoms form a compact blob of
// about 4 face-connected cells, which is what the 32x32 warp tiles need.
#pragma once

#include <climits>

#include "tff_common.cuh"

namespace tff {

// Neighbour clusters per tile-kernel work item (a work item is one cluster I and every
// (ncount/kItemTiles)-th cluster of its list). 4 gives a 9000-atom box ~5,600 warps of work,
// enough to fill 148 SMs; 8 measured 3 % slower there and equal at 300,000 atoms; 3 and 2
// measured 3 % and 6 % slower at 9000 atoms and 4 % and 10 % slower at 300,000 atoms (more
// items hold the SMs longer against the PME kernels of the other stream).
constexpr int kItemTiles = 4;
// Consecutive clusters per super-cluster: the neighbour search screens a super-cluster's
// union box first and tests its members only when that box is within the cutoff.
constexpr int kSuper = 32;
// Histograms up to this many keys are scanned by the last block of the key kernel.
constexpr int64_t kFusedScanMaxKeys = 8192;

template <class T> struct V4;
template <> struct V4<float> { using type = float4; };
struct __align__(16) D4 { double x, y, z, w; };
template <> struct V4<double> { using type = D4; };

__device__ __forceinline__ D4 make_v4(double x, double y, double z, double w) { return D4{x, y, z, w}; }
__device__ __forceinline__ float4 make_v4(float x, float y, float z, float w) { return make_float4(x, y, z, w); }

struct ClusterLayout {
  int nc = 1, bits = 0;
  int64_t nkeys = 1, natoms = 0, nclusters = 0, npad = 0, nsuper = 0;
  int cap = 0;
  size_t keys, hist, fill, status, tmp, sidx, inv, pos, frac, bc, bh, sbc, sbh, nbr, ncount, itemoff, items, boxinfo;
  size_t zero_off, zero_bytes, bytes;
};

// Cell grid side (cells per box vector) and Hilbert bits for `natoms` atoms at about
// `atoms_per_cell` atoms per cell. 8 is the default: runs of 32 atoms along the curve then
// form the most compact clusters (fewest cluster pairs within the cutoff) among 2..32
// atoms per cell on water boxes. From 16 cells per side up, the side is rounded to a power
// of two: on a grid that only partly fills its 2^b key space the curve leaves and
// re-enters the grid, and a 32-atom run across such a jump is not compact (small boxes
// bound the damage).
inline void cell_grid(int64_t natoms, double atoms_per_cell, int &nc, int &bits) {
  const double g = cbrt((double)natoms / atoms_per_cell);
  nc = g >= 16.0 ? (1 << (int)lround(log2(g))) : (int)floor(g);
  nc = std::max(1, std::min(nc, 128));
  bits = 0;
  while ((1 << bits) < nc) ++bits;
}

inline ClusterLayout cluster_layout(int dtype, int64_t natoms, int cap) {
  ClusterLayout L;
  L.natoms = natoms;
  int nc, bits;
  cell_grid(natoms, 8.0, nc, bits);
  L.nc = nc;
  L.bits = bits;
  L.nkeys = (int64_t)1 << (3 * bits);
  L.nclusters = (natoms + kWarp - 1) / kWarp;
  L.npad = L.nclusters * kWarp;
  L.nsuper = (L.nclusters + kSuper - 1) / kSuper;
  L.cap = cap;
  const size_t tsz = dtype == TFF_F64 ? 8 : 4;
  Carver c(nullptr);
  // zero-initialised region first: hist, fill, status
  L.hist = c.off; c.take<unsigned>(L.nkeys + 1);
  L.fill = (c.off + 255) & ~size_t(255); c.take<unsigned>(L.nkeys);
  L.status = (c.off + 255) & ~size_t(255); c.take<unsigned>(64);
  L.zero_off = 0;
  L.zero_bytes = c.bytes();
  L.keys = (c.off + 255) & ~size_t(255); c.take<unsigned>(natoms);
  L.tmp = (c.off + 255) & ~size_t(255); c.take<int>(natoms);
  L.sidx = (c.off + 255) & ~size_t(255); c.take<int>(L.npad);
  L.inv = (c.off + 255) & ~size_t(255); c.take<int>(natoms);
  L.pos = (c.off + 255) & ~size_t(255); c.take<char>(L.npad * 4 * tsz);
  L.frac = (c.off + 255) & ~size_t(255); c.take<char>(L.npad * 4 * tsz);
  L.bc = (c.off + 255) & ~size_t(255); c.take<char>(L.nclusters * 4 * tsz);
  L.bh = (c.off + 255) & ~size_t(255); c.take<char>(L.nclusters * 4 * tsz);
  L.sbc = (c.off + 255) & ~size_t(255); c.take<char>(L.nsuper * 4 * tsz);
  L.sbh = (c.off + 255) & ~size_t(255); c.take<char>(L.nsuper * 4 * tsz);
  L.nbr = (c.off + 255) & ~size_t(255); c.take<int>((size_t)L.nclusters * cap);
  L.ncount = (c.off + 255) & ~size_t(255); c.take<int>(L.nclusters);
  L.itemoff = (c.off + 255) & ~size_t(255); c.take<int>(L.nclusters + 1);
  L.items = (c.off + 255) & ~size_t(255); c.take<int>((size_t)L.nclusters * ((cap + kItemTiles - 1) / kItemTiles));
  L.boxinfo = (c.off + 255) & ~size_t(255); c.take<double>(32);
  L.bytes = c.bytes();
  return L;
}

// One system of a batch (several independent periodic systems evaluated by the same
// launches). Clusters, super-clusters, PME grids and box facts of a batch are laid out
// system after system; every cluster list stays inside its own system.
struct BatchSys {
  int64_t atom_off, natoms;    // caller-order atoms in the batch arrays
  int64_t cl_off, ncl;         // clusters: sorted slots [32 cl_off, 32 (cl_off + ncl))
  int64_t sup_off, nsup;       // super-clusters
  int64_t grid_off, cplx_off;  // PME grids: K^3 real points, K*K*(K/2+1) complex points
  int nc, bits;                // cell grid side and Hilbert bits per axis
  int K, mod_off;              // PME grid side and offset of its B-spline moduli
  int plane_off;               // the system's first DFT plane unit (sum of K before it)
  int conv_blocks;             // work units (and reduction blocks) of its convolution
  int conv_off;                // the system's first convolution unit (sum of conv_blocks before it)
  int gather_blocks;           // work units (and reduction blocks) of its force gather; the spread's too
  int gather_off;              // the system's first gather unit
  int pad;
};

// Totals of a batch, in device memory beside its system table: the batched kernels read
// the batch's composition here, so their launch shapes depend on the batch's capacity
// alone and one captured CUDA graph serves every composition.
struct BatchShape {
  int64_t natoms, nclusters, npad, nsuper, total_grid;
  int nsys;
  int plane_units;  // DFT plane units: sum of K
  int kmax;
  int conv_units;   // convolution units: sum of conv_blocks
  int gather_units; // gather (and spread) units: sum of gather_blocks
  int pad;
};

// Stride of the per-system box facts (see box_info_kernel).
constexpr int kInfoStride = 32;

// Pointers into one workspace.
template <class T>
struct ClusterData {
  using V = typename V4<T>::type;
  unsigned *keys, *hist, *fill, *status;
  int *tmp, *sidx, *inv, *nbr, *ncount;
  int *itemoff;  // work items of the tile kernel: prefix sums of ceil(ncount / kItemTiles)
  int *items;    // owning cluster of each work item
  V *pos, *frac, *bc, *bh;
  V *sbc, *sbh;     // union boxes of kSuper consecutive clusters (fractional centre, half extent)
  double *boxinfo;  // [0..8] box, [9..17] inv, [18] ortho flag, [19..21] perpendicular widths
  int nc, bits, cap;
  int64_t natoms, nclusters, npad, nsuper;
  // batch mode: system table and owners (NULL for one system); boxinfo then holds one
  // record of kInfoStride doubles per system
  const BatchSys *sys;
  int *cl_sys;   // owning system of each cluster
  int *sup_sys;  // owning system of each super-cluster
  const BatchShape *shape;  // batch mode: the sizes below come from here (device memory)
  __device__ __forceinline__ int system_of(int64_t cluster) const { return cl_sys ? cl_sys[cluster] : 0; }
  __device__ __forceinline__ int64_t n_atoms() const { return shape ? shape->natoms : natoms; }
  __device__ __forceinline__ int64_t n_clusters() const { return shape ? shape->nclusters : nclusters; }
  __device__ __forceinline__ int64_t n_pad() const { return shape ? shape->npad : npad; }
  __device__ __forceinline__ int64_t n_super() const { return shape ? shape->nsuper : nsuper; }
  __device__ __forceinline__ const double *info(int system) const { return boxinfo + kInfoStride * system; }
};

template <class T>
inline ClusterData<T> cluster_data(const ClusterLayout &L, void *ws) {
  char *b = static_cast<char *>(ws);
  ClusterData<T> d;
  using V = typename ClusterData<T>::V;
  d.keys = reinterpret_cast<unsigned *>(b + L.keys);
  d.hist = reinterpret_cast<unsigned *>(b + L.hist);
  d.fill = reinterpret_cast<unsigned *>(b + L.fill);
  d.status = reinterpret_cast<unsigned *>(b + L.status);
  d.tmp = reinterpret_cast<int *>(b + L.tmp);
  d.sidx = reinterpret_cast<int *>(b + L.sidx);
  d.inv = reinterpret_cast<int *>(b + L.inv);
  d.nbr = reinterpret_cast<int *>(b + L.nbr);
  d.ncount = reinterpret_cast<int *>(b + L.ncount);
  d.itemoff = reinterpret_cast<int *>(b + L.itemoff);
  d.items = reinterpret_cast<int *>(b + L.items);
  d.pos = reinterpret_cast<V *>(b + L.pos);
  d.frac = reinterpret_cast<V *>(b + L.frac);
  d.bc = reinterpret_cast<V *>(b + L.bc);
  d.bh = reinterpret_cast<V *>(b + L.bh);
  d.sbc = reinterpret_cast<V *>(b + L.sbc);
  d.sbh = reinterpret_cast<V *>(b + L.sbh);
  d.boxinfo = reinterpret_cast<double *>(b + L.boxinfo);
  d.nc = L.nc;
  d.bits = L.bits;
  d.cap = L.cap;
  d.natoms = L.natoms;
  d.nclusters = L.nclusters;
  d.npad = L.npad;
  d.nsuper = L.nsuper;
  d.sys = nullptr;
  d.cl_sys = nullptr;
  d.sup_sys = nullptr;
  d.shape = nullptr;
  return d;
}

// Index of cell (x0, x1, x2) along the 3-D Hilbert curve of a 2^b grid, from J. Skilling,
// "Programming the Hilbert curve", AIP Conf. Proc. 707, 381 (2004): the axes are turned
// into the transposed Hilbert index (inverse undo, then Gray encoding), whose bits are
// interleaved with x0 most significant. Unlike the Morton (Z-order) curve, consecutive
// Hilbert cells are always face neighbours, so a run of 32 atoms never jumps across the box.
__device__ __forceinline__ unsigned hilbert_key(unsigned x0, unsigned x1, unsigned x2, int b) {
  if (b <= 0) return 0u;
  unsigned X[3] = {x0, x1, x2};
  const unsigned M = 1u << (b - 1);
  for (unsigned Q = M; Q > 1u; Q >>= 1) {
    const unsigned P = Q - 1u;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      if (X[i] & Q) {
        X[0] ^= P;
      } else {
        const unsigned t = (X[0] ^ X[i]) & P;
        X[0] ^= t;
        X[i] ^= t;
      }
    }
  }
  X[1] ^= X[0];
  X[2] ^= X[1];
  unsigned t = 0u;
  for (unsigned Q = M; Q > 1u; Q >>= 1)
    if (X[2] & Q) t ^= Q - 1u;
  X[0] ^= t;
  X[1] ^= t;
  X[2] ^= t;
  unsigned key = 0u;
  for (int bit = b - 1; bit >= 0; --bit)
    key = (key << 3) | (((X[0] >> bit) & 1u) << 2) | (((X[1] >> bit) & 1u) << 1) | ((X[2] >> bit) & 1u);
  return key;
}

// Box facts used by the cluster search: inverse, orthorhombic flag, perpendicular widths.
template <class T>
__device__ void write_box_info(const T *box, double *info) {
  Box b;
  load_box(box, b);
  for (int k = 0; k < 9; ++k) {
    info[k] = b.m[k];
    info[9 + k] = b.inv[k];
  }
  const double *m = b.m;
  bool ortho = m[1] == 0.0 && m[2] == 0.0 && m[3] == 0.0 && m[5] == 0.0 && m[6] == 0.0 && m[7] == 0.0;
  info[18] = ortho ? 1.0 : 0.0;
  // width along lattice direction d = V / |cross of the other two rows|
  for (int d = 0; d < 3; ++d) {
    const double *u = m + 3 * ((d + 1) % 3);
    const double *v = m + 3 * ((d + 2) % 3);
    double cx = u[1] * v[2] - u[2] * v[1], cy = u[2] * v[0] - u[0] * v[2], cz = u[0] * v[1] - u[1] * v[0];
    info[19 + d] = b.vol / sqrt(cx * cx + cy * cy + cz * cz);
  }
}

// Box facts of one system; the grid also clears `nz` 8-byte words at `z` and `nz2` at `z2`.
template <class T>
__global__ void box_info_kernel(const T *box, double *info, unsigned long long *z = nullptr, int64_t nz = 0,
                                unsigned long long *z2 = nullptr, int64_t nz2 = 0) {
  pdl_enter();
  if (threadIdx.x == 0 && blockIdx.x == 0) write_box_info(box, info);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nz; k += stride) z[k] = 0ull;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nz2; k += stride) z2[k] = 0ull;
}

// Exclusive scan of hist[0..nkeys) in place; hist[nkeys] = total. One block of 1024
// threads; thread t owns a contiguous segment, so the work is two sweeps of the segment
// plus one block-wide scan of the segment sums.
__device__ __forceinline__ void scan_keys_body(unsigned *hist, int64_t nkeys) {
  __shared__ unsigned s_warp[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  // segments of whole 4-key chunks read as uint4 (hist is 16-byte aligned), several loads in
  // flight per thread
  const int64_t per = ((nkeys + blockDim.x - 1) / blockDim.x + 3) & ~int64_t(3);
  const int64_t beg = min((int64_t)threadIdx.x * per, nkeys), end = min(beg + per, nkeys);
  const int64_t vend = beg + ((end - beg) & ~int64_t(3));
  const uint4 *h4 = reinterpret_cast<const uint4 *>(hist);
  unsigned sum = 0;
#pragma unroll 4
  for (int64_t k = beg; k < vend; k += 4) {
    const uint4 v = h4[k >> 2];
    sum += v.x + v.y + v.z + v.w;
  }
  for (int64_t k = vend; k < end; ++k) sum += hist[k];
  unsigned incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned y = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) s_warp[w] = incl;
  __syncthreads();
  if (w == 0) {
    const unsigned t = (lane < (int)(blockDim.x >> 5)) ? s_warp[lane] : 0u;
    unsigned ti = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned y = __shfl_up_sync(kFull, ti, o);
      if (lane >= o) ti += y;
    }
    s_warp[lane] = ti - t;  // exclusive warp offsets
  }
  __syncthreads();
  unsigned run = s_warp[w] + incl - sum;
  uint4 *o4 = reinterpret_cast<uint4 *>(hist);
#pragma unroll 4
  for (int64_t k = beg; k < vend; k += 4) {
    const uint4 v = h4[k >> 2];
    uint4 o;
    o.x = run;
    run += v.x;
    o.y = run;
    run += v.y;
    o.z = run;
    run += v.z;
    o.w = run;
    run += v.w;
    o4[k >> 2] = o;
  }
  for (int64_t k = vend; k < end; ++k) {
    const unsigned v = hist[k];
    hist[k] = run;
    run += v;
  }
  if (threadIdx.x == blockDim.x - 1) hist[nkeys] = run;
}

template <class T>
// With scan_nkeys > 0 (small systems) the last block to finish also scans the histogram
// (status[4] is its block ticket, zeroed per build), which saves the scan launch.
__global__ void cell_keys_kernel(const T *x, int64_t n, ClusterData<T> d, int64_t scan_nkeys) {
  pdl_enter();
  const double *inv = d.boxinfo + 9;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double rx = x[3 * i], ry = x[3 * i + 1], rz = x[3 * i + 2];
    double f[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double v = rx * inv[c] + ry * inv[3 + c] + rz * inv[6 + c];
      v -= floor(v);
      if (v >= 1.0) v = 0.0;  // guards rounding of tiny negatives
      f[c] = v;
    }
    unsigned cell[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) cell[c] = min((unsigned)(f[c] * d.nc), (unsigned)(d.nc - 1));
    const unsigned key = hilbert_key(cell[0], cell[1], cell[2], d.bits);
    d.keys[i] = key;
    atomicAdd(&d.hist[key], 1u);
  }
  if (scan_nkeys <= 0) return;
  __shared__ bool s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(&d.status[4], 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  scan_keys_body(d.hist, scan_nkeys);
}

static __global__ void scan_keys_kernel(unsigned *hist, int64_t nkeys) {
  pdl_enter();
  scan_keys_body(hist, nkeys);
}

template <class T>
__global__ void scatter_atoms_kernel(int64_t n, ClusterData<T> d) {
  pdl_enter();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    unsigned key = d.keys[i];
    unsigned slot = d.hist[key] + atomicAdd(&d.fill[key], 1u);
    d.tmp[slot] = (int)i;
  }
}

// One warp per key bucket: each atom's slot is its rank (by atom index) inside the bucket,
// found by warp-wide counting, which gives a deterministic order with no serial chain;
// then the sorted SoA is written. q may be NULL (charge slot = 0).
template <class T>
__global__ void sort_buckets_kernel(const T *x, const T *q, int64_t nkeys, ClusterData<T> d) {
  pdl_enter();
  const double *m = d.boxinfo;
  const double *inv = d.boxinfo + 9;
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t k = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); k < nkeys; k += nw) {
    const unsigned b0 = d.hist[k], cnt = d.hist[k + 1] - b0;
    for (unsigned base = 0; base < cnt; base += kWarp) {
      const bool has = base + lane < cnt;
      const int v = has ? d.tmp[b0 + base + lane] : INT_MAX;
      unsigned rank = 0;
      for (unsigned cb = 0; cb < cnt; cb += kWarp) {
        const int other = (cb + lane < cnt) ? d.tmp[b0 + cb + lane] : INT_MAX;
#pragma unroll 8
        for (int s = 0; s < kWarp; ++s) rank += (__shfl_sync(kFull, other, s) < v) ? 1u : 0u;
      }
      if (has) {
        const unsigned slot = b0 + rank;
        const double rx = x[3 * v], ry = x[3 * v + 1], rz = x[3 * v + 2];
        double f[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          double w = rx * inv[c] + ry * inv[3 + c] + rz * inv[6 + c];
          w -= floor(w);
          if (w >= 1.0) w = 0.0;
          f[c] = w;
        }
        const double wx = f[0] * m[0] + f[1] * m[3] + f[2] * m[6];
        const double wy = f[0] * m[1] + f[1] * m[4] + f[2] * m[7];
        const double wz = f[0] * m[2] + f[1] * m[5] + f[2] * m[8];
        d.pos[slot] = make_v4((T)wx, (T)wy, (T)wz, q ? q[v] : T(0));
        d.frac[slot] = make_v4((T)f[0], (T)f[1], (T)f[2], T(0));
        d.sidx[slot] = v;
        d.inv[v] = (int)slot;
      }
    }
  }
  // padding slots
  const int64_t gstride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t s = d.natoms + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < d.npad; s += gstride) {
    d.sidx[s] = -1;
    d.pos[s] = make_v4(T(0), T(0), T(0), T(0));
    d.frac[s] = make_v4(T(0), T(0), T(0), T(0));
  }
}

// Batch mode, steps 1-5 in one launch: one block per system bins its atoms on the
// system's own Hilbert-ordered cell grid in shared memory (counting sort, then an
// insertion sort of each bucket by atom index, which makes the order deterministic and
// equal to the single-system sort), writes the sorted SoA with padding to whole clusters
// and the cluster / super-cluster owners, and zeroes the energy kernel's accumulators of
// those slots (acc: dE/dx of slots_cap slots, then dE/dq). The system count comes from
// d.shape. Limits: kBatchMaxAtoms atoms and
// kBatchMaxKeys keys per system (16 cells per side).
constexpr int kBatchSortThreads = 1024;
constexpr int kBatchMaxAtoms = 16384;
constexpr int kBatchMaxKeys = 4096;
constexpr size_t kBatchSortSmem = (2 * kBatchMaxKeys + 1) * sizeof(unsigned) + 2 * kBatchMaxAtoms * sizeof(unsigned short);

template <class T>
__global__ void __launch_bounds__(kBatchSortThreads) batch_sort_kernel(const T *x, const T *q, const T *boxes,
                                                                       ClusterData<T> d, unsigned long long *acc,
                                                                       int64_t slots_cap) {
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned *hist = reinterpret_cast<unsigned *>(smem);          // kBatchMaxKeys + 1
  unsigned *fill = hist + kBatchMaxKeys + 1;                     // kBatchMaxKeys
  unsigned short *lkey = reinterpret_cast<unsigned short *>(fill + kBatchMaxKeys);  // atom -> key
  unsigned short *order = lkey + kBatchMaxAtoms;                 // sorted position -> atom
  __shared__ double s_info[kInfoStride];
  __shared__ unsigned s_warp[32];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int nsys = d.shape->nsys;
  for (int sy = blockIdx.x; sy < nsys; sy += gridDim.x) {
    const BatchSys b = d.sys[sy];
    const int n = (int)b.natoms;
    const int nkeys = 1 << (3 * b.bits);
    const T *xs = x + 3 * b.atom_off;
    if (tid == 0) {
      write_box_info(boxes + 9 * (int64_t)sy, s_info);
      for (int k = 0; k < kInfoStride; ++k) d.boxinfo[(int64_t)kInfoStride * sy + k] = s_info[k];
    }
    for (int k = tid; k <= nkeys; k += blockDim.x) hist[k] = 0u;
    for (int k = tid; k < nkeys; k += blockDim.x) fill[k] = 0u;
    __syncthreads();
    const double *inv = s_info + 9;
    for (int t = tid; t < n; t += blockDim.x) {
      const double rx = xs[3 * t], ry = xs[3 * t + 1], rz = xs[3 * t + 2];
      unsigned cell[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        double v = rx * inv[c] + ry * inv[3 + c] + rz * inv[6 + c];
        v -= floor(v);
        if (v >= 1.0) v = 0.0;
        cell[c] = min((unsigned)(v * b.nc), (unsigned)(b.nc - 1));
      }
      const unsigned key = hilbert_key(cell[0], cell[1], cell[2], b.bits);
      lkey[t] = (unsigned short)key;
      atomicAdd(&hist[key], 1u);
    }
    __syncthreads();
    // exclusive scan of hist[0, nkeys): thread t owns kBatchMaxKeys / blockDim.x entries
    {
      const int per = (nkeys + blockDim.x - 1) / blockDim.x;
      const int beg = min(tid * per, nkeys), end = min(beg + per, nkeys);
      unsigned sum = 0u;
      for (int k = beg; k < end; ++k) sum += hist[k];
      unsigned incl = sum;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += y;
      }
      if (lane == 31) s_warp[w] = incl;
      __syncthreads();
      if (w == 0) {
        const unsigned v = lane < (int)(blockDim.x >> 5) ? s_warp[lane] : 0u;
        unsigned vi = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const unsigned y = __shfl_up_sync(kFull, vi, o);
          if (lane >= o) vi += y;
        }
        s_warp[lane] = vi - v;
      }
      __syncthreads();
      unsigned run = s_warp[w] + incl - sum;
      for (int k = beg; k < end; ++k) {
        const unsigned v = hist[k];
        hist[k] = run;
        run += v;
      }
      if (tid == 0) hist[nkeys] = (unsigned)n;
    }
    __syncthreads();
    for (int t = tid; t < n; t += blockDim.x) {
      const unsigned key = lkey[t];
      order[hist[key] + atomicAdd(&fill[key], 1u)] = (unsigned short)t;
    }
    __syncthreads();
    for (int k = tid; k < nkeys; k += blockDim.x) {
      const int b0 = (int)hist[k], b1 = (int)hist[k + 1];
      for (int i = b0 + 1; i < b1; ++i) {
        const unsigned short v = order[i];
        int j = i - 1;
        while (j >= b0 && order[j] > v) {
          order[j + 1] = order[j];
          --j;
        }
        order[j + 1] = v;
      }
    }
    __syncthreads();
    const double *m = s_info;
    const int64_t base = b.cl_off * kWarp;
    const int npad = (int)(b.ncl * kWarp);
    for (int p = tid; p < npad; p += blockDim.x) {
      const int64_t slot = base + p;
      // the energy kernel's accumulators of the slot: dE/dx (3 per slot), then dE/dq
      acc[3 * slot] = 0ull;
      acc[3 * slot + 1] = 0ull;
      acc[3 * slot + 2] = 0ull;
      acc[3 * slots_cap + slot] = 0ull;
      if (p < n) {
        const int t = order[p];
        const int64_t a = b.atom_off + t;
        const double rx = xs[3 * t], ry = xs[3 * t + 1], rz = xs[3 * t + 2];
        double f[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          double v = rx * inv[c] + ry * inv[3 + c] + rz * inv[6 + c];
          v -= floor(v);
          if (v >= 1.0) v = 0.0;
          f[c] = v;
        }
        const double wx = f[0] * m[0] + f[1] * m[3] + f[2] * m[6];
        const double wy = f[0] * m[1] + f[1] * m[4] + f[2] * m[7];
        const double wz = f[0] * m[2] + f[1] * m[5] + f[2] * m[8];
        d.pos[slot] = make_v4((T)wx, (T)wy, (T)wz, q ? q[a] : T(0));
        d.frac[slot] = make_v4((T)f[0], (T)f[1], (T)f[2], T(0));
        d.sidx[slot] = (int)a;
        d.inv[a] = (int)slot;
      } else {
        d.sidx[slot] = -1;
        d.pos[slot] = make_v4(T(0), T(0), T(0), T(0));
        d.frac[slot] = make_v4(T(0), T(0), T(0), T(0));
      }
    }
    for (int c = tid; c < b.ncl; c += blockDim.x) d.cl_sys[b.cl_off + c] = sy;
    for (int c = tid; c < b.nsup; c += blockDim.x) d.sup_sys[b.sup_off + c] = sy;
    __syncthreads();
  }
}

// One warp per cluster: bounding box in fractional coordinates. The box is taken around
// the first atom's image so that a cluster straddling the periodic boundary stays compact,
// and the cluster's positions are rewritten as that same contiguous image (anchor +
// nearest-image offset), so that one periodic shift serves a whole cluster pair.
// A block of kSuper warps covers one super-cluster and, once its member boxes are known,
// takes their union around the first member's centre (members shifted to their nearest
// image of it) and widens it by 1e-5 to cover the rounding of centres to T.
template <class T>
__global__ void __launch_bounds__(kWarp * kSuper) cluster_bounds_kernel(ClusterData<T> d) {
  pdl_enter();
  __shared__ double s_box[kSuper][6];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t nsuper = d.n_super();
  for (int64_t S = blockIdx.x; S < nsuper; S += gridDim.x) {
    // members [first, last) of super-cluster S, all in one system
    int64_t first = S * kSuper, last = min(first + kSuper, d.n_clusters());
    int sy = 0;
    if (d.sys) {
      sy = d.sup_sys[S];
      const BatchSys &b = d.sys[sy];
      first = b.cl_off + (S - b.sup_off) * kSuper;
      last = min(first + kSuper, b.cl_off + b.ncl);
    }
    const double *m = d.info(sy);
    const int64_t c = first + w;
    if (c < last) {
      const int64_t s = c * kWarp + lane;
      const bool valid = d.sidx[s] >= 0;
      auto f = d.frac[s];
      T fx = f.x, fy = f.y, fz = f.z;
      const T ax = __shfl_sync(kFull, fx, 0), ay = __shfl_sync(kFull, fy, 0), az = __shfl_sync(kFull, fz, 0);
      fx -= ax; fy -= ay; fz -= az;
      fx -= floor(fx + T(0.5)); fy -= floor(fy + T(0.5)); fz -= floor(fz + T(0.5));
      if (valid) {
        const double ux = (double)ax + (double)fx, uy = (double)ay + (double)fy, uz = (double)az + (double)fz;
        auto p = d.pos[s];
        p.x = (T)(ux * m[0] + uy * m[3] + uz * m[6]);
        p.y = (T)(ux * m[1] + uy * m[4] + uz * m[7]);
        p.z = (T)(ux * m[2] + uy * m[5] + uz * m[8]);
        d.pos[s] = p;
      }
      T lo[3] = {valid ? fx : T(1e30), valid ? fy : T(1e30), valid ? fz : T(1e30)};
      T hi[3] = {valid ? fx : T(-1e30), valid ? fy : T(-1e30), valid ? fz : T(-1e30)};
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          lo[k] = min(lo[k], __shfl_xor_sync(kFull, lo[k], o));
          hi[k] = max(hi[k], __shfl_xor_sync(kFull, hi[k], o));
        }
      }
      if (lane == 0) {
        const auto cc = make_v4(ax + T(0.5) * (lo[0] + hi[0]), ay + T(0.5) * (lo[1] + hi[1]),
                                az + T(0.5) * (lo[2] + hi[2]), T(0));
        const auto hh = make_v4(T(0.5) * (hi[0] - lo[0]), T(0.5) * (hi[1] - lo[1]), T(0.5) * (hi[2] - lo[2]), T(0));
        d.bc[c] = cc;
        d.bh[c] = hh;
        s_box[w][0] = cc.x; s_box[w][1] = cc.y; s_box[w][2] = cc.z;
        s_box[w][3] = hh.x; s_box[w][4] = hh.y; s_box[w][5] = hh.z;
      }
    }
    __syncthreads();
    if (w == 0) {
      const bool v = first + lane < last;
      double lo[3], hi[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const double ref = s_box[0][k];
        double u = v ? s_box[lane][k] - ref : 0.0;
        u -= floor(u + 0.5);
        lo[k] = v ? ref + u - s_box[lane][3 + k] : 1e30;
        hi[k] = v ? ref + u + s_box[lane][3 + k] : -1e30;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          lo[k] = fmin(lo[k], __shfl_xor_sync(kFull, lo[k], o));
          hi[k] = fmax(hi[k], __shfl_xor_sync(kFull, hi[k], o));
        }
      }
      if (lane == 0) {
        d.sbc[S] = make_v4((T)(0.5 * (lo[0] + hi[0])), (T)(0.5 * (lo[1] + hi[1])), (T)(0.5 * (lo[2] + hi[2])), T(0));
        d.sbh[S] = make_v4((T)(0.5 * (hi[0] - lo[0]) + 1e-5), (T)(0.5 * (hi[1] - lo[1]) + 1e-5),
                           (T)(0.5 * (hi[2] - lo[2]) + 1e-5), T(0));
      }
    }
    __syncthreads();
  }
}

// Conservative cluster-pair test on fractional boxes: per axis, the gap between the two
// intervals on the periodic unit circle (nearest image of the centres), converted to a
// distance with the box (exact for orthorhombic, perpendicular widths otherwise). The gap
// only shrinks when one box grows, so a super-cluster's union box that fails the test
// proves that every member fails it too.
template <class T>
__device__ __forceinline__ bool clusters_may_interact(const typename V4<T>::type &ci, const typename V4<T>::type &hi,
                                                      const typename V4<T>::type &cj, const typename V4<T>::type &hj,
                                                      const double *info, double rc) {
  double g[3];
  double dc[3] = {(double)ci.x - (double)cj.x, (double)ci.y - (double)cj.y, (double)ci.z - (double)cj.z};
  double hs[3] = {(double)hi.x + (double)hj.x, (double)hi.y + (double)hj.y, (double)hi.z + (double)hj.z};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    double v = dc[k] - floor(dc[k] + 0.5);
    // 1e-6 margin in fractional units absorbs the FP32 rounding of centres and extents
    g[k] = fmax(0.0, fabs(v) - hs[k] - 1e-6);
  }
  if (info[18] != 0.0) {
    double x = g[0] * info[0], y = g[1] * info[4], z = g[2] * info[8];
    return x * x + y * y + z * z <= rc * rc;
  }
  double m = fmax(g[0] * info[19], fmax(g[1] * info[20], g[2] * info[21]));
  return m <= rc;
}

// The same test in FP32 for float boxes: the box facts of the system are converted once
// (box diagonal for orthorhombic boxes, perpendicular widths otherwise) and the margin is
// 2e-6 in fractional units, above the FP32 rounding of centres, extents and the arithmetic
// (a few 1e-7), so the test stays conservative.
struct BoxTestF {
  float s[3];  // orthorhombic: box lengths; otherwise perpendicular widths
  float lim;   // orthorhombic: rc^2 (1 + 1e-6); otherwise rc (1 + 1e-6)
  bool ortho;
};

__device__ __forceinline__ BoxTestF box_test_f(const double *info, double rc) {
  BoxTestF b;
  b.ortho = info[18] != 0.0;
  b.s[0] = (float)(b.ortho ? info[0] : info[19]);
  b.s[1] = (float)(b.ortho ? info[4] : info[20]);
  b.s[2] = (float)(b.ortho ? info[8] : info[21]);
  b.lim = (float)(b.ortho ? rc * rc * (1.0 + 1e-6) : rc * (1.0 + 1e-6));
  return b;
}

__device__ __forceinline__ bool boxes_may_interact_f(const float4 &ci, const float4 &hi, const float4 &cj,
                                                     const float4 &hj, const BoxTestF &b) {
  const float dc[3] = {ci.x - cj.x, ci.y - cj.y, ci.z - cj.z};
  const float hs[3] = {hi.x + hj.x, hi.y + hj.y, hi.z + hj.z};
  float g[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float v = dc[k] - floorf(dc[k] + 0.5f);
    g[k] = fmaxf(0.f, fabsf(v) - hs[k] - 2e-6f) * b.s[k];
  }
  if (b.ortho) return g[0] * g[0] + g[1] * g[1] + g[2] * g[2] <= b.lim;
  return fmaxf(g[0], fmaxf(g[1], g[2])) <= b.lim;
}

template <class T>
__global__ void cluster_neighbors_kernel(ClusterData<T> d, double rc, int half) {
  pdl_enter();
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
  const int64_t ncl = d.n_clusters();
  for (int64_t I = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); I < ncl; I += nw) {
    const auto ci = d.bc[I];
    const auto hi = d.bh[I];
    int count = 0;
    // candidates: clusters [j0, jend) and super-clusters [s0, send) of I's system
    int64_t j0 = 0, j1 = ncl, s0 = 0;
    int sy = 0;
    if (d.sys) {
      sy = d.cl_sys[I];
      const BatchSys &b = d.sys[sy];
      j0 = b.cl_off;
      j1 = b.cl_off + b.ncl;
      s0 = b.sup_off;
    }
    const double *info = d.info(sy);
    BoxTestF bt{};
    if constexpr (sizeof(T) == 4) bt = box_test_f(info, rc);
    auto test = [&](const typename V4<T>::type &cj, const typename V4<T>::type &hj) {
      if constexpr (sizeof(T) == 4)
        return boxes_may_interact_f(ci, hi, cj, hj, bt);
      else
        return clusters_may_interact<T>(ci, hi, cj, hj, info, rc);
    };
    const int64_t jend = half ? (I + 1) : j1;
    const int64_t send = s0 + (jend - j0 + kSuper - 1) / kSuper;
    // Lanes screen 32 super-clusters at a time; the members of each survivor (one per lane,
    // kSuper == kWarp) are then tested in ascending order, so the list is sorted by J. The
    // member boxes of up to kBatch survivors are loaded before any of them is tested, so a
    // warp waits for one round of loads per kBatch survivors rather than per survivor.
    constexpr int kBatch = 4;
    using V = typename V4<T>::type;
    for (int64_t sb = s0; sb < send; sb += kWarp) {
      const int64_t S = sb + lane;
      const bool sok = S < send && test(d.sbc[S], d.sbh[S]);
      unsigned sm = __ballot_sync(kFull, sok);
      while (sm) {
        int64_t Jb[kBatch];
        V cb[kBatch], hb[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
          Jb[u] = -1;
          if (sm) {
            const int k = __ffs(sm) - 1;
            sm &= sm - 1u;
            const int64_t J = j0 + (sb + k - s0) * kSuper + lane;
            if (J < jend) {
              Jb[u] = J;
              cb[u] = d.bc[J];
              hb[u] = d.bh[J];
            }
          }
        }
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
          const bool ok = Jb[u] >= 0 && test(cb[u], hb[u]);
          const unsigned mm = __ballot_sync(kFull, ok);
          if (ok) {
            const int r = count + __popc(mm & ((1u << lane) - 1u));
            if (r < d.cap) d.nbr[I * d.cap + r] = (int)Jb[u];
          }
          count += __popc(mm);
        }
      }
    }
    if (lane == 0) {
      d.ncount[I] = min(count, d.cap);
      if (count > d.cap) atomicOr(&d.status[0], 1u);
    }
  }
  // The last block to finish turns the counts into work-item offsets (exclusive prefix
  // sums of ceil(count / kItemTiles)); status[1] is the block ticket (zeroed per build).
  // The item -> cluster table is filled by the sorted-parameter kernel that follows.
  __shared__ bool s_last;
  __shared__ int s_warp[32];
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(&d.status[1], 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  const int64_t n = ncl;
  const int64_t per = (n + blockDim.x - 1) / blockDim.x;
  const int64_t beg = min((int64_t)threadIdx.x * per, n), end = min(beg + per, n);
  int sum = 0;
  for (int64_t k = beg; k < end; ++k) sum += (__ldcg(&d.ncount[k]) + kItemTiles - 1) / kItemTiles;
  int incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += y;
  }
  const int w = threadIdx.x >> 5;
  if (lane == 31) s_warp[w] = incl;
  __syncthreads();
  if (w == 0) {
    const int t = (lane < (int)(blockDim.x >> 5)) ? s_warp[lane] : 0;
    int ti = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(kFull, ti, o);
      if (lane >= o) ti += y;
    }
    s_warp[lane] = ti - t;
  }
  __syncthreads();
  int run = s_warp[w] + incl - sum;
  for (int64_t k = beg; k < end; ++k) {
    d.itemoff[k] = run;
    run += (__ldcg(&d.ncount[k]) + kItemTiles - 1) / kItemTiles;
  }
  if (threadIdx.x == blockDim.x - 1) d.itemoff[n] = run;
}

// Host driver for steps 1-6 on `stream`. `zero` (`zero_bytes`, a multiple of 8) is cleared
// on the way. With `pdl` every kernel after the first is a programmatic dependent launch.
template <class T>
int build_clusters(const ClusterLayout &L, const ClusterData<T> &d, void *ws, const T *x, const T *q,
                   const T *box, double rc, int half, cudaStream_t s, void *zero = nullptr, size_t zero_bytes = 0,
                   bool pdl = false) {
  const int sms = sm_count();
  const int64_t nz = (int64_t)(L.zero_bytes / 8);
  const int nb_zero = (int)std::max<int64_t>(1, std::min<int64_t>((nz + 1023) / 1024, sms));
  int st = launch_k(false, box_info_kernel<T>, nb_zero, 256, 0, s, box, d.boxinfo,
                    reinterpret_cast<unsigned long long *>(static_cast<char *>(ws) + L.zero_off), nz,
                    static_cast<unsigned long long *>(zero), (int64_t)(zero_bytes / 8));
  if (st != TFF_OK) return st;
  if (L.natoms == 0) return TFF_OK;
  const int nb_atoms = (int)std::max<int64_t>(1, std::min<int64_t>((L.natoms + 255) / 256, sms * 8));
  // up to kFusedScanMaxKeys keys the last block of the key kernel scans the histogram
  const bool fused_scan = L.nkeys <= kFusedScanMaxKeys;
  if ((st = launch_k(pdl, cell_keys_kernel<T>, nb_atoms, 256, 0, s, x, L.natoms, d,
                     (int64_t)(fused_scan ? L.nkeys : 0))) != TFF_OK)
    return st;
  if (!fused_scan && (st = launch_k(pdl, scan_keys_kernel, 1, 1024, 0, s, d.hist, L.nkeys)) != TFF_OK) return st;
  if ((st = launch_k(pdl, scatter_atoms_kernel<T>, nb_atoms, 256, 0, s, L.natoms, d)) != TFF_OK) return st;
  const int nb_keys = (int)std::max<int64_t>(1, std::min<int64_t>((L.nkeys + 3) / 4, sms * 32));
  if ((st = launch_k(pdl, sort_buckets_kernel<T>, nb_keys, 128, 0, s, x, q, L.nkeys, d)) != TFF_OK) return st;
  const int nb_cl = (int)std::max<int64_t>(1, std::min<int64_t>((L.nclusters + 3) / 4, sms * 16));
  const int nb_super = (int)std::max<int64_t>(1, std::min<int64_t>(L.nsuper, sms * 2));
  if ((st = launch_k(pdl, cluster_bounds_kernel<T>, nb_super, kWarp * kSuper, 0, s, d)) != TFF_OK) return st;
  return launch_k(pdl, cluster_neighbors_kernel<T>, nb_cl, 128, 0, s, d, rc, half);
}

}  // namespace tff

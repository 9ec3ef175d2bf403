// Neighbour lists: the drop-in kernels behind build_neighbor_list_nsquared(_out) and
// build_neighbor_list_cell_list(_out).
//
// Output contract (both): pairs (cap, 2) int64 filled with -1, found pairs written as
// (larger index, smaller index) in arbitrary order, *npairs = number found (may exceed cap).
// Pairs are compacted per warp into a shared-memory buffer that is flushed with one
// global atomic per flush (order of pairs in the output is not deterministic; the SET is).
#include <climits>

#include "cluster.cuh"

namespace tff {
namespace {

constexpr int kNsqBlock = 256;
constexpr int kBufPairs = 128;  // per-warp staging buffer (pairs)

__device__ __forceinline__ bool is_excluded(int64_t i, int64_t j, const int64_t *row_ptr, const int64_t *col) {
  if (col == nullptr) return false;
  for (int64_t e = row_ptr[i]; e < row_ptr[i + 1]; ++e)
    if (col[e] == j) return true;
  return false;
}

// Warp-cooperative staging of found pairs. All 32 lanes must call push() together.
struct PairStage {
  int64_t *buf;  // 2 * kBufPairs
  int count;
  int64_t *out;
  int64_t cap;
  int32_t *counter;

  __device__ __forceinline__ void flush(int lane) {
    __syncwarp();
    int start = 0;
    if (lane == 0 && count > 0) start = atomicAdd(counter, count);
    start = __shfl_sync(kFull, start, 0);
    for (int k = lane; k < count; k += kWarp) {
      const int64_t dst = (int64_t)start + k;
      if (dst < cap) {
        out[2 * dst] = buf[2 * k];
        out[2 * dst + 1] = buf[2 * k + 1];
      }
    }
    __syncwarp();
    count = 0;
  }
  __device__ __forceinline__ void push(bool ok, int64_t a, int64_t b, int lane) {
    const unsigned m = __ballot_sync(kFull, ok);
    if (m == 0u) return;
    if (count + __popc(m) > kBufPairs) flush(lane);
    if (ok) {
      const int r = count + __popc(m & ((1u << lane) - 1u));
      buf[2 * r] = a > b ? a : b;
      buf[2 * r + 1] = a > b ? b : a;
    }
    count += __popc(m);
  }
};

// FP64 re-test of a candidate pair from the caller's (unwrapped) coordinates, with the
// same minimum-image arithmetic as the FP64 path.
template <class T>
__device__ __forceinline__ bool within_fp64(const T *x, int64_t i, int64_t j, const double *m, const double *inv,
                                            bool periodic, double rc2) {
  double dx = (double)x[3 * i] - (double)x[3 * j];
  double dy = (double)x[3 * i + 1] - (double)x[3 * j + 1];
  double dz = (double)x[3 * i + 2] - (double)x[3 * j + 2];
  if (periodic) min_image(dx, dy, dz, m, inv);
  return dx * dx + dy * dy + dz * dz <= rc2;
}

// Decides |r| <= rc for a candidate whose squared distance r2 was computed in T.
template <class T>
__device__ __forceinline__ bool cutoff_test(T r2, T rc2t, const T *x, int64_t i, int64_t j, const double *m,
                                            const double *inv, bool periodic, double rc2) {
  if (sizeof(T) == 8) return r2 <= rc2t;
  const T tol = T(1e-5) * rc2t;
  if (r2 < rc2t - tol) return true;
  if (r2 > rc2t + tol) return false;
  return within_fp64(x, i, j, m, inv, periodic, rc2);
}

// Tiled O(N^2): one block per (i-tile, j-tile) pair with j-tile <= i-tile, j-tile in smem.
template <class T>
__global__ void __launch_bounds__(kNsqBlock) nsquared_kernel(const T *x, const T *box, int64_t n, double rc,
                                                             const int64_t *row_ptr, const int64_t *col,
                                                             int include_self, int64_t *pairs, int64_t cap,
                                                             int32_t *npairs) {
  __shared__ T s_x[kNsqBlock], s_y[kNsqBlock], s_z[kNsqBlock];
  __shared__ int64_t s_buf[(kNsqBlock / kWarp) * 2 * kBufPairs];
  __shared__ double s_m[9], s_inv[9];
  __shared__ T s_mt[9], s_invt[9];
  const bool periodic = box != nullptr;
  if (threadIdx.x == 0 && periodic) {
    Box b;
    load_box(box, b);
    for (int k = 0; k < 9; ++k) {
      s_m[k] = b.m[k];
      s_inv[k] = b.inv[k];
      s_mt[k] = (T)b.m[k];
      s_invt[k] = (T)b.inv[k];
    }
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  PairStage st{s_buf + w * 2 * kBufPairs, 0, pairs, cap, npairs};
  const double rc2 = rc * rc;
  const T rc2t = (T)rc2;
  const int64_t ntiles = (n + kNsqBlock - 1) / kNsqBlock;
  const int64_t ntp = ntiles * (ntiles + 1) / 2;
  for (int64_t tp = blockIdx.x; tp < ntp; tp += gridDim.x) {
    // tile pair index -> (I, J), J <= I
    int64_t I = (int64_t)floor((sqrt(8.0 * (double)tp + 1.0) - 1.0) * 0.5);
    while (I * (I + 1) / 2 > tp) --I;
    while ((I + 1) * (I + 2) / 2 <= tp) ++I;
    const int64_t J = tp - I * (I + 1) / 2;
    __syncthreads();
    const int64_t jl = J * kNsqBlock + threadIdx.x;
    if (jl < n) {
      s_x[threadIdx.x] = x[3 * jl];
      s_y[threadIdx.x] = x[3 * jl + 1];
      s_z[threadIdx.x] = x[3 * jl + 2];
    }
    __syncthreads();
    const int64_t i = I * kNsqBlock + threadIdx.x;
    const bool ivalid = i < n;
    T xi = T(0), yi = T(0), zi = T(0);
    if (ivalid) {
      xi = x[3 * i];
      yi = x[3 * i + 1];
      zi = x[3 * i + 2];
    }
    const int64_t jcount = min((int64_t)kNsqBlock, n - J * kNsqBlock);
    for (int jj = 0; jj < jcount; ++jj) {
      const int64_t j = J * kNsqBlock + jj;
      bool ok = ivalid && (j < i || (include_self && j == i));
      if (ok) {
        T dx = xi - s_x[jj], dy = yi - s_y[jj], dz = zi - s_z[jj];
        if (periodic) min_image(dx, dy, dz, s_mt, s_invt);
        const T r2 = dx * dx + dy * dy + dz * dz;
        ok = cutoff_test<T>(r2, rc2t, x, i, j, s_m, s_inv, periodic, rc2);
        if (ok) ok = !is_excluded(i, j, row_ptr, col);
      }
      st.push(ok, i, j, lane);
    }
  }
  st.flush(lane);
}

// Cell-list emit: one warp per (cluster I, chunk of its half neighbour list).
constexpr int kEmitChunk = 4;
constexpr int kEmitBlock = 128;

template <class T>
__global__ void __launch_bounds__(kEmitBlock) cell_emit_kernel(ClusterData<T> d, const T *x, double rc,
                                                               const int64_t *row_ptr, const int64_t *col,
                                                               int include_self, int64_t *pairs, int64_t cap,
                                                               int32_t *npairs) {
  using V = typename V4<T>::type;
  constexpr int W = kEmitBlock / kWarp;
  __shared__ V s_pos[W][kWarp];
  __shared__ int s_idx[W][kWarp];
  __shared__ int64_t s_buf[W * 2 * kBufPairs];
  __shared__ double s_m[9], s_inv[9];
  __shared__ T s_mt[9], s_invt[9];
  __shared__ int s_ortho;
  if (threadIdx.x < 9) {
    s_m[threadIdx.x] = d.boxinfo[threadIdx.x];
    s_inv[threadIdx.x] = d.boxinfo[9 + threadIdx.x];
    s_mt[threadIdx.x] = (T)d.boxinfo[threadIdx.x];
    s_invt[threadIdx.x] = (T)d.boxinfo[9 + threadIdx.x];
  }
  if (threadIdx.x == 0) s_ortho = d.boxinfo[18] != 0.0;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  PairStage st{s_buf + w * 2 * kBufPairs, 0, pairs, cap, npairs};
  const double rc2 = rc * rc;
  const T rc2t = (T)rc2;
  const T Lx = s_mt[0], Ly = s_mt[4], Lz = s_mt[8];
  const T iLx = s_invt[0], iLy = s_invt[4], iLz = s_invt[8];
  const bool ortho = s_ortho;
  const int nchunks = (d.cap + kEmitChunk - 1) / kEmitChunk;
  const int64_t nitems = d.nclusters * nchunks;
  const int64_t nw = (int64_t)gridDim.x * W;
  for (int64_t item = (int64_t)blockIdx.x * W + w; item < nitems; item += nw) {
    const int64_t I = item / nchunks;
    const int c0 = (int)(item % nchunks) * kEmitChunk;
    const int cnt = d.ncount[I];
    if (c0 >= cnt) continue;
    const int64_t si = I * kWarp + lane;
    const int ai = d.sidx[si];
    const V pi = d.pos[si];
    const int c1 = min(cnt, c0 + kEmitChunk);
    for (int c = c0; c < c1; ++c) {
      const int J = d.nbr[I * d.cap + c];
      __syncwarp();
      s_pos[w][lane] = d.pos[(int64_t)J * kWarp + lane];
      s_idx[w][lane] = d.sidx[(int64_t)J * kWarp + lane];
      __syncwarp();
      for (int s = 0; s < kWarp; ++s) {
        const int aj = s_idx[w][s];
        bool ok = ai >= 0 && aj >= 0;
        if (J == I) ok = ok && (lane > s || (include_self && lane == s));
        if (ok) {
          const V pj = s_pos[w][s];
          T dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
          if (ortho) {
            dx = wrap1(dx, Lx, iLx);
            dy = wrap1(dy, Ly, iLy);
            dz = wrap1(dz, Lz, iLz);
          } else {
            min_image(dx, dy, dz, s_mt, s_invt);
          }
          const T r2 = dx * dx + dy * dy + dz * dz;
          ok = cutoff_test<T>(r2, rc2t, x, ai, aj, s_m, s_inv, true, rc2);
          if (ok) ok = !is_excluded(ai, aj, row_ptr, col);
        }
        st.push(ok, ai, aj, lane);
      }
    }
  }
  st.flush(lane);
}

// Marks an overflowing cluster list: the caller sees npairs > cap.
__global__ void cluster_overflow_kernel(const unsigned *status, int32_t *npairs) {
  if (threadIdx.x == 0 && blockIdx.x == 0 && (status[0] & 1u)) npairs[0] = INT_MAX;
}

int default_cluster_cap(int64_t nclusters, int requested) {
  if (requested > 0) return requested;
  return (int)std::max<int64_t>(1, std::min<int64_t>(nclusters, 1024));
}

template <class T>
int nsquared_impl(int64_t natoms, const T *x, const T *box, double cutoff, const int64_t *rp,
                  const int64_t *col, int include_self, int64_t *pairs, int64_t cap, int32_t *npairs,
                  cudaStream_t s) {
  if (cap > 0) TFF_CUDA(cudaMemsetAsync(pairs, 0xff, sizeof(int64_t) * 2 * cap, s));
  TFF_CUDA(cudaMemsetAsync(npairs, 0, sizeof(int32_t), s));
  if (natoms == 0) return TFF_OK;
  const int64_t ntiles = (natoms + kNsqBlock - 1) / kNsqBlock;
  const int64_t ntp = ntiles * (ntiles + 1) / 2;
  const int nb = (int)std::max<int64_t>(1, std::min<int64_t>(ntp, (int64_t)sm_count() * 8));
  nsquared_kernel<T><<<nb, kNsqBlock, 0, s>>>(x, box, natoms, cutoff, rp, col, include_self, pairs, cap, npairs);
  TFF_LAUNCHED();
  return TFF_OK;
}

template <class T>
int cell_list_impl(int64_t natoms, const T *x, const T *box, double cutoff, const int64_t *rp, const int64_t *col,
                   int include_self, int64_t *pairs, int64_t cap, int32_t *npairs, int ccap, void *ws,
                   size_t ws_bytes, cudaStream_t s) {
  const int dtype = sizeof(T) == 8 ? TFF_F64 : TFF_F32;
  const int64_t ncl = (natoms + kWarp - 1) / kWarp;
  ClusterLayout L = cluster_layout(dtype, natoms, default_cluster_cap(ncl, ccap));
  if (ws == nullptr || ws_bytes < L.bytes) {
    set_error("workspace too small: need %zu bytes, got %zu", L.bytes, ws_bytes);
    return TFF_ERR_WORKSPACE;
  }
  if (cap > 0) TFF_CUDA(cudaMemsetAsync(pairs, 0xff, sizeof(int64_t) * 2 * cap, s));
  TFF_CUDA(cudaMemsetAsync(npairs, 0, sizeof(int32_t), s));
  if (natoms == 0) return TFF_OK;
  ClusterData<T> d = cluster_data<T>(L, ws);
  int st = build_clusters<T>(L, d, ws, x, nullptr, box, cutoff, /*half=*/1, s);
  if (st != TFF_OK) return st;
  const int nchunks = (L.cap + kEmitChunk - 1) / kEmitChunk;
  const int64_t items = L.nclusters * nchunks;
  const int nb = (int)std::max<int64_t>(1, std::min<int64_t>((items + 3) / 4, (int64_t)sm_count() * 16));
  cell_emit_kernel<T><<<nb, kEmitBlock, 0, s>>>(d, x, cutoff, rp, col, include_self, pairs, cap, npairs);
  TFF_LAUNCHED();
  cluster_overflow_kernel<<<1, 32, 0, s>>>(d.status, npairs);
  TFF_LAUNCHED();
  return TFF_OK;
}

}  // namespace
}  // namespace tff

using namespace tff;

extern "C" {

int tff_nblist_nsquared(int dtype, int64_t natoms, const void *coords, const void *box, double cutoff,
                        const int64_t *excl_row_ptr, const int64_t *excl_col, int include_self, int64_t *pairs,
                        int64_t max_npairs, int32_t *npairs, tff_stream_t stream) {
  TFF_NVTX("tff_nblist_nsquared");
  TFF_ARG(dtype == TFF_F32 || dtype == TFF_F64, "dtype must be TFF_F32 or TFF_F64");
  TFF_ARG(natoms >= 0 && max_npairs >= 0, "negative sizes");
  TFF_ARG(npairs != nullptr, "npairs is NULL");
  TFF_ARG(pairs != nullptr || max_npairs == 0, "pairs is NULL");
  TFF_ARG(coords != nullptr || natoms == 0, "coords is NULL");
  TFF_ARG((excl_row_ptr == nullptr) == (excl_col == nullptr), "exclusion CSR needs both arrays");
  TFF_ARG(cutoff >= 0.0, "cutoff must be >= 0");
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == TFF_F32)
    return nsquared_impl<float>(natoms, (const float *)coords, (const float *)box, cutoff, excl_row_ptr, excl_col,
                                include_self, pairs, max_npairs, npairs, s);
  return nsquared_impl<double>(natoms, (const double *)coords, (const double *)box, cutoff, excl_row_ptr, excl_col,
                               include_self, pairs, max_npairs, npairs, s);
}

size_t tff_nblist_cell_list_workspace_bytes(int dtype, int64_t natoms, int max_cluster_neighbors) {
  const int64_t ncl = (natoms + kWarp - 1) / kWarp;
  return cluster_layout(dtype, natoms, default_cluster_cap(ncl, max_cluster_neighbors)).bytes;
}

int tff_nblist_cell_list(int dtype, int64_t natoms, const void *coords, const void *box, double cutoff,
                         const int64_t *excl_row_ptr, const int64_t *excl_col, int include_self, int64_t *pairs,
                         int64_t max_npairs, int32_t *npairs, int max_cluster_neighbors, void *workspace,
                         size_t workspace_bytes, tff_stream_t stream) {
  TFF_NVTX("tff_nblist_cell_list");
  TFF_ARG(dtype == TFF_F32 || dtype == TFF_F64, "dtype must be TFF_F32 or TFF_F64");
  TFF_ARG(box != nullptr, "Cell-list neighbor list requires a periodic box");
  TFF_ARG(natoms >= 0 && max_npairs >= 0, "negative sizes");
  TFF_ARG(npairs != nullptr, "npairs is NULL");
  TFF_ARG(pairs != nullptr || max_npairs == 0, "pairs is NULL");
  TFF_ARG(coords != nullptr || natoms == 0, "coords is NULL");
  TFF_ARG((excl_row_ptr == nullptr) == (excl_col == nullptr), "exclusion CSR needs both arrays");
  TFF_ARG(cutoff >= 0.0, "cutoff must be >= 0");
  TFF_ARG(natoms < (int64_t)INT_MAX, "too many atoms");
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == TFF_F32)
    return cell_list_impl<float>(natoms, (const float *)coords, (const float *)box, cutoff, excl_row_ptr, excl_col,
                                 include_self, pairs, max_npairs, npairs, max_cluster_neighbors, workspace,
                                 workspace_bytes, s);
  return cell_list_impl<double>(natoms, (const double *)coords, (const double *)box, cutoff, excl_row_ptr, excl_col,
                                include_self, pairs, max_npairs, npairs, max_cluster_neighbors, workspace,
                                workspace_bytes, s);
}

}  // extern "C"

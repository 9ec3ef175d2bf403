// Fused fixed-charge system: one evaluation = cluster build (full neighbour-cluster lists)
// -> fused real-space tile kernel (LJ with Lorentz-Berthelot combining + erfc-screened
// Coulomb, Ewald exclusion correction) -> PME (spread, FFT, influence function, FFT,
// gather) -> forces in caller order. It evaluates the nonbonded terms of
// examples/tip3p/model.py:100-133 (NeighborList + Vdw + MultipolarInteraction(rank 0) +
// PME) without materialising an int64 pair list.
//
// Tile kernel: one warp per (cluster I, chunk of kTileChunk clusters J of I's FULL list).
// Lane l owns atom l of I; the 32 atoms of J are staged in shared memory and read with
// broadcast loads, so every lane sweeps all 32 j atoms. Each pair is therefore evaluated
// from both sides, which removes j-side atomics: forces/charge gradients of atom i are
// summed in registers (FP32 per tile, FP64 across tiles) and added once per chunk into
// int64 fixed-point accumulators (mixed) or FP64 atomics (FP64 mode). Energies are halved.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "pme.cuh"

namespace tff {
namespace {

constexpr int kMaxExcl = 8;       // excluded partners per atom (self excluded)
constexpr int kTileChunk = 8;     // J clusters per warp work item
constexpr int kTileBlock = 128;

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
  const int *excl;                 // (N, kMaxExcl) original partner indices, -1 padded
  typename Acc<T>::S *gx;          // (npad, 3) sorted slots, dE/dx
  typename Acc<T>::S *gq;          // (npad) sorted slots, dE/dq
  double rc, alpha, kc;
  double *partials;
  unsigned *tickets;
  double *energies;                // [0] pairs (LJ + erfc Coulomb), [1] exclusion correction
};

// LB parameters in sorted order.
template <class T>
__global__ void sorted_lj_kernel(ClusterData<T> cl, const T *sigma, const T *eps, typename V2<T>::type *lj) {
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < cl.npad; s += (int64_t)gridDim.x * blockDim.x) {
    const int a = cl.sidx[s];
    lj[s] = a >= 0 ? make_v2(T(0.5) * sigma[a], (T)sqrt((double)eps[a])) : make_v2(T(0), T(0));
  }
}

template <class T>
__global__ void __launch_bounds__(kTileBlock) tile_kernel(TileArgs<T> A) {
  using V = typename V4<T>::type;
  using W2 = typename V2<T>::type;
  constexpr int NW = kTileBlock / kWarp;
  __shared__ V s_pos[NW][kWarp];
  __shared__ W2 s_lj[NW][kWarp];
  __shared__ T s_box[6];
  const ClusterData<T> &cl = A.cl;
  if (threadIdx.x < 3) {
    s_box[threadIdx.x] = (T)cl.boxinfo[4 * threadIdx.x];          // L_x, L_y, L_z
    s_box[3 + threadIdx.x] = (T)cl.boxinfo[9 + 4 * threadIdx.x];  // 1/L
  }
  __shared__ T s_m[9], s_inv[9];
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
  const T Lx = s_box[0], Ly = s_box[1], Lz = s_box[2], iLx = s_box[3], iLy = s_box[4], iLz = s_box[5];
  double e_pair = 0.0, e_excl = 0.0;

  const int nchunks = (cl.cap + kTileChunk - 1) / kTileChunk;
  const int64_t nitems = cl.nclusters * nchunks;
  const int64_t nwarps = (int64_t)gridDim.x * NW;
  for (int64_t item = (int64_t)blockIdx.x * NW + w; item < nitems; item += nwarps) {
    const int64_t I = item / nchunks;
    const int c0 = (int)(item % nchunks) * kTileChunk;
    const int cnt = cl.ncount[I];
    if (c0 >= cnt) continue;
    const int c1 = min(cnt, c0 + kTileChunk);
    const int64_t si = I * kWarp + lane;
    const int ai = cl.sidx[si];
    const bool vi = ai >= 0;
    const V pi = cl.pos[si];
    const W2 lji = A.lj[si];
    const T qi = pi.w;
    int ex[kMaxExcl];
#pragma unroll
    for (int k = 0; k < kMaxExcl; ++k) {
      const int pa = vi ? A.excl[(int64_t)ai * kMaxExcl + k] : -1;
      ex[k] = pa >= 0 ? cl.inv[pa] : -1;
    }
    double fx = 0.0, fy = 0.0, fz = 0.0, dq = 0.0;
    for (int c = c0; c < c1; ++c) {
      const int J = cl.nbr[I * cl.cap + c];
      const int64_t sj = (int64_t)J * kWarp + lane;
      __syncwarp();
      s_pos[w][lane] = cl.pos[sj];
      s_lj[w][lane] = A.lj[sj];
      const unsigned jvalid = __ballot_sync(kFull, cl.sidx[sj] >= 0);
      __syncwarp();
      unsigned emask = 0u;
#pragma unroll
      for (int k = 0; k < kMaxExcl; ++k)
        if (ex[k] >= 0 && (ex[k] >> 5) == J) emask |= 1u << (ex[k] & 31);
      unsigned skip = ~jvalid;
      if (J == (int)I) skip |= 1u << lane;
      if (!vi) skip = kFull;
      T tfx = T(0), tfy = T(0), tfz = T(0), tdq = T(0), te = T(0);
#pragma unroll 4
      for (int s = 0; s < kWarp; ++s) {
        const V pj = s_pos[w][s];
        T dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
        if (ortho) {
          dx = wrap1(dx, Lx, iLx);
          dy = wrap1(dy, Ly, iLy);
          dz = wrap1(dz, Lz, iLz);
        } else {
          min_image(dx, dy, dz, s_m, s_inv);
        }
        const T r2 = dx * dx + dy * dy + dz * dz;
        const bool in = !((skip >> s) & 1u) && (r2 <= rc2);
        if (!__any_sync(kFull, in)) continue;
        const bool is_ex = (emask >> s) & 1u;
        const T r2s = in ? r2 : T(1);
        const T rinv = rsqrt_t(r2s);
        const T rinv2 = rinv * rinv;
        const T r = r2s * rinv;
        const T u = alpha * r;
        T ec, ex2;
        erfc_exp(u, ec, ex2);
        T damp = ec;
        if (is_ex) damp = -erf_t(u);  // erfc(u) - 1, computed directly
        const T qq = kc * qi * pj.w;
        const T ecoul = qq * damp * rinv;
        T dedr_r = -qq * (damp * rinv2 + two_a_rpi * ex2 * rinv) * rinv;
        const W2 ljj = s_lj[w][s];
        const T sig = lji.x + ljj.x;
        const T eps = is_ex ? T(0) : lji.y * ljj.y;
        const T sr2 = sig * sig * rinv2;
        const T sr6 = sr2 * sr2 * sr2;
        const T elj = T(4) * eps * sr6 * (sr6 - T(1));
        dedr_r -= T(24) * eps * sr6 * (T(2) * sr6 - T(1)) * rinv2;
        if (in) {
          tfx += dedr_r * dx;
          tfy += dedr_r * dy;
          tfz += dedr_r * dz;
          tdq += kc * pj.w * damp * rinv;
          if (is_ex) e_excl += 0.5 * (double)ecoul;
          else te += ecoul + elj;
        }
      }
      fx += (double)tfx;
      fy += (double)tfy;
      fz += (double)tfz;
      dq += (double)tdq;
      e_pair += 0.5 * (double)te;
    }
    if (vi) {
      Acc<T>::add(&A.gx[3 * si], fx);
      Acc<T>::add(&A.gx[3 * si + 1], fy);
      Acc<T>::add(&A.gx[3 * si + 2], fz);
      Acc<T>::add(&A.gq[si], dq);
    }
  }
  grid_sum<kTileBlock>(e_pair, A.partials, A.tickets, A.energies, false);
  grid_sum<kTileBlock>(e_excl, A.partials + 4096, A.tickets + 1, A.energies + 1, false);
}

// Sorted accumulators -> caller order; energies.
template <class T>
__global__ void finalize_kernel(ClusterData<T> cl, const typename Acc<T>::S *gx, const typename Acc<T>::S *gq,
                                T *forces, double *forces64, T *grad_q, const double *e_tile, const double *e_pme,
                                double kc, double *energy, double *terms) {
  for (int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; a < cl.natoms;
       a += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = cl.inv[a];
    const double x = Acc<T>::get(&gx[3 * s]), y = Acc<T>::get(&gx[3 * s + 1]), z = Acc<T>::get(&gx[3 * s + 2]);
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
    if (grad_q) grad_q[a] = (T)Acc<T>::get(&gq[s]);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
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
  void *cl_ws = nullptr;
  void *pme_ws = nullptr;
  void *acc = nullptr;         // gx (npad*3), gq (npad): zeroed per evaluation
  size_t acc_bytes = 0;
  void *lj = nullptr;          // sorted (sigma/2, sqrt eps)
  void *q = nullptr, *sigma = nullptr, *eps = nullptr;  // per-atom, system dtype
  int *excl = nullptr;         // (N, kMaxExcl)
  void *moduli = nullptr;      // xmod (K), ymod (K), zmod (K/2+1)
  double *scratch = nullptr;   // partials (8192), tickets (64 u32), energies (8)
  void *host_x = nullptr;      // device staging for *_host: coords64 (3N) + box64 (9)
  void *dev_x = nullptr;       // coords/box in system dtype for *_host
  double *dev_f = nullptr;     // forces64 for *_host
  double *dev_e = nullptr;
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
  auto mark = [&](int k) { return ev ? record_event(ev[k], s) : TFF_OK; };
  int st = mark(0);
  if (st != TFF_OK) return st;
  ClusterData<T> cd = cluster_data<T>(sys->cl, sys->cl_ws);
  st = build_clusters<T>(sys->cl, cd, sys->cl_ws, x, static_cast<const T *>(sys->q), box, sys->desc.cutoff,
                         /*half=*/0, s);
  if (st != TFF_OK) return st;
  if ((st = mark(1)) != TFF_OK) return st;
  S *gx = static_cast<S *>(sys->acc);
  S *gq = gx + 3 * sys->cl.npad;
  char *scr = reinterpret_cast<char *>(sys->scratch);
  double *partials = reinterpret_cast<double *>(scr);
  unsigned *tickets = reinterpret_cast<unsigned *>(scr + 8192 * sizeof(double));
  double *energies = reinterpret_cast<double *>(scr + 8192 * sizeof(double) + 256);
  TFF_CUDA(cudaMemsetAsync(sys->acc, 0, sys->acc_bytes, s));
  TFF_CUDA(cudaMemsetAsync(tickets, 0, 256 + 8 * sizeof(double), s));
  const int sms = sm_count();
  auto *lj = static_cast<typename V2<T>::type *>(sys->lj);
  if (n > 0) {
    const int nb = (int)std::max<int64_t>(1, std::min<int64_t>((sys->cl.npad + 255) / 256, sms * 8));
    sorted_lj_kernel<T><<<nb, 256, 0, s>>>(cd, static_cast<const T *>(sys->sigma), static_cast<const T *>(sys->eps),
                                           lj);
    TFF_LAUNCHED();
    TileArgs<T> A;
    A.cl = cd;
    A.lj = lj;
    A.excl = sys->excl;
    A.gx = gx;
    A.gq = gq;
    A.rc = sys->desc.cutoff;
    A.alpha = sys->desc.ewald_alpha;
    A.kc = sys->desc.coul_constant;
    A.partials = partials;
    A.tickets = tickets;
    A.energies = energies;
    const int nchunks = (sys->cl.cap + kTileChunk - 1) / kTileChunk;
    const int64_t items = sys->cl.nclusters * nchunks;
    const int nbt = (int)std::max<int64_t>(1, std::min<int64_t>((items + 3) / 4, (int64_t)sms * 16));
    tile_kernel<T><<<nbt, kTileBlock, 0, s>>>(A);
    TFF_LAUNCHED();
  }
  if ((st = mark(2)) != TFF_OK) return st;
  const double *e_pme = nullptr;
  if (sys->pme && n > 0) {
    const int K = sys->desc.pme_grid;
    const T *xm = static_cast<const T *>(sys->moduli);
    const T *ym = xm + K;
    const T *zm = ym + K;
    char *pw = static_cast<char *>(sys->pme_ws);
    SortedAtoms<T> atoms{cd.pos, cd.sidx, cd.npad};
    T *phi_grid = nullptr;
    st = pme_grid_phase<T>(sys->pme->impl, sys->pl, pw, atoms, cd.npad, box, sys->desc.ewald_alpha, xm, ym, zm, s,
                           &phi_grid);
    if (st != TFF_OK) return st;
    if ((st = mark(3)) != TFF_OK) return st;
    SortedGatherOut<T> out{gx, gq, sys->desc.coul_constant};
    st = pme_gather_phase<T>(sys->pme->impl, sys->pl, pw, atoms, cd.npad, box, sys->desc.ewald_alpha, phi_grid, out,
                             1.0, (T *)nullptr, s);
    if (st != TFF_OK) return st;
    e_pme = reinterpret_cast<const double *>(pw + sys->pl.energies);
  } else {
    if ((st = mark(3)) != TFF_OK) return st;
  }
  if ((st = mark(4)) != TFF_OK) return st;
  const int nbf = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, sms * 8));
  finalize_kernel<T><<<nbf, 256, 0, s>>>(cd, gx, gq, forces, forces64, grad_q, energies, e_pme,
                                         sys->desc.coul_constant, energy, terms);
  TFF_LAUNCHED();
  return mark(5);
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
  void *ptrs[] = {sys->cl_ws, sys->pme_ws, sys->acc, sys->lj, sys->q, sys->sigma, sys->eps, sys->excl,
                  sys->moduli, sys->scratch, sys->host_x, sys->dev_x, sys->dev_f, sys->dev_e};
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
                                             : (int)std::max<int64_t>(1, std::min<int64_t>(ncl, 512));
  sys->cl = cluster_layout(desc->dtype, n, sys->cap);
  const size_t ts = desc->dtype == TFF_F64 ? 8 : 4;
#define TFF_ALLOC(ptr, bytes)                                   \
  do {                                                          \
    cudaError_t _e = cudaMalloc((void **)&(ptr), (bytes) ? (bytes) : 256); \
    if (_e != cudaSuccess) {                                    \
      free_system(sys);                                         \
      return cuda_fail(_e, "cudaMalloc", __FILE__, __LINE__);   \
    }                                                           \
  } while (0)
  TFF_ALLOC(sys->cl_ws, sys->cl.bytes);
  sys->acc_bytes = (size_t)sys->cl.npad * 4 * 8;
  TFF_ALLOC(sys->acc, sys->acc_bytes);
  TFF_ALLOC(sys->lj, (size_t)sys->cl.npad * 2 * ts);
  TFF_ALLOC(sys->q, n * ts);
  TFF_ALLOC(sys->sigma, n * ts);
  TFF_ALLOC(sys->eps, n * ts);
  TFF_ALLOC(sys->excl, ex.size() * sizeof(int));
  TFF_ALLOC(sys->scratch, 8192 * sizeof(double) + 256 + 8 * sizeof(double));
  TFF_ALLOC(sys->host_x, (3 * n + 9) * sizeof(double));
  TFF_ALLOC(sys->dev_x, (3 * n + 9) * ts);
  TFF_ALLOC(sys->dev_f, 3 * n * sizeof(double));
  TFF_ALLOC(sys->dev_e, 8 * sizeof(double));
  cudaError_t e = cudaSuccess;
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
    return cuda_fail(e, "upload", __FILE__, __LINE__);
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
  if (n > 0) TFF_CUDA(cudaMemcpyAsync(stage, coords, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s));
  TFF_CUDA(cudaMemcpyAsync(stage + 3 * n, box, 9 * sizeof(double), cudaMemcpyHostToDevice, s));
  int st;
  const int nb = (int)std::max<int64_t>(1, std::min<int64_t>((3 * n + 255) / 256, sm_count() * 8));
  if (sys->desc.dtype == TFF_F32) {
    float *x = static_cast<float *>(sys->dev_x);
    cast_inputs_kernel<float><<<nb, 256, 0, s>>>(stage, stage + 3 * n, x, x + 3 * n, 3 * n);
    TFF_LAUNCHED();
    st = system_eval_impl<float>(sys, x, x + 3 * n, sys->dev_e, nullptr, sys->dev_f, nullptr, nullptr, s);
  } else {
    double *x = static_cast<double *>(sys->dev_x);
    cast_inputs_kernel<double><<<nb, 256, 0, s>>>(stage, stage + 3 * n, x, x + 3 * n, 3 * n);
    TFF_LAUNCHED();
    st = system_eval_impl<double>(sys, x, x + 3 * n, sys->dev_e, nullptr, sys->dev_f, nullptr, nullptr, s);
  }
  if (st != TFF_OK) return st;
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
  // cluster build 7 + sorted LJ 1 + tile 1 + finalize 1; PME: spread, [to_real], convolve, gather
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

// Pair terms over an explicit (P, 2) pair list: the drop-in kernels behind
// compute_nonbonded_energy_from_atom_pairs, compute_nonbonded_forces_from_atom_pairs,
// compute_coulomb_energy, compute_lennard_jones_energy and rank-0
// compute_multipolar_energy_from_atom_pairs.
//
// One thread per pair (grid-stride over a grid sized to a fixed multiple of the SM
// count, so the work partition - and with it every summation order - is fixed).
// Energies: per-thread FP64, fixed-order block and grid reduction. Gradients: int64
// fixed-point atomics in mixed precision (order-independent, bit-reproducible), FP64
// atomics in FP64 mode.
#include <math.h>

#include <mutex>

#include <cuda.h>   // driver types only: cuCtxGetCurrent / cuCtxGetId are reached via the runtime

#include "tff_common.cuh"

namespace tff {
namespace {

enum CoulMode { C_NONE = 0, C_SHIFT = 1, C_PLAIN = 2, C_EWALD = 3 };
enum LjMode { L_NONE = 0, L_ATOM = 1, L_PAIR = 2, L_TYPE = 3 };

constexpr int kPairBlock = 256;

template <class T>
struct PairArgs {
  const T *x;
  const int64_t *pairs;
  int64_t npairs;
  const int64_t *excl;
  int64_t nexcl;
  const T *box;
  const T *q;
  const T *sig;
  const T *eps;
  const int64_t *types;
  int64_t ntypes;
  double k, rc, alpha;
  typename Acc<T>::S *gx, *gq, *gs, *ge;  // accumulators (nullable)
  T *gs_pair, *ge_pair;                   // per-pair parameter gradients (L_PAIR)
  double *partials;
  unsigned *ticket;
  double *energy;
};

__device__ __forceinline__ float erfc_t(float x) { return erfcf(x); }
__device__ __forceinline__ double erfc_t(double x) { return erfc(x); }
__device__ __forceinline__ float exp_t(float x) { return expf(x); }
__device__ __forceinline__ double exp_t(double x) { return exp(x); }
__device__ __forceinline__ float rsqrt_t(float x) { return rsqrtf(x); }
__device__ __forceinline__ double rsqrt_t(double x) { return rsqrt(x); }
__device__ __forceinline__ float sqrt_t(float x) { return sqrtf(x); }
__device__ __forceinline__ double sqrt_t(double x) { return sqrt(x); }

template <class T, int CM, int LM>
__global__ void __launch_bounds__(kPairBlock) pair_kernel(PairArgs<T> a) {
  using A = Acc<T>;
  __shared__ T s_m[9], s_inv[9];
  const bool periodic = a.box != nullptr;
  if (threadIdx.x == 0 && periodic) {
    Box b;
    load_box(a.box, b);
    for (int k = 0; k < 9; ++k) {
      s_m[k] = (T)b.m[k];
      s_inv[k] = (T)b.inv[k];
    }
  }
  __syncthreads();

  const T rc = (T)a.rc;
  const T rc2 = rc * rc;
  const T kc = (T)a.k;
  const T inv_rc = T(1) / rc;
  const T alpha = (T)a.alpha;
  const T two_a_rpi = (T)(2.0 * a.alpha / 1.7724538509055160273);
  double e_acc = 0.0;

  const int64_t total = a.npairs + ((CM == C_EWALD) ? a.nexcl : 0);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += stride) {
    const bool is_excl = (CM == C_EWALD) && (t >= a.npairs);
    const int64_t p = is_excl ? (t - a.npairs) : t;
    const int64_t *pl = is_excl ? a.excl : a.pairs;
    const int64_t i = pl[2 * p], j = pl[2 * p + 1];
    if (i < 0 || j < 0) continue;
    T dx = a.x[3 * i] - a.x[3 * j];
    T dy = a.x[3 * i + 1] - a.x[3 * j + 1];
    T dz = a.x[3 * i + 2] - a.x[3 * j + 2];
    if (periodic) min_image(dx, dy, dz, s_m, s_inv);
    const T r2 = dx * dx + dy * dy + dz * dz;
    if (!(r2 <= rc2)) continue;
    const T rinv = rsqrt_t(r2);
    const T rinv2 = rinv * rinv;
    T e = T(0);
    T dedr_over_r = T(0);  // (dE/dr) / r

    if (CM != C_NONE) {
      const T qi = a.q[i], qj = a.q[j];
      T f;       // energy per unit k q_i q_j
      T dfdr_r;  // (df/dr) / r
      if (CM == C_SHIFT) {
        f = rinv - inv_rc;
        dfdr_r = -rinv2 * rinv;
      } else if (CM == C_PLAIN) {
        f = rinv;
        dfdr_r = -rinv2 * rinv;
      } else {
        const T r = r2 * rinv;
        const T u = alpha * r;
        T damp = erfc_t(u);
        if (is_excl) damp -= T(1);
        f = damp * rinv;
        dfdr_r = -(damp * rinv2 + two_a_rpi * exp_t(-u * u) * rinv) * rinv;
      }
      e += kc * qi * qj * f;
      dedr_over_r += kc * qi * qj * dfdr_r;
      if (a.gq) {
        A::add(&a.gq[i], (double)(kc * qj * f));
        A::add(&a.gq[j], (double)(kc * qi * f));
      }
    }

    if (LM != L_NONE && !is_excl) {
      T s, ep, sqe_i = T(0), sqe_j = T(0);
      int64_t tidx = 0;
      if (LM == L_ATOM) {
        s = T(0.5) * (a.sig[i] + a.sig[j]);
        sqe_i = a.eps[i];
        sqe_j = a.eps[j];
        ep = sqrt_t(sqe_i * sqe_j);
      } else if (LM == L_PAIR) {
        s = a.sig[p];
        ep = a.eps[p];
      } else {
        tidx = a.types[i] * a.ntypes + a.types[j];
        s = a.sig[tidx];
        ep = a.eps[tidx];
      }
      const T sr2 = s * s * rinv2;
      const T sr6 = sr2 * sr2 * sr2;
      e += T(4) * ep * sr6 * (sr6 - T(1));
      const T g = T(24) * ep * sr6 * (T(2) * sr6 - T(1));  // = -r dE/dr = s dE/ds
      dedr_over_r -= g * rinv2;
      const T de_ds = g / s;
      const T de_de = T(4) * sr6 * (sr6 - T(1));
      if (LM == L_ATOM) {
        if (a.gs) {
          A::add(&a.gs[i], 0.5 * (double)de_ds);
          A::add(&a.gs[j], 0.5 * (double)de_ds);
        }
        if (a.ge && ep > T(0)) {
          const T h = de_de / (T(2) * ep);
          A::add(&a.ge[i], (double)(h * sqe_j));
          A::add(&a.ge[j], (double)(h * sqe_i));
        }
      } else if (LM == L_PAIR) {
        if (a.gs_pair) a.gs_pair[p] = de_ds;
        if (a.ge_pair) a.ge_pair[p] = de_de;
      } else {
        if (a.gs) A::add(&a.gs[tidx], (double)de_ds);
        if (a.ge) A::add(&a.ge[tidx], (double)de_de);
      }
    }

    e_acc += (double)e;
    if (a.gx) {
      const double fx = (double)(dedr_over_r * dx), fy = (double)(dedr_over_r * dy),
                   fz = (double)(dedr_over_r * dz);
      A::add(&a.gx[3 * i], fx);
      A::add(&a.gx[3 * i + 1], fy);
      A::add(&a.gx[3 * i + 2], fz);
      A::add(&a.gx[3 * j], -fx);
      A::add(&a.gx[3 * j + 1], -fy);
      A::add(&a.gx[3 * j + 2], -fz);
    }
  }
  grid_sum<kPairBlock>(e_acc, a.partials, a.ticket, a.energy, false);
}

// Converts accumulators into the caller's arrays: out[k] = scale * acc[k] (or += when add).
template <class T>
__global__ void acc_to_out(const typename Acc<T>::S *acc, T *out, int64_t n, double scale, bool add) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x) {
    double v = scale * Acc<T>::get(&acc[k]);
    out[k] = add ? (T)((double)out[k] + v) : (T)v;
  }
}

template <class T>
__global__ void energy_out(const double *e, T *out, double prefactor) {
  out[0] = (T)(prefactor * e[0]);
}

struct PairLayout {
  size_t bytes;
  size_t acc_off, acc_bytes;  // zeroed region
  size_t gx, gq, gs, ge;      // element offsets (in accumulator units) inside the acc region
  size_t partials, ticket, energy;
};

PairLayout pair_layout(int dtype, int64_t natoms, int64_t ntypes) {
  const size_t es = 8;  // both accumulator types are 8 bytes
  PairLayout L{};
  const size_t npar = (size_t)std::max<int64_t>(natoms, ntypes * ntypes);
  L.gx = 0;
  L.gq = 3 * (size_t)natoms;
  L.gs = L.gq + (size_t)natoms;
  L.ge = L.gs + npar;
  size_t nacc = L.ge + npar;
  L.acc_off = 0;
  L.acc_bytes = ((nacc * es) + 255) & ~size_t(255);
  L.partials = L.acc_bytes;
  const size_t max_blocks = 8 * 1024;
  L.ticket = L.partials + max_blocks * sizeof(double);
  L.energy = L.ticket + 256;
  L.bytes = L.energy + 256;
  (void)dtype;
  return L;
}

int grid_blocks(int64_t work) {
  int64_t want = (work + kPairBlock - 1) / kPairBlock;
  int64_t cap = (int64_t)sm_count() * 8;
  if (want < 1) want = 1;
  return (int)std::min(want, cap);
}

template <class T, int CM, int LM>
int launch_pairs(PairArgs<T> a, int64_t total, cudaStream_t s) {
  pair_kernel<T, CM, LM><<<grid_blocks(total), kPairBlock, 0, s>>>(a);
  TFF_LAUNCHED();
  return TFF_OK;
}

template <class T>
int dispatch_pairs(int cm, int lm, const PairArgs<T> &a, int64_t total, cudaStream_t s) {
#define TFF_PAIR_CASE(C, L) \
  if (cm == C && lm == L) return launch_pairs<T, C, L>(a, total, s);
  TFF_PAIR_CASE(C_SHIFT, L_ATOM)
  TFF_PAIR_CASE(C_PLAIN, L_ATOM)
  TFF_PAIR_CASE(C_SHIFT, L_NONE)
  TFF_PAIR_CASE(C_PLAIN, L_NONE)
  TFF_PAIR_CASE(C_EWALD, L_NONE)
  TFF_PAIR_CASE(C_NONE, L_PAIR)
  TFF_PAIR_CASE(C_NONE, L_TYPE)
#undef TFF_PAIR_CASE
  set_error("unsupported pair-term combination");
  return TFF_ERR_INVALID;
}

// Common driver: zero accumulators, run the pair kernel, convert outputs.
struct PairCall {
  int dtype;
  int cm, lm;
  int64_t natoms, npairs, nexcl, ntypes;
  const void *x, *box, *q, *sig, *eps;
  const int64_t *pairs, *excl, *types;
  double k, rc, alpha;
  void *energy;       // T scalar (nullable)
  double e_scale;
  void *gx; double gx_scale; bool gx_add;
  void *gq, *gs, *ge; // T outputs (per atom / per table / per pair)
  void *ws; size_t ws_bytes;
};

template <class T>
int run_pairs(const PairCall &c, cudaStream_t s) {
  using S = typename Acc<T>::S;
  PairLayout L = pair_layout(c.dtype, c.natoms, c.ntypes);
  if (c.ws_bytes < L.bytes || c.ws == nullptr) {
    set_error("workspace too small: need %zu bytes, got %zu", L.bytes, c.ws_bytes);
    return TFF_ERR_WORKSPACE;
  }
  char *ws = static_cast<char *>(c.ws);
  S *acc = reinterpret_cast<S *>(ws + L.acc_off);
  TFF_CUDA(cudaMemsetAsync(ws, 0, L.acc_bytes, s));
  TFF_CUDA(cudaMemsetAsync(ws + L.ticket, 0, 256, s));
  PairArgs<T> a{};
  a.x = static_cast<const T *>(c.x);
  a.pairs = c.pairs;
  a.npairs = c.npairs;
  a.excl = c.excl;
  a.nexcl = c.nexcl;
  a.box = static_cast<const T *>(c.box);
  a.q = static_cast<const T *>(c.q);
  a.sig = static_cast<const T *>(c.sig);
  a.eps = static_cast<const T *>(c.eps);
  a.types = c.types;
  a.ntypes = c.ntypes;
  a.k = c.k;
  a.rc = c.rc;
  a.alpha = c.alpha;
  a.gx = c.gx ? acc + L.gx : nullptr;
  a.gq = c.gq ? acc + L.gq : nullptr;
  const bool per_pair = (c.lm == L_PAIR);
  a.gs = (c.gs && !per_pair) ? acc + L.gs : nullptr;
  a.ge = (c.ge && !per_pair) ? acc + L.ge : nullptr;
  a.gs_pair = per_pair ? static_cast<T *>(c.gs) : nullptr;
  a.ge_pair = per_pair ? static_cast<T *>(c.ge) : nullptr;
  if (per_pair) {
    if (c.gs) TFF_CUDA(cudaMemsetAsync(c.gs, 0, sizeof(T) * c.npairs, s));
    if (c.ge) TFF_CUDA(cudaMemsetAsync(c.ge, 0, sizeof(T) * c.npairs, s));
  }
  a.partials = reinterpret_cast<double *>(ws + L.partials);
  a.ticket = reinterpret_cast<unsigned *>(ws + L.ticket);
  a.energy = reinterpret_cast<double *>(ws + L.energy);
  const int64_t total = c.npairs + (c.cm == C_EWALD ? c.nexcl : 0);
  int st = dispatch_pairs<T>(c.cm, c.lm, a, total, s);
  if (st != TFF_OK) return st;
  const int nb = std::max(1, std::min(sm_count() * 4, (int)((3 * c.natoms + 255) / 256)));
  if (c.gx) {
    acc_to_out<T><<<nb, 256, 0, s>>>(a.gx, static_cast<T *>(c.gx), 3 * c.natoms, c.gx_scale, c.gx_add);
    TFF_LAUNCHED();
  }
  if (c.gq) {
    acc_to_out<T><<<nb, 256, 0, s>>>(a.gq, static_cast<T *>(c.gq), c.natoms, 1.0, false);
    TFF_LAUNCHED();
  }
  const int64_t npar = (c.lm == L_TYPE) ? c.ntypes * c.ntypes : c.natoms;
  if (a.gs) {
    acc_to_out<T><<<nb, 256, 0, s>>>(a.gs, static_cast<T *>(c.gs), npar, 1.0, false);
    TFF_LAUNCHED();
  }
  if (a.ge) {
    acc_to_out<T><<<nb, 256, 0, s>>>(a.ge, static_cast<T *>(c.ge), npar, 1.0, false);
    TFF_LAUNCHED();
  }
  if (c.energy) {
    energy_out<T><<<1, 1, 0, s>>>(a.energy, static_cast<T *>(c.energy), c.e_scale);
    TFF_LAUNCHED();
  }
  return TFF_OK;
}

int run_pairs_any(const PairCall &c, cudaStream_t s) {
  TFF_ARG(c.dtype == TFF_F32 || c.dtype == TFF_F64, "dtype must be TFF_F32 or TFF_F64");
  TFF_ARG(c.natoms >= 0 && c.npairs >= 0 && c.nexcl >= 0, "negative sizes");
  TFF_ARG(c.x != nullptr || c.natoms == 0, "coords is NULL");
  TFF_ARG(c.pairs != nullptr || c.npairs == 0, "pairs is NULL");
  TFF_ARG(c.rc > 0.0, "cutoff must be positive");
  if (c.cm != C_NONE) TFF_ARG(c.q != nullptr, "charges is NULL");
  if (c.lm != L_NONE) TFF_ARG(c.sig != nullptr && c.eps != nullptr, "sigma/epsilon is NULL");
  if (c.lm == L_TYPE) TFF_ARG(c.types != nullptr && c.ntypes > 0, "atom_types/ntypes invalid");
  return c.dtype == TFF_F32 ? run_pairs<float>(c, s) : run_pairs<double>(c, s);
}

// ---------------------------------------------------------------------------------------
// Scratch for tff_nonbonded_atom_pairs_noalloc: a file-scope device array, so that caller
// never has to allocate. Sized for TFF_NOALLOC_MAX_ATOMS atoms (6 accumulators of 8 bytes
// per atom, the block partials and the reduction ticket/energy); every GPU that loads the
// library holds it until the process exits.
// ---------------------------------------------------------------------------------------
constexpr int64_t kNoAllocMaxAtoms = TFF_NOALLOC_MAX_ATOMS;
constexpr size_t kNoAllocScratchBytes = (size_t)kNoAllocMaxAtoms * 6 * 8 + 8192 * 8 + 512;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Id of the context current on this thread (0 while none is), through the driver's
// cuCtxGetCurrent / cuCtxGetId reached via the runtime (the library does not link the driver
// library). Context ids are unique for the life of the process, so the context the runtime
// creates after a cudaDeviceReset never carries the id of the one it replaced.
int current_context_id(unsigned long long *id) {
  using GetCurrent = CUresult (*)(CUcontext *);
  using GetId = CUresult (*)(CUcontext, unsigned long long *);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  if (get_current == nullptr || get_id == nullptr) {
    void *f1 = nullptr, *f2 = nullptr;
    cudaDriverEntryPointQueryResult r1 = cudaDriverEntryPointSymbolNotFound, r2 = r1;
    TFF_CUDA(cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f1, 12000, cudaEnableDefault, &r1));
    TFF_CUDA(cudaGetDriverEntryPointByVersion("cuCtxGetId", &f2, 12000, cudaEnableDefault, &r2));
    TFF_ARG(r1 == cudaDriverEntryPointSuccess && r2 == cudaDriverEntryPointSuccess && f1 && f2,
            "the driver offers no cuCtxGetCurrent/cuCtxGetId");
    get_current = reinterpret_cast<GetCurrent>(f1);
    get_id = reinterpret_cast<GetId>(f2);
  }
  CUcontext ctx = nullptr;
  TFF_ARG(get_current(&ctx) == CUDA_SUCCESS, "cuCtxGetCurrent failed");
  *id = 0;
  if (ctx != nullptr) TFF_ARG(get_id(ctx, id) == CUDA_SUCCESS, "cuCtxGetId failed");
  return TFF_OK;
}

// Device address of g_noalloc_scratch in the current device's context. In host code the
// symbol is only a host-side stand-in, so the address is looked up with
// cudaGetSymbolAddress (with that device current) at the first call on each device, and
// again whenever the device's context has changed since (after a cudaDeviceReset, the
// old address belongs to a destroyed context).
int noalloc_scratch(void **out) {
  static std::mutex mu;
  static void *addr[64] = {nullptr};
  static unsigned long long ctx_of[64] = {0};
  int dev = 0;
  TFF_CUDA(cudaGetDevice(&dev));
  TFF_ARG(dev >= 0 && dev < 64, "device index %d out of range", dev);
  std::lock_guard<std::mutex> lock(mu);
  unsigned long long ctx = 0;
  int st = current_context_id(&ctx);
  if (st != TFF_OK) return st;
  if (addr[dev] == nullptr || ctx == 0 || ctx != ctx_of[dev]) {
    void *p = nullptr;
    TFF_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));   // makes the context current if none was
    st = current_context_id(&ctx);
    if (st != TFF_OK) return st;
    addr[dev] = p;
    ctx_of[dev] = ctx;
  }
  *out = addr[dev];
  return TFF_OK;
}

}  // namespace
}  // namespace tff

using namespace tff;

extern "C" {

// Same computation as tff_nonbonded_atom_pairs, for callers that cannot allocate device
// memory: a force plugin inside a molecular-dynamics engine that owns every device
// allocation and hands the plugin only its input and output buffers, or a time-critical
// loop that must never reach an allocator (an allocation can synchronise the device or
// fail mid-run). Scratch is the library's static device array instead of a caller
// workspace; the caller still passes inputs and outputs. Limits and sharing:
// natoms <= TFF_NOALLOC_MAX_ATOMS (larger sizes return TFF_ERR_INVALID); the first call on
// each device (and the first after a device reset) looks the array up with
// cudaGetSymbolAddress, so make that first call before any stream capture; all calls share
// the one array (its accumulators are cleared at the start of every call and it keeps the
// last call's contents), so calls that overlap on the GPU, e.g. on two streams at once,
// race and must be serialised by the caller.
int tff_nonbonded_atom_pairs_noalloc(int dtype, int64_t natoms, const void *coords, int64_t npairs,
                                     const int64_t *pairs, const void *box, const void *sigma,
                                     const void *epsilon, const void *charges, double coul_constant,
                                     double cutoff, int do_shift, void *energy, void *grad_coords,
                                     void *grad_sigma, void *grad_epsilon, void *grad_charges,
                                     tff_stream_t stream) {
  TFF_ARG(natoms >= 0 && natoms <= kNoAllocMaxAtoms,
          "natoms=%lld exceeds the static scratch limit of %lld atoms of tff_nonbonded_atom_pairs_noalloc",
          (long long)natoms, (long long)kNoAllocMaxAtoms);
  const size_t need = pair_layout(dtype, natoms, 0).bytes;
  TFF_ARG(need <= kNoAllocScratchBytes, "static scratch too small (%zu > %zu bytes)", need, kNoAllocScratchBytes);
  void *ws = nullptr;
  int st = noalloc_scratch(&ws);
  if (st != TFF_OK) return st;
  PairCall c{};
  c.dtype = dtype;
  c.cm = do_shift ? C_SHIFT : C_PLAIN;
  c.lm = L_ATOM;
  c.natoms = natoms; c.npairs = npairs; c.x = coords; c.box = box; c.q = charges;
  c.sig = sigma; c.eps = epsilon; c.pairs = pairs; c.k = coul_constant; c.rc = cutoff;
  c.energy = energy; c.e_scale = 1.0;
  c.gx = grad_coords; c.gx_scale = 1.0; c.gx_add = false;
  c.gq = grad_charges; c.gs = grad_sigma; c.ge = grad_epsilon;
  c.ws = ws; c.ws_bytes = kNoAllocScratchBytes;
  return run_pairs_any(c, (cudaStream_t)stream);
}

size_t tff_pairs_workspace_bytes(int dtype, int64_t natoms, int64_t ntypes) {
  return pair_layout(dtype, natoms, ntypes).bytes;
}

int tff_nonbonded_atom_pairs(int dtype, int64_t natoms, const void *coords, int64_t npairs,
                             const int64_t *pairs, const void *box, const void *sigma,
                             const void *epsilon, const void *charges, double coul_constant,
                             double cutoff, int do_shift, void *energy, void *grad_coords,
                             void *grad_sigma, void *grad_epsilon, void *grad_charges,
                             void *workspace, size_t workspace_bytes, tff_stream_t stream) {
  TFF_NVTX("tff_nonbonded_atom_pairs");
  PairCall c{};
  c.dtype = dtype;
  c.cm = do_shift ? C_SHIFT : C_PLAIN;
  c.lm = L_ATOM;
  c.natoms = natoms; c.npairs = npairs; c.x = coords; c.box = box; c.q = charges;
  c.sig = sigma; c.eps = epsilon; c.pairs = pairs; c.k = coul_constant; c.rc = cutoff;
  c.energy = energy; c.e_scale = 1.0;
  c.gx = grad_coords; c.gx_scale = 1.0; c.gx_add = false;
  c.gq = grad_charges; c.gs = grad_sigma; c.ge = grad_epsilon;
  c.ws = workspace; c.ws_bytes = workspace_bytes;
  return run_pairs_any(c, (cudaStream_t)stream);
}

int tff_nonbonded_forces_atom_pairs(int dtype, int64_t natoms, const void *coords,
                                    int64_t npairs, const int64_t *pairs, const void *box,
                                    const void *sigma, const void *epsilon, const void *charges,
                                    double coul_constant, double cutoff, void *forces,
                                    void *workspace, size_t workspace_bytes, tff_stream_t stream) {
  TFF_NVTX("tff_nonbonded_forces_atom_pairs");
  TFF_ARG(forces != nullptr || natoms == 0, "forces is NULL");
  PairCall c{};
  c.dtype = dtype;
  c.cm = C_SHIFT;
  c.lm = L_ATOM;
  c.natoms = natoms; c.npairs = npairs; c.x = coords; c.box = box; c.q = charges;
  c.sig = sigma; c.eps = epsilon; c.pairs = pairs; c.k = coul_constant; c.rc = cutoff;
  c.gx = forces; c.gx_scale = -1.0; c.gx_add = true;
  c.ws = workspace; c.ws_bytes = workspace_bytes;
  return run_pairs_any(c, (cudaStream_t)stream);
}

int tff_coulomb_atom_pairs(int dtype, int64_t natoms, const void *coords, int64_t npairs,
                           const int64_t *pairs, const void *box, const void *charges,
                           double coul_constant, double cutoff, int do_shift, void *energy,
                           void *grad_coords, void *grad_charges, void *workspace,
                           size_t workspace_bytes, tff_stream_t stream) {
  TFF_NVTX("tff_coulomb_atom_pairs");
  PairCall c{};
  c.dtype = dtype;
  c.cm = do_shift ? C_SHIFT : C_PLAIN;
  c.lm = L_NONE;
  c.natoms = natoms; c.npairs = npairs; c.x = coords; c.box = box; c.q = charges;
  c.pairs = pairs; c.k = coul_constant; c.rc = cutoff;
  c.energy = energy; c.e_scale = 1.0;
  c.gx = grad_coords; c.gx_scale = 1.0;
  c.gq = grad_charges;
  c.ws = workspace; c.ws_bytes = workspace_bytes;
  return run_pairs_any(c, (cudaStream_t)stream);
}

int tff_lennard_jones_atom_pairs(int dtype, int64_t natoms, const void *coords, int64_t npairs,
                                 const int64_t *pairs, const void *box, const void *sigma,
                                 const void *epsilon, double cutoff, const int64_t *atom_types,
                                 int64_t ntypes, void *energy, void *grad_coords,
                                 void *grad_sigma, void *grad_epsilon, void *workspace,
                                 size_t workspace_bytes, tff_stream_t stream) {
  TFF_NVTX("tff_lennard_jones_atom_pairs");
  PairCall c{};
  c.dtype = dtype;
  c.cm = C_NONE;
  c.lm = atom_types ? L_TYPE : L_PAIR;
  c.natoms = natoms; c.npairs = npairs; c.x = coords; c.box = box;
  c.sig = sigma; c.eps = epsilon; c.types = atom_types; c.ntypes = atom_types ? ntypes : 0;
  c.pairs = pairs; c.rc = cutoff;
  c.energy = energy; c.e_scale = 1.0;
  c.gx = grad_coords; c.gx_scale = 1.0;
  c.gs = grad_sigma; c.ge = grad_epsilon;
  c.ws = workspace; c.ws_bytes = workspace_bytes;
  return run_pairs_any(c, (cudaStream_t)stream);
}

int tff_ewald_real_atom_pairs(int dtype, int64_t natoms, const void *coords, const void *box,
                              int64_t npairs, const int64_t *pairs, int64_t npairs_excl,
                              const int64_t *pairs_excl, const void *charges, double cutoff,
                              double ewald_alpha, double prefactor, void *energy,
                              void *grad_coords, void *grad_charges, void *workspace,
                              size_t workspace_bytes, tff_stream_t stream) {
  TFF_NVTX("tff_ewald_real_atom_pairs");
  PairCall c{};
  c.dtype = dtype;
  const bool ewald = ewald_alpha >= 0.0;
  c.cm = ewald ? C_EWALD : C_PLAIN;
  c.lm = L_NONE;
  c.natoms = natoms; c.npairs = npairs; c.x = coords; c.box = box; c.q = charges;
  c.pairs = pairs;
  // the exclusion correction only exists for a positive Ewald alpha (torchff/multipoles.py:317)
  c.excl = (ewald && ewald_alpha > 0.0) ? pairs_excl : nullptr;
  c.nexcl = (ewald && ewald_alpha > 0.0 && pairs_excl) ? npairs_excl : 0;
  c.k = prefactor; c.rc = cutoff; c.alpha = ewald ? ewald_alpha : 0.0;
  c.energy = energy; c.e_scale = 1.0;
  c.gx = grad_coords; c.gx_scale = 1.0;
  c.gq = grad_charges;
  c.ws = workspace; c.ws_bytes = workspace_bytes;
  return run_pairs_any(c, (cudaStream_t)stream);
}

}  // extern "C"

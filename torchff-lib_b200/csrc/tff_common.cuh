// Shared device/host helpers of libtffb200 (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <nvtx3/nvToolsExt.h>

#include "tffb200.h"

namespace tff {

// ---------------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------------
void set_error(const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what, const char *file, int line);
int sm_count();

#define TFF_ARG(cond, ...)                 \
  do {                                     \
    if (!(cond)) {                         \
      ::tff::set_error(__VA_ARGS__);       \
      return TFF_ERR_INVALID;              \
    }                                      \
  } while (0)

#define TFF_CUDA(call)                                                        \
  do {                                                                        \
    cudaError_t _e = (call);                                                  \
    if (_e != cudaSuccess) return ::tff::cuda_fail(_e, #call, __FILE__, __LINE__); \
  } while (0)

#define TFF_LAUNCHED() TFF_CUDA(cudaGetLastError())

// Host-side NVTX range around the enqueue work of one entry point (shown by Nsight Systems
// beside the kernels it launched; free when no tool is attached).
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};
#define TFF_NVTX(name) ::tff::NvtxRange tff_nvtx_range_(name)

constexpr int kWarp = 32;
constexpr unsigned kFull = 0xffffffffu;

// ---------------------------------------------------------------------------------
// programmatic dependent launch (PTX griddepcontrol, sm_90+)
// ---------------------------------------------------------------------------------
// A kernel of a launch chain calls pdl_enter() before anything else: it waits until the
// grid before it in the stream has completed and its writes are visible (a no-op when the
// kernel was launched normally), then lets the next grid of the chain begin launching, so
// that the next kernel's launch overlaps this kernel's run instead of following its end.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Launches `kernel` on `s`; with `pdl` as a programmatic dependent of the previous kernel in
// the stream (the kernel must begin with pdl_enter()).
template <class... P, class... A>
int launch_k(bool pdl, void (*kernel)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, A &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  TFF_CUDA(cudaLaunchKernelEx(&cfg, kernel, static_cast<P>(args)...));
  return TFF_OK;
}

// Workspace carving: 256-byte aligned sub-buffers out of one caller-provided block.
struct Carver {
  char *base;
  size_t off = 0;
  explicit Carver(void *p) : base(static_cast<char *>(p)) {}
  template <class T>
  T *take(size_t n) {
    off = (off + 255) & ~size_t(255);
    T *p = reinterpret_cast<T *>(base ? base + off : nullptr);
    off += n * sizeof(T);
    return p;
  }
  size_t bytes() const { return (off + 255) & ~size_t(255); }
};

// ---------------------------------------------------------------------------------
// box
// ---------------------------------------------------------------------------------
// Rows of `m` are the box vectors a, b, c (torchff/pbc.py). inv = m^{-1}.
struct Box {
  double m[9];
  double inv[9];
  double vol;
};

template <class T>
__device__ __forceinline__ void load_box(const T *g, Box &b) {
#pragma unroll
  for (int k = 0; k < 9; ++k) b.m[k] = (double)g[k];
  const double *m = b.m;
  double c00 = m[4] * m[8] - m[5] * m[7];
  double c01 = m[5] * m[6] - m[3] * m[8];
  double c02 = m[3] * m[7] - m[4] * m[6];
  double c10 = m[2] * m[7] - m[1] * m[8];
  double c11 = m[0] * m[8] - m[2] * m[6];
  double c12 = m[1] * m[6] - m[0] * m[7];
  double c20 = m[1] * m[5] - m[2] * m[4];
  double c21 = m[2] * m[3] - m[0] * m[5];
  double c22 = m[0] * m[4] - m[1] * m[3];
  double det = m[0] * c00 + m[1] * c01 + m[2] * c02;
  double id = 1.0 / det;
  b.inv[0] = c00 * id; b.inv[1] = c10 * id; b.inv[2] = c20 * id;
  b.inv[3] = c01 * id; b.inv[4] = c11 * id; b.inv[5] = c21 * id;
  b.inv[6] = c02 * id; b.inv[7] = c12 * id; b.inv[8] = c22 * id;
  b.vol = fabs(det);
}

// Minimum image of d = r_i - r_j through fractional coordinates,
// ds - floor(ds + 0.5) (torchff/pbc.py:59-62).
template <class T>
__device__ __forceinline__ void min_image(T &dx, T &dy, T &dz, const T *m, const T *inv) {
  T sa = dx * inv[0] + dy * inv[3] + dz * inv[6];
  T sb = dx * inv[1] + dy * inv[4] + dz * inv[7];
  T sc = dx * inv[2] + dy * inv[5] + dz * inv[8];
  sa -= floor(sa + T(0.5));
  sb -= floor(sb + T(0.5));
  sc -= floor(sc + T(0.5));
  dx = sa * m[0] + sb * m[3] + sc * m[6];
  dy = sa * m[1] + sb * m[4] + sc * m[7];
  dz = sa * m[2] + sb * m[5] + sc * m[8];
}

// Orthorhombic minimum image: same convention, diagonal box.
template <class T>
__device__ __forceinline__ T wrap1(T d, T L, T invL) {
  return d - L * floor(d * invL + T(0.5));
}

// ---------------------------------------------------------------------------------
// fixed-point accumulation (mixed precision) / FP64 atomics (FP64 mode)
// ---------------------------------------------------------------------------------
constexpr double kFixScale = 4294967296.0;          // 2^32
constexpr double kFixInv = 1.0 / 4294967296.0;

__device__ __forceinline__ unsigned long long to_fix(double v) {
  return (unsigned long long)__double2ll_rn(v * kFixScale);
}
// to_fix of a float without the FP64 steps: v * 2^32 is exact in FP32 as in FP64, so the
// rounded integer is the same (|v| < 2^31).
__device__ __forceinline__ unsigned long long to_fix_f(float v) {
  return (unsigned long long)__float2ll_rn(v * 4294967296.0f);
}
__host__ __device__ __forceinline__ double from_fix(unsigned long long v) {
  return (double)(long long)v * kFixInv;
}

// Accumulator storage: float (mixed) -> int64 fixed point, double -> double.
template <class T> struct Acc;
template <> struct Acc<float> {
  using S = unsigned long long;
  static __device__ __forceinline__ void add(S *p, double v) { atomicAdd(p, to_fix(v)); }
  static __device__ __forceinline__ double get(const S *p) { return from_fix(*p); }
};
template <> struct Acc<double> {
  using S = double;
  static __device__ __forceinline__ void add(S *p, double v) { atomicAdd(p, v); }
  static __device__ __forceinline__ double get(const S *p) { return *p; }
};

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// ---------------------------------------------------------------------------------
// deterministic reductions
// ---------------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
  return v;
}

// Fixed-order block sum; result valid on thread 0. BLOCK must be a multiple of 32.
template <int BLOCK>
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double s_part[BLOCK / kWarp];
  v = warp_sum(v);
  const int w = threadIdx.x / kWarp, l = threadIdx.x % kWarp;
  __syncthreads();
  if (l == 0) s_part[w] = v;
  __syncthreads();
  double r = 0.0;
  if (w == 0) {
    r = (l < BLOCK / kWarp) ? s_part[l] : 0.0;
    r = warp_sum(r);
  }
  return r;
}

// Grid-wide deterministic sum: every block contributes `v` (per thread), block partials
// go to `partials[blockIdx.x]`, and the last block to finish sums them in index order
// into `*out` (replacing it, or adding when `accumulate`). `ticket` must be 0 before the
// launch and is reset to 0 by the last block, so repeated launches need no memset.
// Returns true (block-uniform) in the last block, whose thread 0 has written *out.
// grid_sum_n reduces over the blocks bid = 0 .. nblocks-1 of one group (e.g. the blocks of
// one system in a batched launch); grid_sum over the whole grid.
template <int BLOCK>
__device__ __forceinline__ bool grid_sum_n(double v, double *partials, unsigned *ticket, double *out,
                                           bool accumulate, unsigned bid, unsigned nblocks) {
  __shared__ bool s_last;
  double s = block_sum<BLOCK>(v);
  if (threadIdx.x == 0) {
    partials[bid] = s;
    __threadfence();
    unsigned t = atomicAdd(ticket, 1u);
    s_last = (t == nblocks - 1);
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    double a = 0.0;
    for (unsigned i = threadIdx.x; i < nblocks; i += BLOCK)
      a += *((volatile double *)partials + i);
    double tot = block_sum<BLOCK>(a);
    if (threadIdx.x == 0) {
      *out = accumulate ? (*out + tot) : tot;
      *ticket = 0u;
    }
  }
  return s_last;
}

template <int BLOCK>
__device__ __forceinline__ bool grid_sum(double v, double *partials, unsigned *ticket,
                                         double *out, bool accumulate) {
  return grid_sum_n<BLOCK>(v, partials, ticket, out, accumulate, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------------------------
// math
// ---------------------------------------------------------------------------------
// erfc(u) and exp(-u^2) for u >= 0 in FP32 from Abramowitz & Stegun, Handbook of
// Mathematical Functions (1964), eq. 7.1.26 (after C. Hastings):
// erfc(u) = t (a1 + t (a2 + t (a3 + t (a4 + t a5)))) exp(-u^2), t = 1/(1 + p u),
// absolute error <= 1.5e-7.
__device__ __forceinline__ void erfc_exp_as(float u, float &erfc_u, float &exp_mu2) {
  const float p = 0.3275911f;
  const float a1 = 0.254829592f, a2 = -0.284496736f, a3 = 1.421413741f,
              a4 = -1.453152027f, a5 = 1.061405429f;
  float t = __fdividef(1.0f, fmaf(p, u, 1.0f));
  float poly = t * fmaf(t, fmaf(t, fmaf(t, fmaf(t, a5, a4), a3), a2), a1);
  exp_mu2 = __expf(-u * u);
  erfc_u = poly * exp_mu2;
}

// Order-6 cardinal B-spline weights at the 6 stencil points of an atom.
// With w in [0, 1), val[k] = M6(w + k) and der[k] = M6'(w + k), k = 0..5, from the
// recursion of Essmann et al., J. Chem. Phys. 103, 8577 (1995), eq. 4.1:
// M_n(u) = (u M_{n-1}(u) + (n - u) M_{n-1}(u - 1)) / (n - 1), M_2(w) = w, M_2(w+1) = 1-w,
// M_n'(u) = M_{n-1}(u) - M_{n-1}(u - 1).
template <class T>
__device__ __forceinline__ void bspline6(T w, T val[6], T der[6]) {
  T m[6];
  m[0] = w;
  m[1] = T(1) - w;
#pragma unroll
  for (int n = 3; n <= 5; ++n) {
    T inv = T(1) / T(n - 1);
    T prev = T(0);
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      if (k < n) {
        T u = w + T(k);
        T cur = (k < n - 1) ? m[k] : T(0);
        T nv = (u * cur + (T(n) - u) * prev) * inv;
        prev = cur;
        m[k] = nv;
      }
    }
  }
  // m[0..4] = M5(w + k)
  T prev = T(0);
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    T cur = (k < 5) ? m[k] : T(0);
    der[k] = cur - prev;
    T u = w + T(k);
    val[k] = (u * cur + (T(6) - u) * prev) * (T(1) / T(5));
    prev = cur;
  }
}

// As bspline6, plus the second derivative dd[k] = M6''(w + k), from
// M_n''(u) = M_{n-2}(u) - 2 M_{n-2}(u - 1) + M_{n-2}(u - 2) with M4 taken inside the recursion.
template <class T>
__device__ __forceinline__ void bspline6_d2(T w, T val[6], T der[6], T dd[6]) {
  T m[6], m4[6];
  m[0] = w;
  m[1] = T(1) - w;
#pragma unroll
  for (int n = 3; n <= 5; ++n) {
    T inv = T(1) / T(n - 1);
    T prev = T(0);
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      if (k < n) {
        T u = w + T(k);
        T cur = (k < n - 1) ? m[k] : T(0);
        T nv = (u * cur + (T(n) - u) * prev) * inv;
        prev = cur;
        m[k] = nv;
      }
    }
    if (n == 4) {
#pragma unroll
      for (int k = 0; k < 6; ++k) m4[k] = k < 4 ? m[k] : T(0);  // M4(w + k)
    }
  }
  T prev = T(0);
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    T cur = (k < 5) ? m[k] : T(0);
    der[k] = cur - prev;
    T u = w + T(k);
    val[k] = (u * cur + (T(6) - u) * prev) * (T(1) / T(5));
    prev = cur;
    const T a = m4[k], b = k >= 1 ? m4[k - 1] : T(0), c = k >= 2 ? m4[k - 2] : T(0);
    dd[k] = a - T(2) * b + c;
  }
}

// Server lanes: capture a batch's graph for its common DFT class ahead of use (batch.cu).
int batch_warm_graph(tff_batch b, const void *coords, const void *boxes, const void *charges, const void *sigma,
                     const void *epsilon, const int *excl, double *energies, void *forces);

}  // namespace tff

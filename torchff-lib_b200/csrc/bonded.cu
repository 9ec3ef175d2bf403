// Harmonic bonds and angles of flexible water: the kernels behind
// compute_harmonic_bond_energy / _forces, compute_harmonic_angle_energy / _forces and
// compute_angles (torchff/bond.py, torchff/angle.py; schemas csrc/bond/bond_interface.cpp:5-6,
// csrc/angle/angle_interface.cpp:5-8).
//
// One thread per term over a grid of a fixed size (a multiple of the SM count), so every
// summation order is fixed. Energies: per-thread FP64, fixed-order block and grid reduction.
// Coordinate gradients: int64 fixed point (FP32 inputs, order-independent) or FP64 atomics
// (FP64 inputs). Per-term parameter gradients are written directly.
#include <algorithm>

#include "bonded.cuh"

namespace tff {
namespace {

template <class T>
__global__ void bonded_acc_out(const typename Acc<T>::S *acc, T *out, int64_t n, double scale, bool add) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const double v = scale * Acc<T>::get(&acc[k]);
    out[k] = add ? (T)((double)out[k] + v) : (T)v;
  }
}

template <class T>
__global__ void bonded_energy_out(const double *e, T *out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) out[0] = (T)e[0];
}

struct BondedCall {
  int dtype;
  bool angle;  // false: bonds (M,2), true: angles (M,3)
  int64_t natoms, nterms;
  const void *x;
  const int64_t *idx;
  const void *p0, *k;
  void *energy, *gx, *gp0, *gk;
  double gx_scale;
  bool gx_add;
  void *ws;
  size_t ws_bytes;
};

template <class T>
int run_bonded(const BondedCall &c, cudaStream_t s) {
  using S = typename Acc<T>::S;
  const int nb = bonded_blocks(c.nterms);
  const BondedWs w = bonded_ws(c.natoms, nb);
  if (c.ws == nullptr || c.ws_bytes < w.bytes) {
    set_error("workspace too small: need %zu bytes, got %zu", w.bytes, c.ws_bytes);
    return TFF_ERR_WORKSPACE;
  }
  char *b = static_cast<char *>(c.ws);
  S *gx = reinterpret_cast<S *>(b + w.gx);
  double *partials = reinterpret_cast<double *>(b + w.partials);
  unsigned *ticket = reinterpret_cast<unsigned *>(b + w.ticket);
  double *energy = reinterpret_cast<double *>(b + w.energy);
  TFF_CUDA(cudaMemsetAsync(b, 0, w.bytes, s));
  const T *x = static_cast<const T *>(c.x);
  if (c.nterms > 0) {
    if (c.angle)
      harmonic_angle_kernel<T><<<nb, kBondBlock, 0, s>>>(x, c.idx, c.nterms, static_cast<const T *>(c.p0),
                                                         static_cast<const T *>(c.k), c.gx ? gx : nullptr,
                                                         static_cast<T *>(c.gp0), static_cast<T *>(c.gk), partials,
                                                         ticket, c.energy ? energy : nullptr);
    else
      harmonic_bond_kernel<T><<<nb, kBondBlock, 0, s>>>(x, c.idx, c.nterms, static_cast<const T *>(c.p0),
                                                        static_cast<const T *>(c.k), c.gx ? gx : nullptr,
                                                        static_cast<T *>(c.gp0), static_cast<T *>(c.gk), partials,
                                                        ticket, c.energy ? energy : nullptr);
    TFF_LAUNCHED();
  }
  if (c.gx && c.natoms > 0) {
    const int nbx = (int)std::max<int64_t>(1, std::min<int64_t>((3 * c.natoms + 255) / 256, sm_count() * 8));
    bonded_acc_out<T><<<nbx, 256, 0, s>>>(gx, static_cast<T *>(c.gx), 3 * c.natoms, c.gx_scale, c.gx_add);
    TFF_LAUNCHED();
  }
  if (c.energy) {
    bonded_energy_out<T><<<1, 32, 0, s>>>(energy, static_cast<T *>(c.energy));
    TFF_LAUNCHED();
  }
  return TFF_OK;
}

int run_bonded_any(const BondedCall &c, cudaStream_t s) {
  TFF_ARG(c.dtype == TFF_F32 || c.dtype == TFF_F64, "dtype must be TFF_F32 or TFF_F64");
  TFF_ARG(c.natoms >= 0 && c.nterms >= 0, "negative sizes");
  TFF_ARG(c.x != nullptr || c.natoms == 0, "coords is NULL");
  TFF_ARG(c.nterms == 0 || (c.idx != nullptr && c.p0 != nullptr && c.k != nullptr), "terms / parameters are NULL");
  return c.dtype == TFF_F32 ? run_bonded<float>(c, s) : run_bonded<double>(c, s);
}

}  // namespace
}  // namespace tff

using namespace tff;

extern "C" {

size_t tff_bonded_workspace_bytes(int dtype, int64_t natoms, int64_t nterms) {
  (void)dtype;
  return bonded_ws(natoms, bonded_blocks(nterms)).bytes;
}

int tff_harmonic_bond(int dtype, int64_t natoms, const void *coords, int64_t nbonds, const int64_t *bonds,
                      const void *b0, const void *k, void *energy, void *grad_coords, void *grad_b0, void *grad_k,
                      void *workspace, size_t workspace_bytes, tff_stream_t stream) {
  TFF_NVTX("tff_harmonic_bond");
  BondedCall c{dtype, false, natoms, nbonds, coords, bonds, b0, k, energy, grad_coords, grad_b0, grad_k, 1.0,
               false, workspace, workspace_bytes};
  return run_bonded_any(c, (cudaStream_t)stream);
}

int tff_harmonic_bond_forces(int dtype, int64_t natoms, const void *coords, int64_t nbonds, const int64_t *bonds,
                             const void *b0, const void *k, void *forces, void *workspace, size_t workspace_bytes,
                             tff_stream_t stream) {
  TFF_NVTX("tff_harmonic_bond_forces");
  TFF_ARG(forces != nullptr || natoms == 0, "forces is NULL");
  BondedCall c{dtype, false, natoms, nbonds, coords, bonds, b0, k, nullptr, forces, nullptr, nullptr, -1.0,
               true, workspace, workspace_bytes};
  return run_bonded_any(c, (cudaStream_t)stream);
}

int tff_harmonic_angle(int dtype, int64_t natoms, const void *coords, int64_t nangles, const int64_t *angles,
                       const void *theta0, const void *k, void *energy, void *grad_coords, void *grad_theta0,
                       void *grad_k, void *workspace, size_t workspace_bytes, tff_stream_t stream) {
  TFF_NVTX("tff_harmonic_angle");
  BondedCall c{dtype, true, natoms, nangles, coords, angles, theta0, k, energy, grad_coords, grad_theta0, grad_k,
               1.0, false, workspace, workspace_bytes};
  return run_bonded_any(c, (cudaStream_t)stream);
}

int tff_harmonic_angle_forces(int dtype, int64_t natoms, const void *coords, int64_t nangles, const int64_t *angles,
                              const void *theta0, const void *k, void *forces, void *workspace,
                              size_t workspace_bytes, tff_stream_t stream) {
  TFF_NVTX("tff_harmonic_angle_forces");
  TFF_ARG(forces != nullptr || natoms == 0, "forces is NULL");
  BondedCall c{dtype, true, natoms, nangles, coords, angles, theta0, k, nullptr, forces, nullptr, nullptr, -1.0,
               true, workspace, workspace_bytes};
  return run_bonded_any(c, (cudaStream_t)stream);
}

int tff_angles(int dtype, int64_t natoms, const void *coords, int64_t nangles, const int64_t *angles, void *theta,
               const void *grad_theta, void *grad_coords, void *workspace, size_t workspace_bytes,
               tff_stream_t stream) {
  TFF_NVTX("tff_angles");
  TFF_ARG(dtype == TFF_F32 || dtype == TFF_F64, "dtype must be TFF_F32 or TFF_F64");
  TFF_ARG(natoms >= 0 && nangles >= 0, "negative sizes");
  TFF_ARG(nangles == 0 || (coords != nullptr && angles != nullptr), "coords / angles is NULL");
  TFF_ARG((grad_theta == nullptr) == (grad_coords == nullptr), "grad_theta and grad_coords go together");
  cudaStream_t s = (cudaStream_t)stream;
  const int nb = bonded_blocks(nangles);
  const size_t need = bonded_ws(natoms, nb).bytes;
  if (grad_coords) {
    if (workspace == nullptr || workspace_bytes < need) {
      set_error("workspace too small: need %zu bytes, got %zu", need, workspace_bytes);
      return TFF_ERR_WORKSPACE;
    }
    TFF_CUDA(cudaMemsetAsync(workspace, 0, 3 * natoms * 8, s));
  }
  auto go = [&](auto tag) -> int {
    using T = decltype(tag);
    auto *acc = static_cast<typename Acc<T>::S *>(workspace);
    if (nangles > 0) {
      angles_kernel<T><<<nb, kBondBlock, 0, s>>>(static_cast<const T *>(coords), angles, nangles,
                                                 static_cast<T *>(theta), static_cast<const T *>(grad_theta),
                                                 grad_coords ? acc : nullptr);
      TFF_LAUNCHED();
    }
    if (grad_coords && natoms > 0) {
      const int nbx = (int)std::max<int64_t>(1, std::min<int64_t>((3 * natoms + 255) / 256, sm_count() * 8));
      bonded_acc_out<T><<<nbx, 256, 0, s>>>(acc, static_cast<T *>(grad_coords), 3 * natoms, 1.0, false);
      TFF_LAUNCHED();
    }
    return TFF_OK;
  };
  return dtype == TFF_F32 ? go(0.0f) : go(0.0);
}

}  // extern "C"

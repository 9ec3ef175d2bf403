// Fused fixed-charge system: one evaluation = cluster build (full neighbour-cluster lists)
// -> fused real-space tile kernel (LJ with Lorentz-Berthelot combining + erfc-screened
// Coulomb, Ewald exclusion correction) || PME on a second stream (spread, FFT, influence
// function, FFT, gather) -> forces in caller order. It evaluates the nonbonded terms of
// examples/tip3p/model.py:100-133 (NeighborList + Vdw + MultipolarInteraction(rank 0) +
// PME) without materialising an int64 pair list.
// The real-space kernels (cluster-pair tiles) are described in tile.cuh.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "tile.cuh"

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
  cudaEvent_t built_ev = nullptr;  // cluster build done (the PME gather visits its atom order)
  void *cl_ws = nullptr;
  void *pme_ws = nullptr;
  void *acc = nullptr;         // gx (npad*3), gq, gsigma, ga (npad each): zeroed per evaluation
  size_t acc_bytes = 0;
  void *pme_ws2 = nullptr;     // second PME workspace (direction grid of second derivatives)
  void *dir_sorted = nullptr;  // direction of a second-derivative pass per sorted slot
  void *pme_hx = nullptr, *pme_hq = nullptr;  // PME second derivatives (caller order)
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
  // tff_system_eval_host with page-locked caller buffers: one graph that also holds the
  // copies, for the last (coords, box, energy, forces) pointers seen
  cudaGraphExec_t pinned_graph = nullptr;
  const void *pinned_ptrs[2] = {nullptr, nullptr};
  double *pinned_io = nullptr;  // page-locked: box (9) in, energy (1) out
  // bonded terms (flexible water), set by tff_system_set_bonded
  int64_t nbonds = 0, nangles = 0;
  int64_t *bonds = nullptr, *angles = nullptr;  // (M,2), (M,3)
  void *bpar = nullptr;                         // b0, kb (nbonds each), th0, kth (nangles each), system dtype
  void *bacc = nullptr;                         // caller-order dE/dx (3N) + bond, angle energies
  bool has_bonded() const { return nbonds + nangles > 0; }
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

// Bonds and angles of the system into sys->bacc on stream s (zeroed first).
template <class T>
int launch_bonded(tff_system sys, const T *x, cudaStream_t s) {
  const int64_t n = sys->desc.natoms;
  TFF_CUDA(cudaMemsetAsync(sys->bacc, 0, (3 * n + 2) * 8, s));
  const T *p = static_cast<const T *>(sys->bpar);
  const int64_t nt = sys->nbonds + sys->nangles;
  const int nb = (int)std::max<int64_t>(1, std::min<int64_t>((nt + kBondBlock - 1) / kBondBlock, (int64_t)sm_count() * 4));
  system_bonded_kernel<T><<<nb, kBondBlock, 0, s>>>(x, n, sys->bonds, sys->nbonds, p, p + sys->nbonds, sys->angles,
                                                    sys->nangles, p + 2 * sys->nbonds,
                                                    p + 2 * sys->nbonds + sys->nangles,
                                                    static_cast<typename Acc<T>::S *>(sys->bacc));
  TFF_LAUNCHED();
  return TFF_OK;
}

template <class T>
int system_eval_impl(tff_system sys, const T *x, const T *box, double *energy, T *forces, double *forces64, T *grad_q,
                     double *terms, cudaStream_t s, cudaEvent_t *ev = nullptr, unsigned *status_out = nullptr) {
  using S = typename Acc<T>::S;
  const int64_t n = sys->desc.natoms;
  auto mark = [&](int k, cudaStream_t st) { return ev ? record_event(ev[k], st) : TFF_OK; };
  int st = mark(0, s);
  if (st != TFF_OK) return st;
  const int sms = sm_count();
  S *energies = reinterpret_cast<S *>(sys->scratch);  // real-space energy accumulators, zeroed by the build

  // --- PME on the side stream: the grid phase needs only the caller's coordinates and the
  // charges; the gather (enqueued after the cluster build below) visits the atoms in the
  // build's cluster order, so that neighbouring threads read neighbouring grid points
  const bool use_pme = sys->pme && n > 0;
  const double *e_pme = nullptr;
  cudaStream_t ps = sys->pme_stream;
  char *pw = static_cast<char *>(sys->pme_ws);
  T *phi_grid = nullptr;
  if (use_pme) {
    TFF_CUDA(cudaEventRecord(sys->fork_ev, s));
    TFF_CUDA(cudaStreamWaitEvent(ps, sys->fork_ev, 0));
    const int K = sys->desc.pme_grid;
    const T *xm = static_cast<const T *>(sys->moduli);
    const T *ym = xm + K;
    const T *zm = ym + K;
    PlainAtoms<T> atoms{x, static_cast<const T *>(sys->q), n};
    // bonded terms ride on the PME stream (a few microseconds, off the real-space chain)
    if (sys->has_bonded() && (st = launch_bonded<T>(sys, x, ps)) != TFF_OK) return st;
    st = pme_grid_phase<T>(sys->pme->impl, sys->pl, pw, atoms, n, box, sys->desc.ewald_alpha, xm, ym, zm, ps,
                           &phi_grid);
    if (st != TFF_OK) return st;
    if ((st = mark(3, ps)) != TFF_OK) return st;
  }

  if (!use_pme && sys->has_bonded() && n > 0 && (st = launch_bonded<T>(sys, x, s)) != TFF_OK) return st;

  // --- real space on the caller stream
  ClusterData<T> cd = cluster_data<T>(sys->cl, sys->cl_ws);
  // the real-space chain (cluster build, sorted parameters, tile kernel) is one run of
  // programmatic dependent launches unless stage events sit between its kernels
  const bool pdl = ev == nullptr;
  st = build_clusters<T>(sys->cl, cd, sys->cl_ws, x, static_cast<const T *>(sys->q), box, sys->desc.cutoff,
                         kHalfLists<T>, s, sys->scratch, 8 * sizeof(double), pdl);
  if (st != TFF_OK) return st;
  if ((st = mark(1, s)) != TFF_OK) return st;
  if (use_pme) {
    TFF_CUDA(cudaEventRecord(sys->built_ev, s));
    TFF_CUDA(cudaStreamWaitEvent(ps, sys->built_ev, 0));
    IndexedAtoms<T> ia{x, static_cast<const T *>(sys->q), cd.sidx, sys->cl.npad};
    IndexedGatherOut<T> out{static_cast<T *>(sys->pme_phi), static_cast<T *>(sys->pme_grad), cd.sidx};
    st = pme_gather_phase<T>(sys->pme->impl, sys->pl, pw, ia, sys->cl.npad, box, sys->desc.ewald_alpha, phi_grid,
                             out, 1.0, (T *)nullptr, ps);
    if (st != TFF_OK) return st;
    if ((st = mark(4, ps)) != TFF_OK) return st;
    TFF_CUDA(cudaEventRecord(sys->join_ev, ps));
    e_pme = reinterpret_cast<const double *>(pw + sys->pl.energies);
  }
  S *gx = static_cast<S *>(sys->acc);
  S *gq = gx + 3 * sys->cl.npad;
  auto *lj = static_cast<typename V2<T>::type *>(sys->lj);
  if (n > 0) {
    // sorted parameters; also zeroes the accumulators
    const int nb = (int)std::max<int64_t>(1, std::min<int64_t>((sys->cl.npad + 255) / 256, sms * 8));
    st = launch_k(pdl, sorted_params_kernel<T>, nb, 256, 0, s, cd, static_cast<const T *>(sys->sigma),
                  static_cast<const T *>(sys->eps), static_cast<const int *>(sys->excl), lj, sys->exslot,
                  static_cast<const T *>(nullptr), static_cast<typename V4<T>::type *>(nullptr), gx, gq);
    if (st != TFF_OK) return st;
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
    if ((st = launch_real_space<T>(pdl, max_items, sms, s, A)) != TFF_OK) return st;
  }
  if ((st = mark(2, s)) != TFF_OK) return st;
  if (use_pme) TFF_CUDA(cudaStreamWaitEvent(s, sys->join_ev, 0));
  const int nbf = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, sms * 8));
  st = launch_k(pdl, finalize_kernel<T>, nbf, 256, 0, s, cd, static_cast<const S *>(gx), static_cast<const S *>(gq),
                use_pme ? static_cast<const T *>(sys->pme_grad) : static_cast<const T *>(nullptr),
                use_pme ? static_cast<const T *>(sys->pme_phi) : static_cast<const T *>(nullptr), forces, forces64,
                grad_q, static_cast<const S *>(energies), e_pme, sys->desc.coul_constant, energy, terms, 1,
                sys->has_bonded() && n > 0 ? static_cast<const S *>(sys->bacc) : static_cast<const S *>(nullptr),
                status_out);
  if (st != TFF_OK) return st;
  return mark(5, s);
}

// Sorted accumulators -> caller order for MODE 1 (out_x = forces, out_q/out_s/out_e =
// dE/dq, dE/dsigma, dE/deps, energy) and MODE 2 (the same slots hold the derivatives of
// dir . dE/dx). pme_vec / pme_scal are the PME parts (already scaled by kc in MODE 2).
// dE/deps_i = (dE/da_i) / (2 a_i) with a = sqrt(eps), and 0 where eps_i = 0.
// With `bonded` (MODE 1) the bonded dE/dx and energies are added as in finalize_kernel.
template <class T, int MODE>
__global__ void finalize_grads_kernel(ClusterData<T> cl, const typename Acc<T>::S *acc, const T *pme_vec,
                                      const T *pme_scal, const T *eps, double kc, T *out_x, T *out_q, T *out_s,
                                      T *out_e, const typename Acc<T>::S *e_tile, const double *e_pme,
                                      double *energy, const typename Acc<T>::S *bonded) {
  using S = typename Acc<T>::S;
  const int64_t np = cl.npad;
  const S *gx = acc, *gq = acc + 3 * np, *gs = acc + 4 * np, *ga = acc + 5 * np;
  const double ps = MODE == 1 ? kc : 1.0;
  for (int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; a < cl.natoms; a += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = cl.inv[a];
    double x[3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
      x[c] = Acc<T>::get(&gx[3 * s + c]) + (pme_vec ? ps * (double)pme_vec[3 * a + c] : 0.0) +
             (bonded ? Acc<T>::get(&bonded[3 * a + c]) : 0.0);
    if (out_x)
#pragma unroll
      for (int c = 0; c < 3; ++c) out_x[3 * a + c] = (T)(MODE == 1 ? -x[c] : x[c]);
    if (out_q) out_q[a] = (T)(Acc<T>::get(&gq[s]) + (pme_scal ? ps * (double)pme_scal[a] : 0.0));
    if (out_s) out_s[a] = (T)Acc<T>::get(&gs[s]);
    if (out_e) {
      const double ai = sqrt((double)eps[a]);
      out_e[a] = (T)(ai > 0.0 ? Acc<T>::get(&ga[s]) / (2.0 * ai) : 0.0);
    }
  }
  if (MODE == 1 && energy && blockIdx.x == 0 && threadIdx.x == 0) {
    const double rec = e_pme ? kc * e_pme[0] : 0.0, self = e_pme ? kc * e_pme[1] : 0.0;
    const double eb = bonded ? Acc<T>::get(&bonded[3 * cl.natoms]) + Acc<T>::get(&bonded[3 * cl.natoms + 1]) : 0.0;
    energy[0] = Acc<T>::get(&e_tile[0]) + Acc<T>::get(&e_tile[1]) + rec + self + eb;
  }
}

// MODE 1: energy, forces and parameter gradients. MODE 2: derivatives of dir . dE/dx with
// respect to coordinates, charges, sigma and epsilon (one Hessian-vector product; the
// cluster lists and both PME potentials are rebuilt for these coordinates).
template <class T, int MODE>
int system_grad_impl(tff_system sys, const T *x, const T *box, const T *dir, double *energy, T *out_x, T *out_q,
                     T *out_s, T *out_e, cudaStream_t s) {
  using S = typename Acc<T>::S;
  const int64_t n = sys->desc.natoms;
  if (MODE == 2 && sys->has_bonded()) {
    set_error("second derivatives of the bonded terms are not implemented");
    return TFF_ERR_INVALID;
  }
  const int sms = sm_count();
  S *energies = reinterpret_cast<S *>(sys->scratch);
  TFF_CUDA(cudaMemsetAsync(sys->scratch, 0, 8 * sizeof(double), s));
  const bool use_pme = sys->pme && n > 0;
  const double *e_pme = nullptr;
  if (MODE == 1 && !use_pme && sys->has_bonded() && n > 0) {
    const int sb = launch_bonded<T>(sys, x, s);
    if (sb != TFF_OK) return sb;
  }
  if (use_pme) {
    TFF_CUDA(cudaEventRecord(sys->fork_ev, s));
    TFF_CUDA(cudaStreamWaitEvent(sys->pme_stream, sys->fork_ev, 0));
    cudaStream_t ps = sys->pme_stream;
    const int K = sys->desc.pme_grid;
    const T *xm = static_cast<const T *>(sys->moduli), *ym = xm + K, *zm = ym + K;
    char *pw = static_cast<char *>(sys->pme_ws);
    PlainAtoms<T> atoms{x, static_cast<const T *>(sys->q), n};
    T *phi_grid = nullptr;
    if (MODE == 1 && sys->has_bonded()) {
      const int sb = launch_bonded<T>(sys, x, ps);
      if (sb != TFF_OK) return sb;
    }
    int st = pme_grid_phase<T>(sys->pme->impl, sys->pl, pw, atoms, n, box, sys->desc.ewald_alpha, xm, ym, zm, ps,
                               &phi_grid);
    if (st != TFF_OK) return st;
    const int nb = (int)std::max<int64_t>(1, std::min<int64_t>((n * kLanesPerAtom + kPmeBlock - 1) / kPmeBlock, sms * 8));
    if constexpr (MODE == 1) {
      PlainGatherOut<T> out{static_cast<T *>(sys->pme_phi), static_cast<T *>(sys->pme_grad)};
      st = pme_gather_phase<T>(sys->pme->impl, sys->pl, pw, atoms, n, box, sys->desc.ewald_alpha, phi_grid, out, 1.0,
                               (T *)nullptr, ps);
      if (st != TFF_OK) return st;
      e_pme = reinterpret_cast<const double *>(pw + sys->pl.energies);
    } else {
      char *pw2 = static_cast<char *>(sys->pme_ws2);
      TFF_CUDA(cudaMemsetAsync(pw2 + sys->pl.zero_off, 0, sys->pl.zero_bytes, ps));
      pme_spread_dir_kernel<T><<<nb, kPmeBlock, 0, ps>>>(atoms, dir, n, box, K,
                                                         reinterpret_cast<S *>(pw2 + sys->pl.fix));
      TFF_LAUNCHED();
      T *psi_grid = nullptr;
      st = pme_solve_phase<T>(sys->pme->impl, sys->pl, pw2, box, sys->desc.ewald_alpha, xm, ym, zm, ps, &psi_grid);
      if (st != TFF_OK) return st;
      pme_gather_hvp_kernel<T><<<nb, kPmeBlock, 0, ps>>>(atoms, dir, n, box, K, phi_grid, psi_grid,
                                                         sys->desc.coul_constant, static_cast<T *>(sys->pme_hx),
                                                         static_cast<T *>(sys->pme_hq));
      TFF_LAUNCHED();
    }
    TFF_CUDA(cudaEventRecord(sys->join_ev, ps));
  }
  ClusterData<T> cd = cluster_data<T>(sys->cl, sys->cl_ws);
  int st = build_clusters<T>(sys->cl, cd, sys->cl_ws, x, static_cast<const T *>(sys->q), box, sys->desc.cutoff, 0, s);
  if (st != TFF_OK) return st;
  S *acc = static_cast<S *>(sys->acc);
  const int64_t np = sys->cl.npad;
  TFF_CUDA(cudaMemsetAsync(sys->acc, 0, (size_t)np * 6 * 8, s));
  auto *lj = static_cast<typename V2<T>::type *>(sys->lj);
  auto *dsorted = static_cast<typename V4<T>::type *>(sys->dir_sorted);
  if (n > 0) {
    const int nb = (int)std::max<int64_t>(1, std::min<int64_t>((np + 255) / 256, sms * 8));
    sorted_params_kernel<T><<<nb, 256, 0, s>>>(cd, static_cast<const T *>(sys->sigma), static_cast<const T *>(sys->eps),
                                               sys->excl, lj, sys->exslot, MODE == 2 ? dir : nullptr, dsorted);
    TFF_LAUNCHED();
    TileArgs<T> A;
    A.cl = cd;
    A.lj = lj;
    A.exslot = sys->exslot;
    A.gx = acc;
    A.gq = acc + 3 * np;
    A.gs = acc + 4 * np;
    A.ga = acc + 5 * np;
    A.u = dsorted;
    A.rc = sys->desc.cutoff;
    A.alpha = sys->desc.ewald_alpha;
    A.kc = sys->desc.coul_constant;
    A.energies = energies;
    const int64_t max_items = sys->cl.nclusters * ((sys->cl.cap + kItemTiles - 1) / kItemTiles);
    constexpr int NW = TileCfg<T, MODE>::NW;
    const int nbt = (int)std::max<int64_t>(1, std::min<int64_t>((max_items + NW - 1) / NW, (int64_t)sms * 48 / NW));
    tile_kernel<T, MODE><<<nbt, NW * kWarp, 0, s>>>(A);
    TFF_LAUNCHED();
  }
  if (use_pme) TFF_CUDA(cudaStreamWaitEvent(s, sys->join_ev, 0));
  const T *pvec = use_pme ? static_cast<const T *>(MODE == 1 ? sys->pme_grad : sys->pme_hx) : nullptr;
  const T *pscal = use_pme ? static_cast<const T *>(MODE == 1 ? sys->pme_phi : sys->pme_hq) : nullptr;
  const int nbf = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, sms * 8));
  finalize_grads_kernel<T, MODE><<<nbf, 256, 0, s>>>(cd, acc, pvec, pscal, static_cast<const T *>(sys->eps),
                                                     sys->desc.coul_constant, out_x, out_q, out_s, out_e, energies,
                                                     e_pme, energy,
                                                     MODE == 1 && sys->has_bonded() && n > 0
                                                         ? static_cast<const S *>(sys->bacc)
                                                         : nullptr);
  TFF_LAUNCHED();
  return TFF_OK;
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
  if (sys->built_ev) cudaEventDestroy(sys->built_ev);
  if (sys->host_graph) cudaGraphExecDestroy(sys->host_graph);
  if (sys->pinned_graph) cudaGraphExecDestroy(sys->pinned_graph);
  if (sys->pinned_io) cudaFreeHost(sys->pinned_io);
  if (sys->capture_stream) cudaStreamDestroy(sys->capture_stream);
  void *ptrs[] = {sys->cl_ws, sys->pme_ws, sys->pme_ws2, sys->dir_sorted, sys->pme_hx, sys->pme_hq,
                  sys->acc, sys->lj, sys->exslot, sys->pme_grad, sys->pme_phi,
                  sys->q, sys->sigma, sys->eps, sys->excl, sys->moduli, sys->scratch, sys->host_x,
                  sys->dev_x, sys->dev_f, sys->dev_e, sys->bonds, sys->angles, sys->bpar, sys->bacc};
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
    const size_t _b = (bytes);                                             \
    cudaError_t _e = cudaMalloc((void **)&(ptr), _b ? _b : 256);           \
    if (_e != cudaSuccess) {                                               \
      free_system(sys);                                                    \
      return cuda_fail(_e, "cudaMalloc", __FILE__, __LINE__);              \
    }                                                                      \
  } while (0)
  TFF_ALLOC(sys->cl_ws, sys->cl.bytes);
  sys->acc_bytes = (size_t)sys->cl.npad * 6 * 8;
  TFF_ALLOC(sys->acc, sys->acc_bytes);
  TFF_ALLOC(sys->dir_sorted, (size_t)sys->cl.npad * 4 * ts);
  TFF_ALLOC(sys->pme_hx, 3 * n * ts);
  TFF_ALLOC(sys->pme_hq, n * ts);
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
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sys->built_ev, cudaEventDisableTiming);
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
    TFF_ALLOC(sys->pme_ws2, sys->pl.bytes);
    TFF_ALLOC(sys->moduli, (size_t)(2 * K + K / 2 + 1) * ts);
    std::vector<double> mod;
    auto mx = host_moduli(K, K);
    auto mz = host_moduli(K, K / 2 + 1);
    mod.insert(mod.end(), mx.begin(), mx.end());
    mod.insert(mod.end(), mx.begin(), mx.end());
    mod.insert(mod.end(), mz.begin(), mz.end());
    upload(sys->moduli, mod.data(), (int64_t)mod.size());
    if (e == cudaSuccess) e = cudaMemset(sys->pme_ws, 0, sys->pl.bytes);
    if (e == cudaSuccess) e = cudaMemset(sys->pme_ws2, 0, sys->pl.bytes);
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

int tff_system_set_bonded(tff_system sys, int64_t nbonds, const int64_t *bonds, const double *b0, const double *kb,
                          int64_t nangles, const int64_t *angles, const double *theta0, const double *ktheta) {
  TFF_ARG(sys != nullptr, "system is NULL");
  TFF_ARG(nbonds >= 0 && nangles >= 0, "negative sizes");
  TFF_ARG(nbonds == 0 || (bonds && b0 && kb), "bonds / b0 / kb is NULL");
  TFF_ARG(nangles == 0 || (angles && theta0 && ktheta), "angles / theta0 / ktheta is NULL");
  const int64_t n = sys->desc.natoms;
  for (int64_t m = 0; m < 2 * nbonds; ++m) TFF_ARG(bonds[m] >= 0 && bonds[m] < n, "bond atom index out of range");
  for (int64_t m = 0; m < 3 * nangles; ++m)
    TFF_ARG(angles[m] >= 0 && angles[m] < n, "angle atom index out of range");
  TFF_CUDA(cudaDeviceSynchronize());
  for (void *p : {(void *)sys->bonds, (void *)sys->angles, sys->bpar, sys->bacc})
    if (p) cudaFree(p);
  sys->bonds = sys->angles = nullptr;
  sys->bpar = sys->bacc = nullptr;
  sys->nbonds = sys->nangles = 0;
  if (sys->host_graph) {  // the cached host-path graphs do not hold the new terms
    cudaGraphExecDestroy(sys->host_graph);
    sys->host_graph = nullptr;
  }
  if (sys->pinned_graph) {
    cudaGraphExecDestroy(sys->pinned_graph);
    sys->pinned_graph = nullptr;
  }
  if (nbonds + nangles == 0) return TFF_OK;
  const size_t ts = sys->desc.dtype == TFF_F64 ? 8 : 4;
  std::vector<double> par;
  par.insert(par.end(), b0, b0 + nbonds);
  par.insert(par.end(), kb, kb + nbonds);
  par.insert(par.end(), theta0, theta0 + nangles);
  par.insert(par.end(), ktheta, ktheta + nangles);
  std::vector<float> parf(par.begin(), par.end());
  const void *src = ts == 8 ? (const void *)par.data() : (const void *)parf.data();
  TFF_CUDA(cudaMalloc(&sys->bacc, (3 * n + 2) * 8));
  TFF_CUDA(cudaMalloc(&sys->bpar, std::max<size_t>(1, par.size()) * ts));
  TFF_CUDA(cudaMemcpy(sys->bpar, src, par.size() * ts, cudaMemcpyHostToDevice));
  if (nbonds > 0) {
    TFF_CUDA(cudaMalloc(&sys->bonds, 2 * nbonds * sizeof(int64_t)));
    TFF_CUDA(cudaMemcpy(sys->bonds, bonds, 2 * nbonds * sizeof(int64_t), cudaMemcpyHostToDevice));
  }
  if (nangles > 0) {
    TFF_CUDA(cudaMalloc(&sys->angles, 3 * nangles * sizeof(int64_t)));
    TFF_CUDA(cudaMemcpy(sys->angles, angles, 3 * nangles * sizeof(int64_t), cudaMemcpyHostToDevice));
  }
  sys->nbonds = nbonds;
  sys->nangles = nangles;
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
  TFF_NVTX("tff_system_eval");
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

}  // extern "C"

namespace {

// Largest coordinate (and force) array, in bytes, that the page-locked host path moves by
// kernel loads and stores over the host link instead of copies: below it the copies' fixed
// cost dominates (3000 waters, 216 KB: 141 -> 120 us per call), above it their bandwidth
// (100,000 waters, 7.2 MB: 2.1 -> 2.8 ms per call with kernel access).
constexpr int64_t kZeroCopyMaxBytes = 1 << 20;

// Captures the device part of tff_system_eval_host (FP64 -> system dtype cast of the
// coordinates and box, evaluation). Without `coords` the graph reads the staged inputs and
// writes internal buffers (the caller issues the copies around it). With `coords` / `forces`
// (the caller's page-locked host buffers; `dcoords` / `dforces` their device addresses) the
// box comes from the system's page-locked box slot and the energy goes to the slot after
// it. Small systems then need no copy at all: the cast kernel reads coordinates and box
// over the host link and the finalize kernel writes the FP64 forces and the energy straight
// into host memory. Larger ones copy inside the graph.
int capture_host_graph(tff_system sys, const double *coords, double *forces, const double *dcoords, double *dforces,
                       cudaGraphExec_t *out) {
  const int64_t n = sys->desc.natoms;
  double *stage = static_cast<double *>(sys->host_x);
  const double *x_in = stage, *box_in = stage + 3 * n;
  double *e_out = sys->dev_e, *f_out = sys->dev_f;
  const bool zero_copy = coords && 3 * n * (int64_t)sizeof(double) <= kZeroCopyMaxBytes;
  double *io = nullptr;
  TFF_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void **>(&io), sys->pinned_io, 0));
  // the finalize kernel writes the build's overflow word next to the energy slot
  unsigned *status_out = reinterpret_cast<unsigned *>(io + 10);
  if (zero_copy) {
    x_in = dcoords;
    box_in = io;
    e_out = io + 9;
    f_out = dforces;
  }
  if (sys->capture_stream == nullptr)
    TFF_CUDA(cudaStreamCreateWithFlags(&sys->capture_stream, cudaStreamNonBlocking));
  cudaStream_t cs = sys->capture_stream;
  TFF_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  int st = TFF_OK;
  cudaError_t ce = cudaSuccess;
  if (coords && !zero_copy) {
    if (n > 0) ce = cudaMemcpyAsync(stage, coords, 3 * n * sizeof(double), cudaMemcpyHostToDevice, cs);
    if (ce == cudaSuccess)
      ce = cudaMemcpyAsync(stage + 3 * n, sys->pinned_io, 9 * sizeof(double), cudaMemcpyHostToDevice, cs);
  }
  const int nb = (int)std::max<int64_t>(1, std::min<int64_t>((3 * n + 255) / 256, sm_count() * 8));
  if (ce == cudaSuccess) {
    if (sys->desc.dtype == TFF_F32) {
      float *x = static_cast<float *>(sys->dev_x);
      cast_inputs_kernel<float><<<nb, 256, 0, cs>>>(x_in, box_in, x, x + 3 * n, 3 * n);
      st = system_eval_impl<float>(sys, x, x + 3 * n, e_out, nullptr, f_out, nullptr, nullptr, cs, nullptr,
                                    status_out);
    } else {
      double *x = static_cast<double *>(sys->dev_x);
      cast_inputs_kernel<double><<<nb, 256, 0, cs>>>(x_in, box_in, x, x + 3 * n, 3 * n);
      st = system_eval_impl<double>(sys, x, x + 3 * n, e_out, nullptr, f_out, nullptr, nullptr, cs, nullptr,
                                     status_out);
    }
  }
  if (coords && !zero_copy && st == TFF_OK && ce == cudaSuccess) {
    if (n > 0) ce = cudaMemcpyAsync(forces, sys->dev_f, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, cs);
    if (ce == cudaSuccess)
      ce = cudaMemcpyAsync(sys->pinned_io + 9, sys->dev_e, sizeof(double), cudaMemcpyDeviceToHost, cs);
  }
  cudaGraph_t graph = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(cs, &graph);
  if (st != TFF_OK || ce != cudaSuccess || ee != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    if (st != TFF_OK) return st;
    return cuda_fail(ce != cudaSuccess ? ce : ee, "host-path graph capture", __FILE__, __LINE__);
  }
  const cudaError_t ie = cudaGraphInstantiate(out, graph, 0);
  cudaGraphDestroy(graph);
  if (ie != cudaSuccess) {
    *out = nullptr;
    return cuda_fail(ie, "cudaGraphInstantiate", __FILE__, __LINE__);
  }
  return TFF_OK;
}

// Status of the evaluation tff_system_eval_host just waited for: the build's overflow word
// that its finalize kernel copied into the page-locked slot.
int host_status(tff_system sys) {
  unsigned w = 0;
  std::memcpy(&w, sys->pinned_io + 10, sizeof(w));
  if (w & 1u) {
    set_error("a cluster's neighbour list overflowed its capacity (max_cluster_neighbors): pairs were dropped");
    return TFF_ERR_CAPACITY;
  }
  return TFF_OK;
}

// Device address of a page-locked (mapped) host buffer; NULL for other memory.
void *mapped_address(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return a.type == cudaMemoryTypeHost ? a.devicePointer : nullptr;
}

}  // namespace

extern "C" {

int tff_system_eval_host(tff_system sys, const double *coords, const double *box, double *energy, double *forces,
                         tff_stream_t stream) {
  TFF_NVTX("tff_system_eval_host");
  TFF_ARG(sys != nullptr, "system is NULL");
  TFF_ARG(box != nullptr && energy != nullptr, "box/energy is NULL");
  const int64_t n = sys->desc.natoms;
  TFF_ARG(n == 0 || (coords != nullptr && forces != nullptr), "coords/forces is NULL");
  cudaStream_t s = (cudaStream_t)stream;
  double *stage = static_cast<double *>(sys->host_x);
  // Page-locked coordinate and force buffers (the usual case of a caller that reuses them):
  // one graph launch reads the inputs from and writes the results to host memory; it is
  // re-captured when the pointers change.
  const void *dcoords = n > 0 ? mapped_address(coords) : nullptr;
  void *dforces = dcoords ? mapped_address(forces) : nullptr;
  const bool pinned = dcoords != nullptr && dforces != nullptr;
  if (sys->pinned_io == nullptr) TFF_CUDA(cudaHostAlloc(&sys->pinned_io, 16 * sizeof(double), cudaHostAllocMapped));
  if (pinned && (sys->pinned_graph == nullptr || sys->pinned_ptrs[0] != coords || sys->pinned_ptrs[1] != forces)) {
    if (sys->pinned_graph) {
      cudaGraphExecDestroy(sys->pinned_graph);
      sys->pinned_graph = nullptr;
    }
    const int st = capture_host_graph(sys, coords, forces, static_cast<const double *>(dcoords),
                                      static_cast<double *>(dforces), &sys->pinned_graph);
    if (st != TFF_OK) return st;
    sys->pinned_ptrs[0] = coords;
    sys->pinned_ptrs[1] = forces;
  }
  if (pinned) {
    std::memcpy(sys->pinned_io, box, 9 * sizeof(double));
    TFF_CUDA(cudaGraphLaunch(sys->pinned_graph, s));
    TFF_CUDA(cudaStreamSynchronize(s));
    *energy = sys->pinned_io[9];
    return host_status(sys);
  }
  // Other buffers: the device part is captured once (it touches only the system's own
  // buffers) and the copies are issued around it.
  if (sys->host_graph == nullptr) {
    const int st = capture_host_graph(sys, nullptr, nullptr, nullptr, nullptr, &sys->host_graph);
    if (st != TFF_OK) return st;
  }
  if (n > 0) TFF_CUDA(cudaMemcpyAsync(stage, coords, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s));
  TFF_CUDA(cudaMemcpyAsync(stage + 3 * n, box, 9 * sizeof(double), cudaMemcpyHostToDevice, s));
  TFF_CUDA(cudaGraphLaunch(sys->host_graph, s));
  if (n > 0) TFF_CUDA(cudaMemcpyAsync(forces, sys->dev_f, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
  TFF_CUDA(cudaMemcpyAsync(energy, sys->dev_e, sizeof(double), cudaMemcpyDeviceToHost, s));
  TFF_CUDA(cudaStreamSynchronize(s));
  return host_status(sys);
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
  TFF_NVTX("tff_system_eval_timed");
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

int tff_system_eval_grads(tff_system sys, const void *coords, const void *box, double *energy, void *forces,
                          void *grad_charges, void *grad_sigma, void *grad_epsilon, tff_stream_t stream) {
  TFF_NVTX("tff_system_eval_grads");
  TFF_ARG(sys != nullptr && box != nullptr, "system/box is NULL");
  TFF_ARG(sys->desc.natoms == 0 || coords != nullptr, "coords is NULL");
  cudaStream_t s = (cudaStream_t)stream;
  if (sys->desc.dtype == TFF_F32)
    return system_grad_impl<float, 1>(sys, (const float *)coords, (const float *)box, nullptr, energy, (float *)forces,
                                      (float *)grad_charges, (float *)grad_sigma, (float *)grad_epsilon, s);
  return system_grad_impl<double, 1>(sys, (const double *)coords, (const double *)box, nullptr, energy,
                                     (double *)forces, (double *)grad_charges, (double *)grad_sigma,
                                     (double *)grad_epsilon, s);
}

int tff_system_hvp(tff_system sys, const void *coords, const void *box, const void *direction, void *hvp_coords,
                   void *hvp_charges, void *hvp_sigma, void *hvp_epsilon, tff_stream_t stream) {
  TFF_NVTX("tff_system_hvp");
  TFF_ARG(sys != nullptr && box != nullptr, "system/box is NULL");
  TFF_ARG(sys->desc.natoms == 0 || (coords != nullptr && direction != nullptr), "coords/direction is NULL");
  cudaStream_t s = (cudaStream_t)stream;
  if (sys->desc.dtype == TFF_F32)
    return system_grad_impl<float, 2>(sys, (const float *)coords, (const float *)box, (const float *)direction,
                                      nullptr, (float *)hvp_coords, (float *)hvp_charges, (float *)hvp_sigma,
                                      (float *)hvp_epsilon, s);
  return system_grad_impl<double, 2>(sys, (const double *)coords, (const double *)box, (const double *)direction,
                                     nullptr, (double *)hvp_coords, (double *)hvp_charges, (double *)hvp_sigma,
                                     (double *)hvp_epsilon, s);
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

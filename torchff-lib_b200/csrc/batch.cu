// Batched evaluation of many independent periodic systems (the serving path): every stage
// is one launch over all systems of the batch.
//
//   main stream : batch_sort (one block per system: its own box facts and Hilbert cell
//                 grid) -> cluster bounds -> cluster neighbours -> sorted parameters ->
//                 tile kernel -> [join] -> finalize (forces, one energy per system)
//   PME stream  : spread (blockIdx.y = system) -> [fixed point -> FP32] -> 3-D real DFT
//                 (three axis passes over all systems) -> convolution -> inverse DFT
//                 (three passes) -> gather
//
// Systems are laid out one after another in every array; the cluster lists never leave a
// system, and every per-system reduction runs over a block count that depends on that
// system alone, so a system's result does not depend on what else is in the batch. The
// reciprocal-space transforms are the batched direct DFT of pme.cuh (one launch per axis
// pass for all grid sizes): cuFFT transforms grids of one size per plan, and a batch of
// a few hundred sizes would need hundreds of plans and launches per evaluation.
#include <algorithm>
#include <cmath>
#include <utility>
#include <vector>

#include "tile.cuh"

namespace tff {
namespace {

// Largest PME grid side of a batch: the DFT stages two K x K planes in shared memory.
constexpr int kBatchMaxK = 96;
constexpr int kBatchMaxK64 = 64;

// Grid distances inside the batch: every real grid starts on a 256-byte boundary and every
// complex grid on a 256-byte (FP32) boundary, as cuFFT wants aligned transform inputs.
inline int64_t real_dist(int K) { return ((int64_t)K * K * K + 63) / 64 * 64; }
inline int64_t cplx_dist(int K) { return ((int64_t)K * K * (K / 2 + 1) + 31) / 32 * 32; }

// Offset of grid K's moduli (xmod (K), ymod (K), zmod (K/2+1)) in the moduli table.
inline int moduli_offset(int K) {
  int off = 0;
  for (int k = 6; k < K; ++k) off += 2 * k + k / 2 + 1;
  return off;
}

struct BatchLayout {
  int64_t atoms, systems, clusters, supers, grid;
  int cap;
  size_t sys, status, boxinfo, cl_sys, sup_sys, sidx, inv, pos, frac, bc, bh, sbc, sbh, nbr, ncount, itemoff, items;
  size_t lj, exslot, acc, e_tile;
  size_t fix, real, cplx, partials, tickets, e_pme, pme_grad, pme_phi, moduli;
  size_t bytes;
};

inline BatchLayout batch_layout(int dtype, int64_t max_atoms, int64_t max_systems, int64_t max_grid, int cap) {
  BatchLayout L{};
  L.atoms = max_atoms;
  L.systems = max_systems;
  L.clusters = max_atoms / kWarp + max_systems;
  L.supers = L.clusters / kSuper + max_systems;
  L.grid = max_grid;
  L.cap = cap;
  const size_t ts = dtype == TFF_F64 ? 8 : 4;
  const int64_t slots = L.clusters * kWarp;
  Carver c(nullptr);
  auto take = [&](size_t bytes) {
    c.take<char>(bytes);
    return c.off - bytes;
  };
  L.sys = take(max_systems * sizeof(BatchSys));
  L.status = take(64 * sizeof(unsigned));
  L.boxinfo = take(max_systems * kInfoStride * sizeof(double));
  L.cl_sys = take(L.clusters * sizeof(int));
  L.sup_sys = take(L.supers * sizeof(int));
  L.sidx = take(slots * sizeof(int));
  L.inv = take(max_atoms * sizeof(int));
  L.pos = take(slots * 4 * ts);
  L.frac = take(slots * 4 * ts);
  L.bc = take(L.clusters * 4 * ts);
  L.bh = take(L.clusters * 4 * ts);
  L.sbc = take(L.supers * 4 * ts);
  L.sbh = take(L.supers * 4 * ts);
  L.nbr = take((size_t)L.clusters * cap * sizeof(int));
  L.ncount = take(L.clusters * sizeof(int));
  L.itemoff = take((L.clusters + 1) * sizeof(int));
  L.items = take((size_t)L.clusters * ((cap + kItemTiles - 1) / kItemTiles) * sizeof(int));
  L.lj = take(slots * 2 * ts);
  L.exslot = take(slots * kMaxExcl * sizeof(int));
  L.acc = take(slots * 4 * 8);  // gx (3 per slot) + gq, fixed point or double
  L.e_tile = take(2 * max_systems * 8);
  const int64_t grid_cap = max_grid + 64 * max_systems;  // padding of real_dist / cplx_dist
  L.fix = take(grid_cap * 8);
  L.real = take(dtype == TFF_F64 ? 0 : grid_cap * ts);
  L.cplx = take(grid_cap * 2 * ts);  // K*K*(K/2+1) <= K^3 complex points per system
  L.partials = take((size_t)max_systems * kBatchPmeMaxBlocks * sizeof(double));
  L.tickets = take(2 * max_systems * sizeof(unsigned));
  L.e_pme = take(2 * max_systems * sizeof(double));
  L.pme_grad = take(3 * max_atoms * ts);
  L.pme_phi = take(max_atoms * ts);
  L.moduli = take((size_t)moduli_offset(kBatchMaxK + 1) * ts);
  L.bytes = c.bytes();
  return L;
}

}  // namespace
}  // namespace tff

using namespace tff;

struct tff_batch_s {
  tff_batch_desc desc;
  BatchLayout L;
  char *ws = nullptr;
  BatchSys *table = nullptr;       // pinned host copy of the system table
  cudaEvent_t table_ev = nullptr;  // the table upload of the previous evaluation
  cudaStream_t pme_stream = nullptr;
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
  cudaEvent_t sorted_ev = nullptr;  // batch sort done (the PME gather visits its atom order)
  std::vector<BatchSys> host_sys;
  int device = 0;
};

namespace tff {
namespace {

void free_batch(tff_batch b) {
  if (!b) return;
  if (b->ws) cudaFree(b->ws);
  if (b->table) cudaFreeHost(b->table);
  if (b->table_ev) cudaEventDestroy(b->table_ev);
  if (b->pme_stream) cudaStreamDestroy(b->pme_stream);
  if (b->fork_ev) cudaEventDestroy(b->fork_ev);
  if (b->join_ev) cudaEventDestroy(b->join_ev);
  if (b->sorted_ev) cudaEventDestroy(b->sorted_ev);
  delete b;
}

// One direction of the 3-D real DFT of every grid of the batch (three axis passes).
template <class T>
int run_dft(const BatchSys *dsys, int nsys, int kmax, bool forward, T *real, typename CplxOf<T>::type *cplx,
            cudaStream_t s) {
  const dim3 grid((unsigned)kmax, (unsigned)nsys);
  const size_t smem = batch_dft_smem<T>(kmax);
  if (forward) {
    batch_dft_kernel<T, kDftZR2C><<<grid, kDftThreads, smem, s>>>(dsys, real, cplx);
    TFF_LAUNCHED();
    batch_dft_kernel<T, kDftY><<<grid, kDftThreads, smem, s>>>(dsys, real, cplx);
    TFF_LAUNCHED();
    batch_dft_kernel<T, kDftX><<<grid, kDftThreads, smem, s>>>(dsys, real, cplx);
    TFF_LAUNCHED();
  } else {
    batch_dft_kernel<T, kDftXInv><<<grid, kDftThreads, smem, s>>>(dsys, real, cplx);
    TFF_LAUNCHED();
    batch_dft_kernel<T, kDftYInv><<<grid, kDftThreads, smem, s>>>(dsys, real, cplx);
    TFF_LAUNCHED();
    batch_dft_kernel<T, kDftZC2R><<<grid, kDftThreads, smem, s>>>(dsys, real, cplx);
    TFF_LAUNCHED();
  }
  return TFF_OK;
}

template <class T>
int batch_eval_impl(tff_batch b, int nsys, const int64_t *natoms, const int *pme_grid, const T *x, const T *boxes,
                    const T *q, const T *sigma, const T *eps, const int *excl, double *energies, T *forces,
                    cudaStream_t s) {
  using S = typename Acc<T>::S;
  const BatchLayout &L = b->L;
  // --- host: system table, grid order, FFT groups
  auto &hs = b->host_sys;
  hs.assign(nsys, BatchSys{});
  int64_t ao = 0, co = 0, so = 0, go = 0, xo = 0, max_pb = 1;
  for (int i = 0; i < nsys; ++i) {
    const int64_t n = natoms[i];
    const int K = pme_grid[i];
    TFF_ARG(n >= 1 && n <= kBatchMaxAtoms, "system %d: natoms %lld outside [1, %d]", i, (long long)n, kBatchMaxAtoms);
    const int kmax_dtype = sizeof(T) == 8 ? kBatchMaxK64 : kBatchMaxK;
    TFF_ARG(K >= 6 && K <= kmax_dtype, "system %d: PME grid %d outside [6, %d]", i, K, kmax_dtype);
    BatchSys &y = hs[i];
    y.atom_off = ao;
    y.natoms = n;
    y.ncl = (n + kWarp - 1) / kWarp;
    y.cl_off = co;
    y.nsup = (y.ncl + kSuper - 1) / kSuper;
    y.sup_off = so;
    cell_grid(n, b->desc.atoms_per_cell, y.nc, y.bits);
    TFF_ARG((1 << (3 * y.bits)) <= kBatchMaxKeys, "system %d: cell grid too fine", i);
    y.K = K;
    y.mod_off = moduli_offset(K);
    const int64_t ncplx = (int64_t)K * K * (K / 2 + 1);
    y.pme_blocks = (int)std::min<int64_t>(kBatchPmeMaxBlocks, std::max<int64_t>(1, (std::max(n * kLanesPerAtom, ncplx) + kPmeBlock - 1) / kPmeBlock));
    max_pb = std::max<int64_t>(max_pb, y.pme_blocks);
    ao += n;
    co += y.ncl;
    so += y.nsup;
  }
  TFF_ARG(ao <= L.atoms, "batch holds %lld atoms; capacity %lld", (long long)ao, (long long)L.atoms);
  int kmax = 6;
  for (BatchSys &y : hs) {
    y.grid_off = go;
    y.cplx_off = xo;
    go += real_dist(y.K);
    xo += cplx_dist(y.K);
    kmax = std::max(kmax, y.K);
  }
  TFF_ARG(go <= L.grid + 64 * L.systems, "batch holds %lld PME grid points; capacity %lld", (long long)go,
          (long long)L.grid);
  const int64_t ncl = co, nsup = so, npad = co * kWarp, total_atoms = ao, total_grid = go;

  // --- device pointers
  char *w = b->ws;
  ClusterData<T> cd{};
  using V = typename V4<T>::type;
  cd.status = reinterpret_cast<unsigned *>(w + L.status);
  cd.sidx = reinterpret_cast<int *>(w + L.sidx);
  cd.inv = reinterpret_cast<int *>(w + L.inv);
  cd.nbr = reinterpret_cast<int *>(w + L.nbr);
  cd.ncount = reinterpret_cast<int *>(w + L.ncount);
  cd.itemoff = reinterpret_cast<int *>(w + L.itemoff);
  cd.items = reinterpret_cast<int *>(w + L.items);
  cd.pos = reinterpret_cast<V *>(w + L.pos);
  cd.frac = reinterpret_cast<V *>(w + L.frac);
  cd.bc = reinterpret_cast<V *>(w + L.bc);
  cd.bh = reinterpret_cast<V *>(w + L.bh);
  cd.sbc = reinterpret_cast<V *>(w + L.sbc);
  cd.sbh = reinterpret_cast<V *>(w + L.sbh);
  cd.boxinfo = reinterpret_cast<double *>(w + L.boxinfo);
  cd.cap = L.cap;
  cd.natoms = total_atoms;
  cd.nclusters = ncl;
  cd.npad = npad;
  cd.nsuper = nsup;
  cd.sys = reinterpret_cast<const BatchSys *>(w + L.sys);
  cd.cl_sys = reinterpret_cast<int *>(w + L.cl_sys);
  cd.sup_sys = reinterpret_cast<int *>(w + L.sup_sys);

  // --- upload the table (the pinned buffer is reused once the previous upload is done)
  TFF_CUDA(cudaEventSynchronize(b->table_ev));
  std::copy(hs.begin(), hs.end(), b->table);
  TFF_CUDA(cudaMemcpyAsync(w + L.sys, b->table, nsys * sizeof(BatchSys), cudaMemcpyHostToDevice, s));
  TFF_CUDA(cudaEventRecord(b->table_ev, s));
  TFF_CUDA(cudaMemsetAsync(w + L.status, 0, 64 * sizeof(unsigned), s));
  TFF_CUDA(cudaMemsetAsync(w + L.e_tile, 0, 2 * nsys * 8, s));
  TFF_CUDA(cudaMemsetAsync(w + L.acc, 0, npad * 4 * 8, s));
  const int sms = sm_count();

  // --- PME on the side stream
  TFF_CUDA(cudaEventRecord(b->fork_ev, s));
  cudaStream_t ps = b->pme_stream;
  TFF_CUDA(cudaStreamWaitEvent(ps, b->fork_ev, 0));
  TFF_CUDA(cudaMemsetAsync(w + L.fix, 0, total_grid * 8, ps));
  TFF_CUDA(cudaMemsetAsync(w + L.tickets, 0, 2 * nsys * sizeof(unsigned), ps));
  const BatchSys *dsys = cd.sys;
  double *partials = reinterpret_cast<double *>(w + L.partials);
  unsigned *tickets = reinterpret_cast<unsigned *>(w + L.tickets);
  double *e_pme = reinterpret_cast<double *>(w + L.e_pme);
  S *fix = reinterpret_cast<S *>(w + L.fix);
  T *pme_grad = reinterpret_cast<T *>(w + L.pme_grad);
  T *pme_phi = reinterpret_cast<T *>(w + L.pme_phi);
  const dim3 pgrid((unsigned)max_pb, (unsigned)nsys);
  batch_spread_kernel<T><<<pgrid, kPmeBlock, 0, ps>>>(dsys, x, q, boxes, fix);
  TFF_LAUNCHED();
  T *real;
  if (sizeof(T) == 4) {
    real = reinterpret_cast<T *>(w + L.real);
    const int nb = (int)std::max<int64_t>(1, std::min<int64_t>((total_grid + 255) / 256, sms * 8));
    pme_fix_to_real_kernel<<<nb, 256, 0, ps>>>(reinterpret_cast<unsigned long long *>(fix),
                                               reinterpret_cast<float *>(real), total_grid);
    TFF_LAUNCHED();
  } else {
    real = reinterpret_cast<T *>(fix);
  }
  auto *cplx = reinterpret_cast<typename CplxOf<T>::type *>(w + L.cplx);
  int st = run_dft<T>(dsys, nsys, kmax, true, real, cplx, ps);
  if (st != TFF_OK) return st;
  batch_convolve_kernel<T><<<pgrid, kPmeBlock, 0, ps>>>(dsys, cplx, boxes, b->desc.ewald_alpha,
                                                        reinterpret_cast<const T *>(w + L.moduli), partials, tickets,
                                                        e_pme);
  TFF_LAUNCHED();
  if ((st = run_dft<T>(dsys, nsys, kmax, false, real, cplx, ps)) != TFF_OK) return st;

  // --- real space on the caller stream
  batch_sort_kernel<T><<<(int)std::min<int64_t>(nsys, 2 * sms), kBatchSortThreads, kBatchSortSmem, s>>>(x, q, boxes,
                                                                                                     nsys, cd);
  TFF_LAUNCHED();
  // the PME gather follows the sort's atom order
  TFF_CUDA(cudaEventRecord(b->sorted_ev, s));
  TFF_CUDA(cudaStreamWaitEvent(ps, b->sorted_ev, 0));
  batch_gather_kernel<T><<<pgrid, kPmeBlock, 0, ps>>>(dsys, x, q, cd.sidx, boxes, real, b->desc.ewald_alpha, pme_phi,
                                                      pme_grad, partials, tickets, e_pme);
  TFF_LAUNCHED();
  TFF_CUDA(cudaEventRecord(b->join_ev, ps));
  cluster_bounds_kernel<T><<<(int)std::max<int64_t>(1, std::min<int64_t>(nsup, 2 * sms)), kWarp * kSuper, 0, s>>>(cd);
  TFF_LAUNCHED();
  const int nb_cl = (int)std::max<int64_t>(1, std::min<int64_t>((ncl + 3) / 4, sms * 16));
  cluster_neighbors_kernel<T><<<nb_cl, 128, 0, s>>>(cd, b->desc.cutoff, kHalfLists<T>);
  TFF_LAUNCHED();
  auto *lj = reinterpret_cast<typename V2<T>::type *>(w + L.lj);
  int *exslot = reinterpret_cast<int *>(w + L.exslot);
  {
    const int nb = (int)std::max<int64_t>(1, std::min<int64_t>((npad + 255) / 256, sms * 8));
    sorted_params_kernel<T><<<nb, 256, 0, s>>>(cd, sigma, eps, excl, lj, exslot);
    TFF_LAUNCHED();
  }
  S *gx = reinterpret_cast<S *>(w + L.acc);
  S *gq = gx + 3 * npad;
  S *e_tile = reinterpret_cast<S *>(w + L.e_tile);
  {
    TileArgs<T> A;
    A.cl = cd;
    A.lj = lj;
    A.exslot = exslot;
    A.gx = gx;
    A.gq = gq;
    A.rc = b->desc.cutoff;
    A.alpha = b->desc.ewald_alpha;
    A.kc = b->desc.coul_constant;
    A.energies = e_tile;
    const int64_t max_items = ncl * ((L.cap + kItemTiles - 1) / kItemTiles);
    const int st_rs = launch_real_space<T>(false, max_items, sms, s, A);
    if (st_rs != TFF_OK) return st_rs;
  }
  TFF_CUDA(cudaStreamWaitEvent(s, b->join_ev, 0));
  const int nbf = (int)std::max<int64_t>(1, std::min<int64_t>((total_atoms + 255) / 256, sms * 8));
  finalize_kernel<T><<<nbf, 256, 0, s>>>(cd, gx, gq, pme_grad, pme_phi, forces, (double *)nullptr, (T *)nullptr,
                                         e_tile, e_pme, b->desc.coul_constant, energies, (double *)nullptr, nsys);
  TFF_LAUNCHED();
  return TFF_OK;
}

template <class T>
int set_sort_smem() {
  TFF_CUDA(cudaFuncSetAttribute(batch_sort_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kBatchSortSmem));
  const int dft = (int)batch_dft_smem<T>(sizeof(T) == 8 ? kBatchMaxK64 : kBatchMaxK);
  TFF_CUDA(cudaFuncSetAttribute(batch_dft_kernel<T, kDftZR2C>, cudaFuncAttributeMaxDynamicSharedMemorySize, dft));
  TFF_CUDA(cudaFuncSetAttribute(batch_dft_kernel<T, kDftY>, cudaFuncAttributeMaxDynamicSharedMemorySize, dft));
  TFF_CUDA(cudaFuncSetAttribute(batch_dft_kernel<T, kDftX>, cudaFuncAttributeMaxDynamicSharedMemorySize, dft));
  TFF_CUDA(cudaFuncSetAttribute(batch_dft_kernel<T, kDftXInv>, cudaFuncAttributeMaxDynamicSharedMemorySize, dft));
  TFF_CUDA(cudaFuncSetAttribute(batch_dft_kernel<T, kDftYInv>, cudaFuncAttributeMaxDynamicSharedMemorySize, dft));
  TFF_CUDA(cudaFuncSetAttribute(batch_dft_kernel<T, kDftZC2R>, cudaFuncAttributeMaxDynamicSharedMemorySize, dft));
  return TFF_OK;
}

}  // namespace
}  // namespace tff

extern "C" {

size_t tff_batch_device_bytes(const tff_batch_desc *desc) {
  if (!desc) return 0;
  const int cap = desc->max_cluster_neighbors > 0 ? desc->max_cluster_neighbors : kBatchMaxAtoms / kWarp;
  return batch_layout(desc->dtype, desc->max_atoms, desc->max_systems, desc->max_grid_points, cap).bytes;
}

int tff_batch_create(const tff_batch_desc *desc, tff_batch *out) {
  TFF_ARG(desc != nullptr && out != nullptr, "desc/out is NULL");
  TFF_ARG(desc->dtype == TFF_F32 || desc->dtype == TFF_F64, "dtype must be TFF_F32 or TFF_F64");
  TFF_ARG(desc->max_systems >= 1 && desc->max_systems <= 65535, "max_systems must be in [1, 65535]");
  TFF_ARG(desc->max_atoms >= 1 && desc->max_atoms < ((int64_t)1 << 30), "max_atoms out of range");
  TFF_ARG(desc->max_grid_points >= 216, "max_grid_points must be at least 6^3");
  TFF_ARG(desc->cutoff > 0.0 && desc->ewald_alpha > 0.0, "cutoff and ewald_alpha must be positive");
  TFF_ARG(desc->atoms_per_cell == 0.0 || (desc->atoms_per_cell >= 2.0 && desc->atoms_per_cell <= 64.0),
          "atoms_per_cell must be 0 (default 8) or in [2, 64]");
  auto *b = new tff_batch_s();
  b->desc = *desc;
  if (b->desc.atoms_per_cell == 0.0) b->desc.atoms_per_cell = 8.0;
  // a system has at most kBatchMaxAtoms / 32 clusters, so the default cap cannot overflow
  const int cap = desc->max_cluster_neighbors > 0 ? desc->max_cluster_neighbors : kBatchMaxAtoms / kWarp;
  b->L = batch_layout(desc->dtype, desc->max_atoms, desc->max_systems, desc->max_grid_points, cap);
  cudaGetDevice(&b->device);
  cudaError_t e = cudaMalloc(&b->ws, b->L.bytes);
  if (e == cudaSuccess) e = cudaMemset(b->ws, 0, b->L.bytes);
  if (e == cudaSuccess) e = cudaMallocHost((void **)&b->table, desc->max_systems * sizeof(BatchSys));
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->table_ev, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->pme_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork_ev, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->join_ev, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->sorted_ev, cudaEventDisableTiming);
  if (e == cudaSuccess) {
    // B-spline moduli of every grid size the batch accepts
    std::vector<double> mod;
    for (int K = 6; K <= kBatchMaxK; ++K) {
      auto mx = host_moduli(K, K), mz = host_moduli(K, K / 2 + 1);
      mod.insert(mod.end(), mx.begin(), mx.end());
      mod.insert(mod.end(), mx.begin(), mx.end());
      mod.insert(mod.end(), mz.begin(), mz.end());
    }
    if (desc->dtype == TFF_F64) {
      e = cudaMemcpy(b->ws + b->L.moduli, mod.data(), mod.size() * 8, cudaMemcpyHostToDevice);
    } else {
      std::vector<float> mf(mod.begin(), mod.end());
      e = cudaMemcpy(b->ws + b->L.moduli, mf.data(), mf.size() * 4, cudaMemcpyHostToDevice);
    }
  }
  if (e != cudaSuccess) {
    free_batch(b);
    return cuda_fail(e, "batch set-up", __FILE__, __LINE__);
  }
  const int st = desc->dtype == TFF_F64 ? set_sort_smem<double>() : set_sort_smem<float>();
  if (st != TFF_OK) {
    free_batch(b);
    return st;
  }
  *out = b;
  return TFF_OK;
}

int tff_batch_destroy(tff_batch b) {
  free_batch(b);
  return TFF_OK;
}

int tff_batch_eval(tff_batch b, int nsys, const int64_t *natoms, const int *pme_grid, const void *coords,
                   const void *boxes, const void *charges, const void *sigma, const void *epsilon, const int *excl,
                   double *energies, void *forces, tff_stream_t stream) {
  TFF_NVTX("tff_batch_eval");
  TFF_ARG(b != nullptr, "batch is NULL");
  TFF_ARG(nsys >= 1 && nsys <= b->desc.max_systems, "nsys %d outside [1, %d]", nsys, b->desc.max_systems);
  TFF_ARG(natoms && pme_grid && coords && boxes && charges && sigma && epsilon && excl && energies && forces,
          "NULL argument");
  cudaStream_t s = (cudaStream_t)stream;
  if (b->desc.dtype == TFF_F32)
    return batch_eval_impl<float>(b, nsys, natoms, pme_grid, (const float *)coords, (const float *)boxes,
                                  (const float *)charges, (const float *)sigma, (const float *)epsilon, excl, energies,
                                  (float *)forces, s);
  return batch_eval_impl<double>(b, nsys, natoms, pme_grid, (const double *)coords, (const double *)boxes,
                                 (const double *)charges, (const double *)sigma, (const double *)epsilon, excl,
                                 energies, (double *)forces, s);
}

int tff_batch_status(tff_batch b, tff_stream_t stream, int *status) {
  TFF_ARG(b != nullptr && status != nullptr, "batch/status is NULL");
  unsigned v = 0;
  TFF_CUDA(cudaMemcpyAsync(&v, b->ws + b->L.status, sizeof(unsigned), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
  TFF_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
  *status = (int)v;
  return TFF_OK;
}

int tff_batch_kernel_launches(tff_batch b) {
  if (!b) return 0;
  // sort, bounds, neighbours, params, tile, finalize; spread, [to_real], 3 DFT passes,
  // convolve, 3 inverse passes, gather
  return 6 + (b->desc.dtype == TFF_F32 ? 10 : 9);
}

}  // extern "C"

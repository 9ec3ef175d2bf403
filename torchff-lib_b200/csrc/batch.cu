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
#include <cstring>
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

// Bytes before the system table in the uploaded block (the BatchShape sits there).
constexpr size_t kTableOffset = 256;
// Points of a batched convolution work unit: 8 per thread of a 256-thread block.
constexpr int64_t kConvPointsPerUnit = 8 * 256;
// Atoms (sorted slots) of a batched gather work unit: four passes of a 256-thread block at
// 5 atoms per warp.
constexpr int64_t kGatherAtomsPerUnit = 4 * (256 / 32) * 5;
static_assert(sizeof(BatchShape) <= kTableOffset, "BatchShape must fit before the system table");

struct BatchLayout {
  int64_t atoms, systems, clusters, supers, grid;
  int cap;
  size_t shape, sys, status, boxinfo, cl_sys, sup_sys, sidx, inv, pos, frac, bc, bh, sbc, sbh, nbr, ncount, itemoff, items;
  size_t lj, exslot, acc, e_tile;
  size_t fix, real, cplx, partials, tickets, e_pme, pme_grad, pme_phi, moduli, twiddle;
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
  // shape and system table: one upload per evaluation (shape first, the table 256 bytes on)
  L.shape = take(kTableOffset + max_systems * sizeof(BatchSys));
  L.sys = L.shape + kTableOffset;
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
  L.twiddle = take((size_t)twiddle_offset(kBatchMaxK + 1) * 2 * ts);
  L.bytes = c.bytes();
  return L;
}

}  // namespace
}  // namespace tff

using namespace tff;

// Device pointers of one evaluation and the DFT size class: a captured graph replays only
// for the same key.
struct BatchGraphKey {
  const void *ptr[10];
  int dft_class;
  bool operator==(const BatchGraphKey &o) const {
    if (dft_class != o.dft_class) return false;
    for (int k = 0; k < 10; ++k)
      if (ptr[k] != o.ptr[k]) return false;
    return true;
  }
};

struct tff_batch_s {
  tff_batch_desc desc;
  BatchLayout L;
  char *ws = nullptr;
  unsigned char *table = nullptr;  // pinned host copy of the shape + system table block
  cudaEvent_t table_ev = nullptr;  // the table upload of the previous evaluation
  cudaStream_t pme_stream = nullptr;
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
  cudaEvent_t sorted_ev = nullptr;  // batch sort done (the PME gather visits its atom order)
  std::vector<BatchSys> host_sys;
  int device = 0;
  // CUDA graphs of the evaluation (launch shapes depend on the capacity alone, the batch's
  // composition is read from the uploaded shape): captured when a call repeats the
  // previous call's key, replayed for every later call with that key
  cudaStream_t capture_stream = nullptr;
  std::vector<std::pair<BatchGraphKey, cudaGraphExec_t>> graphs;
  BatchGraphKey last_key{};
  bool have_last = false;
  int64_t graph_launches = 0;
};

namespace tff {
namespace {

void free_batch(tff_batch b) {
  if (!b) return;
  for (auto &g : b->graphs) cudaGraphExecDestroy(g.second);
  if (b->capture_stream) cudaStreamDestroy(b->capture_stream);
  if (b->ws) cudaFree(b->ws);
  if (b->table) cudaFreeHost(b->table);
  if (b->table_ev) cudaEventDestroy(b->table_ev);
  if (b->pme_stream) cudaStreamDestroy(b->pme_stream);
  if (b->fork_ev) cudaEventDestroy(b->fork_ev);
  if (b->join_ev) cudaEventDestroy(b->join_ev);
  if (b->sorted_ev) cudaEventDestroy(b->sorted_ev);
  delete b;
}

// DFT shared-memory size class of a batch, part of the graph key: 52 for grid sides up to
// 52 (every water box up to 4,000 waters at 0.1 nm spacing), else the dtype's limit. A
// class costs a capture per lane, and the shared memory of the class sets the resident DFT
// blocks: 5 per SM at 52 (FP32), where a 56 class gave 4 (25 % slower passes) and 64 gave 3.
constexpr int kDftSmallClass = 52;
inline int dft_class(int kmax, int kcap) { return kmax <= kDftSmallClass ? std::min(kcap, kDftSmallClass) : kcap; }

// Host part of an evaluation: system table (offsets, cell grids, PME and DFT work units)
// and shape into the pinned block, after the previous upload out of it is done. Returns
// the table's largest grid side in *kmax.
template <class T>
int batch_prepare(tff_batch b, int nsys, const int64_t *natoms, const int *pme_grid, int *kmax_out) {
  const BatchLayout &L = b->L;
  auto &hs = b->host_sys;
  hs.assign(nsys, BatchSys{});
  int64_t ao = 0, co = 0, so = 0, go = 0, xo = 0;
  int planes = 0, conv = 0, gat = 0;
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
    y.plane_off = planes;
    // the convolution's units cover kConvPointsPerUnit points each (its PME blocks, sized
    // for the atoms, mostly held a few points per thread at most)
    y.conv_blocks = (int)std::min<int64_t>(kBatchPmeMaxBlocks, std::max<int64_t>(1, (ncplx + kConvPointsPerUnit - 1) / kConvPointsPerUnit));
    y.conv_off = conv;
    // the gather's units take kGatherAtomsPerUnit atoms (the sorted slots of its clusters)
    y.gather_blocks = (int)std::min<int64_t>(kBatchPmeMaxBlocks, std::max<int64_t>(1, (y.ncl * kWarp + kGatherAtomsPerUnit - 1) / kGatherAtomsPerUnit));
    y.gather_off = gat;
    planes += K;
    conv += y.conv_blocks;
    gat += y.gather_blocks;
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
  BatchShape sh{};
  sh.natoms = ao;
  sh.nclusters = co;
  sh.npad = co * kWarp;
  sh.nsuper = so;
  sh.total_grid = go;
  sh.nsys = nsys;
  sh.plane_units = planes;
  sh.kmax = kmax;
  sh.conv_units = conv;
  sh.gather_units = gat;
  // the pinned block is reused once the previous upload out of it is done
  TFF_CUDA(cudaEventSynchronize(b->table_ev));
  std::memcpy(b->table, &sh, sizeof(sh));
  std::memcpy(b->table + kTableOffset, hs.data(), nsys * sizeof(BatchSys));
  *kmax_out = kmax;
  return TFF_OK;
}

// Device part of an evaluation on stream s (PME on the batch's second stream, joined back):
// every launch shape depends on the batch's capacity and the DFT class alone, so the
// sequence can be captured once and replayed for any composition of that class.
template <class T>
int batch_enqueue(tff_batch b, int kclass, const T *x, const T *boxes, const T *q, const T *sigma, const T *eps,
                  const int *excl, double *energies, T *forces, cudaStream_t s) {
  using S = typename Acc<T>::S;
  const BatchLayout &L = b->L;
  char *w = b->ws;
  const int sms = sm_count();
  const int64_t slots_cap = L.clusters * kWarp;
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
  // sizes come from the shape on the device; the capacities stand here
  cd.natoms = L.atoms;
  cd.nclusters = L.clusters;
  cd.npad = slots_cap;
  cd.nsuper = L.supers;
  cd.sys = reinterpret_cast<const BatchSys *>(w + L.sys);
  cd.cl_sys = reinterpret_cast<int *>(w + L.cl_sys);
  cd.sup_sys = reinterpret_cast<int *>(w + L.sup_sys);
  cd.shape = reinterpret_cast<const BatchShape *>(w + L.shape);
  const BatchShape *shape = cd.shape;
  const BatchSys *dsys = cd.sys;

  TFF_CUDA(cudaMemsetAsync(w + L.status, 0, 64 * sizeof(unsigned), s));
  TFF_CUDA(cudaMemsetAsync(w + L.e_tile, 0, 2 * L.systems * 8, s));

  // --- PME on the side stream
  TFF_CUDA(cudaEventRecord(b->fork_ev, s));
  cudaStream_t ps = b->pme_stream;
  TFF_CUDA(cudaStreamWaitEvent(ps, b->fork_ev, 0));
  TFF_CUDA(cudaMemsetAsync(w + L.tickets, 0, 2 * L.systems * sizeof(unsigned), ps));
  double *partials = reinterpret_cast<double *>(w + L.partials);
  unsigned *tickets = reinterpret_cast<unsigned *>(w + L.tickets);
  double *e_pme = reinterpret_cast<double *>(w + L.e_pme);
  S *fix = reinterpret_cast<S *>(w + L.fix);
  T *pme_grad = reinterpret_cast<T *>(w + L.pme_grad);
  T *pme_phi = reinterpret_cast<T *>(w + L.pme_phi);
  const int nb_pme = sms * 8;
  batch_zero_grid_kernel<S><<<sms * 8, 256, 0, ps>>>(shape, fix);
  TFF_LAUNCHED();
  // work-unit counters of the persistent PME kernels: status words 16.. (zeroed above)
  unsigned *counters = cd.status + 16;
  batch_spread_kernel<T><<<nb_pme, kPmeBlock, 0, ps>>>(dsys, shape, x, q, boxes, fix, counters);
  TFF_LAUNCHED();
  T *real;
  if (sizeof(T) == 4) {
    real = reinterpret_cast<T *>(w + L.real);
    batch_fix_to_real_kernel<<<sms * 8, 256, 0, ps>>>(shape, reinterpret_cast<unsigned long long *>(fix),
                                                     reinterpret_cast<float *>(real));
    TFF_LAUNCHED();
  } else {
    real = reinterpret_cast<T *>(fix);
  }
  auto *cplx = reinterpret_cast<typename CplxOf<T>::type *>(w + L.cplx);
  const auto *twtab = reinterpret_cast<const typename CplxOf<T>::type *>(w + L.twiddle);
  const size_t dsmem = batch_dft_smem<T>(kclass);
  const int nb_dft = sms * 8;
  batch_dft_kernel<T, kDftZR2C><<<nb_dft, kDftThreads, dsmem, ps>>>(dsys, shape, real, cplx, twtab, counters + 1);
  TFF_LAUNCHED();
  batch_dft_kernel<T, kDftY><<<nb_dft, kDftThreads, dsmem, ps>>>(dsys, shape, real, cplx, twtab, counters + 2);
  TFF_LAUNCHED();
  batch_dft_kernel<T, kDftX><<<nb_dft, kDftThreads, dsmem, ps>>>(dsys, shape, real, cplx, twtab, counters + 3);
  TFF_LAUNCHED();
  batch_convolve_kernel<T><<<nb_pme, kPmeBlock, 0, ps>>>(dsys, shape, cplx, boxes, b->desc.ewald_alpha,
                                                         reinterpret_cast<const T *>(w + L.moduli), partials, tickets,
                                                         e_pme, counters + 4);
  TFF_LAUNCHED();
  batch_dft_kernel<T, kDftXInv><<<nb_dft, kDftThreads, dsmem, ps>>>(dsys, shape, real, cplx, twtab, counters + 5);
  TFF_LAUNCHED();
  batch_dft_kernel<T, kDftYInv><<<nb_dft, kDftThreads, dsmem, ps>>>(dsys, shape, real, cplx, twtab, counters + 6);
  TFF_LAUNCHED();
  batch_dft_kernel<T, kDftZC2R><<<nb_dft, kDftThreads, dsmem, ps>>>(dsys, shape, real, cplx, twtab, counters + 7);
  TFF_LAUNCHED();

  // --- real space on the caller stream
  S *gx = reinterpret_cast<S *>(w + L.acc);
  S *gq = gx + 3 * slots_cap;
  batch_sort_kernel<T><<<(int)std::min<int64_t>(L.systems, 2 * sms), kBatchSortThreads, kBatchSortSmem, s>>>(
      x, q, boxes, cd, reinterpret_cast<unsigned long long *>(gx), slots_cap);
  TFF_LAUNCHED();
  // the PME gather follows the sort's atom order
  TFF_CUDA(cudaEventRecord(b->sorted_ev, s));
  TFF_CUDA(cudaStreamWaitEvent(ps, b->sorted_ev, 0));
  batch_gather_kernel<T><<<nb_pme, kPmeBlock, 0, ps>>>(dsys, shape, x, q, cd.sidx, boxes, real, b->desc.ewald_alpha,
                                                       pme_phi, pme_grad, partials, tickets, e_pme, counters + 8);
  TFF_LAUNCHED();
  TFF_CUDA(cudaEventRecord(b->join_ev, ps));
  cluster_bounds_kernel<T><<<(int)std::max<int64_t>(1, std::min<int64_t>(L.supers, 2 * sms)), kWarp * kSuper, 0, s>>>(cd);
  TFF_LAUNCHED();
  const int nb_cl = (int)std::max<int64_t>(1, std::min<int64_t>((L.clusters + 3) / 4, sms * 16));
  cluster_neighbors_kernel<T><<<nb_cl, 128, 0, s>>>(cd, b->desc.cutoff, kHalfLists<T>);
  TFF_LAUNCHED();
  auto *lj = reinterpret_cast<typename V2<T>::type *>(w + L.lj);
  int *exslot = reinterpret_cast<int *>(w + L.exslot);
  {
    const int nb = (int)std::max<int64_t>(1, std::min<int64_t>((slots_cap + 255) / 256, sms * 8));
    sorted_params_kernel<T><<<nb, 256, 0, s>>>(cd, sigma, eps, excl, lj, exslot);
    TFF_LAUNCHED();
  }
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
    const int64_t max_items = L.clusters * ((L.cap + kItemTiles - 1) / kItemTiles);
    const int st_rs = launch_real_space<T>(false, max_items, sms, s, A);
    if (st_rs != TFF_OK) return st_rs;
  }
  TFF_CUDA(cudaStreamWaitEvent(s, b->join_ev, 0));
  const int nbf = (int)std::max<int64_t>(1, std::min<int64_t>((L.atoms + 255) / 256, sms * 8));
  finalize_kernel<T><<<nbf, 256, 0, s>>>(cd, gx, gq, pme_grad, pme_phi, forces, (double *)nullptr, (T *)nullptr,
                                         e_tile, e_pme, b->desc.coul_constant, energies, (double *)nullptr,
                                         (int)L.systems);
  TFF_LAUNCHED();
  return TFF_OK;
}

// Most graphs a batch keeps (one per DFT class and buffer set; the oldest goes first).
constexpr size_t kBatchMaxGraphs = 8;

// Captures the device part for `key` (nothing runs) and appends the graph to the batch's
// list.
template <class T>
int batch_capture(tff_batch b, const BatchGraphKey &key, const T *x, const T *boxes, const T *q, const T *sigma,
                  const T *eps, const int *excl, double *energies, T *forces) {
  if (b->capture_stream == nullptr) TFF_CUDA(cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking));
  TFF_CUDA(cudaStreamBeginCapture(b->capture_stream, cudaStreamCaptureModeThreadLocal));
  const int st = batch_enqueue<T>(b, key.dft_class, x, boxes, q, sigma, eps, excl, energies, forces,
                                  b->capture_stream);
  cudaGraph_t graph = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(b->capture_stream, &graph);
  if (st != TFF_OK || ee != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    if (st != TFF_OK) return st;
    return cuda_fail(ee, "batch graph capture", __FILE__, __LINE__);
  }
  cudaGraphExec_t exec = nullptr;
  const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ie != cudaSuccess) return cuda_fail(ie, "cudaGraphInstantiate", __FILE__, __LINE__);
  if (b->graphs.size() >= kBatchMaxGraphs) {
    cudaGraphExecDestroy(b->graphs.front().second);
    b->graphs.erase(b->graphs.begin());
  }
  b->graphs.emplace_back(key, exec);
  return TFF_OK;
}

template <class T>
int batch_eval_impl(tff_batch b, int nsys, const int64_t *natoms, const int *pme_grid, const T *x, const T *boxes,
                    const T *q, const T *sigma, const T *eps, const int *excl, double *energies, T *forces,
                    cudaStream_t s) {
  int kmax = 6;
  int st = batch_prepare<T>(b, nsys, natoms, pme_grid, &kmax);
  if (st != TFF_OK) return st;
  const int kclass = dft_class(kmax, sizeof(T) == 8 ? kBatchMaxK64 : kBatchMaxK);
  // upload the shape and the table (exact size), then run the device part
  TFF_CUDA(cudaMemcpyAsync(b->ws + b->L.shape, b->table, kTableOffset + nsys * sizeof(BatchSys),
                           cudaMemcpyHostToDevice, s));
  TFF_CUDA(cudaEventRecord(b->table_ev, s));
  const BatchGraphKey key{{x, boxes, q, sigma, eps, excl, energies, forces, nullptr, nullptr}, kclass};
  auto it = std::find_if(b->graphs.begin(), b->graphs.end(), [&](const auto &g) { return g.first == key; });
  if (it == b->graphs.end() && b->have_last && b->last_key == key) {
    // the same buffers and class twice in a row: capture the device part once
    if ((st = batch_capture<T>(b, key, x, boxes, q, sigma, eps, excl, energies, forces)) != TFF_OK) return st;
    it = b->graphs.end() - 1;
  }
  b->last_key = key;
  b->have_last = true;
  if (it != b->graphs.end()) {
    ++b->graph_launches;
    TFF_CUDA(cudaGraphLaunch(it->second, s));
    return TFF_OK;
  }
  return batch_enqueue<T>(b, kclass, x, boxes, q, sigma, eps, excl, energies, forces, s);
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

// Captures the graph of the batch's common DFT class (grid sides up to 52) for these
// device buffers ahead of use, so that the first evaluations through them need no capture
// (used for the server's lanes, whose staging buffers never change).
int batch_warm_graph(tff_batch b, const void *coords, const void *boxes, const void *charges, const void *sigma,
                     const void *epsilon, const int *excl, double *energies, void *forces) {
  const int kcap = b->desc.dtype == TFF_F64 ? kBatchMaxK64 : kBatchMaxK;
  const BatchGraphKey key{{coords, boxes, charges, sigma, epsilon, excl, energies, forces, nullptr, nullptr},
                          dft_class(6, kcap)};
  if (b->desc.dtype == TFF_F32)
    return batch_capture<float>(b, key, (const float *)coords, (const float *)boxes, (const float *)charges,
                                (const float *)sigma, (const float *)epsilon, excl, energies, (float *)forces);
  return batch_capture<double>(b, key, (const double *)coords, (const double *)boxes, (const double *)charges,
                               (const double *)sigma, (const double *)epsilon, excl, energies, (double *)forces);
}

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
  if (e == cudaSuccess) e = cudaMallocHost((void **)&b->table, kTableOffset + desc->max_systems * sizeof(BatchSys));
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
  if (e == cudaSuccess) {
    // twiddles of every grid side the batch accepts (the DFT passes read them per plane)
    if (desc->dtype == TFF_F64)
      batch_twiddle_kernel<double><<<64, 256>>>(reinterpret_cast<CplxOf<double>::type *>(b->ws + b->L.twiddle),
                                                kBatchMaxK);
    else
      batch_twiddle_kernel<float><<<64, 256>>>(reinterpret_cast<CplxOf<float>::type *>(b->ws + b->L.twiddle),
                                               kBatchMaxK);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(nullptr);  // the PME streams do not wait for stream 0
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

int64_t tff_batch_graph_launches(tff_batch b) { return b ? b->graph_launches : 0; }

int tff_batch_kernel_launches(tff_batch b) {
  if (!b) return 0;
  // sort, bounds, neighbours, params, pair kernel, finalize; grid zeroing, spread,
  // [to_real], 3 DFT passes, convolve, 3 inverse passes, gather
  return 6 + (b->desc.dtype == TFF_F32 ? 11 : 10);
}

}  // extern "C"

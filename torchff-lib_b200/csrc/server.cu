// Continuous-batching server over tff_batch: requests (one periodic system each, host
// arrays) queue up; a worker thread keeps `lanes` batches in flight, each on its own
// stream with its own device memory. Whenever a lane is free and requests wait, the lane
// takes as many of them (in arrival order) as fit its capacity, copies them to the device,
// evaluates them in one batched pass and copies the results back; a lane whose completion
// event has fired hands the results to their requests. Requests that arrive while other
// batches are on the GPU therefore start as soon as a lane frees up, and the batches of
// different lanes overlap on the device.
//
// Device memory: the HBM budget is split evenly over the lanes; each lane's capacity in
// atoms and PME grid points is the largest whose batch workspace plus staging fits its
// share (tff_batch_device_bytes), and a request joins a batch only while the batch stays
// within that capacity.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "tff_common.cuh"

namespace tff {
namespace {

constexpr int kExclSlots = 8;  // partner slots per atom in the batch exclusion table

struct ServerReq {
  int64_t id = 0;
  int64_t n = 0;
  int K = 0;
  std::vector<unsigned char> coords, params, box;  // in the server dtype: (n,3), (3,n) q|sigma|eps, (9)
  std::vector<int> excl;                            // (n, 8) local partner indices, -1 padded
  double *energy_out = nullptr, *forces_out = nullptr;
  double t_submit = 0.0, t_start = 0.0, t_done = 0.0;
  int status = TFF_OK;
  bool done = false;
  int waiters = 0;  // threads inside tff_server_wait on this request (release refuses while > 0)
};

struct Lane {
  tff_batch batch = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t done_ev = nullptr;
  int64_t max_atoms = 0, max_grid = 0;
  int max_systems = 0;
  unsigned char *h_in = nullptr, *h_out = nullptr, *d_in = nullptr, *d_out = nullptr;
  size_t in_bytes = 0, out_bytes = 0;
  std::vector<ServerReq *> reqs;
  std::vector<int64_t> natoms;
  std::vector<int> K;
  bool busy = false;
  // staging offsets (bytes): coords | q | sigma | eps (atoms), boxes (systems), excl
  size_t o_x = 0, o_q = 0, o_s = 0, o_e = 0, o_box = 0, o_excl = 0, o_f = 0;
};

}  // namespace
}  // namespace tff

using namespace tff;

struct tff_server_s {
  tff_server_desc desc;
  size_t ts = 4;
  int device = 0;
  std::vector<Lane> lanes;
  std::deque<ServerReq *> queue;
  std::unordered_map<int64_t, ServerReq *> reqs;
  int64_t next_id = 1;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::thread worker;
  bool stop = false;
  bool hold = false;  // no new batch starts while set (requests keep queueing)
  int waiting = 0;    // threads inside tff_server_wait / tff_server_drain (destroy waits for 0)
  int fatal = TFF_OK;
  std::chrono::steady_clock::time_point t0;
  tff_server_stats stats{};
  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

namespace tff {
namespace {

void free_lane(Lane &l) {
  if (l.batch) tff_batch_destroy(l.batch);
  if (l.stream) cudaStreamDestroy(l.stream);
  if (l.done_ev) cudaEventDestroy(l.done_ev);
  if (l.h_in) cudaFreeHost(l.h_in);
  if (l.h_out) cudaFreeHost(l.h_out);
  if (l.d_in) cudaFree(l.d_in);
  if (l.d_out) cudaFree(l.d_out);
  l = Lane{};
}

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

void lane_offsets(Lane &l, size_t ts) {
  size_t o = 0;
  l.o_x = o; o = align256(o + 3 * l.max_atoms * ts);
  l.o_q = o; o = align256(o + l.max_atoms * ts);
  l.o_s = o; o = align256(o + l.max_atoms * ts);
  l.o_e = o; o = align256(o + l.max_atoms * ts);
  l.o_box = o; o = align256(o + 9 * (size_t)l.max_systems * ts);
  l.o_excl = o; o = align256(o + kExclSlots * l.max_atoms * sizeof(int));
  l.in_bytes = o;
  l.o_f = align256((size_t)l.max_systems * sizeof(double));
  l.out_bytes = align256(l.o_f + 3 * l.max_atoms * ts);
}

tff_batch_desc lane_batch_desc(const tff_server_desc &d, int64_t atoms, int64_t grid) {
  tff_batch_desc b{};
  b.dtype = d.dtype;
  b.max_systems = d.max_systems_per_batch;
  b.max_atoms = atoms;
  b.max_grid_points = grid;
  b.cutoff = d.cutoff;
  b.ewald_alpha = d.ewald_alpha;
  b.coul_constant = d.coul_constant;
  b.max_cluster_neighbors = 0;
  b.atoms_per_cell = d.atoms_per_cell;
  return b;
}

// Device bytes of one lane holding `atoms` atoms (grid capacity in proportion).
size_t lane_device_bytes(const tff_server_desc &d, int64_t atoms, size_t ts) {
  const int64_t grid = (int64_t)(atoms * d.grid_points_per_atom) + 96 * 96 * 96;
  Lane l;
  l.max_atoms = atoms;
  l.max_systems = d.max_systems_per_batch;
  lane_offsets(l, ts);
  tff_batch_desc bd = lane_batch_desc(d, atoms, grid);
  return tff_batch_device_bytes(&bd) + l.in_bytes + l.out_bytes;
}

// Results of requests [i0, i1) of a finished lane into their host buffers.
void unpack_requests(const Lane &l, size_t ts, const std::vector<int64_t> &off, int i0, int i1) {
  const double *e = reinterpret_cast<const double *>(l.h_out);
  for (int i = i0; i < i1; ++i) {
    ServerReq *r = l.reqs[i];
    const int64_t ao = off[i];
    if (r->energy_out) *r->energy_out = e[i];
    if (r->forces_out) {
      const int64_t m = 3 * r->n;
      if (ts == 8) {
        std::memcpy(r->forces_out, l.h_out + l.o_f + 3 * ao * 8, m * 8);
      } else {
        const float *f = reinterpret_cast<const float *>(l.h_out + l.o_f) + 3 * ao;
        for (int64_t k = 0; k < m; ++k) r->forces_out[k] = f[k];
      }
    }
  }
}

// Runs fn(i0, i1) over the requests of a lane, split over up to 4 threads for large batches.
template <class F>
void over_requests(const Lane &l, const std::vector<int64_t> &off, F fn) {
  const int nsys = (int)l.reqs.size();
  const int64_t ao = off[nsys];
  const int nthr = ao >= 65536 ? std::min(4, std::max(1, (int)std::thread::hardware_concurrency() / 2)) : 1;
  if (nthr <= 1) {
    fn(0, nsys);
    return;
  }
  std::vector<std::thread> pool;
  int i0 = 0;
  for (int t = 0; t < nthr; ++t) {
    const int64_t goal = ao * (t + 1) / nthr;
    int i1 = i0;
    while (i1 < nsys && (t == nthr - 1 || off[i1] < goal)) ++i1;
    pool.emplace_back(fn, i0, i1);
    i0 = i1;
  }
  for (auto &th : pool) th.join();
}

std::vector<int64_t> atom_offsets(const Lane &l) {
  std::vector<int64_t> off(l.reqs.size() + 1, 0);
  for (size_t i = 0; i < l.reqs.size(); ++i) off[i + 1] = off[i] + l.reqs[i]->n;
  return off;
}

// Results of a finished lane into the requests' host buffers (worker thread, no lock).
void unpack_lane(tff_server s, Lane &l) {
  const std::vector<int64_t> off = atom_offsets(l);
  const size_t ts = s->ts;
  over_requests(l, off, [&](int i0, int i1) { unpack_requests(l, ts, off, i0, i1); });
}

// Copies requests [i0, i1) of a lane into its pinned staging buffer (atom offsets in off).
void pack_requests(const Lane &l, size_t ts, const std::vector<int64_t> &off, int i0, int i1) {
  for (int i = i0; i < i1; ++i) {
    const ServerReq *r = l.reqs[i];
    const int64_t n = r->n, ao = off[i];
    std::memcpy(l.h_in + l.o_x + 3 * ao * ts, r->coords.data(), 3 * n * ts);
    std::memcpy(l.h_in + l.o_q + ao * ts, r->params.data(), n * ts);
    std::memcpy(l.h_in + l.o_s + ao * ts, r->params.data() + n * ts, n * ts);
    std::memcpy(l.h_in + l.o_e + ao * ts, r->params.data() + 2 * n * ts, n * ts);
    std::memcpy(l.h_in + l.o_box + 9 * (size_t)i * ts, r->box.data(), 9 * ts);
    std::memcpy(l.h_in + l.o_excl + kExclSlots * ao * sizeof(int), r->excl.data(), kExclSlots * n * sizeof(int));
  }
}

int launch_lane(tff_server s, Lane &l) {
  TFF_NVTX("tff_server_batch");
  const size_t ts = s->ts;
  const int nsys = (int)l.reqs.size();
  l.natoms.resize(nsys);
  l.K.resize(nsys);
  for (int i = 0; i < nsys; ++i) {
    l.natoms[i] = l.reqs[i]->n;
    l.K[i] = l.reqs[i]->K;
  }
  // large batches are copied by several threads (one core's memory bandwidth is the limit
  // otherwise), split into runs of about equal atom counts
  const std::vector<int64_t> off = atom_offsets(l);
  const int64_t ao = off[nsys];
  over_requests(l, off, [&](int i0, int i1) { pack_requests(l, ts, off, i0, i1); });
  cudaStream_t st = l.stream;
  auto h2d = [&](size_t off, size_t bytes) {
    return cudaMemcpyAsync(l.d_in + off, l.h_in + off, bytes, cudaMemcpyHostToDevice, st);
  };
  TFF_CUDA(h2d(l.o_x, 3 * ao * ts));
  TFF_CUDA(h2d(l.o_q, ao * ts));
  TFF_CUDA(h2d(l.o_s, ao * ts));
  TFF_CUDA(h2d(l.o_e, ao * ts));
  TFF_CUDA(h2d(l.o_box, 9 * (size_t)nsys * ts));
  TFF_CUDA(h2d(l.o_excl, kExclSlots * ao * sizeof(int)));
  double *d_energy = reinterpret_cast<double *>(l.d_out);
  int rc = tff_batch_eval(l.batch, nsys, l.natoms.data(), l.K.data(), l.d_in + l.o_x, l.d_in + l.o_box,
                          l.d_in + l.o_q, l.d_in + l.o_s, l.d_in + l.o_e,
                          reinterpret_cast<const int *>(l.d_in + l.o_excl), d_energy, l.d_out + l.o_f,
                          (tff_stream_t)st);
  if (rc != TFF_OK) return rc;
  TFF_CUDA(cudaMemcpyAsync(l.h_out, l.d_out, nsys * sizeof(double), cudaMemcpyDeviceToHost, st));
  TFF_CUDA(cudaMemcpyAsync(l.h_out + l.o_f, l.d_out + l.o_f, 3 * ao * ts, cudaMemcpyDeviceToHost, st));
  TFF_CUDA(cudaEventRecord(l.done_ev, st));
  return TFF_OK;
}

void worker_loop(tff_server s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (true) {
    bool progress = false;
    for (Lane &l : s->lanes) {
      if (!l.busy) continue;
      lk.unlock();
      const cudaError_t q = cudaEventQuery(l.done_ev);
      int st = TFF_OK;
      if (q == cudaSuccess) unpack_lane(s, l);
      else if (q != cudaErrorNotReady) st = cuda_fail(q, "batch completion", __FILE__, __LINE__);
      lk.lock();
      if (q == cudaErrorNotReady) continue;
      const double t = s->now();
      for (ServerReq *r : l.reqs) {
        r->t_done = t;
        r->status = st;
        r->done = true;
      }
      s->stats.systems_done += (int64_t)l.reqs.size();
      l.reqs.clear();
      l.busy = false;
      if (st != TFF_OK) s->fatal = st;
      progress = true;
      s->cv_done.notify_all();
    }
    for (Lane &l : s->lanes) {
      if (l.busy || s->queue.empty() || s->fatal != TFF_OK || s->hold) continue;
      int64_t atoms = 0, grid = 0;
      while (!s->queue.empty() && (int)l.reqs.size() < l.max_systems) {
        ServerReq *r = s->queue.front();
        const int64_t g = (int64_t)r->K * r->K * r->K;
        if (atoms + r->n > l.max_atoms || grid + g > l.max_grid) break;
        atoms += r->n;
        grid += g;
        l.reqs.push_back(r);
        s->queue.pop_front();
      }
      if (l.reqs.empty()) continue;
      const double t = s->now();
      for (ServerReq *r : l.reqs) r->t_start = t;
      lk.unlock();
      const int st = launch_lane(s, l);
      lk.lock();
      s->stats.batches += 1;
      s->stats.systems_launched += (int64_t)l.reqs.size();
      s->stats.max_batch_systems = std::max<int64_t>(s->stats.max_batch_systems, (int64_t)l.reqs.size());
      s->stats.max_batch_atoms = std::max<int64_t>(s->stats.max_batch_atoms, atoms);
      if (st != TFF_OK) {
        for (ServerReq *r : l.reqs) {
          r->status = st;
          r->done = true;
          r->t_done = s->now();
        }
        l.reqs.clear();
        s->fatal = st;
        s->cv_done.notify_all();
      } else {
        l.busy = true;
        int inflight = 0;
        for (const Lane &o : s->lanes) inflight += o.busy ? 1 : 0;
        s->stats.max_lanes_in_flight = std::max<int64_t>(s->stats.max_lanes_in_flight, inflight);
      }
      progress = true;
    }
    if (s->fatal != TFF_OK && !s->queue.empty()) {
      // after a failed batch the remaining requests fail too instead of waiting forever
      const double t = s->now();
      for (ServerReq *r : s->queue) {
        r->status = s->fatal;
        r->done = true;
        r->t_done = t;
        s->stats.systems_done += 1;
      }
      s->queue.clear();
      s->cv_done.notify_all();
    }
    bool any_busy = false;
    for (const Lane &l : s->lanes) any_busy |= l.busy;
    if (s->stop && !any_busy && (s->queue.empty() || s->fatal != TFF_OK)) break;
    if (progress) continue;
    if (!any_busy) {
      s->cv_work.wait(lk, [&] { return s->stop || (!s->queue.empty() && !s->hold); });
    } else {
      lk.unlock();
      std::this_thread::yield();
      lk.lock();
    }
  }
}

void free_server(tff_server s) {
  if (!s) return;
  if (s->worker.joinable()) {
    {
      std::lock_guard<std::mutex> g(s->mu);
      s->stop = true;
      s->hold = false;
    }
    s->cv_work.notify_all();
    s->worker.join();
    // every request is done now; let threads still inside a wait leave it before the
    // mutex and the requests go away
    std::unique_lock<std::mutex> lk(s->mu);
    s->cv_done.wait(lk, [&] { return s->waiting == 0; });
  }
  for (Lane &l : s->lanes) free_lane(l);
  for (auto &kv : s->reqs) delete kv.second;  // every queued request is in the map too
  delete s;
}

}  // namespace
}  // namespace tff

extern "C" {

int tff_server_create(const tff_server_desc *desc, tff_server *out) {
  TFF_ARG(desc != nullptr && out != nullptr, "desc/out is NULL");
  TFF_ARG(desc->dtype == TFF_F32 || desc->dtype == TFF_F64, "dtype must be TFF_F32 or TFF_F64");
  TFF_ARG(desc->lanes >= 1 && desc->lanes <= 16, "lanes must be in [1, 16]");
  TFF_ARG(desc->max_systems_per_batch >= 1 && desc->max_systems_per_batch <= 65535,
          "max_systems_per_batch must be in [1, 65535]");
  TFF_ARG(desc->grid_points_per_atom > 0.0, "grid_points_per_atom must be positive");
  TFF_ARG(desc->cutoff > 0.0 && desc->ewald_alpha > 0.0, "cutoff and ewald_alpha must be positive");
  auto *s = new tff_server_s();
  s->desc = *desc;
  s->ts = desc->dtype == TFF_F64 ? 8 : 4;
  s->t0 = std::chrono::steady_clock::now();
  cudaGetDevice(&s->device);
  // largest lane (in atoms, multiple of 1024) whose memory fits budget / lanes
  const size_t share = desc->hbm_budget_bytes / desc->lanes;
  int64_t lo = 0, hi = (int64_t)1 << 22;
  while (hi - lo > 1024) {
    const int64_t mid = (lo + hi) / 2;
    if (lane_device_bytes(*desc, mid, s->ts) <= share) lo = mid;
    else hi = mid;
  }
  if (lo < 16384) {
    delete s;
    set_error("HBM budget %zu bytes over %d lanes is too small for one 16384-atom system per lane",
              desc->hbm_budget_bytes, desc->lanes);
    return TFF_ERR_INVALID;
  }
  s->lanes.resize(desc->lanes);
  for (Lane &l : s->lanes) {
    l.max_atoms = lo;
    l.max_grid = (int64_t)(lo * desc->grid_points_per_atom) + 96 * 96 * 96;
    l.max_systems = desc->max_systems_per_batch;
    lane_offsets(l, s->ts);
    tff_batch_desc bd = lane_batch_desc(*desc, l.max_atoms, l.max_grid);
    int st = tff_batch_create(&bd, &l.batch);
    cudaError_t e = cudaSuccess;
    if (st == TFF_OK) e = cudaStreamCreateWithFlags(&l.stream, cudaStreamNonBlocking);
    if (st == TFF_OK && e == cudaSuccess) e = cudaEventCreateWithFlags(&l.done_ev, cudaEventDisableTiming);
    if (st == TFF_OK && e == cudaSuccess) e = cudaMallocHost((void **)&l.h_in, l.in_bytes);
    if (st == TFF_OK && e == cudaSuccess) e = cudaMallocHost((void **)&l.h_out, l.out_bytes);
    if (st == TFF_OK && e == cudaSuccess) e = cudaMalloc((void **)&l.d_in, l.in_bytes);
    if (st == TFF_OK && e == cudaSuccess) e = cudaMalloc((void **)&l.d_out, l.out_bytes);
    // the lane's staging buffers never change: its graph of the common DFT class is
    // captured now rather than on the way of the first requests
    if (st == TFF_OK && e == cudaSuccess)
      st = batch_warm_graph(l.batch, l.d_in + l.o_x, l.d_in + l.o_box, l.d_in + l.o_q, l.d_in + l.o_s,
                            l.d_in + l.o_e, reinterpret_cast<const int *>(l.d_in + l.o_excl),
                            reinterpret_cast<double *>(l.d_out), l.d_out + l.o_f);
    if (st != TFF_OK || e != cudaSuccess) {
      if (st == TFF_OK) st = cuda_fail(e, "server lane set-up", __FILE__, __LINE__);
      free_server(s);
      return st;
    }
  }
  s->stats.lane_max_atoms = lo;
  s->stats.lane_max_grid_points = s->lanes[0].max_grid;
  s->stats.lane_device_bytes = (int64_t)lane_device_bytes(*desc, lo, s->ts);
  s->worker = std::thread(worker_loop, s);
  *out = s;
  return TFF_OK;
}

int tff_server_destroy(tff_server s) {
  free_server(s);
  return TFF_OK;
}

int tff_server_submit(tff_server s, const tff_request *req, int64_t *ticket) {
  TFF_ARG(s != nullptr && req != nullptr && ticket != nullptr, "server/request/ticket is NULL");
  const int64_t n = req->natoms;
  TFF_ARG(n >= 1 && n <= 16384, "natoms %lld outside [1, 16384]", (long long)n);
  const int kmax = s->desc.dtype == TFF_F64 ? 64 : 96;
  TFF_ARG(req->pme_grid >= 6 && req->pme_grid <= kmax, "pme_grid %d outside [6, %d]", req->pme_grid, kmax);
  TFF_ARG(req->coords && req->box && req->charges && req->sigma && req->epsilon, "NULL input array");
  TFF_ARG(req->nexcl == 0 || req->excl_pairs != nullptr, "exclusion pairs are NULL");
  auto *r = new ServerReq();
  r->n = n;
  r->K = req->pme_grid;
  const size_t ts = s->ts;
  r->coords.resize(3 * n * ts);
  r->params.resize(3 * n * ts);
  r->box.resize(9 * ts);
  auto put = [&](unsigned char *dst, const double *src, int64_t cnt) {
    if (ts == 8) {
      std::memcpy(dst, src, cnt * 8);
    } else {
      float *f = reinterpret_cast<float *>(dst);
      for (int64_t k = 0; k < cnt; ++k) f[k] = (float)src[k];
    }
  };
  put(r->coords.data(), req->coords, 3 * n);
  put(r->params.data(), req->charges, n);
  put(r->params.data() + n * ts, req->sigma, n);
  put(r->params.data() + 2 * n * ts, req->epsilon, n);
  put(r->box.data(), req->box, 9);
  r->excl.assign(kExclSlots * n, -1);
  std::vector<unsigned char> cnt(n, 0);
  for (int64_t e = 0; e < req->nexcl; ++e) {
    const int64_t a = req->excl_pairs[2 * e], b = req->excl_pairs[2 * e + 1];
    if (a < 0 || b < 0 || a >= n || b >= n) {
      delete r;
      set_error("exclusion pair %lld (%lld, %lld) out of range", (long long)e, (long long)a, (long long)b);
      return TFF_ERR_INVALID;
    }
    if (a == b) continue;
    for (int side = 0; side < 2; ++side) {
      const int64_t u = side ? b : a, v = side ? a : b;
      int *row = r->excl.data() + kExclSlots * u;
      bool dup = false;
      for (int k = 0; k < cnt[u]; ++k) dup |= row[k] == (int)v;
      if (dup) continue;
      if (cnt[u] == kExclSlots) {
        delete r;
        set_error("atom %lld has more than %d excluded partners", (long long)u, kExclSlots);
        return TFF_ERR_INVALID;
      }
      row[cnt[u]++] = (int)v;
    }
  }
  for (int64_t a = 0; a < n; ++a) std::sort(r->excl.data() + kExclSlots * a, r->excl.data() + kExclSlots * a + cnt[a]);
  r->energy_out = req->energy;
  r->forces_out = req->forces;
  {
    std::lock_guard<std::mutex> g(s->mu);
    if (s->fatal != TFF_OK) {
      delete r;
      set_error("server stopped after an error (status %d)", s->fatal);
      return s->fatal;
    }
    const Lane &l0 = s->lanes[0];
    if (n > l0.max_atoms || (int64_t)r->K * r->K * r->K > l0.max_grid) {
      delete r;
      set_error("request exceeds a lane's capacity");
      return TFF_ERR_CAPACITY;
    }
    r->id = s->next_id++;
    r->t_submit = s->now();
    s->reqs[r->id] = r;
    s->queue.push_back(r);
    s->stats.submitted += 1;
    *ticket = r->id;
  }
  s->cv_work.notify_one();
  return TFF_OK;
}

int tff_server_wait(tff_server s, int64_t ticket, double timeout_s) {
  TFF_ARG(s != nullptr, "server is NULL");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  TFF_ARG(it != s->reqs.end(), "unknown ticket %lld", (long long)ticket);
  ServerReq *r = it->second;
  const auto pred = [&] { return r->done; };
  r->waiters += 1;  // keeps r alive: tff_server_release refuses a request that has waiters
  s->waiting += 1;
  bool finished = true;
  if (timeout_s < 0)
    s->cv_done.wait(lk, pred);
  else
    finished = s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred);
  r->waiters -= 1;
  s->waiting -= 1;
  s->cv_done.notify_all();
  if (!finished) {
    set_error("request %lld not finished within %.3f s", (long long)ticket, timeout_s);
    return TFF_ERR_TIMEOUT;
  }
  if (r->status != TFF_OK) set_error("request %lld failed with status %d", (long long)ticket, r->status);
  return r->status;
}

int tff_server_poll(tff_server s, int64_t ticket, int *done) {
  TFF_ARG(s != nullptr && done != nullptr, "server/done is NULL");
  std::lock_guard<std::mutex> g(s->mu);
  auto it = s->reqs.find(ticket);
  TFF_ARG(it != s->reqs.end(), "unknown ticket %lld", (long long)ticket);
  *done = it->second->done ? 1 : 0;
  return TFF_OK;
}

int tff_server_request_times(tff_server s, int64_t ticket, double *t_submit, double *t_start, double *t_done) {
  TFF_ARG(s != nullptr, "server is NULL");
  std::lock_guard<std::mutex> g(s->mu);
  auto it = s->reqs.find(ticket);
  TFF_ARG(it != s->reqs.end(), "unknown ticket %lld", (long long)ticket);
  if (t_submit) *t_submit = it->second->t_submit;
  if (t_start) *t_start = it->second->t_start;
  if (t_done) *t_done = it->second->t_done;
  return TFF_OK;
}

int tff_server_release(tff_server s, int64_t ticket) {
  TFF_ARG(s != nullptr, "server is NULL");
  std::lock_guard<std::mutex> g(s->mu);
  auto it = s->reqs.find(ticket);
  TFF_ARG(it != s->reqs.end(), "unknown ticket %lld", (long long)ticket);
  TFF_ARG(it->second->done, "request %lld is still in flight", (long long)ticket);
  TFF_ARG(it->second->waiters == 0, "request %lld has a thread waiting on it", (long long)ticket);
  delete it->second;
  s->reqs.erase(it);
  return TFF_OK;
}

int tff_server_drain(tff_server s, double timeout_s) {
  TFF_ARG(s != nullptr, "server is NULL");
  std::unique_lock<std::mutex> lk(s->mu);
  const auto pred = [&] { return s->stats.systems_done >= s->stats.submitted || s->fatal != TFF_OK; };
  s->waiting += 1;
  bool finished = true;
  if (timeout_s < 0)
    s->cv_done.wait(lk, pred);
  else
    finished = s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred);
  s->waiting -= 1;
  s->cv_done.notify_all();
  if (!finished) {
    set_error("server not drained within %.3f s", timeout_s);
    return TFF_ERR_TIMEOUT;
  }
  return s->fatal;
}

int tff_server_hold(tff_server s, int hold) {
  TFF_ARG(s != nullptr, "server is NULL");
  {
    std::lock_guard<std::mutex> g(s->mu);
    s->hold = hold != 0;
  }
  s->cv_work.notify_all();
  return TFF_OK;
}

int tff_server_get_stats(tff_server s, tff_server_stats *out) {
  TFF_ARG(s != nullptr && out != nullptr, "server/stats is NULL");
  std::lock_guard<std::mutex> g(s->mu);
  *out = s->stats;
  out->now = s->now();
  return TFF_OK;
}

}  // extern "C"

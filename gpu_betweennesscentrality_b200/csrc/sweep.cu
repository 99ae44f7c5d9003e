// sweep.cu -- batched and served source sweeps of libqbc_b200.
//
// RQ of a vertex set Q is BC restricted to Q: the pair sum of RQ.cu:307-463,
// sum over s < t of sigma_sv * sigma_vt / sigma_st over pairs with d_st = d_sv + d_vt, equals
// 0.5 * sum_s delta_s(v) for each v.  Every query set therefore needs the same per-source sweep over
// all sources, and one sweep answers any number of sets:
//
//   batched  a list of query sets answered by one sweep.  The sweep's launches (per chunk of sources:
//            label scan + dependency pass) are captured once into a CUDA graph per source list and
//            tuning, then replayed; the sets' values are picked from the sweep's BC on the device.
//   served   a request loop on a host thread.  The sweep runs chunk after chunk around the source
//            list; each chunk is its own captured graph whose last kernel adds the chunk's BC into
//            the device accumulators of every admitted request.  A request is admitted at a chunk
//            boundary when a slot and room in the accumulator pool are free, and completes after one
//            full turn from there, so it sees every source exactly once whatever else is running.
//   autotune times candidate launch configurations on a sample of sources and keeps the fastest.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>

#include "device_state.h"

namespace qbc {

// acc[e.y] += part[e.x] for the first *count entries (each accumulator index appears once)
__global__ void k_gather_entries(const double *__restrict__ part, const int2 *__restrict__ ent,
                                 const int32_t *__restrict__ count, double *__restrict__ acc) {
  const int c = *count;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < c; k += gridDim.x * blockDim.x) {
    const int2 e = ent[k];
    acc[e.y] += part[e.x];
  }
}

// out[i] = bc_tid[tid_of[points[i]]]
__global__ void k_pick(const double *__restrict__ bc_tid, const int32_t *__restrict__ tid_of,
                       const int32_t *__restrict__ points, int32_t q, int32_t n, double *__restrict__ out,
                       int32_t *err) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < q; i += gridDim.x * blockDim.x) {
    const int v = points[i];
    const bool ok = v >= 0 && v < n;
    out[i] = ok ? bc_tid[tid_of[v]] : 0.0;
    if (!ok) atomicCAS(err, 0, 3);
  }
}

namespace {

uint64_t fnv(uint64_t h, const void *p, size_t bytes) {
  const unsigned char *c = (const unsigned char *)p;
  for (size_t i = 0; i < bytes; i++) h = (h ^ c[i]) * 1099511628211ull;
  return h;
}

uint64_t tuning_key(const Handle &h, const DeviceState *d) {
  const Tuning &t = h.tuning;
  const int32_t f[] = {t.lanes_per_source, t.label_threads, t.split, t.dep_threads, t.dep_form, t.queue_depth, t.label_warps, t.label_tile, t.label_passes, t.sweep_delta, t.sweep_threads, t.label_sources, t.label_stream, d->chunk};
  return fnv(1469598103934665603ull, f, sizeof(f));
}

// Source tids in increasing order (sources of one CTA are neighbours in the tree); nullptr = all.
std::vector<int32_t> source_tids(const Index &ix, const int32_t *sources0, int32_t ns) {
  std::vector<int32_t> t;
  if (!sources0) {
    t.resize((size_t)ix.n);
    for (int32_t i = 0; i < ix.n; i++) t[i] = i;
    return t;
  }
  t.resize((size_t)ns);
  for (int32_t i = 0; i < ns; i++) {
    if (sources0[i] < 0 || sources0[i] >= ix.n) throw Error(QBC_EINVAL, "source id " + std::to_string(sources0[i]) + " out of range");
    t[i] = ix.tid_of[sources0[i]];
  }
  std::sort(t.begin(), t.end());
  return t;
}

struct Counters {
  int64_t launches, label, dep;
};
Counters counters(const DeviceState *d) { return {d->launches, d->label_launches, d->dep_launches}; }

// Captures what `enqueue` puts on `st` into an instantiated graph; the launch counters it bumped are
// returned in `per_replay` and taken back (they are added again at each replay).
template <class F>
cudaGraphExec_t capture(DeviceState *d, cudaStream_t st, Counters &per_replay, F &&enqueue) {
  const bool prof = d->profiling;
  d->profiling = false;  // no timing events inside graphs
  const Counters c0 = counters(d);
  cudaGraph_t g = nullptr;
  CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
  try {
    enqueue();
  } catch (...) {
    cudaStreamEndCapture(st, &g);
    if (g) cudaGraphDestroy(g);
    d->profiling = prof;
    throw;
  }
  cudaError_t e = cudaStreamEndCapture(st, &g);
  d->profiling = prof;
  const Counters c1 = counters(d);
  per_replay = {c1.launches - c0.launches, c1.label - c0.label, c1.dep - c0.dep};
  d->launches = c0.launches;
  d->label_launches = c0.label;
  d->dep_launches = c0.dep;
  CK(e);
  cudaGraphExec_t ex = nullptr;
  e = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  CK(e);
  return ex;
}

void replay(DeviceState *d, cudaGraphExec_t ex, const Counters &c, cudaStream_t st) {
  CK(cudaGraphLaunch(ex, st));
  d->launches += c.launches;
  d->label_launches += c.label;
  d->dep_launches += c.dep;
}

}  // namespace

// ------------------------------------------------------------------------------- batched sweep
// One source list's whole sweep as one graph: clear the BC accumulator, then every chunk.
struct SweepPlan {
  uint64_t key = 0;
  int32_t ns = 0;
  int32_t *d_tids = nullptr;
  cudaGraphExec_t whole = nullptr;
  Counters per_replay{0, 0, 0};
};

struct SweepCache {
  std::vector<std::unique_ptr<SweepPlan>> plans;  // most recent last
  int32_t *d_points = nullptr;
  double *d_out = nullptr;
  int64_t points_cap = 0;
};

static void free_plan(SweepPlan *p) {
  if (p->whole) cudaGraphExecDestroy(p->whole);
  if (p->d_tids) cudaFree(p->d_tids);
  p->whole = nullptr;
  p->d_tids = nullptr;
}

void sweep_cache_free(DeviceState *d) {
  SweepCache *c = d->sweep;
  if (!c) return;
  for (auto &p : c->plans) free_plan(p.get());
  if (c->d_points) cudaFree(c->d_points);
  if (c->d_out) cudaFree(c->d_out);
  delete c;
  d->sweep = nullptr;
}

static constexpr size_t kMaxPlans = 4;

static SweepPlan &plan_for(Handle &h, DeviceState *d, const int32_t *sources0, int32_t ns) {
  if (!d->sweep) d->sweep = new SweepCache();
  SweepCache &c = *d->sweep;
  std::vector<int32_t> tids = source_tids(h.host, sources0, ns);
  uint64_t key = tuning_key(h, d);
  key = fnv(key, tids.data(), tids.size() * 4);
  key = fnv(key, &d->chunk, 4);
  for (size_t i = 0; i < c.plans.size(); i++)
    if (c.plans[i]->key == key && c.plans[i]->ns == (int32_t)tids.size()) {
      std::unique_ptr<SweepPlan> p = std::move(c.plans[i]);
      c.plans.erase(c.plans.begin() + (long)i);
      c.plans.push_back(std::move(p));
      return *c.plans.back();
    }
  if (c.plans.size() >= kMaxPlans) {
    CK(cudaStreamSynchronize(d->s_label));
    free_plan(c.plans.front().get());
    c.plans.erase(c.plans.begin());
  }
  auto p = std::make_unique<SweepPlan>();
  p->key = key;
  p->ns = (int32_t)tids.size();
  cudaStream_t st = d->s_label;
  try {
    CK(cudaMalloc(&p->d_tids, std::max<size_t>(4, tids.size() * 4)));
    if (!tids.empty()) CK(cudaMemcpyAsync(p->d_tids, tids.data(), tids.size() * 4, cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    const int32_t total = p->ns;
    int32_t *dt = p->d_tids;
    p->whole = capture(d, st, p->per_replay, [&] {
      CK(cudaMemsetAsync(d->bc_tid, 0, (size_t)d->n * 8, st));
      for (int32_t off = 0; off < total; off += d->chunk) launch_chunk(h, d, dt + off, std::min(d->chunk, total - off), 0, st);
    });
  } catch (...) {
    free_plan(p.get());
    throw;
  }
  c.plans.push_back(std::move(p));
  return *c.plans.back();
}

void host_bc_sweep(Handle &h, const int32_t *sources0, int32_t ns, double *bc_out) {
  NvtxRange nvtx("qbc.bc_sweep");
  DeviceState *d = need_dev(h);
  SweepPlan &p = plan_for(h, d, sources0, ns);
  cudaStream_t st = d->s_label;
  replay(d, p.whole, p.per_replay, st);
  launch_tid_to_vid(d, d->bc_tid, d->bc_vid, 0, st);
  CK(cudaMemcpyAsync(bc_out, d->bc_vid, (size_t)d->n * 8, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  check_err(d);
}

void host_query_batch(Handle &h, const int32_t *points0, int64_t total, const int32_t *sources0, int32_t ns, double *out) {
  NvtxRange nvtx("qbc.query_batch");
  DeviceState *d = need_dev(h);
  for (int64_t i = 0; i < total; i++)
    if (points0[i] < 0 || points0[i] >= h.host.n) throw Error(QBC_EINVAL, "query id " + std::to_string(points0[i]) + " out of range");
  SweepPlan &p = plan_for(h, d, sources0, ns);
  SweepCache &c = *d->sweep;
  cudaStream_t st = d->s_label;
  if (total > c.points_cap) {
    CK(cudaStreamSynchronize(st));
    if (c.d_points) cudaFree(c.d_points);
    if (c.d_out) cudaFree(c.d_out);
    c.d_points = nullptr;
    c.d_out = nullptr;
    c.points_cap = 0;
    CK(cudaMalloc(&c.d_points, (size_t)total * 4));
    CK(cudaMalloc(&c.d_out, (size_t)total * 8));
    c.points_cap = total;
  }
  if (total) CK(cudaMemcpyAsync(c.d_points, points0, (size_t)total * 4, cudaMemcpyHostToDevice, st));
  replay(d, p.whole, p.per_replay, st);
  if (total) {
    const int blocks = (int)std::min<int64_t>(148 * 4, (total + 255) / 256);
    k_pick<<<blocks, 256, 0, st>>>(d->bc_tid, d->tid_of, c.d_points, (int32_t)total, d->n, c.d_out, d->err);
    CK(cudaGetLastError());
    d->launches++;
    CK(cudaMemcpyAsync(out, c.d_out, (size_t)total * 8, cudaMemcpyDeviceToHost, st));
  }
  CK(cudaStreamSynchronize(st));
  check_err(d);
}

// ------------------------------------------------------------------------------- autotune
// Mean time per source of a sweep over `tids` (device) with the handle's current tuning.
static double time_sample(Handle &h, DeviceState *d, const int32_t *d_tids, int32_t ns, int reps) {
  cudaStream_t st = d->s_label;
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  float best = 1e30f;
  try {
    for (int r = -1; r < reps; r++) {
      CK(cudaMemsetAsync(d->bc_tid, 0, (size_t)d->n * 8, st));
      CK(cudaEventRecord(a, st));
      for (int32_t off = 0; off < ns; off += d->chunk) launch_chunk(h, d, d_tids + off, std::min(d->chunk, ns - off), 0, st);
      CK(cudaEventRecord(b, st));
      CK(cudaEventSynchronize(b));
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, a, b));
      if (r >= 0) best = std::min(best, ms);
    }
    check_err(d);
  } catch (...) {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    throw;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return (double)best / std::max(1, ns);
}

static bool label_fits(const Handle &h, const DeviceState *d, int32_t lanes, int32_t threads) {
  // generic kernel: (32/K sources x 3 rows + one row per warp) x stride ints of shared memory
  const size_t smem = ((size_t)(32 / lanes) * 3 + (size_t)threads / 32) * d->hmax_pad * 4;
  return smem + 2048 <= (size_t)d->smem_optin;
}

void autotune(Handle &h, const int32_t *sources0, int32_t ns, double *ms_per_source) {
  NvtxRange nvtx("qbc.autotune");
  DeviceState *d = need_dev(h);
  std::vector<int32_t> tids = source_tids(h.host, sources0, ns);
  if (tids.empty()) throw Error(QBC_EINVAL, "empty tuning sample");
  int32_t *d_tids = nullptr;
  CK(cudaMalloc(&d_tids, tids.size() * 4));
  const Tuning start = h.tuning;
  try {
    CK(cudaMemcpy(d_tids, tids.data(), tids.size() * 4, cudaMemcpyHostToDevice));
    const int32_t cnt = (int32_t)tids.size();
    Tuning best = h.tuning;
    double best_t = time_sample(h, d, d_tids, cnt, 3);
    auto trial = [&](const Tuning &t) {
      h.tuning = t;
      try {
        if (t.chunk != d->chunk) device_set_chunk(h, t.chunk);
        const double x = time_sample(h, d, d_tids, cnt, 3);
        if (x < best_t * 0.99) {  // a candidate must win by more than the timing noise (~1 %)
          best_t = x;
          best = t;
          best.chunk = d->chunk;
        }
      } catch (const Error &e) {
        // a configuration that does not fit (scratch allocation, shared memory) is skipped
        if (e.code != QBC_ENOMEM && e.code != QBC_EDEVICE) throw;
        cudaGetLastError();
        h.tuning = best;
        if (d->chunk != best.chunk) device_set_chunk(h, best.chunk);
      }
    };
    best.chunk = d->chunk;
    auto chunk_trials = [&] {
      for (int32_t ch : {1024, 2048, 4096, 8192}) {
        if (ch > std::max<int32_t>(32, (cnt + 31) / 32 * 32)) continue;  // the sample must span a chunk
        if (ch == best.chunk) continue;
        Tuning t = best;
        t.chunk = ch;
        trial(t);
      }
    };
    // 0. sources per scratch buffer (again at the end, after the kernels are chosen)
    chunk_trials();
    if (h.host.kind == IndexKind::CSR) {
      // label-free index: the sweep's bucket width (around twice the mean arc weight) and CTA
      // size, then the Kahn/dependency pass's CTA size
      const int32_t auto_delta = d->sweep_delta_auto;
      for (int32_t mult : {2, 4, 8})  // 0.5x, 1x, 2x the default width (wider and narrower measured slower)
        for (int32_t threads : {256, 512, 2048}) {  // 2048: four 512-thread CTAs per SM
          Tuning t = best;
          t.sweep_delta = std::max(1, auto_delta * mult / 4);
          t.sweep_threads = threads;
          trial(t);
        }
      for (int32_t th : {128, 256}) {
        Tuning t = best;
        t.dep_threads = th;
        trial(t);
      }
      chunk_trials();
      h.tuning = best;
      if (d->chunk != best.chunk) device_set_chunk(h, best.chunk);
      *ms_per_source = best_t;
      cudaFree(d_tids);
      return;
    }
    // 1. label kernel: the packed-key kernel with 32 sources per CTA and 8-20 warps (0 lanes) and,
    //    for tall trees, tile passes or a global-memory tail; its 16-source forms (whole source rows
    //    in shared memory, two targets per warp; target rows whole or through a ring) with 8, 12 or
    //    16 warps; or the general kernel with
    //    32/K sources per CTA and 128 or 256 threads
    if (d->packed_bits) {
      for (int32_t warps : {8, 12, 16, 20})  // 12: the two-target kernel
        for (int32_t passes : {0, 2}) {  // rows taller than a 16-warp tile: global tail or tile passes
          if (passes == 2 && (d->hmax_pad <= 644 || warps == 12)) continue;
          Tuning t = best;
          t.lanes_per_source = 0;
          t.label_sources = 32;
          t.label_warps = warps;
          t.label_passes = passes;
          trial(t);
        }
      for (int32_t stream : {1, 2})
        for (int32_t warps : {8, 12, 16}) {
          Tuning t = best;
          t.lanes_per_source = 0;
          t.label_sources = 16;
          t.label_stream = stream;
          t.label_warps = warps;
          t.label_passes = 0;
          t.label_tile = 0;
          trial(t);
        }
    }
    for (int32_t lanes : {4, 8, 16})
      for (int32_t threads : {128, 256}) {
        if (!label_fits(h, d, lanes, threads)) continue;
        Tuning t = best;
        t.lanes_per_source = lanes;
        t.label_threads = threads;
        trial(t);
      }
    // 2. target ranges per source group (the width of each CTA's target tile)
    for (int32_t split : {0, 2, 4, 8, 16, 32}) {
      Tuning t = best;
      t.split = split;
      trial(t);
    }
    // 3. dependency pass: warp per source with its shared level-queue depth, or CTA per source
    for (int32_t form : {1, 3})
      for (int32_t qd : {64, 256, 512, 1024}) {
        Tuning t = best;
        t.dep_form = form;
        t.queue_depth = qd;
        trial(t);
      }
    for (int32_t form : {2, 4})
      for (int32_t th : {128, 256}) {
        Tuning t = best;
        t.dep_form = form;
        t.dep_threads = th;
        trial(t);
      }
    // 4. sources per scratch buffer
    chunk_trials();
    h.tuning = best;
    if (d->chunk != best.chunk) device_set_chunk(h, best.chunk);
    *ms_per_source = best_t;
  } catch (...) {
    cudaFree(d_tids);
    h.tuning = start;
    throw;
  }
  cudaFree(d_tids);
}

// ------------------------------------------------------------------------------- served loop
namespace {

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// first-fit ranges of a pool of `cap` accumulator entries
struct RangeAlloc {
  std::map<int64_t, int64_t> free_;  // offset -> length
  int64_t used = 0;
  explicit RangeAlloc(int64_t cap = 0) {
    if (cap > 0) free_[0] = cap;
  }
  int64_t alloc(int64_t len) {
    for (auto it = free_.begin(); it != free_.end(); ++it)
      if (it->second >= len) {
        const int64_t off = it->first, rest = it->second - len;
        free_.erase(it);
        if (rest) free_[off + len] = rest;
        used += len;
        return off;
      }
    return -1;
  }
  void release(int64_t off, int64_t len) {
    used -= len;
    auto it = free_.emplace(off, len).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
};

enum ReqState { QUEUED, ACTIVE, COPYING, DONE, FAILED };

struct Req {
  int64_t id = 0;
  std::vector<int32_t> tids;
  int64_t off = -1;
  int32_t remaining = 0;
  ReqState state = QUEUED;
  double t_submit = 0, t_admit = 0, t_done = 0;
  std::vector<double> result;
  std::string error;
  int error_code = QBC_EDEVICE;  // QBC_EBUSY: cancelled by qbc_serve_close
};

}  // namespace

struct Server {
  Handle *h = nullptr;
  DeviceState *d = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  int32_t ns = 0, nchunks = 0, chunk = 0;
  int32_t *d_tids = nullptr;
  std::vector<cudaGraphExec_t> graphs;  // one per chunk
  Counters per_chunk{0, 0, 0};
  int64_t cap = 0;  // accumulator pool entries
  int max_active = 64;
  size_t max_queue = 1 << 20;
  double *d_acc = nullptr;
  int2 *d_ent = nullptr;
  int32_t *d_count = nullptr;
  int2 *h_ent[2] = {nullptr, nullptr};  // pinned
  int32_t *h_count = nullptr;          // pinned [2]
  double *h_acc = nullptr;             // pinned, mirrors d_acc
  int32_t *h_err = nullptr;            // pinned [2]
  RangeAlloc pool;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Req *> queue;
  std::vector<Req *> active;
  std::map<int64_t, std::unique_ptr<Req>> reqs;
  int64_t next_id = 1;
  int waiters = 0;  // threads inside serve_wait
  bool stop = false;
  std::string fail;
  std::thread th;
  // statistics
  int64_t chunks_run = 0, done_count = 0;
  double busy_s = 0.0, t_open = 0.0;

  void release_all();
  void loop();
  void fail_all(const std::string &msg);
};

void Server::release_all() {
  for (auto g : graphs)
    if (g) cudaGraphExecDestroy(g);
  graphs.clear();
  void *dp[] = {d_tids, d_acc, d_ent, d_count};
  for (void *p : dp)
    if (p) cudaFree(p);
  void *hp[] = {h_ent[0], h_ent[1], h_count, h_acc, h_err};
  for (void *p : hp)
    if (p) cudaFreeHost(p);
  for (auto e : ev)
    if (e) cudaEventDestroy(e);
  if (st) cudaStreamDestroy(st);
}

void Server::fail_all(const std::string &msg) {
  fail = msg;
  for (Req *r : active) {
    r->state = FAILED;
    r->error = msg;
  }
  for (Req *r : queue) {
    r->state = FAILED;
    r->error = msg;
  }
  for (auto &kv : reqs)
    if (kv.second->state == COPYING) {
      kv.second->state = FAILED;
      kv.second->error = msg;
    }
  active.clear();
  queue.clear();
  cv_done.notify_all();
}

// Engine: admits requests at chunk boundaries, launches chunk graphs around the source list with at
// most two chunks queued on the stream, and completes each request one full turn after admission.
void Server::loop() {
  std::unique_lock<std::mutex> lk(mu);
  try {
    CK(cudaSetDevice(d->device));
    int64_t k = 0;  // chunks launched
    int32_t cursor = 0;
    bool entries_dirty = true, prev = false;
    std::vector<Req *> prev_fin;
    auto finalize = [&](std::vector<Req *> &fin, int slot) {
      if (h_err[slot] != 0) throw Error(QBC_EDEVICE, "device: kernel error word " + std::to_string(h_err[slot]));
      const double t = now_s();
      for (Req *r : fin) {
        r->result.assign(h_acc + r->off, h_acc + r->off + r->tids.size());
        pool.release(r->off, (int64_t)r->tids.size());
        r->off = -1;
        r->t_done = t;
        r->state = DONE;
        done_count++;
      }
      if (!fin.empty()) cv_done.notify_all();
      fin.clear();
    };
    for (;;) {
      if (!stop) {
        while (!queue.empty() && (int)active.size() < max_active) {
          Req *r = queue.front();
          const int64_t off = pool.alloc((int64_t)r->tids.size());
          if (off < 0) break;
          queue.pop_front();
          r->off = off;
          r->remaining = nchunks;
          r->t_admit = now_s();
          r->state = ACTIVE;
          active.push_back(r);
          CK(cudaMemsetAsync(d_acc + off, 0, r->tids.size() * 8, st));
          entries_dirty = true;
        }
      }
      if (active.empty() || stop) {
        if (prev) {
          lk.unlock();
          cudaError_t e = cudaEventSynchronize(ev[(k - 1) & 1]);
          lk.lock();
          CK(e);
          finalize(prev_fin, (int)((k - 1) & 1));
          prev = false;
          continue;
        }
        if (stop) break;
        cv_work.wait(lk);
        continue;
      }
      const int slot = (int)(k & 1);
      NvtxRange nvtx("qbc.serve.chunk");  // one turn of the loop: enqueue a chunk, finish the previous one
      if (entries_dirty) {
        int64_t m = 0;
        for (Req *r : active)
          for (size_t i = 0; i < r->tids.size(); i++) h_ent[slot][m++] = make_int2(r->tids[i], (int32_t)(r->off + (int64_t)i));
        h_count[slot] = (int32_t)m;
        CK(cudaMemcpyAsync(d_ent, h_ent[slot], (size_t)m * 8, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(d_count, h_count + slot, 4, cudaMemcpyHostToDevice, st));
        entries_dirty = false;
      }
      replay(d, graphs[cursor], per_chunk, st);
      cursor = (cursor + 1) % nchunks;
      std::vector<Req *> fin;
      for (size_t i = 0; i < active.size();) {
        Req *r = active[i];
        if (--r->remaining == 0) {
          CK(cudaMemcpyAsync(h_acc + r->off, d_acc + r->off, r->tids.size() * 8, cudaMemcpyDeviceToHost, st));
          r->state = COPYING;
          fin.push_back(r);
          active[i] = active.back();
          active.pop_back();
          entries_dirty = true;
        } else {
          i++;
        }
      }
      CK(cudaMemcpyAsync(h_err + slot, d->err, 4, cudaMemcpyDeviceToHost, st));
      CK(cudaEventRecord(ev[slot], st));
      chunks_run++;
      if (prev) {
        lk.unlock();
        cudaError_t e = cudaEventSynchronize(ev[(k - 1) & 1]);
        lk.lock();
        CK(e);
        finalize(prev_fin, (int)((k - 1) & 1));
      }
      prev_fin = fin;
      prev = true;
      k++;
    }
  } catch (const std::exception &e) {
    cudaStreamSynchronize(st);
    fail_all(e.what());
  }
}

static void check_server(Server *s) {
  if (!s) throw Error(QBC_EINVAL, "null server");
}

Server *serve_open(Handle &h, const int32_t *sources0, int32_t ns, const int64_t *opts, int32_t nopts) {
  DeviceState *d = need_dev(h);
  if (h.server) throw Error(QBC_EBUSY, "the index already has a server");
  auto s = std::make_unique<Server>();
  s->h = &h;
  s->d = d;
  try {
    std::vector<int32_t> tids = source_tids(h.host, sources0, ns);
    if (tids.empty()) throw Error(QBC_EINVAL, "empty source list");
    s->ns = (int32_t)tids.size();
    // sources per served chunk: the admission granularity (at most the scratch's chunk)
    int32_t sc = nopts > 3 && opts[3] > 0 ? (int32_t)std::min<int64_t>(opts[3], d->chunk) : d->chunk;
    sc = std::max<int32_t>(32, (sc + 31) / 32 * 32);
    sc = std::min(sc, d->chunk);
    s->chunk = sc;
    s->nchunks = (s->ns + sc - 1) / sc;
    const int64_t max_active = nopts > 0 && opts[0] > 0 ? opts[0] : 64;
    int64_t pool_bytes = nopts > 1 ? opts[1] : 0;
    if (nopts > 2 && opts[2] > 0) s->max_queue = (size_t)opts[2];
    size_t free_b = 0, total_b = 0;
    CK(cudaMemGetInfo(&free_b, &total_b));
    // admission pool: per accumulator entry 8 B (FP64 sum) + 8 B (target, slot) on the device
    if (pool_bytes <= 0) pool_bytes = (int64_t)std::min<size_t>(free_b / 8, (size_t)64 << 20);
    if ((size_t)pool_bytes > free_b / 2) throw Error(QBC_ENOMEM, "request pool larger than half the free device memory");
    s->max_active = (int)std::min<int64_t>(max_active, 1 << 20);
    s->cap = std::max<int64_t>(1, pool_bytes / 16);
    s->pool = RangeAlloc(s->cap);
    CK(cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking));
    for (auto &e : s->ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    CK(cudaMalloc(&s->d_tids, tids.size() * 4));
    CK(cudaMalloc(&s->d_acc, (size_t)s->cap * 8));
    CK(cudaMalloc(&s->d_ent, (size_t)s->cap * 8));
    CK(cudaMalloc(&s->d_count, 4));
    for (auto &p : s->h_ent) CK(cudaMallocHost(&p, (size_t)s->cap * 8));
    CK(cudaMallocHost(&s->h_count, 8));
    CK(cudaMallocHost(&s->h_acc, (size_t)s->cap * 8));
    CK(cudaMallocHost(&s->h_err, 8));
    s->h_err[0] = s->h_err[1] = 0;
    CK(cudaMemcpyAsync(s->d_tids, tids.data(), tids.size() * 4, cudaMemcpyHostToDevice, s->st));
    CK(cudaMemsetAsync(s->d_count, 0, 4, s->st));
    CK(cudaStreamSynchronize(s->st));
    for (int32_t c = 0; c < s->nchunks; c++) {
      const int32_t off = c * s->chunk, cnt = std::min(s->chunk, s->ns - off);
      Server *sp = s.get();
      s->graphs.push_back(capture(d, s->st, s->per_chunk, [&] {
        CK(cudaMemsetAsync(d->bc_tid, 0, (size_t)d->n * 8, sp->st));
        launch_chunk(h, d, sp->d_tids + off, cnt, 0, sp->st);
        k_gather_entries<<<148 * 2, 256, 0, sp->st>>>(d->bc_tid, sp->d_ent, sp->d_count, sp->d_acc);
        CK(cudaGetLastError());
        d->launches++;
      }));
    }
    s->t_open = now_s();
    h.server = s.get();
    s->th = std::thread([sp = s.get()] { sp->loop(); });
  } catch (...) {
    s->release_all();
    throw;
  }
  return s.release();
}

int64_t serve_submit(Server *s, const int32_t *points0, int32_t q) {
  check_server(s);
  const Index &ix = s->h->host;
  if (q < 0 || (q > 0 && !points0)) throw Error(QBC_EINVAL, "null argument");
  if (q > s->cap) throw Error(QBC_EINVAL, "request of " + std::to_string(q) + " vertices exceeds the request pool (" + std::to_string(s->cap) + ")");
  auto r = std::make_unique<Req>();
  r->tids.resize((size_t)q);
  for (int32_t i = 0; i < q; i++) {
    if (points0[i] < 0 || points0[i] >= ix.n) throw Error(QBC_EINVAL, "query id " + std::to_string(points0[i]) + " out of range");
    r->tids[i] = ix.tid_of[points0[i]];
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (!s->fail.empty()) throw Error(QBC_EDEVICE, "server stopped: " + s->fail);
  if (s->stop) throw Error(QBC_EBUSY, "server is closing");
  if (s->queue.size() >= s->max_queue) throw Error(QBC_EBUSY, "request queue full");
  r->id = s->next_id++;
  r->t_submit = now_s();
  Req *rp = r.get();
  const int64_t id = r->id;
  s->reqs[id] = std::move(r);
  if (q == 0) {
    rp->state = DONE;
    rp->t_admit = rp->t_done = rp->t_submit;
    s->done_count++;
  } else {
    s->queue.push_back(rp);
    s->cv_work.notify_one();
  }
  return id;
}

// 1 and the result when done (the ticket is then released), 0 while pending
static int take_result(Server *s, std::map<int64_t, std::unique_ptr<Req>>::iterator it, double *out, double *times) {
  Req *r = it->second.get();
  if (r->state == FAILED) {
    const std::string msg = r->error;
    const int code = r->error_code;
    s->reqs.erase(it);
    throw Error(code, msg);
  }
  if (r->state != DONE) return 0;
  if (out && !r->result.empty()) std::memcpy(out, r->result.data(), r->result.size() * 8);
  if (times) {
    times[0] = r->t_submit - s->t_open;
    times[1] = r->t_admit - s->t_open;
    times[2] = r->t_done - s->t_open;
  }
  s->reqs.erase(it);
  return 1;
}

int serve_poll(Server *s, int64_t ticket, double *out, double *times) {
  check_server(s);
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) throw Error(QBC_EINVAL, "unknown ticket " + std::to_string(ticket));
  return take_result(s, it, out, times);
}

int serve_wait(Server *s, int64_t ticket, double timeout_s, double *out, double *times) {
  check_server(s);
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) throw Error(QBC_EINVAL, "unknown ticket " + std::to_string(ticket));
  Req *r = it->second.get();
  auto ready = [&] { return r->state == DONE || r->state == FAILED; };
  // counted, so that serve_close frees the server only once every waiter has left
  struct Waiting {
    Server *s;
    explicit Waiting(Server *x) : s(x) { s->waiters++; }
    ~Waiting() {
      s->waiters--;
      s->cv_done.notify_all();
    }
  } waiting(s);
  if (timeout_s < 0) s->cv_done.wait(lk, ready);
  else s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready);
  return take_result(s, it, out, times);
}

void serve_stats(Server *s, double *out, int32_t nout) {
  check_server(s);
  std::lock_guard<std::mutex> lk(s->mu);
  const double v[] = {(double)s->chunks_run,
                      (double)s->chunks_run / std::max(1, s->nchunks),
                      (double)s->done_count,
                      (double)s->active.size(),
                      (double)s->queue.size(),
                      (double)s->pool.used,
                      (double)s->cap,
                      (double)s->nchunks,
                      (double)s->ns};
  for (int32_t i = 0; i < nout && i < (int32_t)(sizeof(v) / sizeof(v[0])); i++) out[i] = v[i];
}

void serve_close(Server *s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    for (Req *r : s->queue) {
      r->state = FAILED;
      r->error = "server closed";
      r->error_code = QBC_EBUSY;
    }
    s->queue.clear();
    for (Req *r : s->active) {
      r->state = FAILED;
      r->error = "server closed";
      r->error_code = QBC_EBUSY;
    }
    s->active.clear();
  }
  s->cv_work.notify_all();
  s->cv_done.notify_all();
  if (s->th.joinable()) s->th.join();
  {  // every request is now done or failed: let threads still in serve_wait collect theirs first
    std::unique_lock<std::mutex> lk(s->mu);
    s->cv_done.notify_all();
    s->cv_done.wait(lk, [&] { return s->waiters == 0; });
  }
  cudaSetDevice(s->d->device);
  cudaStreamSynchronize(s->st);
  if (s->h->server == s) s->h->server = nullptr;
  s->release_all();
  delete s;
}

}  // namespace qbc

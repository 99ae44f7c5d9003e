// device_state.h -- device-resident index and scratch of libqbc_b200 (internal to the library:
// shared by the kernel drivers in device.cu and the sweep / batch / serve engine in sweep.cu).
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <string>
#include <utility>
#include <vector>

#include "../../include/qbc_b200.h"
#include "device.h"

namespace qbc {

// NVTX range over a scope: the library's phases (index build, upload, sweeps, query batches, the
// autotuner, served chunks) appear by name on Nsight timelines; with no tool attached a push/pop
// is a check of one function pointer.
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};

#define CK(call)                                                                                    \
  do {                                                                                              \
    cudaError_t e_ = (call);                                                                        \
    if (e_ != cudaSuccess)                                                                          \
      throw Error(e_ == cudaErrorMemoryAllocation ? QBC_ENOMEM : QBC_ECUDA,                         \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                              \
  } while (0)

enum : int32_t {
  ERR_NONE = 0,
  ERR_HOP_CAP = 1,
  ERR_DISCONNECTED = 2,
  ERR_BAD_SOURCE = 3,
  ERR_COPY_TIMEOUT = 4,
  ERR_SWEEP_BOUND = 5  // a shortest-path sweep ran past its pass bound
};

// Per-source rows (dist/sigma pairs, hop layers) of a buffer with ns source slots are stored
// chunk-blocked: entry (slot, t) lives at ((t / 8) * ns + slot) * 8 + t % 8, so the 8-target
// chunk of the 32 consecutive slots a warp produces is one contiguous block.  With ns = 1 this is
// the plain row layout.
__host__ __device__ __forceinline__ size_t blk(int slot, int t, int ns) {
  return ((size_t)(t >> 3) * (size_t)ns + (size_t)slot) * 8 + (size_t)(t & 7);
}

template <class T>
struct RowView {
  T *p;
  int slot, ns;
  __device__ __forceinline__ T &operator[](int t) const { return p[blk(slot, t, ns)]; }
};

// ------------------------------------------------------------------------------- state
struct SweepCache;  // captured sweep graphs (sweep.cu)

struct DeviceState {
  int device = 0;
  cudaStream_t s_label = nullptr, s_dep = nullptr;
  cudaEvent_t ev_label[2] = {nullptr, nullptr}, ev_dep[2] = {nullptr, nullptr}, ev_start = nullptr;
  int32_t n = 0, n_pad = 0, hmax_pad = 0;
  int32_t *depth = nullptr, *send = nullptr, *arc_off = nullptr, *arc_head = nullptr, *arc_w = nullptr;
  int2 *arc_rng = nullptr, *arc_hw = nullptr;
  int4 *arc4 = nullptr;  // per vertex 2 x int4: (head, weight) of its first four arcs (see k_dependency_cta_pipe)
  int32_t *vid_of = nullptr, *tid_of = nullptr, *parent = nullptr;
  // label distances: one array, shifted left in place by packed_bits when the packed-key scan
  // applies (dis_sh then aliases it); no per-entry ancestor ids or subtree ends are kept -- each
  // launch derives its sources' rows from the parent links (k_src_rows)
  int32_t *dis = nullptr;
  int32_t packed_bits = 0;  // > 0: the packed-key label scan applies
  int32_t sweep_delta_auto = 1;  // CSR sweep's default bucket width (twice the mean arc weight)
  int32_t *dis_sh = nullptr;  // = dis when packed_bits > 0 (the packed kernel's name for it)
  int64_t *lab_off = nullptr;
  int2 *ch = nullptr;
  // scratch: one buffer of `chunk` source slots (index 1 unused)
  int32_t chunk = 0;
  int4 *rec[2] = {nullptr, nullptr};  // per (slot, vertex): dist, sigma bits, delta (f64)
  int32_t *hop[2] = {nullptr, nullptr};
  int32_t *order[2] = {nullptr, nullptr};
  int32_t *lcnt[2] = {nullptr, nullptr};
  int32_t *src[2] = {nullptr, nullptr};
  int32_t *maxhop[2] = {nullptr, nullptr};
  int32_t *src_rows[2] = {nullptr, nullptr};  // per slot: source's ancestors, then their subtree ends (hmax_pad each)
  double *bc_tid = nullptr;
  double *bc_vid = nullptr;
  int32_t *sources = nullptr;  // staging for host source lists
  int32_t sources_cap = 0;
  // device source lists (qbc_bc_sources_device): tids, then the same sorted, and the sort's
  // temporary storage; grown on demand
  int32_t *dsrc_tid = nullptr, *dsrc_sorted = nullptr;
  void *dsrc_tmp = nullptr;
  size_t dsrc_tmp_bytes = 0;
  int32_t dsrc_cap = 0;
  int32_t *err = nullptr;
  int32_t *grid_ctl = nullptr;  // control block of the cooperative plain sweep (kGridCtlBytes)
  int64_t bytes = 0, scratch_bytes = 0;
  int smem_optin = 0;
  // optional per-launch timing of the two main kernels (events on their launching streams)
  bool profiling = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_lab, ev_dp;
  size_t ev_lab_used = 0, ev_dp_used = 0;
  double label_ms = 0.0, dep_ms = 0.0;
  int64_t label_launches = 0, dep_launches = 0, launches = 0;
  SweepCache *sweep = nullptr;
};

static std::pair<cudaEvent_t, cudaEvent_t> take_events(std::vector<std::pair<cudaEvent_t, cudaEvent_t>> &pool,
                                                       size_t &used) {
  if (used == pool.size()) {
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    pool.push_back({a, b});
  }
  return pool[used++];
}

template <class T>
static T *dmalloc(DeviceState *d, size_t count) {
  void *p = nullptr;
  if (count == 0) count = 1;
  CK(cudaMalloc(&p, count * sizeof(T)));
  d->bytes += (int64_t)(count * sizeof(T));
  return (T *)p;
}

template <class T>
static T *dupload(DeviceState *d, const std::vector<T> &v, cudaStream_t s) {
  T *p = dmalloc<T>(d, v.size());
  if (!v.empty()) CK(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
  return p;
}

// Launches of one chunk of sources (their tids at d_src_tid, cnt <= chunk) on stream st, using
// scratch buffer `buf`: the label scan, then the dependency pass, which adds 0.5 * delta into
// d->bc_tid (not cleared here).  Nothing in it synchronises, so it can be stream-captured.
void launch_chunk(const Handle &h, DeviceState *d, const int32_t *d_src_tid, int32_t cnt, int buf, cudaStream_t st);
// CSR index: rows of ns sources by shortest-path sweeps into the given scratch (rec/hop/order/lcnt
// laid out as a buffer of ns slots), one CTA per source (sssp.cu): records (dist, count, 0), hop
// layers and, when maxhop is not null, the largest layer per source -- the label scan's outputs.
// write_hop false: hop layers are left out (the hop row is still the sweep's staging space); the
// CTA pipelined dependency pass does not read them, it walks the wave queue.
void launch_sweep_rows(const Handle &h, DeviceState *d, int4 *rec, int32_t *hop, int32_t *order, int32_t *lcnt,
                       int32_t *maxhop, const int32_t *src, int32_t ns, cudaStream_t st, bool write_hop = true);
int32_t sweep_delta(const Handle &h, const DeviceState *d);
// CSR index, plain path: one source's rows (slot 0 of a one-slot buffer; no largest-layer output)
// by a cooperative launch of the whole GPU
constexpr size_t kGridCtlBytes = 256;
void launch_sweep_rows_grid(const Handle &h, DeviceState *d, int4 *rec, int32_t *hop, int32_t *order, int32_t *lcnt,
                            const int32_t *src, cudaStream_t st);
// out_vid[vid_of[t]] (+)= in_tid[t] for all t
void launch_tid_to_vid(DeviceState *d, const double *in_tid, double *out_vid, int accumulate, cudaStream_t st);
// tids of cnt vids (sets ERR_BAD_SOURCE for ids out of range)
void launch_vid_to_tid(DeviceState *d, const int32_t *vids, int32_t *tids, int32_t cnt, cudaStream_t st);
DeviceState *need_dev(Handle &h);
// frees the captured sweep graphs (they hold scratch pointers; called whenever scratch changes)
void sweep_cache_free(DeviceState *d);
// reads and clears the device error word; throws QBC_EDEVICE when a kernel set it (synchronous)
void check_err(DeviceState *d);

}  // namespace qbc

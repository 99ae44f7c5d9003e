// device.h -- device-resident index, scratch and drivers of libqbc_b200.
#pragma once

#include <cstdint>
#include <vector>

#include "host.h"

namespace qbc {

struct Tuning {
  int32_t lanes_per_source = 0;  // K in {1,2,4,...,32}; sources per CTA = 32/K; 0 = auto
  int32_t label_threads = 256;   // threads per CTA of the label kernel
  int32_t split = 0;             // target ranges per source group; 0 = auto
  int32_t chunk = 0;             // sources per scratch buffer; 0 = auto
  int32_t dep_threads = 256;     // threads per CTA of the CTA-per-source dependency kernel
  int32_t dep_form = 0;          // 0 auto (= 4 for MHL), 1 warp per source, 2 CTA per source, 3 warp per
                                 // source with a software-pipelined backprop, 4 CTA per source, pipelined
  int32_t queue_depth = 0;       // level-queue layers held in shared memory by the warp form; 0 = 512
  int32_t label_warps = 0;       // packed-key label kernel: 8, 16 or 20 warps, 12 = two-target kernel; 0 = auto
  int32_t label_tile = 0;        // label entries per row staged in shared memory; 0 = all that fit
  int32_t label_passes = 0;      // rows longer than the tile: 0/1 one pass + global tail, 2 several tile passes
  int32_t sweep_delta = 0;       // CSR index: distance bucket width of the shortest-path sweep; 0 = auto
  int32_t sweep_threads = 0;     // CSR index: threads per CTA of the sweep (256, 512 or 1024; 0 = 512);
                                 // 2048: 512-thread CTAs, four per SM (32 registers a thread)
  int32_t label_sources = 0;     // packed-key label kernel: sources per CTA (32, or 16 with whole rows of
                                 // tall trees in shared memory); 0 = auto
  int32_t label_stream = 0;      // 16-source kernel: 1 whole target rows double-buffered, 2 64-entry
                                 // blocks through a ring; 0 = auto (whole rows when they fit 16 warps)
};

struct DeviceState;  // opaque, defined in device_state.h
struct Server;       // served request loop, defined in sweep.cu

struct Handle {
  Index host;
  Tuning tuning;
  DeviceState *dev = nullptr;
  Server *server = nullptr;  // while set, the index's device state belongs to that server
};

void device_upload(Handle &h, int device);
// The last dt.r vertices of a min-degree elimination on the device (a dense matrix, one pick and
// one shortcut update per step); fills dt.order / dt.x_off / dt.x.
void device_dense_eliminate(int device, DenseTail &dt);
// Uploads the index structure and fills its label rows on the device (host rows stay empty).
void device_build(Handle &h, int device, const Separators &seps);
// Copies device-built label rows to the host index (no-op when they are there already).
void device_download_rows(Handle &h);
void device_release(Handle &h);
// Reallocates the per-source scratch for `chunk` source slots (0 = sized from free memory).
void device_set_chunk(Handle &h, int32_t chunk);
int64_t device_bytes(const Handle &h);
int device_id(const Handle &h);  // -1 when not uploaded

// BC over `sources0` (0-based vids) accumulated into d_bc_vid (n doubles, vid order, device).
// Enqueued on `stream` (nullptr: the handle's stream); the caller synchronises.
void device_bc_sources(Handle &h, const int32_t *d_sources0, int32_t ns, double *d_bc_vid, void *stream);
// Same with host source list and host output (overwritten); synchronous.
void host_bc_sources(Handle &h, const int32_t *sources0, int32_t ns, double *bc_out);
// plain path: one source per launch pair
void host_bc_plain(Handle &h, const int32_t *sources0, int32_t ns, double *bc_out);
// Per-launch CUDA-event timing of the label and dependency kernels (on their own streams).
void device_profiling(Handle &h, bool on);
// out[0]=label ms, [1]=label launches, [2]=dependency ms, [3]=dependency launches, [4]=all launches
// since the last device_profiling call; synchronises the device.
void device_stats(Handle &h, double *out);
// sources per CTA of the batched label scan under the current tuning (0: label-free index)
int32_t device_label_group(Handle &h);
// name of the kernel the batched rows come from under the current tuning
const char *device_label_kernel(Handle &h);
// rows of each listed source in vid order (cnt/hop may be null)
void host_rows(Handle &h, const int32_t *sources0, int32_t ns, int32_t *dist, uint32_t *cnt, int32_t *hop);

// Batched sweeps (sweep.cu): the sweep over a source list (nullptr = all vertices) is captured once
// into a CUDA graph per source list and tuning, and replayed.
void host_bc_sweep(Handle &h, const int32_t *sources0, int32_t ns, double *bc_out);
// BC of `total` query vertices (the concatenated sets of a batch) from one sweep.
void host_query_batch(Handle &h, const int32_t *points0, int64_t total, const int32_t *sources0, int32_t ns, double *out);
// Times candidate tunings on a sweep over the listed sources and keeps the fastest.
void autotune(Handle &h, const int32_t *sources0, int32_t ns, double *ms_per_source);
// Served request loop (see sweep.cu).
Server *serve_open(Handle &h, const int32_t *sources0, int32_t ns, const int64_t *opts, int32_t nopts);
int64_t serve_submit(Server *s, const int32_t *points0, int32_t q);
int serve_poll(Server *s, int64_t ticket, double *out, double *times);
int serve_wait(Server *s, int64_t ticket, double timeout_s, double *out, double *times);
void serve_stats(Server *s, double *out, int32_t nout);
void serve_close(Server *s);

// One source's BC contribution added into d_bc_vid (device, n doubles, vid order) using only the
// library's static device scratch; enqueued on `stream` (nullptr: the index's stream).
void host_bc_source_static(Handle &h, int32_t source0, double *d_bc_vid, void *stream);

}  // namespace qbc

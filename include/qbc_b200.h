/*
 * qbc_b200.h -- C ABI of the B200-native query-based betweenness-centrality library
 * (libqbc_b200.so).  Plain pointers and sizes only; every call returns a QBC_* status and
 * qbc_last_error() gives the message of the calling thread's last failure.
 *
 * Vertex ids: file ids are 1-based (graph, query batch); every id crossing this ABI is 0-based
 * (Graph's convention, src/Graph.cpp:24-25).  Distances are int32, shortest-path counts are the
 * reference's 32-bit wrapping count bits (count_t = uint32_t, src/TreeCount/Util.h:24, stored in
 * int on the device, MHLQBC.cu:94-101), hop layers int32, BC FP64 with BC(v) = 0.5 * sum_s delta_s(v)
 * (MHLQBC.cu:469-472).
 *
 * Each entry point names the reference interface it replaces (paths relative to the reference).
 */
#ifndef QBC_B200_H
#define QBC_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  QBC_OK = 0,
  QBC_EINVAL = 1,   /* bad argument */
  QBC_EIO = 2,      /* file missing / malformed */
  QBC_EGRAPH = 3,   /* graph violates an input rule (asymmetric, disconnected, weight < 1, ...) */
  QBC_ECUDA = 4,    /* CUDA runtime error */
  QBC_ENOMEM = 5,   /* device or host allocation refused */
  QBC_EDEVICE = 6,  /* a kernel reported an error word (capacity exceeded, bound hit) */
  QBC_ETIMEOUT = 7, /* reserved (a served wait that runs out returns QBC_OK with *done = 0) */
  QBC_EBUSY = 8     /* the index is serving, the request queue is full, or a request was
                       cancelled by qbc_serve_close */
};

enum {
  QBC_INDEX_MHL = 0, /* TreeCount distance + count + hop labels (MHL-QBC, RQ) */
  QBC_INDEX_H2H = 1, /* H2H distance labels from an order file (QBC) */
  /* No labels: each source's (distance, count, hop) row comes from a shortest-path sweep over the
   * arc list on the device (near-far buckets, then the SP-DAG counted in topological waves), the
   * same rows the TreeCount scan gives (MHLQBC.cu:334-412 semantics).  For graphs whose tree
   * decomposition is too wide for label rows, e.g. road grids with random long shortcuts, where
   * the reference's own index build (TreeDecomp.cpp:54-208) does not finish. */
  QBC_INDEX_CSR = 2
};

typedef struct qbc_graph qbc_graph; /* host arc list, Graph::ReadGraph rules */
typedef struct qbc_index qbc_index; /* host index + its device-resident copy + per-source scratch */

const char *qbc_last_error(void);
const char *qbc_version(void);

/* ---- input (replaces Graph::ReadGraph, src/Graph.cpp:4-37) ----------------------------------
 * Lines "u v w" are directed arcs, 1-based; a repeated (u,v) keeps the first arc, weight 0 reads
 * as 1 (src/Graph.cpp:27-35).  Beyond the reference, the graph is validated: every arc needs its
 * reverse with the same weight (the index reader symmetrises, src/TreeCount/Graph.cpp:55-71), no
 * self loops, connected (QBC.cu:525 spins forever otherwise), and total weight < 999999999 so no
 * distance reaches the reference's INF. */
int qbc_graph_read(const char *path, qbc_graph **out);
int qbc_graph_from_lines(int n, int m, const int32_t *u1, const int32_t *v1, const int32_t *w, qbc_graph **out);
int qbc_graph_info(const qbc_graph *g, int32_t *n, int32_t *arcs);
/* arcs in Graph's CSR order (initGraphTravel, MHLQBC.cu:130-160): off[n+1], head[arcs], w[arcs] */
int qbc_graph_arcs(const qbc_graph *g, int32_t *off, int32_t *head, int32_t *w);
void qbc_graph_free(qbc_graph *g);

/* order file "n" + n lines "id order", 0-based ids (Graph::CHconsorderMT, src/buildIndex.cpp:6-20) */
int qbc_read_order(const char *path, int32_t n, int32_t *node_order);
/* query batch "q" + q 1-based ids (processBactch, RQ.cu:589-610); ids0 receives 0-based ids */
int qbc_read_query(const char *path, int32_t n, int32_t cap, int32_t *q, int32_t *ids0);
/* min-degree contraction order (the order-file generator Graph::GraphConstract,
 * src/buildIndex.cpp:759-925); node_order[vid] = rank, 0 contracted first */
int qbc_min_degree_order(const qbc_graph *g, int32_t *node_order);

/* ---- index (replaces TreeDecomp Reduce/MakeTree/MakeIndex, src/TreeCount/TreeDecomp.cpp:54-511,
 * with moveCountIndexToDevice, MHLQBC.cu:6-128; and Graph::CHconsorderMT/makeTree/makeIndex,
 * src/buildIndex.cpp:4-310, with moveDisIndexToDevice, QBC.cu:11-127) -------------------------
 * kind QBC_INDEX_MHL ignores node_order; QBC_INDEX_H2H requires it; QBC_INDEX_CSR ignores it and
 * keeps the arc list in vertex-id order (checked connected).  nthreads <= 0: all cores. */
int qbc_index_build(const qbc_graph *g, int kind, const int32_t *node_order, int nthreads, qbc_index **out);
/* copies the index to HBM of `device` (cudaSetDevice semantics, QBC.cu:601-602) */
int qbc_index_upload(qbc_index *idx, int device);
/* On-disk index (replaces the reference's headerless tmpRoadCountIndex file, TreeDecomp.cpp:243,
 * 460-467,496-506, and TreeQuery::ReadIndex, TreeDecomp.cpp:748-900): the whole index with its rows,
 * a versioned header and a checksum.  save copies device-built rows back first; load returns a
 * host index (then qbc_index_upload).  A damaged, truncated or foreign file gives QBC_EIO. */
int qbc_index_save(qbc_index *idx, const char *path);
int qbc_index_load(const char *path, qbc_index **out);
/* As qbc_index_build, with the label rows filled on the GPU `device` (elimination and tree on the
 * host; the rows, one launch per tree depth, on the device) and left there: the index is uploaded on
 * return and the host holds no label rows until qbc_index_export or qbc_index_release_device copies
 * them back.  Same rows as qbc_index_build (TreeDecomp.cpp:388-450 semantics).  Replaces the CPU
 * label build of TreeDecomp::MakeIndex (TreeDecomp.cpp:388-511) and buildIndex.cpp:246-270. */
int qbc_index_build_device(const qbc_graph *g, int kind, const int32_t *node_order, int device, qbc_index **out);
/* drops the device copy (keeps the host index) */
int qbc_index_release_device(qbc_index *idx);
/* info[0]=n, [1]=arcs, [2]=label entries, [3]=tree height, [4]=tree width, [5]=device bytes,
 * [6]=kind, [7]=sum over vertices of depth (label bytes/12 for MHL) */
int qbc_index_info(const qbc_index *idx, int64_t *info);
/* Sum over the listed sources of the label entries the K2 scan reads (sum_t h(lca(s,t)));
 * the algorithmic-bytes figure of the roofline. */
int qbc_index_scan_entries(const qbc_index *idx, const int32_t *sources0, int32_t ns, int64_t *entries);
/* Label entries the batched label scan copies from target rows when the listed sources, sorted by
 * tree position, form CTAs of `group` consecutive sources: each CTA copies target row t up to the
 * deepest LCA depth of t with one of its sources.  Times 4 bytes, the DRAM-read model of that
 * kernel's target rows (no counterpart in the reference, which reads labels per pair). */
int qbc_index_group_entries(const qbc_index *idx, const int32_t *sources0, int32_t ns, int32_t group, int64_t *entries);
/* Sources per CTA of the batched label scan under the current tuning: 32 for the packed-key
 * kernel, 16 for its tall-tree form, 32/K for the general kernel, 0 for the label-free index (the
 * `group` of qbc_index_group_entries).  Needs the index's device state. */
int qbc_index_label_group(qbc_index *idx, int32_t *sources_per_cta);
/* Name of the kernel that produces the batched per-source rows under the current tuning
 * ("k_label_scan_packed", "k_label_scan_rows16", "k_label_scan_tall", "k_label_scan_pair",
 * "k_label_scan", or "k_sweep_rows" for the label-free index), NUL-terminated in name[0..cap),
 * for matching profiler output to a configuration; no counterpart in the reference.  Needs the
 * index's device state. */
int qbc_index_label_kernel(qbc_index *idx, char *name, int32_t cap);
void qbc_index_free(qbc_index *idx);
/* Copies the host index out (for inspection and tests).  Arrays sized by qbc_index_info:
 * vid_of/depth/send[n], lab_off[n+1], dis/anc[info[2]], ch[2*info[2]] (MHL only; may be NULL). */
int qbc_index_export(const qbc_index *idx, int32_t *vid_of, int32_t *depth, int32_t *send, int64_t *lab_off,
                     int32_t *dis, int32_t *ch, int32_t *anc);

/* Tuning of the batched path: params[0]=lanes per source K of the label scan (0=auto: the
 * packed-key kernel when the index allows it, else the smallest K whose rows fit shared memory;
 * 1..32 forces the general kernel with 32/K sources per CTA), [1]=threads per CTA of the general
 * label kernel, [2]=target split per source group (0=auto), [3]=sources per chunk (0=auto),
 * [4]=threads per CTA of the CTA-per-source dependency kernel, [5]=dependency form (0 auto = 4,
 * 1 one warp per source, 2 one CTA per source, 3 one warp per source with the backprop's
 * layer-independent loads issued one to three steps ahead, 4 one CTA per source, pipelined the
 * same way), [6]=level-queue depth of the warp form (layers
 * counted in shared memory, 64..2048; 0 = 512), [7]=warps per CTA of the packed-key kernel (8 or
 * 16 or 20; 0 = the most warps whose shared memory holds the whole tree height, else 8; 12 = a 12-warp kernel that scans
 * two targets per step against one load of the source words), [8]=label tile: entries of
 * each row staged in shared memory by the packed-key kernel (0 = all that fit; later entries of a
 * scan are read from global memory or taken in further passes, see [9]), [9]=label passes for
 * rows longer than the tile (0 = 1: one launch, entries beyond the tile read from global memory;
 * 2: one launch per tile of entries, the pairs' running minima kept in the output rows between
 * passes), [10]=distance bucket width of the CSR index's shortest-path sweep (0 = auto: twice the
 * mean arc weight), [11]=threads per CTA of that sweep (256, 512 or 1024; 0 = 512; 2048 = 512-thread
 * CTAs, four per SM), [12]=sources
 * per CTA of the packed-key label scan (32; 16 = the tall-tree kernel: whole rows of 16 sources in
 * shared memory, two targets per warp, target rows streamed through a cp.async ring, when the
 * height fits; 0 = auto: 16 when the 32-source kernel cannot hold whole rows and [7]-[9] are 0),
 * [13]=target rows of the 16-source kernel (1 = whole rows, double-buffered per warp side; 2 =
 * 64-entry blocks through a ring; 0 = auto: whole rows when they fit with 16 warps).  Refused
 * with QBC_EBUSY while the index serves. */
int qbc_index_set_tuning(qbc_index *idx, const int32_t *params, int32_t nparams);
int qbc_index_get_tuning(const qbc_index *idx, int32_t *params, int32_t nparams);

/* Kernel timing: after qbc_index_profile(idx, 1) every label-scan and dependency launch is
 * bracketed by CUDA events on its own stream; qbc_index_stats synchronises and returns
 * out[0]=label-scan ms, [1]=label-scan launches, [2]=dependency ms, [3]=dependency launches,
 * [4]=all kernel launches of the library since the profile call. */
int qbc_index_profile(qbc_index *idx, int on);
int qbc_index_stats(qbc_index *idx, double *out);

/* Autotuner (no counterpart in the reference): times candidate tunings -- sources per CTA and
 * threads of the label kernel, target split, dependency form and level-queue depth, chunk size --
 * on a sweep over the listed sources, keeps the fastest on the index and returns it in params
 * (layout of qbc_index_set_tuning, up to 12) with its time per source in ms.  On a CSR index
 * it tunes the sweep's bucket width and threads, the dependency threads and the chunk size. */
int qbc_autotune(qbc_index *idx, const int32_t *sources0, int32_t ns, int32_t *params, int32_t nparams,
                 double *ms_per_source);

/* ---- BC (replaces Graph::brandesBCIndexGPU_5, MHLQBC.cu:495-537 / QBC.cu:419-584) ------------
 * Batched path: many sources per launch, label rows staged in shared memory, level-bucketed
 * backprop.  qbc_bc_all's sweep is captured once into a CUDA graph per tuning and replayed.
 * bc_out: n host doubles (overwritten). */
int qbc_bc_all(qbc_index *idx, double *bc_out);
/* partial BC over a source list (0-based vids) */
int qbc_bc_sources(qbc_index *idx, const int32_t *sources0, int32_t ns, double *bc_out);
/* plain path: one source per launch sequence (label kernel over the whole GPU, then one CTA for its
 * dependency pass, as the reference gives each source one block, MHLQBC.cu:237-475) */
int qbc_bc_plain(qbc_index *idx, const int32_t *sources0, int32_t ns, double *bc_out);
/* Device-resident variant: d_sources0 (ns int32) and d_bc (n doubles, accumulated into, not
 * cleared) are device pointers; stream is a cudaStream_t or NULL for the index's own stream.
 * Sources may come in any order and repeat: they are sorted into tree order on the device (the
 * label kernels run fastest on tree neighbours); the index grows its source buffers (2 x 4 B per
 * source plus the sort's temporary storage) when a longer list arrives, which synchronises the
 * stream once.  Returns after enqueueing; the caller synchronises. */
int qbc_bc_sources_device(qbc_index *idx, const int32_t *d_sources0, int32_t ns, double *d_bc, void *stream);

/* One source's BC contribution without allocating: no counterpart in the reference.
 * For callers that cannot allocate device memory when they need BC -- a host application whose
 * memory manager already holds the GPU's memory, or a serving loop that must stay free of
 * cudaMalloc/cudaFree (they synchronise the device and have unbounded latency).  The per-source
 * scratch lives in a static device array built into the library (about 5 MiB, held by every GPU
 * that loads the library until the process exits), so graphs are limited to
 * QBC_STATIC_MAX_VERTICES vertices (larger ones return QBC_EINVAL).  On a label index the
 * one-source label kernel also holds 44 bytes per tree level in shared memory, so trees taller
 * than about 5,100 levels (long paths, thin strips) return QBC_EINVAL too; a QBC_INDEX_CSR index
 * has no such limit.  The index must already be uploaded.  Adds 0.5*delta_s(v) into d_bc (device
 * pointer, n doubles, 0-based vid order) on `stream` (NULL: the index's stream); the caller
 * synchronises.  A device-side error of the call (a sweep that hit its bound) is recorded in the
 * index's error word and returned by the index's next synchronous call.  The first call on a
 * device looks up the array's device address with that device current and caches it for the
 * process; make that first call before any stream capture, and not across a cudaDeviceReset.
 * All calls share the one array, which keeps the previous call's contents: calls that overlap
 * on the GPU (other streams, other host threads) race, so issue them in one stream. */
#define QBC_STATIC_MAX_VERTICES 131072
int qbc_bc_source_static(qbc_index *idx, int32_t source0, double *d_bc, void *stream);

/* ---- RQ (replaces Graph::brandesBCIndexGPU_PointBatch, RQ.cu:465-531) -----------------------
 * BC of each query vertex over all sources (the reference's pair formula equals BC restricted to
 * the query set).  points0: q 0-based vids; out: q doubles. */
int qbc_bc_query(qbc_index *idx, const int32_t *points0, int32_t q, double *out);
/* Batched RQ: many query sets sharing one source sweep (a replayed CUDA graph, as qbc_bc_all):
 * set i is points0[set_off[i] .. set_off[i+1]), set_off[0] = 0; out has set_off[nsets] doubles.
 * sources0 (ns vids) restricts the sweep to those sources (partial sums), NULL = all. */
int qbc_bc_query_batch(qbc_index *idx, const int32_t *points0, const int32_t *set_off, int32_t nsets,
                       const int32_t *sources0, int32_t ns, double *out);

/* ---- Served RQ (no counterpart in the reference) ------------------------------------------------
 * A request loop on its own host thread and CUDA stream keeps sweeping the source list (NULL = all
 * vertices) chunk by chunk while requests are in flight; each chunk's launches are one captured
 * CUDA graph whose last kernel adds the chunk's BC into the device accumulator of every admitted
 * request.  A request (a vertex set) is admitted at the next chunk boundary when fewer than
 * opts[0] requests are active (default 64) and its q accumulators fit in the request pool of
 * opts[1] bytes (16 B per query vertex; 0 = min(free device memory / 8, 64 MiB)); it completes
 * after one full turn over the sources from its admission, so its values equal qbc_bc_query's
 * (up to FP64 summation order) whatever else runs.  opts[2] = queue capacity (0 = 2^20);
 * opts[3] = sources per served chunk, the admission granularity (0 = the index's chunk).  While a
 * server is open the index refuses every other device call with QBC_EBUSY.
 * times (3 doubles, may be NULL) = submit, admission and completion in seconds since open. */
typedef struct qbc_server qbc_server;
int qbc_serve_open(qbc_index *idx, const int32_t *sources0, int32_t ns, const int64_t *opts, int32_t nopts,
                   qbc_server **out);
/* queues a request of q vertices (0-based vids); QBC_EBUSY when the queue is full */
int qbc_serve_submit(qbc_server *srv, const int32_t *points0, int32_t q, int64_t *ticket);
/* *done = 1 and out (q doubles) filled once the request is complete (the ticket is then released) */
int qbc_serve_poll(qbc_server *srv, int64_t ticket, double *out, double *times, int32_t *done);
/* as qbc_serve_poll, waiting up to timeout_s seconds (< 0: no limit) */
int qbc_serve_wait(qbc_server *srv, int64_t ticket, double timeout_s, double *out, double *times, int32_t *done);
/* out[0]=chunks run, [1]=turns over the sources, [2]=requests done, [3]=active, [4]=queued,
 * [5]=pool entries in use, [6]=pool capacity, [7]=chunks per turn, [8]=sources per turn */
int qbc_serve_stats(qbc_server *srv, double *out, int32_t nout);
/* cancels queued and active requests (their waiters get QBC_EBUSY), waits for the device work in
 * flight and for threads still inside qbc_serve_wait to return, then frees the server; no call on
 * the server may start once qbc_serve_close has been called */
int qbc_serve_close(qbc_server *srv);

/* ---- per-source rows (the K2 output: MHLQBC.cu:334-412, RQ.cu:228-291, QBC.cu:272-331) ------
 * dist/cnt/hop: ns*n each, row k = source sources0[k], column = 0-based vid.  cnt and hop may be
 * NULL; for an H2H index they are filled by the device Kahn pass (QBC.cu:485-555 semantics). */
int qbc_rows(qbc_index *idx, const int32_t *sources0, int32_t ns, int32_t *dist, uint32_t *cnt, int32_t *hop);

#ifdef __cplusplus
}
#endif
#endif

// capi.cpp -- extern "C" boundary of libqbc_b200 (declared in include/qbc_b200.h).
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <string>

#include "../../include/qbc_b200.h"
#include "device.h"
#include "host.h"

struct qbc_graph {
  qbc::Graph g;
};
struct qbc_index {
  qbc::Handle h;
  ~qbc_index() {
    if (h.server) qbc::serve_close(h.server);
    qbc::device_release(h);
  }
};
struct qbc_server {
  qbc::Server *s;
};

namespace {
thread_local std::string g_err;

template <class F>
int guarded(F &&f) {
  try {
    f();
    g_err.clear();
    return QBC_OK;
  } catch (const qbc::Error &e) {
    g_err = e.what();
    return e.code;
  } catch (const std::bad_alloc &) {
    g_err = "host allocation failed";
    return QBC_ENOMEM;
  } catch (const std::exception &e) {
    g_err = e.what();
    return QBC_EINVAL;
  }
}

void need(bool ok, const char *what) {
  if (!ok) throw qbc::Error(QBC_EINVAL, what);
}

constexpr int32_t kTuningFields = 14;  // qbc_index_set_tuning's params layout

void not_serving(const qbc_index *idx) {
  if (idx->h.server) throw qbc::Error(QBC_EBUSY, "the index is serving requests: close its server first");
}
}  // namespace

extern "C" {

const char *qbc_last_error(void) { return g_err.c_str(); }
const char *qbc_version(void) { return "qbc_b200 0.1 (sm_100a)"; }

int qbc_graph_read(const char *path, qbc_graph **out) {
  return guarded([&] {
    need(path && out, "null argument");
    auto p = std::make_unique<qbc_graph>();
    p->g = qbc::graph_read(path);
    *out = p.release();
  });
}

int qbc_graph_from_lines(int n, int m, const int32_t *u1, const int32_t *v1, const int32_t *w, qbc_graph **out) {
  return guarded([&] {
    need(out && (m == 0 || (u1 && v1 && w)), "null argument");
    auto p = std::make_unique<qbc_graph>();
    p->g = qbc::graph_from_lines(n, m, u1, v1, w);
    *out = p.release();
  });
}

int qbc_graph_info(const qbc_graph *g, int32_t *n, int32_t *arcs) {
  return guarded([&] {
    need(g, "null graph");
    if (n) *n = g->g.n;
    if (arcs) *arcs = g->g.arcs();
  });
}

int qbc_graph_arcs(const qbc_graph *g, int32_t *off, int32_t *head, int32_t *w) {
  return guarded([&] {
    need(g, "null graph");
    if (off) std::memcpy(off, g->g.off.data(), g->g.off.size() * 4);
    if (head) std::memcpy(head, g->g.head.data(), g->g.head.size() * 4);
    if (w) std::memcpy(w, g->g.w.data(), g->g.w.size() * 4);
  });
}

void qbc_graph_free(qbc_graph *g) { delete g; }

int qbc_read_order(const char *path, int32_t n, int32_t *node_order) {
  return guarded([&] {
    need(path && node_order, "null argument");
    auto o = qbc::read_order(path, n);
    std::memcpy(node_order, o.data(), o.size() * 4);
  });
}

int qbc_read_query(const char *path, int32_t n, int32_t cap, int32_t *q, int32_t *ids0) {
  return guarded([&] {
    need(path && q, "null argument");
    auto ids = qbc::read_query(path, n);
    *q = (int32_t)ids.size();
    if (ids0) {
      if ((int32_t)ids.size() > cap) throw qbc::Error(QBC_EINVAL, "query batch larger than the output capacity");
      std::memcpy(ids0, ids.data(), ids.size() * 4);
    }
  });
}

int qbc_min_degree_order(const qbc_graph *g, int32_t *node_order) {
  return guarded([&] {
    need(g && node_order, "null argument");
    auto o = qbc::min_degree_order(g->g);
    std::memcpy(node_order, o.data(), o.size() * 4);
  });
}

int qbc_index_build(const qbc_graph *g, int kind, const int32_t *node_order, int nthreads, qbc_index **out) {
  return guarded([&] {
    need(g && out, "null argument");
    auto p = std::make_unique<qbc_index>();
    if (kind == QBC_INDEX_MHL) {
      p->h.host = qbc::build_mhl(g->g, nthreads);
    } else if (kind == QBC_INDEX_H2H) {
      need(node_order != nullptr, "H2H index needs a node order");
      std::vector<int32_t> o(node_order, node_order + g->g.n);
      p->h.host = qbc::build_h2h(g->g, o, nthreads);
    } else if (kind == QBC_INDEX_CSR) {
      p->h.host = qbc::build_csr(g->g);
    } else {
      throw qbc::Error(QBC_EINVAL, "unknown index kind");
    }
    *out = p.release();
  });
}

// Vertices whose min-degree elimination runs on the device (the dense tail, device_dense_eliminate)
// in a device build: the last 16,384 of graphs with at least 262,144 vertices (1M grid: the last
// 16,384 eliminations are 2.9 of the host's 5.0 s).  Test hook: QBC_DENSE_TAIL overrides it (0
// disables the tail; a value >= n eliminates the whole graph on the device).
static int32_t dense_tail_size(int32_t n) {
  const char *e = std::getenv("QBC_DENSE_TAIL");
  if (e && *e) return std::max<int32_t>(0, (int32_t)std::strtol(e, nullptr, 10));
  return n >= 262144 ? 16384 : 0;
}

int qbc_index_build_device(const qbc_graph *g, int kind, const int32_t *node_order, int device, qbc_index **out) {
  return guarded([&] {
    need(g && out, "null argument");
    need(kind == QBC_INDEX_MHL || kind == QBC_INDEX_H2H || kind == QBC_INDEX_CSR, "unknown index kind");
    need(kind != QBC_INDEX_H2H || node_order != nullptr, "H2H index needs a node order");
    auto p = std::make_unique<qbc_index>();
    if (kind == QBC_INDEX_CSR) {  // no label rows to fill: the arc list goes to the device as it is
      p->h.host = qbc::build_csr(g->g);
      qbc::device_upload(p->h, device);
      *out = p.release();
      return;
    }
    qbc::Separators seps;
    std::vector<int32_t> o;
    if (node_order) o.assign(node_order, node_order + g->g.n);
    const qbc::TailEngine tail = [device](qbc::DenseTail &dt) { qbc::device_dense_eliminate(device, dt); };
    p->h.host = qbc::prepare_index(g->g, kind == QBC_INDEX_MHL ? qbc::IndexKind::MHL : qbc::IndexKind::H2H,
                                   node_order ? &o : nullptr, seps, dense_tail_size(g->g.n), tail);
    qbc::device_build(p->h, device, seps);
    *out = p.release();
  });
}

int qbc_index_save(qbc_index *idx, const char *path) {
  return guarded([&] {
    need(idx && path, "null argument");
    if (!idx->h.host.rows_on_host) {
      not_serving(idx);
      qbc::device_download_rows(idx->h);
    }
    qbc::index_save(idx->h.host, path);
  });
}

int qbc_index_load(const char *path, qbc_index **out) {
  return guarded([&] {
    need(path && out, "null argument");
    auto p = std::make_unique<qbc_index>();
    p->h.host = qbc::index_load(path);
    *out = p.release();
  });
}

int qbc_index_upload(qbc_index *idx, int device) {
  return guarded([&] {
    need(idx, "null index");
    not_serving(idx);
    qbc::device_upload(idx->h, device);
  });
}

int qbc_index_release_device(qbc_index *idx) {
  return guarded([&] {
    need(idx, "null index");
    not_serving(idx);
    qbc::device_download_rows(idx->h);  // device-built rows move to the host first
    qbc::device_release(idx->h);
  });
}

int qbc_index_info(const qbc_index *idx, int64_t *info) {
  return guarded([&] {
    need(idx && info, "null argument");
    const qbc::Index &ix = idx->h.host;
    info[0] = ix.n;
    info[1] = (int64_t)ix.arc_head.size();
    info[2] = ix.lab_off.empty() ? 0 : ix.lab_off[ix.n];
    info[3] = ix.tree_height;
    info[4] = ix.tree_width;
    info[5] = qbc::device_bytes(idx->h);
    info[6] = (int64_t)ix.kind;
    info[7] = ix.depth_sum;
  });
}

int qbc_index_scan_entries(const qbc_index *idx, const int32_t *sources0, int32_t ns, int64_t *entries) {
  return guarded([&] {
    need(idx && entries && (ns == 0 || sources0), "null argument");
    for (int32_t i = 0; i < ns; i++)
      if (sources0[i] < 0 || sources0[i] >= idx->h.host.n) throw qbc::Error(QBC_EINVAL, "source id out of range");
    *entries = qbc::scan_entries(idx->h.host, sources0, ns);
  });
}

int qbc_index_group_entries(const qbc_index *idx, const int32_t *sources0, int32_t ns, int32_t group, int64_t *entries) {
  return guarded([&] {
    need(idx && entries && (ns == 0 || sources0) && group > 0, "null argument or group < 1");
    for (int32_t i = 0; i < ns; i++)
      if (sources0[i] < 0 || sources0[i] >= idx->h.host.n) throw qbc::Error(QBC_EINVAL, "source id out of range");
    *entries = qbc::group_entries(idx->h.host, sources0, ns, group);
  });
}

int qbc_index_label_group(qbc_index *idx, int32_t *sources_per_cta) {
  return guarded([&] {
    need(idx && sources_per_cta, "null argument");
    *sources_per_cta = qbc::device_label_group(idx->h);
  });
}

int qbc_index_label_kernel(qbc_index *idx, char *name, int32_t cap) {
  return guarded([&] {
    need(idx && name && cap > 0, "null argument or cap < 1");
    const char *k = qbc::device_label_kernel(idx->h);
    std::strncpy(name, k, (size_t)cap - 1);
    name[cap - 1] = '\0';
  });
}

void qbc_index_free(qbc_index *idx) { delete idx; }

int qbc_index_export(const qbc_index *idx, int32_t *vid_of, int32_t *depth, int32_t *send, int64_t *lab_off,
                     int32_t *dis, int32_t *ch, int32_t *anc) {
  return guarded([&] {
    need(idx, "null index");
    if (!idx->h.host.rows_on_host) {
      not_serving(idx);
      qbc::device_download_rows(const_cast<qbc_index *>(idx)->h);
    }
    const qbc::Index &ix = idx->h.host;
    auto cp = [](void *dst, const void *src, size_t bytes) {
      if (dst && bytes) std::memcpy(dst, src, bytes);
    };
    cp(vid_of, ix.vid_of.data(), ix.vid_of.size() * 4);
    cp(depth, ix.depth.data(), ix.depth.size() * 4);
    cp(send, ix.send.data(), ix.send.size() * 4);
    cp(lab_off, ix.lab_off.data(), ix.lab_off.size() * 8);
    cp(dis, ix.dis.data(), ix.dis.size() * 4);
    cp(ch, ix.ch.data(), ix.ch.size() * 4);
    cp(anc, ix.anc.data(), ix.anc.size() * 4);
  });
}

int qbc_index_set_tuning(qbc_index *idx, const int32_t *params, int32_t nparams) {
  return guarded([&] {
    need(idx && (nparams == 0 || params), "null argument");
    qbc::Tuning &t = idx->h.tuning;
    not_serving(idx);
    int32_t *f[] = {&t.lanes_per_source, &t.label_threads, &t.split, &t.chunk, &t.dep_threads, &t.dep_form, &t.queue_depth, &t.label_warps, &t.label_tile, &t.label_passes, &t.sweep_delta, &t.sweep_threads, &t.label_sources, &t.label_stream};
    if (nparams > 0) {
      int32_t k = params[0];
      need(k == 0 || k == 1 || k == 2 || k == 4 || k == 8 || k == 16 || k == 32, "lanes per source must be 0 or a power of two <= 32");
    }
    const int32_t old_chunk = t.chunk;
    if (nparams > 5) need(params[5] >= 0 && params[5] <= 4, "dependency form must be 0..4");
    if (nparams > 6) need(params[6] == 0 || (params[6] >= 64 && params[6] <= 2048), "queue depth must be 0 or in [64, 2048]");
    if (nparams > 7)
      need(params[7] == 0 || params[7] == 8 || params[7] == 12 || params[7] == 16 || params[7] == 20,
           "label warps must be 0, 8, 12 (two-target kernel), 16 or 20");
    if (nparams > 8) need(params[8] >= 0, "label tile must be >= 0");
    if (nparams > 9) need(params[9] >= 0 && params[9] <= 2, "label passes must be 0, 1 or 2");
    if (nparams > 10) need(params[10] >= 0, "sweep bucket width must be >= 0");
    if (nparams > 11)
      need(params[11] == 0 || params[11] == 256 || params[11] == 512 || params[11] == 1024 || params[11] == 2048,
           "sweep threads must be 0, 256, 512, 1024 or 2048 (four 512-thread CTAs per SM)");
    if (nparams > 12) need(params[12] == 0 || params[12] == 16 || params[12] == 32, "label sources must be 0, 16 or 32");
    if (nparams > 13) need(params[13] >= 0 && params[13] <= 2, "label stream must be 0, 1 or 2");
    for (int32_t i = 0; i < nparams && i < kTuningFields; i++) *f[i] = params[i];
    if (nparams > 3 && t.chunk != old_chunk && idx->h.dev) qbc::device_set_chunk(idx->h, t.chunk);
  });
}

int qbc_index_get_tuning(const qbc_index *idx, int32_t *params, int32_t nparams) {
  return guarded([&] {
    need(idx && (nparams == 0 || params), "null argument");
    const qbc::Tuning &t = idx->h.tuning;
    const int32_t f[] = {t.lanes_per_source, t.label_threads, t.split, t.chunk, t.dep_threads, t.dep_form, t.queue_depth, t.label_warps, t.label_tile, t.label_passes, t.sweep_delta, t.sweep_threads, t.label_sources, t.label_stream};
    for (int32_t i = 0; i < nparams && i < kTuningFields; i++) params[i] = f[i];
  });
}

int qbc_bc_all(qbc_index *idx, double *bc_out) {
  return guarded([&] {
    need(idx && bc_out, "null argument");
    qbc::host_bc_sweep(idx->h, nullptr, 0, bc_out);
  });
}

int qbc_bc_sources(qbc_index *idx, const int32_t *sources0, int32_t ns, double *bc_out) {
  return guarded([&] {
    need(idx && bc_out && ns >= 0 && (ns == 0 || sources0), "null argument");
    qbc::host_bc_sources(idx->h, sources0, ns, bc_out);
  });
}

int qbc_bc_plain(qbc_index *idx, const int32_t *sources0, int32_t ns, double *bc_out) {
  return guarded([&] {
    need(idx && bc_out && ns >= 0 && (ns == 0 || sources0), "null argument");
    qbc::host_bc_plain(idx->h, sources0, ns, bc_out);
  });
}

int qbc_bc_sources_device(qbc_index *idx, const int32_t *d_sources0, int32_t ns, double *d_bc, void *stream) {
  return guarded([&] {
    need(idx && d_bc && ns >= 0 && (ns == 0 || d_sources0), "null argument");
    qbc::device_bc_sources(idx->h, d_sources0, ns, d_bc, stream);
  });
}

int qbc_bc_query(qbc_index *idx, const int32_t *points0, int32_t q, double *out) {
  return guarded([&] {
    need(idx && q >= 0 && (q == 0 || (points0 && out)), "null argument");
    qbc::host_query_batch(idx->h, points0, q, nullptr, 0, out);
  });
}

int qbc_bc_query_batch(qbc_index *idx, const int32_t *points0, const int32_t *set_off, int32_t nsets,
                       const int32_t *sources0, int32_t ns, double *out) {
  return guarded([&] {
    need(idx && set_off && nsets >= 0, "null argument");
    need(set_off[0] == 0, "set offsets must start at 0");
    for (int32_t k = 0; k < nsets; k++) need(set_off[k + 1] >= set_off[k], "set offsets must not decrease");
    const int32_t total = nsets ? set_off[nsets] : 0;
    need(total == 0 || (points0 && out), "null argument");
    need(!sources0 || ns > 0, "empty source list");
    qbc::host_query_batch(idx->h, points0, total, sources0, ns, out);
  });
}

int qbc_index_profile(qbc_index *idx, int on) {
  return guarded([&] {
    need(idx, "null index");
    qbc::device_profiling(idx->h, on != 0);
  });
}

int qbc_index_stats(qbc_index *idx, double *out) {
  return guarded([&] {
    need(idx && out, "null argument");
    qbc::device_stats(idx->h, out);
  });
}

int qbc_bc_source_static(qbc_index *idx, int32_t source0, double *d_bc, void *stream) {
  return guarded([&] {
    need(idx, "null index");
    qbc::host_bc_source_static(idx->h, source0, d_bc, stream);
  });
}

int qbc_rows(qbc_index *idx, const int32_t *sources0, int32_t ns, int32_t *dist, uint32_t *cnt, int32_t *hop) {
  return guarded([&] {
    need(idx && dist && ns >= 0 && (ns == 0 || sources0), "null argument");
    qbc::host_rows(idx->h, sources0, ns, dist, cnt, hop);
  });
}

int qbc_autotune(qbc_index *idx, const int32_t *sources0, int32_t ns, int32_t *params, int32_t nparams,
                 double *ms_per_source) {
  return guarded([&] {
    need(idx && sources0 && ns > 0, "null argument");
    double ms = 0.0;
    qbc::autotune(idx->h, sources0, ns, &ms);
    if (ms_per_source) *ms_per_source = ms;
    const qbc::Tuning &t = idx->h.tuning;
    const int32_t f[] = {t.lanes_per_source, t.label_threads, t.split, t.chunk, t.dep_threads, t.dep_form, t.queue_depth, t.label_warps, t.label_tile, t.label_passes, t.sweep_delta, t.sweep_threads, t.label_sources, t.label_stream};
    for (int32_t i = 0; params && i < nparams && i < kTuningFields; i++) params[i] = f[i];
  });
}

int qbc_serve_open(qbc_index *idx, const int32_t *sources0, int32_t ns, const int64_t *opts, int32_t nopts,
                   qbc_server **out) {
  return guarded([&] {
    need(idx && out && (nopts == 0 || opts) && (!sources0 || ns > 0), "null argument");
    auto p = std::make_unique<qbc_server>();
    p->s = qbc::serve_open(idx->h, sources0, ns, opts, nopts);
    *out = p.release();
  });
}

int qbc_serve_submit(qbc_server *srv, const int32_t *points0, int32_t q, int64_t *ticket) {
  return guarded([&] {
    need(srv && ticket, "null argument");
    *ticket = qbc::serve_submit(srv->s, points0, q);
  });
}

int qbc_serve_poll(qbc_server *srv, int64_t ticket, double *out, double *times, int32_t *done) {
  return guarded([&] {
    need(srv && done, "null argument");
    *done = qbc::serve_poll(srv->s, ticket, out, times);
  });
}

int qbc_serve_wait(qbc_server *srv, int64_t ticket, double timeout_s, double *out, double *times, int32_t *done) {
  return guarded([&] {
    need(srv && done, "null argument");
    *done = qbc::serve_wait(srv->s, ticket, timeout_s, out, times);
  });
}

int qbc_serve_stats(qbc_server *srv, double *out, int32_t nout) {
  return guarded([&] {
    need(srv && (nout == 0 || out), "null argument");
    qbc::serve_stats(srv->s, out, nout);
  });
}

int qbc_serve_close(qbc_server *srv) {
  return guarded([&] {
    if (!srv) return;
    qbc::serve_close(srv->s);
    delete srv;
  });
}

}  // extern "C"

// sssp.cu -- label-free per-source rows of libqbc_b200 (QBC_INDEX_CSR).
//
// The label kernels get a source's (distance, path count, max hop) row from ancestor labels of a
// tree decomposition (MHLQBC.cu:334-412).  That index grows with the graph's tree width: on a road
// grid with 2 % uniformly random long shortcuts the width jumps from 196 to 1,441 at 50k vertices
// and the elimination (the reference's TreeDecomp::Reduce, TreeDecomp.cpp:54-208, as well as this
// library's) does not finish at 200k.  For such graphs the rows come from a shortest-path sweep
// over the arc list instead, one CTA per source (k_sweep_rows):
//
//   distances  near-far buckets.  Vertices whose tentative distance is below the current threshold
//              T form the near list and are relaxed in passes (Bellman-Ford inside the bucket)
//              until no distance below T changes; a relaxation that lands at or beyond T parks the
//              vertex in the far list.  Then T advances by the bucket width and the far list is
//              split: entries now below T become the next near list, entries settled earlier are
//              dropped, the rest stay.  A vertex is relaxed again only when its distance dropped,
//              and the buckets keep the long shortcuts (weights 500..5000 against ~100 on the grid)
//              from flooding the graph with distances that later get undercut.
//   counts     Kahn waves over the SP-DAG (arcs t -> h with d[h] == d[t] + w): a vertex enters
//              wave L once all its DAG predecessors are done, so L is the largest number of arcs
//              on a shortest path (TreeCount's my_cnt) and its count, the 32-bit wrapping sum of
//              its predecessors' counts, is complete (TreeCount's cnt).
//
// It writes the same outputs as the label scan -- records (dist, count, .), hop layers and the
// largest layer per source -- so the dependency passes of the label path run unchanged (they
// write the records' last 8 bytes before reading them).
//
// Memory: the frontier phases visit vertices scattered over the graph (the shortcuts spread every
// wave across it), so each visit costs DRAM sectors, not bytes.  A vertex's whole sweep state is
// therefore its 16-byte record -- distance, list stamp (then count), in-degree -- and one sector
// fetch serves a visit; measured at 1M vertices + 2 % shortcuts, separate 4-byte arrays for the
// same fields cost 8-10 sectors per visit.  Lists use the per-source buffers of the label path:
// near list and Kahn queue in the level-queue row, next near list and far list in the two halves
// of the layer-counter row; hop layers go to the hop row as vertices leave their wave.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <string>

#include "device_state.h"

namespace qbc {

namespace {

constexpr unsigned kSweepFull = 0xffffffffu;
constexpr int kFarTile = 4;  // far-list entries per thread loaded before a compaction step writes

struct SweepArgs {
  const int4 *__restrict__ arc4;    // per vertex its first four arcs as (head, weight) pairs
  const int2 *__restrict__ arc_hw;  // per arc (head, weight)
  const int32_t *__restrict__ src;  // tids of this launch's sources, one per CTA
  int32_t ns, n, n_pad;
  int32_t delta;       // bucket width (distance units)
  int32_t max_rounds;  // bound on passes and on far-list splits (error word beyond it)
  int4 *rec;           // [ns][n_pad] sweep state, then the output records
  int32_t *hop;        // [ns][n_pad] hop layers out
  int32_t *order;      // [ns][n_pad] near list, then the Kahn queue
  int32_t *lcnt;       // [ns][2 (n_pad + 2)]: next near list, far list
  int32_t *maxhop;     // [ns] largest hop layer per source, or null
  int32_t *err;
  int32_t sort_shift;    // frontier lists are visited in order of v >> sort_shift ...
  int32_t sort_buckets;  // ... (n_pad - 1) >> sort_shift < sort_buckets <= kSortBuckets
  int32_t write_hop;     // 0: hop layers not written (the dependency pass reads the wave queue)
};

constexpr int kSortBuckets = 4096;  // shared-memory counters of the frontier ordering
constexpr int kSortMinLen = 1024;   // shorter lists are visited as they are

// Exclusive scan of c[0..len) in place (len <= kSortBuckets), whole CTA; red holds 33 ints.
template <int THREADS>
__device__ __forceinline__ void cta_exclusive_scan(int *c, int len, int *red) {
  constexpr int per = (kSortBuckets + THREADS - 1) / THREADS;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int b = tid * per;
  int local = 0;
#pragma unroll
  for (int k = 0; k < per; k++) local += (b + k < len) ? c[b + k] : 0;
  int x = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(kSweepFull, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) red[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int t = lane < THREADS / 32 ? red[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(kSweepFull, t, o);
      if (lane >= o) t += y;
    }
    red[lane] = t;  // inclusive warp totals
  }
  __syncthreads();
  int run = x - local + (warp > 0 ? red[warp - 1] : 0);
#pragma unroll
  for (int k = 0; k < per; k++)
    if (b + k < len) {
      const int v = c[b + k];
      c[b + k] = run;
      run += v;
    }
  __syncthreads();
}

// Frontier ordering: a list of vertices is rewritten into `out` grouped by v >> shift (a counting
// sort, CTA-wide), so that a pass visits the frontier in vertex-id order.  Near lists and Kahn
// waves are bands of the graph; in id order consecutive visits share record lines, and the rows
// above and below are visited soon after, while their lines are still in L1/L2.
template <int THREADS, class IN, class OUT>
__device__ __forceinline__ void order_frontier(const SweepArgs &a, IN in, int len, OUT out, int *hist, int *red) {
  const int tid = threadIdx.x;
  for (int i = tid; i < a.sort_buckets; i += THREADS) hist[i] = 0;
  __syncthreads();
  for (int i = tid; i < len; i += THREADS) atomicAdd(hist + (in(i) >> a.sort_shift), 1);
  __syncthreads();
  cta_exclusive_scan<THREADS>(hist, a.sort_buckets, red);
  for (int i = tid; i < len; i += THREADS) {
    const int v = in(i);
    out(atomicAdd(hist + (v >> a.sort_shift), 1)) = v;
  }
  __syncthreads();
}

// Shared state of one CTA's sweep.  Record field y while sweeping: > 0 the pass whose next list
// holds the vertex; < 0 the (negated, minus one) far-list split round whose far list holds it; 0
// neither.
struct SweepShared {
  int near_len, next_len, far_len, min_kept;
  int tail;  // Kahn queue length
};

__device__ __forceinline__ void relax(const RowView<int4> &rec, int u, int nd, int T, int pass, int far_tag,
                                      int32_t *next, int32_t *far, SweepShared &sh) {
  int4 &r = rec[u];
  if (nd >= r.x) return;  // a stale (larger) cached value only lets the atomic decide
  const int old = atomicMin(&r.x, nd);
  if (nd >= old) return;
  if (nd < T) {
    if (atomicExch(&r.y, pass) != pass) next[atomicAdd(&sh.next_len, 1)] = u;
  } else if (atomicExch(&r.y, far_tag) != far_tag) {
    far[atomicAdd(&sh.far_len, 1)] = u;
  }
}

// f(head, weight) for each arc of v in CSR order
template <class F>
__device__ __forceinline__ void for_arcs(const SweepArgs &a, int v, F &&f) {
  const int4 p0 = __ldg(a.arc4 + 2 * v), p1 = __ldg(a.arc4 + 2 * v + 1);
  if (p0.x >= 0) f(p0.x, p0.y);
  if (p0.z >= 0) f(p0.z, p0.w);
  if (p1.x >= 0) f(p1.x, p1.y);
  if (p1.z >= 0) {
    f(p1.z, p1.w);
  } else if (p1.z < -1) {  // more than four arcs: the rest are arc_hw[~p1.z, p1.w)
    for (int e = ~p1.z; e < p1.w; e++) {
      const int2 hw = __ldg(a.arc_hw + e);
      f(hw.x, hw.y);
    }
  }
}

// The first four arcs of v as (head, weight) pairs, head -1 where absent; *rest = the range of
// further arcs in arc_hw (empty for at most four arcs).  A visit loads all four heads' records
// before it issues any atomic: a load after an atomic cannot be moved above it (the addresses
// might alias), so checking the arcs one by one made each visit wait for four DRAM round trips.
struct Arcs4 {
  int h[4], w[4];
  int rest_b, rest_e;
};
__device__ __forceinline__ Arcs4 arcs4(const SweepArgs &a, int v) {
  const int4 p0 = __ldg(a.arc4 + 2 * v), p1 = __ldg(a.arc4 + 2 * v + 1);
  Arcs4 r;
  r.h[0] = p0.x; r.w[0] = p0.y;
  r.h[1] = p0.z; r.w[1] = p0.w;
  r.h[2] = p1.x; r.w[2] = p1.y;
  const bool more = p1.z < -1;
  r.h[3] = more ? -1 : p1.z;
  r.w[3] = p1.w;
  r.rest_b = more ? ~p1.z : 0;
  r.rest_e = more ? p1.w : 0;
  return r;
}

// MINB CTAs per SM: 1,536 threads per SM by default (40 registers a thread at 512); <512, 4>
// fits 2,048 threads per SM in 32 registers, for more scattered gathers in flight.
template <int THREADS, int MINB = 1536 / THREADS>
__global__ void __launch_bounds__(THREADS, MINB) k_sweep_rows(SweepArgs a) {
  __shared__ SweepShared sh;
  __shared__ int hist[kSortBuckets];
  __shared__ int red[33];
  const int slot = blockIdx.x;
  if (slot >= a.ns) return;
  const int s = a.src[slot];
  const int tid = threadIdx.x;
  const RowView<int4> rec{a.rec, slot, a.ns};
  const RowView<int32_t> hop{a.hop, slot, a.ns};
  int32_t *near = a.order + (size_t)slot * a.n_pad;
  int32_t *next = a.lcnt + (size_t)slot * 2 * (a.n_pad + 2);
  int32_t *far = next + (a.n_pad + 2);
  for (int v = tid; v < a.n; v += THREADS) rec[v] = make_int4(v == s ? 0 : INT_MAX, 0, 0, 0);
  if (tid == 0) {
    sh.near_len = 1;
    sh.next_len = 0;
    sh.far_len = 0;
    near[0] = s;
  }
  __syncthreads();
  const int delta = a.delta;
  int T = delta, pass = 0, round = 0;
  bool bound_hit = false;
  for (;;) {
    // passes over the near list until no distance below T changes
    for (;;) {
      const int len = sh.near_len;
      if (len == 0) break;
      if (++pass > a.max_rounds) {
        bound_hit = true;
        break;
      }
      const int far_tag = -1 - round;
      // a long list is visited in vertex-id order, staged in the hop row (free until the waves)
      const bool sorted = len >= kSortMinLen;
      if (sorted)
        order_frontier<THREADS>(
            a, [&](int i) { return near[i]; }, len, [&](int i) -> int32_t & { return hop[i]; }, hist, red);
      for (int i = tid; i < len; i += THREADS) {
        const int v = sorted ? hop[i] : near[i];
        const int dv = rec[v].x;
        const Arcs4 q = arcs4(a, v);
        int du[4];
#pragma unroll
        for (int k = 0; k < 4; k++) du[k] = q.h[k] >= 0 ? rec[q.h[k]].x : INT_MIN;
#pragma unroll
        for (int k = 0; k < 4; k++)
          if (dv + q.w[k] < du[k]) relax(rec, q.h[k], dv + q.w[k], T, pass, far_tag, next, far, sh);
        for (int e = q.rest_b; e < q.rest_e; e++) {
          const int2 hw = __ldg(a.arc_hw + e);
          relax(rec, hw.x, dv + hw.y, T, pass, far_tag, next, far, sh);
        }
      }
      __syncthreads();
      if (tid == 0) {
        sh.near_len = sh.next_len;
        sh.next_len = 0;
      }
      int32_t *t = near;
      near = next;
      next = t;
      __syncthreads();
    }
    if (bound_hit) break;
    // split the far list at the next threshold; a split that moves nothing (an empty bucket)
    // is repeated with the threshold just past the smallest distance left
    int T_old = T;
    T += delta;
    bool moved = false;
    while (!moved) {
      const int flen = sh.far_len;
      if (flen == 0 || ++round > a.max_rounds) break;
      const int tag = -1 - round;
      __syncthreads();  // every thread has read far_len
      if (tid == 0) {
        sh.far_len = 0;
        sh.min_kept = INT_MAX;
      }
      __syncthreads();
      for (int base = 0; base < flen; base += THREADS * kFarTile) {
        int u[kFarTile], du[kFarTile];
#pragma unroll
        for (int q = 0; q < kFarTile; q++) {
          const int i = base + q * THREADS + tid;
          u[q] = i < flen ? far[i] : -1;
        }
#pragma unroll
        for (int q = 0; q < kFarTile; q++) du[q] = u[q] >= 0 ? rec[u[q]].x : 0;
        __syncthreads();  // the tile is read before kept entries are written back in front of it
        int mn = INT_MAX;
#pragma unroll
        for (int q = 0; q < kFarTile; q++) {
          if (u[q] < 0 || du[q] < T_old) continue;  // settled in an earlier bucket: stale entry
          if (du[q] < T) {
            near[atomicAdd(&sh.near_len, 1)] = u[q];
          } else {
            far[atomicAdd(&sh.far_len, 1)] = u[q];
            rec[u[q]].y = tag;
            mn = min(mn, du[q]);
          }
        }
        mn = __reduce_min_sync(kSweepFull, mn);
        if ((tid & 31) == 0 && mn != INT_MAX) atomicMin(&sh.min_kept, mn);
        __syncthreads();
      }
      moved = sh.near_len > 0;
      if (!moved) {
        T_old = T;
        const int mk = sh.min_kept;
        if (mk != INT_MAX) T = max(T + delta, (mk / delta + 1) * delta);
      }
    }
    if (round > a.max_rounds) {
      bound_hit = true;
      break;
    }
    if (!moved) break;  // far list empty: every vertex is settled
  }
  if (bound_hit) {
    if (tid == 0) atomicCAS(a.err, ERR_NONE, ERR_SWEEP_BOUND);
    return;
  }
  // ---- counts and hop layers: in-degrees over the DAG (vertex order: neighbours' records are
  // mostly in the same or the next sectors), record (dist, count = [v == s], in-degree, successor
  // mask).  The same neighbour distances give the DAG successors (d[h] == d[v] + w): bit k of the
  // mask for the first four arcs, bit 4 when a further arc is one, so a wave visit touches only its
  // successors' records instead of gathering every neighbour's distance.
  for (int v = tid; v < a.n; v += THREADS) {
    const int dv = rec[v].x;
    const Arcs4 q = arcs4(a, v);
    int dh[4];
#pragma unroll
    for (int k = 0; k < 4; k++) dh[k] = q.h[k] >= 0 ? rec[q.h[k]].x : INT_MIN;
    int c = 0, m = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      c += q.h[k] >= 0 && dh[k] + q.w[k] == dv;
      m |= (q.h[k] >= 0 && dh[k] == dv + q.w[k]) << k;
    }
    for (int e = q.rest_b; e < q.rest_e; e++) {
      const int2 hw = __ldg(a.arc_hw + e);
      const int dx = rec[hw.x].x;
      c += dx + hw.y == dv;
      m |= (dx == dv + hw.y) << 4;
    }
    rec[v] = make_int4(dv, v == s ? 1 : 0, c, m);
  }
  int32_t *queue = a.order + (size_t)slot * a.n_pad;
  if (tid == 0) {
    queue[0] = s;
    sh.tail = 1;
  }
  __syncthreads();
  int L = 0, b = 0, e = 1;
  int32_t *wave = a.lcnt + (size_t)slot * 2 * (a.n_pad + 2);  // the next-list row is free now
  // The queue is the dependency pass's level queue: wave L (hop layer L) is [wstart[L],
  // wstart[L + 1]) of it, the starts kept in the far-list row (free now), so that pass needs no
  // layer sort of its own.
  int32_t *wstart = wave + (a.n_pad + 2);
  while (b < e) {
    if (tid == 0) wstart[L] = b;
    // a long wave is visited in vertex-id order, staged in the next-list row and written back
    // into the queue in that order (each thread rewrites the entries it visits)
    const bool sorted = e - b >= kSortMinLen;
    if (sorted)
      order_frontier<THREADS>(
          a, [&](int i) { return queue[b + i]; }, e - b, [&](int i) -> int32_t & { return wave[i]; }, hist, red);
    for (int i = b + tid; i < e; i += THREADS) {
      const int v = sorted ? wave[i - b] : queue[i];
      if (sorted) queue[i] = v;
      const int4 r = rec[v];
      if (a.write_hop) hop[v] = L;  // a scattered 4-byte write: skipped when no one reads it
      auto push = [&](int h) {
        int4 &rh = rec[h];
        atomicAdd(&rh.y, r.y);                                            // 32-bit wrapping, as count_t
        if (atomicSub(&rh.z, 1) == 1) queue[atomicAdd(&sh.tail, 1)] = h;  // its last predecessor
      };
      const Arcs4 q = arcs4(a, v);
#pragma unroll
      for (int k = 0; k < 4; k++)
        if ((r.w >> k) & 1) push(q.h[k]);
      if (r.w & 16)
        for (int x = q.rest_b; x < q.rest_e; x++) {
          const int2 hw = __ldg(a.arc_hw + x);
          if (rec[hw.x].x == r.x + hw.y) push(hw.x);
        }
    }
    __syncthreads();
    b = e;
    e = sh.tail;
    L++;
    __syncthreads();  // every thread has read the tail before the next wave moves it
  }
  if (e != a.n) {  // a vertex the sweep did not reach (the index build rejects disconnected graphs)
    if (tid == 0) atomicCAS(a.err, ERR_NONE, ERR_DISCONNECTED);
    return;
  }
  if (tid == 0) {
    wstart[L] = e;                    // end of the last wave
    if (a.maxhop) a.maxhop[slot] = L - 1;  // waves 0 .. L-1 hold vertices
  }
}

// ------------------------------------------------------------------------------- plain path
// One source swept by the whole GPU (the plain one-source-per-launch path): the same near-far
// buckets and Kahn waves, every CTA of a cooperative launch working on one shared frontier.  The
// lists' lengths live in a control block in global memory and the steps are separated by a grid
// barrier.  Data written by other CTAs is read through L2 (__ldcg): their atomics do not update
// this SM's L1.
struct GridCtl {
  unsigned arrive, gen;  // grid barrier: arrivals, generation
  int abort;             // a barrier wait ran out: every CTA leaves at its next barrier
  int near_len, next_len, far_len, keep_len, min_kept, tail;
};

constexpr long long kGridSpinLimit = 1ll << 24;  // ~2 s of 64-ns sleeps per barrier wait

// Barrier over all CTAs of a cooperative launch with a bounded wait; false when the grid aborts.
__device__ __forceinline__ bool grid_sync(GridCtl *c, unsigned &gen, int32_t *err) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    __threadfence();
    if (atomicAdd(&c->arrive, 1u) == gridDim.x - 1) {
      c->arrive = 0;
      __threadfence();
      atomicExch(&c->gen, gen + 1);
    } else {
      long long spins = 0;
      while (*(volatile unsigned *)&c->gen == gen) {
        if (*(volatile int *)&c->abort || ++spins > kGridSpinLimit) {
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
      if (!ok) {
        atomicExch(&c->abort, 1);
        atomicCAS(err, ERR_NONE, ERR_SWEEP_BOUND);
      }
    }
    gen++;
    __threadfence();
    s_ok = ok && !*(volatile int *)&c->abort;
  }
  __syncthreads();
  return s_ok;
}

__device__ __forceinline__ int ldcg(const int *p) { return __ldcg(p); }

__device__ __forceinline__ void relax_grid(int4 *rec, int u, int nd, int T, int pass, int far_tag, int32_t *next,
                                           int32_t *far, GridCtl *c) {
  int *r = reinterpret_cast<int *>(rec + u);
  if (nd >= ldcg(r)) return;
  const int old = atomicMin(r, nd);
  if (nd >= old) return;
  if (nd < T) {
    if (atomicExch(r + 1, pass) != pass) next[atomicAdd(&c->next_len, 1)] = u;
  } else if (atomicExch(r + 1, far_tag) != far_tag) {
    far[atomicAdd(&c->far_len, 1)] = u;
  }
}

// rec/hop/order/lcnt: the single slot of a one-source buffer (plain rows); far lists ping-pong
// between the second half of the layer-counter row and the hop row (written only by the waves)
__global__ void __launch_bounds__(1024, 1) k_sweep_rows_grid(SweepArgs a, GridCtl *c) {
  const int s = a.src[0];
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
  int4 *rec = a.rec;
  int32_t *near = a.order, *next = a.lcnt, *far = a.lcnt + (a.n_pad + 2), *far2 = a.hop;
  unsigned gen = 0;
  for (int v = gt; v < a.n; v += gs) __stcg(rec + v, make_int4(v == s ? 0 : INT_MAX, 0, 0, 0));
  if (gt == 0) {
    near[0] = s;
    c->near_len = 1;
  }
  if (!grid_sync(c, gen, a.err)) return;
  const int delta = a.delta;
  int T = delta, pass = 0, round = 0;
  for (;;) {
    for (;;) {
      const int len = ldcg(&c->near_len);
      if (len == 0) break;
      if (++pass > a.max_rounds) {
        if (gt == 0) atomicCAS(a.err, ERR_NONE, ERR_SWEEP_BOUND);
        return;  // uniform: every CTA read the same length and counts the same passes
      }
      const int far_tag = -1 - round;
      for (int i = gt; i < len; i += gs) {
        const int v = ldcg(near + i);
        const int dv = ldcg(reinterpret_cast<const int *>(rec + v));
        const Arcs4 q = arcs4(a, v);
        int du[4];
#pragma unroll
        for (int k = 0; k < 4; k++) du[k] = q.h[k] >= 0 ? ldcg(reinterpret_cast<const int *>(rec + q.h[k])) : INT_MIN;
#pragma unroll
        for (int k = 0; k < 4; k++)
          if (dv + q.w[k] < du[k]) relax_grid(rec, q.h[k], dv + q.w[k], T, pass, far_tag, next, far, c);
        for (int e = q.rest_b; e < q.rest_e; e++) {
          const int2 hw = __ldg(a.arc_hw + e);
          relax_grid(rec, hw.x, dv + hw.y, T, pass, far_tag, next, far, c);
        }
      }
      if (!grid_sync(c, gen, a.err)) return;
      if (gt == 0) {
        c->near_len = c->next_len;
        c->next_len = 0;
      }
      int32_t *t = near;
      near = next;
      next = t;
      if (!grid_sync(c, gen, a.err)) return;
    }
    int T_old = T;
    T += delta;
    bool moved = false;
    while (!moved) {
      const int flen = ldcg(&c->far_len);
      if (flen == 0) break;
      if (++round > a.max_rounds) {
        if (gt == 0) atomicCAS(a.err, ERR_NONE, ERR_SWEEP_BOUND);
        return;
      }
      const int tag = -1 - round;
      if (gt == 0) {
        c->keep_len = 0;
        c->min_kept = INT_MAX;
      }
      if (!grid_sync(c, gen, a.err)) return;
      for (int i = gt; i < flen + (gs - flen % gs) % gs; i += gs) {  // whole warps reach the reduction
        int mn = INT_MAX;
        if (i < flen) {
          const int u = ldcg(far + i);
          const int du = ldcg(reinterpret_cast<const int *>(rec + u));
          if (du >= T_old) {
            if (du < T) {
              near[atomicAdd(&c->near_len, 1)] = u;
            } else {
              far2[atomicAdd(&c->keep_len, 1)] = u;
              reinterpret_cast<int *>(rec + u)[1] = tag;
              mn = du;
            }
          }
        }
        mn = __reduce_min_sync(kSweepFull, mn);
        if ((threadIdx.x & 31) == 0 && mn != INT_MAX) atomicMin(&c->min_kept, mn);
      }
      if (!grid_sync(c, gen, a.err)) return;
      if (gt == 0) c->far_len = c->keep_len;
      int32_t *t = far;
      far = far2;
      far2 = t;
      moved = ldcg(&c->near_len) > 0;
      const int mk = ldcg(&c->min_kept);
      if (!grid_sync(c, gen, a.err)) return;
      if (!moved) {
        T_old = T;
        if (mk != INT_MAX) T = max(T + delta, (mk / delta + 1) * delta);
      }
    }
    if (!moved) break;
  }
  // counts and hop layers (Kahn waves), as in k_sweep_rows
  for (int v = gt; v < a.n; v += gs) {
    const int dv = ldcg(reinterpret_cast<const int *>(rec + v));
    int cnt = 0;
    for_arcs(a, v, [&](int h, int w) { cnt += ldcg(reinterpret_cast<const int *>(rec + h)) + w == dv; });
    __stcg(rec + v, make_int4(dv, v == s ? 1 : 0, cnt, 0));
  }
  int32_t *queue = a.order;
  if (gt == 0) {
    queue[0] = s;
    c->tail = 1;
  }
  if (!grid_sync(c, gen, a.err)) return;
  int L = 0, b = 0, e = 1;
  while (b < e) {
    for (int i = b + gt; i < e; i += gs) {
      const int v = ldcg(queue + i);
      const int dv = ldcg(reinterpret_cast<const int *>(rec + v));
      const int sv = ldcg(reinterpret_cast<const int *>(rec + v) + 1);
      a.hop[v] = L;
      auto push = [&](int h) {
        int *rh = reinterpret_cast<int *>(rec + h);
        atomicAdd(rh + 1, sv);
        if (atomicSub(rh + 2, 1) == 1) queue[atomicAdd(&c->tail, 1)] = h;
      };
      const Arcs4 q = arcs4(a, v);
      int dh[4];
#pragma unroll
      for (int k = 0; k < 4; k++) dh[k] = q.h[k] >= 0 ? ldcg(reinterpret_cast<const int *>(rec + q.h[k])) : INT_MIN;
#pragma unroll
      for (int k = 0; k < 4; k++)
        if (dh[k] == dv + q.w[k]) push(q.h[k]);
      for (int x = q.rest_b; x < q.rest_e; x++) {
        const int2 hw = __ldg(a.arc_hw + x);
        if (ldcg(reinterpret_cast<const int *>(rec + hw.x)) == dv + hw.y) push(hw.x);
      }
    }
    if (!grid_sync(c, gen, a.err)) return;
    b = e;
    e = ldcg(&c->tail);
    L++;
    if (!grid_sync(c, gen, a.err)) return;
  }
  if (e != a.n && gt == 0) atomicCAS(a.err, ERR_NONE, ERR_DISCONNECTED);
}

}  // namespace

// Bucket width: tuned, else twice the mean arc weight.  Capped so that thresholds stay far from
// int32 overflow (distances are below 999,999,999, the graph reader's bound on total weight).
int32_t sweep_delta(const Handle &h, const DeviceState *d) {
  const int32_t w = h.tuning.sweep_delta > 0 ? h.tuning.sweep_delta : d->sweep_delta_auto;
  return std::min<int32_t>(std::max<int32_t>(1, w), 1 << 28);
}

void launch_sweep_rows(const Handle &h, DeviceState *d, int4 *rec, int32_t *hop, int32_t *order, int32_t *lcnt,
                       int32_t *maxhop, const int32_t *src, int32_t ns, cudaStream_t st, bool write_hop) {
  SweepArgs a{};
  a.arc4 = d->arc4;
  a.arc_hw = d->arc_hw;
  a.src = src;
  a.ns = ns;
  a.n = d->n;
  a.n_pad = d->n_pad;
  a.delta = sweep_delta(h, d);
  // passes: at most one per vertex settled plus one per bucket; splits: one per bucket
  a.max_rounds = 2 * d->n + 16;
  a.rec = rec;
  a.hop = hop;
  a.order = order;
  a.lcnt = lcnt;
  a.maxhop = maxhop;
  a.err = d->err;
  a.write_hop = write_hop ? 1 : 0;
  a.sort_shift = 0;
  while (((d->n_pad - 1) >> a.sort_shift) >= kSortBuckets) a.sort_shift++;
  a.sort_buckets = ((d->n_pad - 1) >> a.sort_shift) + 1;
  if (h.tuning.sweep_threads == 256) k_sweep_rows<256><<<ns, 256, 0, st>>>(a);
  else if (h.tuning.sweep_threads == 1024) k_sweep_rows<1024><<<ns, 1024, 0, st>>>(a);
  else if (h.tuning.sweep_threads == 2048) k_sweep_rows<512, 4><<<ns, 512, 0, st>>>(a);  // 4 x 512 per SM
  else k_sweep_rows<512><<<ns, 512, 0, st>>>(a);
  CK(cudaGetLastError());
}

void launch_sweep_rows_grid(const Handle &h, DeviceState *d, int4 *rec, int32_t *hop, int32_t *order, int32_t *lcnt,
                            const int32_t *src, cudaStream_t st) {
  static_assert(sizeof(GridCtl) <= kGridCtlBytes, "grid control block");
  SweepArgs a{};
  a.arc4 = d->arc4;
  a.arc_hw = d->arc_hw;
  a.src = src;
  a.ns = 1;
  a.n = d->n;
  a.n_pad = d->n_pad;
  a.delta = sweep_delta(h, d);
  a.max_rounds = 2 * d->n + 16;
  a.rec = rec;
  a.hop = hop;
  a.order = order;
  a.lcnt = lcnt;
  a.maxhop = nullptr;
  a.err = d->err;
  // one 1,024-thread CTA per SM, all resident at once (the barrier waits on every one of them;
  // fewer, larger CTAs make each barrier cheaper)
  int per_sm = 0, sms = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep_rows_grid, 1024, 0));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d->device));
  if (per_sm < 1) throw Error(QBC_EDEVICE, "plain sweep kernel does not fit an SM");
  GridCtl *c = reinterpret_cast<GridCtl *>(d->grid_ctl);
  CK(cudaMemsetAsync(c, 0, sizeof(GridCtl), st));
  void *args[] = {&a, &c};
  CK(cudaLaunchCooperativeKernel((const void *)k_sweep_rows_grid, dim3((unsigned)sms), dim3(1024), args, 0, st));
}

}  // namespace qbc

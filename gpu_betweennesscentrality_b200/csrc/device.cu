// device.cu -- B200 (sm_100a) kernels and drivers of libqbc_b200.
//
// Per source s the reference runs, inside one CTA (MHLQBC.cu:237-475): LCA of s with every tree
// node, a dist/count/hop label scan per target, SP-DAG arcs with layer counts, a layer queue and a
// layered FP64 backprop.  Here the same quantities come from three kernels:
//
//   k_label_scan   (K1+K2)  G sources x a range of targets per CTA.  The G source rows (label
//                  distances, ancestor ids and subtree ends) sit in shared memory; each target row
//                  is read once from HBM/L2 per G sources (16-byte vector loads) and reused by all
//                  of them.  LCA depth = binary search of the target id in the source's nested
//                  ancestor intervals (DFS preorder), replacing the Euler-tour RMQ gathers.  The
//                  scan tracks min + tie flag; path counts and hops are gathered only at the
//                  minimising entries, so the hot loop reads 4 B per entry instead of 12.
//   k_dependency   (K3-K5)  one CTA per source: layer histogram with shared-memory
//                  atomics, block scan, scatter into a level queue, then a pull-form backprop
//                  (each vertex sums over its own DAG out-arcs, no FP64 atomics on delta) and
//                  an FP64 red into BC.
//   k_kahn_dependency (QBC) distance-only rows from the H2H index; sigma and topological waves
//                  by a device Kahn pass (QBC.cu:485-555 ran it on the host), then the same backprop.
//
// Chunks of sources run through one scratch buffer; the label scan and the dependency pass of a
// chunk run back to back on one stream (concurrent on two streams they thrash each other's caches:
// measured ~2x slower in total).
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <climits>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "device_state.h"

namespace qbc {

constexpr int kInfDist = 999999999;  // unreached label entry (TreeDecomp INF, TreeDecomp.h:58)
constexpr int kLayerCap = 4094;  // shared-memory layer counters; deeper DAGs use global memory
constexpr int kHopBatch = 8;   // hop loads in flight per thread in the dependency pass's layer sort
constexpr unsigned kFull = 0xffffffffu;

// ------------------------------------------------------------------------------- K1 + K2
struct LabelArgs {
  // label distances, shifted left by `bits` when the packed-key kernel applies (one array serves
  // both kernels: the general one shifts back as it loads)
  const int32_t *__restrict__ dis;
  const int32_t *__restrict__ dis_sh;  // the same array (packed kernel: keys and target rows pre-shifted)
  const int2 *__restrict__ ch;
  const int64_t *__restrict__ lab_off;
  const int32_t *__restrict__ depth;
  const int32_t *__restrict__ send;
  const int32_t *__restrict__ src;  // tids of this chunk's sources
  int32_t ns, n, n_pad, stride, split;
  int4 *__restrict__ out_rec;     // [ns][n_pad] records (dist, count bits, delta as f64 = 0)
  int32_t *__restrict__ out_hop;  // [ns][n_pad]
  int32_t *__restrict__ maxhop;   // [ns] largest hop layer per source (atomicMax), or null
  // per slot of the launch: the source's ancestor ids (root first), then their subtree ends, each
  // row `src_stride` ints (k_src_rows writes them from the parent links before the scan)
  const int32_t *__restrict__ src_rows;
  int32_t src_stride;
  int32_t bits;                      // index bits of the packed keys (packed kernel)
  int32_t pass_lo;                   // multi-pass packed kernel: first row entry of this pass's tile
  int32_t multipass;                 // launcher only: rows longer than the tile take several passes
                                     // (kernel variant MP, state in out_rec between passes)
  int32_t row_words;                 // lane-pair kernel: words per target-row buffer
  int32_t *err;                      // device error word (packed kernel's bounded waits)
  uint32_t wait_spins;               // attempts of a row-copy wait before it is reported
};

// largest J with lo[J] <= t < hi[J] (entry 0 is the root and always holds), returned as J+1
__device__ __forceinline__ int lca_depth(const int32_t *lo, const int32_t *hi, int hs, int t) {
  int l = 0, h = hs;
  while (h - l > 1) {
    int mid = (l + h) >> 1;
    bool p = (lo[mid] <= t) && (t < hi[mid]);
    l = p ? mid : l;
    h = p ? h : mid;
  }
  return l + 1;
}

template <int K, bool COUNTS>
__global__ void __launch_bounds__(256, 1) k_label_scan(LabelArgs a) {
  constexpr int G = 32 / K;
  extern __shared__ int4 smem4[];
  int32_t *sm = reinterpret_cast<int32_t *>(smem4);
  const int S = a.stride;
  int32_t *s_dis = sm;
  int32_t *s_lo = s_dis + G * S;
  int32_t *s_hi = s_lo + G * S;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  int32_t *tbuf = s_hi + G * S + warp * S;
  __shared__ int32_t s_tid[G], s_h[G];
  __shared__ int64_t s_off[G];

  const int first = blockIdx.y * G;
  if (first >= a.ns) return;
  const int gcount = min(G, a.ns - first);
  if (threadIdx.x < G) {
    int i = threadIdx.x;
    int s = i < gcount ? a.src[first + i] : 0;
    s_tid[i] = s;
    s_h[i] = i < gcount ? a.depth[s] : 0;
    s_off[i] = a.lab_off[s];
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < G * S; idx += blockDim.x) {
    const int i = idx / S, j = idx - i * S;
    int vd = 0x3fffffff, vlo = INT_MAX, vhi = -1;
    if (i < gcount && j < s_h[i]) {
      const int32_t *row = a.src_rows + (size_t)(first + i) * 2 * a.src_stride;
      vd = (int)((uint32_t)a.dis[s_off[i] + j] >> a.bits);
      vlo = row[j];
      vhi = row[a.src_stride + j];
    }
    s_dis[idx] = vd;
    s_lo[idx] = vlo;
    s_hi[idx] = vhi;
  }
  __syncthreads();

  const int si = lane / K, kq = lane % K;
  const bool have = si < gcount;
  const int hs = have ? s_h[si] : 1;
  const int64_t soff = s_off[si];
  const int32_t *srow = s_dis + si * S;
  const int32_t *slo = s_lo + si * S;
  const int32_t *shi = s_hi + si * S;

  const int nchunk = a.n_pad >> 3;
  const int cbeg = (int)((int64_t)nchunk * blockIdx.x / a.split);
  const int cend = (int)((int64_t)nchunk * (blockIdx.x + 1) / a.split);
  for (int c = cbeg + warp; c < cend; c += nwarps) {
    const int t0 = c << 3;
    int rd[8], rc[8], rh[8];
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const int t = t0 + k;
      rd[k] = 0; rc[k] = 0; rh[k] = 0;
      if (t < a.n) {
        const int64_t toff = a.lab_off[t];
        const int hl = have ? lca_depth(slo, shi, hs, t) : 0;
        const int H = __reduce_max_sync(kFull, hl);
        for (int j = lane * 4; j < H; j += 128) {
          int4 x = __ldg(reinterpret_cast<const int4 *>(a.dis + toff + j));
          x.x = (int)((uint32_t)x.x >> a.bits);
          x.y = (int)((uint32_t)x.y >> a.bits);
          x.z = (int)((uint32_t)x.z >> a.bits);
          x.w = (int)((uint32_t)x.w >> a.bits);
          *reinterpret_cast<int4 *>(tbuf + j) = x;
        }
        __syncwarp();
        if (K == 1) {
          int m = INT_MAX, jm = 0;
          bool tie = false;
          for (int j = 0; j < hl; j += 4) {
            const int4 x = *reinterpret_cast<const int4 *>(srow + j);
            const int4 y = *reinterpret_cast<const int4 *>(tbuf + j);
            int v0 = x.x + y.x, v1 = x.y + y.y, v2 = x.z + y.z, v3 = x.w + y.w;
            v1 = (j + 1 < hl) ? v1 : INT_MAX;
            v2 = (j + 2 < hl) ? v2 : INT_MAX;
            v3 = (j + 3 < hl) ? v3 : INT_MAX;
#define QBC_STEP(v, jj)              \
  if (v < m) {                       \
    m = v; jm = jj; tie = false;     \
  } else if (v == m) {               \
    tie = true;                      \
  }
            QBC_STEP(v0, j) QBC_STEP(v1, j + 1) QBC_STEP(v2, j + 2) QBC_STEP(v3, j + 3)
#undef QBC_STEP
          }
          rd[k] = m;
          if (COUNTS && have) {
            if (!tie) {
              const int2 cs = __ldg(a.ch + soff + jm), ct = __ldg(a.ch + toff + jm);
              rc[k] = (int)((unsigned)cs.x * (unsigned)ct.x);
              rh[k] = cs.y + ct.y;
            } else {
              unsigned cc = 0;
              int hh = 0;
              for (int j = 0; j < hl; j++) {
                if (srow[j] + tbuf[j] == m) {
                  const int2 cs = __ldg(a.ch + soff + j), ct = __ldg(a.ch + toff + j);
                  cc += (unsigned)cs.x * (unsigned)ct.x;
                  hh = max(hh, cs.y + ct.y);
                }
              }
              rc[k] = (int)cc;
              rh[k] = hh;
            }
          }
        } else {
          int m = INT_MAX;
          for (int j = kq * 4; j < hl; j += 4 * K) {
            const int4 x = *reinterpret_cast<const int4 *>(srow + j);
            const int4 y = *reinterpret_cast<const int4 *>(tbuf + j);
            int v0 = x.x + y.x, v1 = x.y + y.y, v2 = x.z + y.z, v3 = x.w + y.w;
            v1 = (j + 1 < hl) ? v1 : INT_MAX;
            v2 = (j + 2 < hl) ? v2 : INT_MAX;
            v3 = (j + 3 < hl) ? v3 : INT_MAX;
            m = min(m, min(min(v0, v1), min(v2, v3)));
          }
#pragma unroll
          for (int o = K / 2; o >= 1; o >>= 1) m = min(m, __shfl_xor_sync(kFull, m, o));
          rd[k] = m;
          if (COUNTS) {
            unsigned cc = 0;
            int hh = 0;
            for (int j = kq * 4; j < hl; j += 4 * K) {
#pragma unroll
              for (int q = 0; q < 4; q++) {
                if (j + q < hl && srow[j + q] + tbuf[j + q] == m) {
                  const int2 cs = __ldg(a.ch + soff + j + q), ct = __ldg(a.ch + toff + j + q);
                  cc += (unsigned)cs.x * (unsigned)ct.x;
                  hh = max(hh, cs.y + ct.y);
                }
              }
            }
#pragma unroll
            for (int o = K / 2; o >= 1; o >>= 1) {
              cc += __shfl_xor_sync(kFull, cc, o);
              hh = max(hh, __shfl_xor_sync(kFull, hh, o));
            }
            rc[k] = (int)cc;
            rh[k] = hh;
          }
        }
        __syncwarp();
      }
    }
    if (have && kq == 0) {
      const size_t slot = (size_t)(first + si);
      if (COUNTS && a.maxhop) {
        int mh = 0;
#pragma unroll
        for (int k = 0; k < 8; k++) mh = max(mh, rh[k]);
        atomicMax(a.maxhop + slot, mh);
      }
      int4 *od = a.out_rec + blk((int)slot, t0, a.ns);
#pragma unroll
      for (int k = 0; k < 8; k++) od[k] = make_int4(rd[k], rc[k], 0, 0);
      if (COUNTS) {
        int4 *oh = reinterpret_cast<int4 *>(a.out_hop + blk((int)slot, t0, a.ns));
        oh[0] = make_int4(rh[0], rh[1], rh[2], rh[3]);
        oh[1] = make_int4(rh[4], rh[5], rh[6], rh[7]);
      }
    }
  }
}

// Packed-key label scan (K=1, 32 sources per CTA).  Each source entry is stored as the key
// (dist << B) | j and target rows are read from a copy of the label distances pre-shifted by B
// (dis_sh), so one add gives (d_s+d_t, j) and a running unsigned min yields the distance and the
// smallest minimising j at
// once; a second min over key ^ (2^B-1) yields the largest minimising j, so a tie exists iff the two
// differ.  Valid when every row has at most 2^B entries and 2*max_label < 2^(32-B) - 1 (checked
// on the host).  Target rows arrive by 1-D TMA bulk copies (cp.async.bulk, no multicast) into two
// per-warp shared buffers, the row of the next target in flight while the current one is scanned;
// ancestor intervals come from the L1-cached global rows anc/aend.
__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void bulk_row_to_smem(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

// Bounded wait of a whole warp for the phase with the given parity: true once every lane has seen
// the phase complete (each lane's own try_wait is its acquire of the copied row), false when
// `spins` attempts ran out.  Warp-uniform, so the lanes leave the wait together.
constexpr uint32_t kRowWaitSpins = 1u << 22;   // a row copy that takes longer is reported
constexpr uint32_t kDrainWaitSpins = 1u << 28;  // copies still in flight when a CTA gives up
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t spins = kRowWaitSpins) {
  for (uint32_t it = 0; it < spins; it++) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    if (__all_sync(kFull, ok)) return true;
  }
  return false;
}

constexpr int kRowBuffers = 2;  // per-warp target-row buffers: 1 copy in flight
constexpr int kStageInt4 = 32 * 5 + 32 * 3;  // per-warp output staging (int4s)

// Shared memory of the packed kernel with `warps` warps and row stride S (entries): 32 source key
// rows, kRowBuffers target rows per warp, per-warp output staging.
__host__ __device__ constexpr size_t packed_smem(int warps, int S) {
  return (size_t)32 * S * 4 + (size_t)warps * (kRowBuffers * (size_t)S * 4 + kStageInt4 * 16);
}

// Rows are held in shared memory up to S entries (S = the padded tree height when it fits);
// entries j >= S of a scan (taller trees) are read from global memory, 4 at a time.
template <bool COUNTS, int WARPS, bool MP>
__global__ void __launch_bounds__(WARPS * 32, 1) k_label_scan_packed(LabelArgs a) {
  constexpr int G = 32;
  extern __shared__ int4 smem4[];
  uint32_t *s_key = reinterpret_cast<uint32_t *>(smem4);
  const int S = a.stride;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  int32_t *tb0 = reinterpret_cast<int32_t *>(s_key + G * S) + warp * kRowBuffers * S;
  int4 *sdc = reinterpret_cast<int4 *>(s_key + G * S + nwarps * kRowBuffers * S) + warp * kStageInt4;
  int4 *shp = sdc + 32 * 5;
  int2 *sdc2 = reinterpret_cast<int2 *>(sdc) + lane * 10;  // this lane's 8 (dist, count) pairs
  int32_t *shp1 = reinterpret_cast<int32_t *>(shp) + lane * 12;  // this lane's 8 hop layers
  __shared__ int32_t s_h[G];
  __shared__ int64_t s_off[G];
  __shared__ __align__(8) uint64_t s_bar[WARPS][kRowBuffers];
  const int first = blockIdx.y * G;
  if (first >= a.ns) return;
  const int gcount = min(G, a.ns - first);
  const uint32_t B = (uint32_t)a.bits, mask = (1u << B) - 1u;
  __shared__ int32_t s_hmax;
  if (threadIdx.x < G) {
    const int i = threadIdx.x;
    const int s = i < gcount ? a.src[first + i] : 0;
    s_h[i] = i < gcount ? a.depth[s] : 0;
    s_off[i] = a.lab_off[s];
    const int hm32 = __reduce_max_sync(kFull, s_h[i]);
    if (i == 0) s_hmax = hm32;
  }
  if (lane == 0)
    for (int b = 0; b < kRowBuffers; b++) mbar_init(&s_bar[warp][b], 1);
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  __syncthreads();
  // Multi-pass: this pass scans row entries [P0, P0 + S); a CTA whose rows all ended in an earlier
  // pass has nothing left, and the pass that reaches its deepest row finalises its pairs.
  const int P0 = MP ? a.pass_lo : 0;
  if (MP && P0 > 0 && s_hmax <= P0) return;
  const bool fin = !MP || s_hmax <= P0 + S;
  for (int idx = threadIdx.x; idx < G * S; idx += blockDim.x) {
    const int i = idx / S, jj = idx - i * S, j = P0 + jj;
    uint32_t key = 0xffffffffu;
    if (i < gcount && j < s_h[i]) key = (uint32_t)a.dis_sh[s_off[i] + j] | (uint32_t)j;
    s_key[idx] = key;
  }
  __syncthreads();

  const bool have = lane < gcount;
  const int hs = have ? s_h[lane] : 1;
  const int64_t soff = s_off[lane];
  const uint32_t *srow = s_key + lane * S;
  const int32_t *lo = a.src_rows + (size_t)(first + (have ? lane : 0)) * 2 * a.src_stride;
  const int32_t *hi = lo + a.src_stride;
  const int nsteps = 32 - __clz(hs);
  int mh = 0;
  bool failed = false;

  const int nchunk = a.n_pad >> 3;
  const int cbeg = (int)((int64_t)nchunk * blockIdx.x / a.split);
  const int cend = (int)((int64_t)nchunk * (blockIdx.x + 1) / a.split);
  uint32_t issued = 0, done = 0;
  int next_c = cbeg + warp, next_k = 0;
  auto issue_next = [&]() {
    if (next_c >= cend) return;
    const int t = next_c * 8 + next_k;
    if (t >= a.n) { next_c = cend; return; }
    if (lane == 0) {
      const uint32_t b = issued % kRowBuffers;
      // entries [P0, P0 + S) of the row (S and P0 are multiples of 4: 16-byte aligned); a row that
      // ends before P0 is not scanned in this pass, 16 bytes of its start are copied instead
      const int rem = ((a.depth[t] + 3) & ~3) - P0;
      const int64_t src = a.lab_off[t] + (rem > 0 ? P0 : 0);
      const uint32_t bytes = (uint32_t)((rem > 0 ? min(rem, S) : 4) * 4);
      bulk_row_to_smem(tb0 + b * S, a.dis_sh + src, bytes, &s_bar[warp][b]);
    }
    issued++;
    if (++next_k == 8) { next_k = 0; next_c += nwarps; }
  };
  for (int q = 0; q < kRowBuffers - 1; q++) issue_next();

  for (int c = cbeg + warp; c < cend && !failed; c += nwarps) {
    const int t0 = c << 3;
    // deepest ancestor interval of this lane's source holding t0 (binary search)
    int J = 0;
    {
      int h = have ? hs : 1;
      for (int it = 0; it < nsteps; it++) {
        if (h - J > 1) {
          const int mid = (J + h) >> 1;
          const bool p = (__ldg(lo + mid) <= t0) && (t0 < __ldg(hi + mid));
          J = p ? mid : J;
          h = p ? h : mid;
        }
      }
    }
    int hiJ = have ? __ldg(hi + J) : 0x7fffffff;
    int loN = (have && J + 1 < hs) ? __ldg(lo + J + 1) : 0x7fffffff;
    uint32_t pending = 0;  // targets whose counts are gathered after the chunk
    const int kend = min(8, a.n - t0);
    if (MP && P0 > 0) {  // (m1, m2) of the earlier passes, kept in the output records
      const int4 *grec = a.out_rec + blk(first, t0, a.ns);
      int2 *sdc_all = reinterpret_cast<int2 *>(sdc);
      for (int p = lane; p < gcount * 8; p += 32) {
        const int4 x = grec[p];
        sdc_all[(p >> 3) * 10 + (p & 7)] = make_int2(x.x, x.y);
      }
      __syncwarp();
    }
    for (int k = 0; k < kend; k++) {
      const int t = t0 + k;
      // advance the interval: targets grow, so t leaves intervals on the right and enters a deeper
      // one only at its first id (one ancestor interval starts at each preorder id)
      if (have && k > 0) {
        if (t >= hiJ) {
          do { J--; hiJ = __ldg(hi + J); } while (t >= hiJ);
          loN = __ldg(lo + J + 1);
        } else if (t == loN) {
          J++;
          hiJ = __ldg(hi + J);
          loN = (J + 1 < hs) ? __ldg(lo + J + 1) : 0x7fffffff;
        }
      }
      issue_next();
      const uint32_t b = done % kRowBuffers;
      if (!mbar_wait(&s_bar[warp][b], (done / kRowBuffers) & 1, a.wait_spins)) {
        failed = true;
        break;
      }
      done++;
      const int32_t *tbuf = tb0 + b * S;
      const int hl = have ? J + 1 : 0;
      const int hm = max(0, min(hl, P0 + S) - P0);  // entries of this pass held in shared memory
      uint32_t m1 = 0xffffffffu, m2 = 0xffffffffu, n1 = 0xffffffffu, n2 = 0xffffffffu;
      if (MP && P0 > 0 && have) {
        const int2 st = sdc2[k];
        m1 = (uint32_t)st.x;
        m2 = (uint32_t)st.y;
      }
      const int full8 = hm & ~7;
      int j = 0;
      for (; j < full8; j += 8) {
        const uint4 x = *reinterpret_cast<const uint4 *>(srow + j);
        const uint4 y = *reinterpret_cast<const uint4 *>(tbuf + j);
        const uint4 x2 = *reinterpret_cast<const uint4 *>(srow + j + 4);
        const uint4 y2 = *reinterpret_cast<const uint4 *>(tbuf + j + 4);
        const uint32_t v0 = x.x + y.x, v1 = x.y + y.y, v2 = x.z + y.z, v3 = x.w + y.w;
        const uint32_t u0 = x2.x + y2.x, u1 = x2.y + y2.y, u2 = x2.z + y2.z, u3 = x2.w + y2.w;
        m1 = __vimin3_u32(m1, v0, v1);
        n1 = __vimin3_u32(n1, u0, u1);
        m1 = __vimin3_u32(m1, v2, v3);
        n1 = __vimin3_u32(n1, u2, u3);
        m2 = __vimin3_u32(m2, v0 ^ mask, v1 ^ mask);
        n2 = __vimin3_u32(n2, u0 ^ mask, u1 ^ mask);
        m2 = __vimin3_u32(m2, v2 ^ mask, v3 ^ mask);
        n2 = __vimin3_u32(n2, u2 ^ mask, u3 ^ mask);
      }
      for (; j < hm; j += 4) {
        const uint4 x = *reinterpret_cast<const uint4 *>(srow + j);
        const uint4 y = *reinterpret_cast<const uint4 *>(tbuf + j);
        const uint32_t v0 = x.x + y.x;
        const uint32_t v1 = (j + 1 < hm) ? x.y + y.y : 0xffffffffu;
        const uint32_t v2 = (j + 2 < hm) ? x.z + y.z : 0xffffffffu;
        const uint32_t v3 = (j + 3 < hm) ? x.w + y.w : 0xffffffffu;
        m1 = __vimin3_u32(m1, v0, v1);
        m1 = __vimin3_u32(m1, v2, v3);
        m2 = __vimin3_u32(m2, v0 ^ mask, (j + 1 < hm) ? v1 ^ mask : 0xffffffffu);
        m2 = __vimin3_u32(m2, (j + 2 < hm) ? v2 ^ mask : 0xffffffffu, (j + 3 < hm) ? v3 ^ mask : 0xffffffffu);
      }
      const int64_t toff_t = (!MP && hl > S) ? a.lab_off[t] : 0;
      for (j = S; !MP && j < hl; j += 4) {  // beyond the shared rows: both rows from global memory
        const uint4 x = __ldg(reinterpret_cast<const uint4 *>(a.dis_sh + soff + j));
        const uint4 y = __ldg(reinterpret_cast<const uint4 *>(a.dis_sh + toff_t + j));
        const uint32_t v0 = (x.x + y.x) | (uint32_t)j;
        const uint32_t v1 = (j + 1 < hl) ? ((x.y + y.y) | (uint32_t)(j + 1)) : 0xffffffffu;
        const uint32_t v2 = (j + 2 < hl) ? ((x.z + y.z) | (uint32_t)(j + 2)) : 0xffffffffu;
        const uint32_t v3 = (j + 3 < hl) ? ((x.w + y.w) | (uint32_t)(j + 3)) : 0xffffffffu;
        m1 = __vimin3_u32(m1, v0, v1);
        m1 = __vimin3_u32(m1, v2, v3);
        m2 = __vimin3_u32(m2, v0 ^ mask, (j + 1 < hl) ? v1 ^ mask : 0xffffffffu);
        m2 = __vimin3_u32(m2, (j + 2 < hl) ? v2 ^ mask : 0xffffffffu, (j + 3 < hl) ? v3 ^ mask : 0xffffffffu);
      }
      m1 = min(m1, n1);
      m2 = min(m2, n2);
      if (!fin) {  // carry (m1, m2) to the next pass
        if (have) sdc2[k] = make_int2((int)m1, (int)m2);
        __syncwarp();
        continue;
      }
      const uint32_t dist = m1 >> B;
      int cnt = 0, hop = 0;
      if (COUNTS && have) {
        if ((m1 ^ m2) == mask) {
          cnt = (int)(m1 & mask);  // the minimising entry; counts resolved after the chunk
          pending |= 1u << k;
        } else {
          const int64_t toff = a.lab_off[t];
          unsigned cc = 0;
          int hh = 0;
          for (int q = 0; q < hl; q++) {
            const bool in_tile = q >= P0 && q < P0 + S;
            const uint32_t dq = in_tile ? (srow[q - P0] + (uint32_t)tbuf[q - P0]) >> B
                                        : ((uint32_t)__ldg(a.dis_sh + soff + q) + (uint32_t)__ldg(a.dis_sh + toff + q)) >> B;
            if (dq == dist) {
              const int2 cs = __ldg(a.ch + soff + q), ct = __ldg(a.ch + toff + q);
              cc += (unsigned)cs.x * (unsigned)ct.x;
              hh = max(hh, cs.y + ct.y);
            }
          }
          cnt = (int)cc;
          hop = hh;
        }
      }
      if (have) {
        sdc2[k] = make_int2((int)dist, cnt);
        if (COUNTS) shp1[k] = hop;
      }
      __syncwarp();
    }
    if (failed) break;
    if (kend < 8 && have) {
      for (int k = kend; k < 8; k++) {
        sdc2[k] = make_int2(0, 0);
        if (COUNTS) shp1[k] = 0;
      }
    }
    if (COUNTS && fin && have && pending) {
      int2 cs8[8], ct8[8];
#pragma unroll
      for (int k = 0; k < 8; k++) {
        if (pending & (1u << k)) {
          const int jm = sdc2[k].y;
          cs8[k] = __ldg(a.ch + soff + jm);
          ct8[k] = __ldg(a.ch + a.lab_off[t0 + k] + jm);
        }
      }
#pragma unroll
      for (int k = 0; k < 8; k++) {
        if (pending & (1u << k)) {
          sdc2[k].y = (int)((unsigned)cs8[k].x * (unsigned)ct8[k].x);
          shp1[k] = cs8[k].y + ct8[k].y;
        }
      }
    }
    if (COUNTS && fin && have) {
#pragma unroll
      for (int k = 0; k < 8; k++) mh = max(mh, shp1[k]);
    }
    __syncwarp();
    {  // the warp's 32 slots x 8 targets are one contiguous block: coalesced 512-byte stores
      int4 *grec = a.out_rec + blk(first, t0, a.ns);  // 16-byte records: 512 B per store instruction
      const int2 *sdc_all = reinterpret_cast<const int2 *>(sdc);
      for (int p = lane; p < gcount * 8; p += 32) {
        const int2 x = sdc_all[(p >> 3) * 10 + (p & 7)];
        grec[p] = make_int4(x.x, x.y, 0, 0);
      }
      if (COUNTS && fin) {
        int4 *ghp = reinterpret_cast<int4 *>(a.out_hop + blk(first, t0, a.ns));
        for (int p = lane; p < gcount * 2; p += 32) ghp[p] = shp[(p >> 1) * 3 + (p & 1)];
      }
    }
    __syncwarp();
  }
  if (failed) {
    // record, then wait out every copy still in flight into this warp's row buffers before the
    // CTA's shared memory can be released (the long bound only keeps a broken copy from hanging)
    if (lane == 0 && a.err) atomicCAS(a.err, ERR_NONE, ERR_COPY_TIMEOUT);
    while (done < issued) {
      mbar_wait(&s_bar[warp][done % kRowBuffers], (done / kRowBuffers) & 1, kDrainWaitSpins);
      done++;
    }
    return;
  }
  if (COUNTS && fin && have && a.maxhop) atomicMax(a.maxhop + first + lane, mh);
}

// ------------------------------------------------------------------------------- K1 + K2, tall trees
// Packed-key label scan for trees too tall for the 32-source CTA to hold its source rows in shared
// memory (MHLQBC.cu:379-392 is the scan it replaces).  A CTA takes 16 sources, so whole rows fit
// (16 x height x 4 bytes: 175 KB at height 2,728).  Each warp scans two targets at once: lane l
// pairs source l / 2 with target A (even lanes) or B (odd lanes).  A 16-byte shared load is served
// per half-warp, at least one wavefront each (measured on B200: a broadcast to all 32 lanes costs
// 2, 16 distinct rows per half-warp cost 2 per half); with the lane pairs of a half-warp sharing a
// source row, each half-warp reads 8 source rows (one wavefront) and the two targets' rows (one
// wavefront, the two rings in different bank groups): 8 wavefronts per 8 entries of 32 pairs,
// against 12 for 32 distinct source rows.  Target rows stream through a per-target ring of RING
// blocks of 64 entries filled by cp.async (16 bytes per lane, RING - 1 blocks ahead of the scan,
// only up to the deepest LCA of that target's pairs), so no entry of a scan is read from global
// memory.  Keys, tie detection, count/hop gathers and the chunk-blocked output are those of
// k_label_scan_packed.
// (Measured: 16 warps with a 3-block ring beat 12 warps with 4 at 1M, 9.3 vs 8.7 entries/clk/SM;
// one stream over a chunk's four targets, instead of a ring refilled per target, was slower:
// its per-block bookkeeping cost more than the latency it hid.)
constexpr int kTallSources = 16;
constexpr int kTallBlock = 64;  // entries per block (16 lanes x 4)
__host__ __device__ constexpr int tall_half_words(int ring) { return ring * kTallBlock + 4; }  // +4: the two rings in different bank groups
__host__ __device__ constexpr int tall_ring_words(int ring) { return 2 * tall_half_words(ring); }  // per warp
constexpr int kTallStageWords = kTallSources * 8 * 2 + kTallSources * 8;  // per warp: (dist, count) and hop of 16 x 8 pairs

__host__ __device__ constexpr size_t tall_smem(int warps, int ring, int S) {
  return (size_t)kTallSources * S * 4 + (size_t)warps * (tall_ring_words(ring) + kTallStageWords) * 4;
}

__device__ __forceinline__ void cp_async16(void *dst, const void *src, bool in) {
  // src-size 0: nothing is read and the 16 bytes are zero-filled
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_addr(dst)), "l"(src), "r"(in ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

template <bool COUNTS, int WARPS, int RING>
__global__ void __launch_bounds__(WARPS * 32, 1) k_label_scan_tall(LabelArgs a) {
  constexpr int G = kTallSources;
  extern __shared__ int4 smem4[];
  uint32_t *s_key = reinterpret_cast<uint32_t *>(smem4);
  const int S = a.stride;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const int side = lane & 1, sl = lane >> 1;  // target side (A, B) and source slot of this lane
  uint32_t *ring = s_key + G * S + warp * tall_ring_words(RING) + side * tall_half_words(RING);
  int32_t *stage = reinterpret_cast<int32_t *>(s_key + G * S + nwarps * tall_ring_words(RING)) + warp * kTallStageWords;
  int2 *sdc = reinterpret_cast<int2 *>(stage);  // slot x 8 targets: (dist, count)
  int2 *sdc2 = sdc + sl * 8;
  int32_t *shp = stage + G * 8 * 2;             // slot x 8 targets: hop layer
  int32_t *shp1 = shp + sl * 8;
  __shared__ int32_t s_h[G];
  __shared__ int64_t s_off[G];
  const int first = blockIdx.y * G;
  if (first >= a.ns) return;
  const int gcount = min(G, a.ns - first);
  const uint32_t B = (uint32_t)a.bits, mask = (1u << B) - 1u;
  if (threadIdx.x < G) {
    const int i = threadIdx.x;
    const int s = i < gcount ? a.src[first + i] : 0;
    s_h[i] = i < gcount ? a.depth[s] : 0;
    s_off[i] = a.lab_off[s];
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < G * S; idx += blockDim.x) {
    const int i = idx / S, j = idx - i * S;
    uint32_t key = 0xffffffffu;
    if (i < gcount && j < s_h[i]) key = (uint32_t)a.dis_sh[s_off[i] + j] | (uint32_t)j;
    s_key[idx] = key;
  }
  __syncthreads();

  const bool have = sl < gcount;
  const int hs = have ? s_h[sl] : 1;
  const int64_t soff = s_off[sl];
  const uint32_t *srow = s_key + sl * S;
  const int32_t *lo = a.src_rows + (size_t)(first + (have ? sl : 0)) * 2 * a.src_stride;
  const int32_t *hi = lo + a.src_stride;
  const int nsteps = 32 - __clz(hs);
  int mh = 0;

  const int nchunk = a.n_pad >> 3;
  const int cbeg = (int)((int64_t)nchunk * blockIdx.x / a.split);
  const int cend = (int)((int64_t)nchunk * (blockIdx.x + 1) / a.split);
  for (int c = cbeg + warp; c < cend; c += nwarps) {
    const int t0 = c << 3;
    const int kend = min(8, a.n - t0);
    const int tb = t0 + 4 * side;  // this side's targets: tb .. tb + 3
    // deepest ancestor interval of this lane's source holding tb (binary search)
    int J = 0;
    if (tb < a.n) {
      int h = have ? hs : 1;
      for (int it = 0; it < nsteps; it++) {
        if (h - J > 1) {
          const int mid = (J + h) >> 1;
          const bool p = (__ldg(lo + mid) <= tb) && (tb < __ldg(hi + mid));
          J = p ? mid : J;
          h = p ? h : mid;
        }
      }
    }
    int hiJ = have ? __ldg(hi + J) : 0x7fffffff;
    int loN = (have && J + 1 < hs) ? __ldg(lo + J + 1) : 0x7fffffff;
    uint32_t pending = 0;
    int64_t toff_next = (4 * side < kend) ? a.lab_off[tb] : 0;
    for (int k = 0; k < 4; k++) {
      const int t = tb + k;
      const bool tv = 4 * side + k < kend;
      const int64_t toff = toff_next;  // loaded one target ahead
      toff_next = (k < 3 && 4 * side + k + 1 < kend) ? a.lab_off[t + 1] : 0;
      if (have && tv && k > 0) {  // advance the interval (targets grow by one)
        if (t >= hiJ) {
          do { J--; hiJ = __ldg(hi + J); } while (t >= hiJ);
          loN = __ldg(lo + J + 1);
        } else if (t == loN) {
          J++;
          hiJ = __ldg(hi + J);
          loN = (J + 1 < hs) ? __ldg(lo + J + 1) : 0x7fffffff;
        }
      }
      const int hl = (have && tv) ? J + 1 : 0;
      int hh = hl;  // the side's deepest scan (lanes of one parity), then the warp's
#pragma unroll
      for (int o = 16; o >= 2; o >>= 1) hh = max(hh, __shfl_xor_sync(kFull, hh, o));
      const int lim = (hh + 3) & ~3;  // entries of this side's target row to bring in
      const int nb = (max(hh, __shfl_xor_sync(kFull, hh, 1)) + kTallBlock - 1) / kTallBlock;
      const int32_t *trow = a.dis_sh + toff;
      auto issue = [&](int b) {  // block b of this side's row; an empty group past the last block
        if (b < nb) {
          const int e = b * kTallBlock + 4 * sl;
          cp_async16(ring + (b % RING) * kTallBlock + 4 * sl, e < lim ? trow + e : trow, e < lim);
        }
        cp_async_commit();
      };
      __syncwarp();  // the ring's slots are no longer read for the previous target
#pragma unroll
      for (int b = 0; b < RING - 1; b++) issue(b);
      uint32_t m1 = 0xffffffffu, m2 = 0xffffffffu, n1 = 0xffffffffu, n2 = 0xffffffffu;
      for (int b = 0; b < nb; b++) {
        cp_async_wait<RING - 2>();  // this lane's part of block b has landed
        __syncwarp();               // every lane's, and block b - 1 is no longer read
        issue(b + RING - 1);        // into block b - 1's slot
        const uint32_t *tbuf = ring + (b % RING) * kTallBlock;
        const uint32_t *xs = srow + b * kTallBlock;
        const int hm = min(hl - b * kTallBlock, kTallBlock);
        const int full8 = hm > 0 ? (hm & ~7) : 0;
        int j = 0;
        for (; j < full8; j += 8) {
          const uint4 x = *reinterpret_cast<const uint4 *>(xs + j);
          const uint4 y = *reinterpret_cast<const uint4 *>(tbuf + j);
          const uint4 x2 = *reinterpret_cast<const uint4 *>(xs + j + 4);
          const uint4 y2 = *reinterpret_cast<const uint4 *>(tbuf + j + 4);
          const uint32_t v0 = x.x + y.x, v1 = x.y + y.y, v2 = x.z + y.z, v3 = x.w + y.w;
          const uint32_t u0 = x2.x + y2.x, u1 = x2.y + y2.y, u2 = x2.z + y2.z, u3 = x2.w + y2.w;
          m1 = __vimin3_u32(m1, v0, v1);
          n1 = __vimin3_u32(n1, u0, u1);
          m1 = __vimin3_u32(m1, v2, v3);
          n1 = __vimin3_u32(n1, u2, u3);
          m2 = __vimin3_u32(m2, v0 ^ mask, v1 ^ mask);
          n2 = __vimin3_u32(n2, u0 ^ mask, u1 ^ mask);
          m2 = __vimin3_u32(m2, v2 ^ mask, v3 ^ mask);
          n2 = __vimin3_u32(n2, u2 ^ mask, u3 ^ mask);
        }
        for (; j < hm; j += 4) {
          const uint4 x = *reinterpret_cast<const uint4 *>(xs + j);
          const uint4 y = *reinterpret_cast<const uint4 *>(tbuf + j);
          const uint32_t v0 = x.x + y.x;
          const uint32_t v1 = (j + 1 < hm) ? x.y + y.y : 0xffffffffu;
          const uint32_t v2 = (j + 2 < hm) ? x.z + y.z : 0xffffffffu;
          const uint32_t v3 = (j + 3 < hm) ? x.w + y.w : 0xffffffffu;
          m1 = __vimin3_u32(m1, v0, v1);
          m1 = __vimin3_u32(m1, v2, v3);
          m2 = __vimin3_u32(m2, v0 ^ mask, (j + 1 < hm) ? v1 ^ mask : 0xffffffffu);
          m2 = __vimin3_u32(m2, (j + 2 < hm) ? v2 ^ mask : 0xffffffffu, (j + 3 < hm) ? v3 ^ mask : 0xffffffffu);
        }
      }
      m1 = min(m1, n1);
      m2 = min(m2, n2);
      const uint32_t dist = m1 >> B;
      int cnt = 0, hop = 0;
      if (COUNTS && have && tv) {
        if ((m1 ^ m2) == mask) {
          cnt = (int)(m1 & mask);  // the minimising entry; counts resolved after the chunk
          pending |= 1u << k;
        } else {  // a tie: sum over every minimising entry (target row from global memory)
          unsigned cc = 0;
          int hx = 0;
          for (int q = 0; q < hl; q++) {
            const uint32_t dq = (srow[q] + (uint32_t)__ldg(trow + q)) >> B;
            if (dq == dist) {
              const int2 cs = __ldg(a.ch + soff + q), ct = __ldg(a.ch + toff + q);
              cc += (unsigned)cs.x * (unsigned)ct.x;
              hx = max(hx, cs.y + ct.y);
            }
          }
          cnt = (int)cc;
          hop = hx;
        }
      }
      if (have) {
        sdc2[4 * side + k] = tv ? make_int2((int)dist, cnt) : make_int2(0, 0);
        if (COUNTS) shp1[4 * side + k] = hop;
      }
    }
    if (COUNTS && have && pending) {
      int2 cs4[4], ct4[4];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        if (pending & (1u << k)) {
          const int jm = sdc2[4 * side + k].y;
          cs4[k] = __ldg(a.ch + soff + jm);
          ct4[k] = __ldg(a.ch + a.lab_off[tb + k] + jm);
        }
      }
#pragma unroll
      for (int k = 0; k < 4; k++) {
        if (pending & (1u << k)) {
          sdc2[4 * side + k].y = (int)((unsigned)cs4[k].x * (unsigned)ct4[k].x);
          shp1[4 * side + k] = cs4[k].y + ct4[k].y;
        }
      }
    }
    if (COUNTS && have) {
#pragma unroll
      for (int k = 0; k < 4; k++) mh = max(mh, shp1[4 * side + k]);
    }
    __syncwarp();
    {  // the warp's 16 slots x 8 targets are one contiguous block of records
      int4 *grec = a.out_rec + blk(first, t0, a.ns);
      for (int p = lane; p < gcount * 8; p += 32) {
        const int2 x = sdc[p];
        grec[p] = make_int4(x.x, x.y, 0, 0);
      }
      if (COUNTS) {
        int4 *ghp = reinterpret_cast<int4 *>(a.out_hop + blk(first, t0, a.ns));
        const int4 *shp4 = reinterpret_cast<const int4 *>(shp);
        for (int p = lane; p < gcount * 2; p += 32) ghp[p] = shp4[p];
      }
    }
    __syncwarp();
  }
  cp_async_wait<0>();
  if (COUNTS && have && a.maxhop) atomicMax(a.maxhop + first + sl, mh);
}

// ------------------------------------------------------------------------------- K1 + K2, lane pairs
// The lane-pair layout of k_label_scan_tall for trees whose whole rows fit twice per warp side:
// 16 sources per CTA, lane l pairs source l / 2 with target A or B (8 shared-memory wavefronts per
// 8 entries of 32 pairs), and each side's target row is copied whole by cp.async into a per-side
// double buffer while the previous target is scanned (the next target's LCA depth is known ahead:
// the four targets of a side are consecutive, so their depths come from one interval walk).  The
// tie re-scan reads the target row from the buffer.
template <class T>
__device__ __forceinline__ T pick4(const T (&x)[4], int k) {  // x[k] without dynamic register indexing
  return k == 0 ? x[0] : k == 1 ? x[1] : k == 2 ? x[2] : x[3];
}

__host__ __device__ constexpr int rows16_side_words(int R) { return 2 * R + 4; }  // +4: the sides in different bank groups
__host__ __device__ constexpr size_t rows16_smem(int warps, int S, int R) {
  return (size_t)kTallSources * S * 4 + (size_t)warps * (2 * rows16_side_words(R) + kTallStageWords) * 4;
}

template <bool COUNTS, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, 1) k_label_scan_rows16(LabelArgs a) {
  constexpr int G = kTallSources;
  extern __shared__ int4 smem4[];
  uint32_t *s_key = reinterpret_cast<uint32_t *>(smem4);
  const int S = a.stride, R = a.row_words;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const int side = lane & 1, sl = lane >> 1;  // target side (A, B) and source slot of this lane
  uint32_t *rbuf = s_key + G * S + warp * 2 * rows16_side_words(R) + side * rows16_side_words(R);
  int32_t *stage = reinterpret_cast<int32_t *>(s_key + G * S + nwarps * 2 * rows16_side_words(R)) + warp * kTallStageWords;
  int2 *sdc = reinterpret_cast<int2 *>(stage);  // slot x 8 targets: (dist, count)
  int2 *sdc2 = sdc + sl * 8;
  int32_t *shp = stage + G * 8 * 2;             // slot x 8 targets: hop layer
  int32_t *shp1 = shp + sl * 8;
  __shared__ int32_t s_h[G];
  __shared__ int64_t s_off[G];
  const int first = blockIdx.y * G;
  if (first >= a.ns) return;
  const int gcount = min(G, a.ns - first);
  const uint32_t B = (uint32_t)a.bits, mask = (1u << B) - 1u;
  if (threadIdx.x < G) {
    const int i = threadIdx.x;
    const int s = i < gcount ? a.src[first + i] : 0;
    s_h[i] = i < gcount ? a.depth[s] : 0;
    s_off[i] = a.lab_off[s];
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < G * S; idx += blockDim.x) {
    const int i = idx / S, j = idx - i * S;
    uint32_t key = 0xffffffffu;
    if (i < gcount && j < s_h[i]) key = (uint32_t)a.dis_sh[s_off[i] + j] | (uint32_t)j;
    s_key[idx] = key;
  }
  __syncthreads();

  const bool have = sl < gcount;
  const int hs = have ? s_h[sl] : 1;
  const int64_t soff = s_off[sl];
  const uint32_t *srow = s_key + sl * S;
  const int32_t *lo = a.src_rows + (size_t)(first + (have ? sl : 0)) * 2 * a.src_stride;
  const int32_t *hi = lo + a.src_stride;
  const int nsteps = 32 - __clz(hs);
  int mh = 0;

  const int nchunk = a.n_pad >> 3;
  const int cbeg = (int)((int64_t)nchunk * blockIdx.x / a.split);
  const int cend = (int)((int64_t)nchunk * (blockIdx.x + 1) / a.split);
  for (int c = cbeg + warp; c < cend; c += nwarps) {
    const int t0 = c << 3;
    const int kend = min(8, a.n - t0);
    const int tb = t0 + 4 * side;  // this side's targets: tb .. tb + 3
    int hl[4], lim[4];
    int64_t toff[4];
    {  // LCA depths of this lane's source with the side's four targets (one interval walk)
      int J = 0;
      if (tb < a.n) {
        int h = have ? hs : 1;
        for (int it = 0; it < nsteps; it++) {
          if (h - J > 1) {
            const int mid = (J + h) >> 1;
            const bool p = (__ldg(lo + mid) <= tb) && (tb < __ldg(hi + mid));
            J = p ? mid : J;
            h = p ? h : mid;
          }
        }
      }
      int hiJ = have ? __ldg(hi + J) : 0x7fffffff;
      int loN = (have && J + 1 < hs) ? __ldg(lo + J + 1) : 0x7fffffff;
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const int t = tb + k;
        const bool tv = 4 * side + k < kend;
        toff[k] = tv ? a.lab_off[t] : 0;
        if (have && tv && k > 0) {
          if (t >= hiJ) {
            do { J--; hiJ = __ldg(hi + J); } while (t >= hiJ);
            loN = __ldg(lo + J + 1);
          } else if (t == loN) {
            J++;
            hiJ = __ldg(hi + J);
            loN = (J + 1 < hs) ? __ldg(lo + J + 1) : 0x7fffffff;
          }
        }
        hl[k] = (have && tv) ? J + 1 : 0;
        int hh = hl[k];  // the side's deepest scan (lanes of one parity)
#pragma unroll
        for (int o = 16; o >= 2; o >>= 1) hh = max(hh, __shfl_xor_sync(kFull, hh, o));
        lim[k] = (hh + 3) & ~3;
      }
    }
    auto issue_row = [&](int k) {  // the side's row of target k, whole, into buffer k & 1
      const int lk = pick4(lim, k);
      const int32_t *trow = a.dis_sh + pick4(toff, k);
      uint32_t *dst = rbuf + (k & 1) * R;
      for (int e = 4 * sl; e < lk; e += 64) cp_async16(dst + e, trow + e, true);
      cp_async_commit();
    };
    uint32_t pending = 0;
    __syncwarp();  // the buffers are no longer read for the previous chunk
    issue_row(0);
    for (int k = 0; k < 4; k++) {
      if (k < 3) issue_row(k + 1);  // into the buffer target k - 1 used
      else cp_async_commit();
      cp_async_wait<1>();  // this lane's pieces of target k's row have landed
      __syncwarp();        // and every lane's
      const int hlk = pick4(hl, k);
      const uint32_t *tbuf = rbuf + (k & 1) * R;
      uint32_t m1 = 0xffffffffu, m2 = 0xffffffffu, n1 = 0xffffffffu, n2 = 0xffffffffu;
      const int full8 = hlk & ~7;
      int j = 0;
      for (; j < full8; j += 8) {
        const uint4 x = *reinterpret_cast<const uint4 *>(srow + j);
        const uint4 y = *reinterpret_cast<const uint4 *>(tbuf + j);
        const uint4 x2 = *reinterpret_cast<const uint4 *>(srow + j + 4);
        const uint4 y2 = *reinterpret_cast<const uint4 *>(tbuf + j + 4);
        const uint32_t v0 = x.x + y.x, v1 = x.y + y.y, v2 = x.z + y.z, v3 = x.w + y.w;
        const uint32_t u0 = x2.x + y2.x, u1 = x2.y + y2.y, u2 = x2.z + y2.z, u3 = x2.w + y2.w;
        m1 = __vimin3_u32(m1, v0, v1);
        n1 = __vimin3_u32(n1, u0, u1);
        m1 = __vimin3_u32(m1, v2, v3);
        n1 = __vimin3_u32(n1, u2, u3);
        m2 = __vimin3_u32(m2, v0 ^ mask, v1 ^ mask);
        n2 = __vimin3_u32(n2, u0 ^ mask, u1 ^ mask);
        m2 = __vimin3_u32(m2, v2 ^ mask, v3 ^ mask);
        n2 = __vimin3_u32(n2, u2 ^ mask, u3 ^ mask);
      }
      for (; j < hlk; j += 4) {
        const uint4 x = *reinterpret_cast<const uint4 *>(srow + j);
        const uint4 y = *reinterpret_cast<const uint4 *>(tbuf + j);
        const uint32_t v0 = x.x + y.x;
        const uint32_t v1 = (j + 1 < hlk) ? x.y + y.y : 0xffffffffu;
        const uint32_t v2 = (j + 2 < hlk) ? x.z + y.z : 0xffffffffu;
        const uint32_t v3 = (j + 3 < hlk) ? x.w + y.w : 0xffffffffu;
        m1 = __vimin3_u32(m1, v0, v1);
        m1 = __vimin3_u32(m1, v2, v3);
        m2 = __vimin3_u32(m2, v0 ^ mask, (j + 1 < hlk) ? v1 ^ mask : 0xffffffffu);
        m2 = __vimin3_u32(m2, (j + 2 < hlk) ? v2 ^ mask : 0xffffffffu, (j + 3 < hlk) ? v3 ^ mask : 0xffffffffu);
      }
      m1 = min(m1, n1);
      m2 = min(m2, n2);
      const bool tv = hlk > 0;
      const uint32_t dist = m1 >> B;
      int cnt = 0, hop = 0;
      if (COUNTS && tv) {
        if ((m1 ^ m2) == mask) {
          cnt = (int)(m1 & mask);  // the minimising entry; counts resolved after the chunk
          pending |= 1u << k;
        } else {  // a tie: sum over every minimising entry
          const int64_t tk = pick4(toff, k);
          unsigned cc = 0;
          int hx = 0;
          for (int q = 0; q < hlk; q++) {
            if (((srow[q] + tbuf[q]) >> B) == dist) {
              const int2 cs = __ldg(a.ch + soff + q), ct = __ldg(a.ch + tk + q);
              cc += (unsigned)cs.x * (unsigned)ct.x;
              hx = max(hx, cs.y + ct.y);
            }
          }
          cnt = (int)cc;
          hop = hx;
        }
      }
      if (have) {
        sdc2[4 * side + k] = tv ? make_int2((int)dist, cnt) : make_int2(0, 0);
        if (COUNTS) shp1[4 * side + k] = hop;
      }
      __syncwarp();  // target k's buffer is free for target k + 2
    }
    if (COUNTS && have && pending) {
      int2 cs4[4], ct4[4];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        if (pending & (1u << k)) {
          const int jm = sdc2[4 * side + k].y;
          cs4[k] = __ldg(a.ch + soff + jm);
          ct4[k] = __ldg(a.ch + toff[k] + jm);
        }
      }
#pragma unroll
      for (int k = 0; k < 4; k++) {
        if (pending & (1u << k)) {
          sdc2[4 * side + k].y = (int)((unsigned)cs4[k].x * (unsigned)ct4[k].x);
          shp1[4 * side + k] = cs4[k].y + ct4[k].y;
        }
      }
    }
    if (COUNTS && have) {
#pragma unroll
      for (int k = 0; k < 4; k++) mh = max(mh, shp1[4 * side + k]);
    }
    __syncwarp();
    {  // the warp's 16 slots x 8 targets are one contiguous block of records
      int4 *grec = a.out_rec + blk(first, t0, a.ns);
      for (int p = lane; p < gcount * 8; p += 32) {
        const int2 x = sdc[p];
        grec[p] = make_int4(x.x, x.y, 0, 0);
      }
      if (COUNTS) {
        int4 *ghp = reinterpret_cast<int4 *>(a.out_hop + blk(first, t0, a.ns));
        const int4 *shp4 = reinterpret_cast<const int4 *>(shp);
        for (int p = lane; p < gcount * 2; p += 32) ghp[p] = shp4[p];
      }
    }
    __syncwarp();
  }
  cp_async_wait<0>();
  if (COUNTS && have && a.maxhop) atomicMax(a.maxhop + first + sl, mh);
}

// ------------------------------------------------------------------------------- K1 + K2, target pairs
// Variant of k_label_scan_packed that scans two targets per step: each lane's source-row words
// are loaded from shared memory once and combined with both target rows, so a step moves 3 instead of
// 5 shared-memory wavefronts per 128 lane-entries.  Two target rows are scanned while the next two
// are in flight (4 row buffers per warp), hence 12 warps per CTA to stay within shared memory.
constexpr int kPairWarps = 12;
constexpr int kPairBuffers = 4;

__host__ __device__ constexpr size_t pair_smem(int S) {
  return (size_t)32 * S * 4 + (size_t)kPairWarps * (kPairBuffers * (size_t)S * 4 + kStageInt4 * 16);
}

// running (min key, min of key ^ mask) over entries [j0, j1) (j1 - j0 a multiple of 8) of one
// source row and one target row held in shared memory, eight at a time
__device__ __forceinline__ void scan8(const uint32_t *srow, const int32_t *tbuf, int j0, int j1, uint32_t mask,
                                      uint32_t &m1, uint32_t &m2) {
  uint32_t n1 = 0xffffffffu, n2 = 0xffffffffu;
  for (int j = j0; j < j1; j += 8) {
    const uint4 x = *reinterpret_cast<const uint4 *>(srow + j);
    const uint4 y = *reinterpret_cast<const uint4 *>(tbuf + j);
    const uint4 x2 = *reinterpret_cast<const uint4 *>(srow + j + 4);
    const uint4 y2 = *reinterpret_cast<const uint4 *>(tbuf + j + 4);
    const uint32_t v0 = x.x + y.x, v1 = x.y + y.y, v2 = x.z + y.z, v3 = x.w + y.w;
    const uint32_t u0 = x2.x + y2.x, u1 = x2.y + y2.y, u2 = x2.z + y2.z, u3 = x2.w + y2.w;
    m1 = __vimin3_u32(m1, v0, v1);
    n1 = __vimin3_u32(n1, u0, u1);
    m1 = __vimin3_u32(m1, v2, v3);
    n1 = __vimin3_u32(n1, u2, u3);
    m2 = __vimin3_u32(m2, v0 ^ mask, v1 ^ mask);
    n2 = __vimin3_u32(n2, u0 ^ mask, u1 ^ mask);
    m2 = __vimin3_u32(m2, v2 ^ mask, v3 ^ mask);
    n2 = __vimin3_u32(n2, u2 ^ mask, u3 ^ mask);
  }
  m1 = min(m1, n1);
  m2 = min(m2, n2);
}

// the same over entries [j0, hm) (j0 a multiple of 4), four at a time with the last group masked
__device__ __forceinline__ void scan_rest(const uint32_t *srow, const int32_t *tbuf, int j0, int hm, uint32_t mask,
                                          uint32_t &m1, uint32_t &m2) {
  for (int j = j0; j < hm; j += 4) {
    const uint4 x = *reinterpret_cast<const uint4 *>(srow + j);
    const uint4 y = *reinterpret_cast<const uint4 *>(tbuf + j);
    const uint32_t v0 = x.x + y.x;
    const uint32_t v1 = (j + 1 < hm) ? x.y + y.y : 0xffffffffu;
    const uint32_t v2 = (j + 2 < hm) ? x.z + y.z : 0xffffffffu;
    const uint32_t v3 = (j + 3 < hm) ? x.w + y.w : 0xffffffffu;
    m1 = __vimin3_u32(m1, v0, v1);
    m1 = __vimin3_u32(m1, v2, v3);
    m2 = __vimin3_u32(m2, v0 ^ mask, (j + 1 < hm) ? v1 ^ mask : 0xffffffffu);
    m2 = __vimin3_u32(m2, (j + 2 < hm) ? v2 ^ mask : 0xffffffffu, (j + 3 < hm) ? v3 ^ mask : 0xffffffffu);
  }
}

// the same over entries [S, hl) read from global memory (rows longer than the shared tile)
__device__ __forceinline__ void scan_global(const int32_t *dis_sh, int64_t soff, int64_t toff, int S, int hl,
                                            uint32_t mask, uint32_t &m1, uint32_t &m2) {
  for (int j = S; j < hl; j += 4) {
    const uint4 x = __ldg(reinterpret_cast<const uint4 *>(dis_sh + soff + j));
    const uint4 y = __ldg(reinterpret_cast<const uint4 *>(dis_sh + toff + j));
    const uint32_t v0 = (x.x + y.x) | (uint32_t)j;
    const uint32_t v1 = (j + 1 < hl) ? ((x.y + y.y) | (uint32_t)(j + 1)) : 0xffffffffu;
    const uint32_t v2 = (j + 2 < hl) ? ((x.z + y.z) | (uint32_t)(j + 2)) : 0xffffffffu;
    const uint32_t v3 = (j + 3 < hl) ? ((x.w + y.w) | (uint32_t)(j + 3)) : 0xffffffffu;
    m1 = __vimin3_u32(m1, v0, v1);
    m1 = __vimin3_u32(m1, v2, v3);
    m2 = __vimin3_u32(m2, v0 ^ mask, (j + 1 < hl) ? v1 ^ mask : 0xffffffffu);
    m2 = __vimin3_u32(m2, (j + 2 < hl) ? v2 ^ mask : 0xffffffffu, (j + 3 < hl) ? v3 ^ mask : 0xffffffffu);
  }
}

// distance, and count/hop (or the minimising entry, resolved after the chunk) of one pair from its
// (m1, m2) keys; ties re-scan the row (shared tile, then global memory)
template <bool COUNTS>
__device__ __forceinline__ void finish_pair(const LabelArgs &a, bool have, int k, int t, int hl, uint32_t m1, uint32_t m2,
                                            uint32_t B, uint32_t mask, const uint32_t *srow, const int32_t *tbuf, int S,
                                            int64_t soff, int2 *sdc2, int32_t *shp1, uint32_t &pending) {
  const uint32_t dist = m1 >> B;
  int cnt = 0, hop = 0;
  if (COUNTS && have) {
    if ((m1 ^ m2) == mask) {
      cnt = (int)(m1 & mask);
      pending |= 1u << k;
    } else {
      const int64_t toff = a.lab_off[t];
      unsigned cc = 0;
      int hh = 0;
      for (int q = 0; q < hl; q++) {
        const uint32_t dq = q < S ? (srow[q] + (uint32_t)tbuf[q]) >> B
                                  : ((uint32_t)__ldg(a.dis_sh + soff + q) + (uint32_t)__ldg(a.dis_sh + toff + q)) >> B;
        if (dq == dist) {
          const int2 cs = __ldg(a.ch + soff + q), ct = __ldg(a.ch + toff + q);
          cc += (unsigned)cs.x * (unsigned)ct.x;
          hh = max(hh, cs.y + ct.y);
        }
      }
      cnt = (int)cc;
      hop = hh;
    }
  }
  if (have) {
    sdc2[k] = make_int2((int)dist, cnt);
    if (COUNTS) shp1[k] = hop;
  }
}

template <bool COUNTS>
__global__ void __launch_bounds__(kPairWarps * 32, 1) k_label_scan_pair(LabelArgs a) {
  constexpr int G = 32;
  extern __shared__ int4 smem4[];
  uint32_t *s_key = reinterpret_cast<uint32_t *>(smem4);
  const int S = a.stride;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  int32_t *tb0 = reinterpret_cast<int32_t *>(s_key + G * S) + warp * kPairBuffers * S;
  int4 *sdc = reinterpret_cast<int4 *>(s_key + G * S + nwarps * kPairBuffers * S) + warp * kStageInt4;
  int4 *shp = sdc + 32 * 5;
  int2 *sdc2 = reinterpret_cast<int2 *>(sdc) + lane * 10;
  int32_t *shp1 = reinterpret_cast<int32_t *>(shp) + lane * 12;
  __shared__ int32_t s_h[G];
  __shared__ int64_t s_off[G];
  __shared__ __align__(8) uint64_t s_bar[kPairWarps][kPairBuffers];
  const int first = blockIdx.y * G;
  if (first >= a.ns) return;
  const int gcount = min(G, a.ns - first);
  const uint32_t B = (uint32_t)a.bits, mask = (1u << B) - 1u;
  if (threadIdx.x < G) {
    const int i = threadIdx.x;
    const int s = i < gcount ? a.src[first + i] : 0;
    s_h[i] = i < gcount ? a.depth[s] : 0;
    s_off[i] = a.lab_off[s];
  }
  if (lane == 0)
    for (int b = 0; b < kPairBuffers; b++) mbar_init(&s_bar[warp][b], 1);
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  __syncthreads();
  for (int idx = threadIdx.x; idx < G * S; idx += blockDim.x) {
    const int i = idx / S, j = idx - i * S;
    uint32_t key = 0xffffffffu;
    if (i < gcount && j < s_h[i]) key = (uint32_t)a.dis_sh[s_off[i] + j] | (uint32_t)j;
    s_key[idx] = key;
  }
  __syncthreads();

  const bool have = lane < gcount;
  const int hs = have ? s_h[lane] : 1;
  const int64_t soff = s_off[lane];
  const uint32_t *srow = s_key + lane * S;
  const int32_t *lo = a.src_rows + (size_t)(first + (have ? lane : 0)) * 2 * a.src_stride;
  const int32_t *hi = lo + a.src_stride;
  const int nsteps = 32 - __clz(hs);
  int mh = 0;
  bool failed = false;

  const int nchunk = a.n_pad >> 3;
  const int cbeg = (int)((int64_t)nchunk * blockIdx.x / a.split);
  const int cend = (int)((int64_t)nchunk * (blockIdx.x + 1) / a.split);
  uint32_t issued = 0, done = 0;
  int next_c = cbeg + warp, next_k = 0;
  auto issue_next = [&]() {
    if (next_c >= cend) return;
    const int t = next_c * 8 + next_k;
    if (t >= a.n) { next_c = cend; return; }
    if (lane == 0) {
      const uint32_t b = issued % kPairBuffers;
      const uint32_t bytes = (uint32_t)(min((a.depth[t] + 3) & ~3, S) * 4);  // S is a multiple of 4
      bulk_row_to_smem(tb0 + b * S, a.dis_sh + a.lab_off[t], bytes, &s_bar[warp][b]);
    }
    issued++;
    if (++next_k == 8) { next_k = 0; next_c += nwarps; }
  };
  auto wait_row = [&](const int32_t *&tbuf) {
    const uint32_t b = done % kPairBuffers;
    if (!mbar_wait(&s_bar[warp][b], (done / kPairBuffers) & 1, a.wait_spins)) return false;
    done++;
    tbuf = tb0 + b * S;
    return true;
  };
  for (int q = 0; q < kPairBuffers - 2; q++) issue_next();

  for (int c = cbeg + warp; c < cend && !failed; c += nwarps) {
    const int t0 = c << 3;
    int J = 0;
    {
      int h = have ? hs : 1;
      for (int it = 0; it < nsteps; it++) {
        if (h - J > 1) {
          const int mid = (J + h) >> 1;
          const bool p = (__ldg(lo + mid) <= t0) && (t0 < __ldg(hi + mid));
          J = p ? mid : J;
          h = p ? h : mid;
        }
      }
    }
    int hiJ = have ? __ldg(hi + J) : 0x7fffffff;
    int loN = (have && J + 1 < hs) ? __ldg(lo + J + 1) : 0x7fffffff;
    // the deepest ancestor interval holding t, moved on from the previous target
    auto advance = [&](int t) {
      if (!have) return;
      if (t >= hiJ) {
        do { J--; hiJ = __ldg(hi + J); } while (t >= hiJ);
        loN = __ldg(lo + J + 1);
      } else if (t == loN) {
        J++;
        hiJ = __ldg(hi + J);
        loN = (J + 1 < hs) ? __ldg(lo + J + 1) : 0x7fffffff;
      }
    };
    uint32_t pending = 0;
    const int kend = min(8, a.n - t0);
    for (int k = 0; k < kend; k += 2) {
      const int ta = t0 + k, tb = ta + 1;
      const bool two = k + 1 < kend;
      if (k > 0) advance(ta);
      const int hla = have ? J + 1 : 0;
      int hlb = 0;
      if (two) {
        advance(tb);
        hlb = have ? J + 1 : 0;
      }
      issue_next();
      if (two) issue_next();
      const int32_t *tba = nullptr, *tbb = nullptr;
      if (!wait_row(tba) || (two && !wait_row(tbb))) {
        failed = true;
        break;
      }
      if (!two) tbb = tba;
      const int hma = min(hla, S), hmb = min(hlb, S);
      const int full8 = min(hma, hmb) & ~7;
      uint32_t a1 = 0xffffffffu, a2 = 0xffffffffu, an1 = 0xffffffffu, an2 = 0xffffffffu;
      uint32_t b1 = 0xffffffffu, b2 = 0xffffffffu, bn1 = 0xffffffffu, bn2 = 0xffffffffu;
      for (int j = 0; j < full8; j += 8) {  // both targets: one load of the source words
        const uint4 x = *reinterpret_cast<const uint4 *>(srow + j);
        const uint4 x2 = *reinterpret_cast<const uint4 *>(srow + j + 4);
        const uint4 y = *reinterpret_cast<const uint4 *>(tba + j);
        const uint4 y2 = *reinterpret_cast<const uint4 *>(tba + j + 4);
        const uint4 z = *reinterpret_cast<const uint4 *>(tbb + j);
        const uint4 z2 = *reinterpret_cast<const uint4 *>(tbb + j + 4);
        uint32_t v0 = x.x + y.x, v1 = x.y + y.y, v2 = x.z + y.z, v3 = x.w + y.w;
        uint32_t u0 = x2.x + y2.x, u1 = x2.y + y2.y, u2 = x2.z + y2.z, u3 = x2.w + y2.w;
        a1 = __vimin3_u32(a1, v0, v1);
        an1 = __vimin3_u32(an1, u0, u1);
        a1 = __vimin3_u32(a1, v2, v3);
        an1 = __vimin3_u32(an1, u2, u3);
        a2 = __vimin3_u32(a2, v0 ^ mask, v1 ^ mask);
        an2 = __vimin3_u32(an2, u0 ^ mask, u1 ^ mask);
        a2 = __vimin3_u32(a2, v2 ^ mask, v3 ^ mask);
        an2 = __vimin3_u32(an2, u2 ^ mask, u3 ^ mask);
        v0 = x.x + z.x, v1 = x.y + z.y, v2 = x.z + z.z, v3 = x.w + z.w;
        u0 = x2.x + z2.x, u1 = x2.y + z2.y, u2 = x2.z + z2.z, u3 = x2.w + z2.w;
        b1 = __vimin3_u32(b1, v0, v1);
        bn1 = __vimin3_u32(bn1, u0, u1);
        b1 = __vimin3_u32(b1, v2, v3);
        bn1 = __vimin3_u32(bn1, u2, u3);
        b2 = __vimin3_u32(b2, v0 ^ mask, v1 ^ mask);
        bn2 = __vimin3_u32(bn2, u0 ^ mask, u1 ^ mask);
        b2 = __vimin3_u32(b2, v2 ^ mask, v3 ^ mask);
        bn2 = __vimin3_u32(bn2, u2 ^ mask, u3 ^ mask);
      }
      a1 = min(a1, an1);
      a2 = min(a2, an2);
      b1 = min(b1, bn1);
      b2 = min(b2, bn2);
      scan8(srow, tba, full8, hma & ~7, mask, a1, a2);
      scan_rest(srow, tba, hma & ~7, hma, mask, a1, a2);
      if (hla > S) scan_global(a.dis_sh, soff, a.lab_off[ta], S, hla, mask, a1, a2);
      finish_pair<COUNTS>(a, have, k, ta, hla, a1, a2, B, mask, srow, tba, S, soff, sdc2, shp1, pending);
      if (two) {
        scan8(srow, tbb, full8, hmb & ~7, mask, b1, b2);
        scan_rest(srow, tbb, hmb & ~7, hmb, mask, b1, b2);
        if (hlb > S) scan_global(a.dis_sh, soff, a.lab_off[tb], S, hlb, mask, b1, b2);
        finish_pair<COUNTS>(a, have, k + 1, tb, hlb, b1, b2, B, mask, srow, tbb, S, soff, sdc2, shp1, pending);
      }
      __syncwarp();
    }
    if (failed) break;
    if (kend < 8 && have) {
      for (int k = kend; k < 8; k++) {
        sdc2[k] = make_int2(0, 0);
        if (COUNTS) shp1[k] = 0;
      }
    }
    if (COUNTS && have && pending) {
      int2 cs8[8], ct8[8];
#pragma unroll
      for (int k = 0; k < 8; k++) {
        if (pending & (1u << k)) {
          const int jm = sdc2[k].y;
          cs8[k] = __ldg(a.ch + soff + jm);
          ct8[k] = __ldg(a.ch + a.lab_off[t0 + k] + jm);
        }
      }
#pragma unroll
      for (int k = 0; k < 8; k++) {
        if (pending & (1u << k)) {
          sdc2[k].y = (int)((unsigned)cs8[k].x * (unsigned)ct8[k].x);
          shp1[k] = cs8[k].y + ct8[k].y;
        }
      }
    }
    if (COUNTS && have) {
#pragma unroll
      for (int k = 0; k < 8; k++) mh = max(mh, shp1[k]);
    }
    __syncwarp();
    {
      int4 *grec = a.out_rec + blk(first, t0, a.ns);
      const int2 *sdc_all = reinterpret_cast<const int2 *>(sdc);
      for (int p = lane; p < gcount * 8; p += 32) {
        const int2 x = sdc_all[(p >> 3) * 10 + (p & 7)];
        grec[p] = make_int4(x.x, x.y, 0, 0);
      }
      if (COUNTS) {
        int4 *ghp = reinterpret_cast<int4 *>(a.out_hop + blk(first, t0, a.ns));
        for (int p = lane; p < gcount * 2; p += 32) ghp[p] = shp[(p >> 1) * 3 + (p & 1)];
      }
    }
    __syncwarp();
  }
  if (failed) {
    if (lane == 0 && a.err) atomicCAS(a.err, ERR_NONE, ERR_COPY_TIMEOUT);
    while (done < issued) {
      mbar_wait(&s_bar[warp][done % kPairBuffers], (done / kPairBuffers) & 1, kDrainWaitSpins);
      done++;
    }
    return;
  }
  if (COUNTS && have && a.maxhop) atomicMax(a.maxhop + first + lane, mh);
}

// ------------------------------------------------------------------------------- K3 - K5
struct DepArgs {
  const int2 *__restrict__ arc_rng;  // per vertex (first arc, end arc)
  const int2 *__restrict__ arc_hw;   // per arc (head, weight)
  const int4 *__restrict__ arc4;     // per vertex its first four arcs in 32 bytes (arc4_of)
  const int32_t *__restrict__ arc_off;
  const int32_t *__restrict__ arc_head;
  const int32_t *__restrict__ arc_w;
  const int32_t *__restrict__ src;
  int32_t ns, n, n_pad;
  int4 *rec;       // [ns][n_pad] records (dist, sigma, delta as f64); sigma written by the Kahn kernel
  int32_t *hop;    // [ns][n_pad] layer (MHL) / indegree then wave (H2H)
  int32_t *order;  // [ns][n_pad] level queue
  int32_t *lcnt;   // [ns][2*(n_pad+2)] global layer counters when shared ones do not suffice
  double *bc;      // [n] tid order, FP64 red target
  int32_t *err;
};
// The label-free sweep's records carry DAG-successor masks in their last word until rho overwrites
// it (bit k for the k-th of the first four arcs, bit 4 for a later arc); k_dependency_cta_pipe<true>
// loads only those successors' records.

__device__ __forceinline__ int block_reduce_max(int v, int *red) {
  v = __reduce_max_sync(kFull, v);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    int x = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : INT_MIN;
    x = __reduce_max_sync(kFull, x);
    if (threadIdx.x == 0) red[32] = x;
  }
  __syncthreads();
  int r = red[32];
  __syncthreads();
  return r;
}

// exclusive scan of cnt[0..len) into itself; cnt[len] = total.  Block-wide.
__device__ __forceinline__ void block_exclusive_scan(int *cnt, int len, int *red) {
  const int nt = blockDim.x;
  const int per = (len + nt - 1) / nt;
  const int b = threadIdx.x * per, e = min(len, b + per);
  int local = 0;
  for (int i = b; i < e; i++) local += cnt[i];
  // block scan of `local`
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int x = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) red[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int nw = nt >> 5;
    int w = lane < nw ? red[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(kFull, w, o);
      if (lane >= o) w += y;
    }
    if (lane < nw) red[lane] = w;  // inclusive warp totals
  }
  __syncthreads();
  int run = x - local + (warp > 0 ? red[warp - 1] : 0);
  for (int i = b; i < e; i++) {
    int c = cnt[i];
    cnt[i] = run;
    run += c;
  }
  __syncthreads();
  if (threadIdx.x == nt - 1) cnt[len] = run;
  __syncthreads();
}

// atomicAdd of 1 on the layer counter ctr[key]; returns this vertex's slot.  Plain shared-memory
// atomics: measured faster on B200 than warp aggregation with __match_any_sync (dependency pass
// 164 -> 153 ms per all-source step at 50k); slots within a layer are then in no fixed order,
// which changes nothing (vertices of one layer are independent).
__device__ __forceinline__ int layer_slot(int *ctr, int key) { return atomicAdd(ctr + key, 1); }

// Dependencies (MHLQBC.cu:452-466): delta_v = sum over DAG arcs v->w of sigma_v * (1 + delta_w) /
// sigma_w.  Factored as delta_v = sigma_v * sum_w rho_w with rho_w = (1 + delta_w) / sigma_w, one
// FP64 division per vertex instead of one per DAG arc; this reassociation changes results only by
// rounding (relative 1e-14 at the tested sizes; the BC tolerance is 1e-9).  A vertex's per-source
// record is 16 bytes: (dist, sigma bits, rho as f64), so one load brings everything the backprop
// needs about a DAG successor.  Records are read with plain (coherent) loads: rho is written
// during the pass.
__device__ __forceinline__ double rec_rho(const int4 r) { return __hiloint2double(r.w, r.z); }
__device__ __forceinline__ void set_rho(int4 *r, double x) { reinterpret_cast<double *>(r)[1] = x; }

// A dependency pass leaves at once when the error word is set: the rows it would read come from a
// label scan or sweep that gave up (its hop layers could index past the layer counters), and the
// call reports the error anyway.
__device__ __forceinline__ bool rows_failed(const DepArgs &a) { return a.err && __ldcg(a.err) != ERR_NONE; }

// delta of v, its rho stored in its record, 0.5 * delta added into BC
template <class RV>
__device__ __forceinline__ void finish_vertex(const DepArgs &a, const RV &rec, int v, double sv, double sum) {
  const double d = sv * sum;
  set_rho(&rec[v], (1.0 + d) / sv);
  atomicAdd(a.bc + v, 0.5 * d);
}

// layered backprop over a level queue by a whole CTA (defined after the 4-wide gather below)
template <class RV>
__device__ void backprop_levels(const DepArgs &a, const RV &rec, const int32_t *order, const int *start, int maxL);

__global__ void __launch_bounds__(256) k_dependency(DepArgs a) {
  if (rows_failed(a)) return;
  __shared__ int sh_cnt[kLayerCap + 2];
  __shared__ int sh_cur[kLayerCap + 2];
  __shared__ int red[33];
  const int slot = blockIdx.x;
  if (slot >= a.ns) return;
  const int s = a.src[slot];
  const size_t base = (size_t)slot * a.n_pad;
  const RowView<int4> rec{a.rec, slot, a.ns};
  const RowView<const int32_t> hop{a.hop, slot, a.ns};
  int32_t *order = a.order + base;

  int mx = 0;
  for (int v = threadIdx.x; v < a.n; v += blockDim.x) mx = max(mx, hop[v]);
  const int maxL = block_reduce_max(mx, red);
  int *cnt = sh_cnt, *cur = sh_cur;
  if (maxL + 2 > kLayerCap) {
    cnt = a.lcnt + (size_t)slot * 2 * (a.n_pad + 2);
    cur = cnt + (a.n_pad + 2);
  }
  for (int i = threadIdx.x; i <= maxL + 1; i += blockDim.x) cnt[i] = 0;
  __syncthreads();
  const int nround = (a.n + blockDim.x - 1) / blockDim.x * blockDim.x;
  for (int v0 = 0; v0 < nround; v0 += blockDim.x) {
    const int v = v0 + threadIdx.x;
    const bool ok = v < a.n && v != s;
    if (ok) layer_slot(cnt, hop[v]);
  }
  __syncthreads();
  block_exclusive_scan(cnt, maxL + 1, red);
  for (int i = threadIdx.x; i <= maxL + 1; i += blockDim.x) cur[i] = cnt[i];
  __syncthreads();
  for (int v0 = 0; v0 < nround; v0 += blockDim.x) {
    const int v = v0 + threadIdx.x;
    const bool ok = v < a.n && v != s;
    if (ok) order[layer_slot(cur, hop[v])] = v;
  }
  __syncthreads();
  backprop_levels(a, rec, order, cnt, maxL);
}

// Warp-per-source form of k_dependency for graphs whose per-source DAG is narrow: no CTA-wide
// barrier per layer (a __syncwarp orders the layer's delta writes), many sources in flight per SM
// to cover the gathers' DRAM latency, and the largest layer taken from the label kernel.
// sum of rho over v's SP-DAG out-arcs gathered four at a time: the (head, weight) pairs of up to
// four arcs are loaded together, then their heads' records together, so a vertex costs two rounds
// of memory latency per four arcs instead of two per arc; arcs are summed in CSR order.
template <class RV>
__device__ __forceinline__ double pull_rho_sum4(const DepArgs &a, const RV &rec, int v, double &sv) {
  const int4 rv = rec[v];
  const int2 rng = a.arc_rng[v];
  sv = (double)rv.y;
  double acc = 0.0;
  for (int e = rng.x; e < rng.y; e += 4) {
    int2 hw[4];
#pragma unroll
    for (int q = 0; q < 4; q++) hw[q] = (e + q < rng.y) ? a.arc_hw[e + q] : make_int2(-1, 0);
    int4 rw[4];
#pragma unroll
    for (int q = 0; q < 4; q++)
      if (hw[q].x >= 0) rw[q] = rec[hw[q].x];
#pragma unroll
    for (int q = 0; q < 4; q++)
      if (hw[q].x >= 0 && rw[q].x == rv.x + hw[q].y) acc += rec_rho(rw[q]);
  }
  return acc;
}

template <class RV>
__device__ void backprop_levels(const DepArgs &a, const RV &rec, const int32_t *order, const int *start, int maxL) {
  for (int L = maxL; L >= 1; --L) {
    const int b = start[L], e = start[L + 1];
    for (int idx = b + threadIdx.x; idx < e; idx += blockDim.x) {
      const int v = order[idx];
      double sv;
      const double sum = pull_rho_sum4(a, rec, v, sv);
      finish_vertex(a, rec, v, sv, sum);
    }
    __syncthreads();
  }
}

// One step of the pipelined backprop: up to 32 vertices of one layer, one per lane.
struct StepIt {
  int L, idx, end;  // layer, first queue position of the step, end of the layer
};

__device__ __forceinline__ StepIt step_first(const int *cnt, int maxL) {
  int L = maxL;
  while (L >= 1 && cnt[L] == cnt[L + 1]) L--;
  return StepIt{L, L >= 1 ? cnt[L] : 0, L >= 1 ? cnt[L + 1] : 0};
}

__device__ __forceinline__ StepIt step_next(const int *cnt, StepIt it, int width = 32) {
  if (it.L < 1) return it;
  it.idx += width;
  if (it.idx < it.end) return it;
  int L = it.L - 1;
  while (L >= 1 && cnt[L] == cnt[L + 1]) L--;
  return StepIt{L, L >= 1 ? cnt[L] : 0, L >= 1 ? cnt[L + 1] : 0};
}

template <bool PIPE>
__global__ void __launch_bounds__(256, 3) k_dependency_warp(DepArgs a, const int32_t *__restrict__ maxhop, int lcap) {
  if (rows_failed(a)) return;
  extern __shared__ int smw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const int slot = blockIdx.x * nwarps + warp;
  if (slot >= a.ns) return;
  const int s = a.src[slot];
  const size_t base = (size_t)slot * a.n_pad;
  const RowView<int4> rec{a.rec, slot, a.ns};
  const RowView<const int32_t> hop{a.hop, slot, a.ns};
  int32_t *order = a.order + base;
  const int maxL = maxhop[slot];
  int *cnt, *cur;
  if (maxL + 2 <= lcap) {
    cnt = smw + warp * 2 * lcap;
    cur = cnt + lcap;
  } else {
    cnt = a.lcnt + (size_t)slot * 2 * (a.n_pad + 2);
    cur = cnt + (a.n_pad + 2);
  }
  for (int i = lane; i <= maxL + 1; i += 32) cnt[i] = 0;
  __syncwarp();
  // layer histogram: four loads in flight per lane before the aggregated shared atomics
  for (int v0 = 0; v0 < a.n; v0 += 128) {
    int hv[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int v = v0 + q * 32 + lane;
      hv[q] = (v < a.n && v != s) ? hop[v] : -1;
    }
#pragma unroll
    for (int q = 0; q < 4; q++)
      if (hv[q] >= 0) layer_slot(cnt, hv[q]);
  }
  __syncwarp();
  {  // exclusive scan of cnt[0..maxL] by the warp
    const int len = maxL + 1;
    const int per = (len + 31) / 32;
    const int b = lane * per, e = min(len, b + per);
    int local = 0;
    for (int i = b; i < e; i++) local += cnt[i];
    int x = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(kFull, x, o);
      if (lane >= o) x += y;
    }
    int run = x - local;
    for (int i = b; i < e; i++) {
      const int c = cnt[i];
      cnt[i] = run;
      cur[i] = run;
      run += c;
    }
    const int total = __shfl_sync(kFull, x, 31);
    if (lane == 0) cnt[len] = total;
  }
  __syncwarp();
  for (int v0 = 0; v0 < a.n; v0 += 128) {
    int hv[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int v = v0 + q * 32 + lane;
      hv[q] = (v < a.n && v != s) ? hop[v] : -1;
    }
#pragma unroll
    for (int q = 0; q < 4; q++)
      if (hv[q] >= 0) order[layer_slot(cur, hv[q])] = v0 + q * 32 + lane;
  }
  __syncwarp();
  if constexpr (PIPE) {
    // Software-pipelined backprop: everything about a vertex that does not change during the pass
    // (its queue entry, its dist/sigma, its arc range, its first four arcs) is loaded one to three
    // steps ahead, so a step waits only for its successors' records (rho written by the previous
    // layer).  Steps never cross a layer; a __syncwarp separates layers.
    StepIt itC = step_first(cnt, maxL);  // step being computed
    StepIt itB = step_next(cnt, itC);    // its successor: records + arc ranges arriving
    StepIt itA = step_next(cnt, itB);    // the one after: queue entry arriving
    auto vertex_at = [&](const StepIt &it) { return (it.L >= 1 && it.idx + lane < it.end) ? order[it.idx + lane] : -1; };
    // stage C (compute) registers
    int vC = vertex_at(itC);
    int4 rC = vC >= 0 ? rec[vC] : make_int4(0, 0, 0, 0);
    int2 gC = vC >= 0 ? a.arc_rng[vC] : make_int2(0, 0);
    int2 hC[4];
#pragma unroll
    for (int q = 0; q < 4; q++) hC[q] = (gC.x + q < gC.y) ? a.arc_hw[gC.x + q] : make_int2(-1, 0);
    // stage B registers
    int vB = vertex_at(itB);
    int4 rB = vB >= 0 ? rec[vB] : make_int4(0, 0, 0, 0);
    int2 gB = vB >= 0 ? a.arc_rng[vB] : make_int2(0, 0);
    // stage A register
    int vA = vertex_at(itA);
    while (itC.L >= 1) {
      // issue the look-ahead loads first
      int2 hB[4];
#pragma unroll
      for (int q = 0; q < 4; q++) hB[q] = (gB.x + q < gB.y) ? a.arc_hw[gB.x + q] : make_int2(-1, 0);
      const int4 rA = vA >= 0 ? rec[vA] : make_int4(0, 0, 0, 0);
      const int2 gA = vA >= 0 ? a.arc_rng[vA] : make_int2(0, 0);
      const StepIt itN = step_next(cnt, itA);
      const int vN = vertex_at(itN);
      // compute step C: its successors' records (rho written by earlier layers)
      if (vC >= 0) {
        int4 rw[4];
#pragma unroll
        for (int q = 0; q < 4; q++)
          if (hC[q].x >= 0) rw[q] = rec[hC[q].x];
        double acc = 0.0;
#pragma unroll
        for (int q = 0; q < 4; q++)
          if (hC[q].x >= 0 && rw[q].x == rC.x + hC[q].y) acc += rec_rho(rw[q]);
        for (int e = gC.x + 4; e < gC.y; e++) {  // arcs beyond the first four, in arc order
          const int2 hw = a.arc_hw[e];
          const int4 r = rec[hw.x];
          if (r.x == rC.x + hw.y) acc += rec_rho(r);
        }
        finish_vertex(a, rec, vC, (double)rC.y, acc);
      }
      // rotate; a layer change needs this layer's rho visible to the whole warp
      if (itB.L != itC.L) __syncwarp();
      itC = itB;
      vC = vB;
      rC = rB;
      gC = gB;
#pragma unroll
      for (int q = 0; q < 4; q++) hC[q] = hB[q];
      itB = itA;
      vB = vA;
      rB = rA;
      gB = gA;
      itA = itN;
      vA = vN;
    }
  } else {
    // layers from the deepest up; two vertices per lane per step so their gathers overlap
    for (int L = maxL; L >= 1; --L) {
      const int b = cnt[L], e = cnt[L + 1];
      for (int idx = b + lane; idx < e; idx += 64) {
        const bool two = idx + 32 < e;
        const int v1 = order[idx];
        const int v2 = two ? order[idx + 32] : v1;
        double sv1, sv2 = 1.0;
        const double r1 = pull_rho_sum4(a, rec, v1, sv1);
        const double r2 = two ? pull_rho_sum4(a, rec, v2, sv2) : 0.0;
        finish_vertex(a, rec, v1, sv1, r1);
        if (two) finish_vertex(a, rec, v2, sv2, r2);
      }
      __syncwarp();
    }
  }
}

// CTA-per-source form with the software-pipelined backprop of k_dependency_warp<true> (steps of
// blockDim.x vertices, a __syncthreads between layers); the largest layer comes from the label
// kernel, so the pass over the hop layers that k_dependency makes to find it is skipped.
//
// The pass is bound by L1 misses, and most of its hits are successors' records: a vertex's own
// record is loaded (through L1) one layer before its predecessors gather it.  So the kernel keeps
// its shared memory small (one layer-counter array of kDepLayerCap + 2 ints, 8 KB, so that the
// driver can leave ~220 KB of the SM's 256 KB to L1 at 3 CTAs per SM; 33 KB of counters measured
// 104 vs 86 ms per all-source step at 50k), and loads the queue and the arc lists, which are read
// once per source, past L1 (ld.global.cg: 86 -> 85 ms).
//
// One counter array serves both phases: after the exclusive scan cnt[L] is the start of layer L;
// the scatter advances it to the end of layer L, i.e. the start of layer L + 1, so the backprop
// reads layer L as [cnt[L - 1], cnt[L]) through the pointer cnt - 1.
constexpr int kDepLayerCap = 2046;

// The label-free sweep leaves its Kahn queue as the level queue (PRE): wave L is hop layer L, kept
// at [ws[L], ws[L + 1]) of the order row with the starts ws in the second half of the slot's
// layer-counter row, so the layer sort below is skipped; cnt[i] = ws[i + 1] is the same array the
// sort would leave (layer L at [cnt[L - 1], cnt[L]), the source alone in layer 0 at the front).
__device__ __forceinline__ const int32_t *sweep_wave_starts(const DepArgs &a, int slot) {
  return a.lcnt + (size_t)slot * 2 * (a.n_pad + 2) + (a.n_pad + 2);
}

template <bool MASK, bool PRE, class CNT>
__device__ __forceinline__ void dep_cta_pipe_body(const DepArgs &a, int slot, int maxL, CNT *cnt, int *red) {
  const int s = a.src[slot];
  const size_t base = (size_t)slot * a.n_pad;
  const RowView<int4> rec{a.rec, slot, a.ns};
  const RowView<const int32_t> hop{a.hop, slot, a.ns};
  int32_t *order = a.order + base;
  const int W = blockDim.x, tid = threadIdx.x;
  if constexpr (PRE) {
    if constexpr (!std::is_const<CNT>::value) {  // shared counters: copy the starts in
      const int32_t *ws = sweep_wave_starts(a, slot);
      for (int i = tid; i <= maxL; i += W) cnt[i] = __ldcg(ws + i + 1);
    }
    __syncthreads();
  } else {
    for (int i = threadIdx.x; i <= maxL + 1; i += blockDim.x) cnt[i] = 0;
    __syncthreads();
    // layer histogram, then the counting sort of the source's vertices by layer; each thread has
    // kHopBatch hop loads in flight before its atomics
    for (int v0 = 0; v0 < a.n; v0 += W * kHopBatch) {
      int hv[kHopBatch];
#pragma unroll
      for (int q = 0; q < kHopBatch; q++) {
        const int v = v0 + q * W + tid;
        hv[q] = (v < a.n && v != s) ? hop[v] : -1;
      }
#pragma unroll
      for (int q = 0; q < kHopBatch; q++)
        if (hv[q] >= 0) layer_slot(cnt, hv[q]);
    }
    __syncthreads();
    block_exclusive_scan(cnt, maxL + 1, red);
    for (int v0 = 0; v0 < a.n; v0 += W * kHopBatch) {
      int hv[kHopBatch];
#pragma unroll
      for (int q = 0; q < kHopBatch; q++) {
        const int v = v0 + q * W + tid;
        hv[q] = (v < a.n && v != s) ? hop[v] : -1;
      }
#pragma unroll
      for (int q = 0; q < kHopBatch; q++)
        if (hv[q] >= 0) order[layer_slot(cnt, hv[q])] = v0 + q * W + tid;
    }
    __syncthreads();
  }
  const CNT *start = cnt - 1;  // layer L is [start[L], start[L + 1]) for L >= 1
  // Pipeline over steps: the queue entry of a step is loaded three steps before it is computed,
  // its own record two, its arcs one; a step then waits only for its successors' records (rho
  // written by the layer before).
  StepIt itC = step_first(start, maxL);
  StepIt itB = step_next(start, itC, W);
  StepIt itA = step_next(start, itB, W);
  auto vertex_at = [&](const StepIt &it) {
    return (it.L >= 1 && it.idx + tid < it.end) ? __ldcg(order + it.idx + tid) : -1;
  };
  const int4 none = make_int4(-1, 0, -1, 0);
  int vC = vertex_at(itC);
  int4 rC = vC >= 0 ? rec[vC] : make_int4(0, 0, 0, 0);
  int4 aC0 = vC >= 0 ? __ldcg(a.arc4 + 2 * vC) : none, aC1 = vC >= 0 ? __ldcg(a.arc4 + 2 * vC + 1) : none;
  int vB = vertex_at(itB);
  int4 rB = vB >= 0 ? rec[vB] : make_int4(0, 0, 0, 0);
  int vA = vertex_at(itA);
  while (itC.L >= 1) {
    const int4 aB0 = vB >= 0 ? __ldcg(a.arc4 + 2 * vB) : none, aB1 = vB >= 0 ? __ldcg(a.arc4 + 2 * vB + 1) : none;
    const int4 rA = vA >= 0 ? rec[vA] : make_int4(0, 0, 0, 0);
    const StepIt itN = step_next(start, itA, W);
    const int vN = vertex_at(itN);
    if (vC >= 0) {
      const int hd[4] = {aC0.x, aC0.z, aC1.x, aC1.z}, wt[4] = {aC0.y, aC0.w, aC1.y, aC1.w};
      const int msk = MASK ? rC.w : 0x1f;  // own record: still the mask, rho comes below
      int4 rw[4];
#pragma unroll
      for (int q = 0; q < 4; q++)
        if (hd[q] >= 0 && ((msk >> q) & 1)) rw[q] = rec[hd[q]];
      double acc = 0.0;
#pragma unroll
      for (int q = 0; q < 4; q++)
        if (hd[q] >= 0 && ((msk >> q) & 1) && rw[q].x == rC.x + wt[q]) acc += rec_rho(rw[q]);
      if (hd[3] < -1 && (msk & 16)) {  // arcs beyond the third, in arc order
        for (int e = ~hd[3]; e < wt[3]; e++) {
          const int2 hw = __ldcg(a.arc_hw + e);
          const int4 r = rec[hw.x];
          if (r.x == rC.x + hw.y) acc += rec_rho(r);
        }
      }
      finish_vertex(a, rec, vC, (double)rC.y, acc);
    }
    if (itB.L != itC.L) __syncthreads();  // this layer's rho visible to the next
    itC = itB;
    vC = vB;
    rC = rB;
    aC0 = aB0;
    aC1 = aB1;
    itB = itA;
    vB = vA;
    rB = rA;
    itA = itN;
    vA = vN;
  }
}

// The body is instantiated for shared counters (the usual case: shared-memory atomics and loads)
// and for the per-slot global counters of DAGs deeper than kDepLayerCap layers; MASK (with PRE) for
// the label-free sweep's rows, whose records carry DAG-successor masks and whose queue is sorted by
// layer already, so the label path's code has neither the mask test nor the wave starts.
template <bool MASK>
__global__ void __launch_bounds__(256, 3) k_dependency_cta_pipe(DepArgs a, const int32_t *__restrict__ maxhop) {
  if (rows_failed(a)) return;
  __shared__ int sh_cnt[kDepLayerCap + 2];
  __shared__ int red[33];
  const int slot = blockIdx.x;
  if (slot >= a.ns) return;
  const int maxL = maxhop[slot];
  if (maxL <= kDepLayerCap)
    dep_cta_pipe_body<MASK, MASK>(a, slot, maxL, sh_cnt, red);
  else if constexpr (MASK)  // the sweep's wave starts, read in place
    dep_cta_pipe_body<true, true>(a, slot, maxL, sweep_wave_starts(a, slot) + 1, red);
  else
    dep_cta_pipe_body<false, false>(a, slot, maxL, a.lcnt + (size_t)slot * 2 * (a.n_pad + 2), red);
}

// QBC: sigma by Kahn waves on the SP-DAG from H2H distances (QBC.cu:335-344, :485-555), then
// the same backprop.  hop[] holds the in-degree until a vertex is queued, then its wave.
__global__ void __launch_bounds__(256) k_kahn_dependency(DepArgs a) {
  if (rows_failed(a)) return;
  __shared__ int sh_wave[kLayerCap + 2];
  __shared__ int s_tail, s_flag;
  const int slot = blockIdx.x;
  if (slot >= a.ns) return;
  const int s = a.src[slot];
  const size_t base = (size_t)slot * a.n_pad;
  const RowView<int4> rec{a.rec, slot, a.ns};
  const RowView<int32_t> deg{a.hop, slot, a.ns};
  int32_t *order = a.order + base;
  int *wave = sh_wave;
  bool global_waves = false;
  int wave_cap = kLayerCap;
  // in-degree over reverse arcs (arcs are symmetric) and sigma = 0
  for (int v = threadIdx.x; v < a.n; v += blockDim.x) {
    const int dv = rec[v].x;
    int c = 0;
    for (int e = a.arc_off[v]; e < a.arc_off[v + 1]; e++) {
      const int u = a.arc_head[e];
      if (rec[u].x + a.arc_w[e] == dv) c++;
    }
    deg[v] = c;
    rec[v].y = (v == s) ? 1 : 0;
  }
  if (threadIdx.x == 0) {
    order[0] = s;
    deg[s] = 0;
    s_tail = 1;
    s_flag = 0;
    wave[0] = 0;
    wave[1] = 1;
  }
  __syncthreads();
  int L = 0;
  for (;;) {
    const int b = wave[L], e = wave[L + 1];
    if (b == e) break;
    for (int idx = b + threadIdx.x; idx < e; idx += blockDim.x) {
      const int v = order[idx];
      const int4 dv = rec[v];
      for (int ee = a.arc_off[v]; ee < a.arc_off[v + 1]; ee++) {
        const int w = a.arc_head[ee];
        if (rec[w].x == dv.x + a.arc_w[ee]) {
          atomicAdd(&rec[w].y, dv.y);
          if (atomicSub(&deg[w], 1) == 1) {
            const int pos = atomicAdd(&s_tail, 1);
            order[pos] = w;
            deg[w] = L + 1;
          }
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      if (!global_waves && L + 2 >= wave_cap) {
        // move wave starts to global memory
        int *g = a.lcnt + (size_t)slot * 2 * (a.n_pad + 2);
        for (int i = 0; i <= L + 1; i++) g[i] = wave[i];
        s_flag = 1;
      }
    }
    __syncthreads();
    if (s_flag && !global_waves) {
      wave = a.lcnt + (size_t)slot * 2 * (a.n_pad + 2);
      global_waves = true;
      wave_cap = a.n_pad + 2;
    }
    if (threadIdx.x == 0) wave[L + 2] = s_tail;
    __syncthreads();
    L++;
    if (L > a.n) break;
  }
  if (threadIdx.x == 0) deg[s] = 0;
  if (s_tail != a.n) {
    if (threadIdx.x == 0) atomicCAS(a.err, ERR_NONE, ERR_DISCONNECTED);
    return;
  }
  __syncthreads();
  // waves 1..L-1 hold vertices; wave L is empty
  backprop_levels(a, rec, order, wave, L - 1);
}

// Each slot's source: its ancestors root first (the tree path, walked up from the source by parent
// links) and their subtree ends -- the nested intervals the label kernels test targets against,
// derived per launch instead of stored for every label entry (4 + 4 bytes per entry saved).
__global__ void k_src_rows(const int32_t *__restrict__ src, int32_t ns, const int32_t *__restrict__ depth,
                           const int32_t *__restrict__ parent, const int32_t *__restrict__ send, int32_t stride,
                           int32_t *__restrict__ rows) {
  for (int slot = blockIdx.x * blockDim.x + threadIdx.x; slot < ns; slot += gridDim.x * blockDim.x) {
    const int s = src[slot];
    int32_t *lo = rows + (size_t)slot * 2 * stride, *hi = lo + stride;
    int x = s;
    for (int j = depth[s] - 1; j >= 0; j--) {
      lo[j] = x;
      hi[j] = send[x];
      x = parent[x];
    }
  }
}

__global__ void k_tid_to_vid_f64(const double *__restrict__ in, const int32_t *__restrict__ vid_of, double *out,
                                 int n, int accumulate) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int v = vid_of[t];
    out[v] = accumulate ? out[v] + in[t] : in[t];
  }
}

__global__ void k_vid_to_tid(const int32_t *__restrict__ vids, const int32_t *__restrict__ tid_of, int32_t *out,
                             int ns, int n, int32_t *err) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += gridDim.x * blockDim.x) {
    const int v = vids[i];
    const bool ok = v >= 0 && v < n;
    out[i] = ok ? tid_of[v] : 0;
    if (!ok) atomicCAS(err, ERR_NONE, ERR_BAD_SOURCE);
  }
}

__global__ void k_rows_to_vid(const int4 *__restrict__ rec, const int32_t *__restrict__ hop,
                              const int32_t *__restrict__ vid_of, int n, int n_pad, int ns, int32_t *dist,
                              uint32_t *cnt, int32_t *hp) {
  const int slot = blockIdx.y;
  if (slot >= ns) return;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int v = vid_of[t];
    const int4 x = rec[blk(slot, t, ns)];
    dist[(size_t)slot * n + v] = x.x;
    if (cnt) cnt[(size_t)slot * n + v] = (uint32_t)x.y;
    if (hp) hp[(size_t)slot * n + v] = hop[blk(slot, t, ns)];
  }
}

// ------------------------------------------------------------------------------- launch config
struct LabelPlan {
  int K, G, S, threads, split;
  size_t smem;
};

static LabelPlan plan_label(const Handle &h, const DeviceState *d, int32_t ns, bool plain) {
  LabelPlan p{};
  p.threads = std::max(64, std::min(256, (h.tuning.label_threads / 32) * 32));
  p.S = d->hmax_pad;
  const size_t budget = (size_t)std::max(48 * 1024, d->smem_optin) - 2048;
  const size_t tb = (size_t)(p.threads / 32) * p.S * 4;
  int K = h.tuning.lanes_per_source;
  if (plain) K = 32;
  if (K <= 0) {
    K = 1;
    while (K < 32 && ((size_t)(32 / K) * 3 * p.S * 4 + tb > budget)) K *= 2;
  }
  p.K = K;
  p.G = 32 / K;
  p.smem = (size_t)p.G * 3 * p.S * 4 + tb;
  if (p.smem > budget) throw Error(QBC_EDEVICE, "tree height " + std::to_string(h.host.tree_height) + " exceeds the label kernel's shared-memory capacity");
  const int groups = (ns + p.G - 1) / p.G;
  int split = h.tuning.split;
  if (split <= 0) {
    // ~8 CTAs per SM in flight over the chunk, at least 1 target chunk of 8 per warp
    const int want = 148 * 8;
    split = std::max(1, (want + groups - 1) / groups);
    split = std::min(split, std::max(1, (d->n_pad / 8) / (p.threads / 32)));
  }
  p.split = split;
  return p;
}

template <int K, bool C>
static void launch_label_k(const LabelPlan &p, const LabelArgs &a, int groups, cudaStream_t st) {
  auto kern = k_label_scan<K, C>;
  CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem));
  dim3 grid(p.split, groups);
  kern<<<grid, p.threads, p.smem, st>>>(a);
  CK(cudaGetLastError());
}

template <bool C>
static void launch_label_c(const LabelPlan &p, const LabelArgs &a, int groups, cudaStream_t st) {
  switch (p.K) {
    case 1: launch_label_k<1, C>(p, a, groups, st); break;
    case 2: launch_label_k<2, C>(p, a, groups, st); break;
    case 4: launch_label_k<4, C>(p, a, groups, st); break;
    case 8: launch_label_k<8, C>(p, a, groups, st); break;
    case 16: launch_label_k<16, C>(p, a, groups, st); break;
    default: launch_label_k<32, C>(p, a, groups, st); break;
  }
}

// Row stride of the packed kernel with `warps` warps: the padded tree height when it fits the
// shared memory (and the tuned label tile), else the largest fitting stride (multiple of 4
// entries, odd in 16-byte units).
static int packed_stride(const Handle &h, const DeviceState *d, int warps) {
  const size_t budget = (size_t)std::max(0, d->smem_optin - 2048);
  int S = d->hmax_pad;
  if (h.tuning.label_tile > 0) S = std::min(S, std::max(8, (h.tuning.label_tile + 3) & ~3));
  // warps == 12: the two-target kernel (4 row buffers per warp)
  auto need = [&](int s) { return warps == 12 ? pair_smem(s) : packed_smem(warps, s); };
  while (S > 8 && need(S) > budget) S -= 4;
  if (((S / 4) & 1) == 0) S -= 4;
  return S;
}

// 20 (or 16) warps when the whole tree height fits, else 8 warps (twice the rows per CTA); or as tuned
static int packed_warps(const Handle &h, const DeviceState *d) {
  const int w = h.tuning.label_warps;
  if (w == 8 || w == 12 || w == 16 || w == 20) return w;
  if (packed_stride(h, d, 20) >= d->hmax_pad) return 20;  // 96 registers/thread: 20 warps fit
  return packed_stride(h, d, 16) >= d->hmax_pad ? 16 : 8;
}

// Target tiles per source group (the label kernels' grid is tiles x groups, one CTA per SM): at
// least four CTAs per SM in all, tiles of at least 8 targets per warp, and among up to twice that
// many tiles the count whose last wave of CTAs is fullest.  A launch of few groups (a 1M-vertex
// chunk holds ~40 groups of 16 sources) otherwise ends in a wave that leaves most SMs idle.
static int label_split(int groups, int warps, int n_pad, int tuned) {
  if (tuned > 0) return tuned;
  const int cap = std::max(1, (n_pad / 8) / warps);
  const int lo = std::min(cap, std::max(1, (148 * 4 + groups - 1) / groups));
  int best = lo;
  double best_fill = 0.0;
  for (int s = lo; s <= std::min(cap, 2 * lo); s++) {
    const long long ctas = (long long)groups * s;
    const double fill = (double)ctas / (double)(((ctas + 147) / 148) * 148);
    if (fill > best_fill + 1e-9) {
      best_fill = fill;
      best = s;
    }
  }
  return best;
}

template <bool C, int W>
static void launch_label_packed_w(const Handle &h, const DeviceState *d, LabelArgs a, int32_t ns, cudaStream_t st) {
  const int S = packed_stride(h, d, W);
  const size_t smem = packed_smem(W, S);
  const int groups = (ns + 31) / 32;
  const int split = label_split(groups, W, d->n_pad, h.tuning.split);
  a.stride = S;
  a.split = split;
  dim3 grid(split, groups);
  // rows longer than the tile: one pass reading the entries beyond the tile from global memory
  // (default), or several passes over tiles of S entries (label_passes = 2; measured slower at 1M:
  // every pass re-walks all targets of the CTA, 3.0 vs 4.6 label entries/clk/SM)
  const int passes = (d->hmax_pad + S - 1) / S;
  a.multipass = (passes > 1 && h.tuning.label_passes == 2) ? 1 : 0;
  auto kern = a.multipass ? k_label_scan_packed<C, W, true> : k_label_scan_packed<C, W, false>;
  CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  for (int p = 0; p < (a.multipass ? passes : 1); p++) {
    a.pass_lo = p * S;
    kern<<<grid, W * 32, smem, st>>>(a);
    CK(cudaGetLastError());
  }
}

template <bool C>
static void launch_label_pair(const Handle &h, const DeviceState *d, LabelArgs a, int32_t ns, cudaStream_t st) {
  const int S = packed_stride(h, d, 12);
  const size_t smem = pair_smem(S);
  const int groups = (ns + 31) / 32;
  const int split = label_split(groups, kPairWarps, d->n_pad, h.tuning.split);
  a.stride = S;
  a.split = split;
  a.multipass = 0;
  a.pass_lo = 0;
  CK(cudaFuncSetAttribute(k_label_scan_pair<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid(split, groups);
  k_label_scan_pair<C><<<grid, kPairWarps * 32, smem, st>>>(a);
  CK(cudaGetLastError());
}

// Tall trees: the 16-source kernel when the 32-source one cannot hold whole rows (its scans would
// read entries beyond the tile from global memory) and the label warps, tile and passes are not
// tuned; the most warps (16, 12 or 8) whose shared memory holds the whole height.  0: not used.
static int tall_stride(const DeviceState *d) {
  int S = d->hmax_pad;
  if (((S / 4) & 1) == 0) S += 4;  // odd in 16-byte units: rows 0-7 start in distinct bank groups
  return S;
}
// The configuration of the 16-source kernels: whole target rows (k_label_scan_rows16) or a ring of
// 64-entry blocks (k_label_scan_tall); warps 16, 12 or 8 (the tuned label_warps when it fits), the
// ring 4 blocks deep, else 3; {0, ...}: the 32-source kernels.  Auto: the 16-source kernels when
// the 32-source kernel cannot hold whole rows and its warps, tile and passes are not tuned; whole
// rows when they fit with 16 warps.
struct TallCfg {
  int warps, ring;
  bool whole;
};
static int rows16_words(const DeviceState *d) { return d->hmax_pad; }
static TallCfg tall_cfg(const Handle &h, const DeviceState *d) {
  const Tuning &t = h.tuning;
  if (t.label_sources == 32) return {0, 0, false};
  if (t.label_sources == 0 &&
      (t.label_warps != 0 || t.label_tile > 0 || t.label_passes != 0 || packed_stride(h, d, 8) >= d->hmax_pad))
    return {0, 0, false};
  const size_t budget = (size_t)std::max(0, d->smem_optin - 1024);
  const int S = tall_stride(d), R = rows16_words(d);
  const int w = t.label_warps;
  auto fits_whole = [&](int x) { return rows16_smem(x, S, R) <= budget; };
  if (t.label_stream == 1 || (t.label_stream == 0 && fits_whole(16))) {
    for (int x : {w, 16, 12, 8})
      if ((x == 8 || x == 12 || x == 16) && fits_whole(x)) return {x, 0, true};
  }
  for (int x : {w, 16, 12, 8}) {
    if (x != 8 && x != 12 && x != 16) continue;
    for (int r : {4, 3})
      if (tall_smem(x, r, S) <= budget) return {x, r, false};
  }
  return {0, 0, false};
}
static int tall_warps(const Handle &h, const DeviceState *d) { return tall_cfg(h, d).warps; }

template <bool C, int W, int R>
static void launch_label_tall(const DeviceState *d, LabelArgs a, int32_t ns, cudaStream_t st) {
  const int S = tall_stride(d);
  const size_t smem = tall_smem(W, R, S);
  const int groups = (ns + kTallSources - 1) / kTallSources;
  const int split = label_split(groups, W, d->n_pad, 0);
  a.stride = S;
  a.split = split;
  CK(cudaFuncSetAttribute(k_label_scan_tall<C, W, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid(split, groups);
  k_label_scan_tall<C, W, R><<<grid, W * 32, smem, st>>>(a);
  CK(cudaGetLastError());
}

template <bool C, int W>
static void launch_label_rows16(const DeviceState *d, LabelArgs a, int32_t ns, cudaStream_t st) {
  const int S = tall_stride(d), R = rows16_words(d);
  const size_t smem = rows16_smem(W, S, R);
  const int groups = (ns + kTallSources - 1) / kTallSources;
  const int split = label_split(groups, W, d->n_pad, 0);
  a.stride = S;
  a.row_words = R;
  a.split = split;
  CK(cudaFuncSetAttribute(k_label_scan_rows16<C, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid(split, groups);
  k_label_scan_rows16<C, W><<<grid, W * 32, smem, st>>>(a);
  CK(cudaGetLastError());
}

template <bool C>
static void launch_label_packed(const Handle &h, const DeviceState *d, LabelArgs a, int32_t ns, cudaStream_t st) {
  const TallCfg tc = tall_cfg(h, d);
  if (tc.whole) {
    if (tc.warps == 16) return launch_label_rows16<C, 16>(d, a, ns, st);
    if (tc.warps == 12) return launch_label_rows16<C, 12>(d, a, ns, st);
    return launch_label_rows16<C, 8>(d, a, ns, st);
  }
  if (tc.warps == 16) return tc.ring == 4 ? launch_label_tall<C, 16, 4>(d, a, ns, st) : launch_label_tall<C, 16, 3>(d, a, ns, st);
  if (tc.warps == 12) return tc.ring == 4 ? launch_label_tall<C, 12, 4>(d, a, ns, st) : launch_label_tall<C, 12, 3>(d, a, ns, st);
  if (tc.warps == 8) return tc.ring == 4 ? launch_label_tall<C, 8, 4>(d, a, ns, st) : launch_label_tall<C, 8, 3>(d, a, ns, st);
  const int w = packed_warps(h, d);
  if (w == 12) launch_label_pair<C>(h, d, a, ns, st);
  else if (w == 16) launch_label_packed_w<C, 16>(h, d, a, ns, st);
  else if (w == 20) launch_label_packed_w<C, 20>(h, d, a, ns, st);
  else launch_label_packed_w<C, 8>(h, d, a, ns, st);
}

// the packed-key kernel applies when its keys fit 32 bits
static bool use_packed(const Handle &h, const DeviceState *d, bool plain) {
  if (plain || d->packed_bits == 0 || h.tuning.lanes_per_source != 0) return false;
  return packed_stride(h, d, packed_warps(h, d)) >= 8 && packed_smem(8, 8) <= (size_t)d->smem_optin;
}

// Attempts of a label-row copy wait before it is reported (ERR_COPY_TIMEOUT).  Test hook: the
// environment variable QBC_TEST_ROW_WAIT_SPINS overrides it (0: every wait gives up at once), so
// the timeout path -- error word, drain of the copies in flight, QBC_EDEVICE, recovery -- can be
// exercised without a slow copy.
static uint32_t row_wait_spins() {
  const char *e = std::getenv("QBC_TEST_ROW_WAIT_SPINS");
  return e && *e ? (uint32_t)std::strtoul(e, nullptr, 10) : kRowWaitSpins;
}

// need_hop false: the caller's next kernel does not read the hop rows (label-free index with the
// CTA pipelined dependency pass, which walks the sweep's wave queue), so the sweep leaves them out.
static void launch_label(const Handle &h, DeviceState *d, int buf, const int32_t *src, int32_t ns, bool plain,
                         cudaStream_t st, bool need_hop = true) {
  if (h.host.kind == IndexKind::CSR) {  // no labels: shortest-path sweeps give the rows
    std::pair<cudaEvent_t, cudaEvent_t> ev{};
    if (d->profiling) {
      ev = take_events(d->ev_lab, d->ev_lab_used);
      CK(cudaEventRecord(ev.first, st));
    }
    if (plain)  // one source over the whole GPU (the buffer's slot 0 has the plain row layout)
      launch_sweep_rows_grid(h, d, d->rec[buf], d->hop[buf], d->order[buf], d->lcnt[buf], src, st);
    else
      launch_sweep_rows(h, d, d->rec[buf], d->hop[buf], d->order[buf], d->lcnt[buf], d->maxhop[buf], src, ns, st,
                        need_hop);
    if (d->profiling) CK(cudaEventRecord(ev.second, st));
    d->label_launches++;
    d->launches++;
    return;
  }
  const bool packed = use_packed(h, d, plain);
  LabelPlan p = packed ? LabelPlan{1, 32, d->hmax_pad, 512, 1, 0} : plan_label(h, d, ns, plain);
  LabelArgs a{};
  a.dis = d->dis;
  a.dis_sh = d->dis_sh;
  a.ch = d->ch;
  a.lab_off = d->lab_off;
  a.depth = d->depth;
  a.send = d->send;
  a.src = src;
  a.ns = ns;
  a.n = d->n;
  a.n_pad = d->n_pad;
  a.stride = p.S;
  a.split = p.split;
  a.out_rec = d->rec[buf];
  a.out_hop = d->hop[buf];
  a.maxhop = d->maxhop[buf];
  a.src_rows = d->src_rows[buf];
  a.src_stride = d->hmax_pad;
  a.bits = d->packed_bits;
  a.err = d->err;
  a.wait_spins = row_wait_spins();
  const int groups = (ns + p.G - 1) / p.G;
  CK(cudaMemsetAsync(d->maxhop[buf], 0, (size_t)ns * 4, st));
  k_src_rows<<<(ns + 127) / 128, 128, 0, st>>>(src, ns, d->depth, d->parent, d->send, d->hmax_pad, d->src_rows[buf]);
  CK(cudaGetLastError());
  d->launches++;
  std::pair<cudaEvent_t, cudaEvent_t> ev{};
  if (d->profiling) {
    ev = take_events(d->ev_lab, d->ev_lab_used);
    CK(cudaEventRecord(ev.first, st));
  }
  if (packed) {
    if (h.host.kind == IndexKind::MHL) launch_label_packed<true>(h, d, a, ns, st);
    else launch_label_packed<false>(h, d, a, ns, st);
  } else if (h.host.kind == IndexKind::MHL) {
    launch_label_c<true>(p, a, groups, st);
  } else {
    launch_label_c<false>(p, a, groups, st);
  }
  if (d->profiling) CK(cudaEventRecord(ev.second, st));
  d->label_launches++;
  d->launches++;
}

static DepArgs dep_args(DeviceState *d, int buf, const int32_t *src, int32_t ns) {
  DepArgs a{};
  a.arc_rng = d->arc_rng;
  a.arc_hw = d->arc_hw;
  a.arc4 = d->arc4;
  a.arc_off = d->arc_off;
  a.arc_head = d->arc_head;
  a.arc_w = d->arc_w;
  a.src = src;
  a.ns = ns;
  a.n = d->n;
  a.n_pad = d->n_pad;
  a.rec = d->rec[buf];
  a.hop = d->hop[buf];
  a.order = d->order[buf];
  a.lcnt = d->lcnt[buf];
  a.bc = d->bc_tid;
  a.err = d->err;
  return a;
}

// plain = a single source: one CTA runs its dependency pass (the warp form would leave 7/8 of the
// CTA idle)
static void launch_dep(const Handle &h, DeviceState *d, int buf, const int32_t *src, int32_t ns, cudaStream_t st,
                       bool plain = false) {
  DepArgs a = dep_args(d, buf, src, ns);
  const int threads = std::max(64, std::min(256, (h.tuning.dep_threads / 32) * 32));
  // auto (0) = the CTA-per-source pipelined pass: measured fastest at 50k (77 ms per all-source
  // step; the pipelined warp form and the plain CTA form measured 153 and 151 ms, when this pass
  // took 146)
  const int form = h.tuning.dep_form == 0 ? 4 : h.tuning.dep_form;
  // MHL and CSR rows carry counts and hop layers; H2H rows are distances only (Kahn pass)
  const bool counted = h.host.kind != IndexKind::H2H;
  const bool warp_form = counted && (form == 1 || form == 3) && !plain;
  std::pair<cudaEvent_t, cudaEvent_t> ev{};
  if (d->profiling) {
    ev = take_events(d->ev_dp, d->ev_dp_used);
    CK(cudaEventRecord(ev.first, st));
  }
  if (warp_form) {
    constexpr int wpb = 8;
    const int lcap = h.tuning.queue_depth > 0 ? std::min(2048, std::max(64, h.tuning.queue_depth)) : 512;
    const size_t smem = (size_t)wpb * 2 * lcap * 4;
    if (smem > 48 * 1024) {
      CK(cudaFuncSetAttribute(k_dependency_warp<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      CK(cudaFuncSetAttribute(k_dependency_warp<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    }
    if (form == 3)
      k_dependency_warp<true><<<(ns + wpb - 1) / wpb, wpb * 32, smem, st>>>(a, d->maxhop[buf], lcap);
    else k_dependency_warp<false><<<(ns + wpb - 1) / wpb, wpb * 32, smem, st>>>(a, d->maxhop[buf], lcap);
  } else if (counted && form == 4 && !plain) {
    if (h.host.kind == IndexKind::CSR)  // the sweep's records carry successor masks
      k_dependency_cta_pipe<true><<<ns, threads, 0, st>>>(a, d->maxhop[buf]);
    else
      k_dependency_cta_pipe<false><<<ns, threads, 0, st>>>(a, d->maxhop[buf]);
  } else if (counted) {
    k_dependency<<<ns, threads, 0, st>>>(a);
  } else {
    k_kahn_dependency<<<ns, threads, 0, st>>>(a);
  }
  CK(cudaGetLastError());
  if (d->profiling) CK(cudaEventRecord(ev.second, st));
  d->dep_launches++;
  d->launches++;
}

// the batched dependency pass of a label-free index reads the wave queue, not the hop rows
static bool dep_reads_hops(const Handle &h) {
  return !(h.host.kind == IndexKind::CSR && (h.tuning.dep_form == 0 || h.tuning.dep_form == 4));
}

void launch_chunk(const Handle &h, DeviceState *d, const int32_t *d_src_tid, int32_t cnt, int buf, cudaStream_t st) {
  launch_label(h, d, buf, d_src_tid, cnt, false, st, dep_reads_hops(h));
  launch_dep(h, d, buf, d_src_tid, cnt, st);
}

void launch_tid_to_vid(DeviceState *d, const double *in_tid, double *out_vid, int accumulate, cudaStream_t st) {
  k_tid_to_vid_f64<<<(d->n + 255) / 256, 256, 0, st>>>(in_tid, d->vid_of, out_vid, d->n, accumulate);
  CK(cudaGetLastError());
  d->launches++;
}

void launch_vid_to_tid(DeviceState *d, const int32_t *vids, int32_t *tids, int32_t cnt, cudaStream_t st) {
  if (cnt <= 0) return;
  k_vid_to_tid<<<(cnt + 255) / 256, 256, 0, st>>>(vids, d->tid_of, tids, cnt, d->n, d->err);
  CK(cudaGetLastError());
  d->launches++;
}

// Per-source scratch: one buffer of `chunk` source slots (24 B per vertex and slot plus the layer
// counters).  `chunk` comes from the tuning, else from the free memory left after the index.
static void free_scratch(DeviceState *d) {
  sweep_cache_free(d);
  for (int b = 0; b < 2; b++) {
    void *q[] = {d->rec[b], d->hop[b], d->order[b], d->lcnt[b], d->src[b], d->maxhop[b], d->src_rows[b]};
    for (void *p : q)
      if (p) cudaFree(p);
    d->rec[b] = nullptr;
    d->hop[b] = d->order[b] = d->lcnt[b] = d->src[b] = d->maxhop[b] = d->src_rows[b] = nullptr;
  }
  d->bytes -= d->scratch_bytes;
  d->scratch_bytes = 0;
  d->chunk = 0;
}

static void alloc_scratch(Handle &h, DeviceState *d) {
  const Index &ix = h.host;
  const int64_t before = d->bytes;
  const size_t per_slot = (size_t)d->n_pad * (16 + 4 + 4) + (size_t)2 * (d->n_pad + 2) * 4 + 4 + (size_t)8 * d->hmax_pad;
  size_t free_b = 0, total_b = 0;
  CK(cudaMemGetInfo(&free_b, &total_b));
  int32_t chunk = h.tuning.chunk;
  if (chunk <= 0) {
    // at most 20 GB: at 1M vertices (32 MB per slot) 608 slots, within 2-4 % of the throughput of
    // 736-1,024 slots (24-33 GB), with the 12 B per entry index the whole state stays near 44 GB
    const size_t budget = std::min<size_t>(free_b / 4, (size_t)20 << 30);
    chunk = (int32_t)std::max<size_t>(32, std::min<size_t>(4096, budget / per_slot));
    chunk = std::max(32, (chunk / 32) * 32);
  }
  chunk = std::min<int32_t>(chunk, std::max(32, (ix.n + 31) / 32 * 32));
  d->chunk = chunk;
  // one buffer: the label scan and dependency pass of consecutive chunks run in order on one stream
  for (int b = 0; b < 1; b++) {
    d->rec[b] = dmalloc<int4>(d, (size_t)chunk * d->n_pad);
    d->hop[b] = dmalloc<int32_t>(d, (size_t)chunk * d->n_pad);
    d->order[b] = dmalloc<int32_t>(d, (size_t)chunk * d->n_pad);
    d->lcnt[b] = dmalloc<int32_t>(d, (size_t)chunk * 2 * (d->n_pad + 2));
    d->src[b] = dmalloc<int32_t>(d, (size_t)chunk);
    d->maxhop[b] = dmalloc<int32_t>(d, (size_t)chunk);
    d->src_rows[b] = dmalloc<int32_t>(d, (size_t)chunk * 2 * d->hmax_pad);
  }
  d->scratch_bytes = d->bytes - before;
}

void device_set_chunk(Handle &h, int32_t chunk) {
  DeviceState *d = need_dev(h);
  CK(cudaDeviceSynchronize());
  free_scratch(d);
  h.tuning.chunk = chunk;
  alloc_scratch(h, d);
}

// ------------------------------------------------------------------------------- dense elimination
// The last r vertices of the min-degree elimination (TreeDecomp.cpp:54-208 semantics, as the host's
// eliminate): near the root the separators are large (hundreds of vertices) and the host spends
// most of its time there on the k^2 shortcut updates of each step.  Here the remaining graph is a
// dense r x r matrix of (length, count bits, max hop) entries, absent = kAbsentLen.  A step picks
// the live vertex x of minimum (degree, id), compacts its row into the separator list in column
// order, and updates every separator vertex u (a warp each): the shortcuts through x to every
// other separator vertex, with the host's rule -- a shorter length replaces, an equal one adds the
// count and keeps the larger hop -- then u's entry for x removed.  All steps run in one
// cooperative launch (k_dense_tail below); where that cannot be resident, each step is two
// launches, k_dense_pick and k_dense_update.  The picks, separators and so the tree and rows are
// the host elimination's: the separator order differs (column order here) and nothing downstream
// depends on it.
constexpr int32_t kAbsentLen = 0x7fffffff;

__global__ void k_dense_clear(int4 *M, int64_t count) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
    M[i] = make_int4(kAbsentLen, 0, 0, 0);
}

__global__ void k_dense_scatter(int4 *M, int32_t r, const int32_t *__restrict__ row, const int4 *__restrict__ ent,
                                int64_t m) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
    const int4 e = ent[i];
    M[(int64_t)row[i] * r + e.x] = make_int4(e.y, e.z, e.w, 0);
  }
}

constexpr int kPickThreads = 1024;

__global__ void __launch_bounds__(kPickThreads) k_dense_pick(const int4 *__restrict__ M, const int32_t *__restrict__ deg,
                                                             uint8_t *alive, int32_t r, int32_t step, int32_t *order,
                                                             int4 *xlist, int32_t *xcount, int4 *sep, int64_t *sep_off) {
  __shared__ unsigned long long s_best[kPickThreads / 32];
  __shared__ int32_t s_cnt[kPickThreads / 32];
  __shared__ int32_t s_x;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  unsigned long long best = ~0ull;
  for (int i = tid; i < r; i += kPickThreads)
    if (alive[i]) best = min(best, ((unsigned long long)(uint32_t)deg[i] << 32) | (uint32_t)i);
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) best = min(best, __shfl_xor_sync(kFull, best, o));
  if (lane == 0) s_best[warp] = best;
  __syncthreads();
  if (warp == 0) {
    best = s_best[lane];
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) best = min(best, __shfl_xor_sync(kFull, best, o));
    if (lane == 0) {
      const int32_t x = (int32_t)(best & 0xffffffffu);
      s_x = x;
      alive[x] = 0;
      order[step] = x;
    }
  }
  __syncthreads();
  const int32_t x = s_x;
  // row x compacted in column order: each thread takes a contiguous range of columns
  const int per = (r + kPickThreads - 1) / kPickThreads;
  const int c0 = min(r, tid * per), c1 = min(r, c0 + per);
  const int4 *row = M + (int64_t)x * r;
  int mine = 0;
  for (int c = c0; c < c1; c++) mine += row[c].x != kAbsentLen;
  int incl = mine;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) s_cnt[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int w = s_cnt[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(kFull, w, o);
      if (lane >= o) w += y;
    }
    s_cnt[lane] = w;  // inclusive warp totals
  }
  __syncthreads();
  int p = incl - mine + (warp > 0 ? s_cnt[warp - 1] : 0);
  const int total = s_cnt[kPickThreads / 32 - 1];
  const int64_t so = sep_off[step];
  for (int c = c0; c < c1; c++) {
    const int4 e = row[c];
    if (e.x != kAbsentLen) {
      const int4 v = make_int4(c, e.x, e.y, e.z);
      xlist[p] = v;
      sep[so + p] = v;
      p++;
    }
  }
  if (tid == 0) {
    *xcount = total;
    sep_off[step + 1] = so + total;
  }
}

__global__ void __launch_bounds__(256) k_dense_update(int4 *M, int32_t *deg, int32_t r, const int4 *__restrict__ xlist,
                                                      const int32_t *__restrict__ xcount,
                                                      const int32_t *__restrict__ order, int32_t step) {
  const int k = *xcount, x = order[step];
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int i = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5); i < k; i += warps) {
    const int4 a = xlist[i];
    int4 *row = M + (int64_t)a.x * r;
    int added = 0;
    for (int j = lane; j < k; j += 32) {
      if (j == i) continue;
      const int4 b = xlist[j];
      const int nl = a.y + b.y;
      const int nc = (int)((unsigned)a.z * (unsigned)b.z);
      const int nh = a.w + b.w;
      const int4 e = row[b.x];
      if (e.x == kAbsentLen) {
        row[b.x] = make_int4(nl, nc, nh, 0);
        added++;
      } else if (nl < e.x) {
        row[b.x] = make_int4(nl, nc, nh, 0);
      } else if (nl == e.x) {
        row[b.x] = make_int4(e.x, (int)((unsigned)e.y + (unsigned)nc), max(e.z, nh), 0);
      }
    }
    added = __reduce_add_sync(kFull, added);
    if (lane == 0) {
      row[x] = make_int4(kAbsentLen, 0, 0, 0);
      deg[a.x] += added - 1;
    }
  }
}

// The whole tail in one cooperative launch (1,024-thread CTAs, all resident): the same
// pick, compaction and update per step, separated by grid barriers instead of kernel boundaries
// (two launches per step cost ~38 us a step at 1M).  The grid is small -- 32 CTAs when they cover
// the row's columns, so a barrier has few arrivals; a step's update takes a warp per separator
// vertex, about 1,000 at most on the 1M grid -- and the barrier polls without sleeping.  Every CTA
// finds the pick from the per-CTA minima; the compaction of row x is split by column ranges, each
// CTA placing its entries after those of the CTAs before it; data written by other CTAs is read
// through L2 (__ldcg).  A barrier wait is bounded (a few million polls, ~1-2 s); when it runs out
// the grid leaves at its next barrier and the host reports the error.
struct DenseCtl {
  unsigned arrive, gen;
  int abort, err;
};
constexpr long long kDenseSpinLimit = 1ll << 22;  // polls of the generation word per barrier wait (~1-2 s)

__device__ __forceinline__ bool dense_grid_sync(DenseCtl *c, unsigned &gen) {
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
        if (*(volatile int *)&c->abort || ++spins > kDenseSpinLimit) {
          ok = 0;
          break;
        }
      }
      if (!ok) {
        atomicExch(&c->abort, 1);
        atomicExch(&c->err, 1);
      }
    }
    gen++;
    __threadfence();
    s_ok = ok && !*(volatile int *)&c->abort;
  }
  __syncthreads();
  return s_ok;
}

constexpr int kTailThreads = 1024;

__device__ __forceinline__ unsigned long long block_min_u64(unsigned long long v, unsigned long long *red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) v = min(v, __shfl_xor_sync(kFull, v, o));
  if (lane == 0) red[warp] = v;
  __syncthreads();
  v = red[lane];  // kTailThreads / 32 == 32 partials
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) v = min(v, __shfl_xor_sync(kFull, v, o));
  __syncthreads();
  return v;
}

// exclusive prefix sum of x over the CTA's kTailThreads threads; *total = the CTA's sum
__device__ __forceinline__ int block_scan_excl(int x, int *red, int *total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) red[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int w = red[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(kFull, w, o);
      if (lane >= o) w += y;
    }
    red[lane] = w;  // inclusive warp totals
  }
  __syncthreads();
  const int r = incl - x + (warp > 0 ? red[warp - 1] : 0);
  *total = red[31];
  __syncthreads();
  return r;
}

// r <= gridDim.x * kTailThreads (one column of row x per thread in the compaction)
__global__ void __launch_bounds__(kTailThreads, 1) k_dense_tail(int4 *M, int32_t *deg, uint8_t *alive, int32_t r,
                                                                int32_t *order, int4 *xlist, int4 *sep,
                                                                int64_t *sep_off, unsigned long long *part_best,
                                                                int32_t *part_cnt, DenseCtl *ctl) {
  __shared__ unsigned long long s_red64[32];
  __shared__ int s_red[32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int G = gridDim.x, b = blockIdx.x;
  const int cols = (r + G - 1) / G;
  const int c_lo = min(r, b * cols), c_hi = min(r, c_lo + cols);
  unsigned gen = 0;
  int64_t so = 0;  // separator entries written by the steps before (the same in every CTA)
  for (int s = 0; s < r; s++) {
    // pick: the live vertex of least (degree, id)
    unsigned long long best = ~0ull;
    for (int i = b * kTailThreads + tid; i < r; i += G * kTailThreads)
      if (__ldcg(alive + i)) best = min(best, ((unsigned long long)(uint32_t)__ldcg(deg + i) << 32) | (uint32_t)i);
    best = block_min_u64(best, s_red64);
    if (tid == 0) part_best[b] = best;
    if (!dense_grid_sync(ctl, gen)) return;
    best = ~0ull;
    for (int i = tid; i < G; i += kTailThreads) best = min(best, __ldcg(part_best + i));
    best = block_min_u64(best, s_red64);
    const int x = (int)(best & 0xffffffffu);
    // row x compacted in column order: this CTA's columns [c_lo, c_hi), one per thread
    const int c = c_lo + tid;
    int4 e = make_int4(kAbsentLen, 0, 0, 0);
    if (c < c_hi) e = __ldcg(M + (int64_t)x * r + c);
    const int pres = e.x != kAbsentLen;
    int mine_total = 0;
    const int my_off = block_scan_excl(pres, s_red, &mine_total);
    if (tid == 0) part_cnt[b] = mine_total;
    if (!dense_grid_sync(ctl, gen)) return;
    int before = 0, all = 0;
    for (int i = tid; i < G; i += kTailThreads) {
      const int v = __ldcg(part_cnt + i);
      all += v;
      if (i < b) before += v;
    }
    before = __reduce_add_sync(kFull, before);
    all = __reduce_add_sync(kFull, all);
    if (lane == 0) {
      s_red[warp] = before;
      s_red64[warp] = (unsigned long long)all;
    }
    __syncthreads();
    before = 0;
    all = 0;
    for (int w = 0; w < kTailThreads / 32; w++) {
      before += s_red[w];
      all += (int)s_red64[w];
    }
    __syncthreads();
    if (pres) {
      const int4 v = make_int4(c, e.x, e.y, e.z);
      xlist[before + my_off] = v;
      sep[so + before + my_off] = v;
    }
    if (b == 0 && tid == 0) {
      order[s] = x;
      alive[x] = 0;
      sep_off[s + 1] = so + all;
    }
    so += all;
    if (!dense_grid_sync(ctl, gen)) return;
    // update: a warp per separator vertex u, the shortcuts through x to every other one
    const int k = all;
    for (int i = b * (kTailThreads / 32) + warp; i < k; i += G * (kTailThreads / 32)) {
      const int4 a = __ldcg(xlist + i);
      int4 *row = M + (int64_t)a.x * r;
      int added = 0;
      for (int j = lane; j < k; j += 32) {
        if (j == i) continue;
        const int4 bb = __ldcg(xlist + j);
        const int nl = a.y + bb.y;
        const int nc = (int)((unsigned)a.z * (unsigned)bb.z);
        const int nh = a.w + bb.w;
        const int4 cur = __ldcg(row + bb.x);
        if (cur.x == kAbsentLen) {
          row[bb.x] = make_int4(nl, nc, nh, 0);
          added++;
        } else if (nl < cur.x) {
          row[bb.x] = make_int4(nl, nc, nh, 0);
        } else if (nl == cur.x) {
          row[bb.x] = make_int4(cur.x, (int)((unsigned)cur.y + (unsigned)nc), max(cur.z, nh), 0);
        }
      }
      added = __reduce_add_sync(kFull, added);
      if (lane == 0) {
        row[x] = make_int4(kAbsentLen, 0, 0, 0);
        deg[a.x] = __ldcg(deg + a.x) + added - 1;
      }
    }
    if (!dense_grid_sync(ctl, gen)) return;
  }
}

// device buffers freed on every exit of the function that owns them
struct DevBufs {
  std::vector<void *> p;
  DevBufs() = default;
  DevBufs(const DevBufs &) = delete;
  DevBufs &operator=(const DevBufs &) = delete;
  ~DevBufs() {
    for (void *q : p) cudaFree(q);
  }
  template <class T>
  T *get(size_t count) {
    void *q = nullptr;
    CK(cudaMalloc(&q, std::max<size_t>(1, count) * sizeof(T)));
    p.push_back(q);
    return (T *)q;
  }
};

void device_dense_eliminate(int device, DenseTail &dt) {
  NvtxRange range("qbc.dense_eliminate");
  CK(cudaSetDevice(device));
  const int32_t r = dt.r;
  if (r <= 0) {
    dt.order.clear();
    dt.x_off.assign(1, 0);
    dt.x.clear();
    return;
  }
  const int64_t m = dt.off[r];
  const int64_t cap = std::max<int64_t>(1, (int64_t)r * (r - 1) / 2);  // every pair at most once
  DevBufs buf;
  int4 *M = buf.get<int4>((size_t)r * r);
  int32_t *deg = buf.get<int32_t>(r);
  uint8_t *alive = buf.get<uint8_t>(r);
  int32_t *order = buf.get<int32_t>(r);
  int4 *xlist = buf.get<int4>(r);
  int32_t *xcount = buf.get<int32_t>(1);
  int4 *sep = buf.get<int4>((size_t)cap);
  int64_t *sep_off = buf.get<int64_t>((size_t)r + 1);
  int32_t *row = buf.get<int32_t>((size_t)m);
  int4 *ent = buf.get<int4>((size_t)m);
  std::vector<int32_t> hrow((size_t)m), hdeg((size_t)r);
  for (int32_t i = 0; i < r; i++) {
    hdeg[i] = (int32_t)(dt.off[i + 1] - dt.off[i]);
    for (int64_t e = dt.off[i]; e < dt.off[i + 1]; e++) hrow[e] = i;
  }
  cudaStream_t st;
  CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  } sg{st};
  CK(cudaMemcpyAsync(row, hrow.data(), (size_t)m * 4, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(ent, dt.ent.data(), (size_t)m * 16, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(deg, hdeg.data(), (size_t)r * 4, cudaMemcpyHostToDevice, st));
  CK(cudaMemsetAsync(alive, 1, (size_t)r, st));
  CK(cudaMemsetAsync(sep_off, 0, sizeof(int64_t), st));
  k_dense_clear<<<148 * 8, 256, 0, st>>>(M, (int64_t)r * r);
  k_dense_scatter<<<148 * 8, 256, 0, st>>>(M, r, row, ent, m);
  CK(cudaGetLastError());
  // one cooperative launch for all r steps when one CTA per SM fits and covers the row's columns;
  // else two launches per step
  int per_sm = 0, sms = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_dense_tail, kTailThreads, 0));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  int coop = 0;
  CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device));
  const int grid = std::min(sms, std::max(32, (int)((r + kTailThreads - 1) / kTailThreads)));
  if (coop && per_sm >= 1 && (int64_t)grid * kTailThreads >= r) {
    unsigned long long *part_best = buf.get<unsigned long long>((size_t)grid);
    int32_t *part_cnt = buf.get<int32_t>((size_t)grid);
    DenseCtl *ctl = buf.get<DenseCtl>(1);
    CK(cudaMemsetAsync(ctl, 0, sizeof(DenseCtl), st));
    int32_t rr = r;
    void *args[] = {&M, &deg, &alive, &rr, &order, &xlist, &sep, &sep_off, &part_best, &part_cnt, &ctl};
    CK(cudaLaunchCooperativeKernel((const void *)k_dense_tail, dim3((unsigned)grid), dim3(kTailThreads), args, 0, st));
    DenseCtl hc{};
    CK(cudaMemcpyAsync(&hc, ctl, sizeof(DenseCtl), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (hc.err || hc.abort) throw Error(QBC_ECUDA, "dense elimination: a grid barrier wait ran out");
  } else {
    for (int32_t s = 0; s < r; s++) {
      k_dense_pick<<<1, kPickThreads, 0, st>>>(M, deg, alive, r, s, order, xlist, xcount, sep, sep_off);
      k_dense_update<<<148 * 4, 256, 0, st>>>(M, deg, r, xlist, xcount, order, s);
    }
  }
  CK(cudaGetLastError());
  dt.order.resize((size_t)r);
  dt.x_off.resize((size_t)r + 1);
  CK(cudaMemcpyAsync(dt.order.data(), order, (size_t)r * 4, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(dt.x_off.data(), sep_off, ((size_t)r + 1) * 8, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  const int64_t total = dt.x_off[r];
  if (total < 0 || total > cap) throw Error(QBC_ECUDA, "dense elimination: separator total out of range");
  dt.x.resize((size_t)total * 4);
  if (total) CK(cudaMemcpyAsync(dt.x.data(), sep, (size_t)total * 16, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
}

// ------------------------------------------------------------------------------- device row fill
// Label rows built on the device (TreeDecomp.cpp:388-450 semantics, as the host builders): node p's
// row only reads rows of its separator vertices and ancestors, which sit at smaller depth, so the
// rows of one depth are independent -- one launch per depth, one warp per node, lanes over the
// row's entries (coalesced reads of the separators' rows).
struct FillArgs {
  const int32_t *__restrict__ depth;
  const int32_t *__restrict__ parent;
  const int64_t *__restrict__ lab_off;
  const int64_t *__restrict__ sep_off;
  const int4 *__restrict__ sep;  // (tid of x, shortcut length, count bits, max hop)
  int32_t *dis;
  int2 *ch;
  int32_t *anc;  // H2H only: ancestor id of each entry (the H2H fill reads rows of ancestors below x)
};

// Merge of one separator's candidate into an entry: shorter replaces, equal adds the count and
// keeps the larger hop (TreeDecomp.cpp:157-193); order-free, so any order of separators gives the
// sequential merge's entry.
template <bool MHL>
__device__ __forceinline__ void fill_merge(int &best, unsigned &c, int &hp, int nd, unsigned nc, int nh) {
  if (nd < best) {
    best = nd;
    c = nc;
    hp = nh;
  } else if (MHL && nd == best) {
    c += nc;
    hp = max(hp, nh);
  }
}

// Entries of a row filled per thread: the separator entries' row loads are issued kFillBatch at a
// time before any is merged, so a thread waits for one round of L2/DRAM latency per batch instead
// of one per separator vertex (the loop was latency-bound: 1M build, 2.9 s of fill kernels).
constexpr int kFillBatch = 8;
constexpr int kFillWarpSpan = 128;  // row entries per warp task of k_fill_level

// A separator entry as the fill reads it: (shortcut length, count bits, max hop), the vertex's
// row offset and depth - 1.
struct FillSep {
  int len;
  unsigned cnt;
  int hop, k;
  long long xoff;
};

// Entry j of a row from separator entries sep(0..nx): MHL reads x's own row at j (ancestors of x
// at depth > k contribute nothing); H2H reads, for ancestors j below x, the ancestor's row at k.
template <bool MHL, class GET>
__device__ __forceinline__ void fill_entry(const FillArgs &f, int j, int64_t ajoff, int nx, GET sep, int &best,
                                           unsigned &c, int &hp) {
  for (int i0 = 0; i0 < nx; i0 += kFillBatch) {
    int dv[kFillBatch];
    int2 cv[kFillBatch];
    FillSep x[kFillBatch];
#pragma unroll
    for (int q = 0; q < kFillBatch; q++) {
      x[q] = sep(min(i0 + q, nx - 1));
      const bool in = i0 + q < nx;
      const bool own = j <= x[q].k;
      const bool use = in && (own || !MHL);
      const int64_t xo = own ? x[q].xoff + j : ajoff + x[q].k;
      dv[q] = use ? f.dis[xo] : 0;
      if (MHL) cv[q] = use ? f.ch[xo] : make_int2(0, 0);
      if (!use) x[q].k = INT_MIN;  // marks the slot unused
    }
#pragma unroll
    for (int q = 0; q < kFillBatch; q++) {
      if (x[q].k == INT_MIN) continue;
      if (MHL)
        fill_merge<true>(best, c, hp, x[q].len + dv[q], x[q].cnt * (unsigned)cv[q].x, x[q].hop + cv[q].y);
      else
        fill_merge<false>(best, c, hp, x[q].len + dv[q], 0u, 0);
    }
  }
}

// One launch per tree depth k (all its nodes have rows of k entries); a warp takes one node's
// entries [span * kFillWarpSpan, ...) so that long rows of few nodes still spread over many warps.
// The node's separator entries (fewer than kBigSeparator here, else as many as needed) are staged
// 32 at a time in registers, lane i holding entry i, and handed round by shuffles.
template <bool MHL>
__global__ void __launch_bounds__(256) k_fill_level(FillArgs f, const int32_t *__restrict__ nodes, int count, int spans) {
  const int w = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (w >= count * spans) return;
  const int p = nodes[w / spans];
  const int jlo = (w % spans) * kFillWarpSpan;
  const int h = f.depth[p];
  if (jlo >= h) return;
  const int jhi = min(h, jlo + kFillWarpSpan);
  const int64_t off = f.lab_off[p];
  if (!MHL) {  // H2H: ancestor ids of this span (the parent's row plus p), read below by the same lane
    const int par = f.parent[p];
    const int64_t poff = par >= 0 ? f.lab_off[par] : 0;
    for (int j = jlo + lane; j < jhi; j += 32) f.anc[off + j] = (j < h - 1) ? f.anc[poff + j] : p;
  }
  const int64_t sb = f.sep_off[p];
  const int nx = (int)(f.sep_off[p + 1] - sb);
  for (int jb = jlo; jb < jhi; jb += 32) {
    const int j = jb + lane;
    const bool live = j < h - 1;
    int best = kInfDist;
    unsigned c = 0;
    int hp = 0;
    const int64_t ajoff = (!MHL && live) ? f.lab_off[f.anc[off + j]] : 0;
    for (int base = 0; base < nx; base += 32) {
      FillSep mine{0, 0u, 0, -1, 0};
      if (base + lane < nx) {
        const int4 xs = f.sep[sb + base + lane];
        mine = FillSep{xs.y, (unsigned)xs.z, xs.w, f.depth[xs.x] - 1, (long long)f.lab_off[xs.x]};
      }
      const int cnt = min(32, nx - base);
      auto get = [&](int i) {
        return FillSep{__shfl_sync(kFull, mine.len, i), (unsigned)__shfl_sync(kFull, (int)mine.cnt, i),
                       __shfl_sync(kFull, mine.hop, i), __shfl_sync(kFull, mine.k, i),
                       __shfl_sync(kFull, mine.xoff, i)};
      };
      // every lane runs the batches (the shuffles need the whole warp); lanes past the row's last
      // separator-filled entry merge nothing
      int b2 = best;
      unsigned c2 = c;
      int h2 = hp;
      fill_entry<MHL>(f, live ? j : 0, ajoff, cnt, get, b2, c2, h2);
      if (live) {
        best = b2;
        c = c2;
        hp = h2;
      }
    }
    if (live) {
      f.dis[off + j] = best;
      if (MHL) f.ch[off + j] = make_int2((int)c, hp);
    } else if (j == h - 1) {  // p's own entry
      f.dis[off + j] = 0;
      if (MHL) f.ch[off + j] = make_int2(1, 0);
    }
  }
}

// The same fill for nodes with large separators (near the root): a CTA per (node, block of
// blockDim.x entries), the separator entries with their vertices' row offsets and depths staged
// in shared memory, a thread per entry.
constexpr int kBigSeparator = 32;  // separators of at least this size take the CTA form
constexpr int kFillStageBytes = 24;  // shared bytes per staged separator entry (FillSep)

template <bool MHL>
__global__ void __launch_bounds__(256) k_fill_node_cta(FillArgs f, const int32_t *__restrict__ nodes) {
  extern __shared__ FillSep fsm_sep[];
  const int p = nodes[blockIdx.y];
  const int h = f.depth[p];
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if ((int)(blockIdx.x * blockDim.x) >= h) return;  // whole CTA, before the barrier
  const int64_t off = f.lab_off[p];
  const int64_t sb = f.sep_off[p];
  const int nx = (int)(f.sep_off[p + 1] - sb);
  for (int i = threadIdx.x; i < nx; i += blockDim.x) {
    const int4 x = f.sep[sb + i];
    fsm_sep[i] = FillSep{x.y, (unsigned)x.z, x.w, f.depth[x.x] - 1, (long long)f.lab_off[x.x]};
  }
  int64_t ajoff = 0;
  if (!MHL && j < h) {  // H2H: this entry's ancestor (the parent's row plus p), read below by this thread
    const int par = f.parent[p];
    const int64_t poff = par >= 0 ? f.lab_off[par] : 0;
    const int a = (j < h - 1) ? f.anc[poff + j] : p;
    f.anc[off + j] = a;
    ajoff = f.lab_off[a];
  }
  __syncthreads();
  if (j < h - 1) {
    int best = kInfDist;
    unsigned c = 0;
    int hp = 0;
    fill_entry<MHL>(f, j, ajoff, nx, [&](int i) { return fsm_sep[i]; }, best, c, hp);
    f.dis[off + j] = best;
    if (MHL) f.ch[off + j] = make_int2((int)c, hp);
  } else if (j == h - 1) {
    f.dis[off + j] = 0;
    if (MHL) f.ch[off + j] = make_int2(1, 0);
  }
}

// x[i] <<= bits in place (the packed-key scan's pre-shifted label distances)
__global__ void k_shift_left(int32_t *x, int64_t n, int bits) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] = (int32_t)((uint32_t)x[i] << bits);
}

__global__ void k_max_i32(const int32_t *__restrict__ x, int64_t n, int32_t *out) {
  int m = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) m = max(m, x[i]);
  m = __reduce_max_sync(kFull, m);
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// ------------------------------------------------------------------------------- upload
// Per vertex its first four arcs in CSR order as (head, weight) pairs in two int4 (one 32-byte
// sector: the dependency pass reads a vertex's arcs with one request instead of a range lookup and
// four pair loads).  Missing arcs have head -1.  A vertex with more than four arcs keeps three in
// place and puts (~e, end) in the fourth pair: its remaining arcs are arc_hw[e, end), e >= 3.
static std::vector<int4> arc4_of(const std::vector<int32_t> &off, const std::vector<int32_t> &head,
                                 const std::vector<int32_t> &w) {
  const size_t n = off.empty() ? 0 : off.size() - 1;
  std::vector<int4> out(2 * n);
  for (size_t v = 0; v < n; v++) {
    int32_t p[8];
    for (int q = 0; q < 4; q++) {
      p[2 * q] = -1;
      p[2 * q + 1] = 0;
    }
    const int32_t b = off[v], e = off[v + 1];
    const int inl = e - b > 4 ? 3 : e - b;
    for (int q = 0; q < inl; q++) {
      p[2 * q] = head[b + q];
      p[2 * q + 1] = w[b + q];
    }
    if (e - b > 4) {
      p[6] = ~(b + 3);
      p[7] = e;
    }
    out[2 * v] = make_int4(p[0], p[1], p[2], p[3]);
    out[2 * v + 1] = make_int4(p[4], p[5], p[6], p[7]);
  }
  return out;
}

static DeviceState *new_state(Handle &h, int device) {
  device_release(h);
  const Index &ix = h.host;
  CK(cudaSetDevice(device));
  DeviceState *d = new DeviceState();
  h.dev = d;
  d->device = device;
  CK(cudaStreamCreateWithFlags(&d->s_label, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&d->s_dep, cudaStreamNonBlocking));
  for (int b = 0; b < 2; b++) {
    CK(cudaEventCreateWithFlags(&d->ev_label[b], cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&d->ev_dep[b], cudaEventDisableTiming));
  }
  CK(cudaEventCreateWithFlags(&d->ev_start, cudaEventDisableTiming));
  CK(cudaDeviceGetAttribute(&d->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
  // the dependency pass wants L1, not shared memory: 3 CTAs x 9.5 KB fit the 32 KB carveout
  // (14 % of 228 KB), which leaves 224 KB of L1 instead of the 192 KB the driver picks by itself
  // (76.6 vs 78.8 ms per all-source step at 50k)
  CK(cudaFuncSetAttribute(k_dependency_cta_pipe<false>, cudaFuncAttributePreferredSharedMemoryCarveout, 14));
  CK(cudaFuncSetAttribute(k_dependency_cta_pipe<true>, cudaFuncAttributePreferredSharedMemoryCarveout, 14));
  d->n = ix.n;
  d->n_pad = (ix.n + 7) & ~7;
  int S = (ix.tree_height + 3) & ~3;
  if (((S / 4) & 1) == 0) S += 4;  // odd number of 16-byte groups: conflict-free LDS.128 across rows
  d->hmax_pad = S;
  cudaStream_t st = d->s_label;
  d->depth = dupload(d, ix.depth, st);
  d->send = dupload(d, ix.send, st);
  d->arc_off = dupload(d, ix.arc_off, st);
  d->arc_head = dupload(d, ix.arc_head, st);
  d->arc_w = dupload(d, ix.arc_w, st);
  {
    std::vector<int2> rng((size_t)ix.n), hw(ix.arc_head.size());
    for (int32_t v = 0; v < ix.n; v++) rng[v] = make_int2(ix.arc_off[v], ix.arc_off[v + 1]);
    for (size_t e = 0; e < hw.size(); e++) hw[e] = make_int2(ix.arc_head[e], ix.arc_w[e]);
    d->arc_rng = dupload(d, rng, st);
    d->arc_hw = dupload(d, hw, st);
    const std::vector<int4> a4 = arc4_of(ix.arc_off, ix.arc_head, ix.arc_w);
    d->arc4 = dupload(d, a4, st);
    CK(cudaStreamSynchronize(st));  // the staging vectors die here
  }
  d->vid_of = dupload(d, ix.vid_of, st);
  d->tid_of = dupload(d, ix.tid_of, st);
  d->parent = dupload(d, ix.parent, st);
  d->lab_off = dupload(d, ix.lab_off, st);
  {
    double wsum = 0.0;
    for (int32_t x : ix.arc_w) wsum += x;
    const double mean = ix.arc_w.empty() ? 1.0 : wsum / (double)ix.arc_w.size();
    d->sweep_delta_auto = (int32_t)std::min(1.0 * (1 << 28), std::max(1.0, 2.0 * mean));
  }
  return d;
}

static void finish_state(Handle &h, DeviceState *d) {
  const Index &ix = h.host;
  cudaStream_t st = d->s_label;
  {
    // packed keys (dist << B) | j need every row index below 2^B and 2*max_label + 1 < 2^(32-B)
    int B = 1;
    while ((1 << B) < ix.tree_height) B++;
    const uint64_t room = (uint64_t)1 << (32 - B);
    d->packed_bits = (ix.kind != IndexKind::CSR && B <= 16 && 2ull * (uint64_t)std::max(ix.max_label, 0) + 2 < room) ? B : 0;
  }
  if (d->packed_bits) {  // label distances pre-shifted by B, in place (one add per entry in the scan)
    const int64_t L = ix.lab_off[ix.n];
    k_shift_left<<<148 * 8, 256, 0, st>>>(d->dis, L, d->packed_bits);
    CK(cudaGetLastError());
    d->dis_sh = d->dis;
  }
  alloc_scratch(h, d);
  d->bc_tid = dmalloc<double>(d, ix.n);
  d->bc_vid = dmalloc<double>(d, ix.n);
  d->err = dmalloc<int32_t>(d, 1);
  d->grid_ctl = dmalloc<int32_t>(d, kGridCtlBytes / 4);
  CK(cudaMemsetAsync(d->err, 0, 4, st));
  CK(cudaStreamSynchronize(st));
}

void device_upload(Handle &h, int device) {
  NvtxRange nvtx("qbc.upload");
  if (!h.host.rows_on_host) {
    if (!h.dev) throw Error(QBC_EINVAL, "index rows exist only on a released device");
    device_download_rows(h);
  }
  const Index &ix = h.host;
  DeviceState *d = nullptr;
  try {
    d = new_state(h, device);
    cudaStream_t st = d->s_label;
    d->dis = dupload(d, ix.dis, st);  // ancestor ids and subtree ends stay on the host
    if (ix.kind == IndexKind::MHL) {
      d->ch = dmalloc<int2>(d, ix.ch.size() / 2);
      CK(cudaMemcpyAsync(d->ch, ix.ch.data(), ix.ch.size() * 4, cudaMemcpyHostToDevice, st));
    }
    finish_state(h, d);
  } catch (...) {
    device_release(h);
    throw;
  }
}

void device_build(Handle &h, int device, const Separators &seps) {
  NvtxRange nvtx("qbc.build_device");
  Index &ix = h.host;
  try {
    DeviceState *d = nullptr;
    {
      TraceScope t("device state and arc upload");
      d = new_state(h, device);
      CK(cudaStreamSynchronize(d->s_label));
    }
    auto t_fill = std::make_unique<TraceScope>("row buffers and separator upload");
    cudaStream_t st = d->s_label;
    const int64_t L = ix.lab_off[ix.n];
    d->dis = dmalloc<int32_t>(d, (size_t)L);
    CK(cudaMemsetAsync(d->dis, 0, (size_t)L * 4, st));

    const bool mhl = ix.kind == IndexKind::MHL;
    if (mhl) {
      d->ch = dmalloc<int2>(d, (size_t)L);
      CK(cudaMemsetAsync(d->ch, 0, (size_t)L * 8, st));
    }
    // nodes grouped by depth (counting sort; preorder keeps each level in increasing tid order);
    // within a level, nodes with small separators first (a warp per 128 entries of a node's row),
    // then large ones (a CTA per 256 entries, separators staged in shared memory; beyond the
    // staging capacity they stay warp-filled)
    const int64_t stage_cap = std::max(kBigSeparator, (d->smem_optin - 1024) / kFillStageBytes);
    auto big = [&](int32_t t) {
      const int64_t nx = seps.off[t + 1] - seps.off[t];
      return nx >= kBigSeparator && nx <= stage_cap;
    };
    std::vector<int64_t> lvl((size_t)ix.tree_height + 2, 0), nbig((size_t)ix.tree_height + 2, 0),
        maxsep((size_t)ix.tree_height + 2, 0);
    for (int32_t t = 0; t < ix.n; t++) {
      lvl[ix.depth[t] + 1]++;
      if (big(t)) {
        nbig[ix.depth[t]]++;
        maxsep[ix.depth[t]] = std::max(maxsep[ix.depth[t]], seps.off[t + 1] - seps.off[t]);
      }
    }
    for (size_t k = 1; k < lvl.size(); k++) lvl[k] += lvl[k - 1];
    std::vector<int32_t> nodes((size_t)ix.n);
    {
      std::vector<int64_t> fs(lvl.begin(), lvl.end() - 1), fb((size_t)ix.tree_height + 2, 0);
      for (size_t k = 0; k + 1 < lvl.size(); k++) fb[k] = lvl[k + 1] - nbig[k];
      for (int32_t t = 0; t < ix.n; t++) {
        if (big(t)) nodes[fb[ix.depth[t]]++] = t;
        else nodes[fs[ix.depth[t]]++] = t;
      }
    }
    // temporaries of the fill, freed at the end; per-entry ancestor ids (f_anc) only for H2H,
    // whose fill reads rows of ancestors below a separator vertex (MHL rows read only the
    // separator vertices' own rows)
    int32_t *d_nodes = nullptr, *d_max = nullptr, *f_anc = nullptr;
    int64_t *d_soff = nullptr;
    int4 *d_sep = nullptr;
    auto free_tmp = [&] {
      void *q[] = {d_nodes, d_max, d_soff, d_sep, f_anc};
      for (void *p : q)
        if (p) cudaFree(p);
    };
    try {
      CK(cudaMalloc(&d_nodes, nodes.size() * 4));
      if (!mhl) {
        CK(cudaMalloc(&f_anc, (size_t)std::max<int64_t>(L, 1) * 4));
        CK(cudaMemsetAsync(f_anc, 0, (size_t)L * 4, st));
      }
      CK(cudaMalloc(&d_soff, seps.off.size() * 8));
      CK(cudaMalloc(&d_sep, std::max<size_t>(16, seps.ent.size() * 4)));
      CK(cudaMalloc(&d_max, 4));
      CK(cudaMemcpyAsync(d_nodes, nodes.data(), nodes.size() * 4, cudaMemcpyHostToDevice, st));
      CK(cudaMemcpyAsync(d_soff, seps.off.data(), seps.off.size() * 8, cudaMemcpyHostToDevice, st));
      if (!seps.ent.empty()) CK(cudaMemcpyAsync(d_sep, seps.ent.data(), seps.ent.size() * 4, cudaMemcpyHostToDevice, st));
      CK(cudaMemsetAsync(d_max, 0, 4, st));
      FillArgs f{d->depth, d->parent, d->lab_off, d_soff, d_sep, d->dis, d->ch, f_anc};
      if (TraceScope::enabled()) {  // split the phase: buffers and upload, then the fill kernels
        CK(cudaStreamSynchronize(st));
        t_fill = std::make_unique<TraceScope>("device row fill kernels");
      }
      const size_t max_stage = (size_t)stage_cap * kFillStageBytes;
      CK(cudaFuncSetAttribute(k_fill_node_cta<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_stage));
      CK(cudaFuncSetAttribute(k_fill_node_cta<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_stage));
      for (int32_t k = 1; k <= ix.tree_height; k++) {
        const int count = (int)(lvl[k + 1] - lvl[k] - nbig[k]);
        if (count > 0) {
          const int spans = (k + kFillWarpSpan - 1) / kFillWarpSpan;  // rows at depth k have k entries
          const int blocks = (int)(((int64_t)count * spans + 7) / 8);
          if (mhl) k_fill_level<true><<<blocks, 256, 0, st>>>(f, d_nodes + lvl[k], count, spans);
          else k_fill_level<false><<<blocks, 256, 0, st>>>(f, d_nodes + lvl[k], count, spans);
          CK(cudaGetLastError());
        }
        if (nbig[k] > 0) {
          const size_t smem = (size_t)maxsep[k] * kFillStageBytes;
          const dim3 grid((unsigned)((k + 255) / 256), (unsigned)nbig[k]);
          if (mhl) k_fill_node_cta<true><<<grid, 256, smem, st>>>(f, d_nodes + lvl[k + 1] - nbig[k]);
          else k_fill_node_cta<false><<<grid, 256, smem, st>>>(f, d_nodes + lvl[k + 1] - nbig[k]);
          CK(cudaGetLastError());
        }
      }
      k_max_i32<<<148 * 4, 256, 0, st>>>(d->dis, L, d_max);
      CK(cudaGetLastError());
      int32_t mx = 0;
      CK(cudaMemcpyAsync(&mx, d_max, 4, cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      ix.max_label = mx;
    } catch (...) {
      free_tmp();
      throw;
    }
    free_tmp();
    ix.rows_on_host = false;
    ix.dis.clear();
    ix.ch.clear();
    ix.anc.clear();
    ix.aend.clear();
    t_fill.reset();
    TraceScope t_fin("per-source scratch");
    finish_state(h, d);
    if (TraceScope::enabled()) CK(cudaDeviceSynchronize());
  } catch (...) {
    device_release(h);
    throw;
  }
}

void device_download_rows(Handle &h) {
  Index &ix = h.host;
  if (ix.rows_on_host) return;
  DeviceState *d = h.dev;
  if (!d) throw Error(QBC_EINVAL, "index rows exist only on a released device");
  CK(cudaSetDevice(d->device));
  const size_t L = (size_t)ix.lab_off[ix.n];
  ix.dis.resize(L);
  CK(cudaMemcpy(ix.dis.data(), d->dis, L * 4, cudaMemcpyDeviceToHost));
  if (d->packed_bits)  // the device keeps them shifted for the packed-key scan
    for (int32_t &x : ix.dis) x = (int32_t)((uint32_t)x >> d->packed_bits);
  fill_ancestor_rows(ix);  // not kept on the device: rebuilt from the parent links
  if (ix.kind == IndexKind::MHL) {
    ix.ch.resize(2 * L);
    CK(cudaMemcpy(ix.ch.data(), d->ch, L * 8, cudaMemcpyDeviceToHost));
  }
  ix.rows_on_host = true;
}

void device_release(Handle &h) {
  DeviceState *d = h.dev;
  if (!d) return;
  cudaSetDevice(d->device);
  cudaDeviceSynchronize();
  void *ptrs[] = {d->depth, d->send, d->arc_off, d->arc_head, d->arc_w, d->arc_rng, d->arc_hw, d->arc4, d->vid_of, d->tid_of, d->parent,
                  d->lab_off, d->dis, d->ch, d->bc_tid, d->bc_vid, d->err, d->grid_ctl, d->sources,
                  d->dsrc_tid, d->dsrc_sorted, d->dsrc_tmp};  // dis_sh aliases dis
  for (void *p : ptrs)
    if (p) cudaFree(p);
  free_scratch(d);
  for (int b = 0; b < 2; b++) {
    if (d->ev_label[b]) cudaEventDestroy(d->ev_label[b]);
    if (d->ev_dep[b]) cudaEventDestroy(d->ev_dep[b]);
  }
  if (d->ev_start) cudaEventDestroy(d->ev_start);
  for (auto &e : d->ev_lab) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
  for (auto &e : d->ev_dp) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
  if (d->s_label) cudaStreamDestroy(d->s_label);
  if (d->s_dep) cudaStreamDestroy(d->s_dep);
  delete d;
  h.dev = nullptr;
}

int64_t device_bytes(const Handle &h) { return h.dev ? h.dev->bytes : 0; }
int device_id(const Handle &h) { return h.dev ? h.dev->device : -1; }

DeviceState *need_dev(Handle &h) {
  if (!h.dev) throw Error(QBC_EINVAL, "index is not on a device: call qbc_index_upload first");
  if (h.server) throw Error(QBC_EBUSY, "the index is serving requests: close its server first");
  CK(cudaSetDevice(h.dev->device));
  return h.dev;
}

void check_err(DeviceState *d) {
  int32_t e = 0;
  CK(cudaMemcpy(&e, d->err, 4, cudaMemcpyDeviceToHost));
  if (e != ERR_NONE) {
    CK(cudaMemset(d->err, 0, 4));
    throw Error(QBC_EDEVICE, e == ERR_DISCONNECTED ? "device: SP-DAG wave pass did not reach every vertex"
                             : e == ERR_BAD_SOURCE ? "device: source id out of range"
                             : e == ERR_COPY_TIMEOUT ? "device: label-row copy wait ran out"
                             : e == ERR_SWEEP_BOUND ? "device: shortest-path sweep ran past its pass bound"
                                                   : "device: kernel error word " + std::to_string(e));
  }
}

// ------------------------------------------------------------------------------- drivers
// A device source list as tids in tree order, on stream st: the label kernels give consecutive
// sources to one CTA, and sources of one subtree share most of their ancestors, so a CTA's scans
// end at similar depths and its target rows are fetched to similar depths (1M grid, 4,096 random
// sources, tall-tree kernel: 1,874 ms per step in tid order against 2,593 ms in vid order).  The
// host entry points sort on the host; here the tids are sorted on the device (a radix sort of ns
// keys over the bits of n - 1).  Buffers grow on demand and stay with the index.
static const int32_t *device_sources_tid_order(DeviceState *d, const int32_t *d_sources0, int32_t ns, cudaStream_t st) {
  int bits = 1;
  while (bits < 31 && ((d->n - 1) >> bits) != 0) bits++;
  size_t tmp = 0;
  CK(cub::DeviceRadixSort::SortKeys(nullptr, tmp, (const int32_t *)nullptr, (int32_t *)nullptr, ns, 0, bits, st));
  if (ns > d->dsrc_cap || tmp > d->dsrc_tmp_bytes) {
    CK(cudaStreamSynchronize(st));
    for (void *p : {(void *)d->dsrc_tid, (void *)d->dsrc_sorted, d->dsrc_tmp})
      if (p) cudaFree(p);
    d->bytes -= (int64_t)d->dsrc_cap * 8 + (int64_t)d->dsrc_tmp_bytes;
    d->dsrc_tid = d->dsrc_sorted = nullptr;
    d->dsrc_tmp = nullptr;
    d->dsrc_cap = 0;
    d->dsrc_tmp_bytes = 0;
    const int32_t cap = std::max(ns, d->dsrc_cap);
    d->dsrc_tid = dmalloc<int32_t>(d, (size_t)cap);
    d->dsrc_sorted = dmalloc<int32_t>(d, (size_t)cap);
    d->dsrc_tmp = dmalloc<unsigned char>(d, tmp);
    d->dsrc_cap = cap;
    d->dsrc_tmp_bytes = std::max<size_t>(1, tmp);
  }
  k_vid_to_tid<<<(ns + 255) / 256, 256, 0, st>>>(d_sources0, d->tid_of, d->dsrc_tid, ns, d->n, d->err);
  CK(cudaGetLastError());
  d->launches++;
  size_t have = d->dsrc_tmp_bytes;
  CK(cub::DeviceRadixSort::SortKeys(d->dsrc_tmp, have, d->dsrc_tid, d->dsrc_sorted, ns, 0, bits, st));
  return d->dsrc_sorted;
}

void device_bc_sources(Handle &h, const int32_t *d_sources0, int32_t ns, double *d_bc_vid, void *stream) {
  NvtxRange nvtx("qbc.bc_sources_device");
  DeviceState *d = need_dev(h);
  cudaStream_t user = stream ? (cudaStream_t)stream : d->s_label;
  CK(cudaEventRecord(d->ev_start, user));
  CK(cudaStreamWaitEvent(d->s_label, d->ev_start, 0));
  CK(cudaStreamWaitEvent(d->s_dep, d->ev_start, 0));
  CK(cudaMemsetAsync(d->bc_tid, 0, (size_t)d->n * 8, d->s_label));
  CK(cudaEventRecord(d->ev_label[1], d->s_label));
  CK(cudaStreamWaitEvent(d->s_dep, d->ev_label[1], 0));
  const int32_t *tids = ns > 0 ? device_sources_tid_order(d, d_sources0, ns, d->s_label) : nullptr;
  for (int32_t off = 0; off < ns; off += d->chunk) {
    const int b = 0;  // stream order frees the buffer for the next chunk
    const int32_t cnt = std::min(d->chunk, ns - off);
    launch_label(h, d, b, tids + off, cnt, false, d->s_label, dep_reads_hops(h));
    // The dependency pass runs right after the scan on the same stream: run concurrently on a
    // second stream the two kernels thrash each other's caches and both slow down ~2x.
    launch_dep(h, d, b, tids + off, cnt, d->s_label);
  }
  CK(cudaEventRecord(d->ev_dep[0], d->s_label));
  CK(cudaStreamWaitEvent(user, d->ev_dep[0], 0));
  k_tid_to_vid_f64<<<(d->n + 255) / 256, 256, 0, user>>>(d->bc_tid, d->vid_of, d_bc_vid, d->n, 1);
  CK(cudaGetLastError());
  d->launches++;
}

void device_profiling(Handle &h, bool on) {
  DeviceState *d = need_dev(h);
  d->profiling = on;
  d->ev_lab_used = d->ev_dp_used = 0;
  d->label_ms = d->dep_ms = 0.0;
  d->label_launches = d->dep_launches = d->launches = 0;
}

void device_stats(Handle &h, double *out) {
  DeviceState *d = need_dev(h);
  CK(cudaDeviceSynchronize());
  for (size_t i = 0; i < d->ev_lab_used; i++) {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, d->ev_lab[i].first, d->ev_lab[i].second));
    d->label_ms += ms;
  }
  for (size_t i = 0; i < d->ev_dp_used; i++) {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, d->ev_dp[i].first, d->ev_dp[i].second));
    d->dep_ms += ms;
  }
  d->ev_lab_used = d->ev_dp_used = 0;
  out[0] = d->label_ms;
  out[1] = (double)d->label_launches;
  out[2] = d->dep_ms;
  out[3] = (double)d->dep_launches;
  out[4] = (double)d->launches;
}

int32_t device_label_group(Handle &h) {
  DeviceState *d = need_dev(h);
  if (h.host.kind == IndexKind::CSR) return 0;
  if (use_packed(h, d, false)) return tall_warps(h, d) ? kTallSources : 32;
  return plan_label(h, d, std::max(1, d->chunk), false).G;
}

const char *device_label_kernel(Handle &h) {
  DeviceState *d = need_dev(h);
  if (h.host.kind == IndexKind::CSR) return "k_sweep_rows";
  if (!use_packed(h, d, false)) return "k_label_scan";
  const TallCfg tc = tall_cfg(h, d);
  if (tc.warps) return tc.whole ? "k_label_scan_rows16" : "k_label_scan_tall";
  return packed_warps(h, d) == 12 ? "k_label_scan_pair" : "k_label_scan_packed";
}

static int32_t *stage_sources(DeviceState *d, const int32_t *sources0, int32_t ns, int32_t n) {
  for (int32_t i = 0; i < ns; i++)
    if (sources0[i] < 0 || sources0[i] >= n) throw Error(QBC_EINVAL, "source id " + std::to_string(sources0[i]) + " out of range");
  if (ns > d->sources_cap) {
    if (d->sources) cudaFree(d->sources);
    d->sources = nullptr;
    d->sources = dmalloc<int32_t>(d, (size_t)ns);
    d->sources_cap = ns;
  }
  if (ns) CK(cudaMemcpyAsync(d->sources, sources0, (size_t)ns * 4, cudaMemcpyHostToDevice, d->s_label));
  return d->sources;
}

// host list, sorted by tid so each CTA's sources are neighbours in the tree
static std::vector<int32_t> tid_sorted(const Index &ix, const int32_t *sources0, int32_t ns) {
  std::vector<int32_t> v(sources0, sources0 + ns);
  for (int32_t x : v)
    if (x < 0 || x >= ix.n) throw Error(QBC_EINVAL, "source id " + std::to_string(x) + " out of range");
  std::sort(v.begin(), v.end(), [&](int32_t a, int32_t b) { return ix.tid_of[a] < ix.tid_of[b]; });
  return v;
}

void host_bc_sources(Handle &h, const int32_t *sources0, int32_t ns, double *bc_out) {
  NvtxRange nvtx("qbc.bc_sources");
  DeviceState *d = need_dev(h);
  std::vector<int32_t> srt = tid_sorted(h.host, sources0, ns);
  int32_t *ds = stage_sources(d, srt.data(), ns, d->n);
  CK(cudaMemsetAsync(d->bc_vid, 0, (size_t)d->n * 8, d->s_label));
  device_bc_sources(h, ds, ns, d->bc_vid, d->s_label);
  CK(cudaMemcpyAsync(bc_out, d->bc_vid, (size_t)d->n * 8, cudaMemcpyDeviceToHost, d->s_label));
  CK(cudaStreamSynchronize(d->s_label));
  check_err(d);
}

void host_bc_plain(Handle &h, const int32_t *sources0, int32_t ns, double *bc_out) {
  NvtxRange nvtx("qbc.bc_plain");
  DeviceState *d = need_dev(h);
  int32_t *ds = stage_sources(d, sources0, ns, d->n);
  cudaStream_t st = d->s_label;
  CK(cudaMemsetAsync(d->bc_tid, 0, (size_t)d->n * 8, st));
  for (int32_t i = 0; i < ns; i++) {
    k_vid_to_tid<<<1, 32, 0, st>>>(ds + i, d->tid_of, d->src[0], 1, d->n, d->err);
    CK(cudaGetLastError());
    launch_label(h, d, 0, d->src[0], 1, true, st);
    launch_dep(h, d, 0, d->src[0], 1, st, true);
  }
  k_tid_to_vid_f64<<<(d->n + 255) / 256, 256, 0, st>>>(d->bc_tid, d->vid_of, d->bc_vid, d->n, 0);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(bc_out, d->bc_vid, (size_t)d->n * 8, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  check_err(d);
}

void host_rows(Handle &h, const int32_t *sources0, int32_t ns, int32_t *dist, uint32_t *cnt, int32_t *hop) {
  NvtxRange nvtx("qbc.rows");
  DeviceState *d = need_dev(h);
  cudaStream_t st = d->s_label;
  const int32_t n = d->n;
  int32_t *o_d = nullptr, *o_h = nullptr;
  uint32_t *o_c = nullptr;
  const int32_t step = std::min<int32_t>(d->chunk, 256);
  o_d = dmalloc<int32_t>(d, (size_t)step * n);
  if (cnt) o_c = dmalloc<uint32_t>(d, (size_t)step * n);
  if (hop) o_h = dmalloc<int32_t>(d, (size_t)step * n);
  try {
    int32_t *ds = stage_sources(d, sources0, ns, n);
    for (int32_t off = 0; off < ns; off += step) {
      const int32_t c = std::min(step, ns - off);
      k_vid_to_tid<<<(c + 255) / 256, 256, 0, st>>>(ds + off, d->tid_of, d->src[0], c, n, d->err);
      CK(cudaGetLastError());
      launch_label(h, d, 0, d->src[0], c, false, st);
      if (h.host.kind == IndexKind::H2H && (cnt || hop)) {
        // sigma and waves by the Kahn pass; BC accumulation goes to a scratch target
        CK(cudaMemsetAsync(d->bc_tid, 0, (size_t)n * 8, st));
        launch_dep(h, d, 0, d->src[0], c, st);
      }
      dim3 grid((n + 255) / 256, c);
      k_rows_to_vid<<<grid, 256, 0, st>>>(d->rec[0], d->hop[0], d->vid_of, n, d->n_pad, c, o_d, o_c, o_h);
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(dist + (size_t)off * n, o_d, (size_t)c * n * 4, cudaMemcpyDeviceToHost, st));
      if (cnt) CK(cudaMemcpyAsync(cnt + (size_t)off * n, o_c, (size_t)c * n * 4, cudaMemcpyDeviceToHost, st));
      if (hop) CK(cudaMemcpyAsync(hop + (size_t)off * n, o_h, (size_t)c * n * 4, cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
    }
    check_err(d);
  } catch (...) {
    cudaFree(o_d); if (o_c) cudaFree(o_c); if (o_h) cudaFree(o_h);
    throw;
  }
  cudaFree(o_d);
  if (o_c) cudaFree(o_c);
  if (o_h) cudaFree(o_h);
  d->bytes -= (int64_t)step * n * 4 * (1 + (cnt ? 1 : 0) + (hop ? 1 : 0));
}

// ------------------------------------------------------------------ allocation-free single source
// qbc_bc_source_static: one source's BC contribution without any device allocation in the call.
// Some callers cannot allocate device memory at the point where they need BC: a host application
// whose memory manager has already reserved the GPU's memory (a framework's caching allocator),
// or a serving loop whose steady state must stay free of cudaMalloc/cudaFree because those calls
// synchronise the device and have unbounded latency.  For them the per-source scratch (distance /
// sigma pairs, hop layers, dependencies, level queue, layer counters, a BC accumulator) lives in
// this statically sized device array instead of the index's allocated scratch buffers.  Every GPU
// that loads the library holds it (kStaticScratchBytes, about 5 MiB) until the process exits.
constexpr int32_t kStaticMaxVertices = 1 << 17;  // largest graph the static scratch serves
constexpr size_t kStaticRec = 0;                                                    // int4[max]
constexpr size_t kStaticHop = kStaticRec + (size_t)kStaticMaxVertices * 16;         // int32[max]
constexpr size_t kStaticOrder = kStaticHop + (size_t)kStaticMaxVertices * 4;        // int32[max]
constexpr size_t kStaticLcnt = kStaticOrder + (size_t)kStaticMaxVertices * 4;       // int32[2*(max+2)]
constexpr size_t kStaticBc = kStaticLcnt + (((size_t)2 * (kStaticMaxVertices + 2) * 4 + 255) / 256) * 256;  // double[max]
constexpr size_t kStaticSrc = kStaticBc + (size_t)kStaticMaxVertices * 8;           // int32[64]
constexpr int32_t kStaticMaxHeight = 8192;  // source-row capacity (the label kernel's own limit is lower)
constexpr size_t kStaticSrcRows = kStaticSrc + 256;                                  // int32[2*height]
constexpr size_t kStaticScratchBytes = kStaticSrcRows + (size_t)2 * kStaticMaxHeight * 4;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

__global__ void k_static_set_source(int32_t *dst, int32_t tid) { *dst = tid; }

// Address of g_static_scratch on `device`.  The symbol name is only a host-side stand-in, so
// the device address is looked up once per device with that device current, and cached for the
// life of the process (a cudaDeviceReset that recreates the device's context invalidates it).
static unsigned char *static_scratch_on(int device) {
  static std::mutex mu;
  static std::vector<unsigned char *> cached;
  std::lock_guard<std::mutex> lock(mu);
  if (device < 0) throw Error(QBC_EINVAL, "bad device");
  if ((size_t)device >= cached.size()) cached.resize((size_t)device + 1, nullptr);
  if (!cached[device]) {
    int cur = -1;
    CK(cudaGetDevice(&cur));
    if (cur != device) throw Error(QBC_EINVAL, "static scratch set-up needs the index's device current");
    void *ptr = nullptr;
    CK(cudaGetSymbolAddress(&ptr, g_static_scratch));
    cached[device] = (unsigned char *)ptr;
  }
  return cached[device];
}

void host_bc_source_static(Handle &h, int32_t source0, double *d_bc_vid, void *stream) {
  if (h.host.n > kStaticMaxVertices)
    throw Error(QBC_EINVAL, "graph has " + std::to_string(h.host.n) + " vertices; the static-scratch entry point serves at most " +
                                std::to_string(kStaticMaxVertices));
  if (source0 < 0 || source0 >= h.host.n) throw Error(QBC_EINVAL, "source id " + std::to_string(source0) + " out of range");
  if (!d_bc_vid) throw Error(QBC_EINVAL, "null BC output");
  DeviceState *d = need_dev(h);
  if (h.host.kind != IndexKind::CSR) {
    // the one-source label kernel keeps a source row and one row per warp in shared memory
    // (44 B per tree level): taller trees need the batched path or a CSR index
    const size_t budget = (size_t)std::max(48 * 1024, d->smem_optin) - 2048;
    if ((size_t)44 * d->hmax_pad > budget || d->hmax_pad > kStaticMaxHeight)
      throw Error(QBC_EINVAL, "tree height " + std::to_string(h.host.tree_height) + " exceeds the " +
                                  std::to_string(budget / 44) + " levels the static-scratch entry point's label kernel holds in "
                                  "shared memory; use qbc_bc_sources_device or a QBC_INDEX_CSR index");
  }
  unsigned char *base = static_scratch_on(d->device);
  cudaStream_t st = stream ? (cudaStream_t)stream : d->s_label;
  int4 *rec = reinterpret_cast<int4 *>(base + kStaticRec);
  int32_t *hop = reinterpret_cast<int32_t *>(base + kStaticHop);
  int32_t *order = reinterpret_cast<int32_t *>(base + kStaticOrder);
  int32_t *lcnt = reinterpret_cast<int32_t *>(base + kStaticLcnt);
  double *bc_tid = reinterpret_cast<double *>(base + kStaticBc);
  int32_t *src = reinterpret_cast<int32_t *>(base + kStaticSrc);
  // the array keeps the previous call's contents: the BC accumulator must start at zero; every
  // other region is fully written by the kernels before it is read
  CK(cudaMemsetAsync(bc_tid, 0, (size_t)d->n * 8, st));
  k_static_set_source<<<1, 1, 0, st>>>(src, h.host.tid_of[source0]);
  CK(cudaGetLastError());
  if (h.host.kind == IndexKind::CSR) {  // label-free index: the shortest-path sweep gives the row
    launch_sweep_rows(h, d, rec, hop, order, lcnt, nullptr, src, 1, st);
  } else {
    const LabelPlan p = plan_label(h, d, 1, true);
    LabelArgs la{};
    int32_t *src_rows = reinterpret_cast<int32_t *>(base + kStaticSrcRows);
    k_src_rows<<<1, 32, 0, st>>>(src, 1, d->depth, d->parent, d->send, d->hmax_pad, src_rows);
    CK(cudaGetLastError());
    la.dis = d->dis;
    la.ch = d->ch;
    la.src_rows = src_rows;
    la.src_stride = d->hmax_pad;
    la.bits = d->packed_bits;
    la.lab_off = d->lab_off;
    la.depth = d->depth;
    la.send = d->send;
    la.src = src;
    la.ns = 1;
    la.n = d->n;
    la.n_pad = d->n_pad;
    la.stride = p.S;
    la.split = p.split;
    la.out_rec = rec;
    la.out_hop = hop;
    la.wait_spins = kRowWaitSpins;
    if (h.host.kind == IndexKind::MHL) launch_label_c<true>(p, la, 1, st);
    else launch_label_c<false>(p, la, 1, st);
  }
  DepArgs da{};
  da.arc_rng = d->arc_rng;
  da.arc_hw = d->arc_hw;
  da.arc_off = d->arc_off;
  da.arc_head = d->arc_head;
  da.arc_w = d->arc_w;
  da.src = src;
  da.ns = 1;
  da.n = d->n;
  da.n_pad = d->n_pad;
  da.rec = rec;
  da.hop = hop;
  da.order = order;
  da.lcnt = lcnt;
  da.bc = bc_tid;
  da.err = d->err;
  const int threads = std::max(64, std::min(256, (h.tuning.dep_threads / 32) * 32));
  if (h.host.kind != IndexKind::H2H) k_dependency<<<1, threads, 0, st>>>(da);  // rows carry counts and hops
  else k_kahn_dependency<<<1, threads, 0, st>>>(da);
  CK(cudaGetLastError());
  k_tid_to_vid_f64<<<(d->n + 255) / 256, 256, 0, st>>>(bc_tid, d->vid_of, d_bc_vid, d->n, 1);
  CK(cudaGetLastError());
}

}  // namespace qbc


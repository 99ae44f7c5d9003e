// index_file.cpp -- on-disk index format of libqbc_b200, so a service can cold-start without a
// rebuild.  Replaces the reference's headerless tmpRoadCountIndex stream (written during
// TreeDecomp::MakeIndex, TreeDecomp.cpp:243,460-467,496-506; read by TreeQuery::ReadIndex,
// TreeDecomp.cpp:748-900) with a self-describing, checksummed file of this library's layout:
//
//   "QBCIDX02"                                   8-byte magic
//   int32 version(2), kind, n, arcs, tree_height, tree_width, max_label, reserved(0)
//   int64 label entries L (= lab_off[n]), depth_sum
//   int32 vid_of[n], tid_of[n], depth[n], parent[n], send[n]
//   int64 lab_off[n+1]
//   int32 arc_off[n+1], arc_head[arcs], arc_w[arcs]
//   int32 dis[L], anc[L], aend[L]
//   int32 ch[2L]                                 (MHL only: count bits, max hop)
//   uint64 checksum of every byte above (WordHash below)
//
// Little-endian, as the hosts this library runs on.  Version 1 files ("QBCIDX01", the same layout
// with the byte-wise FNV-1a as checksum) still load.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>

#include "../../include/qbc_b200.h"
#include "host.h"

namespace qbc {

namespace {

constexpr char kMagicV1[8] = {'Q', 'B', 'C', 'I', 'D', 'X', '0', '1'};
constexpr char kMagic[8] = {'Q', 'B', 'C', 'I', 'D', 'X', '0', '2'};
constexpr int32_t kVersion = 2;
constexpr uint64_t kFnvBasis = 1469598103934665603ull, kFnvPrime = 1099511628211ull;

// Checksum of version 2: FNV-1a's xor-then-multiply step applied to 64-bit little-endian words in
// four interleaved lanes (four independent multiplies per 32 bytes, so hashing runs far faster than
// the disk; the byte-wise FNV-1a of version 1 ran at ~0.5 GB/s and made loading a 200k-vertex index
// slower than rebuilding it).  A partial last block is zero-padded; the lanes and the byte count
// are folded at the end.  Every word passes through a bijection of its lane, so any changed word
// changes its lane.
struct WordHash {
  uint64_t lane[4] = {kFnvBasis, kFnvBasis ^ 1, kFnvBasis ^ 2, kFnvBasis ^ 3};
  unsigned char buf[32];
  size_t nbuf = 0;
  uint64_t total = 0;
  void block(const unsigned char *p) {
    for (int q = 0; q < 4; q++) {
      uint64_t w;
      std::memcpy(&w, p + 8 * q, 8);
      lane[q] = (lane[q] ^ w) * kFnvPrime;
    }
  }
  void update(const void *data, size_t bytes) {
    const unsigned char *p = (const unsigned char *)data;
    total += bytes;
    if (nbuf) {
      const size_t take = std::min(32 - nbuf, bytes);
      std::memcpy(buf + nbuf, p, take);
      nbuf += take;
      p += take;
      bytes -= take;
      if (nbuf < 32) return;
      block(buf);
      nbuf = 0;
    }
    for (; bytes >= 32; p += 32, bytes -= 32) block(p);
    std::memcpy(buf, p, bytes);
    nbuf = bytes;
  }
  uint64_t digest() {
    if (nbuf) {
      std::memset(buf + nbuf, 0, 32 - nbuf);
      block(buf);
      nbuf = 0;
    }
    uint64_t h = kFnvBasis;
    for (int q = 0; q < 4; q++) h = (h ^ lane[q]) * kFnvPrime;
    return (h ^ total) * kFnvPrime;
  }
};

struct File {
  FILE *f = nullptr;
  std::string path;
  bool v1 = false;      // byte-wise FNV-1a (version 1 files)
  uint64_t h1 = kFnvBasis;
  WordHash h2;
  File(const std::string &p, const char *mode) : path(p) {
    f = std::fopen(p.c_str(), mode);
    if (!f) throw Error(QBC_EIO, p + ": cannot open");
  }
  ~File() {
    if (f) std::fclose(f);
  }
  void hash(const void *p, size_t bytes) {
    if (!v1) {
      h2.update(p, bytes);
      return;
    }
    const unsigned char *c = (const unsigned char *)p;
    for (size_t i = 0; i < bytes; i++) h1 = (h1 ^ c[i]) * kFnvPrime;
  }
  uint64_t digest() { return v1 ? h1 : h2.digest(); }
  void put(const void *p, size_t bytes) {
    if (bytes && std::fwrite(p, 1, bytes, f) != bytes) throw Error(QBC_EIO, path + ": write failed");
    hash(p, bytes);
  }
  void get(void *p, size_t bytes) {
    if (bytes && std::fread(p, 1, bytes, f) != bytes) throw Error(QBC_EIO, path + ": truncated index file");
    hash(p, bytes);
  }
  template <class T>
  void put_vec(const std::vector<T> &v, size_t expect) {
    if (v.size() != expect) throw Error(QBC_EINVAL, "index array has an unexpected length");
    put(v.data(), v.size() * sizeof(T));
  }
  template <class T>
  void get_vec(std::vector<T> &v, size_t count) {
    v.resize(count);
    get(v.data(), count * sizeof(T));
  }
};

}  // namespace

void index_save(const Index &ix, const std::string &path) {
  if (!ix.rows_on_host) throw Error(QBC_EINVAL, "index rows are on the device: copy them back first");
  File f(path, "wb");
  const int64_t L = ix.lab_off.empty() ? 0 : ix.lab_off[ix.n];
  const int32_t arcs = (int32_t)ix.arc_head.size();
  f.put(kMagic, 8);
  const int32_t hdr[8] = {kVersion, (int32_t)ix.kind, ix.n, arcs, ix.tree_height, ix.tree_width, ix.max_label, 0};
  f.put(hdr, sizeof(hdr));
  const int64_t hdr2[2] = {L, ix.depth_sum};
  f.put(hdr2, sizeof(hdr2));
  const size_t n = (size_t)ix.n;
  f.put_vec(ix.vid_of, n);
  f.put_vec(ix.tid_of, n);
  f.put_vec(ix.depth, n);
  f.put_vec(ix.parent, n);
  f.put_vec(ix.send, n);
  f.put_vec(ix.lab_off, n + 1);
  f.put_vec(ix.arc_off, n + 1);
  f.put_vec(ix.arc_head, (size_t)arcs);
  f.put_vec(ix.arc_w, (size_t)arcs);
  f.put_vec(ix.dis, (size_t)L);
  f.put_vec(ix.anc, (size_t)L);
  f.put_vec(ix.aend, (size_t)L);
  if (ix.kind == IndexKind::MHL) f.put_vec(ix.ch, (size_t)(2 * L));
  const uint64_t sum = f.digest();
  if (std::fwrite(&sum, 8, 1, f.f) != 1) throw Error(QBC_EIO, path + ": write failed");
  if (std::fflush(f.f) != 0) throw Error(QBC_EIO, path + ": write failed");
}

Index index_load(const std::string &path) {
  File f(path, "rb");
  char magic[8];
  if (std::fread(magic, 1, 8, f.f) != 8) throw Error(QBC_EIO, path + ": not a qbc_b200 index file");
  if (std::memcmp(magic, kMagicV1, 8) == 0) f.v1 = true;
  else if (std::memcmp(magic, kMagic, 8) != 0) throw Error(QBC_EIO, path + ": not a qbc_b200 index file");
  f.hash(magic, 8);
  int32_t hdr[8];
  f.get(hdr, sizeof(hdr));
  if (hdr[0] != (f.v1 ? 1 : kVersion)) throw Error(QBC_EIO, path + ": unsupported index file version " + std::to_string(hdr[0]));
  int64_t hdr2[2];
  f.get(hdr2, sizeof(hdr2));
  Index ix;
  if (hdr[1] != (int32_t)IndexKind::MHL && hdr[1] != (int32_t)IndexKind::H2H && hdr[1] != (int32_t)IndexKind::CSR)
    throw Error(QBC_EIO, path + ": bad index kind");
  const bool csr = hdr[1] == (int32_t)IndexKind::CSR;  // arc list only: no tree, no rows
  ix.kind = (IndexKind)hdr[1];
  ix.n = hdr[2];
  const int32_t arcs = hdr[3];
  ix.tree_height = hdr[4];
  ix.tree_width = hdr[5];
  ix.max_label = hdr[6];
  const int64_t L = hdr2[0];
  ix.depth_sum = hdr2[1];
  if (ix.n <= 0 || arcs < 0 || L < 0 ||
      (csr ? (ix.tree_height != 0 || L != 0) : (ix.tree_height <= 0 || ix.tree_height > ix.n)))
    throw Error(QBC_EIO, path + ": corrupt index header");
  // the payload size the header implies must match the file before anything is allocated
  {
    const long here = std::ftell(f.f);
    std::fseek(f.f, 0, SEEK_END);
    const long end = std::ftell(f.f);
    std::fseek(f.f, here, SEEK_SET);
    const int64_t n = ix.n;
    const int64_t want = 5 * 4 * n + 8 * (n + 1) + 4 * (n + 1) + 8 * (int64_t)arcs + 12 * L +
                         (ix.kind == IndexKind::MHL ? 8 * L : 0) + 8;
    if (end - here != want) throw Error(QBC_EIO, path + ": index file size does not match its header");
  }
  const size_t n = (size_t)ix.n;
  f.get_vec(ix.vid_of, n);
  f.get_vec(ix.tid_of, n);
  f.get_vec(ix.depth, n);
  f.get_vec(ix.parent, n);
  f.get_vec(ix.send, n);
  f.get_vec(ix.lab_off, n + 1);
  f.get_vec(ix.arc_off, n + 1);
  f.get_vec(ix.arc_head, (size_t)arcs);
  f.get_vec(ix.arc_w, (size_t)arcs);
  f.get_vec(ix.dis, (size_t)L);
  f.get_vec(ix.anc, (size_t)L);
  f.get_vec(ix.aend, (size_t)L);
  if (ix.kind == IndexKind::MHL) f.get_vec(ix.ch, (size_t)(2 * L));
  const uint64_t want = f.digest();
  uint64_t sum = 0;
  if (std::fread(&sum, 8, 1, f.f) != 1 || sum != want) throw Error(QBC_EIO, path + ": index file checksum mismatch");
  // structural checks the kernels rely on
  if (ix.lab_off[n] != L || ix.arc_off[n] != arcs) throw Error(QBC_EIO, path + ": inconsistent index arrays");
  for (size_t t = 0; t < n && csr; t++) {
    if (ix.depth[t] != 0 || ix.parent[t] != -1 || ix.send[t] != (int32_t)t + 1 || ix.lab_off[t] != 0 ||
        ix.vid_of[t] < 0 || ix.vid_of[t] >= ix.n || ix.tid_of[ix.vid_of[t]] != (int32_t)t || ix.arc_off[t] > ix.arc_off[t + 1])
      throw Error(QBC_EIO, path + ": inconsistent index arrays");
  }
  for (size_t t = 0; t < n && !csr; t++) {
    if (ix.depth[t] < 1 || ix.depth[t] > ix.tree_height || ix.lab_off[t] % 4 != 0 ||
        ix.lab_off[t + 1] - ix.lab_off[t] < ix.depth[t] || ix.send[t] <= (int32_t)t || ix.send[t] > ix.n ||
        ix.vid_of[t] < 0 || ix.vid_of[t] >= ix.n || ix.tid_of[ix.vid_of[t]] != (int32_t)t ||
        ix.arc_off[t] > ix.arc_off[t + 1] || (t == 0 ? ix.parent[t] != -1 : (ix.parent[t] < 0 || ix.parent[t] >= (int32_t)t)))
      throw Error(QBC_EIO, path + ": inconsistent index arrays");
  }
  for (int32_t hd : ix.arc_head)
    if (hd < 0 || hd >= ix.n) throw Error(QBC_EIO, path + ": inconsistent index arrays");
  for (int32_t a : ix.anc)
    if (a < 0 || a >= ix.n) throw Error(QBC_EIO, path + ": inconsistent index arrays");
  ix.rows_on_host = true;
  return ix;
}

}  // namespace qbc

// cf_igen.cu -- the product-bounded I side (the igen / idump records) through
// two C calls, count then write, as gpu/igen_gpu.py:113-162 counts and writes
// its records in two passes.
//
// Records: every r-subset I of the ascending pool with prod(I) < Icap and at
// most hmax primes at indices >= split_idx; key = mult * prod(I) mod M (mult =
// P0 mod M, taken by cf_pool_prepare), id = colex rank; the order of
// src/mitm64_idump_stream2.cpp with IDUMP_RANK=1 and one thread.
//
//   cf_igen_bounds  the exact bound table H[t][x] = floor((Icap-1) / (a_x ...
//                   a_{x+t})) on the host (128-bit products; a product that
//                   overflows 128 bits gives 0);
//   cf_igen_count   expands the enumeration tree level by level in the
//                   caller's workspace (cf_bgen_count, cf_scan_u64,
//                   cf_bgen_expand) down to the last inner level and returns
//                   the record count; the last frontier stays in the workspace
//                   and its shape in a small host state;
//   cf_igen_write   writes the records [c0, c0+cc) of that frontier.
//
// A level larger than the workspace holds makes cf_igen_count return CF_ENOMEM
// with the node count it needed; cf_igen_tmp_bytes(nodes) sizes the retry.
#include <string.h>
#include "cf_abi_internal.h"

extern "C" size_t cf_scan_tmp_bytes(u64 n);
extern "C" int cf_scan_u64(const u64* in, u64 n, u64* out, void* tmp, size_t tmp_bytes, void* stream);
extern "C" u64 cf_key_of(u64 M, u64 v);
extern "C" int cf_bgen_count(int side, int d, int r, int n, u64 F, const u64* alo, const u64* ahi, const u32* meta,
                             const u64* bounds, int split_idx, int hmax, int xa, int xb, u64* cnt, u32* xs,
                             void* stream);
extern "C" int cf_bgen_expand(int side, int d, int r, int n, u64 F, const void* pool, const u64* key, const u64* alo,
                              const u64* ahi, const u64* id, const u32* meta, const u64* offs, const u32* xs,
                              int split_idx, int bitmask, u64 c0, u64 cc, u64* okey, u64* oalo, u64* oahi, u64* oid,
                              u32* ometa, void* stream);

namespace {

typedef unsigned __int128 u128;

size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }

// Workspace for frontiers of at most C nodes: two node sets (key, alo, ahi, id:
// 8 bytes each; meta: 4), the counts (8), first child indices (4), the offsets
// (8, plus one) and the scan's scratch.
struct IgenLayout {
  size_t set[2], cnt, xs, offs, scan, total;
};
IgenLayout igen_layout(u64 C) {
  IgenLayout L;
  const size_t nodes = a256((size_t)C * 36);
  size_t o = 0;
  L.set[0] = o; o += nodes;
  L.set[1] = o; o += nodes;
  L.cnt = o; o += a256((size_t)C * 8);
  L.xs = o; o += a256((size_t)C * 4);
  L.offs = o; o += a256((size_t)(C + 1) * 8);
  L.scan = o; o += a256(cf_scan_tmp_bytes(C ? C : 1));
  L.total = o;
  return L;
}

// Node set views: key | alo | ahi | id (C words each) | meta (C u32)
struct NodeSet {
  u64 *key, *alo, *ahi, *id;
  u32* meta;
};
NodeSet node_set(unsigned char* base, u64 C) {
  NodeSet s;
  s.key = (u64*)base;
  s.alo = s.key + C;
  s.ahi = s.alo + C;
  s.id = s.ahi + C;
  s.meta = (u32*)(s.id + C);
  return s;
}

// Largest node capacity whose layout fits tmp_bytes.
u64 igen_capacity(size_t tmp_bytes) {
  u64 lo = 0, hi = (u64)(tmp_bytes / 36) + 1;
  while (lo < hi) {
    const u64 mid = lo + (hi - lo + 1) / 2;
    if (igen_layout(mid).total <= tmp_bytes) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// The state cf_igen_count leaves for cf_igen_write (opaque to callers).
struct IgenState {
  u64 magic, F, C, total, set;
  u64 pad[3];
};
constexpr u64 kIgenMagic = 0x6366696765e57a7eull;
static_assert(sizeof(IgenState) == 64, "the igen state is 64 bytes");

}  // namespace

extern "C" size_t cf_igen_bounds_bytes(int n, int r) {
  if (n < 1 || n > CF_MAX_POOL || r < 1 || r > CF_MAX_R) return 0;
  return (size_t)16 * n * r;
}

// Host: the bound table of the ascending pool ins[n] for radius r and exclusive
// cap Icap = icap_hi * 2^64 + icap_lo, as (lo, hi) u64 pairs, row t = positions
// left after the chosen index (the layout cf_bgen_count reads).
extern "C" int cf_igen_bounds(const u64* ins, int n, int r, u64 icap_lo, u64 icap_hi, void* out, size_t out_bytes) {
  if (!ins || !out || n < 1 || n > CF_MAX_POOL || r < 1 || r > CF_MAX_R || out_bytes < cf_igen_bounds_bytes(n, r)) {
    cf_set_error("cf_igen_bounds: bad arguments%s", "");
    return CF_EBADARG;
  }
  for (int i = 1; i < n; ++i)
    if (ins[i] <= ins[i - 1]) { cf_set_error("cf_igen_bounds: pool not strictly ascending%s", ""); return CF_EBADARG; }
  const u128 icap = ((u128)icap_hi << 64) | icap_lo;
  const u128 top = icap ? icap - 1 : 0;
  u64* H = (u64*)out;
  memset(H, 0, cf_igen_bounds_bytes(n, r));
  for (int t = 0; t < r && t < n; ++t)
    for (int x = 0; x + t < n; ++x) {
      u128 w = 1;
      bool over = false;
      for (int j = 0; j <= t && !over; ++j) over = __builtin_mul_overflow(w, (u128)ins[x + j], &w);
      const u128 q = (over || icap == 0) ? 0 : top / w;
      H[2 * ((size_t)t * n + x)] = (u64)q;
      H[2 * ((size_t)t * n + x) + 1] = (u64)(q >> 64);
    }
  return CF_OK;
}

extern "C" size_t cf_igen_tmp_bytes(u64 max_nodes) { return igen_layout(max_nodes ? max_nodes : 1).total; }

// Count the records (see above).  pool_dev: cf_pool_prepare(ins, n, r, M,
// P0 mod M) on the device; bounds_dev: cf_igen_bounds on the device.
// *total receives the record count; state (64 bytes, host) the frontier for
// cf_igen_write.  CF_ENOMEM: a level needs *need_nodes nodes (retry with
// cf_igen_tmp_bytes(*need_nodes) bytes).  Synchronises the stream once per level.
extern "C" int cf_igen_count(const void* pool_dev, const void* bounds_dev, u64 M, u64 mult, int n, int r,
                             int split_idx, int hmax, void* tmp, size_t tmp_bytes, u64* total, u64* need_nodes,
                             void* state, void* stream) {
  if (!pool_dev || !bounds_dev || !tmp || !total || !state || n < 1 || n > CF_MAX_POOL || r < 1 || r > CF_MAX_R ||
      r > n || M < 2 || split_idx < 0 || hmax < 0) {
    cf_set_error("cf_igen_count: bad arguments%s", "");
    return CF_EBADARG;
  }
  const cudaStream_t st = (cudaStream_t)stream;
  const u64 C = igen_capacity(tmp_bytes);
  if (C < 1) { cf_set_error("cf_igen_count: workspace too small%s", ""); return CF_ENOMEM; }
  const IgenLayout L = igen_layout(C);
  unsigned char* w = (unsigned char*)tmp;
  u64* cnt = (u64*)(w + L.cnt);
  u32* xs = (u32*)(w + L.xs);
  u64* offs = (u64*)(w + L.offs);
  void* stmp = w + L.scan;
  // the root: key form of the multiplier, product 1, id 0, no index yet
  NodeSet cur = node_set(w + L.set[0], C);
  const u64 root[4] = {cf_key_of(M, mult % M), 1, 0, 0};
  const u32 root_meta = 0xffffu;
  cudaError_t e = cudaMemcpyAsync(cur.key, &root[0], 8, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(cur.alo, &root[1], 8, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(cur.ahi, &root[2], 8, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(cur.id, &root[3], 8, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(cur.meta, &root_meta, 4, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return cf_cuda_status(e, "cf_igen_count: root");
  u64 F = 1;
  int set = 0;
  for (int d = 0; d < r; ++d) {
    int rc = cf_bgen_count(0, d, r, n, F, cur.alo, cur.ahi, cur.meta, (const u64*)bounds_dev, split_idx, hmax, 0, n,
                           cnt, xs, stream);
    if (rc == CF_OK) rc = cf_scan_u64(cnt, F, offs, stmp, L.total - L.scan, stream);
    if (rc != CF_OK) return rc;
    u64 level = 0;
    e = cudaMemcpyAsync(&level, offs + F, 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cf_cuda_status(e, "cf_igen_count: level size");
    if (d == r - 1 || level == 0) {
      IgenState s = {kIgenMagic, d == r - 1 ? F : 0, C, d == r - 1 ? level : 0, (u64)set, {0, 0, 0}};
      memcpy(state, &s, sizeof s);
      *total = s.total;
      return CF_OK;
    }
    if (level > C) {
      if (need_nodes) *need_nodes = level;
      char buf[160];
      snprintf(buf, sizeof buf, "cf_igen_count: a level has %llu nodes, the workspace holds %llu",
               (unsigned long long)level, (unsigned long long)C);
      cf_set_error("%s", buf);
      return CF_ENOMEM;
    }
    NodeSet nxt = node_set(w + L.set[1 - set], C);
    rc = cf_bgen_expand(0, d, r, n, F, pool_dev, cur.key, cur.alo, cur.ahi, cur.id, cur.meta, offs, xs, split_idx, 0,
                        0, level, nxt.key, nxt.alo, nxt.ahi, nxt.id, nxt.meta, stream);
    if (rc != CF_OK) return rc;
    cur = nxt;
    set = 1 - set;
    F = level;
  }
  return CF_OK;
}

// Write records [c0, c0+cc) of the frontier cf_igen_count left in tmp (same
// pool, n, r, split_idx and workspace) to keys[cc], ids[cc].
extern "C" int cf_igen_write(const void* pool_dev, int n, int r, int split_idx, const void* tmp, const void* state,
                             u64 c0, u64 cc, u64* keys, u64* ids, void* stream) {
  if (!state || !tmp || !pool_dev) { cf_set_error("cf_igen_write: bad arguments%s", ""); return CF_EBADARG; }
  IgenState s;
  memcpy(&s, state, sizeof s);
  if (s.magic != kIgenMagic) { cf_set_error("cf_igen_write: state not from cf_igen_count%s", ""); return CF_EBADARG; }
  if (cc == 0) return CF_OK;
  if (c0 > s.total || cc > s.total - c0 || !keys || !ids) {
    cf_set_error("cf_igen_write: record range outside the counted records%s", "");
    return CF_EBADARG;
  }
  const IgenLayout L = igen_layout(s.C);
  unsigned char* w = (unsigned char*)tmp;
  const NodeSet cur = node_set(w + L.set[s.set], s.C);
  return cf_bgen_expand(0, r - 1, r, n, s.F, pool_dev, cur.key, cur.alo, cur.ahi, cur.id, cur.meta,
                        (const u64*)(w + L.offs), (const u32*)(w + L.xs), split_idx, 0, c0, cc, keys, nullptr,
                        nullptr, ids, nullptr, stream);
}

// cf_bsolve.cu -- one product-bounded exchange instance in one C call: the
// bounded D side (ddump's records), a record table of it, the bounded I side
// expanded to its last inner level and its leaves probed in registers, and the
// candidate pairs handed back -- the device part of the reference driver's
// run_instance (gpu/mitm_gpu_mstar_driver.py:184-286: build_D with DFILTER,
// the igen chunks, the sorted join) without a host round trip per kernel.
//
// The host work per instance was the cost of a census family run (a Python
// loop over levels with a device read after each): this runs the levels from
// C++, in the caller's workspace, with one read of each level's size.
//
//   cf_ddump_bounds   the exact D-side bound table G[t][x] = ceil(Dmin / (b_x
//                     b_{x-1} ... b_{x-t})) on the host (cf_igen_bounds is the I
//                     side's);
//   cf_bounded_join   D records (colex ids), table, I leaves probed; returns the
//                     candidates {D colex id, D key, I colex id} in host arrays
//                     (equal keys and the rare fingerprint collisions, which the
//                     caller removes by recomputing the I key), and the two
//                     side sizes.  CF_ENOMEM: the workspace is too small (*need
//                     holds a size that gets further; retry); CF_EOVERFLOW: more
//                     candidates than max_out (*n_out holds their number).
#include <string.h>
#include "cf_dtab.cuh"

extern "C" size_t cf_scan_tmp_bytes(u64 n);
extern "C" int cf_scan_u64(const u64* in, u64 n, u64* out, void* tmp, size_t tmp_bytes, void* stream);
extern "C" u64 cf_key_of(u64 M, u64 v);
extern "C" size_t cf_dtab_bytes2(int bbits, int fbits);
extern "C" int cf_bgen_count(int side, int d, int r, int n, u64 F, const u64* alo, const u64* ahi, const u32* meta,
                             const u64* bounds, int split_idx, int hmax, int xa, int xb, u64* cnt, u32* xs,
                             void* stream);
extern "C" int cf_bgen_expand(int side, int d, int r, int n, u64 F, const void* pool, const u64* key, const u64* alo,
                              const u64* ahi, const u64* id, const u32* meta, const u64* offs, const u32* xs,
                              int split_idx, int bitmask, u64 c0, u64 cc, u64* okey, u64* oalo, u64* oahi, u64* oid,
                              u32* ometa, void* stream);
extern "C" int cf_rec_build_keyform(const u64* keys, u64 n, void* tab, int bbits, int fbits, const void* pool,
                                    u32* err, void* stream);
extern "C" int cf_bgen_probe_keyform(int r, int n, u64 F, const void* pool, const u64* key, const u64* id,
                                     const u64* offs, const u32* xs, u64 c0, u64 cc, const void* tab, int bbits,
                                     int fbits, void* pairs, u32 max_pairs, u32* npairs, u32* err, void* stream);

namespace {

typedef unsigned __int128 u128;

size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

// Bump allocation in the caller's workspace; a request that does not fit marks
// the run as short of memory and records how much it would have needed.
struct Bump {
  unsigned char* base;
  size_t cap, off, need;
  bool ok;
  void* take(size_t bytes) {
    const size_t o = al256(off);
    if (!ok || o + bytes > cap) {
      ok = false;
      if (o + bytes > need) need = o + bytes;
      return nullptr;
    }
    off = o + bytes;
    return base + o;
  }
};

struct Level {
  u64 F;
  u64 *key, *alo, *ahi, *id;
  u32* meta;
  u64* offs;
  u32* xs;
};

__global__ void k_gather_candidates(const CfPair* __restrict__ pairs, u32 n, const u64* __restrict__ Dk,
                                    const u64* __restrict__ Did, u64* __restrict__ out /*[3][n]*/) {
  for (u32 k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const u64 p = pairs[k].d_id;
    out[k] = Did[p];
    out[(u64)n + k] = Dk[p];
    out[2ull * n + k] = pairs[k].i_id;
  }
}

// Expand one side from the root down to depth `stop` (the leaf level when it
// equals r: records are written to rec_key/rec_id; else the frontier at depth
// stop is returned with its child offsets).  Returns CF_OK, an error, or
// CF_ENOMEM through the bump allocator.
int expand_side(int side, int r, int n, const void* pool, const u64* bounds, u64 root_key, int split_idx, int hmax,
                int bitmask, int stop, Bump& bump, Level& out, u64* total, u64** rec_key, u64** rec_id,
                u64* hostw, cudaStream_t st) {
  Level cur;
  cur.F = 1;
  cur.key = (u64*)bump.take(4 * 8);
  cur.meta = (u32*)bump.take(4);
  if (!bump.ok) return CF_ENOMEM;
  cur.alo = cur.key + 1;
  cur.ahi = cur.key + 2;
  cur.id = cur.key + 3;
  hostw[0] = root_key; hostw[1] = 1; hostw[2] = 0; hostw[3] = 0;
  ((u32*)(hostw + 4))[0] = 0xffffu;
  cudaError_t e = cudaMemcpyAsync(cur.key, hostw, 32, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(cur.meta, hostw + 4, 4, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return cf_cuda_status(e, "cf_bounded_join: root");
  for (int d = 0; d < r; ++d) {
    u64* cnt = (u64*)bump.take(cur.F * 8);
    cur.xs = (u32*)bump.take(cur.F * 4);
    cur.offs = (u64*)bump.take((cur.F + 1) * 8);
    const size_t sb = cf_scan_tmp_bytes(cur.F);
    void* stmp = bump.take(sb);
    if (!bump.ok) return CF_ENOMEM;
    int rc = cf_bgen_count(side, d, r, n, cur.F, cur.alo, cur.ahi, cur.meta, bounds, split_idx, hmax, 0, n, cnt,
                           cur.xs, st);
    if (rc == CF_OK) rc = cf_scan_u64(cnt, cur.F, cur.offs, stmp, sb, st);
    if (rc != CF_OK) return rc;
    e = cudaMemcpyAsync(hostw + 5, cur.offs + cur.F, 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cf_cuda_status(e, "cf_bounded_join: level size");
    const u64 level = hostw[5];
    if (d == stop) {                           // the frontier the caller probes
      out = cur;
      *total = level;
      return CF_OK;
    }
    if (level == 0) {
      out = cur;
      out.F = 0;
      *total = 0;
      return CF_OK;
    }
    if (d == r - 1) {                          // leaves: the side's records
      *rec_key = (u64*)bump.take(level * 8);
      *rec_id = (u64*)bump.take(level * 8);
      if (!bump.ok) return CF_ENOMEM;
      rc = cf_bgen_expand(side, d, r, n, cur.F, pool, cur.key, cur.alo, cur.ahi, cur.id, cur.meta, cur.offs, cur.xs,
                          split_idx, bitmask, 0, level, *rec_key, nullptr, nullptr, *rec_id, nullptr, st);
      if (rc != CF_OK) return rc;
      *total = level;
      return CF_OK;
    }
    Level nxt;
    nxt.F = level;
    nxt.key = (u64*)bump.take(level * 8);
    nxt.alo = (u64*)bump.take(level * 8);
    nxt.ahi = (u64*)bump.take(level * 8);
    nxt.id = (u64*)bump.take(level * 8);
    nxt.meta = (u32*)bump.take(level * 4);
    if (!bump.ok) return CF_ENOMEM;
    rc = cf_bgen_expand(side, d, r, n, cur.F, pool, cur.key, cur.alo, cur.ahi, cur.id, cur.meta, cur.offs, cur.xs,
                        split_idx, bitmask, 0, level, nxt.key, nxt.alo, nxt.ahi, nxt.id, nxt.meta, st);
    if (rc != CF_OK) return rc;
    cur = nxt;
  }
  *total = 0;
  return CF_OK;
}

}  // namespace

extern "C" size_t cf_ddump_bounds_bytes(int n, int r) {
  if (n < 1 || n > CF_MAX_POOL || r < 1 || r > CF_MAX_R) return 0;
  return (size_t)16 * n * r;
}

// Host: the D-side bound table of the ascending base b[n] for radius r and
// inclusive floor Dmin = dmin_hi * 2^64 + dmin_lo, as (lo, hi) u64 pairs (row t
// = positions left after the chosen index; entries x < t unused and saturated).
extern "C" int cf_ddump_bounds(const u64* b, int n, int r, u64 dmin_lo, u64 dmin_hi, void* out, size_t out_bytes) {
  if (!b || !out || n < 1 || n > CF_MAX_POOL || r < 1 || r > CF_MAX_R || out_bytes < cf_ddump_bounds_bytes(n, r)) {
    cf_set_error("cf_ddump_bounds: bad arguments%s", "");
    return CF_EBADARG;
  }
  for (int i = 1; i < n; ++i)
    if (b[i] <= b[i - 1]) { cf_set_error("cf_ddump_bounds: base not strictly ascending%s", ""); return CF_EBADARG; }
  const u128 dmin = ((u128)dmin_hi << 64) | dmin_lo;
  u64* G = (u64*)out;
  memset(G, 0xff, cf_ddump_bounds_bytes(n, r));
  for (int t = 0; t < r && t < n; ++t)
    for (int x = t; x < n; ++x) {
      u128 w = 1;
      bool over = false;
      for (int j = 0; j <= t && !over; ++j) over = __builtin_mul_overflow(w, (u128)b[x - j], &w);
      u128 q;
      if (dmin == 0) q = 0;
      else if (over) q = 1;                     // w > 2^128 > Dmin: any product of the window clears it
      else q = dmin / w + (dmin % w != 0);
      G[2 * ((size_t)t * n + x)] = (u64)q;
      G[2 * ((size_t)t * n + x) + 1] = (u64)(q >> 64);
    }
  return CF_OK;
}

// One bounded instance (see the top of the file).  poolD/boundsD: the base's
// pool table (cf_pool_prepare(B0, nb, r, M, 1)) and cf_ddump_bounds table on
// the device; poolI/boundsI: the insertion pool's (mult = P0 mod M) and
// cf_igen_bounds table.  bbits/fbits: the D record table's shape (0 bits: chosen
// here, about 8 records per bucket, no Bloom level).  out: host array of
// 3 * max_out u64 (D colex ids, D keys, I colex ids, max_out each);
// sizes[2]: host, receives {nD, nI}.  M below 2^64.
extern "C" int cf_bounded_join(const void* poolD, const void* boundsD, int nb, const void* poolI,
                               const void* boundsI, int ni, int r, u64 M, u64 p0_mod_m, int split_idx, int hmax,
                               int bbits, int fbits, void* tmp, size_t tmp_bytes, u64* out, u64 max_out,
                               u64* n_out, u64* sizes, u64* need, void* stream) {
  if (!poolD || !boundsD || !poolI || !boundsI || !tmp || !n_out || !sizes || (max_out && !out) || r < 1 ||
      r > CF_MAX_R || nb < r || ni < r || nb > CF_MAX_POOL || ni > CF_MAX_POOL || M < 2 || split_idx < 0 ||
      hmax < 0 || bbits < 0 || bbits > 28 || fbits < 0 || fbits > 26) {
    cf_set_error("cf_bounded_join: bad arguments%s", "");
    return CF_EBADARG;
  }
  const cudaStream_t st = (cudaStream_t)stream;
  Bump bump{(unsigned char*)tmp, tmp_bytes, 0, 0, true};
  static thread_local u64 hostw[8];
  *n_out = 0;
  sizes[0] = sizes[1] = 0;
  u32* misc = (u32*)bump.take(256);           // [0] npairs, [1] err
  if (!bump.ok) { if (need) *need = bump.need; cf_set_error("cf_bounded_join: workspace too small%s", ""); return CF_ENOMEM; }
  // ---- D side: every record
  Level fd;
  u64 nD = 0, *Dk = nullptr, *Did = nullptr;
  int rc = expand_side(1, r, nb, poolD, (const u64*)boundsD, cf_key_of(M, 1), nb, r, 2, r, bump, fd, &nD, &Dk, &Did,
                       hostw, st);
  if (rc == CF_ENOMEM || !bump.ok) {
    if (need) *need = bump.need;
    cf_set_error("cf_bounded_join: workspace too small (D side)%s", "");
    return CF_ENOMEM;
  }
  if (rc != CF_OK) return rc;
  sizes[0] = nD;
  // ---- I side: the frontier above the leaves
  Level fi;
  u64 nI = 0;
  rc = expand_side(0, r, ni, poolI, (const u64*)boundsI, cf_key_of(M, p0_mod_m % M), split_idx, hmax, 0, r - 1, bump,
                   fi, &nI, nullptr, nullptr, hostw, st);
  if (rc == CF_ENOMEM || !bump.ok) {
    if (need) *need = bump.need;
    cf_set_error("cf_bounded_join: workspace too small (I side)%s", "");
    return CF_ENOMEM;
  }
  if (rc != CF_OK) return rc;
  sizes[1] = nI;
  if (nD == 0 || nI == 0 || fi.F == 0) return CF_OK;
  if (nD >= (1ull << 32)) { cf_set_error("cf_bounded_join: D side of 2^32 records or more%s", ""); return CF_EOVERFLOW; }
  // ---- table of the D records
  if (bbits == 0) {
    bbits = 4;
    while (bbits < 28 && ((u64)1 << bbits) * 8 < nD) ++bbits;
    fbits = 0;
  }
  const u64 nbk = 1ull << bbits;
  const size_t tb = cf_dtab_bytes2(bbits, fbits);
  unsigned char* tab = (unsigned char*)bump.take(tb);
  const u32 cap = max_out > (1u << 20) ? (1u << 20) : (u32)(max_out ? max_out : 1);
  CfPair* pairs = (CfPair*)bump.take((size_t)cap * sizeof(CfPair));
  u64* gath = (u64*)bump.take((size_t)3 * cap * 8);
  if (!bump.ok) {
    if (need) *need = bump.need;
    cf_set_error("cf_bounded_join: workspace too small (table)%s", "");
    return CF_ENOMEM;
  }
  cudaError_t e = cudaMemsetAsync(tab, 0, nbk * 32, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(tab + nbk * 160, 0, tb - nbk * 160, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(misc, 0, 8, st);
  if (e != cudaSuccess) return cf_cuda_status(e, "cf_bounded_join: zero");
  // the D records go in under the key form of the I pool's modulus, the form the I leaves are computed
  // in: the leaves probe without a conversion to canonical residues
  rc = cf_rec_build_keyform(Dk, nD, tab, bbits, fbits, poolI, misc + 1, st);
  if (rc != CF_OK) return rc;
  // ---- probe every I leaf, in launches of at most 2^30 leaves
  constexpr u64 kChunk = 1ull << 30;
  for (u64 c0 = 0; c0 < nI; c0 += kChunk) {
    const u64 cc = nI - c0 < kChunk ? nI - c0 : kChunk;
    rc = cf_bgen_probe_keyform(r, ni, fi.F, poolI, fi.key, fi.id, fi.offs, fi.xs, c0, cc, tab, bbits, fbits, pairs,
                               cap, misc, misc + 1, st);
    if (rc != CF_OK) return rc;
  }
  e = cudaMemcpyAsync(hostw, misc, 8, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cf_cuda_status(e, "cf_bounded_join: candidates");
  const u32 npairs = ((u32*)hostw)[0], err = ((u32*)hostw)[1];
  if (err & CF_ERR_TABLE_FULL) { cf_set_error("cf_bounded_join: table full%s", ""); return CF_EOVERFLOW; }
  *n_out = npairs;
  if (npairs > cap || (err & CF_ERR_PAIR_OVERFLOW)) {
    cf_set_error("cf_bounded_join: more candidates than the output holds%s", "");
    return CF_EOVERFLOW;
  }
  if (err) { cf_set_error("cf_bounded_join: a kernel rejected its work%s", ""); return CF_EBADARG; }
  if (npairs == 0) return CF_OK;
  k_gather_candidates<<<(npairs + 255) / 256, 256, 0, st>>>(pairs, npairs, Dk, Did, gath);
  CF_LAUNCH_CHECK("cf_bounded_join: gather");
  for (int j = 0; j < 3; ++j) {
    e = cudaMemcpyAsync(out + (size_t)j * max_out, gath + (size_t)j * npairs, (size_t)npairs * 8,
                        cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return cf_cuda_status(e, "cf_bounded_join: copy out");
  }
  return cf_cuda_status(cudaStreamSynchronize(st), "cf_bounded_join: copy out");
}

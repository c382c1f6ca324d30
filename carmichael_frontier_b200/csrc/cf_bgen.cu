// cf_bgen.cu -- product-bounded subset generation: the record producers of the
// reference's filtered sides, exact, on the GPU.
//
//   I side (gpu/igen_gpu.py:26-76, src/mitm64_idump_stream2.cpp): every r-subset
//     I of the ascending pool with prod(I) < Icap and at most hmax primes at
//     indices >= split_idx; key = P0 * prod(I) mod M, id = colex rank
//     sum_j C(i_j, j+1); lexicographic order.
//   D side (src/mitm64_ddump.cpp:29-44): every r-subset D of the ascending base
//     with prod(D) >= Dmin; key = prod(D) mod M, id = indices packed 6 bits each
//     (ascending from bit 0) or a 64-bit index mask (bases of at most 64
//     primes, as the dumper), or -- for larger bases, which the dumper does not
//     take -- the colex rank; descending-index depth-first order.
//
// Instead of one depth-first walk per thread (which balances poorly when the
// bound prunes unevenly), the enumeration tree is expanded one level at a time
// over the whole frontier.  A node is a partial subset {key form of its
// residue, exact 128-bit product, partial id, last index, count of large
// primes}.  Because the pool is sorted, the children of a node that can still
// complete within the bound form ONE contiguous index range, found by a binary
// search in a host-computed exact bound table:
//   I side: H[t][x] = floor((Icap-1) / (a_x a_{x+1} ... a_{x+t})), non-increasing
//           in x; child x is kept iff A <= H[t][x]  (t = positions left after x)
//   D side: G[t][x] = ceil(Dmin / (b_x b_{x-1} ... b_{x-t})), non-increasing in
//           x; child x is kept iff A >= G[t][x]
// so a level is: count children per node (k_bgen_count), exclusive scan
// (cf_scan_u64), and write one child per thread (k_bgen_expand), which finds
// its parent by binary search over the scanned offsets -- every thread does the
// same work whatever the shape of the tree.  The last level writes the records
// (canonical keys) directly, in the reference's order.  The product never
// overflows: on the I side the host checks that Icap - 1 < 2^128 (A * a_x <= Icap - 1 for every kept
// child) or, for larger caps (the table then saturates at 2^128 - 1), that r - 1 primes multiply below 2^128;
// on the D side the host checks that the r largest primes multiply below 2^128.
#include "cf_abi_internal.h"

namespace {

struct U128 {
  u64 lo, hi;
};
__device__ __forceinline__ bool u128_le(U128 a, U128 b) { return a.hi < b.hi || (a.hi == b.hi && a.lo <= b.lo); }
__device__ __forceinline__ U128 u128_mul64(U128 a, u64 b) {   // caller guarantees no overflow
  U128 r;
  r.lo = a.lo * b;
  r.hi = a.hi * b + __umul64hi(a.lo, b);
  return r;
}
__device__ __forceinline__ U128 bound_at(const u64* __restrict__ tb, int n, int t, int x) {
  const u64* p = tb + 2 * ((size_t)t * n + x);
  U128 v;
  v.lo = p[0];
  v.hi = p[1];
  return v;
}

constexpr u32 kRoot = 0xffffu;

// Children of every frontier node at depth d: cnt[i] and the first child index xs[i].
template <int SIDE>
__global__ void __launch_bounds__(256)
k_bgen_count(int d, int r, int n, u64 F, const u64* __restrict__ alo, const u64* __restrict__ ahi,
             const u32* __restrict__ meta, const u64* __restrict__ bounds, int split_idx, int hmax, int xa, int xb,
             u64* __restrict__ cnt, u32* __restrict__ xs) {
  const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= F) return;
  const int t = r - d - 1;
  const u32 mt = meta[i];
  const int last = (int)(mt & 0xffffu);
  const int nl = (int)(mt >> 16);
  U128 A;
  A.lo = alo[i];
  A.hi = ahi[i];
  u64 c = 0;
  u32 x0 = 0;
  if (SIDE == 0) {                          // I side: ascending, x in [lo, hi] with H[t][x] >= A
    int lo = (last == (int)kRoot) ? 0 : last + 1;
    int hi = n - 1 - t;
    if (nl + 1 > hmax && hi > split_idx - 1) hi = split_idx - 1;
    if (d == 0) {
      if (lo < xa) lo = xa;
      if (hi > xb - 1) hi = xb - 1;
    }
    if (lo <= hi && u128_le(A, bound_at(bounds, n, t, lo))) {
      int a = lo, b = hi;                    // largest x in [a, b] with A <= H[t][x]
      while (a < b) {
        const int mid = (a + b + 1) >> 1;
        if (u128_le(A, bound_at(bounds, n, t, mid))) a = mid; else b = mid - 1;
      }
      c = (u64)(a - lo + 1);
      x0 = (u32)lo;
    }
  } else {                                  // D side: descending, x in [lo, hi] with G[t][x] <= A
    int hi = (last == (int)kRoot) ? n - 1 : last - 1;
    int lo = t;
    if (d == 0) {
      if (lo < xa) lo = xa;
      if (hi > xb - 1) hi = xb - 1;
    }
    if (lo <= hi && u128_le(bound_at(bounds, n, t, hi), A)) {
      int a = lo, b = hi;                    // smallest x in [a, b] with G[t][x] <= A
      while (a < b) {
        const int mid = (a + b) >> 1;
        if (u128_le(bound_at(bounds, n, t, mid), A)) b = mid; else a = mid + 1;
      }
      c = (u64)(hi - a + 1);
      x0 = (u32)hi;
    }
  }
  cnt[i] = c;
  xs[i] = x0;
}

// One child per thread for the children [c0, c0 + cc) of the level: parent by
// binary search over offs[0..F] (exclusive scan of the counts, offs[F] = total).
// LEAF: write records (canonical key, final id); else write child nodes.
template <int SIDE, bool LEAF>
__global__ void __launch_bounds__(256)
k_bgen_expand(int d, int r, int n, u64 F, const u64* __restrict__ pool, const u64* __restrict__ key,
              const u64* __restrict__ alo, const u64* __restrict__ ahi, const u64* __restrict__ id,
              const u32* __restrict__ meta, const u64* __restrict__ offs, const u32* __restrict__ xs, int split_idx,
              int bitmask, u64 c0, u64 cc, u64* __restrict__ okey, u64* __restrict__ oalo, u64* __restrict__ oahi,
              u64* __restrict__ oid, u32* __restrict__ ometa) {
  const u64 k = (u64)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= cc) return;
  const u64 c = c0 + k;
  u64 a = 0, b = F - 1;                      // largest p with offs[p] <= c
  while (a < b) {
    const u64 mid = (a + b + 1) >> 1;
    if (offs[mid] <= c) a = mid; else b = mid - 1;
  }
  const u64 p = a;
  const u64 j = c - offs[p];
  const int x = SIDE == 0 ? (int)(xs[p] + j) : (int)(xs[p] - j);
  const CfPoolHdr* hd = (const CfPoolHdr*)pool;
  const CfMod md = cf_mod_from_hdr(hd);
  const u64 prime = pool[cf_pool_off_prime(n) + x];
  // M of 2^64 or more (header M = 0, cf_pool_prepare_split): a node key is the odd part alone in
  // Montgomery form (x * 2^64 mod m); x mod 2^a follows from the node's exact product A.
  const bool wide = hd->M == 0;
  const u64 kk = wide ? cf_redc_mul(key[p], cf_redc_mul(prime, hd->r2, md.m, md.minv), md.m, md.minv)
                      : cf_mul_key(key[p], pool[cf_pool_off_pkey(n) + x], md);
  u64 nid;
  if (SIDE == 0) {
    nid = id[p] + pool[cf_pool_off_binom(n) + (size_t)x * (r + 1) + (d + 1)];   // colex: + C(x, d+1)
  } else if (bitmask == 2) {                 // colex rank: x is the (r-d)-th smallest index
    nid = id[p] + pool[cf_pool_off_binom(n) + (size_t)x * (r + 1) + (r - d)];
  } else {
    nid = bitmask ? (id[p] | (1ull << x)) : (id[p] | ((u64)x << (6 * (r - 1 - d))));
  }
  if (LEAF) {
    // wide: the packed residue (x mod m in Montgomery form) << a | x mod 2^a, taken mod 2^64
    okey[k] = wide ? (kk << md.a) | ((hd->x20 * (alo[p] * prime)) & md.mask2)
                   : cf_key_to_canon(kk, md, hd->inv2a, hd->inv2aR);
    oid[k] = nid;
  } else {
    U128 A;
    A.lo = alo[p];
    A.hi = ahi[p];
    const U128 A2 = u128_mul64(A, prime);
    const u32 mt = meta[p];
    const u32 nl = (mt >> 16) + (SIDE == 0 && x >= split_idx ? 1u : 0u);
    okey[k] = kk;
    oalo[k] = A2.lo;
    oahi[k] = A2.hi;
    oid[k] = nid;
    ometa[k] = (nl << 16) | (u32)x;
  }
}

// ---- exclusive scan of u64 counts ---------------------------------------------
constexpr int kScanBlock = 1024;

__global__ void __launch_bounds__(kScanBlock)
k_scan_block(const u64* __restrict__ in, u64 n, u64* __restrict__ out, u64* __restrict__ sums) {
  __shared__ u64 warp_tot[32];
  const u64 i = (u64)blockIdx.x * kScanBlock + threadIdx.x;
  const u64 v = i < n ? in[i] : 0;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  u64 s = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const u64 y = __shfl_up_sync(0xffffffffu, s, o);
    if (lane >= o) s += y;
  }
  if (lane == 31) warp_tot[w] = s;
  __syncthreads();
  if (w == 0) {
    u64 t = warp_tot[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const u64 y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    warp_tot[lane] = t;                       // inclusive over warps
  }
  __syncthreads();
  const u64 before = (w ? warp_tot[w - 1] : 0) + s - v;
  if (i < n) out[i] = before;
  if (threadIdx.x == kScanBlock - 1) sums[blockIdx.x] = warp_tot[31];
}

__global__ void __launch_bounds__(kScanBlock)
k_scan_add(u64* __restrict__ out, u64 n, const u64* __restrict__ add) {
  const u64 i = (u64)blockIdx.x * kScanBlock + threadIdx.x;
  if (i < n) out[i] += add[blockIdx.x];
}

__global__ void k_scan_total(const u64* __restrict__ in, const u64* __restrict__ ex, u64 n, u64* __restrict__ out) {
  out[n] = n ? ex[n - 1] + in[n - 1] : 0;
}

u64 scan_tmp_words(u64 n) {
  u64 w = 0;
  while (n > 1) {
    n = (n + kScanBlock - 1) / kScanBlock;
    w += n + 1;
  }
  return w + 2;
}

void scan_rec(const u64* in, u64 n, u64* out, u64* tmp, cudaStream_t st) {
  const u64 nb = (n + kScanBlock - 1) / kScanBlock;
  u64* sums = tmp;
  k_scan_block<<<(unsigned)nb, kScanBlock, 0, st>>>(in, n, out, sums);
  if (nb > 1) {
    u64* sums_ex = tmp + nb + 1;
    scan_rec(sums, nb, sums_ex, sums_ex + nb + 1, st);
    k_scan_add<<<(unsigned)nb, kScanBlock, 0, st>>>(out, n, sums_ex);
  }
}

}  // namespace

// Workspace (bytes) of cf_scan_u64 for n values.
extern "C" size_t cf_scan_tmp_bytes(u64 n) { return (size_t)(scan_tmp_words(n) * 2 + 64) * 8; }

// out[0..n] = exclusive prefix sums of in[0..n), out[n] = total.
extern "C" int cf_scan_u64(const u64* in, u64 n, u64* out, void* tmp, size_t tmp_bytes, void* stream) {
  if (!out || (n && (!in || !tmp)) || n > (1ull << 40)) { cf_set_error("cf_scan_u64: bad arguments%s", ""); return CF_EBADARG; }
  const cudaStream_t st = (cudaStream_t)stream;
  if (n == 0) {
    cudaMemsetAsync(out, 0, 8, st);
    CF_LAUNCH_CHECK("cf_scan_u64");
    return CF_OK;
  }
  if (tmp_bytes < cf_scan_tmp_bytes(n)) { cf_set_error("cf_scan_u64: workspace too small%s", ""); return CF_EBADARG; }
  scan_rec(in, n, out, (u64*)tmp, st);
  k_scan_total<<<1, 1, 0, st>>>(in, out, n, out);
  CF_LAUNCH_CHECK("cf_scan_u64");
  return CF_OK;
}

// Count the children of F frontier nodes at depth d (side 0 = I, 1 = D).
// Nodes: alo/ahi (exact product), meta (last index | large-prime count << 16; the
// root has last index 0xffff).  bounds: u64 pairs (lo, hi) of H (I side) or G
// (D side), r x n, row t = positions left after the chosen index.  At depth 0
// only first indices in [xa, xb) are taken (blocks of first indices).
extern "C" int cf_bgen_count(int side, int d, int r, int n, u64 F, const u64* alo, const u64* ahi, const u32* meta,
                             const u64* bounds, int split_idx, int hmax, int xa, int xb, u64* cnt, u32* xs,
                             void* stream) {
  if ((side != 0 && side != 1) || r < 1 || r > CF_MAX_R || d < 0 || d >= r || n < 1 || n > CF_MAX_POOL ||
      !bounds || !cnt || !xs || (F && (!alo || !ahi || !meta))) {
    cf_set_error("cf_bgen_count: bad arguments%s", "");
    return CF_EBADARG;
  }
  if (F == 0) return CF_OK;
  const unsigned g = (unsigned)((F + 255) / 256);
  if (side == 0)
    k_bgen_count<0><<<g, 256, 0, (cudaStream_t)stream>>>(d, r, n, F, alo, ahi, meta, bounds, split_idx, hmax, xa, xb,
                                                         cnt, xs);
  else
    k_bgen_count<1><<<g, 256, 0, (cudaStream_t)stream>>>(d, r, n, F, alo, ahi, meta, bounds, split_idx, hmax, xa, xb,
                                                         cnt, xs);
  CF_LAUNCH_CHECK("cf_bgen_count");
  return CF_OK;
}

// Write the children [c0, c0+cc) of the depth-d frontier (offs = cf_scan_u64 of
// the counts).  d < r-1: child nodes (okey, oalo, oahi, oid, ometa); d = r-1:
// records (okey = canonical residue, oid = id).  pool: the side's pool table
// (cf_pool_prepare with mult = P0 for the I side, 1 for the D side).  A pool of
// cf_pool_prepare_split for M >= 2^64: node keys hold the odd part in Montgomery
// form and records the packed residue taken mod 2^64.
extern "C" int cf_bgen_expand(int side, int d, int r, int n, u64 F, const void* pool, const u64* key, const u64* alo,
                              const u64* ahi, const u64* id, const u32* meta, const u64* offs, const u32* xs,
                              int split_idx, int bitmask, u64 c0, u64 cc, u64* okey, u64* oalo, u64* oahi, u64* oid,
                              u32* ometa, void* stream) {
  const bool leaf = d == r - 1;
  if ((side != 0 && side != 1) || r < 1 || r > CF_MAX_R || d < 0 || d >= r || n < 1 || n > CF_MAX_POOL ||
      (side == 1 && bitmask != 2 && n > 64) || bitmask < 0 || bitmask > 2 || !pool || F == 0 || !key || !alo || !ahi || !id || !meta || !offs || !xs ||
      (cc && (!okey || !oid || (!leaf && (!oalo || !oahi || !ometa))))) {
    cf_set_error("cf_bgen_expand: bad arguments%s", "");
    return CF_EBADARG;
  }
  if (cc == 0) return CF_OK;
  const unsigned g = (unsigned)((cc + 255) / 256);
  const cudaStream_t st = (cudaStream_t)stream;
  const u64* P = (const u64*)pool;
#define CF_BGEN_LAUNCH(S, L)                                                                                  \
  k_bgen_expand<S, L><<<g, 256, 0, st>>>(d, r, n, F, P, key, alo, ahi, id, meta, offs, xs, split_idx, bitmask, \
                                         c0, cc, okey, oalo, oahi, oid, ometa)
  if (side == 0) {
    if (leaf) CF_BGEN_LAUNCH(0, true); else CF_BGEN_LAUNCH(0, false);
  } else {
    if (leaf) CF_BGEN_LAUNCH(1, true); else CF_BGEN_LAUNCH(1, false);
  }
#undef CF_BGEN_LAUNCH
  CF_LAUNCH_CHECK("cf_bgen_expand");
  return CF_OK;
}

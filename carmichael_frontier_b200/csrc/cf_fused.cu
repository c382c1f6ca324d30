// cf_fused.cu -- fused generate-and-probe join (no I-side materialisation).
//
// The D side is built once per modulus into a bucketed fingerprint table
// ("D table"): 2^bbits buckets of 16 slots.  A bucket's sixteen 16-bit
// fingerprints (0 = empty) fill one 32-byte sector -- the only data a probe
// reads; at an average load of 5-10 per bucket the fingerprint array of a
// k=64, r=5 D side (7.6M records) is 32 MB and stays in the 126 MB L2.  A side
// array holds, per slot, a second, 32-bit fingerprint and the D rank; it is
// read only when the 16-bit fingerprint matches.  A full bucket continues into
// the next one (linear probing over buckets), so lookups are complete at any
// load; the 48 fingerprint bits leave about 1e-14 false candidates per probe,
// and the exact pair check removes those.
//
// The I side is never written: each warp walks its rank range with the tail
// walker, computes every record's residue in registers and probes the table
// with one 32-byte sector read (SIMD 16-bit compares).  Every candidate is
// appended to the pair buffer and k_check_pairs keeps those whose residues are
// equal -- exactly the pair set of the reference's join_sorted
// (gpu/mitm_gpu2.py:107-119) and mitm64.cpp's probe (src/mitm64.cpp:85-101),
// with all duplicates.
#include "cf_abi_internal.h"
#include "cf_enum.cuh"

namespace {

constexpr int kFuseBlock = 256;
constexpr int kFuseSteps = 64;            // 32 x 64 = 2048 consecutive records per warp range
constexpr size_t kBinomSmemMaxF = 24 * 1024;

// Bucket and fingerprints of a residue, from its canonical odd part X (< m) and
// 2-adic part x2 (< 2^a, a <= 32): the pair is the residue, so equal residues
// give equal bucket and fingerprints.  The bucket and the 16-bit fingerprint
// are the top bbits and the next 16 bits of one 64-bit multiplicative hash;
// the 32-bit side fingerprint is an independent 32-bit fold of the residue.
struct CfFuseKey {
  u32 bucket, f16, f32;
};
__device__ __forceinline__ CfFuseKey cf_fuse_key(u64 X, u32 x2, int bbits) {
  const u64 h = (X ^ ((u64)x2 << 32)) * CF_HASH_MULT;
  CfFuseKey k;
  k.bucket = (u32)(h >> (64 - bbits));
  const u32 f = (u32)(h >> (48 - bbits)) & 0xffffu;
  k.f16 = f ? f : 1u;                       // 0 marks an empty slot
  k.f32 = (u32)X ^ ((u32)(X >> 32) * 0x85EBCA6Bu) ^ (x2 * 0xC2B2AE35u);
  return k;
}

// Canonical odd part and 2-adic part of prefix product q times tail entry e.
__device__ __forceinline__ void cf_fuse_res(CfElt32 q, const CfTailEnt& e, const CfMod32& md, u64 minv, u64& X,
                                            u32& x2) {
  X = cf_redc_mul(q.X, e.X, md.m, minv);            // q.X < 2m, e.X < m: canonical in [0, m)
  x2 = ((u32)q.x2 * e.x2) & (u32)md.mask2;          // a <= 32 on this path
}

// D table: fp16[nb*16] (32 bytes per bucket), then side[nb*16] = {fp32, rank},
// then the per-bucket fill counters used while building.
struct DTab {
  u32* fpw;       // fingerprint words: [nb * 8], two 16-bit fingerprints each
  uint2* side;    // [nb * 16]: .x = 32-bit fingerprint, .y = D rank - rank0
  u32* fill;      // [nb]: slots claimed so far (build only)
  u64 nb;         // buckets (power of two)
  u64 rank0;      // first D rank of the build
  int bbits;
};

// Insert a residue (X, x2) with its rank; returns false if every bucket was full.
// A slot is claimed with one atomicAdd on the bucket's fill counter; the claimed
// 16-bit half is then set with atomicOr (its word is shared with a neighbour slot).
__device__ __forceinline__ bool dtab_insert(const DTab& t, u64 X, u32 x2, u64 rank) {
  const CfFuseKey fk = cf_fuse_key(X, x2, t.bbits);
  const u32 f16 = fk.f16, f32 = fk.f32;
  u64 b = fk.bucket;
  for (u64 tries = 0; tries < t.nb; ++tries) {
    const u32 s = atomicAdd(&t.fill[b], 1u);
    if (s < 16u) {
      uint2 sd;
      sd.x = f32;
      sd.y = (u32)(rank - t.rank0);
      t.side[b * 16 + s] = sd;
      atomicOr(&t.fpw[b * 8 + (s >> 1)], f16 << (16 * (s & 1)));
      return true;
    }
    b = (b + 1) & (t.nb - 1);
  }
  return false;
}

__device__ __forceinline__ void emit_pair(u64 d, u64 i, CfPair* __restrict__ pairs, u32 max_pairs,
                                          u32* __restrict__ npairs, u32* __restrict__ err) {
  const u32 k = atomicAdd(npairs, 1u);
  if (k < max_pairs) {
    CfPair pr;
    pr.d_id = d;
    pr.i_id = i;
    pairs[k] = pr;
  } else {
    atomicOr(err, CF_ERR_PAIR_OVERFLOW);
  }
}

// Cold path: emit the matches of bucket b and continue through full buckets.
__device__ __noinline__ void probe_slow(const DTab& t, u64 b, u32 f16, u32 f32, u64 irank, CfPair* __restrict__ pairs,
                                        u32 max_pairs, u32* __restrict__ npairs, u32* __restrict__ err) {
  for (u64 tries = 0; tries < t.nb; ++tries) {
    const u32* row = t.fpw + b * 8;
    bool full = true;
    for (int s = 0; s < 16; ++s) {
      const u32 v = (row[s >> 1] >> (16 * (s & 1))) & 0xffffu;
      full &= (v != 0u);
      if (v == f16) {
        const uint2 sd = t.side[b * 16 + s];
        if (sd.x == f32) emit_pair(t.rank0 + sd.y, irank, pairs, max_pairs, npairs, err);
      }
    }
    if (!full) return;
    b = (b + 1) & (t.nb - 1);
  }
}

// Nonzero iff some 16-bit half of w is zero (SWAR test; exact, no false positives).
__device__ __forceinline__ u32 cf_zero_half(u32 w) { return (w - 0x00010001u) & ~w & 0x80008000u; }

// Fast test of one bucket: any 16-bit fingerprint equal to f16 (hit), or the
// bucket is full.  Slots are claimed in order, so the bucket is full exactly
// when its last slot (the high half of the last word) is occupied.
__device__ __forceinline__ bool probe_fast(uint4 r0, uint4 r1, u32 f16) {
  const u32 ff = f16 * 0x10001u;
  const u32 eq = cf_zero_half(r0.x ^ ff) | cf_zero_half(r0.y ^ ff) | cf_zero_half(r0.z ^ ff) |
                 cf_zero_half(r0.w ^ ff) | cf_zero_half(r1.x ^ ff) | cf_zero_half(r1.y ^ ff) |
                 cf_zero_half(r1.z ^ ff) | cf_zero_half(r1.w ^ ff);
  return (eq != 0u) | ((r1.w >> 16) != 0u);
}

struct FuseSmem {
  size_t p32, binom, total;
};

__host__ __device__ inline FuseSmem fuse_layout(int n, int R) {
  FuseSmem L;
  L.p32 = 0;
  size_t b = ((size_t)n * 4 + 15) & ~(size_t)15;
  const size_t bb = (size_t)(n + 1) * (R + 1) * 8;
  L.binom = (bb <= kBinomSmemMaxF) ? b : (size_t)-1;
  L.total = (bb <= kBinomSmemMaxF) ? b + bb : b;
  return L;
}

// Shared set-up of both kernels: primes and (if small) binomials in shared memory.
template <int R>
__device__ __forceinline__ const u64* fuse_setup(const u64* __restrict__ pool, unsigned char* smem, u32*& s_p) {
  const CfPoolHdr* hd = (const CfPoolHdr*)pool;
  const int n = (int)hd->n;
  const FuseSmem L = fuse_layout(n, R);
  s_p = (u32*)(smem + L.p32);
  const u64* pr = pool + cf_pool_off_prime(n);
  for (int i = threadIdx.x; i < n; i += blockDim.x) s_p[i] = (u32)pr[i];
  const u64* g_binom = pool + cf_pool_off_binom(n);
  if (L.binom == (size_t)-1) return g_binom;
  u64* sb = (u64*)(smem + L.binom);
  const int nb = (n + 1) * (R + 1);
  for (int i = threadIdx.x; i < nb; i += blockDim.x) sb[i] = g_binom[i];
  return sb;
}

// MODE 0: insert every record of [lo, lo+count) into the D table.
// MODE 1: probe every record of [lo, lo+count) against the D table.
template <int R, int MODE>
__global__ void __launch_bounds__(kFuseBlock)
k_fused(const u64* __restrict__ pool, const CfTailEnt* __restrict__ tail, u64 lo, u64 count, DTab tab,
        CfPair* __restrict__ pairs, u32 max_pairs, u32* __restrict__ npairs, u32* __restrict__ err, u32 steps) {
  constexpr int B = R < 2 ? R : 2;
  extern __shared__ __align__(16) unsigned char smem[];
  const CfPoolHdr* hd = (const CfPoolHdr*)pool;
  if (!hd->fast32 || hd->tail_b != (u64)B) {
    if (threadIdx.x == 0) atomicOr(err, CF_ERR_BAD_ARG);
    return;
  }
  const int n = (int)hd->n;
  u32* s_p;
  const u64* binom = fuse_setup<R>(pool, smem, s_p);
  CfArithFast ar;
  ar.md = cf_mod32_from_hdr(hd);
  ar.p = s_p;
  const u64 minv = hd->minv;
  CfElt32 st;
  st.X = hd->X0s;
  st.x2 = hd->x20;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const u64 per_warp = 32ull * steps;
  const u64 nwarps = (u64)gridDim.x * (kFuseBlock / 32);
  bool bad = false;
  for (u64 wbase = ((u64)blockIdx.x * (kFuseBlock / 32) + (threadIdx.x >> 5)) * per_warp; wbase < count;
       wbase += nwarps * per_warp) {
    const u32 left = (u32)((count - wbase) < per_warp ? (count - wbase) : per_warp);
    CfTailWalker<R, B> w;
    w.init(lo + wbase, n, binom, ar, st, hd->tail_n);
    const u64 rank_base = lo + wbase + (u64)lane;
    for (u32 off = 0; off < left; off += 32) {    // uniform across the warp
      CfElt32 q = st;
      u64 j;
      int unused[R - B > 0 ? R - B : 1];
      w.template step<false>(n, binom, ar, lane, q, j, unused);
      if (off + (u32)lane < left) {
        u64 X;
        u32 x2;
        cf_fuse_res(q, tail[j], ar.md, minv, X, x2);
        if (MODE == 0) {
          bad |= !dtab_insert(tab, X, x2, rank_base + off);
        } else {
          const CfFuseKey fk = cf_fuse_key(X, x2, tab.bbits);
          const uint4* row = (const uint4*)(tab.fpw + (u64)fk.bucket * 8);
          if (probe_fast(__ldg(row), __ldg(row + 1), fk.f16))
            probe_slow(tab, fk.bucket, fk.f16, fk.f32, rank_base + off, pairs, max_pairs, npairs, err);
        }
      }
    }
  }
  if (bad) atomicOr(err, CF_ERR_TABLE_FULL);
}

template <int R, int MODE>
int launch_fused(const u64* pool, const CfTailEnt* tail, int n, u64 lo, u64 count, const DTab& tab, CfPair* pairs,
                 u32 max_pairs, u32* npairs, u32* err, u32 grid, cudaStream_t st) {
  const size_t smem = fuse_layout(n, R).total;
  auto kern = k_fused<R, MODE>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cf_cuda_status(e, "cf_fused: smem attribute");
  const u32 steps = MODE == 0 ? 8u : (u32)kFuseSteps;      // the build is atomic-latency-bound: more warps
  const u64 per_cta = (u64)kFuseBlock * steps;
  u64 g = (count + per_cta - 1) / per_cta;
  if (grid && g > grid) g = grid;
  if (g == 0) g = 1;
  if (g > 0x7fffffffull) g = 0x7fffffffull;
  kern<<<(unsigned)g, kFuseBlock, smem, st>>>(pool, tail, lo, count, tab, pairs, max_pairs, npairs, err, steps);
  return CF_OK;
}

template <int R>
void dispatch_fused(int mode, const u64* pool, const CfTailEnt* tail, int n, u64 lo, u64 count, const DTab& tab,
                    CfPair* pairs, u32 max_pairs, u32* npairs, u32* err, u32 grid, cudaStream_t st, int* rc) {
  *rc = mode == 0 ? launch_fused<R, 0>(pool, tail, n, lo, count, tab, pairs, max_pairs, npairs, err, grid, st)
                  : launch_fused<R, 1>(pool, tail, n, lo, count, tab, pairs, max_pairs, npairs, err, grid, st);
}

DTab make_tab(void* tab, int bbits, u64 rank0) {
  DTab t;
  t.nb = 1ull << bbits;
  t.fpw = (u32*)tab;
  t.side = (uint2*)((unsigned char*)tab + t.nb * 32);
  t.fill = (u32*)((unsigned char*)tab + t.nb * 160);
  t.rank0 = rank0;
  t.bbits = bbits;
  return t;
}

}  // namespace

// Bytes of a D table with 2^bbits buckets (32 bytes of 16-bit fingerprints, 128
// bytes of side data and a 4-byte fill counter each).
extern "C" size_t cf_dtab_bytes(int bbits) {
  if (bbits < 1 || bbits > 30) return 0;
  return ((size_t)1 << bbits) * 164;
}

extern "C" size_t cf_dtab_fp_bytes(int bbits) {
  if (bbits < 1 || bbits > 30) return 0;
  return ((size_t)1 << bbits) * 32;
}

// Build: insert the D-side records of ranks [lo, lo+count), count < 2^32.  The
// caller zeroes the fingerprint array (the first cf_dtab_fp_bytes(bbits) bytes)
// and the fill counters (the last 4 * 2^bbits bytes) first.
extern "C" int cf_dtab_build(const void* pool_dev, const void* tail, int n, int r, u64 lo, u64 count, void* tab,
                             int bbits, u32* err, void* stream) {
  if (!pool_dev || !tail || !tab || !err || n < 1 || n > CF_MAX_POOL || r < 1 || r > CF_MAX_DISPATCH_R ||
      bbits < 1 || bbits > 28) {
    cf_set_error("cf_dtab_build: bad arguments%s", "");
    return CF_EBADARG;
  }
  if (count == 0) return CF_OK;
  if (count >= (1ull << 32)) { cf_set_error("cf_dtab_build: at most 2^32-1 D records per table%s", ""); return CF_EBADARG; }
  const DTab t = make_tab(tab, bbits, lo);
  int rc = CF_OK;
  CF_DISPATCH_R(r, dispatch_fused, 0, (const u64*)pool_dev, (const CfTailEnt*)tail, n, lo, count, t, nullptr, 0u,
                nullptr, err, 0u, (cudaStream_t)stream, &rc);
  if (rc != CF_OK) return rc;
  CF_LAUNCH_CHECK("cf_dtab_build");
  return CF_OK;
}

// Probe: generate the I-side records of ranks [lo, lo+count) in registers and
// append every (D rank, I rank) candidate whose 32-bit fingerprints agree
// through *npairs (zeroed by the caller); cf_check_pairs then keeps the pairs
// whose residues are equal.  d_rank0: first D rank of the table's build.
// grid: CTAs (0 = one per 4096 records).
extern "C" int cf_fused_probe(const void* pool_dev, const void* tail, int n, int r, u64 lo, u64 count,
                              const void* tab, int bbits, u64 d_rank0, void* pairs, u32 max_pairs, u32* npairs,
                              u32* err, u32 grid, void* stream) {
  if (!pool_dev || !tail || !tab || !npairs || !err || (max_pairs && !pairs) || n < 1 || n > CF_MAX_POOL ||
      r < 1 || r > CF_MAX_DISPATCH_R || bbits < 1 || bbits > 28) {
    cf_set_error("cf_fused_probe: bad arguments%s", "");
    return CF_EBADARG;
  }
  if (count == 0) return CF_OK;
  const DTab t = make_tab((void*)tab, bbits, d_rank0);
  int rc = CF_OK;
  CF_DISPATCH_R(r, dispatch_fused, 1, (const u64*)pool_dev, (const CfTailEnt*)tail, n, lo, count, t,
                (CfPair*)pairs, max_pairs, npairs, err, grid, (cudaStream_t)stream, &rc);
  if (rc != CF_OK) return rc;
  CF_LAUNCH_CHECK("cf_fused_probe");
  return CF_OK;
}

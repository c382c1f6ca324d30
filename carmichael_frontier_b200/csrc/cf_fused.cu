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
#include "cf_dtab.cuh"

namespace {

constexpr int kFuseBlock = 256;
constexpr int kFuseSteps = 64;            // 32 x 64 = 2048 consecutive records per warp range
constexpr int kBuildU = 4;                // build: records per lane whose slot claims are in flight together

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

// MODE 0: insert every record of [lo, lo+count) into the D table, claiming slots
//         by fill counter with kBuildU records per lane in flight (the build is
//         bound by the latency of the claims, not by their number).
// MODE 1: probe every record of [lo, lo+count) against the D table.
template <int R, int MODE, bool BLOOM>
__global__ void __launch_bounds__(kFuseBlock, 4)   // 64 registers: four CTAs per SM
k_fused(const u64* __restrict__ pool, const CfTailEnt* __restrict__ tail, u64 lo, u64 count, DTab tab,
        CfPair* __restrict__ pairs, u32 max_pairs, u32* __restrict__ npairs, u32* __restrict__ err, u32 steps,
        u32 swap) {
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
  CfPairSink sink;
  sink.pairs = pairs;
  sink.mods = nullptr;
  sink.npairs = npairs;
  sink.err = err;
  sink.max_pairs = max_pairs;
  sink.mod = 0;
  sink.swap = swap;
  const u64 per_warp = 32ull * steps;
  const u64 nwarps = (u64)gridDim.x * (kFuseBlock / 32);
  bool bad = false;
  const u64 keep = MODE == 0 ? cf_l2_build_policy(tab.nb) : 0ull;   // build: L2 priority of claims and stores
  for (u64 wbase = ((u64)blockIdx.x * (kFuseBlock / 32) + (threadIdx.x >> 5)) * per_warp; wbase < count;
       wbase += nwarps * per_warp) {
    const u32 left = (u32)((count - wbase) < per_warp ? (count - wbase) : per_warp);
    CfTailWalker<R, B> w;
    w.init(lo + wbase, n, binom, ar, st, hd->tail_n);
    const u64 rank_base = lo + wbase + (u64)lane;
    if constexpr (MODE == 0) {
      for (u32 off = 0; off < left; off += 32u * kBuildU) {   // uniform across the warp
        u32 bk[kBuildU], f16[kBuildU], f32[kBuildU], rel[kBuildU];
        bool v[kBuildU];
#pragma unroll
        for (int u = 0; u < kBuildU; ++u) {
          const u32 o = off + 32u * (u32)u;
          v[u] = false;
          if (o < left) {                        // uniform: the walker never steps past the range
            CfElt32 q = st;
            u64 j;
            int unused[R - B > 0 ? R - B : 1];
            w.template step<false>(n, binom, ar, lane, q, j, unused);
            if (o + (u32)lane < left) {
              u64 X;
              u32 x2;
              cf_fuse_res(q, tail[j], ar.md, minv, X, x2);
              if (tab.bloom) {
                const CfBloomKey bl = cf_bloom_key(X, x2, tab.fbits);
                u32* blk = tab.bloom + (u64)bl.block * 8;
                atomicOr(blk + bl.w0, bl.m0);
                atomicOr(blk + bl.w1, bl.m1);
                atomicOr(blk + bl.w2, bl.m2);
              }
              const CfFuseKey fk = cf_fuse_key(X, x2, tab.bbits);
              bk[u] = fk.bucket;
              f16[u] = fk.f16;
              f32[u] = fk.f32;
              rel[u] = (u32)(rank_base + o - tab.rank0);
              v[u] = true;
            }
          }
        }
        u32 slot[kBuildU];
#pragma unroll
        for (int u = 0; u < kBuildU; ++u) slot[u] = v[u] ? cf_atom_add_keep(tab.fill + bk[u], 1u, keep) : 16u;
#pragma unroll
        for (int u = 0; u < kBuildU; ++u)
          if (v[u]) bad |= !dtab_claim_fill(tab, bk[u], slot[u], f16[u], f32[u], rel[u], keep);
      }
    } else {
      for (u32 off = 0; off < left; off += 32) {    // uniform across the warp
        CfElt32 q = st;
        u64 j;
        int unused[R - B > 0 ? R - B : 1];
        w.template step<false>(n, binom, ar, lane, q, j, unused);
        if (off + (u32)lane < left) {
          u64 X;
          u32 x2;
          cf_fuse_res(q, tail[j], ar.md, minv, X, x2);
          if (BLOOM) {
            const CfBloomKey bk = cf_bloom_key(X, x2, tab.fbits);
            const uint4* blk = (const uint4*)(tab.bloom + (u64)bk.block * 8);
            const uint4 a = __ldg(blk), c = __ldg(blk + 1);
            const bool in = (cf_word8(a, c, bk.w0) & bk.m0) && (cf_word8(a, c, bk.w1) & bk.m1) &&
                            (cf_word8(a, c, bk.w2) & bk.m2);
            if (!in) continue;
          }
          dtab_probe(tab, X, x2, rank_base + off, sink);
        }
      }
    }
  }
  if (bad) atomicOr(err, CF_ERR_TABLE_FULL);
}

template <int R, int MODE>
int launch_fused(const u64* pool, const CfTailEnt* tail, int n, u64 lo, u64 count, const DTab& tab, CfPair* pairs,
                 u32 max_pairs, u32* npairs, u32* err, u32 grid, u32 swap, cudaStream_t st) {
  const size_t smem = fuse_layout(n, R).total;
  auto kern = (MODE == 1 && tab.bloom) ? k_fused<R, MODE, true> : k_fused<R, MODE, false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cf_cuda_status(e, "cf_fused: smem attribute");
  const u32 steps = MODE == 0 ? 8u : (u32)kFuseSteps;      // the build is atomic-latency-bound: more warps
  const u64 per_cta = (u64)kFuseBlock * steps;
  u64 g = (count + per_cta - 1) / per_cta;
  if (grid && g > grid) g = grid;
  if (g == 0) g = 1;
  if (g > 0x7fffffffull) g = 0x7fffffffull;
  kern<<<(unsigned)g, kFuseBlock, smem, st>>>(pool, tail, lo, count, tab, pairs, max_pairs, npairs, err, steps,
                                              swap);
  return CF_OK;
}

template <int R>
void dispatch_fused(int mode, const u64* pool, const CfTailEnt* tail, int n, u64 lo, u64 count, const DTab& tab,
                    CfPair* pairs, u32 max_pairs, u32* npairs, u32* err, u32 grid, u32 swap, cudaStream_t st,
                    int* rc) {
  *rc = mode == 0 ? launch_fused<R, 0>(pool, tail, n, lo, count, tab, pairs, max_pairs, npairs, err, grid, 0, st)
                  : launch_fused<R, 1>(pool, tail, n, lo, count, tab, pairs, max_pairs, npairs, err, grid, swap, st);
}

DTab make_tab(void* tab, int bbits, int fbits, u64 rank0, int compact) {
  DTab t;
  t.xb = compact ? kCompactXb : 0u;
  t.nb = 1ull << bbits;
  t.fpw = (u32*)tab;
  t.side = (uint2*)((unsigned char*)tab + t.nb * 32);
  t.fill = (u32*)((unsigned char*)tab + t.nb * 160);
  t.fbits = fbits;
  t.bloom = fbits ? (u32*)((unsigned char*)tab + t.nb * 164) : nullptr;
  t.rank0 = rank0;
  t.bbits = bbits;
  return t;
}

}  // namespace

// Bytes of a D table with 2^bbits buckets (32 bytes of 16-bit fingerprints, 128
// bytes of side data and a 4-byte fill counter each) and, when fbits > 0, a
// Bloom filter of 2^fbits 32-byte blocks after it.
extern "C" size_t cf_dtab_bytes2(int bbits, int fbits) {
  if (bbits < 1 || bbits > 28 || fbits < 0 || fbits > 26) return 0;
  return ((size_t)1 << bbits) * 164 + (fbits ? ((size_t)1 << fbits) * 32 : 0);
}

extern "C" size_t cf_dtab_bytes(int bbits) { return cf_dtab_bytes2(bbits, 0); }

extern "C" size_t cf_dtab_fp_bytes(int bbits) {
  if (bbits < 1 || bbits > 30) return 0;
  return ((size_t)1 << bbits) * 32;
}

// Build: insert the D-side records of ranks [lo, lo+count), count < 2^32, slots
// claimed by fill counter.  side_format 0: wide side entries; 1: compact side
// words (tables of at most 2^20 buckets; the probe must be told the same
// format).  The caller zeroes the fingerprint array (the first
// cf_dtab_fp_bytes(bbits) bytes), the fill counters (4 * 2^bbits bytes from
// offset 160 * 2^bbits) and the Bloom filter (when fbits > 0) first.
extern "C" int cf_dtab_build3(const void* pool_dev, const void* tail, int n, int r, u64 lo, u64 count, void* tab,
                              int bbits, int fbits, int side_format, u32* err, void* stream) {
  if (!pool_dev || !tail || !tab || !err || n < 1 || n > CF_MAX_POOL || r < 1 || r > CF_MAX_DISPATCH_R ||
      bbits < 1 || bbits > 28 || (side_format != 0 && side_format != 1)) {
    cf_set_error("cf_dtab_build: bad arguments%s", "");
    return CF_EBADARG;
  }
  if (count == 0) return CF_OK;
  if (count >= (1ull << 32)) { cf_set_error("cf_dtab_build: at most 2^32-1 D records per table%s", ""); return CF_EBADARG; }
  if (fbits < 0 || fbits > 26) { cf_set_error("cf_dtab_build: fbits must be 0..26%s", ""); return CF_EBADARG; }
  if (side_format == 1 && (bbits > kCompactMaxBbits || count > (1ull << (32 - kCompactXb)))) {
    cf_set_error("cf_dtab_build: compact side words need at most 2^20 buckets and 2^24 records%s", "");
    return CF_EBADARG;
  }
  const DTab t = make_tab(tab, bbits, fbits, lo, side_format);
  int rc = CF_OK;
  CF_DISPATCH_R(r, dispatch_fused, 0, (const u64*)pool_dev, (const CfTailEnt*)tail, n, lo, count, t, nullptr, 0u,
                nullptr, err, 0u, 0u, (cudaStream_t)stream, &rc);
  if (rc != CF_OK) return rc;
  CF_LAUNCH_CHECK("cf_dtab_build");
  return CF_OK;
}

extern "C" int cf_dtab_build2(const void* pool_dev, const void* tail, int n, int r, u64 lo, u64 count, void* tab,
                              int bbits, int fbits, u32* err, void* stream) {
  return cf_dtab_build3(pool_dev, tail, n, r, lo, count, tab, bbits, fbits, 0, err, stream);
}

extern "C" int cf_dtab_build(const void* pool_dev, const void* tail, int n, int r, u64 lo, u64 count, void* tab,
                             int bbits, u32* err, void* stream) {
  return cf_dtab_build3(pool_dev, tail, n, r, lo, count, tab, bbits, 0, 0, err, stream);
}

// Probe: generate the records of ranks [lo, lo+count) of the probing side in
// registers and append every candidate whose fingerprints agree through
// *npairs (zeroed by the caller); cf_check_pairs then keeps the pairs whose
// residues are equal.  tab_rank0: first rank of the table's build.  swap = 0:
// the table holds D records and the I side probes; swap = 1: the table holds I
// records and the D side probes (build on the smaller side).  Pairs are stored
// as {D rank, I rank} either way.  side_format: the table's (as built).  grid:
// CTAs (0 = one per 16384 records).
extern "C" int cf_fused_probe3(const void* pool_dev, const void* tail, int n, int r, u64 lo, u64 count,
                               const void* tab, int bbits, int fbits, int side_format, u64 tab_rank0, int swap,
                               void* pairs, u32 max_pairs, u32* npairs, u32* err, u32 grid, void* stream) {
  if (!pool_dev || !tail || !tab || !npairs || !err || (max_pairs && !pairs) || n < 1 || n > CF_MAX_POOL ||
      r < 1 || r > CF_MAX_DISPATCH_R || bbits < 1 || bbits > 28 || (swap != 0 && swap != 1) ||
      (side_format != 0 && side_format != 1) || (side_format == 1 && bbits > kCompactMaxBbits)) {
    cf_set_error("cf_fused_probe: bad arguments%s", "");
    return CF_EBADARG;
  }
  if (count == 0) return CF_OK;
  if (fbits < 0 || fbits > 26) { cf_set_error("cf_fused_probe: fbits must be 0..26%s", ""); return CF_EBADARG; }
  const DTab t = make_tab((void*)tab, bbits, fbits, tab_rank0, side_format);
  int rc = CF_OK;
  CF_DISPATCH_R(r, dispatch_fused, 1, (const u64*)pool_dev, (const CfTailEnt*)tail, n, lo, count, t,
                (CfPair*)pairs, max_pairs, npairs, err, grid, (u32)swap, (cudaStream_t)stream, &rc);
  if (rc != CF_OK) return rc;
  CF_LAUNCH_CHECK("cf_fused_probe");
  return CF_OK;
}

extern "C" int cf_fused_probe2(const void* pool_dev, const void* tail, int n, int r, u64 lo, u64 count,
                               const void* tab, int bbits, int fbits, u64 tab_rank0, int swap, void* pairs,
                               u32 max_pairs, u32* npairs, u32* err, u32 grid, void* stream) {
  return cf_fused_probe3(pool_dev, tail, n, r, lo, count, tab, bbits, fbits, 0, tab_rank0, swap, pairs, max_pairs,
                         npairs, err, grid, stream);
}

extern "C" int cf_fused_probe(const void* pool_dev, const void* tail, int n, int r, u64 lo, u64 count,
                              const void* tab, int bbits, u64 d_rank0, void* pairs, u32 max_pairs, u32* npairs,
                              u32* err, u32 grid, void* stream) {
  return cf_fused_probe3(pool_dev, tail, n, r, lo, count, tab, bbits, 0, 0, d_rank0, 0, pairs, max_pairs, npairs,
                         err, grid, stream);
}

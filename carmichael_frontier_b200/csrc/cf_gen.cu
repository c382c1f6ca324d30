// cf_gen.cu -- residue generation kernels.
//
//  k_gen_linear : drop-in for the reference's gen_records (gpu/mitm_gpu2.py:24-66).
//                 Record t of a launch is the subset at lexicographic rank lo+t;
//                 key = mult * prod(p) mod M (canonical residue, or internal key),
//                 id  = packed indices (`bits` per position), lex rank or colex rank.
//  k_gen_part   : the solve path's generator.  Same enumeration (fast arithmetic,
//                 primes < 2^31), but each CTA scatters its tile of records straight
//                 into 2^pbits residue partitions (partition = top bits of a
//                 multiplicative hash of the key), staged in shared memory so that
//                 every (tile, partition) run is written contiguously after ONE
//                 global atomic reservation.
#include "cf_abi_internal.h"
#include "cf_enum.cuh"

namespace {

constexpr int kLinBlock = 256;
constexpr int kLinSteps = 16;              // 32 x 16 = 512 consecutive records per warp
constexpr size_t kBinomSmemMax = 24 * 1024;

// One warp writes 32 rank-consecutive records per step straight to global
// memory (coalesced); keys converted to canonical residues when asked.
template <int R, class Ar>
__device__ __forceinline__ void cf_gen_linear_warp(const CfPoolHdr* hd, const Ar& ar, typename Ar::E start,
                                                   const u64* binom, int n, u64 lo, u64 count, int id_mode,
                                                   int bits, int canon, u64* __restrict__ keys,
                                                   u64* __restrict__ ids) {
  const int lane = threadIdx.x & 31;
  const u64 wbase = ((u64)blockIdx.x * (kLinBlock / 32) + (threadIdx.x >> 5)) * (32u * kLinSteps);
  if (wbase >= count) return;
  const CfMod md = cf_mod_from_hdr(hd);
  const bool fast = hd->fast32 != 0;
  const u64 inv2a = hd->inv2a, inv2aR = hd->inv2aR;
  CfWarpWalker<R, Ar> w;
  w.init(lo + wbase, n, binom, ar, start);
  for (int s = 0; s < kLinSteps; ++s) {
    const u64 t0 = wbase + (u64)s * 32;
    if (t0 >= count) break;                       // uniform across the warp
    typename Ar::E myA = start;
    int last;
    int myidx[R > 1 ? R - 1 : 1];
    w.template step_idx<true>(n, ar, lane, myA, last, myidx);
    const u64 t = t0 + lane;
    if (t < count) {
      u64 k = ar.key(ar.mul(myA, last));
      if (canon) {
        // fast keys hold (x mod m) in standard form, wide keys in Montgomery form
        k = fast ? cf_key_to_canon(k, md, inv2aR, inv2aR) : cf_key_to_canon(k, md, inv2a, inv2aR);
      }
      u64 id = 0;
      if (id_mode == 1) {
        id = lo + t;
      } else if (id_mode == 0) {
#pragma unroll
        for (int j = 0; j < R - 1; ++j) id |= ((u64)myidx[j]) << (j * bits);
        id |= ((u64)last) << ((R - 1) * bits);
      } else {
#pragma unroll
        for (int j = 0; j < R - 1; ++j) id += cf_binom(binom, R, myidx[j], j + 1);
        id += cf_binom(binom, R, last, R);
      }
      keys[t] = k;
      ids[t] = id;
    }
  }
}

template <int R>
__global__ void __launch_bounds__(kLinBlock)
k_gen_linear(const u64* __restrict__ pool, u64 lo, u64 count, int id_mode, int bits, int canon,
             u64* __restrict__ keys, u64* __restrict__ ids) {
  __shared__ u64 s_pk[CF_MAX_POOL];
  const CfPoolHdr* hd = (const CfPoolHdr*)pool;
  const int n = (int)hd->n;
  const bool fast = hd->fast32 != 0;
  const u64* binom = pool + cf_pool_off_binom(n);
  if (fast) {
    const u64* pr = pool + cf_pool_off_prime(n);
    u32* s_p = (u32*)s_pk;
    for (int i = threadIdx.x; i < n; i += kLinBlock) s_p[i] = (u32)pr[i];
  } else {
    const u64* pk = pool + cf_pool_off_pkey(n);
    for (int i = threadIdx.x; i < n; i += kLinBlock) s_pk[i] = pk[i];
  }
  __syncthreads();
  if (fast) {
    CfArithFast ar;
    ar.md = cf_mod32_from_hdr(hd);
    ar.p = (const u32*)s_pk;
    CfElt32 st;
    st.X = hd->X0;
    st.x2 = hd->x20;
    cf_gen_linear_warp<R>(hd, ar, st, binom, n, lo, count, id_mode, bits, canon, keys, ids);
  } else {
    CfArithWide ar;
    ar.md = cf_mod_from_hdr(hd);
    ar.pk = s_pk;
    cf_gen_linear_warp<R>(hd, ar, hd->mult_key, binom, n, lo, count, id_mode, bits, canon, keys, ids);
  }
}

// ---------------------------------------------------------------------------
// Partitioned generation.
// ---------------------------------------------------------------------------
template <int BLOCK>
__device__ __forceinline__ void block_exclusive_scan(u32* a, int len, u32* s_warp) {
  // each thread scans a contiguous chunk, then warp and block scans of chunk totals
  const int per = (len + BLOCK - 1) / BLOCK;
  const int b = threadIdx.x * per;
  const int e = min(len, b + per);
  u32 sum = 0;
  for (int i = b; i < e; ++i) sum += a[i];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  u32 incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const u32 v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) s_warp[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    constexpr int NW = BLOCK / 32;
    u32 v = (lane < NW) ? s_warp[lane] : 0;
    u32 vi = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const u32 x = __shfl_up_sync(0xffffffffu, vi, o);
      if (lane >= o) vi += x;
    }
    if (lane < NW) s_warp[lane] = vi - v;  // exclusive warp offsets
  }
  __syncthreads();
  u32 run = s_warp[wid] + incl - sum;
  for (int i = b; i < e; ++i) {
    const u32 v = a[i];
    a[i] = run;
    run += v;
  }
  __syncthreads();
}

struct GenPartSmem {
  size_t stage, part, p32, binom, hist, total;
};

__host__ __device__ inline GenPartSmem gen_part_layout(int block, int steps, int n, int R, int pbits) {
  GenPartSmem L;
  const size_t T = (size_t)block * steps;
  L.stage = 0;
  L.part = L.stage + T * sizeof(CfRec);
  L.p32 = L.part + ((T * 2 + 15) & ~(size_t)15);
  size_t b = L.p32 + (((size_t)n * 4 + 15) & ~(size_t)15);
  const size_t binom_bytes = (size_t)(n + 1) * (R + 1) * 8;
  L.binom = (binom_bytes <= kBinomSmemMax) ? b : (size_t)-1;
  if (binom_bytes <= kBinomSmemMax) b += binom_bytes;
  L.hist = b;
  L.total = b + (size_t)3 * ((size_t)1 << pbits) * 4;
  return L;
}

// Tiles of 4096 records leave room for two CTAs per SM in shared memory; the register budget is
// held to that too (512 threads: 64 registers, 1.36x the single-CTA rate on the k=64 r=5 I side).
template <int R, int BLOCK, int STEPS>
__global__ void __launch_bounds__(BLOCK, BLOCK * STEPS <= 4096 ? 2 : 1)
k_gen_part(const u64* __restrict__ pool, const CfTailEnt* __restrict__ tail, u64 lo, u64 count, int pbits,
           u32 cap, u32* __restrict__ counts, CfRec* __restrict__ out, u32* __restrict__ err) {
  constexpr int T = BLOCK * STEPS;
  static_assert(T <= 8192, "positions within a partition are packed into 13 bits");
  constexpr int B = R < 2 ? R : 2;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ u32 s_warp[BLOCK / 32];
  const CfPoolHdr* hd = (const CfPoolHdr*)pool;
  const int n = (int)hd->n;
  if (!hd->fast32 || hd->tail_b != (u64)B) {   // the solve path needs primes < 2^31 and the tail table
    if (threadIdx.x == 0) atomicOr(err, CF_ERR_BAD_ARG);
    return;
  }
  const u32 nparts = 1u << pbits;
  const GenPartSmem L = gen_part_layout(BLOCK, STEPS, n, R, pbits);
  CfRec* s_stage = (CfRec*)(smem + L.stage);
  unsigned short* s_part = (unsigned short*)(smem + L.part);
  u32* s_p = (u32*)(smem + L.p32);
  u32* s_hist = (u32*)(smem + L.hist);
  u32* s_loff = s_hist + nparts;
  u32* s_gbase = s_loff + nparts;
  const u64* g_binom = pool + cf_pool_off_binom(n);
  const u64* binom = g_binom;
  if (L.binom != (size_t)-1) {
    u64* sb = (u64*)(smem + L.binom);
    const int nb = (n + 1) * (R + 1);
    for (int i = threadIdx.x; i < nb; i += BLOCK) sb[i] = g_binom[i];
    binom = sb;
  }
  const u64* pr = pool + cf_pool_off_prime(n);
  for (int i = threadIdx.x; i < n; i += BLOCK) s_p[i] = (u32)pr[i];
  for (u32 i = threadIdx.x; i < nparts; i += BLOCK) s_hist[i] = 0;
  CfArithFast ar;
  ar.md = cf_mod32_from_hdr(hd);
  ar.p = s_p;
  const u64 minv = hd->minv;
  CfElt32 st;
  st.X = hd->X0s;
  st.x2 = hd->x20;
  __syncthreads();

  // warp w of this CTA owns the 32*STEPS consecutive ranks starting at wbase
  const int lane = threadIdx.x & 31;
  const u64 tile0 = (u64)blockIdx.x * T;
  const u64 wbase = tile0 + (u64)(threadIdx.x >> 5) * (32u * STEPS);
  u64 key[STEPS];
  u32 pp[STEPS];                                // partition << 13 | position in it (T <= 8192)
  if (wbase < count) {
    CfTailWalker<R, B> w;
    w.init(lo + wbase, n, binom, ar, st, hd->tail_n);
#pragma unroll
    for (int s = 0; s < STEPS; ++s) {
      const u64 t0 = wbase + (u64)s * 32;
      if (t0 < count) {                         // uniform across the warp
        CfElt32 q = st;
        u64 j;
        int unused[R - B > 0 ? R - B : 1];
        w.template step<false>(n, binom, ar, lane, q, j, unused);
        if (t0 + lane < count) {
          key[s] = cf_tail_key(q, tail[j], ar.md, minv);
          const u32 pt = cf_part_of(cf_hash(key[s]), pbits);
          pp[s] = (pt << 13) | atomicAdd(&s_hist[pt], 1u);
        }
      }
    }
  }
  __syncthreads();
  // reserve one global run per non-empty partition; independent atomics in flight together
  constexpr int PER = 4;
  for (u32 p0 = threadIdx.x; p0 < nparts; p0 += BLOCK * PER) {
    u32 res[PER];
#pragma unroll
    for (int u = 0; u < PER; ++u) {
      const u32 p = p0 + (u32)u * BLOCK;
      res[u] = 0;
      if (p < nparts) {
        const u32 h = s_hist[p];
        s_loff[p] = h;
        if (h) res[u] = atomicAdd(&counts[p], h);
      }
    }
#pragma unroll
    for (int u = 0; u < PER; ++u) {
      const u32 p = p0 + (u32)u * BLOCK;
      if (p < nparts) s_gbase[p] = res[u];
    }
  }
  __syncthreads();
  block_exclusive_scan<BLOCK>(s_loff, (int)nparts, s_warp);
#pragma unroll
  for (int s = 0; s < STEPS; ++s) {
    const u64 t = wbase + (u64)s * 32 + lane;
    if (t < count) {
      const u32 slot = s_loff[pp[s] >> 13] + (pp[s] & 0x1fffu);
      CfRec rc;
      rc.key = key[s];
      rc.id = lo + t;
      s_stage[slot] = rc;
      s_part[slot] = (unsigned short)(pp[s] >> 13);
    }
  }
  __syncthreads();
  const u64 left = count - tile0;
  const int tv = (int)(left < (u64)T ? left : (u64)T);
  bool ovf = false;
  for (int j = threadIdx.x; j < tv; j += BLOCK) {
    const CfRec rc = s_stage[j];
    const u32 p = s_part[j];
    const u32 dst = s_gbase[p] + ((u32)j - s_loff[p]);
    if (dst < cap) out[(size_t)p * cap + dst] = rc;
    else ovf = true;
  }
  if (ovf) atomicOr(err, CF_ERR_PART_OVERFLOW);
}

template <int R>
void launch_gen_linear(const u64* pool, u64 lo, u64 count, int id_mode, int bits, int canon, u64* keys,
                       u64* ids, cudaStream_t st) {
  const u64 per = (u64)kLinBlock * kLinSteps;
  const unsigned grid = (unsigned)((count + per - 1) / per);
  k_gen_linear<R><<<grid, kLinBlock, 0, st>>>(pool, lo, count, id_mode, bits, canon, keys, ids);
}

// Launch shapes (threads per CTA, warp steps per tile) the autotuner chooses from.
constexpr int kShapes[][2] = {{256, 16}, {512, 8}, {512, 16}, {1024, 8}};
constexpr int kNumShapes = 4;

template <int R, int BLOCK, int STEPS>
int launch_gen_part_shape(const u64* pool, const CfTailEnt* tail, int n, u64 lo, u64 count, int pbits, u32 cap,
                          u32* counts, CfRec* out, u32* err, cudaStream_t st) {
  const size_t smem = gen_part_layout(BLOCK, STEPS, n, R, pbits).total;
  if (smem > 227 * 1024) { cf_set_error("cf_gen_part: shared memory budget exceeded%s", ""); return CF_EBADARG; }
  auto kern = k_gen_part<R, BLOCK, STEPS>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cf_cuda_status(e, "cf_gen_part: smem attribute");
  const u64 per = (u64)BLOCK * STEPS;
  const unsigned grid = (unsigned)((count + per - 1) / per);
  kern<<<grid, BLOCK, smem, st>>>(pool, tail, lo, count, pbits, cap, counts, out, err);
  return CF_OK;
}

template <int R>
void launch_gen_part(const u64* pool, const CfTailEnt* tail, int n, u64 lo, u64 count, int pbits, u32 cap,
                     u32* counts, CfRec* out, u32* err, cudaStream_t st, int shape, int* rc) {
  switch (shape) {
    case 0: *rc = launch_gen_part_shape<R, 256, 16>(pool, tail, n, lo, count, pbits, cap, counts, out, err, st); break;
    case 1: *rc = launch_gen_part_shape<R, 512, 8>(pool, tail, n, lo, count, pbits, cap, counts, out, err, st); break;
    case 2: *rc = launch_gen_part_shape<R, 512, 16>(pool, tail, n, lo, count, pbits, cap, counts, out, err, st); break;
    default: *rc = launch_gen_part_shape<R, 1024, 8>(pool, tail, n, lo, count, pbits, cap, counts, out, err, st); break;
  }
}

// Tail table: entry t = product of the t-th B-subset (lexicographic) of the pool.
template <int R>
__global__ void k_build_tail(const u64* __restrict__ pool, CfTailEnt* __restrict__ tail) {
  constexpr int B = R < 2 ? R : 2;
  const CfPoolHdr* hd = (const CfPoolHdr*)pool;
  if (hd->tail_b != (u64)B) return;
  const int n = (int)hd->n;
  const u64* binom = pool + cf_pool_off_binom(n);
  const u64* pr = pool + cf_pool_off_prime(n);
  const CfMod32 md = cf_mod32_from_hdr(hd);
  const u64 tn = hd->tail_n;
  for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t < tn; t += (u64)gridDim.x * blockDim.x) {
    int idx[B];
    cf_unrank_lex_k<B, R>(t, n, binom, idx);
    CfElt32 e;
    e.X = hd->S0;
    e.x2 = 1ull & md.mask2;
    u32 ij = 0;
#pragma unroll
    for (int j = 0; j < B; ++j) {
      e = cf_mul32(e, (u32)pr[idx[j]], md);
      ij |= (u32)idx[j] << (10 * j);
    }
    CfTailEnt ent;
    ent.X = (e.X >= md.m) ? e.X - md.m : e.X;
    ent.x2 = (u32)e.x2;
    ent.ij = ij;
    tail[t] = ent;
  }
}

template <int R>
void launch_build_tail(const u64* pool, CfTailEnt* tail, u64 tn, cudaStream_t st) {
  const u64 g = (tn + 255) / 256;
  k_build_tail<R><<<(unsigned)(g < 4096 ? (g ? g : 1) : 4096), 256, 0, st>>>(pool, tail);
}

}  // namespace

extern "C" int cf_gen_subsets(const void* pool_dev, int n, int r, u64 lo, u64 count, int id_mode, int bits,
                              int canon, u64* keys, u64* ids, void* stream) {
  if (!pool_dev || n < 1 || n > CF_MAX_POOL || r < 1 || r > CF_MAX_DISPATCH_R || r > n) {
    cf_set_error("cf_gen_subsets: bad pool arguments (n 1..1024, r 1..10)%s", "");
    return CF_EBADARG;
  }
  if (id_mode < 0 || id_mode > 2 || (id_mode == 0 && (bits < 1 || r * bits > 64))) {
    cf_set_error("cf_gen_subsets: bad id mode (0 packed with r*bits<=64, 1 lex rank, 2 colex rank)%s", "");
    return CF_EBADARG;
  }
  if (count == 0) return CF_OK;
  if (!keys || !ids) { cf_set_error("cf_gen_subsets: null output%s", ""); return CF_EBADARG; }
  if (count > (1ull << 40)) { cf_set_error("cf_gen_subsets: count too large for one launch%s", ""); return CF_EBADARG; }
  cudaStream_t st = (cudaStream_t)stream;
  CF_DISPATCH_R(r, launch_gen_linear, (const u64*)pool_dev, lo, count, id_mode, bits, canon, keys, ids, st);
  CF_LAUNCH_CHECK("cf_gen_subsets");
  return CF_OK;
}

extern "C" int cf_gen_part_shapes(void) { return kNumShapes; }

extern "C" size_t cf_gen_part_smem_bytes(int n, int r, int pbits, int shape) {
  if (shape < 0 || shape >= kNumShapes || pbits < 0 || pbits > 12) return 0;
  return gen_part_layout(kShapes[shape][0], kShapes[shape][1], n, r, pbits).total;
}

static u64 host_binom(int n, int k) {
  if (k < 0 || k > n) return 0;
  unsigned __int128 v = 1;
  for (int i = 1; i <= k; ++i) v = v * (unsigned)(n - k + i) / (unsigned)i;
  return (u64)v;
}

extern "C" size_t cf_tail_bytes(int n, int r) {
  if (n < 1 || n > CF_MAX_POOL || r < 1 || r > CF_MAX_DISPATCH_R) return 0;
  return (size_t)host_binom(n, r < 2 ? r : 2) * sizeof(CfTailEnt);
}

extern "C" int cf_build_tail(const void* pool_dev, int n, int r, void* tail, void* stream) {
  if (!pool_dev || !tail || n < 1 || n > CF_MAX_POOL || r < 1 || r > CF_MAX_DISPATCH_R || r > n) {
    cf_set_error("cf_build_tail: bad arguments%s", "");
    return CF_EBADARG;
  }
  CF_DISPATCH_R(r, launch_build_tail, (const u64*)pool_dev, (CfTailEnt*)tail, host_binom(n, r < 2 ? r : 2),
                (cudaStream_t)stream);
  CF_LAUNCH_CHECK("cf_build_tail");
  return CF_OK;
}

extern "C" int cf_gen_part(const void* pool_dev, const void* tail, int n, int r, u64 lo, u64 count, int pbits,
                           u32 cap, u32* counts, void* out, u32* err, int shape, void* stream) {
  if (!pool_dev || n < 1 || n > CF_MAX_POOL || r < 1 || r > CF_MAX_DISPATCH_R || r > n) {
    cf_set_error("cf_gen_part: bad pool arguments (n 1..1024, r 1..10)%s", "");
    return CF_EBADARG;
  }
  if (pbits < 0 || pbits > 12) { cf_set_error("cf_gen_part: pbits must be 0..12%s", ""); return CF_EBADARG; }
  if (shape < 0 || shape >= kNumShapes) { cf_set_error("cf_gen_part: unknown launch shape%s", ""); return CF_EBADARG; }
  if (count == 0) return CF_OK;
  if (!counts || !out || !err || !tail) { cf_set_error("cf_gen_part: null buffer%s", ""); return CF_EBADARG; }
  if (count > (1ull << 40)) { cf_set_error("cf_gen_part: count too large for one launch%s", ""); return CF_EBADARG; }
  int rc = CF_OK;
  CF_DISPATCH_R(r, launch_gen_part, (const u64*)pool_dev, (const CfTailEnt*)tail, n, lo, count, pbits, cap, counts,
                (CfRec*)out, err, (cudaStream_t)stream, shape, &rc);
  if (rc != CF_OK) return rc;
  CF_LAUNCH_CHECK("cf_gen_part");
  return CF_OK;
}

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
constexpr int kLinItems = 8;
constexpr size_t kBinomSmemMax = 24 * 1024;

// Stage the pool's primes (u32 for the fast path, key form otherwise) and, when
// small enough, its binomial table into shared memory.
template <int R, class Ar>
__device__ __forceinline__ void cf_gen_linear_body(const u64* __restrict__ pool, const Ar& ar,
                                                   typename Ar::E start, const u64* binom, int n, u64 lo,
                                                   u64 count, int id_mode, int bits, int canon,
                                                   u64* s_k, u64* s_i) {
  const CfPoolHdr* hd = (const CfPoolHdr*)pool;
  const u64 tile0 = (u64)blockIdx.x * (kLinBlock * kLinItems);
  const u64 my0 = tile0 + (u64)threadIdx.x * kLinItems;
  if (my0 >= count) return;
  const int nv = (int)((count - my0) < (u64)kLinItems ? (count - my0) : (u64)kLinItems);
  const CfMod md = cf_mod_from_hdr(hd);
  const bool fast = hd->fast32 != 0;
  const u64 inv2a = hd->inv2a, inv2aR = hd->inv2aR;
  CfLexWalker<R, Ar> w;
  w.init(lo + my0, n, binom, ar, start);
  for (int i = 0; i < nv; ++i) {
    u64 k = w.key;
    if (canon) {
      // fast keys hold (x mod m) in standard form, wide keys in Montgomery form
      k = fast ? cf_key_to_canon(k, md, inv2aR, inv2aR) : cf_key_to_canon(k, md, inv2a, inv2aR);
    }
    u64 id;
    if (id_mode == 0) id = w.packed(bits);
    else if (id_mode == 1) id = lo + my0 + (u64)i;
    else id = cf_colex_rank<R>(w.idx, binom);
    s_k[threadIdx.x * (kLinItems + 1) + i] = k;
    s_i[threadIdx.x * (kLinItems + 1) + i] = id;
    if (i + 1 < nv) w.next(n, ar);
  }
}

template <int R>
__global__ void __launch_bounds__(kLinBlock)
k_gen_linear(const u64* __restrict__ pool, u64 lo, u64 count, int id_mode, int bits, int canon,
             u64* __restrict__ keys, u64* __restrict__ ids) {
  __shared__ u64 s_pk[CF_MAX_POOL];
  __shared__ u64 s_k[kLinBlock * (kLinItems + 1)];
  __shared__ u64 s_i[kLinBlock * (kLinItems + 1)];
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
    cf_gen_linear_body<R>(pool, ar, st, binom, n, lo, count, id_mode, bits, canon, s_k, s_i);
  } else {
    CfArithWide ar;
    ar.md = cf_mod_from_hdr(hd);
    ar.pk = s_pk;
    cf_gen_linear_body<R>(pool, ar, hd->mult_key, binom, n, lo, count, id_mode, bits, canon, s_k, s_i);
  }
  __syncthreads();
  const u64 tile0 = (u64)blockIdx.x * (kLinBlock * kLinItems);
  for (int j = threadIdx.x; j < kLinBlock * kLinItems; j += kLinBlock) {
    const u64 g = tile0 + (u64)j;
    if (g < count) {
      const int t = j / kLinItems, i = j % kLinItems;
      keys[g] = s_k[t * (kLinItems + 1) + i];
      ids[g] = s_i[t * (kLinItems + 1) + i];
    }
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
  size_t stage, p32, binom, hist, total;
};

__host__ __device__ inline GenPartSmem gen_part_layout(int block, int items, int n, int R, int pbits) {
  GenPartSmem L;
  const size_t T = (size_t)block * items;
  L.stage = 0;
  L.p32 = L.stage + T * sizeof(CfRec);
  size_t b = L.p32 + (((size_t)n * 4 + 15) & ~(size_t)15);
  const size_t binom_bytes = (size_t)(n + 1) * (R + 1) * 8;
  L.binom = (binom_bytes <= kBinomSmemMax) ? b : (size_t)-1;
  if (binom_bytes <= kBinomSmemMax) b += binom_bytes;
  L.hist = b;
  L.total = b + (size_t)3 * ((size_t)1 << pbits) * 4;
  return L;
}

template <int R, int BLOCK, int ITEMS>
__global__ void __launch_bounds__(BLOCK)
k_gen_part(const u64* __restrict__ pool, u64 lo, u64 count, int pbits, u32 cap, u32* __restrict__ counts,
           CfRec* __restrict__ out, u32* __restrict__ err) {
  constexpr int T = BLOCK * ITEMS;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ u32 s_warp[BLOCK / 32];
  const CfPoolHdr* hd = (const CfPoolHdr*)pool;
  const int n = (int)hd->n;
  if (!hd->fast32) {            // the solve path requires pool primes < 2^31
    if (threadIdx.x == 0) atomicOr(err, CF_ERR_BAD_ARG);
    return;
  }
  const u32 nparts = 1u << pbits;
  const GenPartSmem L = gen_part_layout(BLOCK, ITEMS, n, R, pbits);
  CfRec* s_stage = (CfRec*)(smem + L.stage);
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
  CfElt32 st;
  st.X = hd->X0;
  st.x2 = hd->x20;
  __syncthreads();

  const u64 tile0 = (u64)blockIdx.x * T;
  const u64 my0 = tile0 + (u64)threadIdx.x * ITEMS;
  int nv = 0;
  if (my0 < count) nv = (int)((count - my0) < (u64)ITEMS ? (count - my0) : (u64)ITEMS);
  u64 key[ITEMS];
  u32 pos[ITEMS];
  if (nv > 0) {
    CfLexWalker<R, CfArithFast> w;
    w.init(lo + my0, n, binom, ar, st);
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
      if (i < nv) {
        key[i] = w.key;
        pos[i] = atomicAdd(&s_hist[cf_part_of(cf_hash(w.key), pbits)], 1u);
        if (i + 1 < nv) w.next(n, ar);
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
  for (int i = 0; i < ITEMS; ++i) {
    if (i < nv) {
      const u32 p = cf_part_of(cf_hash(key[i]), pbits);
      CfRec rc;
      rc.key = key[i];
      rc.id = lo + my0 + (u64)i;
      s_stage[s_loff[p] + pos[i]] = rc;
    }
  }
  __syncthreads();
  const u64 left = count - tile0;
  const int tv = (int)(left < (u64)T ? left : (u64)T);
  bool ovf = false;
  for (int j = threadIdx.x; j < tv; j += BLOCK) {
    const CfRec rc = s_stage[j];
    const u32 p = cf_part_of(cf_hash(rc.key), pbits);
    const u32 dst = s_gbase[p] + ((u32)j - s_loff[p]);
    if (dst < cap) out[(size_t)p * cap + dst] = rc;
    else ovf = true;
  }
  if (ovf) atomicOr(err, CF_ERR_PART_OVERFLOW);
}

template <int R>
void launch_gen_linear(const u64* pool, u64 lo, u64 count, int id_mode, int bits, int canon, u64* keys,
                       u64* ids, cudaStream_t st) {
  const u64 per = (u64)kLinBlock * kLinItems;
  const unsigned grid = (unsigned)((count + per - 1) / per);
  k_gen_linear<R><<<grid, kLinBlock, 0, st>>>(pool, lo, count, id_mode, bits, canon, keys, ids);
}

// Launch shapes (threads per CTA, records per thread) the autotuner chooses from.
constexpr int kShapes[][2] = {{256, 16}, {512, 8}, {512, 16}, {1024, 8}};
constexpr int kNumShapes = 4;

template <int R, int BLOCK, int ITEMS>
int launch_gen_part_shape(const u64* pool, int n, u64 lo, u64 count, int pbits, u32 cap, u32* counts, CfRec* out,
                          u32* err, cudaStream_t st) {
  const size_t smem = gen_part_layout(BLOCK, ITEMS, n, R, pbits).total;
  if (smem > 227 * 1024) { cf_set_error("cf_gen_part: shared memory budget exceeded%s", ""); return CF_EBADARG; }
  auto kern = k_gen_part<R, BLOCK, ITEMS>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cf_cuda_status(e, "cf_gen_part: smem attribute");
  const u64 per = (u64)BLOCK * ITEMS;
  const unsigned grid = (unsigned)((count + per - 1) / per);
  kern<<<grid, BLOCK, smem, st>>>(pool, lo, count, pbits, cap, counts, out, err);
  return CF_OK;
}

template <int R>
void launch_gen_part(const u64* pool, int n, u64 lo, u64 count, int pbits, u32 cap, u32* counts, CfRec* out,
                     u32* err, cudaStream_t st, int shape, int* rc) {
  switch (shape) {
    case 0: *rc = launch_gen_part_shape<R, 256, 16>(pool, n, lo, count, pbits, cap, counts, out, err, st); break;
    case 1: *rc = launch_gen_part_shape<R, 512, 8>(pool, n, lo, count, pbits, cap, counts, out, err, st); break;
    case 2: *rc = launch_gen_part_shape<R, 512, 16>(pool, n, lo, count, pbits, cap, counts, out, err, st); break;
    default: *rc = launch_gen_part_shape<R, 1024, 8>(pool, n, lo, count, pbits, cap, counts, out, err, st); break;
  }
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

extern "C" int cf_gen_part(const void* pool_dev, int n, int r, u64 lo, u64 count, int pbits, u32 cap,
                           u32* counts, void* out, u32* err, int shape, void* stream) {
  if (!pool_dev || n < 1 || n > CF_MAX_POOL || r < 1 || r > CF_MAX_DISPATCH_R || r > n) {
    cf_set_error("cf_gen_part: bad pool arguments (n 1..1024, r 1..10)%s", "");
    return CF_EBADARG;
  }
  if (pbits < 0 || pbits > 12) { cf_set_error("cf_gen_part: pbits must be 0..12%s", ""); return CF_EBADARG; }
  if (shape < 0 || shape >= kNumShapes) { cf_set_error("cf_gen_part: unknown launch shape%s", ""); return CF_EBADARG; }
  if (count == 0) return CF_OK;
  if (!counts || !out || !err) { cf_set_error("cf_gen_part: null buffer%s", ""); return CF_EBADARG; }
  if (count > (1ull << 40)) { cf_set_error("cf_gen_part: count too large for one launch%s", ""); return CF_EBADARG; }
  int rc = CF_OK;
  CF_DISPATCH_R(r, launch_gen_part, (const u64*)pool_dev, n, lo, count, pbits, cap, counts, (CfRec*)out, err,
                (cudaStream_t)stream, shape, &rc);
  if (rc != CF_OK) return rc;
  CF_LAUNCH_CHECK("cf_gen_part");
  return CF_OK;
}

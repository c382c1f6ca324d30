// cf_gen.cu -- residue generation kernels.
//
//  k_gen_linear : drop-in for the reference's gen_records (gpu/mitm_gpu2.py:24-66).
//                 Record t of a launch is the subset at lexicographic rank lo+t;
//                 key = mult * prod(p) mod M (canonical residue, or key form),
//                 id  = packed indices (`bits` per position), lex rank or colex rank.
//  k_gen_part   : the solve path's generator.  Same enumeration, but each CTA
//                 scatters its tile of records straight into `nparts` residue
//                 partitions (partition = floor(key * nparts / M)), staged in
//                 shared memory so that every (tile, partition) run is written
//                 contiguously after ONE global atomic reservation.
#include "cf_abi_internal.h"
#include "cf_enum.cuh"

namespace {

constexpr int kLinBlock = 256;
constexpr int kLinItems = 8;

template <int R>
__global__ void __launch_bounds__(kLinBlock)
k_gen_linear(const u64* __restrict__ pool, u64 lo, u64 count, int id_mode, int bits, int canon,
             u64* __restrict__ keys, u64* __restrict__ ids) {
  __shared__ u64 s_pk[CF_MAX_POOL];
  __shared__ u64 s_k[kLinBlock * (kLinItems + 1)];
  __shared__ u64 s_i[kLinBlock * (kLinItems + 1)];
  const CfPoolHdr* hd = (const CfPoolHdr*)pool;
  const int n = (int)hd->n;
  const CfMod md = cf_mod_from_hdr(hd);
  const u64 mult = hd->mult_key, inv2a = hd->inv2a, inv2aR = hd->inv2aR;
  const u64* binom = pool + cf_pool_off_binom(n);
  const u64* pk = pool + cf_pool_off_pkey(n);
  for (int i = threadIdx.x; i < n; i += kLinBlock) s_pk[i] = pk[i];
  __syncthreads();

  const u64 tile0 = (u64)blockIdx.x * (kLinBlock * kLinItems);
  const u64 my0 = tile0 + (u64)threadIdx.x * kLinItems;
  if (my0 < count) {
    const int nv = (int)((count - my0) < (u64)kLinItems ? (count - my0) : (u64)kLinItems);
    CfLexWalker<R> w;
    w.init(lo + my0, n, binom, s_pk, mult, md);
    for (int i = 0; i < nv; ++i) {
      const u64 k = canon ? cf_key_to_canon(w.key, md, inv2a, inv2aR) : w.key;
      u64 id;
      if (id_mode == 0) id = w.packed(bits);
      else if (id_mode == 1) id = lo + my0 + (u64)i;
      else id = cf_colex_rank<R>(w.idx, binom);
      s_k[threadIdx.x * (kLinItems + 1) + i] = k;
      s_i[threadIdx.x * (kLinItems + 1) + i] = id;
      if (i + 1 < nv) w.next(n, s_pk, md);
    }
  }
  __syncthreads();
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

template <int R, int BLOCK, int ITEMS>
__global__ void __launch_bounds__(BLOCK)
k_gen_part(const u64* __restrict__ pool, u64 lo, u64 count, u32 nparts, u64 cpart, u32 cap,
           u32* __restrict__ counts, CfRec* __restrict__ out, u32* __restrict__ err) {
  constexpr int T = BLOCK * ITEMS;
  extern __shared__ __align__(16) unsigned char smem[];
  CfRec* s_stage = (CfRec*)smem;                          // T records
  const CfPoolHdr* hd = (const CfPoolHdr*)pool;
  const int n = (int)hd->n;
  u64* s_pk = (u64*)(s_stage + T);                         // n keys
  u32* s_hist = (u32*)(s_pk + n);                          // nparts
  u32* s_loff = s_hist + nparts;                           // nparts
  u32* s_gbase = s_loff + nparts;                          // nparts
  __shared__ u32 s_warp[BLOCK / 32];

  const CfMod md = cf_mod_from_hdr(hd);
  const u64 mult = hd->mult_key;
  const u64* binom = pool + cf_pool_off_binom(n);
  const u64* pk = pool + cf_pool_off_pkey(n);
  for (int i = threadIdx.x; i < n; i += BLOCK) s_pk[i] = pk[i];
  for (u32 i = threadIdx.x; i < nparts; i += BLOCK) s_hist[i] = 0;
  __syncthreads();

  const u64 tile0 = (u64)blockIdx.x * T;
  const u64 my0 = tile0 + (u64)threadIdx.x * ITEMS;
  int nv = 0;
  if (my0 < count) nv = (int)((count - my0) < (u64)ITEMS ? (count - my0) : (u64)ITEMS);
  u64 key[ITEMS];
  u32 pos[ITEMS];
  if (nv > 0) {
    CfLexWalker<R> w;
    w.init(lo + my0, n, binom, s_pk, mult, md);
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
      if (i < nv) {
        key[i] = w.key;
        const u32 p = (u32)cf_mulhi(w.key, cpart);
        pos[i] = atomicAdd(&s_hist[p], 1u);
        if (i + 1 < nv) w.next(n, s_pk, md);
      }
    }
  }
  __syncthreads();
  // reserve one global run per non-empty partition (before the scan overwrites s_hist)
  for (u32 p = threadIdx.x; p < nparts; p += BLOCK) {
    const u32 h = s_hist[p];
    s_loff[p] = h;
    s_gbase[p] = h ? atomicAdd(&counts[p], h) : 0u;
  }
  __syncthreads();
  block_exclusive_scan<BLOCK>(s_loff, (int)nparts, s_warp);
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    if (i < nv) {
      const u32 p = (u32)cf_mulhi(key[i], cpart);
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
    const u32 p = (u32)cf_mulhi(rc.key, cpart);
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

constexpr int kPartBlock = 256;
constexpr int kPartItems = 16;

size_t gen_part_smem(int n, u32 nparts) {
  return (size_t)kPartBlock * kPartItems * sizeof(CfRec) + (size_t)n * 8 + (size_t)nparts * 12;
}

template <int R>
void launch_gen_part(const u64* pool, int n, u64 lo, u64 count, u32 nparts, u64 cpart, u32 cap, u32* counts,
                     CfRec* out, u32* err, cudaStream_t st, int* rc) {
  const size_t smem = gen_part_smem(n, nparts);
  auto kern = k_gen_part<R, kPartBlock, kPartItems>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) { *rc = cf_cuda_status(e, "cf_gen_part: smem attribute"); return; }
  const u64 per = (u64)kPartBlock * kPartItems;
  const unsigned grid = (unsigned)((count + per - 1) / per);
  kern<<<grid, kPartBlock, smem, st>>>(pool, lo, count, nparts, cpart, cap, counts, out, err);
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

extern "C" size_t cf_gen_part_smem_bytes(int n, u32 nparts) { return gen_part_smem(n, nparts); }

extern "C" int cf_gen_part(const void* pool_dev, int n, int r, u64 lo, u64 count, u32 nparts, u64 cpart, u32 cap,
                           u32* counts, void* out, u32* err, void* stream) {
  if (!pool_dev || n < 1 || n > CF_MAX_POOL || r < 1 || r > CF_MAX_DISPATCH_R || r > n) {
    cf_set_error("cf_gen_part: bad pool arguments (n 1..1024, r 1..10)%s", "");
    return CF_EBADARG;
  }
  if (nparts < 1 || nparts > 4096 || (cpart == 0 && nparts > 1)) {
    cf_set_error("cf_gen_part: nparts must be 1..4096 with its multiplier%s", "");
    return CF_EBADARG;
  }
  if (gen_part_smem(n, nparts) > 220 * 1024) { cf_set_error("cf_gen_part: shared memory budget exceeded%s", ""); return CF_EBADARG; }
  if (count == 0) return CF_OK;
  if (!counts || !out || !err) { cf_set_error("cf_gen_part: null buffer%s", ""); return CF_EBADARG; }
  if (count > (1ull << 40)) { cf_set_error("cf_gen_part: count too large for one launch%s", ""); return CF_EBADARG; }
  int rc = CF_OK;
  CF_DISPATCH_R(r, launch_gen_part, (const u64*)pool_dev, n, lo, count, nparts, cpart, cap, counts, (CfRec*)out,
                err, (cudaStream_t)stream, &rc);
  if (rc != CF_OK) return rc;
  CF_LAUNCH_CHECK("cf_gen_part");
  return CF_OK;
}

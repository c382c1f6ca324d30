// cf_stream.cu -- range partitioning of materialised {key, id} records for the
// streamed (out-of-core) join.
//
// A side that does not fit in HBM is split by the top bits of its residue: with
// canonical keys in [0, M), partition p = floor(key * 2^pbits / M), so each
// partition is one residue range and equal residues always meet in the same
// partition.  (The reference's driver instead keeps the D side in NCHUNKS_D
// sorted pieces and streams the I side in I_CHUNK pieces, joining every I piece
// against every D piece, gpu/mitm_gpu_mstar_driver.py:100-118,241-262.)
// Partitions are then streamed through HBM one at a time and joined there.
//
// Scatter: a CTA takes a tile of records; lanes of a warp that share a
// partition are grouped with __match_any_sync and ranked by popcount, the group
// leader reserves the group's slots with one shared-memory atomic, the CTA
// reserves each partition's slots in the output with one global atomic, and
// every record is written to out[part_base[p] + cursor].  Order inside a
// partition is not kept (the join does not need it).
#include "cf_abi_internal.h"

namespace {

constexpr int kPartBlock = 512;
constexpr int kPartTile = 8192;          // records per CTA tile (16 per thread)

__device__ __forceinline__ u32 range_part(u64 key, u64 M, int pbits) {
  // floor(key * 2^pbits / M) for key < M: the quotient is below 2^pbits, found by a
  // binary search on q * M <= key * 2^pbits with both sides as 128-bit (hi, lo).
  // M = 0 stands for 2^64 (keys of a modulus of 2^64 or more, taken mod 2^64).
  const u64 rh = key >> (64 - pbits), rl = key << pbits;
  if (M == 0) return (u32)rh;
  u32 a = 0, z = (1u << pbits) - 1;
  while (a < z) {
    const u32 mid = (a + z + 1) >> 1;
    const u64 ph = __umul64hi((u64)mid, M), pl = (u64)mid * M;
    if (ph < rh || (ph == rh && pl <= rl)) a = mid; else z = mid - 1;
  }
  return a;
}

__global__ void __launch_bounds__(kPartBlock)
k_part_hist(const u64* __restrict__ keys, u64 n, u64 M, int pbits, u64* __restrict__ counts) {
  extern __shared__ u32 s_hist[];
  const int P = 1 << pbits;
  for (int i = threadIdx.x; i < P; i += blockDim.x) s_hist[i] = 0;
  __syncthreads();
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    atomicAdd(&s_hist[range_part(keys[i], M, pbits)], 1u);
  __syncthreads();
  for (int i = threadIdx.x; i < P; i += blockDim.x)
    if (s_hist[i]) atomicAdd((unsigned long long*)&counts[i], (unsigned long long)s_hist[i]);
}

__global__ void __launch_bounds__(kPartBlock)
k_part_scatter(const u64* __restrict__ keys, const u64* __restrict__ ids, u64 n, u64 M, int pbits,
               u64* __restrict__ cursor /* [P]: next free slot of each partition, from its offset */,
               u64* __restrict__ okeys, u64* __restrict__ oids) {
  extern __shared__ u32 s_mem[];
  const int P = 1 << pbits;
  u32* s_cnt = s_mem;                                   // [P] slots of the tile per partition
  unsigned long long* s_base = (unsigned long long*)(s_mem + ((P + 1) & ~1));   // [P] global base per partition
  constexpr int kPer = kPartTile / kPartBlock;
  const int lane = threadIdx.x & 31;
  for (u64 tile = (u64)blockIdx.x * kPartTile; tile < n; tile += (u64)gridDim.x * kPartTile) {
    for (int i = threadIdx.x; i < P; i += blockDim.x) s_cnt[i] = 0;
    __syncthreads();
    u32 part[kPer], rank[kPer];
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      const u64 i = tile + (u64)j * kPartBlock + threadIdx.x;
      const bool live = i < n;
      const u32 p = live ? range_part(keys[i], M, pbits) : 0xffffffffu;
      // lanes with the same partition: rank by popcount below, one shared atomic per group
      const u32 peers = __match_any_sync(0xffffffffu, p);
      const u32 below = __popc(peers & ((1u << lane) - 1u));
      const int leader = __ffs(peers) - 1;
      u32 base = 0;
      if (live && lane == leader) base = atomicAdd(&s_cnt[p], (u32)__popc(peers));
      base = __shfl_sync(0xffffffffu, base, leader);
      part[j] = p;
      rank[j] = base + below;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < P; i += blockDim.x)
      s_base[i] = s_cnt[i] ? atomicAdd((unsigned long long*)&cursor[i], (unsigned long long)s_cnt[i]) : 0ull;
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      const u64 i = tile + (u64)j * kPartBlock + threadIdx.x;
      if (i < n) {
        const u64 dst = s_base[part[j]] + rank[j];
        okeys[dst] = keys[i];
        oids[dst] = ids[i];
      }
    }
    __syncthreads();
  }
}

unsigned grid_of(u64 n, u64 per) {
  const u64 g = (n + per - 1) / per;
  return (unsigned)(g < 148ull * 8 ? (g ? g : 1) : 148ull * 8);
}

}  // namespace

// counts[p] += number of keys[0..n) in residue range p = floor(key * 2^pbits / M)
// (counts zeroed by the caller; 1 <= pbits <= 12, keys canonical, < M).
extern "C" int cf_part_hist(const u64* keys, u64 n, u64 M, int pbits, u64* counts, void* stream) {
  if (!counts || (n && !keys) || pbits < 1 || pbits > 12 || M == 1) {
    cf_set_error("cf_part_hist: bad arguments%s", "");
    return CF_EBADARG;
  }
  if (n == 0) return CF_OK;
  k_part_hist<<<grid_of(n, 1u << 16), kPartBlock, (size_t)4 << pbits, (cudaStream_t)stream>>>(keys, n, M, pbits,
                                                                                              counts);
  CF_LAUNCH_CHECK("cf_part_hist");
  return CF_OK;
}

// Scatter (keys, ids)[0..n) into the partitions: record with partition p goes to
// out[cursor[p]++] (cursor = the partitions' start offsets, advanced in place;
// the caller sizes each partition by cf_part_hist).
extern "C" int cf_part_scatter(const u64* keys, const u64* ids, u64 n, u64 M, int pbits, u64* cursor, u64* okeys,
                               u64* oids, void* stream) {
  if (!cursor || (n && (!keys || !ids || !okeys || !oids)) || pbits < 1 || pbits > 12 || M == 1) {
    cf_set_error("cf_part_scatter: bad arguments%s", "");
    return CF_EBADARG;
  }
  if (n == 0) return CF_OK;
  const size_t P = (size_t)1 << pbits;
  const size_t smem = ((P + 1) & ~(size_t)1) * 4 + P * 8;
  k_part_scatter<<<grid_of(n, kPartTile), kPartBlock, smem, (cudaStream_t)stream>>>(keys, ids, n, M, pbits, cursor,
                                                                                     okeys, oids);
  CF_LAUNCH_CHECK("cf_part_scatter");
  return CF_OK;
}

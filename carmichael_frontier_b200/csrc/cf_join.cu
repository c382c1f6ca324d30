// cf_join.cu -- partitioned equal-residue join (the solve path).
//
// Both sides were scattered by k_gen_part into the same `nparts` residue
// partitions, so equal residues meet inside one partition.  For each
// partition a CTA builds an open-addressing table of the D-side records in
// shared memory, then streams the I-side records of the same partition from
// HBM with 16-byte loads and probes.  Every equal-key (D, I) record pair is
// emitted -- the pair set of the reference's join_sorted
// (gpu/mitm_gpu2.py:107-119), which keeps all duplicates.
//
// Table slot word: (16-bit fingerprint << 16) | local D index, so a slot costs
// 4 bytes; a fingerprint hit is confirmed against the full 64-bit D key in
// global memory before a pair is emitted, so the pair set is exact.
#include "cf_abi_internal.h"

namespace {

constexpr u32 kEmpty = 0xffffffffu;
constexpr int kJoinBlock = 512;
constexpr int kUnroll = 4;

// Slot and 16-bit fingerprint from the hash bits just below the partition bits.
__device__ __forceinline__ void slot_fp(u64 key, int pbits, int sbits, u32& slot, u32& fp) {
  const u64 h = cf_hash(key) << pbits;
  slot = (u32)(h >> (64 - sbits));
  fp = (u32)(h >> (48 - sbits)) & 0xffffu;
}

__global__ void __launch_bounds__(kJoinBlock)
k_join_part(const CfRec* __restrict__ D, const u32* __restrict__ dcount, u32 capD,
            const CfRec* __restrict__ I, const u32* __restrict__ icount, u32 capI, int pbits,
            int sbits, u32 isplit, CfPair* __restrict__ pairs, u32 max_pairs, u32* __restrict__ npairs,
            u32* __restrict__ err) {
  extern __shared__ u32 s_tab[];
  const u32 S = 1u << sbits, smask = S - 1, dmax = S >> 1;
  const u32 nparts = 1u << pbits;
  const u32 nwork = nparts * isplit;
  for (u32 w = blockIdx.x; w < nwork; w += gridDim.x) {
    const u32 p = w / isplit, part = w % isplit;
    const u32 nd = min(dcount[p], capD);
    const u32 niall = min(icount[p], capI);
    const u32 i0 = (u32)(((u64)niall * part) / isplit), i1 = (u32)(((u64)niall * (part + 1)) / isplit);
    const CfRec* Dp = D + (size_t)p * capD;
    const CfRec* Ip = I + (size_t)p * capI;
    for (u32 d0 = 0; d0 < nd; d0 += dmax) {          // one round unless the partition is oversized
      const u32 d1 = min(nd, d0 + dmax);
      for (u32 s = threadIdx.x; s < S; s += kJoinBlock) s_tab[s] = kEmpty;
      __syncthreads();
      for (u32 d = d0 + threadIdx.x; d < d1; d += kJoinBlock) {
        u32 slot, fp;
        slot_fp(Dp[d].key, pbits, sbits, slot, fp);
        const u32 v = (fp << 16) | (d - d0);
        for (u32 tries = 0; tries < S; ++tries) {      // load <= 1/2: always finds a slot
          const u32 old = atomicCAS(&s_tab[slot], kEmpty, v);
          if (old == kEmpty) break;
          slot = (slot + 1) & smask;
        }
      }
      __syncthreads();
      for (u32 ib = i0 + threadIdx.x; ib < i1; ib += kJoinBlock * kUnroll) {
        CfRec rc[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
          const u32 i = ib + (u32)u * kJoinBlock;
          if (i < i1) rc[u] = Ip[i];
        }
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
          const u32 i = ib + (u32)u * kJoinBlock;
          if (i >= i1) continue;
          u32 slot, fp;
          slot_fp(rc[u].key, pbits, sbits, slot, fp);
          for (u32 tries = 0; tries < S; ++tries) {
            const u32 v = s_tab[slot];
            if (v == kEmpty) break;
            if ((v >> 16) == fp) {
              const u32 dl = d0 + (v & 0xffffu);
              const CfRec dr = Dp[dl];
              if (dr.key == rc[u].key) {
                const u32 k = atomicAdd(npairs, 1u);
                if (k < max_pairs) {
                  CfPair pr;
                  pr.d_id = dr.id;
                  pr.i_id = rc[u].id;
                  pairs[k] = pr;
                } else {
                  atomicOr(err, CF_ERR_PAIR_OVERFLOW);
                }
              }
            }
            slot = (slot + 1) & smask;
          }
        }
      }
      __syncthreads();
    }
  }
}

}  // namespace

extern "C" size_t cf_join_part_smem_bytes(int sbits) { return (size_t)4 << sbits; }

extern "C" int cf_join_part(const void* D, const u32* dcount, u32 capD, const void* I, const u32* icount, u32 capI,
                            int pbits, int sbits, u32 isplit, u32 grid, void* pairs, u32 max_pairs,
                            u32* npairs, u32* err, void* stream) {
  if (sbits < 4 || sbits > 15) { cf_set_error("cf_join_part: sbits must be 4..15%s", ""); return CF_EBADARG; }
  if (pbits < 0 || pbits > 12 || isplit < 1 || isplit > 4096) { cf_set_error("cf_join_part: bad partition counts%s", ""); return CF_EBADARG; }
  const u32 nparts = 1u << pbits;
  if (!D || !dcount || !I || !icount || !npairs || !err || (max_pairs && !pairs)) {
    cf_set_error("cf_join_part: null buffer%s", "");
    return CF_EBADARG;
  }
  const size_t smem = (size_t)4 << sbits;
  cudaError_t e = cudaFuncSetAttribute(k_join_part, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cf_cuda_status(e, "cf_join_part: smem attribute");
  const u32 nwork = nparts * isplit;
  const u32 g = (grid == 0 || grid > nwork) ? nwork : grid;
  k_join_part<<<g, kJoinBlock, smem, (cudaStream_t)stream>>>((const CfRec*)D, dcount, capD, (const CfRec*)I, icount,
                                                            capI, pbits, sbits, isplit, (CfPair*)pairs,
                                                            max_pairs, npairs, err);
  CF_LAUNCH_CHECK("cf_join_part");
  return CF_OK;
}

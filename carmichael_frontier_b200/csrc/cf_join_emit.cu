// cf_join_emit.cu -- the equal-key join of two sorted sides with its pairs
// written on the device, in the reference's order: the C entry points behind
// join_sorted (gpu/mitm_gpu2.py:107-119).
//
//   cf_join_count  for every I row the number of D keys equal to it (the
//                  difference of the two searchsorted positions), then an
//                  exclusive scan of those counts: per-row offsets and the
//                  pair total (a device u64);
//   cf_join_emit   every pair {Did[p], Iid[row]} at its row's offset -- I rows
//                  in order and, within a row, D positions in order, which is
//                  the order join_sorted returns.
//
// Each thread of the count takes a run of consecutive I keys, finds the first D
// key not below its first key by binary search and gallops forward (the sides
// are sorted, so the run's positions only grow).  Equal keys are rare, so the
// emit kernel searches again only for the rows with a nonzero count.
#include "cf_abi_internal.h"

extern "C" size_t cf_scan_tmp_bytes(u64 n);
extern "C" int cf_scan_u64(const u64* in, u64 n, u64* out, void* tmp, size_t tmp_bytes, void* stream);

namespace {

constexpr int kJoinBlock = 256;
constexpr int kJoinRun = 16;

__device__ __forceinline__ u64 lower_bound(const u64* __restrict__ a, u64 lo, u64 hi, u64 key) {
  while (lo < hi) {
    const u64 mid = lo + ((hi - lo) >> 1);
    if (a[mid] < key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__global__ void __launch_bounds__(kJoinBlock)
k_join_count(const u64* __restrict__ Dk, u64 nD, const u64* __restrict__ Ik, u64 nI, u64* __restrict__ cnt) {
  const u64 t = (u64)blockIdx.x * kJoinBlock + threadIdx.x;
  const u64 r0 = t * kJoinRun;
  if (r0 >= nI) return;
  const u64 r1 = (r0 + kJoinRun < nI) ? r0 + kJoinRun : nI;
  u64 pos = lower_bound(Dk, 0, nD, Ik[r0]);
  for (u64 r = r0; r < r1; ++r) {
    const u64 key = Ik[r];
    if (pos < nD && Dk[pos] < key) {          // gallop to the first D key >= key
      u64 step = 1, lo = pos + 1, hi = pos + 1;
      while (hi < nD && Dk[hi] < key) { lo = hi + 1; hi = pos + (step <<= 1); }
      if (hi > nD) hi = nD;
      pos = lower_bound(Dk, lo, hi, key);
    }
    u64 q = pos;
    while (q < nD && Dk[q] == key) ++q;
    cnt[r] = q - pos;
  }
}

__global__ void __launch_bounds__(kJoinBlock)
k_join_emit(const u64* __restrict__ Dk, const u64* __restrict__ Did, u64 nD, const u64* __restrict__ Ik,
            const u64* __restrict__ Iid, u64 nI, const u64* __restrict__ offs, u64* __restrict__ oD,
            u64* __restrict__ oI, u64 max_pairs) {
  for (u64 r = (u64)blockIdx.x * kJoinBlock + threadIdx.x; r < nI; r += (u64)gridDim.x * kJoinBlock) {
    const u64 a = offs[r], b = offs[r + 1];
    if (a == b) continue;
    const u64 key = Ik[r], iid = Iid[r];
    const u64 p0 = lower_bound(Dk, 0, nD, key);
    for (u64 k = a; k < b && k < max_pairs; ++k) {
      oD[k] = Did[p0 + (k - a)];
      oI[k] = iid;
    }
  }
}

size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

// Workspace of cf_join_count / cf_join_emit for nI I records: the per-row
// counts, their exclusive scan (nI + 1 offsets) and the scan's scratch.
extern "C" size_t cf_join_tmp_bytes(u64 nI) {
  return up256((size_t)nI * 8) + up256((size_t)(nI + 1) * 8) + cf_scan_tmp_bytes(nI ? nI : 1);
}

// Count the equal-key pairs of sorted Dk[nD] and sorted Ik[nI]: the per-row
// offsets stay in tmp for cf_join_emit, the total goes to *npairs (a device
// u64, read it after the stream reaches this point).
extern "C" int cf_join_count(const u64* Dk, u64 nD, const u64* Ik, u64 nI, void* tmp, size_t tmp_bytes,
                             u64* npairs, void* stream) {
  if (!npairs || (nI && (!Ik || !tmp)) || (nD && !Dk) || nI > (1ull << 40) || nD > (1ull << 40)) {
    cf_set_error("cf_join_count: bad arguments%s", "");
    return CF_EBADARG;
  }
  const cudaStream_t st = (cudaStream_t)stream;
  if (nI == 0) return cf_cuda_status(cudaMemsetAsync(npairs, 0, 8, st), "cf_join_count");
  if (tmp_bytes < cf_join_tmp_bytes(nI)) { cf_set_error("cf_join_count: workspace too small%s", ""); return CF_ENOMEM; }
  unsigned char* w = (unsigned char*)tmp;
  u64* cnt = (u64*)w;
  u64* offs = (u64*)(w + up256((size_t)nI * 8));
  void* stmp = w + up256((size_t)nI * 8) + up256((size_t)(nI + 1) * 8);
  if (nD == 0) {
    const cudaError_t e = cudaMemsetAsync(cnt, 0, (size_t)nI * 8, st);
    if (e != cudaSuccess) return cf_cuda_status(e, "cf_join_count");
  } else {
    const u64 threads = (nI + kJoinRun - 1) / kJoinRun;
    k_join_count<<<(unsigned)((threads + kJoinBlock - 1) / kJoinBlock), kJoinBlock, 0, st>>>(Dk, nD, Ik, nI, cnt);
    CF_LAUNCH_CHECK("cf_join_count");
  }
  const int rc = cf_scan_u64(cnt, nI, offs, stmp, cf_scan_tmp_bytes(nI), stream);
  if (rc != CF_OK) return rc;
  return cf_cuda_status(cudaMemcpyAsync(npairs, offs + nI, 8, cudaMemcpyDeviceToDevice, st), "cf_join_count: total");
}

// Write the pairs counted by cf_join_count (same sides, same tmp): outD[k],
// outI[k] for k < min(total, max_pairs), in join_sorted's order.
extern "C" int cf_join_emit(const u64* Dk, const u64* Did, u64 nD, const u64* Ik, const u64* Iid, u64 nI,
                            const void* tmp, u64* outD, u64* outI, u64 max_pairs, void* stream) {
  if (nI == 0 || nD == 0 || max_pairs == 0) return CF_OK;
  if (!Dk || !Did || !Ik || !Iid || !tmp || !outD || !outI) {
    cf_set_error("cf_join_emit: bad arguments%s", "");
    return CF_EBADARG;
  }
  const u64* offs = (const u64*)((const unsigned char*)tmp + up256((size_t)nI * 8));
  const u64 blocks = (nI + kJoinBlock - 1) / kJoinBlock;
  k_join_emit<<<(unsigned)(blocks < 65535 * 16 ? blocks : 65535 * 16), kJoinBlock, 0, (cudaStream_t)stream>>>(
      Dk, Did, nD, Ik, Iid, nI, offs, outD, outI, max_pairs);
  CF_LAUNCH_CHECK("cf_join_emit");
  return CF_OK;
}

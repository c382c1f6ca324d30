// cf_check.cu -- exact verification of candidate pairs on the device.
//
// For each (D, I) pair from the join: unrank both lexicographic ranks, recompute
// both residues from scratch (they must be equal), run the conservative fp64
// log-size pre-screen  log2 P0 - sum log2 d + sum log2 i <= log2 B + eps, and for
// every survivor the exact checks:
//   size     n = prod(B0 \ D) * prod(I) <= B      (32-bit limbs, exact)
//   Korselt  prod(S) == 1 (mod p-1) for every p in S
//   distinct the k primes of S are pairwise distinct.
// The reference performs the same checks on the host in Python integers
// (gpu/mitm_gpu_mstar_driver.py:226-237) and by ref/ref_carmichael.py:55-72.
#include "cf_check.cuh"

namespace {

template <int R>
__global__ void __launch_bounds__(128)
k_check_pairs(const u64* __restrict__ poolD, const u64* __restrict__ poolI, const CfScreen* __restrict__ scr,
              const CfPair* __restrict__ pairs, const u32* __restrict__ npairs, u32 max_pairs,
              CfPairResult* __restrict__ res, u32* __restrict__ err) {
  (void)err;
  const u32 np = min(*npairs, max_pairs);
  for (u32 t = blockIdx.x * blockDim.x + threadIdx.x; t < np; t += gridDim.x * blockDim.x)
    res[t] = cf_check_one<R>(poolD, poolI, scr, pairs[t]);
}

template <int R>
void launch_check(const u64* poolD, const u64* poolI, const CfScreen* scr, const CfPair* pairs, const u32* npairs,
                  u32 max_pairs, CfPairResult* res, u32* err, cudaStream_t st) {
  const u32 grid = max_pairs ? (u32)((max_pairs + 127) / 128) : 1u;
  k_check_pairs<R><<<grid < 1024u ? grid : 1024u, 128, 0, st>>>(poolD, poolI, scr, pairs, npairs, max_pairs, res,
                                                                err);
}

}  // namespace

extern "C" size_t cf_pair_result_bytes(void) { return sizeof(CfPairResult); }

extern "C" int cf_check_pairs(const void* poolD, const void* poolI, const void* screen, int r, const void* pairs,
                              const u32* npairs, u32 max_pairs, void* results, u32* err, void* stream) {
  if (!poolD || !poolI || !screen || !npairs || !err || r < 1 || r > CF_MAX_DISPATCH_R) {
    cf_set_error("cf_check_pairs: bad arguments%s", "");
    return CF_EBADARG;
  }
  if (max_pairs == 0) return CF_OK;
  if (!pairs || !results) { cf_set_error("cf_check_pairs: null buffer%s", ""); return CF_EBADARG; }
  CF_DISPATCH_R(r, launch_check, (const u64*)poolD, (const u64*)poolI, (const CfScreen*)screen,
                (const CfPair*)pairs, npairs, max_pairs, (CfPairResult*)results, err, (cudaStream_t)stream);
  CF_LAUNCH_CHECK("cf_check_pairs");
  return CF_OK;
}

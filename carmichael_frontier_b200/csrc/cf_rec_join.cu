// cf_rec_join.cu -- hash join of two materialised record sides (the product-
// bounded producers' output): the table of cf_dtab.cuh built from the smaller
// side's keys, probed by the other side's keys.
//
// Keys are canonical residues; equal residues give equal buckets and
// fingerprints (the hash is a function of the key alone), so every equal-key
// pair is emitted, plus rare fingerprint collisions that the caller removes by
// comparing the keys.  Pairs carry record positions {D position, I position};
// this is the join of the reference's sorted sides (gpu/mitm_gpu2.py:107-119,
// as run_instance uses it on the filtered sides, gpu/mitm_gpu_mstar_driver.py:
// 241-262) without sorting either side.
#include "cf_dtab.cuh"

namespace {

DTab rec_tab(void* tab, int bbits, int fbits) {
  DTab t;
  t.xb = 0;                  // wide side entries
  t.nb = 1ull << bbits;
  t.fpw = (u32*)tab;
  t.side = (uint2*)((unsigned char*)tab + t.nb * 32);
  t.fill = (u32*)((unsigned char*)tab + t.nb * 160);
  t.bloom = fbits ? (u32*)((unsigned char*)tab + t.nb * 164) : nullptr;
  t.rank0 = 0;
  t.bbits = bbits;
  t.fbits = fbits;
  return t;
}

__global__ void __launch_bounds__(256)
k_rec_build(const u64* __restrict__ keys, u64 n, DTab tab, u32* __restrict__ err) {
  bool ok = true;
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    ok &= dtab_insert(tab, keys[i], 0u, i);
  if (!ok) atomicOr(err, CF_ERR_TABLE_FULL);
}

// Insert canonical residues keys[0..n) under their key form of the pool's modulus: the odd part in
// Montgomery form (x * 2^64 mod m, one product with 2^128 mod m) over the 2-adic part -- the form in
// which the bounded producers' nodes carry products, so that their leaves probe without converting.
__global__ void __launch_bounds__(256)
k_rec_build_keyform(const u64* __restrict__ keys, u64 n, DTab tab, const u64* __restrict__ pool, u32* __restrict__ err) {
  const CfPoolHdr* hd = (const CfPoolHdr*)pool;
  const CfMod md = cf_mod_from_hdr(hd);
  const u64 r2 = hd->r2;
  bool ok = true;
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
    const u64 k = keys[i];
    const u64 kf = (cf_redc_mul(k, r2, md.m, md.minv) << md.a) | (k & md.mask2);   // k * r2 < 2^64 * m
    ok &= dtab_insert(tab, kf, 0u, i);
  }
  if (!ok) atomicOr(err, CF_ERR_TABLE_FULL);
}

__global__ void __launch_bounds__(256)
k_rec_probe(const u64* __restrict__ keys, u64 n, DTab tab, CfPairSink sink) {
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
    const u64 X = keys[i];
    if (tab.bloom) {
      const CfBloomKey bk = cf_bloom_key(X, 0u, tab.fbits);
      const uint4* blk = (const uint4*)(tab.bloom + (u64)bk.block * 8);
      const uint4 a = __ldg(blk), c = __ldg(blk + 1);
      if (!((cf_word8(a, c, bk.w0) & bk.m0) && (cf_word8(a, c, bk.w1) & bk.m1) && (cf_word8(a, c, bk.w2) & bk.m2)))
        continue;
    }
    dtab_probe(tab, X, 0u, i, sink);
  }
}

unsigned grid_for(u64 n) {
  const u64 g = (n + 255) / 256;
  return (unsigned)(g < 148ull * 32 ? (g ? g : 1) : 148ull * 32);
}

}  // namespace

// Insert keys[0..n) (positions as ranks, n < 2^32) into a table laid out as
// cf_dtab_bytes2(bbits, fbits) (fingerprints, fill counters and Bloom filter
// zeroed by the caller).
extern "C" int cf_rec_build(const u64* keys, u64 n, void* tab, int bbits, int fbits, u32* err, void* stream) {
  if (!tab || !err || (n && !keys) || bbits < 1 || bbits > 28 || fbits < 0 || fbits > 26 || n >= (1ull << 32)) {
    cf_set_error("cf_rec_build: bad arguments%s", "");
    return CF_EBADARG;
  }
  if (n == 0) return CF_OK;
  k_rec_build<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(keys, n, rec_tab(tab, bbits, fbits), err);
  CF_LAUNCH_CHECK("cf_rec_build");
  return CF_OK;
}

// The same table from canonical residues inserted under the key form of the modulus of `pool` (a
// pool table on the device): the table a probe by key-form leaves (cf_bgen_probe_keyform) reads.
extern "C" int cf_rec_build_keyform(const u64* keys, u64 n, void* tab, int bbits, int fbits, const void* pool,
                                    u32* err, void* stream) {
  if (!tab || !err || !pool || (n && !keys) || bbits < 1 || bbits > 28 || fbits < 0 || fbits > 26 ||
      n >= (1ull << 32)) {
    cf_set_error("cf_rec_build_keyform: bad arguments%s", "");
    return CF_EBADARG;
  }
  if (n == 0) return CF_OK;
  k_rec_build_keyform<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(keys, n, rec_tab(tab, bbits, fbits),
                                                                       (const u64*)pool, err);
  CF_LAUNCH_CHECK("cf_rec_build_keyform");
  return CF_OK;
}

// Probe with keys[0..n): every candidate {table position, probe position} --
// stored as {D position, I position}: swap = 0 when the table holds the D side,
// 1 when it holds the I side -- goes to pairs through *npairs (zeroed by the
// caller).  Candidates include rare fingerprint collisions: compare the keys.
extern "C" int cf_rec_probe(const u64* keys, u64 n, const void* tab, int bbits, int fbits, int swap, void* pairs,
                            u32 max_pairs, u32* npairs, u32* err, void* stream) {
  if (!tab || !npairs || !err || (n && !keys) || (max_pairs && !pairs) || bbits < 1 || bbits > 28 || fbits < 0 ||
      fbits > 26 || (swap != 0 && swap != 1)) {
    cf_set_error("cf_rec_probe: bad arguments%s", "");
    return CF_EBADARG;
  }
  if (n == 0) return CF_OK;
  CfPairSink sink;
  sink.pairs = (CfPair*)pairs;
  sink.mods = nullptr;
  sink.npairs = npairs;
  sink.err = err;
  sink.max_pairs = max_pairs;
  sink.mod = 0;
  sink.swap = (u32)swap;
  k_rec_probe<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(keys, n, rec_tab((void*)tab, bbits, fbits), sink);
  CF_LAUNCH_CHECK("cf_rec_probe");
  return CF_OK;
}

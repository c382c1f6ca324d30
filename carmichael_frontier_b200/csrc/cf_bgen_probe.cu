// cf_bgen_probe.cu -- last level of the bounded I-side enumeration fused with the
// probe of a record table: the I leaves are computed and probed in registers and
// never written.
//
// Under a size bound the D side (Dmin filter) is usually small while the I side
// (Icap filter) can stay large; the reference materialises both and sort-joins
// them (gpu/mitm_gpu_mstar_driver.py:241-262, igen chunks against the sorted D
// chunks).  Here the D records are inserted into the table of cf_dtab.cuh
// (cf_rec_build) and every I leaf -- child x of a depth-(r-1) frontier node,
// key = P0 * prod(I) mod M, id = colex rank -- probes it.  Candidates are stored
// as {D record position, I colex id}; the caller removes the rare fingerprint
// collisions by recomputing the I key from the id.
#include "cf_dtab.cuh"

namespace {

constexpr int kLeavesPerThread = 32;       // consecutive leaves per thread: one parent search each

// KEYFORM: the table holds key forms (cf_rec_build_keyform) and the leaves probe with theirs; else the
// table holds canonical residues and every leaf is converted first (two Montgomery products).
template <bool KEYFORM>
__global__ void __launch_bounds__(256)
k_bgen_probe(int r, int n, u64 F, const u64* __restrict__ pool, const u64* __restrict__ key,
             const u64* __restrict__ id, const u64* __restrict__ offs, const u32* __restrict__ xs, u64 c0, u64 cc,
             DTab tab, CfPairSink sink) {
  const u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x;
  const u64 first = t * kLeavesPerThread;
  if (first >= cc) return;
  const u64 end = (first + kLeavesPerThread < cc) ? first + kLeavesPerThread : cc;
  const CfPoolHdr* hd = (const CfPoolHdr*)pool;
  const CfMod md = cf_mod_from_hdr(hd);
  const u64* pkey = pool + cf_pool_off_pkey(n);
  const u64* binom = pool + cf_pool_off_binom(n);
  u64 c = c0 + first;
  u64 a = 0, b = F - 1;                       // parent of the first leaf: largest p with offs[p] <= c
  while (a < b) {
    const u64 mid = (a + b + 1) >> 1;
    if (offs[mid] <= c) a = mid; else b = mid - 1;
  }
  u64 p = a;
  for (u64 k = first; k < end; ++k, ++c) {
    while (p + 1 < F && offs[p + 1] <= c) ++p;  // consecutive leaves share or follow their parent
    const int x = (int)(xs[p] + (c - offs[p]));
    const u64 kk = cf_mul_key(key[p], pkey[x], md);
    const u64 X = KEYFORM ? kk : cf_key_to_canon(kk, md, hd->inv2a, hd->inv2aR);
    const u64 iid = id[p] + binom[(size_t)x * (r + 1) + r];      // colex: + C(x, r)
    if (tab.bloom) {
      const CfBloomKey bk = cf_bloom_key(X, 0u, tab.fbits);
      const uint4* blk = (const uint4*)(tab.bloom + (u64)bk.block * 8);
      const uint4 u = __ldg(blk), v = __ldg(blk + 1);
      if (!((cf_word8(u, v, bk.w0) & bk.m0) && (cf_word8(u, v, bk.w1) & bk.m1) && (cf_word8(u, v, bk.w2) & bk.m2)))
        continue;
    }
    dtab_probe(tab, X, 0u, iid, sink);
  }
}

}  // namespace

// Probe the leaves [c0, c0+cc) of a depth-(r-1) I-side frontier (cf_bgen_count +
// cf_scan_u64 at d = r-1, as for cf_bgen_expand) against a table built by
// cf_rec_build from D records.  Candidates {D position, I colex id} go to pairs
// through *npairs (zeroed by the caller).
static int bgen_probe(bool keyform, int r, int n, u64 F, const void* pool, const u64* key, const u64* id,
                      const u64* offs, const u32* xs, u64 c0, u64 cc, const void* tab, int bbits, int fbits,
                      void* pairs, u32 max_pairs, u32* npairs, u32* err, void* stream) {
  if (r < 1 || r > CF_MAX_R || n < 1 || n > CF_MAX_POOL || F == 0 || !pool || !key || !id || !offs || !xs || !tab ||
      !npairs || !err || (max_pairs && !pairs) || bbits < 1 || bbits > 28 || fbits < 0 || fbits > 26) {
    cf_set_error("cf_bgen_probe: bad arguments%s", "");
    return CF_EBADARG;
  }
  if (cc == 0) return CF_OK;
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
  CfPairSink sink;
  sink.pairs = (CfPair*)pairs;
  sink.mods = nullptr;
  sink.npairs = npairs;
  sink.err = err;
  sink.max_pairs = max_pairs;
  sink.mod = 0;
  sink.swap = 0;
  const u64 threads = (cc + kLeavesPerThread - 1) / kLeavesPerThread;
  auto kern = keyform ? k_bgen_probe<true> : k_bgen_probe<false>;
  kern<<<(unsigned)((threads + 255) / 256), 256, 0, (cudaStream_t)stream>>>(r, n, F, (const u64*)pool, key, id, offs,
                                                                          xs, c0, cc, t, sink);
  CF_LAUNCH_CHECK("cf_bgen_probe");
  return CF_OK;
}

extern "C" int cf_bgen_probe(int r, int n, u64 F, const void* pool, const u64* key, const u64* id, const u64* offs,
                             const u32* xs, u64 c0, u64 cc, const void* tab, int bbits, int fbits, void* pairs,
                             u32 max_pairs, u32* npairs, u32* err, void* stream) {
  return bgen_probe(false, r, n, F, pool, key, id, offs, xs, c0, cc, tab, bbits, fbits, pairs, max_pairs, npairs,
                    err, stream);
}

// The same probe of a table built by cf_rec_build_keyform with the same pool's modulus: the leaves
// probe with their key forms, without the conversion to canonical residues.
extern "C" int cf_bgen_probe_keyform(int r, int n, u64 F, const void* pool, const u64* key, const u64* id,
                                     const u64* offs, const u32* xs, u64 c0, u64 cc, const void* tab, int bbits,
                                     int fbits, void* pairs, u32 max_pairs, u32* npairs, u32* err, void* stream) {
  return bgen_probe(true, r, n, F, pool, key, id, offs, xs, c0, cc, tab, bbits, fbits, pairs, max_pairs, npairs,
                    err, stream);
}

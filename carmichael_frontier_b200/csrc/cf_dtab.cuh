// cf_dtab.cuh -- the D table of the fused join (shared by the single-modulus
// kernels in cf_fused.cu and the batched portfolio kernels in cf_batch.cu).
//
// 2^bbits buckets of 16 slots.  A bucket's sixteen 16-bit fingerprints (0 =
// empty) fill one 32-byte sector -- the only data a probe reads; a side array
// holds, per slot, more fingerprint bits and the D rank (read only when the
// 16-bit fingerprint matches).  Slots are claimed in order -- by a per-bucket
// fill counter (the in-place single-modulus build) or by compare-and-swap on
// the fingerprint words (record tables, batched in-place builds) -- so "bucket
// full" is a test of the last slot, and a full bucket continues into the next
// one.  An optional blocked Bloom filter is a first level for tables too large
// for L2.
#pragma once
#include "cf_abi_internal.h"
#include "cf_enum.cuh"

constexpr size_t kBinomSmemMaxF = 24 * 1024;


// Bucket and fingerprints of a residue, from its canonical odd part X (< m) and
// 2-adic part x2 (< 2^a, a <= 32): the pair is the residue, so equal residues
// give equal bucket and fingerprints.  The bucket and the 16-bit fingerprint
// are the top bbits and the next 16 bits of one 64-bit multiplicative hash;
// the 32-bit side fingerprint is an independent 32-bit fold of the residue.
struct CfFuseKey {
  u32 bucket, f16, f32;
};
__device__ __forceinline__ u32 cf_fuse_f32(u64 X, u32 x2) {
  return (u32)X ^ ((u32)(X >> 32) * 0x85EBCA6Bu) ^ (x2 * 0xC2B2AE35u);
}
__device__ __forceinline__ void cf_fuse_bucket(u64 X, u32 x2, int bbits, u32& bucket, u32& f16) {
  const u64 h = (X ^ ((u64)x2 << 32)) * CF_HASH_MULT;
  bucket = (u32)(h >> (64 - bbits));
  const u32 f = (u32)(h >> (48 - bbits)) & 0xffffu;
  f16 = f ? f : 1u;                         // 0 marks an empty slot
}
__device__ __forceinline__ CfFuseKey cf_fuse_key(u64 X, u32 x2, int bbits) {
  CfFuseKey k;
  cf_fuse_bucket(X, x2, bbits, k.bucket, k.f16);
  k.f32 = cf_fuse_f32(X, x2);
  return k;
}

// Canonical odd part and 2-adic part of prefix product q times tail entry e.
__device__ __forceinline__ void cf_fuse_res(CfElt32 q, const CfTailEnt& e, const CfMod32& md, u64 minv, u64& X,
                                            u32& x2) {
  X = cf_redc_mul(q.X, e.X, md.m, minv);            // q.X < 2m, e.X < m: canonical in [0, m)
  x2 = ((u32)q.x2 * e.x2) & (u32)md.mask2;          // a <= 32 on this path
}

// D table: fp16[nb*16] (32 bytes per bucket), then the side area (128 bytes per
// bucket), then the per-bucket fill counters used while building.  "D table"
// names the structure; it holds whichever side of the join is smaller.
//
// Two side formats.  Wide (xb = 0): side[nb*16] = {fp32, rank - rank0}, 8 bytes
// per slot.  Compact (xb = 8, tables of at most 2^20 buckets, so at most 2^24
// records): one 32-bit word per slot, (rank - rank0) << 8 | the low 8 bits of
// the 32-bit fingerprint, at ((u32*)side)[b*16 + s] -- 64 bytes per bucket, half
// the footprint, so that an in-place build of an L2-sized table keeps its side
// words in L2 instead of evicting partly written sectors.  The 24 fingerprint
// bits (16 + 8) leave about 2e-7 false candidates per probe at 7 records per
// bucket; the exact pair check removes them.
struct DTab {
  u32* fpw;       // fingerprint words: [nb * 8], two 16-bit fingerprints each
  uint2* side;    // wide: [nb * 16] {32-bit fingerprint, rank - rank0}; compact: [nb * 16] u32 words
  u32* fill;      // [nb]: slots claimed so far (builds by fill counter)
  u32* bloom;     // optional first level: [2^fbits * 8] words (256-bit blocks), nullptr if off
  u64 nb;         // buckets (power of two)
  u64 rank0;      // first rank of the build
  int bbits;
  int fbits;
  u32 xb;         // 0: wide side entries; 8: compact side words
};

constexpr u32 kCompactXb = 8;
constexpr int kCompactMaxBbits = 20;

// Blocked Bloom filter over the residues, for D tables too large for L2: a
// 256-bit block (one 32-byte sector) per key, three bits set in it; a probe
// that misses a bit skips the DRAM-resident table.  The block and bit indices
// come from a second 64-bit hash, independent of the table's.
struct CfBloomKey {
  u32 block, w0, w1, w2, m0, m1, m2;
};
__device__ __forceinline__ CfBloomKey cf_bloom_key(u64 X, u32 x2, int fbits) {
  const u64 g = (X * 0xC2B2AE3D27D4EB4Full) ^ ((u64)x2 * 0x165667B19E3779F9ull);
  const u64 h = (g ^ (g >> 29)) * 0xD6E8FEB86659FD93ull;
  CfBloomKey k;
  k.block = (u32)(h >> (64 - fbits));
  const u32 b0 = (u32)(h >> 8) & 255u, b1 = (u32)(h >> 16) & 255u, b2 = (u32)(h >> 24) & 255u;
  k.w0 = b0 >> 5; k.m0 = 1u << (b0 & 31);
  k.w1 = b1 >> 5; k.m1 = 1u << (b1 & 31);
  k.w2 = b2 >> 5; k.m2 = 1u << (b2 & 31);
  return k;
}

__device__ __forceinline__ u32 cf_word8(uint4 a, uint4 b, u32 w) {
  const u32 v[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
  u32 r = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) r = (w == (u32)i) ? v[i] : r;
  return r;
}

// Claim a slot for (f16, side entry sd) in bucket b or, when b is full, in the
// first non-full bucket after it; returns false if every bucket was full.
// A slot is claimed with one compare-and-swap on the fingerprint word holding the
// bucket's first empty 16-bit half: slots are only ever set, and a claim always
// takes the first empty slot it sees, so the occupied slots of a bucket are a
// prefix and "bucket full" is "last slot occupied".  A failed swap means another
// thread filled that word first; the claim retries with the value it returned
// (at most 16 slots per bucket, so the retries are bounded).  The side entry is
// written after the claim; probes run only after the build has completed.
__device__ __forceinline__ bool dtab_claim(const DTab& t, u64 b, u32 f16, uint2 sd) {
  for (u64 tries = 0; tries < t.nb; ++tries) {
    u32* row = t.fpw + b * 8;
    const uint4 r0 = __ldcg((const uint4*)row), r1 = __ldcg((const uint4*)row + 1);
    const u32 w8[8] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w};
    int w = 0;                                     // first word with an empty half
#pragma unroll
    for (int i = 7; i >= 0; --i)
      if ((w8[i] & 0xffff0000u) == 0u) w = i;
    if ((w8[7] & 0xffff0000u) != 0u) w = 8;        // last slot occupied: bucket full
    u32 cur = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) cur = (w == i) ? w8[i] : cur;
    // each pass either claims a slot, sees one more slot filled by another thread,
    // or moves to the next word: at most 16 + 8 passes per bucket
    for (int spin = 0; w < 8 && spin < 32; ++spin) {
      if ((cur & 0xffff0000u) != 0u) {             // this word is full: move to the next one
        ++w;
        cur = (w < 8) ? __ldcg(&row[w]) : 0u;
        continue;
      }
      const bool lo_free = (cur & 0xffffu) == 0u;
      const u32 nv = lo_free ? (cur | f16) : (cur | (f16 << 16));
      const u32 prev = atomicCAS(&row[w], cur, nv);
      if (prev == cur) {
        t.side[b * 16 + 2 * w + (lo_free ? 0 : 1)] = sd;
        return true;
      }
      cur = prev;
    }
    b = (b + 1) & (t.nb - 1);
  }
  return false;
}

// L2 eviction policy of the in-place build's claims and stores.  For tables of at most
// 2^20 buckets (fingerprints, compact side words and fill counters about 100 MB, inside the
// 126 MB L2) it is evict-last, so that the table's partly written sectors stay in L2 until
// the build has filled them instead of leaving for DRAM half written and coming back for the
// next slot (config-2 tables: build 16% faster); larger tables keep the normal priority.
__device__ __forceinline__ u64 cf_l2_build_policy(u64 nb) {
  u64 last, normal;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(last));
  asm volatile("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(normal));
  return nb <= (1ull << kCompactMaxBbits) ? last : normal;
}
__device__ __forceinline__ u32 cf_atom_add_keep(u32* a, u32 v, u64 pol) {
  u32 old;
  asm volatile("atom.global.add.L2::cache_hint.u32 %0, [%1], %2, %3;" : "=r"(old) : "l"(a), "r"(v), "l"(pol)
               : "memory");
  return old;
}
__device__ __forceinline__ void cf_st_keep_u16(unsigned short* a, unsigned short v, u64 pol) {
  asm volatile("st.global.L2::cache_hint.b16 [%0], %1, %2;" ::"l"(a), "h"(v), "l"(pol) : "memory");
}
__device__ __forceinline__ void cf_st_keep_u32(u32* a, u32 v, u64 pol) {
  asm volatile("st.global.L2::cache_hint.b32 [%0], %1, %2;" ::"l"(a), "r"(v), "l"(pol) : "memory");
}

// Fill a claimed slot s of bucket b: its 16-bit fingerprint (a 16-bit store into
// the bucket's row) and its side entry in the table's format.
__device__ __forceinline__ void dtab_place(const DTab& t, u64 b, u32 s, u32 f16, u32 f32, u32 rel, u64 pol) {
  cf_st_keep_u16(reinterpret_cast<unsigned short*>(t.fpw) + b * 16 + s, (unsigned short)f16, pol);
  if (t.xb)
    cf_st_keep_u32(reinterpret_cast<u32*>(t.side) + b * 16 + s,
                   (rel << kCompactXb) | (f32 & ((1u << kCompactXb) - 1u)), pol);
  else
    t.side[b * 16 + s] = make_uint2(f32, rel);
}

// Claim by fill counter: slot s = atomicAdd(fill[b], 1) of bucket b (first_slot,
// claimed by the caller) or, while s >= 16 (bucket full), of the next buckets.
// Every claimed slot is written before the build ends, so when probes run the
// occupied slots of a bucket are a prefix and "bucket full" is "last slot
// occupied" -- the layout the probe expects.  Returns false if every bucket was
// full.
__device__ __forceinline__ bool dtab_claim_fill(const DTab& t, u64 b, u32 first_slot, u32 f16, u32 f32, u32 rel,
                                                u64 pol) {
  u32 s = first_slot;
  for (u64 tries = 0; tries < t.nb; ++tries) {
    if (s < 16u) {
      dtab_place(t, b, s, f16, f32, rel, pol);
      return true;
    }
    b = (b + 1) & (t.nb - 1);
    s = cf_atom_add_keep(t.fill + b, 1u, pol);
  }
  return false;
}

// Insert a residue (X, x2) with its rank; returns false if every bucket was full.
__device__ __forceinline__ bool dtab_insert(const DTab& t, u64 X, u32 x2, u64 rank) {
  if (t.bloom) {
    const CfBloomKey bk = cf_bloom_key(X, x2, t.fbits);
    u32* blk = t.bloom + (u64)bk.block * 8;
    atomicOr(blk + bk.w0, bk.m0);
    atomicOr(blk + bk.w1, bk.m1);
    atomicOr(blk + bk.w2, bk.m2);
  }
  const CfFuseKey fk = cf_fuse_key(X, x2, t.bbits);
  return dtab_claim(t, fk.bucket, fk.f16, make_uint2(fk.f32, (u32)(rank - t.rank0)));
}

// Pair sink: candidates go to pairs[k] through the counter *npairs; in batched
// runs the modulus index goes to mods[k] as well (mods == nullptr otherwise).
// The table holds the smaller side: the D side (swap = 0) or the I side (swap =
// 1, the D side probes); pairs are always stored as {D rank, I rank}.
struct CfPairSink {
  CfPair* pairs;
  u32* mods;
  u32* npairs;
  u32* err;
  u32 max_pairs;
  u32 mod;
  u32 swap;
};

__device__ __forceinline__ void emit_pair(u64 stored, u64 probing, const CfPairSink& o) {
  const u32 k = atomicAdd(o.npairs, 1u);
  if (k < o.max_pairs) {
    CfPair pr;
    pr.d_id = o.swap ? probing : stored;
    pr.i_id = o.swap ? stored : probing;
    o.pairs[k] = pr;
    if (o.mods) o.mods[k] = o.mod;
  } else {
    atomicOr(o.err, CF_ERR_PAIR_OVERFLOW);
  }
}

// Cold path: emit the matches of bucket b and continue through full buckets.
static __device__ __noinline__ void probe_slow(const DTab& t, u64 b, u32 f16, u32 f32, u64 irank,
                                               const CfPairSink& o) {
  for (u64 tries = 0; tries < t.nb; ++tries) {
    const u32* row = t.fpw + b * 8;
    bool full = true;
    for (int s = 0; s < 16; ++s) {
      const u32 v = (row[s >> 1] >> (16 * (s & 1))) & 0xffffu;
      full &= (v != 0u);
      if (v == f16) {
        if (t.xb) {
          const u32 w = reinterpret_cast<const u32*>(t.side)[b * 16 + s];
          if ((w & ((1u << kCompactXb) - 1u)) == (f32 & ((1u << kCompactXb) - 1u)))
            emit_pair(t.rank0 + (w >> kCompactXb), irank, o);
        } else {
          const uint2 sd = t.side[b * 16 + s];
          if (sd.x == f32) emit_pair(t.rank0 + sd.y, irank, o);
        }
      }
    }
    if (!full) return;
    b = (b + 1) & (t.nb - 1);
  }
}

// Nonzero iff some 16-bit half of w is zero (SWAR test; exact, no false positives).
__device__ __forceinline__ u32 cf_zero_half(u32 w) { return (w - 0x00010001u) & ~w & 0x80008000u; }

// Any 16-bit fingerprint of a bucket's row equal to f16 (SWAR over the eight
// words).  Slots are claimed in order, so the bucket is full exactly when its
// last slot (the high half of the last word) is occupied.
__device__ __forceinline__ bool probe_match(uint4 r0, uint4 r1, u32 f16) {
  // (t - 0x00010001) & ~t per word, OR-ed over the words before the one mask: the same
  // bits as OR-ing the eight masked tests, one three-input logic op per word
  const u32 ff = f16 * 0x10001u;
  const u32 w[8] = {r0.x ^ ff, r0.y ^ ff, r0.z ^ ff, r0.w ^ ff, r1.x ^ ff, r1.y ^ ff, r1.z ^ ff, r1.w ^ ff};
  u32 acc = 0u;
#pragma unroll
  for (int i = 0; i < 8; ++i) acc |= (w[i] - 0x00010001u) & ~w[i];
  return (acc & 0x80008000u) != 0u;
}

// Probe the table for one residue.  The bucket's fingerprint row is tested in
// registers and, while that bucket is full, so are the rows after it (a full
// bucket is common at 8-12 records per bucket, and sending it to the cold path
// would hold up the whole warp); only a 16-bit fingerprint match, or a chain
// longer than kProbeHops rows, takes the cold path, which emits the matches of
// the chain from that bucket on.
constexpr int kProbeHops = 4;

// One bucket's 32-byte fingerprint row.  With a 32-byte aligned table it is one
// 256-bit load that bypasses L1 (a random row has no reuse there, and one request
// per probe instead of two halves the L1 traffic that bounds the probe);
// otherwise two 128-bit loads.
__device__ __forceinline__ void dtab_row(const u32* row, bool wide, uint4& r0, uint4& r1) {
  if (wide) {
    asm("ld.global.nc.L1::no_allocate.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(r0.x), "=r"(r0.y), "=r"(r0.z), "=r"(r0.w), "=r"(r1.x), "=r"(r1.y), "=r"(r1.z), "=r"(r1.w)
        : "l"(row));
  } else {
    r0 = __ldg((const uint4*)row);
    r1 = __ldg((const uint4*)row + 1);
  }
}

// The rest of a probe whose first row (bucket b) is already in registers: test it and, while
// the bucket is full, the rows after it.
__device__ __forceinline__ void dtab_probe_rows(const DTab& t, u64 b, u32 f16, uint4 r0, uint4 r1, u64 X, u32 x2,
                                                u64 rank, const CfPairSink& o, bool wide) {
#pragma unroll 1
  for (int hop = 0;; ++hop) {
    const bool full = (r1.w >> 16) != 0u;
    if (probe_match(r0, r1, f16) || (full && hop == kProbeHops - 1)) {
      probe_slow(t, b, f16, cf_fuse_f32(X, x2), rank, o);   // the side fingerprint: cold path only
      return;
    }
    if (!full) return;
    b = (b + 1) & (t.nb - 1);
    dtab_row(t.fpw + b * 8, wide, r0, r1);
  }
}

// Probe for the residue (X, x2) (x2 = 0 for keys that carry the whole residue in X).
__device__ __forceinline__ void dtab_probe(const DTab& t, u64 X, u32 x2, u64 rank, const CfPairSink& o) {
  u32 bucket, f16;
  cf_fuse_bucket(X, x2, t.bbits, bucket, f16);
  const bool wide = ((uintptr_t)t.fpw & 31u) == 0u;
  uint4 r0, r1;
  dtab_row(t.fpw + (u64)bucket * 8, wide, r0, r1);
  dtab_probe_rows(t, bucket, f16, r0, r1, X, x2, rank, o, wide);
}


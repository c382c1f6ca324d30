// cf_common.cuh -- arithmetic and table layouts shared by every kernel of the
// exchange meet-in-the-middle residue join, and by the host code that prepares
// the tables.
//
// Residue representation ("key form").  The modulus M (< 2^64, odd part < 2^63) is split as
// M = 2^a * m with m odd.  A residue x mod M is held as
//     key(x) = (X << a) | (x mod 2^a),   X = x * 2^64 mod m   (Montgomery form)
// which is a bijection of [0, M) onto [0, M): equal keys <=> equal residues,
// exactly as the reference's canonical u64 residues (gpu/mitm_gpu2.py:4-5), so
// the join never needs the canonical value.  Products are computed without any
// 128-bit division: the odd part by one Montgomery reduction (four 64-bit
// multiplies, mul.lo/mul.hi), the 2-adic part by one low-word multiply.
// The drop-in generator converts back to the canonical residue by CRT.
#pragma once
#include <stdint.h>
#include <stddef.h>

#if defined(__CUDACC__)
#define CF_HD __host__ __device__ __forceinline__
#else
#define CF_HD static inline
#endif

typedef unsigned long long u64;
typedef unsigned int u32;

CF_HD u64 cf_mulhi(u64 a, u64 b) {
#if defined(__CUDA_ARCH__)
  return __umul64hi(a, b);
#else
  return (u64)(((unsigned __int128)a * b) >> 64);
#endif
}

// Montgomery product: x*y*2^-64 mod m, for x*y < m*2^64; result in [0, m).
CF_HD u64 cf_redc_mul(u64 x, u64 y, u64 m, u64 minv) {
  const u64 lo = x * y;
  const u64 hi = cf_mulhi(x, y);
  const u64 u = lo * minv;            // u*m == lo (mod 2^64)
  const u64 mh = cf_mulhi(u, m);      // (x*y - u*m) / 2^64 = hi - mh exactly
  const u64 r = hi - mh;
  return (hi < mh) ? r + m : r;
}

// Everything a kernel needs to multiply keys modulo M.
struct CfMod {
  u64 m;      // odd part of M
  u64 minv;   // m^-1 mod 2^64
  u64 mask2;  // 2^a - 1
  int a;      // 2-adic valuation of M
};

// key(x) * key(y) = key(x*y mod M)
CF_HD u64 cf_mul_key(u64 kx, u64 ky, const CfMod& md) {
  const u64 X = cf_redc_mul(kx >> md.a, ky >> md.a, md.m, md.minv);
  return (X << md.a) | ((kx * ky) & md.mask2);
}

// ---------------------------------------------------------------------------
// Fast path for pool primes p < 2^31 (every pool of the search): a lazy
// Montgomery step with a 32-bit radix.  For x < 2m and p < 2^31,
//     cf_redc32(x, p) = x * p * 2^-32 mod m,  result in [0, 2m),
// in five 32x32->64 multiply(-add)s.  A product of R primes therefore carries
// the constant 2^(-32R); the start value is pre-scaled by 2^(32R) so that the
// final value, reduced once to [0, m), is exactly mult * prod(p) mod m.
// Together with the 2-adic part x mod 2^a the pair is the canonical residue
// mod M (Chinese remainder theorem), packed as key = (x mod m) << a | x mod 2^a.
// ---------------------------------------------------------------------------
struct CfMod32 {
  u64 m;      // odd part of M (< 2^63: values stay below 2m < 2^64)
  u64 mask2;  // 2^a - 1
  u32 ninv;   // -m^-1 mod 2^32
  u32 ml, mh; // low and high 32-bit halves of m
  int a;
};

CF_HD u64 cf_redc32(u64 x, u32 p, const CfMod32& md) {
  const u32 xl = (u32)x, xh = (u32)(x >> 32);
  const u64 lo = (u64)xl * p;                  // x = xh*2^32 + xl
  const u32 u = (u32)lo * md.ninv;             // t + u*m == 0 (mod 2^32)
  const u64 s1 = (u64)u * md.ml + (u32)lo;     // < 2^64; its low 32 bits are 0
  u64 r = (u64)xh * p + (lo >> 32);
  r += (u64)u * md.mh;
  return r + (s1 >> 32);
}

// Element of the fast path: odd part X in [0, 2m) (lazily reduced), 2-adic part x2.
struct CfElt32 {
  u64 X, x2;
};

CF_HD CfElt32 cf_mul32(CfElt32 e, u32 p, const CfMod32& md) {
  CfElt32 o;
  o.X = cf_redc32(e.X, p, md);
  o.x2 = (e.x2 * (u64)p) & md.mask2;
  return o;
}

CF_HD u64 cf_key32(CfElt32 e, const CfMod32& md) {
  const u64 X = (e.X >= md.m) ? e.X - md.m : e.X;
  return (X << md.a) | e.x2;
}

// Residue partitions and in-partition hash: a multiplicative (Fibonacci) hash
// of the key, so partitions are balanced whatever the structure of M.
#define CF_HASH_MULT 0x9E3779B97F4A7C15ull
CF_HD u64 cf_hash(u64 key) { return key * CF_HASH_MULT; }
CF_HD u32 cf_part_of(u64 h, int pbits) { return pbits ? (u32)(h >> (64 - pbits)) : 0u; }

// ---------------------------------------------------------------------------
// Pool table: one blob per (prime list, radius, modulus, multiplier), prepared
// on the host by cf_pool_prepare() and copied to the device by the caller.
// Layout (u64 words):
//   [0, CF_POOL_HDR_WORDS)            header (CfPoolHdr)
//   pkey[n]                          key(p_i mod M)
//   prime[n]                         p_i as given
//   lg[n]                            log2(p_i) as IEEE double (bit pattern)
//   binom[(n+1)*(R+1)]               C(x, y) for x <= n, y <= R, saturated at 2^64-1
// ---------------------------------------------------------------------------
#define CF_POOL_MAGIC 0x43464d49544d3031ull /* "CFMITM01" */
#define CF_POOL_HDR_WORDS 32
#define CF_MAX_POOL 1024
#define CF_MAX_R 16

struct CfPoolHdr {
  u64 magic;
  u64 M, m, minv, mask2;
  u64 a, n, R;
  u64 mult_key;    // key(mult mod M): first factor of every product
  u64 total;       // C(n, R) (saturated)
  u64 inv2a;       // (2^a)^-1 mod m                  (canonical conversion)
  u64 inv2aR;      // (2^a)^-1 * 2^64 mod m           (canonical conversion)
  u64 r2;          // 2^128 mod m
  u64 one_key;     // key(1)
  u64 fast32;      // 1 if every prime < 2^31 (fast path available)
  u64 X0;          // fast path start: (mult mod m) * 2^(32R) mod m
  u64 x20;         // fast path start: mult mod 2^a
  u64 ninv32;      // -m^-1 mod 2^32
  u64 tail_b;      // suffix length b of the tail table (0: no tail table for this pool)
  u64 tail_n;      // C(n, b): entries of the tail table
  u64 X0s;         // tail path start: (mult mod m) * 2^(32(R-b)) mod m
  u64 S0;          // tail table start: 2^(64 + 32b) mod m
  u64 reserved[CF_POOL_HDR_WORDS - 22];
};

CF_HD size_t cf_pool_words(int n, int R) {
  return (size_t)CF_POOL_HDR_WORDS + 3 * (size_t)n + (size_t)(n + 1) * (size_t)(R + 1);
}
CF_HD size_t cf_pool_off_pkey(int) { return CF_POOL_HDR_WORDS; }
CF_HD size_t cf_pool_off_prime(int n) { return CF_POOL_HDR_WORDS + (size_t)n; }
CF_HD size_t cf_pool_off_lg(int n) { return CF_POOL_HDR_WORDS + 2 * (size_t)n; }
CF_HD size_t cf_pool_off_binom(int n) { return CF_POOL_HDR_WORDS + 3 * (size_t)n; }

CF_HD CfMod32 cf_mod32_from_hdr(const CfPoolHdr* h) {
  CfMod32 md;
  md.m = h->m;
  md.mask2 = h->mask2;
  md.ninv = (u32)h->ninv32;
  md.ml = (u32)h->m;
  md.mh = (u32)(h->m >> 32);
  md.a = (int)h->a;
  return md;
}

CF_HD CfMod cf_mod_from_hdr(const CfPoolHdr* h) {
  CfMod md;
  md.m = h->m;
  md.minv = h->minv;
  md.mask2 = h->mask2;
  md.a = (int)h->a;
  return md;
}

// key -> canonical residue in [0, M) (Chinese remaindering of the Montgomery
// odd part and the 2-adic part).
CF_HD u64 cf_key_to_canon(u64 k, const CfMod& md, u64 inv2a, u64 inv2aR) {
  const u64 X = k >> md.a;
  const u64 x2 = k & md.mask2;
  const u64 t = cf_redc_mul(X, inv2a, md.m, md.minv);    // x_m * 2^-a
  const u64 s = cf_redc_mul(x2, inv2aR, md.m, md.minv);  // x_2 * 2^-a
  const u64 q = (t >= s) ? (t - s) : (t + md.m - s);     // (x_m - x_2) * 2^-a mod m
  return x2 + (q << md.a);
}

// Tail table entry: the product of one b-subset (b <= 3) of the pool, lexicographic
// order, as odd part in Montgomery form (x * 2^64 mod m, canonical) and 2-adic
// part; the subset's indices packed 10 bits each.
struct __align__(16) CfTailEnt {
  u64 X;
  u32 x2;
  u32 ij;
};

// Record of one subset: residue key and the subset's identifier (its
// lexicographic combinatorial-number-system rank, or a packed index word).
struct __align__(16) CfRec {
  u64 key;
  u64 id;
};

// Candidate pair emitted by the join: D-side and I-side identifiers.
struct __align__(16) CfPair {
  u64 d_id;
  u64 i_id;
};

// Result of the exact check of one pair (see cf_check.cu).
#define CF_HIT_KEY_EQUAL 1u      // residues recomputed from the ranks are equal
#define CF_HIT_SCREEN 2u         // fp64 log-size pre-screen passed (conservative)
#define CF_HIT_SIZE_EXACT 4u     // exact big-integer check prod(S) <= B passed
#define CF_HIT_KORSELT 8u        // (p-1) | (prod(S)-1) for every p in S
#define CF_HIT_DISJOINT 16u      // S has k distinct primes
struct CfPairResult {
  u32 flags;
  u32 r;
  unsigned short d_idx[CF_MAX_R];
  unsigned short i_idx[CF_MAX_R];
};

// Screen table: size bound and base product for the pair check.
#define CF_SCREEN_MAX_LIMBS 64   // B < 2^2048
struct CfScreen {
  double lgP0;      // log2(prod B0)
  double lgB;       // log2(B)
  double eps;       // conservative margin of the fp64 pre-screen
  u32 nlimbs;       // limbs of B (little-endian base 2^32)
  u32 pad;
  u32 limbsB[CF_SCREEN_MAX_LIMBS];
};

// Error word bits written by kernels (the host turns them into statuses).
#define CF_ERR_PART_OVERFLOW 1u  // a partition received more records than its capacity
#define CF_ERR_PAIR_OVERFLOW 2u  // more candidate pairs than the pair buffer holds
#define CF_ERR_TABLE_FULL 4u     // hash table could not place a record (never expected)
#define CF_ERR_SPIN_LIMIT 8u     // a bounded wait gave up (look-back or queue)
#define CF_ERR_KEY_MISMATCH 16u  // a checked pair's residues differ (internal error)
#define CF_ERR_BAD_ARG 32u

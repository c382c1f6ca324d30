// cf_prepare.cu -- host-side preparation of the small tables the kernels read
// (pool tables and the size-screen table), plus the library's error string.
// Pure host code: exact 128-bit integer arithmetic, no device calls.
#include <math.h>
#include <stdio.h>
#include <string.h>
#include "cf_abi_internal.h"

static thread_local char g_err[512] = "ok";

void cf_set_error(const char* fmt, const char* detail) {
  snprintf(g_err, sizeof g_err, fmt, detail ? detail : "");
}

extern "C" const char* cf_last_error_string(void) { return g_err; }

extern "C" int cf_version(void) { return CF_ABI_VERSION; }

typedef unsigned __int128 u128;

static u64 inv_mod_2_64(u64 m) {           // m odd
  u64 x = m;                               // correct to 3 bits
  for (int i = 0; i < 6; ++i) x *= 2 - m * x;
  return x;
}

static u64 mod_pow(u64 b, u64 e, u64 m) {
  if (m == 1) return 0;
  u64 r = 1 % m;
  b %= m;
  while (e) {
    if (e & 1) r = (u64)((u128)r * b % m);
    b = (u64)((u128)b * b % m);
    e >>= 1;
  }
  return r;
}

struct HostMod {
  u64 M, m, minv, mask2, Rm, r2;
  int a;
};

// M = 2^a * m with m odd below 2^63: the lazy 32-bit-radix Montgomery step keeps its values
// below 2m < 2^64.  When M < 2^64, key = X << a | x mod 2^a is a bijection of [0, M) (X < m);
// for larger M (a <= 32) the packed key is taken mod 2^64: equal residues still give equal
// keys, and callers confirm equal keys exactly.
static int host_mod_split(u64 m, int a, HostMod* h) {
  if (!(m & 1) || m >= (1ull << 63) || a < 0 || a > 32 || (m == 1 && a == 0)) return CF_EBADARG;
  h->a = a;
  h->m = m;
  h->M = (a == 0 || (m >> (64 - a)) == 0) ? (m << a) : 0;   // 0: M itself is 2^64 or more
  h->minv = inv_mod_2_64(h->m);
  h->mask2 = (h->a == 0) ? 0 : ((1ull << h->a) - 1);
  h->Rm = (u64)((((u128)1) << 64) % h->m);
  h->r2 = (u64)((u128)h->Rm * h->Rm % h->m);
  return CF_OK;
}

// Any M >= 2 whose odd part is below 2^63 (every even M below 2^64).
static int host_mod_init(u64 M, HostMod* h) {
  if (M < 2) return CF_EBADARG;
  const int a = __builtin_ctzll(M);
  if (a > 32) {                                 // 2-adic part beyond 32 bits: the generic keys
    if ((M >> a) >= (1ull << 63)) return CF_EBADARG;
    h->a = a; h->m = M >> a; h->M = M;
    h->minv = inv_mod_2_64(h->m);
    h->mask2 = (1ull << a) - 1;
    h->Rm = (u64)((((u128)1) << 64) % h->m);
    h->r2 = (u64)((u128)h->Rm * h->Rm % h->m);
    return CF_OK;
  }
  return host_mod_split(M >> a, a, h);
}

static u64 host_key(const HostMod& h, u64 v) {
  const u64 X = (u64)((u128)(v % h.m) * h.Rm % h.m);
  return (X << h.a) | (v & h.mask2);
}

// Key of the residue with odd part v_odd (mod m) and 2-adic part v2 (mod 2^a).
static u64 host_key2(const HostMod& h, u64 v_odd, u64 v2) {
  const u64 X = (u64)((u128)(v_odd % h.m) * h.Rm % h.m);
  return (X << h.a) | (v2 & h.mask2);
}

extern "C" size_t cf_pool_bytes(int n, int r) {
  if (n < 1 || n > CF_MAX_POOL || r < 1 || r > CF_MAX_R) return 0;
  return cf_pool_words(n, r) * sizeof(u64);
}

static int pool_args_ok(const u64* primes, int n, int r, void* out, size_t out_bytes) {
  if (!primes || !out) { cf_set_error("cf_pool_prepare: null pointer%s", ""); return CF_EBADARG; }
  if (n < 1 || n > CF_MAX_POOL) { cf_set_error("cf_pool_prepare: pool size out of range (1..1024)%s", ""); return CF_EBADARG; }
  if (r < 1 || r > CF_MAX_R || r > n) { cf_set_error("cf_pool_prepare: radius out of range (1..16, <= n)%s", ""); return CF_EBADARG; }
  if (out_bytes < cf_pool_bytes(n, r)) { cf_set_error("cf_pool_prepare: table buffer too small%s", ""); return CF_EBADARG; }
  return CF_OK;
}

static int pool_fill(const u64* primes, int n, int r, const HostMod& h, u64 mult_odd, u64 mult2, void* out);

extern "C" int cf_pool_prepare(const u64* primes, int n, int r, u64 M, u64 mult, void* out,
                               size_t out_bytes) {
  const int rc = pool_args_ok(primes, n, r, out, out_bytes);
  if (rc != CF_OK) return rc;
  HostMod h;
  if (host_mod_init(M, &h) != CF_OK) {
    cf_set_error("cf_pool_prepare: need 2 <= M < 2^64 with an odd part below 2^63%s", "");
    return CF_EBADARG;
  }
  return pool_fill(primes, n, r, h, (mult % M) % h.m, (mult % M) & h.mask2, out);
}

// The same table for M = 2^a * m given by its parts (M may be 2^64 or more): m odd below 2^63,
// a <= 32, the multiplier as its residues mod m and mod 2^a.
extern "C" int cf_pool_prepare_split(const u64* primes, int n, int r, u64 m, int a, u64 mult_odd, u64 mult2,
                                     void* out, size_t out_bytes) {
  const int rc = pool_args_ok(primes, n, r, out, out_bytes);
  if (rc != CF_OK) return rc;
  HostMod h;
  if (host_mod_split(m, a, &h) != CF_OK) {
    cf_set_error("cf_pool_prepare_split: need an odd m below 2^63 and 0 <= a <= 32%s", "");
    return CF_EBADARG;
  }
  return pool_fill(primes, n, r, h, mult_odd % m, mult2, out);
}

static int pool_fill(const u64* primes, int n, int r, const HostMod& h, u64 mult_odd, u64 mult2, void* out) {
  u64* w = (u64*)out;
  memset(w, 0, cf_pool_bytes(n, r));
  CfPoolHdr* hd = (CfPoolHdr*)w;
  hd->magic = CF_POOL_MAGIC;
  hd->M = h.M; hd->m = h.m; hd->minv = h.minv; hd->mask2 = h.mask2;
  hd->a = (u64)h.a; hd->n = (u64)n; hd->R = (u64)r;
  hd->mult_key = host_key2(h, mult_odd, mult2);
  hd->one_key = host_key2(h, 1, 1);
  hd->r2 = h.r2;
  const u64 half = (h.m + 1) / 2;          // 2^-1 mod m (m odd)
  hd->inv2a = mod_pow(half, (u64)h.a, h.m);
  hd->inv2aR = (u64)((u128)hd->inv2a * h.Rm % h.m);
  u64 maxp = 0;
  for (int i = 0; i < n; ++i) maxp = primes[i] > maxp ? primes[i] : maxp;
  hd->fast32 = (maxp < (1ull << 31)) ? 1 : 0;
  hd->ninv32 = (u64)(u32)(0u - (u32)h.minv);                 // -m^-1 mod 2^32
  hd->X0 = (u64)((u128)mult_odd * mod_pow(2, 32ull * (u64)r, h.m) % h.m);
  hd->x20 = mult2 & h.mask2;
  // tail table: b = min(R, 2) primes per entry when the fast path applies and 2^a fits 32 bits
  const int b = (hd->fast32 && h.a <= 32) ? (r < 2 ? r : 2) : 0;
  hd->tail_b = (u64)b;
  if (b) {
    hd->X0s = (u64)((u128)mult_odd * mod_pow(2, 32ull * (u64)(r - b), h.m) % h.m);
    hd->S0 = mod_pow(2, 64ull + 32ull * (u64)b, h.m);
  }
  u64* pkey = w + cf_pool_off_pkey(n);
  u64* prime = w + cf_pool_off_prime(n);
  double* lg = (double*)(w + cf_pool_off_lg(n));
  u64* binom = w + cf_pool_off_binom(n);
  for (int i = 0; i < n; ++i) {
    pkey[i] = host_key(h, primes[i]);
    prime[i] = primes[i];
    lg[i] = primes[i] ? log2((double)primes[i]) : -INFINITY;
  }
  const u64 SAT = ~0ull;
  for (int x = 0; x <= n; ++x) {
    for (int y = 0; y <= r; ++y) {
      u64 v;
      if (y == 0) v = 1;
      else if (x == 0) v = 0;
      else {
        const u64 p = binom[(size_t)(x - 1) * (r + 1) + (y - 1)];
        const u64 q = binom[(size_t)(x - 1) * (r + 1) + y];
        v = (p > SAT - q) ? SAT : p + q;
      }
      binom[(size_t)x * (r + 1) + y] = v;
    }
  }
  hd->total = binom[(size_t)n * (r + 1) + r];
  hd->tail_n = b ? binom[(size_t)n * (r + 1) + b] : 0;
  return CF_OK;
}

extern "C" u64 cf_key_of(u64 M, u64 v) {
  HostMod h;
  if (host_mod_init(M, &h) != CF_OK) return ~0ull;
  return host_key(h, v);
}

extern "C" u64 cf_canon_of(u64 M, u64 k) {
  HostMod h;
  if (host_mod_init(M, &h) != CF_OK) return ~0ull;
  CfMod md;
  md.m = h.m; md.minv = h.minv; md.mask2 = h.mask2; md.a = h.a;
  const u64 inv2a = mod_pow((h.m + 1) / 2, (u64)h.a, h.m);
  const u64 inv2aR = (u64)((u128)inv2a * h.Rm % h.m);
  return cf_key_to_canon(k, md, inv2a, inv2aR);
}

extern "C" u64 cf_key_mul(u64 M, u64 kx, u64 ky) {
  HostMod h;
  if (host_mod_init(M, &h) != CF_OK) return ~0ull;
  CfMod md;
  md.m = h.m; md.minv = h.minv; md.mask2 = h.mask2; md.a = h.a;
  return cf_mul_key(kx, ky, md);
}

// Product of the residues x and y mod M through the fast path (two cf_mul32 steps
// from the scaled start), returned as a key: host mirror for tests.
extern "C" u64 cf_key32_mul(u64 M, u64 x, u64 y) {
  HostMod h;
  if (host_mod_init(M, &h) != CF_OK || x >= (1ull << 31) || y >= (1ull << 31)) return ~0ull;
  CfMod32 md;
  md.m = h.m; md.mask2 = h.mask2; md.ninv = (u32)(0u - (u32)h.minv); md.ml = (u32)h.m; md.mh = (u32)(h.m >> 32);
  md.a = h.a;
  CfElt32 e;
  e.X = mod_pow(2, 64, h.m);
  e.x2 = 1 & h.mask2;
  e = cf_mul32(e, (u32)x, md);
  e = cf_mul32(e, (u32)y, md);
  return cf_key32(e, md);
}

extern "C" size_t cf_screen_bytes(void) { return sizeof(CfScreen); }

extern "C" int cf_screen_prepare(const u32* limbsB, int nlimbs, double lgP0, double lgB, double eps,
                                 void* out, size_t out_bytes) {
  if (!limbsB || !out || out_bytes < sizeof(CfScreen)) { cf_set_error("cf_screen_prepare: bad buffer%s", ""); return CF_EBADARG; }
  if (nlimbs < 1 || nlimbs > CF_SCREEN_MAX_LIMBS) { cf_set_error("cf_screen_prepare: B needs 1..64 limbs of 32 bits%s", ""); return CF_EBADARG; }
  if (!(eps >= 0.0)) { cf_set_error("cf_screen_prepare: eps must be >= 0%s", ""); return CF_EBADARG; }
  CfScreen* s = (CfScreen*)out;
  memset(s, 0, sizeof *s);
  s->lgP0 = lgP0; s->lgB = lgB; s->eps = eps; s->nlimbs = (u32)nlimbs;
  for (int i = 0; i < nlimbs; ++i) s->limbsB[i] = limbsB[i];
  return CF_OK;
}

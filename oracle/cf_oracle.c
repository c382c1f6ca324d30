/* cf_oracle.c -- CPU restatement of the reference's exchange-MITM hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (carmichael_frontier_b200/)
 * links, imports or executes this file; only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg use it, as the checker.
 *
 * Plain C (gcc, unsigned __int128), single-threaded, written for clarity, not
 * speed.  Each function restates one reference routine (paths inside
 * AlexanderEastwood/carmichael-frontier):
 *   ora_gen_records  gpu/mitm_gpu2.py:24-66  (CNS unrank + 128-bit mulmod)
 *   ora_join_all     gpu/mitm_gpu2.py:101-119 (stable sort + all equal-key pairs)
 *   ora_idump        src/mitm64_idump_stream2.cpp:44-57 (product-bounded I side)
 *   ora_ddump        src/mitm64_ddump.cpp:29-44 (Dmin-filtered D side)
 *   ora_mitm64       src/mitm64.cpp:50-121 (max-prodD-per-residue hash join)
 * Pinned against the reference's own binaries and kernel source by
 * tests/golden/make_golden.py (fixtures in tests/golden/).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef uint64_t u64;
typedef unsigned __int128 u128;

static u64 binom_sat(int a, int b) {
  if (b < 0 || b > a) return 0;
  if (b > a - b) b = a - b;
  u128 v = 1;
  for (int i = 1; i <= b; ++i) {
    v = v * (u128)(a - b + i) / (u128)i;
    if (v > (u128)~0ull) return ~0ull;
  }
  return (u64)v;
}

/* gen_records: record t = subset of lexicographic rank lo+t (indices ascending);
 * key = mult * prod(p) mod M by repeated 128-bit products; id packs `bits` per position. */
void ora_gen_records(const u64* primes, int n, int R, int bits, u64 M, u64 mult, u64 lo, u64 count,
                     u64* keys, u64* ids) {
  for (u64 t = 0; t < count; ++t) {
    u64 rank = lo + t;
    int idx[16];
    int start = 0;
    for (int pos = 0; pos < R; ++pos) {
      int remaining = R - pos - 1;
      for (int c = start; c <= n - 1; ++c) {
        u64 cnt = binom_sat(n - 1 - c, remaining);
        if (rank < cnt) { idx[pos] = c; start = c + 1; break; }
        rank -= cnt;
      }
    }
    u64 acc = mult % M, id = 0;
    for (int pos = 0; pos < R; ++pos) {
      u64 p = primes[idx[pos]];
      acc = (u64)(((u128)acc * (p % M)) % M);
      id |= ((u64)idx[pos]) << (pos * bits);
    }
    keys[t] = acc;
    ids[t] = id;
  }
}

typedef struct { u64 key, rank; } KR;

static int kr_cmp(const void* a, const void* b) {
  const KR* x = (const KR*)a; const KR* y = (const KR*)b;
  if (x->key != y->key) return x->key < y->key ? -1 : 1;
  return x->rank < y->rank ? -1 : (x->rank > y->rank);
}

/* Walk all r-subsets of pool[0..n-1] in lexicographic order, calling back with
 * (key = mult * prod mod M, rank). */
typedef void (*walk_cb)(u64 key, u64 rank, const int* idx, void* ctx);
static void walk_lex(const u64* pool, int n, int R, u64 M, u64 mult, walk_cb cb, void* ctx) {
  if (R < 1 || R > n) return;
  int idx[16];
  u64 pre[17];
  for (int j = 0; j < R; ++j) idx[j] = j;
  pre[0] = mult % M;
  for (int j = 0; j < R; ++j) pre[j + 1] = (u64)(((u128)pre[j] * (pool[idx[j]] % M)) % M);
  u64 rank = 0;
  for (;;) {
    cb(pre[R], rank++, idx, ctx);
    int j = R - 1;
    while (j >= 0 && idx[j] == n - R + j) --j;
    if (j < 0) break;
    idx[j]++;
    for (int t = j + 1; t < R; ++t) idx[t] = idx[t - 1] + 1;
    for (int t = j; t < R; ++t) pre[t + 1] = (u64)(((u128)pre[t] * (pool[idx[t]] % M)) % M);
  }
}

typedef struct { KR* a; u64 n; } CollectCtx;
static void collect_cb(u64 key, u64 rank, const int* idx, void* ctx) {
  (void)idx;
  CollectCtx* c = (CollectCtx*)ctx;
  c->a[c->n].key = key; c->a[c->n].rank = rank; c->n++;
}

typedef struct {
  const KR* D; u64 nD; u64* d_out; u64* i_out; int64_t cap; int64_t found;
} ProbeCtx;
static void probe_cb(u64 key, u64 rank, const int* idx, void* ctx) {
  (void)idx;
  ProbeCtx* c = (ProbeCtx*)ctx;
  u64 lo = 0, hi = c->nD;
  while (lo < hi) { u64 mid = (lo + hi) / 2; if (c->D[mid].key < key) lo = mid + 1; else hi = mid; }
  for (u64 j = lo; j < c->nD && c->D[j].key == key; ++j) {
    if (c->found < c->cap) { c->d_out[c->found] = c->D[j].rank; c->i_out[c->found] = rank; }
    c->found++;
  }
}

/* Every (D, I) pair with multD*prod(D) == multI*prod(I) (mod M), D an R-subset of
 * Dpool, I an R-subset of Ipool, as lexicographic ranks; ordered by I rank, then D
 * rank (join_sorted's order on stably sorted sides).  Returns the pair count
 * (pairs beyond cap are counted, not written); -1 on allocation failure. */
int64_t ora_join_all(const u64* Dpool, int nD, u64 multD, const u64* Ipool, int nI, u64 multI, int R, u64 M,
                     u64* d_rank, u64* i_rank, int64_t cap) {
  u64 total = binom_sat(nD, R);
  KR* a = (KR*)malloc(sizeof(KR) * (total ? total : 1));
  if (!a) return -1;
  CollectCtx cc = {a, 0};
  walk_lex(Dpool, nD, R, M, multD, collect_cb, &cc);
  qsort(a, cc.n, sizeof(KR), kr_cmp);
  ProbeCtx pc = {a, cc.n, d_rank, i_rank, cap, 0};
  walk_lex(Ipool, nI, R, M, multI, probe_cb, &pc);
  free(a);
  return pc.found;
}

/* ---- product-bounded I side (mitm64_idump_stream2) ----------------------- */
typedef struct {
  const u64* INS; int n, R, split_idx, hmax, rank_ids;
  u64 M, P0m; u128 Icap;
  u64* keys; u64* ids; u64 cap; u64 count;
} IdumpCtx;

static int mul_ge(u128 a, u128 b, u128 cap) {
  u128 r;
  if (__builtin_mul_overflow(a, b, &r)) return 1;
  return r >= cap;
}
static int window_ge(const IdumpCtx* c, u128 np, int a, int t) {
  u128 v = np;
  for (int j = 0; j < t; ++j) if (__builtin_mul_overflow(v, (u128)c->INS[a + j], &v)) return 1;
  return v >= c->Icap;
}
static void idump_rec(IdumpCtx* c, int start, int depth, u128 prod, u64 res, u64 id, int nlarge) {
  if (depth == c->R) {
    if (c->count < c->cap) {
      c->keys[c->count] = (u64)(((u128)c->P0m * res) % c->M);
      c->ids[c->count] = id;
    }
    c->count++;
    return;
  }
  const int t = c->R - depth - 1;
  for (int i = start; i <= c->n - 1 - t; ++i) {
    if (i >= c->split_idx && nlarge + 1 > c->hmax) break;
    if (mul_ge(prod, c->INS[i], c->Icap)) break;
    u128 np = prod * c->INS[i];
    if (t > 0 && window_ge(c, np, i + 1, t)) break;
    u64 nid = c->rank_ids ? id + binom_sat(i, depth + 1) : (id | ((u64)i << (8 * depth)));
    idump_rec(c, i + 1, depth + 1, np, (u64)(((u128)res * (c->INS[i] % c->M)) % c->M), nid,
              nlarge + (i >= c->split_idx));
  }
}

/* Records {key = P0*prod(I) mod M, id} of every R-subset I of the ascending INS
 * with prod(I) < Icap (Icap given as two u64 halves) and at most hmax primes at
 * indices >= split_idx, in the dumper's depth-first order (one thread).
 * Returns the record count (records beyond cap are counted only). */
u64 ora_idump(const u64* INS, int n, int R, u64 M, u64 P0m, u64 icap_lo, u64 icap_hi, int split_idx, int hmax,
              int rank_ids, u64* keys, u64* ids, u64 cap) {
  IdumpCtx c;
  memset(&c, 0, sizeof c);
  c.INS = INS; c.n = n; c.R = R; c.split_idx = split_idx; c.hmax = hmax; c.rank_ids = rank_ids;
  c.M = M; c.P0m = P0m; c.Icap = ((u128)icap_hi << 64) | icap_lo;
  c.keys = keys; c.ids = ids; c.cap = cap;
  const int tt = R - 1;
  for (int i0 = 0; i0 <= n - 1 - tt; ++i0) {
    if (i0 >= split_idx && 1 > hmax) break;
    u128 np = (u128)INS[i0];
    if (np >= c.Icap) continue;
    if (tt > 0 && window_ge(&c, np, i0 + 1, tt)) continue;
    /* depth-0 id is i0 in both encodings: packed i0 << 0, colex C(i0, 1) = i0 */
    idump_rec(&c, i0 + 1, 1, np, INS[i0] % M, (u64)i0, (i0 >= split_idx));
  }
  return c.count;
}

/* ---- Dmin-filtered D side (mitm64_ddump) ------------------------------- */
typedef struct {
  const u64* B; int R, bitmask; u64 M; u128 Dmin;
  u64* keys; u64* ids; u64 cap; u64 count; int idx[16];
} DdumpCtx;

static void ddump_rec(DdumpCtx* c, int hi, int depth, u128 prod, u64 res) {
  if (depth == c->R) {
    u64 id = 0;
    if (c->bitmask) { for (int j = 0; j < c->R; ++j) id |= 1ull << c->idx[j]; }
    else { for (int j = c->R - 1, pos = 0; j >= 0; --j, ++pos) id |= ((u64)c->idx[j]) << (6 * pos); }
    if (c->count < c->cap) { c->keys[c->count] = res % c->M; c->ids[c->count] = id; }
    c->count++;
    return;
  }
  const int t = c->R - depth - 1;
  for (int i = hi; i >= t; --i) {
    u128 np = prod * c->B[i];
    u128 best = np;
    for (int j = 0; j < t; ++j) best *= c->B[i - 1 - j];
    if (best < c->Dmin) break;
    c->idx[depth] = i;
    ddump_rec(c, i - 1, depth + 1, np, (u64)(((u128)res * (c->B[i] % c->M)) % c->M));
  }
}

/* Records {key = prod(D) mod M, id} of every R-subset D of the ascending base B
 * (nB primes) with prod(D) >= Dmin, descending-index depth-first order; ids are
 * 6-bit packed ascending indices, or a 64-bit index mask when bitmask != 0. */
u64 ora_ddump(const u64* B, int nB, int R, u64 M, u64 dmin_lo, u64 dmin_hi, int bitmask, u64* keys, u64* ids,
              u64 cap) {
  DdumpCtx c;
  memset(&c, 0, sizeof c);
  c.B = B; c.R = R; c.bitmask = bitmask || R > 10; c.M = M; c.Dmin = ((u128)dmin_hi << 64) | dmin_lo;
  c.keys = keys; c.ids = ids; c.cap = cap;
  ddump_rec(&c, nB - 1, 0, (u128)1, 1 % M);
  return c.count;
}

/* ---- mitm64.cpp semantics: max prod(D) per residue, inclusive Icap break ---- */
typedef struct { u64 res; u128 prod; int idx[16]; int used; } DSlot;

/* Matches of src/mitm64.cpp: the D side keeps, per residue of prod(D) mod M, the
 * deletion with the largest product (reach-pruned by prodDmin, Bd descending);
 * every I-subset of the ascending INS with prod(I) <= Icap (break on >) probes
 * with key P0m*prod(I) mod M.  Writes (D indices into Bd, I indices into INS) of
 * each match; returns the match count, and d_leaves / i_leaves / d_res. */
int64_t ora_mitm64(const u64* B0asc, int nB, const u64* INS, int nI, int R, u64 M, u64 P0m, u64 icap_lo,
                   u64 icap_hi, u64 dmin_lo, u64 dmin_hi, int* d_out, int* i_out, int64_t cap, u64* stats) {
  u128 Icap = ((u128)icap_hi << 64) | icap_lo, Dmin = ((u128)dmin_hi << 64) | dmin_lo;
  u64* Bd = (u64*)malloc(sizeof(u64) * nB);
  for (int i = 0; i < nB; ++i) Bd[i] = B0asc[nB - 1 - i];
  u64 nslots = 1;
  u64 total = binom_sat(nB, R);
  while (nslots < 2 * total + 16) nslots <<= 1;
  DSlot* tab = (DSlot*)calloc(nslots, sizeof(DSlot));
  if (!tab || !Bd) { free(tab); free(Bd); return -1; }
  u64 d_leaves = 0, d_res = 0;
  /* iterative descent over Bd indices (start, depth, prod) with the reach prune */
  int idx[16];
  u128 prod[17];
  int depth = 0;
  idx[0] = 0;
  prod[0] = 1;
  while (depth >= 0) {
    int need = R - depth;
    int i = idx[depth];
    if (i > nB - need) { --depth; if (depth >= 0) idx[depth]++; continue; }
    u128 reach = prod[depth];
    for (int j = i; j < i + need; ++j) reach *= Bd[j];
    if (reach < Dmin) { --depth; if (depth >= 0) idx[depth]++; continue; }
    prod[depth + 1] = prod[depth] * Bd[i];
    if (depth + 1 == R) {
      d_leaves++;
      u64 res = (u64)(prod[R] % M);
      u64 h = (res * 0x9E3779B97F4A7C15ull) & (nslots - 1);
      while (tab[h].used && tab[h].res != res) h = (h + 1) & (nslots - 1);
      if (!tab[h].used) { tab[h].used = 1; tab[h].res = res; tab[h].prod = 0; d_res++; }
      if (prod[R] > tab[h].prod) { tab[h].prod = prod[R]; memcpy(tab[h].idx, idx, sizeof(int) * R); }
      idx[depth]++;
      continue;
    }
    idx[depth + 1] = i + 1;
    ++depth;
  }
  /* I side */
  int64_t found = 0;
  u64 i_leaves = 0;
  int ii[16];
  u128 ip[17];
  u64 ir[17];
  depth = 0;
  ii[0] = 0;
  ip[0] = 1;
  ir[0] = 1 % M;
  while (depth >= 0) {
    int need = R - depth;
    int i = ii[depth];
    if (i > nI - need) { --depth; if (depth >= 0) ii[depth]++; continue; }
    u128 np = ip[depth] * INS[i];
    if (np > Icap) { --depth; if (depth >= 0) ii[depth]++; continue; }
    ip[depth + 1] = np;
    ir[depth + 1] = (u64)(((u128)ir[depth] * (INS[i] % M)) % M);
    if (depth + 1 == R) {
      i_leaves++;
      u64 key = (u64)(((u128)P0m * ir[R]) % M);
      u64 h = (key * 0x9E3779B97F4A7C15ull) & (nslots - 1);
      while (tab[h].used && tab[h].res != key) h = (h + 1) & (nslots - 1);
      if (tab[h].used) {
        if (found < cap) {
          for (int j = 0; j < R; ++j) { d_out[found * R + j] = tab[h].idx[j]; i_out[found * R + j] = ii[j]; }
        }
        found++;
      }
      ii[depth]++;
      continue;
    }
    ii[depth + 1] = i + 1;
    ++depth;
  }
  if (stats) { stats[0] = d_leaves; stats[1] = d_res; stats[2] = i_leaves; }
  free(tab);
  free(Bd);
  return found;
}

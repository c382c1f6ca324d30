/* cfmitm.h -- C ABI of the B200 exchange meet-in-the-middle residue join.
 *
 * Every function is extern "C", takes plain pointers and sizes, and returns an
 * int status (0 = ok, negative = error; cf_last_error_string() says why).
 * Device buffers are owned by the caller; functions that need scratch take a
 * (tmp, tmp_bytes) workspace whose size a *_tmp_bytes / *_bytes query gives.
 * Work is queued on the caller's CUDA stream (`stream`, a cudaStream_t, may be
 * NULL for the legacy default stream); only the calls documented as
 * synchronising wait for the device.  The library never throws.
 *
 * Residues are held in "key form" (see carmichael_frontier_b200/csrc/cf_common.cuh):
 * a bijection of [0, M) onto itself for M < 2^64, so equal keys <=> equal residues mod M.
 * Tables made by cf_pool_prepare_split for M >= 2^64 hold keys taken mod 2^64: equal
 * residues => equal keys only.  cf_gen_subsets(..., canon=1) emits canonical residues
 * instead (M < 2^64 only).
 *
 * Reference interfaces replaced (paths inside AlexanderEastwood/carmichael-frontier):
 *   gen_records / generate()   gpu/mitm_gpu2.py:24-98
 *   sort_side()                gpu/mitm_gpu2.py:101-104
 *   join_sorted()              gpu/mitm_gpu2.py:107-119
 *   exact pair re-check        gpu/mitm_gpu_mstar_driver.py:226-237, ref/ref_carmichael.py:55-72
 *   CPU join engine            src/mitm64.cpp:50-121 (recD / worker)
 */
#ifndef CFMITM_H
#define CFMITM_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define CF_OK 0
#define CF_EBADARG -1
#define CF_ENOMEM -2
#define CF_ECUDA -3
#define CF_EOVERFLOW -4
#define CF_ETIMEOUT -5

/* error-word bits written by kernels into the caller's u32 `err` word */
#define CF_ERR_PART_OVERFLOW 1u
#define CF_ERR_PAIR_OVERFLOW 2u
#define CF_ERR_TABLE_FULL 4u
#define CF_ERR_SPIN_LIMIT 8u
#define CF_ERR_KEY_MISMATCH 16u

/* pair-check result flags (CfPairResult.flags) */
#define CF_HIT_KEY_EQUAL 1u
#define CF_HIT_SCREEN 2u
#define CF_HIT_SIZE_EXACT 4u
#define CF_HIT_KORSELT 8u
#define CF_HIT_DISJOINT 16u

/* ABI version of this header (1). */
int cf_version(void);

/* Human-readable reason for the last non-zero status on this host thread.
 * Replaces the reference's Python assertion messages (gpu/mitm_gpu2.py:83-85,
 * gpu/igen_gpu.py:103-105). */
const char* cf_last_error_string(void);

/* ---- host-side table preparation (no device calls) ---------------------- */

/* Bytes of the pool table for n primes and radius r (0 if out of range). */
size_t cf_pool_bytes(int n, int r);

/* Fill a pool table (host buffer) for the r-subsets of primes[0..n-1] modulo M
 * (2 <= M < 2^64, odd part below 2^63) with leading multiplier `mult` (the D side of a solve uses
 * (prod B0)^-1 mod M, the I side 1; gen_records' `mult` argument otherwise).
 * Holds each prime in key form, log2 of each prime and the binomial table.
 * Replaces the host half of generate(): gpu/mitm_gpu2.py:70-93. */
int cf_pool_prepare(const uint64_t* primes, int n, int r, uint64_t M, uint64_t mult, void* out,
                    size_t out_bytes);

/* The same table for M = 2^a * m given by its parts, so M may be 2^64 or more: m odd below 2^63,
 * 0 <= a <= 32, the multiplier as mult_odd = mult mod m and mult2 = mult mod 2^a.  Keys of such
 * moduli are the packed residue taken mod 2^64: equal residues give equal keys, and a caller
 * confirms each key match exactly (the Python layer recomputes the residues with Python
 * integers before it reports a pair).  No counterpart in
 * the reference, whose keys are u64 residues below M < 2^64 (gpu/run_mstar_family.py:70-73). */
int cf_pool_prepare_split(const uint64_t* primes, int n, int r, uint64_t m, int a, uint64_t mult_odd,
                          uint64_t mult2, void* out, size_t out_bytes);

/* key(v mod M), its inverse, and the product of two keys computed by the
 * kernels' own Montgomery/CRT code compiled for the host (host helpers). */
uint64_t cf_key_of(uint64_t M, uint64_t v);
uint64_t cf_canon_of(uint64_t M, uint64_t key);
uint64_t cf_key_mul(uint64_t M, uint64_t kx, uint64_t ky);

/* Key of x*y mod M computed by the solve path's fast arithmetic (pool primes
 * below 2^31: lazy 32-bit-radix Montgomery steps), for host-side tests.  The
 * solve path's key is (x mod m) << a | (x mod 2^a) for M = 2^a * m, m odd. */
uint64_t cf_key32_mul(uint64_t M, uint64_t x, uint64_t y);

/* Size-screen table for cf_check_pairs: B as little-endian 32-bit limbs
 * (1..64 limbs), log2(prod B0), log2(B) and the fp64 margin eps. */
size_t cf_screen_bytes(void);
int cf_screen_prepare(const uint32_t* limbsB, int nlimbs, double lgP0, double lgB, double eps, void* out,
                      size_t out_bytes);

/* ---- generation ---------------------------------------------------------- */

/* gen_records drop-in (gpu/mitm_gpu2.py:24-98): record t is the r-subset at
 * lexicographic rank lo+t of the pool in `pool_dev` (a cf_pool_prepare table
 * copied to the device).  keys[t] = mult * prod(p) mod M (canonical residue if
 * canon != 0, else key form).  ids[t]: id_mode 0 = indices packed `bits` per
 * position (gen_records' id), 1 = lexicographic rank, 2 = colexicographic rank
 * sum C(i_j, j+1) (the rank id of src/mitm64_idump_stream2.cpp:26-29).
 * Requires 1 <= r <= 10 and lo + count <= C(n, r). */
int cf_gen_subsets(const void* pool_dev, int n, int r, uint64_t lo, uint64_t count, int id_mode, int bits,
                   int canon, uint64_t* keys, uint64_t* ids, void* stream);

/* Tail table of a pool (device, cf_tail_bytes(n, r) bytes): the products of all
 * b-subsets of the pool, b = min(r, 2), in lexicographic order, 16 bytes each.
 * Built once per pool by cf_build_tail; the generators split every r-subset into
 * an (r-b)-prefix and a b-suffix read from this table.  Requires pool primes
 * below 2^31 and 2^32 not dividing M. */
size_t cf_tail_bytes(int n, int r);
int cf_build_tail(const void* pool_dev, int n, int r, void* tail, void* stream);

/* Partitioned generation for the solve path (pool primes below 2^31): the
 * records of ranks [lo, lo+count) (id = lexicographic rank) are scattered into
 * 2^pbits (pbits 0..12) residue partitions -- the top pbits bits of
 * key * 0x9E3779B97F4A7C15 mod 2^64 -- of capacity cap records each: partition
 * p occupies out[p*cap .. p*cap+cap) as 16-byte {key, id} records (the
 * reference's record layout, src/mitm64_idump_stream.cpp:6-12).  counts[p]
 * (device, zeroed by the caller) receives the number of records routed to p,
 * even beyond cap; then CF_ERR_PART_OVERFLOW is set in *err and the caller
 * retries with a larger cap.  shape selects the launch shape (0..
 * cf_gen_part_shapes()-1: threads x records per thread).  Replaces generate()
 * + sort_side() as the producer of a joinable side. */
int cf_gen_part_shapes(void);
size_t cf_gen_part_smem_bytes(int n, int r, int pbits, int shape);
int cf_gen_part(const void* pool_dev, const void* tail, int n, int r, uint64_t lo, uint64_t count, int pbits,
                uint32_t cap, uint32_t* counts, void* out, uint32_t* err, int shape, void* stream);

/* ---- join ---------------------------------------------------------------- */

/* Partitioned equal-residue join over the 2^pbits partitions of cf_gen_part:
 * every (D, I) record pair with equal keys is appended to pairs[] as
 * {D id, I id} (16 bytes) through the device counter *npairs (zeroed by the
 * caller); beyond max_pairs the count keeps growing and CF_ERR_PAIR_OVERFLOW is
 * set.  sbits (4..15): shared-memory table of 2^sbits slots (4 bytes each) per
 * CTA; isplit: CTAs per partition; grid: 0 = one CTA per (partition, split).
 * Replaces join_sorted (gpu/mitm_gpu2.py:107-119) and mitm64.cpp's hash probe
 * (src/mitm64.cpp:85-101). */
size_t cf_join_part_smem_bytes(int sbits);
int cf_join_part(const void* D, const uint32_t* dcount, uint32_t capD, const void* I, const uint32_t* icount,
                 uint32_t capI, int pbits, int sbits, uint32_t isplit, uint32_t grid, void* pairs,
                 uint32_t max_pairs, uint32_t* npairs, uint32_t* err, void* stream);

/* Fused generate-and-probe join (the I side is never written to memory).
 * D table: 2^bbits buckets of 16 slots, cf_dtab_bytes(bbits) bytes: first an
 * array of 32-byte fingerprint sectors (16 16-bit fingerprints per bucket, the
 * one sector a probe reads; cf_dtab_fp_bytes(bbits) bytes, L2-resident for
 * r <= 5), then a side area of 128 bytes per bucket (per slot more
 * fingerprint bits and the D rank), then a 4-byte fill counter per bucket.
 * Before building, the caller zeroes the fingerprint array and the fill
 * counters (the last 4 * 2^bbits bytes).
 * cf_dtab_build inserts the D records of ranks [lo, lo+count), count < 2^32;
 * cf_fused_probe generates the I records of ranks [lo, lo+count) in
 * registers, probes the table and appends every {D rank, I rank} candidate
 * whose fingerprints agree through *npairs (zeroed by the caller);
 * cf_check_pairs then flags the pairs whose residues are equal
 * (CF_HIT_KEY_EQUAL), which is the exact pair set.  Replaces join_sorted
 * (gpu/mitm_gpu2.py:107-119) and the probe of src/mitm64.cpp:85-101 without
 * materialising the I side. */
size_t cf_dtab_bytes(int bbits);
size_t cf_dtab_fp_bytes(int bbits);
/* Variants with an optional first level for tables larger than L2: a blocked
 * Bloom filter of 2^fbits 32-byte blocks (3 bits per record; fbits 0 = none)
 * placed after the table (cf_dtab_bytes2(bbits, fbits) bytes in all; the caller
 * zeroes the filter with the fingerprint array and fill counters), and the
 * choice of the side the table holds: the table can be built from either
 * side's pool (cf_dtab_build2 does not care); swap = 1 tells the probe that the
 * table holds I records and the D side is probing, so that pairs are still
 * stored as {D rank, I rank}.  A hash join builds on its smaller side. */
size_t cf_dtab_bytes2(int bbits, int fbits);
int cf_dtab_build2(const void* pool_dev, const void* tail, int n, int r, uint64_t lo, uint64_t count, void* tab,
                   int bbits, int fbits, uint32_t* err, void* stream);
int cf_fused_probe2(const void* pool_dev, const void* tail, int n, int r, uint64_t lo, uint64_t count,
                    const void* tab, int bbits, int fbits, uint64_t tab_rank0, int swap, void* pairs,
                    uint32_t max_pairs, uint32_t* npairs, uint32_t* err, uint32_t grid, void* stream);
int cf_dtab_build(const void* pool_dev, const void* tail, int n, int r, uint64_t lo, uint64_t count, void* tab,
                  int bbits, uint32_t* err, void* stream);
/* The same with the side area's format chosen: side_format 0 = wide (per slot a
 * 32-bit fingerprint and the rank, 8 bytes; what the variants above build and
 * probe), 1 = compact (per slot one 32-bit word, rank << 8 | 8 more
 * fingerprint bits; tables of at most 2^20 buckets and 2^24 records).  The
 * compact side of an L2-sized table stays in L2 while it is built, so its
 * sectors are written back whole once.  Build and probe must be given the same
 * format. */
int cf_dtab_build3(const void* pool_dev, const void* tail, int n, int r, uint64_t lo, uint64_t count, void* tab,
                   int bbits, int fbits, int side_format, uint32_t* err, void* stream);
int cf_fused_probe3(const void* pool_dev, const void* tail, int n, int r, uint64_t lo, uint64_t count,
                    const void* tab, int bbits, int fbits, int side_format, uint64_t tab_rank0, int swap,
                    void* pairs, uint32_t max_pairs, uint32_t* npairs, uint32_t* err, uint32_t grid,
                    void* stream);
int cf_fused_probe(const void* pool_dev, const void* tail, int n, int r, uint64_t lo, uint64_t count,
                   const void* tab, int bbits, uint64_t d_rank0, void* pairs, uint32_t max_pairs,
                   uint32_t* npairs, uint32_t* err, uint32_t grid, void* stream);

/* Exact check of candidate pairs (lexicographic-rank ids): recomputed residues,
 * conservative fp64 log-size screen, exact size n <= B, Korselt, distinctness.
 * results[t] (cf_pair_result_bytes() each) for t < min(*npairs, max_pairs).
 * Replaces the driver's exact re-check (gpu/mitm_gpu_mstar_driver.py:226-237). */
size_t cf_pair_result_bytes(void);
int cf_check_pairs(const void* poolD, const void* poolI, const void* screen, int r, const void* pairs,
                   const uint32_t* npairs, uint32_t max_pairs, void* results, uint32_t* err, void* stream);

/* ---- product-bounded producers (filtered I side, Dmin-filtered D side) ---- */

/* Level-by-level expansion of the bounded enumeration tree.  A frontier node is
 * {key (key form), exact product (alo, ahi), partial id, meta = last index |
 * count of large primes << 16}; the root is {key(mult), 1, 0, 0xffff}.
 * bounds: r x n u128 values as (lo, hi) u64 pairs, row t = positions left after
 * the chosen index:
 *   side 0 (I, ascending, id = colex rank): H[t][x] = floor((Icap-1) /
 *     (a_x ... a_{x+t})), child x kept iff product <= H[t][x]; indices >=
 *     split_idx count as large, at most hmax of them.  The records of
 *     src/mitm64_idump_stream2.cpp (IDUMP_RANK=1) and gpu/igen_gpu.py:26-76
 *     (its igen kernel, count and write passes), in the same lexicographic order.
 *   side 1 (D, descending; bitmask 0: 6-bit packed ids, 1: index mask, both
 *     for n <= 64; 2: colex rank, any n): G[t][x] = ceil(Dmin / (b_x b_{x-1}
 *     ... b_{x-t})), child x kept iff product >= G[t][x].  The records of
 *     src/mitm64_ddump.cpp:29-44, same order.
 * cf_bgen_count writes each node's child count and first child index;
 * cf_scan_u64 turns counts into offsets (offs[F] = total); cf_bgen_expand writes
 * children [c0, c0+cc): nodes for d < r-1, records {canonical key, id} for
 * d = r-1.  First indices can be restricted to [xa, xb) at depth 0.  With a
 * cf_pool_prepare_split pool of M >= 2^64, node keys hold x * 2^64 mod m (the root
 * key: mult * 2^64 mod m) and record keys the packed residue
 * (x * 2^64 mod m) << a | x mod 2^a taken mod 2^64; callers confirm matches exactly. */
size_t cf_scan_tmp_bytes(uint64_t n);
int cf_scan_u64(const uint64_t* in, uint64_t n, uint64_t* out, void* tmp, size_t tmp_bytes, void* stream);
int cf_bgen_count(int side, int d, int r, int n, uint64_t F, const uint64_t* alo, const uint64_t* ahi,
                  const uint32_t* meta, const uint64_t* bounds, int split_idx, int hmax, int xa, int xb,
                  uint64_t* cnt, uint32_t* xs, void* stream);
int cf_bgen_expand(int side, int d, int r, int n, uint64_t F, const void* pool, const uint64_t* key,
                   const uint64_t* alo, const uint64_t* ahi, const uint64_t* id, const uint32_t* meta,
                   const uint64_t* offs, const uint32_t* xs, int split_idx, int bitmask, uint64_t c0, uint64_t cc,
                   uint64_t* okey, uint64_t* oalo, uint64_t* oahi, uint64_t* oid, uint32_t* ometa, void* stream);

/* The bounded I side in two calls, as gpu/igen_gpu.py:113-162 counts and then
 * writes its records: cf_igen_bounds computes the bound table H on the host
 * (exact 128-bit, cf_igen_bounds_bytes(n, r) bytes; upload it); cf_igen_count
 * expands the levels in the caller's workspace (pool_dev = cf_pool_prepare(ins,
 * n, r, M, mult = P0 mod M) on the device) and returns the record count and a
 * 64-byte host state, or CF_ENOMEM with the node count a level needs (size the
 * retry with cf_igen_tmp_bytes); cf_igen_write writes records [c0, c0+cc) of
 * the counted frontier, in src/mitm64_idump_stream2.cpp's order (colex ids).
 * split_idx = n and hmax = r impose no stratum.  Moduli below 2^64. */
size_t cf_igen_bounds_bytes(int n, int r);
int cf_igen_bounds(const uint64_t* ins, int n, int r, uint64_t icap_lo, uint64_t icap_hi, void* out,
                   size_t out_bytes);
size_t cf_igen_tmp_bytes(uint64_t max_nodes);
int cf_igen_count(const void* pool_dev, const void* bounds_dev, uint64_t M, uint64_t mult, int n, int r,
                  int split_idx, int hmax, void* tmp, size_t tmp_bytes, uint64_t* total, uint64_t* need_nodes,
                  void* state, void* stream);
int cf_igen_write(const void* pool_dev, int n, int r, int split_idx, const void* tmp, const void* state,
                  uint64_t c0, uint64_t cc, uint64_t* keys, uint64_t* ids, void* stream);

/* One product-bounded exchange instance in one call (the device part of the
 * reference driver's run_instance, gpu/mitm_gpu_mstar_driver.py:184-286):
 * cf_ddump_bounds computes the D side's bound table G (exact 128-bit,
 * cf_ddump_bounds_bytes(n, r) bytes; upload it); cf_bounded_join then expands
 * the D side (prod >= Dmin, colex ids), builds a record table of it, expands the
 * I side (prod < Icap, at most hmax primes at indices >= split_idx) to its last
 * inner level, probes every leaf in registers and returns in out (host,
 * 3 * max_out u64: D colex ids | D keys | I colex ids) the candidates -- the
 * equal-key pairs and rare fingerprint collisions, which the caller drops by
 * recomputing the I key -- and sizes[2] = {nD, nI}.  poolD = cf_pool_prepare(B0,
 * nb, r, M, 1), poolI = cf_pool_prepare(INS, ni, r, M, P0 mod M), both on the
 * device; bbits = 0 picks the table shape.  CF_ENOMEM: retry with at least
 * *need bytes of workspace; CF_EOVERFLOW with *n_out > max_out: retry with a
 * larger out.  Moduli below 2^64, caps below 2^128.  Waits on `stream` once per
 * level. */
size_t cf_ddump_bounds_bytes(int n, int r);
int cf_ddump_bounds(const uint64_t* b, int n, int r, uint64_t dmin_lo, uint64_t dmin_hi, void* out, size_t out_bytes);
int cf_bounded_join(const void* poolD, const void* boundsD, int nb, const void* poolI, const void* boundsI, int ni,
                    int r, uint64_t M, uint64_t p0_mod_m, int split_idx, int hmax, int bbits, int fbits, void* tmp,
                    size_t tmp_bytes, uint64_t* out, uint64_t max_out, uint64_t* n_out, uint64_t* sizes,
                    uint64_t* need, void* stream);

/* Hash join of two materialised sides of {canonical key} records (the bounded
 * producers' output): cf_rec_build inserts the smaller side's keys into a table
 * of cf_dtab_bytes2(bbits, fbits) bytes (zeroed as for cf_dtab_build2);
 * cf_rec_probe probes it with the other side and appends every candidate
 * {D position, I position} (swap = 1 when the table holds the I side); the
 * caller drops the rare candidates whose keys differ.  Replaces sort_side +
 * join_sorted on the filtered sides (gpu/mitm_gpu_mstar_driver.py:241-262). */
int cf_rec_build(const uint64_t* keys, uint64_t n, void* tab, int bbits, int fbits, uint32_t* err, void* stream);
int cf_rec_probe(const uint64_t* keys, uint64_t n, const void* tab, int bbits, int fbits, int swap, void* pairs,
                 uint32_t max_pairs, uint32_t* npairs, uint32_t* err, void* stream);

/* The last level of the bounded I side fused with the probe of a cf_rec_build
 * table of D records: the leaves [c0, c0+cc) of a depth-(r-1) I frontier (the
 * node arrays, offsets and first child indices of cf_bgen_count / cf_scan_u64)
 * are computed in registers and probed, never written; candidates are
 * {D position, I colex id}.  Replaces the igen chunks x sorted D chunks join of
 * gpu/mitm_gpu_mstar_driver.py:241-262 when the I side is the large one.  It hashes
 * canonical residues: pools of M < 2^64 only (write the leaves with cf_bgen_expand and
 * probe them with cf_rec_probe otherwise). */
int cf_bgen_probe(int r, int n, uint64_t F, const void* pool, const uint64_t* key, const uint64_t* id,
                  const uint64_t* offs, const uint32_t* xs, uint64_t c0, uint64_t cc, const void* tab, int bbits,
                  int fbits, void* pairs, uint32_t max_pairs, uint32_t* npairs, uint32_t* err, void* stream);

/* The same pair for a table of D records under their key form (odd part in Montgomery form
 * over the 2-adic part, the form the bounded producers' nodes carry): cf_rec_build_keyform
 * inserts canonical D keys converted with the modulus of `pool` (the I pool table on the
 * device, M < 2^64), and cf_bgen_probe_keyform probes it with the leaves' key forms, with no
 * conversion per leaf.  Same candidates as cf_rec_build + cf_bgen_probe.  No counterpart in
 * the reference. */
int cf_rec_build_keyform(const uint64_t* keys, uint64_t n, void* tab, int bbits, int fbits, const void* pool,
                         uint32_t* err, void* stream);
int cf_bgen_probe_keyform(int r, int n, uint64_t F, const void* pool, const uint64_t* key, const uint64_t* id,
                          const uint64_t* offs, const uint32_t* xs, uint64_t c0, uint64_t cc, const void* tab,
                          int bbits, int fbits, void* pairs, uint32_t max_pairs, uint32_t* npairs, uint32_t* err,
                          void* stream);

/* ---- streamed (out-of-core) join --------------------------------------------- */

/* Range partitioning of canonical {key, id} records (key < M) for sides larger than
 * HBM: partition p = floor(key * 2^pbits / M) (1 <= pbits <= 12), so equal residues
 * meet in the same partition and partitions can be joined one at a time.  M = 0
 * stands for 2^64: any u64 keys (the packed residues mod 2^64 of a modulus of 2^64 or
 * more), p = key >> (64 - pbits).
 * cf_part_hist adds the partition sizes of keys[0..n) to counts[2^pbits];
 * cf_part_scatter writes each record to out[cursor[p]++] (cursor = the partitions'
 * start offsets from a cf_part_hist of the same keys; order inside a partition is
 * not kept).  Replaces the reference's D chunks x I chunks streaming
 * (gpu/mitm_gpu_mstar_driver.py:100-118, 241-262) for sides that do not fit. */
int cf_part_hist(const uint64_t* keys, uint64_t n, uint64_t M, int pbits, uint64_t* counts, void* stream);
int cf_part_scatter(const uint64_t* keys, const uint64_t* ids, uint64_t n, uint64_t M, int pbits, uint64_t* cursor,
                    uint64_t* okeys, uint64_t* oids, void* stream);

/* ---- batched portfolio --------------------------------------------------- */

/* Many moduli (radius 1..cf_batch_max_r() each, mixed) joined by persistent
 * kernels fed from a device work queue: mode 0 builds every modulus's D table,
 * mode 1 probes every modulus's I-rank window, mode 2 checks every candidate.
 * mods: device array of nmod descriptors of cf_batch_mod_bytes() bytes each
 *   {poolD, tailD, poolI, tailI, screen, fpw, side, fill, bloom (8-byte
 *    pointers); nD, i_lo, nI (u64); bbits, fbits, r, swap (i32);
 *    pkw, psd, pcnt (8-byte pointers); pcap, plb (u32)} -- the last five
 *    describe the partitioned build below (pcap = 0: built by mode 0)
 * with the D-table areas laid out as cf_dtab_build2's (fingerprints 32 B, side
 * 128 B, fill 4 B per bucket; Bloom filter 32 B per block) but placed by the
 * caller; fpw, fill and bloom are zeroed before mode 0.  swap = 0: the table
 * holds the D side and the I window probes; swap = 1: the table holds the I
 * window and the D side probes.  tstart: device u64[nmod+1] prefix sums of
 * ceil(side records / ticket) (the table's side for mode 0, the probing side
 * for mode 1); queue: device u64 zeroed before modes 0 and 1;
 * candidates go to pairs/pmod (pair, modulus index) through *npairs, and mode 2
 * writes one result per pair as cf_check_pairs does.  The reference solves one
 * instance at a time (run_instance, gpu/mitm_gpu_mstar_driver.py:184-286,
 * called per instance from the loop at :311); this replaces that loop. */
size_t cf_batch_mod_bytes(void);
int cf_batch_max_r(void);
int cf_batch_run(int mode, const void* mods, const uint64_t* tstart, uint32_t nmod, uint32_t ticket, void* queue,
                 void* pairs, uint32_t* pmod, uint32_t max_pairs, uint32_t* npairs, uint32_t* err, void* results,
                 uint32_t grid, void* stream);

/* Partitioned table build for the batch (moduli with pcap > 0), in place of
 * mode 0 for tables larger than L2: phase 0 generates each table side and
 * scatters its records into bucket ranges of 2^plb buckets (plb 9 or 10, the
 * same for every modulus of one phase-1 launch, given as part_lb; 0 from
 * cf_batch_part_buckets(lb) means lb is not supported)
 * (pkw: range-local bucket << 16 | 16-bit fingerprint, psd: side entry; pcap
 * records per range, counts in pcnt, zeroed by the caller); phase 1 builds each
 * range in shared memory and writes its fingerprint rows and side entries out
 * whole; phase 2 inserts the few records that ran past the end of their range.
 * tstart: phase 0, prefix sums of ceil(table-side records / cf_batch_part_tile());
 * phase 1, prefix sums of the ranges per modulus (2^max(0, bbits - plb), at most
 * cf_batch_part_max_ranges()); 0 for moduli
 * built by mode 0.  queue: device u64 zeroed before phases 0 and 1; ovf:
 * ovf_cap entries of cf_batch_ovf_bytes(), *novf zeroed before phase 1.
 * radius (phase 0): 1..cf_batch_max_r() runs a generator specialised for moduli of that radius (the
 * others must have no tickets in tstart), 0 one for any radius.
 * CF_ERR_PART_OVERFLOW in *err: a range received more than pcap records and
 * the caller rebuilds the batch with mode 0.  The table is the one mode 0 builds
 * (same slots rule), so mode 1 probes it unchanged.  Replaces, like mode 0, the
 * D-side table build of the reference's join (recD, src/mitm64.cpp:51-73;
 * sort_side of the D chunk, gpu/mitm_gpu2.py:101-104). */
uint32_t cf_batch_part_buckets(int lb);
uint32_t cf_batch_part_tile(void);
uint32_t cf_batch_part_max_ranges(void);
size_t cf_batch_ovf_bytes(void);
int cf_batch_part(int phase, const void* mods, const uint64_t* tstart, uint32_t nmod, void* queue, void* ovf,
                  uint32_t ovf_cap, uint32_t* novf, uint32_t* err, int part_lb, int radius, uint32_t grid,
                  void* stream);

/* One prepared batch (the descriptors, ticket sums and buffers a portfolio's
 * prepare step lays out) and the call that runs it: zero the table areas and
 * queue words, the partitioned builds (scatter per radius, range placement,
 * overflow fix-up) when use_part, then cf_batch_run's build, probe and check --
 * every launch on `stream`, with no host wait, so the call can be recorded in a
 * CUDA graph.  misc (64 bytes): +0 build queue, +8 probe queue, +16 candidate
 * count (u32), +20 error word (u32), +24 overflow count, +32 scatter queue,
 * +40 range queue.  Replaces the reference's per-instance loop
 * (gpu/mitm_gpu_mstar_driver.py:296-320). */
typedef struct CfBatchQueue {
  const void* mods;
  void* arena;
  uint64_t zero_bytes;
  void* misc;
  const uint64_t* build_tickets;
  const uint64_t* probe_tickets;
  const uint64_t* place_tickets;
  const uint64_t* const* scatter_tickets;
  const int* scatter_radius;
  void* ovf;
  void* pairs;
  void* pair_mods;
  void* results;
  uint32_t nmod, ticket, grid, max_pairs;
  uint32_t ovf_cap, n_scatter;
  int use_part, part_lb;
  uint32_t n_probe, pad0;                   /* n_probe > 0: one probe launch per radius present, */
  const uint64_t* const* probe_tickets_r;   /* each with the ticket sums of that radius's moduli only */
  const int* probe_radius;
} CfBatchQueue;
int cf_solve_batch(const CfBatchQueue* q, void* stream);

/* ---- sorted-side drop-ins ------------------------------------------------ */

/* Stable LSD radix sort of (keys, ids)[n] by key over key_bits bits, in place;
 * workspace cf_sort_tmp_bytes(n).  Synchronises `stream` once.
 * Replaces sort_side (gpu/mitm_gpu2.py:101-104). */
size_t cf_sort_tmp_bytes(uint64_t n);
int cf_sort_pairs(uint64_t* keys, uint64_t* ids, uint64_t n, int key_bits, void* tmp, size_t tmp_bytes,
                  void* stream);

/* The same sort with the digit width chosen by the caller: digit_bits 8 or 9
 * (other widths return CF_EBADARG), ceil(key_bits / digit_bits) passes, passes
 * whose digit is constant skipped; the result does not depend on the width.
 * Workspace cf_sort_digits_tmp_bytes(n, key_bits, digit_bits) (0 for a bad
 * width or key_bits).  The width is the radix digit width that the autotuner
 * picks per size class for sort_side (gpu/mitm_gpu2.py:101-104), whose call
 * has no such argument. */
size_t cf_sort_digits_tmp_bytes(uint64_t n, int key_bits, int digit_bits);
int cf_sort_pairs_digits(uint64_t* keys, uint64_t* ids, uint64_t n, int key_bits, int digit_bits, void* tmp,
                         size_t tmp_bytes, void* stream);

/* The same sort for callers that cannot allocate device memory (for example
 * when all device memory belongs to another allocator): no workspace argument;
 * the scratch is a fixed array inside this library's own device memory (3 MiB,
 * held by every GPU that loads the library).  n is limited to
 * cf_sort_pairs_noalloc_max() = 131072 records; larger n returns CF_EBADARG.
 * The first call on a device looks up the array's address on that device
 * (make it before any stream capture) and keeps it for the life of the process:
 * after cudaDeviceReset on that device the kept address is stale, so do not use
 * this entry point after a reset.  Like cf_sort_pairs it waits on `stream` once
 * (it reads the digit histogram back).  Calls share the array: device work of
 * two calls must not overlap.  This entry point has no counterpart in the
 * reference. */
uint64_t cf_sort_pairs_noalloc_max(void);
int cf_sort_pairs_noalloc(uint64_t* keys, uint64_t* ids, uint64_t n, int key_bits, void* stream);

/* The equal-key join of sorted Dk[nD] and sorted Ik[nI] with the pairs written
 * on the device in join_sorted's order (I rows in order, D positions in order
 * within a row; gpu/mitm_gpu2.py:107-119).  cf_join_count leaves per-row
 * offsets in tmp (cf_join_tmp_bytes(nI) bytes) and the pair total in the device
 * u64 *npairs; cf_join_emit then writes {Did, Iid} of the first max_pairs pairs
 * to outD, outI. */
size_t cf_join_tmp_bytes(uint64_t nI);
int cf_join_count(const uint64_t* Dk, uint64_t nD, const uint64_t* Ik, uint64_t nI, void* tmp, size_t tmp_bytes,
                  uint64_t* npairs, void* stream);
int cf_join_emit(const uint64_t* Dk, const uint64_t* Did, uint64_t nD, const uint64_t* Ik, const uint64_t* Iid,
                 uint64_t nI, const void* tmp, uint64_t* outD, uint64_t* outI, uint64_t max_pairs, void* stream);

/* Equal-key runs between sorted Dk[nD] and sorted Ik[nI]: runs (24 bytes each,
 * {I row, first D position, count}), unordered, counted in the device u64
 * counters *nruns and *npairs (zeroed by the caller).  The count/emit core of
 * join_sorted (gpu/mitm_gpu2.py:107-119). */
size_t cf_merge_run_bytes(void);
int cf_merge_join_runs(const uint64_t* Dk, uint64_t nD, const uint64_t* Ik, uint64_t nI, void* runs,
                       uint64_t max_runs, uint64_t* nruns, uint64_t* npairs, uint32_t* err, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CFMITM_H */

// cf_batch.cu -- batched portfolio: many moduli with uneven pool sizes and mixed
// radii joined by persistent kernels that pull work from a device queue.
//
// The host describes each modulus once (CfBatchMod: its D and I pool tables,
// tail tables, screen table, D-table areas and the I-rank window to probe) and
// the prefix sums of its work in tickets of `ticket` consecutive records.
// Three launches then cover the whole batch, whatever its radii:
//   k_batch<0>      builds every modulus's D table   (tickets over the D sides)
//   k_batch<1>      probes every I window            (tickets over the I sides)
//   k_batch_check   checks every candidate pair
// A warp takes the next ticket with one atomicAdd on the queue head, finds its
// modulus by binary search over the ticket prefix sums, and runs the walker and
// D-table code of the single-modulus kernels (cf_dtab.cuh) instantiated for the
// modulus's radius.  Tickets are ordered by modulus, so at any moment the SMs
// work on one or two moduli and the D table being probed stays in L2; small
// moduli cost no launches and no host round trips, large ones spread over every
// SM.  The launch sequence is fixed for a batch, so it can be captured in a CUDA
// graph and replayed.
#include "cf_check.cuh"
#include "cf_dtab.cuh"

namespace {

constexpr int kBatchBlock = 256;
constexpr int kBatchMaxR = 8;

// One modulus of a batch.  fpw/fill/bloom are zeroed by the caller before the
// build; side needs no initialisation.  D ranks are [0, nD); I ranks
// [i_lo, i_lo + nI).  swap = 0: the table holds the D side and the I window
// probes; swap = 1: the table holds the I window and the D side probes.
struct CfBatchMod {
  const u64* poolD;
  const CfTailEnt* tailD;
  const u64* poolI;
  const CfTailEnt* tailI;
  const CfScreen* screen;
  u32* fpw;          // 32 B per bucket: sixteen 16-bit fingerprints
  uint2* side;       // 128 B per bucket: {32-bit fingerprint, D rank} per slot
  u32* fill;         // 4 B per bucket
  u32* bloom;        // 2^fbits blocks of 32 B, or null
  u64 nD, i_lo, nI;
  int bbits, fbits;
  int r, swap;
  // partitioned build (pcap > 0): the table side's records are first scattered
  // into 2^max(0, bbits - plb) bucket ranges, then each range is built in
  // shared memory and written out whole
  u32* pkw;          // [nparts * pcap]: bucket within the range << 16 | 16-bit fingerprint
  uint2* psd;        // [nparts * pcap]: side entries {32-bit fingerprint, rank - rank0}
  u32* pcnt;         // [nparts]: records scattered into each range (zeroed by the caller)
  u32 pcap;          // records a range holds (0: this modulus uses the in-place build)
  u32 plb;           // log2 buckets per range (kPlbMin..kPlbMax)
};

template <int R, int MODE>
__device__ __forceinline__ bool batch_ticket(const CfBatchMod& md, u32 mod, u64 first, u32 left, int lane,
                                             const CfPairSink& sink0) {
  constexpr int B = R < 2 ? R : 2;
  const bool d_side = (MODE == 0) == (md.swap == 0);     // this ticket walks the D side
  const u64* pool = d_side ? md.poolD : md.poolI;
  const CfTailEnt* tail = d_side ? md.tailD : md.tailI;
  const CfPoolHdr* hd = (const CfPoolHdr*)pool;
  if (!hd->fast32 || hd->tail_b != (u64)B) return false;
  const int n = (int)hd->n;
  const u64* binom = pool + cf_pool_off_binom(n);
  CfArithFast ar;
  ar.md = cf_mod32_from_hdr(hd);
  ar.p = nullptr;
  ar.p64 = pool + cf_pool_off_prime(n);
  const u64 minv = hd->minv;
  CfElt32 st;
  st.X = hd->X0s;
  st.x2 = hd->x20;
  DTab tab;
  tab.xb = 0;                  // wide side entries
  tab.nb = 1ull << md.bbits;
  tab.fpw = md.fpw;
  tab.side = md.side;
  tab.fill = md.fill;
  tab.bloom = md.bloom;
  tab.rank0 = md.swap ? md.i_lo : 0;
  tab.bbits = md.bbits;
  tab.fbits = md.fbits;
  CfPairSink sink = sink0;
  sink.mod = mod;
  sink.swap = (u32)md.swap;
  CfTailWalker<R, B> w;
  w.init(first, n, binom, ar, st, hd->tail_n);
  const u64 rank_base = first + (u64)lane;
  bool ok = true;
  for (u32 off = 0; off < left; off += 32) {      // uniform across the warp
    CfElt32 q = st;
    u64 j;
    int unused[R - B > 0 ? R - B : 1];
    w.template step<false>(n, binom, ar, lane, q, j, unused);
    if (off + (u32)lane < left) {
      u64 X;
      u32 x2;
      cf_fuse_res(q, tail[j], ar.md, minv, X, x2);
      if (MODE == 0) {
        ok &= dtab_insert(tab, X, x2, rank_base + off);
      } else {
        if (tab.bloom) {
          const CfBloomKey bk = cf_bloom_key(X, x2, tab.fbits);
          const uint4* blk = (const uint4*)(tab.bloom + (u64)bk.block * 8);
          const uint4 a = __ldg(blk), c = __ldg(blk + 1);
          const bool in = (cf_word8(a, c, bk.w0) & bk.m0) && (cf_word8(a, c, bk.w1) & bk.m1) &&
                          (cf_word8(a, c, bk.w2) & bk.m2);
          if (!in) continue;
        }
        dtab_probe(tab, X, x2, rank_base + off, sink);
      }
    }
  }
  return ok;
}

// The modulus of ticket t (tstart[lo] <= t < tstart[lo + 1]).  `hint` is the modulus of the caller's
// previous ticket, 0 before the first: tickets from the queue only grow, so tstart[hint] <= t, and the
// ticket usually falls in that modulus or the next; a binary search over the rest otherwise.
__device__ __forceinline__ u32 ticket_mod(const u64* __restrict__ tstart, u32 nmod, u64 t, u32 hint) {
  if (tstart[hint + 1] > t) return hint;
  u32 lo = hint + 1, hi = nmod;                // tstart[lo] <= t < tstart[hi]
  if (tstart[lo + 1] > t) return lo;
  while (hi - lo > 1) {
    const u32 mid = (lo + hi) >> 1;
    if (tstart[mid] <= t) lo = mid; else hi = mid;
  }
  return lo;
}

// RF = 0: any radius (a switch into the radius-templated code); RF > 0: every
// modulus of the launch has radius RF (its ticket sums hold only those), so the
// kernel carries only that radius's code and registers.
template <int MODE, int RF>
__global__ void __launch_bounds__(kBatchBlock, (MODE == 1 && RF > 0) ? 4 : 1)   // one-radius probes: 4 CTAs per SM
k_batch(const CfBatchMod* __restrict__ mods, const u64* __restrict__ tstart /*[nmod+1]*/, u32 nmod, u32 ticket,
        unsigned long long* __restrict__ queue, CfPair* __restrict__ pairs, u32* __restrict__ pmod, u32 max_pairs,
        u32* __restrict__ npairs, u32* __restrict__ err) {
  const int lane = threadIdx.x & 31;
  const u64 total = tstart[nmod];
  CfPairSink sink;
  sink.pairs = pairs;
  sink.mods = pmod;
  sink.npairs = npairs;
  sink.err = err;
  sink.max_pairs = max_pairs;
  sink.mod = 0;
  sink.swap = 0;
  bool ok = true, badarg = false;
  u32 lo = 0;                                 // modulus of the warp's ticket
  for (;;) {
    u64 t = 0;
    if (lane == 0) t = atomicAdd(queue, 1ull);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= total) break;
    lo = ticket_mod(tstart, nmod, t, lo);
    const CfBatchMod& md = mods[lo];
    const bool d_side = (MODE == 0) == (md.swap == 0);
    const u64 n_side = d_side ? md.nD : md.nI;
    const u64 first = (t - tstart[lo]) * (u64)ticket;
    if (first >= n_side) continue;
    const u32 left = (u32)((n_side - first) < ticket ? (n_side - first) : ticket);
    const u64 rank0 = first + (d_side ? 0 : md.i_lo);
    bool good;
    if constexpr (RF > 0) {
      if (md.r == RF) {
        good = batch_ticket<RF, MODE>(md, lo, rank0, left, lane, sink);
      } else {
        good = true;
        badarg = true;
      }
    } else switch (md.r) {
      case 1: good = batch_ticket<1, MODE>(md, lo, rank0, left, lane, sink); break;
      case 2: good = batch_ticket<2, MODE>(md, lo, rank0, left, lane, sink); break;
      case 3: good = batch_ticket<3, MODE>(md, lo, rank0, left, lane, sink); break;
      case 4: good = batch_ticket<4, MODE>(md, lo, rank0, left, lane, sink); break;
      case 5: good = batch_ticket<5, MODE>(md, lo, rank0, left, lane, sink); break;
      case 6: good = batch_ticket<6, MODE>(md, lo, rank0, left, lane, sink); break;
      case 7: good = batch_ticket<7, MODE>(md, lo, rank0, left, lane, sink); break;
      case 8: good = batch_ticket<8, MODE>(md, lo, rank0, left, lane, sink); break;
      default: good = true; badarg = true; break;
    }
    ok &= good;
  }
  if (!ok) atomicOr(err, MODE == 0 ? CF_ERR_TABLE_FULL : CF_ERR_BAD_ARG);
  if (badarg) atomicOr(err, CF_ERR_BAD_ARG);
}

// ---------------------------------------------------------------------------
// Partitioned table build.  Building a table larger than L2 by compare-and-swap
// in place costs a random DRAM read and write of a fingerprint sector and of a
// side-entry sector per record.  Instead:
//   k_bscatter  generates the table side in tiles of kScTile records, ranks each
//               tile's records by bucket range (2^plb buckets) in shared
//               memory, reserves each range's space with one atomic per tile
//               and writes the records there (the writes of one range land in
//               consecutive addresses, so L2 merges them into whole sectors);
//   k_bplace    takes one bucket range per CTA, claims its records' slots in
//               shared memory with the same rule as dtab_claim, and writes the
//               range's fingerprint rows and side entries out in order;
//   k_bfix      inserts the rare records that ran past the end of their range
//               (every bucket from theirs to the range's last one full) into
//               the finished table with dtab_claim, continuing in the next range.
// The result is a table the probe reads exactly like one built in place: every
// record sits in the first non-full bucket at or after its own.
// ---------------------------------------------------------------------------
constexpr int kPlbMin = 9;                    // 512-bucket ranges: 80 KB, two CTAs per SM
constexpr int kPlbMax = 10;                   // 1024-bucket ranges: 160 KB, one CTA per SM
constexpr int kScBlock = 256;
constexpr int kScMinBlocks = 3;               // CTAs per SM (registers for the pipelined generator)
constexpr int kScTile = 4064;                 // records per scatter ticket (508 per warp; 56 KB of
                                              // shared memory per CTA)
constexpr int kScWarpRecs = kScTile / (kScBlock / 32);
constexpr u32 kScMaxParts = 2048;             // bucket ranges per modulus (bbits <= plb + 11)
constexpr size_t kScSmem = (size_t)kScTile * 12 + (size_t)kScMaxParts * 4;
constexpr int kPlItems = 8;                   // records a thread loads before claiming (more loop if needed)
template <int PLB>
struct PlaceShape {
  static constexpr int kBlock = PLB == kPlbMax ? 1024 : 512;
  static constexpr int kMinBlocks = PLB == kPlbMax ? 1 : 2;
  static constexpr u32 kBuckets = 1u << PLB;
  static constexpr size_t kSmem = (size_t)kBuckets * (32 + 128 + 4);
};

struct CfOvf {
  u32 mod, bucket, f16, f32, rank, pad;
};

template <int R>
__device__ __forceinline__ bool scatter_gen(const CfBatchMod& md, u64 first, u32 count, u32* s_kw, u32* s_pp,
                                            u32* s_f32, u32* s_h) {
  constexpr int B = R < 2 ? R : 2;
  const bool d_side = md.swap == 0;              // the table holds the smaller side
  const u64* pool = d_side ? md.poolD : md.poolI;
  const CfTailEnt* tail = d_side ? md.tailD : md.tailI;
  const CfPoolHdr* hd = (const CfPoolHdr*)pool;
  if (!hd->fast32 || hd->tail_b != (u64)B) return false;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const u32 wbeg = (u32)wid * kScWarpRecs;
  if (wbeg >= count) return true;
  const u32 wcnt = min((u32)kScWarpRecs, count - wbeg);
  const int n = (int)hd->n;
  const u64* binom = pool + cf_pool_off_binom(n);
  CfArithFast ar;
  ar.md = cf_mod32_from_hdr(hd);
  ar.p = nullptr;
  ar.p64 = pool + cf_pool_off_prime(n);
  const u64 minv = hd->minv;
  CfElt32 st;
  st.X = hd->X0s;
  st.x2 = hd->x20;
  const u64 rank0 = d_side ? 0 : md.i_lo;        // enumeration rank of the side's first record
  CfTailWalker<R, B> w;
  w.init(rank0 + first + wbeg, n, binom, ar, st, hd->tail_n);
  const int plb = (int)md.plb;
  const u32 pmask = md.bbits > plb ? ~0u : 0u;
  // software-pipelined: the next step's tail entry is loaded before this step's record is hashed and
  // staged, so the table read overlaps the work instead of stalling the warp
  int unused[R - B > 0 ? R - B : 1];
  CfElt32 qn = st;
  u64 jn;
  w.template step<false>(n, binom, ar, lane, qn, jn, unused);
  CfTailEnt en = (u32)lane < wcnt ? tail[jn] : CfTailEnt{};
  for (u32 off = 0; off < wcnt; off += 32) {     // uniform across the warp
    const CfElt32 q = qn;
    const CfTailEnt e = en;
    if (off + 32 < wcnt) {
      qn = st;
      w.template step<false>(n, binom, ar, lane, qn, jn, unused);
      if (off + 32 + (u32)lane < wcnt) en = tail[jn];
    }
    if (off + (u32)lane < wcnt) {
      u64 X;
      u32 x2;
      cf_fuse_res(q, e, ar.md, minv, X, x2);
      if (md.bloom) {
        const CfBloomKey bk = cf_bloom_key(X, x2, md.fbits);
        u32* blk = md.bloom + (u64)bk.block * 8;
        atomicOr(blk + bk.w0, bk.m0);
        atomicOr(blk + bk.w1, bk.m1);
        atomicOr(blk + bk.w2, bk.m2);
      }
      const CfFuseKey fk = cf_fuse_key(X, x2, md.bbits);
      const u32 p = (fk.bucket >> plb) & pmask;
      const u32 bl = fk.bucket & ((1u << plb) - 1u);
      const u32 pos = atomicAdd(&s_h[p], 1u);
      const u32 i = wbeg + off + (u32)lane;
      s_kw[i] = (bl << 16) | fk.f16;
      s_pp[i] = (p << 12) | pos;
      s_f32[i] = fk.f32;
    }
  }
  return true;
}

// RF = 0: any radius (a switch into the radius-templated generator); RF = 1..8: only
// moduli of that radius (the others have no tickets), with the generator's registers
// sized for it -- fitting four CTAs per SM.
template <int RF>
__global__ void __launch_bounds__(kScBlock, kScMinBlocks)
k_bscatter(const CfBatchMod* __restrict__ mods, const u64* __restrict__ tstart, u32 nmod,
           unsigned long long* __restrict__ queue, u32* __restrict__ err) {
  extern __shared__ __align__(16) unsigned char smem[];
  u32* s_kw = (u32*)smem;                        // [kScTile] bucket within the range << 16 | 16-bit fingerprint
  u32* s_pp = s_kw + kScTile;                    // [kScTile] range << 12 | place among the tile's records of it
  u32* s_f32 = s_pp + kScTile;                   // [kScTile] 32-bit fingerprint (the side entry's rank is first + i)
  u32* s_h = s_f32 + kScTile;                    // [kScMaxParts] tile counts, then global offsets
  __shared__ u64 s_t;
  const u64 total = tstart[nmod];
  bool ok = true;
  u32 lo = 0;                                    // modulus of the CTA's ticket
  for (;;) {
    if (threadIdx.x == 0) s_t = atomicAdd(queue, 1ull);
    __syncthreads();
    const u64 t = s_t;
    if (t >= total) break;
    lo = ticket_mod(tstart, nmod, t, lo);
    const CfBatchMod& md = mods[lo];
    const u64 n_side = md.swap ? md.nI : md.nD;
    const u64 first = (t - tstart[lo]) * (u64)kScTile;
    const bool plb_ok = md.plb >= (u32)kPlbMin && md.plb <= (u32)kPlbMax;
    const u32 nparts = plb_ok && md.bbits > (int)md.plb ? 1u << (md.bbits - (int)md.plb) : 1u;
    const bool good = first < n_side && nparts <= kScMaxParts && md.pcap > 0 && plb_ok;
    const u32 count = good ? (u32)min((u64)kScTile, n_side - first) : 0u;
    for (u32 p = threadIdx.x; p < nparts && good; p += kScBlock) s_h[p] = 0;
    __syncthreads();
    if (good) {
      bool g = true;
      if (RF != 0) {
        g = md.r == RF && scatter_gen<RF != 0 ? RF : 1>(md, first, count, s_kw, s_pp, s_f32, s_h);
      } else switch (md.r) {
        case 1: g = scatter_gen<1>(md, first, count, s_kw, s_pp, s_f32, s_h); break;
        case 2: g = scatter_gen<2>(md, first, count, s_kw, s_pp, s_f32, s_h); break;
        case 3: g = scatter_gen<3>(md, first, count, s_kw, s_pp, s_f32, s_h); break;
        case 4: g = scatter_gen<4>(md, first, count, s_kw, s_pp, s_f32, s_h); break;
        case 5: g = scatter_gen<5>(md, first, count, s_kw, s_pp, s_f32, s_h); break;
        case 6: g = scatter_gen<6>(md, first, count, s_kw, s_pp, s_f32, s_h); break;
        case 7: g = scatter_gen<7>(md, first, count, s_kw, s_pp, s_f32, s_h); break;
        case 8: g = scatter_gen<8>(md, first, count, s_kw, s_pp, s_f32, s_h); break;
        default: g = false; break;
      }
      ok &= g;
    } else if (first < n_side) {
      ok = false;
    }
    __syncthreads();
    // reserve each range's space: a thread's (up to 16) atomics are issued together
    for (u32 p0 = 0; p0 < nparts && good; p0 += kScBlock * 16) {
      u32 c[16], g[16];
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const u32 p = p0 + threadIdx.x + (u32)k * kScBlock;
        c[k] = p < nparts ? s_h[p] : 0u;
      }
#pragma unroll
      for (int k = 0; k < 16; ++k) g[k] = c[k] ? atomicAdd(&md.pcnt[p0 + threadIdx.x + (u32)k * kScBlock], c[k]) : 0u;
#pragma unroll
      for (int k = 0; k < 16; ++k)
        if (c[k]) s_h[p0 + threadIdx.x + (u32)k * kScBlock] = g[k];
    }
    __syncthreads();
    bool over = false;
#pragma unroll 4
    for (u32 i = threadIdx.x; i < count; i += kScBlock) {
      const u32 pp = s_pp[i];
      const u32 p = pp >> 12;
      const u32 g = s_h[p] + (pp & 0xfffu);
      if (g < md.pcap) {
        const u64 at = (u64)p * md.pcap + g;
        md.pkw[at] = s_kw[i];
        md.psd[at] = make_uint2(s_f32[i], (u32)(first + i));
      } else {
        over = true;
      }
    }
    if (over) atomicOr(err, CF_ERR_PART_OVERFLOW);
    __syncthreads();
  }
  if (!ok) atomicOr(err, CF_ERR_BAD_ARG);
}

// Claim a slot in the shared-memory rows of one bucket range.  The range is
// private to this CTA, so a per-bucket fill counter hands out slots 0, 1, 2, ...
// in claim order (one shared atomic per claim): the occupied slots of a bucket
// are a prefix, a bucket is full after 16 claims and later claims continue in the
// next bucket -- the layout dtab_claim produces.  Returns false when the claim
// ran past the range's last bucket (only when the range is not the whole table;
// a whole table wraps around).
__device__ __forceinline__ bool place_claim(unsigned short* s_fp16, uint2* s_side, u32* s_fill, u32 nbp, bool whole,
                                            u32 b, u32 f16, uint2 sd) {
  for (u32 tries = 0; tries < nbp; ++tries) {
    const u32 slot = atomicAdd(&s_fill[b], 1u);
    if (slot < 16u) {
      s_fp16[b * 16 + slot] = (unsigned short)f16;
      s_side[b * 16 + slot] = sd;
      return true;
    }
    if (++b == nbp) {
      if (!whole) return false;
      b = 0;
    }
  }
  return false;
}

template <int PLB>
__global__ void __launch_bounds__(PlaceShape<PLB>::kBlock, PlaceShape<PLB>::kMinBlocks)
k_bplace(const CfBatchMod* __restrict__ mods, const u64* __restrict__ tstart, u32 nmod,
         unsigned long long* __restrict__ queue, CfOvf* __restrict__ ovf, u32 ovf_cap, u32* __restrict__ novf,
         u32* __restrict__ err) {
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr int kPlBlock = PlaceShape<PLB>::kBlock;
  constexpr u32 kPartBuckets = PlaceShape<PLB>::kBuckets;
  u32* s_fp = (u32*)smem;                                    // [kPartBuckets * 8]
  uint2* s_side = (uint2*)(s_fp + kPartBuckets * 8);         // [kPartBuckets * 16]
  u32* s_fill = (u32*)(s_side + kPartBuckets * 16);          // [kPartBuckets] slots claimed
  __shared__ u64 s_t;
  const u64 total = tstart[nmod];
  u32 lo = 0;                                    // modulus of the CTA's ticket
  for (;;) {
    if (threadIdx.x == 0) s_t = atomicAdd(queue, 1ull);
    __syncthreads();
    const u64 t = s_t;
    if (t >= total) break;
    lo = ticket_mod(tstart, nmod, t, lo);
    const CfBatchMod& md = mods[lo];
    const u32 p = (u32)(t - tstart[lo]);
    if (md.plb != (u32)PLB) {                    // the launch's range size must be the modulus's
      if (threadIdx.x == 0) atomicOr(err, CF_ERR_BAD_ARG);
      __syncthreads();
      continue;
    }
    const u64 nb = 1ull << md.bbits;
    const u32 nbp = nb < kPartBuckets ? (u32)nb : kPartBuckets;
    const u64 b0 = (u64)p * nbp;
    const bool whole = nbp == nb;
    for (u32 i = threadIdx.x; i < nbp * 8; i += kPlBlock) s_fp[i] = 0;
    for (u32 i = threadIdx.x; i < nbp; i += kPlBlock) s_fill[i] = 0;
    __syncthreads();
    const u32 cnt = min(md.pcnt[p], md.pcap);
    const u32* kw = md.pkw + (u64)p * md.pcap;
    const uint2* sd = md.psd + (u64)p * md.pcap;
    for (u32 i0 = 0; i0 < cnt; i0 += kPlBlock * kPlItems) {
     u32 kk[kPlItems];
     uint2 ee[kPlItems];
#pragma unroll
     for (int q = 0; q < kPlItems; ++q) {        // this thread's records, loads issued together
       const u32 i = i0 + threadIdx.x + (u32)q * kPlBlock;
       kk[q] = i < cnt ? __ldcs(kw + i) : 0u;
       ee[q] = i < cnt ? __ldcs(sd + i) : make_uint2(0u, 0u);
     }
#pragma unroll
     for (int q = 0; q < kPlItems; ++q) {
      if (i0 + threadIdx.x + (u32)q * kPlBlock >= cnt) continue;
      const u32 k = kk[q];
      const uint2 e = ee[q];
      const u32 b = (k >> 16) & (nbp - 1u);
      if (!place_claim((unsigned short*)s_fp, s_side, s_fill, nbp, whole, b, k & 0xffffu, e)) {
        if (whole) {
          atomicOr(err, CF_ERR_TABLE_FULL);
          continue;
        }
        const u32 o = atomicAdd(novf, 1u);
        if (o < ovf_cap) {
          CfOvf v;
          v.mod = lo;
          v.bucket = (u32)((b0 + nbp) & (nb - 1));
          v.f16 = k & 0xffffu;
          v.f32 = e.x;
          v.rank = e.y;
          v.pad = 0;
          ovf[o] = v;
        } else {
          atomicOr(err, CF_ERR_TABLE_FULL);
        }
      }
     }
    }
    __syncthreads();
    uint4* gfp = (uint4*)(md.fpw + b0 * 8);
    const uint4* sfp = (const uint4*)s_fp;
    for (u32 i = threadIdx.x; i < nbp * 2; i += kPlBlock) gfp[i] = sfp[i];
    uint4* gsd = (uint4*)(md.side + b0 * 16);
    const uint4* ssd = (const uint4*)s_side;
    for (u32 i = threadIdx.x; i < nbp * 8; i += kPlBlock) gsd[i] = ssd[i];
    __syncthreads();
  }
}

__global__ void __launch_bounds__(256)
k_bfix(const CfBatchMod* __restrict__ mods, const CfOvf* __restrict__ ovf, const u32* __restrict__ novf, u32 ovf_cap,
       u32* __restrict__ err) {
  const u32 n = min(*novf, ovf_cap);
  for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const CfOvf v = ovf[i];
    const CfBatchMod& md = mods[v.mod];
    DTab tab;
    tab.xb = 0;                  // wide side entries
    tab.nb = 1ull << md.bbits;
    tab.fpw = md.fpw;
    tab.side = md.side;
    tab.fill = md.fill;
    tab.bloom = md.bloom;
    tab.rank0 = 0;
    tab.bbits = md.bbits;
    tab.fbits = md.fbits;
    if (!dtab_claim(tab, v.bucket, v.f16, make_uint2(v.f32, v.rank))) atomicOr(err, CF_ERR_TABLE_FULL);
  }
}

__global__ void __launch_bounds__(128)
k_batch_check(const CfBatchMod* __restrict__ mods, const CfPair* __restrict__ pairs, const u32* __restrict__ pmod,
              const u32* __restrict__ npairs, u32 max_pairs, CfPairResult* __restrict__ res) {
  const u32 np = min(*npairs, max_pairs);
  for (u32 t = blockIdx.x * blockDim.x + threadIdx.x; t < np; t += gridDim.x * blockDim.x) {
    const CfBatchMod& md = mods[pmod[t]];
    CfPairResult o;
    switch (md.r) {
      case 1: o = cf_check_one<1>(md.poolD, md.poolI, md.screen, pairs[t]); break;
      case 2: o = cf_check_one<2>(md.poolD, md.poolI, md.screen, pairs[t]); break;
      case 3: o = cf_check_one<3>(md.poolD, md.poolI, md.screen, pairs[t]); break;
      case 4: o = cf_check_one<4>(md.poolD, md.poolI, md.screen, pairs[t]); break;
      case 5: o = cf_check_one<5>(md.poolD, md.poolI, md.screen, pairs[t]); break;
      case 6: o = cf_check_one<6>(md.poolD, md.poolI, md.screen, pairs[t]); break;
      case 7: o = cf_check_one<7>(md.poolD, md.poolI, md.screen, pairs[t]); break;
      default: o = cf_check_one<8>(md.poolD, md.poolI, md.screen, pairs[t]); break;
    }
    res[t] = o;
  }
}

}  // namespace

extern "C" size_t cf_batch_mod_bytes(void) { return sizeof(CfBatchMod); }
extern "C" int cf_batch_max_r(void) { return kBatchMaxR; }

static int batch_launch(int mode, int rf, const void* mods, const u64* tstart, u32 nmod, u32 ticket, void* queue,
                        void* pairs, u32* pmod, u32 max_pairs, u32* npairs, u32* err, u32 grid, cudaStream_t st);

// mode 0: build the table of every modulus (from its smaller side); mode 1:
// probe it with the other side; mode 2: check every candidate pair.
//   mods    device array of nmod CfBatchMod descriptors (radius 1..8 each)
//   tstart  device array of nmod+1 ticket prefix sums: tstart[m+1]-tstart[m] =
//           ceil(records of the table's side / ticket) for mode 0, of the
//           probing side for mode 1
//   ticket  records per ticket, a multiple of 32 (modes 0 and 1)
//   queue   device u64, zeroed before each of modes 0 and 1
//   pairs, pmod  candidate (D rank, I rank) pairs and their modulus indices,
//           appended through *npairs (zeroed before mode 1)
//   results mode 2: one CfPairResult per pair
//   grid    persistent CTAs (0 = as many as are resident at once)
extern "C" int cf_batch_run(int mode, const void* mods, const u64* tstart, u32 nmod, u32 ticket, void* queue,
                            void* pairs, u32* pmod, u32 max_pairs, u32* npairs, u32* err, void* results, u32 grid,
                            void* stream) {
  if (mode < 0 || mode > 2 || !mods || !npairs || !err || nmod == 0 ||
      (mode < 2 && (!tstart || !queue || ticket == 0 || (ticket & 31u))) || (max_pairs && (!pairs || !pmod)) ||
      (mode == 2 && max_pairs && !results)) {
    cf_set_error("cf_batch_run: bad arguments%s", "");
    return CF_EBADARG;
  }
  const cudaStream_t st = (cudaStream_t)stream;
  if (mode == 2) {
    if (max_pairs == 0) return CF_OK;
    const u32 g = (max_pairs + 127) / 128;
    k_batch_check<<<g < 1024u ? g : 1024u, 128, 0, st>>>((const CfBatchMod*)mods, (const CfPair*)pairs, pmod, npairs,
                                                          max_pairs, (CfPairResult*)results);
    CF_LAUNCH_CHECK("cf_batch_run(check)");
    return CF_OK;
  }
  return batch_launch(mode, 0, mods, tstart, nmod, ticket, queue, pairs, pmod, max_pairs, npairs, err, grid, st);
}

// (definitions of the launch helpers declared above cf_batch_run)
// Launch k_batch<mode, rf> as a persistent wave (grid 0: as many CTAs as are
// resident at once, looked up once per mode, radius and device).
template <int MODE, int RF>
static int batch_launch_t(const void* mods, const u64* tstart, u32 nmod, u32 ticket, void* queue, void* pairs,
                          u32* pmod, u32 max_pairs, u32* npairs, u32* err, u32 grid, cudaStream_t st) {
  if (grid == 0) {
    static int s_grid[64];                    // per device; benign race (same value)
    int dev = 0;
    cudaGetDevice(&dev);
    int* slot = (dev >= 0 && dev < 64) ? &s_grid[dev] : nullptr;
    if (slot && *slot) {
      grid = (u32)*slot;
    } else {
      int sms = 148, per_sm = 0;
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch<MODE, RF>, kBatchBlock, 0);
      grid = (u32)sms * (u32)(per_sm > 0 ? per_sm : 1);
      if (slot) *slot = (int)grid;
    }
  }
  k_batch<MODE, RF><<<grid, kBatchBlock, 0, st>>>((const CfBatchMod*)mods, tstart, nmod, ticket,
                                                  (unsigned long long*)queue, (CfPair*)pairs, pmod, max_pairs,
                                                  npairs, err);
  CF_LAUNCH_CHECK("cf_batch_run");
  return CF_OK;
}

static int batch_launch(int mode, int rf, const void* mods, const u64* tstart, u32 nmod, u32 ticket, void* queue,
                        void* pairs, u32* pmod, u32 max_pairs, u32* npairs, u32* err, u32 grid, cudaStream_t st) {
#define CF_BL(M, R) batch_launch_t<M, R>(mods, tstart, nmod, ticket, queue, pairs, pmod, max_pairs, npairs, err, grid, st)
  if (mode == 0) return CF_BL(0, 0);
  switch (rf) {
    case 1: return CF_BL(1, 1);
    case 2: return CF_BL(1, 2);
    case 3: return CF_BL(1, 3);
    case 4: return CF_BL(1, 4);
    case 5: return CF_BL(1, 5);
    case 6: return CF_BL(1, 6);
    case 7: return CF_BL(1, 7);
    case 8: return CF_BL(1, 8);
    default: return CF_BL(1, 0);
  }
#undef CF_BL
}

extern "C" u32 cf_batch_part_buckets(int lb) { return lb >= kPlbMin && lb <= kPlbMax ? 1u << lb : 0u; }
extern "C" u32 cf_batch_part_tile(void) { return kScTile; }
extern "C" u32 cf_batch_part_max_ranges(void) { return kScMaxParts; }
extern "C" size_t cf_batch_ovf_bytes(void) { return sizeof(CfOvf); }

// Partitioned table build of the moduli whose descriptor has pcap > 0.
//   phase 0: scatter (tstart: nmod+1 prefix sums of ceil(table-side records /
//            cf_batch_part_tile()), 0 for moduli built in place)
//   phase 1: place (tstart: prefix sums of the bucket ranges per modulus,
//            2^max(0, bbits - log2 cf_batch_part_buckets()), 0 for in-place moduli)
//   phase 2: insert the records that ran past their range (tstart unused)
// queue: a device u64 zeroed before each of phases 0 and 1; ovf: ovf_cap entries of
// cf_batch_ovf_bytes(), *novf zeroed before phase 1.  Errors go to *err:
// CF_ERR_PART_OVERFLOW when a range received more than pcap records (the caller
// rebuilds in place), CF_ERR_TABLE_FULL when the overflow list ran out.
template <int RF>
static cudaError_t launch_scatter(const void* mods, const u64* tstart, u32 nmod, void* queue, u32* err, u32 grid,
                                  int sms, cudaStream_t st) {
  cudaError_t e = cudaFuncSetAttribute(k_bscatter<RF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kScSmem);
  if (e != cudaSuccess) return e;
  k_bscatter<RF><<<grid ? grid : (u32)sms * kScMinBlocks, kScBlock, kScSmem, st>>>(
      (const CfBatchMod*)mods, tstart, nmod, (unsigned long long*)queue, err);
  return cudaGetLastError();
}

extern "C" int cf_batch_part(int phase, const void* mods, const u64* tstart, u32 nmod, void* queue, void* ovf,
                             u32 ovf_cap, u32* novf, u32* err, int part_lb, int radius, u32 grid, void* stream) {
  if (phase < 0 || phase > 2 || !mods || nmod == 0 || !err || (phase < 2 && (!tstart || !queue)) ||
      (phase > 0 && (!novf || (ovf_cap && !ovf))) || (phase == 1 && (part_lb < kPlbMin || part_lb > kPlbMax)) ||
      radius < 0 || radius > kBatchMaxR) {
    cf_set_error("cf_batch_part: bad arguments%s", "");
    return CF_EBADARG;
  }
  const cudaStream_t st = (cudaStream_t)stream;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (phase == 0) {
    cudaError_t e;
    switch (radius) {
      case 1: e = launch_scatter<1>(mods, tstart, nmod, queue, err, grid, sms, st); break;
      case 2: e = launch_scatter<2>(mods, tstart, nmod, queue, err, grid, sms, st); break;
      case 3: e = launch_scatter<3>(mods, tstart, nmod, queue, err, grid, sms, st); break;
      case 4: e = launch_scatter<4>(mods, tstart, nmod, queue, err, grid, sms, st); break;
      case 5: e = launch_scatter<5>(mods, tstart, nmod, queue, err, grid, sms, st); break;
      case 6: e = launch_scatter<6>(mods, tstart, nmod, queue, err, grid, sms, st); break;
      case 7: e = launch_scatter<7>(mods, tstart, nmod, queue, err, grid, sms, st); break;
      case 8: e = launch_scatter<8>(mods, tstart, nmod, queue, err, grid, sms, st); break;
      default: e = launch_scatter<0>(mods, tstart, nmod, queue, err, grid, sms, st); break;
    }
    if (e != cudaSuccess) return cf_cuda_status(e, "cf_batch_part(scatter)");
  } else if (phase == 1) {
    cudaError_t e;
    if (part_lb == kPlbMax) {
      using S = PlaceShape<kPlbMax>;
      e = cudaFuncSetAttribute(k_bplace<kPlbMax>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::kSmem);
      if (e != cudaSuccess) return cf_cuda_status(e, "cf_batch_part: smem attribute");
      k_bplace<kPlbMax><<<grid ? grid : (u32)sms * S::kMinBlocks, S::kBlock, S::kSmem, st>>>(
          (const CfBatchMod*)mods, tstart, nmod, (unsigned long long*)queue, (CfOvf*)ovf, ovf_cap, novf, err);
    } else {
      using S = PlaceShape<kPlbMin>;
      e = cudaFuncSetAttribute(k_bplace<kPlbMin>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::kSmem);
      if (e != cudaSuccess) return cf_cuda_status(e, "cf_batch_part: smem attribute");
      k_bplace<kPlbMin><<<grid ? grid : (u32)sms * S::kMinBlocks, S::kBlock, S::kSmem, st>>>(
          (const CfBatchMod*)mods, tstart, nmod, (unsigned long long*)queue, (CfOvf*)ovf, ovf_cap, novf, err);
    }
  } else {
    k_bfix<<<32, 256, 0, st>>>((const CfBatchMod*)mods, (const CfOvf*)ovf, novf, ovf_cap, err);
  }
  CF_LAUNCH_CHECK("cf_batch_part");
  return CF_OK;
}

// ---------------------------------------------------------------------------
// cf_solve_batch: the whole device sequence of one prepared batch in one call
// (the per-instance loop of gpu/mitm_gpu_mstar_driver.py:296-320 that the
// batch replaces): zero the arena's table prefix and the queue words, then --
// when the batch builds some tables partitioned -- the scatter per radius, the
// range placement and the overflow fix-up, then the table builds, the probes
// and the exact checks.  Every launch goes to `stream` without a host wait, so
// the call can be recorded into a CUDA graph and replayed.
// ---------------------------------------------------------------------------
extern "C" int cf_solve_batch(const CfBatchQueue* q, void* stream) {
  if (!q || !q->mods || !q->misc || q->nmod == 0 || !q->build_tickets || !q->probe_tickets || !q->pairs ||
      !q->pair_mods || !q->results || (q->zero_bytes && !q->arena) ||
      (q->use_part && (!q->place_tickets || !q->ovf || (q->n_scatter && (!q->scatter_tickets || !q->scatter_radius)))) ||
      (q->n_probe && (!q->probe_tickets_r || !q->probe_radius))) {
    cf_set_error("cf_solve_batch: bad arguments%s", "");
    return CF_EBADARG;
  }
  const cudaStream_t st = (cudaStream_t)stream;
  unsigned char* m = (unsigned char*)q->misc;
  // misc: +0 build queue, +8 probe queue, +16 npairs, +20 err, +24 overflow count, +32 scatter queue,
  // +40 range queue
  cudaError_t e = q->zero_bytes ? cudaMemsetAsync(q->arena, 0, q->zero_bytes, st) : cudaSuccess;
  if (e == cudaSuccess) e = cudaMemsetAsync(m, 0, 64, st);
  if (e != cudaSuccess) return cf_cuda_status(e, "cf_solve_batch: zero");
  u32* npairs = (u32*)(m + 16);
  u32* err = (u32*)(m + 20);
  u32* novf = (u32*)(m + 24);
  int rc = CF_OK;
  if (q->use_part) {
    for (u32 i = 0; i < q->n_scatter && rc == CF_OK; ++i) {
      if (i) {
        e = cudaMemsetAsync(m + 32, 0, 8, st);          // the scatter queue head, for the next radius
        if (e != cudaSuccess) return cf_cuda_status(e, "cf_solve_batch: zero");
      }
      rc = cf_batch_part(0, q->mods, q->scatter_tickets[i], q->nmod, m + 32, nullptr, 0, novf, err, q->part_lb,
                         q->scatter_radius[i], 0, stream);
    }
    if (rc == CF_OK)
      rc = cf_batch_part(1, q->mods, q->place_tickets, q->nmod, m + 40, q->ovf, q->ovf_cap, novf, err, q->part_lb, 0,
                         0, stream);
    if (rc == CF_OK)
      rc = cf_batch_part(2, q->mods, nullptr, q->nmod, nullptr, q->ovf, q->ovf_cap, novf, err, q->part_lb, 0, 0,
                         stream);
    if (rc != CF_OK) return rc;
  }
  rc = cf_batch_run(0, q->mods, q->build_tickets, q->nmod, q->ticket, m, q->pairs, (u32*)q->pair_mods, q->max_pairs,
                    npairs, err, nullptr, q->grid, stream);
  if (rc == CF_OK && q->n_probe == 0)
    rc = cf_batch_run(1, q->mods, q->probe_tickets, q->nmod, q->ticket, m + 8, q->pairs, (u32*)q->pair_mods,
                      q->max_pairs, npairs, err, nullptr, q->grid, stream);
  for (u32 i = 0; i < q->n_probe && rc == CF_OK; ++i) {       // one probe launch per radius present
    e = cudaMemsetAsync(m + 8, 0, 8, st);
    if (e != cudaSuccess) return cf_cuda_status(e, "cf_solve_batch: zero");
    const int rr = q->probe_radius[i];
    if (rr < 1 || rr > kBatchMaxR) { cf_set_error("cf_solve_batch: probe radius out of range%s", ""); return CF_EBADARG; }
    rc = batch_launch(1, rr, q->mods, q->probe_tickets_r[i], q->nmod, q->ticket, m + 8, q->pairs, (u32*)q->pair_mods,
                      q->max_pairs, npairs, err, q->grid, st);
  }
  if (rc == CF_OK)
    rc = cf_batch_run(2, q->mods, nullptr, q->nmod, 0, nullptr, q->pairs, (u32*)q->pair_mods, q->max_pairs, npairs,
                      err, q->results, 0, stream);
  return rc;
}

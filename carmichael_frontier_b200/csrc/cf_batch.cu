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
        const CfFuseKey fk = cf_fuse_key(X, x2, tab.bbits);
        const uint4* row = (const uint4*)(tab.fpw + (u64)fk.bucket * 8);
        if (probe_fast(__ldg(row), __ldg(row + 1), fk.f16))
          probe_slow(tab, fk.bucket, fk.f16, fk.f32, rank_base + off, sink);
      }
    }
  }
  return ok;
}

template <int MODE>
__global__ void __launch_bounds__(kBatchBlock)
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
  for (;;) {
    u64 t = 0;
    if (lane == 0) t = atomicAdd(queue, 1ull);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= total) break;
    u32 lo = 0, hi = nmod;                    // the modulus with tstart[lo] <= t < tstart[lo + 1]
    while (hi - lo > 1) {
      const u32 mid = (lo + hi) >> 1;
      if (tstart[mid] <= t) lo = mid; else hi = mid;
    }
    const CfBatchMod& md = mods[lo];
    const bool d_side = (MODE == 0) == (md.swap == 0);
    const u64 n_side = d_side ? md.nD : md.nI;
    const u64 first = (t - tstart[lo]) * (u64)ticket;
    if (first >= n_side) continue;
    const u32 left = (u32)((n_side - first) < ticket ? (n_side - first) : ticket);
    const u64 rank0 = first + (d_side ? 0 : md.i_lo);
    bool good;
    switch (md.r) {
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
  if (grid == 0) {                           // every CTA resident: one wave of persistent CTAs
    static int s_grid[2][64];                 // per mode and device; benign race (same value)
    int dev = 0;
    cudaGetDevice(&dev);
    int* slot = (dev >= 0 && dev < 64) ? &s_grid[mode][dev] : nullptr;
    if (slot && *slot) {
      grid = (u32)*slot;
    } else {
      int sms = 148, per_sm = 0;
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      if (mode == 0) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch<0>, kBatchBlock, 0);
      else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch<1>, kBatchBlock, 0);
      grid = (u32)sms * (u32)(per_sm > 0 ? per_sm : 1);
      if (slot) *slot = (int)grid;
    }
  }
  if (mode == 0)
    k_batch<0><<<grid, kBatchBlock, 0, st>>>((const CfBatchMod*)mods, tstart, nmod, ticket,
                                             (unsigned long long*)queue, (CfPair*)pairs, pmod, max_pairs, npairs, err);
  else
    k_batch<1><<<grid, kBatchBlock, 0, st>>>((const CfBatchMod*)mods, tstart, nmod, ticket,
                                             (unsigned long long*)queue, (CfPair*)pairs, pmod, max_pairs, npairs, err);
  CF_LAUNCH_CHECK("cf_batch_run");
  return CF_OK;
}

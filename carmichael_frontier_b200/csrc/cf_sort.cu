// cf_sort.cu -- stable LSD onesweep radix sort of (u64 key, u64 id) records and
// the sorted-side merge join: the drop-ins for the reference's sort_side
// (gpu/mitm_gpu2.py:101-104, a stable argsort plus two gathers) and
// join_sorted (gpu/mitm_gpu2.py:107-119).
//
// Sort: one histogram kernel reads every key once and counts all digits of all
// passes; each pass is then ONE kernel (onesweep): a CTA takes the next tile
// ticket, ranks its keys stably in shared memory (per warp, item by item over a
// warp-striped tile, lanes of one digit matched through a shared mask, so equal
// digits keep input order), publishes its per-digit counts, resolves its global
// digit offsets by decoupled look-back over the tiles before it (bounded spin),
// and scatters keys, then ids.  The digit is 8 or 9 bits wide (one width for all
// passes of a sort; the autotuner picks it per size class).  Passes whose digit
// is equal for every key are skipped by the host, so keys below M cost at most
// ceil(log2 M / width) passes.
//
// Merge join: every thread takes a run of consecutive sorted I keys, finds the
// first D key >= its first key by binary search and then gallops forward;
// every I row with at least one equal D key is appended as (row, first D
// position, count) to a compact run list (pairs are rare).  The host expands
// runs into pairs in I-row order, which is join_sorted's output order.
#include <type_traits>
#include <vector>
#include "cf_abi_internal.h"

namespace {

using u16 = unsigned short;

constexpr int kSortBlock = 512;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortBlock * kSortItems;  // 4096
constexpr int kWarps = kSortBlock / 32;
constexpr int kMaxPasses = 8;                       // 64 bits at 8 or 9 bits per digit
// Look-back status word of one digit of one tile: flag (aggregate / inclusive) in the top two bits,
// count below.  32-bit words when n < 2^30 (half the status traffic), 64-bit words otherwise.
template <typename SW>
struct Status {
  static constexpr int kBits = (int)sizeof(SW) * 8;
  static constexpr SW kAgg = (SW)1 << (kBits - 2);
  static constexpr SW kInc = (SW)2 << (kBits - 2);
  static constexpr SW kVal = ((SW)1 << (kBits - 2)) - 1;
};
constexpr u32 kSpinLimit = 1u << 24;

// Digit counts of every pass, one read of the keys: hist[p][d] for the digit of
// width db at bit p * db, p < np.  Dynamic shared memory: np << db counters.
__global__ void __launch_bounds__(kSortBlock)
k_sort_hist(const u64* __restrict__ keys, u64 n, u64* __restrict__ hist /*[np][1 << db]*/, int np, int db) {
  extern __shared__ u32 s_h[];
  const int bins = np << db;
  const u64 mask = (1ull << db) - 1;
  for (int i = threadIdx.x; i < bins; i += kSortBlock) s_h[i] = 0;
  __syncthreads();
  for (u64 i = (u64)blockIdx.x * kSortBlock + threadIdx.x; i < n; i += (u64)gridDim.x * kSortBlock) {
    const u64 k = keys[i];
#pragma unroll
    for (int p = 0; p < kMaxPasses; ++p)
      if (p < np) atomicAdd(&s_h[(p << db) + (int)((k >> (p * db)) & mask)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < bins; i += kSortBlock) {
    const u32 v = s_h[i];
    if (v) atomicAdd((unsigned long long*)&hist[i], (unsigned long long)v);
  }
}

// exclusive scan of each pass's histogram of 1 << db bins (one warp per pass)
__global__ void k_sort_hist_scan(const u64* __restrict__ hist, u64* __restrict__ excl, int db) {
  const int p = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int bins = 1 << db;
  u64 run = 0;
  for (int c = 0; c < bins; c += 32) {
    const u64 v = hist[p * bins + c + lane];
    u64 incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const u64 x = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += x;
    }
    excl[p * bins + c + lane] = run + incl - v;
    run += __shfl_sync(0xffffffffu, incl, 31);
  }
}

__device__ __forceinline__ u32 lanemask_lt() {
  u32 m;
  asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Bulk (TMA) copies of a tile into shared memory, completed on an mbarrier.
__device__ __forceinline__ u32 smem_addr(const void* p) { return (u32)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(u64* bar, u32 count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(u64* bar, u32 bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
// global -> shared, `bytes` a multiple of 16, both addresses 16-byte aligned
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, u32 bytes, u64* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}
// Bounded wait for phase `parity` of an mbarrier; false if the limit ran out.
__device__ __forceinline__ bool mbar_wait(u64* bar, u32 parity, u32 limit) {
  const u32 a = smem_addr(bar);
  for (u32 i = 0; i < limit; ++i) {
    u32 done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Global places of the staged elements j = threadIdx.x + k * kSortBlock (staged element j has
// digit s_dj[j]): computed once per tile and used for the keys and again for the ids.
template <typename Dig>
__device__ __forceinline__ void tile_places(const Dig* s_dj, const u64* s_gbase, int tv, u64 (&dst)[kSortItems]) {
  u32 d[kSortItems];
#pragma unroll
  for (int k = 0; k < kSortItems; ++k) {
    const int j = threadIdx.x + k * kSortBlock;
    d[k] = j < tv ? (u32)s_dj[j] : 0u;
  }
#pragma unroll
  for (int k = 0; k < kSortItems; ++k) dst[k] = s_gbase[d[k]] + (u64)(threadIdx.x + k * kSortBlock);
}

// Write a staged tile to its global places, kSortItems elements per thread with their
// shared-memory loads issued together.
__device__ __forceinline__ void write_tile(const u64* s_v, const u64 (&dst)[kSortItems], u64* __restrict__ out,
                                           int tv) {
  u64 v[kSortItems];
#pragma unroll
  for (int k = 0; k < kSortItems; ++k) {
    const int j = threadIdx.x + k * kSortBlock;
    v[k] = s_v[j < tv ? j : 0];
  }
#pragma unroll
  for (int k = 0; k < kSortItems; ++k)
    if (threadIdx.x + k * kSortBlock < tv) out[dst[k]] = v[k];
}

constexpr u32 kMbarLimit = 1u << 22;  // try_wait rounds (each suspends for a while) before giving up

// Dynamic shared memory of one pass with DB-bit digits (R = 2^DB bins):
//   tile keys [4096] u64 | tile ids [4096] u64 | warp digit counters [16][R] Cnt |
//   union { peer masks [16][R] u32 (ranking only),
//           staged digits [4096] Dig, gbase [R] u64, dcnt [R] u32, doff [R] u32 (after ranking) }.
// A warp's count of one digit is at most 256 and the exclusive over warps at most 4096, so the
// 9-bit pass keeps its counters in 16 bits; with the union that keeps it at 112 KB, two CTAs per SM.
template <int DB>
struct PassLayout {
  static constexpr int R = 1 << DB;
  using Cnt = typename std::conditional<DB == 8, u32, u16>::type;
  using Dig = typename std::conditional<DB == 8, unsigned char, u16>::type;
  static constexpr size_t kTile = (size_t)kSortTile * 16;
  static constexpr size_t kWc = (size_t)kWarps * R * sizeof(Cnt);
  static constexpr size_t kMm = (size_t)kWarps * R * 4;
  static constexpr size_t kDj = (size_t)kSortTile * sizeof(Dig);
  static constexpr size_t kAfter = kDj + (size_t)R * 16;
  static constexpr size_t kUnion = kMm > kAfter ? kMm : kAfter;
  static constexpr size_t kSmem = kTile + kWc + kUnion;
  static_assert(R <= kSortBlock, "one thread per digit in the scan and look-back");
  static_assert(kWc % 16 == 0 && kDj % 16 == 0, "aligned sub-arrays");
  static_assert(2 * (kSmem + 1024 + 256) <= 233472, "two CTAs per SM");
};

// One onesweep pass over the DB-bit digit at bit `shift`.  Two CTAs per SM.  BULK:
// the tile's keys and ids are brought into shared memory by two bulk copies at
// the start (every pointer 16-byte aligned), so the id load overlaps the ranking;
// otherwise by plain coalesced loads.  Each item's digit (DB + 1 bits, R = no
// item) rides in the top bits of its local offset.
template <int DB, bool BULK, typename SW>
__global__ void __launch_bounds__(kSortBlock, 2)
k_sort_pass(const u64* __restrict__ kin, const u64* __restrict__ iin, u64* __restrict__ kout,
            u64* __restrict__ iout, u64 n, int shift, const u64* __restrict__ gexcl /*[R]*/,
            SW* __restrict__ status /*[tiles][R]*/, u32* __restrict__ ticket, u32* __restrict__ err) {
  using St = Status<SW>;
  using L = PassLayout<DB>;
  using Cnt = typename L::Cnt;
  using Dig = typename L::Dig;
  constexpr int R = L::R;
  constexpr u32 kNone = (u32)R;
  // predecessor tiles read per look-back round trip: every round reads R status words per tile, so
  // narrow windows win (measured at 2^28 records: 8-bit digits 5 > 4, 6 > 8 > 12; 9-bit 2 > 3, 4 > 8)
  constexpr int kLookWin = DB == 8 ? 5 : 2;
  extern __shared__ __align__(128) unsigned char smem[];
  u64* s_kin = (u64*)smem;                                   // tile keys; later the staging area
  u64* s_iin = s_kin + kSortTile;                            // tile ids
  Cnt* s_wc = (Cnt*)(smem + L::kTile);                       // [kWarps][R] warp digit counts
  unsigned char* s_un = smem + L::kTile + L::kWc;
  u32* s_mm = (u32*)s_un;                                    // [kWarps][R] lanes holding each digit
  Dig* s_dj = (Dig*)s_un;                                    // digit of staged element j
  u64* s_gbase = (u64*)(s_un + L::kDj);  // global position of staged element j of digit d: s_gbase[d] + j
  u32* s_dcnt = (u32*)(s_gbase + R);
  u32* s_doff = s_dcnt + R;
  __shared__ __align__(8) u64 s_bar[2];
  __shared__ u32 s_tile;
  __shared__ u32 s_scan[kWarps];

  if (threadIdx.x == 0) {
    s_tile = atomicAdd(ticket, 1u);
    if (BULK) {
      mbar_init(&s_bar[0], 1);
      mbar_init(&s_bar[1], 1);
      mbar_fence_init();
    }
  }
  __syncthreads();
  const u32 tile = s_tile;
  const u64 base = (u64)tile * kSortTile;
  const u64 left = n - base;
  const int tv = (int)(left < (u64)kSortTile ? left : (u64)kSortTile);
  if (BULK) {
    if (threadIdx.x == 0) {
      const u32 bytes = (u32)(tv & ~1) * 8u;   // whole 16-byte units; an odd last record is loaded below
      mbar_expect_tx(&s_bar[0], bytes);
      if (bytes) bulk_g2s(s_kin, kin + base, bytes, &s_bar[0]);
      mbar_expect_tx(&s_bar[1], bytes);
      if (bytes) bulk_g2s(s_iin, iin + base, bytes, &s_bar[1]);
      if (tv & 1) {
        s_kin[tv - 1] = kin[base + tv - 1];
        s_iin[tv - 1] = iin[base + tv - 1];
      }
    }
  } else {
    for (int j = threadIdx.x; j < tv; j += kSortBlock) {
      s_kin[j] = kin[base + j];
      s_iin[j] = iin[base + j];
    }
  }
  for (int i = threadIdx.x; i < (int)((L::kWc + L::kMm) / 4); i += kSortBlock)   // counters and masks
    ((u32*)(smem + L::kTile))[i] = 0;
  __syncthreads();
  // A tile whose keys never arrived (both bounded waits ran out, practically unreachable) is
  // ranked as empty: it publishes zero counts, so its successors' look-back still ends and
  // every position they compute stays below n, and it writes nothing.  The error word makes
  // the call return CF_ETIMEOUT.
  bool keys_lost = false;
  if (BULK) {
    bool ok = mbar_wait(&s_bar[0], 0, kMbarLimit);
    if (!ok) {
      atomicOr(err, CF_ERR_SPIN_LIMIT);
      ok = mbar_wait(&s_bar[0], 0, kMbarLimit);
    }
    keys_lost = __syncthreads_or(!ok) != 0;
  }
  const int tr = keys_lost ? 0 : tv;          // items ranked and written
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  u64 key[kSortItems];
  u32 loc[kSortItems];                      // local offset (low 16 bits) | digit << 16
  const u32 lt = lanemask_lt();
  Cnt* wc = s_wc + wid * R;
  u32* mm = s_mm + wid * R;
#pragma unroll
  for (int it = 0; it < kSortItems; ++it) {
    const int e = wid * 32 * kSortItems + it * 32 + lane;
    key[it] = e < tr ? s_kin[e] : 0ull;
  }
  // stable rank within the warp, item by item: the lanes of one digit find each other
  // through a shared mask (one atomic OR each), the group's lowest lane takes the
  // group's slice of the warp's digit counter and clears the mask, and the slice's
  // start reaches the group by shuffle
#pragma unroll
  for (int it = 0; it < kSortItems; ++it) {
    const int e = wid * 32 * kSortItems + it * 32 + lane;
    const u32 d = e < tr ? (u32)((key[it] >> shift) & (u64)(R - 1)) : kNone;
    const bool valid = d < kNone;
    if (valid) atomicOr(&mm[d], 1u << lane);
    __syncwarp();
    const u32 peers = valid ? mm[d] : 0u;
    const int leader = valid ? __ffs(peers) - 1 : lane;
    __syncwarp();
    u32 base = 0;
    if (valid && lane == leader) {
      base = wc[d];
      wc[d] = (Cnt)(base + __popc(peers));
      mm[d] = 0u;
    }
    base = __shfl_sync(0xffffffffu, base, leader);
    __syncwarp();
    loc[it] = (d << 16) | (base + __popc(peers & lt));
  }
  __syncthreads();
  if (threadIdx.x < R) {                      // per digit: exclusive over warps, tile total
    const int d = threadIdx.x;
    u32 v[kWarps];
#pragma unroll
    for (int w = 0; w < kWarps; ++w) v[w] = s_wc[w * R + d];
    u32 run = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      s_wc[w * R + d] = (Cnt)run;
      run += v[w];
    }
    s_dcnt[d] = run;
    // flag and count share one 64-bit word and readers read nothing else that this
    // tile writes, so the status store needs no fence before it
    const SW pub = (tile == 0) ? (St::kInc | (SW)run) : (St::kAgg | (SW)run);
    ((volatile SW*)status)[(u64)tile * R + d] = pub;
    u32 incl = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const u32 x = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += x;
    }
    if (lane == 31) s_scan[wid] = incl;
    s_doff[d] = incl - run;
  }
  __syncthreads();
  if (threadIdx.x < R) {
    const int d = threadIdx.x;
    u32 add = 0;
    for (int w = 0; w < wid; ++w) add += s_scan[w];
    s_doff[d] += add;
    u64 excl = 0;
    if (tile > 0) {
      // decoupled look-back, kLookWin predecessors per round trip, bounded.  Tile 0
      // always publishes an inclusive prefix, so the walk ends at tile 0 at the latest.
      int j = (int)tile - 1;
      u32 spins = 0;
      for (;;) {
        SW v[kLookWin];
#pragma unroll
        for (int w = 0; w < kLookWin; ++w)
          v[w] = (j - w >= 0) ? ((volatile const SW*)status)[(u64)(j - w) * R + d] : St::kInc;
        int used = 0;
        bool stop = false, stall = false;
#pragma unroll
        for (int w = 0; w < kLookWin; ++w) {
          if (stop || stall) continue;
          const SW f = v[w] & (SW)~St::kVal;
          if (f == 0) { stall = true; continue; }
          excl += (u64)(v[w] & St::kVal);
          ++used;
          if (f == St::kInc) stop = true;
        }
        if (stop) break;
        j -= used;
        if (used == 0) {                       // predecessor not published yet: back off briefly
          if (++spins > kSpinLimit) { atomicOr(err, CF_ERR_SPIN_LIMIT); break; }
          __nanosleep(64);
        }
      }
      ((volatile SW*)status)[(u64)tile * R + d] = St::kInc | (SW)(excl + s_dcnt[d]);
    }
    s_gbase[d] = gexcl[d] + excl - s_doff[d];   // wraps mod 2^64; j >= s_doff[d] brings it back
  }
  __syncthreads();
  {
    u32 add[kSortItems];
#pragma unroll
    for (int it = 0; it < kSortItems; ++it) {
      const u32 d = loc[it] >> 16;
      add[it] = d < kNone ? s_doff[d] + (u32)wc[d] : 0u;
    }
#pragma unroll
    for (int it = 0; it < kSortItems; ++it) {
      const u32 d = loc[it] >> 16;
      if (d < kNone) {
        const u32 l = (loc[it] & 0xffffu) + add[it];
        loc[it] = l | (d << 16);
        s_kin[l] = key[it];
        s_dj[l] = (Dig)d;
      }
    }
  }
  __syncthreads();
  u64 dst[kSortItems];
  tile_places(s_dj, s_gbase, tr, dst);
  write_tile(s_kin, dst, kout, tr);
  bool ids_lost = false;
  if (BULK) {
    bool ok = mbar_wait(&s_bar[1], 0, kMbarLimit);
    if (!ok) {
      atomicOr(err, CF_ERR_SPIN_LIMIT);
      ok = mbar_wait(&s_bar[1], 0, kMbarLimit);
    }
    ids_lost = __syncthreads_or(!ok) != 0;
  } else {
    __syncthreads();
  }
  if (keys_lost || ids_lost) {
    // nothing more is written; before the CTA gives up its shared memory, wait (bounded) once
    // more for copies still in flight, so a late copy is unlikely to land in a later CTA's tile
    if (keys_lost) mbar_wait(&s_bar[0], 0, kMbarLimit);
    if (ids_lost || keys_lost) mbar_wait(&s_bar[1], 0, kMbarLimit);
    return;
  }
  {
    u64 idv[kSortItems];
#pragma unroll
    for (int it = 0; it < kSortItems; ++it) {
      const int e = wid * 32 * kSortItems + it * 32 + lane;
      idv[it] = (loc[it] >> 16) < kNone ? s_iin[e] : 0ull;
    }
#pragma unroll
    for (int it = 0; it < kSortItems; ++it)
      if ((loc[it] >> 16) < kNone) s_kin[loc[it] & 0xffffu] = idv[it];
  }
  __syncthreads();
  // the 8-bit pass keeps the places in registers across the id wait (1.5% faster); the 9-bit pass
  // reads them again (1% faster there)
  if constexpr (DB != 8) tile_places(s_dj, s_gbase, tr, dst);
  write_tile(s_kin, dst, iout, tr);
}

// ---------------------------------------------------------------------------
// Merge join of two sorted key arrays.
// ---------------------------------------------------------------------------
constexpr int kMergeBlock = 256;
constexpr int kMergeRun = 16;

struct CfRun {
  u64 irow, dlo, cnt;
};

__device__ __forceinline__ u64 lower_bound_u64(const u64* __restrict__ a, u64 lo, u64 hi, u64 key) {
  while (lo < hi) {
    const u64 mid = lo + ((hi - lo) >> 1);
    if (a[mid] < key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__global__ void __launch_bounds__(kMergeBlock)
k_merge_runs(const u64* __restrict__ Dk, u64 nD, const u64* __restrict__ Ik, u64 nI, CfRun* __restrict__ runs,
             u64 max_runs, unsigned long long* __restrict__ nruns, u64* __restrict__ npairs, u32* __restrict__ err) {
  const u64 t = (u64)blockIdx.x * kMergeBlock + threadIdx.x;
  const u64 r0 = t * kMergeRun;
  if (r0 >= nI) return;
  const u64 r1 = (r0 + kMergeRun < nI) ? r0 + kMergeRun : nI;
  u64 pos = lower_bound_u64(Dk, 0, nD, Ik[r0]);
  u64 local_pairs = 0;
  for (u64 r = r0; r < r1; ++r) {
    const u64 key = Ik[r];
    if (pos < nD && Dk[pos] < key) {          // gallop to the first D key >= key
      u64 step = 1, lo = pos + 1, hi = pos + 1;
      while (hi < nD && Dk[hi] < key) { lo = hi + 1; hi = pos + (step <<= 1); }
      if (hi > nD) hi = nD;
      pos = lower_bound_u64(Dk, lo, hi, key);
    }
    u64 q = pos;
    while (q < nD && Dk[q] == key) ++q;
    if (q > pos) {
      const u64 k = atomicAdd(nruns, 1ull);
      if (k < max_runs) {
        CfRun run;
        run.irow = r; run.dlo = pos; run.cnt = q - pos;
        runs[k] = run;
      } else {
        atomicOr(err, CF_ERR_PAIR_OVERFLOW);
      }
      local_pairs += q - pos;
    }
  }
  if (local_pairs) atomicAdd((unsigned long long*)npairs, (unsigned long long)local_pairs);
}

}  // namespace

// Workspace of one sort of n records with np passes of db-bit digits: second
// key/id buffers, histograms, the look-back status words of every pass and the
// tile tickets.
static size_t sort_tmp_bytes(u64 n, int np, int db) {
  const u64 tiles = (n + kSortTile - 1) / kSortTile;
  const u64 bins = (u64)np << db;
  return (size_t)(2 * n * 8) + (size_t)(2 * bins * 8) + (size_t)(tiles * bins * 8) + kMaxPasses * 4 + 64;
}

static int sort_passes(int key_bits, int db) { return (key_bits + db - 1) / db; }

template <int DB, typename SW>
static cudaError_t sort_pass_attrs() {
  cudaError_t e = cudaFuncSetAttribute(k_sort_pass<DB, true, SW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)PassLayout<DB>::kSmem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_sort_pass<DB, false, SW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)PassLayout<DB>::kSmem);
  return e;
}

template <int DB, typename SW>
static void sort_pass_launch(bool bulk, unsigned tiles, cudaStream_t st, const u64* ka, const u64* ia, u64* kb,
                             u64* ib, u64 n, int shift, const u64* excl, SW* status, u32* ticket, u32* errw) {
  if (bulk)
    k_sort_pass<DB, true, SW><<<tiles, kSortBlock, PassLayout<DB>::kSmem, st>>>(ka, ia, kb, ib, n, shift, excl,
                                                                              status, ticket, errw);
  else
    k_sort_pass<DB, false, SW><<<tiles, kSortBlock, PassLayout<DB>::kSmem, st>>>(ka, ia, kb, ib, n, shift, excl,
                                                                               status, ticket, errw);
}

template <typename SW>
static cudaError_t sort_passes_attrs(int db) { return db == 8 ? sort_pass_attrs<8, SW>() : sort_pass_attrs<9, SW>(); }

// The sort behind cf_sort_pairs and cf_sort_pairs_digits: np = ceil(key_bits / db)
// passes of db-bit digits (8 or 9), passes whose digit is constant skipped.
static int sort_pairs(u64* keys, u64* ids, u64 n, int key_bits, int db, void* tmp, size_t tmp_bytes, size_t need,
                      cudaStream_t st) {
  const int np = sort_passes(key_bits, db);
  const int bins = 1 << db;
  const u64 tiles = (n + kSortTile - 1) / kSortTile;
  if (tmp_bytes < need) { cf_set_error("cf_sort_pairs: workspace too small%s", ""); return CF_ENOMEM; }
  unsigned char* w = (unsigned char*)tmp;
  u64* k2 = (u64*)w; w += n * 8;
  u64* i2 = (u64*)w; w += n * 8;
  u64* hist = (u64*)w; w += (size_t)np * bins * 8;
  u64* excl = (u64*)w; w += (size_t)np * bins * 8;
  const bool narrow = n < (1ull << 30);           // 32-bit status words hold every count
  unsigned char* status = w; w += (size_t)np * tiles * bins * 8;   // room for 64-bit words
  u32* tickets = (u32*)w; w += kMaxPasses * 4;
  u32* errw = (u32*)w;
  cudaError_t e = cudaMemsetAsync(hist, 0, (size_t)np * bins * 8, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(status, 0, (size_t)np * tiles * bins * (narrow ? 4 : 8), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(tickets, 0, kMaxPasses * 4 + 4, st);
  if (e != cudaSuccess) return cf_cuda_status(e, "cf_sort_pairs: memset");
  const unsigned hgrid = (unsigned)((n + kSortBlock * 8 - 1) / (kSortBlock * 8));
  k_sort_hist<<<hgrid < 2048 ? hgrid : 2048, kSortBlock, (size_t)(np << db) * 4, st>>>(keys, n, hist, np, db);
  k_sort_hist_scan<<<1, 32 * np, 0, st>>>(hist, excl, db);
  CF_LAUNCH_CHECK("cf_sort_pairs: histogram");
  std::vector<u64> hh((size_t)np * bins);
  e = cudaMemcpyAsync(hh.data(), hist, hh.size() * 8, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cf_cuda_status(e, "cf_sort_pairs: histogram read");
  e = narrow ? sort_passes_attrs<u32>(db) : sort_passes_attrs<u64>(db);
  if (e != cudaSuccess) return cf_cuda_status(e, "cf_sort_pairs: smem attribute");
  u64 *ka = keys, *ia = ids, *kb = k2, *ib = i2;
  int done = 0;
  for (int p = 0; p < np; ++p) {
    bool trivial = false;
    for (int d = 0; d < bins; ++d) if (hh[(size_t)p * bins + d] == n) trivial = true;
    if (trivial) continue;
    // bulk copies read 16-byte units from 16-byte boundaries: every tile starts at
    // a multiple of 4096 records, so aligned source arrays suffice
    const bool bulk = ((((uintptr_t)ka) | ((uintptr_t)ia)) & 15u) == 0;
    const u64 pw = (u64)p * tiles * bins;           // this pass's status words
    const u64* pex = excl + p * bins;
    if (narrow) {
      u32* pst = (u32*)status + pw;
      if (db == 8) sort_pass_launch<8, u32>(bulk, (unsigned)tiles, st, ka, ia, kb, ib, n, 8 * p, pex, pst, tickets + p, errw);
      else sort_pass_launch<9, u32>(bulk, (unsigned)tiles, st, ka, ia, kb, ib, n, 9 * p, pex, pst, tickets + p, errw);
    } else {
      u64* pst = (u64*)status + pw;
      if (db == 8) sort_pass_launch<8, u64>(bulk, (unsigned)tiles, st, ka, ia, kb, ib, n, 8 * p, pex, pst, tickets + p, errw);
      else sort_pass_launch<9, u64>(bulk, (unsigned)tiles, st, ka, ia, kb, ib, n, 9 * p, pex, pst, tickets + p, errw);
    }
    CF_LAUNCH_CHECK("cf_sort_pairs: pass");
    u64* t = ka; ka = kb; kb = t;
    t = ia; ia = ib; ib = t;
    ++done;
  }
  if (done & 1) {      // result sits in the workspace: copy back
    e = cudaMemcpyAsync(keys, ka, n * 8, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ids, ia, n * 8, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return cf_cuda_status(e, "cf_sort_pairs: copy back");
  }
  u32 herr = 0;
  e = cudaMemcpyAsync(&herr, errw, 4, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cf_cuda_status(e, "cf_sort_pairs: error word");
  if (herr & CF_ERR_SPIN_LIMIT) { cf_set_error("cf_sort_pairs: look-back wait exceeded its limit%s", ""); return CF_ETIMEOUT; }
  return CF_OK;
}

static int sort_args_ok(const u64* keys, const u64* ids, u64 n, int key_bits, const void* tmp, const char* who) {
  if (!keys || !ids || !tmp) { cf_set_error("%s: null buffer", who); return CF_EBADARG; }
  if (key_bits < 1 || key_bits > 64) { cf_set_error("%s: key_bits must be 1..64", who); return CF_EBADARG; }
  if (n > (1ull << 40)) { cf_set_error("%s: n too large", who); return CF_EBADARG; }
  return CF_OK;
}

extern "C" size_t cf_sort_tmp_bytes(u64 n) { return sort_tmp_bytes(n, kMaxPasses, 8); }

// Sort (keys, ids) of length n by key, stably, in place (results end in the
// caller's arrays), 8-bit digits.  key_bits: bits of the largest key (1..64);
// passes whose digit is constant are skipped.  Synchronises the stream once (to
// read the digit histogram).
extern "C" int cf_sort_pairs(u64* keys, u64* ids, u64 n, int key_bits, void* tmp, size_t tmp_bytes, void* stream) {
  if (n <= 1) return CF_OK;
  const int rc = sort_args_ok(keys, ids, n, key_bits, tmp, "cf_sort_pairs");
  if (rc != CF_OK) return rc;
  return sort_pairs(keys, ids, n, key_bits, 8, tmp, tmp_bytes, cf_sort_tmp_bytes(n), (cudaStream_t)stream);
}

// Workspace of cf_sort_pairs_digits; 0 for a digit width other than 8 or 9 or
// key_bits outside 1..64.
extern "C" size_t cf_sort_digits_tmp_bytes(u64 n, int key_bits, int digit_bits) {
  if ((digit_bits != 8 && digit_bits != 9) || key_bits < 1 || key_bits > 64) return 0;
  return sort_tmp_bytes(n, sort_passes(key_bits, digit_bits), digit_bits);
}

// cf_sort_pairs with the digit width chosen by the caller (8 or 9 bits):
// ceil(key_bits / digit_bits) passes, constant-digit passes skipped.  Same
// result for every width.
extern "C" int cf_sort_pairs_digits(u64* keys, u64* ids, u64 n, int key_bits, int digit_bits, void* tmp,
                                    size_t tmp_bytes, void* stream) {
  if (digit_bits != 8 && digit_bits != 9) {
    cf_set_error("cf_sort_pairs_digits: digit_bits must be 8 or 9%s", "");
    return CF_EBADARG;
  }
  if (n <= 1) return CF_OK;
  const int rc = sort_args_ok(keys, ids, n, key_bits, tmp, "cf_sort_pairs_digits");
  if (rc != CF_OK) return rc;
  return sort_pairs(keys, ids, n, key_bits, digit_bits, tmp, tmp_bytes,
                    cf_sort_digits_tmp_bytes(n, key_bits, digit_bits), (cudaStream_t)stream);
}

extern "C" size_t cf_merge_run_bytes(void) { return sizeof(CfRun); }

// Equal-key runs between sorted Dk[nD] and sorted Ik[nI]: runs[k] = (I row, first
// D position, count), unordered; *nruns and *npairs (device u64 counters,
// zeroed by the caller) receive the run and pair totals.
extern "C" int cf_merge_join_runs(const u64* Dk, u64 nD, const u64* Ik, u64 nI, void* runs, u64 max_runs,
                                  u64* nruns, u64* npairs, u32* err, void* stream) {
  if (nD == 0 || nI == 0) return CF_OK;
  if (!Dk || !Ik || !nruns || !npairs || !err || (max_runs && !runs)) {
    cf_set_error("cf_merge_join_runs: null buffer%s", "");
    return CF_EBADARG;
  }
  const u64 threads = (nI + kMergeRun - 1) / kMergeRun;
  const u64 grid = (threads + kMergeBlock - 1) / kMergeBlock;
  if (grid > 0x7fffffffull) { cf_set_error("cf_merge_join_runs: n too large%s", ""); return CF_EBADARG; }
  k_merge_runs<<<(unsigned)grid, kMergeBlock, 0, (cudaStream_t)stream>>>(
      Dk, nD, Ik, nI, (CfRun*)runs, max_runs, (unsigned long long*)nruns, npairs, err);
  CF_LAUNCH_CHECK("cf_merge_join_runs");
  return CF_OK;
}

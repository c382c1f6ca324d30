// cf_enum.cuh -- enumeration of r-subsets in lexicographic
// combinatorial-number-system (CNS) rank order, the order of the reference's
// gen_records kernel (gpu/mitm_gpu2.py:40-52), with the running product kept
// in residue form.
//
// A warp owns a contiguous rank range.  It unranks the first rank by binary
// search over the hockey-stick identity (O(R log n) table reads instead of the
// reference's O(n) scan per record), keeps the prefix products
// A[j] = mult * p[i_0] ... p[i_{j-1}], and its lanes take consecutive ranks, so
// a record costs exactly one modular product (A[R-1] * p[i_{R-1}]).
#pragma once
#include "cf_common.cuh"

// C(x, y) from the saturated table (x <= n, y <= R).
__device__ __forceinline__ u64 cf_binom(const u64* __restrict__ binom, int R, int x, int y) {
  return binom[(size_t)x * (R + 1) + y];
}

// Lexicographic CNS unranking of `rank` into idx[0..R-1] (ascending), exactly
// the subset at that rank in gen_records' order.  Requires rank < C(n, R).
template <int R>
__device__ __forceinline__ void cf_unrank_lex(u64 rank, int n, const u64* __restrict__ binom,
                                              int (&idx)[R]) {
  int start = 0;
#pragma unroll
  for (int pos = 0; pos < R - 1; ++pos) {
    const int rem = R - pos - 1;
    // number of subsets whose index at `pos` lies in [start, c) is
    //   cum(c) = C(n-start, rem+1) - C(n-c, rem+1)
    const u64 total = cf_binom(binom, R, n - start, rem + 1);
    const u64 Y = total - rank;               // > 0
    int lo = start, hi = n - 1 - rem;         // answer: largest c with C(n-c, rem+1) >= Y
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (cf_binom(binom, R, n - mid, rem + 1) >= Y) lo = mid; else hi = mid - 1;
    }
    idx[pos] = lo;
    rank -= total - cf_binom(binom, R, n - lo, rem + 1);
    start = lo + 1;
  }
  idx[R - 1] = start + (int)rank;             // last position: one subset per index
}

// Lexicographic rank of the ascending K-subset idx of {0..n-1}; the binomial
// table has R+1 columns (K <= R).
template <int K, int R>
__device__ __forceinline__ u64 cf_rank_lex(const int* idx, int n, const u64* __restrict__ binom) {
  u64 rank = 0;
  int start = 0;
#pragma unroll
  for (int pos = 0; pos < K; ++pos) {
    rank += cf_binom(binom, R, n - start, K - pos) - cf_binom(binom, R, n - idx[pos], K - pos);
    start = idx[pos] + 1;
  }
  return rank;
}

// Unrank a K-subset of {0..n-1} (lexicographic) with a table of R+1 columns.
template <int K, int R>
__device__ __forceinline__ void cf_unrank_lex_k(u64 rank, int n, const u64* __restrict__ binom, int* idx) {
  int start = 0;
#pragma unroll
  for (int pos = 0; pos < K - 1; ++pos) {
    const int rem = K - pos - 1;
    const u64 total = cf_binom(binom, R, n - start, rem + 1);
    const u64 Y = total - rank;
    int lo = start, hi = n - 1 - rem;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (cf_binom(binom, R, n - mid, rem + 1) >= Y) lo = mid; else hi = mid - 1;
    }
    idx[pos] = lo;
    rank -= total - cf_binom(binom, R, n - lo, rem + 1);
    start = lo + 1;
  }
  idx[K - 1] = start + (int)rank;
}

// Colexicographic rank sum_j C(i_j, j+1) (the id of the reference's rank-mode
// dumpers, src/mitm64_idump_stream2.cpp:26-29).
template <int R>
__device__ __forceinline__ u64 cf_colex_rank(const int (&idx)[R], const u64* __restrict__ binom) {
  u64 v = 0;
#pragma unroll
  for (int j = 0; j < R; ++j) v += cf_binom(binom, R, idx[j], j + 1);
  return v;
}

// Arithmetic policies for the walker.
// Fast: primes < 2^31, lazy 32-bit-radix Montgomery (cf_redc32); key = CRT pair.
struct CfArithFast {
  CfMod32 md;
  const u32* p;            // primes as u32 (shared memory), or nullptr to read p64
  const u64* p64 = nullptr; // primes of the pool table (global memory)
  typedef CfElt32 E;
  __device__ __forceinline__ E mul(E a, int i) const { return cf_mul32(a, p ? p[i] : (u32)p64[i], md); }
  __device__ __forceinline__ u64 key(E a) const { return cf_key32(a, md); }
};
// Wide: any prime below 2^64 (reduced mod M on the host), 64-bit Montgomery keys.
struct CfArithWide {
  CfMod md;
  const u64* pk;
  typedef u64 E;
  __device__ __forceinline__ E mul(E a, int i) const { return cf_mul_key(a, pk[i], md); }
  __device__ __forceinline__ u64 key(E a) const { return a; }
};

// Warp-cooperative lexicographic walker: the 32 lanes of a warp produce 32
// CONSECUTIVE ranks per step.  The state is uniform across the warp: the
// current prefix idx[0..R-2] with its product A[R-1] and the next last index
// c.  A step hands lanes f..f+take-1 the current prefix with last indices
// c..c+take-1 and moves to the successor prefix whenever the run of last
// indices ends, so every lane does exactly one modular product per record, the
// warp never diverges, and lane-consecutive records are rank-consecutive
// (coalesced stores).  Unranking happens once per warp range.
template <int R, class Ar>
struct CfWarpWalker {
  int idx[R > 1 ? R - 1 : 1];     // prefix indices (R-1 of them)
  typename Ar::E A[R];            // A[j] = mult * p[idx[0]] ... p[idx[j-1]]
  int c;                          // next last index of the current prefix

  __device__ __forceinline__ void init(u64 rank, int n, const u64* __restrict__ binom, const Ar& ar,
                                       typename Ar::E start) {
    int full[R];
    cf_unrank_lex<R>(rank, n, binom, full);
#pragma unroll
    for (int j = 0; j < R - 1; ++j) idx[j] = full[j];
    c = full[R - 1];
    A[0] = start;
#pragma unroll
    for (int j = 1; j < R; ++j) A[j] = ar.mul(A[j - 1], idx[j - 1]);
  }

  // Move to the successor prefix (R-1 subset of {0..n-2} in lexicographic
  // order); returns false when there is none.  The common case only bumps the
  // last prefix index (one modular product); a deeper carry is rare.
  __device__ __forceinline__ bool next_prefix(int n, const Ar& ar) {
    if constexpr (R == 1) {
      return false;
    } else {
      if (idx[R - 2] < n - 2) {
        idx[R - 2] += 1;
        A[R - 1] = ar.mul(A[R - 2], idx[R - 2]);
        c = idx[R - 2] + 1;
        return true;
      }
      return carry(n, ar);
    }
  }

  __device__ __forceinline__ bool carry(int n, const Ar& ar) {
    if constexpr (R == 1) {
      return false;
    } else {
      int j = R - 3;                    // idx[R-2] is at its maximum n-2
#pragma unroll
      for (int t = R - 3; t >= 0; --t)
        if (t == j && idx[t] == n - R + t) j = t - 1;
      if (j < 0) return false;
#pragma unroll
      for (int t = 0; t < R - 1; ++t) {
        if (t == j) idx[t] += 1;
        else if (t > j) idx[t] = idx[t - 1] + 1;
      }
#pragma unroll
      for (int t = 1; t < R; ++t)
        if (t > j) A[t] = ar.mul(A[t - 1], idx[t - 1]);
      c = idx[R - 2] + 1;
      return true;
    }
  }

  // One warp step: this lane's prefix product and last index for record
  // (current position + lane).  Lanes past the end of the enumeration get
  // last = -1.
  __device__ __forceinline__ void step(int n, const Ar& ar, int lane, typename Ar::E& myA, int& mylast) {
    int dummy[R > 1 ? R - 1 : 1];
    step_idx<false>(n, ar, lane, myA, mylast, dummy);
  }

  // As step(), also copying this lane's prefix indices (for index-word ids).
  template <bool WANT_IDX>
  __device__ __forceinline__ void step_idx(int n, const Ar& ar, int lane, typename Ar::E& myA, int& mylast,
                                           int (&myidx)[R > 1 ? R - 1 : 1]) {
    int f = 0;
    mylast = -1;
    do {
      if (c >= n && !next_prefix(n, ar)) break;
      const int take = min(n - c, 32 - f);
      if ((unsigned)(lane - f) < (unsigned)take) {
        myA = A[R - 1];
        mylast = c + (lane - f);
        if (WANT_IDX) {
#pragma unroll
          for (int j = 0; j < R - 1; ++j) myidx[j] = idx[j];
        }
      }
      f += take;
      c += take;
    } while (f < 32);
  }
};

// ---------------------------------------------------------------------------
// Tail-table walker (fast arithmetic).  A subset of size R is split into a
// prefix of A = R - B indices and a suffix of B indices.  The suffix products
// of all B-subsets sit in a lexicographic table (CfTailEnt, C(n, B) entries,
// L1/L2-resident), and the records of one prefix are exactly the table's tail
// from the first suffix whose smallest index exceeds the prefix's largest.  A
// warp's 32 lanes read 32 consecutive table entries per step (coalesced) and
// do one 64-bit Montgomery product each; the prefix changes once every
// C(n - i_last - 1, B) records, so the per-step bookkeeping is negligible.
// ---------------------------------------------------------------------------
template <int R, int B>
struct CfTailWalker {
  static constexpr int A = R - B;
  int idx[A > 0 ? A : 1];        // prefix indices
  CfElt32 Q[A + 1];              // Q[j] = start * p[idx[0]] ... p[idx[j-1]] (lazy, 32-bit radix)
  u32 cur, tend;                 // position in the tail table and its end (C(n, B) <= 523,776 entries)

  __device__ __forceinline__ void init(u64 rank, int n, const u64* __restrict__ binom, const CfArithFast& ar,
                                       CfElt32 start, u64 tail_n) {
    int full[R];
    cf_unrank_lex<R>(rank, n, binom, full);
#pragma unroll
    for (int j = 0; j < A; ++j) idx[j] = full[j];
    Q[0] = start;
#pragma unroll
    for (int j = 1; j <= A; ++j) Q[j] = ar.mul(Q[j - 1], idx[j - 1]);
    cur = (u32)cf_rank_lex<B, R>(full + A, n, binom);
    tend = (u32)tail_n;
  }

  __device__ __forceinline__ bool next_prefix(int n, const u64* __restrict__ binom, const CfArithFast& ar) {
    if constexpr (A == 0) {
      return false;
    } else {
      const int np = n - B;                       // prefix indices lie in 0..np-1
      if (idx[A - 1] < np - 1) {
        idx[A - 1] += 1;
        Q[A] = ar.mul(Q[A - 1], idx[A - 1]);
      } else {
        int j = A - 2;
#pragma unroll
        for (int t = A - 2; t >= 0; --t)
          if (t == j && idx[t] == np - A + t) j = t - 1;
        if (j < 0) return false;
#pragma unroll
        for (int t = 0; t < A; ++t) {
          if (t == j) idx[t] += 1;
          else if (t > j) idx[t] = idx[t - 1] + 1;
        }
#pragma unroll
        for (int t = 1; t <= A; ++t)
          if (t > j) Q[t] = ar.mul(Q[t - 1], idx[t - 1]);
      }
      cur = tend - (u32)cf_binom(binom, R, n - idx[A - 1] - 1, B);
      return true;
    }
  }

  // This lane's prefix product and tail index for record (position + lane);
  // lanes past the end of the enumeration get j = ~0.
  template <bool WANT_IDX>
  __device__ __forceinline__ void step(int n, const u64* __restrict__ binom, const CfArithFast& ar, int lane,
                                       CfElt32& myQ, u64& myj, int (&myidx)[A > 0 ? A : 1]) {
    if (tend - cur >= 32u) {                      // common case: the whole step lies in one tail
      myQ = Q[A];
      myj = (u64)(cur + (u32)lane);
      cur += 32u;
      if (WANT_IDX) {
#pragma unroll
        for (int j = 0; j < A; ++j) myidx[j] = idx[j];
      }
      return;
    }
    int f = 0;
    myj = ~0ull;
    do {
      if (cur >= tend && !next_prefix(n, binom, ar)) break;
      const u32 avail = tend - cur;
      const int take = avail < (u32)(32 - f) ? (int)avail : 32 - f;
      if ((unsigned)(lane - f) < (unsigned)take) {
        myQ = Q[A];
        myj = (u64)(cur + (u32)(lane - f));
        if (WANT_IDX) {
#pragma unroll
          for (int j = 0; j < A; ++j) myidx[j] = idx[j];
        }
      }
      f += take;
      cur += (u32)take;
    } while (f < 32);
  }
};

// Key of prefix product q times tail entry e: canonical (x mod m) << a | x mod 2^a.
__device__ __forceinline__ u64 cf_tail_key(CfElt32 q, const CfTailEnt& e, const CfMod32& md, u64 minv) {
  const u64 X = cf_redc_mul(q.X, e.X, md.m, minv);   // q.X < 2m, e.X < m: result canonical in [0, m)
  return (X << md.a) | ((q.x2 * (u64)e.x2) & md.mask2);
}

// Product of the subset idx under a policy (used by the pair check).
template <int R, class Ar>
__device__ __forceinline__ u64 cf_subset_key(const int (&idx)[R], const Ar& ar, typename Ar::E start) {
  typename Ar::E a = start;
#pragma unroll
  for (int j = 0; j < R; ++j) a = ar.mul(a, idx[j]);
  return ar.key(a);
}

// Dispatch a templated functor over the supported radii 1..CF_MAX_DISPATCH_R.
#define CF_MAX_DISPATCH_R 10
#define CF_DISPATCH_R(R_RUNTIME, FUNC, ...)                 \
  switch (R_RUNTIME) {                                      \
    case 1: FUNC<1>(__VA_ARGS__); break;                    \
    case 2: FUNC<2>(__VA_ARGS__); break;                    \
    case 3: FUNC<3>(__VA_ARGS__); break;                    \
    case 4: FUNC<4>(__VA_ARGS__); break;                    \
    case 5: FUNC<5>(__VA_ARGS__); break;                    \
    case 6: FUNC<6>(__VA_ARGS__); break;                    \
    case 7: FUNC<7>(__VA_ARGS__); break;                    \
    case 8: FUNC<8>(__VA_ARGS__); break;                    \
    case 9: FUNC<9>(__VA_ARGS__); break;                    \
    case 10: FUNC<10>(__VA_ARGS__); break;                  \
    default: break;                                         \
  }

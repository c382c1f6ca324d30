// cf_enum.cuh -- per-thread enumeration of r-subsets in lexicographic
// combinatorial-number-system (CNS) rank order, the order of the reference's
// gen_records kernel (gpu/mitm_gpu2.py:40-52), with the running product kept
// in residue form.
//
// A thread owns a contiguous rank range.  It unranks the first rank by binary
// search over the hockey-stick identity (O(R log n) table reads instead of the
// reference's O(n) scan), keeps the prefix products A[j] = mult * p[i_0] ...
// p[i_{j-1}], and steps to the lexicographic successor.  The common step only
// moves the last index, so a record costs exactly one modular product
// (A[R-1] * p[i_{R-1}]); a carry at position j costs R-j products.
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
  const u32* p;
  typedef CfElt32 E;
  __device__ __forceinline__ E mul(E a, int i) const { return cf_mul32(a, p[i], md); }
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

// Lexicographic walker over r-subsets of an n-element pool with running products.
template <int R, class Ar>
struct CfLexWalker {
  int idx[R];
  typename Ar::E A[R];   // prefix products; A[0] = mult
  u64 key;               // key of A[R-1] * p[idx[R-1]]

  __device__ __forceinline__ void init(u64 rank, int n, const u64* __restrict__ binom, const Ar& ar,
                                       typename Ar::E start) {
    cf_unrank_lex<R>(rank, n, binom, idx);
    A[0] = start;
#pragma unroll
    for (int j = 1; j < R; ++j) A[j] = ar.mul(A[j - 1], idx[j - 1]);
    key = ar.key(ar.mul(A[R - 1], idx[R - 1]));
  }

  // Advance to the lexicographic successor (the caller guarantees one exists).
  __device__ __forceinline__ void next(int n, const Ar& ar) {
    if (idx[R - 1] < n - 1) {
      idx[R - 1] += 1;
    } else {
      // largest j < R-1 with idx[j] < n - R + j
      int j = R - 2;
#pragma unroll
      for (int t = R - 2; t >= 0; --t)
        if (t == j && idx[t] == n - R + t) j = t - 1;
#pragma unroll
      for (int t = 0; t < R; ++t) {
        if (t == j) idx[t] += 1;
        else if (t > j) idx[t] = idx[t - 1] + 1;
      }
#pragma unroll
      for (int t = 1; t < R; ++t)
        if (t > j) A[t] = ar.mul(A[t - 1], idx[t - 1]);
    }
    key = ar.key(ar.mul(A[R - 1], idx[R - 1]));
  }

  // Index word with `bits` bits per position, position order (gen_records' id,
  // gpu/mitm_gpu2.py:61).
  __device__ __forceinline__ u64 packed(int bits) const {
    u64 id = 0;
#pragma unroll
    for (int j = 0; j < R; ++j) id |= ((u64)idx[j]) << (j * bits);
    return id;
  }
};

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

// cf_check.cuh -- exact check of one candidate (D, I) pair of one modulus
// (shared by the single-modulus and the batched pair-check kernels).
#pragma once
#include "cf_abi_internal.h"
#include "cf_enum.cuh"

// Check one candidate pair (lexicographic ranks) of one modulus.
template <int R>
__device__ __forceinline__ CfPairResult cf_check_one(const u64* __restrict__ poolD, const u64* __restrict__ poolI,
                                     const CfScreen* __restrict__ scr, CfPair pr) {
  const CfPoolHdr* hD = (const CfPoolHdr*)poolD;
  const CfPoolHdr* hI = (const CfPoolHdr*)poolI;
  const int nD = (int)hD->n, nI = (int)hI->n;
  const bool fast = hD->fast32 && hI->fast32;
  CfArithWide wD, wI;
  wD.md = cf_mod_from_hdr(hD);
  wI.md = wD.md;
  const CfMod32 md32 = cf_mod32_from_hdr(hD);
  const u64* bD = poolD + cf_pool_off_binom(nD);
  const u64* bI = poolI + cf_pool_off_binom(nI);
  wD.pk = poolD + cf_pool_off_pkey(nD);
  wI.pk = poolI + cf_pool_off_pkey(nI);
  const u64* pD = poolD + cf_pool_off_prime(nD);
  const u64* pI = poolI + cf_pool_off_prime(nI);
  const double* lD = (const double*)(poolD + cf_pool_off_lg(nD));
  const double* lI = (const double*)(poolI + cf_pool_off_lg(nI));
  CfPairResult out;
  out.flags = 0;
  out.r = R;
  for (int j = 0; j < CF_MAX_R; ++j) { out.d_idx[j] = 0; out.i_idx[j] = 0; }
  int di[R], ii[R];
  cf_unrank_lex<R>(pr.d_id, nD, bD, di);
  cf_unrank_lex<R>(pr.i_id, nI, bI, ii);
  u64 kd, ki;
  if (fast) {
    CfElt32 eD, eI;
    eD.X = hD->X0; eD.x2 = hD->x20;
    eI.X = hI->X0; eI.x2 = hI->x20;
#pragma unroll
    for (int j = 0; j < R; ++j) {
      eD = cf_mul32(eD, (u32)pD[di[j]], md32);
      eI = cf_mul32(eI, (u32)pI[ii[j]], md32);
    }
    kd = cf_key32(eD, md32);
    ki = cf_key32(eI, md32);
  } else {
    kd = cf_subset_key<R>(di, wD, hD->mult_key);
    ki = cf_subset_key<R>(ii, wI, hI->mult_key);
  }
  double lg = scr->lgP0;
#pragma unroll
  for (int j = 0; j < R; ++j) {
    lg += lI[ii[j]] - lD[di[j]];
    out.d_idx[j] = (unsigned short)di[j];
    out.i_idx[j] = (unsigned short)ii[j];
  }
  if (kd == ki) out.flags |= CF_HIT_KEY_EQUAL;
  if (kd == ki && lg <= scr->lgB + scr->eps) {
    out.flags |= CF_HIT_SCREEN;
    // --- distinctness of S = (B0 \ D) u I: D indices are distinct by construction
    //     (strictly increasing), I primes must avoid B0 and each other.
    bool distinct = true;
    for (int j = 0; j < R; ++j) {
      const u64 q = pI[ii[j]];
      for (int x = 0; x < nD; ++x) distinct &= (pD[x] != q);
      for (int y = 0; y < j; ++y) distinct &= (pI[ii[y]] != q);
    }
    if (distinct) out.flags |= CF_HIT_DISJOINT;
    // --- exact size: n = prod(S) in 32-bit limbs against B
    u32 limb[CF_SCREEN_MAX_LIMBS];
    const int L = CF_SCREEN_MAX_LIMBS;
    for (int l = 0; l < L; ++l) limb[l] = 0;
    limb[0] = 1;
    bool over = false;
    int dpos = 0;
    for (int x = 0; x < nD + R; ++x) {
      u64 q;
      if (x < nD) {
        if (dpos < R && di[dpos] == x) { ++dpos; continue; }
        q = pD[x];
      } else {
        q = pI[ii[x - nD]];
      }
      if (q >> 32) { over = true; continue; }
      u64 carry = 0;
      for (int l = 0; l < L; ++l) {
        const u64 v = (u64)limb[l] * q + carry;
        limb[l] = (u32)v;
        carry = v >> 32;
      }
      if (carry) over = true;
    }
    if (!over) {
      int cmp = 0;   // -1 n<B, 0 equal, 1 n>B
      for (int l = L - 1; l >= 0 && cmp == 0; --l) {
        const u32 b = (l < (int)scr->nlimbs) ? scr->limbsB[l] : 0u;
        if (limb[l] != b) cmp = (limb[l] < b) ? -1 : 1;
      }
      if (cmp <= 0) out.flags |= CF_HIT_SIZE_EXACT;
    }
    // --- Korselt: prod(S) == 1 mod (p-1) for every p in S
    bool korselt = true;
    int dp1 = 0;
    for (int x = 0; x < nD + R && korselt; ++x) {
      u64 p;
      if (x < nD) {
        if (dp1 < R && di[dp1] == x) { ++dp1; continue; }
        p = pD[x];
      } else {
        p = pI[ii[x - nD]];
      }
      const u64 mod = p - 1;
      if (mod == 0) { korselt = false; break; }
      u64 prod = 1 % mod;
      int dq = 0;
      for (int y = 0; y < nD + R; ++y) {
        u64 q;
        if (y < nD) {
          if (dq < R && di[dq] == y) { ++dq; continue; }
          q = pD[y];
        } else {
          q = pI[ii[y - nD]];
        }
        prod = (u64)(((unsigned __int128)prod * (q % mod)) % mod);
      }
      korselt = (prod == 1 % mod);
    }
    if (korselt) out.flags |= CF_HIT_KORSELT;
  }
  return out;
}


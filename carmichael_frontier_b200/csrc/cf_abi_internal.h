// cf_abi_internal.h -- status codes and helpers shared by the C-ABI sources.
#pragma once
#include <stdio.h>
#include "cf_common.cuh"

#define CF_ABI_VERSION 1

// Status codes returned by every entry point (0 = ok; negative = error).
#define CF_OK 0
#define CF_EBADARG -1     // argument out of range / inconsistent sizes
#define CF_ENOMEM -2      // caller workspace too small
#define CF_ECUDA -3       // CUDA runtime error (launch or copy)
#define CF_EOVERFLOW -4   // capacity exceeded (partition or pair buffer); retry larger
#define CF_ETIMEOUT -5    // a bounded device wait gave up

void cf_set_error(const char* fmt, const char* detail);

#if defined(__CUDACC__)
#include <cuda_runtime.h>
static inline int cf_cuda_status(cudaError_t e, const char* where) {
  if (e == cudaSuccess) return CF_OK;
  char buf[256];
  snprintf(buf, sizeof buf, "%s: %s", where, cudaGetErrorString(e));
  cf_set_error("%s", buf);
  return CF_ECUDA;
}
#define CF_LAUNCH_CHECK(where)                         \
  do {                                                 \
    cudaError_t _e = cudaGetLastError();               \
    if (_e != cudaSuccess) return cf_cuda_status(_e, where); \
  } while (0)
#endif

// One prepared batch for cf_solve_batch.  The same layout is declared with
// <stdint.h> types in include/cfmitm.h (CfBatchQueue); keep the two in step.
struct CfBatchQueue {
  const void* mods;                    // device CfBatchMod[nmod]
  void* arena;                         // device table areas; the first zero_bytes are zeroed
  u64 zero_bytes;
  void* misc;                          // device, 64 bytes: queue heads, pair count, error word
  const u64* build_tickets;            // device ticket prefix sums [nmod + 1] of the table builds
  const u64* probe_tickets;            // ... of the probes
  const u64* place_tickets;            // partitioned build: range placement tickets
  const u64* const* scatter_tickets;   // host array [n_scatter] of device ticket prefix sums
  const int* scatter_radius;           // host array [n_scatter]: the radius of each scatter launch
  void* ovf;                           // device overflow records of the partitioned build
  void* pairs;                         // device candidate pairs (16 bytes each)
  void* pair_mods;                     // device u32 modulus index of each candidate
  void* results;                       // device check results (cf_pair_result_bytes() each)
  u32 nmod, ticket, grid, max_pairs;
  u32 ovf_cap, n_scatter;
  int use_part, part_lb;
  u32 n_probe, pad0;                   // n_probe > 0: one probe launch per radius instead of probe_tickets
  const u64* const* probe_tickets_r;   // host array [n_probe] of device ticket prefix sums (one radius each)
  const int* probe_radius;             // host array [n_probe]: the radius of each probe launch
};
static_assert(sizeof(CfBatchQueue) == 160, "CfBatchQueue layout");

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

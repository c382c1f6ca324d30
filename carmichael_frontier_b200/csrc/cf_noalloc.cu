// cf_noalloc.cu -- a variant of the radix sort for callers that cannot allocate
// device memory.
//
// cf_sort_pairs needs scratch memory (second key/id buffers, digit histograms,
// look-back words) that its caller normally passes in.  Some callers have no
// way to obtain device memory for that: a host whose device memory is entirely
// owned by another allocator (for example a framework's caching allocator that
// it must not bypass), or a plugin that is not allowed to change the device's
// memory footprint from one call to the next.  cf_sort_pairs_noalloc takes only
// the inputs and outputs (the arrays it sorts in place) and uses a fixed
// scratch area that lives in this library's own device memory: a file-scope
// __device__ array of CF_NOALLOC_SCRATCH_BYTES, which every GPU that loads the
// library holds until the process exits.  It calls no allocation routine.
//
// Limits and rules:
//  * n <= CF_NOALLOC_MAX_RECORDS (131072 records); larger n is rejected.
//  * The first call on a device looks up the array's device address on that
//    device (cudaGetSymbolAddress, with that device current); make that first
//    call before any stream capture on the device.  The address is kept for the
//    life of the process, so it goes stale if the caller resets the device
//    (cudaDeviceReset); the entry point is not for use after a reset.
//  * All calls share the one scratch array and it keeps whatever the last call
//    left there; the parts that must start at zero are cleared on every call.
//    Calls whose device work overlaps (different streams, or different host
//    threads, on one device) race on the scratch and must be serialised by the
//    caller.
#include <mutex>
#include "cf_abi_internal.h"

extern "C" size_t cf_sort_tmp_bytes(u64 n);
extern "C" int cf_sort_pairs(u64* keys, u64* ids, u64 n, int key_bits, void* tmp, size_t tmp_bytes, void* stream);

#define CF_NOALLOC_MAX_RECORDS (1u << 17)
#define CF_NOALLOC_SCRATCH_BYTES (3u << 20)   // >= cf_sort_tmp_bytes(CF_NOALLOC_MAX_RECORDS)
#define CF_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) unsigned char g_noalloc_scratch[CF_NOALLOC_SCRATCH_BYTES];

static std::mutex g_noalloc_mu;
static void* g_noalloc_addr[CF_NOALLOC_MAX_DEVICES];

// Device address of the scratch array on the current device (looked up once per device).
static int noalloc_scratch(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cf_cuda_status(e, "cf_sort_pairs_noalloc: cudaGetDevice");
  if (dev < 0 || dev >= CF_NOALLOC_MAX_DEVICES) {
    cf_set_error("cf_sort_pairs_noalloc: device ordinal beyond the supported 64%s", "");
    return CF_EBADARG;
  }
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cf_cuda_status(e, "cf_sort_pairs_noalloc: cudaGetSymbolAddress");
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return CF_OK;
}

extern "C" u64 cf_sort_pairs_noalloc_max(void) { return CF_NOALLOC_MAX_RECORDS; }

// Same result as cf_sort_pairs (stable sort of (keys, ids)[n] by key, in place)
// with the library's fixed scratch array instead of a caller workspace.
extern "C" int cf_sort_pairs_noalloc(u64* keys, u64* ids, u64 n, int key_bits, void* stream) {
  if (n > CF_NOALLOC_MAX_RECORDS) {
    char buf[160];
    snprintf(buf, sizeof buf, "cf_sort_pairs_noalloc: n = %llu exceeds the fixed scratch limit of %u records",
             (unsigned long long)n, CF_NOALLOC_MAX_RECORDS);
    cf_set_error("%s", buf);
    return CF_EBADARG;
  }
  if (n <= 1) return CF_OK;
  if (cf_sort_tmp_bytes(n) > CF_NOALLOC_SCRATCH_BYTES) {
    cf_set_error("cf_sort_pairs_noalloc: scratch array too small for this n%s", "");
    return CF_ENOMEM;
  }
  void* scratch = nullptr;
  const int rc = noalloc_scratch(&scratch);
  if (rc != CF_OK) return rc;
  // cf_sort_pairs clears the histogram, look-back and ticket words it uses on every call.
  return cf_sort_pairs(keys, ids, n, key_bits, scratch, CF_NOALLOC_SCRATCH_BYTES, stream);
}

// hb_search_noalloc: exact IVF-flat search that allocates nothing.
//
// Some callers cannot allocate device memory while they serve a query: a
// serving process whose device memory is handed out by another allocator (a
// framework's caching allocator, or a fixed pool reserved at start-up) can
// see cudaMalloc fail or fragment that pool mid-request, and cudaFree
// synchronises the whole device, stalling every other stream of a
// latency-bound process.  For them this entry point runs the exact search
// (coarse quantizer, list-major scan, merge) with all of its per-call
// scratch taken from one fixed array compiled into this library:
//
//   g_noalloc_scratch: 32 MiB of device memory, a file-scope static
//   __device__ array.  Every GPU on which the library is loaded holds it
//   until the process exits.
//
// The caller passes device pointers for the queries and the results; the
// index itself is built beforehand with the ordinary calls.  A search whose
// scratch would not fit (queries x nlist coarse distances, the work
// description and the partial top-k slots) is rejected with HB_ERR_INVALID
// and a message giving the bytes needed.
//
// In host code g_noalloc_scratch names a host-side stand-in, not device
// memory, so its device address is looked up once per device, with that
// device current, by cudaGetSymbolAddress on the first call made for an
// index on that device; that first call should therefore come before any
// stream capture.  Every call shares the array and it keeps the previous
// call's contents: the counters the scan needs zeroed are cleared on each
// call, and calls whose GPU work overlaps (two indexes on the same device
// searched from two threads, for instance) race on the array.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "hb_internal.hpp"

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch array on `device`, looked up once.
int scratch_address(int device, void** out) {
  if (device < 0 || device >= kMaxDevices) {
    hb::set_last_error("device ordinal out of range for the fixed scratch");
    return HB_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_addr[device]) {
    int prev = 0;
    cudaGetDevice(&prev);
    cudaError_t e = cudaSetDevice(device);
    void* p = nullptr;
    if (e == cudaSuccess) e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    cudaSetDevice(prev);
    if (e != cudaSuccess || !p) {
      char msg[160];
      std::snprintf(msg, sizeof(msg), "cudaGetSymbolAddress of the fixed scratch failed: %s",
                    cudaGetErrorString(e));
      hb::set_last_error(msg);
      return HB_ERR_CUDA;
    }
    g_scratch_addr[device] = p;
  }
  *out = g_scratch_addr[device];
  return HB_OK;
}

}  // namespace

extern "C" int hb_search_noalloc(hb_index* ix, size_t nq, const float* q, size_t k, float* D, int64_t* I) {
  const int device = hb::index_device(ix);
  if (device < 0) {
    hb::set_last_error("null index handle");
    return HB_ERR_INVALID;
  }
  void* scratch = nullptr;
  const int rc = scratch_address(device, &scratch);
  if (rc != HB_OK) return rc;
  return hb::search_in_scratch(ix, nq, q, k, D, I, scratch, kNoAllocScratchBytes);
}

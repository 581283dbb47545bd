// Device helpers shared by the kernels.
#pragma once
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>

namespace hb {

// 16-byte asynchronous global->shared copy; src_valid = false zero-fills.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool src_valid) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  int sz = src_valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(sz)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Selection key: squared distances are >= 0 (or +inf / NaN), so their IEEE
// bit patterns order like the values; the low word breaks ties.
__device__ __forceinline__ uint64_t make_key(float d, uint32_t tie) {
  return (static_cast<uint64_t>(__float_as_uint(d)) << 32) | tie;
}
__device__ __forceinline__ float key_dist(uint64_t k) { return __uint_as_float(static_cast<uint32_t>(k >> 32)); }
__device__ __forceinline__ uint32_t key_tie(uint64_t k) { return static_cast<uint32_t>(k); }
constexpr uint64_t kEmpty = ~0ull;

// Bitonic sort of n (power of two) keys in shared memory by one warp.
__device__ __forceinline__ void warp_bitonic_sort(uint64_t* s, int n, int lane) {
  for (int size = 2; size <= n; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = lane; i < (n >> 1); i += 32) {
        int lo = 2 * i - (i & (stride - 1));
        int hi = lo + stride;
        bool asc = (lo & size) == 0;
        uint64_t a = s[lo], b = s[hi];
        if ((a > b) == asc) {
          s[lo] = b;
          s[hi] = a;
        }
      }
      __syncwarp();
    }
  }
}

// Bitonic sort of n (power of two) keys in shared memory by the whole block.
__device__ __forceinline__ void block_bitonic_sort(uint64_t* s, int n) {
  for (int size = 2; size <= n; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = threadIdx.x; i < (n >> 1); i += blockDim.x) {
        int lo = 2 * i - (i & (stride - 1));
        int hi = lo + stride;
        bool asc = (lo & size) == 0;
        uint64_t a = s[lo], b = s[hi];
        if ((a > b) == asc) {
          s[lo] = b;
          s[hi] = a;
        }
      }
      __syncthreads();
    }
  }
}

__host__ __device__ __forceinline__ int pow2_ceil(int x) {
  int p = 1;
  while (p < x) p <<= 1;
  return p;
}

}  // namespace hb

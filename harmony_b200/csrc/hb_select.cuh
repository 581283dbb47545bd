// Block-wide selection of the k smallest 64-bit keys: radix selection over
// key bytes (most significant first) until the chosen bucket holds exactly
// the keys still needed, then a bitonic sort of the winners.
#pragma once
#include "hb_device.cuh"

namespace hb {

struct SelectShared {
  int hist[256];
  int bucket;
  int need;
  int count;
  int real;
};

// Radix selection of the kk smallest non-empty keys among key_at(0..m).
// On return s_out[0..kk) holds them (unordered) and the function returns kk.
template <class KeyAt>
__device__ __forceinline__ int block_select(KeyAt key_at, int m, int kk, SelectShared& sh, uint64_t* s_out) {
  const int tid = threadIdx.x;
  uint64_t prefix = 0;
  int shift = 64;
  int need = kk;
  // Narrow the prefix one byte at a time until the chosen bucket holds
  // exactly the keys still needed.
  while (shift > 0) {
    shift -= 8;
    for (int i = tid; i < 256; i += blockDim.x) sh.hist[i] = 0;
    __syncthreads();
    for (int i = tid; i < m; i += blockDim.x) {
      const uint64_t key = key_at(i);
      if (key == kEmpty) continue;
      if (shift == 56 || (key >> (shift + 8)) == (prefix >> (shift + 8)))
        atomicAdd(&sh.hist[(key >> shift) & 255], 1);
    }
    __syncthreads();
    if (tid < 32) {
      // Lane L owns bins [8L, 8L+8).
      int loc[8];
      int sum = 0;
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        loc[b] = sh.hist[tid * 8 + b];
        sum += loc[b];
      }
      int incl = sum;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const int o = __shfl_up_sync(0xffffffffu, incl, off);
        if (tid >= off) incl += o;
      }
      const int excl = incl - sum;
      const unsigned hit = __ballot_sync(0xffffffffu, incl >= need);
      const int lane = __ffs(hit) - 1;
      if (tid == lane) {
        int cum = excl;
        int b = 0;
        for (; b < 8; ++b) {
          if (cum + loc[b] >= need) break;
          cum += loc[b];
        }
        sh.bucket = tid * 8 + b;
        sh.need = need - cum;
        sh.count = loc[b];
      }
    }
    __syncthreads();
    prefix |= static_cast<uint64_t>(sh.bucket) << shift;
    need = sh.need;
    const bool done = sh.count == need;
    __syncthreads();
    if (done) break;
  }
  // Keys whose top (64 - shift) bits are <= the prefix's are the selection.
  if (tid == 0) sh.count = 0;
  __syncthreads();
  const uint64_t lim = prefix >> shift;
  for (int i = tid; i < m; i += blockDim.x) {
    const uint64_t key = key_at(i);
    if (key == kEmpty) continue;
    if ((shift == 64 ? 0 : (key >> shift)) <= lim) {
      const int pos = atomicAdd(&sh.count, 1);
      if (pos < kk) s_out[pos] = key;
    }
  }
  __syncthreads();
  return kk;
}

// Count keys that are not empty.
template <class KeyAt>
__device__ __forceinline__ int block_count_real(KeyAt key_at, int m, SelectShared& sh) {
  if (threadIdx.x == 0) sh.real = 0;
  __syncthreads();
  int c = 0;
  for (int i = threadIdx.x; i < m; i += blockDim.x) c += key_at(i) != kEmpty;
  for (int off = 16; off > 0; off >>= 1) c += __shfl_xor_sync(0xffffffffu, c, off);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(&sh.real, c);
  __syncthreads();
  return sh.real;
}

// Select and sort: s_out gets the min(k, real) smallest keys ascending,
// padded with kEmpty to pow2_ceil(k).
template <class KeyAt>
__device__ __forceinline__ int block_topk_sorted(KeyAt key_at, int m, int k, SelectShared& sh, uint64_t* s_out) {
  const int real = block_count_real(key_at, m, sh);
  const int kk = min(k, real);
  const int n2 = pow2_ceil(max(k, 2));
  for (int i = threadIdx.x; i < n2; i += blockDim.x) s_out[i] = kEmpty;
  __syncthreads();
  if (kk > 0) block_select(key_at, m, kk, sh, s_out);
  block_bitonic_sort(s_out, n2);
  return kk;
}


// The k smallest keys of src[0..m) (sorted, kEmpty-padded to pow2_ceil(k)).
__device__ __forceinline__ int block_topk_keys(const uint64_t* src, int m, int k, uint64_t* s_out) {
  __shared__ SelectShared sh_keys;
  auto key_at = [&](int i) -> uint64_t { return src[i]; };
  return block_topk_sorted(key_at, m, k, sh_keys, s_out);
}

}  // namespace hb

// Block-wide selection of the k smallest 64-bit keys: one pass for the count,
// minimum and maximum of the non-empty keys (the bits above their highest
// differing bit are common to all of them and need no radix pass), then
// radix selection over 8-bit digits from that bit down until the chosen
// bucket holds exactly the keys still needed, then a bitonic sort of the
// winners.  Histogram updates are aggregated per warp over lanes that hit
// the same bin (distances of one row often share their leading digits).
#pragma once
#include "hb_device.cuh"

namespace hb {

struct SelectShared {
  int hist[256];
  int bucket;
  int need;
  int count;
  int real;
  unsigned long long lo;
  unsigned long long hi;
};

// Count, minimum and maximum of the non-empty keys among key_at(0..m);
// returns the count.  Every thread of the block must call it.
template <class KeyAt>
__device__ __forceinline__ int block_key_stats(KeyAt key_at, int m, SelectShared& sh) {
  if (threadIdx.x == 0) {
    sh.real = 0;
    sh.lo = kEmpty;
    sh.hi = 0;
  }
  __syncthreads();
  int c = 0;
  unsigned long long lo = kEmpty, hi = 0;
#pragma unroll 4
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    const uint64_t key = key_at(i);
    if (key == kEmpty) continue;
    ++c;
    lo = key < lo ? key : lo;
    hi = key > hi ? key : hi;
  }
  for (int off = 16; off > 0; off >>= 1) {
    c += __shfl_xor_sync(0xffffffffu, c, off);
    const unsigned long long l2 = __shfl_xor_sync(0xffffffffu, lo, off);
    const unsigned long long h2 = __shfl_xor_sync(0xffffffffu, hi, off);
    lo = l2 < lo ? l2 : lo;
    hi = h2 > hi ? h2 : hi;
  }
  if ((threadIdx.x & 31) == 0 && c) {
    atomicAdd(&sh.real, c);
    atomicMin(&sh.lo, lo);
    atomicMax(&sh.hi, hi);
  }
  __syncthreads();
  return sh.real;
}

// Selection of the kk smallest non-empty keys among key_at(0..m), after
// block_key_stats on the same keys (0 < kk <= count).  On return
// s_out[0..kk) holds them (unordered) and the function returns kk.
template <class KeyAt>
__device__ __forceinline__ int block_select(KeyAt key_at, int m, int kk, SelectShared& sh, uint64_t* s_out) {
  const int tid = threadIdx.x, lane = tid & 31;
  const uint64_t diff = static_cast<uint64_t>(sh.lo ^ sh.hi);
  // Bits [shift, 64) are equal in every non-empty key.
  int shift = diff ? 64 - __clzll(static_cast<long long>(diff)) : 0;
  uint64_t prefix = shift >= 64 ? 0 : (static_cast<uint64_t>(sh.lo) >> shift) << shift;
  int need = kk;
  bool take_all = kk >= sh.real;
  __syncthreads();
  while (!take_all && shift > 0) {
    const int w = shift < 8 ? shift : 8;
    shift -= w;
    const int top = shift + w;  // bits >= top must match the prefix
    const uint64_t want = top >= 64 ? 0 : prefix >> top;
    for (int i = tid; i < 256; i += blockDim.x) sh.hist[i] = 0;
    __syncthreads();
#pragma unroll 2
    for (int base = tid & ~31; base < m; base += blockDim.x) {
      const int i = base + lane;
      bool valid = false;
      unsigned bin = 0;
      if (i < m) {
        const uint64_t key = key_at(i);
        valid = key != kEmpty && (top >= 64 || (key >> top) == want);
        bin = static_cast<unsigned>(key >> shift) & ((1u << w) - 1u);
      }
      const unsigned vmask = __ballot_sync(0xffffffffu, valid);
      if (valid) {
        const unsigned peers = __match_any_sync(vmask, bin);
        if (lane == __ffs(peers) - 1) atomicAdd(&sh.hist[bin], __popc(peers));
      }
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
      const int first = __ffs(hit) - 1;
      if (tid == first) {
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
  // The selection: every non-empty key when all are wanted, else the keys
  // whose bits from `shift` up are <= the prefix's.
  if (tid == 0) sh.count = 0;
  __syncthreads();
  const uint64_t lim = shift >= 64 ? 0 : prefix >> shift;
#pragma unroll 4
  for (int i = tid; i < m; i += blockDim.x) {
    const uint64_t key = key_at(i);
    if (key == kEmpty) continue;
    if (take_all || (key >> shift) <= lim) {
      const int pos = atomicAdd(&sh.count, 1);
      if (pos < kk) s_out[pos] = key;
    }
  }
  __syncthreads();
  return kk;
}

// Select and sort: s_out gets the min(k, real) smallest keys ascending,
// padded with kEmpty to pow2_ceil(k).
template <class KeyAt>
__device__ __forceinline__ int block_topk_sorted(KeyAt key_at, int m, int k, SelectShared& sh, uint64_t* s_out) {
  const int real = block_key_stats(key_at, m, sh);
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

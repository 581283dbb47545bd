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

// Monotone map of a float to uint32 (all signs), and its inverse.
__device__ __forceinline__ uint32_t ordered_bits(float f) {
  const uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ordered_to_float(uint32_t u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// Squared L2 distance of one stored row and one query row (both padded to
// dpad, a multiple of 4, with zeros) with the reference's sequential
// unfused FP32 loop, src/utils.h:480-487: t = q - x, sum += t * t, each
// operation rounded on its own, dimensions in order.  The zero padding adds
// exact zeros.
// The same loop continued from acc over dims [0, n) of x and qrow (n a
// multiple of 4): running it over consecutive pieces of a row in order gives
// the whole row's sum bit for bit.
__device__ __forceinline__ float exact_l2_seq_from(float acc, const float* __restrict__ x,
                                                   const float* __restrict__ qrow, int n) {
#pragma unroll 8
  for (int c = 0; c < n; c += 4) {
    const float4 v = *reinterpret_cast<const float4*>(x + c);
    const float4 w = *reinterpret_cast<const float4*>(qrow + c);
    float t;
    t = __fsub_rn(w.x, v.x);
    acc = __fadd_rn(acc, __fmul_rn(t, t));
    t = __fsub_rn(w.y, v.y);
    acc = __fadd_rn(acc, __fmul_rn(t, t));
    t = __fsub_rn(w.z, v.z);
    acc = __fadd_rn(acc, __fmul_rn(t, t));
    t = __fsub_rn(w.w, v.w);
    acc = __fadd_rn(acc, __fmul_rn(t, t));
  }
  return acc;
}

__device__ __forceinline__ float exact_l2_seq(const float* __restrict__ x, const float* __restrict__ qrow, int dpad) {
  float acc = 0.0f;
#pragma unroll 8
  for (int c = 0; c < dpad; c += 4) {
    const float4 v = *reinterpret_cast<const float4*>(x + c);
    const float4 w = *reinterpret_cast<const float4*>(qrow + c);
    float t;
    t = __fsub_rn(w.x, v.x);
    acc = __fadd_rn(acc, __fmul_rn(t, t));
    t = __fsub_rn(w.y, v.y);
    acc = __fadd_rn(acc, __fmul_rn(t, t));
    t = __fsub_rn(w.z, v.z);
    acc = __fadd_rn(acc, __fmul_rn(t, t));
    t = __fsub_rn(w.w, v.w);
    acc = __fadd_rn(acc, __fmul_rn(t, t));
  }
  return acc;
}

// Columns [c0, c0 + ncol) (ncol <= 64, a multiple of 4) of the rows named by
// the warp's first nv lanes (row r = lane r's `row`, -1: none) of a
// row-major FP32 matrix with ld-float rows, to stage + r * stride: half a warp
// per row, lane L copying floats [4 (L % 16), + 4), two rows per copy
// instruction.  Returns once the copies have landed (a __syncwarp first
// keeps the previous readers ahead of the overwrite).  stride = 68 (64 + 4)
// keeps the per-lane float4 reads of row `lane` conflict-free.
constexpr int kHalfStageStride = 68;
__device__ __forceinline__ void warp_stage_half_rows(const float* __restrict__ base, int row, int ld, int c0,
                                                     int ncol, float* stage, int nv, int lane) {
  __syncwarp();
  const int h = lane >> 4, cl = 4 * (lane & 15);
  for (int r0 = 0; r0 < nv; r0 += 2) {
    const int rr = __shfl_sync(0xffffffffu, row, r0 + h);
    if (r0 + h < nv && rr >= 0 && cl < ncol)
      cp_async16(stage + (r0 + h) * kHalfStageStride + cl, base + static_cast<size_t>(rr) * ld + c0 + cl, true);
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncwarp();
}

// The k-th smallest (1 <= k) of the 256 keys a warp holds, eight per lane
// (v; pad with 0xFFFFFFFF): each lane sorts its keys with Batcher's 19
// compare-exchanges for eight, then k rounds take the smallest head over the
// warp, the lowest lane holding it dropping it.  For small k.
__device__ __forceinline__ uint32_t warp_kth_small8(uint32_t (&v)[8], int k, int lane) {
  auto cx = [&](int a, int b) {
    const uint32_t lo = min(v[a], v[b]), hi = max(v[a], v[b]);
    v[a] = lo;
    v[b] = hi;
  };
  cx(0, 1), cx(2, 3), cx(4, 5), cx(6, 7);
  cx(0, 2), cx(1, 3), cx(4, 6), cx(5, 7);
  cx(1, 2), cx(5, 6);
  cx(0, 4), cx(1, 5), cx(2, 6), cx(3, 7);
  cx(2, 4), cx(3, 5);
  cx(1, 2), cx(3, 4), cx(5, 6);
  uint32_t m = 0;
  for (int r = 0; r < k; ++r) {
    m = v[0];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, o));
    const unsigned who = __ballot_sync(0xffffffffu, v[0] == m);
    if (lane == __ffs(who) - 1) {
#pragma unroll
      for (int i = 0; i < 7; ++i) v[i] = v[i + 1];
      v[7] = 0xFFFFFFFFu;
    }
  }
  return m;
}

// The k-th smallest (k >= 1) of n 32-bit keys get(0 .. n-1), by one warp:
// radix selection over four 8-bit digits with a 256-bin histogram h in
// shared memory.  n >= k.  A digit that the smallest and the largest key
// share (with everything above it) is every key's digit and needs no count:
// keys of one query share their top bits, and counting those digits would
// put every lane's atomic on one bin.
template <class Get>
__device__ uint32_t warp_kth_smallest(Get get, int n, int k, int* h, int lane) {
  // Keys are read eight per lane at a time, the loads issued together.
  constexpr int kB = 8;
  uint32_t lo = 0xFFFFFFFFu, hi = 0u;
  for (int i0 = 0; i0 < n; i0 += 32 * kB) {
    uint32_t v[kB];
#pragma unroll
    for (int u = 0; u < kB; ++u) v[u] = i0 + 32 * u + lane < n ? get(i0 + 32 * u + lane) : 0u;
#pragma unroll
    for (int u = 0; u < kB; ++u)
      if (i0 + 32 * u + lane < n) {
        lo = min(lo, v[u]);
        hi = max(hi, v[u]);
      }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  uint32_t prefix = 0u, pmask = 0u;
  int need = k;  // rank of the wanted key among those matching the prefix
  for (int shift = 24; shift >= 0; shift -= 8) {
    if ((lo >> shift) == (hi >> shift)) {
      prefix |= lo & (255u << shift);
      pmask |= 255u << shift;
      continue;
    }
    for (int i = lane; i < 256; i += 32) h[i] = 0;
    __syncwarp();
    for (int i0 = 0; i0 < n; i0 += 32 * kB) {
      uint32_t v[kB];
#pragma unroll
      for (int u = 0; u < kB; ++u) v[u] = i0 + 32 * u + lane < n ? get(i0 + 32 * u + lane) : 0u;
#pragma unroll
      for (int u = 0; u < kB; ++u)
        if (i0 + 32 * u + lane < n && (v[u] & pmask) == prefix) atomicAdd(&h[(v[u] >> shift) & 255u], 1);
    }
    __syncwarp();
    int loc[8], sum = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      loc[j] = h[8 * lane + j];
      sum += loc[j];
    }
    int incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int x = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += x;
    }
    const int excl = incl - sum;
    const unsigned hit = __ballot_sync(0xffffffffu, excl < need && need <= incl);
    const int src_lane = __ffs(hit) - 1;
    int bin = 0, before = excl;
    if (lane == src_lane) {
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        if (before + loc[j] >= need) {
          bin = 8 * lane + j;
          break;
        }
        before += loc[j];
      }
    }
    bin = __shfl_sync(0xffffffffu, bin, src_lane);
    before = __shfl_sync(0xffffffffu, before, src_lane);
    need -= before;
    prefix |= static_cast<uint32_t>(bin) << shift;
    pmask |= 255u << shift;
    __syncwarp();
  }
  return prefix;
}

__host__ __device__ __forceinline__ int pow2_ceil(int x) {
  int p = 1;
  while (p < x) p <<= 1;
  return p;
}

}  // namespace hb

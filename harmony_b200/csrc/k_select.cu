// Selection and scheduling kernels of the search pipeline.
//
//  * select_rows_kernel -- coarse quantizer: the P smallest (distance,
//    centroid) pairs of each query's row, ascending.  The reference keeps a
//    max-heap of nprobe with strict '<' admission and heap-sorts it
//    (src/IVFScan.hpp:108-138, src/Index.cpp:1440-1448); the selected set is
//    the P smallest distances (ties broken here by the lower centroid id) and
//    centroids at or above FLT_MAX are never admitted.
//  * build-work kernels -- turn the probe table into the list-major work
//    description the persistent scan consumes (which queries probe each
//    list, items per list, output slots per (query, probe)).
//  * merge_kernel -- the k smallest keys over all partial slots of a query
//    (the master's heap merge of worker heaps, src/Index.cpp:1324-1343, done
//    as one selection), decoded to (distance, id).
//  * warmup_tops_kernel -- Index::warmUpSearch (src/Index.cpp:999-1051):
//    k-th smallest distance over the first warm_list_size vectors of the
//    first warm_lists probed lists; FLT_MAX when fewer than k qualify.
//
// All selections are radix selections over 64-bit keys (distance bits, tie)
// followed by a bitonic sort of the k winners in shared memory.
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include "hb_device.cuh"
#include "hb_internal.hpp"
#include "hb_select.cuh"

namespace hb {
namespace {

constexpr int kSelThreads = 256;
constexpr int kMaxSelect = 8192;  // largest k a single selection returns

__global__ void __launch_bounds__(kSelThreads) select_rows_kernel(const float* __restrict__ D, int ncols,
                                                                  int ldD, int k, int32_t* __restrict__ out_idx,
                                                                  float* __restrict__ out_val) {
  extern __shared__ uint64_t s_out[];
  __shared__ SelectShared sh;
  const float* row = D + static_cast<size_t>(blockIdx.x) * ldD;
  auto key_at = [&](int i) -> uint64_t {
    const float v = row[i];
    return v < FLT_MAX ? make_key(v, static_cast<uint32_t>(i)) : kEmpty;
  };
  block_topk_sorted(key_at, ncols, k, sh, s_out);
  for (int j = threadIdx.x; j < k; j += blockDim.x) {
    const uint64_t key = s_out[j];
    const size_t o = static_cast<size_t>(blockIdx.x) * k + j;
    out_idx[o] = key == kEmpty ? -1 : static_cast<int32_t>(key_tie(key));
    if (out_val) out_val[o] = key == kEmpty ? FLT_MAX : key_dist(key);
  }
}

// Row selection for rows of at most 32 * kSelThreads columns and k <= 1024:
// the row is read once into registers (VPT values per thread); a histogram
// of the keys' high words over kBins equal ranges between the row's
// smallest and largest non-empty key finds the bin holding the k-th key;
// the keys in that bin and below (k plus the bin's share) are compacted
// into shared memory and sorted.  The result is the same as
// select_rows_kernel's: the k smallest (value bits, column) keys, ascending.
constexpr int kBins = 1024;
constexpr int kCandCap = 2048;
constexpr int kFlaggedGrid = 296;  // CTAs striding over the rows flagged by the warp kernel

template <int VPT>
__global__ void __launch_bounds__(kSelThreads, 6) select_rows_reg_kernel(const float* __restrict__ D, int nrows,
                                                                      int ncols, int ldD, int kmax,
                                                                      int32_t* __restrict__ out_idx,
                                                                      float* __restrict__ out_val,
                                                                      const int32_t* __restrict__ k_row,
                                                                      const int* __restrict__ only) {
  __shared__ int hist[kBins];
  __shared__ uint64_t s_keys[kCandCap];
  __shared__ SelectShared sh;
  __shared__ unsigned s_lo, s_hi;
  __shared__ int s_real, s_cnt, s_bin, s_cum;
  __shared__ int s_wsum[kSelThreads / 32];
  __shared__ unsigned s_mask;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  // A row per CTA; with `only`, chunks of 32 rows whose flags one warp reads
  // at once, then the flagged ones.
  const int step = only ? 32 : 1;
  for (int r0 = blockIdx.x * step; r0 < nrows; r0 += gridDim.x * step) {
    unsigned mask = 1u;
    if (only) {
      if (wid == 0) {
        const unsigned b = __ballot_sync(0xffffffffu, r0 + lane < nrows && only[r0 + lane] != 0);
        if (lane == 0) s_mask = b;
      }
      __syncthreads();
      mask = s_mask;
      __syncthreads();
    }
    while (mask) {
      const int r = r0 + __ffs(mask) - 1;
      mask &= mask - 1;
      // Row width (rows of width 0 are skipped; the output stride is kmax).
      const int k = k_row ? min(k_row[r], kmax) : kmax;
      if (k <= 0) continue;
      const float* row = D + static_cast<size_t>(r) * ldD;
      // High words of the keys; 0xFFFFFFFF marks empty (a value >= FLT_MAX or
      // NaN has no key; no non-empty value has all-ones bits).
      uint32_t u[VPT];
      unsigned lo = 0xFFFFFFFFu, hi = 0;
      int real = 0;
#pragma unroll
      for (int j = 0; j < VPT; ++j) {
        const int c = tid + j * kSelThreads;
        u[j] = 0xFFFFFFFFu;
        if (c < ncols) {
          const float v = row[c];
          if (v < FLT_MAX) {
            u[j] = __float_as_uint(v);
            lo = min(lo, u[j]);
            hi = max(hi, u[j]);
            ++real;
          }
        }
      }
      if (tid == 0) {
        s_lo = 0xFFFFFFFFu;
        s_hi = 0;
        s_real = 0;
        s_cnt = 0;
      }
      for (int i = tid; i < kBins; i += kSelThreads) hist[i] = 0;
      for (int off = 16; off > 0; off >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, off));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, off));
        real += __shfl_xor_sync(0xffffffffu, real, off);
      }
      __syncthreads();
      if (lane == 0 && real) {
        atomicMin(&s_lo, lo);
        atomicMax(&s_hi, hi);
        atomicAdd(&s_real, real);
      }
      __syncthreads();
      real = s_real;
      lo = s_lo;
      const int kk = min(k, real);
      // Bin of a high word: monotone in the word (float rounding is monotone),
      // below kBins.
      const float scale = static_cast<float>(kBins) / (static_cast<float>(s_hi - lo) + 1.0f);
      auto bin_of = [&](uint32_t x) -> int {
        return min(kBins - 1, static_cast<int>(static_cast<float>(x - lo) * scale));
      };
      // Histogram, then the bin where the count reaches kk.
      if (kk > 0 && kk < real) {
#pragma unroll
        for (int j = 0; j < VPT; ++j)
          if (u[j] != 0xFFFFFFFFu) atomicAdd(&hist[bin_of(u[j])], 1);
      }
      __syncthreads();
      if (kk > 0 && kk < real) {
        constexpr int per = kBins / kSelThreads;
        int loc = 0;
#pragma unroll
        for (int b = 0; b < per; ++b) loc += hist[tid * per + b];
        int incl = loc;
        for (int off = 1; off < 32; off <<= 1) {
          const int o = __shfl_up_sync(0xffffffffu, incl, off);
          if (lane >= off) incl += o;
        }
        if (lane == 31) s_wsum[wid] = incl;
        __syncthreads();
        int base = 0;
        for (int w = 0; w < wid; ++w) base += s_wsum[w];
        int cum = base + incl - loc;
        if (cum < kk && cum + loc >= kk) {
          int b = 0;
          for (; b < per; ++b) {
            cum += hist[tid * per + b];
            if (cum >= kk) break;
          }
          s_bin = tid * per + b;
          s_cum = cum;
        }
      } else if (tid == 0) {
        s_bin = kBins;  // every non-empty key
        s_cum = real;
      }
      __syncthreads();
      const int bstar = s_bin;
      const int ncand = s_cum;
      uint64_t* keys = s_keys;
      int m = 0;
      if (ncand <= kCandCap) {
#pragma unroll
        for (int j = 0; j < VPT; ++j) {
          if (u[j] != 0xFFFFFFFFu && (bstar >= kBins || bin_of(u[j]) <= bstar)) {
            const int pos = atomicAdd(&s_cnt, 1);
            keys[pos] = (static_cast<uint64_t>(u[j]) << 32) | static_cast<uint32_t>(tid + j * kSelThreads);
          }
        }
        m = pow2_ceil(max(ncand, 2));
        __syncthreads();
        for (int i = ncand + tid; i < m; i += kSelThreads) keys[i] = kEmpty;
        __syncthreads();
        block_bitonic_sort(keys, m);
      } else {
        // Many equal high words near the k-th key: the generic selection.
        auto key_at = [&](int i) -> uint64_t {
          const float v = row[i];
          return v < FLT_MAX ? make_key(v, static_cast<uint32_t>(i)) : kEmpty;
        };
        block_topk_sorted(key_at, ncols, k, sh, keys);
      }
      for (int j = tid; j < k; j += kSelThreads) {
        const uint64_t key = j < kk ? keys[j] : kEmpty;
        const size_t o = static_cast<size_t>(r) * kmax + j;
        out_idx[o] = key == kEmpty ? -1 : static_cast<int32_t>(key_tie(key));
        if (out_val) out_val[o] = key == kEmpty ? FLT_MAX : key_dist(key);
      }
      __syncthreads();  // shared state is reused by the next row
    }
  }
}

// The same selection with one warp per row (4 rows per CTA), for k <= 256
// and rows of at most 8192 columns with 16-byte aligned rows: three passes
// over the row from L2 (range; histogram of the keys' high words in a
// per-warp 1024-bin table; ballot compaction of the keys in and under the
// k-th key's bin), then a warp bitonic sort.  A row whose candidates exceed
// kWarpCand is flagged for the CTA kernel.
constexpr int kSelWarps = 4;
constexpr int kWarpCand = 512;

__global__ void __launch_bounds__(kSelWarps * 32) select_rows_warp_kernel(
    const float* __restrict__ D, int nrows, int ncols, int ldD, int kmax, int32_t* __restrict__ out_idx,
    float* __restrict__ out_val, const int32_t* __restrict__ k_row, int* __restrict__ overflow) {
  __shared__ int s_hist[kSelWarps][kBins];
  __shared__ uint64_t s_cand[kSelWarps][kWarpCand];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int r = blockIdx.x * kSelWarps + wib;
  if (r >= nrows) return;
  int* hist = s_hist[wib];
  uint64_t* cand = s_cand[wib];
  const int k = k_row ? min(k_row[r], kmax) : kmax;
  overflow[r] = 0;  // every lane writes the same value
  if (k <= 0) return;
  const float4* row4 = reinterpret_cast<const float4*>(D + static_cast<size_t>(r) * ldD);
  const int n4 = ncols >> 2;
  auto word = [](float v) -> uint32_t { return v < FLT_MAX ? __float_as_uint(v) : 0xFFFFFFFFu; };
  // Range of the finite values.
  unsigned lo = 0xFFFFFFFFu, hi = 0;
#pragma unroll 4
  for (int i = lane; i < n4; i += 32) {
    const float4 v = row4[i];
    const uint32_t u[4] = {word(v.x), word(v.y), word(v.z), word(v.w)};
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (u[j] != 0xFFFFFFFFu) {
        lo = min(lo, u[j]);
        hi = max(hi, u[j]);
      }
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  // Bin of a high word: (x - lo) >> sh clamped to [0, kBins), monotone in x.
  const unsigned span = hi >= lo ? hi - lo : 0u;
  const int sh = max(0, 32 - __clz(static_cast<int>(span | 1u)) - 10);
  auto bin_of = [&](uint32_t x) -> int {
    return x <= lo ? 0 : static_cast<int>(min(static_cast<unsigned>(kBins - 1), (x - lo) >> sh));
  };
  // Histogram of the finite values (and their count).
  for (int i = lane; i < kBins; i += 32) hist[i] = 0;
  __syncwarp();
  int real = 0;
#pragma unroll 4
  for (int i = lane; i < n4; i += 32) {
    const float4 v = row4[i];
    const uint32_t u[4] = {word(v.x), word(v.y), word(v.z), word(v.w)};
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (u[j] != 0xFFFFFFFFu) {
        atomicAdd(&hist[bin_of(u[j])], 1);
        ++real;
      }
  }
  for (int o = 16; o > 0; o >>= 1) real += __shfl_xor_sync(0xffffffffu, real, o);
  __syncwarp();
  const int kk = min(k, real);
  int bstar = kBins, ncand = real;
  if (kk > 0 && kk < real) {
    // Lane L owns bins [32L, 32L + 32).
    int loc = 0;
    for (int b = 0; b < 32; ++b) loc += hist[lane * 32 + b];
    int incl = loc;
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    const int excl = incl - loc;
    const unsigned owner = __ballot_sync(0xffffffffu, excl < kk && incl >= kk);
    const int ol = __ffs(owner) - 1;
    int bb = 0, cum = 0;
    if (lane == ol) {
      cum = excl;
      for (; bb < 32; ++bb) {
        cum += hist[lane * 32 + bb];
        if (cum >= kk) break;
      }
    }
    bstar = __shfl_sync(0xffffffffu, ol * 32 + bb, ol);
    ncand = __shfl_sync(0xffffffffu, cum, ol);
  }
  if (ncand > kWarpCand) {
    overflow[r] = 1;
    return;
  }
  int cnt = 0;
  for (int i = lane; i < ((n4 + 31) & ~31); i += 32) {
    uint32_t u[4] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu};
    if (i < n4) {
      const float4 v = row4[i];
      u[0] = word(v.x), u[1] = word(v.y), u[2] = word(v.z), u[3] = word(v.w);
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const bool take = u[j] != 0xFFFFFFFFu && (bstar >= kBins || bin_of(u[j]) <= bstar);
      const unsigned b = __ballot_sync(0xffffffffu, take);
      if (take) cand[cnt + __popc(b & ((1u << lane) - 1u))] =
          (static_cast<uint64_t>(u[j]) << 32) | static_cast<uint32_t>(4 * i + j);
      cnt += __popc(b);
    }
  }
  const int n2 = pow2_ceil(max(cnt, 2));
  for (int i = cnt + lane; i < n2; i += 32) cand[i] = kEmpty;
  __syncwarp();
  warp_bitonic_sort(cand, n2, lane);
  for (int j = lane; j < k; j += 32) {
    const uint64_t key = j < kk ? cand[j] : kEmpty;
    const size_t o = static_cast<size_t>(r) * kmax + j;
    out_idx[o] = key == kEmpty ? -1 : static_cast<int32_t>(key_tie(key));
    if (out_val) out_val[o] = key == kEmpty ? FLT_MAX : key_dist(key);
  }
}

// The same selection from the chunk minima of coarse_tc (cm[c * nrows + r]
// = the smallest value of columns 16c .. 16c + 15 of row r): the k-th
// smallest chunk minimum T is at least the row's k-th smallest value (those
// k minima are k values of the row), and every value <= T lies in a chunk
// whose minimum is <= T, so the k smallest keys are among the values <= T of
// those chunks -- a little more than k chunks read instead of the row twice.
// A warp per row; rows with fewer than k finite minima or more than
// kWarpCand values <= T are flagged for the CTA kernel.
constexpr int kChunkCols = 16;
constexpr int kChunkMax = 256;  // chunks per row: eight per lane

__global__ void __launch_bounds__(kSelWarps * 32) select_rows_chunk_kernel(
    const float* __restrict__ D, int nrows, int ncols, int ldD, int kmax, int32_t* __restrict__ out_idx,
    float* __restrict__ out_val, const int32_t* __restrict__ k_row, int* __restrict__ overflow,
    const uint32_t* __restrict__ cmins) {
  __shared__ uint64_t s_cand[kSelWarps][kWarpCand];
  __shared__ int s_chk[kSelWarps][kChunkMax];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int r = blockIdx.x * kSelWarps + wib;
  if (r >= nrows) return;
  const int k = k_row ? min(k_row[r], kmax) : kmax;
  const int nch = (ncols + kChunkCols - 1) / kChunkCols;
  overflow[r] = 0;  // every lane writes the same value
  if (k <= 0) return;
  if (k > nch) {
    overflow[r] = 1;
    return;
  }
  uint32_t v[8], w[8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
    w[i] = v[i] = 32 * i + lane < nch ? cmins[static_cast<size_t>(32 * i + lane) * nrows + r] : 0xFFFFFFFFu;
  const uint32_t T = warp_kth_small8(v, k, lane);
  if (T > __float_as_uint(FLT_MAX)) {  // fewer than k finite minima
    overflow[r] = 1;
    return;
  }
  // Chunks with minimum <= T, ascending.
  int nc = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const bool in = 32 * i + lane < nch && w[i] <= T;
    const unsigned b = __ballot_sync(0xffffffffu, in);
    if (in) s_chk[wib][nc + __popc(b & ((1u << lane) - 1u))] = 32 * i + lane;
    nc += __popc(b);
  }
  __syncwarp();
  // Their values <= T: a half-warp per chunk (lane % 16 = column), sixteen
  // chunks' loads in flight at a time.
  const float* row = D + static_cast<size_t>(r) * ldD;
  uint64_t* cand = s_cand[wib];
  const int half = lane >> 4, cl = lane & 15;
  int cnt = 0;
  for (int t0 = 0; t0 < nc; t0 += 16) {
    uint32_t u[8];
    int col[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int t = t0 + 2 * e + half;
      col[e] = t < nc ? s_chk[wib][t] * kChunkCols + cl : ncols;
      const float x = col[e] < ncols ? row[col[e]] : FLT_MAX;
      u[e] = x < FLT_MAX ? __float_as_uint(x) : 0xFFFFFFFFu;
    }
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const bool take = u[e] <= T;
      const unsigned b = __ballot_sync(0xffffffffu, take);
      const int pos = cnt + __popc(b & ((1u << lane) - 1u));
      if (take && pos < kWarpCand) cand[pos] = (static_cast<uint64_t>(u[e]) << 32) | static_cast<uint32_t>(col[e]);
      cnt += __popc(b);
    }
  }
  if (cnt > kWarpCand) {
    overflow[r] = 1;
    return;
  }
  const int n2 = pow2_ceil(max(cnt, 2));
  for (int i = cnt + lane; i < n2; i += 32) cand[i] = kEmpty;
  __syncwarp();
  warp_bitonic_sort(cand, n2, lane);
  for (int j = lane; j < k; j += 32) {
    const uint64_t key = j < cnt ? cand[j] : kEmpty;
    const size_t o = static_cast<size_t>(r) * kmax + j;
    out_idx[o] = key == kEmpty ? -1 : static_cast<int32_t>(key_tie(key));
    if (out_val) out_val[o] = key == kEmpty ? FLT_MAX : key_dist(key);
  }
}

__global__ void __launch_bounds__(kSelThreads) merge_kernel(const uint64_t* __restrict__ part,
                                                            const int64_t* __restrict__ slot_base, int P, int k,
                                                            const int64_t* __restrict__ ids, float* __restrict__ D,
                                                            int64_t* __restrict__ I) {
  extern __shared__ uint64_t s_out[];
  __shared__ SelectShared sh;
  const int q = blockIdx.x;
  const int64_t s0 = slot_base[static_cast<int64_t>(q) * P];
  const int64_t s1 = slot_base[static_cast<int64_t>(q + 1) * P];
  const uint64_t* src = part + s0 * k;
  const int m = static_cast<int>((s1 - s0) * k);
  auto key_at = [&](int i) -> uint64_t { return src[i]; };
  block_topk_sorted(key_at, m, k, sh, s_out);
  for (int j = threadIdx.x; j < k; j += blockDim.x) {
    const uint64_t key = s_out[j];
    const size_t o = static_cast<size_t>(q) * k + j;
    D[o] = key == kEmpty ? FLT_MAX : key_dist(key);
    I[o] = key == kEmpty ? -1 : ids[key_tie(key)];
  }
}

__global__ void __launch_bounds__(kSelThreads) warmup_tops_kernel(const float* __restrict__ q,
                                                                  const int32_t* __restrict__ probes, int P,
                                                                  const float* __restrict__ codes,
                                                                  const int64_t* __restrict__ list_off, int dpad,
                                                                  int k, int wl, int wls, float* __restrict__ tops) {
  extern __shared__ __align__(16) unsigned char wsm[];
  __shared__ SelectShared sh;
  __shared__ int64_t sbeg[64];
  __shared__ int scnt[65];
  const int qi = blockIdx.x;
  float* sq = reinterpret_cast<float*>(wsm);
  float* sd = sq + dpad;
  const int ncap = wl * wls;
  uint64_t* s_out = reinterpret_cast<uint64_t*>(sd + ((ncap + 1) & ~1));
  for (int c = threadIdx.x; c < dpad; c += blockDim.x) sq[c] = q[static_cast<size_t>(qi) * dpad + c];
  if (threadIdx.x == 0) {
    int tot = 0;
    for (int j = 0; j < wl; ++j) {
      const int l = probes[static_cast<size_t>(qi) * P + j];
      int64_t n = 0;
      if (l >= 0) {
        sbeg[j] = list_off[l];
        n = list_off[l + 1] - list_off[l];
      }
      scnt[j] = tot;
      tot += static_cast<int>(n < wls ? n : wls);
    }
    scnt[wl] = tot;
  }
  __syncthreads();
  const int m = scnt[wl];
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    int j = 0;
    while (scnt[j + 1] <= i) ++j;
    const float* x = codes + static_cast<size_t>(sbeg[j] + (i - scnt[j])) * dpad;
    float acc = 0.0f;
    for (int c = 0; c < dpad; c += 4) {
      const float4 v = *reinterpret_cast<const float4*>(x + c);
      float t;
      t = __fsub_rn(sq[c], v.x);
      acc = __fadd_rn(acc, __fmul_rn(t, t));
      t = __fsub_rn(sq[c + 1], v.y);
      acc = __fadd_rn(acc, __fmul_rn(t, t));
      t = __fsub_rn(sq[c + 2], v.z);
      acc = __fadd_rn(acc, __fmul_rn(t, t));
      t = __fsub_rn(sq[c + 3], v.w);
      acc = __fadd_rn(acc, __fmul_rn(t, t));
    }
    sd[i] = acc;
  }
  __syncthreads();
  auto key_at = [&](int i) -> uint64_t {
    const float v = sd[i];
    return v < FLT_MAX ? make_key(v, static_cast<uint32_t>(i)) : kEmpty;
  };
  const int real = block_key_stats(key_at, m, sh);
  if (real < k) {
    if (threadIdx.x == 0) tops[qi] = FLT_MAX;
    return;
  }
  block_select(key_at, m, k, sh, s_out);
  // The k-th smallest is the largest selected key.
  if (threadIdx.x == 0) {
    uint64_t mx = 0;
    for (int i = 0; i < k; ++i) mx = s_out[i] > mx ? s_out[i] : mx;
    tops[qi] = key_dist(mx);
  }
}

// ---------------------------------------------------------------------------
// Work description.

__global__ void count_probes_kernel(const int32_t* __restrict__ probes, int nqp, int P,
                                    const int64_t* __restrict__ list_off, int chunk_rows,
                                    int32_t* __restrict__ list_cnt, int64_t* __restrict__ slot_cnt) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nqp) return;
  const int l = probes[idx];
  int64_t nch = 0;
  if (l >= 0) {
    const int64_t n = list_off[l + 1] - list_off[l];
    if (n > 0) {
      nch = (n + chunk_rows - 1) / chunk_rows;
      atomicAdd(&list_cnt[l], 1);
    }
  }
  if (slot_cnt) slot_cnt[idx] = nch;
}

__global__ void list_items_kernel(const int32_t* __restrict__ list_cnt, const int64_t* __restrict__ list_off,
                                  int nlist, int chunk_rows, int qgroup, int64_t* __restrict__ cnt64,
                                  int64_t* __restrict__ items) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l > nlist) return;
  if (l == nlist) {
    cnt64[l] = 0;
    items[l] = 0;
    return;
  }
  const int64_t n = list_off[l + 1] - list_off[l];
  const int64_t nch = (n + chunk_rows - 1) / chunk_rows;
  const int64_t ng = (list_cnt[l] + qgroup - 1) / qgroup;
  cnt64[l] = list_cnt[l];
  items[l] = nch * ng;
}

// Block-wide exclusive prefix sum of n int64 values given by get(i), each
// thread taking a contiguous run: out[i] for i < n and out[n] = the total.
// Every thread of the block must call it.
constexpr int kWorkThreads = 1024;
constexpr int kSmallWorkPairs = 32768;  // (query, probe) pairs a single CTA builds
constexpr int kSmallWorkLists = 16384;  // lists whose counters fit its shared memory
constexpr int kScanListsOneCta = 65536; // lists whose two exclusive sums one CTA forms

template <class Get>
__device__ void block_exclusive_scan(Get get, int n, int64_t* __restrict__ out, int64_t* s_warp) {
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int per = (n + kWorkThreads - 1) / kWorkThreads;
  const int b = min(n, tid * per), e = min(n, b + per);
  int64_t sum = 0;
  for (int i = b; i < e; ++i) sum += get(i);
  int64_t incl = sum;
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t x = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += x;
  }
  if (lane == 31) s_warp[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    int64_t w = lane < kWorkThreads / 32 ? s_warp[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t x = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += x;
    }
    s_warp[32 + lane] = w;  // inclusive totals of the warps
  }
  __syncthreads();
  int64_t run = incl - sum + (wid > 0 ? s_warp[32 + wid - 1] : 0);
  for (int i = b; i < e; ++i) {
    out[i] = run;
    run += get(i);
  }
  if (tid == kWorkThreads - 1) out[n] = s_warp[32 + kWorkThreads / 32 - 1];
  __syncthreads();
}

// The whole work description of a small batch in one CTA (the multi-kernel
// path's count, prefix sums and scatter, with the counters in shared
// memory): list_cnt, list_qoff, item_off, slot_base and list_q as
// launch_build_work defines them.
__global__ void __launch_bounds__(kWorkThreads) build_work_small_kernel(
    const int32_t* __restrict__ probes, int nqp, int P, const int64_t* __restrict__ list_off, int nlist,
    int chunk_rows, int qgroup, int32_t* __restrict__ list_cnt, int64_t* __restrict__ list_qoff,
    int32_t* __restrict__ list_q, int64_t* __restrict__ item_off, int64_t* __restrict__ slot_base) {
  extern __shared__ int32_t s_work[];  // [nlist] counts, then [nlist] cursors
  __shared__ int64_t s_warp[64];
  int32_t* cnt = s_work;
  int32_t* cur = s_work + nlist;
  for (int l = threadIdx.x; l < nlist; l += blockDim.x) {
    cnt[l] = 0;
    cur[l] = 0;
  }
  __syncthreads();
  auto nch_of = [&](int idx) -> int64_t {
    const int l = probes[idx];
    if (l < 0) return 0;
    const int64_t n = list_off[l + 1] - list_off[l];
    return n > 0 ? (n + chunk_rows - 1) / chunk_rows : 0;
  };
  for (int idx = threadIdx.x; idx < nqp; idx += blockDim.x)
    if (nch_of(idx) > 0) atomicAdd(&cnt[probes[idx]], 1);
  __syncthreads();
  for (int l = threadIdx.x; l < nlist; l += blockDim.x) list_cnt[l] = cnt[l];
  block_exclusive_scan([&](int l) -> int64_t { return cnt[l]; }, nlist, list_qoff, s_warp);
  block_exclusive_scan(
      [&](int l) -> int64_t {
        const int64_t n = list_off[l + 1] - list_off[l];
        return ((n + chunk_rows - 1) / chunk_rows) * ((cnt[l] + qgroup - 1) / qgroup);
      },
      nlist, item_off, s_warp);
  if (slot_base) block_exclusive_scan(nch_of, nqp, slot_base, s_warp);
  for (int idx = threadIdx.x; idx < nqp; idx += blockDim.x) {
    if (nch_of(idx) == 0) continue;
    const int l = probes[idx];
    const int pos = atomicAdd(&cur[l], 1);
    const int q = idx / P, j = idx - q * P;
    list_q[list_qoff[l] + pos] = static_cast<int32_t>((static_cast<uint32_t>(q) << 16) | static_cast<uint32_t>(j));
  }
}

// Per list: queries (list_cnt) and work items (chunks x query groups), and
// their exclusive sums list_qoff and item_off (nlist + 1 each), by one CTA.
__global__ void __launch_bounds__(kWorkThreads) list_scan_kernel(const int32_t* __restrict__ list_cnt,
                                                                 const int64_t* __restrict__ list_off, int nlist,
                                                                 int chunk_rows, int qgroup,
                                                                 int64_t* __restrict__ list_qoff,
                                                                 int64_t* __restrict__ item_off) {
  __shared__ int64_t s_warp[64];
  block_exclusive_scan([&](int l) -> int64_t { return list_cnt[l]; }, nlist, list_qoff, s_warp);
  block_exclusive_scan(
      [&](int l) -> int64_t {
        const int64_t n = list_off[l + 1] - list_off[l];
        return ((n + chunk_rows - 1) / chunk_rows) * ((list_cnt[l] + qgroup - 1) / qgroup);
      },
      nlist, item_off, s_warp);
}

__global__ void scatter_probes_kernel(const int32_t* __restrict__ probes, int nqp, int P,
                                      const int64_t* __restrict__ list_off, const int64_t* __restrict__ list_qoff,
                                      int32_t* __restrict__ cursor, int32_t* __restrict__ list_q) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nqp) return;
  const int l = probes[idx];
  if (l < 0 || list_off[l + 1] == list_off[l]) return;
  const int pos = atomicAdd(&cursor[l], 1);
  const int q = idx / P, j = idx - q * P;
  list_q[list_qoff[l] + pos] = static_cast<int32_t>((static_cast<uint32_t>(q) << 16) | static_cast<uint32_t>(j));
}

// Binary max-heap of (value, id) rows in place, restating the reference's
// heap_replace_top / heap_sort (src/heap.hpp:36-80) 0-based: the new value
// sinks from the root; at each level it goes to the left child when there is
// no right child or the left value is the greater, else to the right child,
// and stops when it is greater than that child.
__device__ __forceinline__ void heap_sink(float* hv, int64_t* hi, int64_t k, float val, int64_t id) {
  int64_t j = 0;
  for (;;) {
    int64_t c = 2 * j + 1;
    if (c >= k) break;
    if (c + 1 < k && !(hv[c] > hv[c + 1])) ++c;
    if (val > hv[c]) break;
    hv[j] = hv[c];
    hi[j] = hi[c];
    j = c;
  }
  hv[j] = val;
  hi[j] = id;
}

// One thread per query: the reference master's merge of the workers' result
// rows (src/Index.cpp:1327-1341): heap of k (FLT_MAX, -1), then for each part
// in order and each of its k entries in order, admit a value strictly below
// the top; finally heap-sort ascending.  The output row is the heap.
__global__ void merge_parts_kernel(const float* __restrict__ Dp, const int64_t* __restrict__ Ip, int nparts,
                                   int64_t nq, int k, float* __restrict__ D, int64_t* __restrict__ I) {
  const int64_t q = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (q >= nq) return;
  float* hv = D + q * k;
  int64_t* hi = I + q * k;
  for (int i = 0; i < k; ++i) {
    hv[i] = FLT_MAX;
    hi[i] = -1;
  }
  for (int p = 0; p < nparts; ++p) {
    const int64_t base = (static_cast<int64_t>(p) * nq + q) * k;
    for (int i = 0; i < k; ++i) {
      const float v = Dp[base + i];
      if (v < hv[0]) heap_sink(hv, hi, k, v, Ip[base + i]);
    }
  }
  for (int64_t i = k - 1; i >= 0; --i) {
    const float v = hv[i];
    const int64_t id = hi[i];
    hv[i] = hv[0];
    hi[i] = hi[0];
    heap_sink(hv, hi, i, v, id);
  }
}

size_t cub_scan_bytes(size_t n) {
  size_t bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, bytes, static_cast<const int64_t*>(nullptr),
                                static_cast<int64_t*>(nullptr), static_cast<int64_t>(n));
  return bytes;
}

void exclusive_sum(const int64_t* in, int64_t* out, size_t n, void* tmp, size_t tmp_bytes, cudaStream_t st) {
  size_t bytes = tmp_bytes;
  HB_CUDA(cub::DeviceScan::ExclusiveSum(tmp, bytes, in, out, static_cast<int64_t>(n), st));
}

}  // namespace

void launch_select_rows(const float* D, int nrows, int ncols, int ldD, int k, int32_t* out_idx, float* out_val,
                        cudaStream_t st, const int32_t* k_row, int* row_flags, const uint32_t* cmins) {
  if (nrows <= 0 || k <= 0) return;
  const int* only = nullptr;
  const int nch = (ncols + kChunkCols - 1) / kChunkCols;
  if (row_flags && cmins && nch <= kChunkMax && 4 * k <= nch) {
    // Chunk minima given and k small against the chunk count (else T would
    // sit near the largest minima): a warp per row reads the chunks that can
    // hold the k smallest; rows it flags go through the CTA kernel below.
    select_rows_chunk_kernel<<<(nrows + kSelWarps - 1) / kSelWarps, kSelWarps * 32, 0, st>>>(
        D, nrows, ncols, ldD, k, out_idx, out_val, k_row, row_flags, cmins);
    HB_CUDA(cudaGetLastError());
    only = row_flags;
  } else if (row_flags && k <= 256 && ncols <= 8192 && ncols % 4 == 0 && ldD % 4 == 0) {
    // Warp per row; rows it flags go through the CTA kernel below.
    select_rows_warp_kernel<<<(nrows + kSelWarps - 1) / kSelWarps, kSelWarps * 32, 0, st>>>(
        D, nrows, ncols, ldD, k, out_idx, out_val, k_row, row_flags);
    HB_CUDA(cudaGetLastError());
    only = row_flags;
  }
  HB_CHECK(k <= kMaxSelect, HB_ERR_INVALID, "nprobe above 8192 is not supported");
  HB_CHECK(!k_row || (k <= 1024 && ncols <= 32 * kSelThreads), HB_ERR_INVALID,
           "per-row widths need k <= 1024 and at most 8192 columns");
  if (k <= 1024 && ncols <= 32 * kSelThreads) {
    const int vpt = (ncols + kSelThreads - 1) / kSelThreads;
    // Behind the warp kernel only its flagged rows (rare) are left: a small
    // grid strides over the flags instead of a CTA per row.
    const int g = only ? std::min((nrows + 31) / 32, kFlaggedGrid) : nrows;
    if (vpt <= 4)
      select_rows_reg_kernel<4><<<g, kSelThreads, 0, st>>>(D, nrows, ncols, ldD, k, out_idx, out_val, k_row, only);
    else if (vpt <= 8)
      select_rows_reg_kernel<8><<<g, kSelThreads, 0, st>>>(D, nrows, ncols, ldD, k, out_idx, out_val, k_row, only);
    else if (vpt <= 16)
      select_rows_reg_kernel<16><<<g, kSelThreads, 0, st>>>(D, nrows, ncols, ldD, k, out_idx, out_val, k_row, only);
    else
      select_rows_reg_kernel<32><<<g, kSelThreads, 0, st>>>(D, nrows, ncols, ldD, k, out_idx, out_val, k_row, only);
    HB_CUDA(cudaGetLastError());
    return;
  }
  const size_t smem = static_cast<size_t>(pow2_ceil(k < 2 ? 2 : k)) * 8;
  HB_CUDA(cudaFuncSetAttribute(select_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(smem)));
  select_rows_kernel<<<nrows, kSelThreads, smem, st>>>(D, ncols, ldD, k, out_idx, out_val);
  HB_CUDA(cudaGetLastError());
}

void launch_merge_parts(const float* Dp, const int64_t* Ip, int nparts, int64_t nq, int k, float* D, int64_t* I,
                        cudaStream_t st) {
  if (nq <= 0) return;
  merge_parts_kernel<<<static_cast<unsigned>((nq + 127) / 128), 128, 0, st>>>(Dp, Ip, nparts, nq, k, D, I);
  HB_CUDA(cudaGetLastError());
}

size_t build_work_tmp_bytes(int nq, int P, int nlist) {
  const size_t n1 = static_cast<size_t>(nlist) + 1;
  const size_t n2 = static_cast<size_t>(nq) * P + 1;
  size_t cub_bytes = std::max(cub_scan_bytes(n1), cub_scan_bytes(n2));
  cub_bytes = (cub_bytes + 255) / 256 * 256;
  // cub scratch + cnt64 + items64 + slot_cnt64
  return cub_bytes + (2 * n1 + n2) * sizeof(int64_t) + 256;
}

int launch_build_work(const int32_t* probes, int nq, int P, const int64_t* list_off, int nlist, int chunk_rows,
                       int qgroup, int32_t* list_cnt, int64_t* list_qoff, int32_t* list_cursor, int32_t* list_q,
                       int64_t* item_off, int64_t* slot_base, void* scan_tmp, size_t scan_tmp_bytes,
                       cudaStream_t st) {
  const size_t n1 = static_cast<size_t>(nlist) + 1;
  const size_t n2 = static_cast<size_t>(nq) * P + 1;
  size_t cub_bytes = std::max(cub_scan_bytes(n1), cub_scan_bytes(n2));
  cub_bytes = (cub_bytes + 255) / 256 * 256;
  HB_CHECK(scan_tmp_bytes >= cub_bytes + (2 * n1 + n2) * sizeof(int64_t), HB_ERR_INVALID,
           "work scratch too small");
  unsigned char* base = static_cast<unsigned char*>(scan_tmp);
  void* cub_tmp = base;
  int64_t* cnt64 = reinterpret_cast<int64_t*>(base + cub_bytes);
  int64_t* items64 = cnt64 + n1;
  int64_t* slot_cnt = items64 + n1;
  const int nqp = nq * P;
  if (nqp <= kSmallWorkPairs && nlist <= kSmallWorkLists) {
    // Small batch: one CTA, one launch.
    const size_t smem = static_cast<size_t>(2) * nlist * sizeof(int32_t);
    HB_CUDA(cudaFuncSetAttribute(build_work_small_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)));
    build_work_small_kernel<<<1, kWorkThreads, smem, st>>>(probes, nqp, P, list_off, nlist, chunk_rows, qgroup,
                                                           list_cnt, list_qoff, list_q, item_off, slot_base);
    HB_CUDA(cudaGetLastError());
    return 1;
  }
  HB_CUDA(cudaMemsetAsync(list_cnt, 0, sizeof(int32_t) * nlist, st));
  HB_CUDA(cudaMemsetAsync(list_cursor, 0, sizeof(int32_t) * nlist, st));
  if (slot_base) HB_CUDA(cudaMemsetAsync(slot_cnt + nqp, 0, sizeof(int64_t), st));
  const int tb = 256;
  count_probes_kernel<<<(nqp + tb - 1) / tb, tb, 0, st>>>(probes, nqp, P, list_off, chunk_rows, list_cnt,
                                                          slot_base ? slot_cnt : nullptr);
  if (nlist <= kScanListsOneCta) {
    // One CTA scans both per-list counts (a few thousand lists).
    list_scan_kernel<<<1, kWorkThreads, 0, st>>>(list_cnt, list_off, nlist, chunk_rows, qgroup, list_qoff, item_off);
  } else {
    list_items_kernel<<<(nlist + 1 + tb - 1) / tb, tb, 0, st>>>(list_cnt, list_off, nlist, chunk_rows, qgroup, cnt64,
                                                                items64);
    HB_CUDA(cudaGetLastError());
    exclusive_sum(cnt64, list_qoff, n1, cub_tmp, cub_bytes, st);
    exclusive_sum(items64, item_off, n1, cub_tmp, cub_bytes, st);
  }
  HB_CUDA(cudaGetLastError());
  // The per-(query, probe) output slots: only the exact scan's partial
  // results use them.
  if (slot_base) exclusive_sum(slot_cnt, slot_base, n2, cub_tmp, cub_bytes, st);
  scatter_probes_kernel<<<(nqp + tb - 1) / tb, tb, 0, st>>>(probes, nqp, P, list_off, list_qoff, list_cursor,
                                                            list_q);
  HB_CUDA(cudaGetLastError());
  return 3;  // count, the per-list sums, scatter (the CUB scans are library kernels)
}

void launch_merge(const uint64_t* part, const int64_t* slot_base, int nq, int P, int k, const int64_t* ids,
                  float* D, int64_t* I, cudaStream_t st) {
  if (nq <= 0) return;
  HB_CHECK(k <= kMaxSelect, HB_ERR_INVALID, "k above 8192 is not supported");
  const size_t smem = static_cast<size_t>(pow2_ceil(k < 2 ? 2 : k)) * 8;
  HB_CUDA(cudaFuncSetAttribute(merge_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  merge_kernel<<<nq, kSelThreads, smem, st>>>(part, slot_base, P, k, ids, D, I);
  HB_CUDA(cudaGetLastError());
}

void launch_warmup_tops(const float* q, int nq, const int32_t* probes, int P, const float* codes,
                        const int64_t* list_off, int dpad, int k, int warm_lists, int warm_list_size, float* tops,
                        cudaStream_t st) {
  if (nq <= 0) return;
  const int wl = warm_lists < P ? warm_lists : P;
  HB_CHECK(wl <= 64, HB_ERR_INVALID, "warm-up over more than 64 lists is not supported");
  const int ncap = wl * warm_list_size;
  HB_CHECK(ncap <= 16384, HB_ERR_INVALID, "warm-up candidate count above 16384 is not supported");
  HB_CHECK(k <= kMaxSelect, HB_ERR_INVALID, "k above 8192 is not supported");
  const size_t smem = static_cast<size_t>(dpad) * 4 + static_cast<size_t>((ncap + 1) & ~1) * 4 +
                      static_cast<size_t>(k) * 8 + 16;
  HB_CUDA(cudaFuncSetAttribute(warmup_tops_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(smem)));
  warmup_tops_kernel<<<nq, kSelThreads, smem, st>>>(q, probes, P, codes, list_off, dpad, k, wl, warm_list_size,
                                                    tops);
  HB_CUDA(cudaGetLastError());
}

}  // namespace hb

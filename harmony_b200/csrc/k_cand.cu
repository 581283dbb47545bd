// BF16 tensor-core list scan through a candidate matrix, for the searches the
// shared-memory heap scan (k_tc.cu) does not hold: vectors wider than 128
// dimensions and more than 64 candidates per query.
//
//  1. gather_queries_kernel writes, for every (list, query probing it) entry
//     of the list-major work description, the query in BF16 (K = kpad, zero
//     padded): one row per entry, so the queries of one work item are 128
//     consecutive rows and reach the tensor cores by plain TMA tiles.
//  2. cand_scan_kernel: persistent, one CTA per SM, 192 threads (4 epilogue
//     warps, a TMA warp, an MMA warp).  Work items are (list, chunk of rows,
//     group of <= 128 queries); the search uses one 128-row tile per item,
//     so the items spread evenly over the CTAs.  For each 128-row tile of the chunk the TMA
//     warp streams 64-column K blocks of both operands (queries: A, 128 x 64;
//     rows: B, 128 x 64; 128-byte swizzle) into a ring of 32 KB stages, the
//     MMA warp issues tcgen05.mma M128 x N128 x K16 into one of four TMEM
//     accumulators, and the epilogue (thread = query, TMEM lane) writes
//     v = ||x||^2 - 2 q~.x~ of the tile's rows into the query's candidate
//     row: the concatenation over its probes, in probe order, of one segment
//     per probed list (the list's length rounded up to 4; +inf past the end).
//  3. cand_select_kernel: one CTA per query selects the R smallest keys
//     (v, position) of its candidate row (block radix selection over the row
//     staged in shared memory; unique keys, so the choice is deterministic)
//     and maps each position back to its stored row.
//  4. cand_exact_kernel: one CTA per query recomputes the R distances with
//     the reference's sequential unfused FP32 loop and returns the k best
//     (distance, row) -- the same rule as the heap scan's rerank, so whenever
//     the true k nearest are among the R candidates the result equals the
//     exact scan's.
// Every mbarrier wait is bounded; on a timeout the kernel records an error
// code, the roles stop, copies and MMAs in flight are waited for and TMEM is
// freed.
#include <cudaTypedefs.h>
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>

#include <algorithm>

#include <cub/cub.cuh>

#include "hb_device.cuh"
#include "hb_internal.hpp"
#include "hb_select.cuh"
#include "hb_sm100.cuh"

namespace hb {
namespace {

using namespace sm100;

constexpr int kT = 128;                    // rows per tile = queries per group
constexpr int kStg = 6;                    // ring stages
constexpr int kThreads = 192;              // 4 epilogue warps, TMA warp, MMA warp
constexpr uint32_t kBlk = kT * 128;        // one 128-row x 64-column BF16 block (16 KB)
constexpr uint32_t kStageBytes = 2 * kBlk;  // A block + B block
constexpr int kAccN = 4;                    // TMEM accumulators of 128 columns (all 512)
constexpr int kSelectThreads = 256;
constexpr int kBins = 2048;                 // histogram bins of the candidate selection
constexpr int kSelUnroll = 4;               // 32-value runs a warp loads at once
constexpr int kExactThreads = 256;
constexpr int kExChunk = 32;                // dimensions per staged chunk of the exact re-rank
constexpr int kExStride = kExChunk + 1;     // odd row stride: column reads hit distinct banks

struct CandShared {
  uint64_t full[kStg];
  uint64_t empty[kStg];
  uint64_t accf[kAccN];
  uint64_t acce[kAccN];
  uint64_t drain;
  uint32_t tmem;
};

struct CandItem {
  int list, chunk, group, qcnt, ntiles;
  int64_t row0;   // first stored row of the chunk
  int64_t tile0;  // its first 128-row norm tile
  int64_t qrow0;  // first query row of the group in the gathered matrix
};

__device__ __forceinline__ CandItem cand_item(const CandArgs& a, int64_t item) {
  int lo = 0, hi = a.nlist;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (a.item_off[mid] <= item) lo = mid; else hi = mid;
  }
  CandItem d;
  const int l = lo;
  const int64_t local = item - a.item_off[l];
  const int ng = (a.list_cnt[l] + kT - 1) / kT;
  d.list = l;
  d.chunk = static_cast<int>(local / ng);
  d.group = static_cast<int>(local % ng);
  d.qcnt = min(kT, a.list_cnt[l] - d.group * kT);
  const int64_t r0 = a.list_off[l] + static_cast<int64_t>(d.chunk) * a.chunk_rows;
  const int64_t r1 = min(a.list_off[l + 1], r0 + static_cast<int64_t>(a.chunk_rows));
  d.row0 = r0;
  d.ntiles = static_cast<int>((r1 - r0 + kT - 1) / kT);
  d.tile0 = a.tile_off[l] + static_cast<int64_t>(d.chunk) * (a.chunk_rows / kT);
  d.qrow0 = a.list_qoff[l] + static_cast<int64_t>(d.group) * kT;
  return d;
}

// FP8 = false: BF16 operands, 64-element K blocks, kind::f16.  FP8 = true:
// E4M3 operands scaled per query and per list (x ~ s_l * code, q ~ s_q *
// code), 128-element K blocks (the same 128-byte swizzled rows), kind::f8f6f4;
// the epilogue multiplies the accumulator by s_q * s_l.
template <bool FP8>
__global__ void __launch_bounds__(kThreads, 1)
    cand_scan_kernel(const __grid_constant__ CUtensorMap tmap_q, const __grid_constant__ CUtensorMap tmap_x,
                     CandArgs a) {
  extern __shared__ uint8_t smem_raw[];
  __shared__ CandShared sh;
  uint8_t* ring = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  constexpr int kEl = FP8 ? 128 : 64;  // elements per 128-byte K block
  const int nkb = a.kpad / kEl;
  const int64_t total = a.item_off[a.nlist];

  if (warp == 5) tmem_alloc(&sh.tmem, kAccN * kT);
  if (tid == 0) {
    for (int s = 0; s < kStg; ++s) {
      mbar_init(&sh.full[s], 1);
      mbar_init(&sh.empty[s], 1);
    }
    for (int b = 0; b < kAccN; ++b) {
      mbar_init(&sh.accf[b], 1);
      mbar_init(&sh.acce[b], 128);
    }
    mbar_init(&sh.drain, 1);
    fence_barrier_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sh.tmem;

  if (warp == 4) {
    if (lane == 0) {
      prefetch_tmap(&tmap_q);
      prefetch_tmap(&tmap_x);
      int64_t it = 0;
      bool ok = true;
      for (int64_t item = blockIdx.x; ok && item < total; item += gridDim.x) {
        const CandItem d = cand_item(a, item);
        for (int t = 0; ok && t < d.ntiles; ++t) {
          for (int kb = 0; kb < nkb; ++kb, ++it) {
            const int s = static_cast<int>(it % kStg);
            if (!mbar_wait(&sh.empty[s], static_cast<uint32_t>((it / kStg) & 1) ^ 1u, a.err, 31)) {
              ok = false;
              break;
            }
            uint8_t* st = ring + static_cast<size_t>(s) * kStageBytes;
            mbar_arrive_expect_tx(&sh.full[s], kStageBytes);
            tma_load_2d(st, &tmap_q, kb * kEl, static_cast<int>(d.qrow0), &sh.full[s]);
            tma_load_2d(st + kBlk, &tmap_x, kb * kEl, static_cast<int>(d.row0 + static_cast<int64_t>(t) * kT),
                        &sh.full[s]);
          }
        }
      }
      // Every issued copy lands before the CTA may exit: wait for the last
      // phase issued on each stage (already complete on the normal path).
      for (int64_t j = it - 1; j >= 0 && j >= it - kStg; --j)
        mbar_wait(&sh.full[j % kStg], static_cast<uint32_t>((j / kStg) & 1), nullptr, 0, 200000000LL);
    }
  } else if (warp == 5) {
    if (lane == 0) {
      const uint32_t idesc = FP8 ? idesc_e4m3_f32(kT, kT) : idesc_bf16_f32(kT, kT);
      const uint32_t rbase = smem_u32(ring);
      int64_t it = 0, tile = 0;
      bool ok = true;
      for (int64_t item = blockIdx.x; ok && item < total; item += gridDim.x) {
        const CandItem d = cand_item(a, item);
        for (int t = 0; t < d.ntiles; ++t, ++tile) {
          const int b = static_cast<int>(tile % kAccN);
          if (!mbar_wait(&sh.acce[b], static_cast<uint32_t>((tile / kAccN) & 1) ^ 1u, a.err, 33)) {
            ok = false;
            break;
          }
          tc_fence_after();
          for (int kb = 0; kb < nkb; ++kb, ++it) {
            const int s = static_cast<int>(it % kStg);
            if (!mbar_wait(&sh.full[s], static_cast<uint32_t>((it / kStg) & 1), a.err, 32)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t sa = rbase + static_cast<uint32_t>(s) * kStageBytes;
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
              if (FP8)
                mma_e4m3(tmem + static_cast<uint32_t>(b * kT), desc_sw128(sa + kk * 32u),
                         desc_sw128(sa + kBlk + kk * 32u), idesc, (kb | kk) != 0 ? 1u : 0u);
              else
                mma_bf16(tmem + static_cast<uint32_t>(b * kT), desc_sw128(sa + kk * 32u),
                         desc_sw128(sa + kBlk + kk * 32u), idesc, (kb | kk) != 0 ? 1u : 0u);
            }
            mma_commit(&sh.empty[s]);
          }
          if (!ok) break;
          mma_commit(&sh.accf[b]);
        }
      }
      // The tensor cores must be done before TMEM is released: one more
      // commit tracks every MMA issued, on the normal and the error path.
      if (it > 0) {
        mma_commit(&sh.drain);
        mbar_wait(&sh.drain, 0u, nullptr, 0, 200000000LL);
      }
    }
  } else {
    const uint32_t lane_base = (32u * static_cast<uint32_t>(warp)) << 16;
    int64_t tile = 0;
    bool ok = true;
    for (int64_t item = blockIdx.x; ok && item < total; item += gridDim.x) {
      const CandItem d = cand_item(a, item);
      // This thread's query (lane tid of the group) and its segment.
      int64_t sbase = 0, slen = 0;
      float f = -2.0f, c0 = 0.0f;  // v = c0 + ||x||^2 + f * acc
      if (tid < d.qcnt) {
        const uint32_t e = static_cast<uint32_t>(a.list_q[d.qrow0 + tid]);
        const int64_t qp = static_cast<int64_t>(e >> 16) * a.P + (e & 0xffffu);
        sbase = a.seg[qp];
        slen = a.seg[qp + 1] - sbase;
        // Residuals: ||q - x||^2 = ||q - c_l||^2 + ||r||^2 - 2 (q - c_l).r
        c0 = a.qcd[d.qrow0 + tid];
        if (FP8) f = -2.0f * a.qscale[d.qrow0 + tid] * a.list_scale[d.list];
      }
      for (int t = 0; t < d.ntiles; ++t, ++tile) {
        const int b = static_cast<int>(tile % kAccN);
        if (ok) ok = mbar_wait(&sh.accf[b], static_cast<uint32_t>((tile / kAccN) & 1), a.err, 34);
        ok = __all_sync(0xffffffffu, ok);
        if (!ok) break;
        tc_fence_after();
        const int64_t rl0 = static_cast<int64_t>(d.chunk) * a.chunk_rows + static_cast<int64_t>(t) * kT;
        // The tile's 128 row norms: one coalesced load per 32 columns, then
        // handed to every lane by shuffles.
        const float* tn = a.tile_norm + (d.tile0 + t) * kT;
        float nrm[kT / 32];
#pragma unroll
        for (int c = 0; c < kT / 32; ++c) nrm[c] = tn[c * 32 + lane];
#pragma unroll
        for (int c = 0; c < kT / 32; ++c) {
          uint32_t r[32];
          tmem_ld32(tmem + lane_base + static_cast<uint32_t>(b * kT + c * 32), r);
          tmem_ld_wait();
#pragma unroll
          for (int j = 0; j < 32; ++j)
            r[j] = __float_as_uint(fmaf(f, __uint_as_float(r[j]), c0 + __shfl_sync(0xffffffffu, nrm[c], j)));
          const int64_t o = rl0 + c * 32;
          if (o < slen) {
            float* out = a.cand + sbase + o;
#pragma unroll
            for (int j4 = 0; j4 < 8; ++j4)
              if (o + 4 * j4 < slen)
                *reinterpret_cast<float4*>(out + 4 * j4) =
                    make_float4(__uint_as_float(r[4 * j4]), __uint_as_float(r[4 * j4 + 1]),
                                __uint_as_float(r[4 * j4 + 2]), __uint_as_float(r[4 * j4 + 3]));
          }
        }
        tc_fence_before();
        mbar_arrive(&sh.acce[b]);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 5) {
    tc_fence_after();
    tmem_dealloc(tmem, kAccN * kT);
  }
}

// 16 floats (times `inv`) -> 16 E4M3 bytes, saturating to +-448.
__device__ __forceinline__ uint4 to_e4m3x16(const float* x, float inv) {
  uint32_t w[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const __nv_fp8x2_storage_t lo =
        __nv_cvt_float2_to_fp8x2(make_float2(x[4 * j] * inv, x[4 * j + 1] * inv), __NV_SATFINITE, __NV_E4M3);
    const __nv_fp8x2_storage_t hi =
        __nv_cvt_float2_to_fp8x2(make_float2(x[4 * j + 2] * inv, x[4 * j + 3] * inv), __NV_SATFINITE, __NV_E4M3);
    w[j] = static_cast<uint32_t>(lo) | (static_cast<uint32_t>(hi) << 16);
  }
  return make_uint4(w[0], w[1], w[2], w[3]);
}

// FP8 copy of the codes as residuals, one CTA per list: r = x - c_l (FP32),
// the list's scale s_l = max |r| / 448 (E4M3's largest finite value), every
// row as E4M3(r / s_l) in kpad8 bytes (columns past dpad zero), and the
// row's FP32 residual norm ||r||^2.
__global__ void list_fp8_kernel(const float* __restrict__ codes, const int64_t* __restrict__ list_off,
                                const float* __restrict__ cent, int dpad, int kpad8, uint8_t* __restrict__ out,
                                float* __restrict__ scale, float* __restrict__ rnorm) {
  __shared__ float s_max[32];
  const int l = blockIdx.x;
  const int64_t r0 = list_off[l], r1 = list_off[l + 1];
  const float* c = cent + static_cast<size_t>(l) * dpad;
  float m = 0.0f;
  for (int64_t i = r0 * dpad + threadIdx.x; i < r1 * dpad; i += blockDim.x)
    m = fmaxf(m, fabsf(codes[i] - c[i % dpad]));
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? s_max[threadIdx.x] : 0.0f;
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) s_max[0] = m;
  }
  __syncthreads();
  const float mx = s_max[0];
  const float inv = mx > 0.0f ? 448.0f / mx : 1.0f;
  if (threadIdx.x == 0) scale[l] = 1.0f / inv;
  const int cpr = kpad8 / 16;
  for (int64_t u = threadIdx.x; u < (r1 - r0) * cpr; u += blockDim.x) {
    const int64_t r = r0 + u / cpr;
    const int cc = static_cast<int>(u % cpr) * 16;
    float x[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) x[j] = cc + j < dpad ? codes[r * dpad + cc + j] - c[cc + j] : 0.0f;
    *reinterpret_cast<uint4*>(out + r * kpad8 + cc) = to_e4m3x16(x, inv);
  }
  // Residual norms, one warp per row.
  const int lane = threadIdx.x & 31;
  for (int64_t r = r0 + (threadIdx.x >> 5); r < r1; r += blockDim.x >> 5) {
    float sq = 0.0f;
    for (int j = lane; j < dpad; j += 32) {
      const float v = codes[r * dpad + j] - c[j];
      sq = fmaf(v, v, sq);
    }
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
    if (lane == 0) rnorm[r] = sq;
  }
}

// One warp per list-major entry e (query q, list l): q' = q - c_l as row e of
// the gathered matrix -- BF16, or (FP8) E4M3(q' / s_e) with the entry's scale
// s_e = max |q'| / 448 -- and ||q'||^2 (the scan's value of a row is
// ||q'||^2 + ||r||^2 - 2 q'.r with r = x - c_l).
template <bool FP8>
__global__ void gather_residual_kernel(const float* __restrict__ q, int dpad, int kpad,
                                       const int32_t* __restrict__ list_q, const int64_t* __restrict__ list_qoff,
                                       int nlist, const float* __restrict__ cent, int64_t max_rows,
                                       float* __restrict__ escale, float* __restrict__ ecd, void* __restrict__ G) {
  const int lane = threadIdx.x & 31;
  const int64_t rows = min(list_qoff[nlist], max_rows);
  for (int64_t e = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5; e < rows;
       e += (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5) {
    int lo = 0, hi = nlist;  // list of entry e: largest l with list_qoff[l] <= e
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (list_qoff[mid] <= e) lo = mid; else hi = mid;
    }
    const int qi = static_cast<int>(static_cast<uint32_t>(list_q[e]) >> 16);
    const float* src = q + static_cast<int64_t>(qi) * dpad;
    const float* c = cent + static_cast<size_t>(lo) * dpad;
    float m = 0.0f, sq = 0.0f;
    for (int j = lane; j < dpad; j += 32) {
      const float v = src[j] - c[j];
      m = fmaxf(m, fabsf(v));
      sq = fmaf(v, v, sq);
    }
    for (int o = 16; o > 0; o >>= 1) {
      m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
      sq += __shfl_xor_sync(0xffffffffu, sq, o);
    }
    if (lane == 0) ecd[e] = sq;
    if (FP8) {
      const float inv = m > 0.0f ? 448.0f / m : 1.0f;
      if (lane == 0) escale[e] = 1.0f / inv;
      uint8_t* row = static_cast<uint8_t*>(G) + e * kpad;
      for (int cc = lane * 16; cc < kpad; cc += 32 * 16) {
        float x[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) x[j] = cc + j < dpad ? src[cc + j] - c[cc + j] : 0.0f;
        *reinterpret_cast<uint4*>(row + cc) = to_e4m3x16(x, inv);
      }
    } else {
      __nv_bfloat16* row = static_cast<__nv_bfloat16*>(G) + e * kpad;
      for (int cc = lane * 8; cc < kpad; cc += 32 * 8) {
        uint32_t w[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const float a0 = cc + 2 * j < dpad ? src[cc + 2 * j] - c[cc + 2 * j] : 0.0f;
          const float a1 = cc + 2 * j + 1 < dpad ? src[cc + 2 * j + 1] - c[cc + 2 * j + 1] : 0.0f;
          __nv_bfloat162 p2 = __floats2bfloat162_rn(a0, a1);
          w[j] = *reinterpret_cast<uint32_t*>(&p2);
        }
        *reinterpret_cast<uint4*>(row + cc) = make_uint4(w[0], w[1], w[2], w[3]);
      }
    }
  }
}

// Segment lengths: the probed list's length rounded up to 4 (0 for a cut
// probe), in (query, probe rank) order; the exclusive sum gives the starts.
__global__ void seg_len_kernel(const int32_t* __restrict__ probes, int nqp, const int64_t* __restrict__ list_off,
                               int64_t* __restrict__ len) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx > nqp) return;
  int64_t n = 0;
  if (idx < nqp) {
    const int l = probes[idx];
    if (l >= 0) n = (list_off[l + 1] - list_off[l] + 3) & ~int64_t(3);
  }
  len[idx] = n;
}

// Histogram bin of a finite candidate value: 2048 equal bins over
// [vmin, vmax]; monotone in v (each step rounds monotonically), so every
// value in a lower bin is below every value in a higher one.
__device__ __forceinline__ int value_bin(float v, float vmin, float scale) {
  const float t = (v - vmin) * scale;
  return t < static_cast<float>(kBins) ? max(0, static_cast<int>(t)) : kBins - 1;
}

// One CTA per query: the R smallest keys (v, position) of the query's
// candidate row -- unique, so the R chosen are the R smallest values with
// ties to the earlier position -- mapped back to their stored rows, in
// ascending key order (-1 past the candidates).  Three coalesced passes over
// the row: the range of its finite values, a 2048-bin histogram over that
// range, and the compaction of every key in the bins up to the one holding
// the R-th value into shared memory, which a bitonic sort orders.  A row
// whose compacted set would exceed the buffer (a dense bin) takes the
// block radix selection instead.  Padding (+inf) is no candidate.
__global__ void __launch_bounds__(kSelectThreads)
    cand_select_kernel(const float* __restrict__ cand, const int64_t* __restrict__ seg,
                       const int32_t* __restrict__ probes, int P, int R, const int64_t* __restrict__ list_off,
                       int cap, int64_t* __restrict__ out_rows) {
  extern __shared__ __align__(16) unsigned char smem_sel[];
  uint64_t* s_cand = reinterpret_cast<uint64_t*>(smem_sel);  // cap keys (a power of two >= 2 * pow2(R))
  __shared__ int s_hist[kBins];
  __shared__ unsigned int s_lo, s_hi;
  __shared__ int s_real, s_bin, s_C, s_cnt;
  __shared__ SelectShared sh_sel;
  const int qi = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t* sq = seg + static_cast<int64_t>(qi) * P;
  const int64_t r0 = sq[0];
  const int m = static_cast<int>(sq[P] - r0);  // a multiple of 4, as is r0
  const float* src = cand + r0;
  for (int i = tid; i < kBins; i += kSelectThreads) s_hist[i] = 0;
  if (tid == 0) {
    s_lo = 0xffffffffu;
    s_hi = 0u;
    s_real = 0;
    s_cnt = 0;
  }
  __syncthreads();
  // Pass 1: count and range of the finite values.
  {
    unsigned int lo = 0xffffffffu, hi = 0u;
    int c = 0;
    const float4* s4 = reinterpret_cast<const float4*>(src);
#pragma unroll 4
    for (int i4 = tid; i4 < m / 4; i4 += kSelectThreads) {
      const float4 v = s4[i4];
      const float e[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (e[j] < INFINITY) {
          const unsigned int o = ordered_bits(e[j]);
          ++c;
          lo = min(lo, o);
          hi = max(hi, o);
        }
    }
    for (int off = 16; off > 0; off >>= 1) {
      c += __shfl_xor_sync(0xffffffffu, c, off);
      lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, off));
      hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, off));
    }
    if (lane == 0 && c) {
      atomicAdd(&s_real, c);
      atomicMin(&s_lo, lo);
      atomicMax(&s_hi, hi);
    }
  }
  __syncthreads();
  const int real = s_real;
  const int need = min(R, real);
  int C = 0;
  if (real > 0) {
    const float vmin = ordered_to_float(s_lo), vmax = ordered_to_float(s_hi);
    const float range = vmax - vmin;
    float scale = range > 0.0f ? static_cast<float>(kBins) / range : 0.0f;
    if (!(scale < 1e30f)) scale = 0.0f;
    // Pass 2: histogram (one shared atomic per value: the values of a run
    // spread over the bins); each warp loads four 32-value runs before it
    // bins them.
    for (int base = tid & ~31; base < m; base += kSelUnroll * kSelectThreads) {
      float vv[kSelUnroll];
#pragma unroll
      for (int u = 0; u < kSelUnroll; ++u) {
        const int i = base + u * kSelectThreads + lane;
        vv[u] = i < m ? src[i] : INFINITY;
      }
#pragma unroll
      for (int u = 0; u < kSelUnroll; ++u)
        if (vv[u] < INFINITY) atomicAdd(&s_hist[value_bin(vv[u], vmin, scale)], 1);
    }
    __syncthreads();
    // The bin holding the need-th value: lane L sums bins [64L, 64L + 64)
    // (read rotated so the lanes hit distinct banks).
    if (warp == 0) {
      int loc = 0;
      for (int j = 0; j < kBins / 32; ++j) loc += s_hist[lane * (kBins / 32) + ((j + lane) & (kBins / 32 - 1))];
      int incl = loc;
      for (int off = 1; off < 32; off <<= 1) {
        const int o = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += o;
      }
      const unsigned hit = __ballot_sync(0xffffffffu, incl >= need);
      if (lane == __ffs(hit) - 1) {
        int cum = incl - loc, b = lane * (kBins / 32);
        for (;; ++b) {
          cum += s_hist[b];
          if (cum >= need) break;
        }
        s_bin = b;
        s_C = cum;
      }
    }
    __syncthreads();
    C = s_C;
    if (C <= cap) {
      // Pass 3: every key in bins <= s_bin, in any order (the keys are unique).
      const int bsel = s_bin;
      for (int base = tid & ~31; base < m; base += kSelUnroll * kSelectThreads) {
        float vv[kSelUnroll];
#pragma unroll
        for (int u = 0; u < kSelUnroll; ++u) {
          const int i = base + u * kSelectThreads + lane;
          vv[u] = i < m ? src[i] : INFINITY;
        }
#pragma unroll
        for (int u = 0; u < kSelUnroll; ++u) {
          const int i = base + u * kSelectThreads + lane;
          const bool take = vv[u] < INFINITY && value_bin(vv[u], vmin, scale) <= bsel;
          const unsigned tm = __ballot_sync(0xffffffffu, take);
          int pos0 = 0;
          if (lane == 0 && tm) pos0 = atomicAdd(&s_cnt, __popc(tm));
          pos0 = __shfl_sync(0xffffffffu, pos0, 0);
          if (take)
            s_cand[pos0 + __popc(tm & ((1u << lane) - 1u))] =
                (static_cast<uint64_t>(ordered_bits(vv[u])) << 32) | static_cast<uint32_t>(i);
        }
      }
      const int c2 = pow2_ceil(C < 2 ? 2 : C);
      for (int i = C + tid; i < c2; i += kSelectThreads) s_cand[i] = kEmpty;
      __syncthreads();
      block_bitonic_sort(s_cand, c2);
    } else {
      // A dense bin: radix selection over the whole row.
      auto key_at = [&](int i) -> uint64_t {
        const float v = src[i];
        return v < INFINITY ? (static_cast<uint64_t>(ordered_bits(v)) << 32) | static_cast<uint32_t>(i) : kEmpty;
      };
      block_topk_sorted(key_at, m, R, sh_sel, s_cand);
    }
  }
  for (int i = tid; i < R; i += kSelectThreads) {
    int64_t row = -1;
    if (i < need) {
      const int64_t pos = r0 + key_tie(s_cand[i]);
      int lo = 0, hi = P;  // the last probe rank whose segment starts at or before pos
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (sq[mid] <= pos) lo = mid; else hi = mid;
      }
      row = list_off[probes[static_cast<int64_t>(qi) * P + lo]] + (pos - sq[lo]);
    }
    out_rows[static_cast<int64_t>(qi) * R + i] = row;
  }
}

// One CTA per query: exact distances of its R candidate rows with the
// reference's sequential unfused FP32 loop (the same operations, in the same
// order, as exact_l2_seq), then the k best (distance, row).  Thread t owns
// candidate t of each batch of blockDim.x (R rounded up to a warp, 64 to
// 256); the batch's rows and the query are staged 32 dimensions at a time
// in shared memory by coalesced loads (four 128-byte rows per warp
// instruction, all of a thread's loads in flight at once), and each thread
// continues its own sum over the chunk from shared memory.
__global__ void __launch_bounds__(kExactThreads)
    cand_exact_kernel(const int64_t* __restrict__ rows, int R, int k, const float* __restrict__ codes,
                      const float* __restrict__ q, int dpad, const int64_t* __restrict__ ids, float* __restrict__ D,
                      int64_t* __restrict__ I) {
  extern __shared__ __align__(16) unsigned char smem_ex[];
  __shared__ int64_t s_rows[kExactThreads];
  __shared__ __align__(16) float s_q[kExChunk];
  const int qi = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
  const int n2 = pow2_ceil(R < 2 ? 2 : R);
  uint64_t* s_ex = reinterpret_cast<uint64_t*>(smem_ex);
  float* s_tile = reinterpret_cast<float*>(s_ex + n2);  // nt x kExStride
  const float* qrow = q + static_cast<size_t>(qi) * dpad;
  for (int i = tid; i < n2; i += nt) s_ex[i] = kEmpty;
  for (int b0 = 0; b0 < R; b0 += nt) {
    const int i = b0 + tid;
    const int64_t row = i < R ? rows[static_cast<int64_t>(qi) * R + i] : -1;
    s_rows[tid] = row;
    float acc = 0.0f;
    for (int c0 = 0; c0 < dpad; c0 += kExChunk) {
      const int w4 = min(kExChunk, dpad - c0) / 4;  // dpad is a multiple of 4
      __syncthreads();                              // rows published / previous chunk consumed
      if (tid < w4) *reinterpret_cast<float4*>(s_q + 4 * tid) = *reinterpret_cast<const float4*>(qrow + c0 + 4 * tid);
#pragma unroll
      for (int j = 0; j < kExChunk / 4; ++j) {
        const int u = tid + j * nt;
        const int r = u / (kExChunk / 4), f = u % (kExChunk / 4);
        const int64_t rr = s_rows[r];
        if (rr >= 0 && f < w4) {
          const float4 v = *reinterpret_cast<const float4*>(codes + rr * dpad + c0 + 4 * f);
          float* dst = s_tile + r * kExStride + 4 * f;
          dst[0] = v.x;
          dst[1] = v.y;
          dst[2] = v.z;
          dst[3] = v.w;
        }
      }
      __syncthreads();
      if (row >= 0) {
        const float* x = s_tile + tid * kExStride;
        for (int c = 0; c < 4 * w4; c += 4) {
          const float4 qq = *reinterpret_cast<const float4*>(s_q + c);
          const float x0 = x[c], x1 = x[c + 1], x2 = x[c + 2], x3 = x[c + 3];
          float t = __fsub_rn(qq.x, x0);
          acc = __fadd_rn(acc, __fmul_rn(t, t));
          t = __fsub_rn(qq.y, x1);
          acc = __fadd_rn(acc, __fmul_rn(t, t));
          t = __fsub_rn(qq.z, x2);
          acc = __fadd_rn(acc, __fmul_rn(t, t));
          t = __fsub_rn(qq.w, x3);
          acc = __fadd_rn(acc, __fmul_rn(t, t));
        }
      }
    }
    if (row >= 0 && acc < FLT_MAX) s_ex[i] = make_key(acc, static_cast<uint32_t>(row));
  }
  __syncthreads();
  block_bitonic_sort(s_ex, n2);
  for (int j = tid; j < k; j += nt) {
    const uint64_t key = j < n2 ? s_ex[j] : kEmpty;
    const size_t o = static_cast<size_t>(qi) * k + j;
    D[o] = key == kEmpty ? FLT_MAX : key_dist(key);
    I[o] = key == kEmpty ? -1 : ids[key_tie(key)];
  }
}

}  // namespace

size_t cand_segments_tmp_bytes(int nq, int P) {
  const size_t n = static_cast<size_t>(nq) * P + 1;
  size_t bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, bytes, static_cast<const int64_t*>(nullptr), static_cast<int64_t*>(nullptr),
                                static_cast<int64_t>(n));
  bytes = (bytes + 255) / 256 * 256;
  return bytes + n * sizeof(int64_t);
}

void launch_cand_segments(const int32_t* probes, int nq, int P, const int64_t* list_off, int64_t* seg, void* tmp,
                          size_t tmp_bytes, cudaStream_t st) {
  const int nqp = nq * P;
  const size_t n = static_cast<size_t>(nqp) + 1;
  size_t cub_bytes = 0;
  HB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, cub_bytes, static_cast<const int64_t*>(nullptr),
                                        static_cast<int64_t*>(nullptr), static_cast<int64_t>(n)));
  const size_t cub_pad = (cub_bytes + 255) / 256 * 256;
  HB_CHECK(tmp_bytes >= cub_pad + n * sizeof(int64_t), HB_ERR_INVALID, "segment scratch too small");
  int64_t* len = reinterpret_cast<int64_t*>(static_cast<unsigned char*>(tmp) + cub_pad);
  seg_len_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(probes, nqp, list_off, len);
  HB_CUDA(cudaGetLastError());
  size_t bytes = cub_bytes;
  HB_CUDA(cub::DeviceScan::ExclusiveSum(tmp, bytes, len, seg, static_cast<int64_t>(n), st));
}

void launch_cand_scan(const void* tmap_q, const void* tmap_x, const CandArgs& a, int num_sms, cudaStream_t st) {
  const int blk = a.fp8 ? 128 : 64;
  HB_CHECK(a.kpad >= blk && a.kpad % blk == 0, HB_ERR_INVALID, "the candidate scan needs whole 128-byte K blocks");
  HB_CHECK(a.qcd && (!a.fp8 || (a.qscale && a.list_scale)), HB_ERR_INVALID, "residual scan without its constants");
  HB_CHECK(a.chunk_rows >= kT && a.chunk_rows % kT == 0, HB_ERR_INVALID, "chunk rows must be a multiple of 128");
  const size_t smem = kStg * static_cast<size_t>(kStageBytes) + 1024;
  const CUtensorMap* mq = static_cast<const CUtensorMap*>(tmap_q);
  const CUtensorMap* mx = static_cast<const CUtensorMap*>(tmap_x);
  if (a.fp8) {
    HB_CUDA(cudaFuncSetAttribute(cand_scan_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)));
    cand_scan_kernel<true><<<num_sms, kThreads, smem, st>>>(*mq, *mx, a);
  } else {
    HB_CUDA(cudaFuncSetAttribute(cand_scan_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)));
    cand_scan_kernel<false><<<num_sms, kThreads, smem, st>>>(*mq, *mx, a);
  }
  HB_CUDA(cudaGetLastError());
}

void launch_fp8_codes(const float* codes, const int64_t* list_off, const float* cent, int nlist, int dpad, int kpad8,
                      void* out, float* scale, float* rnorm, cudaStream_t st) {
  if (nlist <= 0) return;
  HB_CHECK(kpad8 % 128 == 0 && dpad <= kpad8, HB_ERR_INVALID, "bad FP8 row length");
  list_fp8_kernel<<<nlist, 256, 0, st>>>(codes, list_off, cent, dpad, kpad8, static_cast<uint8_t*>(out), scale, rnorm);
  HB_CUDA(cudaGetLastError());
}

void launch_gather_residual(const float* q, int dpad, int kpad, bool fp8, const int32_t* list_q,
                            const int64_t* list_qoff, int nlist, const float* cent, int64_t max_rows, float* escale,
                            float* ecd, void* G, cudaStream_t st) {
  if (max_rows <= 0) return;
  HB_CHECK(kpad % (fp8 ? 128 : 64) == 0 && dpad <= kpad && kpad <= 2048, HB_ERR_INVALID, "bad residual padding");
  int64_t g = (max_rows * 32 + 255) / 256;
  if (g > 148 * 32) g = 148 * 32;
  if (fp8)
    gather_residual_kernel<true><<<static_cast<unsigned>(g), 256, 0, st>>>(q, dpad, kpad, list_q, list_qoff, nlist,
                                                                           cent, max_rows, escale, ecd, G);
  else
    gather_residual_kernel<false><<<static_cast<unsigned>(g), 256, 0, st>>>(q, dpad, kpad, list_q, list_qoff, nlist,
                                                                            cent, max_rows, escale, ecd, G);
  HB_CUDA(cudaGetLastError());
}

void make_u8_tensor_map(void* tmap_out, const void* base, size_t rows, int row_bytes) {
  CUtensorMap* m = static_cast<CUtensorMap*>(tmap_out);
  cuuint64_t dims[2] = {static_cast<cuuint64_t>(row_bytes), static_cast<cuuint64_t>(rows)};
  cuuint64_t strides[1] = {static_cast<cuuint64_t>(row_bytes)};
  cuuint32_t box[2] = {128, kT};
  cuuint32_t es[2] = {1, 1};
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult qr;
  HB_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &qr));
  HB_CHECK(fn && qr == cudaDriverEntryPointSuccess, HB_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  CUresult r = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn)(
      m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base), dims, strides, box, es,
      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  HB_CHECK(r == CUDA_SUCCESS, HB_ERR_CUDA, "cuTensorMapEncodeTiled failed (FP8)");
}

void launch_cand_select(const float* cand, const int64_t* seg, const int32_t* probes, int nq, int P, int R,
                        const int64_t* list_off, int64_t* rows, cudaStream_t st) {
  if (nq <= 0) return;
  HB_CHECK(R >= 1 && R <= kCandMaxR, HB_ERR_INVALID, "candidate count out of range");
  // Compaction buffer: at least 2048 keys and four times the R kept.
  const int cap = std::max(2048, 4 * pow2_ceil(R < 2 ? 2 : R));
  const size_t smem_sel = static_cast<size_t>(cap) * sizeof(uint64_t);
  HB_CUDA(cudaFuncSetAttribute(cand_select_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(smem_sel)));
  cand_select_kernel<<<nq, kSelectThreads, smem_sel, st>>>(cand, seg, probes, P, R, list_off, cap, rows);
  HB_CUDA(cudaGetLastError());
}

void launch_cand_exact(const int64_t* rows, int nq, int R, int k, const float* codes, const float* q, int dpad,
                       const int64_t* ids, float* D, int64_t* I, cudaStream_t st) {
  if (nq <= 0) return;
  HB_CHECK(R >= 1 && R <= kCandMaxR && k <= R, HB_ERR_INVALID, "candidate count out of range");
  const size_t keys = static_cast<size_t>(pow2_ceil(R < 2 ? 2 : R)) * sizeof(uint64_t);
  const int nt = std::min(kExactThreads, std::max(64, (R + 31) / 32 * 32));
  const size_t smem_ex = keys + static_cast<size_t>(nt) * kExStride * sizeof(float);
  HB_CUDA(cudaFuncSetAttribute(cand_exact_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(smem_ex)));
  cand_exact_kernel<<<nq, nt, smem_ex, st>>>(rows, R, k, codes, q, dpad, ids, D, I);
  HB_CUDA(cudaGetLastError());
}

}  // namespace hb

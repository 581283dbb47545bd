// Tensor-core coarse quantizer with an exact FP32 finish.
//
//  1. coarse_tc_kernel: queries and centroids are split into BF16 pairs
//     x = hi + lo (hi = bf16(x), lo = bf16(x - hi)), each stored as one row
//     [hi | lo] of 2 * kpad BF16 (split_rows_kernel).  Per (centroid tile,
//     query tile) of 128 x 128 one tcgen05.mma chain accumulates
//     q_hi.c_hi + q_hi.c_lo + q_lo.c_hi, i.e. q.c to about 2^-16 relative
//     (the 3-term BF16 split).  A CTA keeps one centroid tile resident in
//     shared memory (B, K-major, 128-byte swizzle, one TMA load) and streams
//     query tiles (A) through a ring of 64-column K blocks; accumulators are
//     double-buffered in TMEM.  The (centroid tile, query tile) pairs are
//     ordered centroid tile first and split into equal contiguous ranges, one
//     per CTA, one CTA per SM, so a CTA loads at most a few centroid tiles.
//     The epilogue (thread = query) writes v = max(0, ||q||^2 + ||c||^2 -
//     2 q.c) to an nq x nlist matrix.
//  2. select_rows (k_select.cu) keeps the Pm = P + m smallest values.
//  3. coarse_refine_kernel recomputes those Pm distances exactly (the
//     reference's sequential unfused FP32 loop, src/utils.h:480-487), sorts
//     them by (distance, centroid) and keeps P.  Every centroid outside the
//     Pm has v >= v_last (the Pm-th value), hence an exact distance >=
//     v_last - bound, bound being the error bound of v; when the exact P-th
//     distance is below that, the P kept are exactly the exact quantizer's.
//     Otherwise the query is flagged.
//  4. coarse_fallback_kernel recomputes each flagged query's row exactly.
// The probe rows equal the exact quantizer's (l2_matrix + select_rows) in
// every case; the tensor cores only decide which distances get computed.
//
// Error bound of v: the split leaves |q.c - (q_hi.c_hi + q_hi.c_lo +
// q_lo.c_hi)| <= 3 * 2^-18 * sum|q_i c_i|; the FP32 accumulation of 3 * kpad
// <= 384 exact BF16 products, in any order, adds <= 384 * 2^-23 *
// sum|q_i c_i|; with sum|q_i c_i| <= ||q|| ||c|| the dot error is < 6e-5
// ||q|| ||c||, so 2 q.c is within 1.2e-4 ||q|| ||c||.  The norms, the FP32
// combination and the reference's own FP32 rounding add < 1e-5 (||q||^2 +
// ||c||^2 + v).  The bound used, 4e-4 ||q|| max||c|| + 2e-5 (max||c||^2 +
// ||q||^2 + |v|), is more than three times that.
#include <cudaTypedefs.h>
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "hb_device.cuh"
#include "hb_internal.hpp"
#include "hb_select.cuh"
#include "hb_sm100.cuh"

namespace hb {
namespace {

using namespace sm100;

constexpr int kCT = 128;        // queries per tile = centroids per tile
constexpr int kCStages = 6;     // ring of 64-column K blocks of query tiles (16 KB each)
constexpr int kCEpiWarps = 8;   // epilogue warps: two per TMEM lane quarter, one per half of the columns
constexpr int kCTmaWarp = kCEpiWarps, kCMmaWarp = kCEpiWarps + 1;
constexpr int kCThreads = (kCEpiWarps + 2) * 32;
constexpr uint32_t kBlk = kCT * 128;  // bytes of one 128-row x 64-column BF16 block
constexpr uint32_t kBoxBytes = 32 * 128;  // one 32 x 32 FP32 box of V

struct CoarseShared {
  uint64_t full[kCStages];
  uint64_t empty[kCStages];
  uint64_t accf[2];
  uint64_t acce[2];
  uint64_t bfull;
  uint64_t bempty;
  uint32_t tmem;
};

// Pairs [p0, p1) of CTA b out of G over `pairs`, centroid tile = p / qt.
__device__ __forceinline__ void coarse_range(int b, int G, int pairs, int& p0, int& p1) {
  p0 = static_cast<int>(static_cast<long long>(b) * pairs / G);
  p1 = static_cast<int>(static_cast<long long>(b + 1) * pairs / G);
}

__global__ void __launch_bounds__(kCThreads, 1)
    coarse_tc_kernel(const __grid_constant__ CUtensorMap tmap_c, const __grid_constant__ CUtensorMap tmap_q,
                     const __grid_constant__ CUtensorMap tmap_v, int tma_v, const float* __restrict__ qnorm, int nq,
                     int kpad, const float* __restrict__ cnorm, int nlist, int qt, int pairs, float* __restrict__ V,
                     uint32_t* __restrict__ cmins,
                     int* __restrict__ err) {
  extern __shared__ uint8_t smem_raw[];
  __shared__ CoarseShared sh;
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int nh = kpad / 64;  // K blocks of one half (hi or lo)
  uint8_t* Bt = smem;        // resident centroid tile: [c_hi | c_lo], 2 * nh blocks
  uint8_t* ring = smem + static_cast<size_t>(2 * nh) * kBlk;
  // Per epilogue warp, two 32 x 32 FP32 boxes (128-byte swizzle) for the
  // TMA stores of its two chunks of a tile.
  uint8_t* stg = ring + static_cast<size_t>(kCStages) * kBlk;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  int p0, p1;
  coarse_range(blockIdx.x, gridDim.x, pairs, p0, p1);

  if (warp == kCMmaWarp) tmem_alloc(&sh.tmem, 256);
  if (tid == 0) {
    for (int s = 0; s < kCStages; ++s) {
      mbar_init(&sh.full[s], 1);
      mbar_init(&sh.empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&sh.accf[b], 1);
      mbar_init(&sh.acce[b], kCEpiWarps * 32);
    }
    mbar_init(&sh.bfull, 1);
    mbar_init(&sh.bempty, 1);
    fence_barrier_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sh.tmem;

  if (warp == kCTmaWarp) {
    if (lane == 0) {
      // Centroid tile at each change of tile (after the MMAs that read the
      // previous one), then the query tile's 2 * nh K blocks.
      int it = 0, nb = 0, cur = -1;
      for (int p = p0; p < p1; ++p) {
        const int c = p / qt, qtile = p - c * qt;
        if (c != cur) {
          if (nb > 0 && !mbar_wait(&sh.bempty, (nb - 1) & 1u, err, 25)) break;
          mbar_arrive_expect_tx(&sh.bfull, static_cast<uint32_t>(2 * nh) * kBlk);
          for (int kb = 0; kb < 2 * nh; ++kb) tma_load_2d(Bt + static_cast<size_t>(kb) * kBlk, &tmap_c, kb * 64, c * kCT, &sh.bfull);
          cur = c;
          ++nb;
        }
        bool ok = true;
        for (int kb = 0; kb < 2 * nh; ++kb, ++it) {
          const int s = it % kCStages;
          if (!mbar_wait(&sh.empty[s], ((it / kCStages) & 1u) ^ 1u, err, 21)) {
            ok = false;
            break;
          }
          mbar_arrive_expect_tx(&sh.full[s], kBlk);
          tma_load_2d(ring + static_cast<size_t>(s) * kBlk, &tmap_q, kb * 64, qtile * kCT, &sh.full[s]);
        }
        if (!ok) break;
      }
    }
  } else if (warp == kCMmaWarp) {
    if (lane == 0) {
      const uint32_t idesc = idesc_bf16_f32(kCT, kCT);
      const uint32_t bbase = smem_u32(Bt), rbase = smem_u32(ring);
      int it = 0, nb = 0, cur = -1, issued = 0;
      bool ok = true;
      for (int p = p0; p < p1 && ok; ++p) {
        const int c = p / qt;
        if (c != cur) {
          if (!mbar_wait(&sh.bfull, nb & 1u, err, 26)) break;
          tc_fence_after();
          cur = c;
          ++nb;
        }
        const int i = p - p0, b = i & 1;
        if (!mbar_wait(&sh.acce[b], ((i >> 1) & 1u) ^ 1u, err, 23)) break;
        tc_fence_after();
        const uint32_t d = tmem + static_cast<uint32_t>(b * kCT);
        // A block kb: q_hi block kb (kb < nh) meets c_hi and c_lo block kb;
        // q_lo block kb - nh meets c_hi block kb - nh.
        for (int kb = 0; kb < 2 * nh; ++kb, ++it) {
          const int s = it % kCStages;
          if (!mbar_wait(&sh.full[s], (it / kCStages) & 1u, err, 22)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint64_t ad = desc_sw128(rbase + static_cast<uint32_t>(s) * kBlk);
          const int j = kb < nh ? kb : kb - nh;
          const uint64_t bh = desc_sw128(bbase + static_cast<uint32_t>(j) * kBlk);
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) mma_bf16(d, ad + 2 * kk, bh + 2 * kk, idesc, (kb | kk) != 0 ? 1u : 0u);
          if (kb < nh) {
            const uint64_t bl = desc_sw128(bbase + static_cast<uint32_t>(nh + j) * kBlk);
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) mma_bf16(d, ad + 2 * kk, bl + 2 * kk, idesc, 1u);
          }
          mma_commit(&sh.empty[s]);
        }
        if (!ok) break;
        mma_commit(&sh.accf[b]);
        ++issued;
        // The last tile against this centroid tile: its MMAs free B.
        if (p + 1 == p1 || (p + 1) / qt != c) mma_commit(&sh.bempty);
      }
      // Drain: the tensor cores must be done before TMEM is released.
      if (issued > 0) {
        const int l = issued - 1;
        mbar_wait(&sh.accf[l & 1], (l >> 1) & 1u, nullptr, 0, 200000000LL);
      }
    }
  } else {
    // Warp w: TMEM lanes (queries) 32 (w % 4) .. + 31, columns 64 (w / 4)
    // .. + 63 of each tile (two 32-column chunks).
    const uint32_t lane_base = (32u * static_cast<uint32_t>(warp & 3)) << 16;
    const int half = warp >> 2;
    bool ok = true;
    for (int p = p0; p < p1; ++p) {
      const int c = p / qt, qtile = p - c * qt;
      const int i = p - p0, b = i & 1;
      const int qi = qtile * kCT + (warp & 3) * 32 + lane;
      const float qn = qi < nq ? qnorm[qi] : 0.0f;
      if (ok) ok = mbar_wait(&sh.accf[b], (i >> 1) & 1u, err, 24);
      ok = __all_sync(0xffffffffu, ok);
      if (!ok) break;
      tc_fence_after();
      const uint32_t t0 = tmem + lane_base + static_cast<uint32_t>(b * kCT + half * 64);
      uint32_t ra[32], rb[32];
      tmem_ld32(t0, ra);
      tmem_ld32(t0 + 32, rb);
      tmem_ld_wait(ra);
      tmem_ld_wait(rb);
      tc_fence_before();
      mbar_arrive(&sh.acce[b]);
      uint8_t* box0 = stg + static_cast<size_t>(warp) * 2 * kBoxBytes;
      if (tma_v) {
        // The previous tile's stores have read the boxes.
        if (lane == 0) bulk_wait_read();
        __syncwarp();
      }
      auto chunk = [&](const uint32_t (&r)[32], int cb, uint8_t* box) {
        float* out = V + static_cast<size_t>(qi) * nlist + cb;
        // The smallest value of each 16-column half of the chunk over its
        // columns inside nlist, stored chunk-major (a warp's 32 queries are
        // one 128-byte store).
        uint32_t cm[2] = {0xFFFFFFFFu, 0xFFFFFFFFu};
        const bool full = cb + 32 <= nlist;
        auto cmin4 = [&](const float4& o, int c) {
          const uint32_t e0 = full || c + 0 < nlist ? __float_as_uint(o.x) : 0xFFFFFFFFu;
          const uint32_t e1 = full || c + 1 < nlist ? __float_as_uint(o.y) : 0xFFFFFFFFu;
          const uint32_t e2 = full || c + 2 < nlist ? __float_as_uint(o.z) : 0xFFFFFFFFu;
          const uint32_t e3 = full || c + 3 < nlist ? __float_as_uint(o.w) : 0xFFFFFFFFu;
          uint32_t& m = cm[(c - cb) >> 4];
          m = min(min(m, min(e0, e1)), min(e2, e3));
        };
        auto put_cm = [&]() {
          if (cmins && qi < nq) {
            cmins[static_cast<size_t>(cb / 16) * nq + qi] = cm[0];
            if (cb + 16 < nlist) cmins[static_cast<size_t>(cb / 16 + 1) * nq + qi] = cm[1];
          }
        };
        if (tma_v) {
          // Row `lane` of the box: 16-byte piece j4 at (j4 ^ (lane % 8)).
#pragma unroll
          for (int j4 = 0; j4 < 8; ++j4) {
            float4 cn;
            if (cb + 4 * j4 + 3 < nlist) {
              cn = *reinterpret_cast<const float4*>(cnorm + cb + 4 * j4);
            } else {
              cn.x = cb + 4 * j4 + 0 < nlist ? cnorm[cb + 4 * j4 + 0] : 0.0f;
              cn.y = cb + 4 * j4 + 1 < nlist ? cnorm[cb + 4 * j4 + 1] : 0.0f;
              cn.z = cb + 4 * j4 + 2 < nlist ? cnorm[cb + 4 * j4 + 2] : 0.0f;
              cn.w = 0.0f;
            }
            float4 o;
            o.x = fmaxf(fmaf(-2.0f, __uint_as_float(r[4 * j4 + 0]), qn + cn.x), 0.0f);
            o.y = fmaxf(fmaf(-2.0f, __uint_as_float(r[4 * j4 + 1]), qn + cn.y), 0.0f);
            o.z = fmaxf(fmaf(-2.0f, __uint_as_float(r[4 * j4 + 2]), qn + cn.z), 0.0f);
            o.w = fmaxf(fmaf(-2.0f, __uint_as_float(r[4 * j4 + 3]), qn + cn.w), 0.0f);
            cmin4(o, cb + 4 * j4);
            *reinterpret_cast<float4*>(box + lane * 128 + ((j4 ^ (lane & 7)) << 4)) = o;
          }
          put_cm();
          return;
        }
        if (nlist - cb >= 32 && (nlist & 3) == 0) {
#pragma unroll
          for (int j4 = 0; j4 < 8; ++j4) {
            const float4 cn = *reinterpret_cast<const float4*>(cnorm + cb + 4 * j4);
            float4 o;
            o.x = fmaxf(fmaf(-2.0f, __uint_as_float(r[4 * j4 + 0]), qn + cn.x), 0.0f);
            o.y = fmaxf(fmaf(-2.0f, __uint_as_float(r[4 * j4 + 1]), qn + cn.y), 0.0f);
            o.z = fmaxf(fmaf(-2.0f, __uint_as_float(r[4 * j4 + 2]), qn + cn.z), 0.0f);
            o.w = fmaxf(fmaf(-2.0f, __uint_as_float(r[4 * j4 + 3]), qn + cn.w), 0.0f);
            cmin4(o, cb + 4 * j4);
            if (qi < nq) *reinterpret_cast<float4*>(out + 4 * j4) = o;
          }
        } else {
#pragma unroll
          for (int j = 0; j < 32; ++j)
            if (cb + j < nlist) {
              const float v = fmaxf(fmaf(-2.0f, __uint_as_float(r[j]), qn + cnorm[cb + j]), 0.0f);
              cm[j >> 4] = min(cm[j >> 4], __float_as_uint(v));
              if (qi < nq) out[j] = v;
            }
        }
        put_cm();
      };
      const int cb = c * kCT + half * 64;
      if (cb < nlist) chunk(ra, cb, box0);
      if (cb + 32 < nlist) chunk(rb, cb + 32, box0 + kBoxBytes);
      if (tma_v) {
        // Rows past nq and columns past nlist of a box are not written.
        fence_proxy_async_smem();
        __syncwarp();
        const int row = qtile * kCT + (warp & 3) * 32;
        if (lane == 0 && row < nq) {
          if (cb < nlist) tma_store_2d(&tmap_v, box0, cb, row);
          if (cb + 32 < nlist) tma_store_2d(&tmap_v, box0 + kBoxBytes, cb + 32, row);
          bulk_commit();
        }
      }
    }
    // The stores are complete before the CTA (and its shared memory) ends.
    if (tma_v && lane == 0) bulk_wait_all();
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kCMmaWarp) {
    tc_fence_after();
    tmem_dealloc(tmem, 256);
  }
}

// Rows (FP32, dpad wide) -> [hi | lo] BF16 rows of 2 * kpad (zeros past d),
// and, when norm is given, each row's ||x||^2; a warp per row.
__global__ void split_rows_kernel(const float* __restrict__ x, int n, int dpad, int kpad,
                                  __nv_bfloat16* __restrict__ out, float* __restrict__ norm) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += warps) {
    const float* row = x + static_cast<size_t>(r) * dpad;
    __nv_bfloat16* o = out + static_cast<size_t>(r) * 2 * kpad;
    float s = 0.0f;
    for (int k = lane; k < kpad; k += 32) {
      const float v = k < dpad ? row[k] : 0.0f;
      s = fmaf(v, v, s);
      const __nv_bfloat16 h = __float2bfloat16_rn(v);
      o[k] = h;
      o[kpad + k] = __float2bfloat16_rn(v - __bfloat162float(h));
    }
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (norm && lane == 0) norm[r] = s;
  }
}

// One warp per query: exact distances of its Pm candidates (lane = candidate,
// sequential over the dims), sort by (distance, centroid), keep P; flag the
// query when the exactness bound does not hold.
__device__ __forceinline__ int coarse_extra_dev(int P, int margin) { return margin >= 0 ? margin : max(16, P / 4); }

__global__ void __launch_bounds__(256) coarse_refine_kernel(const float* __restrict__ q, int nq, int dpad,
                                                            const float* __restrict__ cent,
                                                            const int32_t* __restrict__ cand, const float* __restrict__ cval,
                                                            int Pm, int P, int nlist, const float* __restrict__ cmaxnorm,
                                                            int32_t* __restrict__ probes, float* __restrict__ cdist,
                                                            int* __restrict__ flags, CoarseRows rows) {
  // [warps][pow2(Pm)] keys, then a stage of 32 rows x 64 columns per warp.
  extern __shared__ __align__(16) uint8_t s_ref_raw[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int qi = blockIdx.x * (blockDim.x >> 5) + wib;
  if (qi >= nq) return;
  // This row's width and candidate count (P and Pm are the row strides).
  int Pr = P, Pmr = Pm;
  if (rows.width) {
    Pr = min(rows.width[qi], P);
    if (Pr <= 0 || (rows.pre && Pr <= rows.pre_w)) {
      // Already exact from the narrower pass (or empty): copy and pad.
      for (int j = lane; j < P; j += 32)
        probes[static_cast<size_t>(qi) * P + j] =
            (j < Pr && rows.pre) ? rows.pre[static_cast<size_t>(qi) * rows.pre_w + j] : -1;
      if (lane == 0) flags[qi] = 0;
      return;
    }
    Pmr = min(nlist, Pr + coarse_extra_dev(Pr, rows.margin));
  }
  const int n2 = pow2_ceil(Pmr < 2 ? 2 : Pmr);
  // Per-warp buffers are laid out for the launch's widest row.
  const int nmax = pow2_ceil(Pm < 2 ? 2 : Pm);
  uint64_t* buf = reinterpret_cast<uint64_t*>(s_ref_raw) + static_cast<size_t>(wib) * nmax;
  float* stage = reinterpret_cast<float*>(s_ref_raw + static_cast<size_t>(blockDim.x >> 5) * nmax * 8) +
                 static_cast<size_t>(wib) * 32 * kHalfStageStride;
  const float* qrow = q + static_cast<size_t>(qi) * dpad;
  float qn = 0.0f;
  for (int c = lane * 4; c < dpad; c += 128) {
    const float4 v = *reinterpret_cast<const float4*>(qrow + c);
    qn += v.x * v.x + v.y * v.y + v.z * v.z + v.w * v.w;
  }
  for (int o = 16; o > 0; o >>= 1) qn += __shfl_xor_sync(0xffffffffu, qn, o);
  // 32 candidates at a time, lane = candidate: the warp stages 64 columns
  // of their centroid rows at a time, each lane continuing the sequential
  // loop over its row.
  for (int base = 0; base < n2; base += 32) {
    const int i = base + lane;
    const int c = i < Pmr ? cand[static_cast<size_t>(qi) * Pm + i] : -1;
    float acc = 0.0f;
    if (base < Pmr) {
      const int nv = min(32, Pmr - base);
      for (int c0 = 0; c0 < dpad; c0 += 64) {
        const int nc = min(64, dpad - c0);
        warp_stage_half_rows(cent, c, dpad, c0, nc, stage, nv, lane);
        if (c >= 0) acc = exact_l2_seq_from(acc, stage + static_cast<size_t>(lane) * kHalfStageStride, qrow + c0, nc);
      }
    }
    uint64_t key = kEmpty;
    if (c >= 0 && acc < FLT_MAX) key = make_key(acc, static_cast<uint32_t>(c));
    if (i < n2) buf[i] = key;
  }
  __syncwarp();
  warp_bitonic_sort(buf, n2, lane);
  for (int j = lane; j < P; j += 32) {
    const uint64_t key = j < Pr ? buf[j] : kEmpty;
    probes[static_cast<size_t>(qi) * P + j] = key == kEmpty ? -1 : static_cast<int32_t>(key_tie(key));
    if (cdist) cdist[static_cast<size_t>(qi) * P + j] = key == kEmpty ? FLT_MAX : key_dist(key);
  }
  if (lane == 0) {
    bool exact = true;
    if (Pmr < nlist) {
      // Outside the Pmr candidates every value is >= vlast, so every exact
      // distance there is >= vlast - bound.
      const float vlast = cval[static_cast<size_t>(qi) * Pm + Pmr - 1];
      const uint64_t kp = buf[Pr - 1];
      exact = kp != kEmpty && vlast < FLT_MAX;
      if (exact) {
        const float mn = *cmaxnorm;
        const float bound = 4e-4f * sqrtf(qn) * mn + 2e-5f * (mn * mn + qn + fabsf(vlast)) + 1e-30f;
        exact = key_dist(kp) < vlast - bound;
      }
    }
    flags[qi] = exact ? 0 : 1;
  }
}

// The same refinement with one CTA per query, for small batches (a warp per
// query leaves the GPU idle when there are few queries): threads take
// candidates, the CTA sorts them.
__global__ void __launch_bounds__(256) coarse_refine_block_kernel(
    const float* __restrict__ q, int nq, int dpad, const float* __restrict__ cent, const int32_t* __restrict__ cand,
    const float* __restrict__ cval, int Pm, int P, int nlist, const float* __restrict__ cmaxnorm,
    int32_t* __restrict__ probes, float* __restrict__ cdist, int* __restrict__ flags, CoarseRows rows) {
  extern __shared__ uint64_t s_blk[];  // pow2(Pm)
  __shared__ float s_qn[8];
  const int qi = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  int Pr = P, Pmr = Pm;
  if (rows.width) {
    Pr = min(rows.width[qi], P);
    if (Pr <= 0 || (rows.pre && Pr <= rows.pre_w)) {
      for (int j = tid; j < P; j += blockDim.x)
        probes[static_cast<size_t>(qi) * P + j] =
            (j < Pr && rows.pre) ? rows.pre[static_cast<size_t>(qi) * rows.pre_w + j] : -1;
      if (tid == 0) flags[qi] = 0;
      return;
    }
    Pmr = min(nlist, Pr + coarse_extra_dev(Pr, rows.margin));
  }
  const int n2 = pow2_ceil(Pmr < 2 ? 2 : Pmr);
  const float* qrow = q + static_cast<size_t>(qi) * dpad;
  float qn = 0.0f;
  for (int c = tid; c < dpad; c += blockDim.x) qn = fmaf(qrow[c], qrow[c], qn);
  for (int o = 16; o > 0; o >>= 1) qn += __shfl_xor_sync(0xffffffffu, qn, o);
  if (lane == 0) s_qn[wid] = qn;
  for (int i = tid; i < n2; i += blockDim.x) {
    uint64_t key = kEmpty;
    if (i < Pmr) {
      const int c = cand[static_cast<size_t>(qi) * Pm + i];
      if (c >= 0) {
        const float acc = exact_l2_seq(cent + static_cast<size_t>(c) * dpad, qrow, dpad);
        if (acc < FLT_MAX) key = make_key(acc, static_cast<uint32_t>(c));
      }
    }
    s_blk[i] = key;
  }
  __syncthreads();
  block_bitonic_sort(s_blk, n2);
  for (int j = tid; j < P; j += blockDim.x) {
    const uint64_t key = j < Pr ? s_blk[j] : kEmpty;
    probes[static_cast<size_t>(qi) * P + j] = key == kEmpty ? -1 : static_cast<int32_t>(key_tie(key));
    if (cdist) cdist[static_cast<size_t>(qi) * P + j] = key == kEmpty ? FLT_MAX : key_dist(key);
  }
  if (tid == 0) {
    float qs = 0.0f;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) qs += s_qn[w];
    bool exact = true;
    if (Pmr < nlist) {
      const float vlast = cval[static_cast<size_t>(qi) * Pm + Pmr - 1];
      const uint64_t kp = s_blk[Pr - 1];
      exact = kp != kEmpty && vlast < FLT_MAX;
      if (exact) {
        const float mn = *cmaxnorm;
        const float bound = 4e-4f * sqrtf(qs) * mn + 2e-5f * (mn * mn + qs + fabsf(vlast)) + 1e-30f;
        exact = key_dist(kp) < vlast - bound;
      }
    }
    flags[qi] = exact ? 0 : 1;
  }
}

// Exact row for each flagged query (rare): the reference's sequential FP32
// distance to every centroid, written over the query's row of the
// approximate matrix, then the P smallest (distance, centroid).
__global__ void __launch_bounds__(256) coarse_fallback_kernel(const float* __restrict__ q, int nq, int dpad,
                                                              const float* __restrict__ cent, int nlist, int P,
                                                              const int* __restrict__ flags, float* __restrict__ V,
                                                              int32_t* __restrict__ probes, float* __restrict__ cdist,
                                                              const int32_t* __restrict__ width,
                                                              uint32_t* __restrict__ cmins) {
  extern __shared__ uint64_t s_fb[];
  __shared__ SelectShared sh_sel;
  __shared__ unsigned s_mask;
  // Flagged queries are rare: a small grid strides over chunks of 32
  // queries, one warp reading their flags at once.
  for (int q0 = blockIdx.x * 32; q0 < nq; q0 += gridDim.x * 32) {
    if (threadIdx.x < 32) {
      const unsigned b = __ballot_sync(0xffffffffu, q0 + static_cast<int>(threadIdx.x) < nq && flags[q0 + threadIdx.x] != 0);
      if (threadIdx.x == 0) s_mask = b;
    }
    __syncthreads();
    unsigned mask = s_mask;
    __syncthreads();
    while (mask) {
      const int qi = q0 + __ffs(mask) - 1;
      mask &= mask - 1;
      const float* qrow = q + static_cast<size_t>(qi) * dpad;
      float* row = V + static_cast<size_t>(qi) * nlist;
      // The row is overwritten with exact values, and so are its chunk
      // minima (a warp's 32 consecutive columns are two 16-column chunks).
      for (int c0 = 0; c0 < nlist; c0 += blockDim.x) {
        const int c = c0 + static_cast<int>(threadIdx.x);
        float acc = FLT_MAX;
        if (c < nlist) {
          const float* x = cent + static_cast<size_t>(c) * dpad;
          acc = 0.0f;
          for (int j = 0; j < dpad; ++j) {
            const float t = __fsub_rn(qrow[j], x[j]);
            acc = __fadd_rn(acc, __fmul_rn(t, t));
          }
          row[c] = acc;
        }
        uint32_t m = c < nlist ? __float_as_uint(acc) : 0xFFFFFFFFu;
        for (int o = 8; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (cmins && (threadIdx.x & 15) == 0 && c < nlist) cmins[static_cast<size_t>(c / 16) * nq + qi] = m;
      }
      __syncthreads();
      auto key_at = [&](int c) -> uint64_t {
        const float v = row[c];
        return v < FLT_MAX ? make_key(v, static_cast<uint32_t>(c)) : kEmpty;
      };
      const int Pr = width ? min(width[qi], P) : P;
      block_topk_sorted(key_at, nlist, P, sh_sel, s_fb);
      for (int j = threadIdx.x; j < P; j += blockDim.x) {
        const uint64_t key = j < Pr ? s_fb[j] : kEmpty;
        probes[static_cast<size_t>(qi) * P + j] = key == kEmpty ? -1 : static_cast<int32_t>(key_tie(key));
        if (cdist) cdist[static_cast<size_t>(qi) * P + j] = key == kEmpty ? FLT_MAX : key_dist(key);
      }
      __syncthreads();  // s_fb and the selection state are reused by the next query
    }
  }
}

// Candidate count of each row of the wider pass: 0 where the narrower pass
// already holds the row's width, else width + margin (at most nlist).
__global__ void coarse_widths_kernel(const int32_t* __restrict__ width, int nq, int wmax, int pre_w, int margin,
                                     int nlist, int32_t* __restrict__ kq) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nq) return;
  const int w = min(width[r], wmax);
  kq[r] = w <= pre_w ? 0 : min(nlist, w + coarse_extra_dev(w, margin));
}

}  // namespace

void launch_coarse_widths(const int32_t* width, int nq, int wmax, int pre_w, int margin, int nlist, int32_t* kq,
                          cudaStream_t st) {
  if (nq <= 0) return;
  coarse_widths_kernel<<<(nq + 255) / 256, 256, 0, st>>>(width, nq, wmax, pre_w, margin, nlist, kq);
  HB_CUDA(cudaGetLastError());
}

size_t coarse_tc_smem_bytes(int kpad) {
  return 1024 + static_cast<size_t>(2 * kpad / 64 + kCStages) * kBlk + static_cast<size_t>(kCEpiWarps) * 2 * kBoxBytes;
}

void make_centroid_split(const float* cent, int nlist, int dpad, int kpad, void* out, void* tmap_out, cudaStream_t st) {
  HB_CHECK(kpad == 64 || kpad == 128, HB_ERR_INVALID, "the tensor-core coarse quantizer supports d <= 128");
  if (nlist > 0) {
    const unsigned g = static_cast<unsigned>(std::min<int>((nlist + 7) / 8, 148 * 16));
    split_rows_kernel<<<g, 256, 0, st>>>(cent, nlist, dpad, kpad, static_cast<__nv_bfloat16*>(out), nullptr);
  }
  HB_CUDA(cudaGetLastError());
  make_bf16_tensor_map(tmap_out, out, static_cast<size_t>(nlist), 2 * kpad);
}

void launch_coarse_tc(const void* tmap, const float* q, int nq, int dpad, int kpad, const float* cnorm, int nlist,
                      float* V, void* qsplit, float* qnorm, uint32_t* cmins, int* err, int num_sms,
                      cudaStream_t st) {
  if (nq <= 0 || nlist <= 0) return;
  HB_CHECK(kpad == 64 || kpad == 128, HB_ERR_INVALID, "the tensor-core coarse quantizer supports d <= 128");
  // Query rows -> [hi | lo] BF16 and ||q||^2, then their tensor map.
  const unsigned g = static_cast<unsigned>(std::min<int>((nq + 7) / 8, 148 * 16));
  split_rows_kernel<<<g, 256, 0, st>>>(q, nq, dpad, kpad, static_cast<__nv_bfloat16*>(qsplit), qnorm);
  HB_CUDA(cudaGetLastError());
  alignas(64) unsigned char tmap_q[128];
  make_bf16_tensor_map(tmap_q, qsplit, static_cast<size_t>(nq), 2 * kpad);
  // V rows of 16-byte multiples go out by TMA stores; other widths by plain
  // stores.
  alignas(64) unsigned char tmap_v[128] = {};
  const int tma_v = (nlist & 3) == 0 ? 1 : 0;
  if (tma_v) make_f32_store_map(tmap_v, V, static_cast<size_t>(nq), static_cast<size_t>(nlist));
  const int qt = (nq + kCT - 1) / kCT;
  const int ct = (nlist + kCT - 1) / kCT;
  const int pairs = qt * ct;
  const int G = std::max(1, std::min(pairs, num_sms));
  const size_t smem = coarse_tc_smem_bytes(kpad);
  HB_CUDA(cudaFuncSetAttribute(coarse_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  coarse_tc_kernel<<<G, kCThreads, smem, st>>>(*static_cast<const CUtensorMap*>(tmap),
                                                *reinterpret_cast<const CUtensorMap*>(tmap_q),
                                                *reinterpret_cast<const CUtensorMap*>(tmap_v), tma_v, qnorm, nq, kpad,
                                                cnorm, nlist, qt, pairs, V, cmins, err);
  HB_CUDA(cudaGetLastError());
}

void launch_coarse_refine(const float* q, int nq, int dpad, const float* cent, const int32_t* cand, const float* cval,
                          int Pm, int P, int nlist, const float* cmaxnorm, int32_t* probes, float* cdist, int* flags,
                          cudaStream_t st, CoarseRows rows) {
  if (nq <= 0) return;
  HB_CHECK(P >= 1 && P <= Pm && Pm <= kCoarseMaxPm, HB_ERR_INVALID, "coarse candidate count out of range");
  HB_CHECK(dpad % 4 == 0 && dpad <= 128, HB_ERR_INVALID, "the coarse refinement stages rows of at most 128 floats");
  const int n2 = pow2_ceil(Pm < 2 ? 2 : Pm);
  const size_t stage = static_cast<size_t>(32) * kHalfStageStride * sizeof(float);  // per warp
  // A CTA per query for small batches, and for the widening pass of the
  // learned nprobe, whose few wide rows (up to Pm candidates) would
  // otherwise keep one warp each busy long after the narrow rows are done.
  if (nq < 512 || rows.width) {
    const size_t smem = static_cast<size_t>(n2) * 8;
    HB_CUDA(cudaFuncSetAttribute(coarse_refine_block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)));
    coarse_refine_block_kernel<<<nq, 256, smem, st>>>(q, nq, dpad, cent, cand, cval, Pm, P, nlist, cmaxnorm, probes,
                                                      cdist, flags, rows);
    HB_CUDA(cudaGetLastError());
    return;
  }
  // Four warps (one query each) per CTA: with the 32-row x 64-column stages,
  // six CTAs fit an SM.
  const int warps = 4;
  const size_t smem = static_cast<size_t>(warps) * (n2 * 8 + stage);
  HB_CUDA(cudaFuncSetAttribute(coarse_refine_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  coarse_refine_kernel<<<(nq + warps - 1) / warps, warps * 32, smem, st>>>(q, nq, dpad, cent, cand, cval, Pm, P, nlist,
                                                                          cmaxnorm, probes, cdist, flags, rows);
  HB_CUDA(cudaGetLastError());
}

void launch_coarse_fallback(const float* q, int nq, int dpad, const float* cent, int nlist, int P, const int* flags,
                            float* V, int32_t* probes, float* cdist, cudaStream_t st, const int32_t* width,
                            uint32_t* cmins) {
  if (nq <= 0) return;
  const size_t smem = static_cast<size_t>(pow2_ceil(P < 2 ? 2 : P)) * 8;
  HB_CUDA(cudaFuncSetAttribute(coarse_fallback_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  coarse_fallback_kernel<<<std::min((nq + 31) / 32, 296), 256, smem, st>>>(q, nq, dpad, cent, nlist, P, flags, V,
                                                                           probes, cdist, width, cmins);
  HB_CUDA(cudaGetLastError());
}

}  // namespace hb

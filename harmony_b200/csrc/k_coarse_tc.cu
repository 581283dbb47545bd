// Tensor-core coarse quantizer with an exact FP32 finish.
//
//  1. coarse_tc_kernel: queries and centroids are split into BF16 pairs
//     x = hi + lo (hi = bf16(x), lo = bf16(x - hi)); one tcgen05.mma chain
//     over K = 3 * kpad with A = [q_hi | q_hi | q_lo] and
//     B = [c_hi | c_lo | c_hi] gives q_hi.c_hi + q_hi.c_lo + q_lo.c_hi,
//     i.e. q.c to about 2^-16 relative (the 3-term BF16 split).  128
//     queries per CTA (A, K-major, 128-byte swizzle, built in shared memory
//     from the FP32 queries), 128 centroids per TMA tile streamed through a
//     ring of 64-column K blocks, accumulators double-buffered in TMEM.  The
//     epilogue writes v = max(0, ||q||^2 + ||c||^2 - 2 q.c) to an
//     nq x nlist matrix.
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
// <= 384 exact BF16 products adds <= 384 * 2^-23 * sum|q_i c_i|; with
// sum|q_i c_i| <= ||q|| ||c|| the dot error is < 6e-5 ||q|| ||c||, so
// 2 q.c is within 1.2e-4 ||q|| ||c||.  The norms, the FP32 combination and
// the reference's own FP32 rounding add < 1e-5 (||q||^2 + ||c||^2 + v).  The
// bound used, 4e-4 ||q|| max||c|| + 2e-5 (max||c||^2 + ||q||^2 + |v|), is
// more than three times that.
#include <cudaTypedefs.h>
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "hb_device.cuh"
#include "hb_internal.hpp"
#include "hb_select.cuh"
#include "hb_sm100.cuh"

namespace hb {
namespace {

using namespace sm100;

constexpr int kCT = 128;        // queries per CTA = centroids per tile
constexpr int kCStages = 6;     // ring of 64-column K blocks (16 KB each)
constexpr int kCThreads = 192;  // 4 epilogue warps, TMA warp, MMA warp
constexpr uint32_t kBlk = kCT * 128;  // bytes of one 128-row x 64-column BF16 block

struct CoarseShared {
  uint64_t full[kCStages];
  uint64_t empty[kCStages];
  uint64_t accf[2];
  uint64_t acce[2];
  uint32_t tmem;
};

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
  __nv_bfloat162 p = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&p);
}

__global__ void __launch_bounds__(kCThreads, 1)
    coarse_tc_kernel(const __grid_constant__ CUtensorMap tmap, const float* __restrict__ q, int nq, int dpad, int kpad,
                     const float* __restrict__ cnorm, int nlist, int tiles_per_cta, float* __restrict__ V,
                     int* __restrict__ err) {
  extern __shared__ uint8_t smem_raw[];
  __shared__ CoarseShared sh;
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int nkb = 3 * kpad / 64;  // K blocks per tile
  uint8_t* A = smem;
  uint8_t* ring = smem + static_cast<size_t>(nkb) * kBlk;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int q0 = blockIdx.x * kCT;
  const int t0 = blockIdx.y * tiles_per_cta;
  const int t1 = min((nlist + kCT - 1) / kCT, t0 + tiles_per_cta);
  const int ntiles = max(0, t1 - t0);

  if (warp == 5) tmem_alloc(&sh.tmem, 256);
  if (tid == 0) {
    for (int s = 0; s < kCStages; ++s) {
      mbar_init(&sh.full[s], 1);
      mbar_init(&sh.empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&sh.accf[b], 1);
      mbar_init(&sh.acce[b], 128);
    }
    fence_barrier_init();
  }
  float qn = 0.0f;
  if (tid < 128) {
    // Row tid of A: [hi | hi | lo] of query q0 + tid (zeros past nq / dpad).
    const int qi = q0 + tid;
    const float* qrow = q + static_cast<size_t>(qi < nq ? qi : 0) * dpad;
    const uint32_t kb_hi2 = static_cast<uint32_t>(kpad / 64) * kBlk;
    for (int k = 0; k < kpad; k += 8) {
      float x[8];
      if (qi < nq && k < dpad) {
        const float4 lo4 = *reinterpret_cast<const float4*>(qrow + k);
        const float4 hi4 = *reinterpret_cast<const float4*>(qrow + k + 4);
        x[0] = lo4.x, x[1] = lo4.y, x[2] = lo4.z, x[3] = lo4.w, x[4] = hi4.x, x[5] = hi4.y, x[6] = hi4.z, x[7] = hi4.w;
      } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) x[j] = 0.0f;
      }
      uint32_t h[4], l[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const float a = x[2 * j], b = x[2 * j + 1];
        qn = fmaf(a, a, qn);
        qn = fmaf(b, b, qn);
        const float ha = __bfloat162float(__float2bfloat16_rn(a)), hb_ = __bfloat162float(__float2bfloat16_rn(b));
        h[j] = pack_bf16x2(ha, hb_);
        l[j] = pack_bf16x2(a - ha, b - hb_);
      }
      const uint32_t off = sw128_offset_bf16(tid, k, kBlk);
      *reinterpret_cast<uint4*>(A + off) = make_uint4(h[0], h[1], h[2], h[3]);
      *reinterpret_cast<uint4*>(A + kb_hi2 + off) = make_uint4(h[0], h[1], h[2], h[3]);
      *reinterpret_cast<uint4*>(A + 2 * kb_hi2 + off) = make_uint4(l[0], l[1], l[2], l[3]);
    }
    fence_proxy_async_smem();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sh.tmem;

  if (warp == 4) {
    if (lane == 0) {
      int it = 0;
      for (int i = 0; i < ntiles; ++i) {
        for (int kb = 0; kb < nkb; ++kb, ++it) {
          const int s = it % kCStages;
          if (!mbar_wait(&sh.empty[s], ((it / kCStages) & 1u) ^ 1u, err, 21)) goto producer_done;
          mbar_arrive_expect_tx(&sh.full[s], kBlk);
          tma_load_2d(ring + static_cast<size_t>(s) * kBlk, &tmap, kb * 64, (t0 + i) * kCT, &sh.full[s]);
        }
      }
    producer_done:;
    }
  } else if (warp == 5) {
    if (lane == 0) {
      const uint32_t idesc = idesc_bf16_f32(kCT, kCT);
      const uint32_t abase = smem_u32(A), rbase = smem_u32(ring);
      int it = 0;
      int issued = 0;
      for (int i = 0; i < ntiles; ++i) {
        const int b = i & 1;
        if (!mbar_wait(&sh.acce[b], ((i >> 1) & 1u) ^ 1u, err, 23)) break;
        tc_fence_after();
        bool ok = true;
        for (int kb = 0; kb < nkb; ++kb, ++it) {
          const int s = it % kCStages;
          if (!mbar_wait(&sh.full[s], (it / kCStages) & 1u, err, 22)) {
            ok = false;
            break;
          }
          tc_fence_after();
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {
            mma_bf16(tmem + static_cast<uint32_t>(b * kCT),
                     desc_sw128(abase + static_cast<uint32_t>(kb) * kBlk + kk * 32u),
                     desc_sw128(rbase + static_cast<uint32_t>(s) * kBlk + kk * 32u), idesc,
                     (kb | kk) != 0 ? 1u : 0u);
          }
          mma_commit(&sh.empty[s]);
        }
        if (!ok) break;
        mma_commit(&sh.accf[b]);
        ++issued;
      }
      // Drain: the tensor cores must be done before TMEM is released.
      if (issued > 0) {
        const int l = issued - 1;
        mbar_wait(&sh.accf[l & 1], (l >> 1) & 1u, nullptr, 0, 200000000LL);
      }
    }
  } else {
    const int qi = q0 + tid;
    const uint32_t lane_base = (32u * static_cast<uint32_t>(warp)) << 16;
    bool ok = true;
    for (int i = 0; i < ntiles; ++i) {
      const int b = i & 1;
      if (ok) ok = mbar_wait(&sh.accf[b], (i >> 1) & 1u, err, 24);
      ok = __all_sync(0xffffffffu, ok);
      if (!ok) break;
      tc_fence_after();
      const int c0 = (t0 + i) * kCT;
#pragma unroll 1
      for (int c = 0; c < kCT / 32; ++c) {
        uint32_t r[32];
        tmem_ld32(tmem + lane_base + static_cast<uint32_t>(b * kCT + c * 32), r);
        tmem_ld_wait();
        if (qi < nq) {
          const int cb = c0 + c * 32;
          float* out = V + static_cast<size_t>(qi) * nlist + cb;
          if (nlist - cb >= 32 && (nlist & 3) == 0) {
#pragma unroll
            for (int j4 = 0; j4 < 8; ++j4) {
              const float4 cn = *reinterpret_cast<const float4*>(cnorm + cb + 4 * j4);
              float4 o;
              o.x = fmaxf(fmaf(-2.0f, __uint_as_float(r[4 * j4 + 0]), qn + cn.x), 0.0f);
              o.y = fmaxf(fmaf(-2.0f, __uint_as_float(r[4 * j4 + 1]), qn + cn.y), 0.0f);
              o.z = fmaxf(fmaf(-2.0f, __uint_as_float(r[4 * j4 + 2]), qn + cn.z), 0.0f);
              o.w = fmaxf(fmaf(-2.0f, __uint_as_float(r[4 * j4 + 3]), qn + cn.w), 0.0f);
              *reinterpret_cast<float4*>(out + 4 * j4) = o;
            }
          } else {
#pragma unroll
            for (int j = 0; j < 32; ++j)
              if (cb + j < nlist) out[j] = fmaxf(fmaf(-2.0f, __uint_as_float(r[j]), qn + cnorm[cb + j]), 0.0f);
          }
        }
      }
      tc_fence_before();
      mbar_arrive(&sh.acce[b]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 5) {
    tc_fence_after();
    tmem_dealloc(tmem, 256);
  }
}

// Centroid rows -> [hi | lo | hi] BF16 rows of 3 * kpad (zeros past d).
__global__ void split3_kernel(const float* __restrict__ c, int n, int dpad, int kpad, __nv_bfloat16* __restrict__ out) {
  const size_t total = static_cast<size_t>(n) * kpad;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const size_t r = i / kpad;
    const int k = static_cast<int>(i % kpad);
    const float x = k < dpad ? c[r * dpad + k] : 0.0f;
    const __nv_bfloat16 h = __float2bfloat16_rn(x);
    const __nv_bfloat16 l = __float2bfloat16_rn(x - __bfloat162float(h));
    __nv_bfloat16* o = out + r * 3 * kpad;
    o[k] = h;
    o[kpad + k] = l;
    o[2 * kpad + k] = h;
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
  extern __shared__ uint64_t s_ref[];  // [warps][pow2(Pm)]
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
  uint64_t* buf = s_ref + static_cast<size_t>(wib) * pow2_ceil(Pm < 2 ? 2 : Pm);
  const float* qrow = q + static_cast<size_t>(qi) * dpad;
  float qn = 0.0f;
  for (int c = lane * 4; c < dpad; c += 128) {
    const float4 v = *reinterpret_cast<const float4*>(qrow + c);
    qn += v.x * v.x + v.y * v.y + v.z * v.z + v.w * v.w;
  }
  for (int o = 16; o > 0; o >>= 1) qn += __shfl_xor_sync(0xffffffffu, qn, o);
  for (int i = lane; i < n2; i += 32) {
    uint64_t key = kEmpty;
    if (i < Pmr) {
      const int c = cand[static_cast<size_t>(qi) * Pm + i];
      if (c >= 0) {
        const float* x = cent + static_cast<size_t>(c) * dpad;
        float acc = 0.0f;
#pragma unroll 8
        for (int j = 0; j < dpad; j += 4) {
          const float4 v = *reinterpret_cast<const float4*>(x + j);
          const float4 w = *reinterpret_cast<const float4*>(qrow + j);
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
        if (acc < FLT_MAX) key = make_key(acc, static_cast<uint32_t>(c));
      }
    }
    buf[i] = key;
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
        const float* x = cent + static_cast<size_t>(c) * dpad;
        float acc = 0.0f;
#pragma unroll 8
        for (int j = 0; j < dpad; j += 4) {
          const float4 v = *reinterpret_cast<const float4*>(x + j);
          const float4 w = *reinterpret_cast<const float4*>(qrow + j);
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
                                                              const int32_t* __restrict__ width) {
  extern __shared__ uint64_t s_fb[];
  __shared__ SelectShared sh_sel;
  const int qi = blockIdx.x;
  if (qi >= nq || !flags[qi]) return;
  const float* qrow = q + static_cast<size_t>(qi) * dpad;
  float* row = V + static_cast<size_t>(qi) * nlist;
  for (int c = threadIdx.x; c < nlist; c += blockDim.x) {
    const float* x = cent + static_cast<size_t>(c) * dpad;
    float acc = 0.0f;
    for (int j = 0; j < dpad; ++j) {
      const float t = __fsub_rn(qrow[j], x[j]);
      acc = __fadd_rn(acc, __fmul_rn(t, t));
    }
    row[c] = acc;
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
  return 1024 + static_cast<size_t>(3 * kpad / 64 + kCStages) * kBlk;
}

void make_centroid_split(const float* cent, int nlist, int dpad, int kpad, void* out, void* tmap_out, cudaStream_t st) {
  HB_CHECK(kpad == 64 || kpad == 128, HB_ERR_INVALID, "the tensor-core coarse quantizer supports d <= 128");
  const size_t total = static_cast<size_t>(nlist) * kpad;
  const unsigned g = static_cast<unsigned>(std::min<size_t>((total + 255) / 256, 148u * 16u));
  if (total) split3_kernel<<<g, 256, 0, st>>>(cent, nlist, dpad, kpad, static_cast<__nv_bfloat16*>(out));
  HB_CUDA(cudaGetLastError());
  make_bf16_tensor_map(tmap_out, out, static_cast<size_t>(nlist), 3 * kpad);
}

void launch_coarse_tc(const void* tmap, const float* q, int nq, int dpad, int kpad, const float* cnorm, int nlist,
                      float* V, int* err, int num_sms, cudaStream_t st) {
  if (nq <= 0 || nlist <= 0) return;
  HB_CHECK(kpad == 64 || kpad == 128, HB_ERR_INVALID, "the tensor-core coarse quantizer supports d <= 128");
  const int qt = (nq + kCT - 1) / kCT;
  const int ct = (nlist + kCT - 1) / kCT;
  int split = std::max(1, std::min(ct, (2 * num_sms + qt - 1) / qt));
  const int per = (ct + split - 1) / split;
  split = (ct + per - 1) / per;
  const size_t smem = coarse_tc_smem_bytes(kpad);
  HB_CUDA(cudaFuncSetAttribute(coarse_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  coarse_tc_kernel<<<dim3(qt, split), kCThreads, smem, st>>>(*static_cast<const CUtensorMap*>(tmap), q, nq, dpad, kpad,
                                                            cnorm, nlist, per, V, err);
  HB_CUDA(cudaGetLastError());
}

void launch_coarse_refine(const float* q, int nq, int dpad, const float* cent, const int32_t* cand, const float* cval,
                          int Pm, int P, int nlist, const float* cmaxnorm, int32_t* probes, float* cdist, int* flags,
                          cudaStream_t st, CoarseRows rows) {
  if (nq <= 0) return;
  HB_CHECK(P >= 1 && P <= Pm && Pm <= kCoarseMaxPm, HB_ERR_INVALID, "coarse candidate count out of range");
  const int n2 = pow2_ceil(Pm < 2 ? 2 : Pm);
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
  const int warps = std::max(1, std::min(8, 65536 / (n2 * 8)));
  const size_t smem = static_cast<size_t>(warps) * n2 * 8;
  HB_CUDA(cudaFuncSetAttribute(coarse_refine_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  coarse_refine_kernel<<<(nq + warps - 1) / warps, warps * 32, smem, st>>>(q, nq, dpad, cent, cand, cval, Pm, P, nlist,
                                                                          cmaxnorm, probes, cdist, flags, rows);
  HB_CUDA(cudaGetLastError());
}

void launch_coarse_fallback(const float* q, int nq, int dpad, const float* cent, int nlist, int P, const int* flags,
                            float* V, int32_t* probes, float* cdist, cudaStream_t st, const int32_t* width) {
  if (nq <= 0) return;
  const size_t smem = static_cast<size_t>(pow2_ceil(P < 2 ? 2 : P)) * 8;
  HB_CUDA(cudaFuncSetAttribute(coarse_fallback_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  coarse_fallback_kernel<<<nq, 256, smem, st>>>(q, nq, dpad, cent, nlist, P, flags, V, probes, cdist, width);
  HB_CUDA(cudaGetLastError());
}

}  // namespace hb

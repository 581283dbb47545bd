// Learned probe predictor: the kernels of a small MLP (no reference
// counterpart) that predicts, per query, how many lists to probe.
//
// Features (feature_kernel): the query's d components and the log distances
// to its 32 nearest centroids (the nearest as log d0, the others relative to
// it), standardised with training-set mean / std.
// Network: F -> 256 -> 256 -> NB, GELU between layers, NB classes = nprobe
// buckets.  Training runs in FP32 (master weights, Adam); the weights used
// for inference are rounded to BF16 and so are the activations between
// layers, i.e. the predictor is a BF16 MLP with FP32 accumulation.
//
// gemm_kernel is a 64x64-tile SIMT GEMM with optional transposes, fused
// bias + GELU epilogue, used for every layer forward and backward.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>

#include "hb_device.cuh"
#include "hb_internal.hpp"
#include "hb_sm100.cuh"

namespace hb {
namespace {

constexpr int kT = 64;       // tile
constexpr int kKT = 16;      // k tile
constexpr int kGemmThreads = 256;

__device__ __forceinline__ float gelu_f(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
  const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
  return cdf + x * pdf;
}
__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// C[m][n] = sum_k A(m,k) B(k,n) (+ bias[n]) (+ beta * C), optional GELU with
// the pre-activation kept in Z.  A(m,k) = tA ? A[k*lda+m] : A[m*lda+k];
// B(k,n) = tB ? B[n*ldb+k] : B[k*ldb+n].
__global__ void __launch_bounds__(kGemmThreads) gemm_kernel(int M, int N, int K, const float* __restrict__ A, int lda,
                                                            int tA, const float* __restrict__ B, int ldb, int tB,
                                                            float* __restrict__ C, int ldc, const float* __restrict__ bias,
                                                            float beta, int act, float* __restrict__ Z, int round_bf16) {
  __shared__ float sA[kKT][kT + 1];
  __shared__ float sB[kKT][kT + 1];
  const int m0 = blockIdx.y * kT, n0 = blockIdx.x * kT;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;  // 16 x 16 threads, 4 x 4 outputs each
  float acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += kKT) {
    // Consecutive threads walk each operand's contiguous dimension.
    for (int i = threadIdx.x; i < kKT * kT; i += kGemmThreads) {
      {
        const int kk = tA ? i / kT : i % kKT, mm = tA ? i % kT : i / kKT;
        const int m = m0 + mm, k = k0 + kk;
        float va = 0.f;
        if (m < M && k < K) va = tA ? A[static_cast<size_t>(k) * lda + m] : A[static_cast<size_t>(m) * lda + k];
        sA[kk][mm] = va;
      }
      {
        const int kk = tB ? i % kKT : i / kT, nn = tB ? i / kKT : i % kT;
        const int n = n0 + nn, k = k0 + kk;
        float vb = 0.f;
        if (n < N && k < K) vb = tB ? B[static_cast<size_t>(n) * ldb + k] : B[static_cast<size_t>(k) * ldb + n];
        sB[kk][nn] = vb;
      }
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kKT; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        a[i] = sA[kk][ty * 4 + i];
        b[i] = sB[kk][tx * 4 + i];
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + ty * 4 + i;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int n = n0 + tx * 4 + j;
      if (n >= N) continue;
      float v = acc[i][j];
      if (bias) v += bias[n];
      const size_t o = static_cast<size_t>(m) * ldc + n;
      if (beta != 0.f) v += beta * C[o];
      if (Z) Z[o] = v;
      if (act) v = gelu_f(v);
      if (round_bf16) v = bf16r(v);
      C[o] = v;
    }
  }
}

// dZ = dH * gelu'(Z)
__global__ void gelu_backward_kernel(const float* __restrict__ dH, const float* __restrict__ Z, float* __restrict__ dZ,
                                     size_t n) {
  const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
  if (i < n) dZ[i] = dH[i] * gelu_grad(Z[i]);
}

// Per row: softmax cross-entropy gradient (p - onehot) / B, loss summed.
__global__ void softmax_ce_kernel(const float* __restrict__ logits, const int32_t* __restrict__ labels, int B, int NB,
                                  float* __restrict__ dlogits, float* __restrict__ loss) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= B) return;
  const float* z = logits + static_cast<size_t>(r) * NB;
  float mx = -INFINITY;
  for (int j = 0; j < NB; ++j) mx = fmaxf(mx, z[j]);
  float s = 0.f;
  for (int j = 0; j < NB; ++j) s += expf(z[j] - mx);
  const int y = labels[r];
  for (int j = 0; j < NB; ++j) {
    const float p = expf(z[j] - mx) / s;
    dlogits[static_cast<size_t>(r) * NB + j] = (p - (j == y ? 1.f : 0.f)) / static_cast<float>(B);
  }
  atomicAdd(loss, -(z[y] - mx - logf(s)));
}

// db[n] = sum over rows of dY[r][n]
__global__ void colsum_kernel(const float* __restrict__ dY, int B, int N, float* __restrict__ db) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float s = 0.f;
  for (int r = 0; r < B; ++r) s += dY[static_cast<size_t>(r) * N + n];
  db[n] = s;
}

__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, size_t n, float lr, float b1, float b2, float eps, float c1,
                            float c2, float wd) {
  const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i] + wd * w[i];
  m[i] = b1 * m[i] + (1.f - b1) * gi;
  v[i] = b2 * v[i] + (1.f - b2) * gi * gi;
  w[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps);
}

__global__ void round_bf16_kernel(const float* __restrict__ src, float* __restrict__ dst, size_t n) {
  const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
  if (i < n) dst[i] = bf16r(src[i]);
}

// Raw features: query components then log centroid distances.
__global__ void feature_kernel(const float* __restrict__ q, int nq, int d, int dpad, const float* __restrict__ cdist,
                               int P, int C, float* __restrict__ out) {
  const int F = d + C;
  const size_t total = static_cast<size_t>(nq) * F;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int r = static_cast<int>(i / F);
    const int f = static_cast<int>(i - static_cast<size_t>(r) * F);
    float v;
    if (f < d) {
      v = q[static_cast<size_t>(r) * dpad + f];
    } else {
      const int j = f - d;
      const float* cd = cdist + static_cast<size_t>(r) * P;
      const float l0 = logf(fmaxf(cd[0], 1e-20f));
      if (j == 0) {
        v = l0;
      } else {
        const float dj = j < P ? cd[j] : cd[P - 1];
        v = dj < FLT_MAX ? logf(fmaxf(dj, 1e-20f)) - l0 : 0.f;
      }
    }
    out[i] = v;
  }
}

// x = (x - mean) / std per column, then rounded to BF16 when asked.
__global__ void standardize_kernel(float* __restrict__ x, int rows, int F, const float* __restrict__ mean,
                                   const float* __restrict__ inv_std, int round) {
  const size_t total = static_cast<size_t>(rows) * F;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int f = static_cast<int>(i % F);
    float v = (x[i] - mean[f]) * inv_std[f];
    x[i] = round ? bf16r(v) : v;
  }
}

// Column mean and 1/std over rows (one block per column).
__global__ void moments_kernel(const float* __restrict__ x, int rows, int F, float* __restrict__ mean,
                               float* __restrict__ inv_std) {
  const int f = blockIdx.x;
  double s = 0.0, s2 = 0.0;
  for (int r = threadIdx.x; r < rows; r += blockDim.x) {
    const double v = x[static_cast<size_t>(r) * F + f];
    s += v;
    s2 += v * v;
  }
  __shared__ double ss[256], ss2[256];
  ss[threadIdx.x] = s;
  ss2[threadIdx.x] = s2;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      ss[threadIdx.x] += ss[threadIdx.x + o];
      ss2[threadIdx.x] += ss2[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double m = ss[0] / rows;
    const double var = fmax(ss2[0] / rows - m * m, 1e-12);
    mean[f] = static_cast<float>(m);
    inv_std[f] = static_cast<float>(1.0 / sqrt(var));
  }
}

// Per query: the smallest bucket whose predicted cumulative probability
// reaches `thr`; nprobe = bucket value (capped).  Probes past it become -1.
__global__ void choose_nprobe_kernel(const float* __restrict__ logits, int nq, int NB,
                                     const int32_t* __restrict__ bucket_val, float thr, int cap,
                                     int32_t* __restrict__ nprobe_out, int32_t* __restrict__ probes, int P) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nq) return;
  const float* z = logits + static_cast<size_t>(r) * NB;
  float mx = -INFINITY;
  for (int j = 0; j < NB; ++j) mx = fmaxf(mx, z[j]);
  float s = 0.f;
  for (int j = 0; j < NB; ++j) s += expf(z[j] - mx);
  float c = 0.f;
  int pick = bucket_val[NB - 1];
  for (int j = 0; j < NB; ++j) {
    c += expf(z[j] - mx) / s;
    if (c >= thr) {
      pick = bucket_val[j];
      break;
    }
  }
  pick = min(pick, cap);
  if (nprobe_out) nprobe_out[r] = pick;
  if (probes)
    for (int j = pick; j < P; ++j) probes[static_cast<size_t>(r) * P + j] = -1;
}

// Cut each query's probe row at its own nprobe (host- or model-given).
__global__ void cut_probes_kernel(const int32_t* __restrict__ nprobe, int nq, int P, int32_t* __restrict__ probes) {
  const size_t total = static_cast<size_t>(nq) * P;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int r = static_cast<int>(i / P);
    const int j = static_cast<int>(i - static_cast<size_t>(r) * P);
    if (j >= nprobe[r]) probes[i] = -1;
  }
}

// Label of a training query: 1 + the highest probe rank among the lists that
// hold its k results (the smallest nprobe that reproduces them).
__global__ void label_rank_kernel(const int64_t* __restrict__ I, int nq, int k, const int32_t* __restrict__ list_of_id,
                                  const int32_t* __restrict__ probes, int P, int32_t* __restrict__ need,
                                  int32_t* __restrict__ ranks) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nq) return;
  int mx = 0;
  for (int j = 0; j < k; ++j) {
    const int64_t id = I[static_cast<size_t>(r) * k + j];
    int rank = P;  // missing result: needs the full probe range
    if (id >= 0) {
      const int l = list_of_id[id];
      for (int p = 0; p < P; ++p)
        if (probes[static_cast<size_t>(r) * P + p] == l) {
          rank = p;
          break;
        }
    }
    if (ranks) ranks[static_cast<size_t>(r) * k + j] = rank;
    mx = max(mx, rank + 1);
  }
  need[r] = min(mx, P);
}

__global__ void list_of_id_kernel(const int64_t* __restrict__ list_off, int nlist, const int64_t* __restrict__ ids,
                                  int32_t* __restrict__ out, int64_t max_id) {
  const int l = blockIdx.x;
  for (int64_t p = list_off[l] + threadIdx.x; p < list_off[l + 1]; p += blockDim.x) {
    const int64_t id = ids[p];
    if (id >= 0 && id < max_id) out[id] = l;
  }
}

inline unsigned blocks_for(size_t n, int tb = 256, unsigned cap = 148u * 64u) {
  size_t g = (n + tb - 1) / tb;
  return static_cast<unsigned>(g < 1 ? 1 : (g > cap ? cap : g));
}

// ---------------------------------------------------------------------------
// Fused predictor inference on the tensor cores: one CTA per 128 queries
// builds the standardized BF16 features in shared memory (A, K-major,
// 128-byte swizzle), runs the three layers as tcgen05.mma chains (M 128 x
// N 256 / 32 x K 16) into TMEM with the BF16 weights staged in shared memory,
// applies bias + GELU + BF16 rounding between layers (written back as the
// next layer's A operand) and ends with the bucket choice.  Same arithmetic
// as the SIMT path (BF16 operands, FP32 accumulation, BF16 activations); the
// accumulation order differs.

using namespace sm100;

constexpr int kMlpRows = 128;
constexpr int kMlpThreads = 512;

// W (N x K FP32, BF16-valued) -> Wb, the shared-memory image of the layer's
// B operand: Npad rows x Kpad BF16 (zero padding), K-major in 64-column
// blocks with the 128-byte swizzle, so the kernel stages it with one bulk
// copy.
__global__ void pack_bf16_kernel(const float* __restrict__ W, int N, int K, int Npad, int Kpad,
                                 __nv_bfloat16* __restrict__ out) {
  const size_t total = static_cast<size_t>(Npad) * Kpad;
  const uint32_t kblk = static_cast<uint32_t>(Npad) * 128u;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int n = static_cast<int>(i / Kpad), k = static_cast<int>(i % Kpad);
    out[sw128_offset_bf16(n, k, kblk) / 2] =
        __float2bfloat16_rn(n < N && k < K ? W[static_cast<size_t>(n) * K + k] : 0.0f);
  }
}

// Stages a packed weight image (bytes, a multiple of 16) with one bulk copy
// completing on bar (thread 0 issues).
__device__ __forceinline__ void stage_weights(uint8_t* dst, const __nv_bfloat16* __restrict__ Wb, uint32_t bytes,
                                              uint64_t* bar) {
  if (threadIdx.x == 0) {
    mbar_arrive_expect_tx(bar, bytes);
    bulk_load(dst, Wb, bytes, bar);
  }
}

__device__ __forceinline__ uint32_t pack2_bf16(float a, float b) {
  __nv_bfloat162 p = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&p);
}

// One layer: D[tmem] = A (128 x K) x W^T (N x K); issued by thread 0, all
// threads wait for completion.
__device__ __forceinline__ bool mlp_mma(uint32_t tmem, const uint8_t* A, const uint8_t* W, int N, int K,
                                        uint64_t* bar, uint32_t parity, int* err) {
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (threadIdx.x == 0) {
    const uint32_t idesc = idesc_bf16_f32(kMlpRows, N);
    const uint32_t a0 = smem_u32(A), w0 = smem_u32(W);
    for (int k = 0; k < K / 16; ++k) {
      const uint32_t oa = static_cast<uint32_t>(k >> 2) * (kMlpRows * 128u) + static_cast<uint32_t>(k & 3) * 32u;
      const uint32_t ow = static_cast<uint32_t>(k >> 2) * (static_cast<uint32_t>(N) * 128u) +
                          static_cast<uint32_t>(k & 3) * 32u;
      mma_bf16(tmem, desc_sw128(a0 + oa), desc_sw128(w0 + ow), idesc, k > 0 ? 1u : 0u);
    }
    mma_commit(bar);
  }
  const bool ok = mbar_wait(bar, parity, err, 41);
  tc_fence_after();
  return ok;
}

__global__ void __launch_bounds__(kMlpThreads, 1) probe_mlp_tc_kernel(
    const float* __restrict__ q, int nq, int d, int dpad, const float* __restrict__ cdist, int P, int C,
    const float* __restrict__ mean, const float* __restrict__ inv_std, int K1, const __nv_bfloat16* __restrict__ W1b,
    const float* __restrict__ b1, const __nv_bfloat16* __restrict__ W2b, const float* __restrict__ b2,
    const __nv_bfloat16* __restrict__ W3b, const float* __restrict__ b3, int NB, const int32_t* __restrict__ bucket_val,
    float thr, int cap, int32_t* __restrict__ nprobe_out, int* __restrict__ err) {
  extern __shared__ uint8_t mlp_raw[];
  __shared__ uint64_t bar, wbar;
  __shared__ uint32_t s_tmem;
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(mlp_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* A = smem;                       // 128 x 256 BF16 (64 KB)
  uint8_t* W = smem + kMlpRows * 256 * 2;  // up to 256 x 256 BF16 (128 KB)
  const int tid = threadIdx.x, warp = tid >> 5;
  const int r0 = blockIdx.x * kMlpRows;
  const uint32_t akblk = kMlpRows * 128u;
  if (warp == 0) tmem_alloc(&s_tmem, 256);
  if (tid == 0) {
    mbar_init(&bar, 1);
    mbar_init(&wbar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  // Layer-1 weights (in flight while the features are formed).
  stage_weights(W, W1b, 256u * static_cast<uint32_t>(K1) * 2u, &wbar);
  uint32_t wpar = 0;
  // The features: a warp per row, lanes over the features, so the query's
  // coordinates and its centroid distances are read coalesced.
  {
    const int F = d + C;
    const int lane = tid & 31;
    for (int row = warp; row < kMlpRows; row += kMlpThreads / 32) {
      const int r = r0 + row;
      const bool live = r < nq;
      const float* qrow = q + static_cast<size_t>(live ? r : 0) * dpad;
      const float* cd = cdist + static_cast<size_t>(live ? r : 0) * P;
      const float l0 = logf(fmaxf(cd[0], 1e-20f));
      for (int f = lane; f < K1; f += 32) {
        float x = 0.0f;
        if (live && f < F) {
          if (f < d) {
            x = qrow[f];
          } else {
            const int c = f - d;
            if (c == 0) {
              x = l0;
            } else {
              const float dj = c < P ? cd[c] : cd[P - 1];
              x = dj < FLT_MAX ? logf(fmaxf(dj, 1e-20f)) - l0 : 0.f;
            }
          }
          x = bf16r((x - mean[f]) * inv_std[f]);
        }
        *reinterpret_cast<__nv_bfloat16*>(A + sw128_offset_bf16(row, f, akblk)) = __float2bfloat16_rn(x);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  // Epilogue mapping: warp w reads TMEM lanes 32 * (w % 4) (rows), columns
  // [64 * (w / 4), +64).
  const int row = (warp & 3) * 32 + (tid & 31);
  const int cbase = (warp >> 2) * 64;
  const uint32_t taddr = tmem + ((32u * static_cast<uint32_t>(warp & 3)) << 16);
  bool ok = true;
  uint32_t parity = 0;
  // Layers 1 and 2: bias + GELU + BF16 back into A; the next layer's weights
  // are copied in while this layer's epilogue runs.
  for (int layer = 0; layer < 2 && ok; ++layer) {
    ok = mbar_wait(&wbar, wpar, err, 42);
    wpar ^= 1u;
    ok = ok && mlp_mma(tmem, A, W, 256, layer == 0 ? K1 : 256, &bar, parity, err);
    parity ^= 1u;
    ok = __syncthreads_and(ok);
    if (!ok) break;
    stage_weights(W, layer == 0 ? W2b : W3b, (layer == 0 ? 256u : 32u) * 256u * 2u, &wbar);
    const float* bias = layer == 0 ? b1 : b2;
    for (int c = 0; c < 2; ++c) {
      uint32_t rr[32];
      tmem_ld32(taddr + static_cast<uint32_t>(cbase + c * 32), rr);
      tmem_ld_wait();
#pragma unroll
      for (int j8 = 0; j8 < 4; ++j8) {
        float v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int n = cbase + c * 32 + j8 * 8 + j;
          v[j] = bf16r(gelu_f(__uint_as_float(rr[j8 * 8 + j]) + bias[n]));
        }
        *reinterpret_cast<uint4*>(A + sw128_offset_bf16(row, cbase + c * 32 + j8 * 8, akblk)) =
            make_uint4(pack2_bf16(v[0], v[1]), pack2_bf16(v[2], v[3]), pack2_bf16(v[4], v[5]),
                       pack2_bf16(v[6], v[7]));
      }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
  }
  // Layer 3 (N 32, NB used) and the bucket choice: the smallest bucket whose
  // predicted CDF reaches thr.
  if (ok) ok = __syncthreads_and(mbar_wait(&wbar, wpar, err, 42) && mlp_mma(tmem, A, W, 32, 256, &bar, parity, err));
  if (ok && warp < 4) {
    uint32_t rr[32];
    tmem_ld32(taddr, rr);
    tmem_ld_wait();
    const int r = r0 + row;
    if (r < nq) {
      float z[32];
      float mx = -INFINITY;
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        z[j] = j < NB ? __uint_as_float(rr[j]) + b3[j] : -INFINITY;
        mx = fmaxf(mx, z[j]);
      }
      float sum = 0.f;
#pragma unroll
      for (int j = 0; j < 32; ++j)
        if (j < NB) sum += expf(z[j] - mx);
      float cum = 0.f;
      int pick = bucket_val[NB - 1];
      bool found = false;
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        if (j < NB && !found) {
          cum += expf(z[j] - mx) / sum;
          if (cum >= thr) {
            pick = bucket_val[j];
            found = true;
          }
        }
      }
      nprobe_out[r] = min(pick, cap);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, 256);
  }
}

}  // namespace

void mlp_gemm(int M, int N, int K, const float* A, int lda, bool tA, const float* B, int ldb, bool tB, float* C, int ldc,
              const float* bias, float beta, bool gelu, float* Z, bool round_bf16, cudaStream_t st) {
  if (M <= 0 || N <= 0) return;
  dim3 grid((N + kT - 1) / kT, (M + kT - 1) / kT);
  gemm_kernel<<<grid, kGemmThreads, 0, st>>>(M, N, K, A, lda, tA ? 1 : 0, B, ldb, tB ? 1 : 0, C, ldc, bias, beta,
                                             gelu ? 1 : 0, Z, round_bf16 ? 1 : 0);
  HB_CUDA(cudaGetLastError());
}

void mlp_gelu_backward(const float* dH, const float* Z, float* dZ, size_t n, cudaStream_t st) {
  gelu_backward_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(dH, Z, dZ, n);
  HB_CUDA(cudaGetLastError());
}

void mlp_softmax_ce(const float* logits, const int32_t* labels, int B, int NB, float* dlogits, float* loss,
                    cudaStream_t st) {
  softmax_ce_kernel<<<(B + 127) / 128, 128, 0, st>>>(logits, labels, B, NB, dlogits, loss);
  HB_CUDA(cudaGetLastError());
}

void mlp_colsum(const float* dY, int B, int N, float* db, cudaStream_t st) {
  colsum_kernel<<<(N + 127) / 128, 128, 0, st>>>(dY, B, N, db);
  HB_CUDA(cudaGetLastError());
}

void mlp_adam(float* w, const float* g, float* m, float* v, size_t n, float lr, int step, float wd, cudaStream_t st) {
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - std::pow(b1, static_cast<float>(step));
  const float c2 = 1.f - std::pow(b2, static_cast<float>(step));
  adam_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(w, g, m, v, n, lr, b1, b2, 1e-8f, c1, c2, wd);
  HB_CUDA(cudaGetLastError());
}

void mlp_round_bf16(const float* src, float* dst, size_t n, cudaStream_t st) {
  round_bf16_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(src, dst, n);
  HB_CUDA(cudaGetLastError());
}

void mlp_features(const float* q, int nq, int d, int dpad, const float* cdist, int P, int C, float* out,
                  cudaStream_t st) {
  feature_kernel<<<blocks_for(static_cast<size_t>(nq) * (d + C)), 256, 0, st>>>(q, nq, d, dpad, cdist, P, C, out);
  HB_CUDA(cudaGetLastError());
}

void mlp_moments(const float* x, int rows, int F, float* mean, float* inv_std, cudaStream_t st) {
  moments_kernel<<<F, 256, 0, st>>>(x, rows, F, mean, inv_std);
  HB_CUDA(cudaGetLastError());
}

void mlp_standardize(float* x, int rows, int F, const float* mean, const float* inv_std, bool round_bf16,
                     cudaStream_t st) {
  standardize_kernel<<<blocks_for(static_cast<size_t>(rows) * F), 256, 0, st>>>(x, rows, F, mean, inv_std,
                                                                               round_bf16 ? 1 : 0);
  HB_CUDA(cudaGetLastError());
}

void mlp_choose_nprobe(const float* logits, int nq, int NB, const int32_t* bucket_val, float thr, int cap,
                       int32_t* nprobe_out, int32_t* probes, int P, cudaStream_t st) {
  choose_nprobe_kernel<<<(nq + 127) / 128, 128, 0, st>>>(logits, nq, NB, bucket_val, thr, cap, nprobe_out, probes, P);
  HB_CUDA(cudaGetLastError());
}

void launch_cut_probes(const int32_t* nprobe, int nq, int P, int32_t* probes, cudaStream_t st) {
  cut_probes_kernel<<<blocks_for(static_cast<size_t>(nq) * P), 256, 0, st>>>(nprobe, nq, P, probes);
  HB_CUDA(cudaGetLastError());
}

void launch_label_rank(const int64_t* I, int nq, int k, const int32_t* list_of_id, const int32_t* probes, int P,
                       int32_t* need, int32_t* ranks, cudaStream_t st) {
  label_rank_kernel<<<(nq + 127) / 128, 128, 0, st>>>(I, nq, k, list_of_id, probes, P, need, ranks);
  HB_CUDA(cudaGetLastError());
}

void launch_list_of_id(const int64_t* list_off, int nlist, const int64_t* ids, int32_t* out, int64_t max_id,
                       cudaStream_t st) {
  list_of_id_kernel<<<nlist, 128, 0, st>>>(list_off, nlist, ids, out, max_id);
  HB_CUDA(cudaGetLastError());
}

size_t probe_mlp_tc_smem_bytes() { return 1024 + kMlpRows * 256 * 2 + 256 * 256 * 2; }

void mlp_pack_bf16(const float* W, int N, int K, int Npad, int Kpad, void* out, cudaStream_t st) {
  const size_t total = static_cast<size_t>(Npad) * Kpad;
  pack_bf16_kernel<<<static_cast<unsigned>(std::min<size_t>((total + 255) / 256, 148u * 8u)), 256, 0, st>>>(
      W, N, K, Npad, Kpad, static_cast<__nv_bfloat16*>(out));
  HB_CUDA(cudaGetLastError());
}

void mlp_infer_tc(const float* q, int nq, int d, int dpad, const float* cdist, int P, int C, const float* mean,
                  const float* inv_std, int K1, const void* W1b, const float* b1, const void* W2b, const float* b2,
                  const void* W3b, const float* b3, int NB, const int32_t* bucket_val, float thr, int cap,
                  int32_t* nprobe_out, int* err, cudaStream_t st) {
  if (nq <= 0) return;
  HB_CHECK(K1 % 64 == 0 && K1 <= 256 && NB <= 32, HB_ERR_INVALID, "predictor shape outside the tensor-core path");
  const size_t smem = probe_mlp_tc_smem_bytes();
  HB_CUDA(cudaFuncSetAttribute(probe_mlp_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(smem)));
  probe_mlp_tc_kernel<<<(nq + kMlpRows - 1) / kMlpRows, kMlpThreads, smem, st>>>(
      q, nq, d, dpad, cdist, P, C, mean, inv_std, K1, static_cast<const __nv_bfloat16*>(W1b), b1,
      static_cast<const __nv_bfloat16*>(W2b), b2, static_cast<const __nv_bfloat16*>(W3b), b3, NB, bucket_val, thr, cap,
      nprobe_out, err);
  HB_CUDA(cudaGetLastError());
}

}  // namespace hb

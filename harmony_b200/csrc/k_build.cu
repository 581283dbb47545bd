// Index-building kernels: k-means update with FP64 centroid sums, list
// construction for Index::add, norms, and small layout helpers.
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>

#include "hb_device.cuh"
#include "hb_internal.hpp"

namespace hb {
namespace {

__global__ void pad_rows_kernel(const float* __restrict__ src, size_t n, int d, int dpad, float* __restrict__ dst) {
  const size_t total = n * static_cast<size_t>(dpad);
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const size_t r = i / dpad;
    const int c = static_cast<int>(i - r * dpad);
    dst[i] = c < d ? src[r * d + c] : 0.0f;
  }
}

__global__ void gather_rows_kernel(const float* __restrict__ src, const int64_t* __restrict__ idx, size_t n,
                                   int dpad, float* __restrict__ dst) {
  const int c4 = dpad / 4;
  const size_t total = n * c4;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const size_t r = i / c4;
    const int c = static_cast<int>(i - r * c4);
    reinterpret_cast<float4*>(dst)[r * c4 + c] =
        reinterpret_cast<const float4*>(src)[static_cast<size_t>(idx[r]) * c4 + c];
  }
}

// One warp per point: lanes sweep the dimensions so the FP64 atomics of a
// point hit consecutive addresses of its centroid row.
__global__ void kmeans_accumulate_kernel(const float* __restrict__ x, const int32_t* __restrict__ assign, size_t n,
                                         int d, int dpad, double* __restrict__ sums, int32_t* __restrict__ counts) {
  const size_t warp = (blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  const int c = assign[warp];
  const float* row = x + warp * dpad;
  double* srow = sums + static_cast<size_t>(c) * dpad;
  for (int j = lane; j < d; j += 32) atomicAdd(&srow[j], static_cast<double>(row[j]));
  if (lane == 0) atomicAdd(&counts[c], 1);
}

// centroid = float(sum) / float(count), as the reference divides its float
// column sums by the count (src/Clustering.cpp:146-150); empty clusters keep
// their centroid.
__global__ void kmeans_update_kernel(const double* __restrict__ sums, const int32_t* __restrict__ counts, int nlist,
                                     int d, int dpad, float* __restrict__ cent) {
  const size_t total = static_cast<size_t>(nlist) * d;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int c = static_cast<int>(i / d);
    const int j = static_cast<int>(i - static_cast<size_t>(c) * d);
    const int cnt = counts[c];
    if (cnt > 0)
      cent[static_cast<size_t>(c) * dpad + j] =
          __fdiv_rn(static_cast<float>(sums[static_cast<size_t>(c) * dpad + j]), static_cast<float>(cnt));
  }
}

// <x, x> with the reference's sequential inner-product loop
// (src/utils.h:511-518; norms of src/Index.cpp:689-696).
__global__ void row_norms_kernel(const float* __restrict__ x, size_t n, int d, int dpad, float* __restrict__ norms) {
  const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const float* r = x + i * dpad;
  float acc = 0.0f;
  for (int j = 0; j < d; ++j) acc = __fadd_rn(acc, __fmul_rn(r[j], r[j]));
  norms[i] = acc;
}

// Sort key of Index::add: list id, then distance to the centroid; the
// stable radix sort keeps equal keys in row order.
__global__ void add_keys_kernel(const int32_t* __restrict__ assign, const float* __restrict__ dist, size_t n,
                                uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  keys[i] = (static_cast<uint64_t>(static_cast<uint32_t>(assign[i])) << 32) | __float_as_uint(dist[i]);
  vals[i] = static_cast<uint32_t>(i);
}

__global__ void scatter_sorted_kernel(const float* __restrict__ x, const uint32_t* __restrict__ order, size_t n,
                                      int dpad, float* __restrict__ codes, int64_t* __restrict__ ids) {
  const int c4 = dpad / 4;
  const size_t total = n * c4;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const size_t p = i / c4;
    const int c = static_cast<int>(i - p * c4);
    const uint32_t src = order[p];
    reinterpret_cast<float4*>(codes)[p * c4 + c] = reinterpret_cast<const float4*>(x)[static_cast<size_t>(src) * c4 + c];
    if (c == 0) ids[p] = static_cast<int64_t>(src);
  }
}

__global__ void histogram_kernel(const int32_t* __restrict__ assign, size_t n, int64_t* __restrict__ cnt) {
  const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
  if (i < n) atomicAdd(reinterpret_cast<unsigned long long*>(&cnt[assign[i]]), 1ull);
}

__global__ void i64_to_i32_kernel(const int64_t* __restrict__ s, size_t n, int32_t* __restrict__ d) {
  const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
  if (i < n) d[i] = static_cast<int32_t>(s[i]);
}
__global__ void i32_to_i64_kernel(const int32_t* __restrict__ s, size_t n, int64_t* __restrict__ d) {
  const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
  if (i < n) d[i] = static_cast<int64_t>(s[i]);
}
__global__ void fill_results_kernel(float* __restrict__ D, int64_t* __restrict__ I, size_t n) {
  const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
  if (i < n) {
    D[i] = FLT_MAX;
    I[i] = -1;
  }
}

inline unsigned grid_for(size_t n, int tb, unsigned cap = 148u * 32u) {
  size_t g = (n + tb - 1) / tb;
  if (g > cap) g = cap;
  return static_cast<unsigned>(g < 1 ? 1 : g);
}
inline unsigned grid_exact(size_t n, int tb) {
  return static_cast<unsigned>((n + tb - 1) / tb);
}

}  // namespace

void launch_pad_rows(const float* src, size_t n, int d, int dpad, float* dst, cudaStream_t st) {
  if (!n) return;
  pad_rows_kernel<<<grid_for(n * dpad, 256), 256, 0, st>>>(src, n, d, dpad, dst);
  HB_CUDA(cudaGetLastError());
}

void launch_gather_rows(const float* src, const int64_t* idx, size_t n, int dpad, float* dst, cudaStream_t st) {
  if (!n) return;
  gather_rows_kernel<<<grid_for(n * dpad / 4, 256), 256, 0, st>>>(src, idx, n, dpad, dst);
  HB_CUDA(cudaGetLastError());
}

void launch_kmeans_accumulate(const float* x, const int32_t* assign, size_t n, int d, int dpad, double* sums,
                              int32_t* counts, cudaStream_t st) {
  if (!n) return;
  kmeans_accumulate_kernel<<<grid_exact(n * 32, 256), 256, 0, st>>>(x, assign, n, d, dpad, sums, counts);
  HB_CUDA(cudaGetLastError());
}

void launch_kmeans_update(const double* sums, const int32_t* counts, int nlist, int d, int dpad, float* cent,
                          cudaStream_t st) {
  kmeans_update_kernel<<<grid_for(static_cast<size_t>(nlist) * d, 256), 256, 0, st>>>(sums, counts, nlist, d, dpad,
                                                                                      cent);
  HB_CUDA(cudaGetLastError());
}

void launch_row_norms(const float* x, size_t n, int d, int dpad, float* norms, cudaStream_t st) {
  if (!n) return;
  row_norms_kernel<<<grid_exact(n, 256), 256, 0, st>>>(x, n, d, dpad, norms);
  HB_CUDA(cudaGetLastError());
}

void launch_add_keys(const int32_t* assign, const float* dist, size_t n, uint64_t* keys, uint32_t* vals,
                     cudaStream_t st) {
  if (!n) return;
  add_keys_kernel<<<grid_exact(n, 256), 256, 0, st>>>(assign, dist, n, keys, vals);
  HB_CUDA(cudaGetLastError());
}

void sort_pairs_u64(uint64_t* keys_in, uint64_t* keys_out, uint32_t* vals_in, uint32_t* vals_out, size_t n,
                    int end_bit, void* tmp, size_t* tmp_bytes, cudaStream_t st) {
  HB_CUDA(cub::DeviceRadixSort::SortPairs(tmp, *tmp_bytes, keys_in, keys_out, vals_in, vals_out,
                                          static_cast<int64_t>(n), 0, end_bit, st));
}

void launch_scatter_sorted(const float* x, const uint32_t* order, size_t n, int d, int dpad, float* codes,
                           int64_t* ids, cudaStream_t st) {
  (void)d;
  if (!n) return;
  scatter_sorted_kernel<<<grid_for(n * dpad / 4, 256), 256, 0, st>>>(x, order, n, dpad, codes, ids);
  HB_CUDA(cudaGetLastError());
}

size_t list_offsets_tmp_bytes(int nlist) {
  size_t bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, bytes, static_cast<const int64_t*>(nullptr), static_cast<int64_t*>(nullptr),
                                static_cast<int64_t>(nlist) + 1);
  return (bytes + 255) / 256 * 256 + (static_cast<size_t>(nlist) + 1) * sizeof(int64_t);
}

void launch_list_offsets(const int32_t* assign, size_t n, int nlist, int64_t* list_off, void* tmp, size_t tmp_bytes,
                         cudaStream_t st) {
  size_t cub_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, cub_bytes, static_cast<const int64_t*>(nullptr),
                                static_cast<int64_t*>(nullptr), static_cast<int64_t>(nlist) + 1);
  const size_t cub_al = (cub_bytes + 255) / 256 * 256;
  HB_CHECK(tmp_bytes >= cub_al + (static_cast<size_t>(nlist) + 1) * sizeof(int64_t), HB_ERR_INVALID,
           "list offset scratch too small");
  int64_t* cnt = reinterpret_cast<int64_t*>(static_cast<unsigned char*>(tmp) + cub_al);
  HB_CUDA(cudaMemsetAsync(cnt, 0, (static_cast<size_t>(nlist) + 1) * sizeof(int64_t), st));
  if (n) {
    histogram_kernel<<<grid_exact(n, 256), 256, 0, st>>>(assign, n, cnt);
    HB_CUDA(cudaGetLastError());
  }
  HB_CUDA(cub::DeviceScan::ExclusiveSum(tmp, cub_bytes, cnt, list_off, static_cast<int64_t>(nlist) + 1, st));
}

void launch_i64_to_i32(const int64_t* src, size_t n, int32_t* dst, cudaStream_t st) {
  if (!n) return;
  i64_to_i32_kernel<<<grid_exact(n, 256), 256, 0, st>>>(src, n, dst);
  HB_CUDA(cudaGetLastError());
}
void launch_i32_to_i64(const int32_t* src, size_t n, int64_t* dst, cudaStream_t st) {
  if (!n) return;
  i32_to_i64_kernel<<<grid_exact(n, 256), 256, 0, st>>>(src, n, dst);
  HB_CUDA(cudaGetLastError());
}
void launch_fill_results(float* D, int64_t* I, size_t n, cudaStream_t st) {
  if (!n) return;
  fill_results_kernel<<<grid_exact(n, 256), 256, 0, st>>>(D, I, n);
  HB_CUDA(cudaGetLastError());
}


namespace {
__global__ void gather_words_kernel(const uint32_t* __restrict__ src, const int32_t* __restrict__ idx, int n, int w,
                                    uint32_t* __restrict__ dst) {
  const size_t total = static_cast<size_t>(n) * w;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const size_t r = i / w, c = i - r * w;
    dst[i] = src[static_cast<size_t>(idx[r]) * w + c];
  }
}

__global__ void scatter_words_kernel(const uint32_t* __restrict__ src, const int32_t* __restrict__ idx, int n, int w,
                                     uint32_t* __restrict__ dst) {
  const size_t total = static_cast<size_t>(n) * w;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const size_t r = i / w, c = i - r * w;
    dst[static_cast<size_t>(idx[r]) * w + c] = src[i];
  }
}
}  // namespace

void launch_gather_words(const uint32_t* src, const int32_t* idx, int n, int w, uint32_t* dst, cudaStream_t st) {
  if (n <= 0 || w <= 0) return;
  const size_t total = static_cast<size_t>(n) * w;
  const unsigned g = static_cast<unsigned>(std::min<size_t>((total + 255) / 256, 148 * 32));
  gather_words_kernel<<<g, 256, 0, st>>>(src, idx, n, w, dst);
  HB_CUDA(cudaGetLastError());
}

void launch_scatter_words(const uint32_t* src, const int32_t* idx, int n, int w, uint32_t* dst, cudaStream_t st) {
  if (n <= 0 || w <= 0) return;
  const size_t total = static_cast<size_t>(n) * w;
  const unsigned g = static_cast<unsigned>(std::min<size_t>((total + 255) / 256, 148 * 32));
  scatter_words_kernel<<<g, 256, 0, st>>>(src, idx, n, w, dst);
  HB_CUDA(cudaGetLastError());
}

}  // namespace hb

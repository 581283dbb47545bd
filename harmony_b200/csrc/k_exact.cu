// Exact FP32 L2 kernels: the arithmetic of the reference's distance loop
// (src/utils.h:480-487) -- for every (query, vector) pair one sequential sum
// over the dimensions in order, each (q-x)^2 rounded before it is added
// (__fmul_rn / __fadd_rn keep nvcc from contracting to FMA).
//
// Layout on the device: vectors and queries are row-major with rows padded
// to dpad (multiple of 16) zero floats.  A CTA stages a tile of TV vector
// rows in shared memory with 16-byte cp.async copies (row stride dpad+4
// floats, so the 8 lanes of a 128-bit load phase hit 8 different 4-bank
// groups), keeps QG queries in shared memory, and gives each thread one
// vector row and QT queries: per 4 dims it issues one LDS.128 of its row,
// QT broadcast LDS.128 of the queries and 12*QT FP32 instructions.
//
// The list scan (scan_exact_kernel) is persistent: one CTA per SM pulls work
// items (list, chunk of rows, group of queries that probe the list) from a
// global counter, so every row chunk is read once per query group and the
// query groups of one chunk run back to back (they share L2).  Each query
// keeps a candidate buffer in shared memory: pairs at or under the query's
// running k-th distance are appended; a warp sorts the buffer back to k
// entries when it could overflow.  The per-(query, chunk) top-k goes to a
// slot in global memory; k_select.cu merges the slots of a query.
#include <cuda_runtime.h>

#include <algorithm>

#include "hb_device.cuh"
#include "hb_internal.hpp"

namespace hb {
namespace {

constexpr int kThreads = 256;

// ----------------------------------------------------------------------------
// Distance micro-kernels.

template <int QT>
__device__ __forceinline__ void dist_plain(const float* __restrict__ xr, const float* __restrict__ qb,
                                           int qstride, int dpad, float (&acc)[QT]) {
#pragma unroll
  for (int i = 0; i < QT; ++i) acc[i] = 0.0f;
#pragma unroll 2
  for (int c = 0; c < dpad; c += 4) {
    const float4 x = *reinterpret_cast<const float4*>(xr + c);
#pragma unroll
    for (int i = 0; i < QT; ++i) {
      const float4 v = *reinterpret_cast<const float4*>(qb + i * qstride + c);
      float t;
      t = __fsub_rn(v.x, x.x);
      acc[i] = __fadd_rn(acc[i], __fmul_rn(t, t));
      t = __fsub_rn(v.y, x.y);
      acc[i] = __fadd_rn(acc[i], __fmul_rn(t, t));
      t = __fsub_rn(v.z, x.z);
      acc[i] = __fadd_rn(acc[i], __fmul_rn(t, t));
      t = __fsub_rn(v.w, x.w);
      acc[i] = __fadd_rn(acc[i], __fmul_rn(t, t));
    }
  }
}

// Packed FP32 pairs (sm_100a f32x2): two queries' differences and squares in
// one 64-bit register; every operation rounds on its own, so each query's sum
// is exactly the scalar sequential sum above.
__device__ __forceinline__ uint64_t f2_pack(float a, float b) {
  uint64_t r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
// acc0 / acc1 += (q - x)^2 for two queries: the subtraction and the square
// packed, the two additions scalar.  (A packed multiply followed by a packed
// add is contracted into one fused multiply-add by the compiler even with
// .rn on both -- measured: a third of 128-term sums then differ from the
// unfused loop -- while this form matches it bit for bit.)
__device__ __forceinline__ void f2_sq_acc(float& acc0, float& acc1, uint64_t q2, uint64_t x2) {
  uint64_t t;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(t) : "l"(q2), "l"(x2));
  asm("mul.rn.f32x2 %0, %1, %1;" : "=l"(t) : "l"(t));
  float s0, s1;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(s0), "=f"(s1) : "l"(t));
  acc0 = __fadd_rn(acc0, s0);
  acc1 = __fadd_rn(acc1, s1);
}

// One row against NP query pairs stored pair-interleaved: qp[(p * dpad + c)
// * 2 + {0,1}] = dim c of the pair's two queries.
template <int NP>
__device__ __forceinline__ void dist_plain_x2(const float* __restrict__ xr, const float* __restrict__ qp, int dpad,
                                              float (&out)[2 * NP]) {
  float acc[2 * NP];
#pragma unroll
  for (int p = 0; p < 2 * NP; ++p) acc[p] = 0.0f;
#pragma unroll 2
  for (int c = 0; c < dpad; c += 4) {
    const float4 x = *reinterpret_cast<const float4*>(xr + c);
    const uint64_t x0 = f2_pack(x.x, x.x), x1 = f2_pack(x.y, x.y), x2 = f2_pack(x.z, x.z), x3 = f2_pack(x.w, x.w);
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      const ulonglong2 qa = *reinterpret_cast<const ulonglong2*>(qp + (static_cast<size_t>(p) * dpad + c) * 2);
      const ulonglong2 qb = *reinterpret_cast<const ulonglong2*>(qp + (static_cast<size_t>(p) * dpad + c) * 2 + 4);
      f2_sq_acc(acc[2 * p], acc[2 * p + 1], qa.x, x0);
      f2_sq_acc(acc[2 * p], acc[2 * p + 1], qa.y, x1);
      f2_sq_acc(acc[2 * p], acc[2 * p + 1], qb.x, x2);
      f2_sq_acc(acc[2 * p], acc[2 * p + 1], qb.y, x3);
    }
  }
#pragma unroll
  for (int p = 0; p < 2 * NP; ++p) out[p] = acc[p];
}

// Segmented sums: the dimension range is cut at bnd[0..nb) (ascending, in
// true dims); part[i][s] is the fresh sequential sum of segment s.
template <int QT, int MAXSEG>
__device__ __forceinline__ void dist_segments(const float* __restrict__ xr, const float* __restrict__ qb,
                                              int qstride, int dpad, const int* bnd, int nseg,
                                              float (&part)[QT][MAXSEG]) {
  float cur[QT];
#pragma unroll
  for (int i = 0; i < QT; ++i) {
    cur[i] = 0.0f;
#pragma unroll
    for (int s = 0; s < MAXSEG; ++s) part[i][s] = 0.0f;
  }
  int s = 0;
  int next = nseg > 1 ? bnd[0] : 0x7fffffff;
  for (int c = 0; c < dpad; c += 4) {
    const float4 x = *reinterpret_cast<const float4*>(xr + c);
    float xv[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int dim = c + e;
      while (dim == next) {
#pragma unroll
        for (int i = 0; i < QT; ++i) {
#pragma unroll
          for (int ss = 0; ss < MAXSEG; ++ss)
            if (ss == s) part[i][ss] = cur[i];
          cur[i] = 0.0f;
        }
        ++s;
        next = (s < nseg - 1) ? bnd[s] : 0x7fffffff;
      }
#pragma unroll
      for (int i = 0; i < QT; ++i) {
        const float t = __fsub_rn(qb[i * qstride + dim], xv[e]);
        cur[i] = __fadd_rn(cur[i], __fmul_rn(t, t));
      }
    }
  }
  // Close the open segment and any empty trailing ones.
  while (s < nseg) {
#pragma unroll
    for (int i = 0; i < QT; ++i) {
#pragma unroll
      for (int ss = 0; ss < MAXSEG; ++ss)
        if (ss == s) part[i][ss] = cur[i];
      cur[i] = 0.0f;
    }
    ++s;
  }
}

// Copy `rows` rows of dpad floats (global, stride dpad) to shared memory
// (stride lds), zero-filling rows at or past `valid`.
__device__ __forceinline__ void load_rows_async(float* s, int lds, const float* g, int rows, int valid,
                                                int dpad) {
  const int cpr = dpad >> 2;  // 16-byte chunks per row
  const int total = rows * cpr;
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int r = idx / cpr;
    const int c = idx - r * cpr;
    const bool ok = r < valid;
    const float* src = ok ? g + static_cast<size_t>(r) * dpad + c * 4 : g;
    cp_async16(s + r * lds + c * 4, src, ok);
  }
}

// ----------------------------------------------------------------------------
// Distance matrix: D[q][c] for a (TV rows x QG queries) tile per CTA.

template <int TV, int QT>
__global__ void __launch_bounds__(kThreads) l2_matrix_kernel(const float* __restrict__ q, int nq,
                                                             const float* __restrict__ rows, int nrows,
                                                             int dpad, float* __restrict__ D, int ldD) {
  constexpr int G = kThreads / TV;
  constexpr int QG = G * QT;
  extern __shared__ __align__(16) float smem[];
  const int lds = dpad + 4;
  float* sr = smem;
  float* sq = smem + TV * lds;
  const int r0 = blockIdx.x * TV;
  const int q0 = blockIdx.y * QG;
  load_rows_async(sr, lds, rows + static_cast<size_t>(r0) * dpad, TV, nrows - r0, dpad);
  load_rows_async(sq, dpad, q + static_cast<size_t>(q0) * dpad, QG, nq - q0, dpad);
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  const int r = threadIdx.x % TV;
  const int g = threadIdx.x / TV;
  float acc[QT];
  dist_plain<QT>(sr + r * lds, sq + g * QT * dpad, dpad, dpad, acc);
  if (r0 + r < nrows) {
#pragma unroll
    for (int i = 0; i < QT; ++i) {
      const int qi = q0 + g * QT + i;
      if (qi < nq) D[static_cast<size_t>(qi) * ldD + r0 + r] = acc[i];
    }
  }
}

// Nearest row per query: each CTA owns QG queries and sweeps all rows with a
// double-buffered tile; lexicographic (distance, row) minimum = the
// reference's strict '<' scan in row order.  Distances >= FLT_MAX never
// win; a query with no admissible row gets row 0 (Clustering's initial
// closest_centroid, src/Clustering.cpp:103-104).
template <int TV, int QT>
__global__ void __launch_bounds__(kThreads) l2_argmin_kernel(const float* __restrict__ q, int nq,
                                                             const float* __restrict__ rows, int nrows,
                                                             int dpad, int32_t* __restrict__ arg,
                                                             float* __restrict__ dist) {
  constexpr int G = kThreads / TV;
  constexpr int QG = G * QT;
  extern __shared__ __align__(16) float smem[];
  const int lds = dpad + 4;
  float* sr0 = smem;
  float* sr1 = smem + TV * lds;
  float* sq = smem + 2 * TV * lds;
  const int q0 = blockIdx.x * QG;
  load_rows_async(sq, dpad, q + static_cast<size_t>(q0) * dpad, QG, nq - q0, dpad);
  load_rows_async(sr0, lds, rows, TV, nrows, dpad);
  cp_async_commit();
  const int r = threadIdx.x % TV;
  const int g = threadIdx.x / TV;
  uint64_t best[QT];
#pragma unroll
  for (int i = 0; i < QT; ++i) best[i] = kEmpty;
  const int ntiles = (nrows + TV - 1) / TV;
  for (int t = 0; t < ntiles; ++t) {
    float* cur = (t & 1) ? sr1 : sr0;
    float* nxt = (t & 1) ? sr0 : sr1;
    if (t + 1 < ntiles) {
      const int rn = (t + 1) * TV;
      load_rows_async(nxt, lds, rows + static_cast<size_t>(rn) * dpad, TV, nrows - rn, dpad);
    }
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    float acc[QT];
    dist_plain<QT>(cur + r * lds, sq + g * QT * dpad, dpad, dpad, acc);
    const int row = t * TV + r;
    if (row < nrows) {
#pragma unroll
      for (int i = 0; i < QT; ++i)
        if (acc[i] < FLT_MAX) {
          const uint64_t key = make_key(acc[i], static_cast<uint32_t>(row));
          best[i] = key < best[i] ? key : best[i];
        }
    }
    __syncthreads();
  }
  // Reduce over the TV threads of each query group through shared memory
  // (the row tiles are free now): red[(g * QT + i) * TV + r].
  uint64_t* red = reinterpret_cast<uint64_t*>(sr0);
#pragma unroll
  for (int i = 0; i < QT; ++i) red[(g * QT + i) * TV + r] = best[i];
  __syncthreads();
  if (threadIdx.x < QG) {
    uint64_t v = kEmpty;
    for (int rr = 0; rr < TV; ++rr) {
      const uint64_t o = red[threadIdx.x * TV + rr];
      v = o < v ? o : v;
    }
    const int qi = q0 + threadIdx.x;
    if (qi < nq) {
      arg[qi] = v == kEmpty ? 0 : static_cast<int32_t>(key_tie(v));
      if (dist) dist[qi] = v == kEmpty ? FLT_MAX : key_dist(v);
    }
  }
}

// ----------------------------------------------------------------------------
// Persistent list scan.

struct ItemShared {
  int list, chunk, group, qcnt;
  int64_t row0, row1;
};

template <int TV, int QT, int MODE>
__global__ void __launch_bounds__(kThreads, 1) scan_exact_kernel(ScanArgs a, int cap) {
  constexpr int G = kThreads / TV;
  constexpr int QG = G * QT;
  constexpr int MAXSEG = (MODE == SCAN_DIMBLOCK) ? 8 : 4;
  extern __shared__ __align__(16) float smem[];
  const int dpad = a.dpad;
  const int lds = dpad + 4;
  float* const srowA = smem;
  float* const srowB = smem + TV * lds;
  float* sq = smem + 2 * TV * lds;
  uint64_t* sbuf = reinterpret_cast<uint64_t*>(sq + QG * dpad);
  int* scnt = reinterpret_cast<int*>(sbuf + QG * cap);
  float* sthr = reinterpret_cast<float*>(scnt + QG);
  float* stop = sthr + QG;
  int* sqid = reinterpret_cast<int*>(stop + QG);   // packed (q << 16 | j) as uint32; -1 if unused
  int* sord = sqid + QG;                           // DIMBLOCK: query block index, -1 = unsearched
  __shared__ ItemShared it;
  __shared__ int sbnd[8];

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int r = tid % TV;
  const int g = tid / TV;
  const int64_t total_items = a.item_off[a.nlist];

  if (MODE == SCAN_CHUNK4 && tid == 0) {
    const int cd = a.d / 4;
    sbnd[0] = cd;
    sbnd[1] = 2 * cd;
    sbnd[2] = 3 * cd;
  }
  if (MODE == SCAN_DIMBLOCK && tid < 8) sbnd[tid] = (tid + 1) * (a.d / a.nseg);

  for (;;) {
    __syncthreads();
    if (tid == 0) {
      const int64_t item = static_cast<int64_t>(atomicAdd(a.work_counter, 1u));
      if (item >= total_items) {
        it.list = -1;
      } else {
        // Largest l with item_off[l] <= item.
        int lo = 0, hi = a.nlist;  // invariant item_off[lo] <= item < item_off[hi]
        while (hi - lo > 1) {
          const int mid = (lo + hi) >> 1;
          if (a.item_off[mid] <= item) lo = mid; else hi = mid;
        }
        const int l = lo;
        // Items of a list: chunk-major, so the query groups of one row
        // chunk run back to back and share it through L2.
        const int64_t local = item - a.item_off[l];
        const int ng = (a.list_cnt[l] + a.qgroup - 1) / a.qgroup;
        it.list = l;
        it.chunk = static_cast<int>(local / ng);
        it.group = static_cast<int>(local % ng);
        it.qcnt = min(a.qgroup, a.list_cnt[l] - it.group * a.qgroup);
        it.row0 = a.list_off[l] + static_cast<int64_t>(it.chunk) * a.chunk_rows;
        it.row1 = min(a.list_off[l + 1], it.row0 + a.chunk_rows);
      }
    }
    __syncthreads();
    if (it.list < 0) break;
    const int qcnt = it.qcnt;
    const int64_t row0 = it.row0;
    const int nrow = static_cast<int>(it.row1 - row0);

    // Queries of this item.
    if (tid < QG) {
      int packed = -1, blk = -1;
      float top = FLT_MAX;
      if (tid < qcnt) {
        packed = a.list_q[a.list_qoff[it.list] + static_cast<int64_t>(it.group) * a.qgroup + tid];
        const int qq = static_cast<int>(static_cast<unsigned>(packed) >> 16);
        if (MODE != SCAN_PLAIN && a.tops) top = a.tops[qq];
        if (MODE == SCAN_DIMBLOCK) {
          const int b = a.qblock > 0 ? qq / a.qblock : 0;
          blk = (a.qblock > 0 && b < a.nblocks) ? b : -1;
        }
      }
      sqid[tid] = packed;
      sord[tid] = blk;
      stop[tid] = top;
      scnt[tid] = 0;
      sthr[tid] = FLT_MAX;
    }
    __syncthreads();
    {
      const int cpr = dpad >> 2;
      for (int idx = tid; idx < QG * cpr; idx += kThreads) {
        const int e = idx / cpr, c = idx - e * cpr;
        const bool ok = e < qcnt;
        const float* src = ok ? a.q + static_cast<size_t>(static_cast<unsigned>(sqid[e]) >> 16) * dpad + c * 4 : a.q;
        cp_async16(sq + e * dpad + c * 4, src, ok);
      }
    }
    const int ntiles = (nrow + TV - 1) / TV;
    load_rows_async(srowA, lds, a.codes + static_cast<size_t>(row0) * dpad, TV, nrow, dpad);
    cp_async_commit();

    for (int t = 0; t < ntiles; ++t) {
      const float* cur = (t & 1) ? srowB : srowA;
      if (t + 1 < ntiles) {
        const int rn = (t + 1) * TV;
        load_rows_async((t & 1) ? srowA : srowB, lds, a.codes + static_cast<size_t>(row0 + rn) * dpad, TV,
                        nrow - rn, dpad);
      }
      cp_async_commit();
      cp_async_wait<1>();
      const bool need = __syncthreads_or(tid < QG && scnt[tid] > cap - TV);
      if (need) {
        for (int e = warp; e < QG; e += kThreads / 32) {
          const int c = scnt[e];
          if (c > cap - TV) {
            uint64_t* b = sbuf + e * cap;
            for (int i = c + lane; i < cap; i += 32) b[i] = kEmpty;
            __syncwarp();
            warp_bitonic_sort(b, cap, lane);
            if (lane == 0) {
              scnt[e] = a.k;
              sthr[e] = key_dist(b[a.k - 1]);
            }
            __syncwarp();
          }
        }
        __syncthreads();
      }

      // Distances for row t*TV + r against queries g*QT ...
      const int rloc = t * TV + r;
      const bool rvalid = rloc < nrow;
      float dist[QT];
      const float* xr = cur + r * lds;
      const float* qb = sq + g * QT * dpad;
      if (MODE == SCAN_PLAIN) {
        dist_plain<QT>(xr, qb, dpad, dpad, dist);
      } else if (MODE == SCAN_CHUNK4) {
        float part[QT][4];
        dist_segments<QT, 4>(xr, qb, dpad, dpad, sbnd, 4, part);
#pragma unroll
        for (int i = 0; i < QT; ++i) {
          const float top = stop[g * QT + i];
          float acc = 0.0f;
          bool dead = false;
#pragma unroll
          for (int s = 0; s < 4; ++s) {
            if (!dead) {
              acc = __fadd_rn(acc, part[i][s]);
              if (a.cut && s < 3 && acc > top) dead = true;
            }
          }
          dist[i] = dead ? INFINITY : acc;
        }
      } else {
        float part[QT][MAXSEG];
        dist_segments<QT, MAXSEG>(xr, qb, dpad, dpad, sbnd, a.nseg, part);
#pragma unroll
        for (int i = 0; i < QT; ++i) {
          const int blk = sord[g * QT + i];
          const float top = stop[g * QT + i];
          float acc = 0.0f;
          bool dead = blk < 0;
          for (int t2 = 0; t2 < a.nseg && !dead; ++t2) {
            const int s = blk >= 0 ? a.seg_order[blk * a.nseg + t2] : 0;
            float p = 0.0f;
#pragma unroll
            for (int ss = 0; ss < MAXSEG; ++ss)
              if (ss == s) p = part[i][ss];
            acc = __fadd_rn(acc, p);
            if (a.cut && acc > top) dead = true;
          }
          dist[i] = dead ? INFINITY : acc;
        }
      }
      if (rvalid) {
#pragma unroll
        for (int i = 0; i < QT; ++i) {
          const int e = g * QT + i;
          if (e < qcnt && dist[i] < FLT_MAX && dist[i] <= sthr[e]) {
            const int pos = atomicAdd(&scnt[e], 1);
            sbuf[e * cap + pos] = make_key(dist[i], static_cast<uint32_t>(row0 + rloc));
          }
        }
      }
      __syncthreads();
    }
    cp_async_wait<0>();
    __syncthreads();

    // Final sort of every buffer and write of the k best to the query's slot.
    for (int e = warp; e < qcnt; e += kThreads / 32) {
      uint64_t* b = sbuf + e * cap;
      const int c = scnt[e];
      for (int i = c + lane; i < cap; i += 32) b[i] = kEmpty;
      __syncwarp();
      warp_bitonic_sort(b, cap, lane);
      const int packed = sqid[e];
      const int qq = static_cast<int>(static_cast<unsigned>(packed) >> 16), j = packed & 0xffff;
      const int64_t slot = a.slot_base[static_cast<int64_t>(qq) * a.P + j] + it.chunk;
      uint64_t* out = a.part + slot * a.k;
      for (int i = lane; i < a.k; i += 32) out[i] = b[i];
      __syncwarp();
    }
  }
}

// ----------------------------------------------------------------------------
// Persistent list scan of the ORIGINAL / BRUTE_FORCE searches (plain
// sequential sums) with 16 warps per SM: kPackThreads threads, each one row
// of the TV-row tile against QT queries.  PK: packed f32x2 arithmetic (QT / 2
// pairs; the item's queries sit pair-interleaved in shared memory); else the
// scalar loop with the queries row-major.  Same items, candidate buffers,
// slots and results as scan_exact_kernel in SCAN_PLAIN mode.
constexpr int kPackThreads = 512;
constexpr bool kPackedExact = true;

template <int TV, int QT, bool PK>
__global__ void __launch_bounds__(kPackThreads, 1) scan_plain_x2_kernel(ScanArgs a, int cap) {
  constexpr int NT = kPackThreads;
  constexpr int G = NT / TV;
  constexpr int QG = G * QT;
  constexpr int NP = QT / 2;
  extern __shared__ __align__(16) float smem[];
  const int dpad = a.dpad;
  const int lds = dpad + 4;
  float* const srowA = smem;
  float* const srowB = smem + TV * lds;
  float* sq = smem + 2 * TV * lds;  // PK: [QG / 2][dpad][2]; else [QG][dpad]
  uint64_t* sbuf = reinterpret_cast<uint64_t*>(sq + QG * dpad);
  int* scnt = reinterpret_cast<int*>(sbuf + QG * cap);
  float* sthr = reinterpret_cast<float*>(scnt + QG);
  int* sqid = reinterpret_cast<int*>(sthr + QG);   // packed (q << 16 | j) as uint32; -1 if unused
  __shared__ ItemShared it;

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int r = tid % TV;
  const int g = tid / TV;
  const int64_t total_items = a.item_off[a.nlist];

  for (;;) {
    __syncthreads();
    if (tid == 0) {
      const int64_t item = static_cast<int64_t>(atomicAdd(a.work_counter, 1u));
      if (item >= total_items) {
        it.list = -1;
      } else {
        int lo = 0, hi = a.nlist;  // invariant item_off[lo] <= item < item_off[hi]
        while (hi - lo > 1) {
          const int mid = (lo + hi) >> 1;
          if (a.item_off[mid] <= item) lo = mid; else hi = mid;
        }
        const int l = lo;
        const int64_t local = item - a.item_off[l];
        const int ng = (a.list_cnt[l] + a.qgroup - 1) / a.qgroup;
        it.list = l;
        it.chunk = static_cast<int>(local / ng);
        it.group = static_cast<int>(local % ng);
        it.qcnt = min(a.qgroup, a.list_cnt[l] - it.group * a.qgroup);
        it.row0 = a.list_off[l] + static_cast<int64_t>(it.chunk) * a.chunk_rows;
        it.row1 = min(a.list_off[l + 1], it.row0 + a.chunk_rows);
      }
    }
    __syncthreads();
    if (it.list < 0) break;
    const int qcnt = it.qcnt;
    const int64_t row0 = it.row0;
    const int nrow = static_cast<int>(it.row1 - row0);
    const int ntiles = (nrow + TV - 1) / TV;
    load_rows_async(srowA, lds, a.codes + static_cast<size_t>(row0) * dpad, TV, nrow, dpad);
    cp_async_commit();
    if (tid < QG) {
      int packed = -1;
      if (tid < qcnt) packed = a.list_q[a.list_qoff[it.list] + static_cast<int64_t>(it.group) * a.qgroup + tid];
      sqid[tid] = packed;
      scnt[tid] = 0;
      sthr[tid] = FLT_MAX;
    }
    __syncthreads();
    // Queries, pair-interleaved (zeros for unused query slots).
    {
      const int cpr = dpad >> 2;
      for (int idx = tid; idx < QG * cpr; idx += NT) {
        const int e = idx / cpr, c = (idx - e * cpr) * 4;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (e < qcnt) v = *reinterpret_cast<const float4*>(a.q + static_cast<size_t>(static_cast<unsigned>(sqid[e]) >> 16) * dpad + c);
        if (PK) {
          float* dst = sq + (static_cast<size_t>(e >> 1) * dpad + c) * 2 + (e & 1);
          dst[0] = v.x;
          dst[2] = v.y;
          dst[4] = v.z;
          dst[6] = v.w;
        } else {
          *reinterpret_cast<float4*>(sq + static_cast<size_t>(e) * dpad + c) = v;
        }
      }
    }

    for (int t = 0; t < ntiles; ++t) {
      const float* cur = (t & 1) ? srowB : srowA;
      if (t + 1 < ntiles) {
        const int rn = (t + 1) * TV;
        load_rows_async((t & 1) ? srowA : srowB, lds, a.codes + static_cast<size_t>(row0 + rn) * dpad, TV,
                        nrow - rn, dpad);
      }
      cp_async_commit();
      cp_async_wait<1>();
      const bool need = __syncthreads_or(tid < QG && scnt[tid] > cap - TV);
      if (need) {
        for (int e = warp; e < QG; e += NT / 32) {
          const int c = scnt[e];
          if (c > cap - TV) {
            uint64_t* b = sbuf + e * cap;
            for (int i = c + lane; i < cap; i += 32) b[i] = kEmpty;
            __syncwarp();
            warp_bitonic_sort(b, cap, lane);
            if (lane == 0) {
              scnt[e] = a.k;
              sthr[e] = key_dist(b[a.k - 1]);
            }
            __syncwarp();
          }
        }
        __syncthreads();
      }
      const int rloc = t * TV + r;
      float dist[QT];
      if (PK)
        dist_plain_x2<NP>(cur + r * lds, sq + static_cast<size_t>(g) * NP * dpad * 2, dpad, dist);
      else
        dist_plain<QT>(cur + r * lds, sq + static_cast<size_t>(g) * QT * dpad, dpad, dpad, dist);
      if (rloc < nrow) {
#pragma unroll
        for (int i = 0; i < QT; ++i) {
          const int e = g * QT + i;
          if (e < qcnt && dist[i] < FLT_MAX && dist[i] <= sthr[e]) {
            const int pos = atomicAdd(&scnt[e], 1);
            sbuf[e * cap + pos] = make_key(dist[i], static_cast<uint32_t>(row0 + rloc));
          }
        }
      }
      __syncthreads();
    }
    cp_async_wait<0>();
    __syncthreads();

    for (int e = warp; e < qcnt; e += NT / 32) {
      uint64_t* b = sbuf + e * cap;
      const int c = scnt[e];
      for (int i = c + lane; i < cap; i += 32) b[i] = kEmpty;
      __syncwarp();
      warp_bitonic_sort(b, cap, lane);
      const int packed = sqid[e];
      const int qq = static_cast<int>(static_cast<unsigned>(packed) >> 16), j = packed & 0xffff;
      const int64_t slot = a.slot_base[static_cast<int64_t>(qq) * a.P + j] + it.chunk;
      uint64_t* out = a.part + slot * a.k;
      for (int i = lane; i < a.k; i += 32) out[i] = b[i];
      __syncwarp();
    }
  }
}

// ----------------------------------------------------------------------------
// Tile shape choice.

struct Shape {
  int tv, qt;
};

inline Shape matrix_shape(int dpad) {
  if (dpad <= 128) return {128, 8};
  if (dpad <= 256) return {64, 8};
  if (dpad <= 512) return {32, 4};
  return {16, 2};
}

template <int TV, int QT>
void matrix_launch(const float* q, int nq, const float* rows, int nrows, int dpad, float* D, int ldD,
                   cudaStream_t st) {
  constexpr int QG = (kThreads / TV) * QT;
  const size_t smem = (static_cast<size_t>(TV) * (dpad + 4) + static_cast<size_t>(QG) * dpad) * 4;
  HB_CUDA(cudaFuncSetAttribute(l2_matrix_kernel<TV, QT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(smem)));
  dim3 grid((nrows + TV - 1) / TV, (nq + QG - 1) / QG);
  l2_matrix_kernel<TV, QT><<<grid, kThreads, smem, st>>>(q, nq, rows, nrows, dpad, D, ldD);
  HB_CUDA(cudaGetLastError());
}

template <int TV, int QT>
void argmin_launch(const float* q, int nq, const float* rows, int nrows, int dpad, int32_t* arg,
                   float* dist, cudaStream_t st) {
  constexpr int QG = (kThreads / TV) * QT;
  const size_t smem = (2 * static_cast<size_t>(TV) * (dpad + 4) + static_cast<size_t>(QG) * dpad) * 4;
  // The final reduction reuses the first row tile (kThreads * QT * 8 bytes,
  // below TV * (dpad + 4) * 4 for every shape launched here).
  HB_CUDA(cudaFuncSetAttribute(l2_argmin_kernel<TV, QT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(smem)));
  dim3 grid((nq + QG - 1) / QG);
  l2_argmin_kernel<TV, QT><<<grid, kThreads, smem, st>>>(q, nq, rows, nrows, dpad, arg, dist);
  HB_CUDA(cudaGetLastError());
}

}  // namespace

void launch_l2_matrix(const float* q, int nq, const float* rows, int nrows, int dpad, float* D, int ldD,
                      cudaStream_t st) {
  if (nq <= 0 || nrows <= 0) return;
  HB_CHECK(dpad <= 1024, HB_ERR_INVALID, "dimension above 1024 is not supported");
  const Shape s = matrix_shape(dpad);
  if (s.tv == 128) matrix_launch<128, 8>(q, nq, rows, nrows, dpad, D, ldD, st);
  else if (s.tv == 64) matrix_launch<64, 8>(q, nq, rows, nrows, dpad, D, ldD, st);
  else if (s.tv == 32) matrix_launch<32, 4>(q, nq, rows, nrows, dpad, D, ldD, st);
  else matrix_launch<32, 2>(q, nq, rows, nrows, dpad, D, ldD, st);
}

void launch_l2_argmin(const float* q, int nq, const float* rows, int nrows, int dpad, int32_t* arg,
                      float* dist, cudaStream_t st) {
  if (nq <= 0) return;
  HB_CHECK(nrows > 0, HB_ERR_STATE, "no centroids");
  HB_CHECK(dpad <= 1024, HB_ERR_INVALID, "dimension above 1024 is not supported");
  if (dpad <= 128) argmin_launch<128, 8>(q, nq, rows, nrows, dpad, arg, dist, st);
  else if (dpad <= 256) argmin_launch<64, 8>(q, nq, rows, nrows, dpad, arg, dist, st);
  else if (dpad <= 512) argmin_launch<32, 4>(q, nq, rows, nrows, dpad, arg, dist, st);
  else argmin_launch<16, 1>(q, nq, rows, nrows, dpad, arg, dist, st);
}

// ----------------------------------------------------------------------------

namespace {
size_t scan_smem(int tv, int qt, int dpad, int cap) {
  const int qg = (kThreads / tv) * qt;
  return (2 * static_cast<size_t>(tv) * (dpad + 4) + static_cast<size_t>(qg) * dpad) * 4 +
         static_cast<size_t>(qg) * cap * 8 + static_cast<size_t>(qg) * 5 * 4;
}
constexpr size_t kSmemLimit = 220 * 1024;

// The packed PLAIN scan (dpad <= 256): kPackThreads threads, QT even.
size_t scan_x2_smem(int tv, int qt, int dpad, int cap) {
  const int qg = (kPackThreads / tv) * qt;
  return (2 * static_cast<size_t>(tv) * (dpad + 4) + static_cast<size_t>(qg) * dpad) * 4 +
         static_cast<size_t>(qg) * cap * 8 + static_cast<size_t>(qg) * 3 * 4;
}
// The 16-warp kernel serves PLAIN scans up to dpad 256; its packed f32x2
// arithmetic is used only where it has been checked to equal the scalar
// sequential sum bit for bit (kPackedExact), else the scalar loop.
bool use_x2(int dpad, int mode) { return mode == SCAN_PLAIN && dpad <= 256; }
}  // namespace

size_t scan_exact_smem_bytes(int d, int dpad, int k, int mode, int* tv, int* qt, int* qgroup) {
  (void)d;
  if (use_x2(dpad, mode)) {
    const int TV = dpad <= 128 ? 128 : 64;
    int QT = 8;
    const int cap = pow2_ceil(k + TV);
    while (QT > 2 && scan_x2_smem(TV, QT, dpad, cap) > kSmemLimit) QT >>= 1;
    const size_t s = scan_x2_smem(TV, QT, dpad, cap);
    if (s <= kSmemLimit) {
      *tv = TV;
      *qt = QT;
      *qgroup = (kPackThreads / TV) * QT;
      return s;
    }
  }
  int TV = dpad <= 128 ? 128 : dpad <= 256 ? 64 : dpad <= 512 ? 32 : 16;
  int QT = mode == SCAN_DIMBLOCK ? 4 : (TV >= 64 ? 8 : 4);
  const int cap = pow2_ceil(k + TV);
  while (QT > 1 && scan_smem(TV, QT, dpad, cap) > kSmemLimit) QT >>= 1;
  const size_t s = scan_smem(TV, QT, dpad, cap);
  if (s > kSmemLimit) return 0;
  *tv = TV;
  *qt = QT;
  *qgroup = (kThreads / TV) * QT;
  return s;
}

namespace {
template <int TV, int QT, int MODE>
void scan_launch(const ScanArgs& a, int cap, size_t smem, int num_sms, cudaStream_t st) {
  HB_CUDA(cudaFuncSetAttribute(scan_exact_kernel<TV, QT, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(smem)));
  scan_exact_kernel<TV, QT, MODE><<<num_sms, kThreads, smem, st>>>(a, cap);
  HB_CUDA(cudaGetLastError());
}

template <int MODE>
void scan_dispatch(const ScanArgs& a, int tv, int qt, int cap, size_t smem, int num_sms, cudaStream_t st) {
#define HB_SCAN_CASE(TV_, QT_) \
  if (tv == TV_ && qt == QT_) return scan_launch<TV_, QT_, MODE>(a, cap, smem, num_sms, st);
  HB_SCAN_CASE(128, 8) HB_SCAN_CASE(128, 4) HB_SCAN_CASE(128, 2) HB_SCAN_CASE(128, 1)
  HB_SCAN_CASE(64, 8) HB_SCAN_CASE(64, 4) HB_SCAN_CASE(64, 2) HB_SCAN_CASE(64, 1)
  HB_SCAN_CASE(32, 4) HB_SCAN_CASE(32, 2) HB_SCAN_CASE(32, 1)
  HB_SCAN_CASE(16, 4) HB_SCAN_CASE(16, 2) HB_SCAN_CASE(16, 1)
#undef HB_SCAN_CASE
  throw Error(HB_ERR_INVALID, "no scan kernel for this tile shape");
}
}  // namespace

namespace {
template <int TV, int QT>
void x2_launch(const ScanArgs& a, int cap, size_t smem, int num_sms, cudaStream_t st) {
  HB_CUDA(cudaFuncSetAttribute(scan_plain_x2_kernel<TV, QT, kPackedExact>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  scan_plain_x2_kernel<TV, QT, kPackedExact><<<num_sms, kPackThreads, smem, st>>>(a, cap);
  HB_CUDA(cudaGetLastError());
}
}  // namespace

void launch_scan_exact(const ScanArgs& a, int num_sms, cudaStream_t st) {
  int tv = 0, qt = 0, qg = 0;
  const size_t smem = scan_exact_smem_bytes(a.d, a.dpad, a.k, a.mode, &tv, &qt, &qg);
  HB_CHECK(smem > 0, HB_ERR_INVALID, "k too large for the fused scan at this dimension");
  HB_CHECK(qg == a.qgroup, HB_ERR_INVALID, "scan plan built for another query group");
  const int cap = pow2_ceil(a.k + tv);
  if (use_x2(a.dpad, a.mode) && qg == (kPackThreads / tv) * qt) {
#define HB_X2_CASE(TV_, QT_) \
  if (tv == TV_ && qt == QT_) return x2_launch<TV_, QT_>(a, cap, smem, num_sms, st);
    HB_X2_CASE(128, 8) HB_X2_CASE(128, 4) HB_X2_CASE(128, 2)
    HB_X2_CASE(64, 8) HB_X2_CASE(64, 4) HB_X2_CASE(64, 2)
#undef HB_X2_CASE
  }
  if (a.mode == SCAN_PLAIN) scan_dispatch<SCAN_PLAIN>(a, tv, qt, cap, smem, num_sms, st);
  else if (a.mode == SCAN_CHUNK4) scan_dispatch<SCAN_CHUNK4>(a, tv, qt, cap, smem, num_sms, st);
  else scan_dispatch<SCAN_DIMBLOCK>(a, tv, qt, cap, smem, num_sms, st);
}

}  // namespace hb

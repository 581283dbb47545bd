// BF16 tensor-core list scan (tcgen05 + TMA) and the exact FP32 re-rank.
//
// Work items are the list-major items of the exact scan (list, chunk of
// rows, group of <= 128 queries probing the list).  Per item the CTA holds
// the group's queries as the MMA's A operand (128 x K, BF16, K-major,
// 128-byte swizzle) and streams the chunk's rows as B operand tiles of 128
// rows (TMA 2-D loads with the same swizzle into a ring of stages).  One
// thread issues tcgen05.mma (M 128 queries x N 128 rows x K 16) into one of
// four TMEM accumulators; the epilogue warps read their TMEM lanes back
// (thread = query, 128 columns = rows), form ||x||^2 - 2 q.x (the query's
// ||q||^2 does not change its ranking) and keep the R smallest per query in
// a thread-private max-heap in shared memory.  The R best keys (approximate
// distance, row position) of every (query, chunk) go to a slot;
// rerank_kernel takes each query's R best over its slots, recomputes their
// distances exactly in FP32 with the reference's sequential unfused loop and
// returns the k best -- so whenever the true k nearest are among the R
// candidates the result equals the exact scan's.
//
// Warp roles (384 threads), all running ahead of each other through
// mbarriers, with no CTA-wide barrier between items:
//   warps 0-7   two epilogue groups (TMEM lane quarters); tile t of the
//               CTA's global tile sequence goes to group t % 2, which keeps
//               its own heaps per item;
//   warp 8      TMA producer of the B tiles;
//   warp 9      MMA issuer; it also copies each tile's 128 row norms
//               (a padded per-tile norm array) next to the accumulator;
//   warps 10-11 item builders: fetch the next item from the global work
//               counter, gather its query ids and seed bounds and write its
//               A tile into the second A buffer while the current item runs.
// Every mbarrier wait is bounded; on a timeout the kernel records an error,
// the roles stop taking work, copies and MMAs in flight are drained and
// TMEM is freed.
#include <cudaTypedefs.h>
#include <cuda.h>
#include <cuda_runtime.h>

#include <cuda_bf16.h>

#include "hb_device.cuh"
#include "hb_internal.hpp"
#include "hb_select.cuh"
#include "hb_sm100.cuh"

namespace hb {
namespace {

using namespace sm100;

constexpr int kGroups = 2;                         // epilogue warpgroups, alternate tiles
constexpr int kEpiThreads = 128;                   // threads per epilogue group (= queries per item)
constexpr int kBuildWarps = 2;
constexpr int kProdWarp = kGroups * 4, kMmaWarp = kGroups * 4 + 1, kBuildWarp0 = kGroups * 4 + 2;
constexpr int kTcThreads = (kBuildWarp0 + kBuildWarps) * 32;
constexpr int kTile = 128;     // rows per B tile, queries per item (M)
constexpr int kMaxStages = 4;
constexpr int kAcc = 2 * kGroups;                  // TMEM accumulators of 128 columns
constexpr size_t kSmemCap = 225 * 1024;            // dynamic shared memory budget

struct ItemDesc {
  int list, chunk, group, qcnt, ntiles;  // ntiles < 0: no more work
  int row0;                              // first row (vector position) of the chunk
  long long tile0;                       // index of the chunk's first tile in the per-tile norm array
};

struct TcShared {
  uint64_t full[kMaxStages];
  uint64_t empty[kMaxStages];
  uint64_t accf[kAcc];
  uint64_t acce[kAcc];
  uint64_t normf[kAcc];
  uint64_t itemf[2];
  uint64_t aempty[2];
  uint64_t drain;
  uint32_t tmem;
  ItemDesc desc[2];
};

// Thread-private max-heap of R keys stored with stride kEpiThreads: the
// top is replaced by `key` and sifted down; returns the new top (known from
// the sift, so no reload).
__device__ __forceinline__ uint64_t heap_replace_top(uint64_t* h, int R, uint64_t key) {
  int i = 0;
  uint64_t new_top = key;
  for (;;) {
    const int c1 = 2 * i + 1;
    if (c1 >= R) break;
    const int c2 = c1 + 1;
    uint64_t vc = h[c1 * kEpiThreads];
    int c = c1;
    if (c2 < R) {
      const uint64_t v2 = h[c2 * kEpiThreads];
      if (v2 > vc) {
        vc = v2;
        c = c2;
      }
    }
    if (key >= vc) break;
    h[i * kEpiThreads] = vc;
    if (i == 0) new_top = vc;
    i = c;
  }
  h[i * kEpiThreads] = key;
  return new_top;
}

// Next work item from the global counter (one thread).
__device__ ItemDesc fetch_item(const TcArgs& a, int64_t total_items) {
  ItemDesc d;
  d.ntiles = -1;
  if (*reinterpret_cast<volatile int*>(a.err) != 0) return d;
  const int64_t item = static_cast<int64_t>(atomicAdd(a.work_counter, 1u));
  if (item >= total_items) return d;
  int lo = 0, hi = a.nlist;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (a.item_off[mid] <= item) lo = mid; else hi = mid;
  }
  const int l = lo;
  const int64_t local = item - a.item_off[l];
  const int ng = (a.list_cnt[l] + kTile - 1) / kTile;
  d.list = l;
  d.chunk = static_cast<int>(local / ng);
  d.group = static_cast<int>(local % ng);
  d.qcnt = min(kTile, a.list_cnt[l] - d.group * kTile);
  const int64_t lb = a.list_off[l];
  const int64_t r0 = lb + static_cast<int64_t>(d.chunk) * a.chunk_rows;
  const int64_t r1 = min(a.list_off[l + 1], r0 + static_cast<int64_t>(a.chunk_rows));
  d.row0 = static_cast<int>(r0);
  d.ntiles = static_cast<int>((r1 - r0 + kTile - 1) / kTile);
  d.tile0 = a.tile_off[l] + static_cast<int64_t>(d.chunk) * (a.chunk_rows / kTile);
  return d;
}

__global__ void __launch_bounds__(kTcThreads, 1)
    scan_bf16_kernel(const __grid_constant__ CUtensorMap tmap, TcArgs a) {
  extern __shared__ uint8_t smem_raw[];
  __shared__ TcShared sh;
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int kpad = a.kpad;
  const int S = a.stages;
  const uint32_t kblk_bytes = kTile * 128;                 // one 64-element K block of 128 rows
  const uint32_t tile_bytes = static_cast<uint32_t>(kpad / 64) * kblk_bytes;
  uint8_t* Abuf = smem;                                    // [2] A tiles
  uint8_t* stages = smem + 2 * tile_bytes;                 // [S] B tiles
  uint64_t* heap = reinterpret_cast<uint64_t*>(stages + static_cast<size_t>(S) * tile_bytes);  // [kGroups][R][128]
  float* nrm = reinterpret_cast<float*>(heap + static_cast<size_t>(kGroups) * a.R * kEpiThreads);  // [kAcc][128]
  int* meta_q = reinterpret_cast<int*>(nrm + kAcc * kTile);                 // [2][128]
  int* meta_j = meta_q + 2 * kTile;                                          // [2][128]
  uint64_t* meta_tau = reinterpret_cast<uint64_t*>(meta_j + 2 * kTile);      // [2][128]

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  int* err = a.err;

  if (warp == kMmaWarp) tmem_alloc(&sh.tmem, 512);
  if (tid == 0) {
    for (int s = 0; s < kMaxStages; ++s) {
      mbar_init(&sh.full[s], 1);
      mbar_init(&sh.empty[s], 1);
    }
    for (int b = 0; b < kAcc; ++b) {
      mbar_init(&sh.accf[b], 1);
      mbar_init(&sh.acce[b], kEpiThreads);
      mbar_init(&sh.normf[b], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&sh.itemf[i], kBuildWarps * 32);
      // A buffer / item slot free: the MMA warp's commit, the producer and
      // every epilogue thread.
      mbar_init(&sh.aempty[i], 2 + kGroups * kEpiThreads);
    }
    mbar_init(&sh.drain, 1);
    fence_barrier_init();
  }
  if (warp == kProdWarp && lane == 0) prefetch_tmap(&tmap);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sh.tmem;
  const int64_t total_items = a.item_off[a.nlist];

  if (warp >= kBuildWarp0) {
    // ---- item builders ---------------------------------------------------
    const int bt = tid - kBuildWarp0 * 32;
    ItemDesc nd;
    nd.ntiles = -1;
    if (bt == 0) nd = fetch_item(a, total_items);
    for (uint32_t it = 0;; ++it) {
      const int ab = static_cast<int>(it & 1u);
      bool okw = true;
      if (bt == 0) {
        okw = mbar_wait(&sh.aempty[ab], ((it >> 1) & 1u) ^ 1u, err, 31);
        if (!okw) nd.ntiles = -1;
        sh.desc[ab] = nd;
      }
      asm volatile("bar.sync 3, %0;\n" ::"n"(kBuildWarps * 32) : "memory");
      const ItemDesc d = sh.desc[ab];
      if (d.ntiles >= 0) {
        const int64_t qbase = a.list_qoff[d.list] + static_cast<int64_t>(d.group) * kTile;
        uint8_t* A = Abuf + ab * tile_bytes;
        for (int r = bt; r < kTile; r += kBuildWarps * 32) {
          int q = -1, j = 0;
          uint64_t tau = kEmpty;
          if (r < d.qcnt) {
            const uint32_t packed = static_cast<uint32_t>(a.list_q[qbase + r]);
            q = static_cast<int>(packed >> 16);
            j = static_cast<int>(packed & 0xffffu);
            // Best known R-th key of this query over the items finished so
            // far: an upper bound of its overall R-th key.
            tau = *reinterpret_cast<volatile unsigned long long*>(a.tau + q);
          }
          meta_q[ab * kTile + r] = q;
          meta_j[ab * kTile + r] = j;
          meta_tau[ab * kTile + r] = tau;
          const float* qrow = a.q + static_cast<size_t>(q < 0 ? 0 : q) * a.dpad;
#pragma unroll 4
          for (int k = 0; k < kpad; k += 8) {
            float4 lo = make_float4(0.f, 0.f, 0.f, 0.f), hi = lo;
            if (q >= 0 && k < a.dpad) {  // dpad is a multiple of 16: a row's 8 values are all in or all out
              lo = *reinterpret_cast<const float4*>(qrow + k);
              hi = *reinterpret_cast<const float4*>(qrow + k + 4);
            }
            __nv_bfloat162 p0 = __floats2bfloat162_rn(lo.x, lo.y), p1 = __floats2bfloat162_rn(lo.z, lo.w);
            __nv_bfloat162 p2 = __floats2bfloat162_rn(hi.x, hi.y), p3 = __floats2bfloat162_rn(hi.z, hi.w);
            *reinterpret_cast<uint4*>(A + sw128_offset_bf16(r, k, kblk_bytes)) =
                make_uint4(*reinterpret_cast<uint32_t*>(&p0), *reinterpret_cast<uint32_t*>(&p1),
                           *reinterpret_cast<uint32_t*>(&p2), *reinterpret_cast<uint32_t*>(&p3));
          }
        }
        fence_proxy_async_smem();
      }
      mbar_arrive(&sh.itemf[ab]);
      if (d.ntiles < 0) break;
      if (bt == 0) nd = fetch_item(a, total_items);
    }
  } else if (warp == kProdWarp) {
    // ---- TMA producer ------------------------------------------------------
    uint32_t p_idx = 0;
    if (lane == 0) {
      for (uint32_t it = 0;; ++it) {
        const int ab = static_cast<int>(it & 1u);
        if (!mbar_wait(&sh.itemf[ab], (it >> 1) & 1u, err, 32)) break;
        const ItemDesc d = sh.desc[ab];
        mbar_arrive(&sh.aempty[ab]);
        if (d.ntiles < 0) break;
        bool ok = true;
        for (int t = 0; t < d.ntiles; ++t, ++p_idx) {
          const int s = static_cast<int>(p_idx % static_cast<uint32_t>(S));
          const uint32_t par = ((p_idx / static_cast<uint32_t>(S)) & 1u) ^ 1u;
          if (!mbar_wait(&sh.empty[s], par, err, 11)) {
            ok = false;
            break;
          }
          uint8_t* dst = stages + s * tile_bytes;
          mbar_arrive_expect_tx(&sh.full[s], tile_bytes);
          const int r = d.row0 + t * kTile;
          for (int kb = 0; kb < kpad / 64; ++kb) tma_load_2d(dst + kb * kblk_bytes, &tmap, kb * 64, r, &sh.full[s]);
        }
        if (!ok) break;
      }
      // Drain: the last S loads may still be landing.
      const uint32_t first = p_idx > static_cast<uint32_t>(S) ? p_idx - static_cast<uint32_t>(S) : 0u;
      for (uint32_t i = first; i < p_idx; ++i)
        mbar_wait(&sh.full[i % static_cast<uint32_t>(S)], (i / static_cast<uint32_t>(S)) & 1u, nullptr, 0,
                  200000000LL);
    }
  } else if (warp == kMmaWarp) {
    // ---- MMA issuer (+ per-tile norms) --------------------------------------
    if (lane == 0) {
      const uint32_t idesc = idesc_bf16_f32(kTile, kTile);
      const int nk = kpad / 16;
      uint32_t m_idx = 0, m_cnt[kGroups] = {}, G = 0;
      for (uint32_t it = 0;; ++it) {
        const int ab = static_cast<int>(it & 1u);
        if (!mbar_wait(&sh.itemf[ab], (it >> 1) & 1u, err, 33)) break;
        const ItemDesc d = sh.desc[ab];
        if (d.ntiles < 0) break;
        tc_fence_after();
        const uint32_t a_base = smem_u32(Abuf + ab * tile_bytes);
        bool ok = true;
        for (int t = 0; t < d.ntiles; ++t, ++m_idx) {
          const int s = static_cast<int>(m_idx % static_cast<uint32_t>(S));
          if (!mbar_wait(&sh.full[s], (m_idx / static_cast<uint32_t>(S)) & 1u, err, 12)) {
            ok = false;
            break;
          }
          const int g = static_cast<int>((G + static_cast<uint32_t>(t)) & 1u);
          const uint32_t c = m_cnt[g];
          const int b = 2 * g + static_cast<int>(c & 1u);
          if (!mbar_wait(&sh.acce[b], ((c >> 1) & 1u) ^ 1u, err, 13)) {
            ok = false;
            break;
          }
          ++m_cnt[g];
          tc_fence_after();
          mbar_arrive_expect_tx(&sh.normf[b], kTile * 4);
          bulk_load(nrm + b * kTile, a.tile_norm + (d.tile0 + t) * kTile, kTile * 4, &sh.normf[b]);
          const uint32_t b_base = smem_u32(stages + s * tile_bytes);
          for (int k = 0; k < nk; ++k) {
            const uint32_t off = static_cast<uint32_t>(k >> 2) * kblk_bytes + static_cast<uint32_t>(k & 3) * 32u;
            mma_bf16(tmem + static_cast<uint32_t>(b * kTile), desc_sw128(a_base + off), desc_sw128(b_base + off),
                     idesc, k > 0 ? 1u : 0u);
          }
          mma_commit(&sh.empty[s]);
          mma_commit(&sh.accf[b]);
        }
        // A buffer ab is free once these MMAs have completed.
        mma_commit(&sh.aempty[ab]);
        if (!ok) break;
        G += static_cast<uint32_t>(d.ntiles);
      }
      // Drain: every MMA done before TMEM is released.
      mma_commit(&sh.drain);
      mbar_wait(&sh.drain, 0, nullptr, 0, 200000000LL);
    }
  } else {
    // ---- epilogue: thread = query (TMEM lane etid) ---------------------------
    const int grp = warp >> 2;
    const int etid = tid - grp * kEpiThreads;
    uint64_t* hp = heap + static_cast<size_t>(grp) * a.R * kEpiThreads + etid;
    const uint32_t lane_base = (32u * static_cast<uint32_t>(warp & 3)) << 16;
    uint32_t e_cnt = 0, G = 0;
    for (uint32_t it = 0;; ++it) {
      const int ab = static_cast<int>(it & 1u);
      bool ok = mbar_wait(&sh.itemf[ab], (it >> 1) & 1u, err, 34);
      if (!__all_sync(0xffffffffu, ok)) break;
      const ItemDesc d = sh.desc[ab];
      const int my_q = meta_q[ab * kTile + etid];
      const int my_j = meta_j[ab * kTile + etid];
      const uint64_t my_tau = meta_tau[ab * kTile + etid];
      mbar_arrive(&sh.aempty[ab]);
      if (d.ntiles < 0) break;
      // The heap starts full of the query's bound: only keys below enter.
      for (int e = 0; e < a.R; ++e) hp[e * kEpiThreads] = my_tau;
      uint64_t top = my_tau;
      // An all-ones top (no bound yet) admits every finite value.
      float thr_f = top == kEmpty ? FLT_MAX : ordered_to_float(static_cast<uint32_t>(top >> 32));
      for (int t = static_cast<int>((static_cast<uint32_t>(grp) ^ G) & 1u); t < d.ntiles; t += kGroups, ++e_cnt) {
        const int b = 2 * grp + static_cast<int>(e_cnt & 1u);
        const uint32_t par = (e_cnt >> 1) & 1u;
        ok = ok && mbar_wait(&sh.accf[b], par, err, 14) && mbar_wait(&sh.normf[b], par, err, 15);
        ok = __all_sync(0xffffffffu, ok);
        tc_fence_after();
        const float* nb = nrm + b * kTile;
        const uint32_t pos_t = static_cast<uint32_t>(d.row0 + t * kTile);
#pragma unroll 1
        for (int c = 0; c < kTile / 32; ++c) {
          uint32_t r[32];
          if (ok) {
            tmem_ld32(tmem + lane_base + static_cast<uint32_t>(b * kTile + c * 32), r);
            tmem_ld_wait();
          }
          if (ok && my_q >= 0) {
            // v = ||x||^2 - 2 q.x (rows past the list carry an infinite
            // norm); the columns' minimum against the bound decides whether
            // any of them needs a look.
            const float4* n4 = reinterpret_cast<const float4*>(nb + c * 32);
            float mn = INFINITY;
#pragma unroll
            for (int j4 = 0; j4 < 8; ++j4) {
              const float4 nv = n4[j4];
              const float v0 = fmaf(-2.0f, __uint_as_float(r[4 * j4 + 0]), nv.x);
              const float v1 = fmaf(-2.0f, __uint_as_float(r[4 * j4 + 1]), nv.y);
              const float v2 = fmaf(-2.0f, __uint_as_float(r[4 * j4 + 2]), nv.z);
              const float v3 = fmaf(-2.0f, __uint_as_float(r[4 * j4 + 3]), nv.w);
              r[4 * j4 + 0] = __float_as_uint(v0);
              r[4 * j4 + 1] = __float_as_uint(v1);
              r[4 * j4 + 2] = __float_as_uint(v2);
              r[4 * j4 + 3] = __float_as_uint(v3);
              mn = fminf(mn, fminf(fminf(v0, v1), fminf(v2, v3)));
            }
            if (mn <= thr_f) {
              uint32_t mq[4] = {0u, 0u, 0u, 0u};
#pragma unroll
              for (int j = 0; j < 32; ++j) mq[j & 3] |= (__uint_as_float(r[j]) <= thr_f ? 1u : 0u) << j;
              uint32_t mask = (mq[0] | mq[1]) | (mq[2] | mq[3]);
              const uint32_t pos0 = pos_t + static_cast<uint32_t>(c * 32);
              while (mask) {
                const int j = __ffs(mask) - 1;
                mask &= mask - 1;
                // r[j] by a 5-level select tree (no register indexing).
                uint32_t t16[16], t8[8], t4[4], t2[2];
#pragma unroll
                for (int i = 0; i < 16; ++i) t16[i] = (j & 1) ? r[2 * i + 1] : r[2 * i];
#pragma unroll
                for (int i = 0; i < 8; ++i) t8[i] = (j & 2) ? t16[2 * i + 1] : t16[2 * i];
#pragma unroll
                for (int i = 0; i < 4; ++i) t4[i] = (j & 4) ? t8[2 * i + 1] : t8[2 * i];
#pragma unroll
                for (int i = 0; i < 2; ++i) t2[i] = (j & 8) ? t4[2 * i + 1] : t4[2 * i];
                const uint32_t hv = (j & 16) ? t2[1] : t2[0];
                const uint64_t key = (static_cast<uint64_t>(ordered_bits(__uint_as_float(hv))) << 32) |
                                     (pos0 + static_cast<uint32_t>(j));
                if (key < top) {
                  top = heap_replace_top(hp, a.R, key);
                  thr_f = top == kEmpty ? FLT_MAX : ordered_to_float(static_cast<uint32_t>(top >> 32));
                }
              }
            }
          }
        }
        tc_fence_before();
        mbar_arrive(&sh.acce[b]);
      }
      // Partial result of this (query, chunk): the group's R keys; seed
      // entries are not results.
      if (my_q >= 0) {
        const int64_t slot = a.slot_base[static_cast<int64_t>(my_q) * a.P + my_j] + d.chunk;
        uint64_t* out = a.part + (slot * kGroups + grp) * a.R;
        for (int e = 0; e < a.R; ++e) {
          const uint64_t v = hp[e * kEpiThreads];
          out[e] = v == my_tau ? kEmpty : v;
        }
        // A heap holding R real keys bounds the query's R-th key: publish it.
        if (top < my_tau) atomicMin(reinterpret_cast<unsigned long long*>(a.tau + my_q), top);
      }
      if (!ok) break;
      G += static_cast<uint32_t>(d.ntiles);
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == kMmaWarp) {
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

__global__ void __launch_bounds__(512) rerank_kernel(const uint64_t* __restrict__ part,
                                                     const int64_t* __restrict__ slot_base, int P, int R, int k,
                                                     const float* __restrict__ codes, const float* __restrict__ q,
                                                     int dpad, const int64_t* __restrict__ ids, float* __restrict__ D,
                                                     int64_t* __restrict__ I, const uint64_t* __restrict__ part2,
                                                     const int64_t* __restrict__ slot_base2, int P2,
                                                     const uint64_t* __restrict__ tau, const int* __restrict__ only) {
  extern __shared__ uint64_t s_keys[];  // pow2(R) approx, then pow2(R) exact
  __shared__ SelectShared sh_sel;
  const int qi = blockIdx.x;
  if (only && !only[qi]) return;
  const int n2 = pow2_ceil(R < 2 ? 2 : R);
  uint64_t* s_appr = s_keys;
  uint64_t* s_exact = s_keys + n2;
  const int64_t s0 = slot_base[static_cast<int64_t>(qi) * P];
  const int64_t s1 = slot_base[static_cast<int64_t>(qi + 1) * P];
  const uint64_t* src = part + s0 * kGroups * R;
  const int m1 = static_cast<int>((s1 - s0) * kGroups * R);
  const uint64_t* src2 = nullptr;
  int m2 = 0;
  if (part2) {
    const int64_t t0 = slot_base2[static_cast<int64_t>(qi) * P2];
    const int64_t t1 = slot_base2[static_cast<int64_t>(qi + 1) * P2];
    src2 = part2 + t0 * kGroups * R;
    m2 = static_cast<int>((t1 - t0) * kGroups * R);
  }
  // The query's final bound is at or above its R-th key: keys above it
  // cannot be among the R best, so they drop out of the selection.
  const uint64_t lim = tau ? tau[qi] : kEmpty;
  auto key_at = [&](int i) -> uint64_t {
    const uint64_t key = i < m1 ? src[i] : src2[i - m1];
    return key <= lim ? key : kEmpty;
  };
  block_topk_sorted(key_at, m1 + m2, R, sh_sel, s_appr);
  const float* qrow = q + static_cast<size_t>(qi) * dpad;
  for (int i = threadIdx.x; i < n2; i += blockDim.x) {
    uint64_t key = kEmpty;
    if (i < R && s_appr[i] != kEmpty) {
      const uint32_t pos = key_tie(s_appr[i]);
      const float acc = exact_l2_seq(codes + static_cast<size_t>(pos) * dpad, qrow, dpad);
      if (acc < FLT_MAX) key = make_key(acc, pos);
    }
    s_exact[i] = key;
  }
  __syncthreads();
  block_bitonic_sort(s_exact, n2);
  for (int j = threadIdx.x; j < k; j += blockDim.x) {
    const uint64_t key = j < n2 ? s_exact[j] : kEmpty;
    const size_t o = static_cast<size_t>(qi) * k + j;
    D[o] = key == kEmpty ? FLT_MAX : key_dist(key);
    I[o] = key == kEmpty ? -1 : ids[key_tie(key)];
  }
}

// Re-rank with one warp per query: the keys at or under the query's final
// bound (at most a few times R of them) are compacted by ballot into a
// per-warp buffer, sorted, the best R recomputed exactly (sequential FP32,
// one candidate per lane) and sorted again.  A query with more than 8192
// slot keys or more than kRerankCap keys under its bound is flagged for the
// CTA kernel.
constexpr int kRerankCap = 256;
constexpr int kRerankWarps = 8;

__global__ void __launch_bounds__(kRerankWarps * 32) rerank_warp_kernel(
    const uint64_t* __restrict__ part, const int64_t* __restrict__ slot_base, int nq, int P, int R, int k,
    const float* __restrict__ codes, const float* __restrict__ q, int dpad, const int64_t* __restrict__ ids,
    float* __restrict__ D, int64_t* __restrict__ I, const uint64_t* __restrict__ tau, int* __restrict__ overflow) {
  __shared__ uint64_t s_cand[kRerankWarps][kRerankCap];
  __shared__ uint64_t s_ex[kRerankWarps][64];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int qi = blockIdx.x * kRerankWarps + wib;
  if (qi >= nq) return;
  uint64_t* cand = s_cand[wib];
  uint64_t* ex = s_ex[wib];
  const int64_t s0 = slot_base[static_cast<int64_t>(qi) * P];
  const int64_t s1 = slot_base[static_cast<int64_t>(qi + 1) * P];
  const uint64_t* src = part + s0 * kGroups * R;
  const int m = static_cast<int>((s1 - s0) * kGroups * R);
  const uint64_t lim = tau[qi];
  if (m > 256 * 32) {
    // Many slots (a wide nprobe): the CTA kernel scans them faster.
    if (lane == 0) overflow[qi] = 1;
    return;
  }
  int cnt = 0;
#pragma unroll 4
  for (int base = 0; base < m; base += 32) {
    const int i = base + lane;
    const uint64_t key = i < m ? src[i] : kEmpty;
    const bool pass = key != kEmpty && key <= lim;
    const unsigned b = __ballot_sync(0xffffffffu, pass);
    const int pos = cnt + __popc(b & ((1u << lane) - 1u));
    if (pass && pos < kRerankCap) cand[pos] = key;
    cnt += __popc(b);
  }
  if (cnt > kRerankCap) {
    if (lane == 0) overflow[qi] = 1;
    return;
  }
  if (lane == 0) overflow[qi] = 0;
  const int n2 = pow2_ceil(cnt < 2 ? 2 : cnt);
  for (int i = cnt + lane; i < n2; i += 32) cand[i] = kEmpty;
  __syncwarp();
  warp_bitonic_sort(cand, n2, lane);
  const int nr = min(R, cnt);
  const float* qrow = q + static_cast<size_t>(qi) * dpad;
  for (int j = lane; j < 64; j += 32) {
    uint64_t key = kEmpty;
    if (j < nr) {
      const uint32_t pos = key_tie(cand[j]);
      const float acc = exact_l2_seq(codes + static_cast<size_t>(pos) * dpad, qrow, dpad);
      if (acc < FLT_MAX) key = make_key(acc, pos);
    }
    ex[j] = key;
  }
  __syncwarp();
  const int e2 = pow2_ceil(nr < 2 ? 2 : nr);
  warp_bitonic_sort(ex, e2, lane);
  for (int j = lane; j < k; j += 32) {
    const uint64_t key = j < e2 ? ex[j] : kEmpty;
    const size_t o = static_cast<size_t>(qi) * k + j;
    D[o] = key == kEmpty ? FLT_MAX : key_dist(key);
    I[o] = key == kEmpty ? -1 : ids[key_tie(key)];
  }
}

// Upper bound of each query's R-th approximate key before the scan, from the
// first S rows of the query's nearest list.  The bound is computed from the
// same BF16 operands the scan multiplies (the query rounded to BF16 exactly
// as the scan's A tile, the BF16 codes), so the scan's value
// ||x||^2 - 2 q~.x~ and the one here differ only by the order and width of
// the FP32 accumulation of 128 exact BF16 products: each is within
// 128 * 2^-19 * sum|q~_i x~_i| <= 2.5e-4 ||q|| max||x|| of the exact sum even
// if the tensor cores kept only 19 bits per addition.  The margin,
// 1e-3 ||q|| max||x|| + 2e-5 (max||x||^2 + |v|), covers twice that plus the
// FP32 rounding of the combination, so the R-th value here plus the margin
// is never below the R-th value the scan sees, and a seed never drops a key
// of the scan's top R.
//
// List-major: one CTA per list stages the list's first S BF16 rows in shared
// memory once; for each query whose nearest list it is (probe rank 0 in the
// list-major work description) in turn, thread t computes row t's value with
// the query broadcast from shared memory, and a 32-step radix selection over
// the CTA (one barrier count per bit) finds the R-th smallest.
constexpr int kSeedRows = 256;
constexpr int kSeedWarps = 8;

__global__ void __launch_bounds__(kSeedWarps * 32) tau_seed_kernel(
    const float* __restrict__ q, int dpad, int kpad, const __nv_bfloat16* __restrict__ codes,
    const int64_t* __restrict__ list_off, const int64_t* __restrict__ list_qoff, const int32_t* __restrict__ list_q,
    const float* __restrict__ xnorm, int S, int R, const float* __restrict__ maxnorm, uint64_t* __restrict__ tau,
    const int32_t* __restrict__ probes, int P) {
  extern __shared__ __align__(16) uint8_t s_seed_raw[];
  __shared__ float s_xn[kSeedRows];
  __shared__ int s_qs[kSeedWarps * 32];
  __shared__ int s_nq;
  __shared__ float s_qn;
  const int tid = threadIdx.x, lane = tid & 31, wib = tid >> 5;
  // One CTA per list (its rows serve every query whose nearest list it is),
  // or, for small batches (probes given), one CTA per query.
  const bool by_query = probes != nullptr;
  int l;
  int64_t e0, e1;
  if (by_query) {
    l = probes[static_cast<size_t>(blockIdx.x) * P];
    if (l < 0) return;
    e0 = 0;
    e1 = 1;
  } else {
    l = blockIdx.x;
    e0 = list_qoff[l];
    e1 = list_qoff[l + 1];
    bool mine = false;
    for (int64_t e = e0 + tid; e < e1 && !mine; e += blockDim.x) mine = (list_q[e] & 0xffff) == 0;
    if (!__syncthreads_or(mine)) return;
  }
  const int64_t b = list_off[l];
  const int n = static_cast<int>(min(static_cast<int64_t>(S), list_off[l + 1] - b));
  if (n < R) return;  // no seed: tau stays empty
  const int stride = kpad * 2 + 16;  // bytes per staged row (padding spreads banks)
  uint8_t* rows = s_seed_raw;
  float* qbuf = reinterpret_cast<float*>(s_seed_raw + static_cast<size_t>(S) * stride);
  const int cpr = kpad / 8;  // 16-byte chunks per row
  for (int i = tid; i < n * cpr; i += blockDim.x) {
    const int r = i / cpr, c = i - r * cpr;
    cp_async16(rows + static_cast<size_t>(r) * stride + c * 16, codes + static_cast<size_t>(b + r) * kpad + c * 8, true);
  }
  cp_async_commit();
  for (int r = tid; r < n; r += blockDim.x) s_xn[r] = xnorm[b + r];
  const float mn = *maxnorm;
  cp_async_wait<0>();
  // Rounds over the list's entries: the queries whose nearest list this is
  // are gathered in shared memory, then one warp per query.
  for (int64_t r0 = e0; r0 < e1; r0 += blockDim.x) {
    if (tid == 0) s_nq = 0;
    __syncthreads();
    if (r0 + tid < e1) {
      const uint32_t ent =
          by_query ? (static_cast<uint32_t>(blockIdx.x) << 16) : static_cast<uint32_t>(list_q[r0 + tid]);
      if ((ent & 0xffff) == 0) s_qs[atomicAdd(&s_nq, 1)] = static_cast<int>(ent >> 16);
    }
    __syncthreads();
    const int nqr = s_nq;
    // Each query in turn, the whole CTA: thread t takes row t, then a
    // 32-step radix selection over the CTA finds the R-th smallest value.
    for (int t = 0; t < nqr; ++t) {
      const int qi = s_qs[t];
      const float* qrow = q + static_cast<size_t>(qi) * dpad;
      for (int c = tid; c < kpad; c += blockDim.x) qbuf[c] = c < dpad ? __bfloat162float(__float2bfloat16_rn(qrow[c])) : 0.0f;
      if (wib == 0) {
        float qn = 0.0f;
        for (int c = lane; c < dpad; c += 32) qn = fmaf(qrow[c], qrow[c], qn);
        for (int o = 16; o > 0; o >>= 1) qn += __shfl_xor_sync(0xffffffffu, qn, o);
        if (lane == 0) s_qn = qn;
      }
      __syncthreads();
      uint32_t key = 0xFFFFFFFFu;
      if (tid < n) {
        const uint8_t* xr = rows + static_cast<size_t>(tid) * stride;
        // Four partial sums (any order is within the margin).
        float d0 = 0.0f, d1 = 0.0f, d2 = 0.0f, d3 = 0.0f;
#pragma unroll 4
        for (int c = 0; c < kpad; c += 8) {
          const uint4 xv = *reinterpret_cast<const uint4*>(xr + c * 2);
          const float4 qa = *reinterpret_cast<const float4*>(qbuf + c);
          const float4 qb = *reinterpret_cast<const float4*>(qbuf + c + 4);
          d0 = fmaf(qa.x, __uint_as_float(xv.x << 16), d0);
          d1 = fmaf(qa.y, __uint_as_float(xv.x & 0xffff0000u), d1);
          d2 = fmaf(qa.z, __uint_as_float(xv.y << 16), d2);
          d3 = fmaf(qa.w, __uint_as_float(xv.y & 0xffff0000u), d3);
          d0 = fmaf(qb.x, __uint_as_float(xv.z << 16), d0);
          d1 = fmaf(qb.y, __uint_as_float(xv.z & 0xffff0000u), d1);
          d2 = fmaf(qb.z, __uint_as_float(xv.w << 16), d2);
          d3 = fmaf(qb.w, __uint_as_float(xv.w & 0xffff0000u), d3);
        }
        key = ordered_bits(fmaf(-2.0f, (d0 + d1) + (d2 + d3), s_xn[tid]));
      }
      uint32_t prefix = 0;
      int need = R;
      for (int bit = 31; bit >= 0; --bit) {
        const uint32_t hmask = bit == 31 ? 0u : (0xFFFFFFFFu << (bit + 1));
        const bool zero_here = (key & hmask) == prefix && ((key >> bit) & 1u) == 0u;
        const int c0 = __syncthreads_count(zero_here);
        if (c0 < need) {
          need -= c0;
          prefix |= 1u << bit;
        }
      }
      if (tid == 0) {
        const float vR = ordered_to_float(prefix);
        const float margin = 1e-3f * sqrtf(s_qn) * mn + 2e-5f * (mn * mn + fabsf(vR)) + 1e-30f;
        tau[qi] = (static_cast<uint64_t>(ordered_bits(vR + margin)) << 32) | 0xffffffffull;
      }
      __syncthreads();
    }
    __syncthreads();
  }
}

// One block per list: the list's norms in 128-row tiles, +inf past its end
// (so rows a tile reads beyond its list can never pass a bound).
__global__ void tile_norms_kernel(const float* __restrict__ norms, const int64_t* __restrict__ list_off,
                                  const int64_t* __restrict__ tile_off, float* __restrict__ tile_norm) {
  const int l = blockIdx.x;
  const int64_t b = list_off[l], n = list_off[l + 1] - b;
  float* dst = tile_norm + tile_off[l] * kTile;
  const int64_t m = (tile_off[l + 1] - tile_off[l]) * kTile;
  for (int64_t i = threadIdx.x; i < m; i += blockDim.x) dst[i] = i < n ? norms[b + i] : INFINITY;
}

__global__ void max_norm_kernel(const float* __restrict__ norms, size_t n, float* __restrict__ out) {
  float m = 0.0f;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    m = fmaxf(m, norms[i]);
  for (int off = 16; off > 0; off >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, off));
  if ((threadIdx.x & 31) == 0) atomicMax(reinterpret_cast<int*>(out), __float_as_int(m));
}

__global__ void sqrt_inplace_kernel(float* v) { *v = sqrtf(*v) * 1.0001f; }

__global__ void to_bf16_kernel(const float* __restrict__ src, size_t n, int dpad, int kpad,
                               __nv_bfloat16* __restrict__ dst) {
  const size_t total = n * static_cast<size_t>(kpad);
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const size_t r = i / kpad;
    const int c = static_cast<int>(i - r * kpad);
    dst[i] = __float2bfloat16_rn(c < dpad ? src[r * dpad + c] : 0.0f);
  }
}

// Self-test of the bounded mbarrier wait: one thread initialises an mbarrier
// that nothing ever arrives on and waits for its first phase with a budget of
// `budget` clock cycles.  No copy or MMA is in flight, so giving up is the
// only way out; the wait records `code` in *err and the kernel returns.
__global__ void wait_selftest_kernel(long long budget, int code, int* err, long long* waited) {
  __shared__ uint64_t bar;
  if (threadIdx.x != 0) return;
  mbar_init(&bar, 1);
  fence_barrier_init();
  const long long t0 = clock64();
  const bool done = mbar_wait(&bar, 0u, err, code, budget);
  *waited = done ? -1 : clock64() - t0;
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    HB_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    HB_CHECK(p && q == cudaDriverEntryPointSuccess, HB_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

}  // namespace

size_t scan_bf16_smem_bytes(int kpad, int R, int stages) {
  const size_t tile = static_cast<size_t>(kpad / 64) * kTile * 128;
  return 1024 + tile * (2 + stages) + static_cast<size_t>(kGroups) * R * kEpiThreads * 8 +
         static_cast<size_t>(kAcc) * kTile * 4 + 2 * kTile * (4 + 4 + 8);
}

int scan_bf16_keys_per_slot(int R) { return kGroups * R; }

int scan_bf16_stages(int kpad, int R) {
  int s = kMaxStages;
  while (s > 2 && scan_bf16_smem_bytes(kpad, R, s) > kSmemCap) --s;
  return s;
}

int scan_bf16_max_R(int kpad) {
  int R = 64;
  while (R > 1 && scan_bf16_smem_bytes(kpad, R, 2) > kSmemCap) --R;
  return R;
}

void make_bf16_tensor_map(void* tmap_out, const void* codes_bf16, size_t rows, int kpad) {
  CUtensorMap* m = static_cast<CUtensorMap*>(tmap_out);
  cuuint64_t dims[2] = {static_cast<cuuint64_t>(kpad), static_cast<cuuint64_t>(rows)};
  cuuint64_t strides[1] = {static_cast<cuuint64_t>(kpad) * 2};
  cuuint32_t box[2] = {64, kTile};
  cuuint32_t es[2] = {1, 1};
  CUresult r = tensor_map_encoder()(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(codes_bf16), dims,
                                    strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  HB_CHECK(r == CUDA_SUCCESS, HB_ERR_CUDA, "cuTensorMapEncodeTiled failed");
}

void launch_to_bf16(const float* src, size_t n, int dpad, int kpad, void* dst, cudaStream_t st) {
  if (!n) return;
  size_t g = (n * kpad + 255) / 256;
  if (g > 148u * 64u) g = 148u * 64u;
  to_bf16_kernel<<<static_cast<unsigned>(g), 256, 0, st>>>(src, n, dpad, kpad, static_cast<__nv_bfloat16*>(dst));
  HB_CUDA(cudaGetLastError());
}

void launch_scan_bf16(const void* tmap, const TcArgs& a, int num_sms, cudaStream_t st) {
  HB_CHECK(a.kpad == 64 || a.kpad == 128, HB_ERR_INVALID, "the BF16 scan supports d <= 128");
  HB_CHECK(a.R >= 1 && a.R <= 64, HB_ERR_INVALID, "rerank candidates per query must be in [1, 64]");
  HB_CHECK(a.chunk_rows % kTile == 0, HB_ERR_INVALID, "BF16 scan chunks must be whole tiles");
  HB_CHECK(a.stages >= 2 && a.stages <= kMaxStages, HB_ERR_INVALID, "bad stage count");
  const size_t smem = scan_bf16_smem_bytes(a.kpad, a.R, a.stages);
  HB_CHECK(smem <= kSmemCap, HB_ERR_INVALID, "rerank candidates too many for the BF16 scan's shared memory");
  HB_CUDA(cudaFuncSetAttribute(scan_bf16_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  scan_bf16_kernel<<<num_sms, kTcThreads, smem, st>>>(*static_cast<const CUtensorMap*>(tmap), a);
  HB_CUDA(cudaGetLastError());
}

void launch_rerank(const uint64_t* part, const int64_t* slot_base, int nq, int P, int R, int k, const float* codes,
                   const float* q, int dpad, const int64_t* ids, float* D, int64_t* I, cudaStream_t st,
                   const uint64_t* part2, const int64_t* slot_base2, int P2, const uint64_t* tau, int* overflow) {
  if (nq <= 0) return;
  if (tau && !part2 && overflow && R <= 64 && nq >= 1024) {
    // Warp per query; the rare query with too many keys under its bound
    // goes through the CTA kernel.
    HB_CHECK(k <= R, HB_ERR_INVALID, "k must not exceed the re-ranked candidates");
    rerank_warp_kernel<<<(nq + kRerankWarps - 1) / kRerankWarps, kRerankWarps * 32, 0, st>>>(
        part, slot_base, nq, P, R, k, codes, q, dpad, ids, D, I, tau, overflow);
    HB_CUDA(cudaGetLastError());
    const int n2 = pow2_ceil(R < 2 ? 2 : R);
    const size_t smem = static_cast<size_t>(2 * n2) * 8 + 64;
    rerank_kernel<<<nq, 512, smem, st>>>(part, slot_base, P, R, k, codes, q, dpad, ids, D, I, nullptr, nullptr, 0, tau,
                                         overflow);
    HB_CUDA(cudaGetLastError());
    return;
  }
  HB_CHECK(k <= R, HB_ERR_INVALID, "k must not exceed the re-ranked candidates");
  const int n2 = pow2_ceil(R < 2 ? 2 : R);
  const size_t smem = static_cast<size_t>(2 * n2) * 8 + 64;
  // Small batches get wider CTAs (each query's selection is the whole job).
  rerank_kernel<<<nq, nq < 1024 ? 256 : 128, smem, st>>>(part, slot_base, P, R, k, codes, q, dpad, ids, D, I, part2,
                                                         slot_base2, P2, tau, nullptr);
  HB_CUDA(cudaGetLastError());
}

void launch_tau_seed(const float* q, int nq, int dpad, int kpad, const void* codes_bf16, const int64_t* list_off,
                     int nlist, const int64_t* list_qoff, const int32_t* list_q, const float* xnorm, int S, int R,
                     const float* maxnorm, uint64_t* tau, cudaStream_t st, const int32_t* probes, int P) {
  if (nq <= 0) return;
  HB_CHECK(kpad == 64 || kpad == 128, HB_ERR_INVALID, "the BF16 scan supports d <= 128");
  HB_CHECK(S >= 1 && S <= kSeedRows && R >= 1 && R <= S, HB_ERR_INVALID, "seed sample out of range");
  HB_CUDA(cudaMemsetAsync(tau, 0xff, static_cast<size_t>(nq) * sizeof(uint64_t), st));
  const size_t smem = static_cast<size_t>(S) * (kpad * 2 + 16) + static_cast<size_t>(kpad) * 4;
  HB_CUDA(cudaFuncSetAttribute(tau_seed_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  const bool by_query = probes && static_cast<long long>(nq) * 4 < nlist;
  tau_seed_kernel<<<by_query ? nq : nlist, kSeedWarps * 32, smem, st>>>(
      q, dpad, kpad, static_cast<const __nv_bfloat16*>(codes_bf16), list_off, list_qoff, list_q, xnorm, S, R, maxnorm,
      tau, by_query ? probes : nullptr, P);
  HB_CUDA(cudaGetLastError());
}

void launch_wait_selftest(long long budget, int code, int* err, long long* waited, cudaStream_t st) {
  HB_CHECK(budget >= 0, HB_ERR_INVALID, "wait budget must be non-negative");
  wait_selftest_kernel<<<1, 32, 0, st>>>(budget, code, err, waited);
  HB_CUDA(cudaGetLastError());
}

void launch_tile_norms(const float* norms, const int64_t* list_off, int nlist, const int64_t* tile_off,
                       float* tile_norm, cudaStream_t st) {
  if (nlist <= 0) return;
  tile_norms_kernel<<<nlist, 256, 0, st>>>(norms, list_off, tile_off, tile_norm);
  HB_CUDA(cudaGetLastError());
}

void launch_max_norm(const float* norms, size_t n, float* out, cudaStream_t st) {
  HB_CUDA(cudaMemsetAsync(out, 0, sizeof(float), st));
  if (n) {
    size_t g = (n + 255) / 256;
    if (g > 1024) g = 1024;
    max_norm_kernel<<<static_cast<unsigned>(g), 256, 0, st>>>(norms, n, out);
  }
  sqrt_inplace_kernel<<<1, 1, 0, st>>>(out);
  HB_CUDA(cudaGetLastError());
}

}  // namespace hb

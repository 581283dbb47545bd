// BF16 tensor-core list scan (tcgen05 + TMA) and the exact FP32 re-rank,
// whose result equals the exact FP32 scan's bit for bit.
//
// Error bound.  The tensor cores work on residuals to the list centroid c_l:
// for a query q, a probed list l and a stored row x of l the scan forms
//   w(x) = cd + ||r||^2 - 2 q~'.r~   (q' = q - c_l, r = x - c_l in FP32; q~', r~
//                                    their BF16 roundings; cd = ||q'||^2 and
//                                    ||r||^2 FP32 sums; the dot product on the
//                                    tensor cores with FP32 accumulation)
// and the reference's distance is d(x) = the sequential unfused FP32 sum of
// (q_i - x_i)^2 (src/utils.h:480-487).  With Q = ||q'||, R = the list's largest
// ||r||, u = 2^-24 and D = ||q - x||^2 = ||q' - r||^2 <= (Q + R)^2:
//   |2 q~'.r~ - 2 q'.r| <= 2 (2^-8 + 2^-16) Q R   BF16 (and FP32 residual)
//                                                 rounding of both operands
//                        + 2 * 2^-10 Q R           FP32 accumulation of kpad <= 128
//                                                 exact products (even with only
//                                                 17 bits kept per addition)
//   |cd - Q^2|, | ||r||^2 stored - R-part |  <= (d + 3) u (Q^2 + R^2)
//   rounding of w (two additions)            <= 2 u (Q + R)^2
//   | d(x) - D |                             <= (d + 3) u D
// so |w(x) - d(x)| <= eps(q, l) = 1.0625 * (2 (2^-8 + 2^-10 + 2^-16) Q R
// + (d + 3) u (Q^2 + R^2) + (d + 5) u (Q + R)^2), a bound per (query, list)
// (d may be replaced by dpad >= d).  Residuals keep Q and R at the scale of
// a list's spread, not of the data's distance from the origin.  Each row
// therefore has a lower bound lb(x) = w(x) - eps(q, l_x) and an upper bound
// ub(x) = w(x) + eps(q, l_x) of its distance (rounded outwards).  Let U be
// any value at least the k-th smallest ub over some k probed rows: k rows
// have d <= U, so the k-th smallest distance d_k is at most U, and every row
// of the exact top k (ties at the k-th distance included) has
// lb <= d <= d_k <= U.  Re-ranking exactly every row with lb <= U, by (FP32
// distance, position) like the exact scan, therefore returns the exact
// scan's result.  A bound per list rather than the largest over the probed
// lists keeps one far or wide list from loosening every other list's test.
//
// Admission.  A row is appended to its query's candidate buffer (key = its
// lower bound, position; its upper bound alongside) when lb <= U(q), i.e.
// w <= U + eps(q, l).  U starts at the seed bound (the k-th smallest upper
// bound over the first rows of the query's nearest list) and, for k <= 16,
// falls to the k-th smallest upper bound a thread knows for the query as the
// scan goes, shared between work items through an atomicMin; a published U
// stands in for k upper bounds.  Every row of the exact top k is admitted
// whatever the order.  The re-rank takes U as the k-th smallest upper bound
// over the appended rows and recomputes those with lb <= U with the
// reference's loop.  A query whose buffer overflows is flagged; the host
// searches it again with the exact FP32 scan.
//
// Work items are the list-major items of the exact scan (list, chunk of
// rows, group of <= 128 queries probing the list).  Per item the CTA holds
// the group's BF16 queries as the MMA's A operand (128 x K, K-major, 128-byte
// swizzle) and streams the chunk's rows as B operand tiles of 128 rows (TMA
// 2-D loads with the same swizzle into a ring of stages).  One thread issues
// tcgen05.mma (M 128 queries x N 128 rows x K 16) into one of four TMEM
// accumulators; the epilogue warps read their TMEM lanes back (thread =
// query, 128 columns = rows), form w and append the rows under the query's
// bound.  The builders form the A tile, BF16(q - c_l) for the item's list,
// from the FP32 queries.
//
// Warp roles (512 threads, 128 registers each), all running ahead of each
// other through mbarriers, with no CTA-wide barrier between items:
//   warps 0-11  three epilogue groups (each four warps = the four TMEM lane
//               quarters); tile t of the CTA's global tile sequence goes to
//               group t % 3 and accumulator t % 4 (three groups keep more
//               warps on the epilogue, which bounds the kernel);
//   warp 12     TMA producer of the B tiles;
//   warp 13     MMA issuer; it also copies each tile's 128 row norms
//               (a padded per-tile norm array) next to the accumulator;
//   warps 14-15 item builders: fetch the next item from the global work
//               counter, gather its BF16 query rows and bounds and write its
//               A tile into the second A buffer while the current item runs.
// Every mbarrier wait is bounded (TcArgs::wait_budget cycles); on a timeout
// the kernel records an error, the roles stop taking work, copies and MMAs
// in flight are drained and TMEM is freed.
#include <cudaTypedefs.h>
#include <cuda.h>
#include <cuda_runtime.h>

#include <cuda_bf16.h>

#include <algorithm>

#include "hb_device.cuh"
#include "hb_internal.hpp"
#include "hb_select.cuh"
#include "hb_sm100.cuh"

namespace hb {
namespace {

using namespace sm100;

constexpr int kGroups = 3;                         // epilogue warpgroups, tile t -> group t % 3
constexpr int kEpiThreads = 128;                   // threads per epilogue group (= queries per item)
constexpr int kBuildWarps = 2;
constexpr int kProdWarp = kGroups * 4, kMmaWarp = kGroups * 4 + 1, kBuildWarp0 = kGroups * 4 + 2;
constexpr int kTcThreads = (kBuildWarp0 + kBuildWarps) * 32;
constexpr int kTile = 128;     // rows per B tile, queries per item (M)
constexpr int kMaxStages = 4;
constexpr int kAcc = 4;                            // TMEM accumulators of 128 columns, tile t -> t % 4
constexpr size_t kSmemCap = 225 * 1024;            // dynamic shared memory budget
constexpr int kTightK = kFilterTightK;             // largest k whose bound tightens during the scan
constexpr int kStage = 8;                          // admitted keys staged per epilogue thread before a flush

// The error bound of one (query, list) pair (see the top of this file):
// Q = ||q - c_l|| from its FP32 square cd, R = the list's largest residual
// norm, d the dimension.
__device__ __forceinline__ float pair_eps(float cd, float R, int d) {
  const float Q = sqrtf(cd) * 1.0001f + 1e-30f;
  const float u = 5.9604645e-8f;  // 2^-24
  const float c1 = 0.00390625f + 0.0009765625f + 1.52587890625e-5f;
  return 1.0625f * (2.0f * c1 * Q * R + (d + 3) * u * (R * R + Q * Q) + (d + 5) * u * (Q + R) * (Q + R));
}

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

// Next work item from the global counter, by one warp: lane 0 takes the
// item, the warp finds its list with a 32-way search of item_off (three
// rounds for 4096 lists instead of twelve dependent loads).
__device__ ItemDesc fetch_item(const TcArgs& a, int64_t total_items, int lane) {
  ItemDesc d;
  d.ntiles = -1;
  int64_t item = 0;
  if (lane == 0)
    item = *reinterpret_cast<volatile int*>(a.err) != 0 ? total_items
                                                        : static_cast<int64_t>(atomicAdd(a.work_counter, 1u));
  item = __shfl_sync(0xffffffffu, item, 0);
  if (item >= total_items) return d;
  // item_off[lo] <= item < item_off[hi]
  int lo = 0, hi = a.nlist;
  while (hi - lo > 1) {
    const int step = max(1, (hi - lo) / 32);
    const int p = lo + (lane + 1) * step;
    const bool le = p < hi && a.item_off[p] <= item;
    const int n = __popc(__ballot_sync(0xffffffffu, le));  // the true lanes are a prefix
    // With every probe at or under the item the list lies past the last
    // probe and hi stays; otherwise probe n is above it.
    if (n < 32) hi = min(hi, lo + (n + 1) * step);
    lo += n * step;
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

// KT = kTightK: the bound tightens (k <= 16); KT = 0: it stays at the seed.
template <int KT>
__global__ void __launch_bounds__(kTcThreads, 1)
    scan_bf16_kernel(const __grid_constant__ CUtensorMap tmap, TcArgs a) {
  constexpr int KB = KT > 0 ? KT : 1;
  extern __shared__ uint8_t smem_raw[];
  __shared__ TcShared sh;
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int kpad = a.kpad;
  const int S = a.stages;
  const long long budget = a.wait_budget;
  const uint32_t kblk_bytes = kTile * 128;                 // one 64-element K block of 128 rows
  const uint32_t tile_bytes = static_cast<uint32_t>(kpad / 64) * kblk_bytes;
  uint8_t* Abuf = smem;                                    // [2] A tiles
  uint8_t* stages = smem + 2 * tile_bytes;                 // [S] B tiles
  float* nrm = reinterpret_cast<float*>(stages + static_cast<size_t>(S) * tile_bytes);  // [kAcc][128]
  int* meta_q = reinterpret_cast<int*>(nrm + kAcc * kTile);                 // [2][128]
  float* meta_thr = reinterpret_cast<float*>(meta_q + 2 * kTile);           // [2][128]
  float* meta_eps = meta_thr + 2 * kTile;                                   // [2][128] eps(q, l)
  float* meta_cd = meta_eps + 2 * kTile;                                    // [2][128] ||q - c_l||^2
  float* s_cent = meta_cd + 2 * kTile;                                      // [2][128] the item's centroid
  uint64_t* staging = reinterpret_cast<uint64_t*>(s_cent + 2 * kTile);      // [kGroups][kStage][128]

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
    constexpr int kBt = kBuildWarps * 32;
    const int bw = bt >> 5;  // builder warp
    ItemDesc nd;
    nd.ntiles = -1;
    if (bw == 0) nd = fetch_item(a, total_items, lane);
    for (uint32_t it = 0;; ++it) {
      const int ab = static_cast<int>(it & 1u);
      if (bt == 0) {
        if (!mbar_wait(&sh.aempty[ab], ((it >> 1) & 1u) ^ 1u, err, 31, budget)) nd.ntiles = -1;
        sh.desc[ab] = nd;
      }
      asm volatile("bar.sync 3, %0;\n" ::"n"(kBt) : "memory");
      const ItemDesc d = sh.desc[ab];
      if (d.ntiles >= 0) {
        const int64_t qbase = a.list_qoff[d.list] + static_cast<int64_t>(d.group) * kTile;
        float* cen = s_cent + ab * kTile;
        for (int c = bt; c < kpad; c += kBt) cen[c] = c < a.dpad ? a.cent[static_cast<size_t>(d.list) * a.dpad + c] : 0.0f;
        // Row r holds the group's query (r % 32) * 4 + r / 32, so the queries
        // of a partial group spread over the four epilogue warps.  Two rows
        // per thread, their loads issued together.
        int q2[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int r = bt + h * kBt;
          const int i = (r & 31) * 4 + (r >> 5);
          q2[h] = i < d.qcnt ? static_cast<int>(static_cast<uint32_t>(a.list_q[qbase + i]) >> 16) : -1;
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int r = bt + h * kBt;
          const int q = q2[h];
          // The query's bound as other items have lowered it so far.
          meta_q[ab * kTile + r] = q;
          meta_thr[ab * kTile + r] =
              q >= 0 ? ordered_to_float(*reinterpret_cast<volatile uint32_t*>(a.thr + q)) : -INFINITY;
        }
        asm volatile("bar.sync 3, %0;\n" ::"n"(kBt) : "memory");
        // A row r = BF16(q - c_l) of the row's query, and ||q - c_l||^2: a
        // warp per row (lane = 4 consecutive columns), 16 rows in flight.
        uint8_t* A = Abuf + ab * tile_bytes;
        const int c0 = 4 * lane;
        const bool col_in = c0 < a.dpad, col_k = c0 < kpad;
        const float4 cv = col_k ? *reinterpret_cast<const float4*>(cen + c0) : make_float4(0.f, 0.f, 0.f, 0.f);
        const float Rl = a.rmax[d.list];
        constexpr int kRowsInFlight = 8;
        // Rows without a query are left as they are: their TMEM lanes belong
        // to no query and the epilogue ignores them.  A block's rows with a
        // query come first (query (r % 32) * 4 + r / 32 grows with r % 32).
        for (int r0 = bw; r0 < kTile; r0 += kBuildWarps * kRowsInFlight) {
          if (meta_q[ab * kTile + r0] < 0) continue;
          float4 x[kRowsInFlight];
#pragma unroll
          for (int j = 0; j < kRowsInFlight; ++j) {
            const int q = meta_q[ab * kTile + r0 + j * kBuildWarps];
            x[j] = q >= 0 && col_in ? __ldg(reinterpret_cast<const float4*>(a.q + static_cast<size_t>(q) * a.dpad + c0))
                                    : cv;  // q - c = 0 for a padding column
          }
#pragma unroll
          for (int j = 0; j < kRowsInFlight; ++j) {
            const int r = r0 + j * kBuildWarps;
            if (meta_q[ab * kTile + r] < 0) break;
            const float v0 = x[j].x - cv.x, v1 = x[j].y - cv.y, v2 = x[j].z - cv.z, v3 = x[j].w - cv.w;
            float cd = fmaf(v3, v3, fmaf(v2, v2, fmaf(v1, v1, v0 * v0)));
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) cd += __shfl_xor_sync(0xffffffffu, cd, o);
            if (col_k) {
              __nv_bfloat162 p01 = __floats2bfloat162_rn(v0, v1), p23 = __floats2bfloat162_rn(v2, v3);
              *reinterpret_cast<uint2*>(A + sw128_offset_bf16(r, c0, kblk_bytes)) =
                  make_uint2(*reinterpret_cast<uint32_t*>(&p01), *reinterpret_cast<uint32_t*>(&p23));
            }
            if (lane == 0) {
              meta_cd[ab * kTile + r] = cd;
              meta_eps[ab * kTile + r] = pair_eps(cd, Rl, a.dpad);  // eps(q, l) of this row's query
            }
          }
        }
        fence_proxy_async_smem();
      }
      mbar_arrive(&sh.itemf[ab]);
      if (d.ntiles < 0) break;
      if (bw == 0) nd = fetch_item(a, total_items, lane);
    }
  } else if (warp == kProdWarp) {
    // ---- TMA producer ------------------------------------------------------
    uint32_t p_idx = 0;
    if (lane == 0) {
      for (uint32_t it = 0;; ++it) {
        const int ab = static_cast<int>(it & 1u);
        if (!mbar_wait(&sh.itemf[ab], (it >> 1) & 1u, err, 32, budget)) break;
        const ItemDesc d = sh.desc[ab];
        mbar_arrive(&sh.aempty[ab]);
        if (d.ntiles < 0) break;
        bool ok = true;
        for (int t = 0; t < d.ntiles; ++t, ++p_idx) {
          const int s = static_cast<int>(p_idx % static_cast<uint32_t>(S));
          const uint32_t par = ((p_idx / static_cast<uint32_t>(S)) & 1u) ^ 1u;
          if (!mbar_wait(&sh.empty[s], par, err, 11, budget)) {
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
      uint32_t m_idx = 0;
      for (uint32_t it = 0;; ++it) {
        const int ab = static_cast<int>(it & 1u);
        if (!mbar_wait(&sh.itemf[ab], (it >> 1) & 1u, err, 33, budget)) break;
        const ItemDesc d = sh.desc[ab];
        if (d.ntiles < 0) break;
        tc_fence_after();
        const uint64_t a_desc = desc_sw128(smem_u32(Abuf + ab * tile_bytes));
        bool ok = true;
        for (int t = 0; t < d.ntiles; ++t, ++m_idx) {
          const int s = static_cast<int>(m_idx % static_cast<uint32_t>(S));
          if (!mbar_wait(&sh.full[s], (m_idx / static_cast<uint32_t>(S)) & 1u, err, 12, budget)) {
            ok = false;
            break;
          }
          const int b = static_cast<int>(m_idx % kAcc);
          if (!mbar_wait(&sh.acce[b], ((m_idx / kAcc) & 1u) ^ 1u, err, 13, budget)) {
            ok = false;
            break;
          }
          tc_fence_after();
          mbar_arrive_expect_tx(&sh.normf[b], kTile * 4);
          bulk_load(nrm + b * kTile, a.tile_norm + (d.tile0 + t) * kTile, kTile * 4, &sh.normf[b]);
          const uint64_t b_desc = desc_sw128(smem_u32(stages + s * tile_bytes));
          const uint32_t d_tmem = tmem + static_cast<uint32_t>(b * kTile);
          for (int k = 0; k < nk; ++k) {
            // The start-address field is (address >> 4) in the low 14 bits.
            const uint64_t off16 = (static_cast<uint32_t>(k >> 2) * kblk_bytes + static_cast<uint32_t>(k & 3) * 32u) >> 4;
            mma_bf16(d_tmem, a_desc + off16, b_desc + off16, idesc, k > 0 ? 1u : 0u);
          }
          mma_commit(&sh.empty[s]);
          mma_commit(&sh.accf[b]);
        }
        // A buffer ab is free once these MMAs have completed.
        mma_commit(&sh.aempty[ab]);
        if (!ok) break;
      }
      // Drain: every MMA done before TMEM is released, and the last norm copy
      // of each accumulator landed (at most one per accumulator is pending:
      // the next one waits for the epilogue to release the accumulator).
      mma_commit(&sh.drain);
      mbar_wait(&sh.drain, 0, nullptr, 0, 200000000LL);
      for (int b = 0; b < kAcc; ++b) {
        const uint32_t copies = m_idx > static_cast<uint32_t>(b) ? (m_idx - static_cast<uint32_t>(b) + kAcc - 1) / kAcc : 0u;
        if (copies) mbar_wait(&sh.normf[b], (copies - 1u) & 1u, nullptr, 0, 200000000LL);
      }
    }
  } else {
    // ---- epilogue: thread = query (TMEM lane etid) ---------------------------
    const int grp = warp >> 2;
    const int etid = tid - grp * kEpiThreads;
    const uint32_t lane_base = (32u * static_cast<uint32_t>(warp & 3)) << 16;
    uint32_t G = 0;
    for (uint32_t it = 0;; ++it) {
      const int ab = static_cast<int>(it & 1u);
      bool ok = mbar_wait(&sh.itemf[ab], (it >> 1) & 1u, err, 34, budget);
      if (!__all_sync(0xffffffffu, ok)) break;
      const ItemDesc d = sh.desc[ab];
      const int my_q = meta_q[ab * kTile + etid];
      const float thr0 = meta_thr[ab * kTile + etid];
      const float eps = meta_eps[ab * kTile + etid];
      const float cd = meta_cd[ab * kTile + etid];
      mbar_arrive(&sh.aempty[ab]);
      if (d.ntiles < 0) break;
      // Queries are spread over the four warps (row r holds query
      // (r % 32) * 4 + r / 32), so a warp without one skips its loads.
      const bool warp_on = __any_sync(0xffffffffu, my_q >= 0);
      // thr = U, the query's bound on its k-th distance (FLT_MAX: none yet).
      float thr = thr0;
      // Columns hold w' = ||r||^2 - 2 q'.r; a row's value is w = cd + w'
      // and it is admitted when w - eps <= U.  A column is looked at when
      // w' <= thr_s, thr_s = U + eps - cd rounded up with a margin (every row
      // with w - eps <= U passes; a few more may), and never above FLT_MAX:
      // the +inf values of rows past a list's end must not pass.
      auto shifted = [&](float t) {
        const float te = t < FLT_MAX ? __fadd_ru(t, eps) : FLT_MAX;
        return fminf(__fadd_ru(__fsub_ru(te, cd), 1e-6f * (fminf(fabsf(te), 1e30f) + cd)), FLT_MAX);
      };
      float thr_s = shifted(thr);
      // The KT smallest upper bounds this thread knows for the query,
      // ascending, and the k-th of them (KT = 0: no tightening).  A published
      // U says that k rows have upper bounds <= U, so U may stand in for k of
      // them: the k-th of a mix of stand-ins and real values is the k-th of k
      // distinct rows or U itself.  Only a value under the current k-th
      // changes the set.
      float best[KB];
      float kth_loc = thr < FLT_MAX ? thr : INFINITY;
#pragma unroll
      for (int i = 0; i < KB; ++i) best[i] = kth_loc;
      uint64_t* cbuf = a.cand + static_cast<size_t>(my_q < 0 ? 0 : my_q) * a.cap;
      uint32_t* ubuf = a.cand_ub + static_cast<size_t>(my_q < 0 ? 0 : my_q) * a.cap;
      // Admitted keys (lower bound, position) wait here (stride kEpiThreads:
      // conflict-free) in two halves of kHalf.  A full half takes its slots in
      // the query's buffer with one atomicAdd and is written out only when
      // the other half fills (or at the item's end), so the atomic's round
      // trip overlaps the scan instead of stalling the warp once per lane.
      // Staged entries hold (w, position); every entry of an item shares eps,
      // so the written key (w - eps rounded down, position) and upper bound
      // (w + eps rounded up) are formed at write time.
      constexpr int kHalf = kStage / 2;
      uint64_t* stg = staging + static_cast<size_t>(grp) * kStage * kEpiThreads + etid;
      int ns = 0, half = 0, pend_base = 0;
      bool pend = false;
      auto write_half = [&](int h, int base, int n) {
        for (int i = 0; i < n; ++i) {
          if (base + i < a.cap) {
            const uint64_t e = stg[(h * kHalf + i) * kEpiThreads];
            const float wv = ordered_to_float(static_cast<uint32_t>(e >> 32));
            cbuf[base + i] = (static_cast<uint64_t>(ordered_bits(__fsub_rd(wv, eps))) << 32) | (e & 0xffffffffull);
            ubuf[base + i] = ordered_bits(__fadd_ru(wv, eps));
          }
        }
      };
      auto stage = [&](uint64_t key) {
        stg[(half * kHalf + ns) * kEpiThreads] = key;
        if (++ns == kHalf) {
          if (pend) write_half(half ^ 1, pend_base, kHalf);
          pend_base = atomicAdd(a.cand_cnt + my_q, kHalf);
          pend = true;
          half ^= 1;
          ns = 0;
        }
      };
      auto flush = [&]() {
        if (pend) write_half(half ^ 1, pend_base, kHalf);
        if (ns > 0) write_half(half, atomicAdd(a.cand_cnt + my_q, ns), ns);
        pend = false;
        ns = 0;
      };
      // One 32-column chunk of the accumulator in r: w' = ||r||^2 - 2 q'.r
      // (rows past the list carry an infinite norm), their minimum against
      // the bound, and the admission of the columns under it.
      auto chunk = [&](uint32_t(&r)[32], const float* nb, uint32_t pos0) {
        const float4* n4 = reinterpret_cast<const float4*>(nb);
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
        if (my_q >= 0 && mn <= thr_s) {
          uint32_t mq[4] = {0u, 0u, 0u, 0u};
#pragma unroll
          for (int j = 0; j < 32; ++j) mq[j & 3] |= (__uint_as_float(r[j]) <= thr_s ? 1u : 0u) << j;
          uint32_t mask = (mq[0] | mq[1]) | (mq[2] | mq[3]);
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
            const float wv = cd + __uint_as_float((j & 16) ? t2[1] : t2[0]);
            stage((static_cast<uint64_t>(ordered_bits(wv)) << 32) | (pos0 + static_cast<uint32_t>(j)));
            const float ub = __fadd_ru(wv, eps);
            if (KT > 0 && ub < kth_loc) {
              // Insert into the ascending KT smallest upper bounds; their k-th
              // is a new U.
              float v = ub;
#pragma unroll
              for (int i = 0; i < KB; ++i) {
                const float o = best[i];
                best[i] = fminf(o, v);
                v = fmaxf(o, v);
              }
              // best is ascending: its k-th entry is the largest of the first k
              // (a max, so the array stays in registers).
              float kth = best[0];
#pragma unroll
              for (int i = 1; i < KB; ++i) kth = i < a.k ? fmaxf(kth, best[i]) : kth;
              kth_loc = kth;
              if (kth < thr) {
                thr = kth;
                thr_s = shifted(thr);
                atomicMin(a.thr + my_q, ordered_bits(thr));  // shared at once (no return value used)
              }
            }
          }
        }
      };
      // The query's bound as other threads have lowered it, read one tile
      // ahead (the load is in flight while a tile is processed).
      uint32_t g_thr = my_q >= 0 ? *reinterpret_cast<volatile uint32_t*>(a.thr + my_q) : 0u;
      constexpr uint32_t kG = kGroups;
      for (int t = static_cast<int>((static_cast<uint32_t>(grp) + kG - G % kG) % kG); t < d.ntiles; t += kGroups) {
        const uint32_t gt = G + static_cast<uint32_t>(t);  // the CTA's global tile index
        const int b = static_cast<int>(gt % kAcc);
        const uint32_t par = (gt / kAcc) & 1u;
        ok = ok && mbar_wait(&sh.accf[b], par, err, 14, budget) && mbar_wait(&sh.normf[b], par, err, 15, budget);
        ok = __all_sync(0xffffffffu, ok);
        tc_fence_after();
        if (my_q >= 0 && ordered_to_float(g_thr) < thr) {
          thr = ordered_to_float(g_thr);
          thr_s = shifted(thr);
          if (KT > 0) {
            kth_loc = fminf(kth_loc, thr);
#pragma unroll
            for (int i = 0; i < KB; ++i) best[i] = fminf(best[i], kth_loc);
          }
        }
        g_thr = my_q >= 0 ? *reinterpret_cast<volatile uint32_t*>(a.thr + my_q) : 0u;
        if (ok && warp_on) {
          const float* nb = nrm + b * kTile;
          const uint32_t col = tmem + lane_base + static_cast<uint32_t>(b * kTile);
          const uint32_t pos_t = static_cast<uint32_t>(d.row0 + t * kTile);
          // One register set (a second one, to load the next chunk while this
          // one is processed, measured slower: it held the kernel to two
          // epilogue warpgroups within the register file).
          uint32_t ra[32];
#pragma unroll 1
          for (int c = 0; c < kTile / 32; ++c) {
            tmem_ld32(col + static_cast<uint32_t>(32 * c), ra);
            tmem_ld_wait(ra);
            chunk(ra, nb + 32 * c, pos_t + static_cast<uint32_t>(32 * c));
          }
        }
        tc_fence_before();
        mbar_arrive(&sh.acce[b]);
      }
      if (my_q >= 0) flush();
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


// Per query, before the scan: the bound U reset to FLT_MAX (none yet; +inf
// padding rows never pass) and the candidate counter reset.
__global__ void query_prep_kernel(int nq, uint32_t* __restrict__ thr, int* __restrict__ cnt) {
  const int qi = blockIdx.x * blockDim.x + threadIdx.x;
  if (qi >= nq) return;
  thr[qi] = ordered_bits(FLT_MAX);
  cnt[qi] = 0;
}

// BF16 residual codes for the tensor-core scans, one CTA per list: row r of
// list l becomes BF16(x_r - c_l) (kpad columns, zero past dpad), its FP32
// residual norm ||x_r - c_l||^2, and the list's largest residual norm
// (slightly rounded up).
__global__ void residual_bf16_kernel(const float* __restrict__ codes, const int64_t* __restrict__ list_off,
                                     const float* __restrict__ cent, int dpad, int kpad,
                                     __nv_bfloat16* __restrict__ dst, float* __restrict__ rnorm,
                                     float* __restrict__ rmax) {
  __shared__ float s_max[32];
  const int l = blockIdx.x;
  const int64_t r0 = list_off[l], r1 = list_off[l + 1];
  const float* c = cent + static_cast<size_t>(l) * dpad;
  for (int64_t i = threadIdx.x; i < (r1 - r0) * kpad; i += blockDim.x) {
    const int64_t r = r0 + i / kpad;
    const int col = static_cast<int>(i % kpad);
    dst[r * kpad + col] = __float2bfloat16_rn(col < dpad ? codes[r * dpad + col] - c[col] : 0.0f);
  }
  const int lane = threadIdx.x & 31;
  float m = 0.0f;
  for (int64_t r = r0 + (threadIdx.x >> 5); r < r1; r += blockDim.x >> 5) {
    float sq = 0.0f;
    for (int j = lane; j < dpad; j += 32) {
      const float v = codes[r * dpad + j] - c[j];
      sq = fmaf(v, v, sq);
    }
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
    if (lane == 0) rnorm[r] = sq;
    m = fmaxf(m, sq);
  }
  if (lane == 0) s_max[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < static_cast<int>(blockDim.x >> 5); ++w) m = fmaxf(m, s_max[w]);
    rmax[l] = sqrtf(m) * 1.0001f;
  }
}

constexpr int kSmallKth = 32;  // largest k for warp_kth_small8


// Re-rank, one warp per query with at most kRrWarpCap candidates: U = the
// k-th smallest upper bound among them (radix selection), the candidates
// whose lower bound is at most U recomputed with the reference's sequential
// FP32 loop, sorted by (distance, position) and cut at k.  A query with more
// candidates goes to the flat kernels below (flag 1); one whose buffer
// overflowed to the host's exact search (flag 2, and listed).
constexpr int kRrWarpCap = 256;
constexpr int kRrWarps = 8;

__global__ void __launch_bounds__(kRrWarps * 32) rerank_warp_kernel(
    const uint64_t* __restrict__ cand, const uint32_t* __restrict__ cand_ub, const int* __restrict__ cnt, int cap,
    int nq, int k, const float* __restrict__ codes, const float* __restrict__ q, int dpad,
    const int64_t* __restrict__ ids, float* __restrict__ D, int64_t* __restrict__ I, int* __restrict__ flag,
    int* __restrict__ over_list, int* __restrict__ over_n, int* __restrict__ m_out, int* __restrict__ big_list) {
  __shared__ uint64_t s_c[kRrWarps][kRrWarpCap];
  __shared__ uint64_t s_x[kRrWarps][kRrWarpCap];
  __shared__ int s_h[kRrWarps][256];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int qi = blockIdx.x * kRrWarps + wib;
  if (qi >= nq) return;
  const int c = cnt[qi];
  if (c > cap) {
    if (lane == 0) {
      flag[qi] = 2;
      m_out[qi] = 0;
      over_list[atomicAdd(over_n, 1)] = qi;
    }
    return;
  }
  if (c > kRrWarpCap) {
    if (lane == 0) {
      flag[qi] = 1;
      big_list[atomicAdd(over_n + 1, 1)] = qi;
    }
    return;
  }
  if (lane == 0) flag[qi] = 0;
  uint64_t* buf = s_c[wib];
  uint64_t* ex = s_x[wib];
  const uint64_t* src = cand + static_cast<size_t>(qi) * cap;
  const uint32_t* usrc = cand_ub + static_cast<size_t>(qi) * cap;
  // U (every candidate when there are fewer than k): for small k from the
  // upper bounds held eight per lane, else by radix from the upper bounds
  // staged in ex (free until the exact phase) so its passes read shared
  // memory.
  uint32_t u_bits = 0xFFFFFFFFu;
  if (c >= k && k <= kSmallKth) {
    static_assert(kRrWarpCap == 256, "eight upper bounds per lane");
    uint32_t v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = 32 * i + lane < c ? usrc[32 * i + lane] : 0xFFFFFFFFu;
    u_bits = warp_kth_small8(v, k, lane);
  } else if (c >= k) {
    uint32_t* ubs = reinterpret_cast<uint32_t*>(ex);
    for (int i = lane; i < c; i += 32) ubs[i] = usrc[i];
    __syncwarp();
    u_bits = warp_kth_smallest([&](int i) { return ubs[i]; }, c, k, s_h[wib], lane);
  }
  // The candidates with lower bound <= U, compacted into buf (c <= 256:
  // eight keys per lane, their loads in flight together).
  int m = 0;
  {
    uint64_t key[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) key[u] = 32 * u + lane < c ? src[32 * u + lane] : kEmpty;
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const bool in = 32 * u + lane < c && static_cast<uint32_t>(key[u] >> 32) <= u_bits;
      const unsigned bal = __ballot_sync(0xffffffffu, in);
      if (in) buf[m + __popc(bal & ((1u << lane) - 1u))] = key[u];
      m += __popc(bal);
    }
  }
  __syncwarp();
  if (lane == 0) m_out[qi] = m;
  // Every line of the rows to recompute requested at once (the lane loops
  // below then wait for one DRAM round trip, not one per batch of loads).
  for (int j = lane; j < m; j += 32) {
    const char* rp = reinterpret_cast<const char*>(codes + static_cast<size_t>(key_tie(buf[j])) * dpad);
    for (int o = 0; o < dpad * 4; o += 128) asm volatile("prefetch.global.L2 [%0];" ::"l"(rp + o));
  }
  const float* qrow = q + static_cast<size_t>(qi) * dpad;
  const int e2n = pow2_ceil(m < 2 ? 2 : m);
  for (int j = lane; j < e2n; j += 32) {
    uint64_t key = kEmpty;
    if (j < m) {
      const uint32_t pos = key_tie(buf[j]);
      const float acc = exact_l2_seq(codes + static_cast<size_t>(pos) * dpad, qrow, dpad);
      if (acc < FLT_MAX) key = make_key(acc, pos);
    }
    ex[j] = key;
  }
  __syncwarp();
  warp_bitonic_sort(ex, e2n, lane);
  for (int j = lane; j < k; j += 32) {
    const uint64_t key = j < m ? ex[j] : kEmpty;
    const size_t o = static_cast<size_t>(qi) * k + j;
    D[o] = key == kEmpty ? FLT_MAX : key_dist(key);
    I[o] = key == kEmpty ? -1 : ids[key_tie(key)];
  }
}

// The bound of the second stage of a batch with k > kTightK: the first stage
// scanned only each query's nearest list, so the k-th smallest upper bound
// admitted there (a radix selection, 8 bits per pass) is a U for the whole
// probe set.  One warp per query; a query with fewer than k admitted rows, or
// an overflowed buffer, keeps its bound.
constexpr int kKthWarps = 8;

__global__ void __launch_bounds__(kKthWarps * 32) kth_bound_kernel(const uint32_t* __restrict__ cand_ub,
                                                                  const int* __restrict__ cnt, int cap, int nq, int k,
                                                                  uint32_t* __restrict__ thr) {
  __shared__ int s_h[kKthWarps][256];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int qi = blockIdx.x * kKthWarps + wib;
  if (qi >= nq) return;
  const int c = cnt[qi];
  if (c < k || c > cap) return;
  const uint32_t* src = cand_ub + static_cast<size_t>(qi) * cap;
  const uint32_t u = warp_kth_smallest([&](int i) { return src[i]; }, c, k, s_h[wib], lane);
  if (lane == 0 && u < thr[qi]) thr[qi] = u;
}

// Probe table split for the two stages: first[q] = the query's nearest list,
// rest = the table with that column set to -1.
__global__ void split_first_probe_kernel(const int32_t* __restrict__ probes, int nq, int P,
                                         int32_t* __restrict__ first, int32_t* __restrict__ rest) {
  const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (i >= static_cast<int64_t>(nq) * P) return;
  const int j = static_cast<int>(i % P);
  const int32_t v = probes[i];
  rest[i] = j == 0 ? -1 : v;
  if (j == 0) first[i / P] = v;
}

// The queries the warp kernel listed in big_list (more than kRrWarpCap
// candidates, at most cap; *big_n of them) in three flat kernels, so the
// exact distances -- the bulk of the work -- run with every SM's threads
// loading rows rather than behind per-query sorts:
//   rerank_big_bound_kernel  a warp per query: U, the k-th smallest upper
//                            bound, by radix selection, then the candidates
//                            whose lower bound is at most U compacted in
//                            place at the front of the query's buffer (m of
//                            them);
//   rerank_big_exact_kernel  a CTA per query: the exact distance of each of
//                            the m rows (two rows per thread in flight),
//                            written back in place as (distance, position)
//                            keys;
//   rerank_big_topk_kernel   a CTA per query: the k smallest keys, sorted.
constexpr int kBigWarps = 8;
constexpr int kRerankMaxDim = 128;  // dpad of the BF16 scan's rows (d <= 128)

__global__ void __launch_bounds__(kBigWarps * 32) rerank_big_bound_kernel(
    uint64_t* __restrict__ cand, const uint32_t* __restrict__ cand_ub, const int* __restrict__ cnt, int cap, int k,
    const int* __restrict__ big_list, const int* __restrict__ big_n, int* __restrict__ m_out) {
  __shared__ int s_h[kBigWarps][256];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int nbig = *big_n;
  for (int w = blockIdx.x * kBigWarps + wib; w < nbig; w += gridDim.x * kBigWarps) {
    const int qi = big_list[w];
    const int c = cnt[qi];
    uint64_t* buf = cand + static_cast<size_t>(qi) * cap;
    const uint32_t* ubs = cand_ub + static_cast<size_t>(qi) * cap;
    const uint32_t lim_bits = warp_kth_smallest([&](int i) { return ubs[i]; }, c, k, s_h[wib], lane);
    // In-place compaction: a block of 256 keys (eight per lane, their loads
    // in flight together) is read before any of it is written, and writes
    // land at or below the read position.
    int m = 0;
    for (int base = 0; base < c; base += 256) {
      uint64_t key[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) key[u] = base + 32 * u + lane < c ? buf[base + 32 * u + lane] : kEmpty;
      __syncwarp();
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const bool in = base + 32 * u + lane < c && static_cast<uint32_t>(key[u] >> 32) <= lim_bits;
        const unsigned bal = __ballot_sync(0xffffffffu, in);
        if (in) buf[m + __popc(bal & ((1u << lane) - 1u))] = key[u];
        m += __popc(bal);
      }
    }
    if (lane == 0) m_out[qi] = m;
    __syncwarp();
  }
}

__global__ void __launch_bounds__(256) rerank_big_exact_kernel(uint64_t* __restrict__ cand, int cap,
                                                               const float* __restrict__ codes,
                                                               const float* __restrict__ q, int dpad,
                                                               const int* __restrict__ big_list,
                                                               const int* __restrict__ big_n,
                                                               const int* __restrict__ m_in) {
  __shared__ __align__(16) float s_q[kRerankMaxDim];
  const int nbig = *big_n;
  for (int w = blockIdx.x; w < nbig; w += gridDim.x) {
    const int qi = big_list[w];
    const int m = m_in[qi];
    uint64_t* buf = cand + static_cast<size_t>(qi) * cap;
    __syncthreads();  // the previous query's readers of s_q are done
    for (int c = threadIdx.x; c < dpad; c += blockDim.x) s_q[c] = q[static_cast<size_t>(qi) * dpad + c];
    __syncthreads();
    // Rows j and j + blockDim.x together: two independent chains, each the
    // reference's sequential loop (many small CTAs per SM keep the loads in
    // flight).
    for (int j0 = threadIdx.x; j0 < m; j0 += 2 * blockDim.x) {
      const int j1 = j0 + blockDim.x;
      const uint32_t p0 = key_tie(buf[j0]);
      const uint32_t p1 = j1 < m ? key_tie(buf[j1]) : p0;
      const float4* x0 = reinterpret_cast<const float4*>(codes + static_cast<size_t>(p0) * dpad);
      const float4* x1 = reinterpret_cast<const float4*>(codes + static_cast<size_t>(p1) * dpad);
      float a0 = 0.0f, a1 = 0.0f;
#pragma unroll 4
      for (int i = 0; i < dpad / 4; ++i) {
        const float4 u = __ldg(x0 + i), v = __ldg(x1 + i);
        const float4 g = *reinterpret_cast<const float4*>(s_q + 4 * i);
        float t;
        t = __fsub_rn(g.x, u.x);
        a0 = __fadd_rn(a0, __fmul_rn(t, t));
        t = __fsub_rn(g.x, v.x);
        a1 = __fadd_rn(a1, __fmul_rn(t, t));
        t = __fsub_rn(g.y, u.y);
        a0 = __fadd_rn(a0, __fmul_rn(t, t));
        t = __fsub_rn(g.y, v.y);
        a1 = __fadd_rn(a1, __fmul_rn(t, t));
        t = __fsub_rn(g.z, u.z);
        a0 = __fadd_rn(a0, __fmul_rn(t, t));
        t = __fsub_rn(g.z, v.z);
        a1 = __fadd_rn(a1, __fmul_rn(t, t));
        t = __fsub_rn(g.w, u.w);
        a0 = __fadd_rn(a0, __fmul_rn(t, t));
        t = __fsub_rn(g.w, v.w);
        a1 = __fadd_rn(a1, __fmul_rn(t, t));
      }
      buf[j0] = a0 < FLT_MAX ? make_key(a0, p0) : kEmpty;
      if (j1 < m) buf[j1] = a1 < FLT_MAX ? make_key(a1, p1) : kEmpty;
    }
  }
}

__global__ void __launch_bounds__(256) rerank_big_topk_kernel(const uint64_t* __restrict__ cand, int cap, int k,
                                                              const int64_t* __restrict__ ids, float* __restrict__ D,
                                                              int64_t* __restrict__ I, const int* __restrict__ big_list,
                                                              const int* __restrict__ big_n,
                                                              const int* __restrict__ m_in) {
  extern __shared__ uint64_t s_top[];  // pow2_ceil(k)
  __shared__ SelectShared sh_sel;
  const int nbig = *big_n;
  for (int w = blockIdx.x; w < nbig; w += gridDim.x) {
    const int qi = big_list[w];
    const int m = m_in[qi];
    const uint64_t* buf = cand + static_cast<size_t>(qi) * cap;
    auto key_at = [&](int i) -> uint64_t { return buf[i]; };
    __syncthreads();  // the previous query's readers of s_top are done
    block_topk_sorted(key_at, m, k, sh_sel, s_top);
    for (int j = threadIdx.x; j < k; j += blockDim.x) {
      const uint64_t key = s_top[j];
      const size_t o = static_cast<size_t>(qi) * k + j;
      D[o] = key == kEmpty ? FLT_MAX : key_dist(key);
      I[o] = key == kEmpty ? -1 : ids[key_tie(key)];
    }
  }
}

// Seed bound per query before the scan: U = the k-th smallest w over the
// first S rows of the query's nearest list, computed from the same BF16
// operands as the scan (these values obey the same eps), + eps(q, l): k rows
// of the probe set have upper bounds at most that.  Queries whose nearest
// list holds fewer than k rows keep FLT_MAX.
//
// List-major: one CTA per list; the queries whose nearest list it is (probe
// rank 0 in the list-major work description) go kSeedQ at a time: warp j
// forms query j's BF16 residual row in shared memory, thread t streams row t
// of the list's first S rows from global memory once (16-byte loads) and
// forms its value for each of those queries (their rows broadcast from
// shared memory), then a warp per query selects its k-th smallest by radix
// (four 8-bit passes).  Nothing is staged in shared memory, so several CTAs
// share an SM and keep their row loads in flight.  Small batches (probes
// given): one CTA per query.
constexpr int kSeedRows = 256;
constexpr int kSeedWarps = 8;
constexpr int kSeedQ = 4;  // queries per pass
static_assert(kSeedWarps * 32 >= kSeedRows, "the seed forms a row per thread");
static_assert(kSeedQ <= kSeedWarps, "a warp per query of a pass");

__global__ void __launch_bounds__(kSeedWarps * 32, 4) seed_bound_kernel(
    const float* __restrict__ q, int dpad, const float* __restrict__ cent, int kpad,
    const __nv_bfloat16* __restrict__ codes,
    const int64_t* __restrict__ list_off, const int64_t* __restrict__ list_qoff, const int32_t* __restrict__ list_q,
    const float* __restrict__ xnorm, const float* __restrict__ rmax, int S, int k, uint32_t* __restrict__ thr,
    const int32_t* __restrict__ probes, int P) {
  __shared__ __align__(16) float s_q[kSeedQ][kRerankMaxDim];
  __shared__ int s_qs[kSeedWarps * 32];
  __shared__ int s_nq;
  __shared__ float s_cd[kSeedQ];
  __shared__ uint32_t s_keys[kSeedQ][kSeedRows];
  __shared__ int s_hist[kSeedQ][256];
  const int tid = threadIdx.x, lane = tid & 31, wib = tid >> 5;
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
  }
  const int64_t b = list_off[l];
  const int n = static_cast<int>(min(static_cast<int64_t>(S), list_off[l + 1] - b));
  if (n < k) return;  // no seed: the bound stays FLT_MAX
  const bool row_ok = tid < n;
  if (row_ok) {
    // Row tid's fetch from DRAM overlaps the query gathering below.
    const char* rp = reinterpret_cast<const char*>(codes + static_cast<size_t>(b + tid) * kpad);
    for (int o = 0; o < kpad * 2; o += 128) asm volatile("prefetch.global.L2 [%0];" ::"l"(rp + o));
  }
  const uint4* xrow = reinterpret_cast<const uint4*>(codes + static_cast<size_t>(b + (row_ok ? tid : 0)) * kpad);
  const float xn = row_ok ? xnorm[b + tid] : 0.0f;
  for (int64_t r0 = e0; r0 < e1; r0 += blockDim.x) {
    if (tid == 0) s_nq = 0;
    __syncthreads();
    if (r0 + tid < e1) {
      const uint32_t ent =
          by_query ? (static_cast<uint32_t>(blockIdx.x) << 16) : static_cast<uint32_t>(list_q[r0 + tid]);
      if ((ent & 0xffff) == 0) s_qs[atomicAdd(&s_nq, 1)] = static_cast<int>(ent >> 16);
    }
    __syncthreads();
    const int nqr = s_nq;  // 0 for a list that is no query's nearest: nothing to do
    for (int t0 = 0; t0 < nqr; t0 += kSeedQ) {
      const int nb = min(kSeedQ, nqr - t0);
      if (wib < nb) {
        const int qi = s_qs[t0 + wib];
        const float* qrow = q + static_cast<size_t>(qi) * dpad;
        const float* crow = cent + static_cast<size_t>(l) * dpad;
        float cd = 0.0f;
        float qv[kRerankMaxDim / 32], cv[kRerankMaxDim / 32];
#pragma unroll
        for (int i = 0; i < kRerankMaxDim / 32; ++i) {
          const int c = lane + 32 * i;
          qv[i] = c < dpad ? qrow[c] : 0.0f;
          cv[i] = c < dpad ? crow[c] : 0.0f;
        }
#pragma unroll
        for (int i = 0; i < kRerankMaxDim / 32; ++i) {
          const int c = lane + 32 * i;
          if (c < kpad) {
            const float v = qv[i] - cv[i];
            cd = fmaf(v, v, cd);
            s_q[wib][c] = __bfloat162float(__float2bfloat16_rn(v));
          }
        }
        for (int o = 16; o > 0; o >>= 1) cd += __shfl_xor_sync(0xffffffffu, cd, o);
        if (lane == 0) s_cd[wib] = cd;
      }
      __syncthreads();
      if (row_ok) {
        // Four partial sums per query (any order is within eps).
        float d[kSeedQ][4];
#pragma unroll
        for (int j = 0; j < kSeedQ; ++j) d[j][0] = d[j][1] = d[j][2] = d[j][3] = 0.0f;
        // 64-byte pieces of the row: four loads in flight, then their values.
        for (int c0 = 0; c0 < kpad; c0 += 32) {
          uint4 xq[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) xq[u] = __ldg(xrow + c0 / 8 + u);
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int c = c0 + 8 * u;
            const uint4 xv = xq[u];
            const float x0 = __uint_as_float(xv.x << 16), x1 = __uint_as_float(xv.x & 0xffff0000u);
            const float x2 = __uint_as_float(xv.y << 16), x3 = __uint_as_float(xv.y & 0xffff0000u);
            const float x4 = __uint_as_float(xv.z << 16), x5 = __uint_as_float(xv.z & 0xffff0000u);
            const float x6 = __uint_as_float(xv.w << 16), x7 = __uint_as_float(xv.w & 0xffff0000u);
#pragma unroll
            for (int j = 0; j < kSeedQ; ++j) {
              if (j < nb) {
                const float4 qa = *reinterpret_cast<const float4*>(&s_q[j][c]);
                const float4 qc = *reinterpret_cast<const float4*>(&s_q[j][c + 4]);
                d[j][0] = fmaf(qa.x, x0, d[j][0]);
                d[j][1] = fmaf(qa.y, x1, d[j][1]);
                d[j][2] = fmaf(qa.z, x2, d[j][2]);
                d[j][3] = fmaf(qa.w, x3, d[j][3]);
                d[j][0] = fmaf(qc.x, x4, d[j][0]);
                d[j][1] = fmaf(qc.y, x5, d[j][1]);
                d[j][2] = fmaf(qc.z, x6, d[j][2]);
                d[j][3] = fmaf(qc.w, x7, d[j][3]);
              }
            }
          }
        }
#pragma unroll
        for (int j = 0; j < kSeedQ; ++j)
          if (j < nb)
            s_keys[j][tid] = ordered_bits(s_cd[j] + fmaf(-2.0f, (d[j][0] + d[j][1]) + (d[j][2] + d[j][3]), xn));
      }
      __syncthreads();
      if (wib < nb) {
        const int qi = s_qs[t0 + wib];
        uint32_t kth;
        if (k <= kSmallKth) {
          uint32_t v[8];
#pragma unroll
          for (int i = 0; i < 8; ++i) v[i] = 32 * i + lane < n ? s_keys[wib][32 * i + lane] : 0xFFFFFFFFu;
          kth = warp_kth_small8(v, k, lane);
        } else {
          kth = warp_kth_smallest([&](int i) { return s_keys[wib][i]; }, n, k, s_hist[wib], lane);
        }
        // U = the k-th smallest w + eps(q, l): every one of those k rows has
        // an upper bound at most that.
        if (lane == 0)
          thr[qi] = ordered_bits(
              fminf(__fadd_ru(ordered_to_float(kth), pair_eps(s_cd[wib], rmax[l], dpad)), FLT_MAX));
      }
      __syncthreads();
    }
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

size_t scan_bf16_smem_bytes(int kpad, int stages) {
  const size_t tile = static_cast<size_t>(kpad / 64) * kTile * 128;
  return 1024 + tile * (2 + stages) + static_cast<size_t>(kAcc) * kTile * 4 + 2 * kTile * (4 + 4 + 4 + 4 + 4) +
         static_cast<size_t>(kGroups) * kStage * kEpiThreads * 8;
}

int scan_bf16_stages(int kpad) {
  int s = kMaxStages;
  while (s > 2 && scan_bf16_smem_bytes(kpad, s) > kSmemCap) --s;
  return s;
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

void make_f32_store_map(void* tmap_out, const float* base, size_t rows, size_t cols) {
  HB_CHECK(cols % 4 == 0, HB_ERR_INVALID, "FP32 tensor map rows must be 16-byte multiples");
  CUtensorMap* m = static_cast<CUtensorMap*>(tmap_out);
  cuuint64_t dims[2] = {static_cast<cuuint64_t>(cols), static_cast<cuuint64_t>(rows)};
  cuuint64_t strides[1] = {static_cast<cuuint64_t>(cols) * 4};
  cuuint32_t box[2] = {32, 32};
  cuuint32_t es[2] = {1, 1};
  CUresult r = tensor_map_encoder()(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides,
                                    box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                    CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
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
  HB_CHECK(a.chunk_rows % kTile == 0, HB_ERR_INVALID, "BF16 scan chunks must be whole tiles");
  HB_CHECK(a.stages >= 2 && a.stages <= kMaxStages, HB_ERR_INVALID, "bad stage count");
  HB_CHECK(a.k >= 1 && a.cap >= a.k, HB_ERR_INVALID, "candidate buffer smaller than k");
  HB_CHECK(a.wait_budget > 0, HB_ERR_INVALID, "wait budget must be positive");
  const size_t smem = scan_bf16_smem_bytes(a.kpad, a.stages);
  HB_CHECK(smem <= kSmemCap, HB_ERR_INVALID, "BF16 scan tiles exceed shared memory");
  if (a.k <= kTightK) {
    HB_CUDA(cudaFuncSetAttribute(scan_bf16_kernel<kTightK>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)));
    scan_bf16_kernel<kTightK><<<num_sms, kTcThreads, smem, st>>>(*static_cast<const CUtensorMap*>(tmap), a);
  } else {
    HB_CUDA(cudaFuncSetAttribute(scan_bf16_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)));
    scan_bf16_kernel<0><<<num_sms, kTcThreads, smem, st>>>(*static_cast<const CUtensorMap*>(tmap), a);
  }
  HB_CUDA(cudaGetLastError());
}

void launch_query_prep(int nq, uint32_t* thr, int* cnt, cudaStream_t st) {
  if (nq <= 0) return;
  query_prep_kernel<<<(nq + 255) / 256, 256, 0, st>>>(nq, thr, cnt);
  HB_CUDA(cudaGetLastError());
}

void launch_residual_bf16(const float* codes, const int64_t* list_off, const float* cent, int nlist, int dpad, int kpad,
                          void* dst, float* rnorm, float* rmax, cudaStream_t st) {
  if (nlist <= 0) return;
  residual_bf16_kernel<<<nlist, 256, 0, st>>>(codes, list_off, cent, dpad, kpad, static_cast<__nv_bfloat16*>(dst),
                                              rnorm, rmax);
  HB_CUDA(cudaGetLastError());
}

void launch_seed_bound(const float* q, int d, int dpad, const float* cent, int nq, int kpad, const void* codes_bf16,
                       const int64_t* list_off, int nlist, const int64_t* list_qoff, const int32_t* list_q,
                       const float* rnorm, const float* rmax, int S, int k, uint32_t* thr, cudaStream_t st,
                       const int32_t* probes, int P) {
  if (nq <= 0) return;
  HB_CHECK(kpad == 64 || kpad == 128, HB_ERR_INVALID, "the BF16 scan supports d <= 128");
  HB_CHECK(S >= 1 && S <= kSeedRows && k >= 1, HB_ERR_INVALID, "seed sample out of range");
  if (k > S) return;  // no sample holds k rows: every bound stays FLT_MAX
  const bool by_query = probes && static_cast<long long>(nq) * 4 < nlist;
  seed_bound_kernel<<<by_query ? nq : nlist, kSeedWarps * 32, 0, st>>>(
      q, dpad, cent, kpad, static_cast<const __nv_bfloat16*>(codes_bf16), list_off, list_qoff, list_q, rnorm, rmax, S, k,
      thr, by_query ? probes : nullptr, P);
  HB_CUDA(cudaGetLastError());
}

void launch_rerank_bf16(uint64_t* cand, const uint32_t* cand_ub, const int* cnt, int cap, int nq, int k,
                        const float* codes, const float* q, int dpad, const int64_t* ids, float* D, int64_t* I,
                        int* flag, int* over_list, int* over_n, int* m_out, int num_sms, cudaStream_t st) {
  if (nq <= 0) return;
  HB_CHECK(k >= 1 && cap >= k && cap <= kRerankMaxCap && (cap & (cap - 1)) == 0, HB_ERR_INVALID,
           "candidate buffer size out of range");
  HB_CHECK(dpad % 4 == 0 && dpad <= kRerankMaxDim, HB_ERR_INVALID, "re-rank rows wider than 128 floats");
  rerank_warp_kernel<<<(nq + kRrWarps - 1) / kRrWarps, kRrWarps * 32, 0, st>>>(
      cand, cand_ub, cnt, cap, nq, k, codes, q, dpad, ids, D, I, flag, over_list, over_n, m_out, over_list + nq);
  HB_CUDA(cudaGetLastError());
  if (cap > kRrWarpCap) {
    // At most nq queries are big (*big_n of them, known on the device
    // only): grids of at most eight CTAs per SM stride over the list.
    const int* big_list = over_list + nq;
    const int* big_n = over_n + 1;
    const int gmax = 8 * std::max(1, num_sms);
    rerank_big_bound_kernel<<<std::min((nq + kBigWarps - 1) / kBigWarps, gmax), kBigWarps * 32, 0, st>>>(
        cand, cand_ub, cnt, cap, k, big_list, big_n, m_out);
    rerank_big_exact_kernel<<<std::min(nq, gmax), 256, 0, st>>>(cand, cap, codes, q, dpad, big_list, big_n, m_out);
    const size_t smem = static_cast<size_t>(pow2_ceil(k < 2 ? 2 : k)) * sizeof(uint64_t);
    rerank_big_topk_kernel<<<std::min(nq, gmax), 256, smem, st>>>(cand, cap, k, ids, D, I, big_list, big_n, m_out);
    HB_CUDA(cudaGetLastError());
  }
}

void launch_kth_bound(const uint32_t* cand_ub, const int* cnt, int cap, int nq, int k, uint32_t* thr,
                      cudaStream_t st) {
  if (nq <= 0) return;
  kth_bound_kernel<<<(nq + kKthWarps - 1) / kKthWarps, kKthWarps * 32, 0, st>>>(cand_ub, cnt, cap, nq, k, thr);
  HB_CUDA(cudaGetLastError());
}

void launch_split_first_probe(const int32_t* probes, int nq, int P, int32_t* first, int32_t* rest, cudaStream_t st) {
  const int64_t n = static_cast<int64_t>(nq) * P;
  if (n <= 0) return;
  split_first_probe_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(probes, nq, P, first, rest);
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

// Internal declarations of the B200 IVF-flat core (host side + kernel
// launchers).  Nothing here is part of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/harmony_b200.h"

namespace hb {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define HB_CUDA(x)                                                                          \
  do {                                                                                      \
    cudaError_t e_ = (x);                                                                   \
    if (e_ != cudaSuccess)                                                                  \
      throw ::hb::Error(e_ == cudaErrorMemoryAllocation ? HB_ERR_NOMEM : HB_ERR_CUDA,       \
                        std::string(#x) + ": " + cudaGetErrorString(e_));                   \
  } while (0)

#define HB_CHECK(cond, code, msg)                     \
  do {                                                \
    if (!(cond)) throw ::hb::Error((code), (msg));    \
  } while (0)

// Bumped on every device allocation of a DevBuf: CUDA graphs that captured
// buffer addresses are valid only while it is unchanged.
inline std::atomic<uint64_t>& devbuf_generation() {
  static std::atomic<uint64_t> g{0};
  return g;
}

// Device allocation owned by the index.  Grows, never shrinks.
template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  T* reserve(size_t count) {
    if (count > n) {
      release();
      size_t bytes = count * sizeof(T);
      if (bytes == 0) bytes = sizeof(T);
      HB_CUDA(cudaMalloc(&p, bytes));
      n = count;
      devbuf_generation().fetch_add(1);
    }
    return p;
  }
  T* get() const { return p; }
};

// Rows are padded to a multiple of 16 elements so that fp32, bf16 and fp8
// rows all start on 16-byte boundaries; padding is zero in codes and queries,
// which leaves every sequential sum unchanged (adding +0.0f is exact).
inline size_t pad_dim(size_t d) { return (d + 15) / 16 * 16; }

constexpr uint64_t kEmptyKey = ~0ull;

// ---- kernel launchers (defined in the .cu files) --------------------------

struct ScanPlan;  // device-resident work description of one search batch

// k_exact.cu
// Exact FP32 distance matrix D[q][c] for q < nq, c < nrows (sequential
// unfused sums over dpad dims).
void launch_l2_matrix(const float* q, int nq, const float* rows, int nrows, int dpad, float* D,
                      int ldD, cudaStream_t st);
// Exact nearest row per query (strict '<', lowest row index wins ties).
void launch_l2_argmin(const float* q, int nq, const float* rows, int nrows, int dpad, int32_t* arg,
                      float* dist, cudaStream_t st);

// Scan modes: the reference's three per-candidate accumulations.
enum ScanMode : int { SCAN_PLAIN = 0, SCAN_CHUNK4 = 1, SCAN_DIMBLOCK = 2 };

struct ScanArgs {
  // index
  const float* codes;      // nb x dpad
  const int64_t* list_off; // nlist + 1
  int nlist;
  int d, dpad;
  // queries
  const float* q;          // nq x dpad
  int nq, P, k;
  // work description
  const int32_t* list_cnt;     // queries per list
  const int64_t* list_qoff;    // exclusive scan of list_cnt (nlist + 1)
  const int32_t* list_q;       // (query << 16 | probe rank) as uint32, grouped by list
  const int64_t* item_off;     // exclusive scan of items per list (nlist + 1)
  const int64_t* slot_base;    // nq*P + 1 exclusive scan of chunks per (q, j)
  int chunk_rows;              // vectors per chunk
  int qgroup;                  // queries per work item
  unsigned int* work_counter;  // persistent scheduler counter (zeroed per launch)
  uint64_t* part;              // slots x k partial top-k keys
  // pruning
  int mode;                    // ScanMode
  const float* tops;           // per-query heap tops (CHUNK4 / DIMBLOCK)
  int cut;                     // pruning on
  int nseg;                    // DIMBLOCK slices
  const int32_t* seg_order;    // DIMBLOCK: order[b * nseg + t]
  int qblock;                  // DIMBLOCK: queries per block
  int nblocks;                 // DIMBLOCK: blocks
};
void launch_scan_exact(const ScanArgs& a, int num_sms, cudaStream_t st);
size_t scan_exact_smem_bytes(int d, int dpad, int k, int mode, int* tv, int* qt, int* qgroup);

// k_select.cu
// Row-wise selection of the k smallest (value, column) pairs of a float
// matrix; out_idx gets columns, out_val the values, ascending.
// row_flags (optional, nrows ints of scratch): enables the warp-per-row
// path for k <= 256.
// cmins (optional, ceil(ncols / 16) x nrows, chunk-major): each 16-column
// chunk's smallest value (bit pattern), as coarse_tc writes it; given with
// row_flags and k <= a quarter of the chunk count (<= 256 chunks), a row
// reads only the chunks whose minimum is at most the k-th smallest chunk
// minimum.
void launch_select_rows(const float* D, int nrows, int ncols, int ldD, int k, int32_t* out_idx,
                        float* out_val, cudaStream_t st, const int32_t* k_row = nullptr, int* row_flags = nullptr,
                        const uint32_t* cmins = nullptr);
// Build the list-major work description from probes (nq x P, -1 = none).
// slot_base (the exact scan's per-(query, probe) output slots) may be null:
// it is then not built.  Returns the number of this library's kernels it
// launched.
int launch_build_work(const int32_t* probes, int nq, int P, const int64_t* list_off, int nlist,
                       int chunk_rows, int qgroup, int32_t* list_cnt, int64_t* list_qoff,
                       int32_t* list_cursor, int32_t* list_q, int64_t* item_off, int64_t* slot_base,
                       void* scan_tmp, size_t scan_tmp_bytes, cudaStream_t st);
size_t build_work_tmp_bytes(int nq, int P, int nlist);
// The reference master's heap merge of nparts result rows per query
// (Dp, Ip: nparts x nq x k, part-major) into D, I (nq x k, ascending).
void launch_merge_parts(const float* Dp, const int64_t* Ip, int nparts, int64_t nq, int k, float* D, int64_t* I,
                        cudaStream_t st);
// Merge partial top-k slots of each query to the final top-k.
void launch_merge(const uint64_t* part, const int64_t* slot_base, int nq, int P, int k,
                  const int64_t* ids, float* D, int64_t* I, cudaStream_t st);
// Warm-up heap tops (k-th smallest distance over the warm-up candidates).
void launch_warmup_tops(const float* q, int nq, const int32_t* probes, int P, const float* codes,
                        const int64_t* list_off, int dpad, int k, int warm_lists,
                        int warm_list_size, float* tops, cudaStream_t st);

// k_build.cu
void launch_pad_rows(const float* src, size_t n, int d, int dpad, float* dst, cudaStream_t st);
void launch_gather_rows(const float* src, const int64_t* idx, size_t n, int dpad, float* dst,
                        cudaStream_t st);
void launch_kmeans_accumulate(const float* x, const int32_t* assign, size_t n, int d, int dpad,
                              double* sums, int32_t* counts, cudaStream_t st);
void launch_kmeans_update(const double* sums, const int32_t* counts, int nlist, int d, int dpad,
                          float* cent, cudaStream_t st);
void launch_row_norms(const float* x, size_t n, int d, int dpad, float* norms, cudaStream_t st);
void launch_add_keys(const int32_t* assign, const float* dist, size_t n, uint64_t* keys,
                     uint32_t* vals, cudaStream_t st);
void sort_pairs_u64(uint64_t* keys_in, uint64_t* keys_out, uint32_t* vals_in, uint32_t* vals_out,
                    size_t n, int end_bit, void* tmp, size_t* tmp_bytes, cudaStream_t st);
void launch_scatter_sorted(const float* x, const uint32_t* order, size_t n, int d, int dpad,
                           float* codes, int64_t* ids, cudaStream_t st);
void launch_list_offsets(const int32_t* assign, size_t n, int nlist, int64_t* list_off,
                         void* tmp, size_t tmp_bytes, cudaStream_t st);
size_t list_offsets_tmp_bytes(int nlist);
void launch_i64_to_i32(const int64_t* src, size_t n, int32_t* dst, cudaStream_t st);
// Rows of w 32-bit words: dst[i] = src[idx[i]] (gather) / dst[idx[i]] = src[i]
// (scatter), i < n.
void launch_gather_words(const uint32_t* src, const int32_t* idx, int n, int w, uint32_t* dst, cudaStream_t st);
void launch_scatter_words(const uint32_t* src, const int32_t* idx, int n, int w, uint32_t* dst, cudaStream_t st);
void launch_i32_to_i64(const int32_t* src, size_t n, int64_t* dst, cudaStream_t st);
void launch_fill_results(float* D, int64_t* I, size_t n, cudaStream_t st);

// k_tc.cu: BF16 tensor-core scan whose exact FP32 re-rank reproduces the
// exact scan bit for bit (the error bound and the admission rule are
// described at the top of k_tc.cu).
struct TcArgs {
  const int64_t* list_off;
  int nlist;
  int kpad;                    // BF16 row length (d rounded up to 64)
  const float* q;              // nq x dpad FP32 queries (zero padded)
  int dpad;
  const float* cent;           // nlist x dpad FP32 centroids (the A rows are BF16(q - c_l))
  const float* tile_norm;      // ||x||^2 per 128-row tile of each list, +inf past the list's end
  const int64_t* tile_off;     // first tile of each list in tile_norm (nlist + 1)
  const int32_t* list_cnt;
  const int64_t* list_qoff;
  const int32_t* list_q;
  const int64_t* item_off;
  int chunk_rows;              // multiple of 128
  unsigned int* work_counter;
  uint32_t* thr;               // per query: U, an upper bound of the k-th distance (ordered float bits),
                               // lowered by atomicMin
  const float* rmax;           // per list: the largest residual norm (the error bound's R)
  uint64_t* cand;              // nq x cap candidate keys (ordered lower-bound bits << 32 | position)
  uint32_t* cand_ub;           // nq x cap: each candidate's upper bound (ordered float bits)
  int* cand_cnt;               // per query: candidates appended (may exceed cap: overflow)
  int cap;
  int k;
  int* err;                    // non-zero after a bounded wait gave up
  int stages;                  // B tile ring depth (scan_bf16_stages)
  long long wait_budget;       // clock cycles a bounded mbarrier wait spends before giving up
};
constexpr int kRerankMaxCap = 8192;  // largest candidate buffer per query
constexpr int kFilterMaxK = 256;     // largest k of the bounded scan (its seed samples <= 256 rows)
constexpr long long kDefaultWaitBudget = 2000000000LL;  // clock cycles before a device wait gives up
size_t scan_bf16_smem_bytes(int kpad, int stages);
int scan_bf16_stages(int kpad);  // deepest B tile ring that fits
// Per-tile norm array: tile_off (nlist + 1, prefix of ceil(n_l / 128)) and
// tile_norm (tiles x 128 floats, +inf past each list's end).
void launch_tile_norms(const float* norms, const int64_t* list_off, int nlist, const int64_t* tile_off,
                       float* tile_norm, cudaStream_t st);
void make_bf16_tensor_map(void* tmap_out, const void* codes_bf16, size_t rows, int kpad);
// Tensor map of a row-major FP32 matrix (rows x cols, cols a multiple of 4)
// for TMA stores of 32 x 32 boxes with the 128-byte swizzle.
void make_f32_store_map(void* tmap_out, const float* base, size_t rows, size_t cols);
// Per query: bound reset to FLT_MAX (none yet), candidate count 0.
void launch_query_prep(int nq, uint32_t* thr, int* cnt, cudaStream_t st);
// Residual BF16 codes BF16(x - c_l) (kpad columns), FP32 residual norms per row
// and the largest residual norm per list.
void launch_residual_bf16(const float* codes, const int64_t* list_off, const float* cent, int nlist, int dpad, int kpad,
                          void* dst, float* rnorm, float* rmax, cudaStream_t st);
// Seed bound from the first S <= 256 rows of each query's nearest list (probe
// rank 0 in the list-major work description; with probes given and a small
// batch, one CTA per query).
void launch_seed_bound(const float* q, int d, int dpad, const float* cent, int nq, int kpad, const void* codes_bf16,
                       const int64_t* list_off, int nlist, const int64_t* list_qoff, const int32_t* list_q,
                       const float* rnorm, const float* rmax, int S, int k, uint32_t* thr, cudaStream_t st,
                       const int32_t* probes = nullptr, int P = 0);
// Exact re-rank of the admitted rows whose lower bound is at most U, the k-th
// smallest admitted upper bound (cand_ub); flag[q] = 2 and
// over_list[0 .. over_n[0]) for queries whose buffer overflowed (left
// unwritten); over_list[nq ..] / over_n[1] list the queries with more than
// 256 candidates, re-ranked by the flat kernels, which overwrite their
// buffers (over_list holds 2 nq ints, over_n 2, zeroed by the caller);
// m_out[q] = rows re-ranked.
void launch_rerank_bf16(uint64_t* cand, const uint32_t* cand_ub, const int* cnt, int cap, int nq, int k,
                        const float* codes, const float* q, int dpad, const int64_t* ids, float* D, int64_t* I,
                        int* flag, int* over_list, int* over_n, int* m_out, int num_sms, cudaStream_t st);

// Largest k whose bound tightens inside the BF16 scan; a larger k takes two
// stages (the nearest list of every query first, then the rest under the
// k-th value the first stage admitted).
constexpr int kFilterTightK = 16;
// Per query: thr = min(thr, k-th smallest admitted upper bound) when the
// buffer holds at least k rows and did not overflow.
void launch_kth_bound(const uint32_t* cand_ub, const int* cnt, int cap, int nq, int k, uint32_t* thr,
                      cudaStream_t st);
// first[q] = probes[q][0]; rest = probes with column 0 set to -1.
void launch_split_first_probe(const int32_t* probes, int nq, int P, int32_t* first, int32_t* rest, cudaStream_t st);

// Candidate-matrix BF16 scan (k_cand.cu): any kpad (a multiple of 64) and up
// to kCandMaxR candidates per query.
constexpr int kCandMaxR = 4096;
struct CandArgs {
  const int64_t* list_off;
  int nlist;
  int kpad;
  const float* tile_norm;   // residual norms ||x - c_l||^2 per 128-row tile, +inf past each list's end
  const int64_t* tile_off;
  const int32_t* list_cnt;  // the list-major work description (launch_build_work, groups of 128)
  const int64_t* list_qoff;
  const int32_t* list_q;
  const int64_t* item_off;
  int chunk_rows;           // multiple of 128
  int P;
  const int64_t* seg;       // nq x P + 1: start of each (query, probe rank) segment of `cand`
  float* cand;              // candidate rows: ||x||^2 - 2 q~.x~, +inf padding
  int* err;
  int fp8;                  // 1: E4M3 residual operands (kpad = FP8 row bytes, a multiple of 128)
  const float* qscale;      // FP8: per list-major entry s_e (q - c_l ~ s_e * code)
  const float* qcd;         // per entry ||q - c_l||^2 (the operands are residuals to c_l)
  const float* list_scale;  // FP8: per list s_l (x - c_l ~ s_l * code)
};
size_t cand_segments_tmp_bytes(int nq, int P);
void launch_cand_segments(const int32_t* probes, int nq, int P, const int64_t* list_off, int64_t* seg, void* tmp,
                          size_t tmp_bytes, cudaStream_t st);
void launch_cand_scan(const void* tmap_q, const void* tmap_x, const CandArgs& a, int num_sms, cudaStream_t st);
// FP8 E4M3 copies for the candidate scan, as residuals to the list centroid:
// codes per list with s_l = max |x - c_l| / 448 (and the rows' FP32 residual
// norms), and per list-major entry (q, l) the row q - c_l with its own scale
// and ||q - c_l||^2.
void launch_fp8_codes(const float* codes, const int64_t* list_off, const float* cent, int nlist, int dpad, int kpad8,
                      void* out, float* scale, float* rnorm, cudaStream_t st);
// Per list-major entry e (query q, list l): row e of G = q - c_l in BF16, or
// (fp8) E4M3 with its scale escale[e]; ecd[e] = ||q - c_l||^2.
void launch_gather_residual(const float* q, int dpad, int kpad, bool fp8, const int32_t* list_q,
                            const int64_t* list_qoff, int nlist, const float* cent, int64_t max_rows, float* escale,
                            float* ecd, void* G, cudaStream_t st);
void make_u8_tensor_map(void* tmap_out, const void* base, size_t rows, int row_bytes);
// Selection of each query's R candidates (rows: nq x R stored rows, -1 past
// the candidates), then their exact re-rank to the k best.
void launch_cand_select(const float* cand, const int64_t* seg, const int32_t* probes, int nq, int P, int R,
                        const int64_t* list_off, int64_t* rows, cudaStream_t st);
void launch_cand_exact(const int64_t* rows, int nq, int R, int k, const float* codes, const float* q, int dpad,
                       const int64_t* ids, float* D, int64_t* I, cudaStream_t st);
void launch_to_bf16(const float* src, size_t n, int dpad, int kpad, void* dst, cudaStream_t st);
void launch_scan_bf16(const void* tmap, const TcArgs& a, int num_sms, cudaStream_t st);
// One thread waits on an mbarrier nothing arrives on, with a budget of
// `budget` cycles: *err gets `code` and *waited the cycles spent (-1 if the
// wait had completed, which cannot happen).
void launch_wait_selftest(long long budget, int code, int* err, long long* waited, cudaStream_t st);
// *out = max over i of sqrt(norms[i]) (slightly rounded up), on the device.
void launch_max_norm(const float* norms, size_t n, float* out, cudaStream_t st);
// probes (nq x P) -> first column (nq x 1) and the rest (nq x (P-1)).

// k_coarse_tc.cu: tensor-core coarse quantizer (3-term BF16 split) with an
// exact FP32 finish; the probe rows equal the exact quantizer's.
constexpr int kCoarseMaxPm = 1024;  // largest candidate count per query
size_t coarse_tc_smem_bytes(int kpad);
// cent (nlist x dpad FP32) -> out (nlist x 2*kpad BF16 [hi|lo]) + its tensor map.
void make_centroid_split(const float* cent, int nlist, int dpad, int kpad, void* out, void* tmap_out, cudaStream_t st);
// V (nq x nlist) = max(0, ||q||^2 + ||c||^2 - 2 q.c) on the tensor cores;
// qsplit (nq x 2*kpad BF16) and qnorm (nq) are scratch for the queries'
// [hi|lo] rows and norms.
// cmins (optional, ceil(nlist / 16) x nq, chunk-major) gets the bit pattern
// of the smallest value of each 16-column chunk of each row, for
// launch_select_rows' chunk path.
void launch_coarse_tc(const void* tmap, const float* q, int nq, int dpad, int kpad, const float* cnorm, int nlist,
                      float* V, void* qsplit, float* qnorm, uint32_t* cmins, int* err, int num_sms, cudaStream_t st);
// Per-row widths of a coarse pass: row r keeps width[r] <= P probes out of
// width[r] + margin candidates; rows whose width is <= pre_w are copied from
// an earlier pass of width pre_w (pre, nq x pre_w).  width == nullptr: every
// row keeps P of Pm.
struct CoarseRows {
  const int32_t* width = nullptr;
  int margin = -1;
  const int32_t* pre = nullptr;
  int pre_w = 0;
};
// Exact distances of the Pm candidates, top P, exactness flag per query.
void launch_coarse_refine(const float* q, int nq, int dpad, const float* cent, const int32_t* cand, const float* cval,
                          int Pm, int P, int nlist, const float* cmaxnorm, int32_t* probes, float* cdist, int* flags,
                          cudaStream_t st, CoarseRows rows = CoarseRows());
// Exact row and top P (or width[r]) for every flagged query (V rows are overwritten).
// cmins (optional): the rewritten rows' chunk minima are rewritten too.
void launch_coarse_fallback(const float* q, int nq, int dpad, const float* cent, int nlist, int P, const int* flags,
                            float* V, int32_t* probes, float* cdist, cudaStream_t st, const int32_t* width = nullptr,
                            uint32_t* cmins = nullptr);
// With w = min(width[r], wmax): kq[r] = 0 if w <= pre_w, else
// min(nlist, w + margin).
void launch_coarse_widths(const int32_t* width, int nq, int wmax, int pre_w, int margin, int nlist, int32_t* kq,
                          cudaStream_t st);

// k_mlp.cu: learned probe predictor kernels.
// Fused tensor-core inference (features -> 3 layers -> bucket choice) for
// K1 = roundup(d + C, 64) <= 256 and NB <= 32; weights packed by
// mlp_pack_bf16 (N x K FP32 -> Npad x Kpad BF16).
void mlp_pack_bf16(const float* W, int N, int K, int Npad, int Kpad, void* out, cudaStream_t st);
void mlp_infer_tc(const float* q, int nq, int d, int dpad, const float* cdist, int P, int C, const float* mean,
                  const float* inv_std, int K1, const void* W1b, const float* b1, const void* W2b, const float* b2,
                  const void* W3b, const float* b3, int NB, const int32_t* bucket_val, float thr, int cap,
                  int32_t* nprobe_out, int* err, cudaStream_t st);
void mlp_gemm(int M, int N, int K, const float* A, int lda, bool tA, const float* B, int ldb, bool tB, float* C, int ldc,
              const float* bias, float beta, bool gelu, float* Z, bool round_bf16, cudaStream_t st);
void mlp_gelu_backward(const float* dH, const float* Z, float* dZ, size_t n, cudaStream_t st);
void mlp_softmax_ce(const float* logits, const int32_t* labels, int B, int NB, float* dlogits, float* loss,
                    cudaStream_t st);
void mlp_colsum(const float* dY, int B, int N, float* db, cudaStream_t st);
void mlp_adam(float* w, const float* g, float* m, float* v, size_t n, float lr, int step, float wd, cudaStream_t st);
void mlp_round_bf16(const float* src, float* dst, size_t n, cudaStream_t st);
void mlp_features(const float* q, int nq, int d, int dpad, const float* cdist, int P, int C, float* out,
                  cudaStream_t st);
void mlp_moments(const float* x, int rows, int F, float* mean, float* inv_std, cudaStream_t st);
void mlp_standardize(float* x, int rows, int F, const float* mean, const float* inv_std, bool round_bf16,
                     cudaStream_t st);
void mlp_choose_nprobe(const float* logits, int nq, int NB, const int32_t* bucket_val, float thr, int cap,
                       int32_t* nprobe_out, int32_t* probes, int P, cudaStream_t st);
void launch_cut_probes(const int32_t* nprobe, int nq, int P, int32_t* probes, cudaStream_t st);
void launch_label_rank(const int64_t* I, int nq, int k, const int32_t* list_of_id, const int32_t* probes, int P,
                       int32_t* need, int32_t* ranks, cudaStream_t st);
void launch_list_of_id(const int64_t* list_off, int nlist, const int64_t* ids, int32_t* out, int64_t max_id,
                       cudaStream_t st);

// hb_index.cu: pieces the no-allocation entry point (hb_noalloc.cu) uses.
// Device ordinal of an index (-1 for a null handle).
int index_device(const hb_index* ix);
// ORIGINAL-mode exact search with every per-call device buffer carved from
// `scratch` (device memory of `scratch_bytes`); device pointers only; makes
// no device allocation.  Returns an hb_status and sets the last error.
int search_in_scratch(hb_index* ix, size_t nq, const float* q, size_t k, float* D, int64_t* I, void* scratch,
                      size_t scratch_bytes);
void set_last_error(const char* msg);

}  // namespace hb

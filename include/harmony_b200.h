/*
 * harmony_b200 -- C ABI of the B200 IVF-flat index.
 *
 * This is the drop-in boundary for the IVF-flat train/add/search path of
 * xuqianmamba/Harmony.  Each entry point replaces one member of the
 * reference's C++ class harmony::Index (src/Index.h) and keeps its argument
 * meaning; errors come back as status codes plus a thread-local message
 * instead of C++ exceptions (the reference throws std::runtime_error at
 * src/Index.cpp:60, 464, 1644, 1711, 1737).
 *
 * Conventions
 *   - Every function returns HB_OK (0) or an hb_status error code; the text
 *     of the last error on the calling thread is hb_last_error().
 *   - Array arguments may be host or device pointers (CUDA unified
 *     addressing tells them apart).  Results land where the caller's pointer
 *     points.  Host arrays are copied through the index's own stream.
 *   - One CUDA stream per index (hb_stream).  An index is not re-entrant,
 *     like the reference (search mutates nprobe, src/Index.cpp:1646-1648).
 *   - Vector ids are int64 (idx_t in src/common.h:83); distances are squared
 *     L2 in float32, ascending per query; missing results are FLT_MAX / -1
 *     (heap_init, src/heap.hpp:13-25).
 */
#ifndef HARMONY_B200_H
#define HARMONY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hb_index hb_index;

typedef enum {
  HB_OK = 0,
  HB_ERR_INVALID = 1,   /* bad argument or unsupported option            */
  HB_ERR_CUDA = 2,      /* CUDA runtime error (message has the detail)   */
  HB_ERR_IO = 3,        /* index file could not be opened / parsed       */
  HB_ERR_STATE = 4,     /* call out of order (e.g. add before train)     */
  HB_ERR_NOMEM = 5,     /* device or host allocation failed              */
  HB_ERR_NODEVICE = 6   /* no CUDA device / library built without it     */
} hb_status;

/* MetricType, src/common.h:20-21 (same values). Only L2 is implemented. */
enum { HB_METRIC_IP = 0, HB_METRIC_L2 = 1 };

/* Index::SearchMode, src/Index.h:29-35 (same order). */
enum {
  HB_MODE_BRUTE_FORCE = 0,
  HB_MODE_ORIGINAL = 1,   /* single-process search, src/Index.cpp:1664-1703   */
  HB_MODE_DIVIDE_IVF = 2, /* list partition + warm-up pruning, node.cpp:606  */
  HB_MODE_DIVIDE_DIM = 3, /* dimension relay + pruning, node.cpp:297-431     */
  HB_MODE_DIVIDE_GROUP = 4
};

/* Arithmetic of the list scan. FP32 reproduces the reference's distances
 * bit for bit; BF16 / FP8 scan on tensor cores and re-rank a widened
 * candidate set in exact FP32.  BF16 with d <= 128 and k <= 256 re-ranks every
 * row within its proven error bound, so its result equals FP32's; FP8 (E4M3
 * with per-list and per-query scales, the candidate-matrix scan) re-ranks
 * rerank_mult * k candidates, and its agreement with FP32 is measured, not
 * guaranteed. */
enum { HB_PREC_FP32 = 0, HB_PREC_BF16 = 1, HB_PREC_FP8 = 2 };

/* Search options: the fields of Index::Param that steer search
 * (src/Index.h:48-68) plus the GPU-only knobs.  hb_search_params_init()
 * fills the reference defaults. */
typedef struct {
  int32_t mode;               /* HB_MODE_*; default ORIGINAL                    */
  int32_t pruning;            /* Param::pruning / !--disablePruning            */
  int32_t order_optimize;     /* Param::orderOptimize                          */
  int32_t period;             /* Param::period                                 */
  int32_t n_dim_blocks;       /* DIVIDE_DIM workers = dimension slices (d % n == 0) */
  int32_t n_query_blocks;     /* DIVIDE_DIM blockCount                         */
  int32_t warmup_lists;       /* preSearch warmUpSearchList (default 10)        */
  int32_t warmup_list_size;   /* preSearch warmUpSearchListSize (0 -> k)        */
  int32_t precision;          /* HB_PREC_*                                     */
  int32_t rerank_mult;        /* FP8, and BF16 with d > 128 or k > 256 (the candidate-
                                 matrix scan): candidates re-ranked = rerank_mult * k, at
                                 most 4096, k itself up to 4096 (default 2).  For
                                 d <= 128 and k <= 256 the re-ranked set is every row
                                 within the scan's error bound of the k-th, and the
                                 result equals the FP32 scan's; this field is unused */
  int32_t learned_probe;      /* 1: per-query nprobe from the learned predictor */
  float learned_target;       /* predictor target recall (0 -> trained target)   */
  const int32_t* nprobe_per_query; /* optional nq array (host or device); overrides nprobe */
  int32_t max_nprobe;         /* cap for per-query nprobe (0 -> index nprobe)    */
  int32_t seed_rows;          /* BF16: rows of each query's nearest list behind
                                 the scan's initial bound (0 -> 256, max 256)  */
  int32_t use_graph;          /* 1: run the batch as one CUDA-graph launch,
                                 captured on first use per batch shape (see
                                 hb_search); ORIGINAL / BRUTE_FORCE, one batch */
  int32_t full_warmup;        /* Param::fullWarmUp: DIVIDE_DIM prunes against the
                                 caller's heap_tops instead of running the warm-up
                                 search (src/Index.cpp:1235-1241); the other modes
                                 ignore it, as the reference does                */
  const float* heap_tops;     /* Param::heapTops: nq floats (host or device); must
                                 be set when full_warmup is (the reference exits
                                 with "heapTop not exist"; here HB_ERR_INVALID)   */
  int32_t reserved[2];
} hb_search_params;

void hb_search_params_init(hb_search_params* p);

/* Thread-local text of the last error ("" if none). */
const char* hb_last_error(void);

/* Version string and build info. */
const char* hb_version(void);

/* Index(d, nlist, nprobe, metric, ...), src/Index.h:15-25 and
 * src/Index.cpp:24-43.  device: CUDA ordinal. */
int hb_create(size_t d, size_t nlist, size_t nprobe, int metric, int device, hb_index** out);
int hb_destroy(hb_index* ix);

/* Index::train(n, codes), src/Index.cpp:381-425: k-means, 20 iterations
 * (2 with lite), seed 6666, at most 256 points per centroid. */
int hb_train(hb_index* ix, size_t n, const float* x, int lite);

/* Index::add(n, codes), src/Index.cpp:581-698: replaces the lists with the
 * n vectors, ids 0..n-1. */
int hb_add(hb_index* ix, size_t n, const float* x);

/* Index::search(n, queries, k, distances, labels), src/Index.cpp:1638-1706.
 * params may be NULL (ORIGINAL, FP32).  D: nq*k floats, I: nq*k int64. */
int hb_search(hb_index* ix, size_t nq, const float* q, size_t k, const hb_search_params* params,
              float* D, int64_t* I);

/* Index::save_index / load_index, src/Index.cpp:1708-1770 (byte format of
 * the reference). */
int hb_save_index(hb_index* ix, const char* path);
int hb_load_index(hb_index* ix, const char* path);

/* The public field Index::nprobe (mutated between searches by the
 * reference driver, src/query.cpp:683). */
int hb_set_nprobe(hb_index* ix, size_t nprobe);
int hb_get_nprobe(const hb_index* ix, size_t* nprobe);

/* Shape of the index. ntotal = vectors added. */
int hb_get_info(const hb_index* ix, size_t* d, size_t* nlist, size_t* ntotal, int* metric);

/* Copies of the index content (host or device destinations). */
int hb_get_centroids(const hb_index* ix, float* out);        /* nlist * d          */
int hb_get_list_sizes(const hb_index* ix, int64_t* out);     /* nlist              */

/* List sharding across GPUs (the reference's DIVIDE_IVF partition,
 * src/Index.cpp:79-104 and 1279-1347, with the merge on the device).
 * hb_retain_lists keeps lists [first, first + count) and empties the others;
 * ids are unchanged, so every shard reports the full index's ids.
 * hb_merge_topk merges nparts result rows per query (D_parts, I_parts:
 * nparts x nq x k, part-major, device memory) into D, I (nq x k, device) with
 * the reference master's rule (src/Index.cpp:1327-1341): a max-heap of k,
 * parts in order, a value admitted when strictly below the top, then sorted
 * ascending.  Runs on the index's stream and returns when done. */
int hb_retain_lists(hb_index* ix, size_t first, size_t count);
int hb_merge_topk(hb_index* ix, size_t nparts, size_t nq, size_t k, const float* D_parts, const int64_t* I_parts,
                  float* D, int64_t* I);

/* Exact search that allocates no device memory.  No counterpart in the
 * reference (its search allocates freely).  For callers that cannot allocate
 * while serving a query: a process whose device memory belongs to another
 * allocator or a fixed pool (cudaMalloc there can fail or fragment it), or a
 * latency-bound one (cudaFree synchronises the whole device).  Same results
 * as hb_search in ORIGINAL mode at the index's nprobe; q, D and I must be
 * device pointers.  All per-call scratch comes from one 32 MiB array built
 * into the library (held on every GPU that loads it); searches needing more
 * (about nq*nlist*4 bytes of coarse distances plus the work description and
 * partial top-k) are rejected with HB_ERR_INVALID.  The first call for an
 * index on a device looks the array's address up (make it before any stream
 * capture); calls share the array, so calls whose GPU work overlaps race. */
int hb_search_noalloc(hb_index* ix, size_t nq, const float* q, size_t k, float* D, int64_t* I);

/* Coarse quantizer only: probe lists of each query, ascending by exact
 * centroid distance (Index::findNearNprobeOfCentroidIds,
 * src/Index.cpp:967-995).  probes: nq*nprobe int64, cdist may be NULL. */
int hb_probe_lists(hb_index* ix, size_t nq, const float* q, size_t nprobe, int64_t* probes,
                   float* cdist);

/* Coarse quantizer route (no reference counterpart; the probe rows are the
 * same on every route).  AUTO: tensor cores for d <= 128 (a 3-term BF16
 * split picks nprobe + margin candidates, re-ranked in exact FP32; queries
 * whose candidates cannot be proven to hold the exact top nprobe are
 * recomputed exactly), else the FP32 distance matrix.  EXACT: always the
 * FP32 matrix.  TENSOR: tensor cores or HB_ERR_INVALID.  margin -1 picks
 * max(16, nprobe / 4). */
enum { HB_COARSE_AUTO = 0, HB_COARSE_EXACT = 1, HB_COARSE_TENSOR = 2 };
int hb_set_coarse_quantizer(hb_index* ix, int kind, int margin);
/* Queries of the most recent tensor-core coarse call that were recomputed
 * exactly (0 after an EXACT call). */
int hb_coarse_fallbacks(hb_index* ix, int64_t* n);

/* Warm-up heap tops (Index::warmUpSearch, src/Index.cpp:999-1051). */
int hb_warmup_tops(hb_index* ix, size_t nq, const float* q, size_t k, size_t warm_lists,
                   size_t warm_list_size, float* tops);

/* The CUDA stream this index launches on (a cudaStream_t). */
void* hb_stream(hb_index* ix);

/* Number of kernels this index has launched so far (for launch accounting). */
uint64_t hb_launch_count(const hb_index* ix);

/* Device allocations (cudaMalloc calls) the library has made in this process,
 * over all indexes.  No reference counterpart: a diagnostic that lets a
 * caller check that a call allocated nothing. */
uint64_t hb_device_allocations(void);

/* Autotuner of the bounded BF16 scan (no reference counterpart).  With
 * hb_set_autotune(ix, 1) the first BF16 search of each (batch size rounded up
 * to a power of two, nprobe rounded up likewise, k) times the scan for chunk
 * lengths of 1/4 to 4 times the default (128 to 4096 rows) and ring depths of
 * 2 to 4 tiles, twice each, and keeps the fastest for later searches of that
 * bucket (every choice gives the same results).  hb_autotune_table writes the
 * table as text, one line "nb_bucket nprobe_bucket k kpad chunk_rows stages
 * best_ms default_ms" per bucket (*needed = bytes including the terminating
 * zero); hb_set_autotune_table replaces it with such text (lines for another
 * kpad are dropped), so a tuned table can be saved and reloaded. */
int hb_set_autotune(hb_index* ix, int on);
int hb_autotune_table(hb_index* ix, char* buf, size_t len, size_t* needed);
int hb_set_autotune_table(hb_index* ix, const char* text);

/* Clock cycles a device-side wait of the BF16 scan spends before it gives
 * up (no reference counterpart; cycles <= 0 restores the default, 2e9).  A
 * wait that gives up makes the search return HB_ERR_CUDA with "gave up
 * waiting" and leaves the index usable. */
int hb_set_wait_budget(hb_index* ix, int64_t cycles);

/* Queries of the most recent BF16 search (d <= 128, k <= 256) whose
 * candidate buffer overflowed and that were searched again with the exact
 * FP32 scan (no reference counterpart). */
int hb_bf16_fallbacks(hb_index* ix, int64_t* n);

/* Admission statistics of the latest bounded BF16 batch (no reference
 * counterpart): stats[0] queries, [1] overflows (searched exactly), [2] rows
 * admitted over all queries, [3] the most any query admitted, [4] rows
 * re-ranked exactly over all queries. */
int hb_bf16_stats(hb_index* ix, int64_t* stats);

/* Self-test of the device-side bounded waits (no reference counterpart).
 * Every mbarrier wait in the tensor-core kernels gives up after a clock
 * budget, records an error code in a device flag and lets its kernel return,
 * and the host reports HB_ERR_CUDA.  This launches one kernel whose single
 * thread waits, with budget_cycles, on an mbarrier nothing arrives on (no
 * copy or MMA in flight), so it returns HB_ERR_CUDA with "gave up waiting
 * (code 99)" and the cycles the wait took in *waited_cycles; the index stays
 * usable afterwards. */
int hb_selftest_bounded_wait(hb_index* ix, int64_t budget_cycles, int64_t* waited_cycles);

/* Per-kernel timing: when enabled, the index records CUDA events around each
 * of its kernels on its own stream.  hb_profile_read synchronises the stream,
 * returns per kernel name (newline-separated in `names`) the summed device
 * time in ms and the number of launches, and clears the record. */
int hb_profile_enable(hb_index* ix, int on);
int hb_profile_read(hb_index* ix, char* names, size_t names_len, double* ms, int64_t* counts,
                    int max_entries, int* n_entries);

/* Learned probe predictor (no reference counterpart): train from nt training
 * queries labelled by the plain search at nprobe = label_nprobe, for a recall
 * target in (0, 1]. */
int hb_train_probe_predictor(hb_index* ix, size_t nt, const float* q, size_t k, size_t label_nprobe,
                             float target);

/* Validation curve of the trained predictor: for each probability threshold,
 * the recall against the label search and the average nprobe it gives. */
int hb_probe_calibration(const hb_index* ix, float* thr, float* recall, float* avg_nprobe, int max_n, int* n);

#ifdef __cplusplus
}
#endif
#endif /* HARMONY_B200_H */

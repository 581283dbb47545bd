/* CPU restatement of the reference's IVF-flat train/add/search algorithm.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path:
 * only tests/, the package smoke check and the bench's CPU-baseline leg may
 * load it.  Nothing in the product links it.
 *
 * Index layout used by every function (CSR, lists concatenated in list order):
 *   list_off[nlist + 1]   vector offsets of each list
 *   ids[nb]               int64 ids in list order
 *   codes[nb * d]         float32 rows in list order
 *
 * Arithmetic: every L2 distance is the reference's sequential, unfused FP32
 * loop (src/utils.h:480-487): acc = acc + (a-b)*(a-b), dims in order, each
 * product rounded before the add.  Built with -ffp-contract=off.
 */
#ifndef IVF_ORACLE_H
#define IVF_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

float orc_l2(const float* a, const float* b, size_t d);

/* Max-heap of k (val, id) pairs: src/heap.hpp:13-90. */
void orc_heap_init(size_t k, float* val, int64_t* ids);
void orc_heap_replace_top(size_t k, float* val, int64_t* ids, float v, int64_t id);
void orc_heap_sort(size_t k, float* val, int64_t* ids);
void orc_heap_topk(size_t n, const float* vals, size_t k, float* D, int64_t* I);

/* Coarse quantizer: nprobe nearest centroids per query, ascending
 * (src/IVFScan.hpp:108-138 + src/Index.cpp:1440-1448). */
void orc_coarse(size_t nq, const float* q, size_t d, size_t nlist, const float* cent,
                size_t nprobe, float* cd, int64_t* cl);

/* ORIGINAL-mode search (src/Index.cpp:1420-1554, 1638-1706). */
void orc_search(size_t nq, const float* q, size_t d, size_t nlist, const float* cent,
                const int64_t* list_off, const int64_t* ids, const float* codes,
                size_t nprobe, size_t k, float* D, int64_t* I);

/* Search with a caller-given probe table (nq x nprobe list ids, -1 = skip). */
void orc_search_probes(size_t nq, const float* q, size_t d, const int64_t* list_off,
                       const int64_t* ids, const float* codes, size_t nprobe,
                       const int64_t* probes, size_t k, float* D, int64_t* I);

/* Warm-up heap tops (src/Index.cpp:999-1051, 1300-1305). */
void orc_warmup_tops(size_t nq, const float* q, size_t d, const int64_t* list_off,
                     const int64_t* ids, const float* codes, size_t nprobe,
                     const int64_t* probes, size_t k, size_t warm_lists,
                     size_t warm_list_size, float* tops);

/* Base-mode worker scan with 4-chunk early abandon (src/node.cpp:606-678). */
void orc_search_pruned(size_t nq, const float* q, size_t d, const int64_t* list_off,
                       const int64_t* ids, const float* codes, size_t nprobe,
                       const int64_t* probes, const float* tops, int cut, size_t k,
                       float* D, int64_t* I);

/* Dimension-partition relay (src/node.cpp:297-431, src/Index.cpp:1188-1278):
 * W dimension slices of d/W dims; query block b = queries
 * [b*bs, (b+1)*bs) with bs = nq / B; order[b*W + t] = slice visited at hop t.
 * Queries past B*bs are never searched (they keep FLT_MAX / -1). */
void orc_search_dimblock(size_t nq, const float* q, size_t d, const int64_t* list_off,
                         const int64_t* ids, const float* codes, size_t nprobe,
                         const int64_t* probes, const float* tops, int cut, size_t W,
                         size_t B, const int64_t* order, size_t k, float* D, int64_t* I);

/* Block visit order of the dimension-partition mode:
 * src/order.h:38-96, with the "period" variant of src/Index.cpp:183-197. */
void orc_block_order(size_t W, size_t B, int order_optimize, int period, int64_t* order);

/* k-means (src/Clustering.cpp:14-152, params from src/Index.cpp:385-394):
 * subsample with std::shuffle(default_random_engine(seed)) when
 * n > nlist*max_pts, initialise from a second shuffle, niter Lloyd steps,
 * argmin with strict '<' (lowest index wins), sums in point order, empty
 * clusters keep their centroid.  cent_out: nlist * d. */
void orc_kmeans(size_t n, const float* x, size_t d, size_t nlist, int niter, int seed,
                size_t max_pts, float* cent_out);

/* Subsample / init index draws of the k-means above (for checking the
 * device trainer's host-side sampling). sample_idx: min(n, nlist*max_pts);
 * init_idx: nlist. */
void orc_kmeans_indices(size_t n, size_t nlist, int seed, size_t max_pts, int64_t* sample_idx,
                        int64_t* init_idx);

/* Index::add (src/Index.cpp:581-698): nearest centroid by strict '<',
 * list sizes, then every vector in ascending order of its centroid distance
 * (ties: ascending row index), ids = row index, norms = sequential <x,x>.
 * Outputs sized nlist+1 / n / n*d / n. */
void orc_add(size_t n, const float* x, size_t d, size_t nlist, const float* cent,
             int64_t* list_off, int64_t* ids, float* codes, float* norms);

/* FP64 brute-force ground truth: k smallest by (double distance, id). */
void orc_bruteforce_f64(size_t nq, const float* q, size_t nb, const float* x, size_t d,
                        size_t k, double* D, int64_t* I);

#ifdef __cplusplus
}
#endif
#endif

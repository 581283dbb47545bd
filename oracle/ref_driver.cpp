// Test-oracle driver: a C ABI over the reference's own harmony::Index, built
// from the unmodified reference sources (src/Index.cpp, src/IVF.cpp,
// src/Clustering.cpp, src/node.cpp) with the stand-ins in ref_shim/.
//
// This file is test infrastructure.  Only tests/, the package smoke check and
// the bench's CPU-baseline leg load the library it builds (oracle/_ref/).
//
// Entry points follow the reference's single-process call sequence:
//   Index(d, nlist, nprobe, METRIC_L2, OPT_NONE, 0, 1, 1, false)   src/Index.h:15-25
//   train / add                                                     src/Index.cpp:381, 581
//   preSearch(nb, 0, 0, 0, 0, &param{ORIGINAL}, "")                 src/Index.cpp:45-55
//   search                                                          src/Index.cpp:1638-1706
//   save_index / load_index                                         src/Index.cpp:1708-1770
// The pruned path drives BaseWorker::single_thread_search_simple
// (src/node.cpp:606-678) directly, with heap tops computed by
// Index::warmUpSearch (src/Index.cpp:999-1051) as search_divide_ivf does
// (src/Index.cpp:1300-1305).
#define private public
#define protected public
#include "tribase.h"
#include "node.h"
#include "order.h"
#undef private
#undef protected

#include <omp.h>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

using namespace harmony;

namespace {
struct RefHandle {
  std::unique_ptr<Index> index;
  Index::Param param;
};

void set_original(RefHandle* h) {
  h->param = Index::Param();
  h->param.mode = Index::SearchMode::ORIGINAL;
  h->param.pruning = false;
  h->param.hardInBalance = false;
  h->index->preSearch(0, 0, 0, 0, 0, &h->param, "");
}

// The reference prints a banner on every search; keep test output readable.
struct QuietStdout {
  std::streambuf* old;
  std::ostringstream sink;
  QuietStdout() : old(std::cout.rdbuf(sink.rdbuf())) {}
  ~QuietStdout() { std::cout.rdbuf(old); }
};
}  // namespace

extern "C" {

void ref_set_threads(int n) { omp_set_num_threads(n > 0 ? n : omp_get_num_procs()); }
int ref_max_threads(void) { return omp_get_max_threads(); }

void* ref_index_new(size_t d, size_t nlist, size_t nprobe) {
  auto* h = new RefHandle();
  h->index = std::make_unique<Index>(d, nlist, nprobe, METRIC_L2, OPT_NONE, 0, 1, 1, false);
  h->index->added_opt_level = OPT_NONE;
  set_original(h);
  return h;
}

void ref_index_free(void* p) { delete static_cast<RefHandle*>(p); }

void ref_train(void* p, size_t n, const float* x) {
  QuietStdout q;
  static_cast<RefHandle*>(p)->index->train(n, x);
}

void ref_add(void* p, size_t n, const float* x) {
  QuietStdout q;
  static_cast<RefHandle*>(p)->index->add(n, x);
}

void ref_set_nprobe(void* p, size_t nprobe) { static_cast<RefHandle*>(p)->index->nprobe = nprobe; }

size_t ref_nprobe(void* p) { return static_cast<RefHandle*>(p)->index->nprobe; }
size_t ref_d(void* p) { return static_cast<RefHandle*>(p)->index->d; }
size_t ref_nlist(void* p) { return static_cast<RefHandle*>(p)->index->nlist; }

void ref_search(void* p, size_t nq, const float* q, size_t k, float* D, int64_t* I) {
  QuietStdout quiet;
  auto* h = static_cast<RefHandle*>(p);
  h->index->search(nq, q, k, D, I);
}

int ref_save(void* p, const char* path) {
  try {
    static_cast<RefHandle*>(p)->index->save_index(path);
  } catch (...) {
    return 1;
  }
  return 0;
}

void* ref_load(const char* path) {
  auto* h = new RefHandle();
  h->index = std::make_unique<Index>();
  try {
    QuietStdout q;
    h->index->load_index(path);
  } catch (...) {
    delete h;
    return nullptr;
  }
  set_original(h);
  return h;
}

void ref_centroids(void* p, float* out) {
  auto* ix = static_cast<RefHandle*>(p)->index.get();
  std::memcpy(out, ix->centroid_codes.get(), sizeof(float) * ix->nlist * ix->d);
}

size_t ref_list_size(void* p, size_t list) {
  auto* ix = static_cast<RefHandle*>(p)->index.get();
  return ix->lists[list].get_list_size();
}

// Copies one inverted list: ids (size_t in the reference), codes, norms.
void ref_list_copy(void* p, size_t list, int64_t* ids, float* codes, float* norms) {
  auto* ix = static_cast<RefHandle*>(p)->index.get();
  IVF& l = ix->lists[list];
  for (size_t i = 0; i < l.list_size; ++i) ids[i] = static_cast<int64_t>(l.candidate_id[i]);
  if (codes) std::memcpy(codes, l.candidate_codes.get(), sizeof(float) * l.list_size * ix->d);
  if (norms) std::memcpy(norms, l.candidate_norms.get(), sizeof(float) * l.list_size);
}

// Probe lists as the DIVIDE_IVF / DIVIDE_DIM masters compute them
// (Index::findNearNprobeOfCentroidIds, src/Index.cpp:967-995).
void ref_probe_lists(void* p, size_t nq, const float* q, int64_t* out) {
  QuietStdout quiet;
  auto* h = static_cast<RefHandle*>(p);
  h->index->findNearNprobeOfCentroidIds(nq, q);
  std::memcpy(out, h->index->listidqueries.get(), sizeof(int64_t) * nq * h->index->nprobe);
}

// Heap tops after warm-up (src/Index.cpp:999-1051, 1300-1305).
void ref_warmup_tops(void* p, size_t nq, const float* q, size_t k, size_t warm_lists,
                     size_t warm_list_size, float* tops) {
  QuietStdout quiet;
  auto* h = static_cast<RefHandle*>(p);
  Index* ix = h->index.get();
  ix->findNearNprobeOfCentroidIds(nq, q);
  ix->warmUpSearchList = warm_lists;
  ix->warmUpSearchListSize = warm_list_size;
  std::vector<float> D(nq * k);
  std::vector<idx_t> I(nq * k);
  init_result(METRIC_L2, nq * k, D.data(), I.data());
  ix->warmUpSearch(nq, q, k, D.data(), I.data(), ix->listidqueries.get());
  for (size_t i = 0; i < nq; ++i) tops[i] = D[i * k];
}

// Base-mode worker scan over all lists with the chunked early abandon
// (cut=true) or without it (cut=false): src/node.cpp:606-678.  Results are
// sorted as the master's merge does (src/Index.cpp:1324-1343).
void ref_search_pruned(void* p, size_t nq, const float* q, size_t k, size_t warm_lists,
                       size_t warm_list_size, int cut, float* D, int64_t* I) {
  QuietStdout quiet;
  auto* h = static_cast<RefHandle*>(p);
  Index* ix = h->index.get();
  if (ix->nprobe > ix->nlist) ix->nprobe = ix->nlist;
  std::vector<float> tops(nq);
  ref_warmup_tops(p, nq, q, k, warm_lists, warm_list_size, tops.data());
  BaseWorker w;
  w.info = BaseWorker::InitInfo(ix->d, 1, ix->nlist, ix->nprobe, 0, 0, ix->nlist);
  w.cut = cut != 0;
  // The worker reads index->lists and index->d; lend it the loaded index.
  w.index.reset(ix);
  init_result(METRIC_L2, nq * k, D, I);
  w.single_thread_search_simple(nq, q, k, D, I, ix->listidqueries.get(), tops.data());
  (void)w.index.release();
  for (size_t i = 0; i < nq; ++i) sort_result(METRIC_L2, k, D + i * k, I + i * k);
}

// Worker visit order for the dimension-partition mode (src/order.h:38-96):
// out[b * W + t] = 0-based worker (dimension slice) that processes block b at
// its t-th hop.
void ref_block_order(size_t workers, size_t blocks, int order_optimize, int64_t* out) {
  SearchOrder so(workers, blocks, order_optimize != 0);
  for (size_t b = 0; b < blocks; ++b)
    for (size_t t = 0; t < workers; ++t) out[b * workers + t] = so.searchedWorkerOrder[b][t] - 1;
}

// Reference heap primitives (src/heap.hpp:13-90), exposed for the heap tests.
void ref_heap_topk(size_t n, const float* vals, size_t k, float* D, int64_t* I) {
  heap_init<METRIC_L2>(k, D, I);
  for (size_t i = 0; i < n; ++i)
    if (vals[i] < D[0]) heap_replace_top<METRIC_L2>(k, D, I, vals[i], static_cast<idx_t>(i));
  heap_sort<METRIC_L2>(k, D, I);
}

float ref_l2(const float* a, const float* b, size_t d) { return calculatedEuclideanDistance(a, b, d); }

// The query driver's evaluation helpers (src/utils.h:187-407, 631-755;
// src/stats.h:101-125), exposed for the harness tests.  Loaders copy rows
// a..b (1-based, inclusive; b = 0 for all) into out when out is non-null
// and return the row count, *d_out the dimension.
size_t ref_load_fvecs(const char* path, int a, int b, float* out, int* d_out) {
  auto [v, n, d] = loadFvecs(path, {a, b});
  *d_out = d;
  if (out && v) std::memcpy(out, v.get(), n * static_cast<size_t>(d) * sizeof(float));
  return n;
}

size_t ref_load_bvecs(const char* path, int a, int b, uint8_t* out, int* d_out) {
  auto [v, n, d] = loadBvecs(path, {a, b});
  *d_out = d;
  if (out && v) std::memcpy(out, v.get(), n * static_cast<size_t>(d));
  return n;
}

size_t ref_load_xvecs(const char* path, int a, int b, float* out, int* d_out) {
  auto [v, n, d] = loadXvecs(path, {a, b});
  *d_out = d;
  if (out && v) std::memcpy(out, v.get(), n * static_cast<size_t>(d) * sizeof(float));
  return n;
}

float ref_calculate_recall(const int64_t* I, const float* D, const int64_t* GT, const float* GD, size_t nq,
                           size_t k, size_t gt_k) {
  QuietStdout quiet;
  return calculate_recall(I, D, GT, GD, nq, k, METRIC_L2, gt_k);
}

float ref_calculate_recall_loose(const int64_t* I, const float* D, const int64_t* GT, const float* GD, size_t nq,
                                 size_t k, size_t gt_k) {
  QuietStdout quiet;
  return calculate_recall_loose(I, D, GT, GD, nq, k, METRIC_L2, gt_k);
}

float ref_calculate_r2(const int64_t* I, const float* D, const int64_t* GT, const float* GD, size_t nq, size_t k,
                       size_t gt_k) {
  return calculate_r2(I, D, GT, GD, nq, k, METRIC_L2, gt_k);
}

// Result files of the query driver (src/utils.h:565-620): ground truth and
// search results, text ("...txt": "label distance" pairs) or binary (labels
// then distances).
void ref_write_results(const int64_t* I, const float* D, size_t nq, size_t k, const char* path) {
  writeResultsToFile(I, D, nq, k, path);
}

void ref_load_results(const char* path, int64_t* I, float* D, size_t nq, size_t k) {
  loadResults(path, I, D, nq, k);
}

// Stats::toCsv (which = 0) or Stats::myToCsv (which = 1) of a Stats whose
// fields are iv = {nlist, nprobe, opt_level, total_count, skip_triangle_count,
// skip_triangle_large_count, skip_subnn_L2_count, skip_subnn_IP_count,
// simi_update_count, check_subnn_L2_ele_count, check_subnn_IP_ele_count,
// check_subnn_L2_count, check_subnn_IP_count, nb, nq, d, k, divideIVF,
// disableOrderOptimize, blockSend, pruning, block, worker, group, team} and
// dv = {simi_ratio, faiss_query_time, query_time, original_time, recall, r2,
// variance, trainTime, addTime, preSearchTime, inBalanceRatio,
// inBalanceRatioTeam, brute_ratio}.
void ref_stats_csv(const char* path, int append, const char* dataset, const char* mode, int which,
                   const int64_t* iv, const double* dv) {
  Stats s;
  s.nlist = iv[0];
  s.nprobe = iv[1];
  s.opt_level = static_cast<OptLevel>(iv[2]);
  s.total_count = iv[3];
  s.skip_triangle_count = iv[4];
  s.skip_triangle_large_count = iv[5];
  s.skip_subnn_L2_count = iv[6];
  s.skip_subnn_IP_count = iv[7];
  s.simi_update_count = iv[8];
  s.check_subnn_L2_ele_count = iv[9];
  s.check_subnn_IP_ele_count = iv[10];
  s.check_subnn_L2_count = iv[11];
  s.check_subnn_IP_count = iv[12];
  s.nb = iv[13];
  s.nq = iv[14];
  s.d = iv[15];
  s.k = iv[16];
  s.divideIVF = iv[17] != 0;
  s.disableOrderOptimize = iv[18] != 0;
  s.blockSend = iv[19] != 0;
  s.pruning = iv[20] != 0;
  s.block = iv[21];
  s.worker = iv[22];
  s.group = iv[23];
  s.team = iv[24];
  s.simi_ratio = static_cast<float>(dv[0]);
  s.faiss_query_time = dv[1];
  s.query_time = dv[2];
  s.original_time = dv[3];
  s.recall = dv[4];
  s.r2 = dv[5];
  s.variance = dv[6];
  s.trainTime = dv[7];
  s.addTime = dv[8];
  s.preSearchTime = dv[9];
  s.inBalanceRatio = dv[10];
  s.inBalanceRatioTeam = dv[11];
  s.brute_ratio = dv[12];
  s.mode = mode;
  if (which == 0)
    s.toCsv(path, append != 0, dataset);
  else
    s.myToCsv(path, append != 0, dataset);
}

}  // extern "C"

// Header-only C++ drop-in for the reference's harmony::Index (src/Index.h),
// forwarding to the C ABI of libharmony_b200.so (include/harmony_b200.h).
//
// Driver code written against the reference's Index -- construct, train,
// add, preSearch, set the public nprobe field, search into caller-owned
// float/idx_t arrays, save_index / load_index -- compiles against this header
// unchanged.  Errors become std::runtime_error, as the reference throws
// (src/Index.cpp:60, 464, 1644, 1711, 1737).  Pointers may be host or device.
#pragma once

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>

#include "harmony_b200.h"

namespace harmony {

using idx_t = int64_t;  // src/common.h:83
enum MetricType { METRIC_IP = 0, METRIC_L2 };  // src/common.h:20-21
enum OptLevel {  // src/common.h:23-32
  OPT_NONE = 0b000, OPT_TRIANGLE = 0b001, OPT_SUBNN_L2 = 0b010, OPT_SUBNN_IP = 0b100,
  OPT_TRI_SUBNN_L2 = 0b011, OPT_TRI_SUBNN_IP = 0b101, OPT_SUBNN_ONLY = 0b110, OPT_ALL = 0b111
};
enum EdgeDevice { EDGEDEVIVE_ENABLED, EDGEDEVIVE_DISABLED };  // src/common.h:34-37

struct Stats {};  // the reference's search return value (src/stats.h); not filled here

class Index {
 public:
  enum class SearchMode { BRUTE_FORCE, ORIGINAL, DIVIDE_IVF, DIVIDE_DIM, DIVIDE_GROUP };  // src/Index.h:29-35

  struct Param {  // src/Index.h:48-68 (the fields that steer search)
    bool orderOptimize = true;
    SearchMode mode = SearchMode::ORIGINAL;
    bool pruning = false;
    bool period = false;
    bool fullWarmUp = false;
    float* heapTops = nullptr;  // per-query pruning thresholds used when fullWarmUp (DIVIDE_DIM)
  };

  Index(size_t d = 0, size_t nlist = 0, size_t nprobe = 0, MetricType metric = METRIC_L2,
        OptLevel opt_level = OPT_NONE, size_t sub_k = 0, size_t sub_nlist = 1, size_t sub_nprobe = 1,
        bool verbose = false, EdgeDevice edge = EDGEDEVIVE_DISABLED, int device = 0)
      : d(d), nlist(nlist), nprobe(nprobe), metric(metric), opt_level(opt_level), sub_k(sub_k),
        sub_nlist(sub_nlist), sub_nprobe(sub_nprobe), verbose(verbose), edge_device_enabled(edge) {
    check(hb_create(d ? d : 16, nlist ? nlist : 1, nprobe, static_cast<int>(metric), device, &h_));
  }
  ~Index() { hb_destroy(h_); }
  Index(const Index&) = delete;
  Index& operator=(const Index&) = delete;

  void train(size_t n, const float* codes, bool faiss = false, bool lite = false) {
    if (faiss) throw std::runtime_error("faiss training is not part of harmony_b200");
    check(hb_train(h_, n, codes, lite ? 1 : 0));
  }
  void add(size_t n, const float* codes) { check(hb_add(h_, n, codes)); }

  void preSearch(size_t /*nb*/, size_t workerCount, size_t blockCount, size_t warmUpSearchList,
                 size_t warmUpSearchListSize, Param* p, std::string /*path*/ = "") {
    param = p;
    this->workerCount = workerCount;
    this->blockCount = blockCount;
    this->warmUpSearchList = warmUpSearchList;
    this->warmUpSearchListSize = warmUpSearchListSize;
  }
  void postSearch() {}

  // Without preSearch the reference leaves `param` unset and only initialises
  // the results (src/Index.cpp:1652-1654); so does this wrapper.
  Stats search(size_t n, const float* queries, size_t k, float* distances, idx_t* labels, float /*ratio*/ = 1) {
    if (n == 0) return Stats();
    check(hb_set_nprobe(h_, nprobe));
    hb_search_params sp;
    hb_search_params_init(&sp);
    if (!param) {
      sp.mode = HB_MODE_ORIGINAL;
      sp.learned_probe = 0;
      size_t zero = 0;
      check(hb_set_nprobe(h_, zero));
    } else {
      sp.mode = static_cast<int32_t>(param->mode);
      sp.pruning = param->pruning;
      sp.order_optimize = param->orderOptimize;
      sp.period = param->period;
      sp.n_dim_blocks = static_cast<int32_t>(workerCount ? workerCount : 1);
      sp.n_query_blocks = static_cast<int32_t>(blockCount ? blockCount : 1);
      if (warmUpSearchList) sp.warmup_lists = static_cast<int32_t>(warmUpSearchList);
      sp.warmup_list_size = static_cast<int32_t>(warmUpSearchListSize);
      sp.full_warmup = param->fullWarmUp ? 1 : 0;
      sp.heap_tops = param->heapTops;
    }
    check(hb_search(h_, n, queries, k, &sp, distances, labels));
    size_t np = 0;
    check(hb_get_nprobe(h_, &np));
    if (param) nprobe = np;  // search clamps nprobe to nlist (src/Index.cpp:1646-1648)
    else check(hb_set_nprobe(h_, nprobe));
    return Stats();
  }

  void save_index(std::string path) const { check(hb_save_index(h_, path.c_str())); }
  void load_index(std::string path) {
    check(hb_load_index(h_, path.c_str()));
    int m = 0;
    check(hb_get_info(h_, &d, &nlist, nullptr, &m));
    metric = static_cast<MetricType>(m);
    opt_level = OPT_NONE;  // src/Index.cpp:1744
  }

  // Public fields of the reference's Index that drivers read or mutate.
  size_t d, nlist, nprobe;
  MetricType metric;
  OptLevel opt_level;
  size_t sub_k, sub_nlist, sub_nprobe;
  bool verbose;
  EdgeDevice edge_device_enabled;
  size_t workerCount = 0, blockCount = 0, warmUpSearchList = 0, warmUpSearchListSize = 0;
  Param* param = nullptr;

  hb_index* handle() const { return h_; }

 private:
  static void check(int rc) {
    if (rc != HB_OK) throw std::runtime_error(std::string("harmony_b200: ") + hb_last_error());
  }
  hb_index* h_ = nullptr;
};

}  // namespace harmony

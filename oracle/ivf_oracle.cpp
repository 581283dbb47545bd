// CPU restatement of the reference's IVF-flat algorithm (see ivf_oracle.h).
// TEST INFRASTRUCTURE ONLY: the checker for the CUDA path, never the product.
// Compiled with -ffp-contract=off so every a*b+c below rounds twice, as the
// reference's distance loop does (src/utils.h:480-487).
#include "ivf_oracle.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>

namespace {
// Fresh sequential sum over dims [0, n): src/utils.h:480-487.
inline float seq_l2(const float* a, const float* b, size_t n) {
  float acc = 0.0f;
  for (size_t i = 0; i < n; ++i) {
    float t = a[i] - b[i];
    float sq = t * t;
    acc = acc + sq;
  }
  return acc;
}
}  // namespace

extern "C" {

float orc_l2(const float* a, const float* b, size_t d) { return seq_l2(a, b, d); }

// src/heap.hpp:13-25 (L2 branch).
void orc_heap_init(size_t k, float* val, int64_t* ids) {
  for (size_t i = 0; i < k; ++i) {
    val[i] = FLT_MAX;
    ids[i] = -1;
  }
}

// Sift-down replacing the root of a 1-based max-heap: src/heap.hpp:35-71.
void orc_heap_replace_top(size_t k, float* val, int64_t* ids, float v, int64_t id) {
  float* hv = val - 1;
  int64_t* hi = ids - 1;
  size_t i = 1;
  for (;;) {
    size_t c1 = 2 * i, c2 = c1 + 1;
    if (c1 > k) break;
    size_t c = (c2 == k + 1 || hv[c1] > hv[c2]) ? c1 : c2;
    if (v > hv[c]) break;
    hv[i] = hv[c];
    hi[i] = hi[c];
    i = c;
  }
  hv[i] = v;
  hi[i] = id;
}

// In-place heap sort to ascending order: src/heap.hpp:73-82.
void orc_heap_sort(size_t k, float* val, int64_t* ids) {
  for (int64_t i = static_cast<int64_t>(k) - 1; i >= 0; --i) {
    float v = val[i];
    int64_t id = ids[i];
    val[i] = val[0];
    ids[i] = ids[0];
    orc_heap_replace_top(static_cast<size_t>(i), val, ids, v, id);
  }
}

void orc_heap_topk(size_t n, const float* vals, size_t k, float* D, int64_t* I) {
  orc_heap_init(k, D, I);
  for (size_t i = 0; i < n; ++i)
    if (vals[i] < D[0]) orc_heap_replace_top(k, D, I, vals[i], static_cast<int64_t>(i));
  orc_heap_sort(k, D, I);
}

// lite_scan_codes over the centroids with a heap of nprobe, then sort_result
// (src/IVFScan.hpp:108-138; src/Index.cpp:1440-1448).
void orc_coarse(size_t nq, const float* q, size_t d, size_t nlist, const float* cent,
                size_t nprobe, float* cd, int64_t* cl) {
#pragma omp parallel for schedule(dynamic, 16)
  for (size_t i = 0; i < nq; ++i) {
    float* hv = cd + i * nprobe;
    int64_t* hi = cl + i * nprobe;
    orc_heap_init(nprobe, hv, hi);
    for (size_t c = 0; c < nlist; ++c) {
      float dis = seq_l2(q + i * d, cent + c * d, d);
      if (dis < hv[0]) orc_heap_replace_top(nprobe, hv, hi, dis, static_cast<int64_t>(c));
    }
    orc_heap_sort(nprobe, hv, hi);
  }
}

// scan_codes over each probed list in probe order (src/IVFScan.hpp:240-288).
void orc_search_probes(size_t nq, const float* q, size_t d, const int64_t* list_off,
                       const int64_t* ids, const float* codes, size_t nprobe,
                       const int64_t* probes, size_t k, float* D, int64_t* I) {
#pragma omp parallel for schedule(dynamic, 4)
  for (size_t i = 0; i < nq; ++i) {
    float* hv = D + i * k;
    int64_t* hi = I + i * k;
    orc_heap_init(k, hv, hi);
    for (size_t j = 0; j < nprobe; ++j) {
      int64_t l = probes[i * nprobe + j];
      if (l < 0) continue;
      for (int64_t v = list_off[l]; v < list_off[l + 1]; ++v) {
        float dis = seq_l2(q + i * d, codes + static_cast<size_t>(v) * d, d);
        if (dis < hv[0]) orc_heap_replace_top(k, hv, hi, dis, ids[v]);
      }
    }
    orc_heap_sort(k, hv, hi);
  }
}

// Index::search in ORIGINAL mode: nprobe is clamped to nlist
// (src/Index.cpp:1646-1648), then per query coarse + scan + sort.
void orc_search(size_t nq, const float* q, size_t d, size_t nlist, const float* cent,
                const int64_t* list_off, const int64_t* ids, const float* codes,
                size_t nprobe, size_t k, float* D, int64_t* I) {
  if (nprobe > nlist) nprobe = nlist;
  std::vector<float> cd(nq * nprobe);
  std::vector<int64_t> cl(nq * nprobe);
  orc_coarse(nq, q, d, nlist, cent, nprobe, cd.data(), cl.data());
  orc_search_probes(nq, q, d, list_off, ids, codes, nprobe, cl.data(), k, D, I);
}

// Index::warmUpSearch: the first warm_list_size vectors of the first
// warm_lists probed lists fill a k-heap; its top is the threshold.
// warm_lists is clamped to nprobe (src/Index.cpp:1008-1011).
void orc_warmup_tops(size_t nq, const float* q, size_t d, const int64_t* list_off,
                     const int64_t* ids, const float* codes, size_t nprobe,
                     const int64_t* probes, size_t k, size_t warm_lists,
                     size_t warm_list_size, float* tops) {
  if (warm_lists > nprobe) warm_lists = nprobe;
#pragma omp parallel for schedule(dynamic, 16)
  for (size_t i = 0; i < nq; ++i) {
    std::vector<float> hv(k);
    std::vector<int64_t> hi(k);
    orc_heap_init(k, hv.data(), hi.data());
    for (size_t j = 0; j < warm_lists; ++j) {
      int64_t l = probes[i * nprobe + j];
      int64_t n = list_off[l + 1] - list_off[l];
      int64_t m = std::min<int64_t>(n, static_cast<int64_t>(warm_list_size));
      for (int64_t v = list_off[l]; v < list_off[l] + m; ++v) {
        float dis = seq_l2(q + i * d, codes + static_cast<size_t>(v) * d, d);
        if (dis < hv[0]) orc_heap_replace_top(k, hv.data(), hi.data(), dis, ids[v]);
      }
    }
    tops[i] = hv[0];
  }
}

// BaseWorker::single_thread_search_simple (src/node.cpp:606-678): distance in
// 4 chunks of d/4 dims (last chunk takes the rest), each chunk a fresh
// sequential sum added to the running total; after each of the first three
// chunks the candidate is abandoned when the total exceeds the query's heap
// top.  The result heap is sorted at the end, as the master's merge does.
void orc_search_pruned(size_t nq, const float* q, size_t d, const int64_t* list_off,
                       const int64_t* ids, const float* codes, size_t nprobe,
                       const int64_t* probes, const float* tops, int cut, size_t k,
                       float* D, int64_t* I) {
  const size_t nchk = 4, cd = d / nchk;
#pragma omp parallel for schedule(dynamic, 4)
  for (size_t i = 0; i < nq; ++i) {
    float* hv = D + i * k;
    int64_t* hi = I + i * k;
    const float* qi = q + i * d;
    orc_heap_init(k, hv, hi);
    for (size_t j = 0; j < nprobe; ++j) {
      int64_t l = probes[i * nprobe + j];
      if (l < 0) continue;
      for (int64_t v = list_off[l]; v < list_off[l + 1]; ++v) {
        const float* x = codes + static_cast<size_t>(v) * d;
        float dis = 0.0f;
        if (cut) {
          for (size_t c = 0; c < nchk; ++c) {
            if (c == nchk - 1) {
              dis = dis + seq_l2(qi + cd * c, x + cd * c, d - c * cd);
            } else {
              dis = dis + seq_l2(qi + cd * c, x + cd * c, cd);
              if (dis > tops[i]) {
                dis = INFINITY;
                break;
              }
            }
          }
        } else {
          dis = seq_l2(qi, x, d);
        }
        if (dis < hv[0]) orc_heap_replace_top(k, hv, hi, dis, ids[v]);
      }
    }
    orc_heap_sort(k, hv, hi);
  }
}

// Worker::searchBlock relay (src/node.cpp:326-381) collapsed onto one host:
// for query block b the slices are added in order[b*W ..], each slice a fresh
// sequential sum over its d/W dims.  With cut, a running total above the
// query's heap top becomes INFINITY and later slices skip it; only the last
// slice's worker admits candidates into the heap (shouldSendHeap,
// src/node.h:338-340).
void orc_search_dimblock(size_t nq, const float* q, size_t d, const int64_t* list_off,
                         const int64_t* ids, const float* codes, size_t nprobe,
                         const int64_t* probes, const float* tops, int cut, size_t W,
                         size_t B, const int64_t* order, size_t k, float* D, int64_t* I) {
  const size_t bd = d / W;
  const size_t bs = B ? nq / B : 0;
  for (size_t i = 0; i < nq; ++i) orc_heap_init(k, D + i * k, I + i * k);
#pragma omp parallel for schedule(dynamic, 4)
  for (size_t i = 0; i < B * bs; ++i) {
    const size_t b = i / bs;
    float* hv = D + i * k;
    int64_t* hi = I + i * k;
    const float* qi = q + i * d;
    for (size_t j = 0; j < nprobe; ++j) {
      int64_t l = probes[i * nprobe + j];
      for (int64_t v = list_off[l]; v < list_off[l + 1]; ++v) {
        const float* x = codes + static_cast<size_t>(v) * d;
        float buf = 0.0f;
        for (size_t t = 0; t < W; ++t) {
          const size_t s = static_cast<size_t>(order[b * W + t]);
          const bool last = (t == W - 1);
          if (cut && buf == INFINITY) continue;
          buf = buf + seq_l2(qi + s * bd, x + s * bd, bd);
          if (cut && buf > tops[i]) {
            buf = INFINITY;
          } else if (last && buf < hv[0]) {
            orc_heap_replace_top(k, hv, hi, buf, ids[v]);
          }
        }
      }
    }
    orc_heap_sort(k, hv, hi);
  }
}

void orc_block_order(size_t W, size_t B, int order_optimize, int period, int64_t* order) {
  // wsbo[r][t] = block that worker r (1-based) processes at step t.
  std::vector<std::vector<int64_t>> wsbo(W + 1, std::vector<int64_t>(B, 0));
  if (order_optimize) {
    if (period && B % W == 0) {
      const size_t layer = B / W;
      for (size_t p = 1; p <= W; ++p)
        for (size_t t = (p - 1) * layer; t < p * layer; ++t) {
          const size_t start = (t % layer) * W;
          for (size_t r = p; r < p + W; ++r) wsbo[(r + W - 1) % W + 1][t] = start + r - p;
        }
    } else {
      const size_t gap = (B + W - 1) / W;
      for (size_t r = 1; r <= W; ++r)
        for (size_t blk = 0; blk < B; ++blk) wsbo[r][(blk + gap * (r - 1)) % B] = blk;
    }
  } else {
    for (size_t r = 1; r <= W; ++r)
      for (size_t t = r - 1; t < r - 1 + B; ++t) wsbo[r][t % B] = t - (r - 1);
  }
  // Workers of each block in visiting order (src/order.h:72-77).
  std::vector<std::vector<int64_t>> seq(B);
  for (size_t t = 0; t < B; ++t)
    for (size_t r = 1; r <= W; ++r) seq[wsbo[r][t]].push_back(static_cast<int64_t>(r) - 1);
  for (size_t b = 0; b < B; ++b)
    for (size_t t = 0; t < W; ++t) order[b * W + t] = t < seq[b].size() ? seq[b][t] : -1;
}

void orc_kmeans_indices(size_t n, size_t nlist, int seed, size_t max_pts, int64_t* sample_idx,
                        int64_t* init_idx) {
  size_t m = n;
  std::vector<size_t> sidx(n);
  std::iota(sidx.begin(), sidx.end(), 0);
  if (n > nlist * max_pts) {
    std::shuffle(sidx.begin(), sidx.end(), std::default_random_engine(seed));
    m = nlist * max_pts;
  }
  for (size_t i = 0; i < m; ++i) sample_idx[i] = static_cast<int64_t>(sidx[i]);
  std::vector<size_t> iidx(m);
  std::iota(iidx.begin(), iidx.end(), 0);
  std::shuffle(iidx.begin(), iidx.end(), std::default_random_engine(seed));
  for (size_t i = 0; i < nlist; ++i) init_idx[i] = static_cast<int64_t>(iidx[i]);
}

void orc_kmeans(size_t n, const float* x, size_t d, size_t nlist, int niter, int seed,
                size_t max_pts, float* cent_out) {
  const size_t m = std::min(n, nlist * max_pts);
  std::vector<int64_t> sidx(m), iidx(nlist);
  orc_kmeans_indices(n, nlist, seed, max_pts, sidx.data(), iidx.data());
  std::vector<float> s(m * d);
  for (size_t i = 0; i < m; ++i) std::memcpy(&s[i * d], x + sidx[i] * d, d * sizeof(float));
  for (size_t c = 0; c < nlist; ++c) std::memcpy(cent_out + c * d, &s[iidx[c] * d], d * sizeof(float));
  std::vector<size_t> assign(m);
  std::vector<float> sums(nlist * d);
  std::vector<size_t> counts(nlist);
  for (int it = 0; it < niter; ++it) {
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < m; ++i) {
      size_t best = 0;
      float bd = FLT_MAX;
      for (size_t c = 0; c < nlist; ++c) {
        float dis = seq_l2(cent_out + c * d, &s[i * d], d);
        if (dis < bd) {
          bd = dis;
          best = c;
        }
      }
      assign[i] = best;
    }
    std::fill(sums.begin(), sums.end(), 0.0f);
    std::fill(counts.begin(), counts.end(), 0);
    for (size_t i = 0; i < m; ++i) {
      counts[assign[i]]++;
      for (size_t j = 0; j < d; ++j) sums[assign[i] * d + j] += s[i * d + j];
    }
    for (size_t c = 0; c < nlist; ++c)
      if (counts[c] > 0)
        for (size_t j = 0; j < d; ++j)
          cent_out[c * d + j] = sums[c * d + j] / static_cast<float>(counts[c]);
  }
}

void orc_add(size_t n, const float* x, size_t d, size_t nlist, const float* cent,
             int64_t* list_off, int64_t* ids, float* codes, float* norms) {
  std::vector<float> cdist(n);
  std::vector<int64_t> clist(n);
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < n; ++i) {
    float bd = FLT_MAX;
    int64_t best = -1;
    for (size_t c = 0; c < nlist; ++c) {
      float dis = seq_l2(x + i * d, cent + c * d, d);
      if (dis < bd) {
        bd = dis;
        best = static_cast<int64_t>(c);
      }
    }
    cdist[i] = bd;
    clist[i] = best;
  }
  std::vector<int64_t> cnt(nlist + 1, 0);
  for (size_t i = 0; i < n; ++i) cnt[clist[i] + 1]++;
  for (size_t c = 0; c < nlist; ++c) cnt[c + 1] += cnt[c];
  std::memcpy(list_off, cnt.data(), sizeof(int64_t) * (nlist + 1));
  std::vector<size_t> ord(n);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](size_t a, size_t b) { return cdist[a] < cdist[b]; });
  std::vector<int64_t> fill(cnt.begin(), cnt.end() - 1);
  for (size_t oi = 0; oi < n; ++oi) {
    size_t i = ord[oi];
    int64_t pos = fill[clist[i]]++;
    ids[pos] = static_cast<int64_t>(i);
    std::memcpy(codes + static_cast<size_t>(pos) * d, x + i * d, d * sizeof(float));
  }
  // Norms are <x,x> with the sequential inner-product loop (src/Index.cpp:689-696,
  // src/utils.h:511-518).
  for (size_t v = 0; v < n; ++v) {
    const float* r = codes + v * d;
    float acc = 0.0f;
    for (size_t j = 0; j < d; ++j) {
      float p = r[j] * r[j];
      acc = acc + p;
    }
    norms[v] = acc;
  }
}

void orc_bruteforce_f64(size_t nq, const float* q, size_t nb, const float* x, size_t d,
                        size_t k, double* D, int64_t* I) {
#pragma omp parallel for schedule(dynamic, 1)
  for (size_t i = 0; i < nq; ++i) {
    std::vector<std::pair<double, int64_t>> v(nb);
    for (size_t b = 0; b < nb; ++b) {
      double acc = 0.0;
      for (size_t j = 0; j < d; ++j) {
        double t = static_cast<double>(q[i * d + j]) - static_cast<double>(x[b * d + j]);
        acc += t * t;
      }
      v[b] = {acc, static_cast<int64_t>(b)};
    }
    size_t kk = std::min(k, nb);
    std::partial_sort(v.begin(), v.begin() + kk, v.end());
    for (size_t j = 0; j < k; ++j) {
      D[i * k + j] = j < kk ? v[j].first : INFINITY;
      I[i * k + j] = j < kk ? v[j].second : -1;
    }
  }
}

}  // extern "C"

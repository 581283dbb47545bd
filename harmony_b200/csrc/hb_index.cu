// Host side of the B200 IVF-flat index and its C ABI (include/harmony_b200.h).
//
// The index mirrors harmony::Index (src/Index.h:13-149): centroids, nlist
// inverted lists of (id, code, norm), nprobe, train / add / search /
// save_index / load_index.  Everything it owns lives in device memory:
//
//   centroids  float [nlist x dpad]          (rows zero-padded to dpad)
//   list_off   int64 [nlist + 1]             CSR offsets of the lists
//   codes      float [ntotal x dpad]         vectors in list order
//   ids        int64 [ntotal]                ids in list order
//   norms      float [ntotal]                <x, x> (the reference stores them too)
//
// Search runs per batch of queries, all on the index's stream:
//   pad queries -> exact coarse distance matrix -> per-query top-nprobe
//   -> [warm-up heap tops] -> list-major work description -> persistent
//   exact list scan -> per-query merge of the partial top-k slots.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cstdio>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <random>
#include <string>
#include <tuple>
#include <vector>

#include "hb_internal.hpp"

namespace hb {

namespace {
thread_local std::string g_last_error;

bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int pow2_floor(long long x) {
  int p = 1;
  while (static_cast<long long>(p) * 2 <= x && p < (1 << 30)) p <<= 1;
  return p;
}
}  // namespace

// Order of the dimension slices for each query block in the
// dimension-partition mode: src/order.h:38-96 and the "period" variant of
// src/Index.cpp:183-197.  order[b * W + t] = slice visited at hop t.
std::vector<int32_t> block_visit_order(int W, int B, bool order_optimize, bool period) {
  std::vector<std::vector<int>> wsbo(W + 1, std::vector<int>(B, 0));
  if (order_optimize) {
    if (period && B % W == 0) {
      const int layer = B / W;
      for (int p = 1; p <= W; ++p)
        for (int t = (p - 1) * layer; t < p * layer; ++t) {
          const int start = (t % layer) * W;
          for (int r = p; r < p + W; ++r) wsbo[(r + W - 1) % W + 1][t] = start + r - p;
        }
    } else {
      const int gap = (B + W - 1) / W;
      for (int r = 1; r <= W; ++r)
        for (int blk = 0; blk < B; ++blk) wsbo[r][(blk + gap * (r - 1)) % B] = blk;
    }
  } else {
    for (int r = 1; r <= W; ++r)
      for (int t = r - 1; t < r - 1 + B; ++t) wsbo[r][t % B] = t - (r - 1);
  }
  std::vector<std::vector<int>> seq(B);
  for (int t = 0; t < B; ++t)
    for (int r = 1; r <= W; ++r) seq[wsbo[r][t]].push_back(r - 1);
  std::vector<int32_t> order(static_cast<size_t>(B) * W, -1);
  for (int b = 0; b < B; ++b)
    for (int t = 0; t < W && t < static_cast<int>(seq[b].size()); ++t) order[static_cast<size_t>(b) * W + t] = seq[b][t];
  return order;
}

// Per-kernel timing with CUDA events on the index's stream (enabled by
// hb_profile_enable; read and cleared by hb_profile_read).
struct ProfRecord {
  const char* name;
  cudaEvent_t a, b;
};

class IndexCore {
 public:
  IndexCore(size_t d, size_t nlist, size_t nprobe, int metric, int device)
      : d_(d), nlist_(nlist), nprobe_(nprobe), metric_(metric), device_(device) {
    HB_CHECK(metric == HB_METRIC_L2, HB_ERR_INVALID, "only METRIC_L2 is implemented");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      cudaGetLastError();
      throw Error(HB_ERR_NODEVICE, "no CUDA device");
    }
    HB_CHECK(device >= 0 && device < ndev, HB_ERR_INVALID, "bad device ordinal");
    HB_CUDA(cudaSetDevice(device));
    HB_CUDA(cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, device));
    HB_CUDA(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    HB_CUDA(cudaMallocHost(&err_host_, sizeof(int)));
    reshape(d, nlist);
  }
  ~IndexCore() {
    cudaSetDevice(device_);
    drop_graphs();
    if (st_) {
      cudaStreamSynchronize(st_);
      cudaStreamDestroy(st_);
    }
    if (err_host_) cudaFreeHost(err_host_);
  }

  // Index ctor state: zero centroids, empty lists (src/Index.cpp:24-43).
  void reshape(size_t d, size_t nlist) {
    HB_CHECK(d > 0 && d <= 1024, HB_ERR_INVALID, "d must be in [1, 1024]");
    HB_CHECK(nlist > 0 && nlist <= (1u << 20), HB_ERR_INVALID, "nlist must be in [1, 2^20]");
    d_ = d;
    nlist_ = nlist;
    dpad_ = pad_dim(d);
    cent_.reserve(nlist_ * dpad_);
    HB_CUDA(cudaMemsetAsync(cent_.p, 0, nlist_ * dpad_ * sizeof(float), st_));
    list_off_.reserve(nlist_ + 1);
    HB_CUDA(cudaMemsetAsync(list_off_.p, 0, (nlist_ + 1) * sizeof(int64_t), st_));
    host_off_.assign(nlist_ + 1, 0);
    ntotal_ = 0;
    coarse_ready_ = false;
    coarse_last_nq_ = 0;
    drop_graphs();
    HB_CUDA(cudaStreamSynchronize(st_));
  }

  size_t d() const { return d_; }
  size_t nlist() const { return nlist_; }
  size_t ntotal() const { return ntotal_; }
  size_t nprobe() const { return nprobe_; }
  void set_nprobe(size_t p) { nprobe_ = p; }
  int metric() const { return metric_; }
  cudaStream_t stream() const { return st_; }
  uint64_t launches() const { return launches_; }

  // ---- profiling -------------------------------------------------------------
  struct Scope {
    IndexCore* ix;
    const char* name;
    cudaEvent_t a = nullptr;
    Scope(IndexCore* i, const char* n) : ix(i), name(n) {
      if (ix->prof_ && !ix->capturing_) {
        a = ix->event();
        cudaEventRecord(a, ix->st_);
      }
    }
    ~Scope() {
      if (a) {
        cudaEvent_t b = ix->event();
        cudaEventRecord(b, ix->st_);
        ix->prof_log_.push_back({name, a, b});
      }
    }
  };
  cudaEvent_t event() {
    if (!ev_pool_.empty()) {
      cudaEvent_t e = ev_pool_.back();
      ev_pool_.pop_back();
      return e;
    }
    cudaEvent_t e;
    HB_CUDA(cudaEventCreate(&e));
    return e;
  }
  void profile_enable(bool on) { prof_ = on; }
  // Sums of the recorded intervals per name (ms) and their counts.
  int profile_read(char* names, size_t names_len, double* ms, int64_t* counts, int max_entries) {
    HB_CUDA(cudaStreamSynchronize(st_));
    std::vector<std::string> keys;
    std::vector<double> tot;
    std::vector<int64_t> cnt;
    for (auto& r : prof_log_) {
      float t = 0.f;
      HB_CUDA(cudaEventElapsedTime(&t, r.a, r.b));
      size_t i = 0;
      for (; i < keys.size(); ++i)
        if (keys[i] == r.name) break;
      if (i == keys.size()) {
        keys.push_back(r.name);
        tot.push_back(0.0);
        cnt.push_back(0);
      }
      tot[i] += t;
      cnt[i] += 1;
      ev_pool_.push_back(r.a);
      ev_pool_.push_back(r.b);
    }
    prof_log_.clear();
    std::string joined;
    for (size_t i = 0; i < keys.size(); ++i) {
      if (static_cast<int>(i) < max_entries) {
        if (ms) ms[i] = tot[i];
        if (counts) counts[i] = cnt[i];
      }
      joined += keys[i];
      joined += '\n';
    }
    if (names && names_len) {
      std::strncpy(names, joined.c_str(), names_len - 1);
      names[names_len - 1] = 0;
    }
    return static_cast<int>(keys.size());
  }

  // ---- input staging -------------------------------------------------------

  // Copies n x d floats (host or device) to a padded device buffer.
  void stage_rows(const float* x, size_t n, DevBuf<float>& dst, DevBuf<float>& tmp) {
    dst.reserve(std::max<size_t>(n * dpad_, 1));
    if (!n) return;
    const float* src = x;
    if (!is_device_ptr(x)) {
      tmp.reserve(n * d_);
      HB_CUDA(cudaMemcpyAsync(tmp.p, x, n * d_ * sizeof(float), cudaMemcpyHostToDevice, st_));
      src = tmp.p;
    }
    launch_pad_rows(src, n, static_cast<int>(d_), static_cast<int>(dpad_), dst.p, st_);
    ++launches_;
  }

  // ---- train: src/Index.cpp:381-425 + src/Clustering.cpp:14-152 ------------

  void train(size_t n, const float* x, bool lite) {
    HB_CHECK(x || n == 0, HB_ERR_INVALID, "null training data");
    HB_CHECK(n >= nlist_, HB_ERR_INVALID, "train needs at least nlist points");
    HB_CHECK(n < (1ull << 31), HB_ERR_INVALID, "train supports fewer than 2^31 points");
    HB_CUDA(cudaSetDevice(device_));
    const int niter = lite ? 2 : 20;
    const int seed = 6666;
    const size_t max_pts = 256;
    // Sampling draws exactly as the reference: std::shuffle with
    // std::default_random_engine(seed) over the point indices, the first
    // nlist*max_pts when n exceeds it, then a second shuffle over the
    // sample whose first nlist entries seed the centroids.
    size_t m = n;
    std::vector<int64_t> sample;
    if (n > nlist_ * max_pts) {
      std::vector<size_t> idx(n);
      std::iota(idx.begin(), idx.end(), 0);
      std::shuffle(idx.begin(), idx.end(), std::default_random_engine(seed));
      m = nlist_ * max_pts;
      sample.assign(idx.begin(), idx.begin() + m);
    }
    std::vector<size_t> iidx(m);
    std::iota(iidx.begin(), iidx.end(), 0);
    std::shuffle(iidx.begin(), iidx.end(), std::default_random_engine(seed));
    std::vector<int64_t> init(nlist_);
    for (size_t c = 0; c < nlist_; ++c) init[c] = static_cast<int64_t>(iidx[c]);

    DevBuf<float> xall, tmp, xs;
    stage_rows(x, n, xall, tmp);
    tmp.release();
    const float* pts = xall.p;
    if (!sample.empty()) {
      DevBuf<int64_t> sidx;
      sidx.reserve(m);
      HB_CUDA(cudaMemcpyAsync(sidx.p, sample.data(), m * sizeof(int64_t), cudaMemcpyHostToDevice, st_));
      xs.reserve(m * dpad_);
      launch_gather_rows(xall.p, sidx.p, m, static_cast<int>(dpad_), xs.p, st_);
      ++launches_;
      HB_CUDA(cudaStreamSynchronize(st_));
      xall.release();
      pts = xs.p;
    }
    {
      DevBuf<int64_t> cidx;
      cidx.reserve(nlist_);
      HB_CUDA(cudaMemcpyAsync(cidx.p, init.data(), nlist_ * sizeof(int64_t), cudaMemcpyHostToDevice, st_));
      launch_gather_rows(pts, cidx.p, nlist_, static_cast<int>(dpad_), cent_.p, st_);
      ++launches_;
      HB_CUDA(cudaStreamSynchronize(st_));
    }
    DevBuf<int32_t> assign, counts;
    DevBuf<double> sums;
    assign.reserve(m);
    counts.reserve(nlist_);
    sums.reserve(nlist_ * dpad_);
    for (int it = 0; it < niter; ++it) {
      launch_l2_argmin(pts, static_cast<int>(m), cent_.p, static_cast<int>(nlist_), static_cast<int>(dpad_), assign.p,
                       nullptr, st_);
      HB_CUDA(cudaMemsetAsync(sums.p, 0, nlist_ * dpad_ * sizeof(double), st_));
      HB_CUDA(cudaMemsetAsync(counts.p, 0, nlist_ * sizeof(int32_t), st_));
      launch_kmeans_accumulate(pts, assign.p, m, static_cast<int>(d_), static_cast<int>(dpad_), sums.p, counts.p,
                               st_);
      launch_kmeans_update(sums.p, counts.p, static_cast<int>(nlist_), static_cast<int>(d_), static_cast<int>(dpad_),
                           cent_.p, st_);
      launches_ += 3;
    }
    HB_CUDA(cudaStreamSynchronize(st_));
    trained_ = true;
    coarse_ready_ = false;
    drop_graphs();
  }

  // ---- add: src/Index.cpp:581-698 ------------------------------------------

  void add(size_t n, const float* x) {
    if (n == 0) return;  // the reference returns before touching the lists
    HB_CHECK(x, HB_ERR_INVALID, "null data");
    HB_CHECK(n < (1ull << 32) - 1, HB_ERR_INVALID, "add supports fewer than 2^32 - 1 vectors");
    HB_CUDA(cudaSetDevice(device_));
    DevBuf<float> xpad, tmp;
    stage_rows(x, n, xpad, tmp);
    tmp.release();
    DevBuf<int32_t> assign;
    DevBuf<float> dist;
    assign.reserve(n);
    dist.reserve(n);
    launch_l2_argmin(xpad.p, static_cast<int>(n), cent_.p, static_cast<int>(nlist_), static_cast<int>(dpad_), assign.p,
                     dist.p, st_);
    DevBuf<uint64_t> k0, k1;
    DevBuf<uint32_t> v0, v1;
    k0.reserve(n);
    k1.reserve(n);
    v0.reserve(n);
    v1.reserve(n);
    launch_add_keys(assign.p, dist.p, n, k0.p, v0.p, st_);
    int list_bits = 1;
    while ((1ull << list_bits) < nlist_) ++list_bits;
    size_t sort_bytes = 0;
    sort_pairs_u64(k0.p, k1.p, v0.p, v1.p, n, 32 + list_bits, nullptr, &sort_bytes, st_);
    DevBuf<unsigned char> sort_tmp;
    sort_tmp.reserve(sort_bytes);
    sort_pairs_u64(k0.p, k1.p, v0.p, v1.p, n, 32 + list_bits, sort_tmp.p, &sort_bytes, st_);
    codes_.reserve(n * dpad_);
    ids_.reserve(n);
    norms_.reserve(n);
    launch_scatter_sorted(xpad.p, v1.p, n, static_cast<int>(d_), static_cast<int>(dpad_), codes_.p, ids_.p, st_);
    const size_t ob = list_offsets_tmp_bytes(static_cast<int>(nlist_));
    DevBuf<unsigned char> otmp;
    otmp.reserve(ob);
    launch_list_offsets(assign.p, n, static_cast<int>(nlist_), list_off_.p, otmp.p, ob, st_);
    launch_row_norms(codes_.p, n, static_cast<int>(d_), static_cast<int>(dpad_), norms_.p, st_);
    launches_ += 6;
    host_off_.resize(nlist_ + 1);
    HB_CUDA(cudaMemcpyAsync(host_off_.data(), list_off_.p, (nlist_ + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost,
                            st_));
    HB_CUDA(cudaStreamSynchronize(st_));
    ntotal_ = n;
    plan_rows_ = 0;
    build_bf16();
    drop_graphs();
  }

  // BF16 copy of the codes (rows padded to kpad = d rounded up to 64) and its
  // TMA tensor map, for the tensor-core scans (the heap scan takes d <= 128,
  // the candidate-matrix scan any d).
  // E4M3 copy of the codes for the FP8 candidate scan (rows padded to kpad8
  // = d rounded up to 128 bytes) with a per-list scale, built on the first
  // FP8 search after the lists change.
  void ensure_fp8() {
    if (fp8_ready_) return;
    kpad8_ = static_cast<int>((d_ + 127) / 128 * 128);
    codes8_.reserve(std::max<size_t>(ntotal_ * static_cast<size_t>(kpad8_), 1));
    list_scale8_.reserve(nlist_);
    rnorm8_.reserve(std::max<size_t>(ntotal_, 1));
    launch_fp8_codes(codes_.p, list_off_.p, cent_.p, static_cast<int>(nlist_), static_cast<int>(dpad_), kpad8_,
                     codes8_.p, list_scale8_.p, rnorm8_.p, st_);
    tile_rnorm8_.reserve(std::max<size_t>(tile_norm_.n, 1));
    launch_tile_norms(rnorm8_.p, list_off_.p, static_cast<int>(nlist_), tile_off_.p, tile_rnorm8_.p, st_);
    launches_ += 2;
    make_u8_tensor_map(tmap8_, codes8_.p, std::max<size_t>(ntotal_, 1), kpad8_);
    HB_CUDA(cudaStreamSynchronize(st_));
    fp8_ready_ = true;
  }

  void build_bf16() {
    bf16_ready_ = false;
    fp8_ready_ = false;
    kpad_ = static_cast<int>((d_ + 63) / 64 * 64);
    if (ntotal_ == 0) return;
    // Residuals to the list centroids: BF16(x - c_l), their FP32 norms and
    // each list's largest residual norm (the scans' error bound uses it).
    codes_bf16_.reserve(ntotal_ * static_cast<size_t>(kpad_));
    rnorm_.reserve(ntotal_);
    rmax_.reserve(nlist_);
    launch_residual_bf16(codes_.p, list_off_.p, cent_.p, static_cast<int>(nlist_), static_cast<int>(dpad_), kpad_,
                         codes_bf16_.p, rnorm_.p, rmax_.p, st_);
    ++launches_;
    make_bf16_tensor_map(tmap_, codes_bf16_.p, ntotal_, kpad_);
    // Residual norms in 128-row tiles per list (+inf past each list's end),
    // copied next to each accumulator by the scan.
    std::vector<int64_t> toff(nlist_ + 1, 0);
    for (size_t l = 0; l < nlist_; ++l) toff[l + 1] = toff[l] + (host_off_[l + 1] - host_off_[l] + 127) / 128;
    tile_off_.reserve(nlist_ + 1);
    HB_CUDA(cudaMemcpyAsync(tile_off_.p, toff.data(), toff.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st_));
    tile_norm_.reserve(std::max<size_t>(static_cast<size_t>(toff[nlist_]) * 128, 1));
    launch_tile_norms(rnorm_.p, list_off_.p, static_cast<int>(nlist_), tile_off_.p, tile_norm_.p, st_);
    launches_ += 2;
    HB_CUDA(cudaStreamSynchronize(st_));
    bf16_ready_ = true;
  }

  // ---- coarse quantizer ----------------------------------------------------

  // probes_out (device, nq x P int32, ascending), cdist_out optional.
  // Coarse quantizer (src/IVFScan.hpp:108-138, src/Index.cpp:1440-1448):
  // probes_out (nq x P) = the P nearest centroids of each query by the
  // reference's sequential FP32 distance, ascending, ties by lower centroid.
  // For d <= 128 the tensor cores pick P + m candidates (3-term BF16 split),
  // which are re-ranked exactly; a query whose candidate set cannot be
  // proven to contain the exact top P is recomputed exactly.  Both routes
  // give the same rows.
  void coarse(const float* qpad, int nq, int P, int32_t* probes_out, float* cdist_out) {
    dmat_.reserve(static_cast<size_t>(nq) * nlist_);
    const int Pm = std::min<int>(static_cast<int>(nlist_), P + coarse_extra(P));
    const bool tc = coarse_kind_ != HB_COARSE_EXACT && d_ <= 128 && Pm <= kCoarseMaxPm && nq > 0;
    HB_CHECK(tc || coarse_kind_ != HB_COARSE_TENSOR, HB_ERR_INVALID,
             "the tensor-core coarse quantizer needs d <= 128 and nprobe + margin <= 1024");
    if (!tc) {
      {
        Scope sc(this, "coarse_l2_matrix");
        launch_l2_matrix(qpad, nq, cent_.p, static_cast<int>(nlist_), static_cast<int>(dpad_), dmat_.p,
                         static_cast<int>(nlist_), st_);
      }
      Scope sc(this, "coarse_select");
      cflags_.reserve(static_cast<size_t>(nq));
      launch_select_rows(dmat_.p, nq, static_cast<int>(nlist_), static_cast<int>(nlist_), P, probes_out, cdist_out,
                         st_, nullptr, cflags_.p);
      launches_ += 3;  // matrix, warp selection, its CTA kernel
      coarse_last_nq_ = 0;
      return;
    }
    ensure_coarse_tc();
    qsplit_.reserve(static_cast<size_t>(nq) * 2 * ckpad_);
    qsnorm_.reserve(static_cast<size_t>(nq));
    cmins_.reserve(static_cast<size_t>(nq) * ((nlist_ + 15) / 16));
    ccand_.reserve(static_cast<size_t>(nq) * Pm);
    cval_.reserve(static_cast<size_t>(nq) * Pm);
    cflags_.reserve(static_cast<size_t>(nq));
    {
      Scope sc(this, "coarse_tc");
      launch_coarse_tc(ctmap_, qpad, nq, static_cast<int>(dpad_), ckpad_, cnorm_.p, static_cast<int>(nlist_), dmat_.p,
                       qsplit_.p, qsnorm_.p, cmins_.p, cerr_dev_.p, num_sms_, st_);
    }
    {
      Scope sc(this, "coarse_select");
      launch_select_rows(dmat_.p, nq, static_cast<int>(nlist_), static_cast<int>(nlist_), Pm, ccand_.p, cval_.p, st_,
                         nullptr, cflags_.p, cmins_.p);
    }
    {
      Scope sc(this, "coarse_refine");
      launch_coarse_refine(qpad, nq, static_cast<int>(dpad_), cent_.p, ccand_.p, cval_.p, Pm, P,
                           static_cast<int>(nlist_), cmaxnorm_.p, probes_out, cdist_out, cflags_.p, st_);
      launch_coarse_fallback(qpad, nq, static_cast<int>(dpad_), cent_.p, static_cast<int>(nlist_), P, cflags_.p,
                             dmat_.p, probes_out, cdist_out, st_, nullptr, cmins_.p);
    }
    launches_ += 6;
    coarse_last_nq_ = nq;
  }

  int coarse_extra(int P) const { return coarse_margin_ >= 0 ? coarse_margin_ : std::max(16, P / 4); }

  bool coarse_tc_route(int P) const {
    const int Pm = std::min<int>(static_cast<int>(nlist_), P + coarse_extra(P));
    return coarse_kind_ != HB_COARSE_EXACT && d_ <= 128 && Pm <= kCoarseMaxPm;
  }

  // Learned probe on the tensor-core route: the exact nearest C centroids
  // (the predictor's features) from one narrow pass, the predictor's
  // per-query nprobe, then a second pass over the same approximate distance
  // matrix that widens only the rows whose nprobe exceeds C (each to its own
  // width plus margin).  probes_out (nq x P, -1 past each row's nprobe) is the
  // exact quantizer's rows cut at the predicted nprobe, as the wide route
  // gives.
  void coarse_learned(const float* qpad, int nq, int P, int32_t* probes_out, float thr, int cap) {
    const ProbeModel& m = probe_;
    const int C = std::min<int>(m.C, P);
    dmat_.reserve(static_cast<size_t>(nq) * nlist_);
    ensure_coarse_tc();
    qsplit_.reserve(static_cast<size_t>(nq) * 2 * ckpad_);
    qsnorm_.reserve(static_cast<size_t>(nq));
    cmins_.reserve(static_cast<size_t>(nq) * ((nlist_ + 15) / 16));
    const int nl = static_cast<int>(nlist_);
    const int PmA = std::min(nl, C + coarse_extra(C));
    const int PmB = std::min(nl, P + coarse_extra(P));
    ccand_.reserve(static_cast<size_t>(nq) * PmB);
    cval_.reserve(static_cast<size_t>(nq) * PmB);
    cflags_.reserve(static_cast<size_t>(nq));
    probes1_.reserve(static_cast<size_t>(nq) * C);
    cdist_.reserve(static_cast<size_t>(nq) * C);
    npq_.reserve(static_cast<size_t>(nq));
    kq_.reserve(static_cast<size_t>(nq));
    {
      Scope sc(this, "coarse_tc");
      launch_coarse_tc(ctmap_, qpad, nq, static_cast<int>(dpad_), ckpad_, cnorm_.p, nl, dmat_.p, qsplit_.p, qsnorm_.p,
                       cmins_.p, cerr_dev_.p, num_sms_, st_);
    }
    {
      Scope sc(this, "coarse_select");
      launch_select_rows(dmat_.p, nq, nl, nl, PmA, ccand_.p, cval_.p, st_, nullptr, cflags_.p, cmins_.p);
    }
    {
      Scope sc(this, "coarse_refine");
      launch_coarse_refine(qpad, nq, static_cast<int>(dpad_), cent_.p, ccand_.p, cval_.p, PmA, C, nl, cmaxnorm_.p,
                           probes1_.p, cdist_.p, cflags_.p, st_);
      launch_coarse_fallback(qpad, nq, static_cast<int>(dpad_), cent_.p, nl, C, cflags_.p, dmat_.p, probes1_.p,
                             cdist_.p, st_, nullptr, cmins_.p);
    }
    {
      Scope sc(this, "probe_mlp");
      probe_infer(nq, qpad, cdist_.p, C, nullptr, thr, cap, npq_.p);
    }
    {
      Scope sc(this, "coarse_widen_select");
      launch_coarse_widths(npq_.p, nq, P, C, coarse_margin_, nl, kq_.p, st_);
      launch_select_rows(dmat_.p, nq, nl, nl, PmB, ccand_.p, cval_.p, st_, kq_.p, cflags_.p, cmins_.p);
    }
    {
      Scope sc(this, "coarse_widen_refine");
      CoarseRows rows;
      rows.width = npq_.p;
      rows.margin = coarse_margin_;
      rows.pre = probes1_.p;
      rows.pre_w = C;
      launch_coarse_refine(qpad, nq, static_cast<int>(dpad_), cent_.p, ccand_.p, cval_.p, PmB, P, nl, cmaxnorm_.p,
                           probes_out, nullptr, cflags_.p, st_, rows);
      launch_coarse_fallback(qpad, nq, static_cast<int>(dpad_), cent_.p, nl, P, cflags_.p, dmat_.p, probes_out, nullptr,
                             st_, npq_.p);
    }
    // narrow pass: query split, matrix, selection + its CTA kernel,
    // refinement, fallback; widening pass: widths, selection, refinement,
    // fallback (the predictor counts its own).
    launches_ += 10;
    coarse_last_nq_ = nq;
  }

  // Split BF16 centroids, their tensor map, ||c||^2 and max ||c||, built once
  // per set of centroids.
  void ensure_coarse_tc() {
    if (coarse_ready_) return;
    ckpad_ = static_cast<int>((d_ + 63) / 64 * 64);
    csplit_.reserve(nlist_ * 2 * static_cast<size_t>(ckpad_));
    make_centroid_split(cent_.p, static_cast<int>(nlist_), static_cast<int>(dpad_), ckpad_, csplit_.p, ctmap_, st_);
    cnorm_.reserve(nlist_);
    launch_row_norms(cent_.p, nlist_, static_cast<int>(d_), static_cast<int>(dpad_), cnorm_.p, st_);
    cmaxnorm_.reserve(1);
    launch_max_norm(cnorm_.p, nlist_, cmaxnorm_.p, st_);
    cerr_dev_.reserve(1);
    HB_CUDA(cudaMemsetAsync(cerr_dev_.p, 0, sizeof(int), st_));
    launches_ += 3;
    coarse_ready_ = true;
  }

  // Raises when a bounded wait of the tensor-core quantizer gave up since the
  // last check (the flag is sticky until read here).
  void coarse_err_check() {
    if (!cerr_dev_.p) return;
    HB_CUDA(cudaMemcpyAsync(err_host_, cerr_dev_.p, sizeof(int), cudaMemcpyDeviceToHost, st_));
    HB_CUDA(cudaStreamSynchronize(st_));
    if (*err_host_ != 0) {
      const int code = *err_host_;
      HB_CUDA(cudaMemsetAsync(cerr_dev_.p, 0, sizeof(int), st_));
      throw Error(HB_ERR_CUDA, "tensor-core coarse quantizer gave up waiting (code " + std::to_string(code) + ")");
    }
  }

  void set_wait_budget(long long cycles) { wait_budget_ = cycles > 0 ? cycles : kDefaultWaitBudget; }
  int last_overflow() const { return last_overflow_; }
  // Admission statistics of the latest bounded BF16 batch: queries,
  // overflows, rows admitted (total, largest per query), rows re-ranked.
  void bf16_stats(int64_t* out) {
    HB_CUDA(cudaSetDevice(device_));
    std::vector<int> cnt(last_nb_), m(last_nb_);
    if (last_nb_) {
      HB_CUDA(cudaMemcpyAsync(cnt.data(), ccnt_.p, cnt.size() * sizeof(int), cudaMemcpyDeviceToHost, st_));
      HB_CUDA(cudaMemcpyAsync(m.data(), rr_m_.p, m.size() * sizeof(int), cudaMemcpyDeviceToHost, st_));
      HB_CUDA(cudaStreamSynchronize(st_));
    }
    int64_t tot = 0, mx = 0, mt = 0;
    for (int i = 0; i < last_nb_; ++i) {
      tot += cnt[i];
      mx = std::max<int64_t>(mx, cnt[i]);
      mt += m[i];
    }
    out[0] = last_nb_;
    out[1] = last_overflow_;
    out[2] = tot;
    out[3] = mx;
    out[4] = mt;
  }

  void set_coarse(int kind, int margin) {
    HB_CHECK(kind >= HB_COARSE_AUTO && kind <= HB_COARSE_TENSOR, HB_ERR_INVALID, "unknown coarse quantizer kind");
    HB_CHECK(margin >= -1 && margin <= kCoarseMaxPm, HB_ERR_INVALID, "coarse margin must be in [-1, 1024]");
    coarse_kind_ = kind;
    coarse_margin_ = margin;
  }

  // Queries of the most recent tensor-core coarse call whose rows were
  // recomputed exactly.
  int64_t coarse_fallbacks() {
    HB_CUDA(cudaSetDevice(device_));
    if (coarse_last_nq_ == 0) return 0;
    std::vector<int> f(coarse_last_nq_);
    HB_CUDA(cudaMemcpyAsync(f.data(), cflags_.p, f.size() * sizeof(int), cudaMemcpyDeviceToHost, st_));
    HB_CUDA(cudaStreamSynchronize(st_));
    int64_t n = 0;
    for (int v : f) n += v != 0;
    return n;
  }

  // ---- search: src/Index.cpp:1638-1706 --------------------------------------

  void search(size_t nq, const float* q, size_t k, const hb_search_params* prm, float* D, int64_t* I) {
    if (nq == 0) return;
    HB_CHECK(q && D && I, HB_ERR_INVALID, "null query or result pointer");
    HB_CHECK(k > 0, HB_ERR_INVALID, "k must be positive");
    HB_CUDA(cudaSetDevice(device_));
    hb_search_params p;
    hb_search_params_init(&p);
    if (prm) p = *prm;
    if (nprobe_ > nlist_) nprobe_ = nlist_;  // src/Index.cpp:1646-1648 (mutates the field)
    HB_CHECK(p.precision == HB_PREC_FP32 || p.precision == HB_PREC_BF16 || p.precision == HB_PREC_FP8,
             HB_ERR_INVALID, "precision must be FP32, BF16 or FP8");
    // bf16: a tensor-core scan (BF16, or the FP8 variant) with an exact re-rank.
    const bool bf16 = p.precision != HB_PREC_FP32;
    fp8_ = p.precision == HB_PREC_FP8;
    if (bf16) {
      HB_CHECK(p.mode == HB_MODE_ORIGINAL || p.mode == HB_MODE_BRUTE_FORCE, HB_ERR_INVALID,
               "the BF16 scan implements ORIGINAL / BRUTE_FORCE search (pruning and the dimension relay are FP32 modes)");
      HB_CHECK(ntotal_ == 0 || bf16_ready_, HB_ERR_STATE, "BF16 codes not built");
    }
    HB_CHECK(p.seed_rows >= 0 && p.seed_rows <= 256, HB_ERR_INVALID, "seed_rows must be in [0, 256]");
    seed_rows_ = p.seed_rows > 0 ? p.seed_rows : 256;
    // BF16 route: the bounded filter scan (exact result) for d <= 128 and
    // k <= 256, else the candidate-matrix scan with a fixed re-rank width.
    const int want_R = std::max(static_cast<int>(k), p.rerank_mult * static_cast<int>(k));
    int etv = 0, eqt = 0, eqg = 0;
    const bool exact_k = scan_exact_smem_bytes(static_cast<int>(d_), static_cast<int>(dpad_), static_cast<int>(k),
                                               SCAN_PLAIN, &etv, &eqt, &eqg) > 0;
    // FP8 (E4M3: 3 mantissa bits, a rounding bound 16 times BF16's) always
    // takes the candidate-matrix scan with its fixed re-rank width.
    cand_path_ = bf16 && (fp8_ || !(kpad_ <= 128 && static_cast<int>(k) <= kFilterMaxK && exact_k));
    const int R = cand_path_ ? std::min(kCandMaxR, want_R) : 0;
    if (cand_path_)
      HB_CHECK(static_cast<int>(k) <= R, HB_ERR_INVALID,
               "BF16 search supports k up to " + std::to_string(kCandMaxR));
    int mode = SCAN_PLAIN;
    size_t P = nprobe_;
    int W = 1, B = 1;
    std::vector<int32_t> order;
    bool need_tops = false;
    switch (p.mode) {
      case HB_MODE_ORIGINAL:
        break;
      case HB_MODE_BRUTE_FORCE:
        P = nlist_;
        break;
      case HB_MODE_DIVIDE_IVF:
        if (p.pruning) {
          mode = SCAN_CHUNK4;
          need_tops = true;
        }
        break;
      case HB_MODE_DIVIDE_DIM: {
        W = p.n_dim_blocks;
        B = p.n_query_blocks;
        HB_CHECK(W >= 1 && W <= 8, HB_ERR_INVALID, "n_dim_blocks must be in [1, 8]");
        HB_CHECK(d_ % W == 0, HB_ERR_INVALID, "d must be divisible by n_dim_blocks (src/Index.cpp:125)");
        HB_CHECK(B >= 1, HB_ERR_INVALID, "n_query_blocks must be >= 1");
        mode = SCAN_DIMBLOCK;
        need_tops = true;  // heap tops are always computed (src/Index.cpp:1241-1252)
        order = block_visit_order(W, B, p.order_optimize != 0, p.period != 0);
        break;
      }
      default:
        throw Error(HB_ERR_INVALID, "search mode not supported");
    }
    // Param::fullWarmUp: the dimension relay prunes against the caller's heap
    // tops instead of the warm-up search's (src/Index.cpp:1235-1241); the
    // reference reads the flag in no other mode.
    ext_tops_ = nullptr;
    if (p.mode == HB_MODE_DIVIDE_DIM && p.full_warmup) {
      HB_CHECK(p.heap_tops, HB_ERR_INVALID, "fullWarmUp needs heap_tops (the reference exits: heapTop not exist)");
      ext_tops_ = p.heap_tops;
    }
    // Per-query nprobe: the learned predictor or a caller-given array.  The
    // coarse quantizer selects the widest probe row, each query's row is then
    // cut at its own nprobe (cut entries become -1 and are never scanned).
    const bool learned = p.learned_probe != 0;
    cut_mode_ = 0;
    if (learned) {
      HB_CHECK(probe_.trained, HB_ERR_STATE, "learned probe predictor not trained (hb_train_probe_predictor)");
      HB_CHECK(!p.nprobe_per_query, HB_ERR_INVALID, "learned probe and nprobe_per_query are exclusive");
      P = std::min<size_t>(probe_.pmax, nlist_);
      cut_mode_ = 1;
      cut_cap_ = p.max_nprobe > 0 ? std::min<int>(p.max_nprobe, static_cast<int>(P)) : static_cast<int>(P);
      cut_thr_ = probe_.threshold_for(p.learned_target);
    } else if (p.nprobe_per_query) {
      if (p.max_nprobe > 0) P = std::min<size_t>(static_cast<size_t>(p.max_nprobe), nlist_);
      cut_mode_ = 2;
      cut_src_ = p.nprobe_per_query;
    }

    const bool dev_out = is_device_ptr(D) && is_device_ptr(I);
    const bool dev_in = is_device_ptr(q);
    size_t bs = std::min<size_t>(nq, batch_limit(P, k));
    if (cand_path_ && P > 0) bs = std::min(bs, cand_batch_limit(P));
    if (bf16 && !cand_path_)
      bs = std::min(bs, std::max<size_t>(1, (size_t(1) << 30) / (static_cast<size_t>(filter_cap(k)) * 8)));
    const int warm_lists = p.warmup_lists;
    const int warm_size = p.warmup_list_size > 0 ? p.warmup_list_size : static_cast<int>(k);
    // DIVIDE_DIM query blocks cover queries [0, B * (nq / B)); the rest stay
    // unsearched (src/Index.cpp:1189, 1266-1270).
    const int qblock = mode == SCAN_DIMBLOCK ? static_cast<int>(nq / B) : 0;
    if (mode == SCAN_DIMBLOCK) HB_CHECK(nq <= bs, HB_ERR_INVALID, "DIVIDE_DIM search is limited to one batch");
    if (!order.empty()) {
      order_dev_.reserve(order.size());
      HB_CUDA(cudaMemcpyAsync(order_dev_.p, order.data(), order.size() * sizeof(int32_t), cudaMemcpyHostToDevice, st_));
    }

    if (p.use_graph) {
      HB_CHECK(mode == SCAN_PLAIN && (p.mode == HB_MODE_ORIGINAL || p.mode == HB_MODE_BRUTE_FORCE) && nq <= bs,
               HB_ERR_INVALID, "graph search runs ORIGINAL / BRUTE_FORCE searches of one batch");
      search_graph(static_cast<int>(nq), q, static_cast<int>(k), static_cast<int>(P), R, bf16, p, D, I);
      return;
    }
    for (size_t b0 = 0; b0 < nq; b0 += bs) {
      const int nb = static_cast<int>(std::min(bs, nq - b0));
      cut_b0_ = b0;
      float* Dd = dev_out ? D + b0 * k : nullptr;
      int64_t* Id = dev_out ? I + b0 * k : nullptr;
      if (!dev_out) {
        dout_.reserve(static_cast<size_t>(nb) * k);
        iout_.reserve(static_cast<size_t>(nb) * k);
        Dd = dout_.p;
        Id = iout_.p;
      }
      // Queries.
      qpad_.reserve(static_cast<size_t>(nb) * dpad_);
      const float* qsrc = q + b0 * d_;
      if (!dev_in) {
        qtmp_.reserve(static_cast<size_t>(nb) * d_);
        HB_CUDA(cudaMemcpyAsync(qtmp_.p, qsrc, static_cast<size_t>(nb) * d_ * sizeof(float), cudaMemcpyHostToDevice,
                                st_));
        qsrc = qtmp_.p;
      }
      launch_pad_rows(qsrc, nb, static_cast<int>(d_), static_cast<int>(dpad_), qpad_.p, st_);
      ++launches_;
      if (P == 0 || ntotal_ == 0) {
        launch_fill_results(Dd, Id, static_cast<size_t>(nb) * k, st_);
        ++launches_;
      } else {
        if (bf16)
          search_batch_bf16(nb, static_cast<int>(P), static_cast<int>(k), R, Dd, Id);
        else
          search_batch(nb, static_cast<int>(P), static_cast<int>(k), mode, p.pruning != 0, need_tops, warm_lists,
                       warm_size, W, B, qblock, Dd, Id);
      }
      if (!dev_out) {
        HB_CUDA(cudaMemcpyAsync(D + b0 * k, Dd, static_cast<size_t>(nb) * k * sizeof(float), cudaMemcpyDeviceToHost,
                                st_));
        HB_CUDA(cudaMemcpyAsync(I + b0 * k, Id, static_cast<size_t>(nb) * k * sizeof(int64_t),
                                cudaMemcpyDeviceToHost, st_));
      }
    }
    HB_CUDA(cudaStreamSynchronize(st_));
    coarse_err_check();
  }

  // ---- one batch as a CUDA graph --------------------------------------------
  //
  // The batch's inputs are copied into fixed buffers (queries, per-query
  // nprobe), the device pipeline runs as one graph launch, and the results
  // are copied out of fixed buffers.  A graph is captured per batch shape
  // (batch size, k, nprobe, precision, candidate count, nprobe mode and its
  // settings) after one ordinary run of the same shape has sized every buffer;
  // any later device allocation of the library, and any change to the index
  // (train / add / load), drops the cached graphs.
  struct GraphEntry {
    cudaGraphExec_t exec = nullptr;
    uint64_t gen = 0;
    uint64_t launches = 0;
  };

  void drop_graphs() {
    for (auto& kv : graphs_)
      if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    graphs_.clear();
  }

  void run_batch_pipeline(int nb, int k, int P, int R, bool bf16) {
    launch_pad_rows(qtmp_.p, nb, static_cast<int>(d_), static_cast<int>(dpad_), qpad_.p, st_);
    ++launches_;
    if (P == 0 || ntotal_ == 0) {
      launch_fill_results(dout_.p, iout_.p, static_cast<size_t>(nb) * k, st_);
      ++launches_;
    } else if (bf16) {
      search_batch_bf16(nb, P, k, R, dout_.p, iout_.p);
    } else {
      search_batch(nb, P, k, SCAN_PLAIN, false, false, 0, k, 1, 1, 0, dout_.p, iout_.p);
    }
  }

  void search_graph(int nb, const float* q, int k, int P, int R, bool bf16, const hb_search_params& p, float* D,
                    int64_t* I) {
    qtmp_.reserve(static_cast<size_t>(nb) * d_);
    qpad_.reserve(static_cast<size_t>(nb) * dpad_);
    dout_.reserve(static_cast<size_t>(nb) * k);
    iout_.reserve(static_cast<size_t>(nb) * k);
    HB_CUDA(cudaMemcpyAsync(qtmp_.p, q, static_cast<size_t>(nb) * d_ * sizeof(float), cudaMemcpyDefault, st_));
    if (cut_mode_ == 2) {
      npqin_.reserve(static_cast<size_t>(nb));
      HB_CUDA(cudaMemcpyAsync(npqin_.p, cut_src_, static_cast<size_t>(nb) * sizeof(int32_t), cudaMemcpyDefault, st_));
      cut_src_ = npqin_.p;
    }
    cut_b0_ = 0;
    char key[256];
    std::snprintf(key, sizeof(key), "%d/%d/%d/%d/%d/%d/%d/%08x/%d/%d/%d/%d/%d", nb, k, P, R, p.precision, p.mode,
                  cut_mode_, cut_mode_ == 1 ? *reinterpret_cast<const uint32_t*>(&cut_thr_) : 0u, cut_cap_,
                  seed_rows_, coarse_kind_, coarse_margin_, static_cast<int>(nprobe_));
    auto it = graphs_.find(key);
    if (it != graphs_.end() && it->second.gen != devbuf_generation().load()) {
      cudaGraphExecDestroy(it->second.exec);
      graphs_.erase(it);
      it = graphs_.end();
    }
    if (it != graphs_.end()) {
      if (bf16) HB_CUDA(cudaMemsetAsync(err_dev_.p, 0, sizeof(int), st_));
      HB_CUDA(cudaGraphLaunch(it->second.exec, st_));
      launches_ += it->second.launches;
    } else {
      // An ordinary run sizes every buffer (and gives this call's results),
      // then the same sequence is captured.
      run_batch_pipeline(nb, k, P, R, bf16);
      HB_CUDA(cudaStreamSynchronize(st_));
      const uint64_t gen = devbuf_generation().load();
      const uint64_t l0 = launches_;
      HB_CUDA(cudaStreamBeginCapture(st_, cudaStreamCaptureModeRelaxed));
      capturing_ = true;
      cudaGraph_t graph = nullptr;
      try {
        run_batch_pipeline(nb, k, P, R, bf16);
      } catch (...) {
        capturing_ = false;
        cudaStreamEndCapture(st_, &graph);
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        throw;
      }
      capturing_ = false;
      HB_CUDA(cudaStreamEndCapture(st_, &graph));
      if (devbuf_generation().load() == gen) {
        GraphEntry e;
        const cudaError_t ie = cudaGraphInstantiate(&e.exec, graph, 0);
        if (ie == cudaSuccess) {
          e.gen = gen;
          e.launches = launches_ - l0;
          graphs_[key] = e;
        } else {
          cudaGetLastError();
        }
      }
      cudaGraphDestroy(graph);
      launches_ = l0;
    }
    if (bf16 && !cand_path_) {
      bf16_err_check();
      fix_overflow(nb, P, k, dout_.p, iout_.p);
    }
    HB_CUDA(cudaMemcpyAsync(D, dout_.p, static_cast<size_t>(nb) * k * sizeof(float), cudaMemcpyDefault, st_));
    HB_CUDA(cudaMemcpyAsync(I, iout_.p, static_cast<size_t>(nb) * k * sizeof(int64_t), cudaMemcpyDefault, st_));
    HB_CUDA(cudaStreamSynchronize(st_));
    if (bf16) bf16_err_check();
    coarse_err_check();
  }

  void probe_lists(size_t nq, const float* q, size_t P, int64_t* probes, float* cdist) {
    if (nq == 0) return;
    HB_CUDA(cudaSetDevice(device_));
    HB_CHECK(P >= 1 && P <= nlist_, HB_ERR_INVALID, "nprobe must be in [1, nlist]");
    DevBuf<float> qp, tmp, cd;
    stage_rows(q, nq, qp, tmp);
    DevBuf<int32_t> pr;
    DevBuf<int64_t> pr64;
    pr.reserve(nq * P);
    pr64.reserve(nq * P);
    cd.reserve(nq * P);
    coarse(qp.p, static_cast<int>(nq), static_cast<int>(P), pr.p, cd.p);
    launch_i32_to_i64(pr.p, nq * P, pr64.p, st_);
    ++launches_;
    HB_CUDA(cudaMemcpyAsync(probes, pr64.p, nq * P * sizeof(int64_t), cudaMemcpyDefault, st_));
    if (cdist) HB_CUDA(cudaMemcpyAsync(cdist, cd.p, nq * P * sizeof(float), cudaMemcpyDefault, st_));
    HB_CUDA(cudaStreamSynchronize(st_));    coarse_err_check();
  }

  void warmup_tops(size_t nq, const float* q, size_t k, size_t wl, size_t wls, float* tops) {
    if (nq == 0) return;
    HB_CUDA(cudaSetDevice(device_));
    size_t P = std::min(nprobe_, nlist_);
    DevBuf<float> qp, tmp, t;
    stage_rows(q, nq, qp, tmp);
    DevBuf<int32_t> pr;
    pr.reserve(std::max<size_t>(nq * P, 1));
    t.reserve(nq);
    if (P > 0) coarse(qp.p, static_cast<int>(nq), static_cast<int>(P), pr.p, nullptr);
    launch_warmup_tops(qp.p, static_cast<int>(nq), pr.p, static_cast<int>(P), codes_.p, list_off_.p,
                       static_cast<int>(dpad_), static_cast<int>(k), static_cast<int>(wl), static_cast<int>(wls), t.p,
                       st_);
    ++launches_;
    HB_CUDA(cudaMemcpyAsync(tops, t.p, nq * sizeof(float), cudaMemcpyDefault, st_));
    HB_CUDA(cudaStreamSynchronize(st_));    coarse_err_check();
  }

  // ---- save / load: src/Index.cpp:1708-1770, src/IVF.cpp:76-134 --------------

  void save(const char* path) {
    HB_CUDA(cudaSetDevice(device_));
    std::ofstream out(path, std::ios::binary);
    HB_CHECK(out.is_open(), HB_ERR_IO, std::string("Cannot open file ") + path);
    std::vector<float> cent(nlist_ * dpad_);
    HB_CUDA(cudaMemcpyAsync(cent.data(), cent_.p, cent.size() * sizeof(float), cudaMemcpyDeviceToHost, st_));
    std::vector<float> codes(ntotal_ * dpad_);
    std::vector<int64_t> ids(ntotal_);
    std::vector<float> norms(ntotal_);
    if (ntotal_) {
      HB_CUDA(cudaMemcpyAsync(codes.data(), codes_.p, codes.size() * sizeof(float), cudaMemcpyDeviceToHost, st_));
      HB_CUDA(cudaMemcpyAsync(ids.data(), ids_.p, ids.size() * sizeof(int64_t), cudaMemcpyDeviceToHost, st_));
      HB_CUDA(cudaMemcpyAsync(norms.data(), norms_.p, norms.size() * sizeof(float), cudaMemcpyDeviceToHost, st_));
    }
    HB_CUDA(cudaStreamSynchronize(st_));
    const size_t sub_k = 0, sub_nlist = 1, sub_nprobe = 1;
    const int32_t metric = metric_, opt = 0;
    out.write(reinterpret_cast<const char*>(&d_), sizeof(size_t));
    out.write(reinterpret_cast<const char*>(&nlist_), sizeof(size_t));
    out.write(reinterpret_cast<const char*>(&metric), sizeof(int32_t));
    out.write(reinterpret_cast<const char*>(&opt), sizeof(int32_t));
    out.write(reinterpret_cast<const char*>(&sub_k), sizeof(size_t));
    out.write(reinterpret_cast<const char*>(&sub_nlist), sizeof(size_t));
    out.write(reinterpret_cast<const char*>(&sub_nprobe), sizeof(size_t));
    std::vector<float> row(d_);
    for (size_t c = 0; c < nlist_; ++c)
      out.write(reinterpret_cast<const char*>(&cent[c * dpad_]), d_ * sizeof(float));
    for (size_t l = 0; l < nlist_; ++l) {
      const size_t n = static_cast<size_t>(host_off_[l + 1] - host_off_[l]);
      if (!n) continue;
      const size_t b = static_cast<size_t>(host_off_[l]);
      out.write(reinterpret_cast<const char*>(&l), sizeof(size_t));
      out.write(reinterpret_cast<const char*>(&n), sizeof(size_t));
      out.write(reinterpret_cast<const char*>(&d_), sizeof(size_t));
      out.write(reinterpret_cast<const char*>(&sub_k), sizeof(size_t));
      out.write(reinterpret_cast<const char*>(&opt), sizeof(int32_t));
      for (size_t i = 0; i < n; ++i) {
        const size_t id = static_cast<size_t>(ids[b + i]);
        out.write(reinterpret_cast<const char*>(&id), sizeof(size_t));
      }
      for (size_t i = 0; i < n; ++i) out.write(reinterpret_cast<const char*>(&codes[(b + i) * dpad_]), d_ * sizeof(float));
      out.write(reinterpret_cast<const char*>(&norms[b]), n * sizeof(float));
    }
    HB_CHECK(out.good(), HB_ERR_IO, std::string("write failed: ") + path);
  }

  void load(const char* path) {
    HB_CUDA(cudaSetDevice(device_));
    std::ifstream in(path, std::ios::binary);
    HB_CHECK(in.is_open(), HB_ERR_IO, std::string("Cannot open file ") + path);
    size_t d = 0, nlist = 0, sub_k = 0, sub_nlist = 0, sub_nprobe = 0;
    int32_t metric = 0, opt = 0;
    in.read(reinterpret_cast<char*>(&d), sizeof(size_t));
    in.read(reinterpret_cast<char*>(&nlist), sizeof(size_t));
    in.read(reinterpret_cast<char*>(&metric), sizeof(int32_t));
    in.read(reinterpret_cast<char*>(&opt), sizeof(int32_t));
    in.read(reinterpret_cast<char*>(&sub_k), sizeof(size_t));
    in.read(reinterpret_cast<char*>(&sub_nlist), sizeof(size_t));
    in.read(reinterpret_cast<char*>(&sub_nprobe), sizeof(size_t));
    HB_CHECK(in.good(), HB_ERR_IO, "truncated index header");
    HB_CHECK(metric == HB_METRIC_L2, HB_ERR_IO, "index metric is not L2");
    HB_CHECK(d > 0 && d <= 1024 && nlist > 0 && nlist <= (1u << 20), HB_ERR_IO, "implausible index shape");
    std::vector<float> cent(nlist * d);
    in.read(reinterpret_cast<char*>(cent.data()), cent.size() * sizeof(float));
    HB_CHECK(in.good(), HB_ERR_IO, "truncated centroids");
    struct ListRec {
      std::vector<int64_t> ids;
      std::vector<float> codes, norms;
    };
    std::vector<ListRec> lists(nlist);
    for (;;) {
      size_t lid = 0;
      in.read(reinterpret_cast<char*>(&lid), sizeof(size_t));
      if (in.eof()) break;
      HB_CHECK(in.good() && lid < nlist, HB_ERR_IO, "bad list record");
      size_t n = 0, ld = 0, lsk = 0;
      int32_t lopt = 0;
      in.read(reinterpret_cast<char*>(&n), sizeof(size_t));
      in.read(reinterpret_cast<char*>(&ld), sizeof(size_t));
      in.read(reinterpret_cast<char*>(&lsk), sizeof(size_t));
      in.read(reinterpret_cast<char*>(&lopt), sizeof(int32_t));
      HB_CHECK(in.good() && ld == d && n < (1ull << 32), HB_ERR_IO, "bad list header");
      ListRec& r = lists[lid];
      std::vector<size_t> ids(n);
      r.codes.resize(n * d);
      r.norms.resize(n);
      in.read(reinterpret_cast<char*>(ids.data()), n * sizeof(size_t));
      in.read(reinterpret_cast<char*>(r.codes.data()), n * d * sizeof(float));
      in.read(reinterpret_cast<char*>(r.norms.data()), n * sizeof(float));
      r.ids.assign(ids.begin(), ids.end());
      // Opt-level extras (src/IVF.cpp:190-211) are read and dropped.
      size_t skip = 0;
      if ((lopt & 1) || (lopt & 4)) skip += 2 * n * sizeof(float);
      if (lopt & 2) skip += n * lsk * (sizeof(int64_t) + sizeof(float));
      if (lopt & 4) skip += 2 * n * lsk * (sizeof(int64_t) + sizeof(float));
      if (skip) in.seekg(static_cast<std::streamoff>(skip), std::ios::cur);
      HB_CHECK(in.good(), HB_ERR_IO, "truncated list record");
    }
    reshape(d, nlist);
    metric_ = metric;
    std::vector<float> cpad(nlist * dpad_, 0.0f);
    for (size_t c = 0; c < nlist; ++c) std::copy(&cent[c * d], &cent[c * d] + d, &cpad[c * dpad_]);
    HB_CUDA(cudaMemcpyAsync(cent_.p, cpad.data(), cpad.size() * sizeof(float), cudaMemcpyHostToDevice, st_));
    host_off_.assign(nlist + 1, 0);
    for (size_t l = 0; l < nlist; ++l) host_off_[l + 1] = host_off_[l] + static_cast<int64_t>(lists[l].ids.size());
    const size_t nt = static_cast<size_t>(host_off_[nlist]);
    std::vector<float> codes(nt * dpad_, 0.0f);
    std::vector<int64_t> ids(nt);
    std::vector<float> norms(nt);
    for (size_t l = 0; l < nlist; ++l) {
      const size_t b = static_cast<size_t>(host_off_[l]);
      const ListRec& r = lists[l];
      for (size_t i = 0; i < r.ids.size(); ++i) {
        ids[b + i] = r.ids[i];
        norms[b + i] = r.norms[i];
        std::copy(&r.codes[i * d], &r.codes[i * d] + d, &codes[(b + i) * dpad_]);
      }
    }
    codes_.reserve(std::max<size_t>(nt * dpad_, 1));
    ids_.reserve(std::max<size_t>(nt, 1));
    norms_.reserve(std::max<size_t>(nt, 1));
    if (nt) {
      HB_CUDA(cudaMemcpyAsync(codes_.p, codes.data(), codes.size() * sizeof(float), cudaMemcpyHostToDevice, st_));
      HB_CUDA(cudaMemcpyAsync(ids_.p, ids.data(), ids.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st_));
      HB_CUDA(cudaMemcpyAsync(norms_.p, norms.data(), norms.size() * sizeof(float), cudaMemcpyHostToDevice, st_));
    }
    HB_CUDA(cudaMemcpyAsync(list_off_.p, host_off_.data(), (nlist + 1) * sizeof(int64_t), cudaMemcpyHostToDevice,
                            st_));
    HB_CUDA(cudaStreamSynchronize(st_));
    ntotal_ = nt;
    trained_ = true;
    plan_rows_ = 0;
    build_bf16();
    drop_graphs();
  }

  // Exact ORIGINAL search of one batch whose per-call buffers all come from
  // the caller's device scratch; no DevBuf grows here.
  void search_in_scratch(size_t nq, const float* q, size_t k, float* D, int64_t* I, unsigned char* scratch,
                         size_t bytes) {
    if (nq == 0) return;
    HB_CHECK(q && D && I && scratch, HB_ERR_INVALID, "null query, result or scratch pointer");
    HB_CHECK(k > 0, HB_ERR_INVALID, "k must be positive");
    HB_CUDA(cudaSetDevice(device_));
    HB_CHECK(is_device_ptr(q) && is_device_ptr(D) && is_device_ptr(I), HB_ERR_INVALID,
             "queries and results must be device pointers");
    HB_CHECK(nq <= 65535, HB_ERR_INVALID, "at most 65535 queries per call");
    if (nprobe_ > nlist_) nprobe_ = nlist_;  // src/Index.cpp:1646-1648
    const int P = static_cast<int>(nprobe_);
    if (P == 0 || ntotal_ == 0) {
      launch_fill_results(D, I, nq * k, st_);
      HB_CUDA(cudaStreamSynchronize(st_));
      return;
    }
    int tv = 0, qt = 0, qg = 0;
    HB_CHECK(scan_exact_smem_bytes(static_cast<int>(d_), static_cast<int>(dpad_), static_cast<int>(k), SCAN_PLAIN,
                                   &tv, &qt, &qg) > 0,
             HB_ERR_INVALID, "k too large for the fused scan at this dimension");
    const int nb = static_cast<int>(nq);
    const int cr = chunk_rows_for(nb, P, tv);
    // Slot bound without host allocation: min(P * largest chunk count,
    // all chunks) per query.
    int64_t max_ch = 0, all_ch = 0;
    for (size_t l = 0; l < nlist_; ++l) {
      const int64_t c = (host_off_[l + 1] - host_off_[l] + cr - 1) / cr;
      max_ch = std::max(max_ch, c);
      all_ch += c;
    }
    const size_t slots = nq * static_cast<size_t>(std::max<int64_t>(1, std::min<int64_t>(P * max_ch, all_ch)));
    size_t off = 0;
    auto carve = [&](size_t nbytes) {
      unsigned char* p = scratch + off;
      off += (nbytes + 255) / 256 * 256;
      return p;
    };
    float* qpad = reinterpret_cast<float*>(carve(nq * dpad_ * sizeof(float)));
    float* dmat = reinterpret_cast<float*>(carve(nq * nlist_ * sizeof(float)));
    int32_t* probes = reinterpret_cast<int32_t*>(carve(nq * P * sizeof(int32_t)));
    int32_t* list_cnt = reinterpret_cast<int32_t*>(carve(nlist_ * sizeof(int32_t)));
    int32_t* cursor = reinterpret_cast<int32_t*>(carve(nlist_ * sizeof(int32_t)));
    int64_t* list_qoff = reinterpret_cast<int64_t*>(carve((nlist_ + 1) * sizeof(int64_t)));
    int64_t* item_off = reinterpret_cast<int64_t*>(carve((nlist_ + 1) * sizeof(int64_t)));
    int32_t* list_q = reinterpret_cast<int32_t*>(carve(nq * P * sizeof(int32_t)));
    int64_t* slot_base = reinterpret_cast<int64_t*>(carve((nq * P + 1) * sizeof(int64_t)));
    const size_t wtmp = build_work_tmp_bytes(nb, P, static_cast<int>(nlist_));
    unsigned char* work_tmp = carve(wtmp);
    uint64_t* part = reinterpret_cast<uint64_t*>(carve(slots * k * sizeof(uint64_t)));
    unsigned int* counter = reinterpret_cast<unsigned int*>(carve(sizeof(unsigned int)));
    if (off > bytes) {
      char msg[200];
      std::snprintf(msg, sizeof(msg),
                    "this search needs %zu bytes of scratch; the fixed scratch holds %zu (use fewer queries, "
                    "a smaller nprobe or k, or hb_search)",
                    off, bytes);
      throw Error(HB_ERR_INVALID, msg);
    }
    launch_pad_rows(q, nq, static_cast<int>(d_), static_cast<int>(dpad_), qpad, st_);
    launch_l2_matrix(qpad, nb, cent_.p, static_cast<int>(nlist_), static_cast<int>(dpad_), dmat,
                     static_cast<int>(nlist_), st_);
    launch_select_rows(dmat, nb, static_cast<int>(nlist_), static_cast<int>(nlist_), P, probes, nullptr, st_);
    const int nbw = launch_build_work(probes, nb, P, list_off_.p, static_cast<int>(nlist_), cr, qg, list_cnt, list_qoff,
                                      cursor, list_q, item_off, slot_base, work_tmp, wtmp, st_);
    HB_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned int), st_));
    ScanArgs a{};
    a.codes = codes_.p;
    a.list_off = list_off_.p;
    a.nlist = static_cast<int>(nlist_);
    a.d = static_cast<int>(d_);
    a.dpad = static_cast<int>(dpad_);
    a.q = qpad;
    a.nq = nb;
    a.P = P;
    a.k = static_cast<int>(k);
    a.list_cnt = list_cnt;
    a.list_qoff = list_qoff;
    a.list_q = list_q;
    a.item_off = item_off;
    a.slot_base = slot_base;
    a.chunk_rows = cr;
    a.qgroup = qg;
    a.work_counter = counter;
    a.part = part;
    a.mode = SCAN_PLAIN;
    a.nseg = 1;
    launch_scan_exact(a, num_sms_, st_);
    launch_merge(part, slot_base, nb, P, static_cast<int>(k), ids_.p, D, I, st_);
    launches_ += 5 + nbw;  // pad, distance matrix, selection, scan, merge, work description
    HB_CUDA(cudaStreamSynchronize(st_));
  }

  int device() const { return device_; }

  // Self-test of the device waits' give-up path: a kernel waits on an
  // mbarrier that nothing arrives on, with a budget of `budget` cycles, and
  // must return with its error code recorded; the host turns the code into
  // HB_ERR_CUDA exactly as after a real scan.
  void wait_selftest(long long budget, long long* waited) {
    HB_CUDA(cudaSetDevice(device_));
    DevBuf<long long> w;
    w.reserve(1);
    err_dev_.reserve(1);
    HB_CUDA(cudaMemsetAsync(err_dev_.p, 0, sizeof(int), st_));
    launch_wait_selftest(budget, 99, err_dev_.p, w.p, st_);
    ++launches_;
    long long wh = 0;
    HB_CUDA(cudaMemcpyAsync(&wh, w.p, sizeof(long long), cudaMemcpyDeviceToHost, st_));
    HB_CUDA(cudaStreamSynchronize(st_));
    if (waited) *waited = wh;
    bf16_err_check();
  }

  void get_centroids(float* out) {
    HB_CUDA(cudaSetDevice(device_));
    HB_CUDA(cudaMemcpy2DAsync(out, d_ * sizeof(float), cent_.p, dpad_ * sizeof(float), d_ * sizeof(float), nlist_,
                              cudaMemcpyDefault, st_));
    HB_CUDA(cudaStreamSynchronize(st_));
  }
  // Keep lists [first, first + count) and empty the others (one rank's share
  // of the reference's DIVIDE_IVF partition, src/Index.cpp:79-104): the kept
  // lists are one contiguous block of rows, moved to the front with their
  // ids (which stay the index's own), norms and offsets.
  void retain_lists(size_t first, size_t count) {
    HB_CHECK(trained_, HB_ERR_STATE, "index not trained");
    HB_CHECK(first <= nlist_ && count <= nlist_ - first, HB_ERR_INVALID, "list range outside the index");
    HB_CUDA(cudaSetDevice(device_));
    const int64_t r0 = host_off_[first], r1 = host_off_[first + count];
    const size_t kept = static_cast<size_t>(r1 - r0);
    if (kept && r0 > 0) {
      DevBuf<float> c;
      DevBuf<int64_t> i;
      DevBuf<float> n;
      c.reserve(kept * dpad_);
      i.reserve(kept);
      n.reserve(kept);
      HB_CUDA(cudaMemcpyAsync(c.p, codes_.p + r0 * dpad_, kept * dpad_ * sizeof(float), cudaMemcpyDeviceToDevice,
                              st_));
      HB_CUDA(cudaMemcpyAsync(i.p, ids_.p + r0, kept * sizeof(int64_t), cudaMemcpyDeviceToDevice, st_));
      HB_CUDA(cudaMemcpyAsync(n.p, norms_.p + r0, kept * sizeof(float), cudaMemcpyDeviceToDevice, st_));
      HB_CUDA(cudaMemcpyAsync(codes_.p, c.p, kept * dpad_ * sizeof(float), cudaMemcpyDeviceToDevice, st_));
      HB_CUDA(cudaMemcpyAsync(ids_.p, i.p, kept * sizeof(int64_t), cudaMemcpyDeviceToDevice, st_));
      HB_CUDA(cudaMemcpyAsync(norms_.p, n.p, kept * sizeof(float), cudaMemcpyDeviceToDevice, st_));
      HB_CUDA(cudaStreamSynchronize(st_));
    }
    for (size_t l = 0; l <= nlist_; ++l) {
      const int64_t o = host_off_[l];
      host_off_[l] = l <= first ? 0 : (l >= first + count ? r1 - r0 : o - r0);
    }
    HB_CUDA(cudaMemcpyAsync(list_off_.p, host_off_.data(), (nlist_ + 1) * sizeof(int64_t), cudaMemcpyHostToDevice,
                            st_));
    HB_CUDA(cudaStreamSynchronize(st_));
    ntotal_ = kept;
    plan_rows_ = 0;
    build_bf16();
    drop_graphs();
  }

  // The reference master's merge of per-worker results (src/Index.cpp:1327-1341)
  // on the index stream; device arrays only.
  void merge_parts(size_t nparts, size_t nq, size_t k, const float* Dp, const int64_t* Ip, float* D, int64_t* I) {
    HB_CHECK(nparts >= 1 && k >= 1, HB_ERR_INVALID, "need at least one part and k >= 1");
    HB_CHECK(is_device_ptr(Dp) && is_device_ptr(Ip) && is_device_ptr(D) && is_device_ptr(I), HB_ERR_INVALID,
             "merge takes device arrays");
    HB_CUDA(cudaSetDevice(device_));
    launch_merge_parts(Dp, Ip, static_cast<int>(nparts), static_cast<int64_t>(nq), static_cast<int>(k), D, I, st_);
    ++launches_;
    HB_CUDA(cudaStreamSynchronize(st_));
  }

  void get_list_sizes(int64_t* out) {
    std::vector<int64_t> s(nlist_);
    for (size_t l = 0; l < nlist_; ++l) s[l] = host_off_[l + 1] - host_off_[l];
    HB_CUDA(cudaMemcpy(out, s.data(), nlist_ * sizeof(int64_t), cudaMemcpyDefault));
  }

 private:
  // Queries per batch: bounded so the coarse matrix and the partial top-k
  // slots stay within a few GB.
  size_t batch_limit(size_t P, size_t k) {
    const size_t by_matrix = std::max<size_t>(1, (size_t(1) << 30) / (nlist_ * sizeof(float)));
    const size_t by_slots = std::max<size_t>(1, (size_t(2) << 30) / (std::max<size_t>(P, 1) * k * 8 * 2));
    return std::max<size_t>(1, std::min<size_t>({size_t(65535), by_matrix, by_slots}));
  }

  // Chunk length of the list scan: keep at least ~4 work items per SM even
  // for tiny batches, and at most 4096 rows per item.
  int chunk_rows_for(int nq, int P, int tv) {
    const double avg = ntotal_ / static_cast<double>(std::max<size_t>(nlist_, 1));
    const long long rows = static_cast<long long>(nq) * P * std::max(avg, 1.0);
    int cr = pow2_floor(std::max<long long>(rows / (4LL * num_sms_), 1));
    cr = std::max(cr, tv);
    cr = std::min(cr, 4096);
    return cr;
  }

  // Upper bound of the output slots of a batch: nq x (sum of the P largest
  // per-list chunk counts).
  size_t max_slots(int nq, int P, int cr) {
    std::vector<int64_t> ch(nlist_);
    for (size_t l = 0; l < nlist_; ++l) ch[l] = (host_off_[l + 1] - host_off_[l] + cr - 1) / cr;
    const size_t take = std::min<size_t>(P, nlist_);
    std::partial_sort(ch.begin(), ch.begin() + take, ch.end(), std::greater<int64_t>());
    int64_t s = 0;
    for (size_t i = 0; i < take; ++i) s += ch[i];
    return static_cast<size_t>(nq) * static_cast<size_t>(std::max<int64_t>(s, 1));
  }

  void search_batch(int nb, int P, int k, int mode, bool cut, bool need_tops, int warm_lists, int warm_size, int W,
                    int B, int qblock, float* Dd, int64_t* Id) {
    int tv = 0, qt = 0, qg = 0;
    const size_t smem = scan_exact_smem_bytes(static_cast<int>(d_), static_cast<int>(dpad_), k, mode, &tv, &qt, &qg);
    HB_CHECK(smem > 0, HB_ERR_INVALID, "k too large for the fused scan at this dimension");
    HB_CHECK(P <= 8192, HB_ERR_INVALID, "nprobe above 8192 is not supported");
    probes_.reserve(static_cast<size_t>(nb) * P);
    coarse_and_cut(nb, P);
    if (need_tops) {
      tops_.reserve(nb);
      if (ext_tops_) {
        HB_CUDA(cudaMemcpyAsync(tops_.p, ext_tops_ + cut_b0_, static_cast<size_t>(nb) * sizeof(float),
                                cudaMemcpyDefault, st_));
      } else {
        Scope sc(this, "warmup_tops");
        launch_warmup_tops(qpad_.p, nb, probes_.p, P, codes_.p, list_off_.p, static_cast<int>(dpad_), k, warm_lists,
                           warm_size, tops_.p, st_);
        ++launches_;
      }
    }
    scan_exact_from(nb, P, k, qpad_.p, probes_.p, mode, cut, need_tops ? tops_.p : nullptr, W, B, qblock, Dd, Id);
  }

  // The exact list scan and merge of nb queries (qpad, nb x dpad) over the
  // probe table `probes` (nb x P).
  void scan_exact_from(int nb, int P, int k, const float* qpad, const int32_t* probes, int mode, bool cut,
                       const float* tops, int W, int B, int qblock, float* Dd, int64_t* Id) {
    int tv = 0, qt = 0, qg = 0;
    const size_t smem = scan_exact_smem_bytes(static_cast<int>(d_), static_cast<int>(dpad_), k, mode, &tv, &qt, &qg);
    HB_CHECK(smem > 0, HB_ERR_INVALID, "k too large for the fused scan at this dimension");
    const int cr = chunk_rows_for(nb, P, tv);
    list_cnt_.reserve(nlist_);
    list_cursor_.reserve(nlist_);
    list_qoff_.reserve(nlist_ + 1);
    item_off_.reserve(nlist_ + 1);
    list_q_.reserve(static_cast<size_t>(nb) * P);
    slot_base_.reserve(static_cast<size_t>(nb) * P + 1);
    const size_t wtmp = build_work_tmp_bytes(nb, P, static_cast<int>(nlist_));
    work_tmp_.reserve(wtmp);
    {
      Scope sc(this, "build_work");
      launches_ += launch_build_work(probes, nb, P, list_off_.p, static_cast<int>(nlist_), cr, qg, list_cnt_.p,
                                     list_qoff_.p, list_cursor_.p, list_q_.p, item_off_.p, slot_base_.p, work_tmp_.p,
                                     wtmp, st_);
    }
    part_.reserve(max_slots(nb, P, cr) * static_cast<size_t>(k));
    counter_.reserve(1);
    HB_CUDA(cudaMemsetAsync(counter_.p, 0, sizeof(unsigned int), st_));
    ScanArgs a{};
    a.codes = codes_.p;
    a.list_off = list_off_.p;
    a.nlist = static_cast<int>(nlist_);
    a.d = static_cast<int>(d_);
    a.dpad = static_cast<int>(dpad_);
    a.q = qpad;
    a.nq = nb;
    a.P = P;
    a.k = k;
    a.list_cnt = list_cnt_.p;
    a.list_qoff = list_qoff_.p;
    a.list_q = list_q_.p;
    a.item_off = item_off_.p;
    a.slot_base = slot_base_.p;
    a.chunk_rows = cr;
    a.qgroup = qg;
    a.work_counter = counter_.p;
    a.part = part_.p;
    a.mode = mode;
    a.tops = tops;
    a.cut = cut ? 1 : 0;
    a.nseg = W;
    a.seg_order = order_dev_.p;
    a.qblock = qblock;
    a.nblocks = B;
    {
      Scope sc(this, "scan_exact");
      launch_scan_exact(a, num_sms_, st_);
    }
    Scope sc(this, "merge");
    launch_merge(part_.p, slot_base_.p, nb, P, k, ids_.p, Dd, Id, st_);
    launches_ += 2;
  }

  // Candidate buffer per query of the bounded BF16 scan: room for 16 k
  // candidates (at least 2048), rounded up to a power of two (the re-rank
  // sorts a buffer in place); a query needing more is searched again with the
  // exact scan.
  static int filter_cap(size_t k) {
    size_t c = 4096;
    while (c < 16 * k) c <<= 1;
    return static_cast<int>(std::min<size_t>(kRerankMaxCap, c));
  }

  // BF16 search of one batch, equal to the exact FP32 scan bit for bit: exact
  // coarse probes, per-query BF16 rows / error bounds, the list-major work
  // description, a per-query admission bound seeded from the nearest list,
  // one tensor-core pass appending the rows under each query's bound, then
  // the exact re-rank of the rows under W_k + 2 eps.  Queries whose candidate
  // buffer overflowed are searched again with the exact scan.
  void search_batch_bf16(int nb, int P, int k, int R, float* Dd, int64_t* Id) {
    if (cand_path_) {
      search_batch_cand(nb, P, k, R, Dd, Id);
      return;
    }
    probes_.reserve(static_cast<size_t>(nb) * P);
    coarse_and_cut(nb, P);
    err_dev_.reserve(1);
    HB_CUDA(cudaMemsetAsync(err_dev_.p, 0, sizeof(int), st_));
    const int cap = filter_cap(k);
    thr_.reserve(nb);
    ccnt_.reserve(nb);
    cflag_.reserve(nb);
    rr_m_.reserve(nb);
    over_list_.reserve(2 * static_cast<size_t>(nb));
    last_nb_ = nb;
    over_n_.reserve(2);
    cbuf_.reserve(static_cast<size_t>(nb) * cap);
    cbuf_ub_.reserve(static_cast<size_t>(nb) * cap);
    const int cr0 = std::max(128, chunk_rows_for(nb, P, 128));
    const int s0 = scan_bf16_stages(kpad_);
    const TuneKey key = tune_key(nb, P, k);
    if (autotune_ && !capturing_ && !tune_.count(key)) autotune(nb, P, k, cap, Dd, Id, key, cr0, s0);
    const auto it = tune_.find(key);
    const int cr = it != tune_.end() ? it->second.chunk_rows : cr0;
    const int stages = it != tune_.end() ? it->second.stages : s0;
    filter_pipeline(nb, P, k, cap, cr, stages, Dd, Id);
    if (!capturing_) {
      bf16_err_check();
      fix_overflow(nb, P, k, Dd, Id);
    }
  }

  // The bounded scan of one batch after the coarse probes: per-query prep,
  // work description (chunks of cr rows), seed bounds, the scan with a ring
  // of `stages` B tiles, and the exact re-rank.  For k > kFilterTightK the
  // scan runs in two stages: every query's nearest list first, whose k-th
  // admitted value bounds the second stage over the other lists.  Every
  // (cr, stages) gives the same result.
  void filter_pipeline(int nb, int P, int k, int cap, int cr, int stages, float* Dd, int64_t* Id) {
    HB_CUDA(cudaMemsetAsync(over_n_.p, 0, 2 * sizeof(int), st_));
    {
      Scope sc(this, "query_prep");
      launch_query_prep(nb, thr_.p, ccnt_.p, st_);
    }
    list_cnt_.reserve(nlist_);
    list_cursor_.reserve(nlist_);
    list_qoff_.reserve(nlist_ + 1);
    item_off_.reserve(nlist_ + 1);
    list_q_.reserve(static_cast<size_t>(nb) * P);
    const size_t wtmp = build_work_tmp_bytes(nb, P, static_cast<int>(nlist_));
    work_tmp_.reserve(wtmp);
    const bool two_stage = k > kFilterTightK && P > 1;
    const int32_t* probes_a = probes_.p;
    int P_a = P, cr_a = cr;
    if (two_stage) {
      probe0_.reserve(static_cast<size_t>(nb));
      probes_rest_.reserve(static_cast<size_t>(nb) * P);
      launch_split_first_probe(probes_.p, nb, P, probe0_.p, probes_rest_.p, st_);
      probes_a = probe0_.p;
      P_a = 1;
      cr_a = std::max(128, chunk_rows_for(nb, 1, 128));
      launches_ += 1;
    }
    {
      Scope sc(this, "build_work");
      launches_ += launch_build_work(probes_a, nb, P_a, list_off_.p, static_cast<int>(nlist_), cr_a, 128, list_cnt_.p,
                                     list_qoff_.p, list_cursor_.p, list_q_.p, item_off_.p, nullptr, work_tmp_.p, wtmp,
                                     st_);
    }
    {
      Scope sc(this, "seed");
      launch_seed_bound(qpad_.p, static_cast<int>(d_), static_cast<int>(dpad_), cent_.p, nb, kpad_, codes_bf16_.p,
                        list_off_.p, static_cast<int>(nlist_), list_qoff_.p, list_q_.p, rnorm_.p, rmax_.p,
                        std::max(seed_rows_, k), k, thr_.p, st_, probes_a, P_a);
    }
    counter_.reserve(1);
    HB_CUDA(cudaMemsetAsync(counter_.p, 0, sizeof(unsigned int), st_));
    TcArgs a{};
    a.list_off = list_off_.p;
    a.nlist = static_cast<int>(nlist_);
    a.kpad = kpad_;
    a.q = qpad_.p;
    a.dpad = static_cast<int>(dpad_);
    a.cent = cent_.p;
    a.tile_norm = tile_norm_.p;
    a.tile_off = tile_off_.p;
    a.list_cnt = list_cnt_.p;
    a.list_qoff = list_qoff_.p;
    a.list_q = list_q_.p;
    a.item_off = item_off_.p;
    a.chunk_rows = cr_a;
    a.work_counter = counter_.p;
    a.thr = thr_.p;
    a.rmax = rmax_.p;
    a.cand = cbuf_.p;
    a.cand_ub = cbuf_ub_.p;
    a.cand_cnt = ccnt_.p;
    a.cap = cap;
    a.k = k;
    a.err = err_dev_.p;
    a.stages = stages;
    a.wait_budget = wait_budget_;
    {
      Scope sc(this, "scan_bf16");
      launch_scan_bf16(tmap_, a, num_sms_, st_);
    }
    if (two_stage) {
      // Second stage: the other lists, appended to the same buffers.
      {
        Scope sc(this, "kth_bound");
        launch_kth_bound(cbuf_ub_.p, ccnt_.p, cap, nb, k, thr_.p, st_);
      }
      {
        Scope sc(this, "build_work");
        launches_ += launch_build_work(probes_rest_.p, nb, P, list_off_.p, static_cast<int>(nlist_), cr, 128,
                                       list_cnt_.p, list_qoff_.p, list_cursor_.p, list_q_.p, item_off_.p, nullptr,
                                       work_tmp_.p, wtmp, st_);
      }
      HB_CUDA(cudaMemsetAsync(counter_.p, 0, sizeof(unsigned int), st_));
      a.chunk_rows = cr;
      {
        Scope sc(this, "scan_bf16");
        launch_scan_bf16(tmap_, a, num_sms_, st_);
      }
      launches_ += 2;  // kth_bound, the second scan
    }
    {
      Scope sc(this, "rerank");
      launch_rerank_bf16(cbuf_.p, cbuf_ub_.p, ccnt_.p, cap, nb, k, codes_.p, qpad_.p, static_cast<int>(dpad_), ids_.p, Dd,
                         Id, cflag_.p, over_list_.p, over_n_.p, rr_m_.p, num_sms_, st_);
    }
    // query prep, seed, scan, warp re-rank, and the three flat re-rank
    // kernels when the buffers can hold more than a warp's candidates.
    launches_ += 4 + (cap > 256 ? 3 : 0);
  }

  // ---- autotuner of the bounded scan ----------------------------------------
  // Per (batch-size bucket, nprobe bucket, k) the first search times the scan
  // pipeline for chunk lengths around the default (x1/4 .. x4, 128 .. 4096
  // rows) and ring depths 2..4, twice each, and keeps the fastest; later
  // searches of the bucket use it.  The table can be read and written as text
  // ("nb_bucket P_bucket k kpad chunk_rows stages best_ms default_ms" lines).
  struct TuneKey {
    int nb_bucket, p_bucket, k;
    bool operator<(const TuneKey& o) const {
      return std::tie(nb_bucket, p_bucket, k) < std::tie(o.nb_bucket, o.p_bucket, o.k);
    }
  };
  struct TuneChoice {
    int chunk_rows, stages;
    float best_ms, default_ms;
  };
  static int pow2_bucket(int x) {
    int b = 1;
    while (b < x) b <<= 1;
    return b;
  }
  TuneKey tune_key(int nb, int P, int k) const { return {pow2_bucket(nb), pow2_bucket(P), k}; }

  void autotune(int nb, int P, int k, int cap, float* Dd, int64_t* Id, const TuneKey& key, int cr0, int s0) {
    std::vector<int> crs;
    for (int f : {-2, -1, 0, 1, 2}) {
      int c = f < 0 ? cr0 >> (-f) : cr0 << f;
      c = std::min(4096, std::max(128, c));
      if (std::find(crs.begin(), crs.end(), c) == crs.end()) crs.push_back(c);
    }
    cudaEvent_t e0 = event(), e1 = event();
    TuneChoice best{cr0, s0, 1e30f, 0.0f};
    for (int S = 2; S <= 4; ++S) {
      if (scan_bf16_smem_bytes(kpad_, S) > scan_bf16_smem_bytes(kpad_, s0) && S > s0) continue;
      for (int c : crs) {
        float ms = 1e30f;
        for (int rep = 0; rep < 2; ++rep) {
          HB_CUDA(cudaEventRecord(e0, st_));
          filter_pipeline(nb, P, k, cap, c, S, Dd, Id);
          HB_CUDA(cudaEventRecord(e1, st_));
          HB_CUDA(cudaEventSynchronize(e1));
          float t = 0.f;
          HB_CUDA(cudaEventElapsedTime(&t, e0, e1));
          ms = std::min(ms, t);
        }
        if (c == cr0 && S == s0) best.default_ms = ms;
        if (ms < best.best_ms) {
          best.best_ms = ms;
          best.chunk_rows = c;
          best.stages = S;
        }
      }
    }
    ev_pool_.push_back(e0);
    ev_pool_.push_back(e1);
    bf16_err_check();
    tune_[key] = best;
  }

 public:
  void set_autotune(bool on) { autotune_ = on; }
  std::string autotune_table() const {
    std::string out;
    char line[160];
    for (const auto& kv : tune_) {
      std::snprintf(line, sizeof(line), "%d %d %d %d %d %d %.4f %.4f\n", kv.first.nb_bucket, kv.first.p_bucket,
                    kv.first.k, kpad_, kv.second.chunk_rows, kv.second.stages, kv.second.best_ms,
                    kv.second.default_ms);
      out += line;
    }
    return out;
  }
  void set_autotune_table(const char* text) {
    std::map<TuneKey, TuneChoice> t;
    const char* p = text;
    while (p && *p) {
      TuneKey key{};
      TuneChoice c{};
      int kp = 0, used = 0;
      if (std::sscanf(p, "%d %d %d %d %d %d %f %f%n", &key.nb_bucket, &key.p_bucket, &key.k, &kp, &c.chunk_rows,
                      &c.stages, &c.best_ms, &c.default_ms, &used) != 8)
        throw Error(HB_ERR_INVALID, "autotune table: expected 8 numbers per line");
      HB_CHECK(c.chunk_rows >= 128 && c.chunk_rows <= 4096 && c.chunk_rows % 128 == 0 && c.stages >= 2 &&
                   c.stages <= 4 && key.k >= 1,
               HB_ERR_INVALID, "autotune table: value out of range");
      if (kp == kpad_) t[key] = c;
      p += used;
      while (*p == '\n' || *p == ' ' || *p == '\r') ++p;
    }
    tune_ = t;
  }

 private:


  // Queries whose candidate buffer overflowed (listed by the re-rank, left
  // unwritten) are searched with the exact scan over their own probe rows,
  // and their result rows are written into Dd / Id.
  void fix_overflow(int nb, int P, int k, float* Dd, int64_t* Id) {
    int n_over = 0;
    HB_CUDA(cudaMemcpyAsync(err_host_, over_n_.p, sizeof(int), cudaMemcpyDeviceToHost, st_));
    HB_CUDA(cudaStreamSynchronize(st_));
    n_over = *err_host_;
    last_overflow_ = n_over;
    if (n_over <= 0) return;
    HB_CHECK(n_over <= nb, HB_ERR_CUDA, "overflow list longer than the batch");
    Scope sc(this, "overflow_exact");
    const int dp = static_cast<int>(dpad_);
    oq_.reserve(static_cast<size_t>(n_over) * dpad_);
    op_.reserve(static_cast<size_t>(n_over) * P);
    od_.reserve(static_cast<size_t>(n_over) * k);
    oi_.reserve(static_cast<size_t>(n_over) * k);
    launch_gather_words(reinterpret_cast<const uint32_t*>(qpad_.p), over_list_.p, n_over, dp,
                        reinterpret_cast<uint32_t*>(oq_.p), st_);
    launch_gather_words(reinterpret_cast<const uint32_t*>(probes_.p), over_list_.p, n_over, P,
                        reinterpret_cast<uint32_t*>(op_.p), st_);
    scan_exact_from(n_over, P, k, oq_.p, op_.p, SCAN_PLAIN, false, nullptr, 1, 1, 0, od_.p, oi_.p);
    launch_scatter_words(reinterpret_cast<const uint32_t*>(od_.p), over_list_.p, n_over, k,
                         reinterpret_cast<uint32_t*>(Dd), st_);
    launch_scatter_words(reinterpret_cast<const uint32_t*>(oi_.p), over_list_.p, n_over, 2 * k,
                         reinterpret_cast<uint32_t*>(Id), st_);
    launches_ += 4;
  }

  // Longest candidate row a query can have at nprobe P: the P largest lists,
  // each rounded up to 4 entries.
  int64_t cand_row_bound(int P) {
    std::vector<int64_t> n(nlist_);
    for (size_t l = 0; l < nlist_; ++l) n[l] = (host_off_[l + 1] - host_off_[l] + 3) & ~int64_t(3);
    const size_t take = std::min<size_t>(static_cast<size_t>(P), nlist_);
    std::partial_sort(n.begin(), n.begin() + take, n.end(), std::greater<int64_t>());
    int64_t s = 0;
    for (size_t i = 0; i < take; ++i) s += n[i];
    return s;
  }

  // Queries per batch of the candidate-matrix scan: at most 2^30 candidate
  // entries (4 GiB) and 2 GiB of gathered BF16 queries.
  size_t cand_batch_limit(size_t P) {
    const int64_t L = std::max<int64_t>(cand_row_bound(static_cast<int>(P)), 1);
    HB_CHECK(L <= (int64_t(1) << 30), HB_ERR_INVALID, "candidate row of one query above 2^30 entries");
    const size_t by_cand = static_cast<size_t>((int64_t(1) << 30) / L);
    const size_t by_q = (size_t(2) << 30) / (P * static_cast<size_t>(kpad_) * 2);
    return std::max<size_t>(1, std::min(by_cand, by_q));
  }

  // BF16 search of one batch through the candidate matrix: exact coarse
  // probes, the list-major work description, every probed row's
  // approximate value on the tensor cores, then per query the R smallest
  // re-ranked exactly.
  void search_batch_cand(int nb, int P, int k, int R, float* Dd, int64_t* Id) {
    probes_.reserve(static_cast<size_t>(nb) * P);
    coarse_and_cut(nb, P);
    err_dev_.reserve(1);
    HB_CUDA(cudaMemsetAsync(err_dev_.p, 0, sizeof(int), st_));
    // One 128-row tile per work item: the queries' tile is fetched per row
    // tile anyway, and small items balance the persistent CTAs.
    const int cr = 128;
    const size_t nqp = static_cast<size_t>(nb) * P;
    list_cnt_.reserve(nlist_);
    list_cursor_.reserve(nlist_);
    list_qoff_.reserve(nlist_ + 1);
    item_off_.reserve(nlist_ + 1);
    list_q_.reserve(nqp);
    slot_base_.reserve(nqp + 1);
    const size_t wtmp = std::max(build_work_tmp_bytes(nb, P, static_cast<int>(nlist_)), cand_segments_tmp_bytes(nb, P));
    work_tmp_.reserve(wtmp);
    {
      Scope sc(this, "build_work");
      launches_ += launch_build_work(probes_.p, nb, P, list_off_.p, static_cast<int>(nlist_), cr, 128, list_cnt_.p,
                                     list_qoff_.p, list_cursor_.p, list_q_.p, item_off_.p, slot_base_.p, work_tmp_.p,
                                     wtmp, st_);
    }
    seg_.reserve(nqp + 1);
    {
      Scope sc(this, "cand_segments");
      launch_cand_segments(probes_.p, nb, P, list_off_.p, seg_.p, work_tmp_.p, wtmp, st_);
    }
    launches_ += 2;
    if (fp8_) {
      ensure_fp8();
      qscale8_.reserve(nqp);
      qcd8_.reserve(nqp);
      gq8_.reserve(nqp * static_cast<size_t>(kpad8_));
      Scope sc(this, "gather_queries");
      launch_gather_residual(qpad_.p, static_cast<int>(dpad_), kpad8_, true, list_q_.p, list_qoff_.p,
                             static_cast<int>(nlist_), cent_.p, static_cast<int64_t>(nqp), qscale8_.p, qcd8_.p,
                             gq8_.p, st_);
      make_u8_tensor_map(gqmap_, gq8_.p, nqp, kpad8_);
      ++launches_;
    } else {
      gq_.reserve(nqp * static_cast<size_t>(kpad_));
      qcd8_.reserve(nqp);
      Scope sc(this, "gather_queries");
      launch_gather_residual(qpad_.p, static_cast<int>(dpad_), kpad_, false, list_q_.p, list_qoff_.p,
                             static_cast<int>(nlist_), cent_.p, static_cast<int64_t>(nqp), nullptr, qcd8_.p, gq_.p,
                             st_);
      make_bf16_tensor_map(gqmap_, gq_.p, nqp, kpad_);
      ++launches_;
    }
    const int64_t row_bound = cand_row_bound(P);
    cand_.reserve(std::max<size_t>(static_cast<size_t>(nb) * row_bound, 1));
    cand_rows_.reserve(static_cast<size_t>(nb) * R);
    CandArgs a{};
    a.list_off = list_off_.p;
    a.nlist = static_cast<int>(nlist_);
    a.kpad = kpad_;
    a.tile_norm = tile_norm_.p;
    a.tile_off = tile_off_.p;
    a.list_cnt = list_cnt_.p;
    a.list_qoff = list_qoff_.p;
    a.list_q = list_q_.p;
    a.item_off = item_off_.p;
    a.chunk_rows = cr;
    a.P = P;
    a.seg = seg_.p;
    a.cand = cand_.p;
    a.err = err_dev_.p;
    a.qcd = qcd8_.p;
    if (fp8_) {
      a.fp8 = 1;
      a.kpad = kpad8_;
      a.qscale = qscale8_.p;
      a.list_scale = list_scale8_.p;
      a.tile_norm = tile_rnorm8_.p;
    }
    {
      Scope sc(this, "cand_scan");
      launch_cand_scan(gqmap_, fp8_ ? tmap8_ : tmap_, a, num_sms_, st_);
    }
    ++launches_;
    {
      Scope sc(this, "cand_select");
      launch_cand_select(cand_.p, seg_.p, probes_.p, nb, P, R, list_off_.p, cand_rows_.p, st_);
    }
    {
      Scope sc(this, "cand_exact");
      launch_cand_exact(cand_rows_.p, nb, R, k, codes_.p, qpad_.p, static_cast<int>(dpad_), ids_.p, Dd, Id, st_);
    }
    launches_ += 2;
    if (!capturing_) bf16_err_check();
  }

  void bf16_err_check() {
    HB_CUDA(cudaMemcpyAsync(err_host_, err_dev_.p, sizeof(int), cudaMemcpyDeviceToHost, st_));
    HB_CUDA(cudaStreamSynchronize(st_));
    if (*err_host_ != 0)
      throw Error(HB_ERR_CUDA, "tensor-core scan gave up waiting (code " + std::to_string(*err_host_) + ")");
  }

  // Coarse probes of the batch in qpad_, then the per-query cut.
  void coarse_and_cut(int nb, int P) {
    if (cut_mode_ == 1 && coarse_tc_route(P) && probe_.C <= P) {
      coarse_learned(qpad_.p, nb, P, probes_.p, cut_thr_, cut_cap_);
    } else if (cut_mode_ == 1) {
      cdist_.reserve(static_cast<size_t>(nb) * P);
      coarse(qpad_.p, nb, P, probes_.p, cdist_.p);
      Scope sc(this, "probe_mlp");
      probe_infer(nb, qpad_.p, cdist_.p, P, probes_.p, cut_thr_, cut_cap_, nullptr);
    } else {
      coarse(qpad_.p, nb, P, probes_.p, nullptr);
      if (cut_mode_ == 2) {
        npq_.reserve(static_cast<size_t>(nb));
        HB_CUDA(cudaMemcpyAsync(npq_.p, cut_src_ + cut_b0_, static_cast<size_t>(nb) * sizeof(int32_t), cudaMemcpyDefault,
                                st_));
        launch_cut_probes(npq_.p, nb, P, probes_.p, st_);
        ++launches_;
      }
    }
  }

  // ---- learned probe predictor ------------------------------------------------
  struct ProbeModel {
    bool trained = false;
    int F = 0, H = 256, NB = 0, C = 32, pmax = 0;
    std::vector<int32_t> buckets;
    DevBuf<float> W1, B1, W2, B2, W3, B3;  // BF16-rounded inference weights
    DevBuf<uint16_t> W1b, W2b, W3b;        // the same, packed BF16 for the tensor cores
    int K1 = 0;
    bool tc = false;
    DevBuf<float> mean, inv_std;
    DevBuf<int32_t> bucket_val;
    std::vector<float> cal_thr, cal_recall, cal_avgp;
    float thr = 1.0f;
    // Smallest-average-nprobe threshold whose validation recall reaches the
    // target (the trained one for target 0).
    float threshold_for(float target) const {
      if (target <= 0.f) return thr;
      float best = 1.0f, bestp = 1e30f;
      for (size_t i = 0; i < cal_thr.size(); ++i)
        if (cal_recall[i] >= target && cal_avgp[i] < bestp) {
          bestp = cal_avgp[i];
          best = cal_thr[i];
        }
      return best;
    }
  };

  // Features -> 3 GEMMs (BF16 weights and activations, FP32 accumulation)
  // -> per-query nprobe; probes (nb x P) are cut in place.
  void probe_infer(int nb, const float* qpad, const float* cdist, int P, int32_t* probes, float thr, int cap,
                   int32_t* nprobe_out) {
    ProbeModel& m = probe_;
    if (m.tc) {
      if (!cerr_dev_.p) {
        cerr_dev_.reserve(1);
        HB_CUDA(cudaMemsetAsync(cerr_dev_.p, 0, sizeof(int), st_));
      }
      int32_t* np = nprobe_out;
      if (!np) {
        npq_.reserve(static_cast<size_t>(nb));
        np = npq_.p;
      }
      mlp_infer_tc(qpad, nb, static_cast<int>(d_), static_cast<int>(dpad_), cdist, P, m.C, m.mean.p, m.inv_std.p, m.K1,
                   m.W1b.p, m.B1.p, m.W2b.p, m.B2.p, m.W3b.p, m.B3.p, m.NB, m.bucket_val.p, thr, cap, np,
                   cerr_dev_.p, st_);
      ++launches_;
      if (probes) {
        launch_cut_probes(np, nb, P, probes, st_);
        ++launches_;
      }
      return;
    }
    pf_.reserve(static_cast<size_t>(nb) * m.F);
    ph1_.reserve(static_cast<size_t>(nb) * m.H);
    ph2_.reserve(static_cast<size_t>(nb) * m.H);
    plog_.reserve(static_cast<size_t>(nb) * m.NB);
    mlp_features(qpad, nb, static_cast<int>(d_), static_cast<int>(dpad_), cdist, P, m.C, pf_.p, st_);
    mlp_standardize(pf_.p, nb, m.F, m.mean.p, m.inv_std.p, true, st_);
    mlp_gemm(nb, m.H, m.F, pf_.p, m.F, false, m.W1.p, m.F, true, ph1_.p, m.H, m.B1.p, 0.f, true, nullptr, true, st_);
    mlp_gemm(nb, m.H, m.H, ph1_.p, m.H, false, m.W2.p, m.H, true, ph2_.p, m.H, m.B2.p, 0.f, true, nullptr, true, st_);
    mlp_gemm(nb, m.NB, m.H, ph2_.p, m.H, false, m.W3.p, m.H, true, plog_.p, m.NB, m.B3.p, 0.f, false, nullptr, false,
             st_);
    mlp_choose_nprobe(plog_.p, nb, m.NB, m.bucket_val.p, thr, cap, nprobe_out, probes, P, st_);
    launches_ += 6;
  }

 public:
  // Trains the predictor on nt queries labelled by the exact FP32 search at
  // nprobe = label_P: a query's label is the smallest nprobe that finds its
  // k results (1 + the highest probe rank among their lists).  90% of the
  // queries train the MLP (Adam), 10% calibrate the probability threshold
  // to the recall target.
  void train_probe(size_t nt, const float* q, size_t k, size_t label_P, float target) {
    HB_CUDA(cudaSetDevice(device_));
    HB_CHECK(ntotal_ > 0, HB_ERR_STATE, "train the probe predictor after add");
    HB_CHECK(nt >= 1000, HB_ERR_INVALID, "at least 1000 training queries");
    HB_CHECK(label_P >= 32 && label_P <= nlist_, HB_ERR_INVALID, "label nprobe must be in [32, nlist]");
    HB_CHECK(target > 0.f && target <= 1.f, HB_ERR_INVALID, "target recall must be in (0, 1]");
    HB_CHECK(k >= 1 && k <= 64, HB_ERR_INVALID, "k must be in [1, 64]");
    ProbeModel& m = probe_;
    const int P = static_cast<int>(label_P);
    m.C = 32;
    m.F = static_cast<int>(d_) + m.C;
    m.H = 256;
    m.buckets.clear();
    for (int b : {1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256, 384, 512, 768, 1024, 1536, 2048})
      if (b < P) m.buckets.push_back(b);
    m.buckets.push_back(P);
    m.NB = static_cast<int>(m.buckets.size());
    m.pmax = P;
    m.trained = false;
    // Labels from the plain exact search.
    DevBuf<float> Dtr;
    DevBuf<int64_t> Itr;
    Dtr.reserve(nt * k);
    Itr.reserve(nt * k);
    const size_t saved = nprobe_;
    nprobe_ = label_P;
    hb_search_params sp;
    hb_search_params_init(&sp);
    search(nt, q, k, &sp, Dtr.p, Itr.p);
    nprobe_ = saved;
    // Probe tables with distances, and padded queries, for all nt.
    DevBuf<float> qall, tmp, cd;
    DevBuf<int32_t> pr;
    stage_rows(q, nt, qall, tmp);
    tmp.release();
    pr.reserve(nt * P);
    cd.reserve(nt * P);
    const size_t cb = std::max<size_t>(1, (size_t(1) << 30) / (nlist_ * sizeof(float)));
    for (size_t b0 = 0; b0 < nt; b0 += cb) {
      const int nb = static_cast<int>(std::min(cb, nt - b0));
      coarse(qall.p + b0 * dpad_, nb, P, pr.p + b0 * P, cd.p + b0 * P);
    }
    // id -> list, labels and per-result probe ranks.
    std::vector<int64_t> ids_h(ntotal_);
    HB_CUDA(cudaMemcpyAsync(ids_h.data(), ids_.p, ntotal_ * sizeof(int64_t), cudaMemcpyDeviceToHost, st_));
    HB_CUDA(cudaStreamSynchronize(st_));
    coarse_err_check();
    int64_t max_id = 0;
    for (int64_t v : ids_h) max_id = std::max(max_id, v);
    DevBuf<int32_t> lid, need, ranks;
    lid.reserve(static_cast<size_t>(max_id) + 1);
    HB_CUDA(cudaMemsetAsync(lid.p, 0xff, (static_cast<size_t>(max_id) + 1) * sizeof(int32_t), st_));
    launch_list_of_id(list_off_.p, static_cast<int>(nlist_), ids_.p, lid.p, max_id + 1, st_);
    need.reserve(nt);
    ranks.reserve(nt * k);
    launch_label_rank(Itr.p, static_cast<int>(nt), static_cast<int>(k), lid.p, pr.p, P, need.p, ranks.p, st_);
    // Features.
    DevBuf<float> X;
    X.reserve(nt * m.F);
    mlp_features(qall.p, static_cast<int>(nt), static_cast<int>(d_), static_cast<int>(dpad_), cd.p, P, m.C, X.p, st_);
    m.mean.reserve(m.F);
    m.inv_std.reserve(m.F);
    mlp_moments(X.p, static_cast<int>(nt), m.F, m.mean.p, m.inv_std.p, st_);
    mlp_standardize(X.p, static_cast<int>(nt), m.F, m.mean.p, m.inv_std.p, false, st_);
    std::vector<int32_t> need_h(nt), ranks_h(nt * k);
    HB_CUDA(cudaMemcpyAsync(need_h.data(), need.p, nt * sizeof(int32_t), cudaMemcpyDeviceToHost, st_));
    HB_CUDA(cudaMemcpyAsync(ranks_h.data(), ranks.p, nt * k * sizeof(int32_t), cudaMemcpyDeviceToHost, st_));
    HB_CUDA(cudaStreamSynchronize(st_));
    std::vector<int32_t> y(nt);
    for (size_t i = 0; i < nt; ++i) {
      int b = 0;
      while (b < m.NB - 1 && m.buckets[b] < need_h[i]) ++b;
      y[i] = b;
    }
    const size_t nval = std::max<size_t>(500, nt / 10);
    const size_t ntr = nt - nval;
    // Parameters: Kaiming-uniform, fixed seed.
    const int F = m.F, H = m.H, NB = m.NB;
    const size_t n1 = static_cast<size_t>(H) * F, n2 = static_cast<size_t>(H) * H, n3 = static_cast<size_t>(NB) * H;
    const size_t nparam = n1 + H + n2 + H + n3 + NB;
    std::vector<float> w0(nparam, 0.f);
    std::mt19937 rng(1234);
    auto fill = [&](size_t off, size_t n, int fan_in) {
      std::uniform_real_distribution<float> u(-std::sqrt(6.f / fan_in), std::sqrt(6.f / fan_in));
      for (size_t i = 0; i < n; ++i) w0[off + i] = u(rng);
    };
    fill(0, n1, F);
    fill(n1 + H, n2, H);
    fill(n1 + H + n2 + H, n3, H);
    DevBuf<float> W, G, Mo, Vo;
    W.reserve(nparam);
    G.reserve(nparam);
    Mo.reserve(nparam);
    Vo.reserve(nparam);
    HB_CUDA(cudaMemcpyAsync(W.p, w0.data(), nparam * sizeof(float), cudaMemcpyHostToDevice, st_));
    HB_CUDA(cudaMemsetAsync(Mo.p, 0, nparam * sizeof(float), st_));
    HB_CUDA(cudaMemsetAsync(Vo.p, 0, nparam * sizeof(float), st_));
    float *w1 = W.p, *b1 = w1 + n1, *w2 = b1 + H, *b2 = w2 + n2, *w3 = b2 + H, *b3 = w3 + n3;
    float *g1 = G.p, *gb1 = g1 + n1, *g2 = gb1 + H, *gb2 = g2 + n2, *g3 = gb2 + H, *gb3 = g3 + n3;
    const int B = 2048;
    DevBuf<float> Xb, Z1, A1, Z2, A2, L, dL, dA, dZ, loss;
    DevBuf<int32_t> yb;
    DevBuf<int64_t> perm_d;
    Xb.reserve(static_cast<size_t>(B) * F);
    Z1.reserve(static_cast<size_t>(B) * H);
    A1.reserve(static_cast<size_t>(B) * H);
    Z2.reserve(static_cast<size_t>(B) * H);
    A2.reserve(static_cast<size_t>(B) * H);
    L.reserve(static_cast<size_t>(B) * NB);
    dL.reserve(static_cast<size_t>(B) * NB);
    dA.reserve(static_cast<size_t>(B) * H);
    dZ.reserve(static_cast<size_t>(B) * H);
    loss.reserve(1);
    yb.reserve(ntr);
    perm_d.reserve(ntr);
    DevBuf<float> Xs;
    Xs.reserve(ntr * F);
    std::vector<int64_t> perm(ntr);
    std::vector<int32_t> yperm(ntr);
    const int epochs = 12;
    int step = 0;
    const float lr = 2e-3f;
    for (int ep = 0; ep < epochs; ++ep) {
      std::iota(perm.begin(), perm.end(), 0);
      std::shuffle(perm.begin(), perm.end(), std::mt19937(777 + ep));
      for (size_t i = 0; i < ntr; ++i) yperm[i] = y[perm[i]];
      HB_CUDA(cudaMemcpyAsync(perm_d.p, perm.data(), ntr * sizeof(int64_t), cudaMemcpyHostToDevice, st_));
      HB_CUDA(cudaMemcpyAsync(yb.p, yperm.data(), ntr * sizeof(int32_t), cudaMemcpyHostToDevice, st_));
      launch_gather_rows(X.p, perm_d.p, ntr, F, Xs.p, st_);
      const float lr_ep = lr * (ep < epochs - 4 ? 1.f : 0.25f);
      for (size_t r0 = 0; r0 + B <= ntr; r0 += B, ++step) {
        const float* xb = Xs.p + r0 * F;
        HB_CUDA(cudaMemsetAsync(loss.p, 0, sizeof(float), st_));
        mlp_gemm(B, H, F, xb, F, false, w1, F, true, A1.p, H, b1, 0.f, true, Z1.p, false, st_);
        mlp_gemm(B, H, H, A1.p, H, false, w2, H, true, A2.p, H, b2, 0.f, true, Z2.p, false, st_);
        mlp_gemm(B, NB, H, A2.p, H, false, w3, H, true, L.p, NB, b3, 0.f, false, nullptr, false, st_);
        mlp_softmax_ce(L.p, yb.p + r0, B, NB, dL.p, loss.p, st_);
        // layer 3
        mlp_gemm(NB, H, B, dL.p, NB, true, A2.p, H, false, g3, H, nullptr, 0.f, false, nullptr, false, st_);
        mlp_colsum(dL.p, B, NB, gb3, st_);
        mlp_gemm(B, H, NB, dL.p, NB, false, w3, H, false, dA.p, H, nullptr, 0.f, false, nullptr, false, st_);
        mlp_gelu_backward(dA.p, Z2.p, dZ.p, static_cast<size_t>(B) * H, st_);
        // layer 2
        mlp_gemm(H, H, B, dZ.p, H, true, A1.p, H, false, g2, H, nullptr, 0.f, false, nullptr, false, st_);
        mlp_colsum(dZ.p, B, H, gb2, st_);
        mlp_gemm(B, H, H, dZ.p, H, false, w2, H, false, dA.p, H, nullptr, 0.f, false, nullptr, false, st_);
        mlp_gelu_backward(dA.p, Z1.p, dZ.p, static_cast<size_t>(B) * H, st_);
        // layer 1
        mlp_gemm(H, F, B, dZ.p, H, true, xb, F, false, g1, F, nullptr, 0.f, false, nullptr, false, st_);
        mlp_colsum(dZ.p, B, H, gb1, st_);
        mlp_adam(W.p, G.p, Mo.p, Vo.p, nparam, lr_ep, step + 1, 1e-5f, st_);
      }
    }
    // Inference copies: BF16-rounded weights.
    m.W1.reserve(n1);
    m.B1.reserve(H);
    m.W2.reserve(n2);
    m.B2.reserve(H);
    m.W3.reserve(n3);
    m.B3.reserve(NB);
    mlp_round_bf16(w1, m.W1.p, n1, st_);
    mlp_round_bf16(b1, m.B1.p, H, st_);
    mlp_round_bf16(w2, m.W2.p, n2, st_);
    mlp_round_bf16(b2, m.B2.p, H, st_);
    mlp_round_bf16(w3, m.W3.p, n3, st_);
    mlp_round_bf16(b3, m.B3.p, NB, st_);
    // Packed BF16 weights for the fused tensor-core inference.
    m.K1 = (F + 63) / 64 * 64;
    m.tc = m.K1 <= 256 && NB <= 32 && H == 256;
    if (m.tc) {
      m.W1b.reserve(static_cast<size_t>(H) * m.K1);
      m.W2b.reserve(static_cast<size_t>(H) * H);
      m.W3b.reserve(static_cast<size_t>(32) * H);
      mlp_pack_bf16(m.W1.p, H, F, H, m.K1, m.W1b.p, st_);
      mlp_pack_bf16(m.W2.p, H, H, H, H, m.W2b.p, st_);
      mlp_pack_bf16(m.W3.p, NB, H, 32, H, m.W3b.p, st_);
    }
    m.bucket_val.reserve(NB);
    HB_CUDA(cudaMemcpyAsync(m.bucket_val.p, m.buckets.data(), NB * sizeof(int32_t), cudaMemcpyHostToDevice, st_));
    // Calibration on the held-out queries: predicted nprobe for a grid of
    // thresholds -> recall against the label search's results.
    m.trained = true;
    const float grid[] = {0.3f,  0.4f,  0.5f,  0.6f,   0.7f,   0.75f,  0.8f,   0.85f,  0.88f,  0.9f,   0.92f,
                          0.94f, 0.95f, 0.96f, 0.97f,  0.975f, 0.98f,  0.985f, 0.99f,  0.993f, 0.995f, 0.997f,
                          0.998f, 0.999f, 0.9995f, 0.9999f, 1.0f};
    DevBuf<int32_t> npv;
    npv.reserve(nval);
    std::vector<int32_t> np_h(nval);
    m.cal_thr.clear();
    m.cal_recall.clear();
    m.cal_avgp.clear();
    const float* qv = qall.p + ntr * dpad_;
    const float* cv = cd.p + ntr * P;
    for (float t : grid) {
      probe_infer(static_cast<int>(nval), qv, cv, P, nullptr, t, P, npv.p);
      HB_CUDA(cudaMemcpyAsync(np_h.data(), npv.p, nval * sizeof(int32_t), cudaMemcpyDeviceToHost, st_));
      HB_CUDA(cudaStreamSynchronize(st_));
      double hit = 0, sp_sum = 0;
      for (size_t i = 0; i < nval; ++i) {
        const int32_t* rr = &ranks_h[(ntr + i) * k];
        for (size_t j = 0; j < k; ++j) hit += rr[j] < np_h[i];
        sp_sum += np_h[i];
      }
      m.cal_thr.push_back(t);
      m.cal_recall.push_back(static_cast<float>(hit / (nval * k)));
      m.cal_avgp.push_back(static_cast<float>(sp_sum / nval));
    }
    m.thr = 1.0f;
    float bestp = 1e30f;
    for (size_t i = 0; i < m.cal_thr.size(); ++i)
      if (m.cal_recall[i] >= target && m.cal_avgp[i] < bestp) {
        bestp = m.cal_avgp[i];
        m.thr = m.cal_thr[i];
      }
    HB_CUDA(cudaStreamSynchronize(st_));
  }

  int probe_calibration(float* thr, float* recall, float* avgp, int max_n) const {
    const int n = static_cast<int>(probe_.cal_thr.size());
    for (int i = 0; i < n && i < max_n; ++i) {
      if (thr) thr[i] = probe_.cal_thr[i];
      if (recall) recall[i] = probe_.cal_recall[i];
      if (avgp) avgp[i] = probe_.cal_avgp[i];
    }
    return n;
  }

 private:
  ProbeModel probe_;
  const float* ext_tops_ = nullptr;  // caller's heap tops (fullWarmUp) for the current search
  int cut_mode_ = 0;
  int cut_cap_ = 0;
  float cut_thr_ = 1.0f;
  const int32_t* cut_src_ = nullptr;
  size_t cut_b0_ = 0;
  DevBuf<float> cdist_, pf_, ph1_, ph2_, plog_;
  DevBuf<int32_t> npq_;

  size_t d_, nlist_, nprobe_;
  size_t dpad_ = 16;
  int kpad_ = 0;
  bool bf16_ready_ = false;
  bool fp8_ = false, fp8_ready_ = false;
  int kpad8_ = 0;
  alignas(64) unsigned char tmap8_[128];
  DevBuf<uint8_t> codes8_, gq8_;
  DevBuf<float> list_scale8_, qscale8_, qcd8_, rnorm8_, tile_rnorm8_;
  alignas(64) unsigned char tmap_[128];
  alignas(64) unsigned char gqmap_[128];  // gathered BF16 queries of the candidate-matrix scan
  bool cand_path_ = false;
  DevBuf<int64_t> seg_;
  DevBuf<uint16_t> gq_;
  DevBuf<float> cand_;
  DevBuf<int64_t> cand_rows_;
  // tensor-core coarse quantizer
  bool coarse_ready_ = false;
  int coarse_kind_ = HB_COARSE_AUTO;
  int coarse_margin_ = -1;
  int seed_rows_ = 256;  // rows of the nearest list behind the BF16 scan's seed bound
  int coarse_last_nq_ = 0;
  int ckpad_ = 0;
  alignas(64) unsigned char ctmap_[128];
  DevBuf<uint16_t> csplit_;
  DevBuf<uint16_t> qsplit_;  // queries' [hi | lo] BF16 rows for the tensor-core quantizer
  DevBuf<float> qsnorm_;     // their ||q||^2
  DevBuf<uint32_t> cmins_;   // per 16-column chunk of dmat_ and query: the chunk's smallest value
  DevBuf<float> cnorm_, cmaxnorm_, cval_;
  DevBuf<int32_t> ccand_;
  DevBuf<int> cflags_, cerr_dev_;
  bool capturing_ = false;
  std::map<std::string, GraphEntry> graphs_;
  DevBuf<int32_t> npqin_;
  // bounded BF16 scan
  DevBuf<uint32_t> thr_;
  DevBuf<int> ccnt_, cflag_, over_list_, over_n_, rr_m_;
  int last_nb_ = 0;
  DevBuf<uint64_t> cbuf_;
  DevBuf<uint32_t> cbuf_ub_;  // each candidate's upper bound
  DevBuf<float> oq_, od_;
  DevBuf<int32_t> op_;
  DevBuf<int64_t> oi_;
  long long wait_budget_ = kDefaultWaitBudget;
  bool autotune_ = false;
  std::map<TuneKey, TuneChoice> tune_;
  int last_overflow_ = 0;
  DevBuf<int32_t> kq_;
  DevBuf<uint16_t> codes_bf16_;
  DevBuf<float> tile_norm_, rnorm_, rmax_;
  DevBuf<int64_t> tile_off_;
  DevBuf<int32_t> probes1_;
  DevBuf<int32_t> probe0_, probes_rest_;  // the two stages' probe tables (k > kFilterTightK)
  DevBuf<int> err_dev_;
  int* err_host_ = nullptr;
  bool prof_ = false;
  std::vector<ProfRecord> prof_log_;
  std::vector<cudaEvent_t> ev_pool_;
  int metric_;
  int device_;
  int num_sms_ = 148;
  cudaStream_t st_ = nullptr;
  bool trained_ = false;
  size_t ntotal_ = 0;
  size_t plan_rows_ = 0;
  uint64_t launches_ = 0;
  std::vector<int64_t> host_off_;

  DevBuf<float> cent_, codes_, norms_;
  DevBuf<int64_t> list_off_, ids_;
  // search workspace
  DevBuf<float> qpad_, qtmp_, dmat_, tops_, dout_;
  DevBuf<int64_t> iout_, list_qoff_, item_off_, slot_base_;
  DevBuf<int32_t> probes_, list_cnt_, list_cursor_, list_q_, order_dev_;
  DevBuf<uint64_t> part_;
  DevBuf<unsigned int> counter_;
  DevBuf<unsigned char> work_tmp_;
};

}  // namespace hb

// ---------------------------------------------------------------------------
// C ABI

struct hb_index {
  std::unique_ptr<hb::IndexCore> core;
};

namespace {
template <class F>
int guarded(F&& f) {
  try {
    hb::g_last_error.clear();
    f();
    return HB_OK;
  } catch (const hb::Error& e) {
    hb::g_last_error = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    hb::g_last_error = "host allocation failed";
    return HB_ERR_NOMEM;
  } catch (const std::exception& e) {
    hb::g_last_error = e.what();
    return HB_ERR_INVALID;
  }
}
#define HB_NEED_INDEX(ix)                                           \
  do {                                                              \
    if (!(ix) || !(ix)->core) {                                     \
      hb::g_last_error = "null index handle";                       \
      return HB_ERR_INVALID;                                        \
    }                                                               \
  } while (0)
}  // namespace

namespace hb {
int index_device(const hb_index* ix) { return (ix && ix->core) ? ix->core->device() : -1; }

int search_in_scratch(hb_index* ix, size_t nq, const float* q, size_t k, float* D, int64_t* I, void* scratch,
                      size_t scratch_bytes) {
  HB_NEED_INDEX(ix);
  return guarded([&] {
    ix->core->search_in_scratch(nq, q, k, D, I, static_cast<unsigned char*>(scratch), scratch_bytes);
  });
}

void set_last_error(const char* msg) { g_last_error = msg ? msg : ""; }
}  // namespace hb

extern "C" {

void hb_search_params_init(hb_search_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->mode = HB_MODE_ORIGINAL;
  p->pruning = 0;
  p->order_optimize = 1;  // Param::orderOptimize default (src/Index.h:49)
  p->period = 0;
  p->n_dim_blocks = 1;
  p->n_query_blocks = 1;
  p->warmup_lists = 10;      // --warmup_list default (src/query.cpp:100-103)
  p->warmup_list_size = 0;   // 0 -> k (src/query.cpp:330-333)
  p->precision = HB_PREC_FP32;
  p->rerank_mult = 2;  // 2k candidates reproduce the exact scan on the 10M x 128 workload
  p->learned_probe = 0;
  p->learned_target = 0.0f;
  p->nprobe_per_query = nullptr;
  p->max_nprobe = 0;
  p->seed_rows = 0;
}

const char* hb_last_error(void) { return hb::g_last_error.c_str(); }

const char* hb_version(void) { return "harmony_b200 0.1 (sm_100a)"; }

int hb_create(size_t d, size_t nlist, size_t nprobe, int metric, int device, hb_index** out) {
  if (!out) {
    hb::g_last_error = "null output handle";
    return HB_ERR_INVALID;
  }
  *out = nullptr;
  return guarded([&] {
    auto h = std::make_unique<hb_index>();
    h->core = std::make_unique<hb::IndexCore>(d, nlist, nprobe, metric, device);
    *out = h.release();
  });
}

int hb_destroy(hb_index* ix) {
  delete ix;
  return HB_OK;
}

int hb_train(hb_index* ix, size_t n, const float* x, int lite) {
  HB_NEED_INDEX(ix);
  return guarded([&] { ix->core->train(n, x, lite != 0); });
}

int hb_add(hb_index* ix, size_t n, const float* x) {
  HB_NEED_INDEX(ix);
  return guarded([&] { ix->core->add(n, x); });
}

int hb_search(hb_index* ix, size_t nq, const float* q, size_t k, const hb_search_params* params, float* D,
              int64_t* I) {
  HB_NEED_INDEX(ix);
  return guarded([&] { ix->core->search(nq, q, k, params, D, I); });
}

int hb_save_index(hb_index* ix, const char* path) {
  HB_NEED_INDEX(ix);
  if (!path) return HB_ERR_INVALID;
  return guarded([&] { ix->core->save(path); });
}

int hb_load_index(hb_index* ix, const char* path) {
  HB_NEED_INDEX(ix);
  if (!path) return HB_ERR_INVALID;
  return guarded([&] { ix->core->load(path); });
}

int hb_set_nprobe(hb_index* ix, size_t nprobe) {
  HB_NEED_INDEX(ix);
  ix->core->set_nprobe(nprobe);
  return HB_OK;
}

int hb_get_nprobe(const hb_index* ix, size_t* nprobe) {
  HB_NEED_INDEX(ix);
  if (!nprobe) return HB_ERR_INVALID;
  *nprobe = ix->core->nprobe();
  return HB_OK;
}

int hb_get_info(const hb_index* ix, size_t* d, size_t* nlist, size_t* ntotal, int* metric) {
  HB_NEED_INDEX(ix);
  if (d) *d = ix->core->d();
  if (nlist) *nlist = ix->core->nlist();
  if (ntotal) *ntotal = ix->core->ntotal();
  if (metric) *metric = ix->core->metric();
  return HB_OK;
}

int hb_get_centroids(const hb_index* ix, float* out) {
  HB_NEED_INDEX(ix);
  return guarded([&] { ix->core->get_centroids(out); });
}

int hb_retain_lists(hb_index* ix, size_t first, size_t count) {
  HB_NEED_INDEX(ix);
  return guarded([&] { ix->core->retain_lists(first, count); });
}

int hb_merge_topk(hb_index* ix, size_t nparts, size_t nq, size_t k, const float* D_parts, const int64_t* I_parts,
                  float* D, int64_t* I) {
  HB_NEED_INDEX(ix);
  if (nq == 0) return HB_OK;
  return guarded([&] {
    HB_CHECK(D_parts && I_parts && D && I, HB_ERR_INVALID, "null pointer");
    ix->core->merge_parts(nparts, nq, k, D_parts, I_parts, D, I);
  });
}

int hb_get_list_sizes(const hb_index* ix, int64_t* out) {
  HB_NEED_INDEX(ix);
  return guarded([&] { ix->core->get_list_sizes(out); });
}

int hb_probe_lists(hb_index* ix, size_t nq, const float* q, size_t nprobe, int64_t* probes, float* cdist) {
  HB_NEED_INDEX(ix);
  return guarded([&] { ix->core->probe_lists(nq, q, nprobe, probes, cdist); });
}

int hb_warmup_tops(hb_index* ix, size_t nq, const float* q, size_t k, size_t warm_lists, size_t warm_list_size,
                   float* tops) {
  HB_NEED_INDEX(ix);
  return guarded([&] { ix->core->warmup_tops(nq, q, k, warm_lists, warm_list_size, tops); });
}

int hb_set_coarse_quantizer(hb_index* ix, int kind, int margin) {
  HB_NEED_INDEX(ix);
  return guarded([&] { ix->core->set_coarse(kind, margin); });
}

int hb_coarse_fallbacks(hb_index* ix, int64_t* n) {
  HB_NEED_INDEX(ix);
  return guarded([&] {
    HB_CHECK(n, HB_ERR_INVALID, "null output pointer");
    *n = ix->core->coarse_fallbacks();
  });
}

void* hb_stream(hb_index* ix) { return (ix && ix->core) ? static_cast<void*>(ix->core->stream()) : nullptr; }

uint64_t hb_launch_count(const hb_index* ix) { return (ix && ix->core) ? ix->core->launches() : 0; }

uint64_t hb_device_allocations(void) { return hb::devbuf_generation().load(); }

int hb_set_autotune(hb_index* ix, int on) {
  HB_NEED_INDEX(ix);
  ix->core->set_autotune(on != 0);
  return HB_OK;
}

int hb_autotune_table(hb_index* ix, char* buf, size_t len, size_t* needed) {
  HB_NEED_INDEX(ix);
  return guarded([&] {
    const std::string t = ix->core->autotune_table();
    if (needed) *needed = t.size() + 1;
    if (buf && len) {
      std::strncpy(buf, t.c_str(), len - 1);
      buf[len - 1] = 0;
    }
  });
}

int hb_set_autotune_table(hb_index* ix, const char* text) {
  HB_NEED_INDEX(ix);
  if (!text) return HB_ERR_INVALID;
  return guarded([&] { ix->core->set_autotune_table(text); });
}

int hb_set_wait_budget(hb_index* ix, int64_t cycles) {
  HB_NEED_INDEX(ix);
  ix->core->set_wait_budget(cycles);
  return HB_OK;
}

int hb_bf16_stats(hb_index* ix, int64_t* stats) {
  HB_NEED_INDEX(ix);
  if (!stats) return HB_ERR_INVALID;
  return guarded([&] { ix->core->bf16_stats(stats); });
}

int hb_bf16_fallbacks(hb_index* ix, int64_t* n) {
  HB_NEED_INDEX(ix);
  if (!n) return HB_ERR_INVALID;
  *n = ix->core->last_overflow();
  return HB_OK;
}

int hb_selftest_bounded_wait(hb_index* ix, int64_t budget_cycles, int64_t* waited_cycles) {
  HB_NEED_INDEX(ix);
  return guarded([&] {
    long long w = 0;
    try {
      ix->core->wait_selftest(budget_cycles, &w);
    } catch (...) {
      if (waited_cycles) *waited_cycles = w;
      throw;
    }
    if (waited_cycles) *waited_cycles = w;
  });
}

int hb_profile_enable(hb_index* ix, int on) {
  HB_NEED_INDEX(ix);
  ix->core->profile_enable(on != 0);
  return HB_OK;
}

int hb_profile_read(hb_index* ix, char* names, size_t names_len, double* ms, int64_t* counts, int max_entries,
                    int* n_entries) {
  HB_NEED_INDEX(ix);
  return guarded([&] {
    const int n = ix->core->profile_read(names, names_len, ms, counts, max_entries);
    if (n_entries) *n_entries = n;
  });
}

int hb_train_probe_predictor(hb_index* ix, size_t nt, const float* q, size_t k, size_t label_nprobe, float target) {
  HB_NEED_INDEX(ix);
  return guarded([&] { ix->core->train_probe(nt, q, k, label_nprobe, target); });
}

int hb_probe_calibration(const hb_index* ix, float* thr, float* recall, float* avg_nprobe, int max_n, int* n) {
  HB_NEED_INDEX(ix);
  const int c = ix->core->probe_calibration(thr, recall, avg_nprobe, max_n);
  if (n) *n = c;
  return HB_OK;
}

}  // extern "C"

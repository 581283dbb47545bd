"""harmony_b200 -- B200-native IVF-flat search behind Harmony's ``Index`` API.

The compute path is ``libharmony_b200.so`` (hand-written sm_100a CUDA kernels
behind the C ABI in ``include/harmony_b200.h``).  This module is the Python
host mirror of the reference's C++ class ``harmony::Index`` (src/Index.h):
same member names, argument meaning and error behaviour, so driver code and
tests read like the reference's own::

    index = Index(d, nlist, nprobe)              # src/Index.h:15-25
    index.train(n, base)                         # src/Index.cpp:381
    index.add(n, base)                           # src/Index.cpp:581
    param = Index.Param(); param.mode = Index.SearchMode.ORIGINAL
    index.preSearch(nb, 0, 0, 0, 0, param, "")   # src/Index.cpp:45-55
    index.search(nq, queries, k, distances, labels)   # src/Index.cpp:1638
    index.save_index(path); index.load_index(path)    # src/Index.cpp:1708-1770

Arrays may be numpy arrays (host) or CUDA tensors / device pointers; results
are written in place like the reference's ``float* distances, idx_t* labels``.
There is no CPU fallback: without the built library or a CUDA device every
call raises.
"""
from __future__ import annotations

import ctypes
import enum
import os
import time
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libharmony_b200.so")

__all__ = ["Index", "MetricType", "OptLevel", "EdgeDevice", "SearchMode", "Precision", "CoarseQuantizer", "HarmonyError",
           "SearchParams", "lib", "LIB_PATH"]


class HarmonyError(RuntimeError):
    """Raised for a non-zero hb_status (the reference throws std::runtime_error)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[hb_status {code}] {msg}")
        self.code = code


class MetricType(enum.IntEnum):  # src/common.h:20-21
    METRIC_IP = 0
    METRIC_L2 = 1


class OptLevel(enum.IntEnum):  # src/common.h:23-32
    OPT_NONE = 0b000
    OPT_TRIANGLE = 0b001
    OPT_SUBNN_L2 = 0b010
    OPT_SUBNN_IP = 0b100
    OPT_TRI_SUBNN_L2 = 0b011
    OPT_TRI_SUBNN_IP = 0b101
    OPT_SUBNN_ONLY = 0b110
    OPT_ALL = 0b111


class EdgeDevice(enum.IntEnum):  # src/common.h:34-37
    EDGEDEVIVE_ENABLED = 0
    EDGEDEVIVE_DISABLED = 1


class SearchMode(enum.IntEnum):  # Index::SearchMode, src/Index.h:29-35
    BRUTE_FORCE = 0
    ORIGINAL = 1
    DIVIDE_IVF = 2
    DIVIDE_DIM = 3
    DIVIDE_GROUP = 4


class Precision(enum.IntEnum):
    FP32 = 0
    BF16 = 1
    FP8 = 2


class CoarseQuantizer(enum.IntEnum):
    """Route of the coarse quantizer; every route gives the same probe rows."""
    AUTO = 0
    EXACT = 1
    TENSOR = 2


class _SearchParamsC(ctypes.Structure):
    _fields_ = [
        ("mode", ctypes.c_int32),
        ("pruning", ctypes.c_int32),
        ("order_optimize", ctypes.c_int32),
        ("period", ctypes.c_int32),
        ("n_dim_blocks", ctypes.c_int32),
        ("n_query_blocks", ctypes.c_int32),
        ("warmup_lists", ctypes.c_int32),
        ("warmup_list_size", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("rerank_mult", ctypes.c_int32),
        ("learned_probe", ctypes.c_int32),
        ("learned_target", ctypes.c_float),
        ("nprobe_per_query", ctypes.c_void_p),
        ("max_nprobe", ctypes.c_int32),
        ("seed_rows", ctypes.c_int32),
        ("use_graph", ctypes.c_int32),
        ("full_warmup", ctypes.c_int32),
        ("heap_tops", ctypes.c_void_p),
        ("reserved", ctypes.c_int32 * 2),
    ]


_lib = None


def lib() -> ctypes.CDLL:
    """Load the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"harmony_b200 CUDA library not built: {LIB_PATH} "
                          "(run __graft_entry__.build() or make -C harmony_b200/csrc)")
    L = ctypes.CDLL(LIB_PATH)
    vp, sz, f, i64 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p
    L.hb_last_error.restype = ctypes.c_char_p
    L.hb_version.restype = ctypes.c_char_p
    L.hb_search_params_init.argtypes = [ctypes.POINTER(_SearchParamsC)]
    L.hb_create.argtypes = [sz, sz, sz, ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)]
    L.hb_destroy.argtypes = [vp]
    L.hb_train.argtypes = [vp, sz, f, ctypes.c_int]
    L.hb_add.argtypes = [vp, sz, f]
    L.hb_search.argtypes = [vp, sz, f, sz, ctypes.POINTER(_SearchParamsC), f, i64]
    L.hb_save_index.argtypes = [vp, ctypes.c_char_p]
    L.hb_load_index.argtypes = [vp, ctypes.c_char_p]
    L.hb_set_nprobe.argtypes = [vp, sz]
    L.hb_get_nprobe.argtypes = [vp, ctypes.POINTER(sz)]
    L.hb_get_info.argtypes = [vp, ctypes.POINTER(sz), ctypes.POINTER(sz), ctypes.POINTER(sz),
                              ctypes.POINTER(ctypes.c_int)]
    L.hb_get_centroids.argtypes = [vp, f]
    L.hb_get_list_sizes.argtypes = [vp, i64]
    L.hb_probe_lists.argtypes = [vp, sz, f, sz, i64, f]
    L.hb_warmup_tops.argtypes = [vp, sz, f, sz, sz, sz, f]
    L.hb_set_coarse_quantizer.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    L.hb_coarse_fallbacks.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
    L.hb_stream.restype = vp
    L.hb_stream.argtypes = [vp]
    L.hb_launch_count.restype = ctypes.c_uint64
    L.hb_launch_count.argtypes = [vp]
    L.hb_device_allocations.restype = ctypes.c_uint64
    L.hb_device_allocations.argtypes = []
    L.hb_selftest_bounded_wait.argtypes = [vp, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]
    L.hb_set_wait_budget.argtypes = [vp, ctypes.c_int64]
    L.hb_set_autotune.argtypes = [vp, ctypes.c_int]
    L.hb_autotune_table.argtypes = [vp, ctypes.c_char_p, sz, ctypes.POINTER(sz)]
    L.hb_set_autotune_table.argtypes = [vp, ctypes.c_char_p]
    L.hb_bf16_fallbacks.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
    L.hb_bf16_stats.argtypes = [vp, ctypes.c_void_p]
    L.hb_train_probe_predictor.argtypes = [vp, sz, f, sz, sz, ctypes.c_float]
    L.hb_search_noalloc.argtypes = [vp, sz, f, sz, f, i64]
    L.hb_retain_lists.argtypes = [vp, sz, sz]
    L.hb_merge_topk.argtypes = [vp, sz, sz, sz, f, i64, f, i64]
    L.hb_probe_calibration.argtypes = [vp, f, f, f, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    L.hb_profile_enable.argtypes = [vp, ctypes.c_int]
    L.hb_profile_read.argtypes = [vp, ctypes.c_char_p, sz, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                  ctypes.POINTER(ctypes.c_int)]
    _lib = L
    return L


def _check(code: int) -> None:
    if code != 0:
        raise HarmonyError(code, lib().hb_last_error().decode(errors="replace"))


def _wait_for_torch(stream_handle: int, *arrays) -> None:
    """Order the index's stream after torch's current stream when any of
    `arrays` is a CUDA tensor.  The library launches on its own non-blocking
    stream and never waits on other streams, so a tensor that torch is still
    producing (or a buffer a collective is still filling) must be finished
    on that stream before the library reads it."""
    if not any(getattr(a, "is_cuda", False) for a in arrays):
        return
    import torch
    dev = next(a.device for a in arrays if getattr(a, "is_cuda", False))
    torch.cuda.ExternalStream(stream_handle, device=dev).wait_stream(torch.cuda.current_stream(dev))


def _ptr(a, dtype, writable=False):
    """(pointer, keepalive) for a numpy array, torch tensor or raw int pointer."""
    if a is None:
        return None, None
    if isinstance(a, int):
        return a, None
    if hasattr(a, "data_ptr") and hasattr(a, "is_contiguous"):  # torch tensor
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        want = {np.float32: "torch.float32", np.int64: "torch.int64", np.int32: "torch.int32"}[dtype]
        if str(a.dtype) != want:
            raise TypeError(f"tensor dtype {a.dtype} != {want}")
        return a.data_ptr(), a
    arr = np.asarray(a)
    if arr.dtype != dtype or not arr.flags.c_contiguous:
        if writable:
            raise TypeError(f"output array must be C-contiguous {np.dtype(dtype).name}")
        arr = np.ascontiguousarray(arr, dtype=dtype)
    return arr.ctypes.data, arr


@dataclass
class Stats:
    """Subset of the reference's Stats (src/stats.h:14-135) a search fills."""
    query_time: float = 0.0
    nprobe: int = 0
    k: int = 0
    nq: int = 0


@dataclass
class SearchParams:
    """GPU search knobs beyond Index::Param (see include/harmony_b200.h)."""
    precision: Precision = Precision.FP32
    rerank_mult: int = 2
    learned_probe: bool = False
    learned_target: float = 0.0
    nprobe_per_query: Optional[object] = None
    max_nprobe: int = 0
    seed_rows: int = 0
    use_graph: bool = False


class Index:
    """harmony::Index (src/Index.h:13-149) on one B200."""

    SearchMode = SearchMode

    @dataclass
    class Param:
        """Index::Param (src/Index.h:48-68): the fields that steer search.
        fullWarmUp with heapTops (nq floats, e.g. each query's k-th ground-truth
        distance as src/query.cpp:716-725 fills it) replaces the warm-up search's
        pruning thresholds in DIVIDE_DIM (src/Index.cpp:1235-1241)."""
        orderOptimize: bool = True
        mode: SearchMode = SearchMode.ORIGINAL
        pruning: bool = False
        period: bool = False
        fullWarmUp: bool = False
        heapTops: Optional[object] = None
        block_dim: int = 0
        groupCount: int = 0
        teamCount: int = 0
        teamSize: int = 0

    def __init__(self, d: int = 0, nlist: int = 0, nprobe: int = 0,
                 metric: MetricType = MetricType.METRIC_L2, opt_level: OptLevel = OptLevel.OPT_NONE,
                 sub_k: int = 0, sub_nlist: int = 1, sub_nprobe: int = 1, verbose: bool = False,
                 edge_device_enabled: EdgeDevice = EdgeDevice.EDGEDEVIVE_DISABLED, device: int = 0):
        self._L = lib()
        self._h = ctypes.c_void_p()
        self.metric = MetricType(metric)
        self.opt_level = OptLevel(opt_level)
        self.sub_k, self.sub_nlist, self.sub_nprobe = sub_k, sub_nlist, sub_nprobe
        self.verbose = verbose
        self.edge_device_enabled = edge_device_enabled
        self.device = device
        # The reference's default Index() has d = nlist = 0 and is filled by
        # load_index; the device index needs a shape, so a placeholder is used.
        self._placeholder = d == 0 or nlist == 0
        _check(self._L.hb_create(d or 16, nlist or 1, nprobe, int(self.metric), device, ctypes.byref(self._h)))
        self.param: Optional[Index.Param] = None
        self.workerCount = self.blockCount = 0
        self.warmUpSearchList = self.warmUpSearchListSize = 0
        self.search_params = SearchParams()
        self.trainTime = self.addTime = 0.0

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._L.hb_destroy(h)
            self._h = ctypes.c_void_p()

    # -- public fields -----------------------------------------------------
    @property
    def nprobe(self) -> int:
        v = ctypes.c_size_t()
        _check(self._L.hb_get_nprobe(self._h, ctypes.byref(v)))
        return v.value

    @nprobe.setter
    def nprobe(self, v: int) -> None:
        _check(self._L.hb_set_nprobe(self._h, int(v)))

    def _info(self):
        d, nl, nt, m = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_int()
        _check(self._L.hb_get_info(self._h, ctypes.byref(d), ctypes.byref(nl), ctypes.byref(nt), ctypes.byref(m)))
        return d.value, nl.value, nt.value, m.value

    @property
    def d(self) -> int:
        return 0 if self._placeholder else self._info()[0]

    @property
    def nlist(self) -> int:
        return 0 if self._placeholder else self._info()[1]

    @property
    def ntotal(self) -> int:
        return self._info()[2]

    @property
    def centroid_codes(self) -> np.ndarray:
        d, nl, _, _ = self._info()
        out = np.empty((nl, d), np.float32)
        _check(self._L.hb_get_centroids(self._h, out.ctypes.data))
        return out

    def list_sizes(self) -> np.ndarray:
        _, nl, _, _ = self._info()
        out = np.empty(nl, np.int64)
        _check(self._L.hb_get_list_sizes(self._h, out.ctypes.data))
        return out

    def retain_lists(self, first: int, count: int) -> None:
        """Keep lists [first, first + count) and empty the others: one rank's
        share of the reference's DIVIDE_IVF partition (src/Index.cpp:79-104).
        Ids are unchanged."""
        _check(self._L.hb_retain_lists(self._h, int(first), int(count)))

    def merge_topk(self, D_parts, I_parts, D, I) -> None:
        """Merge per-shard results (device tensors of shape (parts, nq, k)) into
        D, I (nq, k) with the reference master's heap rule
        (src/Index.cpp:1327-1341), on this index's stream."""
        parts, nq, k = D_parts.shape
        for t in (D_parts, I_parts, D, I):
            if not (hasattr(t, "is_cuda") and t.is_cuda and t.is_contiguous()):
                raise TypeError("merge_topk takes contiguous CUDA tensors")
        if tuple(I_parts.shape) != (parts, nq, k) or tuple(D.shape) != (nq, k) or tuple(I.shape) != (nq, k):
            raise ValueError("shape mismatch")
        # The parts usually come from a collective queued on torch's stream.
        _wait_for_torch(self.stream, D_parts, I_parts, D, I)
        _check(self._L.hb_merge_topk(self._h, parts, nq, k, D_parts.data_ptr(), I_parts.data_ptr(), D.data_ptr(),
                                     I.data_ptr()))

    @property
    def stream(self) -> int:
        """The cudaStream_t this index launches on."""
        return self._L.hb_stream(self._h) or 0

    def launch_count(self) -> int:
        return int(self._L.hb_launch_count(self._h))

    def profile(self, on: bool = True) -> None:
        """Record CUDA events around every kernel on the index's stream."""
        _check(self._L.hb_profile_enable(self._h, int(on)))

    def profile_read(self) -> dict:
        """{kernel name: (total ms, launches)} since the last read."""
        names = ctypes.create_string_buffer(4096)
        ms = np.zeros(64, np.float64)
        cnt = np.zeros(64, np.int64)
        n = ctypes.c_int()
        _check(self._L.hb_profile_read(self._h, names, 4096, ms.ctypes.data, cnt.ctypes.data, 64, ctypes.byref(n)))
        keys = names.value.decode().split("\n")[: n.value]
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(keys)}

    # -- train / add -------------------------------------------------------
    def train(self, n: int, codes, faiss: bool = False, lite: bool = False) -> None:
        """Index::train (src/Index.cpp:381-425); faiss=True is not available."""
        if faiss:
            raise HarmonyError(1, "faiss training is not part of this build")
        p, keep = _ptr(codes, np.float32)
        t0 = time.perf_counter()
        _check(self._L.hb_train(self._h, int(n), p, int(lite)))
        self.trainTime = time.perf_counter() - t0

    def add(self, n: int, codes) -> None:
        """Index::add (src/Index.cpp:581-698)."""
        p, keep = _ptr(codes, np.float32)
        t0 = time.perf_counter()
        _check(self._L.hb_add(self._h, int(n), p))
        self.addTime = time.perf_counter() - t0

    # -- search ------------------------------------------------------------
    def preSearch(self, nb: int, workerCount: int, blockCount: int, warmUpSearchList: int,
                  warmUpSearchListSize: int, param: "Index.Param", path: str = "") -> None:
        """Index::preSearch (src/Index.cpp:45-335): records the search setup.

        The multi-process modes map onto one GPU: workerCount becomes the
        number of dimension slices in DIVIDE_DIM and blockCount the number of
        query blocks; nothing is distributed and no partition file is written.
        """
        if param is None:
            raise HarmonyError(1, "param must not be null")
        self.param = param
        self.workerCount, self.blockCount = int(workerCount), int(blockCount)
        self.warmUpSearchList, self.warmUpSearchListSize = int(warmUpSearchList), int(warmUpSearchListSize)

    def postSearch(self) -> None:
        pass

    def _params_c(self, k: int) -> _SearchParamsC:
        c = _SearchParamsC()
        self._L.hb_search_params_init(ctypes.byref(c))
        prm = self.param
        c.mode = int(prm.mode)
        c.pruning = int(bool(prm.pruning))
        c.order_optimize = int(bool(prm.orderOptimize))
        c.period = int(bool(prm.period))
        c.full_warmup = int(bool(prm.fullWarmUp))
        if prm.mode == SearchMode.DIVIDE_DIM:
            c.n_dim_blocks = max(1, self.workerCount)
            c.n_query_blocks = max(1, self.blockCount)
        if self.warmUpSearchList:
            c.warmup_lists = self.warmUpSearchList
        c.warmup_list_size = self.warmUpSearchListSize
        sp = self.search_params
        c.precision = int(sp.precision)
        c.rerank_mult = int(sp.rerank_mult)
        c.learned_probe = int(bool(sp.learned_probe))
        c.learned_target = float(sp.learned_target)
        c.max_nprobe = int(sp.max_nprobe)
        c.seed_rows = int(sp.seed_rows)
        c.use_graph = 1 if sp.use_graph else 0
        return c

    def search(self, n: int, queries, k: int, distances, labels, ratio: float = 1.0) -> Stats:
        """Index::search (src/Index.cpp:1638-1706): fills distances / labels.

        Without preSearch the reference's ``param`` is unset and search only
        initialises the results (FLT_MAX / -1); the same happens here.
        """
        if n == 0:
            return Stats()
        qp, qk = _ptr(queries, np.float32)
        dp, dk = _ptr(distances, np.float32, writable=True)
        ip, ik = _ptr(labels, np.int64, writable=True)
        t0 = time.perf_counter()
        if self.param is None:
            _fill_unsearched(distances, labels)
            return Stats(nq=n, k=k)
        c = self._params_c(k)
        keep_pq = None
        if self.search_params.nprobe_per_query is not None:
            pq, keep_pq = _ptr(self.search_params.nprobe_per_query, np.int32)
            c.nprobe_per_query = pq
        keep_tops = None
        if getattr(self.param, "fullWarmUp", False) and self.param.heapTops is not None:
            tp, keep_tops = _ptr(self.param.heapTops, np.float32)
            c.heap_tops = tp
        _wait_for_torch(self.stream, queries, distances, labels, keep_pq, keep_tops)
        _check(self._L.hb_search(self._h, int(n), qp, int(k), ctypes.byref(c), dp, ip))
        return Stats(query_time=time.perf_counter() - t0, nprobe=self.nprobe, k=k, nq=n)

    def search_arrays(self, queries, k: int, mode: SearchMode = SearchMode.ORIGINAL):
        """Convenience: returns (D, I) numpy arrays for host queries."""
        q = np.ascontiguousarray(queries, dtype=np.float32)
        nq = q.shape[0]
        D = np.empty((nq, k), np.float32)
        I = np.empty((nq, k), np.int64)
        if self.param is None:
            self.preSearch(0, 0, 0, 0, 0, Index.Param(mode=mode))
        self.search(nq, q, k, D, I)
        return D, I

    def probe_lists(self, queries, nprobe: Optional[int] = None):
        """Coarse quantizer only (Index::findNearNprobeOfCentroidIds)."""
        q = np.ascontiguousarray(queries, dtype=np.float32)
        P = self.nprobe if nprobe is None else nprobe
        probes = np.empty((q.shape[0], P), np.int64)
        cd = np.empty((q.shape[0], P), np.float32)
        _check(self._L.hb_probe_lists(self._h, q.shape[0], q.ctypes.data, P, probes.ctypes.data, cd.ctypes.data))
        return probes, cd

    def warmup_tops(self, queries, k: int, warm_lists: int = 10, warm_list_size: Optional[int] = None):
        q = np.ascontiguousarray(queries, dtype=np.float32)
        tops = np.empty(q.shape[0], np.float32)
        _check(self._L.hb_warmup_tops(self._h, q.shape[0], q.ctypes.data, k, warm_lists,
                                      k if warm_list_size is None else warm_list_size, tops.ctypes.data))
        return tops

    def set_coarse_quantizer(self, kind: "CoarseQuantizer" = CoarseQuantizer.AUTO, margin: int = -1) -> None:
        """Pick the coarse quantizer's route (tensor cores + exact re-rank, or
        the exact FP32 distance matrix) and the tensor-core candidate margin
        (-1: max(16, nprobe / 4)).  The probe rows do not depend on it."""
        _check(self._L.hb_set_coarse_quantizer(self._h, int(kind), int(margin)))

    def bf16_fallbacks(self) -> int:
        """Queries of the latest BF16 search (d <= 128, k <= 256) whose candidate
        buffer overflowed and were searched again with the exact scan."""
        n = ctypes.c_int64()
        _check(self._L.hb_bf16_fallbacks(self._h, ctypes.byref(n)))
        return int(n.value)

    def bf16_stats(self) -> dict:
        """Admission statistics of the latest bounded BF16 batch."""
        st = np.zeros(5, np.int64)
        _check(self._L.hb_bf16_stats(self._h, st.ctypes.data))
        return {"queries": int(st[0]), "overflows": int(st[1]), "admitted": int(st[2]),
                "admitted_max": int(st[3]), "reranked": int(st[4])}

    def set_autotune(self, on: bool = True) -> None:
        """Time the bounded BF16 scan's chunk length and ring depth on the first
        search of each (batch, nprobe, k) bucket and keep the fastest."""
        _check(self._L.hb_set_autotune(self._h, int(on)))

    def autotune_table(self) -> str:
        """The tuned choices as text (one line per bucket)."""
        need = ctypes.c_size_t()
        _check(self._L.hb_autotune_table(self._h, None, 0, ctypes.byref(need)))
        buf = ctypes.create_string_buffer(max(1, need.value))
        _check(self._L.hb_autotune_table(self._h, buf, len(buf), None))
        return buf.value.decode()

    def set_autotune_table(self, text: str) -> None:
        _check(self._L.hb_set_autotune_table(self._h, text.encode()))

    def set_wait_budget(self, cycles: int = 0) -> None:
        """Clock cycles a device wait of the BF16 scan spends before giving up
        (0: the default)."""
        _check(self._L.hb_set_wait_budget(self._h, int(cycles)))

    def coarse_fallbacks(self) -> int:
        """Queries of the latest tensor-core coarse call recomputed exactly."""
        n = ctypes.c_int64()
        _check(self._L.hb_coarse_fallbacks(self._h, ctypes.byref(n)))
        return int(n.value)

    # -- learned probe predictor (no reference counterpart) -----------------
    def train_probe_predictor(self, n: int, queries, k: int = 10, label_nprobe: int = 256,
                              target: float = 0.95) -> None:
        """Train the per-query nprobe predictor on n training queries labelled by
        the exact search at nprobe = label_nprobe, calibrated to `target` recall."""
        p, keep = _ptr(queries, np.float32)
        _check(self._L.hb_train_probe_predictor(self._h, int(n), p, int(k), int(label_nprobe), float(target)))

    def probe_calibration(self):
        """(thresholds, recall, average nprobe) measured on the held-out split."""
        thr = np.zeros(64, np.float32)
        rec = np.zeros(64, np.float32)
        avg = np.zeros(64, np.float32)
        n = ctypes.c_int()
        _check(self._L.hb_probe_calibration(self._h, thr.ctypes.data, rec.ctypes.data, avg.ctypes.data, 64,
                                            ctypes.byref(n)))
        return thr[: n.value], rec[: n.value], avg[: n.value]

    # -- persistence -------------------------------------------------------
    def save_index(self, path: str) -> None:
        d = os.path.dirname(os.path.abspath(path))
        os.makedirs(d, exist_ok=True)  # prepareDirectory (src/Index.cpp:1709)
        _check(self._L.hb_save_index(self._h, path.encode()))

    def load_index(self, path: str) -> None:
        _check(self._L.hb_load_index(self._h, path.encode()))
        self._placeholder = False
        self.opt_level = OptLevel.OPT_NONE  # src/Index.cpp:1744


def _fill_unsearched(D, I):
    if hasattr(D, "fill_"):
        D.fill_(np.finfo(np.float32).max)
        I.fill_(-1)
    else:
        D[...] = np.finfo(np.float32).max
        I[...] = -1

"""CPU oracle for the IVF-flat search path.

TEST INFRASTRUCTURE ONLY.  Two checkers live here:

* ``restated`` -- ``libivf_oracle.so``, this project's own CPU restatement of
  the reference algorithm (ivf_oracle.cpp; every function cites the reference
  file:line it follows).
* ``reference`` -- ``_ref/libharmony_ref.so``, the reference's own
  ``harmony::Index`` compiled from its unmodified sources with the stand-ins in
  ``ref_shim/`` (see Makefile).  It pins the restatement.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package.  The product (``harmony_b200``) never
does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libivf_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libharmony_ref.so")
REF_RELEASE_SO = os.path.join(HERE, "_ref", "libharmony_ref_release.so")
# Where the reference sources lie (only the build reads them).
REFERENCE_SRC = os.environ.get("HARMONY_REFERENCE", "/root/reference")
_AVX512 = ("avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl")


def host_cpu():
    """(model name, logical cores, has the AVX-512 subsets x86-64-v4 needs)."""
    model, flags = "unknown", set()
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name") and model == "unknown":
                    model = line.split(":", 1)[1].strip()
                elif line.startswith("flags") and not flags:
                    flags = set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return model, os.cpu_count() or 1, all(f in flags for f in _AVX512)


def reference_build():
    """(path, description) of the reference library this host loads: the
    Release-flag build where the CPU has AVX-512, else the portable one."""
    if os.path.exists(REF_RELEASE_SO) and host_cpu()[2]:
        return REF_RELEASE_SO, "release flags (-Ofast -mavx512f -march=x86-64-v4 -O3 -DNDEBUG)"
    return REF_SO, "portable flags (-O3 -DNDEBUG -ffp-contract=off)"

_f = ctypes.POINTER(ctypes.c_float)
_d = ctypes.POINTER(ctypes.c_double)
_i = ctypes.POINTER(ctypes.c_int64)
_sz = ctypes.c_size_t
_vp = ctypes.c_void_p


def build(reference: bool = True) -> None:
    """Compile the restatement, and the reference library when its sources exist."""
    subprocess.check_call(["make", "-s", "-C", HERE, "libivf_oracle.so"])
    if reference and os.path.isdir(os.path.join(REFERENCE_SRC, "src")):
        subprocess.check_call(["make", "-s", "-C", HERE, "ref", f"REF={REFERENCE_SRC}"])


def _fp(a):
    return a.ctypes.data_as(_f)


def _ip(a):
    return a.ctypes.data_as(_i)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _i64(a):
    return np.ascontiguousarray(a, dtype=np.int64)


class _Restated:
    def __init__(self):
        if not os.path.exists(ORACLE_SO):
            build(reference=False)
        L = ctypes.CDLL(ORACLE_SO)
        L.orc_l2.restype = ctypes.c_float
        L.orc_l2.argtypes = [_f, _f, _sz]
        L.orc_heap_topk.argtypes = [_sz, _f, _sz, _f, _i]
        L.orc_coarse.argtypes = [_sz, _f, _sz, _sz, _f, _sz, _f, _i]
        L.orc_search.argtypes = [_sz, _f, _sz, _sz, _f, _i, _i, _f, _sz, _sz, _f, _i]
        L.orc_search_probes.argtypes = [_sz, _f, _sz, _i, _i, _f, _sz, _i, _sz, _f, _i]
        L.orc_warmup_tops.argtypes = [_sz, _f, _sz, _i, _i, _f, _sz, _i, _sz, _sz, _sz, _f]
        L.orc_search_pruned.argtypes = [_sz, _f, _sz, _i, _i, _f, _sz, _i, _f, ctypes.c_int, _sz, _f, _i]
        L.orc_search_dimblock.argtypes = [_sz, _f, _sz, _i, _i, _f, _sz, _i, _f, ctypes.c_int, _sz, _sz,
                                          _i, _sz, _f, _i]
        L.orc_block_order.argtypes = [_sz, _sz, ctypes.c_int, ctypes.c_int, _i]
        L.orc_kmeans.argtypes = [_sz, _f, _sz, _sz, ctypes.c_int, ctypes.c_int, _sz, _f]
        L.orc_kmeans_indices.argtypes = [_sz, _sz, ctypes.c_int, _sz, _i, _i]
        L.orc_add.argtypes = [_sz, _f, _sz, _sz, _f, _i, _i, _f, _f]
        L.orc_bruteforce_f64.argtypes = [_sz, _f, _sz, _f, _sz, _sz, _d, _i]
        self.L = L

    def l2(self, a, b):
        a, b = _f32(a), _f32(b)
        return self.L.orc_l2(_fp(a), _fp(b), a.size)

    def heap_topk(self, vals, k):
        vals = _f32(vals)
        D = np.empty(k, np.float32)
        I = np.empty(k, np.int64)
        self.L.orc_heap_topk(vals.size, _fp(vals), k, _fp(D), _ip(I))
        return D, I

    def coarse(self, q, cent, nprobe):
        q, cent = _f32(q), _f32(cent)
        nq, d = q.shape
        D = np.empty((nq, nprobe), np.float32)
        I = np.empty((nq, nprobe), np.int64)
        self.L.orc_coarse(nq, _fp(q), d, cent.shape[0], _fp(cent), nprobe, _fp(D), _ip(I))
        return D, I

    def search(self, ix, q, k, nprobe):
        q = _f32(q)
        nq = q.shape[0]
        D = np.empty((nq, k), np.float32)
        I = np.empty((nq, k), np.int64)
        self.L.orc_search(nq, _fp(q), ix.d, ix.nlist, _fp(ix.centroids), _ip(ix.list_off), _ip(ix.ids),
                          _fp(ix.codes), nprobe, k, _fp(D), _ip(I))
        return D, I

    def search_probes(self, ix, q, probes, k):
        q, probes = _f32(q), _i64(probes)
        nq, P = probes.shape
        D = np.empty((nq, k), np.float32)
        I = np.empty((nq, k), np.int64)
        self.L.orc_search_probes(nq, _fp(q), ix.d, _ip(ix.list_off), _ip(ix.ids), _fp(ix.codes), P,
                                 _ip(probes), k, _fp(D), _ip(I))
        return D, I

    def warmup_tops(self, ix, q, probes, k, warm_lists, warm_list_size):
        q, probes = _f32(q), _i64(probes)
        nq, P = probes.shape
        tops = np.empty(nq, np.float32)
        self.L.orc_warmup_tops(nq, _fp(q), ix.d, _ip(ix.list_off), _ip(ix.ids), _fp(ix.codes), P,
                               _ip(probes), k, warm_lists, warm_list_size, _fp(tops))
        return tops

    def search_pruned(self, ix, q, probes, tops, k, cut=True):
        q, probes, tops = _f32(q), _i64(probes), _f32(tops)
        nq, P = probes.shape
        D = np.empty((nq, k), np.float32)
        I = np.empty((nq, k), np.int64)
        self.L.orc_search_pruned(nq, _fp(q), ix.d, _ip(ix.list_off), _ip(ix.ids), _fp(ix.codes), P,
                                 _ip(probes), _fp(tops), int(cut), k, _fp(D), _ip(I))
        return D, I

    def search_dimblock(self, ix, q, probes, tops, k, W, B, order, cut=True):
        q, probes, tops, order = _f32(q), _i64(probes), _f32(tops), _i64(order)
        nq, P = probes.shape
        D = np.empty((nq, k), np.float32)
        I = np.empty((nq, k), np.int64)
        self.L.orc_search_dimblock(nq, _fp(q), ix.d, _ip(ix.list_off), _ip(ix.ids), _fp(ix.codes), P,
                                   _ip(probes), _fp(tops), int(cut), W, B, _ip(order), k, _fp(D), _ip(I))
        return D, I

    def block_order(self, W, B, order_optimize=True, period=False):
        out = np.empty((B, W), np.int64)
        self.L.orc_block_order(W, B, int(order_optimize), int(period), _ip(out))
        return out

    def kmeans(self, x, nlist, niter=20, seed=6666, max_pts=256):
        x = _f32(x)
        n, d = x.shape
        c = np.empty((nlist, d), np.float32)
        self.L.orc_kmeans(n, _fp(x), d, nlist, niter, seed, max_pts, _fp(c))
        return c

    def kmeans_indices(self, n, nlist, seed=6666, max_pts=256):
        m = min(n, nlist * max_pts)
        s = np.empty(m, np.int64)
        i = np.empty(nlist, np.int64)
        self.L.orc_kmeans_indices(n, nlist, seed, max_pts, _ip(s), _ip(i))
        return s, i

    def add(self, x, cent):
        x, cent = _f32(x), _f32(cent)
        n, d = x.shape
        nlist = cent.shape[0]
        off = np.empty(nlist + 1, np.int64)
        ids = np.empty(n, np.int64)
        codes = np.empty((n, d), np.float32)
        norms = np.empty(n, np.float32)
        self.L.orc_add(n, _fp(x), d, nlist, _fp(cent), _ip(off), _ip(ids), _fp(codes), _fp(norms))
        return IndexData(cent.copy(), off, ids, codes, norms)

    def bruteforce_f64(self, q, x, k):
        q, x = _f32(q), _f32(x)
        nq, d = q.shape
        D = np.empty((nq, k), np.float64)
        I = np.empty((nq, k), np.int64)
        self.L.orc_bruteforce_f64(nq, _fp(q), x.shape[0], _fp(x), d, k, D.ctypes.data_as(_d), _ip(I))
        return D, I


class IndexData:
    """CSR view of an IVF index (centroids, list offsets, ids, codes, norms)."""

    def __init__(self, centroids, list_off, ids, codes, norms=None):
        self.centroids = _f32(centroids)
        self.list_off = _i64(list_off)
        self.ids = _i64(ids)
        self.codes = _f32(codes)
        self.norms = None if norms is None else _f32(norms)
        self.nlist, self.d = self.centroids.shape

    @property
    def list_sizes(self):
        return np.diff(self.list_off)


class RefIndex:
    """The reference's own harmony::Index (ORIGINAL mode), via oracle/_ref."""

    _L = None
    build_kind = ""

    @classmethod
    def lib(cls):
        if cls._L is None:
            path, cls.build_kind = reference_build()
            if not os.path.exists(path):
                raise FileNotFoundError(f"reference oracle not built: {path}")
            L = ctypes.CDLL(path)
            L.ref_index_new.restype = _vp
            L.ref_index_new.argtypes = [_sz, _sz, _sz]
            L.ref_index_free.argtypes = [_vp]
            L.ref_train.argtypes = [_vp, _sz, _f]
            L.ref_add.argtypes = [_vp, _sz, _f]
            L.ref_set_nprobe.argtypes = [_vp, _sz]
            L.ref_nprobe.restype = _sz
            L.ref_nprobe.argtypes = [_vp]
            L.ref_d.restype = _sz
            L.ref_d.argtypes = [_vp]
            L.ref_nlist.restype = _sz
            L.ref_nlist.argtypes = [_vp]
            L.ref_search.argtypes = [_vp, _sz, _f, _sz, _f, _i]
            L.ref_save.restype = ctypes.c_int
            L.ref_save.argtypes = [_vp, ctypes.c_char_p]
            L.ref_load.restype = _vp
            L.ref_load.argtypes = [ctypes.c_char_p]
            L.ref_centroids.argtypes = [_vp, _f]
            L.ref_list_size.restype = _sz
            L.ref_list_size.argtypes = [_vp, _sz]
            L.ref_list_copy.argtypes = [_vp, _sz, _i, _f, _f]
            L.ref_probe_lists.argtypes = [_vp, _sz, _f, _i]
            L.ref_warmup_tops.argtypes = [_vp, _sz, _f, _sz, _sz, _sz, _f]
            L.ref_search_pruned.argtypes = [_vp, _sz, _f, _sz, _sz, _sz, ctypes.c_int, _f, _i]
            L.ref_block_order.argtypes = [_sz, _sz, ctypes.c_int, _i]
            L.ref_heap_topk.argtypes = [_sz, _f, _sz, _f, _i]
            L.ref_l2.restype = ctypes.c_float
            L.ref_l2.argtypes = [_f, _f, _sz]
            _cp, _ip32 = ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)
            L.ref_load_fvecs.restype = _sz
            L.ref_load_fvecs.argtypes = [_cp, ctypes.c_int, ctypes.c_int, _f, _ip32]
            L.ref_load_bvecs.restype = _sz
            L.ref_load_bvecs.argtypes = [_cp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_uint8), _ip32]
            L.ref_load_xvecs.restype = _sz
            L.ref_load_xvecs.argtypes = [_cp, ctypes.c_int, ctypes.c_int, _f, _ip32]
            for fn in ("ref_calculate_recall", "ref_calculate_recall_loose", "ref_calculate_r2"):
                getattr(L, fn).restype = ctypes.c_float
                getattr(L, fn).argtypes = [_i, _f, _i, _f, _sz, _sz, _sz]
            L.ref_stats_csv.argtypes = [_cp, ctypes.c_int, _cp, _cp, ctypes.c_int, _i, _d]
            L.ref_write_results.argtypes = [_i, _f, _sz, _sz, _cp]
            L.ref_load_results.argtypes = [_cp, _i, _f, _sz, _sz]
            L.ref_set_threads.argtypes = [ctypes.c_int]
            L.ref_max_threads.restype = ctypes.c_int
            cls._L = L
        return cls._L

    @classmethod
    def available(cls):
        return os.path.exists(REF_SO)

    def __init__(self, d=0, nlist=0, nprobe=0, _handle=None):
        self.L = self.lib()
        self.h = _handle if _handle is not None else self.L.ref_index_new(d, nlist, nprobe)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_index_free(self.h)
            self.h = None

    @classmethod
    def load(cls, path):
        h = cls.lib().ref_load(path.encode())
        if not h:
            raise IOError(f"reference load_index failed: {path}")
        return cls(_handle=h)

    @property
    def d(self):
        return self.L.ref_d(self.h)

    @property
    def nlist(self):
        return self.L.ref_nlist(self.h)

    @property
    def nprobe(self):
        return self.L.ref_nprobe(self.h)

    @nprobe.setter
    def nprobe(self, v):
        self.L.ref_set_nprobe(self.h, v)

    def train(self, x):
        x = _f32(x)
        self.L.ref_train(self.h, x.shape[0], _fp(x))

    def add(self, x):
        x = _f32(x)
        self.L.ref_add(self.h, x.shape[0], _fp(x))

    def search(self, q, k):
        q = _f32(q)
        nq = q.shape[0]
        D = np.empty((nq, k), np.float32)
        I = np.empty((nq, k), np.int64)
        self.L.ref_search(self.h, nq, _fp(q), k, _fp(D), _ip(I))
        return D, I

    def save(self, path):
        if self.L.ref_save(self.h, path.encode()) != 0:
            raise IOError(f"reference save_index failed: {path}")

    def probe_lists(self, q):
        q = _f32(q)
        out = np.empty((q.shape[0], self.nprobe), np.int64)
        self.L.ref_probe_lists(self.h, q.shape[0], _fp(q), _ip(out))
        return out

    def warmup_tops(self, q, k, warm_lists=10, warm_list_size=None):
        q = _f32(q)
        tops = np.empty(q.shape[0], np.float32)
        self.L.ref_warmup_tops(self.h, q.shape[0], _fp(q), k, warm_lists,
                               k if warm_list_size is None else warm_list_size, _fp(tops))
        return tops

    def search_pruned(self, q, k, warm_lists=10, warm_list_size=None, cut=True):
        q = _f32(q)
        nq = q.shape[0]
        D = np.empty((nq, k), np.float32)
        I = np.empty((nq, k), np.int64)
        self.L.ref_search_pruned(self.h, nq, _fp(q), k, warm_lists, k if warm_list_size is None else warm_list_size,
                                 int(cut), _fp(D), _ip(I))
        return D, I

    def index_data(self) -> IndexData:
        d, nlist = self.d, self.nlist
        cent = np.empty((nlist, d), np.float32)
        self.L.ref_centroids(self.h, _fp(cent))
        sizes = np.array([self.L.ref_list_size(self.h, l) for l in range(nlist)], np.int64)
        off = np.zeros(nlist + 1, np.int64)
        np.cumsum(sizes, out=off[1:])
        nb = int(off[-1])
        ids = np.empty(nb, np.int64)
        codes = np.empty((nb, d), np.float32)
        norms = np.empty(nb, np.float32)
        for l in range(nlist):
            if sizes[l]:
                a, b = off[l], off[l + 1]
                sl_i = ids[a:b]
                sl_c = codes[a:b]
                sl_n = norms[a:b]
                self.L.ref_list_copy(self.h, l, _ip(sl_i), _fp(sl_c), _fp(sl_n))
        return IndexData(cent, off, ids, codes, norms)

    @classmethod
    def block_order(cls, W, B, order_optimize=True):
        out = np.empty((B, W), np.int64)
        cls.lib().ref_block_order(W, B, int(order_optimize), _ip(out))
        return out

    @classmethod
    def heap_topk(cls, vals, k):
        vals = _f32(vals)
        D = np.empty(k, np.float32)
        I = np.empty(k, np.int64)
        cls.lib().ref_heap_topk(vals.size, _fp(vals), k, _fp(D), _ip(I))
        return D, I

    # ---- the query driver's evaluation helpers (src/utils.h, src/stats.h) ----

    @classmethod
    def _load(cls, fn, path, bounds, dtype):
        d = ctypes.c_int()
        p = path.encode()
        n = fn(p, bounds[0], bounds[1], None, ctypes.byref(d))
        out = np.empty((n, d.value), dtype)
        fn(p, bounds[0], bounds[1], out.ctypes.data_as(ctypes.POINTER(np.ctypeslib.as_ctypes_type(dtype))),
           ctypes.byref(d))
        return out

    @classmethod
    def load_fvecs(cls, path, bounds=(1, 0)):
        return cls._load(cls.lib().ref_load_fvecs, path, bounds, np.float32)

    @classmethod
    def load_bvecs(cls, path, bounds=(1, 0)):
        return cls._load(cls.lib().ref_load_bvecs, path, bounds, np.uint8)

    @classmethod
    def load_xvecs(cls, path, bounds=(1, 0)):
        return cls._load(cls.lib().ref_load_xvecs, path, bounds, np.float32)

    @classmethod
    def _measure(cls, fn, I, D, GT, GD, k, gt_k):
        I, GT = _i64(I), _i64(GT)
        D, GD = _f32(D), _f32(GD)
        return np.float32(fn(_ip(I), _fp(D), _ip(GT), _fp(GD), I.size // k, k, gt_k))

    @classmethod
    def calculate_recall(cls, I, D, GT, GD, k, gt_k=0):
        return cls._measure(cls.lib().ref_calculate_recall, I, D, GT, GD, k, gt_k)

    @classmethod
    def calculate_recall_loose(cls, I, D, GT, GD, k, gt_k=0):
        return cls._measure(cls.lib().ref_calculate_recall_loose, I, D, GT, GD, k, gt_k)

    @classmethod
    def calculate_r2(cls, I, D, GT, GD, k, gt_k=0):
        return cls._measure(cls.lib().ref_calculate_r2, I, D, GT, GD, k, gt_k)

    @classmethod
    def write_results(cls, I, D, path):
        I, D = _i64(I), _f32(D)
        nq, k = I.shape
        cls.lib().ref_write_results(_ip(I), _fp(D), nq, k, path.encode())

    @classmethod
    def load_results(cls, path, nq, k):
        I = np.zeros((nq, k), np.int64)
        D = np.zeros((nq, k), np.float32)
        cls.lib().ref_load_results(path.encode(), _ip(I), _fp(D), nq, k)
        return I, D

    _STATS_INT = ["nlist", "nprobe", "opt_level", "total_count", "skip_triangle_count", "skip_triangle_large_count",
                  "skip_subnn_L2_count", "skip_subnn_IP_count", "simi_update_count", "check_subnn_L2_ele_count",
                  "check_subnn_IP_ele_count", "check_subnn_L2_count", "check_subnn_IP_count", "nb", "nq", "d", "k",
                  "divideIVF", "disableOrderOptimize", "blockSend", "pruning", "block", "worker", "group", "team"]
    _STATS_DBL = ["simi_ratio", "faiss_query_time", "query_time", "original_time", "recall", "r2", "variance",
                  "trainTime", "addTime", "preSearchTime", "inBalanceRatio", "inBalanceRatioTeam", "brute_ratio"]

    @classmethod
    def stats_csv(cls, path, append, dataset, record, my=False):
        """The reference's Stats::toCsv / myToCsv of the fields of `record`."""
        iv = np.array([int(getattr(record, f)) for f in cls._STATS_INT], np.int64)
        dv = np.array([float(getattr(record, f)) for f in cls._STATS_DBL], np.float64)
        cls.lib().ref_stats_csv(path.encode(), int(append), dataset.encode(), record.mode.encode(), int(my),
                                _ip(iv), dv.ctypes.data_as(_d))

    @classmethod
    def l2(cls, a, b):
        a, b = _f32(a), _f32(b)
        return cls.lib().ref_l2(_fp(a), _fp(b), a.size)

    @classmethod
    def set_threads(cls, n):
        cls.lib().ref_set_threads(n)


_restated = None


def restated() -> _Restated:
    global _restated
    if _restated is None:
        _restated = _Restated()
    return _restated

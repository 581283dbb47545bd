"""Evaluation harness of the reference's query driver, so that runs of this
library give numbers and CSV rows that compare directly with the reference's:

* the vector-file loaders of src/utils.h:187-407 (fvecs, bvecs, text rows,
  and the extension dispatch), with the reference's 1-based inclusive row
  bounds, and its result / ground-truth files (src/utils.h:565-620);
* the recall measures and r2 of src/utils.h:631-755;
* the Stats CSV rows of src/stats.h:101-125 (``toCsv`` and ``myToCsv``),
  with the reference's column names and number formatting.

Host-side numpy only: none of this runs on the GPU.
"""
from __future__ import annotations

import os
from dataclasses import dataclass
from typing import Optional, Tuple

import numpy as np

FEPS = 1e-4  # src/utils.h:630, 660


def _rows(bounds: Tuple[int, int], nmax: int) -> Tuple[int, int]:
    """Rows a..b, 1-based and inclusive, b = 0 meaning the last row (the
    loaders' ``bounds`` argument).  Bounds outside 1..nmax raise ValueError
    where the reference asserts."""
    a, b = int(bounds[0]), int(bounds[1])
    b = nmax if b == 0 else b
    if not (a >= 1 and b <= nmax and b >= a):
        raise ValueError(f"rows {a}..{b} outside 1..{nmax}")
    return a, b


def _header_dim(path: str) -> int:
    with open(path, "rb") as f:
        head = f.read(4)
    if len(head) < 4:
        raise ValueError(f"{path}: no dimension header")
    return int(np.frombuffer(head, "<i4")[0])


def fvecs_info(path: str) -> Tuple[int, int]:
    """(rows, d) of an fvecs file, src/utils.h:187-202."""
    d = _header_dim(path)
    return os.path.getsize(path) // (4 + 4 * d), d


def bvecs_info(path: str) -> Tuple[int, int]:
    """(rows, d) of a bvecs file as src/utils.h:269-284 counts them:
    file size // (4 + d)."""
    d = _header_dim(path)
    return os.path.getsize(path) // (4 + d), d


def tvecs_info(path: str) -> Tuple[int, int]:
    """(rows, d) of a text vector file, src/utils.h:238-267: every line is a
    row; d is the first line's field count minus its leading label."""
    with open(path, "r") as f:
        lines = f.read().splitlines()
    d = lines[0].count(",") if lines else 0
    return len(lines), d


def xvecs_info(path: str) -> Tuple[int, int]:
    """loadXvecsInfo (src/utils.h:321-332): dispatch on the extension."""
    if path.endswith(".fvecs"):
        return fvecs_info(path)
    if path.endswith(".bvecs"):
        return bvecs_info(path)
    if path.endswith(".txt"):
        return tvecs_info(path)
    raise ValueError("no support file")


def load_fvecs(path: str, bounds: Tuple[int, int] = (1, 0)) -> np.ndarray:
    """Rows a..b of an fvecs file (per row: int32 d, then d float32), as
    src/utils.h:204-237 reads them; returns a (rows, d) float32 array."""
    d = _header_dim(path)
    vs = 4 + 4 * d
    nmax = os.path.getsize(path) // vs
    a, b = _rows(bounds, nmax)
    m = np.memmap(path, dtype=np.uint8, mode="r")
    rec = np.asarray(m[(a - 1) * vs:b * vs]).reshape(b - a + 1, vs)
    return np.ascontiguousarray(rec[:, 4:]).view("<f4").astype(np.float32, copy=False)


def load_bvecs(path: str, bounds: Tuple[int, int] = (1, 0), reference_offsets: bool = False) -> np.ndarray:
    """Rows a..b of a bvecs file (per row: int32 d, then d uint8) as a
    (rows, d) uint8 array.

    The reference's loadBvecs (src/utils.h:286-319) counts (size - 4) // (4 + d)
    rows, seeks to 4 + (a - 1)(4 + d) and then skips 4 more bytes before each
    row, so every row it returns starts 4 bytes into its record: the record's
    bytes 4..d-1 followed by the next record's 4-byte dimension.
    ``reference_offsets=True`` returns exactly those bytes (for numbers that
    must match a reference run); the default reads the records as written.
    """
    d = _header_dim(path)
    vs = 4 + d
    size = os.path.getsize(path)
    m = np.memmap(path, dtype=np.uint8, mode="r")
    if not reference_offsets:
        a, b = _rows(bounds, size // vs)
        rec = np.asarray(m[(a - 1) * vs:b * vs]).reshape(b - a + 1, vs)
        return np.ascontiguousarray(rec[:, 4:])
    a, b = _rows(bounds, (size - 4) // vs)
    n = b - a + 1
    start = 8 + (a - 1) * vs
    flat = np.zeros(n * vs, np.uint8)
    chunk = np.asarray(m[start:min(size, start + n * vs)])
    flat[:chunk.size] = chunk
    return np.ascontiguousarray(flat.reshape(n, vs)[:, :d])


def load_bvecs_as_float(path: str, bounds: Tuple[int, int] = (1, 0), reference_offsets: bool = False) -> np.ndarray:
    """loadBvecs2Fvecs (src/utils.h:321-331): the bvecs rows as float32."""
    return load_bvecs(path, bounds, reference_offsets).astype(np.float32)


def load_tvecs(path: str, bounds: Tuple[int, int] = (1, 0)) -> np.ndarray:
    """Text rows 'label,v1,...,vd' (src/utils.h:346-390): the first field of
    every line is skipped, the others are float32; d is the first row's
    length, and every row must hold at least d values."""
    with open(path, "r") as f:
        lines = f.read().splitlines()
    rows = [ln.split(",")[1:] for ln in lines]
    d = len(rows[0]) if rows else 0
    a, b = _rows(bounds, len(rows))
    out = np.empty((b - a + 1, d), np.float32)
    for i in range(a - 1, b):
        if len(rows[i]) < d:
            raise ValueError(f"{path}: line {i + 1} holds {len(rows[i])} values, the first line {d}")
        out[i - (a - 1)] = np.array([float(v) for v in rows[i][:d]], np.float32)
    return out


def load_xvecs(path: str, bounds: Tuple[int, int] = (1, 0), reference_offsets: bool = False) -> np.ndarray:
    """loadXvecs (src/utils.h:392-403): fvecs, bvecs (as float32) or text rows
    by extension; text files are read whole (the reference passes no bounds)."""
    if path.endswith(".fvecs"):
        return load_fvecs(path, bounds)
    if path.endswith(".bvecs"):
        return load_bvecs_as_float(path, bounds, reference_offsets)
    if path.endswith(".txt"):
        return load_tvecs(path)
    raise ValueError("no support file")


def write_results(I, D, path: str) -> None:
    """writeResultsToFile (src/utils.h:565-594): a result or ground-truth file.
    A path ending in "txt" gets one line per query of "label distance" pairs
    (distances fixed to 6 decimals); any other path gets the int64 labels then
    the float32 distances, raw.  Missing parent directories are created."""
    I = np.ascontiguousarray(I, np.int64)
    D = np.ascontiguousarray(D, np.float32)
    if I.shape != D.shape or I.ndim != 2:
        raise ValueError("labels and distances must both be nq x k")
    parent = os.path.dirname(path)
    if parent:
        os.makedirs(parent, exist_ok=True)
    if path.endswith("txt"):
        with open(path, "w") as f:
            for li, di in zip(I, D):
                f.write(" ".join(f"{int(a)} {float(b):.6f}" for a, b in zip(li, di)) + "\n")
    else:
        with open(path, "wb") as f:
            f.write(I.tobytes())
            f.write(D.tobytes())


def load_results(path: str, nq: int, k: int) -> Tuple[np.ndarray, np.ndarray]:
    """loadResults (src/utils.h:596-620): (labels int64, distances float32),
    each nq x k, from a file written by write_results or by the reference."""
    if path.endswith("txt"):
        with open(path, "r") as f:
            tok = f.read().split()
        if len(tok) < 2 * nq * k:
            raise ValueError(f"{path}: {len(tok) // 2} pairs, {nq * k} expected")
        pairs = np.array(tok[:2 * nq * k], dtype=object).reshape(nq * k, 2)
        I = np.array([int(t) for t in pairs[:, 0]], np.int64).reshape(nq, k)
        D = np.array([float(t) for t in pairs[:, 1]], np.float32).reshape(nq, k)
        return I, D
    raw = np.fromfile(path, dtype=np.uint8)
    need = nq * k * 12
    if raw.size < need:
        raise ValueError(f"{path}: {raw.size} bytes, {need} expected")
    I = raw[:nq * k * 8].view(np.int64).reshape(nq, k).copy()
    D = raw[nq * k * 8:need].view(np.float32).reshape(nq, k).copy()
    return I, D


def _valid_prefix(I: np.ndarray) -> np.ndarray:
    """Per row, True up to (not including) the first -1: the reference's
    loops stop there."""
    return np.cumprod(I != -1, axis=1).astype(bool)


def _prep(I, D, GT, GD, k, gt_k):
    I = np.asarray(I, np.int64).reshape(-1, k)
    D = np.asarray(D, np.float32).reshape(-1, k)
    gt_k = k if gt_k == 0 else gt_k
    if k > gt_k:
        raise ValueError("k should be less than or equal to gt_k.")
    GT = np.asarray(GT, np.int64).reshape(-1)
    GD = np.asarray(GD, np.float32).reshape(-1)
    return I, D, GT, GD, gt_k


def calculate_recall(I, D, GT, GD, k: int, gt_k: int = 0) -> np.float32:
    """calculate_recall (src/utils.h:661-732), L2: the fraction of the nq x k
    result slots (up to each row's first -1) whose id is among the query's
    first k ground-truth ids.  A negative first distance gives 0."""
    I, D, GT, GD, gt_k = _prep(I, D, GT, GD, k, gt_k)
    nq = I.shape[0]
    if D.size and D.flat[0] < 0:
        return np.float32(0.0)
    G = GT.reshape(nq, gt_k)[:, :k]
    valid = _valid_prefix(I)
    hits = sum(int(np.count_nonzero(np.isin(I[i][valid[i]], G[i]))) for i in range(nq))
    return np.float32(hits) / np.float32(nq * k)


def calculate_recall_loose(I, D, GT, GD, k: int, gt_k: int = 0) -> np.float32:
    """calculate_recall_loose (src/utils.h:631-658), L2: a result slot counts
    when its id is a ground-truth id, or its distance is below the k-th
    ground-truth distance or within 1e-4 of it.  The k-th distance is read at
    GD[i * k + k - 1], with stride k as the reference reads it, whatever gt_k."""
    I, D, GT, GD, gt_k = _prep(I, D, GT, GD, k, gt_k)
    nq = I.shape[0]
    if D.size and D.flat[0] < 0:
        return np.float32(0.0)
    G = GT.reshape(nq, gt_k)[:, :k]
    maxdis = GD[np.arange(nq) * k + k - 1][:, None]
    valid = _valid_prefix(I)
    ok = np.zeros(I.shape, bool)
    for i in range(nq):
        ok[i] = np.isin(I[i], G[i])
    close = np.abs(D - maxdis) <= FEPS
    hits = np.count_nonzero(valid & (ok | (D < maxdis) | close))
    return np.float32(hits) / np.float32(nq * k)


def calculate_r2(I, D, GT, GD, k: int, gt_k: int = 0) -> np.float32:
    """calculate_r2 (src/utils.h:734-755): sum(D) / sum(GD) - 1 over the result
    slots up to each row's first -1, both sums accumulated in float32 in row
    order."""
    I, D, GT, GD, gt_k = _prep(I, D, GT, GD, k, gt_k)
    nq = I.shape[0]
    valid = _valid_prefix(I)
    G = GD.reshape(nq, gt_k)[:, :k]
    s = np.cumsum(D[valid], dtype=np.float32)
    g = np.cumsum(G[valid], dtype=np.float32)
    s_sum = s[-1] if s.size else np.float32(0.0)
    g_sum = g[-1] if g.size else np.float32(0.0)
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.float32(np.float32(s_sum) / np.float32(g_sum)) - np.float32(1.0)


# ---- Stats CSV rows -------------------------------------------------------

_TO_CSV = ["dataset", "nlist", "nprobe", "opt_level", "simi_ratio", "tri", "tri_large", "subnn_L2", "subnn_IP",
           "simi_update_rate", "check_L2", "check_IP", "time_speedup", "pruning_speedup", "query_time", "recall",
           "r2"]
_MY_TO_CSV = ["dataset", "mode", "nb", "nq", "d", "nlist", "nprobe", "k", "divideIVF", "orderOptimize",
              "UnblockSend", "cut", "block", "worker", "group", "team", "time_speedup", "query_time",
              "original_time", "recall", "r2", "variance", "train_time", "add_time", "preSearch_time", "ratio",
              "teamRatio", "brute_ratio"]


def _f32s(x) -> str:
    """A float field as the reference's CsvWriter writes it: fixed, 7 digits."""
    return f"{float(np.float32(x)):.7f}"


def _f64s(x) -> str:
    """A double field: fixed, 16 digits."""
    return f"{float(x):.16f}"


@dataclass
class StatsRecord:
    """The fields of the reference's Stats (src/stats.h:14-56) that its CSV
    rows carry, under the reference's names.  Counters of the reference's
    pruning statistics stay 0 for a GPU search (it does not count them)."""
    nlist: int = 0
    nprobe: int = 0
    opt_level: int = 0
    simi_ratio: float = 0.0
    total_count: int = 0
    skip_triangle_count: int = 0
    skip_triangle_large_count: int = 0
    skip_subnn_L2_count: int = 0
    skip_subnn_IP_count: int = 0
    simi_update_count: int = 0
    check_subnn_L2_ele_count: int = 0
    check_subnn_IP_ele_count: int = 0
    check_subnn_L2_count: int = 0
    check_subnn_IP_count: int = 0
    nb: int = 0
    nq: int = 0
    d: int = 0
    k: int = 0
    mode: str = ""
    divideIVF: bool = False
    disableOrderOptimize: bool = False
    blockSend: bool = False
    pruning: bool = False
    block: int = 0
    worker: int = 0
    group: int = 0
    team: int = 0
    faiss_query_time: float = 0.0
    query_time: float = 0.0
    original_time: float = 0.0
    recall: float = 0.0
    r2: float = 0.0
    variance: float = 0.0
    trainTime: float = 0.0
    addTime: float = 0.0
    preSearchTime: float = 0.0
    inBalanceRatio: float = 0.0
    inBalanceRatioTeam: float = 0.0
    brute_ratio: float = 0.0

    def summary(self) -> dict:
        """Stats::summary (src/stats.h:70-82): the derived rates, each computed
        in double and stored as float32."""
        dis = (self.total_count - self.skip_triangle_count - self.skip_triangle_large_count
               - self.skip_subnn_L2_count - self.skip_subnn_IP_count) % (1 << 64)
        f = np.float32
        return {
            "dis_calculate_count": dis,
            "simi_update_rate": f(0) if dis == 0 else f(100.0 * self.simi_update_count / dis),
            "check_subnn_IP": f(0) if self.check_subnn_IP_count == 0 else
            f(1.0 * self.check_subnn_IP_ele_count / self.check_subnn_IP_count),
            "check_subnn_L2": f(0) if self.check_subnn_L2_count == 0 else
            f(1.0 * self.check_subnn_L2_ele_count / self.check_subnn_L2_count),
            "time_speedup": f(0) if self.query_time == 0 else f(100.0 * self.faiss_query_time / self.query_time),
            "pruning_speedup": f(0) if dis == 0 else f(100.0 * self.total_count / dis),
        }

    @staticmethod
    def _write(path: str, header, row, append: bool) -> None:
        exists = append and os.path.exists(path)
        with open(path, "a" if exists else "w") as f:
            if not exists:
                f.write(",".join(header) + "\n")
            f.write(",".join(row) + "\n")

    def to_csv(self, path: str, append: bool, dataset: str = "Unknown") -> None:
        """Stats::toCsv (src/stats.h:90-103): one row, with the header when the
        file is new or append is False."""
        s = self.summary()
        hundred = np.float32(100)
        row = [dataset, str(self.nlist), str(self.nprobe), str(int(self.opt_level)), _f32s(self.simi_ratio),
               str(self.skip_triangle_count), str(self.skip_triangle_large_count), str(self.skip_subnn_L2_count),
               str(self.skip_subnn_IP_count), _f32s(s["simi_update_rate"] / hundred), _f32s(s["check_subnn_L2"]),
               _f32s(s["check_subnn_IP"]), _f32s(s["time_speedup"] / hundred), _f32s(s["pruning_speedup"] / hundred),
               _f64s(self.query_time), _f64s(self.recall), _f64s(self.r2)]
        self._write(path, _TO_CSV, row, append)

    def my_to_csv(self, path: str, append: bool, dataset: str = "Unknown") -> None:
        """Stats::myToCsv (src/stats.h:104-125)."""
        s = self.summary()
        b = lambda v: "1" if v else "0"  # noqa: E731
        row = [dataset, self.mode, str(self.nb), str(self.nq), str(self.d), str(self.nlist), str(self.nprobe),
               str(self.k), b(self.divideIVF), b(not self.disableOrderOptimize), b(not self.blockSend), b(self.pruning),
               str(self.block), str(self.worker), str(self.group), str(self.team), _f32s(s["time_speedup"]),
               _f64s(self.query_time), _f64s(self.original_time), _f64s(self.recall), _f64s(self.r2),
               _f64s(self.variance), _f64s(self.trainTime), _f64s(self.addTime), _f64s(self.preSearchTime),
               _f64s(self.inBalanceRatio), _f64s(self.inBalanceRatioTeam), _f64s(self.brute_ratio)]
        self._write(path, _MY_TO_CSV, row, append)

    @classmethod
    def from_search(cls, index, stats, nb: Optional[int] = None, **fields) -> "StatsRecord":
        """A record for one ``Index.search`` call: nlist, d and nb from the
        index, nprobe, k, nq and query_time from the returned Stats; any other
        field by keyword (recall, r2, mode, ...)."""
        d, nlist, ntotal, _ = index._info()
        rec = cls(nlist=nlist, nprobe=stats.nprobe, nb=ntotal if nb is None else nb, nq=stats.nq, d=d, k=stats.k,
                  query_time=stats.query_time)
        for key, val in fields.items():
            if not hasattr(rec, key):
                raise AttributeError(f"StatsRecord has no field {key}")
            setattr(rec, key, val)
        return rec

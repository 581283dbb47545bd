"""Parity checks between two top-k results of the IVF-flat search.

The reference admits a candidate only when its distance is strictly below
the heap top (src/IVFScan.hpp:267) and heap-sorts the result, so which of
several equal distances it keeps depends on its heap's history.  Parity is
therefore: per query the sorted distances are identical bit for bit, and the
ids agree for every distance value below the k-th; at the k-th distance
(an exact tie across the boundary) ids may differ but each must really be at
that distance.
"""
import numpy as np

FLT_MAX = np.finfo(np.float32).max


def assert_topk_parity(D, I, Dr, Ir, dist_of=None, label=""):
    D = np.asarray(D, np.float32)
    Dr = np.asarray(Dr, np.float32)
    I = np.asarray(I, np.int64)
    Ir = np.asarray(Ir, np.int64)
    assert D.shape == Dr.shape and I.shape == Ir.shape, (D.shape, Dr.shape)
    bad = np.nonzero(np.any(D.view(np.uint32) != Dr.view(np.uint32), axis=1))[0]
    assert bad.size == 0, (f"{label}: distances differ for {bad.size} queries; first q={bad[0]}\n"
                           f" got {D[bad[0]]}\n want {Dr[bad[0]]}")
    nq, k = D.shape
    for q in range(nq):
        if np.array_equal(I[q], Ir[q]):
            continue
        kth = Dr[q, -1]
        for v in np.unique(Dr[q]):
            sel = Dr[q] == v
            a, b = set(I[q][sel].tolist()), set(Ir[q][sel].tolist())
            if v == kth and v != FLT_MAX:
                if dist_of is not None:
                    for i in a - b:
                        assert dist_of(q, i) == v, f"{label}: q={q} id {i} is not at the tied k-th distance"
                continue
            assert a == b, f"{label}: q={q} ids at distance {v} differ: {sorted(a)} vs {sorted(b)}"
    return True


def recall_at_k(I, gt, k):
    I = np.asarray(I)[:, :k]
    gt = np.asarray(gt)[:, :k]
    hit = 0
    for a, b in zip(I, gt):
        hit += len(set(a.tolist()) & set(b.tolist()))
    return hit / float(gt.shape[0] * k)


def assert_probe_parity(P, D, Pr, Dr, dist_of=None, label=""):
    """Probe rows of the coarse quantizer: same distances bit for bit; the
    ids of each run of equal distances agree as sets, except the run at the
    last position, whose ids must each lie at that distance."""
    assert_topk_parity(D, P, Dr, Pr, dist_of, label)


def write_index_file(path, cent, lists=()):
    """Index file in the reference's format (src/Index.cpp:1708-1770,
    src/IVF.cpp:76-134): header, centroids, then per non-empty list its id,
    size, d, sub_k, opt, ids, codes and norms.  lists: (list_id, ids, codes)."""
    import struct
    cent = np.ascontiguousarray(cent, np.float32)
    nlist, d = cent.shape
    with open(path, "wb") as f:
        f.write(struct.pack("<QQiiQQQ", d, nlist, 1, 0, 0, 1, 1))
        f.write(cent.tobytes())
        for l, ids, codes in lists:
            ids = np.ascontiguousarray(ids, np.int64)
            codes = np.ascontiguousarray(codes, np.float32).reshape(len(ids), d)
            if len(ids) == 0:
                continue
            f.write(struct.pack("<QQQQi", l, len(ids), d, 0, 0))
            f.write(ids.astype(np.uint64).tobytes())
            f.write(codes.tobytes())
            f.write(np.einsum("ij,ij->i", codes, codes).astype(np.float32).tobytes())

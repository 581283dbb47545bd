"""GPU tests of the tensor-core coarse quantizer (3-term BF16 split, exact
FP32 re-rank of nprobe + margin candidates, exact recomputation of queries
whose candidates cannot be proven sufficient).  Its probe rows must equal the
exact FP32 quantizer's and the oracle's (src/IVFScan.hpp:108-138)."""
import os
import tempfile

import numpy as np
import pytest

from harmony_b200 import CoarseQuantizer, HarmonyError, Index, SearchMode, datasets
from tests.parity import assert_probe_parity, assert_topk_parity, write_index_file

pytestmark = pytest.mark.gpu


def probes(ix, q, P, kind, margin=-1):
    ix.set_coarse_quantizer(kind, margin)
    try:
        return ix.probe_lists(q, P)
    finally:
        ix.set_coarse_quantizer(CoarseQuantizer.AUTO, -1)


def trained(d, nlist, nb, seed, offset=0.0):
    rng = np.random.default_rng(seed)
    centres = rng.standard_normal((max(nlist // 2, 4), d)).astype(np.float32) * np.float32(3.0)
    lab = rng.integers(0, centres.shape[0], nb)
    base = centres[lab] + rng.standard_normal((nb, d)).astype(np.float32) + np.float32(offset)
    ix = Index(d, nlist, 8)
    ix.train(nb, base)
    lab = rng.integers(0, centres.shape[0], 1200)
    q = centres[lab] + rng.standard_normal((1200, d)).astype(np.float32) + np.float32(offset)
    return ix, np.ascontiguousarray(q, np.float32)


@pytest.mark.parametrize("d,nlist,nq,P", [
    (128, 1000, 300, 40),
    (128, 1000, 1100, 40),  # large batch: one warp per query in the refinement
    (64, 500, 700, 120),
    (16, 37, 5, 8),
    (33, 300, 129, 17),
    (100, 130, 257, 64),
    (64, 2048, 200, 256),
    (128, 200, 50, 200),   # nprobe = nlist: every centroid is a candidate
    (128, 300, 1, 290),    # candidates reach nlist through the margin
    # The selection from 16-column chunk minima (nprobe + margin at most a
    # quarter of the chunks): full chunks; a partial last chunk with TMA
    # stores of the matrix; a partial last chunk with plain stores (nlist not
    # a multiple of 4) and the CTA-per-query refinement.
    (128, 2048, 700, 8),
    (128, 1100, 600, 1),
    (96, 3000, 520, 30),
    (64, 4090, 300, 20),
])
def test_tensor_coarse_matches_exact_and_oracle(restated, d, nlist, nq, P):
    ix, q = trained(d, nlist, max(4 * nlist, 3000), seed=d * 131 + nlist)
    q = q[:nq]
    Pt, Dt = probes(ix, q, P, CoarseQuantizer.TENSOR)
    Pe, De = probes(ix, q, P, CoarseQuantizer.EXACT)
    assert np.array_equal(Pt, Pe) and np.array_equal(Dt.view(np.uint32), De.view(np.uint32))
    Dr, Ir = restated.coarse(q, ix.centroid_codes, P)
    cent = ix.centroid_codes
    assert_probe_parity(Pt, Dt, Ir, Dr, lambda qi, c: restated.l2(q[qi], cent[c]), "tensor coarse")


def test_fallback_rows_are_exact(restated):
    """Margin 0 leaves no room for the exactness proof on most queries; the
    flagged rows are recomputed and the probes still match."""
    ix, q = trained(128, 512, 4000, seed=7)
    Pt, Dt = probes(ix, q, 32, CoarseQuantizer.TENSOR, margin=0)
    n_fb = ix.coarse_fallbacks()
    assert n_fb > 0
    Pe, De = probes(ix, q, 32, CoarseQuantizer.EXACT)
    assert np.array_equal(Pt, Pe) and np.array_equal(Dt, De)
    Pt2, _ = probes(ix, q, 32, CoarseQuantizer.TENSOR, margin=64)
    assert np.array_equal(Pt2, Pe)
    assert ix.coarse_fallbacks() < n_fb


def test_fallback_rows_on_the_chunk_selection(restated):
    """The chunk-minimum selection with margin 0: flagged rows are
    recomputed exactly (their matrix rows and chunk minima rewritten) and the
    probes still match the exact quantizer."""
    ix, q = trained(128, 2048, 8192, seed=11)
    Pt, Dt = probes(ix, q, 16, CoarseQuantizer.TENSOR, margin=0)
    assert ix.coarse_fallbacks() > 0
    Pe, De = probes(ix, q, 16, CoarseQuantizer.EXACT)
    assert np.array_equal(Pt, Pe) and np.array_equal(Dt.view(np.uint32), De.view(np.uint32))


def test_offset_data_large_norms(restated):
    """Points far from the origin: the split's error bound grows with the
    norms, so more queries take the exact route; rows stay identical."""
    ix, q = trained(96, 400, 4000, seed=11, offset=300.0)
    Pt, Dt = probes(ix, q, 24, CoarseQuantizer.TENSOR)
    Pe, De = probes(ix, q, 24, CoarseQuantizer.EXACT)
    assert np.array_equal(Pt, Pe) and np.array_equal(Dt, De)


def test_duplicate_centroids_and_ties(restated):
    """Equal centroids and integer data: exact distance ties, broken by the
    lower centroid id on both routes."""
    rng = np.random.default_rng(5)
    cent = rng.integers(0, 8, (300, 64)).astype(np.float32)
    cent[17] = cent[5]
    cent[200] = cent[5]
    cent[299] = cent[5]
    q = np.concatenate([cent[[5, 17, 42]], rng.integers(0, 8, (150, 64)).astype(np.float32)])
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "cent.index")
        write_index_file(p, cent)
        ix = Index()
        ix.load_index(p)
    Pt, Dt = probes(ix, q, 20, CoarseQuantizer.TENSOR)
    Pe, De = probes(ix, q, 20, CoarseQuantizer.EXACT)
    assert np.array_equal(Pt, Pe) and np.array_equal(Dt, De)
    assert list(Pt[0, :4]) == [5, 17, 200, 299] and (Dt[0, :4] == 0).all()
    Dr, Ir = restated.coarse(q, cent, 20)
    assert_probe_parity(Pt, Dt, Ir, Dr, lambda qi, c: restated.l2(q[qi], cent[c]), "ties")


def test_search_results_identical_across_routes():
    base, q = datasets.config2(seed=9, nb=60_000, nq=500, ncomp=200)
    ix = Index(128, 512, 24)
    ix.train(base.shape[0], base)
    ix.add(base.shape[0], base)
    ix.preSearch(0, 0, 0, 0, 0, Index.Param(mode=SearchMode.ORIGINAL), "")
    out = {}
    for kind in (CoarseQuantizer.TENSOR, CoarseQuantizer.EXACT):
        ix.set_coarse_quantizer(kind, -1)
        D = np.empty((q.shape[0], 10), np.float32)
        I = np.empty((q.shape[0], 10), np.int64)
        ix.search(q.shape[0], q, 10, D, I)
        out[kind] = (D, I)
    ix.set_coarse_quantizer(CoarseQuantizer.AUTO, -1)
    assert np.array_equal(out[CoarseQuantizer.TENSOR][0], out[CoarseQuantizer.EXACT][0])
    assert np.array_equal(out[CoarseQuantizer.TENSOR][1], out[CoarseQuantizer.EXACT][1])


def test_tensor_route_limits():
    ix, q = trained(200, 64, 2000, seed=3)
    with pytest.raises(HarmonyError):
        probes(ix, q[:4], 8, CoarseQuantizer.TENSOR)  # d > 128
    P, D = probes(ix, q[:4], 8, CoarseQuantizer.AUTO)  # AUTO takes the exact route there
    assert P.shape == (4, 8)
    with pytest.raises(HarmonyError):
        ix.set_coarse_quantizer(CoarseQuantizer.AUTO, 5000)

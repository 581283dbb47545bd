"""GPU tests of the bounded BF16 tensor-core scan (tcgen05) with exact FP32
re-rank, d <= 128 and k <= 256.

The scan appends every row whose approximate value lies under the query's
bound, and the re-rank recomputes every appended row within twice the proven
error bound of the k-th approximate value; so the result is the exact FP32
scan's, distances bit for bit and ids identical (ties broken by position like
the exact scan).  These tests demand exact equality, on every query."""
import os
import tempfile

import numpy as np
import pytest

from harmony_b200 import HarmonyError, Index, Precision, SearchMode, datasets
from tests.parity import FLT_MAX, assert_topk_parity

pytestmark = pytest.mark.gpu


def search(ix, q, k, precision=Precision.BF16, mode=SearchMode.ORIGINAL, npq=None, max_nprobe=0):
    q = np.ascontiguousarray(q, np.float32)
    ix.preSearch(0, 0, 0, 0, 0, Index.Param(mode=mode), "")
    sp = ix.search_params
    sp.precision, sp.nprobe_per_query, sp.max_nprobe = precision, npq, max_nprobe
    D = np.empty((q.shape[0], k), np.float32)
    I = np.empty((q.shape[0], k), np.int64)
    try:
        ix.search(q.shape[0], q, k, D, I)
    finally:
        sp.precision, sp.nprobe_per_query, sp.max_nprobe = Precision.FP32, None, 0
    return D, I


def assert_identical(a, b, label=""):
    (D, I), (De, Ie) = a, b
    bad = np.nonzero(np.any(D.view(np.uint32) != De.view(np.uint32), axis=1) | np.any(I != Ie, axis=1))[0]
    assert bad.size == 0, (f"{label}: {bad.size} of {D.shape[0]} queries differ; first q={bad[0]}\n"
                           f" bf16 {D[bad[0]]} {I[bad[0]]}\n fp32 {De[bad[0]]} {Ie[bad[0]]}")


def test_bf16_exact_on_integer_data(ref_lib, restated):
    """Config-1 value range, against the reference's own Index::search on its
    saved index."""
    base, q = datasets.config1()
    ref = ref_lib(128, 100, 10)
    ref.train(base)
    ref.add(base)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "c1.index")
        ref.save(p)
        ix = Index()
        ix.load_index(p)
    ix.nprobe = 10
    D, I = search(ix, q, 10)
    Dr, Ir = ref.search(q, 10)
    assert_topk_parity(D, I, Dr, Ir, lambda qi, i: restated.l2(q[qi], base[i]), "bf16 config1")


@pytest.fixture(scope="module")
def fidx():
    base, q = datasets.config2(seed=41, nb=150_000, nq=700, ncomp=300)
    ix = Index(128, 256, 16)
    ix.train(base.shape[0], base)
    ix.add(base.shape[0], base)
    return base, q, ix


@pytest.mark.parametrize("nprobe,k", [(16, 10), (64, 10), (8, 1), (32, 16), (32, 17), (16, 100), (8, 256)])
def test_bf16_equals_exact_scan(fidx, restated, nprobe, k):
    base, q, ix = fidx
    ix.nprobe = nprobe
    got = search(ix, q, k)
    exact = search(ix, q, k, precision=Precision.FP32)
    assert_identical(got, exact, f"P={nprobe} k={k}")
    # Queries whose candidate buffer overflowed were searched with the exact
    # scan (part of the design); on this far-from-origin data they are few.
    st = ix.bf16_stats()
    assert st["overflows"] == ix.bf16_fallbacks() <= 0.25 * q.shape[0], st
    assert st["reranked"] >= (q.shape[0] - st["overflows"]) * min(k, 1), st
    D, I = got
    for qi in range(0, q.shape[0], 97):
        assert D[qi, 0] == restated.l2(q[qi], base[I[qi, 0]])


def test_bf16_equals_exact_on_uniform_and_far_data():
    """Data without cluster structure (every distance close to every other),
    and data far from the origin (large norms, so the bound is wide)."""
    rng = np.random.default_rng(5)
    for shift, d in ((0.0, 128), (40.0, 96), (0.0, 33)):
        base = (rng.random((40_000, d)) + shift).astype(np.float32)
        q = (rng.random((300, d)) + shift).astype(np.float32)
        ix = Index(d, 64, 8)
        ix.train(base.shape[0], base)
        ix.add(base.shape[0], base)
        for k in (1, 10, 50):
            assert_identical(search(ix, q, k), search(ix, q, k, precision=Precision.FP32), f"shift={shift} d={d} k={k}")


def test_bf16_small_batches_and_padding(fidx):
    base, q, ix = fidx
    ix.nprobe = 24
    for n in (1, 3, 129, 257):
        assert_identical(search(ix, q[:n], 10), search(ix, q[:n], 10, precision=Precision.FP32), f"n={n}")
    rng = np.random.default_rng(3)
    b = rng.standard_normal((30, 16), dtype=np.float32)
    small = Index(16, 4, 2)
    small.train(30, b)
    small.add(30, b)
    D, I = search(small, b[:5], 20)
    De, Ie = search(small, b[:5], 20, precision=Precision.FP32)
    assert np.array_equal(D, De) and np.array_equal(I, Ie)
    assert (I == -1).any()  # fewer candidates than k: padded like heap_init
    assert ((I == -1) == (D == FLT_MAX)).all()


def test_bf16_per_query_nprobe(fidx):
    base, q, ix = fidx
    ix.nprobe = 8
    rng = np.random.default_rng(11)
    npq = rng.integers(0, 40, size=q.shape[0]).astype(np.int32)  # some queries probe nothing
    got = search(ix, q, 10, npq=npq, max_nprobe=40)
    exact = search(ix, q, 10, precision=Precision.FP32, npq=npq, max_nprobe=40)
    assert_identical(got, exact, "per-query nprobe")
    assert (got[1][npq == 0] == -1).all()


def test_bf16_duplicates_and_ties(restated):
    """Every row repeated four times and queries on top of stored rows: many
    exact ties at the k-th distance.  The bounded set holds every tied row, so
    the tie goes to the lowest position, as in the exact scan."""
    rng = np.random.default_rng(13)
    uniq = rng.standard_normal((5000, 64)).astype(np.float32)
    base = np.repeat(uniq, 4, axis=0)
    ix = Index(64, 32, 6)
    ix.train(base.shape[0], base)
    ix.add(base.shape[0], base)
    q = np.concatenate([base[::53], base[1::71] + np.float32(1e-3)])
    for k in (1, 3, 10, 30):
        assert_identical(search(ix, q, k), search(ix, q, k, precision=Precision.FP32), f"dups k={k}")


def test_bf16_overflow_is_searched_exactly(restated):
    """6000 identical rows next to the query: every one of them is within the
    bound, so the candidate buffer overflows and the query is searched again
    with the exact scan -- the result is still the exact one."""
    rng = np.random.default_rng(31)
    d = 96
    same = np.repeat(rng.standard_normal((1, d)).astype(np.float32), 6000, axis=0)
    other = (rng.standard_normal((3000, d)) * 3 + 10).astype(np.float32)
    base = np.concatenate([same, other])
    ix = Index(d, 8, 8)
    ix.train(base.shape[0], base)
    ix.add(base.shape[0], base)
    q = np.concatenate([same[:3] + np.float32(0.05), other[:5] + np.float32(0.01)])
    for k in (10, 100):
        got = search(ix, q, k)
        assert ix.bf16_fallbacks() == 3, ix.bf16_fallbacks()
        assert_identical(got, search(ix, q, k, precision=Precision.FP32), f"overflow k={k}")
        assert (got[1][:3] < 6000).all()


def test_bf16_wait_budget_gives_up_and_recovers(fidx):
    """With a budget of a few hundred cycles the scan's waits give up: the
    search fails with HB_ERR_CUDA, and with the default budget restored the
    index searches correctly."""
    base, q, ix = fidx
    ix.nprobe = 16
    exact = search(ix, q, 10, precision=Precision.FP32)
    ix.set_wait_budget(300)
    try:
        with pytest.raises(HarmonyError, match="gave up waiting"):
            search(ix, q, 10)
    finally:
        ix.set_wait_budget(0)
    assert_identical(search(ix, q, 10), exact, "after the budget test")


def test_bf16_rejects_unsupported(fidx):
    base, q, ix = fidx
    with pytest.raises(HarmonyError):
        search(ix, q[:4], 5000)  # k above the BF16 candidate capacity (4096)
    with pytest.raises(HarmonyError):
        search(ix, q[:4], 10, mode=SearchMode.DIVIDE_IVF)


def test_bf16_autotune_picks_a_config_and_keeps_results(fidx):
    """The autotuner times chunk lengths and ring depths on the first search of
    a bucket; every choice gives the exact result, and the table written out
    can be read back."""
    base, q, ix = fidx
    ix.nprobe = 16
    exact = search(ix, q, 10, precision=Precision.FP32)
    ix.set_autotune(True)
    try:
        assert_identical(search(ix, q, 10), exact, "tuning search")
        assert_identical(search(ix, q, 10), exact, "tuned search")
        table = ix.autotune_table()
        rows = [list(map(float, line.split())) for line in table.strip().splitlines()]
        assert len(rows) == 1
        nb_b, p_b, k, kpad, cr, stages, best, dflt = rows[0]
        assert (nb_b, p_b, k, kpad) == (1024, 16, 10, 128)
        assert 128 <= cr <= 4096 and 2 <= stages <= 4 and 0 < best <= dflt
        ix.set_autotune_table("1024 16 10 128 256 3 0.1 0.2\n")
        assert ix.autotune_table().split()[4:6] == ["256", "3"]
        assert_identical(search(ix, q, 10), exact, "loaded table")
        with pytest.raises(HarmonyError):
            ix.set_autotune_table("1024 16 10 128 100 3 0.1 0.2\n")  # not whole tiles
    finally:
        ix.set_autotune(False)
        ix.set_autotune_table("")

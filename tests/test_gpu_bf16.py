"""GPU tests of the BF16 tensor-core scan (tcgen05) with exact FP32 re-rank."""
import os
import tempfile

import numpy as np
import pytest

from harmony_b200 import HarmonyError, Index, Precision, SearchMode, datasets
from tests.parity import FLT_MAX, assert_topk_parity

pytestmark = pytest.mark.gpu


def search(ix, q, k, precision=Precision.BF16, mult=4, mode=SearchMode.ORIGINAL):
    q = np.ascontiguousarray(q, np.float32)
    ix.preSearch(0, 0, 0, 0, 0, Index.Param(mode=mode), "")
    ix.search_params.precision = precision
    ix.search_params.rerank_mult = mult
    D = np.empty((q.shape[0], k), np.float32)
    I = np.empty((q.shape[0], k), np.int64)
    try:
        ix.search(q.shape[0], q, k, D, I)
    finally:
        ix.search_params.precision = Precision.FP32
    return D, I


def test_bf16_exact_on_integer_data(ref_lib, restated):
    """Config-1 value range: BF16 holds every value exactly and every FP32 sum is
    exact, so the tensor-core scan ranks exactly and must match the reference."""
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


@pytest.mark.parametrize("nprobe,k", [(16, 10), (64, 10), (8, 1), (32, 16)])
def test_bf16_rerank_matches_exact_scan(fidx, restated, nprobe, k):
    base, q, ix = fidx
    ix.nprobe = nprobe
    D, I = search(ix, q, k)
    De, Ie = search(ix, q, k, precision=Precision.FP32)
    # Every returned distance is the exact FP32 distance of its id.
    for qi in range(0, q.shape[0], 37):
        for j in range(k):
            if I[qi, j] >= 0:
                assert D[qi, j] == restated.l2(q[qi], base[I[qi, j]])
    same = [np.array_equal(a, b) for a, b in zip(D.view(np.uint32), De.view(np.uint32))]
    assert np.mean(same) >= 0.995, np.mean(same)
    # Where they differ the BF16 result can only be worse, never better.
    assert (D[:, -1] >= De[:, -1]).all()


def test_bf16_small_batches_and_padding(fidx):
    base, q, ix = fidx
    ix.nprobe = 24
    for n in (1, 3, 129, 257):
        D, I = search(ix, q[:n], 10)
        De, Ie = search(ix, q[:n], 10, precision=Precision.FP32)
        assert np.mean(np.all(D == De, axis=1)) >= 0.99
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


def test_bf16_rejects_unsupported(fidx):
    base, q, ix = fidx
    with pytest.raises(HarmonyError):
        search(ix, q[:4], 5000)  # k above the BF16 candidate capacity (4096)
    with pytest.raises(HarmonyError):
        search(ix, q[:4], 10, mode=SearchMode.DIVIDE_IVF)

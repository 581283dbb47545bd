"""GPU tests of the CUDA-graph search (params.use_graph): a batch is one graph
launch captured per batch shape; results must equal the ordinary search on
every call, for new inputs of the same shape, for a new shape, and after the
index changes."""
import numpy as np
import pytest

from harmony_b200 import HarmonyError, Index, Precision, SearchMode, datasets
from tests.parity import assert_topk_parity

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    base, q = datasets.config2(seed=61, nb=120_000, nq=900, ncomp=300)
    ix = Index(128, 256, 12)
    ix.train(base.shape[0], base)
    ix.add(base.shape[0], base)
    ix.preSearch(0, 0, 0, 0, 0, Index.Param(mode=SearchMode.ORIGINAL), "")
    return base, q, ix


def run(ix, q, k, graph, precision=Precision.FP32, npq=None, max_nprobe=0):
    q = np.ascontiguousarray(q, np.float32)
    sp = ix.search_params
    sp.use_graph, sp.precision, sp.nprobe_per_query, sp.max_nprobe = graph, precision, npq, max_nprobe
    D = np.empty((q.shape[0], k), np.float32)
    I = np.empty((q.shape[0], k), np.int64)
    try:
        ix.search(q.shape[0], q, k, D, I)
    finally:
        sp.use_graph, sp.precision, sp.nprobe_per_query, sp.max_nprobe = False, Precision.FP32, None, 0
    return D, I


@pytest.mark.parametrize("prec", [Precision.FP32, Precision.BF16])
def test_graph_equals_ordinary_over_calls(setup, prec):
    base, q, ix = setup
    before = ix.launch_count()
    for call, (lo, n) in enumerate([(0, 64), (64, 64), (128, 64), (200, 17), (300, 17), (400, 64)]):
        Dg, Ig = run(ix, q[lo:lo + n], 10, True, prec)
        Do, Io = run(ix, q[lo:lo + n], 10, False, prec)
        assert np.array_equal(Dg, Do) and np.array_equal(Ig, Io), (prec, call)
    assert ix.launch_count() > before


def test_graph_per_query_nprobe(setup):
    base, q, ix = setup
    rng = np.random.default_rng(3)
    for call in range(3):
        qq = q[call * 50:(call + 1) * 50]
        npq = rng.integers(1, 40, size=qq.shape[0]).astype(np.int32)
        for prec in (Precision.FP32, Precision.BF16):
            Dg, Ig = run(ix, qq, 10, True, prec, npq=npq, max_nprobe=40)
            Do, Io = run(ix, qq, 10, False, prec, npq=npq, max_nprobe=40)
            assert_topk_parity(Dg, Ig, Do, Io, label=f"{prec.name} call {call}")


def test_graph_after_index_change(setup):
    base, q, ix = setup
    run(ix, q[:32], 10, True, Precision.BF16)
    ix2 = Index(128, 256, 12)
    ix2.train(base.shape[0], base)
    ix2.add(base.shape[0] // 2, base[: base.shape[0] // 2])
    ix2.preSearch(0, 0, 0, 0, 0, Index.Param(mode=SearchMode.ORIGINAL), "")
    for prec in (Precision.FP32, Precision.BF16):
        Dg, Ig = run(ix2, q[:32], 10, True, prec)
        Do, Io = run(ix2, q[:32], 10, False, prec)
        assert np.array_equal(Dg, Do) and np.array_equal(Ig, Io)
    ix2.add(base.shape[0], base)  # the lists change: cached graphs are dropped
    Dg, Ig = run(ix2, q[:32], 10, True, Precision.BF16)
    Do, Io = run(ix2, q[:32], 10, False, Precision.BF16)
    assert np.array_equal(Dg, Do) and np.array_equal(Ig, Io)


def test_graph_rejects_other_modes(setup):
    base, q, ix = setup
    ix.preSearch(0, 0, 0, 10, 10, Index.Param(mode=SearchMode.DIVIDE_IVF, pruning=True), "")
    try:
        with pytest.raises(HarmonyError):
            run(ix, q[:8], 10, True)
    finally:
        ix.preSearch(0, 0, 0, 0, 0, Index.Param(mode=SearchMode.ORIGINAL), "")

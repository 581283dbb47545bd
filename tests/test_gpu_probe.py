"""GPU tests of per-query nprobe: a caller-given array and the learned
predictor (a BF16 MLP trained on labels from the exact search)."""
import numpy as np
import pytest

from harmony_b200 import Index, Precision, SearchMode, datasets
from tests.parity import assert_topk_parity, recall_at_k

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    base, test, train = datasets.config5(seed=51, nb=200_000, nq=600, ntrain=12_000, ncomp=512)
    ix = Index(128, 256, 16)
    ix.train(base.shape[0], base)
    ix.add(base.shape[0], base)
    ix.preSearch(0, 0, 0, 0, 0, Index.Param(mode=SearchMode.ORIGINAL), "")
    return base, test, train, ix


def run(ix, q, k, precision=Precision.FP32, learned=False, npq=None, max_nprobe=0, target=0.0):
    q = np.ascontiguousarray(q, np.float32)
    sp = ix.search_params
    sp.precision, sp.learned_probe, sp.nprobe_per_query, sp.max_nprobe, sp.learned_target = (
        precision, learned, npq, max_nprobe, target)
    D = np.empty((q.shape[0], k), np.float32)
    I = np.empty((q.shape[0], k), np.int64)
    try:
        ix.search(q.shape[0], q, k, D, I)
    finally:
        sp.precision, sp.learned_probe, sp.nprobe_per_query, sp.max_nprobe, sp.learned_target = (
            Precision.FP32, False, None, 0, 0.0)
    return D, I


def test_nprobe_per_query_equals_fixed_nprobe(setup):
    base, test, train, ix = setup
    q = test[:48]
    npq = np.random.default_rng(5).integers(1, 40, size=q.shape[0]).astype(np.int32)
    for prec in (Precision.FP32, Precision.BF16):
        D, I = run(ix, q, 10, prec, npq=npq, max_nprobe=40)
        for i in range(q.shape[0]):
            ix.nprobe = int(npq[i])
            Dr, Ir = run(ix, q[i:i + 1], 10, prec)
            assert_topk_parity(D[i:i + 1], I[i:i + 1], Dr, Ir, label=f"{prec.name} q{i}")


def test_learned_probe_meets_calibrated_recall(setup):
    base, test, train, ix = setup
    ix.train_probe_predictor(train.shape[0], train, k=10, label_nprobe=64, target=0.95)
    thr, rec, avgp = ix.probe_calibration()
    assert len(thr) > 5 and rec.max() > 0.95 and avgp.min() < 64
    ix.nprobe = 64
    Dl, Il = run(ix, test, 10)  # the label search on the test queries
    for prec in (Precision.FP32, Precision.BF16):
        D, I = run(ix, test, 10, prec, learned=True)
        r = recall_at_k(I, Il, 10)
        assert r >= 0.93, (prec, r)
        # Every returned distance is exact.
        dl = {(qi, i): d for qi in range(test.shape[0]) for i, d in zip(Il[qi], Dl[qi])}
        for qi in range(0, test.shape[0], 50):
            for j in range(10):
                if (qi, I[qi, j]) in dl:
                    assert D[qi, j] == dl[(qi, I[qi, j])]
    # The bounded BF16 scan over the predicted probes returns the exact scan's
    # result over the same probes.
    Db, Ib = run(ix, test, 10, Precision.BF16, learned=True)
    De, Ie = run(ix, test, 10, Precision.FP32, learned=True)
    assert np.array_equal(Db.view(np.uint32), De.view(np.uint32)) and np.array_equal(Ib, Ie)
    # A higher target never lowers recall.
    D2, I2 = run(ix, test, 10, Precision.BF16, learned=True, target=0.99)
    assert recall_at_k(I2, Il, 10) >= recall_at_k(I, Il, 10) - 1e-9


def test_learned_probe_same_on_every_coarse_route(setup):
    """The tensor-core route computes the predictor's features from a narrow
    exact pass and widens only the rows that need more probes; the exact
    route selects the full width and cuts it.  Same probes, same results."""
    from harmony_b200 import CoarseQuantizer
    base, test, train, ix = setup
    ix.train_probe_predictor(train.shape[0], train, k=10, label_nprobe=64, target=0.95)
    for prec in (Precision.FP32, Precision.BF16):
        out = {}
        for kind in (CoarseQuantizer.TENSOR, CoarseQuantizer.EXACT):
            ix.set_coarse_quantizer(kind, -1)
            try:
                out[kind] = run(ix, test, 10, prec, learned=True)
                if kind == CoarseQuantizer.TENSOR:
                    # The widening pass proves nearly every row exact; a row
                    # that fails is recomputed, so many failures mean a
                    # broken candidate set.
                    assert ix.coarse_fallbacks() <= 0.05 * test.shape[0]
            finally:
                ix.set_coarse_quantizer(CoarseQuantizer.AUTO, -1)
        (Dt, It), (De, Ie) = out[CoarseQuantizer.TENSOR], out[CoarseQuantizer.EXACT]
        assert np.array_equal(Dt, De) and np.array_equal(It, Ie), prec

"""The query-driver harness (harmony_b200.harness) against the reference's
own loaders, recall / r2 measures and Stats CSV writer, compiled from its
sources into the oracle library: same arrays, same floats bit for bit, same
CSV bytes."""
import os

import numpy as np
import pytest

from harmony_b200 import harness
from harmony_b200.datasets import write_fvecs


def write_bvecs(path, x):
    x = np.asarray(x, np.uint8)
    n, d = x.shape
    rec = np.empty((n, 4 + d), np.uint8)
    rec[:, :4] = np.frombuffer(np.int32(d).tobytes(), np.uint8)
    rec[:, 4:] = x
    rec.tofile(path)


@pytest.fixture
def tmp(tmp_path):
    return str(tmp_path)


def test_fvecs_loader_matches_reference(ref_lib, tmp):
    rng = np.random.default_rng(1)
    x = rng.standard_normal((37, 24)).astype(np.float32)
    p = os.path.join(tmp, "a.fvecs")
    write_fvecs(p, x)
    for bounds in ((1, 0), (1, 1), (5, 17), (37, 37), (2, 0)):
        got = harness.load_fvecs(p, bounds)
        want = ref_lib.load_fvecs(p, bounds)
        assert got.dtype == np.float32 and np.array_equal(got.view(np.uint32), want.view(np.uint32)), bounds
    assert np.array_equal(harness.load_xvecs(p), ref_lib.load_xvecs(p))
    assert harness.fvecs_info(p) == (37, 24) == harness.xvecs_info(p)
    with pytest.raises(ValueError):
        harness.load_fvecs(p, (0, 3))
    with pytest.raises(ValueError):
        harness.load_fvecs(p, (3, 38))


def test_bvecs_loader_matches_reference(ref_lib, tmp):
    rng = np.random.default_rng(2)
    x = rng.integers(0, 256, (29, 40), dtype=np.uint8)
    p = os.path.join(tmp, "a.bvecs")
    write_bvecs(p, x)
    # The records as written.
    assert np.array_equal(harness.load_bvecs(p), x)
    assert np.array_equal(harness.load_bvecs(p, (3, 9)), x[2:9])
    # The reference's reads start 4 bytes into each record.
    for bounds in ((1, 0), (1, 1), (4, 20), (28, 28)):
        got = harness.load_bvecs(p, bounds, reference_offsets=True)
        want = ref_lib.load_bvecs(p, bounds)
        assert np.array_equal(got, want), bounds
    assert np.array_equal(harness.load_bvecs(p, reference_offsets=True)[0, :36], x[0, 4:])
    got = harness.load_xvecs(p, (2, 11), reference_offsets=True)
    assert got.dtype == np.float32 and np.array_equal(got, ref_lib.load_xvecs(p, (2, 11)))


def test_text_loader_matches_reference(ref_lib, tmp):
    rng = np.random.default_rng(3)
    x = (rng.standard_normal((12, 7)) * 100).astype(np.float32)
    p = os.path.join(tmp, "a.txt")
    with open(p, "w") as f:
        for i, row in enumerate(x):
            f.write(",".join([f"id{i}"] + [repr(float(v)) for v in row]) + "\n")
    got = harness.load_xvecs(p)
    want = ref_lib.load_xvecs(p)
    assert np.array_equal(got, want) and np.array_equal(got, x)
    assert harness.tvecs_info(p) == (12, 7)
    assert np.array_equal(harness.load_tvecs(p, (3, 5)), x[2:5])


def results(rng, nq, k, gt_k, holes=True):
    GT = np.stack([rng.permutation(1000)[:gt_k] for _ in range(nq)]).astype(np.int64)
    GD = np.sort(rng.uniform(1, 50, (nq, gt_k)).astype(np.float32), axis=1)
    I = np.where(rng.random((nq, k)) < 0.7, GT[:, :k][:, rng.permutation(k)], rng.integers(1000, 2000, (nq, k)))
    D = np.sort((GD[:, :k] + rng.normal(0, 0.5, (nq, k))).astype(np.float32), axis=1)
    D = np.abs(D)
    # Some exact ties with, and values near, the k-th ground-truth distance.
    D[:, -1] = GD[:, k - 1]
    if k > 1:
        D[::3, -2] = GD[::3, k - 1] + np.float32(5e-5)
        D[1::3, -2] = GD[1::3, k - 1] + np.float32(0.3)
    if holes:
        I[::5, k // 2:] = -1
    return I, D, GT, GD


@pytest.mark.parametrize("k,gt_k", [(10, 0), (10, 10), (10, 100), (1, 0), (100, 100)])
def test_recall_and_r2_match_reference(ref_lib, k, gt_k):
    rng = np.random.default_rng(10 + k + gt_k)
    I, D, GT, GD = results(rng, 200, k, gt_k or k)
    for ours, theirs in ((harness.calculate_recall, ref_lib.calculate_recall),
                         (harness.calculate_recall_loose, ref_lib.calculate_recall_loose),
                         (harness.calculate_r2, ref_lib.calculate_r2)):
        a = ours(I, D, GT, GD, k, gt_k)
        b = theirs(I, D, GT, GD, k, gt_k)
        assert isinstance(a, np.float32)
        assert np.float32(a).tobytes() == np.float32(b).tobytes(), (ours.__name__, a, b)


def test_recall_edge_cases(ref_lib):
    rng = np.random.default_rng(5)
    I, D, GT, GD = results(rng, 20, 10, 10, holes=False)
    D[0, 0] = -1.0  # a negative first distance gives 0
    assert harness.calculate_recall(I, D, GT, GD, 10) == ref_lib.calculate_recall(I, D, GT, GD, 10) == 0
    assert harness.calculate_recall_loose(I, D, GT, GD, 10) == 0
    with pytest.raises(ValueError):
        harness.calculate_recall(I, np.abs(D), GT, GD, 10, 5)
    # Loose recall: within 1e-4 of the k-th ground-truth distance counts,
    # 0.3 or 0.9 above it does not (a float |x|, not an integer one).
    GT3 = np.arange(10, dtype=np.int64)[None].repeat(4, 0)
    GD3 = np.linspace(1, 10, 10, dtype=np.float32)[None].repeat(4, 0)
    I3 = np.full((4, 10), 999, np.int64)
    D3 = np.full((4, 10), 10.3, np.float32)
    D3[1], D3[2], D3[3] = 10.00005, 9.0, 10.9
    assert harness.calculate_recall_loose(I3, D3, GT3, GD3, 10) == np.float32(0.5)
    assert ref_lib.calculate_recall_loose(I3, D3, GT3, GD3, 10) == np.float32(0.5)
    I2 = np.full_like(I, -1)  # no results at all
    assert harness.calculate_recall(I2, np.abs(D), GT, GD, 10) == ref_lib.calculate_recall(I2, np.abs(D), GT, GD, 10)
    a = harness.calculate_r2(I2, np.abs(D), GT, GD, 10)
    b = ref_lib.calculate_r2(I2, np.abs(D), GT, GD, 10)
    assert np.isnan(a) and np.isnan(b)


def record(**kw):
    rec = harness.StatsRecord(nlist=1024, nprobe=32, opt_level=0, simi_ratio=0.8, total_count=123456789,
                              skip_triangle_count=1234, skip_triangle_large_count=0, skip_subnn_L2_count=77,
                              skip_subnn_IP_count=5, simi_update_count=4321, check_subnn_L2_ele_count=91,
                              check_subnn_IP_ele_count=13, check_subnn_L2_count=7, check_subnn_IP_count=3,
                              nb=1000000, nq=10000, d=128, k=100, mode="ORIGINAL", divideIVF=True,
                              disableOrderOptimize=False, blockSend=True, pruning=True, block=4, worker=8, group=2,
                              team=1, faiss_query_time=21.6, query_time=0.0123456789, original_time=0.5,
                              recall=0.9517, r2=0.00123, variance=0.25, trainTime=65.5, addTime=10.6,
                              preSearchTime=0.01, inBalanceRatio=1.2, inBalanceRatioTeam=1.1, brute_ratio=0.03)
    for key, val in kw.items():
        setattr(rec, key, val)
    return rec


@pytest.mark.parametrize("my", [False, True])
def test_stats_csv_matches_reference(ref_lib, tmp, my):
    recs = [record(), record(query_time=0.0, total_count=0, skip_triangle_count=0, skip_subnn_L2_count=0,
                             skip_subnn_IP_count=0, mode="DIVIDE_IVF", divideIVF=False), record(recall=1.0, r2=-0.5)]
    ours, theirs = os.path.join(tmp, "ours.csv"), os.path.join(tmp, "theirs.csv")
    for i, rec in enumerate(recs):
        # The first call starts the file (header), the later ones append; a
        # non-append call on an existing file starts it again.
        append = i > 0
        (rec.my_to_csv if my else rec.to_csv)(ours, append, "sift1m")
        ref_lib.stats_csv(theirs, append, "sift1m", rec, my=my)
    with open(ours, "rb") as a, open(theirs, "rb") as b:
        assert a.read() == b.read()
    record().to_csv(ours, False, "x") if not my else record().my_to_csv(ours, False, "x")
    ref_lib.stats_csv(theirs, False, "x", record(), my=my)
    with open(ours, "rb") as a, open(theirs, "rb") as b:
        assert a.read() == b.read()


def test_stats_record_from_search(tmp):
    """A record filled from one search call carries the index's shape and the
    call's Stats, and writes a row the reference's reader would parse."""
    from harmony_b200 import Stats

    class FakeIndex:
        def _info(self):
            return 128, 1024, 1_000_000, 0

    st = Stats(query_time=0.25, nprobe=32, k=10, nq=10_000)
    rec = harness.StatsRecord.from_search(FakeIndex(), st, recall=0.95, mode="ORIGINAL")
    assert (rec.d, rec.nlist, rec.nb, rec.nprobe, rec.k, rec.nq) == (128, 1024, 1_000_000, 32, 10, 10_000)
    p = os.path.join(tmp, "s.csv")
    rec.my_to_csv(p, True, "c5")
    rec.my_to_csv(p, True, "c5")
    lines = open(p).read().splitlines()
    assert len(lines) == 3 and lines[0].startswith("dataset,mode,nb,nq,d,nlist,nprobe,k,")
    row = dict(zip(lines[0].split(","), lines[1].split(",")))
    assert row["recall"] == "0.9500000000000000" and row["query_time"] == "0.2500000000000000"
    with pytest.raises(AttributeError):
        harness.StatsRecord.from_search(FakeIndex(), st, no_such_field=1)


@pytest.mark.parametrize("ext", ["txt", "bin"])
def test_result_files_match_reference(ref_lib, tmp, ext):
    rng = np.random.default_rng(9)
    I = rng.integers(-1, 1_000_000, (13, 7)).astype(np.int64)
    D = (rng.standard_normal((13, 7)) * 1000).astype(np.float32)
    D[0, -1] = np.finfo(np.float32).max  # padding slots as searches leave them
    ours = os.path.join(tmp, "sub", f"gt_7.{ext}")
    theirs = os.path.join(tmp, "ref", f"gt_7.{ext}")
    harness.write_results(I, D, ours)
    ref_lib.write_results(I, D, theirs)
    with open(ours, "rb") as a, open(theirs, "rb") as b:
        assert a.read() == b.read()
    for path in (ours, theirs):
        Ia, Da = harness.load_results(path, 13, 7)
        Ib, Db = ref_lib.load_results(path, 13, 7)
        assert np.array_equal(Ia, Ib) and np.array_equal(Da.view(np.uint32), Db.view(np.uint32))
        assert np.array_equal(Ia, I)
        if ext == "bin":
            assert np.array_equal(Da, D)


def test_golden_harness_fixtures(tmp):
    """The reference's outputs stored by tests/golden/make_golden_harness.py:
    the harness reproduces them without the reference library present."""
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_harness.npz"))
    p = os.path.join(tmp, "g.bvecs")
    g["bvecs_file"].tofile(p)
    assert np.array_equal(harness.load_bvecs(p, (1, 0), reference_offsets=True), g["bvecs_all"])
    assert np.array_equal(harness.load_bvecs(p, (3, 9), reference_offsets=True), g["bvecs_3_9"])
    for name, (k, gt_k) in {"k10": (10, 10), "k10_gt100": (10, 100)}.items():
        args = [g[f"recall_{name}_{s}"] for s in ("I", "D", "GT", "GD")]
        got = np.array([harness.calculate_recall(*args, k, gt_k), harness.calculate_recall_loose(*args, k, gt_k),
                        harness.calculate_r2(*args, k, gt_k)], np.float32)
        assert got.tobytes() == g[f"recall_{name}_values"].tobytes(), name
    rec = record(skip_triangle_large_count=0, check_subnn_IP_ele_count=0, check_subnn_IP_count=0,
                 disableOrderOptimize=False, blockSend=False)
    for name, my in (("csv_to", False), ("csv_my", True)):
        p = os.path.join(tmp, f"{name}.csv")
        (rec.my_to_csv if my else rec.to_csv)(p, False, "sift1m")
        (rec.my_to_csv if my else rec.to_csv)(p, True, "sift1m")
        assert open(p, "rb").read() == g[name].tobytes(), name
    p = os.path.join(tmp, "r.txt")
    harness.write_results(g["results_I"], g["results_D"], p)
    assert open(p, "rb").read() == g["results_txt"].tobytes()

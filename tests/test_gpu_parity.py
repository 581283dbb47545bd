"""GPU parity tests: the CUDA path (libharmony_b200.so through the C ABI)
against the reference's own Index (oracle/_ref), the restated oracle and the
committed golden vectors.  Bit-exact distances, ids equal except at exact
distance ties at the k-th position (tests/parity.py)."""
import os
import tempfile

import numpy as np
import pytest

import oracle
from harmony_b200 import Index, HarmonyError, SearchMode, datasets
from tests.parity import FLT_MAX, assert_topk_parity, recall_at_k

pytestmark = pytest.mark.gpu


def gpu_index_from_file(path, nprobe):
    ix = Index()
    ix.load_index(path)
    ix.nprobe = nprobe
    ix.preSearch(0, 0, 0, 0, 0, Index.Param(mode=SearchMode.ORIGINAL), "")
    return ix


def search(ix, q, k, param=None, workers=0, blocks=0, wl=0, wls=0):
    q = np.ascontiguousarray(q, np.float32)
    ix.preSearch(0, workers, blocks, wl, wls, param or Index.Param(mode=SearchMode.ORIGINAL), "")
    D = np.empty((q.shape[0], k), np.float32)
    I = np.empty((q.shape[0], k), np.int64)
    ix.search(q.shape[0], q, k, D, I)
    return D, I


def dist_checker(restated, base, q):
    return lambda qi, i: restated.l2(q[qi], base[i])


# -- golden vectors ------------------------------------------------------------

def test_golden_float_index_file(golden):
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "g.index")
        golden["f32_index_file"].tofile(p)
        ix = gpu_index_from_file(p, 6)
        assert ix.d == 20 and ix.nlist == 16
        D, I = search(ix, golden["f32_queries"], 7)
    assert_topk_parity(D, I, golden["f32_D"], golden["f32_I"], label="golden f32")


def test_golden_int_train_add_search(golden, restated):
    base = golden["int_base"].astype(np.float32)
    q = golden["int_queries"].astype(np.float32)
    ix = Index(32, 24, 4)
    ix.train(base.shape[0], base)
    # Integer data: FP64 centroid sums are exact, so the centroids equal the
    # reference's bit for bit.
    assert np.array_equal(ix.centroid_codes.view(np.uint32), golden["int_centroids"].view(np.uint32))
    ix.add(base.shape[0], base)
    assert np.array_equal(np.concatenate([[0], np.cumsum(ix.list_sizes())]), golden["int_list_off"])
    chk = dist_checker(restated, base, q)
    D, I = search(ix, q, 10)
    assert_topk_parity(D, I, golden["int_D4"], golden["int_I4"], chk, "nprobe 4")
    probes, _ = ix.probe_lists(q, 4)
    assert np.array_equal(probes, golden["int_probes4"])
    tops = ix.warmup_tops(q, 10, 3, 10)
    assert np.array_equal(tops, golden["int_tops"])
    D, I = search(ix, q, 10, Index.Param(mode=SearchMode.DIVIDE_IVF, pruning=True), wl=3, wls=10)
    assert_topk_parity(D, I, golden["int_Dp"], golden["int_Ip"], chk, "pruned")
    ix.nprobe = 24
    D, I = search(ix, q, 100)
    assert_topk_parity(D, I, golden["int_D24"], golden["int_I24"], chk, "exhaustive")


# -- config 1 against the reference ------------------------------------------

@pytest.fixture(scope="module")
def c1(ref_lib):
    base, q = datasets.config1()
    ref = ref_lib(128, 100, 10)
    ref.train(base)
    ref.add(base)
    td = tempfile.mkdtemp()
    path = os.path.join(td, "c1.index")
    ref.save(path)
    return base, q, ref, path


def test_config1_frozen_index_original(c1, restated):
    base, q, ref, path = c1
    ix = gpu_index_from_file(path, 10)
    D, I = search(ix, q, 10)
    Dr, Ir = ref.search(q, 10)
    assert_topk_parity(D, I, Dr, Ir, dist_checker(restated, base, q), "config1")
    gD, gI = restated.bruteforce_f64(q, base, 10)
    assert recall_at_k(I, gI, 10) > 0.9


def test_config1_frozen_index_pruned(c1, restated):
    base, q, ref, path = c1
    ix = gpu_index_from_file(path, 10)
    D, I = search(ix, q, 10, Index.Param(mode=SearchMode.DIVIDE_IVF, pruning=True), wl=10, wls=10)
    Dr, Ir = ref.search_pruned(q, 10, 10, 10, cut=True)
    assert_topk_parity(D, I, Dr, Ir, dist_checker(restated, base, q), "config1 pruned")
    assert np.array_equal(ix.warmup_tops(q, 10, 10, 10), ref.warmup_tops(q, 10, 10, 10))


def test_config1_gpu_build_matches_oracle(c1, restated):
    base, q, ref, path = c1
    ix = Index(128, 100, 10)
    ix.train(base.shape[0], base)
    cent = restated.kmeans(base, 100)
    assert np.array_equal(ix.centroid_codes.view(np.uint32), cent.view(np.uint32))
    ix.add(base.shape[0], base)
    mine = restated.add(base, cent)
    assert np.array_equal(np.concatenate([[0], np.cumsum(ix.list_sizes())]), mine.list_off)
    D, I = search(ix, q, 10)
    Dr, Ir = restated.search(mine, q, 10, 10)
    assert_topk_parity(D, I, Dr, Ir, dist_checker(restated, base, q), "gpu build")


def test_save_load_roundtrip_with_reference(c1, ref_lib):
    base, q, ref, path = c1
    ix = gpu_index_from_file(path, 10)
    with tempfile.TemporaryDirectory() as td:
        p2 = os.path.join(td, "again.index")
        ix.save_index(p2)
        assert open(p2, "rb").read() == open(path, "rb").read()
        back = ref_lib.load(p2)
        back.nprobe = 10
        Dr, Ir = back.search(q, 10)
    D, I = search(ix, q, 10)
    assert np.array_equal(D, Dr)


# -- float data, larger k, several nprobe --------------------------------------

@pytest.fixture(scope="module")
def c2small(ref_lib):
    base, q = datasets.config2(nb=120_000, nq=300, ncomp=300)
    ix = Index(128, 256, 8)
    ix.train(base.shape[0], base)
    ix.add(base.shape[0], base)
    td = tempfile.mkdtemp()
    path = os.path.join(td, "c2.index")
    ix.save_index(path)
    ref = ref_lib.load(path)
    return base, q, ix, ref


@pytest.mark.parametrize("nprobe,k", [(8, 100), (32, 100), (128, 10), (256, 1)])
def test_config2_shape_against_reference(c2small, restated, nprobe, k):
    base, q, ix, ref = c2small
    ix.nprobe = nprobe
    ref.nprobe = nprobe
    D, I = search(ix, q, k)
    Dr, Ir = ref.search(q, k)
    assert_topk_parity(D, I, Dr, Ir, dist_checker(restated, base, q), f"c2 P={nprobe} k={k}")


def test_config2_pruned_and_dimblock(c2small, restated):
    base, q, ix, ref = c2small
    ix.nprobe = ref.nprobe = 16
    D, I = search(ix, q, 100, Index.Param(mode=SearchMode.DIVIDE_IVF, pruning=True), wl=10, wls=100)
    Dr, Ir = ref.search_pruned(q, 100, 10, 100, cut=True)
    assert_topk_parity(D, I, Dr, Ir, label="c2 pruned")
    data = ref.index_data()
    probes = ref.probe_lists(q)
    tops = restated.warmup_tops(data, q, probes, 100, 10, 100)
    for W, B, opt, cut in ((4, 4, True, True), (4, 3, False, True), (8, 5, True, False), (2, 1, True, True)):
        prm = Index.Param(mode=SearchMode.DIVIDE_DIM, pruning=cut, orderOptimize=opt)
        D, I = search(ix, q, 100, prm, workers=W, blocks=B, wl=10, wls=100)
        order = restated.block_order(W, B, opt)
        Do, Io = restated.search_dimblock(data, q, probes, tops, 100, W, B, order, cut=cut)
        assert_topk_parity(D, I, Do, Io, label=f"dimblock W={W} B={B}")


def test_config2_dimblock_full_warmup(c2small, restated):
    """Param::fullWarmUp: DIVIDE_DIM prunes against the caller's heap tops --
    the query driver fills them with each query's k-th ground-truth distance
    (src/query.cpp:716-725) -- and runs no warm-up search
    (src/Index.cpp:1235-1241)."""
    import torch
    base, q, ix, ref = c2small
    k = 100
    ix.nprobe = ref.nprobe = 16
    Dgt, _ = search(ix, q, k, Index.Param(mode=SearchMode.BRUTE_FORCE))
    tops = np.ascontiguousarray(Dgt[:, k - 1])
    data = ref.index_data()
    probes = ref.probe_lists(q)
    for W, B, opt in ((4, 4, True), (8, 3, False)):
        order = restated.block_order(W, B, opt)
        Do, Io = restated.search_dimblock(data, q, probes, tops, k, W, B, order, cut=True)
        for t in (tops, torch.from_numpy(tops).cuda()):
            prm = Index.Param(mode=SearchMode.DIVIDE_DIM, pruning=True, orderOptimize=opt, fullWarmUp=True,
                              heapTops=t)
            D, I = search(ix, q, k, prm, workers=W, blocks=B)
            assert_topk_parity(D, I, Do, Io, label=f"full warm-up W={W} B={B}")
    with pytest.raises(HarmonyError, match="heapTop"):
        search(ix, q, k, Index.Param(mode=SearchMode.DIVIDE_DIM, pruning=True, fullWarmUp=True), workers=4, blocks=4)


def test_single_query_batches_split_lists(c2small):
    """A one-query batch splits every list into many chunks (many slots)."""
    base, q, ix, ref = c2small
    ix.nprobe = ref.nprobe = 64
    for i in range(3):
        D, I = search(ix, q[i:i + 1], 50)
        Dr, Ir = ref.search(q[i:i + 1], 50)
        assert_topk_parity(D, I, Dr, Ir, label=f"single {i}")


def test_config3_shape_d500(ref_lib, restated):
    base, q = datasets.config3(nb=20_000, nq=60, ncomp=100)
    ix = Index(500, 64, 8)
    ix.train(base.shape[0], base)
    ix.add(base.shape[0], base)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "c3.index")
        ix.save_index(p)
        ref = ref_lib.load(p)
    ref.nprobe = 8
    D, I = search(ix, q, 100)
    Dr, Ir = ref.search(q, 100)
    assert_topk_parity(D, I, Dr, Ir, dist_checker(restated, base, q), "d500")


# -- edge cases ------------------------------------------------------------------

@pytest.mark.parametrize("d", [3, 4, 20, 33])
def test_odd_dimensions(d, restated):
    rng = np.random.default_rng(d)
    base = rng.standard_normal((700, d), dtype=np.float32)
    q = rng.standard_normal((25, d), dtype=np.float32)
    ix = Index(d, 8, 3)
    ix.train(base.shape[0], base)
    ix.add(base.shape[0], base)
    cent = ix.centroid_codes
    data = restated.add(base, cent)
    D, I = search(ix, q, 9)
    Dr, Ir = restated.search(data, q, 9, 3)
    assert_topk_parity(D, I, Dr, Ir, dist_checker(restated, base, q), f"d={d}")


def test_k_larger_than_candidates_and_nprobe_clamp(restated):
    rng = np.random.default_rng(5)
    base = rng.standard_normal((40, 8), dtype=np.float32)
    q = rng.standard_normal((5, 8), dtype=np.float32)
    ix = Index(8, 4, 2)
    ix.train(40, base)
    ix.add(40, base)
    D, I = search(ix, q, 64)
    data = restated.add(base, ix.centroid_codes)
    Dr, Ir = restated.search(data, q, 64, 2)
    assert_topk_parity(D, I, Dr, Ir, label="k>n")
    assert (I[:, -1] == -1).all() and (D[:, -1] == FLT_MAX).all()
    ix.nprobe = 100  # clamped to nlist by search, as src/Index.cpp:1646-1648
    search(ix, q, 5)
    assert ix.nprobe == 4


def test_nprobe_zero_and_empty_queries():
    rng = np.random.default_rng(6)
    base = rng.standard_normal((100, 8), dtype=np.float32)
    ix = Index(8, 4, 0)
    ix.train(100, base)
    ix.add(100, base)
    D, I = search(ix, base[:3], 4)
    assert (I == -1).all() and (D == FLT_MAX).all()
    ix.preSearch(0, 0, 0, 0, 0, Index.Param())
    ix.search(0, np.zeros((0, 8), np.float32), 4, np.zeros((0, 4), np.float32), np.zeros((0, 4), np.int64))


def test_search_without_presearch_only_initialises():
    rng = np.random.default_rng(7)
    base = rng.standard_normal((100, 8), dtype=np.float32)
    ix = Index(8, 4, 2)
    ix.train(100, base)
    ix.add(100, base)
    D = np.zeros((2, 3), np.float32)
    I = np.zeros((2, 3), np.int64)
    ix.search(2, base[:2], 3, D, I)
    assert (I == -1).all() and (D == FLT_MAX).all()


def test_brute_force_mode_equals_exhaustive(c2small):
    base, q, ix, ref = c2small
    D, I = search(ix, q[:50], 10, Index.Param(mode=SearchMode.BRUTE_FORCE))
    ref.nprobe = 256
    Dr, Ir = ref.search(q[:50], 10)
    assert_topk_parity(D, I, Dr, Ir, label="brute")


def test_device_pointers_in_and_out(c2small):
    import torch
    base, q, ix, ref = c2small
    ix.nprobe = ref.nprobe = 16
    qt = torch.from_numpy(q[:64]).cuda()
    Dt = torch.empty((64, 10), dtype=torch.float32, device="cuda")
    It = torch.empty((64, 10), dtype=torch.int64, device="cuda")
    ix.preSearch(0, 0, 0, 0, 0, Index.Param())
    ix.search(64, qt, 10, Dt, It)
    Dr, Ir = ref.search(q[:64], 10)
    assert_topk_parity(Dt.cpu().numpy(), It.cpu().numpy(), Dr, Ir, label="device ptrs")


def test_errors_are_reported():
    with pytest.raises(HarmonyError):
        Index(8, 4, 2, metric=0)  # METRIC_IP is not implemented
    ix = Index(8, 4, 2)
    with pytest.raises(HarmonyError):
        ix.train(2, np.zeros((2, 8), np.float32))  # fewer points than nlist
    with pytest.raises(HarmonyError):
        ix.load_index("/nonexistent/file.index")
    ix2 = Index(10, 4, 2)
    rng = np.random.default_rng(8)
    b = rng.standard_normal((50, 10), dtype=np.float32)
    ix2.train(50, b)
    ix2.add(50, b)
    with pytest.raises(HarmonyError):  # d % workers != 0 (src/Index.cpp:125)
        search(ix2, b[:4], 3, Index.Param(mode=SearchMode.DIVIDE_DIM), workers=3, blocks=1)

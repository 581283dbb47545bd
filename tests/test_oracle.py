"""CPU tests: pin the restated oracle (oracle/ivf_oracle.cpp) to the reference.

The reference's own harmony::Index (oracle/_ref, built from its unmodified
sources) and the committed golden vectors (tests/golden/make_golden.py) are
the two pins.  No GPU is used here.
"""
import os
import tempfile

import numpy as np
import pytest

import oracle
from harmony_b200 import datasets
from tests.parity import assert_topk_parity


def _golden_int_index(g):
    return oracle.IndexData(g["int_centroids"], g["int_list_off"], g["int_ids"],
                            g["int_base"].astype(np.float32)[g["int_ids"]], g["int_norms"])


# -- golden vectors (no reference needed) ------------------------------------

def test_heap_golden(restated, golden):
    D, I = restated.heap_topk(golden["heap_vals"], 20)
    assert np.array_equal(D, golden["heap_D"]) and np.array_equal(I, golden["heap_I"])
    # HeapTest's own assertions (src/tests/heap_test.cpp:39-47).
    v = golden["heap_vals"]
    assert np.array_equal(v[I], D)
    assert np.array_equal(np.sort(v)[:20], D)


def test_l2_sequential_unfused(restated):
    rng = np.random.default_rng(0)
    a = rng.standard_normal(128, dtype=np.float32)
    b = rng.standard_normal(128, dtype=np.float32)
    acc = np.float32(0)
    for x, y in zip(a, b):
        t = np.float32(x - y)
        acc = np.float32(acc + np.float32(t * t))
    assert restated.l2(a, b) == acc


def test_kmeans_add_golden(restated, golden):
    base = golden["int_base"].astype(np.float32)
    cent = restated.kmeans(base, 24)
    assert np.array_equal(cent.view(np.uint32), golden["int_centroids"].view(np.uint32))
    ix = restated.add(base, cent)
    assert np.array_equal(ix.list_off, golden["int_list_off"])
    assert np.array_equal(ix.norms[np.argsort(ix.ids)], golden["int_norms"][np.argsort(golden["int_ids"])])
    # In-list order: ascending centroid distance; ties are unordered in the
    # reference (std::sort), so compare each list as a set.
    for l in range(24):
        a, b = ix.list_off[l], ix.list_off[l + 1]
        assert set(ix.ids[a:b].tolist()) == set(golden["int_ids"][a:b].tolist())


def test_search_golden(restated, golden):
    ix = _golden_int_index(golden)
    q = golden["int_queries"].astype(np.float32)
    D, I = restated.search(ix, q, 10, 4)
    assert_topk_parity(D, I, golden["int_D4"], golden["int_I4"], label="nprobe4")
    D, I = restated.search(ix, q, 100, 24)
    assert_topk_parity(D, I, golden["int_D24"], golden["int_I24"], label="exhaustive")
    cd, cl = restated.coarse(q, ix.centroids, 4)
    assert np.array_equal(cl, golden["int_probes4"])


def test_pruned_golden(restated, golden):
    ix = _golden_int_index(golden)
    q = golden["int_queries"].astype(np.float32)
    probes = golden["int_probes4"]
    tops = restated.warmup_tops(ix, q, probes, 10, 3, 10)
    assert np.array_equal(tops, golden["int_tops"])
    D, I = restated.search_pruned(ix, q, probes, tops, 10, cut=True)
    assert_topk_parity(D, I, golden["int_Dp"], golden["int_Ip"], label="pruned")


def test_exhaustive_equals_bruteforce(restated, golden):
    """IndexTest (src/tests/index_test.cpp:71-122): nprobe = nlist gives recall 1."""
    base = golden["int_base"].astype(np.float32)
    q = golden["int_queries"].astype(np.float32)
    gD, gI = restated.bruteforce_f64(q, base, 10)
    D = golden["int_D24"][:, :10]
    # Integer data: every FP32 distance is exact, so it equals the FP64 one.
    assert np.array_equal(D.astype(np.float64), gD)


# -- against the reference library --------------------------------------------

def test_l2_matches_reference(restated, ref_lib):
    rng = np.random.default_rng(1)
    for _ in range(200):
        a = rng.standard_normal(128, dtype=np.float32)
        b = rng.standard_normal(128, dtype=np.float32)
        assert restated.l2(a, b) == ref_lib.l2(a, b)


def test_heap_matches_reference(restated, ref_lib):
    rng = np.random.default_rng(2)
    for k in (1, 7, 20, 64):
        v = rng.random(300, dtype=np.float32)
        v[::7] = v[3]  # ties
        D, I = restated.heap_topk(v, k)
        Dr, Ir = ref_lib.heap_topk(v, k)
        assert np.array_equal(D, Dr) and np.array_equal(I, Ir)


@pytest.fixture(scope="module")
def c1_ref(ref_lib):
    base, q = datasets.config1()
    ix = ref_lib(128, 100, 10)
    ix.train(base)
    ix.add(base)
    return base, q, ix


def test_config1_search_matches_reference(restated, c1_ref):
    base, q, ix = c1_ref
    data = ix.index_data()
    Dr, Ir = ix.search(q, 10)
    D, I = restated.search(data, q, 10, 10)
    assert_topk_parity(D, I, Dr, Ir, label="config1")
    gD, gI = restated.bruteforce_f64(q, base, 10)
    rec = np.mean([len(set(a) & set(b)) / 10 for a, b in zip(Ir, gI)])
    assert rec > 0.9


def test_config1_kmeans_add_match_reference(restated, c1_ref):
    base, q, ix = c1_ref
    data = ix.index_data()
    cent = restated.kmeans(base, 100)
    assert np.array_equal(cent.view(np.uint32), data.centroids.view(np.uint32))
    mine = restated.add(base, cent)
    assert np.array_equal(mine.list_off, data.list_off)
    assert np.array_equal(mine.codes, base[mine.ids])


def test_config1_pruned_matches_reference(restated, c1_ref):
    base, q, ix = c1_ref
    data = ix.index_data()
    probes = ix.probe_lists(q)
    cd, cl = restated.coarse(q, data.centroids, 10)
    assert np.array_equal(cl, probes)
    for wl, wls in ((10, 10), (2, 5), (10, 0)):
        tops_r = ix.warmup_tops(q, 10, wl, wls)
        tops = restated.warmup_tops(data, q, probes, 10, wl, wls)
        assert np.array_equal(tops, tops_r)
    Dr, Ir = ix.search_pruned(q, 10, 10, 10, cut=True)
    tops = restated.warmup_tops(data, q, probes, 10, 10, 10)
    D, I = restated.search_pruned(data, q, probes, tops, 10, cut=True)
    assert_topk_parity(D, I, Dr, Ir, label="pruned")
    Dr, Ir = ix.search_pruned(q, 10, 10, 10, cut=False)
    D, I = restated.search_pruned(data, q, probes, tops, 10, cut=False)
    assert_topk_parity(D, I, Dr, Ir, label="unpruned worker")


def test_float_index_file_roundtrip(restated, ref_lib, golden):
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "g.index")
        golden["f32_index_file"].tofile(p)
        ix = ref_lib.load(p)
        ix.nprobe = 6
        D, I = ix.search(golden["f32_queries"], 7)
        assert np.array_equal(D, golden["f32_D"]) and np.array_equal(I, golden["f32_I"])
        data = ix.index_data()
        D2, I2 = restated.search(data, golden["f32_queries"], 7, 6)
        assert_topk_parity(D2, I2, D, I, label="f32")


def test_block_order_matches_reference(restated, ref_lib):
    for W, B in ((4, 4), (4, 8), (3, 7), (2, 5), (8, 3)):
        for opt in (True, False):
            assert np.array_equal(restated.block_order(W, B, opt), ref_lib.block_order(W, B, opt))


def test_block_order_period(restated):
    # Index.cpp:183-197: with period, block order of B % W == 0 layouts.
    o = restated.block_order(2, 4, True, period=True)
    assert sorted(o[0].tolist()) == [0, 1]
    assert (o >= 0).all()


def test_dimblock_no_cut_is_slice_fold(restated, golden):
    """Without pruning the relay sum is the fold of the slices in visit order."""
    ix = _golden_int_index(golden)
    q = golden["int_queries"].astype(np.float32)
    probes = golden["int_probes4"]
    order = restated.block_order(4, 4, True)
    tops = np.full(q.shape[0], np.finfo(np.float32).max, np.float32)
    D, I = restated.search_dimblock(ix, q, probes, tops, 10, 4, 4, order, cut=False)
    # Integer data: all partial sums are exact, so any fold order gives the
    # ORIGINAL distances.
    assert_topk_parity(D, I, golden["int_D4"], golden["int_I4"], label="dimblock")

"""Generate the golden fixtures of the IVF-flat path from the reference itself.

Runs the reference's own harmony::Index (oracle/_ref/libharmony_ref.so, built
from the unmodified reference sources by oracle/Makefile) on small seeded
inputs and stores inputs and outputs in ``golden_ivf.npz``:

  small_int   1500 x 32 integer-valued vectors (config-1 value range),
              nlist 24, 40 queries: centroids and lists after train + add,
              ORIGINAL search ids / distances at nprobe 4 (k 10) and nprobe 24
              (k 100, exhaustive), the probe table, warm-up heap tops and the
              pruned base-worker search (src/node.cpp:606-678).
  small_f32   1200 x 20 Gaussian float vectors loaded from a reference-written
              index file (the file bytes are stored), 30 queries, nprobe 6,
              k 7: ORIGINAL search.
  heap        100 values -> heap top-20 (src/heap.hpp), as HeapTest does
              (src/tests/heap_test.cpp:7-48) but seeded.

Usage:  python tests/golden/make_golden.py   (needs the reference sources)
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from harmony_b200 import datasets  # noqa: E402


def main():
    oracle.build(reference=True)
    R = oracle.RefIndex
    R.set_threads(1)
    out = {}

    # --- small integer-valued set ------------------------------------------
    base, qs = datasets.config1(seed=11, nb=1500, nq=40, d=32, ncomp=12)
    ix = R(32, 24, 4)
    ix.train(base)
    ix.add(base)
    data = ix.index_data()
    D4, I4 = ix.search(qs, 10)
    ix.nprobe = 24
    D24, I24 = ix.search(qs, 100)
    ix.nprobe = 4
    probes = ix.probe_lists(qs)
    tops = ix.warmup_tops(qs, 10, warm_lists=3, warm_list_size=10)
    Dp, Ip = ix.search_pruned(qs, 10, warm_lists=3, warm_list_size=10, cut=True)
    out.update({
        "int_base": base.astype(np.uint8), "int_queries": qs.astype(np.uint8),
        "int_centroids": data.centroids, "int_list_off": data.list_off, "int_ids": data.ids,
        "int_norms": data.norms,
        "int_D4": D4, "int_I4": I4, "int_D24": D24, "int_I24": I24, "int_probes4": probes,
        "int_tops": tops, "int_Dp": Dp, "int_Ip": Ip,
    })

    # --- float set through a reference-written index file -----------------
    rng = np.random.default_rng(12)
    fbase = rng.standard_normal((1200, 20), dtype=np.float32)
    fq = rng.standard_normal((30, 20), dtype=np.float32)
    fx = R(20, 16, 6)
    fx.train(fbase)
    fx.add(fbase)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "f.index")
        fx.save(p)
        blob = np.fromfile(p, dtype=np.uint8)
        lx = R.load(p)
        lx.nprobe = 6
        Df, If = lx.search(fq, 7)
    out.update({"f32_queries": fq, "f32_index_file": blob, "f32_D": Df, "f32_I": If})

    # --- heap ---------------------------------------------------------------
    vals = np.random.default_rng(13).random(100, dtype=np.float32)
    hD, hI = R.heap_topk(vals, 20)
    out.update({"heap_vals": vals, "heap_D": hD, "heap_I": hI})

    path = os.path.join(HERE, "golden_ivf.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({os.path.getsize(path)} bytes)")


if __name__ == "__main__":
    main()

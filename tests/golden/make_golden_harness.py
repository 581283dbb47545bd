"""Generate the golden fixtures of the query-driver harness from the reference itself.

Runs the reference's own helpers (src/utils.h loaders, recall measures and
result files; src/stats.h CSV rows), exported by oracle/_ref/libharmony_ref.so,
on small seeded inputs and stores inputs and outputs in ``golden_harness.npz``:

  bvecs        a 12 x 20 bvecs file (its bytes) and the rows the reference's
               loadBvecs returns for bounds (1, 0) and (3, 9);
  recall_*     result / ground-truth tables (k 10, gt_k 10 and 100) and the
               reference's calculate_recall, calculate_recall_loose and
               calculate_r2 on them;
  csv_*        the bytes of Stats::toCsv and Stats::myToCsv for one record
               (header + two appended rows);
  results_txt  the bytes of writeResultsToFile for a 5 x 4 table (text form).

Usage:  python tests/golden/make_golden_harness.py   (needs the reference sources)
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from harmony_b200 import harness  # noqa: E402  (StatsRecord: the field set)


def tables(rng, nq, k, gt_k):
    GT = np.stack([rng.permutation(500)[:gt_k] for _ in range(nq)]).astype(np.int64)
    GD = np.sort(rng.uniform(1, 40, (nq, gt_k)).astype(np.float32), axis=1)
    I = np.where(rng.random((nq, k)) < 0.7, GT[:, :k][:, rng.permutation(k)], rng.integers(500, 900, (nq, k)))
    D = np.abs(np.sort((GD[:, :k] + rng.normal(0, 0.4, (nq, k))).astype(np.float32), axis=1))
    D[:, -1] = GD[:, k - 1]
    D[::3, -2] = GD[::3, k - 1] + np.float32(5e-5)
    I[::4, k // 2:] = -1
    return I.astype(np.int64), D, GT, GD


def main():
    if not oracle.RefIndex.available():
        oracle.build(reference=True)
    R = oracle.RefIndex
    rng = np.random.default_rng(2024)
    out = {}
    with tempfile.TemporaryDirectory() as td:
        x = rng.integers(0, 256, (12, 20), dtype=np.uint8)
        rec = np.empty((12, 24), np.uint8)
        rec[:, :4] = np.frombuffer(np.int32(20).tobytes(), np.uint8)
        rec[:, 4:] = x
        p = os.path.join(td, "g.bvecs")
        rec.tofile(p)
        out["bvecs_file"] = np.frombuffer(open(p, "rb").read(), np.uint8)
        out["bvecs_all"] = R.load_bvecs(p, (1, 0))
        out["bvecs_3_9"] = R.load_bvecs(p, (3, 9))
        for name, (k, gt_k) in {"k10": (10, 10), "k10_gt100": (10, 100)}.items():
            I, D, GT, GD = tables(rng, 60, k, gt_k)
            out[f"recall_{name}_I"], out[f"recall_{name}_D"] = I, D
            out[f"recall_{name}_GT"], out[f"recall_{name}_GD"] = GT, GD
            out[f"recall_{name}_values"] = np.array(
                [R.calculate_recall(I, D, GT, GD, k, gt_k), R.calculate_recall_loose(I, D, GT, GD, k, gt_k),
                 R.calculate_r2(I, D, GT, GD, k, gt_k)], np.float32)
        stats = harness.StatsRecord(nlist=1024, nprobe=32, opt_level=0, simi_ratio=0.8, total_count=123456789,
                                    skip_triangle_count=1234, skip_subnn_L2_count=77, skip_subnn_IP_count=5,
                                    simi_update_count=4321, check_subnn_L2_ele_count=91, check_subnn_L2_count=7,
                                    nb=1000000, nq=10000, d=128, k=100, mode="ORIGINAL", divideIVF=True,
                                    pruning=True, block=4, worker=8, group=2, team=1, faiss_query_time=21.6,
                                    query_time=0.0123456789, original_time=0.5, recall=0.9517, r2=0.00123,
                                    variance=0.25, trainTime=65.5, addTime=10.6, preSearchTime=0.01,
                                    inBalanceRatio=1.2, inBalanceRatioTeam=1.1, brute_ratio=0.03)
        for name, my in (("csv_to", False), ("csv_my", True)):
            p = os.path.join(td, f"{name}.csv")
            R.stats_csv(p, False, "sift1m", stats, my=my)
            R.stats_csv(p, True, "sift1m", stats, my=my)
            out[name] = np.frombuffer(open(p, "rb").read(), np.uint8)
        I = rng.integers(-1, 10_000, (5, 4)).astype(np.int64)
        D = (rng.standard_normal((5, 4)) * 100).astype(np.float32)
        p = os.path.join(td, "r.txt")
        R.write_results(I, D, p)
        out["results_I"], out["results_D"] = I, D
        out["results_txt"] = np.frombuffer(open(p, "rb").read(), np.uint8)
    np.savez_compressed(os.path.join(HERE, "golden_harness.npz"), **out)
    print("wrote", os.path.join(HERE, "golden_harness.npz"), sorted(out))


if __name__ == "__main__":
    main()

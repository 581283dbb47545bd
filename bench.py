#!/usr/bin/env python
"""Benchmark of the IVF-flat search path on B200.

Metric: queries per second of the whole search (coarse quantizer + list scan
+ top-k merge) at the smallest fixed nprobe whose recall@10 against the FP64
ground truth reaches the target (0.95), on the 10M x 128 / nlist 4096 / k 10
workload (synthetic: seeded 4096-component Gaussian mixture drawn on the GPU).

One step = one search of the 10,000 test queries.  ``value`` is measured with
the queries and results resident in HBM (CUDA events on the index's stream,
max over ranks); ``e2e`` is the same search through the public API with the
queries in pinned host memory and the results copied back, copies inside the
timed region.  The index (5.1 GB of codes) is larger than the 126 MB L2, and
every step touches every list, so no L2 flush is needed between steps.

  python bench.py [--steps K] [--warmup W] [--gpus N]        (our CUDA path)
  python bench.py --impl reference                           (the reference's
        own CPU search, oracle/_ref, on the same frozen index and queries)
  python bench.py --workload c4     (10M x 96, Zipf list sizes, batches of 1..4096)
  python bench.py --workload c3     (270k x 500, k 100: the candidate-matrix BF16 path)
  python bench.py --workload c2     (1M x 128, nlist 1024, k 100: the nprobe 8..128 sweep)
  python bench.py --workload c5-batches  (learned vs fixed nprobe by batch size, 10M x 128)

Multi-GPU: the path is query-parallel with no exchange step, so N ranks run
N independent replicas (weak scaling, each rank its own 10k queries).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = {
    "workload": "ivf-flat 10M x 128 (config5: 4096-component mixture), nlist 4096, k 10, 10k queries",
    "nb": 10_000_000, "d": 128, "nlist": 4096, "k": 10, "nq": 10_000,
}
# DRAM bytes (read + write) of one scan_bf16 launch over its algorithmic bytes, from the
# ncu capture of a 3M x 128 / nlist 1229 / nprobe 40 launch: 866.8 MB for 764.6 MB
# (profiles/scan_bf16_3m_ncu_full.md).  The traffic grows with the lists read, so the
# bench scales it by each launch's algorithmic bytes.
SCAN_TRAFFIC_RATIO = 1.134
NPROBE_SWEEP = [1, 2, 3, 4, 5, 6, 8, 10, 12, 14, 16, 20, 24, 28, 32, 40, 48, 56, 64, 80, 96, 128, 160, 192, 256]


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), float(p["bf16_tflops"]), "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.out = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()

    def summary(self):
        self.out.flush()
        rows = []
        try:
            with open(self.out.name) as f:
                for line in f:
                    parts = [x.strip() for x in line.split(",")]
                    if len(parts) >= 9:
                        rows.append(parts)
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def build_index(torch, seed=5, nb=None, nq=None, ntrain=0):
    from harmony_b200 import Index, datasets
    nb = nb or WORKLOAD["nb"]
    nq = nq or WORKLOAD["nq"]
    base, test, train = datasets.config5_device(seed=seed, nb=nb, nq=nq, ntrain=ntrain)
    ix = Index(WORKLOAD["d"], WORKLOAD["nlist"], 16)
    t0 = time.perf_counter()
    ix.train(base.shape[0], base)
    t1 = time.perf_counter()
    ix.add(base.shape[0], base)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    info = {"train_s": round(t1 - t0, 2), "add_s": round(t2 - t1, 2)}
    if ntrain:
        return ix, base, test, train, info
    return ix, base, test, info


def ground_truth(torch, ix, base, test, k):
    """FP32 exhaustive top-32 on the GPU, re-ranked in FP64 on the host."""
    from harmony_b200 import Index, SearchMode
    nq = test.shape[0]
    ix.preSearch(0, 0, 0, 0, 0, Index.Param(mode=SearchMode.BRUTE_FORCE), "")
    G = torch.empty((nq, 32), dtype=torch.float32, device="cuda")
    GI = torch.empty((nq, 32), dtype=torch.int64, device="cuda")
    ix.search(nq, test, 32, G, GI)
    gi = GI.cpu().numpy()
    cand = base[torch.from_numpy(gi.reshape(-1)).cuda()].double().reshape(nq, 32, -1)
    d64 = ((cand - test.double()[:, None, :]) ** 2).sum(-1).cpu().numpy()
    order = np.argsort(d64, axis=1, kind="stable")
    return np.take_along_axis(gi, order, 1)[:, :k]


def recall(I, gt, k):
    I = np.asarray(I)[:, :k]
    return float(np.mean([len(set(a.tolist()) & set(b.tolist())) / k for a, b in zip(I, gt)]))


def parity_count(D, I, Dr, Ir):
    """Queries whose top-k equals the other result's: distances identical bit
    for bit, and ids identical except among those at the k-th distance (an
    exact tie across the boundary, where the reference's heap history decides,
    src/IVFScan.hpp:267).  Returns (identical queries, queries)."""
    D, Dr = np.ascontiguousarray(D, np.float32), np.ascontiguousarray(Dr, np.float32)
    I, Ir = np.asarray(I), np.asarray(Ir)
    same_d = np.all(D.view(np.uint32) == Dr.view(np.uint32), axis=1)
    ok = 0
    for q in np.nonzero(same_d)[0]:
        if np.array_equal(I[q], Ir[q]):
            ok += 1
            continue
        below = Dr[q] < Dr[q, -1]
        ok += set(I[q][below].tolist()) == set(Ir[q][below].tolist())
    return int(ok), int(D.shape[0])


def max_rel_err_vs_fp64(torch, base, test, D, I):
    """Largest relative error of returned distances against FP64 recomputation."""
    Dt = torch.as_tensor(np.asarray(D)).cuda().double()
    It = torch.as_tensor(np.asarray(I)).cuda()
    valid = It >= 0
    x = base[It.clamp(min=0).reshape(-1)].double().reshape(It.shape[0], It.shape[1], -1)
    d64 = ((x - test.double()[:, None, :]) ** 2).sum(-1)
    err = ((Dt - d64).abs() / d64.clamp(min=1e-30))[valid]
    return float(err.max().item()) if err.numel() else 0.0


def pick_nprobe(ix, test, gt, k, target, precision):
    import torch
    nq = test.shape[0]
    D = torch.empty((nq, k), dtype=torch.float32, device="cuda")
    I = torch.empty((nq, k), dtype=torch.int64, device="cuda")
    ix.search_params.precision = precision
    rec = 0.0
    for p in NPROBE_SWEEP:
        ix.nprobe = p
        ix.search(nq, test, k, D, I)
        rec = recall(I.cpu().numpy(), gt, k)
        if rec >= target:
            return p, rec
    return NPROBE_SWEEP[-1], rec


def time_arm(torch, ix, test, k, P, precision, steps, warmup, world, dist, learned=False, target=0.0, tag="arm"):
    """Device-resident timing of `steps` searches (CUDA events on the index stream).
    The timed loop is an NVTX range `timed_<tag>` (for `ncu --nvtx-include`)."""
    nq = test.shape[0]
    ix.nprobe = P
    ix.search_params.precision = precision
    ix.search_params.learned_probe = learned
    ix.search_params.learned_target = target
    D = torch.empty((nq, k), dtype=torch.float32, device="cuda")
    I = torch.empty((nq, k), dtype=torch.int64, device="cuda")
    stream = torch.cuda.ExternalStream(ix.stream)
    for _ in range(warmup):
        ix.search(nq, test, k, D, I)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches0 = ix.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push(f"timed_{tag}")
    e0.record(stream)
    for _ in range(steps):
        ix.search(nq, test, k, D, I)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.nvtx.range_pop()
    ms = e0.elapsed_time(e1)
    launches = ix.launch_count() - launches0
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    # Per-kernel device time of the same step.
    ix.profile(True)
    for _ in range(steps):
        ix.search(nq, test, k, D, I)
    prof = ix.profile_read()
    ix.profile(False)
    return {"ms_per_step": ms / steps, "launches_per_step": launches / steps, "I": I, "D": D,
            "kernel_ms": {n: v[0] / steps for n, v in prof.items()}}


def run_ours(args):
    import torch
    import torch.distributed as dist
    from harmony_b200 import Index, Precision, SearchMode

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    k, nq, d = WORKLOAD["k"], WORKLOAD["nq"], WORKLOAD["d"]
    ntrain = args.ntrain
    ix, base, test, train, build = build_index(torch, seed=5, ntrain=ntrain)
    gt = ground_truth(torch, ix, base, test, k)
    ix.preSearch(0, 0, 0, 0, 0, Index.Param(mode=SearchMode.ORIGINAL), "")
    # Learned probe: labels from the exact search at nprobe 256 on the
    # training queries, calibrated to the recall target on a held-out 10%.
    t0 = time.perf_counter()
    ix.train_probe_predictor(train.shape[0], train, k=k, label_nprobe=256, target=args.target)
    torch.cuda.synchronize()
    build["probe_train_s"] = round(time.perf_counter() - t0, 2)
    build["probe_train_queries"] = int(train.shape[0])
    del train

    arms, outs = {}, {}
    with ClockSampler(local) as clk:
        for name, prec in (("fp32", Precision.FP32), ("bf16", Precision.BF16)):
            if args.fixed_nprobe:
                P = args.fixed_nprobe
            else:
                P, rec = pick_nprobe(ix, test, gt, k, args.target, prec)
            r = time_arm(torch, ix, test, k, P, prec, args.steps, args.warmup, world, dist, tag=name)
            outs[name] = (r.pop("D").cpu().numpy(), r.pop("I").cpu().numpy())
            r.update({"nprobe": P, "recall_at_10": recall(outs[name][1], gt, k),
                      "qps": world * nq / (r["ms_per_step"] / 1e3)})
            if prec == Precision.BF16:
                r["bounded_scan"] = ix.bf16_stats()
            arms[name] = r
        # Learned nprobe + BF16: raise the predictor's target until the test
        # recall against the FP64 ground truth reaches the bench target.
        Dl = torch.empty((nq, k), dtype=torch.float32, device="cuda")
        Il = torch.empty((nq, k), dtype=torch.int64, device="cuda")
        ix.search_params.precision, ix.search_params.learned_probe = Precision.BF16, True
        tgt = args.target
        for tgt in [args.target + 0.005 * i for i in range(10)]:
            ix.search_params.learned_target = min(tgt, 0.9999)
            ix.search(nq, test, k, Dl, Il)
            if recall(Il.cpu().numpy(), gt, k) >= args.target:
                break
        tgt = min(tgt, 0.9999)
        r = time_arm(torch, ix, test, k, 256, Precision.BF16, args.steps, args.warmup, world, dist, learned=True,
                     target=tgt, tag="learned_bf16")
        r["bounded_scan"] = ix.bf16_stats()
        outs["learned_bf16"] = (r.pop("D").cpu().numpy(), r.pop("I").cpu().numpy())
        r.update({"nprobe": "learned", "predictor_target": round(tgt, 4),
                  "recall_at_10": recall(outs["learned_bf16"][1], gt, k),
                  "qps": world * nq / (r["ms_per_step"] / 1e3)})
        thr, crec, cavg = ix.probe_calibration()
        i_sel = int(np.argmin(np.where(crec >= tgt, cavg, 1e9)))
        r["avg_nprobe_validation"] = round(float(cavg[i_sel]), 2)
        arms["learned_bf16"] = r
        head = arms["learned_bf16"] if arms["learned_bf16"]["recall_at_10"] >= args.target else arms["bf16"]
        # Keep the GPU busy with the headline step for ~1 s so the clock
        # samples describe the timed load.
        t_end = time.perf_counter() + 1.0
        ix.search_params.precision = Precision.BF16
        ix.search_params.learned_probe = head is arms["learned_bf16"]
        ix.search_params.learned_target = tgt if head is arms["learned_bf16"] else 0.0
        ix.nprobe = 256 if head is arms["learned_bf16"] else head["nprobe"]
        Dw = torch.empty((nq, k), dtype=torch.float32, device="cuda")
        Iw = torch.empty((nq, k), dtype=torch.int64, device="cuda")
        while time.perf_counter() < t_end:
            ix.search(nq, test, k, Dw, Iw)
        torch.cuda.synchronize()

    # End to end through the public API: pinned host queries in, host results out
    # (same search settings as the headline step above).
    qh = test.cpu().pin_memory()
    Dh = torch.empty((nq, k), dtype=torch.float32).pin_memory()
    Ih = torch.empty((nq, k), dtype=torch.int64).pin_memory()
    qh_np, Dh_np, Ih_np = qh.numpy(), Dh.numpy(), Ih.numpy()
    for _ in range(args.warmup):
        ix.search(nq, qh_np, k, Dh_np, Ih_np)
    stream = torch.cuda.ExternalStream(ix.stream)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(args.steps):
        ix.search(nq, qh_np, k, Dh_np, Ih_np)
    e3.record(stream)
    e3.synchronize()
    e2e_ms = max(e2.elapsed_time(e3), (time.perf_counter() - t0) * 1e3) / args.steps
    if world > 1:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_recall = recall(Ih_np, gt, k)

    # Parity at this configuration (untimed).  The BF16 arms against the exact
    # FP32 scan over the same probe lists: the fixed-nprobe arm at its nprobe,
    # the learned arm with the same predicted per-query nprobe (the predictor
    # cuts the probe rows the same way for either precision).  The FP32 scan
    # against the reference's own Index::search is checked on the CPU-baseline
    # sample below.
    def exact_fp32(P, learned=False, target=0.0):
        sp = ix.search_params
        sp.precision, sp.learned_probe, sp.learned_target = Precision.FP32, learned, target
        ix.nprobe = P
        Dx = torch.empty((nq, k), dtype=torch.float32, device="cuda")
        Ix = torch.empty((nq, k), dtype=torch.int64, device="cuda")
        ix.search(nq, test, k, Dx, Ix)
        return Dx.cpu().numpy(), Ix.cpu().numpy()

    Pf, Pb = arms["fp32"]["nprobe"], arms["bf16"]["nprobe"]
    ref_b = outs["fp32"] if Pb == Pf else exact_fp32(Pb)
    ok_b, n_b = parity_count(*outs["bf16"], *ref_b)
    ref_l = exact_fp32(256, learned=True, target=tgt)
    ok_l, n_l = parity_count(*outs["learned_bf16"], *ref_l)
    Dh, Ih = outs["learned_bf16"] if head is arms["learned_bf16"] else outs["bf16"]
    parity = {
        "rule": "per query: distances bit-identical, ids identical except among ties at the k-th distance",
        "bf16_fixed_vs_fp32_exact": {"nprobe": Pb, "identical": ok_b, "queries": n_b},
        "learned_bf16_vs_learned_fp32_exact": {"identical": ok_l, "queries": n_l},
        "headline_max_rel_dist_err_vs_fp64": max_rel_err_vs_fp64(torch, base, test, Dh, Ih),
        "fp32_max_rel_dist_err_vs_fp64": max_rel_err_vs_fp64(torch, base, test, *outs["fp32"]),
    }

    # Roofline of the headline step's dominant kernel.
    hbm_peak, bf16_peak, peak_kind = load_peaks()
    P = head["nprobe"] if isinstance(head["nprobe"], int) else arms["bf16"]["nprobe"]
    probes, _ = ix.probe_lists(test.cpu().numpy(), P)
    sizes = ix.list_sizes()
    rows = int(sizes[probes].sum())
    kpad = (d + 63) // 64 * 64
    distinct = np.unique(probes)
    comp_bytes = int(sizes[distinct].sum()) * kpad * 2 + nq * d * 4
    flops = 2.0 * d * rows
    kms = head["kernel_ms"]
    top = max(kms, key=kms.get)
    roof = {"kernel": top, "kernel_ms": round(kms[top], 4), "peak_kind": peak_kind}
    if top == "scan_bf16":
        t = kms[top] / 1e3
        t_hbm, t_tc = comp_bytes / (hbm_peak * 1e9), flops / (bf16_peak * 1e12)
        if t_hbm >= t_tc:
            roof.update({"bound": "hbm", "achieved": round(comp_bytes / t / 1e9, 1), "peak": hbm_peak, "unit": "GB/s",
                         "frac": round(comp_bytes / t / 1e9 / hbm_peak, 3)})
        else:
            roof.update({"bound": "tensor", "achieved": round(flops / t / 1e12, 2), "peak": bf16_peak,
                         "unit": "TFLOP/s", "frac": round(flops / t / 1e12 / bf16_peak, 3)})
        roof.update({"traffic": int(SCAN_TRAFFIC_RATIO * comp_bytes), "bytes_compulsory_per_launch": comp_bytes,
                     "flops_per_launch": flops,
                     "note": "bytes = each probed list read once in BF16 (+ queries); flops = 2*d per "
                             "(query, probed vector); frac = max(bytes/BW, flops/TC) / t; traffic = DRAM "
                             f"read + write per launch, {SCAN_TRAFFIC_RATIO} x the algorithmic bytes as measured "
                             "by ncu on a 3M x 128 launch (profiles/scan_bf16_3m_ncu_full.md), scaled to this "
                             "launch by its algorithmic bytes"})
    else:
        t = kms[top] / 1e3
        nq_f = float(nq)
        if top.startswith("coarse"):
            fl = 3.0 * nq_f * WORKLOAD["nlist"] * d
            roof.update({"bound": "hbm", "achieved": round(nq_f * d * 4 / t / 1e9, 1), "peak": hbm_peak,
                         "unit": "GB/s", "frac": round(nq_f * d * 4 / t / 1e9 / hbm_peak, 4), "traffic": None,
                         "fp32_ops_per_launch": fl,
                         "note": "exact FP32 coarse distances: FP32-pipe bound (3 unfused ops per element pair)"})
        else:
            roof.update({"bound": "hbm", "achieved": None, "peak": hbm_peak, "unit": "GB/s", "frac": None,
                         "traffic": None})
    fp = arms["fp32"]
    fp_pairs = int(sizes[ix.probe_lists(test.cpu().numpy(), fp["nprobe"])[0]].sum())
    fp_bytes_alg = fp_pairs * d * 4
    fp_scan = fp["kernel_ms"].get("scan_exact", 0.0) / 1e3
    clocks = clk.summary()
    sm_mhz = clocks.get("sm_mhz") or 1965.0
    # The exact scan's own roofline is the FP32 pipe, not HBM (each probed list
    # is read once per group of 32 queries): 3 FP32 operations per (query,
    # vector, dimension), against SMs x 128 lanes x 2 (packed f32x2) x clock.
    fp_ops = 3.0 * fp_pairs * d
    fp_peak = 148 * 128 * 2 * sm_mhz * 1e6
    fp_roof = ({"bound": "fp32 pipe", "achieved": round(fp_ops / fp_scan / 1e12, 2), "peak": round(fp_peak / 1e12, 2),
                "unit": "TFLOP/s (FP32 ops)", "frac": round(fp_ops / fp_scan / fp_peak, 3),
                "note": "3 unfused FP32 ops per element pair; peak = 148 SMs x 128 lanes x 2 (f32x2) x sampled SM clock"}
               if fp_scan else None)
    result = None
    if rank == 0:
        result = {
            "metric": "QPS at recall@10>=0.95 (10M x 128, nlist 4096, k 10): learned-nprobe + BF16 tensor-core "
                      "scan + exact FP32 rerank vs plain FP32",
            "value": round(head["qps"], 1),
            "unit": "queries/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(head["ms_per_step"], 4),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "bf16",
            "data": "synthetic (seeded Gaussian mixture drawn on the GPU; no public dataset offline)",
            "config": {"workload": WORKLOAD["workload"], "nprobe": head["nprobe"],
                       "predictor_target": head.get("predictor_target"),
                       "avg_nprobe_validation": head.get("avg_nprobe_validation"),
                       "precision": "bf16 scan + fp32 rerank of 2k candidates",
                       "recall_at_10": round(head["recall_at_10"], 4), "queries_per_step": nq,
                       "parallelism": f"replicas x{world}",
                       "l2_flush": "not needed: 2.6-5.1 GB of codes > L2, every step touches every list",
                       **build},
            "plain_fp32": {"qps": round(fp["qps"], 1), "nprobe": fp["nprobe"],
                           "recall_at_10": round(fp["recall_at_10"], 4), "ms_per_step": round(fp["ms_per_step"], 3),
                           "kernel_ms_per_step": {n: round(v, 4) for n, v in fp["kernel_ms"].items()},
                           "scan_bytes_alg_gbs": round(fp_bytes_alg / fp_scan / 1e9, 1) if fp_scan else None,
                           "roofline": fp_roof},
            "bf16_fixed_nprobe": {"qps": round(arms["bf16"]["qps"], 1), "nprobe": arms["bf16"]["nprobe"],
                                  "bounded_scan": arms["bf16"].get("bounded_scan"),
                                  "recall_at_10": round(arms["bf16"]["recall_at_10"], 4),
                                  "ms_per_step": round(arms["bf16"]["ms_per_step"], 3),
                                  "kernel_ms_per_step": {n: round(v, 4) for n, v in arms["bf16"]["kernel_ms"].items()}},
            "speedup_vs_plain_fp32": round(head["qps"] / fp["qps"], 2),
            "e2e": {"value": round(world * nq / (e2e_ms / 1e3), 1), "unit": "queries/s",
                    "h2d_bytes_per_step": nq * d * 4, "d2h_bytes_per_step": nq * k * 12,
                    "recall_at_10": round(e2e_recall, 4)},
            "parity": parity,
            "roofline": roof,
            "kernel_ms_per_step": {n: round(v, 4) for n, v in kms.items()},
            "bounded_scan": head.get("bounded_scan"),
            "gpu_launches": int(round(head["launches_per_step"] * args.steps)),
            "clocks": clocks,
        }
        if world == 1 and not args.no_cpu_baseline:
            ix.search_params.precision, ix.search_params.learned_probe = Precision.FP32, False
            cb, Dr, Ir = cpu_baseline(ix, test.cpu().numpy(), fp["nprobe"], k, gt)
            result["cpu_baseline"] = cb
            n = Dr.shape[0]
            ok_r, _ = parity_count(outs["fp32"][0][:n], outs["fp32"][1][:n], Dr, Ir)
            parity["fp32_vs_reference_index_search"] = {
                "nprobe": fp["nprobe"], "identical": ok_r, "queries": n,
                "reference": "Index::search (ORIGINAL) of oracle/_ref on the same frozen index, the CPU-baseline sample"}
        print(json.dumps(result), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return result


def _ref_from_index(ix):
    """Freeze our index in the reference's file format and load it with the
    reference's own Index::load_index (oracle/_ref)."""
    import oracle
    if not oracle.RefIndex.available():
        oracle.build(reference=True)
    d = "/dev/shm" if os.path.isdir("/dev/shm") else tempfile.gettempdir()
    path = os.path.join(d, f"hb_bench_{os.getpid()}.index")
    ix.save_index(path)
    try:
        ref = oracle.RefIndex.load(path)
    finally:
        os.unlink(path)
    return ref


def cpu_baseline(ix, test_np, P, k, gt, budget_s=12.0):
    """The reference's own ORIGINAL-mode search (oracle/_ref) on all host cores."""
    import oracle
    ref = _ref_from_index(ix)
    ref.nprobe = P
    cores = os.cpu_count() or 1
    oracle.RefIndex.set_threads(cores)
    probe = test_np[:64]
    t0 = time.perf_counter()
    ref.search(probe, k)
    per_q = (time.perf_counter() - t0) / probe.shape[0]
    n = int(max(64, min(test_np.shape[0], budget_s / max(per_q, 1e-6))))
    sample = test_np[:n]
    t0 = time.perf_counter()
    Dr, Ir = ref.search(sample, k)
    t = time.perf_counter() - t0
    model, _, _ = oracle.host_cpu()
    return ({"value": round(n / t, 1), "unit": "queries/s", "cores": cores, "kind": "reference", "cpu_model": model,
             "reference_build": oracle.RefIndex.build_kind,
             "sample": f"first {n} of the 10k test queries, nprobe {P}, k {k}, one Index::search call "
                       f"(ORIGINAL mode, OpenMP over {cores} threads)",
             "recall_at_10": round(recall(Ir, gt[:n], k), 4)}, Dr, Ir)


def freeze_index(args):
    """Child process of the reference arm: build the 10M x 128 index on the GPU
    (the reference's CPU k-means over 10M x 4096 would take hours), pick the
    smallest nprobe whose exact search reaches the recall target against the
    FP64 ground truth, and write the frozen index in the reference's file
    format with the queries and ground truth into args.freeze_to."""
    import torch
    from harmony_b200 import Index, SearchMode
    _, _, local = dist_setup()
    torch.cuda.set_device(local)
    k, nq = WORKLOAD["k"], WORKLOAD["nq"]
    ix, base, test, build = build_index(torch, seed=5)
    gt = ground_truth(torch, ix, base, test, k)
    ix.preSearch(0, 0, 0, 0, 0, Index.Param(mode=SearchMode.ORIGINAL), "")
    D = torch.empty((nq, k), dtype=torch.float32, device="cuda")
    I = torch.empty((nq, k), dtype=torch.int64, device="cuda")
    P = NPROBE_SWEEP[-1]
    for p in NPROBE_SWEEP:
        ix.nprobe = p
        ix.search(nq, test, k, D, I)
        if recall(I.cpu().numpy(), gt, k) >= args.target:
            P = p
            break
    ix.save_index(os.path.join(args.freeze_to, "index"))
    np.save(os.path.join(args.freeze_to, "test.npy"), test.cpu().numpy())
    np.save(os.path.join(args.freeze_to, "gt.npy"), gt)
    with open(os.path.join(args.freeze_to, "meta.json"), "w") as f:
        json.dump({"nprobe": P, **build}, f)


def run_reference(args):
    """The reference's own CPU search (oracle/_ref: Index::search, ORIGINAL
    mode, OpenMP over every host core) on the frozen index.  The index is
    built and frozen by a child process, so this process loads only the
    reference library (no torch, no CUDA library of this project)."""
    world, rank, local = dist_setup()
    if rank != 0:
        return None
    import shutil
    import oracle
    k, nq = WORKLOAD["k"], WORKLOAD["nq"]
    d = tempfile.mkdtemp(prefix="hb_ref_", dir="/dev/shm" if os.path.isdir("/dev/shm") else None)
    try:
        cmd = [sys.executable, os.path.abspath(__file__), "--freeze-to", d, "--target", str(args.target)]
        if args.nb:
            cmd += ["--nb", str(args.nb)]
        subprocess.run(cmd, check=True)
        with open(os.path.join(d, "meta.json")) as f:
            meta = json.load(f)
        test_np = np.load(os.path.join(d, "test.npy"))
        gt = np.load(os.path.join(d, "gt.npy"))
        if not oracle.RefIndex.available():
            oracle.build(reference=True)
        ref = oracle.RefIndex.load(os.path.join(d, "index"))
    finally:
        shutil.rmtree(d, ignore_errors=True)
    P = int(meta.pop("nprobe"))
    ref.nprobe = P
    cores = os.cpu_count() or 1
    oracle.RefIndex.set_threads(cores)
    model, _, _ = oracle.host_cpu()
    # Bounded sample per step so the whole run stays within a few minutes.
    t0 = time.perf_counter()
    ref.search(test_np[:64], k)
    per_q = (time.perf_counter() - t0) / 64
    n = int(max(64, min(nq, args.ref_step_seconds / max(per_q, 1e-6))))
    sample = test_np[:n]
    for _ in range(args.warmup):
        ref.search(sample, k)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        Dr, Ir = ref.search(sample, k)
    t = (time.perf_counter() - t0) / args.steps
    value = n / t
    res = {
        "metric": "QPS at recall@10>=0.95 (10M x 128, nlist 4096, k 10): learned-nprobe + BF16 tensor-core "
                  "scan + exact FP32 rerank vs plain FP32",
        "impl": "reference",
        "value": round(value, 1), "unit": "queries/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(t * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Gaussian mixture drawn on the GPU)",
        "config": {"workload": WORKLOAD["workload"], "nprobe": P, "queries_per_step": n,
                   "recall_at_10": round(recall(Ir, gt[:n], k), 4), **meta},
        "cpu_baseline": {"value": round(value, 1), "unit": "queries/s", "cores": cores, "kind": "reference",
                         "cpu_model": model, "reference_build": oracle.RefIndex.build_kind,
                         "sample": f"first {n} test queries per step; reference Index::search, ORIGINAL mode; "
                                   f"index frozen by a child process, loaded with the reference's load_index"},
        "e2e": {"value": round(value, 1), "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(res), flush=True)
    return res


def run_c4(args):
    """Config 4: 10M x 96 with Zipf(1.1) list sizes, nlist 4096, k 10, 50k
    queries with per-query nprobe in U[4, 256], searched in batches of 1, 8,
    64, 512 and 4096.  Each batch is one public-API call with the queries in
    pinned host memory and the results copied back (end to end, wall clock
    around the synchronous calls) and, separately, with queries and results
    resident on the device (CUDA events); each both as ordinary calls and as
    one CUDA-graph launch per batch (params.use_graph).  QPS per batch size,
    FP32 exact and BF16 + rerank."""
    import torch
    from harmony_b200 import Index, Precision, SearchMode, datasets
    k, nq, nb, d = 10, args.nq or 50_000, args.nb or 10_000_000, 96
    base, queries = datasets.config4_device(nb=nb, nq=nq)
    ix = Index(d, 4096, 16)
    t0 = time.perf_counter()
    ix.train(base.shape[0], base)
    ix.add(base.shape[0], base)
    torch.cuda.synchronize()
    build_s = round(time.perf_counter() - t0, 2)
    sizes = ix.list_sizes()
    npq = datasets.config4_nprobes(nq)
    ix.preSearch(0, 0, 0, 0, 0, Index.Param(mode=SearchMode.ORIGINAL), "")
    # Ground truth on the first 2000 queries (FP32 exhaustive + FP64 re-rank).
    ng = min(2000, nq)
    gt = ground_truth(torch, ix, base, queries[:ng], k)
    ix.preSearch(0, 0, 0, 0, 0, Index.Param(mode=SearchMode.ORIGINAL), "")
    q_host = torch.empty((nq, d), dtype=torch.float32).pin_memory()
    q_host.copy_(queries.cpu())
    npq_dev = torch.from_numpy(npq).cuda()
    D_host = torch.empty((nq, k), dtype=torch.float32).pin_memory()
    I_host = torch.empty((nq, k), dtype=torch.int64).pin_memory()
    D_dev = torch.empty((nq, k), dtype=torch.float32, device="cuda")
    I_dev = torch.empty((nq, k), dtype=torch.int64, device="cuda")
    stream = torch.cuda.ExternalStream(ix.stream)
    sizes_b = [1, 8, 64, 512, 4096]
    out = {}
    for name, prec in (("fp32", Precision.FP32), ("bf16", Precision.BF16)):
        sp = ix.search_params
        sp.precision, sp.rerank_mult, sp.max_nprobe = prec, 2, 256
        res = {}
        for mode in ("e2e", "device", "e2e_graph", "device_graph"):
            sp.use_graph = mode.endswith("_graph")
            by = {}
            for B in sizes_b:
                calls = max(1, min(nq // B, 200 if B < 512 else 48))
                def one(off):
                    if mode.startswith("device"):
                        sp.nprobe_per_query = npq_dev[off:off + B]
                        ix.search(B, queries[off:off + B], k, D_dev[off:off + B], I_dev[off:off + B])
                    else:
                        sp.nprobe_per_query = npq[off:off + B]
                        ix.search(B, q_host[off:off + B], k, D_host[off:off + B], I_host[off:off + B])
                for c in range(3):  # warm-up
                    one((c * B) % (nq - B + 1))
                torch.cuda.synchronize()
                if mode.startswith("device"):
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    for c in range(calls):
                        one(c * B)
                    e1.record(stream)
                    e1.synchronize()
                    dt = e0.elapsed_time(e1) / 1e3
                else:
                    t1 = time.perf_counter()
                    for c in range(calls):
                        one(c * B)
                    dt = time.perf_counter() - t1
                by[str(B)] = {"qps": round(calls * B / dt, 1), "ms_per_call": round(1e3 * dt / calls, 3),
                              "calls": calls}
            res[mode] = by
        sp.use_graph = False
        # Device time per kernel of one batch at the small sizes (no graph).
        kern = {}
        for B in (1, 64):
            reps = 10
            ix.profile(True)
            for c in range(reps):
                sp.nprobe_per_query = npq_dev[c * B:(c + 1) * B]
                ix.search(B, queries[c * B:(c + 1) * B], k, D_dev[:B], I_dev[:B])
            prof = ix.profile_read()
            ix.profile(False)
            kern[str(B)] = {n: round(v[0] / reps, 4) for n, v in prof.items()}
        res["kernel_ms"] = kern
        # Recall of the first 2000 queries at their own nprobe, one call.
        sp.nprobe_per_query = npq[:ng]
        ix.search(ng, q_host[:ng], k, D_host[:ng], I_host[:ng])
        I_check = I_host[:ng].numpy()
        res["recall_at_10_first_2000"] = round(recall(I_check, gt, k), 4)
        if prec == Precision.BF16:
            res["bounded_scan_first_2000"] = ix.bf16_stats()
        res["max_rel_dist_err_vs_fp64_first_2000"] = max_rel_err_vs_fp64(
            torch, base, queries[:ng], D_host[:ng].numpy(), I_check)
        out[name] = res
        ix.search_params.nprobe_per_query = None
        ix.search_params.max_nprobe = 0
        ix.search_params.precision = Precision.FP32
    line = {"metric": "QPS per batch size, config4 stream (10M x 96, Zipf list sizes, nlist 4096, k 10, "
                      "per-query nprobe U[4,256], batches of 1..4096)",
            "workload": "c4", "unit": "queries/s", "n_gpus": 1, "dtype": "f32 / bf16",
            "data": "synthetic (seeded Zipf(1.1) Gaussian mixture drawn on the GPU)",
            "config": {"nb": nb, "d": d, "nlist": 4096, "k": k, "nq": nq, "batch_sizes": sizes_b,
                       "list_size_min": int(sizes.min()), "list_size_max": int(sizes.max()),
                       "build_s": build_s},
            "arms": out}
    print(json.dumps(line))


def run_c3(args):
    """Config 3: 270k x 500 anisotropic mixture (per-dimension variance
    proportional to (j + 1)^-1.2), nlist 512, nprobe 32, k 100, 5000 queries.
    Arms: the exact FP32 scan, the BF16 candidate-matrix scan with the exact
    FP32 re-rank of the 2k (rerank_mult 2) and 4k best, and the FP8 E4M3
    variant (per-list and per-query scales) re-ranking the 4k and 8k best.  Each arm is timed with
    queries and results resident on the device (CUDA events on the index
    stream) and end to end (pinned host queries and results, wall clock around
    the synchronous calls).  Recall@100 and the largest relative distance error
    are taken against FP64 ground truth on the first 1000 queries; same_as_fp32
    is the fraction of queries whose k results equal the exact scan's bit for
    bit."""
    import torch
    from harmony_b200 import Index, Precision, SearchMode, datasets
    k, nq, nb, d, nlist, P = 100, args.nq or 5000, args.nb or 270_000, 500, 512, 32
    base_np, q_np = datasets.config3(nb=nb, nq=nq)
    base = torch.from_numpy(base_np).cuda()
    queries = torch.from_numpy(q_np).cuda()
    ix = Index(d, nlist, P)
    t0 = time.perf_counter()
    ix.train(nb, base)
    ix.add(nb, base)
    torch.cuda.synchronize()
    build_s = round(time.perf_counter() - t0, 2)
    # FP64 ground truth of the first 1000 queries: exhaustive FP32 top 128,
    # re-ranked in FP64.
    ng = min(1000, nq)
    ix.preSearch(0, 0, 0, 0, 0, Index.Param(mode=SearchMode.BRUTE_FORCE), "")
    GI = torch.empty((ng, 128), dtype=torch.int64, device="cuda")
    G = torch.empty((ng, 128), dtype=torch.float32, device="cuda")
    ix.search(ng, queries[:ng], 128, G, GI)
    cand = base[GI.reshape(-1)].double().reshape(ng, 128, d)
    d64 = ((cand - queries[:ng].double()[:, None, :]) ** 2).sum(-1)
    order = torch.argsort(d64, dim=1, stable=True)
    gt = torch.gather(GI, 1, order)[:, :k].cpu().numpy()
    del cand, d64
    ix.preSearch(0, 0, 0, 0, 0, Index.Param(mode=SearchMode.ORIGINAL), "")
    ix.nprobe = P
    q_host = torch.empty((nq, d), dtype=torch.float32).pin_memory()
    q_host.copy_(queries.cpu())
    D_host = torch.empty((nq, k), dtype=torch.float32).pin_memory()
    I_host = torch.empty((nq, k), dtype=torch.int64).pin_memory()
    D_dev = torch.empty((nq, k), dtype=torch.float32, device="cuda")
    I_dev = torch.empty((nq, k), dtype=torch.int64, device="cuda")
    stream = torch.cuda.ExternalStream(ix.stream)
    arms, ref = {}, None
    for name, prec, mult in (("fp32", Precision.FP32, 2), ("bf16_rerank2k", Precision.BF16, 2),
                             ("bf16_rerank4k", Precision.BF16, 4), ("fp8_rerank4k", Precision.FP8, 4),
                             ("fp8_rerank8k", Precision.FP8, 8)):
        sp = ix.search_params
        sp.precision, sp.rerank_mult = prec, mult
        reps = 3 if prec == Precision.FP32 else 10
        for _ in range(3):
            ix.search(nq, queries, k, D_dev, I_dev)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            ix.search(nq, queries, k, D_dev, I_dev)
        e1.record(stream)
        e1.synchronize()
        ms_dev = e0.elapsed_time(e1) / reps
        t1 = time.perf_counter()
        for _ in range(reps):
            ix.search(nq, q_host, k, D_host, I_host)
        ms_e2e = 1e3 * (time.perf_counter() - t1) / reps
        ix.profile(True)
        ix.search(nq, queries, k, D_dev, I_dev)
        kern = {kk: round(v[0], 3) for kk, v in ix.profile_read().items()}
        ix.profile(False)
        Dn, In = D_dev.cpu().numpy(), I_dev.cpu().numpy()
        # Largest relative error of the returned distances against FP64.
        sel = torch.from_numpy(In[:ng]).cuda()
        x = base[sel.reshape(-1)].double().reshape(ng, k, d)
        e64 = ((x - queries[:ng].double()[:, None, :]) ** 2).sum(-1).cpu().numpy()
        del x
        err = float(np.max(np.abs(Dn[:ng].astype(np.float64) - e64) / np.maximum(e64, 1e-30)))
        arm = {"ms_device": round(ms_dev, 3), "qps_device": round(nq / ms_dev * 1e3, 1),
               "ms_e2e": round(ms_e2e, 3), "qps_e2e": round(nq / ms_e2e * 1e3, 1),
               "recall_at_100_vs_fp64_first_1000": round(recall(In[:ng], gt, k), 4),
               "max_rel_dist_err_vs_fp64": err, "kernels_ms": kern}
        if ref is None:
            ref = Dn
        else:
            arm["same_as_fp32"] = round(float(np.mean([np.array_equal(a, b) for a, b in
                                                       zip(Dn.view(np.uint32), ref.view(np.uint32))])), 4)
        arms[name] = arm
    ix.search_params.precision = Precision.FP32
    line = {"metric": "QPS, config3 (270k x 500 anisotropic mixture, nlist 512, nprobe 32, k 100, 5000 queries)",
            "workload": "c3", "unit": "queries/s", "n_gpus": 1, "dtype": "f32 / bf16",
            "data": "synthetic (seeded anisotropic Gaussian mixture; stands in for nuswide's shape)",
            "config": {"nb": nb, "d": d, "nlist": nlist, "nprobe": P, "k": k, "nq": nq, "build_s": build_s,
                       "inputs": "8.6 MB of queries per step; the index (540 MB FP32 + 276 MB BF16) exceeds L2"},
            "arms": arms}
    print(json.dumps(line))


def run_c2(args):
    """Config 2: 1,000,000 x 128 (1000 unit-variance components, centres
    N(0, 4^2)), 10,000 queries, nlist 1024, k 100, the reference driver's
    nprobe sweep 8 / 16 / 32 / 64 / 128 (src/query.cpp:680-777).  Per nprobe:
    the plain FP32 scan (the reference's arithmetic) and the bounded BF16 scan
    (whose result must equal it), device-timed (CUDA events on the index
    stream, queries and results resident), with the scan kernel's own time,
    its algorithmic bytes (every probed list read once per probing query, the
    reference's traffic) and its FP32-pipe fraction (3 FP32 operations per
    element pair against SMs x 128 lanes x 2 (packed f32x2) x the sampled
    clock); recall@100 against FP64 ground truth on the first 1000 queries."""
    import torch
    from harmony_b200 import Index, Precision, SearchMode, datasets
    k, nq, nb, d, nlist = 100, args.nq or 10_000, args.nb or 1_000_000, 128, 1024
    base_np, q_np = datasets.config2(nb=nb, nq=nq)
    base = torch.from_numpy(base_np).cuda()
    queries = torch.from_numpy(q_np).cuda()
    ix = Index(d, nlist, 8)
    t0 = time.perf_counter()
    ix.train(nb, base)
    ix.add(nb, base)
    torch.cuda.synchronize()
    build_s = round(time.perf_counter() - t0, 2)
    ng = min(1000, nq)
    ix.preSearch(0, 0, 0, 0, 0, Index.Param(mode=SearchMode.BRUTE_FORCE), "")
    GI = torch.empty((ng, 128), dtype=torch.int64, device="cuda")
    G = torch.empty((ng, 128), dtype=torch.float32, device="cuda")
    ix.search(ng, queries[:ng], 128, G, GI)
    cand = base[GI.reshape(-1)].double().reshape(ng, 128, d)
    d64 = ((cand - queries[:ng].double()[:, None, :]) ** 2).sum(-1)
    gt = torch.gather(GI, 1, torch.argsort(d64, dim=1, stable=True))[:, :k].cpu().numpy()
    del cand, d64
    ix.preSearch(0, 0, 0, 0, 0, Index.Param(mode=SearchMode.ORIGINAL), "")
    sizes = ix.list_sizes()
    D = torch.empty((nq, k), dtype=torch.float32, device="cuda")
    I = torch.empty((nq, k), dtype=torch.int64, device="cuda")
    stream = torch.cuda.ExternalStream(ix.stream)
    sweep = []
    with ClockSampler(0) as clk:
        for P in (8, 16, 32, 64, 128):
            ix.nprobe = P
            probes, _ = ix.probe_lists(q_np, P)
            pairs = int(sizes[probes].sum())
            row = {"nprobe": P, "probed_vectors_per_query": round(pairs / nq, 1)}
            outs = {}
            for name, prec in (("fp32", Precision.FP32), ("bf16", Precision.BF16)):
                ix.search_params.precision = prec
                reps = 3 if prec == Precision.FP32 else 10
                for _ in range(3):
                    ix.search(nq, queries, k, D, I)
                torch.cuda.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                for _ in range(reps):
                    ix.search(nq, queries, k, D, I)
                e1.record(stream)
                e1.synchronize()
                ms = e0.elapsed_time(e1) / reps
                ix.profile(True)
                ix.search(nq, queries, k, D, I)
                kern = {kk: round(v[0], 4) for kk, v in ix.profile_read().items()}
                ix.profile(False)
                outs[name] = (D.cpu().numpy().copy(), I.cpu().numpy().copy())
                stats = ix.bf16_stats() if prec == Precision.BF16 else None
                arm = {"ms": round(ms, 3), "qps": round(nq / ms * 1e3, 1), "kernels_ms": kern,
                       "recall_at_100_first_1000": round(recall(outs[name][1][:ng], gt, k), 4)}
                if stats:
                    arm["bounded_scan"] = stats
                scan = kern.get("scan_exact" if prec == Precision.FP32 else "scan_bf16")
                if scan:
                    elem = 2 if prec == Precision.BF16 else 4
                    arm["scan_bytes_alg_gbs"] = round(pairs * d * elem / (scan / 1e3) / 1e9, 1)
                    if prec == Precision.FP32:
                        arm["scan_fp32_ops_per_s"] = 3.0 * pairs * d / (scan / 1e3)
                row[name] = arm
            ok, n = parity_count(*outs["bf16"], *outs["fp32"])
            row["bf16_identical_to_fp32"] = {"identical": ok, "queries": n}
            # Largest relative error of the returned distances against FP64
            # recomputation, first 1000 queries.
            for name in ("fp32", "bf16"):
                Dn, In = outs[name]
                row[name]["max_rel_dist_err_vs_fp64_first_1000"] = max_rel_err_vs_fp64(
                    torch, base, queries[:ng], Dn[:ng], In[:ng])
            sweep.append(row)
        ix.search_params.precision = Precision.FP32
    ck = clk.summary()
    sm = ck.get("sm_mhz") or 1965.0
    peak = 148 * 128 * 2 * sm * 1e6
    for row in sweep:
        v = row["fp32"].get("scan_fp32_ops_per_s")
        if v:
            row["fp32"]["scan_fp32_pipe_frac"] = round(v / peak, 3)
            row["fp32"]["scan_fp32_ops_per_s"] = round(v / 1e12, 2)
    line = {"metric": "QPS per nprobe, config2 (1M x 128, nlist 1024, k 100, 10k queries)",
            "workload": "c2", "unit": "queries/s", "n_gpus": 1, "dtype": "f32 / bf16",
            "data": "synthetic (seeded 1000-component Gaussian mixture, centres N(0, 4^2); stands in for sift1m's shape)",
            "config": {"nb": nb, "d": d, "nlist": nlist, "k": k, "nq": nq, "build_s": build_s,
                       "list_size_min": int(sizes.min()), "list_size_max": int(sizes.max()),
                       "fp32_pipe_peak": "148 SMs x 128 lanes x 2 (f32x2) x sampled SM clock, 3 ops per element pair",
                       "inputs": "512 MB of FP32 codes > L2; every step reads each probed list"},
            "clocks": ck, "sweep": sweep}
    print(json.dumps(line))


def run_c5_batches(args):
    """Learned nprobe against fixed nprobe on the 10M x 128 index, by batch size.

    Both arms search in BF16 (the bounded scan, exact results) with the
    queries and results resident on the device, one CUDA-graph launch per
    batch.  The fixed arm uses the smallest nprobe whose recall@10 over the
    10k test queries reaches the target; the learned arm the smallest predictor
    target whose recall reaches it too.  A query's results do not depend on the
    other queries of its batch, so the recall of either arm is that of the
    whole test set.  Per batch size: QPS of each arm, their ratio, and the
    probed lists per batch (the distinct lists read)."""
    import torch
    from harmony_b200 import Index, Precision, SearchMode
    k, nq = WORKLOAD["k"], WORKLOAD["nq"]
    ix, base, test, train, build = build_index(torch, seed=5, ntrain=args.ntrain)
    gt = ground_truth(torch, ix, base, test, k)
    del base
    ix.preSearch(0, 0, 0, 0, 0, Index.Param(mode=SearchMode.ORIGINAL), "")
    ix.train_probe_predictor(train.shape[0], train, k=k, label_nprobe=256, target=args.target)
    del train
    P, rec_f = pick_nprobe(ix, test, gt, k, args.target, Precision.BF16)
    sp = ix.search_params
    D = torch.empty((nq, k), dtype=torch.float32, device="cuda")
    I = torch.empty((nq, k), dtype=torch.int64, device="cuda")
    sp.precision, sp.learned_probe = Precision.BF16, True
    ix.nprobe = 256
    tgt, rec_l = args.target, 0.0
    for tgt in [args.target + 0.005 * i for i in range(10)]:
        sp.learned_target = min(tgt, 0.9999)
        ix.search(nq, test, k, D, I)
        rec_l = recall(I.cpu().numpy(), gt, k)
        if rec_l >= args.target:
            break
    tgt = min(tgt, 0.9999)
    stream = torch.cuda.ExternalStream(ix.stream)
    q_np = test.cpu().numpy()
    rows = []
    for B in (1, 16, 64, 256, 1024, 4096):
        row = {"batch": B}
        calls = max(8, min(400, 20_000 // B))
        for name, learned in (("fixed", False), ("learned", True)):
            sp.use_graph, sp.learned_probe = True, learned
            sp.learned_target = tgt if learned else 0.0
            ix.nprobe = 256 if learned else P
            offs = [(c * B) % (nq - B + 1) for c in range(calls)]
            for o in offs[:3]:
                ix.search(B, test[o:o + B], k, D[o:o + B], I[o:o + B])
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for o in offs:
                ix.search(B, test[o:o + B], k, D[o:o + B], I[o:o + B])
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / calls
            row[name] = {"ms_per_batch": round(ms, 4), "qps": round(B / ms * 1e3, 1)}
        sp.use_graph = False
        # Lists read per batch (distinct probed lists of the first batch).
        sp.learned_probe = False
        pr_f, _ = ix.probe_lists(q_np[:B], P)
        row["fixed"]["lists_per_batch"] = int(np.unique(pr_f).size)
        row["learned_over_fixed"] = round(row["learned"]["qps"] / row["fixed"]["qps"], 3)
        if B in (16, 256, 4096):
            # Device time per kernel of one batch (no graph; the sum is a
            # little above the graph's time per batch).
            for name, learned in (("fixed", False), ("learned", True)):
                sp.learned_probe = learned
                sp.learned_target = tgt if learned else 0.0
                ix.nprobe = 256 if learned else P
                reps = 8
                ix.profile(True)
                for c in range(reps):
                    o = (c * B) % (nq - B + 1)
                    ix.search(B, test[o:o + B], k, D[o:o + B], I[o:o + B])
                prof = ix.profile_read()
                ix.profile(False)
                row[name]["kernel_ms"] = {n: round(v[0] / reps, 4) for n, v in prof.items()}
        rows.append(row)
    sp.use_graph, sp.learned_probe, sp.learned_target, sp.precision = False, False, 0.0, Precision.FP32
    thr, crec, cavg = ix.probe_calibration()
    i_sel = int(np.argmin(np.where(crec >= tgt, cavg, 1e9)))
    line = {"metric": "QPS by batch size, learned nprobe vs fixed nprobe (both BF16 bounded scan, exact results), "
                      "10M x 128, nlist 4096, k 10",
            "workload": "c5-batches", "unit": "queries/s", "n_gpus": 1, "dtype": "bf16",
            "data": "synthetic (seeded Gaussian mixture drawn on the GPU)",
            "config": {"fixed_nprobe": P, "fixed_recall_at_10": round(rec_f, 4), "predictor_target": round(tgt, 4),
                       "learned_recall_at_10": round(rec_l, 4),
                       "learned_avg_nprobe_validation": round(float(cavg[i_sel]), 2),
                       "timing": "CUDA events on the index stream, one CUDA-graph launch per batch, device-resident "
                                 "queries and results", **build},
            "batches": rows}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--target", type=float, default=0.95)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-step-seconds", type=float, default=6.0)
    ap.add_argument("--nb", type=int, default=None, help="smaller base for profiling runs (not a bench line)")
    ap.add_argument("--nq", type=int, default=None, help="fewer queries for profiling runs (not a bench line)")
    ap.add_argument("--nlist", type=int, default=None, help="other nlist for profiling runs (not a bench line)")
    ap.add_argument("--fixed-nprobe", type=int, default=None,
                    help="skip the recall sweep and use this nprobe (profiling runs; not a bench line)")
    ap.add_argument("--ntrain", type=int, default=200_000, help="training queries of the learned probe")
    ap.add_argument("--freeze-to", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--workload", choices=["c5", "c4", "c3", "c2", "c5-batches"], default="c5",
                    help="c5: the headline bench line; c4: the batch-stream measurement of config 4; "
                         "c3: the 500-dimensional k = 100 measurement of config 3; c2: the 1M x 128 nprobe sweep")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.nb and args.workload in ("c5", "c5-batches"):
        WORKLOAD["nb"] = args.nb
        WORKLOAD["workload"] += f" [reduced: nb={args.nb}]"
    if args.nlist and args.workload in ("c5", "c5-batches"):
        WORKLOAD["nlist"] = args.nlist
        WORKLOAD["workload"] += f" [reduced: nlist={args.nlist}]"
    if args.nq and args.workload in ("c5", "c5-batches"):
        WORKLOAD["nq"] = args.nq
        WORKLOAD["workload"] += f" [reduced: nq={args.nq}]"
    if args.freeze_to:
        freeze_index(args)
    elif args.workload == "c4":
        run_c4(args)
    elif args.workload == "c3":
        run_c3(args)
    elif args.workload == "c2":
        run_c2(args)
    elif args.workload == "c5-batches":
        run_c5_batches(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

"""Seeded synthetic stand-ins for the benchmark datasets of the IVF-flat path.

The reference benchmarks sift10k / sift1m / nuswide / msong files
(src/query.cpp:296-300); only sift10k ships with it and none of the large ones
is available offline, so every workload here is a seeded Gaussian mixture of
the named shape, drawn with ``numpy.random.default_rng(seed)`` (identical on
every machine).  Each generator returns ``(base, queries)`` as float32 C
arrays; sizes can be scaled down for tests with the same distribution.

  config1  10,000 x 128 (+100 queries), integers in [0, 255]: 100 components,
           centres uniform in [32, 224], sd 20, rounded and clipped (the shape
           and value range of the bundled sift10k).
  config2  1,000,000 x 128 (+10,000 queries): 1000 unit-variance components,
           centres N(0, 4^2).
  config3  270,000 x 500 (+5,000 queries): 1000 components, per-dimension
           scale (j+1)^-0.6 (variance decaying as (j+1)^-1.2) applied to
           centres N(0, 4^2) and unit noise alike.
  config4  10,000,000 x 96 (+50,000 queries): 4096 components with mixture
           weights proportional to rank^-1.1 (Zipf, s = 1.1), centres
           N(0, 4^2), unit noise.
  config5  10,000,000 x 128 (+10,000 test and 200,000 training queries):
           4096 unit-variance components, centres N(0, CONFIG5_SPREAD^2).
           The spread is chosen so that fixed-nprobe recall@10 reaches 0.95
           only at nprobe in the tens (config2's spread of 4 saturates recall
           at nprobe = 8).
"""
from __future__ import annotations

import numpy as np

CONFIG5_SPREAD = 0.68
CONFIG5_NOISE = 1.0


def _mixture(rng, n, centres, weights, noise_scale, chunk=1 << 20):
    k, d = centres.shape
    out = np.empty((n, d), np.float32)
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        comp = rng.choice(k, size=e - s, p=weights) if weights is not None else rng.integers(0, k, size=e - s)
        x = rng.standard_normal((e - s, d), dtype=np.float32)
        x *= noise_scale
        x += centres[comp]
        out[s:e] = x
    return out


def config1(seed: int = 1, nb: int = 10_000, nq: int = 100, d: int = 128, ncomp: int = 100):
    rng = np.random.default_rng(seed)
    centres = rng.uniform(32.0, 224.0, size=(ncomp, d)).astype(np.float32)
    base = _mixture(rng, nb, centres, None, np.float32(20.0))
    qs = _mixture(rng, nq, centres, None, np.float32(20.0))
    return (np.clip(np.rint(base), 0, 255).astype(np.float32),
            np.clip(np.rint(qs), 0, 255).astype(np.float32))


def config2(seed: int = 2, nb: int = 1_000_000, nq: int = 10_000, d: int = 128, ncomp: int = 1000):
    rng = np.random.default_rng(seed)
    centres = (rng.standard_normal((ncomp, d), dtype=np.float32) * np.float32(4.0))
    return _mixture(rng, nb, centres, None, np.float32(1.0)), _mixture(rng, nq, centres, None, np.float32(1.0))


def config3(seed: int = 3, nb: int = 270_000, nq: int = 5_000, d: int = 500, ncomp: int = 1000):
    rng = np.random.default_rng(seed)
    scale = ((np.arange(d, dtype=np.float64) + 1.0) ** -0.6).astype(np.float32)
    centres = rng.standard_normal((ncomp, d), dtype=np.float32) * np.float32(4.0) * scale
    return (_mixture(rng, nb, centres, None, scale), _mixture(rng, nq, centres, None, scale))


def zipf_weights(ncomp: int, s: float = 1.1):
    w = (np.arange(1, ncomp + 1, dtype=np.float64)) ** -s
    return w / w.sum()


def config4(seed: int = 4, nb: int = 10_000_000, nq: int = 50_000, d: int = 96, ncomp: int = 4096):
    rng = np.random.default_rng(seed)
    centres = rng.standard_normal((ncomp, d), dtype=np.float32) * np.float32(4.0)
    w = zipf_weights(ncomp)
    return _mixture(rng, nb, centres, w, np.float32(1.0)), _mixture(rng, nq, centres, w, np.float32(1.0))


def config4_nprobes(nq: int = 50_000, seed: int = 44, lo: int = 4, hi: int = 256):
    """Per-query nprobe, uniform in [lo, hi]."""
    return np.random.default_rng(seed).integers(lo, hi + 1, size=nq).astype(np.int32)


def config4_batches(nq: int = 50_000, seed: int = 45, lo: int = 1, hi: int = 4096):
    """Arrival batch sizes, uniform in [lo, hi], summing to nq."""
    rng = np.random.default_rng(seed)
    sizes = []
    left = nq
    while left > 0:
        b = int(min(left, rng.integers(lo, hi + 1)))
        sizes.append(b)
        left -= b
    return sizes


def config5(seed: int = 5, nb: int = 10_000_000, nq: int = 10_000, ntrain: int = 200_000, d: int = 128,
            ncomp: int = 4096, spread: float = CONFIG5_SPREAD):
    """Returns (base, test_queries, train_queries)."""
    rng = np.random.default_rng(seed)
    centres = rng.standard_normal((ncomp, d), dtype=np.float32) * np.float32(spread)
    base = _mixture(rng, nb, centres, None, np.float32(CONFIG5_NOISE))
    test = _mixture(rng, nq, centres, None, np.float32(CONFIG5_NOISE))
    train = _mixture(rng, ntrain, centres, None, np.float32(CONFIG5_NOISE)) if ntrain else None
    return base, test, train


def read_fvecs(path: str) -> np.ndarray:
    """fvecs: per row an int32 dimension then d float32 (reference README.md)."""
    raw = np.fromfile(path, dtype=np.int32)
    if raw.size == 0:
        return np.zeros((0, 0), np.float32)
    d = int(raw[0])
    return raw.reshape(-1, d + 1)[:, 1:].copy().view(np.float32)


def write_fvecs(path: str, x: np.ndarray) -> None:
    x = np.ascontiguousarray(x, dtype=np.float32)
    n, d = x.shape
    out = np.empty((n, d + 1), np.int32)
    out[:, 0] = d
    out[:, 1:] = x.view(np.int32)
    out.tofile(path)


def device_mixture(n, d, ncomp, spread, noise=1.0, seed=0, weights=None, device="cuda", gen_chunk=1 << 22):
    """The same Gaussian-mixture family generated on the GPU with a seeded
    torch generator (for the 10M-vector workloads, where host generation
    takes tens of seconds).  Returns (base, centres) as CUDA tensors.
    Deterministic for a given seed, torch build and GPU model."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    centres = torch.randn((ncomp, d), generator=g, device=device, dtype=torch.float32) * spread
    out = torch.empty((n, d), device=device, dtype=torch.float32)
    w = None if weights is None else torch.as_tensor(weights, device=device, dtype=torch.float32)
    for s in range(0, n, gen_chunk):
        e = min(n, s + gen_chunk)
        if w is None:
            comp = torch.randint(0, ncomp, (e - s,), generator=g, device=device)
        else:
            comp = torch.multinomial(w, e - s, replacement=True, generator=g)
        torch.randn((e - s, d), generator=g, device=device, dtype=torch.float32, out=out[s:e])
        out[s:e].mul_(noise).add_(centres[comp])
    return out, centres


def config5_device(seed: int = 5, nb: int = 10_000_000, nq: int = 10_000, ntrain: int = 200_000,
                   d: int = 128, ncomp: int = 4096, spread: float = CONFIG5_SPREAD, device="cuda"):
    """config5 drawn on the GPU: (base, test, train) CUDA tensors."""
    import torch
    allx, _ = device_mixture(nb + nq + ntrain, d, ncomp, spread, CONFIG5_NOISE, seed, None, device)
    return allx[:nb], allx[nb:nb + nq], (allx[nb + nq:] if ntrain else None)


def config4_device(seed: int = 4, nb: int = 10_000_000, nq: int = 50_000, d: int = 96, ncomp: int = 4096,
                   device="cuda"):
    """config4 drawn on the GPU: (base, queries) CUDA tensors, Zipf(1.1) weights."""
    allx, _ = device_mixture(nb + nq, d, ncomp, 4.0, 1.0, seed, zipf_weights(ncomp), device)
    return allx[:nb], allx[nb:]

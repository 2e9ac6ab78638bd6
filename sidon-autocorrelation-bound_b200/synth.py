"""Seeded synthetic heights for the benchmark and parity workloads.

No public dataset is involved: every workload is generated here from a fixed
seed.  Each candidate has its own numpy PCG64 stream seeded with
``SeedSequence([seed, index])``, so any candidate can be regenerated alone.

Generators (sizes are arguments):

* ``structured``: the plain-method profile -- a_i ~ U[0,1], each cell zeroed
  with probability 1/3, cells [n/50, n/8) forced to zero (support gap), cell 0
  set to 8x the mean (endpoint atom), then a_i *= (1 + i/n) (asymmetry).
* ``lognormal``: the precision-sweep profile -- a_i ~ lognormal(0, 1) in
  fp32, 1/3 exact zeros, a support gap of width n/10 at [n/50, n/50 + n/10),
  cell 0 set to 8x the mean.

Both optionally normalise each row to sum 1 (the reference driver seeds its
population normalised, src/main.cu:549-552).
"""
from __future__ import annotations

import numpy as np


def _rng(seed: int, index: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(np.random.SeedSequence([int(seed), int(index)])))


def structured_one(n: int, seed: int, index: int = 0) -> np.ndarray:
    r = _rng(seed, index)
    a = r.uniform(0.0, 1.0, n)
    a[r.uniform(0.0, 1.0, n) < 1.0 / 3.0] = 0.0
    a[n // 50: n // 8] = 0.0
    a[0] = 8.0 * a.mean()
    a *= 1.0 + np.arange(n) / n
    return a


def lognormal_one(n: int, seed: int, index: int = 0) -> np.ndarray:
    r = _rng(seed, index)
    a = r.lognormal(0.0, 1.0, n).astype(np.float32).astype(np.float64)
    a[r.uniform(0.0, 1.0, n) < 1.0 / 3.0] = 0.0
    g0 = n // 50
    a[g0: g0 + n // 10] = 0.0
    a[0] = 8.0 * a.mean()
    return a


def population(kind: str, n: int, P: int, seed: int, normalise: bool = True,
               dtype=np.float32) -> np.ndarray:
    gen = {"structured": structured_one, "lognormal": lognormal_one}[kind]
    out = np.empty((P, n), dtype=np.float64)
    for p in range(P):
        out[p] = gen(n, seed, p)
    if normalise:
        s = out.sum(axis=1, keepdims=True)
        s[s <= 0] = 1.0
        out /= s
    return out.astype(dtype)


def uneven_sizes(P: int, seed: int, levels=(512, 1024, 2048, 4096, 8400)) -> np.ndarray:
    """n per candidate drawn uniformly from the ladder levels (batched islands)."""
    r = _rng(seed, 1 << 30)
    return np.asarray(levels)[r.integers(0, len(levels), P)]


def ragged_population(sizes, seed: int, kind: str = "structured",
                      normalise: bool = True, dtype=np.float32) -> list[np.ndarray]:
    """One candidate per entry of sizes (candidate p from stream [seed, p])."""
    gen = {"structured": structured_one, "lognormal": lognormal_one}[kind]
    rows = []
    for p, n in enumerate(sizes):
        a = gen(int(n), seed, p)
        if normalise:
            s = a.sum()
            a = a / (s if s > 0 else 1.0)
        rows.append(a.astype(dtype))
    return rows

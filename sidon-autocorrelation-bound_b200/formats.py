"""The reference's vector and certificate formats.

* text vector (saveVec / loadVec, src/main.cu:329-352): two ``#`` comment
  lines, ``n <count>``, ``F <value>`` in scientific notation with 17
  significant digits, then one height per line at 17 significant digits;
  the reader skips blank/``#`` lines and checks the count;
* JSON certificate (certificates/*.json, checked by verify.py:81-100): keys
  problem, page, claim, formula, n, F, non_zero_cells, found_by, weights.
"""
from __future__ import annotations

import json
import pathlib

import numpy as np


def save_vec(path, a, f: float) -> None:
    a = np.asarray(a, dtype=np.float64)
    lines = [
        "# AlphaEvolve problem 2 -- autocorrelation / Sidon",
        "# F = 2*n*max_k b_k / (sum a)^2  is an upper bound on C",
        f"n {a.size}",
        f"F {f:.16e}",
    ]
    lines += [f"{x:.17g}" for x in a]
    pathlib.Path(path).write_text("\n".join(lines) + "\n")


def load_vec(path) -> np.ndarray:
    n = 0
    vals = []
    for line in pathlib.Path(path).read_text().splitlines():
        if not line or line[0] == "#":
            continue
        if line.startswith("n "):
            n = int(line[2:])
            continue
        if line.startswith("F "):
            continue
        vals.append(float(line))
    if not vals or (n and len(vals) != n):
        raise ValueError(f"{path}: expected {n} heights, read {len(vals)}")
    return np.asarray(vals, dtype=np.float64)


CERT_KEYS = ("problem", "page", "claim", "formula", "n", "F", "non_zero_cells", "found_by",
             "weights")


def write_certificate(path, a, F: float, found_by: str) -> dict:
    a = np.asarray(a, dtype=np.float64)
    cert = {
        "problem": "AlphaEvolve problem 2 - an autocorrelation problem related to Sidon sets",
        "page": "https://google-deepmind.github.io/alphaevolve_repository_of_problems/problems/2.html",
        "claim": "C <= F, where C is the largest constant in the problem statement",
        "formula": "F = 2*n*max_k b_k / (sum_i a_i)^2,  b_k = sum_{i+j=k} a_i a_j,  a_i >= 0",
        "n": int(a.size),
        "F": float(F),
        "non_zero_cells": int(np.count_nonzero(a)),
        "found_by": found_by,
        "weights": [float(x) for x in a],
    }
    pathlib.Path(path).write_text(json.dumps(cert))
    return cert


def read_certificate(path) -> dict:
    cert = json.loads(pathlib.Path(path).read_text())
    missing = [k for k in ("n", "F", "weights") if k not in cert]
    if missing:
        raise ValueError(f"{path}: missing keys {missing}")
    return cert

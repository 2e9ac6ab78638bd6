"""The precision sweep at the benchmark's size (n = 8400, lognormal heights
with 1/3 exact zeros, an endpoint atom and a support gap of width n/10):
the reported objective F = 2n max b / S^2, the smoothed objective G_p and
its gradient, for every arithmetic mode, against the long-double oracle.
Needs a B200.  Run with -s to see the table.

Bars per mode (relative; gradient errors relative to max |grad|):
  F                 every mode: 1e-6 (max b is refined in fp64)
  G_p               fp32: 1e-5, TF32x3 / BF16x3: 1e-4, BF16x1: 5e-2
  gradient          fp32: 1e-4 p, TF32x3 / BF16x3: max(2e-3, 2e-5 p),
                    BF16x1: 0.5
TF32x3 splits each operand into two TF32 parts (about 22 significant bits,
three products); like BF16x3 it is bound by the tensor pipe's fp32
accumulation.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

N, SAMPLE = 8400, 3
BARS = {
    "fp32": (1e-6, 1e-5, lambda p: 1e-4 * p),
    "bf16x3": (1e-6, 1e-4, lambda p: max(2e-3, 2e-5 * p)),
    "bf16x1": (1e-6, 5e-2, lambda p: 0.5),
    "tf32x3": (1e-6, 1e-4, lambda p: max(2e-3, 2e-5 * p)),
}


def test_precision_sweep_n8400(cuda, orc):
    from sidon_b200 import kernels as K, synth
    pop = synth.population("lognormal", N, SAMPLE, seed=8400)
    a = torch.as_tensor(pop, device=cuda)
    hostF = [orc.host_f(pop[r].astype(np.float64)) for r in range(SAMPLE)]
    ref = {p: [orc.lp_grad(pop[r].astype(np.float64), p) for r in range(SAMPLE)]
           for p in (8.0, 64.0, 512.0)}
    rows = []
    for mode, (bF, bG, bg) in BARS.items():
        for p in (8.0, 64.0, 512.0):
            val, saved, _ = K.lp_forward(a, p, precision=mode)
            g = K.lp_backward(a, saved, p, precision=mode).cpu().numpy()
            S = saved[:, 1].double().cpu().numpy()
            M = saved[:, 0].double().cpu().numpy()
            eF = max(abs(2 * N * M[r] / S[r] ** 2 - hostF[r]) / hostF[r] for r in range(SAMPLE))
            eG = max(abs(val[r].item() - ref[p][r][1]) / ref[p][r][1] for r in range(SAMPLE))
            eg = max(np.max(np.abs(g[r] - ref[p][r][0])) / np.abs(ref[p][r][0]).max()
                     for r in range(SAMPLE))
            rows.append((mode, p, eF, eG, eg))
            assert eF <= bF and eG <= bG and eg <= bg(p), (mode, p, eF, eG, eg)
    print("\nmode    p     F rel err   G_p rel err  grad rel err")
    for mode, p, eF, eG, eg in rows:
        print(f"{mode:7s} {p:5.0f} {eF:11.2e} {eG:12.2e} {eg:12.2e}")

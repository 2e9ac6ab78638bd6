"""The fp64 polish of the elite (src/main.cu:798-874) through sidon_polish.
Needs a B200.

Bar: the stream-ordered entry point equals the same schedule run pass by
pass through the fp64 local search and evaluation entry points bit for bit,
and it never reports a worse vector than the one it started from.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def K():
    from sidon_b200 import kernels
    return kernels


def test_polish_equals_pass_by_pass(cuda):
    from sidon_b200 import synth
    a = synth.structured_one(300, 5)
    a = a / a.sum()
    Kc, iters, passes = 4, 60, 6
    best_a, best_F, fit = K().polish(a, K=Kc, iters=iters, passes=passes, seed=3)
    pop = torch.as_tensor(K().polish_population(a, Kc, 3), device=cuda)
    ref_best = torch.as_tensor(a, device=cuda).clone()
    ref_F = K().run_eval(ref_best[None, :], with_nactive=False)[0].item()
    for q in range(passes):
        pA = 200.0 * 4.0 ** q
        lA = 0.010 * 0.45 ** q
        K().run_local_search(pop, iters // passes, pA, pA * 30.0, lA, lA * 0.02)
        f, _ = K().run_eval(pop, active_tol=1e-6)
        f = f.cpu().numpy()
        bk = int(np.argmin(f))
        if f[bk] < ref_F:
            ref_F = float(f[bk])
            ref_best = pop[bk].clone()
    assert best_F == ref_F
    np.testing.assert_array_equal(best_a, ref_best.cpu().numpy())
    np.testing.assert_array_equal(fit, f)
    assert best_F == K().host_f(best_a)


def test_polish_never_reports_worse(cuda, certs):
    w, meta = certs[512]
    F0 = K().host_f(w)
    best_a, best_F, _ = K().polish(w, K=4, iters=24, passes=6, seed=1)
    assert best_F <= F0
    assert best_F == K().host_f(best_a)
    assert (best_a >= 0).all()

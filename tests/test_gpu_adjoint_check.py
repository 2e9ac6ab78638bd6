"""The adjoint check at its configured size: n = 4096, B = 64 plain-method
candidates, p in {8, 64, 512}; the fp32 and BF16x3 forward / adjoint pair
against the long-double oracle gradient on sampled candidates, against fp64
central differences (step 1e-6 max a) on 32 random coordinates, and the
recompute-b backward against the stored-b backward (equal results; memory
and time printed with -s).  Needs a B200.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

N, B = 4096, 64


def _timed(fn, reps=5):
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    fn()
    s.record()
    for _ in range(reps):
        fn()
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e) / reps


@pytest.mark.parametrize("p", [8.0, 64.0, 512.0])
def test_adjoint_config(cuda, orc, p):
    from sidon_b200 import kernels as K, synth
    pop = synth.population("structured", N, B, seed=1)
    a = torch.as_tensor(pop, device=cuda)
    rng = np.random.default_rng(int(p))
    sample = rng.choice(B, 3, replace=False)
    for prec, tol in (("fp32", 1e-4 * p), ("bf16x3", max(2e-3, 2e-5 * p))):
        val, saved, _ = K.lp_forward(a, p, precision=prec)
        g = K.lp_backward(a, saved, p, precision=prec).cpu().numpy()
        for r in sample:
            ref_g, ref_v = orc.lp_grad(pop[r].astype(np.float64), p)
            assert abs(val[r].item() - ref_v) <= 1e-4 * ref_v
            assert np.max(np.abs(g[r] - ref_g)) / np.abs(ref_g).max() <= tol, (prec, r)
        # scale invariance of G_p: sum_i a_i dG/da_i = 0
        ad = (g.astype(np.float64) * pop.astype(np.float64)).sum(1)
        assert np.max(np.abs(ad)) <= 1e-3 * np.abs(g).max() * 1.0
    # central differences on 32 coordinates of one candidate (fp32 adjoint)
    r = int(sample[0])
    x = pop[r].astype(np.float64)
    _, saved, _ = K.lp_forward(a[r:r + 1].contiguous(), p)
    g = K.lp_backward(a[r:r + 1].contiguous(), saved, p).cpu().numpy()[0]
    h = 1e-6 * x.max()
    gmax = np.abs(g).max()
    for i in rng.choice(np.flatnonzero(x > 2 * h), 32, replace=False):
        e = np.zeros(N)
        e[i] = h
        fd = (orc.lp_value(x + e, p) - orc.lp_value(x - e, p)) / (2 * h)
        assert abs(fd - g[i]) <= 5e-3 * gmax


def test_recompute_vs_stored_b(cuda):
    from sidon_b200 import kernels as K, synth
    a = torch.as_tensor(synth.population("structured", N, B, seed=2), device=cuda)
    p = 64.0
    for prec in ("fp32", "bf16x3"):
        _, saved, b = K.lp_forward(a, p, store_b=True, precision=prec)
        g1 = K.lp_backward(a, saved, p, precision=prec)
        g2 = K.lp_backward(a, saved, p, b=b, precision=prec)
        assert torch.equal(g1, g2)
        t_re = _timed(lambda: K.lp_backward(a, saved, p, precision=prec))
        t_st = _timed(lambda: K.lp_backward(a, saved, p, b=b, precision=prec))
        print(f"\n{prec}: backward with b recomputed {t_re:.3f} ms (no per-candidate b "
              f"stored), with stored b {t_st:.3f} ms ({b.numel() * 4 / 1e6:.1f} MB of b)")

"""Tensor-core (tcgen05 BF16x3 / BF16x1) path vs the oracle.  Needs a B200.

Tolerances (relative to max b or max |grad|), from the split arithmetic:
BF16x3 represents each height to ~2^-17 and drops lo*lo (~2^-18), with fp32
accumulation -> b within 3e-5 of max b; BF16x1 keeps 8 bits -> 1e-2.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def K():
    from sidon_b200 import kernels
    return kernels


def T(x, dev, dtype=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(x), dtype=dtype, device=dev)


def _status():
    import sidon_b200
    return sidon_b200.load().sidon_device_status(1)


@pytest.mark.parametrize("n", [1, 100, 128, 129, 300, 1000, 4096, 8400])
def test_tc_conv_bf16x3_vs_fp64(cuda, n):
    rng = np.random.default_rng(n)
    a = rng.lognormal(0, 1, (2, n)).astype(np.float32)
    a[:, rng.uniform(size=n) < 1 / 3] = 0
    a[:, 0] = 8 * a.mean() + 1.0          # endpoint atom (never an all-zero row)
    _, saved, b = K().lp_forward(T(a, cuda), 8.0, store_b=True, precision="bf16x3")
    b = b.cpu().numpy().astype(np.float64)
    assert _status() == 0
    for p in range(2):
        ref = np.convolve(a[p].astype(np.float64), a[p].astype(np.float64))
        err = np.max(np.abs(b[p] - ref)) / ref.max()
        assert err <= 3e-5, (n, err)
        assert abs(saved[p, 0].item() - ref.max()) <= 3e-5 * ref.max()


def test_tc_conv_bf16x1_tolerance(cuda):
    rng = np.random.default_rng(0)
    a = rng.uniform(0, 1, (1, 700)).astype(np.float32)
    _, _, b = K().lp_forward(T(a, cuda), 8.0, store_b=True, precision="bf16x1")
    ref = np.convolve(a[0].astype(np.float64), a[0].astype(np.float64))
    err = np.max(np.abs(b.cpu().numpy()[0] - ref)) / ref.max()
    assert err <= 1e-2
    assert _status() == 0


@pytest.mark.parametrize("n,p", [(300, 8.0), (1000, 64.0), (4096, 64.0), (4096, 512.0)])
def test_tc_gradient_vs_long_double(cuda, orc, n, p):
    """BF16x3 adjoint vs the long-double oracle gradient; the weights
    (b/M)^(p-1) amplify the split error by p-1, so the bound is
    max(2e-3, 2e-5 p) of max|grad|."""
    from sidon_b200 import synth
    pop = synth.population("structured", n, 2, seed=n)
    a = T(pop, cuda)
    val, saved, _ = K().lp_forward(a, p, precision="bf16x3")
    g = K().lp_backward(a, saved, p, precision="bf16x3").cpu().numpy()
    assert _status() == 0
    tol = max(2e-3, 2e-5 * p)
    for r in range(2):
        ref_g, ref_v = orc.lp_grad(pop[r].astype(np.float64), p)
        assert abs(val[r].item() - ref_v) <= 1e-4 * ref_v
        err = np.max(np.abs(g[r] - ref_g)) / np.abs(ref_g).max()
        assert err <= tol, (n, p, err)


def test_tc_backward_stored_b_matches_recompute(cuda):
    from sidon_b200 import synth
    a = T(synth.population("structured", 2048, 3, seed=5), cuda)
    _, saved, b = K().lp_forward(a, 64.0, store_b=True, precision="bf16x3")
    g1 = K().lp_backward(a, saved, 64.0, precision="bf16x3")
    g2 = K().lp_backward(a, saved, 64.0, b=b, precision="bf16x3")
    assert torch.equal(g1, g2)


def test_tc_local_search_selftest(cuda, kat, orc):
    """src/main.cu:258-288 with the tensor-core step: F decreases, heights
    stay >= 0 and finite, and the run is bitwise reproducible."""
    case = kat["ls128"]
    start = np.asarray(case["a"], dtype=np.float32)
    x1, x2 = T(start, cuda), T(start, cuda)
    for x in (x1, x2):
        K().run_local_search(x, 800, 4.0, 300.0, 0.06, 0.002, precision="bf16x3")
    assert _status() == 0
    assert torch.equal(x1, x2)
    h = x1.cpu().numpy()
    assert np.all(h >= 0) and np.all(np.isfinite(h))
    F1, _ = K().run_eval(x1)
    for p in range(4):
        assert F1[p].item() < case["F"][p]


def test_tc_local_search_tracks_fp32(cuda, orc):
    """A short anneal at n=1000 with BF16x3 and with FP32 SIMT from the same
    start: certified F agree to 1e-3 relative (different rounding, same
    dynamics)."""
    from sidon_b200 import synth
    pop = synth.population("structured", 1000, 4, seed=77)
    xt, xs = T(pop, cuda), T(pop, cuda)
    K().run_local_search(xt, 30, 4.0, 64.0, 0.01, 0.004, precision="bf16x3")
    K().run_local_search(xs, 30, 4.0, 64.0, 0.01, 0.004, precision="fp32")
    assert _status() == 0
    Ft, _ = K().run_eval(xt)
    Fs, _ = K().run_eval(xs)
    F0, _ = K().run_eval(T(pop, cuda))
    for p in range(4):
        assert Ft[p].item() < F0[p].item()
        assert abs(Ft[p].item() - Fs[p].item()) <= 1e-3 * Fs[p].item()


def test_tc_local_search_skip_modes_and_full_size(cuda):
    from sidon_b200 import synth
    pop = synth.population("lognormal", 8400, 3, seed=3)
    x = T(pop, cuda)
    skip = T(np.array([0, 1, 0], dtype=np.int32), cuda, torch.int32)
    mode = T(np.array([0, 0, 1], dtype=np.int32), cuda, torch.int32)
    K().run_local_search(x, 5, 2.0, 16.0, 1e-3, 1e-3, skip=skip, mode_arr=mode,
                         precision="bf16x3")
    assert _status() == 0
    assert torch.equal(x[1], T(pop[1], cuda))
    h = x.cpu().numpy()
    assert np.all(h >= 0) and np.all(np.isfinite(h))
    assert np.all(h[2] > 0) == np.all(pop[2] > 0)      # mirror steps keep zeros zero
    assert abs(h[0].sum() - 1) < 1e-4 and abs(h[2].sum() - 1) < 1e-4


@pytest.mark.parametrize("n,rounds,pdhg,steps", [(200, 2, 100, "reference"),
                                                 (1000, 1, 200, "unit"),
                                                 (4096, 1, 200, "unit")])
def test_frank_wolfe_tc_tracks_oracle(cuda, orc, n, rounds, pdhg, steps):
    """Chambolle-Pock Frank-Wolfe with BF16x3 convolutions vs the fp32 oracle:
    F never increases (moves are accepted on fp64-refined maxima), and F after
    the step is within 2e-3 relative of the oracle's (the PDHG iterates round
    differently; the line search may settle on a neighbouring t)."""
    from sidon_b200 import synth
    pop = synth.population("structured", n, 3, seed=37 + n)
    x = T(pop, cuda)
    tau, sig = (0.0, 0.0) if steps == "reference" else (0.9, 0.9)
    K().run_frank_wolfe_tc(x, rounds, pdhg, tau=tau, sigma=sig)
    assert _status() == 0
    tc_ = orc.frank_wolfe(pop, rounds, pdhg) if steps == "reference" else None
    got = x.cpu().numpy()
    assert (got >= 0).all()
    for p in range(3):
        F0 = orc.host_f(pop[p].astype(np.float64))
        Fg = orc.host_f(got[p].astype(np.float64))
        assert Fg <= F0 * (1 + 1e-9), (p, F0, Fg)
        if tc_ is not None:
            Fw = orc.host_f(tc_[p].astype(np.float64))
            assert abs(Fg - Fw) <= 2e-3 * Fw, (p, Fg, Fw)
        assert abs(got[p].astype(np.float64).sum() - 1.0) < 1e-5


def test_frank_wolfe_tc_improves_like_simt(cuda):
    """At the batched-island step sizes (tau = sigma = 0.9 on normalised
    heights) the tensor-core step lowers F about as much as the fp32 step."""
    from sidon_b200 import synth
    pop = synth.population("structured", 2048, 4, seed=41)
    a = T(pop, cuda)
    b = T(pop, cuda)
    K().run_frank_wolfe_tc(a, 1, 200, tau=0.9, sigma=0.9)
    assert K().run_frank_wolfe(b, 1, 200, tau=0.9, sigma=0.9)
    Fa, _ = K().run_eval(a, with_nactive=False)
    Fb, _ = K().run_eval(b, with_nactive=False)
    F0, _ = K().run_eval(T(pop, cuda), with_nactive=False)
    gain_a = (F0 - Fa).cpu().numpy()
    gain_b = (F0 - Fb).cpu().numpy()
    assert (gain_a >= 0).all()
    assert gain_a.sum() >= 0.8 * gain_b.sum(), (gain_a, gain_b)


def test_tc_largest_n(cuda):
    """The top of the single-CTA ranges.  n = 9728 (152 blocks, 512 TMEM
    columns, all shared memory) runs every tensor-core kernel; the fused
    local search, whose window ring shares its region with the scratch,
    reaches n = 9984 (26 cells per thread, 512 TMEM columns); one cell more
    is refused with SIDON_ERR_N, and the size query agrees."""
    from sidon_b200 import synth, _lib
    n = 9728
    a = T(synth.population("structured", n, 2, seed=97), cuda)
    _, saved, b = K().lp_forward(a, 8.0, store_b=True, precision="bf16x3")
    ref = np.convolve(a[0].double().cpu().numpy(), a[0].double().cpu().numpy())
    assert np.max(np.abs(b[0].cpu().numpy() - ref)) <= 3e-5 * ref.max()
    x = a.clone()
    K().run_local_search(x, 2, 2.0, 4.0, 1e-3, 1e-3, precision="bf16x3")
    y = a.clone()
    K().run_frank_wolfe_tc(y, 1, 3, 3, 0.3, tau=0.9, sigma=0.9)
    F0, _ = K().run_eval(a, with_nactive=False)
    F1, _ = K().run_eval(y, with_nactive=False)
    assert bool((F1 <= F0 * (1 + 1e-9)).all())
    assert _status() == 0
    top = 9984
    pop = synth.population("structured", top, 2, seed=98)
    z = T(pop, cuda)
    K().run_local_search(z, 6, 2.0, 16.0, 1e-3, 1e-3, precision="bf16x3")
    assert _status() == 0
    Fz, _ = K().run_eval(z, with_nactive=False)
    Fp, _ = K().run_eval(T(pop, cuda), with_nactive=False)
    assert bool((Fz < Fp).all())
    assert bool((z >= 0).all())
    big = torch.full((1, top + 1), 1.0 / (top + 1), device=cuda)
    with pytest.raises(_lib.SidonError) as ei:
        K().run_local_search(big, 1, 2.0, 4.0, 1e-3, 1e-3, precision="bf16x3")
    assert ei.value.status == _lib.ERR_N
    assert K().max_n(_lib.OP_LOCAL_SEARCH_TC) == top


@pytest.mark.parametrize("iters", [1, 7, 30])
def test_balanced_segments_equal_one_wave(cuda, iters):
    """A uniform batch larger than the SM count runs the balanced-segment
    kernel (step chains split across CTAs); each candidate's result equals the
    one-wave kernel's
    (two halves of the batch, each within one wave) bit for bit, with skips,
    mirror-mode candidates and an all-zero candidate (M <= 0) in the batch."""
    from sidon_b200 import synth
    sms = torch.cuda.get_device_properties(cuda).multi_processor_count
    P = sms + 9
    n = 700
    pop = synth.population("lognormal", n, P, seed=iters)
    pop[5] = 0.0
    skip = torch.zeros(P, dtype=torch.int32, device=cuda)
    skip[[3, P - 1]] = 1
    mode = torch.zeros(P, dtype=torch.int32, device=cuda)
    mode[[2, 100]] = 1
    whole = T(pop, cuda)
    K().run_local_search(whole, iters, 2.0, 256.0, 1e-3, 5e-4, precision="bf16x3", skip=skip,
                         mode_arr=mode)
    assert _status() == 0
    h = P // 2
    for lo, hi in ((0, h), (h, P)):
        part = T(pop[lo:hi], cuda)
        K().run_local_search(part, iters, 2.0, 256.0, 1e-3, 5e-4, precision="bf16x3",
                             skip=skip[lo:hi].contiguous(), mode_arr=mode[lo:hi].contiguous())
        assert torch.equal(part, whole[lo:hi]), (lo, hi)
    np.testing.assert_array_equal(whole[5].cpu().numpy(), pop[5])
    np.testing.assert_array_equal(whole[3].cpu().numpy(), pop[3])


def test_nonfinite_heights_are_reported(cuda):
    """NaN, Inf or negative heights do not stop the kernels (or hang them):
    the device status word reports SIDON_ERR_NONFINITE; clean input leaves
    it at SIDON_OK."""
    from sidon_b200 import _lib
    assert _status() == 0
    base = np.full((2, 300), 1.0 / 300, dtype=np.float32)
    for bad in (np.nan, np.inf, -1e-3):
        x = base.copy()
        x[1, 17] = bad
        K().run_local_search(T(x, cuda), 2, 2.0, 4.0, 1e-3, 1e-3, precision="bf16x3")
        assert _status() == _lib.ERR_NONFINITE, bad
        K().lp_forward(T(x, cuda), 8.0, precision="bf16x3")
        assert _status() == _lib.ERR_NONFINITE, bad
    K().run_local_search(T(base, cuda), 2, 2.0, 4.0, 1e-3, 1e-3, precision="bf16x3")
    assert _status() == 0

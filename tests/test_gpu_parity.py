"""CUDA path vs the oracle, through the C ABI.  Needs a B200.

Bars: bit-exact where the arithmetic is specified bit for bit (hostF-order
fp64 evaluation, exact certification, fp32 convolution / correlation chains,
copies, ranking); stated tolerances elsewhere (written in each test).
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


# ------------------------------ certifying eval ----------------------------
@pytest.mark.parametrize("n", [512, 4096, 8400])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_eval_certificates_bitwise_hostF(cuda, certs, n, dtype):
    w, meta = certs[n]
    F, na = K().run_eval(T(w[None, :], cuda, dtype), active_tol=1e-9)
    assert F.item() == meta["ref_hostF"]          # bit for bit
    assert na.item() == meta["probe_verify"]["nactive"]


def test_eval_selftest_kat_257(cuda, kat, orc):
    # src/main.cu:228-256 (reference tolerance 1e-13; here bit for bit)
    pop = np.asarray([c["a"] for c in kat["eval257"]], dtype=np.float32)
    F, na = K().run_eval(T(pop, cuda), active_tol=1e-9)
    Fo, nao = orc.eval_pop(pop.astype(np.float64), tol=1e-9)
    for p, c in enumerate(kat["eval257"]):
        assert F[p].item() == c["F"]
    assert np.array_equal(na.cpu().numpy(), nao)


def test_eval_population_and_degenerate(cuda, orc):
    from sidon_b200 import synth
    pop = synth.population("structured", 1000, 7, seed=5)
    pop[3] = 0.0
    F, na = K().run_eval(T(pop, cuda), active_tol=1e-4)
    Fo, nao = orc.eval_pop(pop.astype(np.float64), tol=1e-4)
    assert np.array_equal(F.cpu().numpy(), Fo)
    assert np.array_equal(na.cpu().numpy(), nao)
    assert F[3].item() == 1e30


# ------------------------------ exact certify ------------------------------
@pytest.mark.parametrize("n", [512, 4096, 8400])
def test_certify_certificates(cuda, certs, orc, n):
    w, meta = certs[n]
    F, M, S, k = K().certify(T(w[None, :], cuda))
    assert abs(F.item() - meta["ref_hostF"]) <= 1e-12 * meta["ref_hostF"]
    assert k.item() == meta["probe_verify"]["kmax"]
    if n <= 4096:
        Fo, Mo, So, ko = orc.certify_exact(w)
        assert F.item() == Fo and M.item() == Mo and S.item() == So


@pytest.mark.parametrize("n,splits", [(512, 3), (4096, 2), (8400, 1)])
def test_certify_bit_exact_across_cell_splits(cuda, certs, n, splits):
    w, _ = certs[n]
    x = T(w[None, :], cuda)
    F0 = K().certify(x)[0].item()
    for _ in range(splits):
        x = K().refine(x)
        assert K().certify(x)[0].item() == F0


def test_certify_fp64_heights(cuda, orc):
    rng = np.random.default_rng(9)
    a = rng.uniform(0, 1, (3, 300))
    a[:, ::7] = 0
    F, M, S, k = K().certify(T(a, cuda, torch.float64))
    for p in range(3):
        Fo, Mo, So, ko = orc.certify_exact(a[p])
        assert F[p].item() == Fo and M[p].item() == Mo and S[p].item() == So and k[p].item() == ko


# ------------------------- convolution / gradient --------------------------
@pytest.mark.parametrize("n", [1, 2, 37, 512, 1000, 4096])
def test_conv_bitwise_oracle(cuda, orc, n):
    rng = np.random.default_rng(n)
    a = rng.uniform(0, 1, (2, n)).astype(np.float32)
    a[:, rng.uniform(size=n) < 0.3] = 0
    _, _, b = K().lp_forward(T(a, cuda), 8.0, store_b=True)
    b = b.cpu().numpy()
    for p in range(2):
        assert np.array_equal(b[p], orc.conv_f32(a[p], a[p]))


@pytest.mark.parametrize("p", [8.0, 64.0, 512.0])
def test_lp_forward_backward_vs_long_double(cuda, orc, p):
    """Adjoint check (n=4096, B=64 scaled down to B=8 here): fp32 G_p and its
    gradient vs the long-double oracle; rel. error bounds 1e-5 (value) and
    2e-3 of max|grad| (gradient, fp32 with (p-1)-amplified weights)."""
    from sidon_b200 import synth
    n, B = 4096, 8
    pop = synth.population("structured", n, B, seed=100)
    a = T(pop, cuda)
    val, saved, _ = K().lp_forward(a, p)
    g = K().lp_backward(a, saved, p).cpu().numpy()
    rng = np.random.default_rng(int(p))
    for r in range(2):
        ref_g, ref_v = orc.lp_grad(pop[r].astype(np.float64), p)
        assert abs(val[r].item() - ref_v) <= 1e-5 * ref_v
        idx = rng.choice(n, 32, replace=False)
        err = np.max(np.abs(g[r, idx] - ref_g[idx]))
        assert err <= 2e-3 * np.abs(ref_g).max(), (p, err)


def test_lp_backward_stored_b_equals_recompute(cuda):
    from sidon_b200 import synth
    a = T(synth.population("structured", 2048, 4, seed=3), cuda)
    _, saved, b = K().lp_forward(a, 64.0, store_b=True)
    g1 = K().lp_backward(a, saved, 64.0)
    g2 = K().lp_backward(a, saved, 64.0, b=b)
    assert torch.equal(g1, g2)


def test_lp_gradient_vs_central_differences(cuda, orc):
    """fp64 central differences (step 1e-6 max a) of the long-double G_p vs
    the fp32 adjoint on 32 random coordinates; tolerance 5e-3 of max|grad|."""
    from sidon_b200 import synth
    n = 512
    a = synth.population("structured", n, 1, seed=8)[0].astype(np.float64)
    p = 64.0
    _, saved, _ = K().lp_forward(T(a[None], cuda), p)
    g = K().lp_backward(T(a[None], cuda), saved, p).cpu().numpy()[0]
    h = 1e-6 * a.max()
    rng = np.random.default_rng(0)
    gmax = np.abs(g).max()
    for i in rng.choice(np.flatnonzero(a > 2 * h), 32, replace=False):
        e = np.zeros(n)
        e[i] = h
        fd = (orc.lp_value(a + e, p) - orc.lp_value(a - e, p)) / (2 * h)
        assert abs(fd - g[i]) <= 5e-3 * gmax


# -------------------------------- local search -----------------------------
def test_local_search_selftest(cuda, kat, orc):
    """src/main.cu:258-288: n=128, P=4, 800 steps p 4->300, lr 0.06->0.002:
    F strictly decreases, heights stay >= 0 and finite, and the certifying
    eval of the polished vector matches hostF within 1e-12."""
    case = kat["ls128"]
    pop = T(np.asarray(case["a"], dtype=np.float32), cuda)
    K().run_local_search(pop, 800, 4.0, 300.0, 0.06, 0.002)
    F1, _ = K().run_eval(pop)
    h = pop.cpu().numpy()
    assert np.all(h >= 0) and np.all(np.isfinite(h))
    for p in range(4):
        assert F1[p].item() < case["F"][p]
    assert abs(F1[0].item() - orc.host_f(h[0].astype(np.float64))) < 1e-12


def test_local_search_matches_oracle_f32(cuda, orc):
    """Same arithmetic as the oracle up to exp/log1p ulps and reduction order;
    F after 60 steps agrees to 1e-4 relative."""
    from sidon_b200 import synth
    pop = synth.population("structured", 256, 6, seed=21)
    mode = np.array([0, 0, 0, 1, 1, 0], dtype=np.int32)
    x = T(pop, cuda)
    K().run_local_search(x, 60, 4.0, 64.0, 0.02, 0.005, mode_arr=T(mode, cuda, torch.int32))
    got = x.cpu().numpy()
    want = orc.local_search(pop, 60, 4.0, 64.0, 0.02, 0.005, mode_arr=mode)
    for p in range(6):
        Fg, Fw = orc.host_f(got[p].astype(np.float64)), orc.host_f(want[p].astype(np.float64))
        assert abs(Fg - Fw) <= 1e-4 * Fw, (p, Fg, Fw)


def test_local_search_first_step_bitwise_conv_path(cuda, orc):
    """One step at p=2 with identical inputs: the conv is bit-identical, so the
    new heights agree to a few fp32 ulps (exp/log1p and reduction order)."""
    from sidon_b200 import synth
    pop = synth.population("lognormal", 300, 2, seed=4)
    x = T(pop, cuda)
    K().run_local_search(x, 1, 2.0, 2.0, 0.01, 0.01)
    want = orc.local_search(pop, 1, 2.0, 2.0, 0.01, 0.01)
    assert np.allclose(x.cpu().numpy(), want, rtol=2e-5, atol=1e-9)


def test_local_search_deterministic_and_skip(cuda):
    from sidon_b200 import synth
    pop = synth.population("structured", 777, 5, seed=2)
    skip = T(np.array([0, 1, 0, 0, 1], dtype=np.int32), cuda, torch.int32)
    x1, x2 = T(pop, cuda), T(pop, cuda)
    for x in (x1, x2):
        K().run_local_search(x, 40, 6.0, 400.0, 0.05, 0.002, skip=skip)
    assert torch.equal(x1, x2)                         # bitwise reproducible
    assert torch.equal(x1[1], T(pop[1], cuda)) and torch.equal(x1[4], T(pop[4], cuda))
    assert not torch.equal(x1[0], T(pop[0], cuda))


def test_local_search_fp64_matches_oracle(cuda, orc):
    from sidon_b200 import synth
    pop = synth.population("structured", 200, 3, seed=6, dtype=np.float64)
    x = T(pop, cuda, torch.float64)
    K().run_local_search(x, 50, 200.0, 6000.0, 0.01, 0.0002)
    want = orc.local_search(pop, 50, 200.0, 6000.0, 0.01, 0.0002)
    for p in range(3):
        Fg, Fw = orc.host_f(x[p].cpu().numpy()), orc.host_f(want[p])
        assert abs(Fg - Fw) <= 1e-9 * Fw


def test_local_search_uniform_reset_on_zero_sum(cuda):
    x = torch.zeros((1, 64), dtype=torch.float32, device=cuda)
    K().run_local_search(x, 3, 4.0, 8.0, 0.01, 0.01)     # M <= 0: loop breaks, a untouched
    assert torch.equal(x, torch.zeros_like(x))


# ------------------------------- Frank-Wolfe -------------------------------
def test_frank_wolfe_matches_oracle(cuda, orc):
    """Reference step sizes; F after 2 rounds of 100 PDHG iterations agrees
    with the oracle to 1e-4 relative and does not increase."""
    from sidon_b200 import synth
    pop = synth.population("structured", 200, 4, seed=31)
    x = T(pop, cuda)
    assert K().run_frank_wolfe(x, rounds=2, pdhg_iters=100)
    want = orc.frank_wolfe(pop, 2, 100)
    got = x.cpu().numpy()
    for p in range(4):
        F0 = orc.host_f(pop[p].astype(np.float64))
        Fg, Fw = orc.host_f(got[p].astype(np.float64)), orc.host_f(want[p].astype(np.float64))
        assert Fg <= F0 * (1 + 1e-6)
        assert abs(Fg - Fw) <= 1e-4 * Fw


def test_frank_wolfe_too_large_reports_false(cuda):
    from sidon_b200 import kernels
    n = kernels.max_n(2) + 1
    x = torch.full((1, n), 1.0 / n, device=cuda)
    assert kernels.run_frank_wolfe(x, 1, 1) is False


# ---------------------------- ladder and islands ---------------------------
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_refine_coarsen_exact(cuda, dtype):
    rng = np.random.default_rng(1)
    a = rng.uniform(0, 1, (5, 1001))
    x = T(a, cuda, dtype)
    r = K().refine(x)
    assert torch.equal(r[:, ::2], x) and torch.equal(r[:, 1::2], x)
    assert torch.equal(K().coarsen(r), x)


@pytest.mark.parametrize("m,n", [(64, 128), (1000, 1500), (1500, 1000), (7, 3), (5, 5)])
def test_resample_matches_oracle(cuda, orc, m, n):
    """Nearest-neighbour resample + fp64 renormalisation (main.cu:496-497,
    555-562) = the oracle bit for bit; without normalisation a 2x resample
    is the cell split."""
    rng = np.random.default_rng(m + n)
    pop = rng.uniform(0, 1, (6, m)).astype(np.float32)
    pop[2] = 0.0                                        # a zero row stays zero
    got = K().resample(T(pop, cuda), n).cpu().numpy()
    for p in range(6):
        want = orc.resample(pop[p], n)
        assert np.array_equal(got[p], want) or (p == 2 and not got[p].any())
    if n == 2 * m:
        raw = K().resample(T(pop, cuda), n, normalise=False)
        assert torch.equal(raw, K().refine(T(pop, cuda)))


def test_island_migrate_matches_oracle(cuda, orc):
    rng = np.random.default_rng(12)
    P, NI, n, k = 64, 8, 333, 2
    pop = rng.uniform(0, 1, (P, n)).astype(np.float32)
    fit = rng.uniform(1.5, 1.6, P)
    fit[5] = fit[6]                                     # a tie
    x, f = T(pop, cuda), T(fit, cuda, torch.float64)
    order = K().island_migrate(x, f, NI, k)
    po, fo, oo = orc.island_migrate(pop, fit, NI, k)
    assert np.array_equal(order.cpu().numpy(), oo)
    assert np.array_equal(x.cpu().numpy(), po)
    assert np.array_equal(f.cpu().numpy(), fo)


# ------------------------------- error paths -------------------------------
def test_errors_are_status_codes_not_exits(cuda):
    from sidon_b200 import kernels
    from sidon_b200._lib import SidonError
    x = torch.ones((2, 10), device=cuda)
    with pytest.raises(SidonError) as e:
        kernels.island_migrate(x, torch.ones(2, dtype=torch.float64, device=cuda), 3, 1)
    assert e.value.status == 1
    big = kernels.max_n(0) + 1
    y = torch.ones((1, big), device=cuda)
    with pytest.raises(SidonError) as e:
        kernels.run_local_search(y, 1, 2.0, 2.0, 0.01, 0.01)
    assert e.value.status == 3

"""The oracle (oracle/sidon_oracle.c) pinned against the reference's own
outputs: certificates, self-test known answers, probe --verify and the
probe's fp64 local search.  CPU only."""
import numpy as np
import pytest


# ---------------------------- hostF / verifier -----------------------------
@pytest.mark.parametrize("n", [512, 4096, 8400])
def test_hostF_matches_reference_bitwise(orc, certs, n):
    w, meta = certs[n]
    F = orc.host_f(w)
    assert F == meta["ref_hostF"]            # reference hostF, compiled from its sources
    assert F == meta["stored_F"]             # certificate JSON
    assert F == meta["ref_verify_py_F"]      # reference verify.py


@pytest.mark.parametrize("n", [512, 4096, 8400])
def test_verify_ld_matches_probe(orc, certs, n):
    w, meta = certs[n]
    pv = meta["probe_verify"]
    r = orc.verify_ld(w)
    # probe prints 20 significant digits of the long double values
    for key in ("F", "S", "M"):
        want = float(pv[key])
        assert abs(r[key] - want) <= 1e-18 * abs(want), key
    assert r["kmax"] == pv["kmax"]
    assert r["nactive"] == pv["nactive"]
    assert f"{r['relbound']:.3g}" == pv["relbound"]
    assert not r["negative"]
    assert abs(r["F"] - meta["stored_F"]) <= 1e-12


def test_selftest_hand_values(orc, kat):
    # src/main.cu:196-207
    for case in kat["hand"]:
        F = orc.host_f(case["a"])
        assert F == case["F"]
        assert abs(F - case["want"]) <= 1e-12 * max(1.0, abs(case["want"]))


def test_selftest_refine_and_scale_invariance(orc, kat):
    # src/main.cu:209-226
    for case in kat["refine"]:
        a = np.asarray(case["a"])
        assert orc.host_f(a) == case["F"]
        assert orc.host_f(np.repeat(a, 2)) == case["F_refined"]
        assert abs(case["F_refined"] - case["F"]) <= 1e-12
    s = kat["scale"]
    assert orc.host_f(s["a"]) == s["F"]
    assert abs(s["F_scaled"] - s["F"]) <= 1e-12


def test_eval_population_equals_hostF(orc, kat):
    pop = np.asarray([c["a"] for c in kat["eval257"]])
    F, na = orc.eval_pop(pop, tol=1e-9)
    for p, c in enumerate(kat["eval257"]):
        assert F[p] == c["F"]
    assert F[0] == 2.0 and na[0] >= 1


def test_eval_degenerate_sum_sentinel(orc):
    F, _ = orc.eval_pop(np.zeros((1, 16)))
    assert F[0] == 1e30      # src/kernels.cuh:376


# ------------------------------ exact certify ------------------------------
@pytest.mark.parametrize("n", [512, 4096])
def test_certify_exact_close_to_hostF_and_split_invariant(orc, certs, n):
    w, meta = certs[n]
    F, M, S, k = orc.certify_exact(w)
    assert abs(F - meta["ref_hostF"]) <= 1e-12 * F
    assert k == meta["probe_verify"]["kmax"]
    F2, M2, S2, k2 = orc.certify_exact(np.repeat(w, 2))
    assert F2 == F                           # bit for bit across the cell split
    assert M2 == 2 * M and S2 == 2 * S


def test_certify_exact_random_split_chain(orc):
    rng = np.random.default_rng(7)
    a = rng.uniform(0, 1, 37).astype(np.float32).astype(np.float64)
    a[rng.uniform(size=37) < 0.3] = 0
    F0 = orc.certify_exact(a)[0]
    for _ in range(3):
        a = np.repeat(a, 2)
        assert orc.certify_exact(a)[0] == F0


def test_exact_bk_matches_long_double(orc):
    rng = np.random.default_rng(3)
    a = rng.uniform(0, 1, 64)
    for k in (0, 17, 63, 100, 126):
        ilo, ihi = max(0, k - 63), min(k, 63)
        want = sum(np.longdouble(a[i]) * np.longdouble(a[k - i]) for i in range(ilo, ihi + 1))
        assert abs(orc.exact_bk(a, k) - float(want)) <= 2e-16 * float(want)


# ------------------------------- local search ------------------------------
def test_f64_local_search_tracks_reference_probe(orc, probe_ls):
    """Oracle fp64 L^p-Adam vs the reference CPU twin (tools/probe.cpp:62-116).
    Arithmetic differs at the ulp level (fma use), so trajectories are
    compared through F and the heights at a loose tolerance."""
    for s, start, end in probe_ls:
        got = orc.local_search(start[None, :], s["iters"], s["pA"], s["pB"], s["lrA"], s["lrB"],
                               mode_default=s["mode"])[0]
        Fg = orc.host_f(got)
        assert abs(Fg - s["F"]) <= 1e-6 * s["F"], (s, Fg)
        assert np.max(np.abs(got - end)) <= 1e-4 * np.max(end)


def test_f32_local_search_selftest_improves(orc, kat):
    # src/main.cu:258-288 on the oracle
    case = kat["ls128"]
    pop = np.asarray(case["a"], dtype=np.float32)
    out = orc.local_search(pop, 200, 4.0, 300.0, 0.06, 0.002)
    for p in range(4):
        assert orc.host_f(out[p].astype(np.float64)) < case["F"][p]
    assert np.all(out >= 0) and np.all(np.isfinite(out))


def test_local_search_skip_and_modes(orc):
    rng = np.random.default_rng(1)
    pop = rng.uniform(0.1, 1, (3, 40)).astype(np.float32)
    out = orc.local_search(pop, 20, 4.0, 50.0, 0.05, 0.01, skip=[0, 1, 0], mode_arr=[0, 0, 1])
    assert np.array_equal(out[1], pop[1])
    assert not np.array_equal(out[0], pop[0]) and not np.array_equal(out[2], pop[2])
    assert np.all(out[2] > 0)                # mirror descent keeps support


# ------------------------------ conv / gradient ----------------------------
def test_conv_corr_f32_against_numpy(orc):
    rng = np.random.default_rng(2)
    a = rng.uniform(0, 1, 50).astype(np.float32)
    b = orc.conv_f32(a, a)
    assert np.allclose(b, np.convolve(a.astype(np.float64), a.astype(np.float64)), rtol=1e-5)
    c = rng.uniform(0, 1, 99).astype(np.float32)
    G = orc.corr_f32(a, c)
    want = np.array([np.dot(c[i:i + 50].astype(np.float64), a) for i in range(50)])
    assert np.allclose(G, want, rtol=1e-5)


@pytest.mark.parametrize("p", [8.0, 64.0])
def test_lp_gradient_oracle_vs_finite_differences(orc, p):
    rng = np.random.default_rng(5)
    a = rng.uniform(0.2, 1, 48)
    g, v = orc.lp_grad(a, p)
    assert abs(v - orc.lp_value(a, p)) <= 1e-14 * v
    h = 1e-6 * a.max()
    for i in (0, 7, 23, 47):
        e = np.zeros_like(a)
        e[i] = h
        fd = (orc.lp_value(a + e, p) - orc.lp_value(a - e, p)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * max(1e-3, np.abs(g).max())
    assert abs(np.dot(a, g)) <= 1e-9 * np.abs(g).max() * a.sum()   # scale invariance


# ------------------------------ FW / ladder / islands ----------------------
def test_frank_wolfe_does_not_increase_F(orc):
    from sidon_b200 import synth
    pop = synth.population("structured", 64, 2, seed=11)
    F0 = [orc.host_f(r.astype(np.float64)) for r in pop]
    out = orc.frank_wolfe(pop, rounds=2, pdhg=100)
    F1 = [orc.host_f(r.astype(np.float64)) for r in out]
    assert all(f1 <= f0 * (1 + 1e-6) for f0, f1 in zip(F0, F1))


def test_refine_coarsen_roundtrip(orc):
    rng = np.random.default_rng(4)
    pop = rng.uniform(0, 1, (3, 21))
    r = orc.refine(pop)
    assert np.array_equal(r[:, ::2], pop) and np.array_equal(r[:, 1::2], pop)
    assert np.array_equal(orc.coarsen(r), pop)


def test_island_migrate_semantics(orc):
    P, NI, n = 12, 3, 5
    pop = np.arange(P * n, dtype=np.float32).reshape(P, n)
    fit = np.array([5, 1, 3, 2, 9, 8, 7, 6, 0.5, 4, 4, 10.0])
    out, f2, order = orc.island_migrate(pop, fit, NI, 1)
    # island 0 = slots 0..3 ranked by fit: 1(1) 3(2) 2(3) 0(5)
    assert list(order[:4]) == [1, 3, 2, 0]
    assert list(order[4:8]) == [7, 6, 5, 4]
    assert list(order[8:]) == [8, 9, 10, 11]     # tie 4,4 broken by slot index
    # best of island i -> worst of island i+1
    assert np.array_equal(out[4], pop[1]) and f2[4] == fit[1]
    assert np.array_equal(out[11], pop[7]) and f2[11] == fit[7]
    assert np.array_equal(out[0], pop[8]) and f2[0] == fit[8]


def test_oracle_resample_restates_injection(orc):
    """so_resample_f32 against a direct restatement of src/main.cu:555-562
    (dst_i = src[min(m-1, i m / n)], S = sum in fp64, dst_i = fl32(x_i / S))."""
    rng = np.random.default_rng(3)
    for m, n in [(3, 7), (7, 3), (100, 100), (512, 8400), (8400, 512), (1, 9)]:
        src = rng.uniform(0, 1, m).astype(np.float32)
        xs = [float(src[min(m - 1, i * m // n)]) for i in range(n)]
        S = 0.0
        for x in xs:
            S += x
        want = np.array([np.float32(x / S) for x in xs], dtype=np.float32)
        np.testing.assert_array_equal(orc.resample(src, n), want)


def test_oracle_ragged_migration_rules(orc):
    sizes = [4, 4, 6, 6, 4, 6, 4, 4]
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    flat = np.arange(off[-1], dtype=np.float32) + 1
    fit = np.array([1.0, np.nan, 3.0, 0.5, 2.0, 0.1, 0.2, 0.3])
    out, f2, order = orc.island_migrate_ragged(flat, off, fit, 2, 1)
    # island 0 = slots 0..3 ranked 3, 0, 2, 1 (NaN last); island 1 = 5, 6, 7, 4
    assert order.tolist() == [3, 0, 2, 1, 5, 6, 7, 4]
    # best of island 0 (slot 3, n=6) -> worst of island 1 (slot 4, n=4): resampled
    np.testing.assert_array_equal(out[off[4]:off[5]], orc.resample(flat[off[3]:off[4]], 4))
    assert np.isnan(f2[4])
    # best of island 1 (slot 5, n=6) -> worst of island 0 (slot 1, n=4): resampled
    np.testing.assert_array_equal(out[off[1]:off[2]], orc.resample(flat[off[5]:off[6]], 4))
    # untouched rows keep their values and fitness
    np.testing.assert_array_equal(out[off[0]:off[1]], flat[off[0]:off[1]])
    assert f2[0] == 1.0 and f2[5] == 0.1


def test_oracle_philox_known_answers(orc):
    """Philox4x32-10 against its authors' known-answer vectors (Random123)."""
    cases = [
        ([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
        ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
        ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
         [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
    ]
    for ctr, key, want in cases:
        assert orc.philox4x32(ctr, key).tolist() == want


def test_oracle_variation_semantics(orc):
    """Operator meanings on the oracle: clone copies, reflect reverses (or
    symmetrises), segment/splice take cells from the right parent, every
    offspring sums to 1 and is non-negative."""
    rng = np.random.default_rng(4)
    pop = rng.uniform(0, 1, (3, 50)).astype(np.float32)
    ops = list(range(14)) + [20]
    J = len(ops)
    out = orc.variation(pop, [0] * J, [1] * J, ops, [0.2] * J, seed=7, gen=3)
    assert (out >= 0).all()
    np.testing.assert_allclose(out.sum(1), 1.0, rtol=1e-5)
    clone = out[ops.index(20)]
    np.testing.assert_allclose(clone, pop[0] / pop[0].sum(dtype=np.float64), rtol=1e-6)
    refl = out[6]
    hard = np.allclose(refl, (pop[0][::-1] / pop[0].sum()), rtol=1e-5)
    soft = np.allclose(refl, 0.5 * (pop[0] + pop[0][::-1]) / pop[0].sum(), rtol=1e-5)
    assert hard or soft
    for k in (1, 8):                       # each cell from one parent, then one common scale
        ok = False
        for c in (out[k][0] / pop[0][0], out[k][0] / pop[1][0]):
            from_a = np.isclose(out[k], c * pop[0], rtol=1e-5)
            from_b = np.isclose(out[k], c * pop[1], rtol=1e-5)
            ok = ok or bool(np.all(from_a | from_b))
        assert ok, k
    sig, nnz = orc.support_sig(np.array([[0, 1, 0, 2, 0, 3]], np.float32), tol=0.02)
    assert nnz[0] == 3 and sig[0] != 0
    sig2, _ = orc.support_sig(np.array([[0, 5, 0, 1, 0, 9]], np.float32), tol=0.02)
    assert sig2[0] == sig[0]                # same support, same signature

"""The memetic generation loop on the device (sidon_generation_*) against the
same generation composed on the host the way the reference driver composes
it (src/main.cu:586-785): the public device calls for the three local-search
tiers, Frank-Wolfe, the fp64 evaluation, the support signatures and the
variation, with the selection policy of the oracle (so_gen_*) in between.
After every generation the population, every plan array, the tabu table and
the whole state must agree bit for bit.  Needs a B200.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

SEED = 20260905


def K():
    from sidon_b200 import kernels
    return kernels


def L():
    from sidon_b200 import _lib
    return _lib


def seeds(n, P, rng):
    """Normalised synthetic heights: lognormal cells, a third zeroed, an
    endpoint atom on every other row."""
    a = rng.lognormal(0.0, 1.0, (P, n))
    a[rng.uniform(size=(P, n)) < 1 / 3] = 0.0
    a[::2, 0] += 4.0 * a[::2].mean(axis=1)
    a /= a.sum(axis=1, keepdims=True)
    return a.astype(np.float32)


def seed_ops(P, rng):
    """Operator record of the seeds: fresh restarts, structured seeds,
    carried-over rows and a few structural operators, so every tier fills."""
    return rng.choice([9, 11, 20, 20, 5, 0, 12], size=P).astype(np.int32)


def poke_state(G, pol, **kw):
    """Set state fields on the device and in the oracle alike."""
    s = L().GenerationState()
    L().call("sidon_generation_read_state", G._h, C.byref(s), None)
    for k, v in kw.items():
        setattr(s, k, v)
        setattr(pol.s, k, v)
    raw = torch.frombuffer(bytearray(bytes(s)), dtype=torch.uint8)
    off = G._views.state - G.workspace.data_ptr()
    G.workspace[off:off + raw.numel()].copy_(raw)


class HostComposition:
    """One generation as the reference driver composes it, with the oracle's
    policy and the library's public device calls."""

    def __init__(self, orc, cfg, n, P, pop0, seed_op, level, cuda):
        self.cfg, self.n, self.P, self.dev = cfg, n, P, cuda
        self.pol = orc.GenerationPolicy(P, cfg.n_islands, cfg.elite, cfg.tabu_tenure, cfg.seed, n)
        self.pol.begin_level(n, level, seed_op)
        self.pop = torch.tensor(pop0, device=cuda)
        self.mom = torch.empty_like(self.pop)
        self.vel = torch.empty_like(self.pop)
        self.mode = torch.tensor(self.pol.mode, device=cuda)
        self.prec = {0: "fp32", 1: "bf16x1", 2: "bf16x3"}[cfg.precision]
        self.fw_prec = {0: "fp32", 1: "bf16x1", 2: "bf16x3"}[cfg.fw_precision]

    def step(self):
        K_, c, pol = K(), self.cfg, self.pol
        cold, med, warm = c.cold_iters, c.cold_iters // 3, c.ls_iters
        skip = pol.tiers(cold, med, warm)
        p_top = np.float32(c.p_max)
        sched = [(cold, 6.0, p_top, 0.085, 0.0015), (med, 40.0, p_top, 0.04, 0.001),
                 (warm, 400.0, np.float32(p_top * np.float32(3.0)), 0.012, 0.0003)]
        for t, (it, pa, pb, la, lb) in enumerate(sched):
            if it > 0:
                K_.run_local_search(self.pop, it, float(np.float32(pa)), float(pb),
                                    float(np.float32(la)), float(np.float32(lb)),
                                    mode_arr=self.mode,
                                    skip=torch.tensor(skip[t], device=self.dev),
                                    mom=self.mom, vel=self.vel, beta1=float(np.float32(0.9)),
                                    beta2=float(np.float32(0.999)), precision=self.prec)
        fw_ran = 0
        if c.fw_rounds > 0:
            if self.fw_prec == "fp32":
                fw_ran = int(K_.run_frank_wolfe(self.pop, c.fw_rounds, c.fw_iters, c.fw_nT,
                                                c.fw_t_max))
            else:
                K_.run_frank_wolfe_tc(self.pop, c.fw_rounds, c.fw_iters, c.fw_nT, c.fw_t_max,
                                      precision=self.fw_prec, g_scratch=self.mom,
                                      gbar_scratch=self.vel)
                fw_ran = 1
        fit, nact = K_.run_eval(self.pop, 1e-4)
        sig, nnz = K_.support_sig(self.pop, 0.02)
        host = self.pop.cpu().numpy()
        self.sig = sig.cpu().numpy().view(np.uint64).copy()
        self.fit = fit.cpu().numpy()
        plan = pol.select(host, self.fit, nact.cpu().numpy(), self.sig, nnz.cpu().numpy(),
                          fw_ran, c.fw_rounds, c.fw_iters)
        self.pop.copy_(torch.from_numpy(host))
        nxt = K_.variation(self.pop, plan["p1"], plan["p2"], plan["op"], plan["strength"],
                           c.seed, int(pol.var_gen[0]))
        host = nxt.cpu().numpy()
        pol.post(host)
        self.pop.copy_(torch.from_numpy(host))
        child, _ = K_.run_eval(self.pop, 1e-4)
        self.child = child.cpu().numpy()
        pol.credit(self.child)


def device_tabu(G):
    v = G.views()
    key = v["tabu_key"].cpu().numpy().view(np.uint64)
    used = v["tabu_used"].cpu().numpy()
    best = v["tabu_best"].cpu().numpy()
    hits = v["tabu_hits"].cpu().numpy()
    return {int(key[i]): (float(best[i]), int(hits[i])) for i in np.nonzero(used)[0]}


def check_same(G, pop_dev, hc, where):
    torch.cuda.synchronize()
    got_pop = pop_dev.cpu().numpy()
    want_pop = hc.pop.cpu().numpy()
    assert np.array_equal(got_pop.view(np.uint32), want_pop.view(np.uint32)), f"{where}: pop"
    st = G.state()
    want = hc.pol.s.as_dict()
    for k, w in want.items():
        assert st[k] == w, f"{where}: state.{k} {st[k]} != {w}"
    v = G.views()
    pl = hc.pol.plan
    for k in ("parent_fit", "rank", "p1", "p2", "op", "strength"):
        got = v[k].cpu().numpy()
        assert np.array_equal(got.view(np.uint8), pl[k].view(np.uint8)), f"{where}: {k}"
    assert np.array_equal(v["fit"].cpu().numpy(), hc.fit), f"{where}: fit"
    assert np.array_equal(v["child_fit"].cpu().numpy(), hc.child), f"{where}: child_fit"
    assert np.array_equal(v["sig"].cpu().numpy().view(np.uint64), hc.sig), f"{where}: sig"
    assert np.array_equal(v["cur_op"].cpu().numpy(), hc.pol.cur_op), f"{where}: cur_op"
    assert device_tabu(G) == hc.pol.tabu(), f"{where}: tabu table"


def make(cuda, orc, n, P, NI, rng, **kw):
    args = dict(n_islands=NI, elite=2, ls_iters=8, cold_iters=12, p_max=300.0,
                precision="fp32", fw_rounds=1, fw_iters=10, fw_nT=4, fw_t_max=0.3,
                fw_precision="fp32", tabu_tenure=6, tabu_capacity=1 << 12, seed=SEED)
    args.update(kw)
    cfg = K().generation_config(**args)
    pop0 = seeds(n, P, rng)
    so = seed_ops(P, rng)
    G = K().Generation(n, P, cfg)
    G.begin_level(n, 0, torch.tensor(so, device=cuda))
    pop = torch.tensor(pop0, device=cuda)
    hc = HostComposition(orc, cfg, n, P, pop0, so, 0, cuda)
    return G, pop, hc


@pytest.mark.parametrize("n,P,NI,gens,prec", [
    (96, 64, 4, 26, "fp32"),       # migration at 12, 24; reinjection at 9, 19; credit every 5
    (200, 32, 4, 13, "bf16x3"),    # tensor-core local search (mirror island 3) and Frank-Wolfe
])
def test_generation_matches_host_composition(cuda, orc, n, P, NI, gens, prec):
    rng = np.random.default_rng(n + P)
    G, pop, hc = make(cuda, orc, n, P, NI, rng, precision=prec, fw_precision=prec)
    for g in range(gens):
        G.step(pop)
        hc.step()
        check_same(G, pop, hc, f"generation {g}")
    st = G.state()
    assert st["gen"] == gens and st["evals"] == gens * P
    assert st["best_F"] < 1e30 and st["best_n"] == n


def test_generation_tabu_and_stagnation_paths(cuda, orc):
    """Tenure 0 diversifies every revisited cell that is not near the
    incumbent; a stagnation of 0.8 turns about a tenth of the plan into
    restarts."""
    rng = np.random.default_rng(5)
    n, P = 64, 48
    G, pop, hc = make(cuda, orc, n, P, 3, rng, tabu_tenure=0, ls_iters=4, cold_iters=6)
    for g in range(6):
        if g == 3:
            poke_state(G, hc.pol, since_improve=20, level_best_F=0.0)
        G.step(pop)
        hc.step()
        check_same(G, pop, hc, f"generation {g}")
    ops = hc.pol.plan["op"]
    assert (ops == 9).any()


@pytest.mark.parametrize("prec,n,P", [("bf16x3", 80, 32), ("fp32", 1000, 320)])
def test_generation_graph_equals_eager(cuda, orc, prec, n, P):
    """A captured graph of generations equals the eager ones bit for bit, on
    the tensor cores and on the fp32 path (narrow-tile kernels, P over two
    waves)."""
    rng = np.random.default_rng(11)
    NI, gens = 4, 7
    cfg = K().generation_config(n_islands=NI, elite=2, ls_iters=6, cold_iters=9, p_max=300.0,
                                precision=prec, fw_rounds=1, fw_iters=8, fw_nT=4,
                                fw_t_max=0.3, fw_precision=prec, tabu_capacity=1 << 10,
                                seed=SEED)
    pop0 = seeds(n, P, rng)
    so = torch.tensor(seed_ops(P, rng), device=cuda)
    A = K().Generation(n, P, cfg)
    B = K().Generation(n, P, cfg)
    A.begin_level(n, 0, so)
    B.begin_level(n, 0, so)
    pa = torch.tensor(pop0, device=cuda)
    pb = torch.tensor(pop0, device=cuda)
    for _ in range(gens):
        A.step(pa)
    graph = B.capture(pb, gens)
    graph.launch()
    torch.cuda.synchronize()
    assert torch.equal(pa.view(torch.int32), pb.view(torch.int32))
    assert A.state() == B.state()
    va, vb = A.views(), B.views()
    for k in ("fit", "child_fit", "rank", "p1", "op", "strength", "cur_op", "best_row"):
        assert torch.equal(va[k], vb[k]), k
    graph.close()


def test_generation_incumbent_is_certified(cuda, orc):
    """The incumbent row's F is its fp64 evaluation, and improves on every
    evaluated candidate; set_best adopts a resumed vector."""
    rng = np.random.default_rng(2)
    n, P = 128, 32
    G, pop, hc = make(cuda, orc, n, P, 2, rng)
    fits = []
    for _ in range(6):
        G.step(pop)
        fits.append(G.views()["fit"].cpu().numpy().copy())
    st = G.state()
    row = G.best()
    assert row.size == n
    assert abs(orc.host_f(row.astype(np.float64)) - st["best_F"]) <= 1e-14 * st["best_F"]
    assert st["best_F"] <= min(f.min() for f in fits) + 1e-12
    # a resumed incumbent: reinjected over island 0's worst slot at generation 9
    G2 = K().Generation(n, P, G.cfg)
    G2.begin_level(n, 0)
    G2.set_best(torch.tensor(row, device=cuda), st["best_F"])
    s2 = G2.state()
    assert s2["best_F"] == st["best_F"] and s2["best_n"] == n


def test_generation_tabu_capacity_reported(cuda, orc):
    rng = np.random.default_rng(9)
    n, P = 64, 64
    G, pop, _ = make(cuda, orc, n, P, 4, rng, tabu_capacity=8, ls_iters=2, cold_iters=3)
    G.step(pop)
    st = G.state()
    assert st["status"] == L().ERR_CAPACITY
    assert st["cells"] <= 9
    assert np.isfinite(pop.cpu().numpy()).all()


@pytest.mark.parametrize("P,NI,elite", [(8, 1, 2), (4, 4, 0), (12, 3, 5)])
def test_generation_edge_islands(cuda, orc, P, NI, elite):
    """One island (migration onto itself), single-slot islands (migration
    chained through every island in order) and more elites than slots."""
    rng = np.random.default_rng(P * 10 + NI)
    n = 48
    G, pop, hc = make(cuda, orc, n, P, NI, rng, elite=elite, ls_iters=3, cold_iters=6)
    for g in range(14):                        # a migration at generation 12
        G.step(pop)
        hc.step()
        check_same(G, pop, hc, f"generation {g}")
    if elite >= P // NI:
        assert (hc.pol.plan["op"] == 20).all()


def test_search_driver_eager_remainder(cuda, orc):
    """gens_per_level not a multiple of gens_per_graph: one graph replay, then
    single eager generations."""
    gen = K().generation_config(n_islands=2, elite=1, ls_iters=4, cold_iters=6, p_max=200.0,
                                precision="fp32", fw_rounds=0, tabu_capacity=1 << 10, seed=9)
    seen = []
    best, F = K().search(ladder=(40,), P=8, seconds=1e9, gens_per_level=3, gens_per_graph=2,
                         polish_iters=0, polish_top=0, gen=gen,
                         progress=lambda d, b: seen.append(d["gen"]))
    assert seen == [2, 3]
    assert best.size == 40 and F == orc.host_f(best)

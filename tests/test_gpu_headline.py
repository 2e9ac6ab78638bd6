"""The timed path at the benchmark's own configuration, against the oracle.

The benchmark times a BF16x3 local search of n = 8400 lognormal candidates
(1/3 exact zeros, a support gap of width n/10, an endpoint atom, normalised),
p 2 -> 1024, lr 1e-3, on more candidates than the GPU has SMs, so that the
balanced-segment kernel runs (step chains split between CTAs, the hand-over
through memory).  Here the same kernel runs P = SMs + 12 such candidates for
20 steps and three of them -- the first, the first whose chain is split
between two CTAs, and the last -- are compared with the oracle's fp32 local
search (oracle/sidon_oracle.c, the update order of src/kernels.cuh:177-289
and tools/probe.cpp:62-116): certified F within 1e-3 relative for BF16x3
(the plain-method case's bar) and 1e-4 for the fp32 SIMT step, heights
exactly non-negative and summing to 1.  The balanced form equals the
one-CTA-per-candidate form bit for bit at this size, two balanced launches
on concurrent streams (each with its own flag words) equal the same
launches run one after the other, and the balanced form captured in a CUDA
graph (the island anneal of a uniform batch) equals its eager run.
Needs a B200.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

N, STEPS = 8400, 20
ANNEAL = dict(p_start=2.0, p_end=1024.0, lr_start=1e-3, lr_end=1e-3)


def _sms(dev):
    return torch.cuda.get_device_properties(dev).multi_processor_count


def _population(P, seed=8400):
    from sidon_b200 import synth
    return synth.population("lognormal", N, P, seed=seed)


def split_candidates(P, iters, G):
    """Candidates whose step chain crosses a segment boundary of the
    balanced-segment kernel (CTA c runs steps [c T / G, (c+1) T / G) of the
    P chains laid end to end, T = P iters)."""
    T = P * iters
    cuts = {c * T // G for c in range(1, G)}
    return [p for p in range(P) if any(p * iters < b < (p + 1) * iters for b in cuts)]


@pytest.fixture(scope="module")
def headline(cuda, orc):
    P = _sms(cuda) + 12
    pop = _population(P)
    split = split_candidates(P, STEPS, _sms(cuda))
    assert split, "the configuration must split some chain between two CTAs"
    picks = sorted({0, split[0], P - 1})
    want = orc.local_search(pop[picks], STEPS, **{k: v for k, v in zip(
        ("pS", "pE", "lrS", "lrE"), ANNEAL.values())})
    return P, pop, picks, want


@pytest.mark.parametrize("prec,tol", [("bf16x3", 1e-3), ("fp32", 1e-4)])
def test_headline_search_tracks_the_oracle(cuda, orc, headline, prec, tol):
    from sidon_b200 import kernels
    P, pop, picks, want = headline
    x = torch.as_tensor(pop, device=cuda)
    kernels.run_local_search(x, STEPS, precision=prec, **ANNEAL)
    assert kernels.device_status(reset=True) == 0
    got = x.cpu().numpy()
    assert (got >= 0).all()
    assert np.abs(got.astype(np.float64).sum(axis=1) - 1.0).max() < 1e-5
    F0 = [orc.host_f(pop[p].astype(np.float64)) for p in picks]
    for j, p in enumerate(picks):
        Fg = orc.host_f(got[p].astype(np.float64))
        Fw = orc.host_f(want[j].astype(np.float64))
        assert Fw < F0[j]
        assert abs(Fg - Fw) <= tol * Fw, (prec, p, Fg, Fw, F0[j])
    Fc = kernels.certify(x)[0].cpu().numpy()
    for p in picks:                                   # certified F is hostF's to 1e-12
        Fh = orc.host_f(got[p].astype(np.float64))
        assert abs(Fc[p] - Fh) <= 1e-12 * Fh


def test_headline_balanced_equals_one_cta_per_candidate(cuda, headline):
    from sidon_b200 import kernels
    P, pop, _, _ = headline
    a = torch.as_tensor(pop, device=cuda)
    b = torch.as_tensor(pop, device=cuda)
    kernels.run_local_search(a, STEPS, precision="bf16x3", **ANNEAL)
    kernels.run_local_search(b, STEPS, precision="bf16x3", balanced=False, **ANNEAL)
    torch.cuda.synchronize()
    assert kernels.device_status(reset=True) == 0
    assert torch.equal(a, b)


def test_balanced_launches_on_concurrent_streams(cuda):
    """Each balanced launch keeps its hand-over flags in its own workspace, so
    two launches on concurrent streams do not interfere: both equal the same
    launches run one after the other."""
    from sidon_b200 import kernels, synth
    P, n, iters = _sms(cuda) + 30, 2048, 12
    pops = [synth.population("lognormal", n, P, seed=s) for s in (5, 6)]
    serial = []
    for p in pops:
        x = torch.as_tensor(p, device=cuda)
        kernels.run_local_search(x, iters, precision="bf16x3", **ANNEAL)
        serial.append(x)
    torch.cuda.synchronize()
    xs = [torch.as_tensor(p, device=cuda) for p in pops]
    ws = [kernels.local_search_workspace(n, P, "bf16x3", cuda) for _ in pops]
    moms = [(torch.empty_like(x), torch.empty_like(x)) for x in xs]
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    torch.cuda.synchronize()
    for x, w, (m, v), s in zip(xs, ws, moms, streams):
        kernels.run_local_search(x, iters, precision="bf16x3", mom=m, vel=v, workspace=w,
                                 stream=s, **ANNEAL)
    torch.cuda.synchronize()
    assert kernels.device_status(reset=True) == 0
    for x, y in zip(xs, serial):
        assert torch.equal(x, y)


def test_balanced_segments_in_a_captured_anneal(cuda):
    """A uniform batch of more candidates than SMs keeps the balanced-segment
    kernel inside a CUDA graph (sidon_anneal_capture; the rank buffer holds
    the flags between migrations): replay equals the eager anneal bit for bit."""
    from sidon_b200 import kernels, synth
    P, n = _sms(cuda) + 20, 1024
    pop = synth.population("structured", n, P, seed=3)
    cfg = kernels.anneal_config(steps=40, p_start=2.0, p_end=64.0, lr_start=1e-3, lr_end=1e-3,
                                precision="bf16x3", fw_every=0, migrate_every=20,
                                n_islands=4, k_migrate=2)
    eager = torch.as_tensor(pop, device=cuda)
    fit_e = kernels.anneal(eager, cfg)
    graphed = torch.as_tensor(pop, device=cuda)
    g = kernels.AnnealGraph(graphed, cfg)
    g.launch()
    torch.cuda.synchronize()
    g.close()
    assert kernels.device_status(reset=True) == 0
    assert torch.equal(eager, graphed)
    assert torch.equal(fit_e, g.fit)

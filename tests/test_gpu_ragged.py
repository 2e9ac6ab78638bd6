"""Ragged batches (candidates of different n in one launch), the persistent
tensor-core kernel, and the stream-ordered anneal driver with its CUDA-graph
capture.  Needs a B200.

Bar: a candidate's result in a ragged batch is bit-identical to the uniform
entry point's result for that candidate alone (the kernels give each
candidate the threads and reduction order of a uniform launch at its n);
ragged migration is bit-identical to the oracle; a graph replay is
bit-identical to the eager enqueue of the same schedule.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

SIZES = [1, 37, 64, 65, 300, 512, 129, 1000, 2048, 777, 4096, 8400]


def K():
    from sidon_b200 import kernels
    return kernels


def _status():
    import sidon_b200
    return sidon_b200.load().sidon_device_status(1)


def _batch(sizes, seed, dev):
    from sidon_b200 import synth
    rows = synth.ragged_population(sizes, seed)
    for r in rows:                       # never an all-zero candidate
        r[0] = max(r[0], np.float32(1e-3))
    return rows, K().RaggedBatch(rows, device=dev)


def test_ragged_order(cuda):
    sizes = [5, 9, 9, 1, 300, 5, 8400, 9]
    _, b = _batch(sizes, 1, cuda)
    want = sorted(range(len(sizes)), key=lambda p: (-sizes[p], p))
    assert b.order.cpu().tolist() == want


@pytest.mark.parametrize("precision", ["bf16x3", "bf16x1", "fp32"])
def test_ragged_local_search_matches_uniform(cuda, precision):
    rows, b = _batch(SIZES, 7, cuda)
    K().run_local_search_ragged(b, 25, 2.0, 64.0, 1e-3, 1e-3, precision=precision)
    got = b.rows()
    assert _status() == 0
    for p, r in enumerate(rows):
        u = torch.as_tensor(r[None, :], device=cuda)
        K().run_local_search(u, 25, 2.0, 64.0, 1e-3, 1e-3, precision=precision)
        np.testing.assert_array_equal(got[p], u.cpu().numpy()[0], err_msg=f"candidate {p}")
        assert (got[p] >= 0).all()


@pytest.mark.parametrize("n_max", [9216, 9728])
def test_window_ring_shape_does_not_change_results(cuda, n_max):
    """The tensor-core CTA sizes its window ring from the batch's largest
    row: two stages of three windows for a uniform n = 8400 or 2048, of two
    at n_max = 9216, three single windows at n = 300 and at n_max = 9728.
    The same rows give the same heights bit for bit under every shape."""
    rows, b = _batch([300, 2048, 8400, n_max], 21, cuda)
    K().run_local_search_ragged(b, 12, 2.0, 512.0, 1e-3, 1e-3, precision="bf16x3")
    got = b.rows()
    assert _status() == 0
    for p, r in enumerate(rows[:3]):
        u = torch.as_tensor(r[None, :], device=cuda)
        K().run_local_search(u, 12, 2.0, 512.0, 1e-3, 1e-3, precision="bf16x3")
        np.testing.assert_array_equal(got[p], u.cpu().numpy()[0], err_msg=f"candidate {p}")


def test_ragged_local_search_order_and_skip(cuda):
    rows, b1 = _batch(SIZES, 9, cuda)
    _, b2 = _batch(SIZES, 9, cuda)
    skip = torch.zeros(len(SIZES), dtype=torch.int32, device=cuda)
    skip[3] = 1
    mode = torch.zeros(len(SIZES), dtype=torch.int32, device=cuda)
    mode[5] = 1
    K().run_local_search_ragged(b1, 12, 2.0, 32.0, 1e-3, 1e-3, skip=skip, mode_arr=mode)
    K().run_local_search_ragged(b2, 12, 2.0, 32.0, 1e-3, 1e-3, skip=skip, mode_arr=mode,
                                use_order=False)
    assert torch.equal(b1.flat, b2.flat)
    np.testing.assert_array_equal(b1.rows()[3], rows[3])
    assert _status() == 0


def test_ragged_eval_matches_uniform_and_hostF(cuda):
    rows, b = _batch(SIZES, 11, cuda)
    F, N = K().run_eval_ragged(b)
    F, N = F.cpu().numpy(), N.cpu().numpy()
    for p, r in enumerate(rows):
        u = torch.as_tensor(r[None, :], device=cuda)
        Fu, Nu = K().run_eval(u)
        assert F[p] == Fu.item() == K().host_f(r.astype(np.float64)), p
        assert N[p] == Nu.item()


def test_ragged_frank_wolfe_matches_uniform(cuda):
    sizes = [64, 300, 1000, 129, 2048]
    rows, b = _batch(sizes, 13, cuda)
    K().run_frank_wolfe_ragged(b, 1, 20, 6, 0.3, tau=0.9, sigma=0.9)
    got = b.rows()
    for p, r in enumerate(rows):
        u = torch.as_tensor(r[None, :], device=cuda)
        assert K().run_frank_wolfe(u, 1, 20, 6, 0.3, tau=0.9, sigma=0.9)
        np.testing.assert_array_equal(got[p], u.cpu().numpy()[0], err_msg=f"candidate {p}")


def test_ragged_frank_wolfe_tc_matches_uniform(cuda):
    sizes = [64, 300, 1000, 129, 2048]
    rows, b = _batch(sizes, 13, cuda)
    K().run_frank_wolfe_tc_ragged(b, 2, 20, 6, 0.3, tau=0.9, sigma=0.9)
    got = b.rows()
    assert _status() == 0
    for p, r in enumerate(rows):
        u = torch.as_tensor(r[None, :], device=cuda)
        K().run_frank_wolfe_tc(u, 2, 20, 6, 0.3, tau=0.9, sigma=0.9)
        np.testing.assert_array_equal(got[p], u.cpu().numpy()[0], err_msg=f"candidate {p}")


def test_ragged_migrate_vs_oracle(cuda, orc):
    rng = np.random.default_rng(5)
    sizes = [int(x) for x in rng.choice([16, 40, 64, 100], 24)]
    rows, b = _batch(sizes, 17, cuda)
    fit = rng.uniform(1.4, 1.8, 24)
    fit[[2, 9]] = fit[4]                                   # ties
    fit[13] = np.nan                                       # unevaluated
    want_flat, want_fit, want_order = orc.island_migrate_ragged(
        np.concatenate(rows), b.host_offsets, fit, 4, 2)
    f = torch.as_tensor(fit, device=cuda)
    order = K().island_migrate_ragged(b, f, 4, 2)
    np.testing.assert_array_equal(order.cpu().numpy(), want_order)
    np.testing.assert_array_equal(b.flat.cpu().numpy(), want_flat)
    np.testing.assert_array_equal(f.cpu().numpy(), want_fit)     # NaN == NaN here


def _small_cfg(precision="bf16x3", fw_precision="bf16x3"):
    return K().anneal_config(steps=60, p_start=2.0, p_end=64.0, precision=precision,
                             fw_every=20, pdhg_iters=10, fw_nT=4, fw_precision=fw_precision,
                             n_islands=3, migrate_every=30, k_migrate=1)


@pytest.mark.parametrize("fw_precision", ["bf16x3", "fp32"])
def test_anneal_matches_manual_schedule(cuda, fw_precision):
    sizes = [64, 300, 129, 1000, 64, 512]
    _, b1 = _batch(sizes, 21, cuda)
    _, b2 = _batch(sizes, 21, cuda)
    cfg = _small_cfg(fw_precision=fw_precision)
    fit = K().anneal(b1, cfg)
    # the same schedule by hand: cuts at 20, 30, 40, 60
    steps, pS, pE, lr = 60, 2.0, 64.0, 1e-3

    def sch(s):
        return pS * (pE / pS) ** (s / (steps - 1))
    f2 = torch.empty(len(sizes), dtype=torch.float64, device=cuda)
    for s0, s1 in [(0, 20), (20, 30), (30, 40), (40, 60)]:
        K().run_local_search_ragged(b2, s1 - s0, sch(s0), sch(s1 - 1), lr, lr)
        if s1 % 20 == 0:
            if fw_precision == "fp32":
                K().run_frank_wolfe_ragged(b2, 1, 10, 4, 0.3, tau=0.9, sigma=0.9)
            else:
                K().run_frank_wolfe_tc_ragged(b2, 1, 10, 4, 0.3, tau=0.9, sigma=0.9)
        if s1 % 30 == 0 and s1 < steps:
            f2, _ = K().run_eval_ragged(b2, with_nactive=False)
            K().island_migrate_ragged(b2, f2, 3, 1)
    f2, _ = K().run_eval_ragged(b2, with_nactive=False)
    assert torch.equal(b1.flat, b2.flat)
    assert torch.equal(fit, f2)
    assert bool((b1.flat >= 0).all())
    assert _status() == 0


@pytest.mark.parametrize("ragged", [True, False])
def test_anneal_graph_replay_matches_eager(cuda, ragged):
    sizes = [64, 300, 129, 1000, 64, 512] if ragged else [256] * 6
    _, b1 = _batch(sizes, 23, cuda)
    _, b2 = _batch(sizes, 23, cuda)
    cfg = _small_cfg()
    if ragged:
        x1, x2 = b1, b2
        flat1, flat2 = b1.flat, b2.flat
    else:
        x1, x2 = b1.flat.view(6, 256), b2.flat.view(6, 256)
        flat1, flat2 = b1.flat, b2.flat
    fit1 = K().anneal(x1, cfg)
    g = K().AnnealGraph(x2, cfg)
    g.launch()
    torch.cuda.synchronize()
    assert torch.equal(flat1, flat2)
    assert torch.equal(fit1, g.fit)
    g.close()
    assert _status() == 0


def test_torch_graph_capture_of_ragged_step(cuda):
    """The ragged local search captured by torch.cuda.CUDAGraph replays
    bit-identically to an eager call on the same input."""
    sizes = [64, 300, 1000, 129]
    rows, b = _batch(sizes, 29, cuda)
    start = b.flat.clone()
    mom, vel = torch.empty_like(b.flat), torch.empty_like(b.flat)
    K().run_local_search_ragged(b, 8, 2.0, 16.0, 1e-3, 1e-3, mom=mom, vel=vel)   # warm-up
    eager = b.flat.clone()
    b.flat.copy_(start)
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            K().run_local_search_ragged(b, 8, 2.0, 16.0, 1e-3, 1e-3, mom=mom, vel=vel)
    b.flat.copy_(start)
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(b.flat, eager)


def test_uniform_anneal_graph_beyond_one_wave(cuda):
    """A uniform batch larger than the SM count: the eager anneal takes the
    balanced-segment kernel, the captured graph the one-CTA-per-candidate
    kernel (no cooperative launch inside a capture); results are equal."""
    from sidon_b200 import synth
    sms = torch.cuda.get_device_properties(cuda).multi_processor_count
    P = 4 * ((sms + 12) // 4)                      # > SMs, divisible by 4 islands
    pop = synth.population("structured", 256, P, seed=31)
    x1 = torch.as_tensor(pop, device=cuda)
    x2 = torch.as_tensor(pop, device=cuda)
    cfg = K().anneal_config(steps=40, p_start=2.0, p_end=64.0, fw_every=20, pdhg_iters=5,
                            fw_nT=3, n_islands=4, migrate_every=20, k_migrate=1)
    fit1 = K().anneal(x1, cfg)
    g = K().AnnealGraph(x2, cfg)
    g.launch()
    torch.cuda.synchronize()
    assert torch.equal(x1, x2)
    assert torch.equal(fit1, g.fit)
    g.close()
    assert _status() == 0

"""Variation operators and support signatures on the device against the C
oracle (same Philox4x32-10 draws, same fixed-order sums).  Needs a B200.

Bars: operators whose arithmetic is plain products and sums (selection,
blend, shift, sparsify, spike, gap, atom, clone) and the signatures are
bit-identical to the oracle; operators that go through a libm function
(exp / cos / log of the normals and cosine modes: ops 2, 3, 4, 9, 11) agree
to 2e-6 relative, the difference between the device's and the host's
correctly-rounded-or-nearly implementations.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

EXACT = (0, 1, 5, 6, 7, 8, 10, 12, 13, 20)
LIBM = (2, 3, 4, 9, 11)


def K():
    from sidon_b200 import kernels
    return kernels


@pytest.mark.parametrize("n", [1, 7, 300, 1000, 8400])
def test_variation_matches_oracle(cuda, orc, n):
    rng = np.random.default_rng(n)
    pop = rng.uniform(0, 1, (4, n)).astype(np.float32)
    pop[:, rng.uniform(size=n) < 1 / 3] = 0
    pop[:, 0] += 0.5
    ops = list(EXACT + LIBM) * 2
    J = len(ops)
    p1 = rng.integers(0, 4, J)
    p2 = rng.integers(0, 4, J)
    st = rng.uniform(0.03, 0.5, J).astype(np.float32)
    want = orc.variation(pop, p1, p2, ops, st, seed=12345, gen=7)
    got = K().variation(torch.as_tensor(pop, device=cuda), p1, p2, ops, st, 12345, 7).cpu().numpy()
    for j, o in enumerate(ops):
        if o in EXACT:
            np.testing.assert_array_equal(got[j], want[j], err_msg=f"op {o}")
        else:
            np.testing.assert_allclose(got[j], want[j], rtol=2e-6, atol=2e-6 * want[j].max(),
                                       err_msg=f"op {o}")
    assert (got >= 0).all()
    np.testing.assert_allclose(got.astype(np.float64).sum(1), 1.0, rtol=1e-5)


def test_variation_streams_depend_on_seed_and_generation(cuda):
    pop = torch.rand((2, 500), device=cuda)
    a = K().variation(pop, [0], [1], [2], [0.3], 1, 1)
    b = K().variation(pop, [0], [1], [2], [0.3], 1, 2)
    c = K().variation(pop, [0], [1], [2], [0.3], 2, 1)
    d = K().variation(pop, [0], [1], [2], [0.3], 1, 1)
    assert torch.equal(a, d)
    assert not torch.equal(a, b) and not torch.equal(a, c)


def test_variation_fp64_and_lognormal_statistics(cuda):
    """fp64 heights work; log(offspring / parent) of the log-normal operator
    has the requested spread (strength 0.2 over 20000 cells)."""
    n = 20000
    a = torch.full((1, n), 1.0 / n, dtype=torch.float64, device=cuda)
    o = K().variation(a, [0], [0], [2], [0.2], 99, 0)
    r = torch.log(o[0] / a[0]).cpu().numpy()
    r -= r.mean()
    assert abs(r.std() - 0.2) < 0.01


@pytest.mark.parametrize("n", [6, 300, 8400])
def test_support_sig_matches_oracle(cuda, orc, n):
    rng = np.random.default_rng(n + 1)
    pop = rng.uniform(0, 1, (5, n)).astype(np.float32)
    pop[:, rng.uniform(size=n) < 0.4] = 0
    pop[1] = pop[0] * 3.0                      # same support as candidate 0
    sig, nnz = K().support_sig(torch.as_tensor(pop, device=cuda))
    ws, wn = orc.support_sig(pop)
    np.testing.assert_array_equal(sig.cpu().numpy().view(np.uint64), ws)
    np.testing.assert_array_equal(nnz.cpu().numpy(), wn)
    assert sig[0].item() == sig[1].item()

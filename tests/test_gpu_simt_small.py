"""The fp32 local search and Frank-Wolfe step of small and middle uniform
candidates (n <= 1664: the CTA kernels with 7-, 9-, 11- or 13-output lane
tiles) against the 15-output kernels that a ragged batch of the same rows
runs: bit-identical heights
(every output is the same fma chain, the team and its sums are the same),
with skip[] and mirror-descent candidates; and against the oracle within the
fp32 bars.  Needs a B200.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def K():
    from sidon_b200 import kernels
    return kernels


@pytest.mark.parametrize("n,P", [(1, 9), (33, 40), (128, 512), (300, 77), (512, 400), (896, 160),
                                 (1000, 60), (1300, 40), (1600, 40), (1700, 20)])
def test_small_tiles_are_bitwise_the_large_tiles(cuda, n, P):
    rng = np.random.default_rng(n)
    pop = rng.uniform(0.2, 1.0, (P, n)).astype(np.float32)
    pop[:, rng.uniform(size=n) < 0.2] = 0.0
    mode = torch.tensor((np.arange(P) % 5 == 3).astype(np.int32), device=cuda)
    skip = torch.tensor((np.arange(P) % 7 == 6).astype(np.int32), device=cuda)
    x = torch.tensor(pop, device=cuda)
    K().run_local_search(x, 25, 4.0, 300.0, 0.05, 0.005, mode_arr=mode, skip=skip,
                         precision="fp32")
    batch = K().RaggedBatch(list(pop), device=cuda)       # the ragged path: 15-output tiles
    K().run_local_search_ragged(batch, 25, 4.0, 300.0, 0.05, 0.005, precision="fp32",
                                mode_arr=mode, skip=skip)
    torch.cuda.synchronize()
    y = batch.flat.view(P, n)
    assert torch.equal(x.view(torch.int32), y.view(torch.int32))
    live = skip == 0
    assert torch.equal(x[~live], torch.tensor(pop, device=cuda)[~live])


def test_small_tiles_against_the_oracle(cuda, orc):
    n, P = 256, 64
    rng = np.random.default_rng(3)
    pop = rng.uniform(0.2, 1.0, (P, n)).astype(np.float32)
    x = torch.tensor(pop, device=cuda)
    K().run_local_search(x, 1, 2.0, 2.0, 0.01, 0.01)
    want = orc.local_search(pop[:16], 1, 2.0, 2.0, 0.01, 0.01)
    assert np.allclose(x[:16].cpu().numpy(), want, rtol=2e-5, atol=1e-9)
    x = torch.tensor(pop, device=cuda)
    K().run_local_search(x, 40, 4.0, 64.0, 0.02, 0.005)
    got = K().run_eval(x, with_nactive=False)[0].cpu().numpy()
    ref = orc.local_search(pop[:8], 40, 4.0, 64.0, 0.02, 0.005)
    for p in range(8):
        Fw = orc.host_f(ref[p].astype(np.float64))
        assert abs(got[p] - Fw) <= 1e-4 * Fw


@pytest.mark.parametrize("n,P", [(33, 20), (300, 50), (896, 30), (1100, 20), (1500, 16)])
def test_small_tile_frank_wolfe_is_bitwise_the_large_tiles(cuda, n, P):
    """The fp32 Frank-Wolfe step with narrow tiles (uniform, n <= 1664) = the
    15-output kernel of a ragged batch of the same rows, bit for bit."""
    rng = np.random.default_rng(n + 1)
    pop = rng.uniform(0.2, 1.0, (P, n)).astype(np.float32)
    pop[:, rng.uniform(size=n) < 0.2] = 0.0
    skip = torch.tensor((np.arange(P) % 6 == 5).astype(np.int32), device=cuda)
    x = torch.tensor(pop, device=cuda)
    assert K().run_frank_wolfe(x, 2, 30, skip=skip)
    batch = K().RaggedBatch(list(pop), device=cuda)
    K().run_frank_wolfe_ragged(batch, 2, 30, skip=skip)
    torch.cuda.synchronize()
    assert torch.equal(x.view(torch.int32), batch.flat.view(P, n).view(torch.int32))

"""The fp32 local search for many small candidates (one warp per candidate,
taken when P >= 2 x SMs and n <= 512) against the one-CTA-per-candidate
kernel it stands in for: bit-identical heights and moments (the convolution
and correlation outputs are the same fma chains, the sums are formed in the
CTA kernel's order), with skip[] and mirror-descent candidates; and against
the oracle within the fp32 bars.  Needs a B200.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def K():
    from sidon_b200 import kernels
    return kernels


@pytest.mark.parametrize("n", [1, 33, 128, 300, 512])
def test_warp_kernel_is_bitwise_the_cta_kernel(cuda, n):
    P = 400                      # >= 2 x 148 SMs: the warp kernel
    rng = np.random.default_rng(n)
    pop = rng.uniform(0.2, 1.0, (P, n)).astype(np.float32)
    pop[:, rng.uniform(size=n) < 0.2] = 0.0
    mode = (np.arange(P) % 5 == 3).astype(np.int32)
    skip = (np.arange(P) % 7 == 6).astype(np.int32)
    x = torch.tensor(pop, device=cuda)
    mom, vel = torch.empty_like(x), torch.empty_like(x)
    K().run_local_search(x, 25, 4.0, 300.0, 0.05, 0.005, mom=mom, vel=vel,
                         mode_arr=torch.tensor(mode, device=cuda),
                         skip=torch.tensor(skip, device=cuda))
    # the same candidates in batches of 50: the CTA kernel
    y = torch.tensor(pop, device=cuda)
    my, vy = torch.empty_like(y), torch.empty_like(y)
    for s in range(0, P, 50):
        K().run_local_search(y[s:s + 50], 25, 4.0, 300.0, 0.05, 0.005, mom=my[s:s + 50],
                             vel=vy[s:s + 50], mode_arr=torch.tensor(mode[s:s + 50], device=cuda),
                             skip=torch.tensor(skip[s:s + 50], device=cuda))
    torch.cuda.synchronize()
    assert torch.equal(x.view(torch.int32), y.view(torch.int32))
    live = torch.tensor(skip == 0, device=cuda)
    assert torch.equal(mom[live].view(torch.int32), my[live].view(torch.int32))
    assert torch.equal(vel[live].view(torch.int32), vy[live].view(torch.int32))
    assert torch.equal(x[~live], torch.tensor(pop, device=cuda)[~live])


def test_warp_kernel_against_the_oracle(cuda, orc):
    n, P = 256, 320
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

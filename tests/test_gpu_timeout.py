"""Bounded device-side waits: a wait that runs out ends the kernel with
SIDON_ERR_TIMEOUT in the status word instead of hanging it, and leaves the
context usable.

The reference has no such path: its CUDA_OK macro prints and exits the
process on any CUDA error (src/kernels.cuh:20-28).  Here every wait of the
tensor-core pipeline (and the balanced-segment kernel's hand-over flag) has
a clock-cycle limit, settable for tests with sidon_set_wait_limit.  With a
limit of one cycle the pipeline's first wait that does not succeed at once
runs out: the kernel records the timeout, sets its abort flag, still drains
the MMAs it issued, frees its tensor memory and returns.  The limit is then
restored and the same call must equal a clean run bit for bit (nothing of
the aborted launch -- abort flag, barrier phases, tensor memory -- carries
over).  No wait here is left unbounded and nothing faults.  Needs a B200.
"""
import pytest
import torch

pytestmark = pytest.mark.gpu

ANNEAL = dict(p_start=2.0, p_end=64.0, lr_start=1e-3, lr_end=1e-3)


def _cases(dev):
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    # (candidates, n): one wave of the one-CTA-per-candidate kernel, and a
    # batch of more candidates than SMs (balanced segments, hand-over flags)
    return [(3, 1024), (sms + 4, 512)]


@pytest.mark.parametrize("case", [0, 1])
def test_short_wait_limit_times_out_and_recovers(cuda, case):
    from sidon_b200 import kernels, synth
    P, n = _cases(cuda)[case]
    pop = synth.population("lognormal", n, P, seed=11 + case)
    kernels.set_wait_limit(0)
    kernels.device_status(reset=True)
    clean = torch.as_tensor(pop, device=cuda)
    kernels.run_local_search(clean, 6, precision="bf16x3", **ANNEAL)
    torch.cuda.synchronize()
    assert kernels.device_status(reset=True) == 0
    try:
        kernels.set_wait_limit(1)
        x = torch.as_tensor(pop, device=cuda)
        kernels.run_local_search(x, 6, precision="bf16x3", **ANNEAL)
        torch.cuda.synchronize()                         # the kernel returned
        assert kernels.device_status(reset=True) == kernels._lib.ERR_TIMEOUT
    finally:
        kernels.set_wait_limit(0)
    again = torch.as_tensor(pop, device=cuda)
    kernels.run_local_search(again, 6, precision="bf16x3", **ANNEAL)
    torch.cuda.synchronize()
    assert kernels.device_status(reset=True) == 0
    assert torch.equal(again, clean)


def test_wait_limit_applies_to_frank_wolfe_and_forward(cuda):
    """The same recovery for the tensor-core Frank-Wolfe step and G_p forward."""
    from sidon_b200 import kernels, synth
    pop = synth.population("structured", 2048, 2, seed=4)
    kernels.set_wait_limit(0)
    kernels.device_status(reset=True)
    y0 = torch.as_tensor(pop, device=cuda)
    kernels.run_frank_wolfe_tc(y0, 1, 4, 3, 0.3, tau=0.9, sigma=0.9)
    v0, s0, _ = kernels.lp_forward(torch.as_tensor(pop, device=cuda), 8.0, precision="bf16x3")
    torch.cuda.synchronize()
    assert kernels.device_status(reset=True) == 0
    try:
        kernels.set_wait_limit(1)
        y = torch.as_tensor(pop, device=cuda)
        kernels.run_frank_wolfe_tc(y, 1, 4, 3, 0.3, tau=0.9, sigma=0.9)
        torch.cuda.synchronize()
        assert kernels.device_status(reset=True) == kernels._lib.ERR_TIMEOUT
        kernels.lp_forward(torch.as_tensor(pop, device=cuda), 8.0, precision="bf16x3")
        torch.cuda.synchronize()
        assert kernels.device_status(reset=True) == kernels._lib.ERR_TIMEOUT
    finally:
        kernels.set_wait_limit(0)
    y1 = torch.as_tensor(pop, device=cuda)
    kernels.run_frank_wolfe_tc(y1, 1, 4, 3, 0.3, tau=0.9, sigma=0.9)
    v1, s1, _ = kernels.lp_forward(torch.as_tensor(pop, device=cuda), 8.0, precision="bf16x3")
    torch.cuda.synchronize()
    assert kernels.device_status(reset=True) == 0
    assert torch.equal(y0, y1)
    assert torch.equal(v0, v1) and torch.equal(s0, s1)

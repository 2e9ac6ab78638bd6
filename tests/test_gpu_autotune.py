"""The fused local search's schedule tuner (sidon_autotune_local_search).

The reference fixes its tiling at compile time (TK = TI = 8,
src/kernels.cuh:30-33).  Here the lane tile of the fp32 kernel, the window
ring of the tensor-core kernel and, for more candidates than SMs, balanced
segments vs waves are chosen per (device, n, P, precision) by timing each on
a short anneal.  Every choice computes the same fma chains and MMAs in the
same order, so the tuner may pick any of them without changing a bit: the
search after tuning equals the search before it, and the schedule the
library reports afterwards is the tuned one.  Needs a B200.
"""
import pytest
import torch

pytestmark = pytest.mark.gpu

ANNEAL = dict(p_start=2.0, p_end=128.0, lr_start=1e-3, lr_end=1e-3)


def _sms(dev):
    return torch.cuda.get_device_properties(dev).multi_processor_count


@pytest.mark.parametrize("prec,n,P", [("fp32", 512, 96), ("fp32", 1300, 40),
                                      ("bf16x3", 2048, "sms+40"), ("bf16x3", 8400, "sms+2"),
                                      ("bf16x1", 4096, 60)])
def test_tuned_schedule_is_used_and_changes_no_bit(cuda, prec, n, P):
    from sidon_b200 import kernels, synth
    if isinstance(P, str):
        P = _sms(cuda) + int(P.split("+")[1])
    pop = synth.population("lognormal", n, P, seed=n + P)
    before = kernels.local_search_schedule(n, P, prec)
    assert before["tuned"] == 0
    x0 = torch.as_tensor(pop, device=cuda)
    kernels.run_local_search(x0, 6, precision=prec, **ANNEAL)
    s = kernels.autotune_local_search(n, P, prec)
    assert s["tuned"] == 1 and s["ms_per_step"] > 0
    if prec == "fp32":
        assert s["lane_tile"] in (7, 9, 11, 13, 15) and 128 * s["lane_tile"] >= min(n, 1920)
    else:
        assert 1 <= s["ring_tiles"] <= 16
        assert s["balanced"] in (0, 1) and (s["balanced"] == 0 or P > _sms(cuda))
    assert kernels.local_search_schedule(n, P, prec) == s
    x1 = torch.as_tensor(pop, device=cuda)
    kernels.run_local_search(x1, 6, precision=prec, **ANNEAL)
    torch.cuda.synchronize()
    assert kernels.device_status(reset=True) == 0
    assert torch.equal(x0, x1), (prec, n, P, s)

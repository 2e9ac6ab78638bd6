"""The allocation-free local search (sidon_local_search_noalloc) against the
regular entry point, through the C ABI.  Needs a B200.

It serves callers that cannot allocate device memory (a plugin inside an
application that owns every device byte, or a hot path that must not call
cudaMalloc/cudaFree): they pass only the population and the library keeps
the Adam moments in its own fixed device array.  The result must equal what
sidon_local_search produces with caller-provided moment buffers -- the same
kernel on the same inputs, so bit for bit -- on two calls in a row (the
second call reuses the array the first one left behind).  This file is
collected last on purpose.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _start(n, P, seed):
    from sidon_b200 import synth
    return synth.population("structured", n, P, seed=seed)


# (fp32, 700, 6): narrow-tile SIMT kernel; (fp32, 2048, 8): 15-output SIMT
# kernel; (bf16x3, 1000, 4): one CTA per candidate; (bf16x3, 4096, 200): more
# candidates than SMs, so the balanced-segment kernel runs with its hand-over
# flags in the library's array (P n = 819200 cells, within the limit).
@pytest.mark.parametrize("precision,n,P", [("fp32", 700, 6), ("fp32", 2048, 8),
                                           ("bf16x3", 1000, 4), ("bf16x3", 4096, 200)])
def test_noalloc_matches_regular_entry_point_twice(cuda, precision, n, P):
    from sidon_b200 import kernels
    args = (25, 4.0, 64.0, 0.02, 0.005)
    for call in range(2):
        start = _start(n, P, seed=40 + call)
        mode = torch.as_tensor(np.array([0, 1] * (P // 2), dtype=np.int32), device=cuda)
        x_ref = torch.as_tensor(start, device=cuda)
        x_new = torch.as_tensor(start, device=cuda)
        kernels.run_local_search(x_ref, *args, mode_arr=mode, precision=precision)
        kernels.run_local_search_noalloc(x_new, *args, mode_arr=mode, precision=precision)
        torch.cuda.synchronize()
        assert torch.equal(x_ref, x_new), (precision, call)
        assert not torch.equal(x_new, torch.as_tensor(start, device=cuda))


def test_noalloc_rejects_sizes_beyond_its_capacity(cuda):
    from sidon_b200 import kernels
    from sidon_b200._lib import SidonError, ERR_CAPACITY
    n = 8400
    P = kernels.NOALLOC_MAX_CELLS // n + 1
    x = torch.full((P, n), 1.0 / n, device=cuda)
    with pytest.raises(SidonError) as e:
        kernels.run_local_search_noalloc(x, 2, 2.0, 2.0, 1e-3, 1e-3)
    assert e.value.status == ERR_CAPACITY
    assert torch.equal(x, torch.full_like(x, 1.0 / n))      # untouched

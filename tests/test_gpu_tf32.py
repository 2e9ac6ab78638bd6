"""TF32x3 products on the tensor cores (tcgen05.mma kind::tf32): the
autoconvolution and the adjoint correlation of the G_p forward / backward
pair with each operand split into two TF32 parts.  Needs a B200.

Bars: b within 3e-5 of max b against fp64 and the gradient against the
long-double oracle within max(2e-3, 2e-5 p) of max |grad| -- BF16x3's bars:
the products are more exact than BF16x3's (2^-22 against 2^-18 per split
operand) but both are bound by the tensor pipe's fp32 accumulation, which
TF32 goes through twice as often (K = 8 per instruction against 16); the
measured errors are printed with -s.  The backward
with b recomputed equals the one with b stored bit for bit; beyond its
shared-memory plan the call returns SIDON_ERR_SMEM, and the fused local
search does not offer the mode (SIDON_ERR_DTYPE).
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def K():
    from sidon_b200 import kernels
    return kernels


def T(x, dev):
    return torch.as_tensor(np.ascontiguousarray(x), dtype=torch.float32, device=dev)


@pytest.mark.parametrize("n", [1, 100, 128, 129, 300, 1000, 4096, 8400])
def test_tf32x3_conv_vs_fp64(cuda, n):
    rng = np.random.default_rng(n + 7)
    a = rng.lognormal(0, 1, (2, n)).astype(np.float32)
    a[:, rng.uniform(size=n) < 1 / 3] = 0
    a[:, 0] = 8 * a.mean() + 1.0
    _, saved, b = K().lp_forward(T(a, cuda), 8.0, store_b=True, precision="tf32x3")
    _, _, b16 = K().lp_forward(T(a, cuda), 8.0, store_b=True, precision="bf16x3")
    b = b.cpu().numpy().astype(np.float64)
    b16 = b16.cpu().numpy().astype(np.float64)
    assert K().device_status(reset=True) == 0
    for p in range(2):
        ref = np.convolve(a[p].astype(np.float64), a[p].astype(np.float64))
        err = np.max(np.abs(b[p] - ref)) / ref.max()
        err16 = np.max(np.abs(b16[p] - ref)) / ref.max()
        print(f"n={n} candidate {p}: TF32x3 {err:.2e}, BF16x3 {err16:.2e} of max b")
        assert err <= 3e-5, (n, err, err16)
        assert abs(saved[p, 0].item() - ref.max()) <= 3e-5 * ref.max()


@pytest.mark.parametrize("p", [8.0, 64.0])
def test_tf32x3_gradient_vs_long_double(cuda, orc, p):
    from sidon_b200 import synth
    n = 1000
    pop = synth.population("structured", n, 3, seed=17)
    a = T(pop, cuda)
    val, saved, b = K().lp_forward(a, p, store_b=True, precision="tf32x3")
    g = K().lp_backward(a, saved, p, precision="tf32x3").cpu().numpy()
    g_stored = K().lp_backward(a, saved, p, b=b, precision="tf32x3").cpu().numpy()
    assert K().device_status(reset=True) == 0
    np.testing.assert_array_equal(g, g_stored)
    for r in range(3):
        want_g, want_v = orc.lp_grad(pop[r].astype(np.float64), p)
        assert abs(val[r].item() - want_v) <= 1e-4 * want_v
        err = np.max(np.abs(g[r] - want_g)) / np.abs(want_g).max()
        assert err <= max(2e-3, 2e-5 * p), (r, err)


def test_tf32x3_limits(cuda):
    from sidon_b200 import _lib
    big = torch.full((1, 9728), 1.0 / 9728, device=cuda)
    with pytest.raises(_lib.SidonError) as e:
        K().lp_forward(big, 8.0, precision="tf32x3")
    assert e.value.status == _lib.ERR_SMEM
    x = torch.full((2, 500), 1.0 / 500, device=cuda)
    with pytest.raises(_lib.SidonError) as e:
        K().run_local_search(x, 2, 2.0, 4.0, 1e-3, 1e-3, precision="tf32x3")
    assert e.value.status == _lib.ERR_DTYPE

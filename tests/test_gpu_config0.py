"""The plain-method case at its configured size (n = 512, one candidate:
U[0,1] heights, a third zeroed, the support gap [n/50, n/8), the endpoint
atom, the (1 + i/n) tilt; 2000 fp32 L^p-Adam steps with p 2 -> 128, lr 1e-3,
beta 0.9 / 0.999): F in fp64 before and after, the device search (fp32 SIMT
and BF16x3) against the fp32 oracle and, where oracle/_ref was built, the
reference's own fp64 CPU twin (tools/probe.cpp localSearch).  Needs a B200.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

N, STEPS = 512, 2000


def start():
    from sidon_b200 import synth
    return synth.population("structured", N, 1, seed=0)[0]


@pytest.mark.parametrize("prec,tol", [("fp32", 1e-4), ("bf16x3", 1e-3)])
def test_config0_device_search_tracks_the_oracle(cuda, orc, prec, tol):
    from sidon_b200 import kernels
    a = start()
    F0 = orc.host_f(a.astype(np.float64))
    x = torch.tensor(a[None, :], device=cuda)
    kernels.run_local_search(x, STEPS, 2.0, 128.0, 1e-3, 1e-3, precision=prec)
    got = x[0].cpu().numpy()
    Fg = kernels.run_eval(x, with_nactive=False)[0].item()
    assert (got >= 0).all() and abs(got.sum() - 1.0) < 1e-5
    assert Fg == orc.host_f(got.astype(np.float64))        # the certifying F is hostF
    want = orc.local_search(a[None, :], STEPS, 2.0, 128.0, 1e-3, 1e-3)[0]
    Fw = orc.host_f(want.astype(np.float64))
    assert Fg < F0 and Fw < F0
    assert abs(Fg - Fw) <= tol * Fw, (prec, Fg, Fw, F0)


def test_config0_against_the_reference_cpu_twin(cuda, orc):
    if not orc.have_ref():
        pytest.skip("oracle/_ref not built on this machine")
    from sidon_b200 import kernels
    a = start()
    x = torch.tensor(a[None, :], device=cuda)
    kernels.run_local_search(x, STEPS, 2.0, 128.0, 1e-3, 1e-3)
    Fg = kernels.run_eval(x, with_nactive=False)[0].item()
    r = np.ascontiguousarray(a.astype(np.float64))
    orc.ref_probe().ref_probe_local_search(r.ctypes.data, N, STEPS, 2.0, 128.0, 1e-3, 1e-3, 0.9,
                                           0.999, 0)
    Fr = orc.host_f(r)
    assert abs(Fg - Fr) <= 1e-3 * Fr, (Fg, Fr)

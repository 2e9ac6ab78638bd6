"""The reference's own GPU kernels, built unmodified for sm_100a from its
sources (oracle/_ref/libref_main.so: kLocalSearch<float>, kEval<float,double>
launched as runLocalSearch / runEval do), beside this library's kernels on
the same heights.  Needs a B200 and the built reference (skipped without
it).  Run with -s to see the timing line (the reference's SIMT step is the
second SIMT baseline of the benchmark's configuration).

Bars: the certifying evaluation equals the reference kEval bit for bit;
after 20 fp32 Adam steps F of the FP32 SIMT step and of the BF16x3 step
agree with the reference kernel's to 1e-4 relative (different tile orders
and __expf in the reference's weights).
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

N, B, STEPS = 8400, 256, 20


@pytest.fixture(scope="module")
def ref(cuda):
    import oracle
    if not oracle.have_ref():
        pytest.skip("reference not built (oracle/_ref)")
    return oracle.ref_main()


def _timed(fn):
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    fn()
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e)


def test_reference_local_search_beside_ours(cuda, ref):
    from sidon_b200 import kernels as K, synth
    pop = torch.as_tensor(synth.population("lognormal", N, B, seed=8400), device=cuda)
    x_ref, x_32, x_tc = pop.clone(), pop.clone(), pop.clone()
    mom, vel = torch.empty_like(pop), torch.empty_like(pop)
    args = (2.0, 1024.0, 1e-3, 1e-3)

    def run_ref(x, it):
        rc = ref.ref_gpu_local_search(x.data_ptr(), mom.data_ptr(), vel.data_ptr(), N, B, it,
                                      *args, None)
        assert rc == 0, rc
    run_ref(pop.clone(), 2)                               # warm-up
    t_ref = _timed(lambda: run_ref(x_ref, STEPS))
    K.run_local_search(pop.clone(), 2, *args, mom=mom, vel=vel)
    t_32 = _timed(lambda: K.run_local_search(x_32, STEPS, *args, mom=mom, vel=vel))
    K.run_local_search(pop.clone(), 2, *args, mom=mom, vel=vel, precision="bf16x3")
    t_tc = _timed(lambda: K.run_local_search(x_tc, STEPS, *args, mom=mom, vel=vel,
                                             precision="bf16x3"))
    F_ref, _ = K.run_eval(x_ref, with_nactive=False)
    F_32, _ = K.run_eval(x_32, with_nactive=False)
    F_tc, _ = K.run_eval(x_tc, with_nactive=False)
    assert torch.allclose(F_32, F_ref, rtol=1e-4, atol=0)
    assert torch.allclose(F_tc, F_ref, rtol=1e-4, atol=0)
    print(f"\nn={N} B={B}: reference kLocalSearch<float> {STEPS * 1e3 / t_ref:.1f} steps/s, "
          f"FP32 SIMT {STEPS * 1e3 / t_32:.1f} steps/s, BF16x3 {STEPS * 1e3 / t_tc:.1f} steps/s")


def test_reference_eval_bit_identical(cuda, ref):
    from sidon_b200 import kernels as K, synth
    pop = torch.as_tensor(synth.population("structured", 4096, 8, seed=9), device=cuda)
    Fr = torch.empty(8, dtype=torch.float64, device=cuda)
    Nr = torch.empty(8, dtype=torch.int32, device=cuda)
    rc = ref.ref_gpu_eval(pop.data_ptr(), 4096, 8, Fr.data_ptr(), Nr.data_ptr(), 1e-4, None)
    assert rc == 0, rc
    F, Nn = K.run_eval(pop, active_tol=1e-4)
    torch.cuda.synchronize()
    assert torch.equal(F, Fr)
    assert torch.equal(Nn, Nr)

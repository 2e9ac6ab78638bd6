"""The search driver (sidon_search, src/main.cu:400-874) end to end on small
settings: a two-level ladder, the device-side generations replayed from CUDA
graphs, the carry-over, the fp64 polish and the host recheck; and the resume
path.  Needs a B200.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def K():
    from sidon_b200 import kernels
    return kernels


def small_gen(seed=5):
    return K().generation_config(n_islands=4, elite=2, ls_iters=30, cold_iters=60, p_max=400.0,
                                 precision="bf16x3", fw_rounds=1, fw_iters=20, fw_nT=6,
                                 fw_t_max=0.3, fw_precision="bf16x3", tabu_capacity=1 << 12,
                                 seed=seed)


def test_search_two_levels_polish_and_recheck(cuda, orc):
    reports = []

    def progress(d, best):
        reports.append((d, None if best is None else best.copy()))

    best, F = K().search(ladder=(64, 128), P=32, seconds=1e9, gens_per_level=4,
                         gens_per_graph=2, polish_iters=600, polish_top=4, gen=small_gen(),
                         progress=progress)
    assert best.size == 128 and (best >= 0).all()
    hf = orc.host_f(best)
    assert F >= hf and F - hf <= 1e-13 * hf            # max(search F, host recheck)
    assert F < 1.7
    # two replays of two generations per level
    assert [(d["level"], d["n"], d["gen"]) for d, _ in reports] == [
        (0, 64, 2), (0, 64, 4), (1, 128, 2), (1, 128, 4)]
    fs = [d["best_F"] for d, _ in reports]
    assert all(b <= a for a, b in zip(fs, fs[1:]))      # the incumbent never worsens
    assert reports[-1][0]["evals"] == 8 * 32
    # the polish can only improve on the search's incumbent
    assert F <= fs[-1] * (1 + 1e-13) or np.isclose(F, hf)


def test_search_resume_drops_coarser_levels(cuda, orc):
    best, F = K().search(ladder=(64,), P=32, seconds=1e9, gens_per_level=2, gens_per_graph=2,
                         polish_iters=0, polish_top=0, gen=small_gen(7))
    assert best.size == 64
    seen = []
    best2, F2 = K().search(ladder=(32, 64), P=32, seconds=1e9, gens_per_level=2,
                           gens_per_graph=2, polish_iters=0, polish_top=0, gen=small_gen(8),
                           resume=best, progress=lambda d, b: seen.append((d["level"], d["n"])))
    assert seen == [(0, 64)]                            # the 32-cell level is skipped
    assert F2 <= orc.host_f(best) * (1 + 1e-15)         # never worse than the resumed vector
    assert best2.size == 64

"""The C-ABI library loads and exports every symbol include/sidon_b200.h
declares; host-only entry points work without a GPU.  CPU only (no kernel
launches)."""
import ctypes
import pathlib
import re
import subprocess

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "sidon_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sidon_[A-Za-z0-9_]+)\s*\(", text)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("sidon_hostF", "sidon_eval", "sidon_local_search", "sidon_frank_wolfe",
                 "sidon_refine", "sidon_island_migrate", "sidon_lp_forward", "sidon_lp_backward",
                 "sidon_certify", "sidon_smem_bytes"):
        assert must in names


def test_header_is_plain_c_and_cxx(tmp_path):
    """A C caller (cgo, ctypes stubs, a plain C driver) and a C++ caller can
    both include the header: it compiles as C99 and as C++17, and a C file
    can call an entry point and lay out the structs."""
    import shutil
    inc = str(ROOT / "include")
    src = tmp_path / "use.c"
    src.write_text(
        "#include <sidon_b200.h>\n"
        "int main(void) {\n"
        "  sidon_generation_config g = {8, 2, 4000, 20000, 20000.f, SIDON_PREC_BF16X3, 6, 500,\n"
        "                               12, 0.30f, SIDON_PREC_FP32_SIMT, 6, 1 << 16, 1ull};\n"
        "  sidon_generation_state st; sidon_anneal_config a; sidon_search_config sc;\n"
        "  (void)st; (void)a; (void)sc;\n"
        "  double h[4] = {1, 2, 2, 1};\n"
        "  return (int)(sidon_hostF(h, 4) > 0) + g.n_islands * 0;\n"
        "}\n")
    for cc, std in (("gcc", "-std=c99"), ("g++", "-std=c++17")):
        exe = shutil.which(cc)
        if exe is None:
            continue
        flags = [std] + (["-x", "c++"] if cc == "g++" else [])
        r = subprocess.run([exe, *flags, "-Wall", "-Werror", "-fsyntax-only", "-I", inc, str(src)],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr


def test_library_exports_every_declared_symbol(lib):
    import sidon_b200._lib as L
    so = pathlib.Path(L.LIB_PATH)
    out = subprocess.run(["nm", "-D", "--defined-only", str(so)], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    for name in declared_functions():
        assert name in exported, name
        assert hasattr(lib, name)
    # and the ctypes signature table covers exactly the declared set
    assert set(L.SIGNATURES) == set(declared_functions())


def test_abi_version_and_status_strings(lib):
    assert lib.sidon_abi_version() == 1
    import sidon_b200._lib as L
    assert L.status_string(0) == "ok"
    assert "shared-memory" in L.status_string(3)


@pytest.mark.parametrize("n", [512, 4096, 8400])
def test_host_entry_hostF_bitwise_reference(lib, certs, n):
    w, meta = certs[n]
    a = np.ascontiguousarray(w)
    assert lib.sidon_hostF(a.ctypes.data, a.size) == meta["ref_hostF"]


def test_host_entry_hostF_kat(lib, kat):
    for case in kat["hand"] + kat["eval257"]:
        a = np.ascontiguousarray(case["a"], dtype=np.float64)
        assert lib.sidon_hostF(a.ctypes.data, a.size) == case["F"]


def test_smem_sizers_are_monotone_and_cover_the_working_set(lib):
    import sidon_b200._lib as L
    prev = 0
    for n in (64, 512, 4096, 8400, 16384):
        s = lib.sidon_smem_bytes(L.OP_LOCAL_SEARCH, n, L.F32)
        assert s >= 4 * 3 * n                 # a + b/c at least, like localSearchSmem<float>
        assert s > prev
        prev = s
    assert lib.sidon_smem_bytes(L.OP_EVAL, 8400, L.F64) >= 8 * 8400
    assert lib.sidon_smem_bytes(L.OP_FRANK_WOLFE, 8400, L.F32) >= 4 * 5 * 8400
    assert lib.sidon_smem_bytes(L.OP_LOCAL_SEARCH, 0, L.F32) == 0
    assert lib.sidon_smem_bytes(99, 100, L.F32) == 0


def test_tensor_core_plan_fits_the_optin_up_to_9984(lib):
    """The fused tensor-core local search's shared-memory plan (heights,
    B copies, and a window ring that shares its region with the scratch)
    stays within the sm_100 per-block opt-in (227 KB) at every n of its
    range, which ends where the accumulators fill the 512 TMEM columns and
    the update's 26 cells per thread run out (n = 9984); the size query
    reports 0 beyond it."""
    import sidon_b200._lib as L
    optin = 232448
    sizes = [lib.sidon_smem_bytes(L.OP_LOCAL_SEARCH_TC, n, L.F32) for n in range(1, 9985)]
    assert all(0 < s <= optin for s in sizes)
    assert max(sizes) > optin - 4096                        # the top of the range uses it
    assert lib.sidon_smem_bytes(L.OP_LOCAL_SEARCH_TC, 9985, L.F32) == 0
    # the multi-tile ring leaves room for the kernels' static shared variables
    assert all(s <= optin - 1024 for n, s in enumerate(sizes, 1) if 1024 <= n)


def test_formats_roundtrip_with_reference_loadvec(tmp_path):
    """Our saveVec text is read back by the reference's loadVec and vice versa."""
    import oracle
    if not oracle.have_ref():
        pytest.skip("oracle/_ref not built (reference tree absent)")
    from sidon_b200 import formats
    rng = np.random.default_rng(0)
    a = rng.uniform(0, 1, 33)
    p1 = tmp_path / "ours.txt"
    formats.save_vec(p1, a, 1.2345)
    buf = np.zeros(64)
    m = oracle.ref_main().ref_loadVec(str(p1).encode(), buf.ctypes.data, 64)
    assert m == 33 and np.array_equal(buf[:33], a)
    p2 = tmp_path / "ref.txt"
    oracle.ref_main().ref_saveVec(str(p2).encode(), np.ascontiguousarray(a).ctypes.data, 33, 1.5)
    assert np.array_equal(formats.load_vec(p2), a)


def test_synth_is_deterministic_and_shaped():
    from sidon_b200 import synth
    a = synth.population("structured", 512, 3, seed=1)
    b = synth.population("structured", 512, 3, seed=1)
    assert a.dtype == np.float32 and a.shape == (3, 512)
    assert np.array_equal(a, b)
    assert np.all(a[:, 512 // 50: 512 // 8] == 0)                  # support gap
    assert np.all(a >= 0) and np.allclose(a.sum(1), 1, atol=1e-5)
    L = synth.population("lognormal", 8400, 2, seed=3)
    g0 = 8400 // 50
    assert np.all(L[:, g0: g0 + 840] == 0)
    frac0 = np.mean(L == 0)
    assert 0.3 < frac0 < 0.5


def test_polish_population_shape_and_norm():
    """Basin-hopping start of the polish: candidate 0 is the input, the rest
    are bounded multiplicative perturbations; all non-negative, sum 1."""
    from sidon_b200 import kernels
    rng = np.random.default_rng(0)
    a = rng.uniform(0, 1, 200)
    a[::3] = 0
    pop = kernels.polish_population(a, 8, seed=2)
    assert pop.shape == (8, 200)
    np.testing.assert_allclose(pop[0], a / a.sum(), rtol=0, atol=0)
    assert (pop >= 0).all()
    np.testing.assert_allclose(pop.sum(1), 1.0, rtol=1e-12)
    assert (pop[:, ::3] == 0).all()                 # zeros stay zero
    r = pop[1:, 1::3] / (a[1::3] / a.sum())
    assert np.abs(np.log(r)).max() < 0.3            # bounded perturbation

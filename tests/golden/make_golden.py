"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run in a container that has the reference tree (the argument, else the
SIDON_REFERENCE_ROOT environment variable) and oracle/_ref built
(``make -C oracle ref REF=<root>``):

    python tests/golden/make_golden.py [REFERENCE_ROOT]

Outputs (committed; the tests read only these, never the reference tree):

* certificates.npz -- for n in (512, 4096, 8400): the certificate heights,
  the stored F, the reference hostF (src/main.cu:95-105, compiled from the
  reference sources), the reference verify.py F, and the output of the
  reference ``probe --verify`` (tools/probe.cpp:146-195) as printed
  (F, M, S, argmax k, active peaks, round-off bound, as decimal strings).
* kat.json -- the self-test known answers of src/main.cu:196-288: hand
  vectors, the refine/scale-invariance vectors drawn with std::mt19937 at the
  self-test's seeds, the n=257 P=5 GPU-eval vectors (seed 3, fp32-rounded)
  and the n=128 P=4 local-search start (seed 5, U[0.1,1) floats), each with
  the reference hostF of the exact values.
* probe_ls.npz -- the reference fp64 CPU twin localSearch
  (tools/probe.cpp:62-116) on seeded inputs: start vectors, settings and
  the resulting vectors and F.
"""
from __future__ import annotations

import ctypes as C
import importlib.util
import json
import pathlib
import re
import subprocess
import sys
import tempfile

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))
import oracle  # noqa: E402

OUT = pathlib.Path(__file__).resolve().parent

# std::mt19937 + std::uniform_real_distribution draws at the self-test's seeds
# (src/main.cu:209-262); the generator program uses only the standard library.
_GEN_CPP = r"""
#include <cstdio>
#include <random>
int main() {
  { std::mt19937 rng(7); std::uniform_real_distribution<double> U(0, 1);
    for (int rep = 0; rep < 3; ++rep) { int n = 23 + rep * 11; std::printf("refine %d", n);
      for (int i = 0; i < n; ++i) std::printf(" %.17g", U(rng)); std::printf("\n"); } }
  { std::mt19937 rng(11); std::uniform_real_distribution<double> U(0, 1);
    std::printf("scale 40"); for (int i = 0; i < 40; ++i) std::printf(" %.17g", U(rng));
    std::printf("\n"); }
  { std::mt19937 rng(3); std::uniform_real_distribution<double> U(0, 1);
    for (int p = 0; p < 5; ++p) { std::printf("eval257 %d", p);
      for (int i = 0; i < 257; ++i) { double x = (p == 0) ? 1.0 : U(rng);
        std::printf(" %.17g", (double)(float)x); } std::printf("\n"); } }
  { std::mt19937 rng(5); std::uniform_real_distribution<float> U(0.1f, 1.0f);
    std::printf("ls128"); for (int i = 0; i < 128 * 4; ++i) std::printf(" %.17g", (double)U(rng));
    std::printf("\n"); }
  return 0;
}
"""


def _mt_vectors() -> dict:
    with tempfile.TemporaryDirectory() as td:
        src = pathlib.Path(td) / "gen.cpp"
        exe = pathlib.Path(td) / "gen"
        src.write_text(_GEN_CPP)
        subprocess.run(["/usr/bin/g++", "-O1", "-std=c++17", str(src), "-o", str(exe)], check=True)
        out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    vec = {"refine": [], "eval257": [], "scale": None, "ls128": None}
    for line in out.splitlines():
        parts = line.split()
        if parts[0] == "refine":
            vec["refine"].append([float(x) for x in parts[2:]])
        elif parts[0] == "scale":
            vec["scale"] = [float(x) for x in parts[2:]]
        elif parts[0] == "eval257":
            vec["eval257"].append([float(x) for x in parts[2:]])
        elif parts[0] == "ls128":
            vec["ls128"] = [float(x) for x in parts[1:]]
    return vec


def _ref_hostf(a) -> float:
    a = np.ascontiguousarray(a, dtype=np.float64)
    return oracle.ref_main().ref_hostF(a.ctypes.data, a.size)


def _probe_verify(a: np.ndarray) -> dict:
    with tempfile.TemporaryDirectory() as td:
        path = pathlib.Path(td) / "v.txt"
        a = np.ascontiguousarray(a, dtype=np.float64)
        oracle.ref_main().ref_saveVec(str(path).encode(), a.ctypes.data, a.size, 0.0)
        txt = subprocess.run([str(oracle.REF_PROBE_EXE), "--verify", str(path)], check=True,
                             capture_output=True, text=True).stdout
    def grab(pat):
        m = re.search(pat, txt)
        return m.group(1)
    return {
        "F": grab(r"F\s+=\s+(\S+)"),
        "S": grab(r"sum a_i\s+=\s+(\S+)"),
        "M": grab(r"max_k b_k\s+=\s+(\S+)"),
        "kmax": int(grab(r"at k = (\d+)")),
        "nactive": int(grab(r"active peaks\s+=\s+(\d+)")),
        "relbound": grab(r"round-off bnd\s+=\s+(\S+)"),
    }


def main(ref_root: str | None = None) -> None:
    ref = pathlib.Path(ref_root) if ref_root else oracle.REFERENCE_TREE
    if ref is None:
        raise SystemExit("give the reference root as the argument or in SIDON_REFERENCE_ROOT")
    if not oracle.have_ref():
        oracle.build(ref)
    spec = importlib.util.spec_from_file_location("ref_verify", ref / "verify.py")
    ref_verify = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ref_verify)

    arrays = {}
    meta = {}
    for n in (512, 4096, 8400):
        cert = json.loads((ref / "certificates" / f"sidon-{n}.json").read_text())
        w = np.asarray(cert["weights"], dtype=np.float64)
        arrays[f"w{n}"] = w
        pv = _probe_verify(w)
        F_py, M_py, k_py = ref_verify.ratio([float(x) for x in cert["weights"]])
        meta[str(n)] = {
            "stored_F": cert["F"],
            "non_zero_cells": cert["non_zero_cells"],
            "ref_hostF": _ref_hostf(w),
            "ref_verify_py_F": F_py,
            "ref_verify_py_kmax": k_py,
            "probe_verify": pv,
        }
    np.savez_compressed(OUT / "certificates.npz", **arrays)
    (OUT / "certificates.json").write_text(json.dumps(meta, indent=1))

    mt = _mt_vectors()
    kat = {"hand": [], "refine": [], "scale": None, "eval257": [], "ls128": None}
    for n in (4, 8, 37, 128):
        a = [1.0] * n
        kat["hand"].append({"a": a, "F": _ref_hostf(a), "want": 2.0})
    for a, want in (([1, 2, 2, 1], 80.0 / 36.0), ([1, 0, 0, 1], 4.0), ([0, 1, 0, 0], 8.0)):
        kat["hand"].append({"a": [float(x) for x in a], "F": _ref_hostf(a), "want": want})
    for a in mt["refine"]:
        a2 = np.repeat(np.asarray(a), 2)
        kat["refine"].append({"a": a, "F": _ref_hostf(a), "F_refined": _ref_hostf(a2)})
    s = mt["scale"]
    kat["scale"] = {"a": s, "F": _ref_hostf(s), "F_scaled": _ref_hostf([x * 37.5 for x in s])}
    for a in mt["eval257"]:
        kat["eval257"].append({"a": a, "F": _ref_hostf(a)})
    ls = np.asarray(mt["ls128"]).reshape(4, 128)
    kat["ls128"] = {"a": ls.tolist(), "F": [_ref_hostf(r) for r in ls],
                    "iters": 800, "p": [4.0, 300.0], "lr": [0.06, 0.002]}
    (OUT / "kat.json").write_text(json.dumps(kat))

    # reference fp64 CPU twin on seeded structured inputs
    sys.path.insert(0, str(ROOT))
    import sidon_b200.synth as synth
    cases = [(64, 300, 6.0, 400.0, 0.08, 0.002, 0), (128, 200, 8.0, 200.0, 0.05, 0.005, 0),
             (96, 150, 6.0, 100.0, 0.05, 0.01, 1)]
    ls_arrays = {}
    settings = []
    for idx, (n, iters, pA, pB, lA, lB, mode) in enumerate(cases):
        a0 = synth.population("structured", n, 1, seed=2024 + idx, normalise=True,
                              dtype=np.float64)[0]
        a = a0.copy()
        F = oracle.ref_probe().ref_probe_local_search(a.ctypes.data, n, iters, pA, pB, lA, lB,
                                                      0.9, 0.999, mode)
        ls_arrays[f"start{idx}"] = a0
        ls_arrays[f"end{idx}"] = a
        settings.append({"n": n, "iters": iters, "pA": pA, "pB": pB, "lrA": lA, "lrB": lB,
                         "mode": mode, "F": F})
    ls_arrays["settings"] = np.asarray(json.dumps(settings))
    np.savez_compressed(OUT / "probe_ls.npz", **ls_arrays)
    print("golden fixtures written to", OUT)


if __name__ == "__main__":
    main(*sys.argv[1:])

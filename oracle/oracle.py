"""ctypes wrapper over the CPU checker.

TEST INFRASTRUCTURE ONLY: tests/, the smoke check in __graft_entry__ and the
cpu_baseline / reference legs of bench.py load this module; the product path
never does.

* ``lib()``  -- the C restatement (oracle/sidon_oracle.c), built by
  ``make -C oracle``;
* ``ref_probe()`` / ``ref_main()`` / ``REF_PROBE_EXE`` -- the reference's own
  code compiled from its sources (``make -C oracle ref``), present wherever
  oracle/_ref was built (it is not rebuilt on machines without the reference
  tree).
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB = HERE / "_build" / "libsidon_oracle.so"
REF_DIR = HERE / "_ref"
REF_PROBE = REF_DIR / "libref_probe.so"
REF_MAIN = REF_DIR / "libref_main.so"
REF_PROBE_EXE = REF_DIR / "probe"
# Where the reference project's sources lie, for building oracle/_ref: the
# SIDON_REFERENCE_ROOT environment variable, or the root given to build().
# Machines without the reference (the GPU boxes) use the oracle/_ref built
# beforehand.
_env_root = os.environ.get("SIDON_REFERENCE_ROOT")
REFERENCE_TREE = pathlib.Path(_env_root) if _env_root else None

_vp, _i, _d, _f = C.c_void_p, C.c_int, C.c_double, C.c_float
_LD = C.c_longdouble

_SIG = {
    "so_hostF": (_d, [_vp, _i]),
    "so_hostF_b": (_d, [_vp, _i, _vp]),
    "so_eval": (None, [_vp, _i, _i, _d, _vp, _vp]),
    "so_verify_ld": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _vp, _vp]),
    "so_conv_f32": (None, [_vp, _vp, _vp, _i]),
    "so_corr_f32": (None, [_vp, _vp, _vp, _i]),
    "so_local_search_f32": (None, [_vp, _i, _i, _i, _f, _f, _f, _f, _f, _f, _vp, _vp, _i]),
    "so_local_search_f64": (None, [_vp, _i, _i, _i, _d, _d, _d, _d, _d, _d, _vp, _vp, _i]),
    "so_lp_step_terms_f32": (None, [_vp, _i, _f, _vp, _vp, _vp, _vp]),
    "so_lp_value_ld": (_d, [_vp, _i, _d]),
    "so_lp_grad_ld": (None, [_vp, _i, _d, _vp, _vp]),
    "so_frank_wolfe_f32": (None, [_vp, _i, _i, _i, _i, _i, _f, _f, _f, _vp]),
    "so_refine_f64": (None, [_vp, _i, _i, _vp]),
    "so_coarsen_f64": (None, [_vp, _i, _i, _vp]),
    "so_island_migrate_f32": (_i, [_vp, _i, _vp, _i, _i, _i, _vp]),
    "so_resample_f32": (None, [_vp, _i, _vp, _i]),
    "so_philox4x32": (None, [_vp, _vp, _vp]),
    "so_variation_f32": (None, [_vp, _vp, _i, _i, _vp, _vp, _vp, _vp, C.c_ulonglong,
                                C.c_ulonglong]),
    "so_support_sig_f32": (None, [_vp, _i, _i, _f, _vp, _vp]),
    "so_island_migrate_ragged_f32": (_i, [_vp, _vp, _vp, _i, _i, _i, _vp]),
    "so_certify_exact": (_d, [_vp, _i, _vp, _vp, _vp]),
    "so_exact_bk": (_d, [_vp, _i, _i]),
    "so_num_threads": (_i, []),
    "so_gen_init": (None, [_vp]),
    "so_gen_begin": (None, [_vp, _vp, _vp, _i, _i, _i, _i, _vp]),
    "so_gen_tiers": (None, [_vp, _vp, _i, _i, _i, _i, _i, _vp]),
    "so_gen_select": (None, [_vp, _vp, _i, _i, _i, _i, _i, C.c_ulonglong, _i, _i, _i, _vp, _vp,
                             _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                             _i, _vp]),
    "so_gen_post": (None, [_vp, _vp, _i, _i, _i, _vp, _vp, _vp, _vp]),
    "so_gen_credit": (None, [_vp, _i, _vp, _vp, _vp, _vp]),
}

_lib = None
_probe = None
_main = None


def build(reference_root=None) -> None:
    """Build the C restatement, and oracle/_ref when a reference tree is given
    (reference_root, else SIDON_REFERENCE_ROOT) and present."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    root = pathlib.Path(reference_root) if reference_root else REFERENCE_TREE
    if root is not None and (root / "src").exists():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF={root}"],
                       check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        for k, (r, a) in _SIG.items():
            fn = getattr(L, k)
            fn.restype = r
            fn.argtypes = a
        _lib = L
    return _lib


def have_ref() -> bool:
    return REF_PROBE.exists() and REF_MAIN.exists() and REF_PROBE_EXE.exists()


def ref_probe() -> C.CDLL:
    global _probe
    if _probe is None:
        L = C.CDLL(str(REF_PROBE))
        L.ref_probe_local_search.restype = _d
        L.ref_probe_local_search.argtypes = [_vp, _i, _i, _d, _d, _d, _d, _d, _d, _i]
        L.ref_probe_local_search_batch.restype = None
        L.ref_probe_local_search_batch.argtypes = [_vp, _i, _i, _i, _d, _d, _d, _d, _d, _d, _i, _vp]
        L.ref_probe_objective_ld.restype = _LD
        L.ref_probe_objective_ld.argtypes = [_vp, _i]
        L.ref_probe_threads.restype = _i
        _probe = L
    return _probe


def ref_main() -> C.CDLL:
    """The reference driver's host functions (loads libcudart statically linked; no GPU needed
    for hostF / loadVec / saveVec)."""
    global _main
    if _main is None:
        L = C.CDLL(str(REF_MAIN))
        L.ref_hostF.restype = _d
        L.ref_hostF.argtypes = [_vp, _i]
        L.ref_loadVec.restype = _i
        L.ref_loadVec.argtypes = [C.c_char_p, _vp, _i]
        L.ref_saveVec.restype = None
        L.ref_saveVec.argtypes = [C.c_char_p, _vp, _i, _d]
        L.ref_gpu_local_search.restype = _i
        L.ref_gpu_local_search.argtypes = [_vp, _vp, _vp, _i, _i, _i, _f, _f, _f, _f, _vp]
        L.ref_gpu_eval.restype = _i
        L.ref_gpu_eval.argtypes = [_vp, _i, _i, _vp, _vp, _d, _vp]
        L.ref_gpu_frank_wolfe.restype = _i
        L.ref_gpu_frank_wolfe.argtypes = [_vp, _i, _i, _i, _i, _i, _f, _vp]
        L.ref_gpu_generation_search.restype = _i
        L.ref_gpu_generation_search.argtypes = [_vp] * 6 + [_i] * 4 + [_f, _i, _i] + [_vp] * 8
        L.ref_gpu_generation_vary.restype = _i
        L.ref_gpu_generation_vary.argtypes = ([_vp, _vp, _i, _i] + [_vp] * 8
                                              + [C.c_ulonglong, C.c_ulonglong])
        _main = L
    return _main


# ------------------------------ numpy helpers ------------------------------
def _c(a, dtype):
    return np.ascontiguousarray(np.asarray(a, dtype=dtype))


def host_f(a) -> float:
    a = _c(a, np.float64)
    return lib().so_hostF(a.ctypes.data, a.size)


def host_f_b(a):
    a = _c(a, np.float64)
    b = np.empty(2 * a.size - 1, dtype=np.float64)
    F = lib().so_hostF_b(a.ctypes.data, a.size, b.ctypes.data)
    return F, b


def eval_pop(pop, tol=1e-4):
    pop = _c(pop, np.float64)
    P, n = pop.shape
    F = np.empty(P, np.float64)
    na = np.empty(P, np.int32)
    lib().so_eval(pop.ctypes.data, n, P, tol, F.ctypes.data, na.ctypes.data)
    return F, na


def verify_ld(a):
    a = _c(a, np.float64)
    F, M, S, rb = (_LD() for _ in range(4))
    km, na = C.c_int(), C.c_int()
    neg = lib().so_verify_ld(a.ctypes.data, a.size, C.byref(F), C.byref(M), C.byref(S),
                             C.byref(km), C.byref(na), C.byref(rb))
    return {"F": F.value, "M": M.value, "S": S.value, "kmax": km.value, "nactive": na.value,
            "relbound": rb.value, "negative": bool(neg)}


def conv_f32(x, y):
    x = _c(x, np.float32)
    y = _c(y, np.float32)
    b = np.empty(2 * x.size - 1, np.float32)
    lib().so_conv_f32(x.ctypes.data, y.ctypes.data, b.ctypes.data, x.size)
    return b


def corr_f32(a, c):
    a = _c(a, np.float32)
    cc = np.zeros(2 * a.size, np.float32)
    cc[: 2 * a.size - 1] = c
    G = np.empty(a.size, np.float32)
    lib().so_corr_f32(a.ctypes.data, cc.ctypes.data, G.ctypes.data, a.size)
    return G


def local_search(pop, iters, pS, pE, lrS, lrE, b1=0.9, b2=0.999, skip=None, mode_arr=None,
                 mode_default=0):
    """In-place on a copy; returns the new population (dtype of the input: f32 or f64)."""
    is64 = np.asarray(pop).dtype == np.float64
    out = _c(pop, np.float64 if is64 else np.float32).copy()
    P, n = out.shape
    sk = None if skip is None else _c(skip, np.int32)
    ma = None if mode_arr is None else _c(mode_arr, np.int32)
    fn = lib().so_local_search_f64 if is64 else lib().so_local_search_f32
    fn(out.ctypes.data, n, P, int(iters), pS, pE, lrS, lrE, b1, b2,
       None if sk is None else sk.ctypes.data, None if ma is None else ma.ctypes.data,
       int(mode_default))
    return out


def lp_step_terms(a, p):
    a = _c(a, np.float32)
    n = a.size
    b = np.empty(2 * n - 1, np.float32)
    c = np.empty(2 * n - 1, np.float32)
    G = np.empty(n, np.float32)
    MR = np.empty(2, np.float32)
    lib().so_lp_step_terms_f32(a.ctypes.data, n, float(p), b.ctypes.data, c.ctypes.data,
                               G.ctypes.data, MR.ctypes.data)
    return b, c, G, float(MR[0]), float(MR[1])


def lp_value(a, p) -> float:
    a = _c(a, np.float64)
    return lib().so_lp_value_ld(a.ctypes.data, a.size, float(p))


def lp_grad(a, p):
    a = _c(a, np.float64)
    g = np.empty(a.size, np.float64)
    v = C.c_double()
    lib().so_lp_grad_ld(a.ctypes.data, a.size, float(p), g.ctypes.data, C.byref(v))
    return g, v.value


def frank_wolfe(pop, rounds, pdhg, nT=12, tMax=0.30, tau_c=0.9, sig_c=0.9, skip=None):
    out = _c(pop, np.float32).copy()
    P, n = out.shape
    sk = None if skip is None else _c(skip, np.int32)
    lib().so_frank_wolfe_f32(out.ctypes.data, n, P, int(rounds), int(pdhg), int(nT), float(tMax),
                             float(tau_c), float(sig_c), None if sk is None else sk.ctypes.data)
    return out


def refine(pop):
    pop = _c(pop, np.float64)
    P, n = pop.shape
    out = np.empty((P, 2 * n), np.float64)
    lib().so_refine_f64(pop.ctypes.data, n, P, out.ctypes.data)
    return out


def coarsen(pop):
    pop = _c(pop, np.float64)
    P, n2 = pop.shape
    out = np.empty((P, n2 // 2), np.float64)
    lib().so_coarsen_f64(pop.ctypes.data, n2, P, out.ctypes.data)
    return out


def island_migrate(pop, fit, NI, k):
    pop = _c(pop, np.float32).copy()
    fit = _c(fit, np.float64).copy()
    P, n = pop.shape
    order = np.empty(P, np.int32)
    rc = lib().so_island_migrate_f32(pop.ctypes.data, n, fit.ctypes.data, P, NI, k,
                                     order.ctypes.data)
    if rc:
        raise ValueError(f"island_migrate: bad arguments ({rc})")
    return pop, fit, order


def resample(src, n):
    """Nearest-neighbour resample to n cells + fp64 renormalisation
    (src/main.cu:555-562)."""
    src = _c(src, np.float32)
    dst = np.empty(n, np.float32)
    lib().so_resample_f32(src.ctypes.data, src.size, dst.ctypes.data, n)
    return dst


def island_migrate_ragged(flat, offsets, fit, NI, k):
    flat = _c(flat, np.float32).copy()
    off = _c(offsets, np.int64)
    fit = _c(fit, np.float64).copy()
    P = off.size - 1
    order = np.empty(P, np.int32)
    rc = lib().so_island_migrate_ragged_f32(flat.ctypes.data, off.ctypes.data, fit.ctypes.data,
                                            P, NI, k, order.ctypes.data)
    if rc:
        raise ValueError(f"island_migrate_ragged: bad arguments ({rc})")
    return flat, fit, order


def philox4x32(ctr, key):
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.empty(4, np.uint32)
    lib().so_philox4x32(c.ctypes.data, k.ctypes.data, out.ctypes.data)
    return out


def variation(pop, p1, p2, op, strength, seed, gen):
    pop = _c(pop, np.float32)
    P, n = pop.shape
    p1, p2, op = (_c(x, np.int32) for x in (p1, p2, op))
    st = _c(strength, np.float32)
    out = np.empty((op.size, n), np.float32)
    lib().so_variation_f32(pop.ctypes.data, out.ctypes.data, n, op.size, p1.ctypes.data,
                           p2.ctypes.data, op.ctypes.data, st.ctypes.data, int(seed), int(gen))
    return out


def support_sig(pop, tol=0.02):
    pop = _c(pop, np.float32)
    P, n = pop.shape
    sig = np.empty(P, np.uint64)
    nnz = np.empty(P, np.int32)
    lib().so_support_sig_f32(pop.ctypes.data, n, P, float(tol), sig.ctypes.data, nnz.ctypes.data)
    return sig, nnz


def certify_exact(a):
    a = _c(a, np.float64)
    k = C.c_int()
    M = C.c_double()
    S = C.c_double()
    F = lib().so_certify_exact(a.ctypes.data, a.size, C.byref(k), C.byref(M), C.byref(S))
    return F, M.value, S.value, k.value


def exact_bk(a, k) -> float:
    a = _c(a, np.float64)
    return lib().so_exact_bk(a.ctypes.data, a.size, int(k))


# ----------------------- memetic generation policy -------------------------
class GenState(C.Structure):
    """struct sidon_generation_state (include/sidon_b200.h), for the oracle."""

    _fields_ = [
        ("best_F", _d), ("level_best_F", _d),
        ("op_weight", _d * 14), ("op_use", _d * 14), ("op_win", _d * 14),
        ("flop", _d),
        ("ls_steps", C.c_longlong), ("evals", C.c_longlong), ("fw_steps", C.c_longlong),
        ("gen", _i), ("level", _i), ("n", _i), ("since_improve", _i),
        ("best_n", _i), ("best_slot", _i), ("improved", _i),
        ("best_nactive", _i), ("best_nnz", _i),
        ("n_cold", _i), ("n_med", _i),
        ("cells", _i), ("status", _i), ("pad_", _i),
    ]

    def as_dict(self) -> dict:
        out = {}
        for k, _ in self._fields_:
            if k == "pad_":
                continue
            x = getattr(self, k)
            out[k] = list(x) if k.startswith("op_") else x
        return out


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class GenerationPolicy:
    """The generation loop's selection policy on the host (so_gen_*): the
    state, the operator record, the descent modes and the tabu list."""

    def __init__(self, P: int, n_islands: int, elite: int, tabu_tenure: int, seed: int,
                 n_max: int, tabu_list: int = 1 << 16):
        self.P, self.NI, self.PI = P, n_islands, P // n_islands
        self.elite, self.tenure, self.seed = elite, tabu_tenure, seed
        self.s = GenState()
        lib().so_gen_init(C.byref(self.s))
        self.cur_op = np.zeros(P, np.int32)
        self.mode = np.zeros(P, np.int32)
        self.best_row = np.zeros(n_max, np.float32)
        self.tcap = tabu_list
        self.tkey = np.zeros(tabu_list, np.uint64)
        self.tbest = np.zeros(tabu_list, np.float64)
        self.thits = np.zeros(tabu_list, np.int32)
        self.tcount = np.zeros(1, np.int32)
        self.var_gen = np.zeros(1, np.uint64)
        self.n = 0

    def begin_level(self, n: int, level: int, seed_op=None) -> None:
        keep = None if seed_op is None else _c(seed_op, np.int32)
        so = None if keep is None else _p(keep)
        lib().so_gen_begin(C.byref(self.s), _p(self.cur_op), _p(self.mode), self.P, self.PI, n,
                           level, so)
        self.n = n

    def set_best(self, row, F: float) -> None:
        row = _c(row, np.float32)
        self.best_row[:row.size] = row
        self.s.best_F = F
        self.s.best_n = row.size

    def tiers(self, cold: int, med: int, warm: int) -> np.ndarray:
        skip = np.zeros((3, self.P), np.int32)
        lib().so_gen_tiers(C.byref(self.s), _p(self.cur_op), self.P, self.n, cold, med, warm,
                           _p(skip))
        return skip

    def select(self, pop: np.ndarray, fit, nact, sig, nnz, fw_ran: int, fw_rounds: int,
               fw_iters: int) -> dict:
        """pop: host fp32 [P][n], updated in place (migration); sig updated."""
        P = self.P
        fit = _c(fit, np.float64)
        nact = _c(nact, np.int32)
        nnz = _c(nnz, np.int32)
        out = {k: np.zeros(P, t) for k, t in (("parent_fit", np.float64), ("rank", np.int32),
                                               ("p1", np.int32), ("p2", np.int32),
                                               ("op", np.int32), ("strength", np.float32))}
        lib().so_gen_select(C.byref(self.s), _p(pop), self.n, P, self.NI, self.elite,
                            self.tenure, self.seed & 0xFFFFFFFFFFFFFFFF, int(fw_ran),
                            int(fw_rounds), int(fw_iters), _p(fit), _p(nact), _p(sig), _p(nnz),
                            _p(out["parent_fit"]), _p(out["rank"]), _p(out["p1"]),
                            _p(out["p2"]), _p(out["op"]), _p(out["strength"]),
                            _p(self.best_row), _p(self.tkey), _p(self.tbest), _p(self.thits),
                            _p(self.tcount), self.tcap, _p(self.var_gen))
        self.plan = out
        return out

    def post(self, pop: np.ndarray) -> None:
        pl = self.plan
        lib().so_gen_post(C.byref(self.s), _p(pop), self.n, self.P, self.PI, _p(pl["op"]),
                          _p(self.cur_op), _p(pl["rank"]), _p(self.best_row))

    def credit(self, child_fit) -> None:
        pl = self.plan
        child_fit = _c(child_fit, np.float64)
        lib().so_gen_credit(C.byref(self.s), self.P, _p(pl["op"]), _p(pl["p1"]), _p(child_fit),
                            _p(pl["parent_fit"]))

    def tabu(self) -> dict:
        """signature -> (best F, revisits)."""
        k = int(self.tcount[0])
        return {int(self.tkey[i]): (float(self.tbest[i]), int(self.thits[i])) for i in range(k)}

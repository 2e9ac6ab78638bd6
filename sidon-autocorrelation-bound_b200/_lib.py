"""ctypes binding of ``libsidon_b200.so`` (the C ABI in include/sidon_b200.h).

There is no fallback: if the library is missing or cannot be loaded, every
entry point raises.  ``load(build=True)`` compiles it first (nvcc, sm_100a).
"""
from __future__ import annotations

import ctypes as C
import pathlib
import threading

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "libsidon_b200.so"

# status codes (enum sidon_status)
OK, ERR_ARG, ERR_N, ERR_SMEM, ERR_CUDA, ERR_DTYPE, ERR_NONFINITE, ERR_TIMEOUT, ERR_DEVICE = range(9)
ERR_CAPACITY = 9
F32, F64 = 0, 1
PREC_FP32_SIMT, PREC_BF16X1, PREC_BF16X3, PREC_FP64_SIMT, PREC_TF32X3 = 0, 1, 2, 3, 4
OP_LOCAL_SEARCH, OP_EVAL, OP_FRANK_WOLFE, OP_LOCAL_SEARCH_TC = 0, 1, 2, 3

_vp, _i, _d, _f, _sz = C.c_void_p, C.c_int, C.c_double, C.c_float, C.c_size_t

# name -> (restype, argtypes); every symbol declared in include/sidon_b200.h
SIGNATURES = {
    "sidon_status_string": (C.c_char_p, [_i]),
    "sidon_last_cuda_error": (_i, []),
    "sidon_abi_version": (_i, []),
    "sidon_device_status": (_i, [_i]),
    "sidon_set_wait_limit": (_i, [C.c_longlong]),
    "sidon_smem_bytes": (_sz, [_i, _i, _i]),
    "sidon_max_n": (_i, [_i, _i]),
    "sidon_hostF": (_d, [_vp, _i]),
    "sidon_eval": (_i, [_vp, _i, _i, _i, _vp, _vp, _d, _vp]),
    "sidon_certify": (_i, [_vp, _i, _i, _i, _vp, _vp, _vp, _vp, _vp]),
    "sidon_local_search": (_i, [_vp, _vp, _vp, _vp, _vp, _i, _i, _i, _d, _d, _d, _d, _d, _d, _i,
                                _i, _i, _vp]),
    "sidon_local_search_workspace_bytes": (_sz, [_i, _i, _i, _i]),
    "sidon_local_search_ws": (_i, [_vp, _vp, _vp, _vp, _vp, _i, _i, _i, _d, _d, _d, _d, _d, _d,
                                   _i, _i, _i, _vp, _sz, _vp]),
    "sidon_local_search_noalloc": (_i, [_vp, _vp, _vp, _i, _i, _i, _d, _d, _d, _d, _d, _d, _i, _i,
                                        _vp]),
    "sidon_lp_forward": (_i, [_vp, _i, _i, _d, _vp, _vp, _vp, _i, _vp]),
    "sidon_lp_backward": (_i, [_vp, _vp, _vp, _i, _i, _d, _vp, _i, _vp]),
    "sidon_frank_wolfe": (_i, [_vp, _vp, _i, _i, _i, _i, _i, _f, _f, _f, _vp]),
    "sidon_frank_wolfe_tc": (_i, [_vp, _vp, _vp, _vp, _i, _i, _i, _i, _i, _f, _f, _f, _i, _vp]),
    "sidon_refine": (_i, [_vp, _i, _i, _vp, _i, _vp]),
    "sidon_coarsen": (_i, [_vp, _i, _i, _vp, _i, _vp]),
    "sidon_resample": (_i, [_vp, _i, _i, _vp, _i, _i, _vp]),
    "sidon_island_migrate": (_i, [_vp, _i, _vp, _i, _i, _i, _vp, _vp]),
    "sidon_variation": (_i, [_vp, _vp, _i, _i, _i, _vp, _vp, _vp, _vp, C.c_ulonglong,
                             C.c_ulonglong, _vp]),
    "sidon_support_sig": (_i, [_vp, _i, _i, _i, _f, _vp, _vp, _vp]),
    "sidon_polish": (_i, [_vp, _vp, _vp, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp]),
    "sidon_large_workspace_bytes": (_sz, [_i, _i, _i, _i]),
    "sidon_autotune_large": (_i, [_i, _i, _i, _vp, _vp]),
    "sidon_autotune_local_search": (_i, [_i, _i, _i, _vp]),
    "sidon_local_search_schedule": (_i, [_i, _i, _i, _vp]),
    "sidon_local_search_large": (_i, [_vp, _vp, _vp, _vp, _vp, _i, _i, _i, _d, _d, _d, _d, _d, _d,
                                      _i, _i, _i, _vp, _sz, _vp]),
    "sidon_frank_wolfe_large": (_i, [_vp, _vp, _i, _i, _i, _i, _i, _f, _f, _f, _i, _i, _vp, _sz,
                                     _vp]),
    "sidon_certify_workspace_bytes": (_sz, [_i]),
    "sidon_certify_large": (_i, [_vp, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp]),
    "sidon_ragged_order": (_i, [_vp, _i, _vp, _vp]),
    "sidon_local_search_ragged": (_i, [_vp, _vp, _vp, _vp, _vp, _i, _vp, _vp, _i, _i, _d, _d, _d,
                                       _d, _d, _d, _i, _i, _vp]),
    "sidon_eval_ragged": (_i, [_vp, _i, _vp, _vp, _i, _i, _vp, _vp, _d, _vp]),
    "sidon_frank_wolfe_ragged": (_i, [_vp, _vp, _vp, _i, _vp, _i, _i, _i, _i, _f, _f, _f, _vp]),
    "sidon_frank_wolfe_tc_ragged": (_i, [_vp, _vp, _vp, _vp, _vp, _i, _vp, _i, _i, _i, _i, _f,
                                         _f, _f, _i, _vp]),
    "sidon_island_migrate_ragged": (_i, [_vp, _vp, _vp, _i, _i, _i, _vp, _vp]),
    "sidon_anneal": (_i, [_vp, _vp, _vp, _vp, _vp, _i, _i, _vp, _vp, _vp, _vp]),
    "sidon_anneal_capture": (_i, [_vp, _vp, _vp, _vp, _vp, _i, _i, _vp, _vp, _vp, _vp]),
    "sidon_graph_launch": (_i, [_vp, _vp]),
    "sidon_graph_destroy": (_i, [_vp]),
    "sidon_generation_workspace_bytes": (_sz, [_i, _i, _i]),
    "sidon_generation_create": (_i, [_vp, _sz, _i, _i, _vp, _vp, _vp]),
    "sidon_generation_destroy": (_i, [_vp]),
    "sidon_generation_views_of": (_i, [_vp, _vp]),
    "sidon_generation_begin_level": (_i, [_vp, _i, _i, _vp, _vp]),
    "sidon_generation_set_best": (_i, [_vp, _vp, _i, _d, _vp]),
    "sidon_generation_step": (_i, [_vp, _vp, _vp]),
    "sidon_generation_capture": (_i, [_vp, _vp, _i, _vp]),
    "sidon_generation_read_state": (_i, [_vp, _vp, _vp]),
    "sidon_seed_level": (_i, [_vp, _vp, _i, _i, _i, _vp, _i, C.c_ulonglong]),
    "sidon_search": (_i, [_vp, _vp, _i, _vp, _i, _vp, _vp, _vp, _vp]),
}


class LsSchedule(C.Structure):
    """struct sidon_ls_schedule."""

    _fields_ = [("lane_tile", _i), ("ring_tiles", _i), ("balanced", _i), ("ms_per_step", _f),
                ("tuned", _i)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class AnnealConfig(C.Structure):
    """struct sidon_anneal_config."""

    _fields_ = [
        ("steps", _i),
        ("p_start", _d), ("p_end", _d),
        ("lr_start", _d), ("lr_end", _d),
        ("beta1", _d), ("beta2", _d),
        ("precision", _i),
        ("fw_every", _i),
        ("fw_rounds", _i), ("pdhg_iters", _i), ("fw_nT", _i),
        ("fw_t_max", _f), ("fw_tau", _f), ("fw_sigma", _f),
        ("fw_precision", _i),
        ("n_islands", _i),
        ("migrate_every", _i),
        ("k_migrate", _i),
    ]


class GenerationConfig(C.Structure):
    """struct sidon_generation_config."""

    _fields_ = [
        ("n_islands", _i), ("elite", _i),
        ("ls_iters", _i), ("cold_iters", _i),
        ("p_max", _f),
        ("precision", _i),
        ("fw_rounds", _i), ("fw_iters", _i), ("fw_nT", _i),
        ("fw_t_max", _f),
        ("fw_precision", _i),
        ("tabu_tenure", _i), ("tabu_capacity", _i),
        ("seed", C.c_ulonglong),
    ]


NOPS = 14


class GenerationState(C.Structure):
    """struct sidon_generation_state."""

    _fields_ = [
        ("best_F", _d), ("level_best_F", _d),
        ("op_weight", _d * NOPS), ("op_use", _d * NOPS), ("op_win", _d * NOPS),
        ("flop", _d),
        ("ls_steps", C.c_longlong), ("evals", C.c_longlong), ("fw_steps", C.c_longlong),
        ("gen", _i), ("level", _i), ("n", _i), ("since_improve", _i),
        ("best_n", _i), ("best_slot", _i), ("improved", _i),
        ("best_nactive", _i), ("best_nnz", _i),
        ("n_cold", _i), ("n_med", _i),
        ("cells", _i), ("status", _i), ("pad_", _i),
    ]


class GenerationViews(C.Structure):
    """struct sidon_generation_views (device pointers into the workspace)."""

    _fields_ = [(k, _vp) for k in (
        "fit", "parent_fit", "child_fit", "nactive", "sig", "nnz", "p1", "p2", "op", "strength",
        "cur_op", "mode", "rank", "tier_skip", "best_row", "state", "tabu_key", "tabu_best",
        "tabu_hits", "tabu_used")]


class SearchProgress(C.Structure):
    """struct sidon_search_progress."""

    _fields_ = [
        ("seconds", _d), ("level", _i), ("n", _i), ("gen", _i), ("improved", _i),
        ("best_F", _d), ("level_best_F", _d),
        ("evals", C.c_longlong), ("ls_steps", C.c_longlong), ("fw_steps", C.c_longlong),
        ("pflop", _d), ("cells", _i), ("best_nactive", _i), ("best_nnz", _i),
        ("n_cold", _i), ("n_med", _i),
    ]


SEARCH_CALLBACK = C.CFUNCTYPE(None, C.POINTER(SearchProgress), C.POINTER(_d), _i, _vp)


class SearchConfig(C.Structure):
    """struct sidon_search_config."""

    _fields_ = [
        ("ladder", C.POINTER(_i)), ("n_levels", _i), ("P", _i), ("seconds", _d),
        ("gens_per_level", _i), ("gens_per_graph", _i), ("polish_iters", _i),
        ("polish_top", _i), ("gen", GenerationConfig),
    ]


_lock = threading.Lock()
_lib: C.CDLL | None = None


class SidonError(RuntimeError):
    """A non-zero status from the C ABI."""

    def __init__(self, fn: str, status: int, cuda_error: int = 0):
        self.status = status
        self.cuda_error = cuda_error
        msg = f"{fn}: {status_string(status)} (status {status})"
        if status == ERR_CUDA:
            msg += f", cudaError {cuda_error}"
        super().__init__(msg)


def load(build: bool = False) -> C.CDLL:
    """Load (optionally building first) the CUDA library; raises if absent."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if build:
            from . import build as _b
            _b.build()
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH.name} is not built; run `python sidon-autocorrelation-bound_b200/build.py` "
                "(no CPU fallback exists for the sidon_b200 kernels)")
        lib = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def status_string(status: int) -> str:
    return load().sidon_status_string(status).decode()


def call(name: str, *args) -> None:
    """Invoke an int-returning entry point and raise SidonError on failure."""
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc != OK:
        raise SidonError(name, rc, lib.sidon_last_cuda_error() if rc == ERR_CUDA else 0)

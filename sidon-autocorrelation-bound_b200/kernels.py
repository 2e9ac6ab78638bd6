"""Host-side mirror of the reference operator surface (src/kernels.cuh plus
the launch helpers and hostF of src/main.cu) over the C ABI.

Tensors are torch CUDA tensors (device memory and streams only); every call
goes through libsidon_b200.so.  Names and argument meaning follow the
reference: ``local_search_smem`` <-> ``localSearchSmem<T>``,
``run_local_search`` <-> ``runLocalSearch``, ``run_eval`` <-> ``runEval``,
``run_frank_wolfe`` <-> ``runFrankWolfe``, ``host_f`` <-> ``hostF``.  Where
the reference aborts the process (``CUDA_OK``, src/kernels.cuh:20-28) these
raise ``SidonError``; where ``runFrankWolfe`` returns false
(src/main.cu:173) ``run_frank_wolfe`` returns False.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import SidonError

PRECISIONS = {
    "fp32": _lib.PREC_FP32_SIMT,
    "bf16x1": _lib.PREC_BF16X1,
    "bf16x3": _lib.PREC_BF16X3,
    "fp64": _lib.PREC_FP64_SIMT,
    "tf32x3": _lib.PREC_TF32X3,
}


def _dtype_code(t: torch.Tensor) -> int:
    if t.dtype == torch.float32:
        return _lib.F32
    if t.dtype == torch.float64:
        return _lib.F64
    raise TypeError(f"heights must be float32 or float64, got {t.dtype}")


def _dev(t: torch.Tensor, name: str, dtype=None) -> int:
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if dtype is not None and t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, got {t.dtype}")
    return t.data_ptr()


def _opt(t, name, dtype=None) -> int | None:
    return None if t is None else _dev(t, name, dtype)


def _stream(stream) -> int | None:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream or None


def _pop_shape(pop: torch.Tensor) -> tuple[int, int]:
    if pop.dim() != 2:
        raise ValueError("population must be [P, n]")
    return pop.shape[1], pop.shape[0]


# ------------------------------ smem sizers --------------------------------
def local_search_smem(n: int, dtype=torch.float32, precision: str | None = None) -> int:
    """Bytes of dynamic shared memory per candidate (src/kernels.cuh:161-162)."""
    if precision in ("bf16x1", "bf16x3"):
        return _lib.load().sidon_smem_bytes(_lib.OP_LOCAL_SEARCH_TC, n, _lib.F32)
    code = _lib.F32 if dtype == torch.float32 else _lib.F64
    return _lib.load().sidon_smem_bytes(_lib.OP_LOCAL_SEARCH, n, code)


def eval_smem(n: int) -> int:
    """src/kernels.cuh:379-380 (evalSmem<double>)."""
    return _lib.load().sidon_smem_bytes(_lib.OP_EVAL, n, _lib.F64)


def fw_smem(n: int) -> int:
    """src/kernels.cuh:405-406 (fwSmem<float>)."""
    return _lib.load().sidon_smem_bytes(_lib.OP_FRANK_WOLFE, n, _lib.F32)


def max_n(op: int, dtype_code: int = _lib.F32) -> int:
    return _lib.load().sidon_max_n(op, dtype_code)


# ------------------------------ host oracle --------------------------------
def device_status(reset: bool = False) -> int:
    """The device-side status word of the tensor-core kernels (0, or the first
    SIDON_ERR_TIMEOUT / SIDON_ERR_NONFINITE since the last reset)."""
    rc = _lib.load().sidon_device_status(1 if reset else 0)
    if rc < 0:
        raise SidonError("sidon_device_status", rc)
    return rc


def set_wait_limit(cycles: int = 0) -> None:
    """Clock-cycle limit of the kernels' bounded waits (0: the default 2^31)."""
    _lib.call("sidon_set_wait_limit", int(cycles))


def host_f(a) -> float:
    """fp64 F on the host, bit-identical to hostF (src/main.cu:95-105)."""
    arr = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    return _lib.load().sidon_hostF(arr.ctypes.data, arr.size)


# ------------------------------ operators ----------------------------------
def local_search_workspace(n: int, P: int, precision: str = "bf16x3", device="cuda",
                           dtype=torch.float32) -> torch.Tensor | None:
    """Workspace of run_local_search's balanced-segment form (None if the call
    needs none)."""
    code = _lib.F32 if dtype == torch.float32 else _lib.F64
    nb = _lib.load().sidon_local_search_workspace_bytes(n, P, code, PRECISIONS[precision])
    return torch.empty(nb, dtype=torch.uint8, device=device) if nb else None


def run_local_search(pop: torch.Tensor, iters: int, p_start: float, p_end: float,
                     lr_start: float, lr_end: float, mode_arr: torch.Tensor | None = None,
                     skip: torch.Tensor | None = None, mom: torch.Tensor | None = None,
                     vel: torch.Tensor | None = None, beta1: float = 0.9, beta2: float = 0.999,
                     mode_default: int = 0, precision: str | None = None, stream=None,
                     workspace: torch.Tensor | None = None, balanced: bool = True) -> None:
    """L^p-annealed projected Adam / mirror descent on every non-skipped
    candidate, in place (kLocalSearch + runLocalSearch,
    src/kernels.cuh:177-289, src/main.cu:152-159).

    With ``balanced`` (default) a tensor-core batch of more candidates than
    SMs runs as balanced step segments through sidon_local_search_ws, its
    flag words in ``workspace`` (allocated here when None); ``balanced=False``
    calls sidon_local_search, one CTA per candidate.  Results are the same
    bit for bit."""
    n, P = _pop_shape(pop)
    code = _dtype_code(pop)
    if precision is None:
        precision = "fp32" if code == _lib.F32 else "fp64"
    if mom is None:
        mom = torch.empty_like(pop)
    if vel is None:
        vel = torch.empty_like(pop)
    args = (_dev(pop, "pop"), _dev(mom, "mom", pop.dtype), _dev(vel, "vel", pop.dtype),
            _opt(skip, "skip", torch.int32), _opt(mode_arr, "mode_arr", torch.int32), n, P,
            int(iters), float(p_start), float(p_end), float(lr_start), float(lr_end),
            float(beta1), float(beta2), int(mode_default), code, PRECISIONS[precision])
    nb = _lib.load().sidon_local_search_workspace_bytes(n, P, code, PRECISIONS[precision])
    if not balanced or nb == 0:
        _lib.call("sidon_local_search", *args, _stream(stream))
        return
    if workspace is None:
        workspace = torch.empty(nb, dtype=torch.uint8, device=pop.device)
        if stream is not None:
            workspace.record_stream(stream)      # freed here, in use on `stream`
    _dev(workspace, "workspace")
    _lib.call("sidon_local_search_ws", *args, workspace.data_ptr(), workspace.numel(),
              _stream(stream))


# P * n limit of run_local_search_noalloc (the library's fixed moment array)
NOALLOC_MAX_CELLS = 1 << 20


def run_local_search_noalloc(pop: torch.Tensor, iters: int, p_start: float, p_end: float,
                             lr_start: float, lr_end: float, mode_arr: torch.Tensor | None = None,
                             skip: torch.Tensor | None = None, beta1: float = 0.9,
                             beta2: float = 0.999, mode_default: int = 0, precision: str = "fp32",
                             stream=None) -> None:
    """run_local_search for callers that cannot allocate device memory: only
    the population is passed; the Adam moments live in a fixed device array
    inside the library (P * n <= NOALLOC_MAX_CELLS).  Calls share that array,
    so calls overlapping on the GPU race on it.  fp32 heights only."""
    n, P = _pop_shape(pop)
    _lib.call("sidon_local_search_noalloc", _dev(pop, "pop", torch.float32),
              _opt(skip, "skip", torch.int32), _opt(mode_arr, "mode_arr", torch.int32), n, P,
              int(iters), float(p_start), float(p_end), float(lr_start), float(lr_end),
              float(beta1), float(beta2), int(mode_default), PRECISIONS[precision],
              _stream(stream))


def run_eval(pop: torch.Tensor, active_tol: float = 1e-4, with_nactive: bool = True,
             out_F: torch.Tensor | None = None, out_nactive: torch.Tensor | None = None,
             stream=None):
    """Certifying fp64 F per candidate (+ active-peak counts) (kEval + runEval,
    src/kernels.cuh:301-377, src/main.cu:161-166).  Returns (F, nactive|None)."""
    n, P = _pop_shape(pop)
    code = _dtype_code(pop)
    if out_F is None:
        out_F = torch.empty(P, dtype=torch.float64, device=pop.device)
    if with_nactive and out_nactive is None:
        out_nactive = torch.empty(P, dtype=torch.int32, device=pop.device)
    _lib.call("sidon_eval", _dev(pop, "pop"), code, n, P, _dev(out_F, "out_F", torch.float64),
              _opt(out_nactive if with_nactive else None, "out_nactive", torch.int32),
              float(active_tol), _stream(stream))
    return out_F, (out_nactive if with_nactive else None)


def certify(pop: torch.Tensor, stream=None):
    """Exact certification (F, M, S, argmax k) per candidate; F is split-invariant."""
    n, P = _pop_shape(pop)
    code = _dtype_code(pop)
    dev = pop.device
    F = torch.empty(P, dtype=torch.float64, device=dev)
    M = torch.empty(P, dtype=torch.float64, device=dev)
    S = torch.empty(P, dtype=torch.float64, device=dev)
    K = torch.empty(P, dtype=torch.int32, device=dev)
    try:
        _lib.call("sidon_certify", _dev(pop, "pop"), code, n, P, F.data_ptr(), M.data_ptr(),
                  S.data_ptr(), K.data_ptr(), _stream(stream))
    except SidonError as e:
        if e.status != _lib.ERR_SMEM:
            raise
        return certify_large(pop, stream)     # beyond shared memory: streamed + list path
    return F, M, S, K


def run_frank_wolfe(pop: torch.Tensor, rounds: int, pdhg_iters: int, nT: int = 12,
                    t_max: float = 0.30, skip: torch.Tensor | None = None, tau: float = 0.0,
                    sigma: float = 0.0, stream=None) -> bool:
    """Chambolle-Pock Frank-Wolfe step in place (kFrankWolfe + runFrankWolfe,
    src/kernels.cuh:408-532, src/main.cu:170-178).  Returns False when the
    candidate does not fit shared memory, like the reference."""
    n, P = _pop_shape(pop)
    try:
        _lib.call("sidon_frank_wolfe", _dev(pop, "pop", torch.float32),
                  _opt(skip, "skip", torch.int32), n, P, int(rounds), int(pdhg_iters), int(nT),
                  float(t_max), float(tau), float(sigma), _stream(stream))
    except SidonError as e:
        if e.status == _lib.ERR_SMEM:
            return False
        raise
    return True


def run_frank_wolfe_tc(pop: torch.Tensor, rounds: int, pdhg_iters: int, nT: int = 12,
                       t_max: float = 0.30, skip: torch.Tensor | None = None, tau: float = 0.0,
                       sigma: float = 0.0, precision: str = "bf16x3",
                       g_scratch: torch.Tensor | None = None,
                       gbar_scratch: torch.Tensor | None = None, stream=None) -> None:
    """run_frank_wolfe with the Chambolle-Pock convolutions on the tensor cores."""
    n, P = _pop_shape(pop)
    if g_scratch is None:
        g_scratch = torch.empty_like(pop)
    if gbar_scratch is None:
        gbar_scratch = torch.empty_like(pop)
    _lib.call("sidon_frank_wolfe_tc", _dev(pop, "pop", torch.float32),
              _dev(g_scratch, "g_scratch", torch.float32),
              _dev(gbar_scratch, "gbar_scratch", torch.float32), _opt(skip, "skip", torch.int32),
              n, P, int(rounds), int(pdhg_iters), int(nT), float(t_max), float(tau), float(sigma),
              PRECISIONS[precision], _stream(stream))


def refine(pop: torch.Tensor, out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    """n -> 2n cell split (kRefine, src/kernels.cuh:538-547)."""
    n, P = _pop_shape(pop)
    if out is None:
        out = torch.empty((P, 2 * n), dtype=pop.dtype, device=pop.device)
    _lib.call("sidon_refine", _dev(pop, "pop"), n, P, _dev(out, "out", pop.dtype),
              _dtype_code(pop), _stream(stream))
    return out


def coarsen(pop: torch.Tensor, out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    """2n -> n pairwise average (kCoarsen, src/kernels.cuh:550-557)."""
    n2, P = _pop_shape(pop)
    if out is None:
        out = torch.empty((P, n2 // 2), dtype=pop.dtype, device=pop.device)
    _lib.call("sidon_coarsen", _dev(pop, "pop"), n2, P, _dev(out, "out", pop.dtype),
              _dtype_code(pop), _stream(stream))
    return out


def resample(pop: torch.Tensor, n: int, normalise: bool = True,
             out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    """Nearest-neighbour resample of every row to n cells, optionally
    normalised to sum 1 (src/main.cu:496-497, 555-562)."""
    m, P = _pop_shape(pop)
    if out is None:
        out = torch.empty((P, int(n)), dtype=torch.float32, device=pop.device)
    _lib.call("sidon_resample", _dev(pop, "pop", torch.float32), m, P,
              _dev(out, "out", torch.float32), int(n), int(bool(normalise)), _stream(stream))
    return out


def lp_forward(a: torch.Tensor, p: float, store_b: bool = False, precision: str = "fp32",
               stream=None):
    """G_p(a) = 2n ||a*a||_p / (sum a)^2 per row.  Returns (value, saved, b|None)."""
    n, P = _pop_shape(a)
    dev = a.device
    value = torch.empty(P, dtype=torch.float32, device=dev)
    saved = torch.empty((P, 4), dtype=torch.float32, device=dev)
    b = torch.empty((P, 2 * n - 1), dtype=torch.float32, device=dev) if store_b else None
    _lib.call("sidon_lp_forward", _dev(a, "a", torch.float32), n, P, float(p), value.data_ptr(),
              saved.data_ptr(), None if b is None else b.data_ptr(), PRECISIONS[precision],
              _stream(stream))
    return value, saved, b


def lp_backward(a: torch.Tensor, saved: torch.Tensor, p: float, b: torch.Tensor | None = None,
                precision: str = "fp32", stream=None) -> torch.Tensor:
    """dG_p/da per row; b recomputed from a unless a stored b is given."""
    n, P = _pop_shape(a)
    grad = torch.empty_like(a)
    _lib.call("sidon_lp_backward", _dev(a, "a", torch.float32), _dev(saved, "saved", torch.float32),
              _opt(b, "b", torch.float32), n, P, float(p), grad.data_ptr(), PRECISIONS[precision],
              _stream(stream))
    return grad


def island_migrate(pop: torch.Tensor, fit: torch.Tensor, n_islands: int, k: int = 1,
                   order: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    """Rank each island by fit and migrate best-of-i over worst-of-(i+1)
    (src/main.cu:676-692), in place on pop and fit.  Returns the ranking."""
    n, P = _pop_shape(pop)
    if order is None:
        order = torch.empty(P, dtype=torch.int32, device=pop.device)
    _lib.call("sidon_island_migrate", _dev(pop, "pop", torch.float32), n,
              _dev(fit, "fit", torch.float64), P, int(n_islands), int(k),
              _dev(order, "order", torch.int32), _stream(stream))
    return order


# ------------------------- variation and signatures -------------------------
VARIATION_OPS = {
    "blend": 0, "segment": 1, "lognormal": 2, "smooth": 3, "gaussian": 4, "sparsify": 5,
    "reflect": 6, "shift": 7, "splice": 8, "restart": 9, "spike": 10, "structured": 11,
    "gap": 12, "atom": 13, "clone": 20,
}


def variation(pop: torch.Tensor, p1, p2, op, strength, seed: int, gen: int,
              out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    """Offspring of the variation operators (kVariation, src/kernels.cuh:558-801):
    row j = operator op[j] on parents p1[j], p2[j] with strength[j], sum 1."""
    n, P = _pop_shape(pop)
    dev = pop.device
    p1, p2, op = (torch.as_tensor(x, dtype=torch.int32, device=dev).contiguous()
                  for x in (p1, p2, op))
    st = torch.as_tensor(strength, dtype=torch.float32, device=dev).contiguous()
    if out is None:
        out = torch.empty((op.numel(), n), dtype=pop.dtype, device=dev)
    _lib.call("sidon_variation", _dev(pop, "pop"), _dev(out, "out", pop.dtype),
              _dtype_code(pop), n, op.numel(), p1.data_ptr(), p2.data_ptr(), op.data_ptr(),
              st.data_ptr(), int(seed) & (2**64 - 1), int(gen) & (2**64 - 1), _stream(stream))
    return out


def support_sig(pop: torch.Tensor, tol: float = 0.02, stream=None):
    """(signature uint64 as int64 [P], nnz int32 [P]) (kSupportSig + runSig,
    src/kernels.cuh:803-849, src/main.cu:180-184)."""
    n, P = _pop_shape(pop)
    sig = torch.empty(P, dtype=torch.int64, device=pop.device)
    nnz = torch.empty(P, dtype=torch.int32, device=pop.device)
    _lib.call("sidon_support_sig", _dev(pop, "pop"), _dtype_code(pop), n, P, float(tol),
              sig.data_ptr(), nnz.data_ptr(), _stream(stream))
    return sig, nnz


# ------------------------------- fp64 polish -------------------------------
def polish_population(best_a, K: int = 8, seed: int = 0) -> np.ndarray:
    """The polish's starting candidates (src/main.cu:810-821): candidate 0 is
    the best vector, candidate k > 0 multiplies every height by
    exp(0.003 (1 + k mod 8) z) with z standard normal (basin hopping), all
    clipped at 0 and normalised to sum 1.  z comes from numpy's PCG64 with
    the given seed (the reference draws it from std::mt19937_64)."""
    a = np.asarray(best_a, dtype=np.float64)
    rng = np.random.Generator(np.random.PCG64(np.random.SeedSequence([int(seed), 0xABCDEF])))
    out = np.empty((K, a.size))
    for k in range(K):
        x = a.copy()
        if k:
            x = x * np.exp(0.003 * (1 + (k % 8)) * rng.standard_normal(a.size))
        x = np.maximum(x, 0.0)
        out[k] = x / x.sum()
    return out


def polish(best_a, K: int = 8, iters: int = 40000, passes: int = 6, seed: int = 0,
           best_F: float | None = None, device="cuda", stream=None):
    """fp64 polish of the elite (src/main.cu:798-874) on the device: returns
    (best heights, best F, per-candidate F after the last pass).  best_F
    (default: the certifying F of best_a) is what a pass must beat."""
    a = np.asarray(best_a, dtype=np.float64)
    n = a.size
    pop = torch.as_tensor(polish_population(a, K, seed), device=device)
    mom, vel = torch.empty_like(pop), torch.empty_like(pop)
    fit = torch.empty(K, dtype=torch.float64, device=device)
    nact = torch.empty(K, dtype=torch.int32, device=device)
    best = torch.as_tensor(a, device=device).clone()
    if best_F is None:
        best_F = run_eval(best[None, :], with_nactive=False)[0].item()
    bF = torch.tensor([float(best_F)], dtype=torch.float64, device=device)
    _lib.call("sidon_polish", pop.data_ptr(), mom.data_ptr(), vel.data_ptr(), n, int(K),
              int(iters), int(passes), fit.data_ptr(), nact.data_ptr(), best.data_ptr(),
              bF.data_ptr(), _stream(stream))
    return best.cpu().numpy(), bF.item(), fit.cpu().numpy()


# ----------------------------- large candidates ----------------------------
def autotune_local_search(n: int, P: int, precision: str = "bf16x3") -> dict:
    """Time every schedule of the fused local search at (n, P, precision) --
    lane tile (fp32), window ring and segments vs waves (tensor cores) --
    and keep the fastest for this process; results are unchanged bit for bit.
    Returns the chosen schedule."""
    s = _lib.LsSchedule()
    _lib.call("sidon_autotune_local_search", int(n), int(P), PRECISIONS[precision], C.byref(s))
    return s.as_dict()


def local_search_schedule(n: int, P: int, precision: str = "bf16x3") -> dict:
    """The schedule the next uniform local search at (n, P, precision) uses."""
    s = _lib.LsSchedule()
    _lib.call("sidon_local_search_schedule", int(n), int(P), PRECISIONS[precision], C.byref(s))
    return s.as_dict()


def autotune_large(n: int, P: int, precision: str = "bf16x3") -> tuple[int, float]:
    """Measure and remember the fastest schedule for (n, P): returns (q, ms
    per step); q >= n is the fused single-CTA kernel."""
    q = C.c_int()
    ms = C.c_float()
    _lib.call("sidon_autotune_large", int(n), int(P), PRECISIONS[precision], C.byref(q),
              C.byref(ms))
    return q.value, ms.value


def large_workspace(n: int, P: int, q: int = 0, device="cuda",
                    precision: str = "bf16x3") -> torch.Tensor:
    """Workspace for run_local_search_large / run_frank_wolfe_large."""
    nbytes = _lib.load().sidon_large_workspace_bytes(int(n), int(P), int(q),
                                                     PRECISIONS[precision])
    if nbytes == 0:
        raise ValueError("bad large-candidate geometry")
    return torch.empty(nbytes, dtype=torch.uint8, device=device)


def run_local_search_large(pop: torch.Tensor, iters: int, p_start: float, p_end: float,
                           lr_start: float, lr_end: float, precision: str = "bf16x3",
                           q: int = 0, workspace: torch.Tensor | None = None,
                           mode_arr: torch.Tensor | None = None,
                           skip: torch.Tensor | None = None, mom: torch.Tensor | None = None,
                           vel: torch.Tensor | None = None, beta1: float = 0.9,
                           beta2: float = 0.999, mode_default: int = 0, stream=None) -> None:
    """run_local_search for candidates of any n (super-block tensor-core jobs)."""
    n, P = _pop_shape(pop)
    if workspace is None:
        workspace = large_workspace(n, P, q, pop.device, precision)
    if mom is None:
        mom = torch.empty_like(pop)
    if vel is None:
        vel = torch.empty_like(pop)
    _lib.call("sidon_local_search_large", _dev(pop, "pop", torch.float32),
              _dev(mom, "mom", torch.float32), _dev(vel, "vel", torch.float32),
              _opt(skip, "skip", torch.int32), _opt(mode_arr, "mode_arr", torch.int32), n, P,
              int(iters), float(p_start), float(p_end), float(lr_start), float(lr_end),
              float(beta1), float(beta2), int(mode_default), PRECISIONS[precision], int(q),
              workspace.data_ptr(), workspace.numel(), _stream(stream))


def run_frank_wolfe_large(pop: torch.Tensor, rounds: int, pdhg_iters: int, nT: int = 12,
                          t_max: float = 0.30, skip: torch.Tensor | None = None,
                          tau: float = 0.0, sigma: float = 0.0, precision: str = "bf16x3",
                          q: int = 0, workspace: torch.Tensor | None = None,
                          stream=None) -> None:
    """run_frank_wolfe_tc for candidates of any n."""
    n, P = _pop_shape(pop)
    if workspace is None:
        workspace = large_workspace(n, P, q, pop.device, precision)
    _lib.call("sidon_frank_wolfe_large", _dev(pop, "pop", torch.float32),
              _opt(skip, "skip", torch.int32), n, P, int(rounds), int(pdhg_iters), int(nT),
              float(t_max), float(tau), float(sigma), PRECISIONS[precision], int(q),
              workspace.data_ptr(), workspace.numel(), _stream(stream))


def certify_large(pop: torch.Tensor, stream=None):
    """certify for candidates of any n: (F, M, S, kmax)."""
    n, P = _pop_shape(pop)
    code = _dtype_code(pop)
    dev = pop.device
    ws = torch.empty(_lib.load().sidon_certify_workspace_bytes(P), dtype=torch.uint8, device=dev)
    F = torch.empty(P, dtype=torch.float64, device=dev)
    M = torch.empty(P, dtype=torch.float64, device=dev)
    S = torch.empty(P, dtype=torch.float64, device=dev)
    K = torch.empty(P, dtype=torch.int32, device=dev)
    _lib.call("sidon_certify_large", _dev(pop, "pop"), code, n, P, F.data_ptr(), M.data_ptr(),
              S.data_ptr(), K.data_ptr(), ws.data_ptr(), _stream(stream))
    return F, M, S, K


# ------------------------------ ragged batches ------------------------------
class RaggedBatch:
    """P candidates of different sizes back to back in one fp32 tensor:
    candidate p is ``flat[offsets[p]:offsets[p+1]]``.  ``offsets`` lives on
    the device (int64, P+1 entries) with a host copy in ``sizes``;
    ``order`` is the longest-first processing order (device int32)."""

    def __init__(self, rows, device="cuda", dtype=torch.float32):
        sizes = [int(len(r)) for r in rows]
        if not sizes or min(sizes) < 1:
            raise ValueError("a ragged batch needs candidates of at least one cell")
        self.sizes = sizes
        self.P = len(sizes)
        self.n_max = max(sizes)
        off = np.zeros(self.P + 1, dtype=np.int64)
        off[1:] = np.cumsum(sizes)
        self.host_offsets = off
        flat = np.concatenate([np.asarray(r, dtype=np.float64) for r in rows])
        self.flat = torch.tensor(flat, dtype=dtype, device=device)
        self.offsets = torch.tensor(off, device=device)
        self.order = ragged_order(self.offsets, self.P)

    def rows(self) -> list[np.ndarray]:
        """The candidates as host arrays (copies)."""
        h = self.flat.detach().cpu().numpy()
        return [h[self.host_offsets[p]:self.host_offsets[p + 1]].copy() for p in range(self.P)]

    def row(self, p: int) -> torch.Tensor:
        """Device view of candidate p."""
        return self.flat[int(self.host_offsets[p]):int(self.host_offsets[p + 1])]


def ragged_order(offsets: torch.Tensor, P: int, out: torch.Tensor | None = None,
                 stream=None) -> torch.Tensor:
    """Longest-first order of a ragged batch (ties by index)."""
    if out is None:
        out = torch.empty(P, dtype=torch.int32, device=offsets.device)
    _lib.call("sidon_ragged_order", _dev(offsets, "offsets", torch.int64), int(P),
              _dev(out, "order", torch.int32), _stream(stream))
    return out


def run_local_search_ragged(batch: RaggedBatch, iters: int, p_start: float, p_end: float,
                            lr_start: float, lr_end: float, precision: str = "bf16x3",
                            mode_arr: torch.Tensor | None = None,
                            skip: torch.Tensor | None = None, mom: torch.Tensor | None = None,
                            vel: torch.Tensor | None = None, beta1: float = 0.9,
                            beta2: float = 0.999, mode_default: int = 0, use_order: bool = True,
                            stream=None) -> None:
    """run_local_search over a ragged batch, in place."""
    if mom is None:
        mom = torch.empty_like(batch.flat)
    if vel is None:
        vel = torch.empty_like(batch.flat)
    _lib.call("sidon_local_search_ragged", _dev(batch.flat, "pop", torch.float32),
              _dev(mom, "mom", torch.float32), _dev(vel, "vel", torch.float32),
              batch.offsets.data_ptr(), batch.order.data_ptr() if use_order else None,
              batch.n_max, _opt(skip, "skip", torch.int32),
              _opt(mode_arr, "mode_arr", torch.int32), batch.P, int(iters), float(p_start),
              float(p_end), float(lr_start), float(lr_end), float(beta1), float(beta2),
              int(mode_default), PRECISIONS[precision], _stream(stream))


def run_eval_ragged(batch: RaggedBatch, active_tol: float = 1e-4, with_nactive: bool = True,
                    stream=None):
    """run_eval over a ragged batch: (F fp64 [P], nactive int32 [P] | None)."""
    dev = batch.flat.device
    F = torch.empty(batch.P, dtype=torch.float64, device=dev)
    N = torch.empty(batch.P, dtype=torch.int32, device=dev) if with_nactive else None
    _lib.call("sidon_eval_ragged", batch.flat.data_ptr(), _dtype_code(batch.flat),
              batch.offsets.data_ptr(), batch.order.data_ptr(), batch.n_max, batch.P,
              F.data_ptr(), None if N is None else N.data_ptr(), float(active_tol),
              _stream(stream))
    return F, N


def run_frank_wolfe_ragged(batch: RaggedBatch, rounds: int, pdhg_iters: int, nT: int = 12,
                           t_max: float = 0.30, skip: torch.Tensor | None = None,
                           tau: float = 0.0, sigma: float = 0.0, stream=None) -> None:
    """run_frank_wolfe over a ragged batch, in place."""
    _lib.call("sidon_frank_wolfe_ragged", _dev(batch.flat, "pop", torch.float32),
              batch.offsets.data_ptr(), batch.order.data_ptr(), batch.n_max,
              _opt(skip, "skip", torch.int32), batch.P, int(rounds), int(pdhg_iters), int(nT),
              float(t_max), float(tau), float(sigma), _stream(stream))


def run_frank_wolfe_tc_ragged(batch: RaggedBatch, rounds: int, pdhg_iters: int, nT: int = 12,
                              t_max: float = 0.30, skip: torch.Tensor | None = None,
                              tau: float = 0.0, sigma: float = 0.0, precision: str = "bf16x3",
                              stream=None) -> None:
    """run_frank_wolfe_tc over a ragged batch, in place."""
    g = torch.empty_like(batch.flat)
    gb = torch.empty_like(batch.flat)
    _lib.call("sidon_frank_wolfe_tc_ragged", _dev(batch.flat, "pop", torch.float32),
              g.data_ptr(), gb.data_ptr(), batch.offsets.data_ptr(), batch.order.data_ptr(),
              batch.n_max, _opt(skip, "skip", torch.int32), batch.P, int(rounds),
              int(pdhg_iters), int(nT), float(t_max), float(tau), float(sigma),
              PRECISIONS[precision], _stream(stream))


def island_migrate_ragged(batch: RaggedBatch, fit: torch.Tensor, n_islands: int, k: int = 1,
                          order: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    """island_migrate over a ragged batch (migrants of another size are
    resampled and renormalised; their fit becomes NaN).  Returns the ranking."""
    if order is None:
        order = torch.empty(batch.P, dtype=torch.int32, device=batch.flat.device)
    _lib.call("sidon_island_migrate_ragged", _dev(batch.flat, "pop", torch.float32),
              batch.offsets.data_ptr(), _dev(fit, "fit", torch.float64), batch.P,
              int(n_islands), int(k), _dev(order, "order", torch.int32), _stream(stream))
    return order


# ------------------------------ anneal driver -------------------------------
def anneal_config(steps: int = 5000, p_start: float = 2.0, p_end: float = 1024.0,
                  lr_start: float = 1e-3, lr_end: float = 1e-3, beta1: float = 0.9,
                  beta2: float = 0.999, precision: str = "bf16x3", fw_every: int = 250,
                  fw_rounds: int = 1, pdhg_iters: int = 200, fw_nT: int = 12,
                  fw_t_max: float = 0.30, fw_tau: float = 0.9, fw_sigma: float = 0.9,
                  fw_precision: str = "bf16x3", n_islands: int = 16, migrate_every: int = 500,
                  k_migrate: int = 4) -> _lib.AnnealConfig:
    """struct sidon_anneal_config; the defaults are the batched island anneal
    (5000 steps, p 2 -> 1024, Frank-Wolfe every 250 steps with 200
    Chambolle-Pock iterations at tau = sigma = 0.9 / ||a||_1 = 0.9 on the
    normalised heights, 16 islands, top-4 migration every 500 steps)."""
    return _lib.AnnealConfig(int(steps), float(p_start), float(p_end), float(lr_start),
                             float(lr_end), float(beta1), float(beta2), PRECISIONS[precision],
                             int(fw_every), int(fw_rounds), int(pdhg_iters), int(fw_nT),
                             float(fw_t_max), float(fw_tau), float(fw_sigma),
                             PRECISIONS[fw_precision], int(n_islands), int(migrate_every),
                             int(k_migrate))


def _anneal_args(batch, cfg, fit, rank, mom, vel):
    if isinstance(batch, RaggedBatch):
        pop, off, order, n_max, P = (batch.flat, batch.offsets.data_ptr(),
                                     batch.order.data_ptr(), batch.n_max, batch.P)
    else:
        n_max, P = _pop_shape(batch)
        pop, off, order = batch, None, None
    dev = pop.device
    if fit is None:
        fit = torch.empty(P, dtype=torch.float64, device=dev)
    if rank is None:
        rank = torch.empty(P, dtype=torch.int32, device=dev)
    if mom is None:
        mom = torch.empty_like(pop)
    if vel is None:
        vel = torch.empty_like(pop)
    args = (_dev(pop, "pop", torch.float32), _dev(mom, "mom", torch.float32),
            _dev(vel, "vel", torch.float32), off, order, n_max, P,
            _dev(fit, "fit", torch.float64), _dev(rank, "rank", torch.int32))
    return args, fit, rank, (mom, vel)


def anneal(batch, cfg: _lib.AnnealConfig, fit: torch.Tensor | None = None,
           rank: torch.Tensor | None = None, mom: torch.Tensor | None = None,
           vel: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    """Enqueue the whole island anneal on a stream (a RaggedBatch or a
    uniform [P, n] fp32 tensor); returns fit (fp64 F at the end)."""
    args, fit, rank, _ = _anneal_args(batch, cfg, fit, rank, mom, vel)
    _lib.call("sidon_anneal", *args, C.byref(cfg), _stream(stream))
    return fit


class AnnealGraph:
    """The anneal recorded once as a CUDA graph (sidon_anneal_capture);
    ``launch`` replays it.  Holds the scratch tensors it was recorded with."""

    def __init__(self, batch, cfg: _lib.AnnealConfig, fit=None, rank=None, mom=None, vel=None):
        args, self.fit, self.rank, self._scratch = _anneal_args(batch, cfg, fit, rank, mom, vel)
        self._batch = batch
        self._cfg = cfg
        h = C.c_void_p()
        _lib.call("sidon_anneal_capture", *args, C.byref(cfg), C.byref(h))
        self._h = h

    def launch(self, stream=None) -> None:
        if not self._h:
            raise RuntimeError("graph destroyed")
        _lib.call("sidon_graph_launch", self._h, _stream(stream))

    def close(self) -> None:
        if self._h:
            _lib.load().sidon_graph_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# memetic generations (sidon_generation_*)
# ---------------------------------------------------------------------------
def generation_config(n_islands: int = 8, elite: int = 2, ls_iters: int = 4000,
                      cold_iters: int = 20000, p_max: float = 20000.0,
                      precision: str = "bf16x3", fw_rounds: int = 6, fw_iters: int = 500,
                      fw_nT: int = 12, fw_t_max: float = 0.30, fw_precision: str = "fp32",
                      tabu_tenure: int = 6, tabu_capacity: int = 1 << 16,
                      seed: int = 20260905) -> _lib.GenerationConfig:
    """struct sidon_generation_config; the defaults are the reference driver's
    (src/main.cu:41-58, 472: 8 islands, 2 elites, warm 4000 / cold 20000
    steps, p up to 20000, 6 Frank-Wolfe rounds of 500 iterations, tabu
    tenure 6)."""
    return _lib.GenerationConfig(int(n_islands), int(elite), int(ls_iters), int(cold_iters),
                                 float(p_max), PRECISIONS[precision], int(fw_rounds),
                                 int(fw_iters), int(fw_nT), float(fw_t_max),
                                 PRECISIONS[fw_precision], int(tabu_tenure), int(tabu_capacity),
                                 int(seed) & 0xFFFFFFFFFFFFFFFF)


class GenerationGraph:
    """Generations recorded once as a CUDA graph (sidon_generation_capture);
    ``launch`` replays them."""

    def __init__(self, handle, pop: torch.Tensor, generations: int):
        h = C.c_void_p()
        _lib.call("sidon_generation_capture", handle, _dev(pop, "pop", torch.float32),
                  int(generations), C.byref(h))
        self._h = h
        self._pop = pop
        self.generations = int(generations)

    def launch(self, stream=None) -> None:
        if not self._h:
            raise RuntimeError("graph destroyed")
        _lib.call("sidon_graph_launch", self._h, _stream(stream))

    def close(self) -> None:
        if self._h:
            _lib.load().sidon_graph_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Generation:
    """The memetic island search, one generation at a time on the device
    (src/main.cu:586-785): anneal tiers, Frank-Wolfe, fp64 evaluation,
    support signatures, incumbent, tabu table, island ranking and
    migration, offspring plan, variation, reinjection and bandit credit.

    The workspace is one device byte tensor owned by this object; the state
    (incumbent, bandit, tabu table, counters) lives in it across levels.
    """

    def __init__(self, n_max: int, P: int, cfg: _lib.GenerationConfig | None = None,
                 device="cuda", stream=None):
        self.cfg = cfg if cfg is not None else generation_config()
        self.n_max, self.P = int(n_max), int(P)
        lib = _lib.load()
        nbytes = lib.sidon_generation_workspace_bytes(self.n_max, self.P,
                                                      int(self.cfg.tabu_capacity))
        if nbytes == 0:
            raise SidonError("sidon_generation_workspace_bytes", _lib.ERR_ARG)
        self.workspace = torch.empty(nbytes, dtype=torch.uint8, device=device)
        h = C.c_void_p()
        _lib.call("sidon_generation_create", self.workspace.data_ptr(), nbytes, self.n_max,
                  self.P, C.byref(self.cfg), C.byref(h), _stream(stream))
        self._h = h
        v = _lib.GenerationViews()
        _lib.call("sidon_generation_views_of", self._h, C.byref(v))
        self._views = v
        self.n = 0

    def _view(self, name: str, count: int, dtype) -> torch.Tensor:
        off = getattr(self._views, name) - self.workspace.data_ptr()
        size = torch.tensor([], dtype=dtype).element_size() * count
        return self.workspace[off:off + size].view(dtype)

    def views(self) -> dict:
        """Device tensors over the workspace arrays (current level's P)."""
        P, cap1 = self.P, int(self.cfg.tabu_capacity) + 1
        return {
            "fit": self._view("fit", P, torch.float64),
            "parent_fit": self._view("parent_fit", P, torch.float64),
            "child_fit": self._view("child_fit", P, torch.float64),
            "nactive": self._view("nactive", P, torch.int32),
            "sig": self._view("sig", P, torch.int64),
            "nnz": self._view("nnz", P, torch.int32),
            "p1": self._view("p1", P, torch.int32),
            "p2": self._view("p2", P, torch.int32),
            "op": self._view("op", P, torch.int32),
            "strength": self._view("strength", P, torch.float32),
            "cur_op": self._view("cur_op", P, torch.int32),
            "mode": self._view("mode", P, torch.int32),
            "rank": self._view("rank", P, torch.int32),
            "tier_skip": self._view("tier_skip", 3 * P, torch.int32).view(3, P),
            "best_row": self._view("best_row", self.n_max, torch.float32),
            "tabu_key": self._view("tabu_key", cap1, torch.int64),
            "tabu_best": self._view("tabu_best", cap1, torch.float64),
            "tabu_hits": self._view("tabu_hits", cap1, torch.int32),
            "tabu_used": self._view("tabu_used", cap1, torch.int32),
        }

    def begin_level(self, n: int, level: int, seed_op: torch.Tensor | None = None,
                    stream=None) -> None:
        """Start a ladder level of n cells; seed_op: int32 [P] operator per slot
        (None: all 9, fresh restarts)."""
        _lib.call("sidon_generation_begin_level", self._h, int(n), int(level),
                  _opt(seed_op, "seed_op", torch.int32), _stream(stream))
        self.n = int(n)

    def set_best(self, row: torch.Tensor, F: float, stream=None) -> None:
        """Adopt row (fp32 device [n]) with fp64 F as the incumbent."""
        _lib.call("sidon_generation_set_best", self._h, _dev(row, "row", torch.float32),
                  int(row.numel()), float(F), _stream(stream))

    def step(self, pop: torch.Tensor, stream=None) -> None:
        """Enqueue one generation on pop (fp32 [P][n], in place)."""
        if tuple(pop.shape) != (self.P, self.n):
            raise ValueError(f"pop must be [{self.P}][{self.n}]")
        _lib.call("sidon_generation_step", self._h, _dev(pop, "pop", torch.float32),
                  _stream(stream))

    def capture(self, pop: torch.Tensor, generations: int) -> GenerationGraph:
        if tuple(pop.shape) != (self.P, self.n):
            raise ValueError(f"pop must be [{self.P}][{self.n}]")
        return GenerationGraph(self._h, pop, generations)

    def state(self, stream=None) -> dict:
        """The device state after the stream's work so far (synchronises it)."""
        s = _lib.GenerationState()
        _lib.call("sidon_generation_read_state", self._h, C.byref(s), _stream(stream))
        out = {}
        for k, _ in _lib.GenerationState._fields_:
            if k == "pad_":
                continue
            x = getattr(s, k)
            out[k] = list(x) if k.startswith("op_") else x
        return out

    def best(self) -> np.ndarray:
        """The incumbent heights (host fp32, its own n cells)."""
        n = self.state()["best_n"]
        return self.views()["best_row"][:n].cpu().numpy()

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.load().sidon_generation_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# search driver (sidon_seed_level, sidon_search)
# ---------------------------------------------------------------------------
def seed_level(n: int, P: int, level: int, prev: np.ndarray | None = None,
               seed: int = 20260905) -> tuple[np.ndarray, np.ndarray]:
    """Host seeding of a ladder level (src/main.cu:483-553): (pop float32
    [P][n], seed_op int32 [P]); prev is the previous level's population."""
    pop = np.zeros((P, n), np.float32)
    op = np.zeros(P, np.int32)
    pv = None if prev is None else np.ascontiguousarray(prev, dtype=np.float32)
    _lib.call("sidon_seed_level", pop.ctypes.data, op.ctypes.data, int(n), int(P), int(level),
              None if pv is None else pv.ctypes.data, 0 if pv is None else pv.shape[1],
              int(seed) & 0xFFFFFFFFFFFFFFFF)
    return pop, op


def search(ladder=(64, 128, 256, 512, 1024, 2048), P: int = 256, seconds: float = 600.0,
           gens_per_level: int = 0, gens_per_graph: int = 5, polish_iters: int = 40000,
           polish_top: int = 8, gen: _lib.GenerationConfig | None = None, resume=None,
           progress=None) -> tuple[np.ndarray, float]:
    """The reference driver's whole search (src/main.cu:400-874) in one call:
    returns (incumbent heights fp64, F).  progress(dict, best ndarray) is
    called after every replay of gens_per_graph generations."""
    lad = (C.c_int * len(ladder))(*[int(x) for x in ladder])
    cfg = _lib.SearchConfig(C.cast(lad, C.POINTER(C.c_int)), len(ladder), int(P), float(seconds),
                            int(gens_per_level), int(gens_per_graph), int(polish_iters),
                            int(polish_top), gen if gen is not None else generation_config())
    res = None if resume is None else np.ascontiguousarray(resume, dtype=np.float64)
    cap = max(max(ladder), 0 if res is None else res.size)
    out = np.zeros(cap, np.float64)
    nb, fb = C.c_int(0), C.c_double(0.0)

    def _cb(pr, best, best_n, _user):
        if progress is not None:
            p = pr.contents
            d = {k: getattr(p, k) for k, _ in _lib.SearchProgress._fields_}
            progress(d, np.ctypeslib.as_array(best, shape=(best_n,)).copy() if best_n else None)

    cb = _lib.SEARCH_CALLBACK(_cb)
    _lib.call("sidon_search", C.byref(cfg), None if res is None else res.ctypes.data,
              0 if res is None else res.size, out.ctypes.data, cap, C.byref(nb), C.byref(fb),
              cb, None)
    return out[:nb.value].copy(), fb.value

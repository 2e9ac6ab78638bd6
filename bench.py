"""Benchmark: batched L^p-annealed projected-Adam steps (forward convolution +
adjoint correlation + update) at n = 8400 cells, B = 256 candidates per GPU.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision bf16x3|bf16x1|fp32]
                    [--impl ours|reference] [--workload lp_adam|islands|ladder|memetic|micro|search]

One *step* = every candidate of the batch advances one Adam step.  The timed
region is ONE launch of the fused local-search kernel running K steps (the
population stays resident in shared memory), bracketed by a barrier and
device synchronisation, timed with CUDA events on the launching stream, max
over ranks.  ``value`` = whole-job batched steps/s (N GPUs x K steps / max
time) of the BF16x3 tensor-core step (default ``--precision``); the FP32 SIMT
form of the same step is timed after it for ``speedup_vs_fp32_simt``.  ``e2e`` = the same metric through the public call with host buffers:
per step an H2D copy of the population from pinned memory, one
``run_local_search`` step and a D2H copy of the updated population, on three
streams so that a step's compute overlaps the neighbouring steps' copies.

Synthetic data: lognormal(0,1) fp32 heights with 1/3 exact zeros, a support
gap of width n/10 at [n/50, n/50+n/10) and an endpoint atom (seeded PCG64,
seed 8400 + rank), normalised to sum 1.

``--impl reference`` times the reference's own CPU implementation of the
path, the fp64 L^p-Adam twin of tools/probe.cpp (localSearch, OpenMP over
candidates as in probe.cpp:239) compiled from the reference sources into
oracle/_ref, on all host cores, on a bounded sample of the same workload.
With ``--workload islands|ladder|memetic|micro`` it times the reference's own
GPU kernels (built for sm_100a from its sources into oracle/_ref, launched
through its own helpers) on the same workload instead, and with ``search``
its unmodified search driver under the same wall-clock budget.
"""
from __future__ import annotations

import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_CELLS = 8400
BATCH = 256
FLOP_PER_CAND_STEP = 4.0 * N_CELLS * N_CELLS        # conv 2n^2 + correlation 2n^2 (src/main.cu:313,625)
ANNEAL = dict(p_start=2.0, p_end=1024.0, lr_start=1e-3, lr_end=1e-3)


def _peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d["hbm_gbs"], "bf16_tflops": d["bf16_tflops"],
                "bf16_tflops_sustained": d.get("bf16_tflops_sustained"), "src": "measured",
                "sm_max_mhz": d.get("sm_max_mhz", 1965.0)}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0,
            "src": "fallback", "sm_max_mhz": 1965.0}


class Clocks:
    """nvidia-smi sampler for the timed region (SM clock, throttle reasons)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self) -> dict:
        mhz, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                mhz.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(mhz)}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _config(prec: str, ws: int) -> dict:
    """The workload both arms report (the metric's configuration)."""
    return {"workload": f"lp_adam n={N_CELLS} B={BATCH}/GPU lognormal heights, "
                        f"p {ANNEAL['p_start']}->{ANNEAL['p_end']} (one batched step = conv + "
                        f"adjoint correlation + Adam update of every candidate)",
            "global_batch": BATCH * ws, "n": N_CELLS, "precision": prec,
            "parallelism": f"candidates sharded, {ws} x {BATCH}",
            "l2": "single launch of K steps, population resident in shared memory; "
                  "L2 flushed (256 MB write) before the timed launch"}


# --------------------------------- reference arm ---------------------------
def _ref_batch_call(probe, pop: np.ndarray, iters: int) -> float:
    """One call of the reference CPU twin over the whole batch: `iters` Adam
    steps of every candidate (OpenMP over candidates, probe.cpp:239), p and lr
    along the benchmark's schedule.  Returns its wall time in seconds."""
    x = np.ascontiguousarray(pop.copy())
    t0 = time.perf_counter()
    probe.ref_probe_local_search_batch(x.ctypes.data, N_CELLS, x.shape[0], int(iters),
                                       ANNEAL["p_start"], ANNEAL["p_end"], ANNEAL["lr_start"],
                                       ANNEAL["lr_end"], 0.9, 0.999, 0, None)
    return time.perf_counter() - t0


def reference_arm(args) -> None:
    """The reference's CPU implementation of the path (tools/probe.cpp
    localSearch, fp64) on the whole workload: the same 256 candidates, W
    warm-up steps in one call, then the K timed steps in one call (each call
    anneals p over its own steps, as the GPU arm's launch does)."""
    ws, rank, _ = _dist()
    if rank != 0:
        return
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    if not oracle.have_ref():
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref not built (reference sources absent here)"}))
        return
    from sidon_b200 import synth
    probe = oracle.ref_probe()
    threads = probe.ref_probe_threads()
    pop = synth.population("lognormal", N_CELLS, BATCH, seed=8400, dtype=np.float64)
    _ref_batch_call(probe, pop, max(1, args.warmup))
    t = _ref_batch_call(probe, pop, args.steps)
    v = args.steps / t                      # batched (256-candidate) steps per second
    line = {
        "impl": "reference", "metric": "lp_adam_batched_steps_per_s", "value": v,
        "unit": "steps/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": _config(args.precision, args.gpus),
        "cpu_baseline": {"value": v, "unit": "steps/s", "cores": threads, "kind": "reference",
                         "sample": f"tools/probe.cpp localSearch (fp64 CPU twin) on all {BATCH} "
                                   f"candidates x {args.steps} steps in one call, OpenMP over "
                                   f"candidates on {threads} threads ({_cpu_model()}); the call "
                                   f"adds one final objective per candidate (1/(2K) of a step)"},
        "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def _cpu_model() -> str:
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown CPU"


def cpu_baseline(budget_s: float = 10.0) -> dict:
    """The reference CPU twin on this host's cores: whole 256-candidate steps,
    as many as fit the budget (one step first to size the call)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    from sidon_b200 import synth
    if not oracle.have_ref():
        return {"value": None, "unit": "steps/s", "cores": 0, "kind": "reference",
                "sample": "unavailable: oracle/_ref not built"}
    probe = oracle.ref_probe()
    threads = probe.ref_probe_threads()
    pop = synth.population("lognormal", N_CELLS, BATCH, seed=8400, dtype=np.float64)
    t1 = _ref_batch_call(probe, pop, 1)
    iters = max(1, int(budget_s / max(t1, 1e-3)))
    t = _ref_batch_call(probe, pop, iters)
    return {"value": iters / t, "unit": "steps/s", "cores": threads, "kind": "reference",
            "sample": f"tools/probe.cpp localSearch fp64 twin, n={N_CELLS}, all {BATCH} "
                      f"candidates x {iters} steps in one call ({t:.1f}s on {threads} threads, "
                      f"{_cpu_model()})"}


# ----------------------------------- our arm -------------------------------
def our_arm(args) -> None:
    import torch
    import torch.distributed as dist
    ws, rank, local = _dist()
    if ws > 1:
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    import sidon_b200
    sidon_b200.load(build=not (ROOT / "sidon-autocorrelation-bound_b200" / "libsidon_b200.so").exists())
    from sidon_b200 import kernels, synth

    prec = args.precision
    host = synth.population("lognormal", N_CELLS, BATCH, seed=8400 + rank)
    pop = torch.as_tensor(host, device=dev)
    mom = torch.empty_like(pop)
    vel = torch.empty_like(pop)
    # flag words of the balanced-segment launch (None where the call needs none)
    wsp = kernels.local_search_workspace(N_CELLS, BATCH, prec, dev)
    stream = torch.cuda.current_stream()

    def run(x, iters):
        kernels.run_local_search(x, iters, mom=mom, vel=vel, precision=prec, workspace=wsp,
                                 **ANNEAL)

    def barrier():
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # warm-up: W steps, untimed (once here, and again on a scratch copy right
    # before the timed launch: the clock sampler's start-up leaves the GPU
    # idle for 0.3 s, and a kernel started from idle runs its first
    # milliseconds at lower clocks)
    run(pop, max(3, args.warmup))
    scratch = torch.empty_like(pop)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    pop.copy_(torch.as_tensor(host, device=dev))
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        scratch.copy_(pop)
        run(scratch, max(3, args.warmup))
        flush.fill_(1.0)                               # evict L2 before the timed launch
        barrier()
        start.record(stream)
        run(pop, args.steps)
        end.record(stream)
        torch.cuda.synchronize()
    ms = start.elapsed_time(end)
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if ws > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = t.item()
    launches = 1

    # the FP32 SIMT form of the same step, for the speed-up the metric names
    simt = None
    if prec != "fp32":
        k32 = max(3, min(args.steps, 20))
        kernels.run_local_search(pop, 3, mom=mom, vel=vel, precision="fp32", **ANNEAL)
        pop.copy_(torch.as_tensor(host, device=dev))
        flush.fill_(1.0)
        torch.cuda.synchronize()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        kernels.run_local_search(pop, k32, mom=mom, vel=vel, precision="fp32", **ANNEAL)
        s1.record(stream)
        torch.cuda.synchronize()
        simt = k32 / (s0.elapsed_time(s1) / 1e3)
        pop.copy_(torch.as_tensor(host, device=dev))
        run(pop, args.steps)

    # F error vs fp64 (hostF-identical certifying evaluation) on the final
    # population: the reported search-time objective (max b refined in fp64
    # over the near-maximal k, sum in fp64) and the raw step arithmetic (max
    # of the b the step itself forms, fp32 sum of the heights)
    Fcert, _ = kernels.run_eval(pop, with_nactive=False)
    _, saved, b_step = kernels.lp_forward(pop, 2.0, store_b=True, precision=prec)
    S = saved[:, 1].double()
    F32 = 2.0 * N_CELLS * saved[:, 0].double() / (S * S)
    f_rel = (F32 - Fcert).abs().div(Fcert).max().item()
    S_raw = pop.sum(dim=1, dtype=torch.float32).double()
    F_raw = 2.0 * N_CELLS * b_step.max(dim=1).values.double() / (S_raw * S_raw)
    f_rel_raw = (F_raw - Fcert).abs().div(Fcert).max().item()
    del b_step

    # end-to-end through the public call with host buffers: every step copies
    # its population in from pinned host memory, runs one step and copies the
    # result out.  Three streams overlap step s's compute with the copy-in of
    # step s+1 and the copy-out of step s-1; three device buffers, so that a
    # copy-in waits only for the copy-out of step s-3 (with two, the chain
    # copy-out -> copy-in -> compute of alternate steps bounds the rate).
    NBUF = 3
    hpin = torch.as_tensor(host).pin_memory()
    houts = [torch.empty_like(hpin).pin_memory() for _ in range(NBUF)]
    xs = [torch.empty_like(pop) for _ in range(NBUF)]
    s_in, s_cp, s_out = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()

    def e2e_loop(nsteps, start_ev):
        ev_cp, ev_out = [None] * NBUF, [None] * NBUF
        for sidx in (s_in, s_cp, s_out):
            sidx.wait_event(start_ev)
        for step in range(nsteps):
            b = step % NBUF
            if ev_out[b] is not None:
                s_in.wait_event(ev_out[b])        # x[b] of step - NBUF fully read back
            with torch.cuda.stream(s_in):
                xs[b].copy_(hpin, non_blocking=True)
            ev_in = torch.cuda.Event()
            ev_in.record(s_in)
            s_cp.wait_event(ev_in)
            kernels.run_local_search(xs[b], 1, mom=mom, vel=vel, precision=prec, stream=s_cp,
                                     workspace=wsp, **ANNEAL)
            ev_cp[b] = torch.cuda.Event()
            ev_cp[b].record(s_cp)
            s_out.wait_event(ev_cp[b])
            with torch.cuda.stream(s_out):
                houts[b].copy_(xs[b], non_blocking=True)
            ev_out[b] = torch.cuda.Event()
            ev_out[b].record(s_out)
        for sidx in (s_in, s_cp, s_out):
            stream.wait_stream(sidx)

    e2e_steps = max(3, min(args.steps, 20))
    w0 = torch.cuda.Event()
    w0.record(stream)
    e2e_loop(2 * NBUF, w0)                 # untimed: every buffer and stream used once first
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    e2e_loop(e2e_steps, e0)
    e1.record(stream)
    torch.cuda.synchronize()
    e_ms = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=dev)
    if ws > 1:
        dist.all_reduce(e_ms, op=dist.ReduceOp.MAX)
    e2e_val = ws * e2e_steps / (e_ms.item() / 1e3)
    hout = houts[0]

    if rank == 0:
        peaks = _peaks()
        value = ws * args.steps / (ms_max / 1e3)
        per_launch_flop = FLOP_PER_CAND_STEP * BATCH * args.steps
        achieved_tf = per_launch_flop / (ms / 1e3) / 1e12
        ck = clk.summary()
        if prec == "fp32":
            mhz = ck["sm_mhz"] or peaks["sm_max_mhz"]
            peak = 148 * 128 * 2 * mhz * 1e6 / 1e12     # FFMA lanes x 2 flop x clock
            roof = {"bound": "fp32_simt", "achieved": achieved_tf, "peak": peak,
                    "unit": "TFLOP/s", "frac": achieved_tf / peak, "traffic": _traffic(prec),
                    "peak_src": f"derived: 148 SMs x 128 FFMA/clk x 2 x {mhz:.0f} MHz (sampled)"}
        else:
            peak = peaks["bf16_tflops"]
            roof = {"bound": "tensor", "achieved": achieved_tf, "peak": peak, "unit": "TFLOP/s",
                    "frac": achieved_tf / peak, "traffic": _traffic(prec),
                    "peak_src": f"bf16_tflops ({peaks['src']}, burst)",
                    "frac_of_3_product_ceiling": 3.0 * achieved_tf / peak if prec == "bf16x3"
                    else achieved_tf / peak}
        line = {
            "metric": "lp_adam_batched_steps_per_s", "value": value, "unit": "steps/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": {"fp32": "f32", "bf16x3": "bf16x3(f32 acc)",
                                            "bf16x1": "bf16(f32 acc)"}[prec],
            "data": "synthetic",
            "config": _config(prec, ws),
            "candidate_steps_per_s": value * BATCH,
            "fp32_simt_steps_per_s": simt,
            "speedup_vs_fp32_simt": (value / ws) / simt if simt else None,
            "f_evals_per_s": value * BATCH,
            "f_rel_err_vs_fp64": f_rel,
            "f_rel_err_vs_fp64_raw_step": f_rel_raw,
            "roofline": roof,
            "clocks": {"sm_mhz": ck["sm_mhz"], "sm_max_mhz": ck["sm_max_mhz"],
                       "reasons": ck["reasons"]},
            "e2e": {"value": e2e_val, "unit": "steps/s",
                    "h2d_bytes_per_step": int(hpin.numel() * 4),
                    "d2h_bytes_per_step": int(hout.numel() * 4)},
            "gpu_launches": launches,
        }
        if ws == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(args.cpu_budget)
        print(json.dumps(line))
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()


# ------------------------------ batched islands -----------------------------
ISLAND_LEVELS = (512, 1024, 2048, 4096, 8400)


def islands_arm(args) -> None:
    """The batched uneven-island anneal: 1024 candidates with n uniform over
    the ladder levels (plain-method heights), one CUDA graph holding the
    5000-step anneal (p 2 -> 1024), a Frank-Wolfe step every 250 steps (200
    Chambolle-Pock iterations, tau = sigma = 0.9 / ||a||_1), 16 islands with
    top-4 migration every 500 steps ranked by fp64 F.  Prints one JSON line
    (its own metric; not the headline line)."""
    import torch
    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    import sidon_b200
    sidon_b200.load(build=not (ROOT / "sidon-autocorrelation-bound_b200" / "libsidon_b200.so").exists())
    from sidon_b200 import kernels, synth

    P = args.islands_P
    sizes = synth.uneven_sizes(P, seed=3 + rank, levels=ISLAND_LEVELS)
    rows = synth.ragged_population(sizes, seed=3 + rank)
    batch = kernels.RaggedBatch(rows, device=dev)
    start_flat = batch.flat.clone()
    cfg = kernels.anneal_config(steps=args.anneal_steps, precision=args.precision,
                                pdhg_iters=args.pdhg_iters, fw_every=args.fw_every,
                                fw_tau=0.9, fw_sigma=0.9, fw_precision=args.fw_precision)
    F0, _ = kernels.run_eval_ragged(batch, with_nactive=False)
    F0 = F0.cpu().numpy()

    # warm-up: a short anneal with the same kernels (untimed)
    wcfg = kernels.anneal_config(steps=max(3, args.warmup) * 2, precision=args.precision,
                                 pdhg_iters=4, fw_every=max(3, args.warmup), migrate_every=0,
                                 fw_precision=args.fw_precision)
    kernels.anneal(batch, wcfg)
    batch.flat.copy_(start_flat)
    graph = kernels.AnnealGraph(batch, cfg)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    flush.fill_(1.0)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        e0.record(stream)
        graph.launch()
        e1.record(stream)
        torch.cuda.synchronize()
    total_ms = e0.elapsed_time(e1)
    F1 = graph.fit.cpu().numpy()
    assert bool((batch.flat >= 0).all())

    # phase split: one 250-step local-search segment and one Frank-Wolfe step
    batch.flat.copy_(start_flat)
    seg = min(cfg.fw_every or cfg.steps, cfg.steps)

    def timed(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b)
    ls_ms = timed(lambda: kernels.run_local_search_ragged(batch, seg, 2.0, 4.0, 1e-3, 1e-3,
                                                           precision=args.precision))
    fw_ms = timed(lambda: kernels.run_frank_wolfe_tc_ragged(
        batch, 1, cfg.pdhg_iters, cfg.fw_nT, cfg.fw_t_max, tau=0.9, sigma=0.9,
        precision=args.precision if args.precision != "fp32" else "bf16x3"))
    fw_simt_ms = timed(lambda: kernels.run_frank_wolfe_ragged(batch, 1, cfg.pdhg_iters, cfg.fw_nT,
                                                               cfg.fw_t_max, tau=0.9, sigma=0.9))
    graph.close()

    n2 = float(np.sum(np.asarray(sizes, dtype=np.float64) ** 2))
    adam_flop = 4.0 * n2 * cfg.steps
    n_fw = cfg.steps // cfg.fw_every if cfg.fw_every else 0
    fw_flop = (4.0 * n2 * cfg.pdhg_iters + 26.0 * n2) * n_fw
    ck = clk.summary()
    if rank == 0:
        line = {
            "metric": "island_anneal_candidate_steps_per_s",
            "value": P * cfg.steps / (total_ms / 1e3), "unit": "candidate-steps/s",
            "n_gpus": 1, "higher_is_better": True, "data": "synthetic",
            "anneal_seconds": total_ms / 1e3,
            "config": {"workload": f"batched uneven islands: P={P}, n uniform over "
                                   f"{list(ISLAND_LEVELS)}, {cfg.steps} steps p 2->1024, "
                                   f"FW every {cfg.fw_every} ({cfg.pdhg_iters} PDHG), "
                                   f"16 islands top-4 every 500, one CUDA graph",
                       "precision": args.precision, "sizes_hist":
                       {int(l): int(np.sum(sizes == l)) for l in ISLAND_LEVELS}},
            "flop": {"adam": adam_flop, "frank_wolfe": fw_flop,
                     "tflops_overall": (adam_flop + fw_flop) / (total_ms / 1e3) / 1e12},
            "fw_precision": args.fw_precision,
            "phase_ms": {"local_search_segment": ls_ms, "segment_steps": seg,
                         "frank_wolfe_step": fw_ms, "frank_wolfe_step_fp32_simt": fw_simt_ms,
                         "adam_tflops": 4.0 * n2 * seg / (ls_ms / 1e3) / 1e12,
                         "fw_tflops": (4.0 * n2 * cfg.pdhg_iters + 26.0 * n2) / (fw_ms / 1e3) / 1e12},
            "F": {"start_median": float(np.median(F0)), "end_median": float(np.nanmedian(F1)),
                  "end_best": float(np.nanmin(F1))},
            "clocks": {"sm_mhz": ck["sm_mhz"], "sm_max_mhz": ck["sm_max_mhz"],
                       "reasons": ck["reasons"]},
        }
        print(json.dumps(line))


# ------------------------- the reference's own micro-benchmark ---------------
MICRO_N = (128, 256, 512, 1024, 2048, 4096)


def _micro_setup(n: int, seed: int = 1):
    """The settings of src/main.cu:294-320: P = max(32, min(512, 4M / n)),
    heights uniform in [0.2, 1) (seeded PCG64 standing in for its
    mt19937(1)), a 10-iteration warm-up at p = 8, then 100 iterations with p
    8 -> 200 and lr 0.05 -> 0.005; TFLOP/s = 4 n^2 P iters / time."""
    P = max(32, min(512, 4 * 1024 * 1024 // n))
    h = np.random.default_rng(seed).uniform(0.2, 1.0, (P, n)).astype(np.float32)
    return P, h


def _micro_line(impl: str, rows: list, extra: dict) -> dict:
    return {"metric": "micro_lp_adam_tflops", "impl": impl, "unit": "TFLOP/s",
            "higher_is_better": True, "n_gpus": 1, "data": "synthetic",
            "config": {"workload": "src/main.cu:294-320 benchmark: n = 128 .. 4096, "
                                   "P = max(32, min(512, 4M/n)), 100 local-search iterations "
                                   "p 8->200, lr 0.05->0.005, then one fp64 evaluation",
                       **extra},
            "rows": rows}


def micro_arm(args) -> None:
    """Our kernels on the reference's own benchmark (--bench of src/main.cu):
    the tensor-core step (BF16x3) and the FP32 SIMT step per n, and the fp64
    evaluation; CUDA events on the launching stream."""
    import torch
    ws, rank, local = _dist()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    import sidon_b200
    sidon_b200.load(build=not (ROOT / "sidon-autocorrelation-bound_b200" / "libsidon_b200.so").exists())
    from sidon_b200 import kernels
    stream = torch.cuda.current_stream()

    def timed(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / 1e3

    rows = []
    for n in MICRO_N:
        P, h = _micro_setup(n)
        row = {"n": n, "P": P}
        flop = 4.0 * n * n * P * 100
        for prec in ("bf16x3", "fp32"):
            x = torch.as_tensor(h, device=dev)
            mom, vel = torch.empty_like(x), torch.empty_like(x)
            kernels.run_local_search(x, 10, 8.0, 8.0, 0.01, 0.01, mom=mom, vel=vel, precision=prec)
            dt = timed(lambda: kernels.run_local_search(x, 100, 8.0, 200.0, 0.05, 0.005, mom=mom,
                                                        vel=vel, precision=prec))
            row[f"ls_ms_{prec}"] = dt * 1e3
            row[f"tflops_{prec}"] = flop / dt / 1e12
        F = torch.empty(P, dtype=torch.float64, device=dev)
        nact = torch.empty(P, dtype=torch.int32, device=dev)
        kernels.run_eval(x, out_F=F, out_nactive=nact)
        row["eval_ms"] = timed(lambda: kernels.run_eval(x, out_F=F, out_nactive=nact)) * 1e3
        rows.append(row)
    print(json.dumps(_micro_line("ours", rows, {"precision": "bf16x3 and fp32 SIMT"})))


def reference_micro_arm(args) -> None:
    """The reference's kernels on its own benchmark: kLocalSearch<float> and
    kEval<float,double> built for sm_100a from its sources (oracle/_ref),
    launched as runLocalSearch / runEval do."""
    ws, rank, local = _dist()
    if rank != 0:
        return
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    if not oracle.have_ref():
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref not built (reference sources absent here)"}))
        return
    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ref = oracle.ref_main()
    stream = torch.cuda.current_stream()
    rows = []
    for n in MICRO_N:
        P, h = _micro_setup(n)
        x = torch.as_tensor(h, device=dev)
        mom, vel = torch.empty_like(x), torch.empty_like(x)
        F = torch.empty(P, dtype=torch.float64, device=dev)
        nact = torch.empty(P, dtype=torch.int32, device=dev)
        assert ref.ref_gpu_local_search(x.data_ptr(), mom.data_ptr(), vel.data_ptr(), n, P, 10,
                                        8.0, 8.0, 0.01, 0.01, None) == 0
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        rc = ref.ref_gpu_local_search(x.data_ptr(), mom.data_ptr(), vel.data_ptr(), n, P, 100,
                                      8.0, 200.0, 0.05, 0.005, None)
        b.record(stream)
        torch.cuda.synchronize()
        assert rc == 0
        dt = a.elapsed_time(b) / 1e3
        a.record(stream)
        rc = ref.ref_gpu_eval(x.data_ptr(), n, P, F.data_ptr(), nact.data_ptr(), 1e-4, None)
        b.record(stream)
        torch.cuda.synchronize()
        assert rc == 0
        rows.append({"n": n, "P": P, "ls_ms": dt * 1e3,
                     "tflops": 4.0 * n * n * P * 100 / dt / 1e12,
                     "eval_ms": a.elapsed_time(b)})
    print(json.dumps(_micro_line("reference", rows, {"kernels": "reference kLocalSearch<float>, "
                                                     "kEval<float,double>, sm_100a build"})))


# ----------------------------- memetic generations ---------------------------
def memetic_arm(args) -> None:
    """The reference driver's generation (src/main.cu:586-785) at its default
    settings -- 256 candidates in 8 islands, 2 elites, warm / medium / cold
    tiers of 4000 / 6666 / 20000 steps with p up to 20000, 6 Frank-Wolfe
    rounds of 500 iterations, tabu tenure 6 -- at one ladder level of n
    cells, on the device with the policy included.  One warm-up generation,
    then --steps generations replayed from one CUDA graph.  Prints one JSON
    line (its own metric; not the headline line)."""
    import torch
    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    import sidon_b200
    sidon_b200.load(build=not (ROOT / "sidon-autocorrelation-bound_b200" / "libsidon_b200.so").exists())
    from sidon_b200 import kernels, synth

    n, P, G = args.memetic_n, 256, max(1, args.steps)
    cfg = kernels.generation_config(precision=args.precision, fw_precision=args.fw_precision,
                                    seed=20260905 + rank)
    pop = torch.as_tensor(synth.population("lognormal", n, P, seed=2048 + rank), device=dev)
    gen = kernels.Generation(n, P, cfg, device=dev)
    seed_op = torch.full((P,), 9, dtype=torch.int32, device=dev)   # fresh level: restarts
    gen.begin_level(n, 0, seed_op)
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    gen.step(pop)                                    # warm-up: generation 0 (eager)
    e1.record(stream)
    torch.cuda.synchronize()
    first_ms = e0.elapsed_time(e1)
    s0 = gen.state()
    graph = gen.capture(pop, G)
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        e0.record(stream)
        graph.launch()
        e1.record(stream)
        torch.cuda.synchronize()
    total_ms = e0.elapsed_time(e1)
    s1 = gen.state()
    graph.close()
    ck = clk.summary()
    if rank == 0:
        steps = s1["ls_steps"] - s0["ls_steps"]
        flop = s1["flop"] - s0["flop"]
        line = {
            "metric": "memetic_generations_per_s", "value": G / (total_ms / 1e3),
            "unit": "generations/s", "n_gpus": 1, "higher_is_better": True,
            "data": "synthetic", "steps": G, "ms_per_generation": total_ms / G,
            "first_generation_ms": first_ms,
            "config": {"workload": f"memetic generation n={n} P={P} 8 islands, tiers "
                                   f"4000/6666/20000 steps p<=20000, FW 6x500, one CUDA graph "
                                   f"of {G} generations",
                       "precision": args.precision, "fw_precision": args.fw_precision},
            "local_search": {"candidate_steps_per_s": steps / (total_ms / 1e3),
                             "tflops_algorithmic_overall": flop / (total_ms / 1e3) / 1e12},
            "search": {"best_F": s1["best_F"], "level_best_F": s1["level_best_F"],
                       "cells": s1["cells"], "n_cold_last": s1["n_cold"],
                       "n_med_last": s1["n_med"], "status": s1["status"]},
            "clocks": {"sm_mhz": ck["sm_mhz"], "sm_max_mhz": ck["sm_max_mhz"],
                       "reasons": ck["reasons"]},
        }
        print(json.dumps(line))


def reference_memetic_arm(args) -> None:
    """The same generations with the reference's own implementation: its
    kernels (kLocalSearch<float> per non-empty tier, kFrankWolfe<float>,
    kEval, kSupportSig, kVariation<float>) launched through its own helpers
    (src/main.cu:152-184, 606-741, compiled from its sources into
    oracle/_ref), one after another with the driver's synchronous copies; the
    host policy between them is the oracle's restatement of the driver's
    rules.  Wall clock per generation (the driver is synchronous)."""
    ws, rank, local = _dist()
    if rank != 0:
        return
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    if not oracle.have_ref():
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref not built (reference sources absent here)"}))
        return
    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    from sidon_b200 import synth
    ref = oracle.ref_main()
    n, P, NI, seed = args.memetic_n, 256, 8, 20260905
    cold, warm, p_top, fw_rounds, fw_iters = 20000, 4000, 20000.0, 6, 500
    pol = oracle.GenerationPolicy(P, NI, 2, 6, seed, n)
    pol.begin_level(n, 0)
    pop = torch.as_tensor(synth.population("lognormal", n, P, seed=2048), device=dev)
    nxt, mom, vel = torch.empty_like(pop), torch.empty_like(pop), torch.empty_like(pop)
    i32 = dict(dtype=torch.int32, device=dev)
    skip_d, p1_d, p2_d, op_d = (torch.zeros(P, **i32) for _ in range(4))
    mode_d = torch.as_tensor(pol.mode, device=dev)
    str_d = torch.zeros(P, dtype=torch.float32, device=dev)
    fit_d = torch.zeros(P, dtype=torch.float64, device=dev)
    nact_d, nnz_d = torch.zeros(P, **i32), torch.zeros(P, **i32)
    sig_d = torch.zeros(P, dtype=torch.int64, device=dev)
    fit_h, nact_h = np.zeros(P), np.zeros(P, np.int32)
    sig_h, nnz_h = np.zeros(P, np.uint64), np.zeros(P, np.int32)
    times = []
    for g in range(1 + max(1, args.steps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        tier = np.ascontiguousarray(np.argmin(pol.tiers(cold, cold // 3, warm), axis=0),
                                    dtype=np.int32)
        fw = ref.ref_gpu_generation_search(
            pop.data_ptr(), mom.data_ptr(), vel.data_ptr(), skip_d.data_ptr(), mode_d.data_ptr(),
            tier.ctypes.data, n, P, cold, warm, p_top, fw_rounds, fw_iters, fit_d.data_ptr(),
            nact_d.data_ptr(), sig_d.data_ptr(), nnz_d.data_ptr(), fit_h.ctypes.data,
            nact_h.ctypes.data, sig_h.ctypes.data, nnz_h.ctypes.data)
        assert fw >= 0, f"reference generation failed ({fw})"
        host = pop.cpu().numpy()
        plan = pol.select(host, fit_h, nact_h, sig_h, nnz_h, fw, fw_rounds, fw_iters)
        pop.copy_(torch.from_numpy(host))
        rc = ref.ref_gpu_generation_vary(
            pop.data_ptr(), nxt.data_ptr(), n, P, p1_d.data_ptr(), p2_d.data_ptr(),
            op_d.data_ptr(), str_d.data_ptr(), plan["p1"].ctypes.data, plan["p2"].ctypes.data,
            plan["op"].ctypes.data, plan["strength"].ctypes.data, seed, int(pol.var_gen[0]))
        assert rc == 0, f"reference variation failed ({rc})"
        pop, nxt = nxt, pop
        host = pop.cpu().numpy()
        pol.post(host)
        pop.copy_(torch.from_numpy(host))
        child = np.zeros(P)
        if pol.s.gen > 0 and pol.s.gen % 5 == 0:
            assert ref.ref_gpu_eval(pop.data_ptr(), n, P, fit_d.data_ptr(), nact_d.data_ptr(),
                                    1e-4, None) == 0
            child = fit_d.cpu().numpy()
        pol.credit(child)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    timed = times[1:]
    sec = sum(timed) / len(timed)
    print(json.dumps({
        "impl": "reference", "metric": "memetic_generations_per_s", "value": 1.0 / sec,
        "unit": "generations/s", "n_gpus": 1, "higher_is_better": True, "data": "synthetic",
        "steps": len(timed), "ms_per_generation": 1e3 * sec, "first_generation_ms": 1e3 * times[0],
        "config": {"workload": f"memetic generation n={n} P={P} 8 islands, tiers "
                               f"4000/6666/20000 steps p<=20000, FW 6x500",
                   "kernels": "reference kLocalSearch/kFrankWolfe/kEval/kSupportSig/"
                              "kVariation<float>, sm_100a build of its sources, sequential"},
        "search": {"best_F": pol.s.best_F, "cells": pol.s.cells},
    }))


def reference_islands_arm(args) -> None:
    """The batched uneven islands with the reference's own kernels
    (kLocalSearch<float>, kFrankWolfe<float>, kEval<float,double>, built for
    sm_100a from its sources into oracle/_ref).  The reference launches one
    size at a time, so the candidates run as one launch per size, one after
    another; one 250-step segment, one Frank-Wolfe step (200 iterations) and
    one evaluation per size are timed with CUDA events and the 5000-step
    anneal is composed from them (20 segments and Frank-Wolfe steps, 10
    evaluations for the migrations)."""
    ws, rank, local = _dist()
    if rank != 0:
        return
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    if not oracle.have_ref():
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref not built (reference sources absent here)"}))
        return
    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    from sidon_b200 import synth
    ref = oracle.ref_main()
    P, steps, seg, pdhg = args.islands_P, args.anneal_steps, args.fw_every, args.pdhg_iters
    sizes = synth.uneven_sizes(P, seed=3, levels=ISLAND_LEVELS)
    rows = synth.ragged_population(sizes, seed=3)
    stream = torch.cuda.current_stream()

    def timed(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        rc = fn()
        b.record(stream)
        torch.cuda.synchronize()
        assert rc >= 0, rc
        return a.elapsed_time(b)

    pA = 2.0
    pB = 2.0 * (1024.0 / 2.0) ** ((seg - 1) / (steps - 1))
    per_size = {}
    for n in ISLAND_LEVELS:
        idx = np.nonzero(sizes == n)[0]
        if idx.size == 0:
            continue
        x = torch.tensor(np.stack([rows[i] for i in idx]).astype(np.float32), device=dev)
        Pg = x.shape[0]
        mom, vel = torch.empty_like(x), torch.empty_like(x)
        F = torch.empty(Pg, dtype=torch.float64, device=dev)
        nact = torch.empty(Pg, dtype=torch.int32, device=dev)
        ref.ref_gpu_local_search(x.data_ptr(), mom.data_ptr(), vel.data_ptr(), n, Pg, 2, pA, pA,
                                 1e-3, 1e-3, None)
        ls = timed(lambda: ref.ref_gpu_local_search(x.data_ptr(), mom.data_ptr(), vel.data_ptr(),
                                                    n, Pg, seg, pA, pB, 1e-3, 1e-3, None))
        fw = timed(lambda: ref.ref_gpu_frank_wolfe(x.data_ptr(), n, Pg, 1, pdhg, 12, 0.30, None))
        ev = timed(lambda: ref.ref_gpu_eval(x.data_ptr(), n, Pg, F.data_ptr(), nact.data_ptr(),
                                            1e-4, None))
        per_size[int(n)] = {"candidates": int(Pg), "segment_ms": ls, "frank_wolfe_ms": fw,
                            "eval_ms": ev}
    n_seg = steps // seg
    seg_ms = sum(v["segment_ms"] for v in per_size.values())
    fw_ms = sum(v["frank_wolfe_ms"] for v in per_size.values())
    ev_ms = sum(v["eval_ms"] for v in per_size.values())
    total_s = (n_seg * (seg_ms + fw_ms) + (steps // 500) * ev_ms) / 1e3
    print(json.dumps({
        "impl": "reference", "metric": "island_anneal_candidate_steps_per_s",
        "value": P * steps / total_s, "unit": "candidate-steps/s", "n_gpus": 1,
        "higher_is_better": True, "data": "synthetic", "anneal_seconds": total_s,
        "config": {"workload": f"batched uneven islands: P={P}, n uniform over "
                               f"{list(ISLAND_LEVELS)}, {steps} steps, FW every {seg} "
                               f"({pdhg} PDHG), reference kernels one launch per size",
                   "composition": f"{n_seg} x (one {seg}-step segment + one Frank-Wolfe step) "
                                  f"+ {steps // 500} evaluations, each timed once per size"},
        "phase_ms": {"local_search_segment": seg_ms, "frank_wolfe_step": fw_ms,
                     "evaluation": ev_ms},
        "per_size": per_size,
    }))


def reference_ladder_arm(args) -> None:
    """The large ladder's levels with the reference's own kernels
    (kLocalSearch<float>, kFrankWolfe<float>, built for sm_100a from its
    sources): per level the Adam segment and one Frank-Wolfe round on the
    same B candidates, timed with CUDA events, where the reference's kernels
    fit one CTA's shared memory; the others are reported as not runnable
    (its driver refuses n > 16384, src/main.cu:391-399)."""
    ws, rank, local = _dist()
    if rank != 0:
        return
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    if not oracle.have_ref():
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref not built (reference sources absent here)"}))
        return
    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    from sidon_b200 import synth
    ref = oracle.ref_main()
    B, steps, pdhg = args.ladder_B, args.ladder_steps, args.ladder_pdhg
    ladder = [int(x) for x in args.ladder_levels.split(",")]
    optin = torch.cuda.get_device_properties(dev).shared_memory_per_block_optin
    stream = torch.cuda.current_stream()

    def timed(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        rc = fn()
        b.record(stream)
        torch.cuda.synchronize()
        return rc, a.elapsed_time(b)

    levels = []
    for n in ladder:
        x = torch.as_tensor(synth.population("structured", n, B, seed=4), device=dev)
        mom, vel = torch.empty_like(x), torch.empty_like(x)
        row = {"n": n}
        if 4 * (3 * n + 8 + 8 + 64) > optin:      # localSearchSmem<float> (kernels.cuh:161-162)
            row["adam"] = "not runnable: the reference's local search does not fit shared memory"
        else:
            ref.ref_gpu_local_search(x.data_ptr(), mom.data_ptr(), vel.data_ptr(), n, B, 2, 4.0,
                                     4.0, 1e-3, 1e-3, None)
            rc, ms = timed(lambda: ref.ref_gpu_local_search(x.data_ptr(), mom.data_ptr(),
                                                            vel.data_ptr(), n, B, steps, 4.0,
                                                            64.0, 1e-3, 1e-3, None))
            assert rc == 0, rc
            row["adam_steps_per_s"] = steps / (ms / 1e3)
            row["adam_tflops_algorithmic"] = 4.0 * n * n * B * steps / (ms / 1e3) / 1e12
        rc, ms = timed(lambda: ref.ref_gpu_frank_wolfe(x.data_ptr(), n, B, 1, pdhg, 12, 0.30, None))
        assert rc >= 0, rc
        if rc == 1:
            row["fw_round_ms"] = ms
        else:
            row["fw"] = "not runnable: kFrankWolfe does not fit shared memory (main.cu:173)"
        if n > 16384:
            row["driver"] = "refused by the reference driver (n > 16384, main.cu:391-399)"
        levels.append(row)
    print(json.dumps({
        "impl": "reference", "metric": "ladder_adam_steps_per_s_at_65536",
        "value": levels[-1].get("adam_steps_per_s"), "unit": "batched steps/s",
        "n_gpus": 1, "higher_is_better": True, "data": "synthetic",
        "config": {"workload": f"large ladder B={B}: {ladder}, {steps} Adam steps + 1 FW round "
                               f"({pdhg} PDHG) per level, reference kernels"},
        "levels": levels,
    }))


# --------------------------------- whole search ------------------------------
SEARCH_LADDER = (64, 128, 256, 512, 1024, 2048)     # the reference driver's default ladder


def search_arm(args) -> None:
    """The whole search at the reference driver's defaults (src/main.cu:41-58:
    ladder 64 ... 2048, 256 candidates in 8 islands, 2 elites, warm / cold
    4000 / 20000 steps, p up to 20000, 6 Frank-Wolfe rounds of 500 iterations,
    40000-step fp64 polish of 8 starts) for --search-seconds of wall clock,
    through sidon_search (BF16x3 local search; the Frank-Wolfe step in fp32
    as the reference, or --fw-precision).  Prints the certified F reached
    (lower is better)."""
    import torch
    ws, rank, local = _dist()
    if rank != 0:
        return
    fw = args.fw_precision or "fp32"
    torch.cuda.set_device(local)
    import sidon_b200
    sidon_b200.load(build=not (ROOT / "sidon-autocorrelation-bound_b200" / "libsidon_b200.so").exists())
    from sidon_b200 import kernels
    gens = []
    t0 = time.perf_counter()
    best, F = kernels.search(ladder=SEARCH_LADDER, P=256, seconds=args.search_seconds,
                             gens_per_graph=2, polish_iters=40000, polish_top=8,
                             gen=kernels.generation_config(precision=args.precision,
                                                           fw_precision=fw,
                                                           seed=20260905),
                             progress=lambda d, b: gens.append((d["n"], d["gen"])))
    wall = time.perf_counter() - t0
    if args.search_out:
        from sidon_b200 import formats
        formats.write_certificate(args.search_out, best, F, "sidon_b200 sidon_search")
    per_level = {}
    for n, g in gens:
        per_level[n] = max(per_level.get(n, 0), g)
    print(json.dumps({
        "metric": "search_F_at_budget", "value": F, "unit": "F (certified, hostF)",
        "higher_is_better": False, "n_gpus": 1, "data": "synthetic seeds",
        "seconds": wall, "n": int(best.size), "generations_per_level": per_level,
        "config": {"workload": f"whole search, reference defaults, {args.search_seconds:.0f} s "
                               f"budget, ladder {list(SEARCH_LADDER)}",
                   "precision": args.precision, "fw_precision": fw},
    }))


def reference_search_arm(args) -> None:
    """The reference's own search driver, unmodified (src/main.cu built for
    sm_100a into oracle/_ref/sidon_ref), with its defaults and the same
    wall-clock budget; its result file gives the F it reports."""
    ws, rank, local = _dist()
    if rank != 0:
        return
    exe = ROOT / "oracle" / "_ref" / "sidon_ref"
    if not exe.exists():
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/sidon_ref not built (reference sources absent here)"}))
        return
    import tempfile
    from sidon_b200 import formats
    with tempfile.TemporaryDirectory() as td:
        out = pathlib.Path(td) / "best"
        t0 = time.perf_counter()
        r = subprocess.run([str(exe), "--seconds", str(args.search_seconds), "--out", str(out),
                            "--quiet"], capture_output=True, text=True,
                           env={**os.environ, "CUDA_VISIBLE_DEVICES": str(local)})
        wall = time.perf_counter() - t0
        if r.returncode != 0:
            print(json.dumps({"impl": "reference",
                              "unavailable": f"reference driver exited {r.returncode}"}))
            return
        text = (pathlib.Path(str(out) + ".txt")).read_text()
        a = formats.load_vec(str(out) + ".txt")
    F = None
    for ln in text.splitlines():
        if ln.startswith("F "):
            F = float(ln.split()[1])
    levels = {}
    for ln in r.stdout.splitlines():
        if ln.startswith("=== level n=") and "done" in ln:
            parts = ln.split()
            levels[int(parts[2].split("=")[1].rstrip(":"))] = int(parts[parts.index("after") + 1])
    import sidon_b200
    hostF = sidon_b200.load().sidon_hostF(np.ascontiguousarray(a).ctypes.data, int(a.size))
    print(json.dumps({
        "impl": "reference", "metric": "search_F_at_budget", "value": F,
        "unit": "F (its own report)", "hostF_of_its_vector": hostF,
        "higher_is_better": False, "n_gpus": 1,
        "data": "synthetic seeds", "seconds": wall, "n": int(a.size),
        "generations_per_level": levels,
        "config": {"workload": f"whole search, reference defaults, {args.search_seconds:.0f} s "
                               f"budget, ladder {list(SEARCH_LADDER)}",
                   "program": "the unmodified reference driver (src/main.cu), sm_100a build"},
    }))


# --------------------------------- large ladder -----------------------------
LADDER = (8192, 16384, 32768, 65536)


def ladder_arm(args) -> None:
    """The large ladder: B = 32 plain-method candidates at n = 8192, cell
    split n -> 2n up to 65536 with the certified F checked bit for bit at
    every split; at each level an Adam + adjoint segment (b recomputed every
    step, never stored), one Chambolle-Pock Frank-Wolfe round and an fp64
    island ranking + migration (4 islands of 8, top 1); BF16x3 search, exact
    fp64 certification of the final F.  Prints one JSON line (its own metric)."""
    import torch
    import torch.distributed as dist
    ws, rank, local = _dist()
    if ws > 1:
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    import sidon_b200
    sidon_b200.load(build=not (ROOT / "sidon-autocorrelation-bound_b200" / "libsidon_b200.so").exists())
    from sidon_b200 import islands, kernels, synth

    B = args.ladder_B
    prec = args.precision if args.precision != "fp32" else "bf16x3"
    stream = torch.cuda.current_stream()
    ladder = [int(x) for x in args.ladder_levels.split(",")]
    pop = torch.as_tensor(synth.population("structured", ladder[0], B, seed=4 + rank), device=dev)
    F_start = kernels.certify(pop)[0].cpu().numpy()

    def timed(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b)

    # warm-up of every kernel on a small case
    w = torch.as_tensor(synth.population("structured", 1024, 2, seed=1), device=dev)
    kernels.run_local_search_large(w, 3, 2.0, 4.0, 1e-3, 1e-3, precision=prec, q=512)
    kernels.run_frank_wolfe_large(w, 1, 2, 2, 0.3, tau=0.9, sigma=0.9, precision=prec, q=512)
    torch.cuda.synchronize()

    levels = []
    steps, pdhg = args.ladder_steps, args.ladder_pdhg
    total_ms = 0.0
    with Clocks(local) as clk:
        for li, n in enumerate(ladder):
            if li > 0:
                before = kernels.certify_large(pop)[0]
                pop = kernels.refine(pop)
                after = kernels.certify_large(pop)[0]
                split_exact = bool(torch.equal(before, after))
            else:
                split_exact = None
            if args.ladder_q > 0:
                q_sel = args.ladder_q
            else:
                q_sel, _ = kernels.autotune_large(n, B, prec)
            ws_t = kernels.large_workspace(n, B, q_sel, dev, prec)
            mom, vel = torch.empty_like(pop), torch.empty_like(pop)
            # p grows geometrically over the ladder, one range per level
            pA = 2.0 * (512.0 ** (li / len(ladder)))
            pB = 2.0 * (512.0 ** ((li + 1) / len(ladder)))
            ls_ms = timed(lambda: kernels.run_local_search_large(
                pop, steps, pA, pB, 1e-3, 1e-3, precision=prec, q=q_sel, workspace=ws_t, mom=mom,
                vel=vel))
            fw_ms = timed(lambda: kernels.run_frank_wolfe_large(
                pop, 1, pdhg, 12, 0.3, tau=0.9, sigma=0.9, precision=prec, q=q_sel,
                workspace=ws_t))
            fit = torch.empty(B, dtype=torch.float64, device=dev)
            n_isl = 4 if B % 4 == 0 and B >= 8 else 1

            def mig():
                f, _ = kernels.run_eval(pop, with_nactive=False)
                fit.copy_(f)
                # islands per rank on one global ring (NCCL hop between ranks)
                islands.migrate_across_ranks(pop, fit, n_isl, 1 if B // n_isl >= 2 else 0)
            mig_ms = timed(mig)
            ls_ms = islands.max_over_ranks(ls_ms, dev)
            fw_ms = islands.max_over_ranks(fw_ms, dev)
            mig_ms = islands.max_over_ranks(mig_ms, dev)
            total_ms += ls_ms + fw_ms + mig_ms
            Fl = kernels.certify_large(pop)[0].cpu().numpy()
            flop = 4.0 * n * n * B * steps
            levels.append({"n": n, "split_F_bit_exact": split_exact,
                           "schedule": "fused" if q_sel >= n else f"super-blocks q={q_sel}",
                           "adam_steps_per_s": steps / (ls_ms / 1e3),
                           "adam_tflops_algorithmic": flop / (ls_ms / 1e3) / 1e12,
                           "fw_round_ms": fw_ms, "fw_pdhg_iters": pdhg,
                           "fw_tflops_algorithmic": (4.0 * n * n * pdhg + 26.0 * n * n) * B
                           / (fw_ms / 1e3) / 1e12,
                           "migrate_ms": mig_ms,
                           "F_median": float(np.nanmedian(Fl)), "F_best": float(np.nanmin(Fl))})
            del ws_t
    Fc, _, _, _ = kernels.certify_large(pop)
    Fe, _ = kernels.run_eval(pop, with_nactive=False)
    host_check = [abs(Fc[p].item() - kernels.host_f(pop[p].cpu().double().numpy())) /
                  Fc[p].item() for p in range(min(2, B))]
    ck = clk.summary()
    best = islands.global_best(Fc) if ws > 1 else None
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps({
            "metric": "ladder_adam_steps_per_s_at_65536", "value": levels[-1]["adam_steps_per_s"],
            "unit": "batched steps/s (per rank; ranks run B candidates each)", "n_gpus": ws,
            "global_best": best, "higher_is_better": True,
            "data": "synthetic", "dtype": prec,
            "config": {"workload": f"large ladder B={B}: {ladder}, cell splits, "
                                   f"{steps} Adam steps + 1 FW round ({pdhg} PDHG) + "
                                   f"migration per level", "precision": prec},
            "levels": levels, "ladder_seconds": total_ms / 1e3,
            "F": {"start_median": float(np.median(F_start)),
                  "final_certified_median": float(np.nanmedian(Fc.cpu().numpy())),
                  "final_certified_best": float(np.nanmin(Fc.cpu().numpy())),
                  "certified_vs_eval_max_rel": float(((Fc - Fe).abs() / Fe).max().item()),
                  "certified_vs_hostF_rel": host_check},
            "clocks": {"sm_mhz": ck["sm_mhz"], "sm_max_mhz": ck["sm_max_mhz"],
                       "reasons": ck["reasons"]},
        }))


def _traffic(prec: str):
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get(prec)
    return None


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default=os.environ.get("SIDON_BENCH_PRECISION", "bf16x3"),
                    choices=["fp32", "bf16x3", "bf16x1"])
    ap.add_argument("--workload", default="lp_adam",
                    choices=["lp_adam", "islands", "ladder", "memetic", "micro", "search"])
    ap.add_argument("--search-seconds", type=float, default=60.0)
    ap.add_argument("--search-out", default="", help="write the certificate (JSON) here")
    ap.add_argument("--memetic-n", type=int, default=2048)
    ap.add_argument("--ladder-B", type=int, default=32)
    ap.add_argument("--ladder-steps", type=int, default=200)
    ap.add_argument("--ladder-pdhg", type=int, default=100)
    ap.add_argument("--ladder-levels", default=",".join(str(x) for x in LADDER))
    ap.add_argument("--ladder-q", type=int, default=0, help="super-block size (0: autotune)")
    ap.add_argument("--islands-P", type=int, default=1024)
    ap.add_argument("--anneal-steps", type=int, default=5000)
    ap.add_argument("--fw-every", type=int, default=250)
    ap.add_argument("--pdhg-iters", type=int, default=200)
    ap.add_argument("--fw-precision", default=None, choices=["fp32", "bf16x3", "bf16x1"],
                    help="Frank-Wolfe arithmetic (default: bf16x3; fp32 for --workload search)")
    ap.add_argument("--cpu-budget", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.fw_precision is None and args.workload != "search":
        args.fw_precision = "bf16x3"
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        if args.workload == "memetic":
            reference_memetic_arm(args)
        elif args.workload == "micro":
            reference_micro_arm(args)
        elif args.workload == "islands":
            reference_islands_arm(args)
        elif args.workload == "ladder":
            reference_ladder_arm(args)
        elif args.workload == "search":
            reference_search_arm(args)
        else:
            reference_arm(args)
    elif args.workload == "islands":
        islands_arm(args)
    elif args.workload == "ladder":
        ladder_arm(args)
    elif args.workload == "memetic":
        memetic_arm(args)
    elif args.workload == "micro":
        micro_arm(args)
    elif args.workload == "search":
        search_arm(args)
    else:
        our_arm(args)


if __name__ == "__main__":
    main()

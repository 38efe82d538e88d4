#!/usr/bin/env python
"""bench.py -- grid-cell time steps per second of the PaScaL_TCS step on B200.

One "step" is one full time step of main.f90:129-223 (energy ADI, momentum
ADI, FFT pressure Poisson solve, projection, Div/CFL/Nu/KE) on one
HBM-resident case.  Default workload: the largest single-GPU case, 512^3
plain FP64 with temperature-dependent water properties (Ra = 1e9, Pr = 7,
dt = 5e-5, tanh y-stretching gamma = 2, seeded conduction profile + 0.01
noise, seed 2), where the FP32-mixed target is stated.  A plain-FP64 workload
also times its FP32-mixed counterpart and states the mixed form's error
against the FP64 form after the same steps; the default run adds the 256^3
water case (gamma 1.5, Ra 1e8, dt 2e-4, seed 1) in both forms as an extra key.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

With N > 1 (torchrun, one process per GPU) every rank advances its own
replica of the case: a single case does not shard on this path, so there is
no data-path collective; the barrier and the max-over-ranks timing use NCCL.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
TUNE_CACHE = os.path.join(ROOT, "pascal_tcs_b200", "tune_cache.txt")

_CASES = {
    # the 256^3 water case the headline metric is quoted on
    "rb256_water": dict(n1m=256, n2m=256, n3m=256, gamma2=1.5, property_set=1, Pr=7.0, Ra=1e8,
                        DeltaT=10.0, dtStart=2e-4, fixed_dt=1, seed=1, noise_amp=0.01),
    "rb64_const": dict(n1m=64, n2m=64, n3m=64, gamma2=1.5, property_set=0, Pr=0.71, Ra=1e5,
                       dtStart=1e-3, fixed_dt=1, seed=0, noise_amp=0.01),
    "rb512_water": dict(n1m=512, n2m=512, n3m=512, gamma2=2.0, property_set=1, Pr=7.0, Ra=1e9,
                        DeltaT=10.0, dtStart=5e-5, fixed_dt=1, seed=2, noise_amp=0.01),
    # profiling size: inputs still larger than L2, about 1.3 GB on the device
    "rb192_water": dict(n1m=192, n2m=192, n3m=192, gamma2=1.5, property_set=1, Pr=7.0, Ra=1e8,
                        DeltaT=10.0, dtStart=2e-4, fixed_dt=1, seed=1, noise_amp=0.01),
    # profiling size of the 512^3 case's line shapes: the same 512-row z lines on
    # 128^2 planes (67 MB per field, about 1.7 GB on the device)
    "rbz512_water": dict(n1m=128, n2m=128, n3m=512, gamma2=2.0, property_set=1, Pr=7.0, Ra=1e9,
                         DeltaT=10.0, dtStart=5e-5, fixed_dt=1, seed=2, noise_amp=0.01),
}
# precision 0: plain FP64; 1: FP32-mixed
WORKLOADS = {f"{k}_{form}": dict(v, precision=prec) for k, v in _CASES.items()
             for form, prec in (("fp64", 0), ("mixed", 1))}
# the batched ensemble: 48 independent cases advanced together on one GPU
WORKLOADS.update({"ens48_fp64": dict(ensemble=48, precision=0), "ens48_mixed": dict(ensemble=48, precision=1)})


def ensemble_cases(n: int, precision: int, seed: int = 2026) -> list[dict]:
    """n seeded cases: every axis drawn from {64, 96, 128, 160, 192}, Ra
    log-uniform in [1e5, 1e7], Pr = 7 with water properties or Pr = 0.71 with
    constant properties, noise seed = case index, fixed dt 2e-4 (CFL-safe)."""
    rng = np.random.default_rng(seed)
    sizes = [64, 96, 128, 160, 192]
    out = []
    for i in range(n):
        n1, n2, n3 = (int(rng.choice(sizes)) for _ in range(3))
        ra = float(10.0 ** rng.uniform(5.0, 7.0))
        water = bool(rng.integers(0, 2))
        out.append(dict(n1m=n1, n2m=n2, n3m=n3, gamma2=1.5, property_set=1 if water else 0,
                        Pr=7.0 if water else 0.71, Ra=ra, DeltaT=10.0, dtStart=2e-4, fixed_dt=1, seed=i,
                        noise_amp=0.01, precision=precision))
    return out


def lpt_shard(cases: list[dict], ws: int, rank: int) -> list[dict]:
    """Longest-processing-time bin packing of the cases over the ranks by cell count."""
    load = [0] * ws
    mine = []
    order = sorted(range(len(cases)), key=lambda i: -cases[i]["n1m"] * cases[i]["n2m"] * cases[i]["n3m"])
    for i in order:
        r = min(range(ws), key=lambda q: load[q])
        load[r] += cases[i]["n1m"] * cases[i]["n2m"] * cases[i]["n3m"]
        if r == rank:
            mine.append(cases[i])
    return mine


# Water cases restart from their seeded state every ENSEMBLE_RESET steps
# (they blow up after ~20 steps in the reference algorithm).
ENSEMBLE_RESET = 8
# The water cases blow up after ~10 steps (256^3) in the reference algorithm itself (the
# non-Boussinesq pressure term sees dPhat = 0 in the wall ghost row and dPhat grows
# ~1.6x per step at the bottom wall; the oracle restatement and this library stop at
# the same step).  Their timed steps therefore restart from the seeded initial state,
# kept on the device, every RESET_EVERY steps; the restore copies are timed too.
RESET_EVERY = {f"{k}_{form}": n for k, n in (("rb256_water", 8), ("rb512_water", 5), ("rb192_water", 8),
                                             ("rbz512_water", 5))
               for form in ("fp64", "mixed")}

# Compulsory-traffic model: arrays each kernel must stream once (reads +
# writes) per interior cell; properties and tridiagonal coefficients are
# recomputed, 1-D metrics, 2-D property tables and ghosts ignored.  Whole step:
# 109 arrays at 8 B (872 B per cell-step) in the FP64 form.  The FP32-mixed
# form stores every array in FP32 (its FP64 parts live in registers and shared
# memory) and adds the velocity's low words: read and written by the pressure
# right-hand side (6) and the projection (6), read by the diagnostics (3), so
# 124 arrays at 4 B = 496 B per cell-step.
STEP_ARRAYS = 109
LO_ARRAYS = {"prhs_fftx": 6, "projection": 6, "post": 3}


def step_bytes_per_cell(esize: int) -> int:
    return STEP_ARRAYS * esize if esize == 8 else (STEP_ARRAYS + sum(LO_ARRAYS.values())) * esize
KERNEL_ARRAYS = {"thermal_z": 5, "thermal_x": 4, "thermal_y": 4,
                 "du_z": 6, "du_x": 4, "du_y": 4, "dv_z": 7, "dv_x": 4, "dv_y": 4,
                 "dw_z": 8, "dw_x": 4, "dw_y": 4, "blockld_v": 5, "blockld_u": 6,
                 "prhs_fftx": 11, "fftz_fwd": 2, "modal_tdma": 2, "fftz_inv": 2, "ifftx": 2,
                 "projection": 14, "post": 4}


def kernel_bytes(name: str, n1: int, n2: int, n3: int, esize: int = 8) -> float:
    cells = n1 * n2 * n3
    h1p = n1 // 2 + 1
    spec = 2.0 * esize * h1p * n2 * n3                # one pass over the complex half-spectrum
    if name in ("fftz_fwd", "modal_tdma", "fftz_inv"):
        return 2 * spec
    if name == "ifftx":
        return spec + esize * cells
    lo = LO_ARRAYS.get(name, 0) if esize == 4 else 0
    if name == "prhs_fftx":
        return (10 + lo) * esize * cells + spec
    if name.startswith("dv_") or name == "blockld_v":
        cells = n1 * (n2 - 1) * n3
    return (KERNEL_ARRAYS[name] + lo) * esize * cells


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(kernel: str, workload: str):
    """dram__bytes_read.sum + dram__bytes_write.sum per launch from the committed
    ncu summary (profiles/traffic.json), or None."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    return d.get(workload, {}).get(kernel)


def profiled_fp64_flop_per_cell(kernel: str):
    """FP64 FLOP per cell of an FP64 line kernel (DFMA = 2) from the committed
    ncu instruction counts (profiles/fp64_flops.json), or None."""
    p = os.path.join(ROOT, "profiles", "fp64_flops.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    return d.get(kernel, {}).get("fp64_flop_per_cell")


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 100 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device, self.proc, self.lines = device, None, []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", str(self.device)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def wait_first(self, timeout: float = 5.0):
        """Block until nvidia-smi has produced a sample, so the timed region is covered."""
        t0 = time.time()
        while self.proc and not self.lines and time.time() - t0 < timeout:
            time.sleep(0.02)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1])); mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(n_gpus: int):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def dist_max(x: float, ws: int) -> float:
    """Max over ranks (the slowest replica sets the job time)."""
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(ws: int):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_baseline(cfg: dict, target_s: float = 20.0, threads: int | None = None) -> dict:
    """The oracle (one-rank C restatement of the reference's CPU path; the
    Fortran/MPI/FFTW reference has no toolchain here) on the host cores: one
    untimed step, then as many whole steps as fit about target_s (at least 1)."""
    from oracle import oracle as O
    threads = threads or os.cpu_count() or 1
    O.set_threads(threads)
    o = O.Oracle(**{k: v for k, v in cfg.items() if k not in ("device", "precision")})
    t0 = time.perf_counter(); o.step(1); t1 = time.perf_counter()
    first = t1 - t0
    n = max(1, min(20, int(target_s / max(first, 1e-3))))
    t0 = time.perf_counter(); o.step(n); t1 = time.perf_counter()
    cells = cfg["n1m"] * cfg["n2m"] * cfg["n3m"]
    del o
    return {"value": cells * n / (t1 - t0), "unit": "cell-steps/s", "cores": threads, "kind": "port",
            "sample": f"{n} full time step(s) of the same {cfg['n1m']}x{cfg['n2m']}x{cfg['n3m']} case "
                      f"(after 1 untimed), oracle C restatement with OpenMP",
            "seconds": t1 - t0}


def run_reference_ensemble(args, cfg, workload, O, threads) -> int:
    """The CPU restatement on a bounded sample of the ensemble: the first two
    cases, each for K steps (one case at a time, as one MPI job would)."""
    cases = ensemble_cases(cfg["ensemble"], cfg["precision"])[:2]
    cells_steps, el = 0, 0.0
    for c in cases:
        fresh = lambda: O.Oracle(**{k: v for k, v in c.items() if k not in ("device", "precision")})
        el += oracle_steps(fresh, args.steps, ENSEMBLE_RESET)
        cells_steps += c["n1m"] * c["n2m"] * c["n3m"] * args.steps
    v = cells_steps / el
    sample = (f"{args.steps} steps of each of the first 2 of the {cfg['ensemble']} cases, one at a time, "
              f"restarting from the seeded state every {ENSEMBLE_RESET} steps as the GPU arm does")
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    line = {"impl": "reference", "metric": ensemble_metric(cfg), "value": v, "unit": "cell-steps/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": None,
            "higher_is_better": True, "scaling": "strong" if ws > 1 else "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded conduction profiles + uniform noise 0.01, zero velocity",
            "config": ensemble_config(cfg, workload, ws),
            "cpu_baseline": {"value": v, "unit": "cell-steps/s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def form_name(cfg: dict) -> str:
    return "FP32-mixed" if cfg.get("precision", 0) else "FP64 plain"


def l2_note(field_mb: float, step_mb: float) -> str:
    """How the timed steps stand against the 126 MB L2 (no flush between steps)."""
    if field_mb > 126.0:
        return "inputs larger than L2 (each field %.0f MB)" % field_mb
    return "each field %.1f MB, but a step streams %.0f MB, more than the 126 MB L2" % (field_mb, step_mb)


def single_metric(cfg: dict) -> str:
    return f"cell-steps/s ({form_name(cfg)}, one {cfg['n1m']}x{cfg['n2m']}x{cfg['n3m']} case per GPU)"


def single_config(cfg: dict, workload: str, ws: int) -> dict:
    """The workload a one-case line describes (the same dict in both arms)."""
    n1, n2, n3 = cfg["n1m"], cfg["n2m"], cfg["n3m"]
    esize = 4 if cfg.get("precision", 0) else 8
    return {"workload": workload, "grid": [n1, n2, n3],
            "properties": "water" if cfg["property_set"] == 1 else "constant",
            "Ra": cfg["Ra"], "Pr": cfg["Pr"], "dt": cfg["dtStart"], "precision": form_name(cfg),
            "parallelism": "replicas" if ws > 1 else "single",
            "l2": l2_note(esize * (n1 + 2) * (n2 + 2) * (n3 + 2) / 1e6, step_bytes_per_cell(esize) * n1 * n2 * n3 / 1e6),
            "timing": "eager launches with one event-probed kernel; CUDA events on the solver stream",
            "restart_every_steps": RESET_EVERY.get(workload, 0) or None}


def ensemble_metric(cfg: dict) -> str:
    return f"cell-steps/s ({form_name(cfg)}, ensemble of {cfg['ensemble']} cases)"


def ensemble_config(cfg: dict, workload: str, ws: int) -> dict:
    """The workload an ensemble line describes (the same dict in both arms)."""
    allcases = ensemble_cases(cfg["ensemble"], cfg["precision"])
    total_cells = sum(c["n1m"] * c["n2m"] * c["n3m"] for c in allcases)
    esize = 4 if cfg["precision"] else 8
    return {"workload": workload, "cases": len(allcases), "cases_on_rank0": len(lpt_shard(allcases, ws, 0)),
            "grids": "each axis from {64,96,128,160,192}, seed 2026", "Ra": "log-uniform 1e5..1e7",
            "Pr": "7 (water) or 0.71 (constant)", "dt": 2e-4, "precision": form_name(cfg),
            "parallelism": f"LPT bin-packing of cases over {ws} GPU(s)" if ws > 1 else "single",
            "l2": "working set of %.1f GB, larger than L2" % (total_cells * esize * 24 / 1e9 / ws),
            "timing": "one CUDA graph per ensemble step, in the form the auto selection keeps; CUDA events around the region",
            "restart_every_steps": ENSEMBLE_RESET}


def oracle_steps(fresh, k: int, reset: int, warmup: int = 0) -> float:
    """Run the oracle for `warmup` untimed then k timed steps; with a reset
    period, restart from the seeded state (a fresh oracle, built outside the
    timed region) before it reaches the step at which the case blows up.
    Returns the timed seconds."""
    o, since, el = fresh(), 0, 0.0
    for n_total, timed in ((warmup, False), (k, True)):
        done = 0
        while done < n_total:
            n = n_total - done if not reset else min(n_total - done, reset - since)
            t0 = time.perf_counter()
            o.step(n)
            if timed:
                el += time.perf_counter() - t0
            done += n
            since += n
            if reset and since == reset:
                o, since = fresh(), 0
    return el


# The reference arm's CPU work per run, seconds: its timed steps are a bounded
# sample of the workload (whole time steps, as many as fit, at least 1) so that
# a --steps K --warmup W run ends within a few minutes at 512^3, where one
# oracle step takes about 20 s on 16 host cores.
REFERENCE_BUDGET_S = 90.0


def run_reference(args, cfg, workload):
    ws, rank, _ = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0
    if rank != 0:
        return 0
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    if "ensemble" in cfg:
        return run_reference_ensemble(args, cfg, workload, O, threads)
    fresh = lambda: O.Oracle(**{k: v for k, v in cfg.items() if k not in ("device", "precision")})
    reset = RESET_EVERY.get(workload, 0)
    # one untimed step sizes the sample; then min(W, the budget's share) warm-up
    # steps and min(K, the rest of the budget) timed steps
    o = fresh()
    t0 = time.perf_counter(); o.step(1); t1 = time.perf_counter()
    del o
    per = t1 - t0
    warm = max(0, min(args.warmup - 1, int(0.2 * REFERENCE_BUDGET_S / per)))
    steps = max(1, min(args.steps, int(0.8 * REFERENCE_BUDGET_S / per)))
    el = oracle_steps(fresh, steps, reset, warmup=warm)
    cells = cfg["n1m"] * cfg["n2m"] * cfg["n3m"]
    v = cells * steps / el
    sample = (f"{steps} full time step(s) after {warm + 1} warm-up step(s)"
              + (f" (the K = {args.steps} steps bounded to about {REFERENCE_BUDGET_S:.0f} s of CPU work)"
                 if steps < args.steps else "")
              + (f", restarting from the seeded state every {reset} steps as the GPU arm does" if reset else "")
              + "; the Fortran/MPI/FFTW reference has no toolchain on this image, so its one-rank C restatement runs")
    line = {"impl": "reference", "metric": single_metric(cfg), "value": v,
            "unit": "cell-steps/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * el / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic: seeded conduction profile + uniform noise 0.01, zero velocity",
            "config": single_config(cfg, workload, ws),
            "cpu_baseline": {"value": v, "unit": "cell-steps/s", "cores": threads, "kind": "port", "sample": sample,
                             "steps_timed": steps},
            "e2e": {"value": v, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def device_run(P, torch, cfg: dict, workload: str, args, ws: int, local: int, stream):
    """Warm-up, per-kernel probe, then K device-timed steps of one case.  Returns
    the solver (left at its seeded snapshot) and the measurements."""
    n1, n2, n3 = cfg["n1m"], cfg["n2m"], cfg["n3m"]
    cells = n1 * n2 * n3
    esize = 4 if cfg.get("precision", 0) else 8
    s = P.Solver(**cfg)
    s.set_stream(stream.cuda_stream)
    tuned = None
    if not args.no_autotune:
        # launch shapes from the committed cache (tuned on B200); a shape not in
        # it is tuned here, before the warm-up and outside every timed region
        knobs, hit = s.autotune(trial_steps=3, cache_path=TUNE_CACHE)
        tuned = {"knobs": knobs, "from_cache": hit}
    reset = RESET_EVERY.get(workload, 0)
    s.snapshot()

    def run_steps(k: int) -> int:
        """k time steps; with a reset period, restart from the snapshot before
        the state would reach the step at which the case blows up."""
        done = 0
        while done < k:
            chunk = k - done if not reset else min(k - done, reset - s.scalars_step_mod(reset))
            done += s.step(chunk)
            if reset and s.scalars_step_mod(reset) == 0:
                s.restore()
        return done

    # warm-up; the last warm-up step probes every kernel to find the dominant one
    run_steps(max(0, args.warmup - 1))
    names = P.kernel_names()
    s.probe(names)
    run_steps(1)
    per = {k: s.probe_read(k) for k in names}
    s.probe_reset()
    top = max((k for k in per if per[k][1] > 0 and k in KERNEL_ARRAYS), key=lambda k: per[k][0])
    s.probe([top])
    if reset:
        s.restore()
    torch.cuda.synchronize()

    # timed region: K steps, device events on the launching stream
    launches0 = P.launch_count()
    with ClockSampler(local) as clk:
        clk.wait_first()
        dist_barrier(ws)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        done = run_steps(args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
        dist_barrier(ws)
        time.sleep(0.15)          # one more sample after the region
    launches = P.launch_count() - launches0
    ms = dist_max(e0.elapsed_time(e1), ws)
    assert done == args.steps
    tk, nk = s.probe_read(top)
    s.probe([])
    peak, peak_kind = measured_peaks()
    kb = kernel_bytes(top, n1, n2, n3, esize)
    achieved = kb / (tk / nk * 1e-3) / 1e9 if nk else None
    roof = {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak if achieved else None, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
            "algorithmic_bytes_per_launch": kb, "launches": nk, "avg_launch_ms": tk / nk if nk else None,
            "traffic": profiled_traffic(top, workload)}
    fpc = profiled_fp64_flop_per_cell(top) if esize == 8 else None
    if fpc and nk:
        # the line kernels' stencil builds and eliminations are FP64 arithmetic above the
        # FP64 ridge point: their second roof is the FP64 pipe, measured live on this GPU
        peak64 = P.measure_fp64_peak(local)
        kcells = n1 * (n2 - 1) * n3 if top.startswith("dv_") else cells
        ach64 = fpc * kcells / (tk / nk * 1e-3) / 1e12
        roof["fp64_pipe"] = {"achieved_tflops": ach64, "peak_tflops": peak64, "frac": ach64 / peak64,
                             "flop_per_cell": fpc,
                             "flop_source": "ncu FP64 instruction counts, DFMA = 2 (profiles/fp64_flops.json)",
                             "peak_source": "measured (tcs_measure_fp64_peak: FP64 FMA chains on every SM)"}
    step_bytes = step_bytes_per_cell(esize) * cells
    whole = {"algorithmic_bytes_per_step": step_bytes, "bytes_per_cell_step": step_bytes_per_cell(esize),
             "achieved_gbs": step_bytes / (ms / args.steps * 1e-3) / 1e9}
    whole["frac_of_peak"] = whole["achieved_gbs"] / peak
    kernel_split = {k: round(v[0], 4) for k, v in sorted(per.items(), key=lambda kv: -kv[1][0]) if v[1]}
    # the same split under the reference's stage timers (main.f90:55-72)
    tmap = P.timer_of_kernel()
    stages = {t: 0.0 for t in P.timer_names()}
    for k, v in per.items():
        if v[1] and tmap.get(k):
            stages[tmap[k]] += v[0]
    stage_split = {t: round(v, 4) for t, v in stages.items()}
    if reset:
        s.restore()
    return s, {"value": ws * cells * args.steps / (ms * 1e-3), "ms_per_step": ms / args.steps, "tuning": tuned,
               "launches": launches, "roofline": roof, "whole_step": whole,
               "kernel_ms_one_step": kernel_split, "stage_ms_one_step": stage_split, "clocks": clk.summary(),
               "reset": reset}


def tdma_api_timing(P, torch, n_sys: int = 256 * 256, n_row: int = 256, reps: int = 5) -> dict:
    """The reference-facing PaScaL_TDMA interface as the reference calls it:
    a plan created, one many-systems solve and the plan destroyed per sweep
    (module_solve_thermal.f90:364-366), on a z sweep's worth of cyclic systems
    (256^2 systems of 256 rows), from host arrays (4 arrays up, 3 down per
    solve) and from device arrays.  Seconds per sweep, best of reps after one
    untimed sweep."""
    rng = np.random.default_rng(5)
    A = rng.uniform(-0.3, 0.3, (n_row, n_sys)); C = rng.uniform(-0.3, 0.3, (n_row, n_sys))
    B = 1.0 + rng.uniform(0.0, 1.0, (n_row, n_sys)); D = rng.uniform(-1.0, 1.0, (n_row, n_sys))
    out = {"systems": n_sys, "rows": n_row, "cyclic": True}

    def sweep(arrs):
        plan = P.TdmaPlan(n_sys)
        plan.many_solve_cycle(*arrs, n_sys, n_row)
        plan.destroy()

    host = [x.copy() for x in (A, B, C, D)]
    best = None
    for r in range(reps + 1):
        for h, x in zip(host, (A, B, C, D)):
            h[...] = x
        t0 = time.perf_counter(); sweep(host); el = time.perf_counter() - t0
        best = el if r and (best is None or el < best) else best
    out["host_arrays_s_per_sweep"] = best
    out["host_arrays_rows_per_s"] = n_sys * n_row / best
    out["host_bytes_per_sweep"] = 7 * 8 * n_sys * n_row
    dev = [torch.tensor(x, device="cuda") for x in (A, B, C, D)]
    src = [d.clone() for d in dev]
    best = None
    for r in range(reps + 1):
        for d, x in zip(dev, src):
            d.copy_(x)
        torch.cuda.synchronize()
        t0 = time.perf_counter(); sweep(dev); el = time.perf_counter() - t0
        best = el if r and (best is None or el < best) else best
    out["device_arrays_s_per_sweep"] = best
    out["device_arrays_rows_per_s"] = n_sys * n_row / best
    return out


def rel_l2(a, b) -> float:
    nb = float(np.linalg.norm(b))
    d = float(np.linalg.norm(a - b))
    return d / nb if nb > 0 else d


def mixed_error(s64, s32, nsteps: int) -> dict:
    """Both forms from the same seeded state for nsteps: relative L2 of the
    interior fields, of the velocity vector and of the Nusselt / kinetic-energy
    series."""
    s64.restore(); s32.restore()
    s64.step(nsteps); s32.step(nsteps)
    out, du2, u2 = {}, 0.0, 0.0
    for f in ("U", "V", "W", "T", "P"):
        a, b = s32.get(f)[1:-1, 1:-1, 1:-1], s64.get(f)[1:-1, 1:-1, 1:-1]
        out[f] = rel_l2(a, b)
        if f in "UVW":
            du2 += float(np.linalg.norm(a - b)) ** 2
            u2 += float(np.linalg.norm(b)) ** 2
    out["velocity"] = (du2 / u2) ** 0.5 if u2 > 0 else du2 ** 0.5
    h64, h32 = s64.history(0, nsteps), s32.history(0, nsteps)
    for col, n in ((4, "Nu_bot"), (5, "Nu_top"), (6, "KE")):
        out[n] = rel_l2(h32[:, col], h64[:, col])
    out["steps"] = nsteps
    s64.restore(); s32.restore()
    return out


def ensemble_measure(P, torch, args, cfg: dict, workload: str, ws: int, rank: int, local: int) -> dict:
    """The batched ensemble: this rank's share of the cases (LPT by cell count)
    advanced together by one CUDA graph per step, against the same cases
    stepped one at a time.  Returns the fields of the JSON line."""
    allcases = ensemble_cases(cfg["ensemble"], cfg["precision"])
    cases = lpt_shard(allcases, ws, rank)
    solvers = [P.Solver(device=local, **c) for c in cases]
    for s in solvers:
        s.snapshot()
    ens = P.Ensemble(solvers)
    reset = ENSEMBLE_RESET

    def grouped(k: int):
        done = 0
        while done < k:
            n = min(k - done, reset)
            ens.step(n)
            done += n
            if n == reset:
                for s in solvers:
                    s.restore()

    def one_at_a_time(k: int):
        for s in solvers:
            done = 0
            while done < k:
                n = min(k - done, reset)
                s.step(n)
                done += n
                if n == reset:
                    s.restore()

    def timed(fn, k: int) -> float:
        dist_barrier(ws)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn(k)
        torch.cuda.synchronize()
        e1.record()
        torch.cuda.synchronize()
        dist_barrier(ws)
        return dist_max(e0.elapsed_time(e1), ws)

    one_at_a_time(args.warmup)
    for s in solvers:
        s.restore()
    # the auto form selection's 8 measuring steps (real steps) are part of the warm-up
    while ens.form()[0] < 0:
        ens.step(1)
    ens_form, tune_br, tune_bat = ens.form()
    for s in solvers:
        s.restore()
    grouped(args.warmup)
    for s in solvers:
        s.restore()
    launches0 = P.launch_count()
    with ClockSampler(local) as clk:
        clk.wait_first()
        ms = timed(grouped, args.steps)
        time.sleep(0.15)
    launches = P.launch_count() - launches0
    # the same ensemble in the other form
    ens.set_batched(not ens_form)
    for s in solvers:
        s.restore()
    grouped(args.warmup)
    for s in solvers:
        s.restore()
    ms_other = timed(grouped, args.steps)
    ens.set_batched(None)
    ms_bat, ms_br = (ms, ms_other) if ens_form == 1 else (ms_other, ms)
    for s in solvers:
        s.restore()
    ms_seq = timed(one_at_a_time, args.steps)
    total_cells = sum(c["n1m"] * c["n2m"] * c["n3m"] for c in allcases)
    value = total_cells * args.steps / (ms * 1e-3)
    seq = total_cells * args.steps / (ms_seq * 1e-3)
    br = total_cells * args.steps / (ms_br * 1e-3)
    bat = total_cells * args.steps / (ms_bat * 1e-3)
    esize = 4 if cfg["precision"] else 8
    peak, peak_kind = measured_peaks()
    step_bytes = step_bytes_per_cell(esize) * total_cells
    achieved = step_bytes * args.steps / (ms * 1e-3) / 1e9
    del ens
    for s in solvers:
        s.close()
    return {"metric": ensemble_metric(cfg), "value": value,
            "unit": "cell-steps/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong" if ws > 1 else "weak",
            "vs_baseline": None, "dtype": "f32+f64" if cfg["precision"] else "f64",
            "data": "synthetic: seeded conduction profiles + uniform noise 0.01, zero velocity",
            "config": ensemble_config(cfg, workload, ws),
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "kernel": "whole ensemble step", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                         "algorithmic_bytes_per_step": step_bytes, "traffic": None},
            "form": {"chosen": "batched" if ens_form == 1 else "one branch per case",
                     "measured_ms_per_step": {"one_branch_per_case": tune_br, "batched": tune_bat}},
            "batched": {"value": bat, "ms_per_step": ms_bat / args.steps},
            "one_branch_per_case": {"value": br, "ms_per_step": ms_br / args.steps},
            "one_at_a_time": {"value": seq, "ms_per_step": ms_seq / args.steps},
            "speedup_vs_one_at_a_time": value / seq,
            "clocks": clk.summary()}


def run_ensemble(args, cfg: dict, workload: str) -> int:
    """The ensemble workloads (ens48_*) as the line's own workload."""
    ws, rank, local = dist_setup(args.gpus)
    import torch
    import pascal_tcs_b200 as P

    torch.cuda.set_device(local)
    line = ensemble_measure(P, torch, args, cfg, workload, ws, rank, local)
    if rank == 0:
        line.update({"e2e": None, "cpu_baseline": None})
        print(json.dumps(line))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="rb512_water_fp64", choices=sorted(WORKLOADS))
    ap.add_argument("--no-extra", action="store_true", help="skip the 256^3 cases the default workload adds")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the FP32-mixed counterpart of an FP64 workload")
    ap.add_argument("--no-autotune", action="store_true", help="run with the default launch shapes")
    args = ap.parse_args()
    workload = args.workload
    cfg = dict(WORKLOADS[workload])
    if args.impl == "reference":
        return run_reference(args, cfg, workload)
    if "ensemble" in cfg:
        return run_ensemble(args, cfg, workload)

    ws, rank, local = dist_setup(args.gpus)
    import torch
    import pascal_tcs_b200 as P

    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    cfg["device"] = local
    n1, n2, n3 = cfg["n1m"], cfg["n2m"], cfg["n3m"]
    cells = n1 * n2 * n3
    fp32 = bool(cfg.get("precision", 0))
    s, m = device_run(P, torch, cfg, workload, args, ws, local, stream)
    reset = m["reset"]

    # end to end through the C ABI with host buffers: fields uploaded from pinned
    # host memory, K steps driven one reference routine at a time (each step
    # returns maxDivU, CFL and dt to the host), fields downloaded back.
    e2e = None
    if not args.no_e2e:
        host = {f: torch.empty(s.shape, dtype=torch.float64, pin_memory=True) for f in ("T", "U", "V", "W", "P")}
        if reset:
            s.restore()
        for f, t in host.items():
            t.numpy()[...] = s.get(f)
        dist_barrier(ws)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for f, t in host.items():
            s.upload_async(f, t.data_ptr())
        for n in range(args.steps):
            if reset and n and n % reset == 0:
                s.restore()
            s.driver_step()
        for f, t in host.items():
            s.download_async(f, t.data_ptr())
        s.synchronize()
        el = dist_max(time.perf_counter() - t0, ws)
        nbytes = 8 * int(np.prod(s.shape))
        e2e = {"value": ws * cells * args.steps / el, "unit": "cell-steps/s",
               "h2d_bytes_per_step": 5 * nbytes / args.steps,
               "d2h_bytes_per_step": 5 * nbytes / args.steps + 2 * 11 * 8,
               "what": "upload T,U,V,W,P (FP64) from pinned host memory, K steps through the per-routine C-ABI "
                       "entry points (maxDivU, CFL, dt read back every step), download T,U,V,W,P (FP64)"}

    # the FP32-mixed counterpart of an FP64 workload, with its error against FP64
    mixed = None
    twin = workload.replace("_fp64", "_mixed")
    if not fp32 and twin in WORKLOADS and not args.no_mixed:
        cfg32 = dict(WORKLOADS[twin], device=local)
        s32, m32 = device_run(P, torch, cfg32, twin, args, ws, local, stream)
        nerr = reset if reset else 200
        err = mixed_error(s, s32, nerr)
        mixed = {"workload": twin, "value": m32["value"], "unit": "cell-steps/s", "ms_per_step": m32["ms_per_step"],
                 "speedup_vs_fp64": m32["value"] / m["value"], "error_vs_fp64": err,
                 "roofline": m32["roofline"], "whole_step": m32["whole_step"], "gpu_launches": m32["launches"],
                 "kernel_ms_one_step": m32["kernel_ms_one_step"], "tuning": m32["tuning"], "clocks": m32["clocks"]}
        del s32

    # the 256^3 water case in both forms, as an extra key of the default run
    extra = None
    if workload == "rb512_water_fp64" and not args.no_extra:
        del s
        extra = {}
        keep = {}
        for w in ("rb256_water_fp64", "rb256_water_mixed"):
            cw = dict(WORKLOADS[w], device=local)
            sw, mw = device_run(P, torch, cw, w, args, ws, local, stream)
            keep[w] = sw
            extra[w] = {"value": mw["value"], "unit": "cell-steps/s", "ms_per_step": mw["ms_per_step"],
                        "roofline": mw["roofline"], "whole_step": mw["whole_step"], "gpu_launches": mw["launches"],
                        "kernel_ms_one_step": mw["kernel_ms_one_step"], "tuning": mw["tuning"], "clocks": mw["clocks"]}
        extra["rb256_water_mixed"]["speedup_vs_fp64"] = extra["rb256_water_mixed"]["value"] / extra["rb256_water_fp64"]["value"]
        extra["rb256_water_mixed"]["error_vs_fp64"] = mixed_error(keep["rb256_water_fp64"], keep["rb256_water_mixed"],
                                                                  RESET_EVERY["rb256_water_fp64"])
        del keep

    tdma = tdma_api_timing(P, torch) if (workload == "rb512_water_fp64" and not args.no_extra) else None
    # the 48-case ensemble (FP64), as an extra key of the default run on one GPU
    if extra is not None and ws == 1:
        extra["ens48_fp64"] = ensemble_measure(P, torch, args, dict(WORKLOADS["ens48_fp64"]), "ens48_fp64", ws, rank,
                                               local)

    base = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        base = cpu_baseline(cfg)
        base.pop("seconds", None)

    if rank == 0:
        line = {"metric": single_metric(cfg), "value": m["value"],
                "unit": "cell-steps/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": m["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32+f64" if fp32 else "f64",
                "data": "synthetic: seeded conduction profile + uniform noise 0.01, zero velocity",
                "config": single_config(cfg, workload, ws),
                "gpu_launches": m["launches"], "roofline": m["roofline"], "whole_step": m["whole_step"],
                "kernel_ms_one_step": m["kernel_ms_one_step"], "stage_ms_one_step": m["stage_ms_one_step"],
                "tuning": m["tuning"], "clocks": m["clocks"], "e2e": e2e,
                "fp32_mixed": mixed, "cpu_baseline": base}
        if extra is not None:
            line["also"] = extra
        if tdma is not None:
            line["tdma_api"] = tdma
        print(json.dumps(line))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())

"""Benchmark: 2-D largest-Lyapunov-exponent maps, grid points per second.

Default workload (chen-surrogate-8192; one step = one full map): the LLE and
peak-count regime class of the Chen system x'=a(y-x), y'=(c-a)x-xz+cy, z'=xy-bz
on an 8192x8192 (a, c) grid over a in [30,45], c in [20,30], b=3, h=0.002,
Benettin two-trajectory LLE (offset 1e-8, renormalised every NT=0.5 over
tMax=1000 after a 500-unit transient; seed chunk 200000), regime class from the
first 50 time units after the transient (DBSCAN eps 0.02 on (peak, interval),
range below 1e-6 -> 0, LLE above 0.05 -> 15), produced surrogate-refined
(cbf_lle_map_surrogate: plain labels on a 512x512 sub-grid + 65536 random
points, BF16 tensor-core MLP trained on the GPU, plain FP64 recompute of
boundary, low-confidence, 1 % audit and expansion points).  The plain FP64 map
of the same grid is computed once per run: its throughput is reported beside the
surrogate's, and the regime agreement and LLE error of the refined map are
measured against it point by point.

chen-lle2d-2048: the plain LLE map alone on 2048x2048 (the FP64 roofline case).
Inputs are synthetic by nature: the grid itself.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    python bench.py --workload chen-lle2d-2048|lorenz-dbscan-1024|lorenz-kde256-1024|lorenz-kde-1024|
                               lorenz-ls2d-1024|rossler-bif1d-1000|batch64

Multi-GPU (torchrun, one rank per GPU): every rank computes its own 2048x2048 map
of one c-stripe (weak scaling, no data-path collective); time = max over ranks.
The JSON line reports:
  value    device-resident throughput (points/s, all ranks), CUDA events on the
           launching stream around each map, L2 flushed between maps;
  e2e      the same through the public host API (cbf_lle2d: host output buffer,
           device allocation, launch, D2H copy inside the timed region);
  roofline achieved FP64 flops of the LLE kernel vs the FP64 peak (the larger of
           the nominal 64 lanes/SM x 2 x clock and the library's FMA probe), plus
           the FP64-pipe instruction utilisation;
  cpu_baseline the CPU oracle (restatement of the reference per-point code) on a
           strided sample, all host threads.
"""
from __future__ import annotations

import argparse
import ctypes as C
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG_DIR = ROOT / "cudabifurcation3.0_b200"

WORKLOAD = dict(system="chen", nPts=2048, ranges=[30.0, 45.0, 20.0, 30.0], idxMut=[1, 3],
                ic=[0.1, 0.1, 0.1], values=[0.5, 35.0, 3.0, 28.0], h=0.002, NT=0.5, tMax=1000.0,
                transientTime=500.0, lleEps=1e-8, maxValue=1e4, seedChunk=200000)
METRIC = "grid points/s, 2D LLE map (plain FP64)"
SUR_METRIC = "grid points/s, 2D LLE map: plain FP64 vs surrogate-refined at \u226599.5% agreement"
SUR_WORKLOAD = dict(WORKLOAD, nPts=8192, seedChunk=200000, maxAmountOfPeaks=512, dbscanEps=0.02,
                    regimeTime=50.0, regimeMinAmp=1e-6, regimeChaosLle=0.05, flags=1)
# FP64 work of one CD step of each system (csrc/systems.cuh; FMA = 2 flops)
FLOPS_PER_STEP = {"chen": 19, "lorenz": 19, "rossler": 17, "memristive5": 66}
FP64_INSTR_PER_STEP = {"chen": 14, "lorenz": 14, "rossler": 10, "memristive5": 52}
# the rescaled Chen/Lorenz step (systems.cuh QuadScaled): (flops, FP64 instructions)
# per step for s = 1/2 (6 FMA + 2 MUL) and for other s (one more MUL), keyed by
# cbf_job_scaled_step
SCALED_COST = {2: (14, 8, "rescaled 8-instruction CD step (s = 1/2)"), 1: (15, 9, "rescaled 9-instruction CD step")}
FP64_LANES_PER_SM = 64
# the same Chen CD step written unfused, as the formula reads (each add, sub, mul
# and div of the explicit half z, y, x and the implicit half x, y, z counted once,
# parameter-only factors hoisted): 5 + 7 + 3 + 3 + 6 + 4 = 28
UNFUSED_CD_FLOPS_PER_STEP = {"chen": 28}

# The other measured configurations (printed as their own JSON lines with
# --workload NAME; the default run is the LLE map above).
_LORENZ = dict(system="lorenz", nPts=1024, ranges=[5.0, 20.0, 20.0, 200.0], idxMut=[1, 2],
               ic=[0.1, 0.1, 0.1], values=[0.5, 10.0, 28.0, 8.0 / 3.0], h=0.005, tMax=200.0,
               transientTime=500.0, maxValue=1e4, writableVar=0, preScaller=1,
               maxAmountOfPeaks=10000)
SECONDARY = {
    # 2-D DBSCAN cluster-count map, Lorenz (sigma, rho) 1024^2, eps 1e-3
    "lorenz-dbscan-1024": dict(_LORENZ, task=2, dbscanEps=1e-3),
    # 2-D KDE mode-count map with 256 samples per point (fixed-sample mode)
    "lorenz-kde256-1024": dict(_LORENZ, task=1, kdeSampling=256, flags=2, kdeI1=-60.0,
                               kdeI2=60.0, kdeH=1.0),
    # the same with the reference's per-peak sampling (k1 = 4 * peaks)
    "lorenz-kde-1024": dict(_LORENZ, task=1, kdeSampling=4, kdeI1=-60.0, kdeI2=60.0, kdeH=0.5),
    # 2-D Lyapunov-spectrum map (LS2D), Lorenz (sigma, rho) 1024^2, 3 exponents per point
    "lorenz-ls2d-1024": dict(system="lorenz", nPts=1024, ranges=[5.0, 20.0, 20.0, 200.0], idxMut=[1, 2],
                             ic=[0.1, 0.1, 0.1], values=[0.5, 10.0, 28.0, 8.0 / 3.0], h=0.005, NT=0.5,
                             tMax=1000.0, transientTime=50.0, lleEps=1e-8, maxValue=1e4, task=6),
    # 1-D bifurcation diagram, Rossler a in [0.05, 0.40], 1000 points
    "rossler-bif1d-1000": dict(system="rossler", nPts=1000, ranges=[0.05, 0.40], idxMut=[1],
                               ic=[0.1, 0.1, 0.1], values=[0.5, 0.2, 0.2, 5.7], h=0.01,
                               tMax=500.0, transientTime=1000.0, maxValue=1e4, writableVar=0,
                               preScaller=1, task=0),
}


BATCH_SEED = 20240101
_BATCH_SYSTEMS = {
    "rossler": dict(values=[0.5, 0.2, 0.2, 5.7], idxMut=[1, 2], ranges=[0.05, 0.35, 0.05, 0.35]),
    "lorenz": dict(values=[0.5, 10.0, 28.0, 8.0 / 3.0], idxMut=[1, 2], ranges=[5.0, 20.0, 20.0, 200.0]),
    "chen": dict(values=[0.5, 35.0, 3.0, 28.0], idxMut=[1, 3], ranges=[30.0, 45.0, 20.0, 30.0]),
}


def batch_specs(seed: int = BATCH_SEED, n: int = 64):
    """The ragged-batch configuration: n jobs drawn from `seed` -- system in
    {Rossler, Lorenz, Chen}, task in {2-D KDE, 2-D DBSCAN, 2-D LLE}, grid side
    U{64..1024}, record U[200, 5000] time units, h U[0.001, 0.01], transient 100."""
    rng = np.random.default_rng(seed)
    specs = []
    for _ in range(n):
        system = ["rossler", "lorenz", "chen"][rng.integers(0, 3)]
        task = ["kde", "dbscan", "lle"][rng.integers(0, 3)]
        side = int(rng.integers(64, 1025))
        record = float(rng.uniform(200.0, 5000.0))
        h = float(rng.uniform(0.001, 0.01))
        spec = dict(system=system, nPts=side, ic=[0.1, 0.1, 0.1], h=h, tMax=record,
                    transientTime=100.0, maxValue=1e4, **_BATCH_SYSTEMS[system])
        if task == "lle":
            spec.update(task=3, NT=0.5, lleEps=1e-8)
        elif task == "kde":
            spec.update(task=1, maxAmountOfPeaks=1000, kdeSampling=4, kdeI1=-60.0, kdeI2=60.0,
                        kdeH=0.5)
        else:
            spec.update(task=2, maxAmountOfPeaks=1000, dbscanEps=0.05)
        specs.append(spec)
    return specs


def run_batch(args) -> int:
    """Ragged batch: the seeded 64 jobs in one persistent launch (CUDA graph) vs one by one."""
    import torch
    torch.cuda.set_device(0)
    cbf = load_cbf()
    specs = batch_specs()
    jobs, outs = [], []
    for sp in specs:
        sp = dict(sp)
        task = sp.pop("task")
        jobs.append(cbf.make_job(task=task, **sp))
        n = sp["nPts"] ** 2
        outs.append(torch.empty(n, dtype=torch.float64 if task == cbf.TASK_LLE else torch.int32,
                                device="cuda"))
    batch = cbf.Batch(jobs, [o.data_ptr() for o in outs])
    stream = torch.cuda.Stream()
    s = stream.cuda_stream
    bps, tune_ms = batch.autotune(s)
    batch.capture(s)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    for _ in range(args.warmup):
        batch.launch(s)
    stream.synchronize()
    sampler = ClockSampler(0)
    sampler.start()
    launches0 = cbf.kernel_launches()
    ms = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        batch.launch(s)
        with torch.cuda.stream(stream):
            e1.record(stream)
        stream.synchronize()
        ms.append(e0.elapsed_time(e1))
    launches = cbf.kernel_launches() - launches0
    clocks = sampler.stop()
    batch.check()
    got = [o.cpu().numpy().copy() for o in outs]
    # the same jobs one by one (per-job kernels), timed the same way
    with torch.cuda.stream(stream):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
    batch.run_sequential(s)
    with torch.cuda.stream(stream):
        e1.record(stream)
    stream.synchronize()
    seq_ms = e0.elapsed_time(e1)
    same = all(np.array_equal(a, o.cpu().numpy(), equal_nan=True) for a, o in zip(got, outs))
    t = statistics.mean(ms)
    pts = batch.points()
    line = {"metric": "grid points/s, ragged batch of 64 jobs in one persistent launch",
            "value": pts / (t / 1e3), "unit": "points/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded job mix)",
            "config": {"workload": "batch64", "seed": BATCH_SEED, "jobs": len(specs),
                       "points": pts,
                       "tasks": {k: sum(1 for sp in specs if sp["task"] == v)
                                 for k, v in (("lle", 3), ("kde", 1), ("dbscan", 2))},
                       "cache": "L2 flushed before every timed run",
                       "blocks_per_sm": bps, "autotune_trial_ms": [round(float(x), 3) for x in tune_ms],
                       "launch": "one CUDA graph (queue reset + persistent kernel)"},
            "one_by_one": {"value": pts / (seq_ms / 1e3), "ms": seq_ms,
                           "speedup_batch_over_one_by_one": seq_ms / t,
                           "results_identical": bool(same)},
            "gpu_launches": int(launches), "clocks": clocks, "kernel_ms": ms}
    print(json.dumps(line), flush=True)
    batch.close()
    return 0 if same else 1


def load_cbf():
    spec = importlib.util.spec_from_file_location("cbf_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["cbf_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def steps_per_point(w) -> int:
    skip = int(w["transientTime"] / w["h"])
    blocks = int(w["tMax"] / w["NT"])
    nt = int(w["NT"] / w["h"])
    return skip + 2 * blocks * nt


def stripe(w: dict, rank: int, world: int) -> dict:
    """Weak scaling: rank r maps the r-th of `world` equal c-stripes (axis 1) at the
    full resolution; the stripes tile the c range with no overlap or gap."""
    w = dict(w)
    if world > 1:
        lo, hi = w["ranges"][2], w["ranges"][3]
        step = (hi - lo) / world
        top = hi if rank == world - 1 else lo + (rank + 1) * step
        w["ranges"] = [w["ranges"][0], w["ranges"][1], lo + rank * step, top]
    return w


def rank_workload(rank: int, world: int) -> dict:
    return stripe(WORKLOAD, rank, world)


def max_over_ranks(values, dist=None, device=None):
    """Element-wise maximum of per-rank timings (all ranks take part)."""
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


class ClockSampler:
    """nvidia-smi samples (clocks, throttle reasons) during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self._t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except (FileNotFoundError, OSError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self._t:
            self._t.join(timeout=2)
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "power_w_median": statistics.median(power), "samples": len(sm),
                "reasons": sorted(reasons)}


def step_cost(cbf, job, system: str):
    """(flops, FP64 instructions, form) of one CD step of the job: the rescaled
    Chen/Lorenz form (6 FMA + 2 MUL at s = 1/2, one more MUL otherwise) where the
    job's grid admits it (cbf_job_scaled_step), the 14-instruction forms
    otherwise."""
    L = cbf.lib()
    L.cbf_job_scaled_step.restype = C.c_int32
    L.cbf_job_scaled_step.argtypes = [C.c_void_p]
    form = L.cbf_job_scaled_step(C.addressof(job))
    if form in SCALED_COST:
        return SCALED_COST[form]
    return FLOPS_PER_STEP[system], FP64_INSTR_PER_STEP[system], "reference-order CD step"


def fp64_roofline(torch, device: int, cost, n_points: int, spp: int, mean_ms: float,
                  clocks: dict, probe_tflops: float, system: str = "chen") -> dict:
    """FP64 roofline of one map: algorithmic flops and FP64-pipe instructions;
    cost = step_cost(...)."""
    flops_step, instr_step, form = cost
    props = torch.cuda.get_device_properties(device)
    max_mhz = clocks.get("sm_max_mhz") or 1965.0
    nominal = props.multi_processor_count * FP64_LANES_PER_SM * 2 * max_mhz * 1e6 / 1e12
    peak = max(nominal, probe_tflops)
    flops = float(n_points) * spp * flops_step
    achieved = flops / (mean_ms / 1e3) / 1e12
    sm_mhz = clocks.get("sm_mhz") or max_mhz
    instr = float(n_points) * spp * instr_step
    pipe = instr / (mean_ms / 1e3) / (props.multi_processor_count * FP64_LANES_PER_SM * sm_mhz * 1e6)
    return {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak,
            "peak_source": "max(nominal SMs x 64 FP64 lanes x 2 flops x max SM clock, FP64 FMA "
                           "probe measured in this run); MEASURED_PEAKS.json has no FP64 figure",
            "peak_nominal": nominal, "peak_probe": probe_tflops, "flops_per_launch": flops,
            "flops_per_step": flops_step, "fp64_instr_per_step": instr_step, "step_form": form,
            "fp64_pipe_frac": pipe, **unfused_cd(system, n_points, spp, mean_ms, peak)}


def unfused_cd(system: str, n_points: int, spp: int, mean_ms: float, peak: float) -> dict:
    """The same map's rate counted with the unfused formula of the CD step (the
    work of the method as written, whatever form computes it)."""
    f = UNFUSED_CD_FLOPS_PER_STEP.get(system)
    if not f:
        return {}
    achieved = float(n_points) * spp * f / (mean_ms / 1e3) / 1e12
    return {"unfused_cd_flops_per_step": f, "unfused_cd_achieved": achieved, "unfused_cd_frac": achieved / peak}


def cpu_baseline(w: dict, target_s: float = 15.0) -> dict:
    """Oracle port of the reference per-point code on a strided sample, all threads."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    threads = O.host_threads()
    job = O.make_job(**w)
    n_total = w["nPts"] ** 2
    probe = np.arange(threads, dtype=np.int64) * (n_total // max(threads, 1))
    t0 = time.perf_counter()
    O.map_lle_list(job, probe, threads)
    per_round = max(time.perf_counter() - t0, 1e-3)
    count = max(1, int(target_s / per_round)) * threads
    idx = grid_sample(n_total, count)
    t0 = time.perf_counter()
    O.map_lle_list(job, idx, threads)
    dt = time.perf_counter() - t0
    return {"value": count / dt, "unit": "points/s", "cores": threads, "kind": "port",
            "sample": f"{count} of {n_total} points spread over the whole grid (golden-ratio sequence), "
                      f"{steps_per_point(w)} steps each"}


def traffic_from_profiles():
    """Per-launch DRAM bytes of the LLE kernel from the committed ncu summary, if any."""
    p = ROOT / "profiles" / "lle_chen_2048_traffic.json"
    try:
        return json.loads(p.read_text()).get("dram_bytes_per_full_launch")
    except (OSError, ValueError):
        return None


def _orc_kw(w):
    """The oracle job of a workload: the same fields, the grid flag included."""
    return dict(w)


def grid_sample(n_total: int, count: int, offset: float = 0.0) -> np.ndarray:
    """`count` grid indices spread over the whole grid (a golden-ratio sequence:
    every row and column range is sampled evenly, whatever the grid side); a
    different `offset` in [0, 1) gives another sample of the same kind."""
    k = np.arange(count, dtype=np.float64)
    frac = np.mod(k * 0.6180339887498949 + offset, 1.0)
    return np.minimum((frac * n_total).astype(np.int64), n_total - 1)


def regime_traffic(points):
    """DRAM bytes of the plain regime kernel for `points` points, scaled from the
    committed ncu capture (traffic grows with the points computed)."""
    p = ROOT / "profiles" / "lle_regime_chen_512_traffic.json"
    try:
        return float(json.loads(p.read_text())["dram_bytes_per_point"]) * points
    except (OSError, ValueError, KeyError):
        return None


def run_reference(args) -> int:
    """The reference's per-point code (oracle port) on the host cores: the plain
    LLE (+ regime class for the default workload) of strided grid points."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sur = args.workload == "chen-surrogate-8192"
    w = SUR_WORKLOAD if sur else WORKLOAD
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    if not O.LIB_PATH.exists():
        O.build(with_ref=False)
    threads = O.host_threads()
    job = O.make_job(**_orc_kw(w))
    n_total = w["nPts"] ** 2
    if sur:
        def compute(idx):
            O.map_lle_regime(job, idx, threads=threads)
    else:
        def compute(idx):
            O.map_lle_list(job, idx, threads)
    # Calibrate on one point per thread, then size every step to ~target seconds.
    target = float(os.environ.get("CBF_REF_STEP_SECONDS", "5"))
    cal = (np.arange(threads, dtype=np.int64) * 7919) % n_total
    t0 = time.perf_counter()
    compute(cal)
    t_cal = max(time.perf_counter() - t0, 1e-3)
    per_step = threads * max(1, int(target / t_cal))
    times = []
    for s in range(args.warmup + args.steps):
        # every step (warm-up and timed) samples the whole grid, each another sample
        idx = grid_sample(n_total, per_step, (s + 0.5) / (args.warmup + args.steps))
        t0 = time.perf_counter()
        compute(idx)
        dt = time.perf_counter() - t0
        if s >= args.warmup:
            times.append(dt)
    tot = sum(times)
    value = per_step * args.steps / tot
    line = {
        "impl": "reference", "metric": SUR_METRIC if sur else METRIC, "value": value, "unit": "points/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "grid": f"{w['nPts']}x{w['nPts']}", "tMax": 1000,
                   "NT": 0.5, "h": 0.002, "transient": 500, "steps_per_point": steps_per_point(w),
                   "method": "plain LLE + regime class per point (the reference has no surrogate)"
                   if sur else "plain LLE per point",
                   "exact_grid": bool(w.get("flags", 0) & 1),
                   "cache": "inputs are scalars; CPU arm"},
        "cpu_baseline": {"value": value, "unit": "points/s", "cores": threads, "kind": "port",
                         "sample": f"{per_step} points per step spread over the whole {n_total}-point grid "
                                   "(golden-ratio sequence, another sample each step)"},
        "e2e": {"value": value, "unit": "points/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_secondary(args, name: str) -> int:
    """One of the other configurations: device-resident points/s, oracle sample."""
    import torch
    torch.cuda.set_device(0)
    cbf = load_cbf()
    w = dict(SECONDARY[name])
    if args.nPts:
        w["nPts"] = args.nPts
    task = w.pop("task")
    job = cbf.make_job(task=task, **w)
    dims = len(w["idxMut"])
    n = w["nPts"] ** dims
    rec = cbf.record_length(job)
    if task == cbf.TASK_LS:  # the base + D perturbed trajectories per interval
        spp = int(w["transientTime"] / w["h"]) + (len(w["ic"]) + 1) * rec * int(w["NT"] / w["h"])
    else:
        spp = int(w["transientTime"] / w["h"]) + rec * w.get("preScaller", 1)
    if task == cbf.TASK_LS:
        out = torch.empty(n * len(w["ic"]), dtype=torch.float64, device="cuda")
        aux_ptr = 0
    elif task == cbf.TASK_PEAKS:
        cap = cbf.lib().cbf_peak_capacity(C.byref(job))
        job.peakCapacity = cap
        out = torch.empty(n * cap, dtype=torch.float64, device="cuda")
        aux = torch.empty(n, dtype=torch.int32, device="cuda")
        aux_ptr = aux.data_ptr()
    else:
        out = torch.empty(n, dtype=torch.int32, device="cuda")
        aux_ptr = 0
    stream = torch.cuda.Stream()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    for _ in range(args.warmup):
        cbf.run_device(job, out.data_ptr(), aux_ptr, stream.cuda_stream)
    stream.synchronize()
    sampler = ClockSampler(0)
    torch.cuda.synchronize()
    sampler.start()
    launches0 = cbf.kernel_launches()
    ms = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        cbf.run_device(job, out.data_ptr(), aux_ptr, stream.cuda_stream)
        with torch.cuda.stream(stream):
            e1.record(stream)
        stream.synchronize()
        ms.append(e0.elapsed_time(e1))
    launches = cbf.kernel_launches() - launches0
    clocks = sampler.stop()
    t = statistics.mean(ms)
    probe = cbf.probe_fp64_peak(300.0)
    roof = fp64_roofline(torch, 0, step_cost(cbf, job, w["system"]), n, spp, t, clocks, probe, w["system"])
    roof["traffic"] = None
    roof["note"] = ("integration flops only (base + perturbed trajectories); Gram-Schmidt and log "
                    "per interval on top") if task == cbf.TASK_LS else \
        "integration flops only; the peak/KDE/DBSCAN work is on top"
    # oracle on a small contiguous sample
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    threads = O.host_threads()
    oj = O.make_job(**{k: v for k, v in w.items() if k != "flags"})
    cnt = min(n, threads * 2)
    t0 = time.perf_counter()
    if task == cbf.TASK_LS:
        O.map_ls(oj, np.arange(n // 2, n // 2 + cnt), threads=threads)
    elif task == cbf.TASK_DBSCAN:
        O.map_dbscan(oj, n // 2, cnt, threads)
    elif task == cbf.TASK_KDE and not (w.get("flags", 0) & 2):
        O.map_kde(oj, n // 2, cnt, threads)
    else:
        O.map_peaks(oj, n // 2, cnt, max(rec // 2, 1), threads)
    cpu_pps = cnt / (time.perf_counter() - t0)
    line = {"metric": f"grid points/s, {name}", "value": n / (t / 1e3), "unit": "points/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (the parameter grid is the input)",
            "config": {"workload": name, "grid": f"{w['nPts']}^{dims}", "steps_per_point": spp,
                       "record": rec, "cache": "L2 flushed before every timed map"},
            "roofline": roof,
            "cpu_baseline": {"value": cpu_pps, "unit": "points/s", "cores": threads,
                             "kind": "port", "sample": f"{cnt} contiguous points"},
            "gpu_launches": int(launches), "clocks": clocks, "kernel_ms": ms}
    print(json.dumps(line), flush=True)
    return 0


def cpu_baseline_regime(w: dict, target_s: float = 15.0) -> dict:
    """Oracle port of the plain LLE + regime per-point code on a strided sample."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    threads = O.host_threads()
    job = O.make_job(**_orc_kw(w))
    n_total = w["nPts"] ** 2
    probe = np.arange(threads, dtype=np.int64) * (n_total // max(threads, 1))
    t0 = time.perf_counter()
    O.map_lle_regime(job, probe, threads=threads)
    per_round = max(time.perf_counter() - t0, 1e-3)
    count = max(1, int(target_s / per_round)) * threads
    idx = grid_sample(n_total, count)
    t0 = time.perf_counter()
    O.map_lle_regime(job, idx, threads=threads)
    dt = time.perf_counter() - t0
    return {"value": count / dt, "unit": "points/s", "cores": threads, "kind": "port",
            "sample": f"{count} of {n_total} points spread over the whole grid (golden-ratio sequence), "
                      f"plain LLE + regime, {steps_per_point(w)} steps each"}


def run_surrogate(args) -> int:
    """Surrogate-refined 8192^2 LLE + regime map against the plain map."""
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900),
                                device_id=torch.device("cuda", local))
    cbf = load_cbf()
    cbf.check(cbf.lib().cbf_set_device(local))
    w = stripe(SUR_WORKLOAD, rank, world)
    if args.nPts:
        w["nPts"] = args.nPts
    n = w["nPts"] ** 2
    job = cbf.make_job(task=cbf.TASK_LLE_REGIME, **w)
    spp = steps_per_point(w)
    cfg = cbf.surrogate_config()
    probe = cbf.probe_fp64_peak(300.0)
    stream = torch.cuda.Stream()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")  # > 126 MB L2

    # plain FP64 map of the same grid, once: throughput and the agreement reference
    p_lle = torch.empty(n, dtype=torch.float64, device="cuda")
    p_cls = torch.empty(n, dtype=torch.int32, device="cuda")
    with torch.cuda.stream(stream):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
    cbf.run_device(job, p_lle.data_ptr(), p_cls.data_ptr(), stream.cuda_stream)
    with torch.cuda.stream(stream):
        e1.record(stream)
    stream.synchronize()
    plain_ms = e0.elapsed_time(e1)
    if args.plain_only:
        if rank == 0:
            print(json.dumps({"workload": "chen-surrogate-8192 (plain map only)",
                              "grid": f"{w['nPts']}x{w['nPts']}", "plain_ms": plain_ms,
                              "plain_points_per_s": n / (plain_ms / 1e3)}), flush=True)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return 0

    s_lle = torch.empty(n, dtype=torch.float64, device="cuda")
    s_cls = torch.empty(n, dtype=torch.int32, device="cuda")
    s_src = torch.empty(n, dtype=torch.uint8, device="cuda")

    def one_map():
        with torch.cuda.stream(stream):
            return cbf.lle_map_surrogate(job, cfg, s_lle.data_ptr(), s_cls.data_ptr(), s_src.data_ptr(),
                                         stream=stream.cuda_stream)

    for _ in range(args.warmup):
        one_map()
    stream.synchronize()

    sampler = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    launches0 = cbf.kernel_launches()
    evs, reps = [], []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        reps.append(one_map())
        with torch.cuda.stream(stream):
            e1.record(stream)
        evs.append((e0, e1))
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches = cbf.kernel_launches() - launches0
    clocks = sampler.stop()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms, plain_max = max_over_ranks([sum(step_ms), plain_ms], dist, "cuda")
    value = world * n * args.steps / (total_ms / 1e3)
    plain_value = world * n / (plain_max / 1e3)

    # agreement and LLE error against the plain map, point by point
    same_cls = (s_cls == p_cls)
    agree = float(same_cls.double().mean().item())
    kept = s_src == 0
    err = (s_lle - p_lle).abs()
    fin = torch.isfinite(err) & kept
    kept_err = err[fin]
    computed = s_src > 0
    exact = bool(torch.equal(s_cls[computed], p_cls[computed]) and
                 torch.equal(torch.nan_to_num(s_lle[computed], nan=7.0, posinf=8.0, neginf=9.0),
                             torch.nan_to_num(p_lle[computed], nan=7.0, posinf=8.0, neginf=9.0)))
    stats = torch.tensor([agree], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(stats, op=dist.ReduceOp.MIN)
    agree_min = float(stats.item())

    # End to end through the reference-facing host entry point: LLE2D's arguments
    # as host arrays, the refined LLE and class maps returned in host arrays
    # (cbf_lle2d_surrogate: inputs, compute and the D2H copies inside the call).
    h_lle = np.zeros(n, np.float64)  # touched once here, so no page faults are timed
    h_cls = np.zeros(n, np.int32)
    rules = cbf.regime_rules(regimeTime=w["regimeTime"], maxAmountOfPeaks=w["maxAmountOfPeaks"],
                             dbscanEps=w["dbscanEps"], regimeMinAmp=w["regimeMinAmp"],
                             regimeChaosLle=w["regimeChaosLle"], flags=w["flags"])
    e2e_in = [np.array(w["ic"], np.float64), np.array(w["ranges"], np.float64),
              np.array(w["idxMut"], np.int32), np.array(w["values"], np.float64)]
    e2e_times = []
    for _ in range(max(1, args.e2e_steps)):
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        cbf.LLE2D_surrogate(w["tMax"], w["NT"], w["nPts"], w["h"], w["lleEps"], e2e_in[0], 3, e2e_in[1],
                            e2e_in[2], 0, w["maxValue"], w["transientTime"], e2e_in[3], 4, system="chen",
                            seedChunk=w["seedChunk"], rules=rules, config=cfg, out_lle=h_lle, out_cls=h_cls)
        e2e_times.append(time.perf_counter() - t0)
    e2e_total = torch.tensor([sum(e2e_times)], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(e2e_total, op=dist.ReduceOp.MAX)
    e2e_value = world * n * len(e2e_times) / float(e2e_total.item())
    e2e_same = bool(np.array_equal(h_cls, s_cls.cpu().numpy()) and
                    np.array_equal(h_lle, s_lle.cpu().numpy(), equal_nan=True))
    e2e_h2d = int(sum(a.nbytes for a in e2e_in) + C.sizeof(rules) + C.sizeof(cfg))

    # What the learning adds: one map with the network replaced by the nearest
    # coarse-grid label (same labels, mask, audit and expansion rules).
    abl_cfg = cbf.surrogate_config(predictor=1)
    with torch.cuda.stream(stream):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
    abl_rep = cbf.lle_map_surrogate(job, abl_cfg, s_lle.data_ptr(), s_cls.data_ptr(), s_src.data_ptr(),
                                    stream=stream.cuda_stream)
    with torch.cuda.stream(stream):
        e1.record(stream)
    stream.synchronize()
    abl_err = (s_lle - p_lle).abs()
    abl_kept = (s_src == 0) & torch.isfinite(abl_err)
    ablation = {"predictor": "nearest coarse-grid label, no network", "ms": e0.elapsed_time(e1),
                "regime_agreement": float((s_cls == p_cls).double().mean().item()),
                "computed_fraction": float((s_src > 0).double().mean().item()),
                "kept_lle_mean_abs_err": float(abl_err[abl_kept].mean().item()) if abl_kept.any() else None,
                "refined": int(abl_rep.refined), "waves": int(abl_rep.waves)}
    # The two predictors alone (refine 0: no recompute), on every point that is
    # not a label: class agreement and LLE error against the plain map.
    raw = {}
    for name, kind in (("network", 0), ("nearest_label", 1)):
        cbf.lle_map_surrogate(job, cbf.surrogate_config(refine=0, predictor=kind), s_lle.data_ptr(),
                              s_cls.data_ptr(), s_src.data_ptr(), stream=stream.cuda_stream)
        stream.synchronize()
        pred = s_src == 0
        lerr = (s_lle - p_lle).abs()
        fin = pred & torch.isfinite(lerr)
        raw[name] = {"class_agreement": float((s_cls[pred] == p_cls[pred]).double().mean().item()),
                     "lle_mean_abs_err": float(lerr[fin].mean().item())}
    ablation["raw_predictions"] = raw

    r = reps[-1].as_dict()
    plain_points = r["labelled"] + r["refined"]
    plain_phase_ms = r["msLabel"] + r["msRefine"]
    props = torch.cuda.get_device_properties(local)
    max_mhz = clocks.get("sm_max_mhz") or 1965.0
    nominal = props.multi_processor_count * FP64_LANES_PER_SM * 2 * max_mhz * 1e6 / 1e12
    peak = max(nominal, probe)
    flops_step, instr_step, form = step_cost(cbf, job, "chen")
    flops = float(plain_points) * spp * flops_step
    achieved = flops / (plain_phase_ms / 1e3) / 1e12
    plain_achieved = float(n) * spp * flops_step / (plain_ms / 1e3) / 1e12
    pipe_den = props.multi_processor_count * FP64_LANES_PER_SM * (clocks.get("sm_mhz") or max_mhz) * 1e6
    roof = {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak,
            "kernel": "lle_regime_kernel (plain FP64 labels + recompute rounds of the refined map)",
            "peak_source": "max(nominal SMs x 64 FP64 lanes x 2 flops x max SM clock, FP64 FMA "
                           "probe measured in this run); MEASURED_PEAKS.json has no FP64 figure",
            "peak_nominal": nominal, "peak_probe": probe,
            "flops_per_step": flops_step, "fp64_instr_per_step": instr_step, "step_form": form,
            "fp64_pipe_frac": float(plain_points) * spp * instr_step / (plain_phase_ms / 1e3) / pipe_den,
            "plain_map_fp64_pipe_frac": float(n) * spp * instr_step / (plain_ms / 1e3) / pipe_den,
            "steps_per_point": spp,
            "plain_points_in_step": plain_points, "plain_phase_ms": plain_phase_ms,
            "plain_map_achieved": plain_achieved, "plain_map_frac": plain_achieved / peak,
            **unfused_cd("chen", plain_points, spp, plain_phase_ms, peak),
            "plain_map_unfused_cd_frac": unfused_cd("chen", n, spp, plain_ms, peak).get("unfused_cd_frac"),
            "traffic": regime_traffic(plain_points)}

    ok = agree_min >= 0.995 and exact and e2e_same
    if rank == 0:
        base = None
        if world == 1 and not args.no_cpu_baseline:
            base = cpu_baseline_regime(w)
        line = {
            "metric": SUR_METRIC, "value": value, "unit": "points/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (the parameter grid is the input)",
            "config": {"workload": "chen-surrogate-8192", "grid": f"{w['nPts']}x{w['nPts']}",
                       "system": "chen", "tMax": w["tMax"], "NT": w["NT"], "h": w["h"],
                       "transient": w["transientTime"], "eps": w["lleEps"], "regimeTime": 50.0,
                       "exact_grid": bool(w["flags"] & 1),
                       "grid_note": "integer grid cells (CBF_FLAG_EXACT_GRID); the reference's LLE2D "
                                    "derives the column from an FP32 index, which moves 33.5 M of "
                                    "the 67 M points of an 8192^2 grid by one or more cells",
                       "steps_per_point": spp, "points_per_rank": n,
                       "surrogate": {k: getattr(cfg, k) for k, _ in cfg._fields_},
                       "cache": "L2 flushed (256 MB write) before every timed map; the outputs "
                                "(805 MB) exceed L2",
                       "parallelism": f"{world} independent c-stripes, one per GPU"},
            "plain": {"value": plain_value, "unit": "points/s", "ms": plain_max,
                      "note": "plain FP64 LLE + regime map of the same grid, CUDA events, once"},
            "speedup_vs_plain": plain_max / (total_ms / args.steps),
            "agreement": {"regime_agreement": agree, "min_over_ranks": agree_min,
                          "computed_fraction": float(computed.double().mean().item()),
                          "plain_points_bit_exact": exact,
                          "kept_lle_mean_abs_err": float(kept_err.mean().item()) if kept_err.numel() else None,
                          "kept_lle_p99_abs_err": float(torch.quantile(kept_err[:1 << 24].float(), 0.99).item())
                          if kept_err.numel() else None},
            "report": r,
            "ablation_no_network": ablation,
            "e2e": {"value": e2e_value, "unit": "points/s", "h2d_bytes_per_step": e2e_h2d,
                    "d2h_bytes_per_step": n * 12, "matches_device_api": e2e_same,
                    "call": "cbf_lle2d_surrogate (LLE2D's arguments, host arrays in and out)"},
            "roofline": roof,
            "cpu_baseline": base,
            "gpu_launches": int(launches),
            "clocks": clocks,
            "step_ms": step_ms,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0 if ok else 1


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--nPts", type=int, default=None, help="override the grid side (testing)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--lle-variant", type=int, default=None,
                    help="chen-lle2d-2048: run this LLE kernel shape instead of autotuning (profiling)")
    ap.add_argument("--plain-only", action="store_true",
                    help="chen-surrogate-8192: compute and time only the plain map (profiling)")
    ap.add_argument("--workload", default="chen-surrogate-8192",
                    choices=["chen-surrogate-8192", "chen-lle2d-2048", "batch64", *SECONDARY])
    args = ap.parse_args(argv)

    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch64":
        return run_batch(args)
    if args.workload == "chen-surrogate-8192":
        return run_surrogate(args)
    if args.workload != "chen-lle2d-2048":
        return run_secondary(args, args.workload)

    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))

    cbf = load_cbf()
    cbf.check(cbf.lib().cbf_set_device(local))
    w = rank_workload(rank, world)
    if args.nPts:
        w["nPts"] = args.nPts
    n = w["nPts"] ** 2
    job = cbf.make_job(task=cbf.TASK_LLE, **w)
    spp = steps_per_point(w)

    probe = cbf.probe_fp64_peak(300.0)  # TFLOP/s, FMA = 2 flops
    # the same step and divergence tracking as a bare instruction stream (two
    # chains per thread, six blocks of 128 per SM): the issue rate the map kernel
    # is compared with
    step_stream = cbf.probe_fp64_step(2, True, 6, 300.0)
    if args.lle_variant is None:
        variant, trial_ms = cbf.autotune(job)  # picks the LLE kernel shape for this device
    else:  # a fixed shape (profiling a chosen kernel): no autotuning launches
        variant, trial_ms = args.lle_variant, []
        cbf.set_lle_variant(w["system"], variant)

    stream = torch.cuda.Stream()
    out = torch.empty(n, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")  # > 126 MB L2

    def one_map():
        with torch.cuda.stream(stream):
            cbf.run_device(job, out.data_ptr(), 0, stream.cuda_stream)

    for _ in range(args.warmup):
        one_map()
    stream.synchronize()

    sampler = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    launches0 = cbf.kernel_launches()
    evs = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        one_map()
        with torch.cuda.stream(stream):
            e1.record(stream)
        evs.append((e0, e1))
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches = cbf.kernel_launches() - launches0
    clocks = sampler.stop()
    kernel_ms = [a.elapsed_time(b) for a, b in evs]
    t = torch.tensor([sum(kernel_ms)], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    value = world * n * args.steps / (total_ms / 1e3)

    # End to end through the public host API: host buffer, D2H inside the region.
    res = np.empty(n, np.float64)
    e2e_times = []
    L = cbf.lib()
    icv = np.array(w["ic"], np.float64)
    rv = np.array(w["ranges"], np.float64)
    iv = np.array(w["idxMut"], np.int32)
    vv = np.array(w["values"], np.float64)
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int32)
    for _ in range(max(1, args.e2e_steps)):
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        cbf.check(L.cbf_lle2d(3, w["tMax"], w["NT"], w["nPts"], w["h"], w["lleEps"],
                              icv.ctypes.data_as(dp), 3, rv.ctypes.data_as(dp),
                              iv.ctypes.data_as(ip), 0, w["maxValue"], w["transientTime"],
                              vv.ctypes.data_as(dp), 4, w["seedChunk"], res.ctypes.data_as(dp)))
        e2e_times.append(time.perf_counter() - t0)
    e2e_total = torch.tensor([sum(e2e_times)], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(e2e_total, op=dist.ReduceOp.MAX)
    e2e_value = world * n * len(e2e_times) / float(e2e_total.item())
    same = np.array_equal(res, out.cpu().numpy(), equal_nan=True)

    roof = fp64_roofline(torch, local, step_cost(cbf, job, w["system"]), n, spp, statistics.mean(kernel_ms),
                         clocks, probe, w["system"])
    roof["traffic"] = traffic_from_profiles()
    sm_props = torch.cuda.get_device_properties(local)
    roof["step_stream_fp64_pipe_frac"] = step_stream / (
        sm_props.multi_processor_count * FP64_LANES_PER_SM * (clocks.get("sm_mhz") or 1965.0) * 1e6)
    roof["step_stream_note"] = ("FP64 issue rate of the same 8-instruction step and divergence tracking alone "
                                "(2 chains per thread, 6 blocks of 128 per SM; cbf_probe_fp64_step)")

    if rank == 0:
        base = None
        if world == 1 and not args.no_cpu_baseline:
            base = cpu_baseline(w)
        line = {
            "metric": METRIC, "value": value, "unit": "points/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (the parameter grid is the input)",
            "config": {"workload": "chen-lle2d-2048", "grid": f"{w['nPts']}x{w['nPts']}",
                       "system": "chen", "tMax": w["tMax"], "NT": w["NT"], "h": w["h"],
                       "transient": w["transientTime"], "eps": w["lleEps"],
                       "steps_per_point": spp, "points_per_rank": n,
                       "cache": "L2 flushed (256 MB write) before every timed map; inputs are scalars",
                       "parallelism": f"{world} independent c-stripes, one per GPU",
                       "lle_kernel_variant": variant,
                       "autotune_trial_ms": [round(float(x), 3) for x in trial_ms]},
            "e2e": {"value": e2e_value, "unit": "points/s", "h2d_bytes_per_step": C.sizeof(cbf.Job),
                    "d2h_bytes_per_step": n * 8, "matches_device_api": bool(same)},
            "roofline": roof,
            "cpu_baseline": base,
            "gpu_launches": int(launches),
            "clocks": clocks,
            "kernel_ms": kernel_ms,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0 if same else 1


if __name__ == "__main__":
    sys.exit(main())

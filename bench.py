"""Benchmark: 2-D largest-Lyapunov-exponent map, grid points per second.

Workload (one step = one full map): Chen system x'=a(y-x), y'=(c-a)x-xz+cy,
z'=xy-bz on a 2048x2048 (a, c) grid over a in [30,45], c in [20,30], b=3,
h=0.002, Benettin two-trajectory LLE with initial offset 1e-8 renormalised every
NT=0.5 over tMax=1000 after a 500-unit transient (LLE2D semantics of the
reference, seed chunk 200000).  FP64 throughout.  Inputs are synthetic by
nature: the grid itself.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun, one rank per GPU): every rank computes its own 2048x2048 map
of one c-stripe (weak scaling, no data-path collective); time = max over ranks.
The JSON line reports:
  value    device-resident throughput (points/s, all ranks), CUDA events on the
           launching stream around each map, L2 flushed between maps;
  e2e      the same through the public host API (cbf_lle2d: host output buffer,
           device allocation, launch, D2H copy inside the timed region);
  roofline achieved FP64 flops of the LLE kernel vs the FP64 FMA peak measured on
           the same GPU by the library's probe kernel;
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
CHEN_FLOPS_PER_STEP = 26   # FP64 flops of one Chen CD step, FMA = 2 (systems.cuh)
METRIC = "grid points/s, 2D LLE map (plain FP64)"


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


def rank_workload(rank: int, world: int) -> dict:
    w = dict(WORKLOAD)
    if world > 1:
        lo, hi = w["ranges"][2], w["ranges"][3]
        step = (hi - lo) / world
        w["ranges"] = [w["ranges"][0], w["ranges"][1], lo + rank * step, lo + (rank + 1) * step]
    return w


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


def cpu_baseline(w: dict, target_s: float = 15.0) -> dict:
    """Oracle port of the reference per-point code on a strided sample, all threads."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    threads = O.host_threads()
    job = O.make_job(**{k: v for k, v in w.items()})
    n_total = w["nPts"] ** 2
    # calibrate: one point per thread
    probe = np.arange(threads, dtype=np.int64) * (n_total // max(threads, 1))
    t0 = time.perf_counter()
    O.map_lle_list(job, probe, threads)
    dt = time.perf_counter() - t0
    per_round = max(dt, 1e-3)
    rounds = max(1, int(target_s / per_round))
    count = rounds * threads
    stride = max(1, n_total // count)
    idx = (np.arange(count, dtype=np.int64) * stride) % n_total
    t0 = time.perf_counter()
    O.map_lle_list(job, idx, threads)
    dt = time.perf_counter() - t0
    return {"value": count / dt, "unit": "points/s", "cores": threads, "kind": "port",
            "sample": f"{count} of {n_total} points (every {stride}th), full 1.25e6 steps each",
            "seconds": dt}


def traffic_from_profiles():
    """Per-launch DRAM bytes of the LLE kernel from the committed ncu summary, if any."""
    p = ROOT / "profiles" / "lle_chen_2048_ncu.json"
    try:
        d = json.loads(p.read_text())
        return d.get("dram_bytes_per_full_launch")
    except (OSError, ValueError):
        return None


def run_reference(args) -> int:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    w = WORKLOAD
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    if not O.LIB_PATH.exists():
        O.build(with_ref=False)
    threads = O.host_threads()
    job = O.make_job(**w)
    n_total = w["nPts"] ** 2
    # Calibrate on one point per thread, then size every step to ~target seconds.
    target = float(os.environ.get("CBF_REF_STEP_SECONDS", "5"))
    cal = (np.arange(threads, dtype=np.int64) * 7919) % n_total
    t0 = time.perf_counter()
    O.map_lle_list(job, cal, threads)
    t_cal = max(time.perf_counter() - t0, 1e-3)
    per_step = threads * max(1, int(target / t_cal))
    stride = max(1, n_total // (per_step * (args.steps + args.warmup)))
    times = []
    for s in range(args.warmup + args.steps):
        idx = ((np.arange(per_step, dtype=np.int64) + s * per_step) * stride) % n_total
        t0 = time.perf_counter()
        O.map_lle_list(job, idx, threads)
        dt = time.perf_counter() - t0
        if s >= args.warmup:
            times.append(dt)
    tot = sum(times)
    value = per_step * args.steps / tot
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "points/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "chen-lle2d-2048", "grid": "2048x2048", "tMax": 1000, "NT": 0.5,
                   "h": 0.002, "transient": 500, "steps_per_point": steps_per_point(w),
                   "cache": "inputs are scalars; CPU arm"},
        "cpu_baseline": {"value": value, "unit": "points/s", "cores": threads, "kind": "port",
                         "sample": f"{per_step} strided points per step of {n_total}"},
        "e2e": {"value": value, "unit": "points/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--nPts", type=int, default=None, help="override the grid side (testing)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args(argv)

    if args.impl == "reference":
        return run_reference(args)

    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(local)

    cbf = load_cbf()
    cbf.check(cbf.lib().cbf_set_device(local))
    w = rank_workload(rank, world)
    if args.nPts:
        w["nPts"] = args.nPts
    n = w["nPts"] ** 2
    job = cbf.make_job(task=cbf.TASK_LLE, **w)
    spp = steps_per_point(w)

    fp64_peak = cbf.probe_fp64_peak(300.0)  # TFLOP/s, FMA = 2 flops

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
    total_ms = sum(kernel_ms)
    t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
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
    assert np.array_equal(res, out.cpu().numpy(), equal_nan=True), "host and device API maps differ"

    flops_per_launch = float(n) * spp * CHEN_FLOPS_PER_STEP
    achieved = flops_per_launch / (ms_per_step / 1e3) / 1e12 if world == 1 else \
        flops_per_launch / (statistics.mean(kernel_ms) / 1e3) / 1e12
    traffic = traffic_from_profiles()

    if rank == 0:
        base = None
        if world == 1 and not args.no_cpu_baseline:
            base = cpu_baseline(w)
            base.pop("seconds", None)
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
                       "parallelism": f"{world} independent c-stripes, one per GPU"},
            "e2e": {"value": e2e_value, "unit": "points/s", "h2d_bytes_per_step": C.sizeof(cbf.Job),
                    "d2h_bytes_per_step": n * 8},
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": fp64_peak,
                         "unit": "TFLOP/s", "frac": achieved / fp64_peak,
                         "traffic": traffic,
                         "peak_source": "FP64 FMA-chain probe kernel on this GPU, same run "
                                        "(MEASURED_PEAKS.json has no FP64 figure)",
                         "flops_per_launch": flops_per_launch,
                         "flops_per_step": CHEN_FLOPS_PER_STEP},
            "cpu_baseline": base,
            "gpu_launches": int(launches),
            "clocks": clocks,
            "kernel_ms": kernel_ms,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())

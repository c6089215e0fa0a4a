"""Benchmark of the batched FP32 FFT size sweep (packed split-complex, pack 8).

Workload (one step): for every N = 2^6 .. 2^20, a forward and an inverse
(1/N) transform over a 1 GiB buffer of complex64 (batch = 2^27 / N rows),
N(0,1) synthetic data, out of place between two resident 1 GiB buffers (each
larger than the 126 MB L2, so no L2 flush is needed between iterations).

metric: algorithmic GB/s = 16 B per complex point per direction / time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun, one rank per GPU): every rank runs the same sweep on its
own buffers (independent transforms, no collective on the data path: weak
scaling); the step time is the max over ranks.
"""
from __future__ import annotations

import argparse
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
sys.path.insert(0, str(ROOT))

METRIC = "FP32 FFT/fxcorr GB/s, % of HBM peak; tensor-core vs plain at ≤2e-6 rel err"
LOG_NS = list(range(6, 21))
POINTS = 1 << 27    # complex64 points per 1 GiB buffer (overridable by --points for profiling captures)
BYTES_PER_POINT_DIR = 16


def peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d["hbm_gbs"], "src": "measured"}
    return {"hbm_gbs": 6650.0, "src": "fallback"}


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples: list[list[str]] = []
        self._stop = threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.samples.append([s.strip() for s in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self) -> dict:
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[2 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# --------------------------------------------------------------- CPU leg
def cpu_reference(budget_s: float = 12.0) -> dict:
    """The reference fft_unit<float> (compiled from its headers) on the host
    cores: a bounded sample of every size of the sweep, forward + inverse."""
    import oracle as O
    if not O.ref_available():
        return {"value": None, "unit": "GB/s", "cores": 0, "kind": "reference",
                "sample": "unavailable: oracle/_ref/libpcx_ref.so not built"}
    import ctypes
    threads = O.host_threads()
    fp = ctypes.POINTER(ctypes.c_float)
    per_size = budget_s / len(LOG_NS)
    tot_bytes, tot_t, rows_used = 0.0, 0.0, {}
    rng = np.random.default_rng(1)
    for lg in LOG_NS:
        n = 1 << lg
        rows = max(threads, min((POINTS // n), (1 << 22) // n))
        data = rng.standard_normal(rows * 2 * n).astype(np.float32)
        ptr = data.ctypes.data_as(fp)
        # one calibration pass, then as many passes as fit the per-size budget
        t0 = time.perf_counter()
        O.ref().ref_fft_batch_f32(0, n, rows, ptr, 0, threads)
        O.ref().ref_fft_batch_f32(0, n, rows, ptr, 1, threads)
        dt = time.perf_counter() - t0
        reps = max(1, int(per_size / max(dt, 1e-6)) - 1)
        t0 = time.perf_counter()
        for _ in range(reps):
            O.ref().ref_fft_batch_f32(0, n, rows, ptr, 0, threads)
            O.ref().ref_fft_batch_f32(0, n, rows, ptr, 1, threads)
        dt = time.perf_counter() - t0
        tot_t += dt
        tot_bytes += reps * rows * n * BYTES_PER_POINT_DIR * 2
        rows_used[n] = rows * reps
    return {"value": tot_bytes / tot_t / 1e9, "unit": "GB/s", "cores": threads, "kind": "reference",
            "sample": f"fft_unit<float> normal order fwd+inv, per N in 2^6..2^20 a batch of "
                      f"max({threads}, 2^22/N) rows repeated for ~{per_size:.1f} s "
                      f"({sum(rows_used.values())} transforms pairs total)"}


# --------------------------------------------------------------- GPU leg
def run_gpu(args, rank: int, world: int) -> dict | None:
    import torch
    import torch.distributed as dist
    from packed_b200 import fft_unit

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    g = torch.Generator(device=dev).manual_seed(1 + rank)
    reals = 2 * POINTS
    x = torch.randn(reals, device=dev, generator=g)
    y = torch.empty_like(x)
    units = {lg: fft_unit(1 << lg) for lg in LOG_NS}
    stream = torch.cuda.current_stream()

    def step(events=None):
        for lg in LOG_NS:
            n = 1 << lg
            b = POINTS // n
            if events is not None:
                events[lg][0].record(stream)
            units[lg].exec(y, x, batch=b, direction=0)
            units[lg].exec(x, y, batch=b, direction=1)
            if events is not None:
                events[lg][1].record(stream)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        step()
    barrier()
    per = {lg: [] for lg in LOG_NS}
    with ClockSampler(dev.index) as clk:
        t_start = torch.cuda.Event(enable_timing=True)
        t_end = torch.cuda.Event(enable_timing=True)
        barrier()
        t_start.record(stream)
        for _ in range(args.steps):
            ev = {lg: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for lg in LOG_NS}
            step(ev)
            torch.cuda.synchronize()
            for lg in LOG_NS:
                per[lg].append(ev[lg][0].elapsed_time(ev[lg][1]))
        t_end.record(stream)
        barrier()
    ms = t_start.elapsed_time(t_end)
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = t.item()
    clocks = clk.summary()

    # e2e through the public API with host buffers: per size one batch of the
    # same 1 GiB, pinned host -> device, forward + inverse, device -> host
    e2e = None
    if rank == 0:
        host_in = torch.empty(reals, dtype=torch.float32).pin_memory()
        host_in.copy_(x.cpu())
        host_out = torch.empty_like(host_in).pin_memory()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for lg in LOG_NS:
            n = 1 << lg
            x.copy_(host_in, non_blocking=True)
            units[lg].exec(y, x, batch=POINTS // n, direction=0)
            units[lg].exec(x, y, batch=POINTS // n, direction=1)
            host_out.copy_(x, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = e0.elapsed_time(e1)
        e2e_bytes = len(LOG_NS) * POINTS * BYTES_PER_POINT_DIR * 2
        e2e = {"value": e2e_bytes / (e2e_ms / 1e3) / 1e9, "unit": "GB/s",
               "h2d_bytes_per_step": reals * 4 * len(LOG_NS), "d2h_bytes_per_step": reals * 4 * len(LOG_NS),
               "ms_per_step": e2e_ms}
    bytes_step = len(LOG_NS) * POINTS * BYTES_PER_POINT_DIR * 2 * world
    return {"ms": ms, "per": per, "bytes_step": bytes_step, "clocks": clocks, "e2e": e2e, "units": units}


def launches_per_step(units) -> int:
    total = 0
    for lg, u in units.items():
        n = 1 << lg
        b = POINTS // n
        if lg <= 12:
            total += 2
        else:
            chunk = max(1, u.workspace_size(b) // (n * 8))
            total += 2 * 2 * ((b + chunk - 1) // chunk)
    return total


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--points", type=int, default=27, help="log2 complex points per buffer (profiling captures)")
    ap.add_argument("--sizes", type=str, default=None, help="comma list of log2 N (profiling captures)")
    args = ap.parse_args()
    global POINTS, LOG_NS
    POINTS = 1 << args.points
    if args.sizes:
        LOG_NS = [int(v) for v in args.sizes.split(",")]
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    config = {"workload": "C2 FP32 FFT size sweep: N=2^6..2^20, 1 GiB complex64 per size (batch 2^27/N), "
                          "fwd+inv(1/N), pack 8 split-complex, natural order, out of place",
              "global_batch_points": POINTS * world, "sizes": [1 << lg for lg in LOG_NS],
              "l2": "inputs 1 GiB > L2 (no flush needed)", "parallelism": f"independent shards x{world}"}

    if args.impl == "reference":
        if rank != 0:
            return
        times = []
        cb = None
        for i in range(args.warmup + args.steps):
            cb = cpu_reference(budget_s=max(3.0, 12.0 / max(1, args.steps)))
            if i >= args.warmup:
                times.append(cb["value"])
        v = statistics.median(times) if times and times[0] else None
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "GB/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic N(0,1)", "config": config,
                "cpu_baseline": {**cb, "value": v},
                "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    res = run_gpu(args, rank, world)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank != 0:
        return
    pk = peaks()
    ms_step = res["ms"] / args.steps
    value = res["bytes_step"] / (ms_step / 1e3) / 1e9
    # dominant kernel family: the size with the largest share of the step
    mean = {lg: statistics.mean(v) for lg, v in res["per"].items()}
    top = max(mean, key=mean.get)
    alg = POINTS * BYTES_PER_POINT_DIR * 2
    ach = alg / (mean[top] / 1e3) / 1e9
    per_size = {str(1 << lg): round(alg / (mean[lg] / 1e3) / 1e9, 1) for lg in LOG_NS}
    traffic = None
    tp = ROOT / "profiles" / "traffic.json"
    if tp.exists():
        traffic = json.loads(tp.read_text()).get(str(1 << top))
    line = {
        "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic N(0,1), seed 1+rank", "config": config,
        "pct_hbm": 100.0 * value / world / pk["hbm_gbs"],
        "per_size_gbs": per_size,
        "roofline": {"bound": "hbm", "achieved": ach, "peak": pk["hbm_gbs"], "unit": "GB/s",
                     "frac": ach / pk["hbm_gbs"], "traffic": traffic, "peak_src": pk["src"],
                     "kernel": f"N={1 << top} fwd+inv ({'single-pass' if top <= 12 else 'four-step'})",
                     "algorithmic_bytes_per_launch": alg // 2},
        "clocks": res["clocks"], "e2e": res["e2e"], "gpu_launches": launches_per_step(res["units"]) * args.steps,
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_reference()
    print(json.dumps(line))


if __name__ == "__main__":
    main()

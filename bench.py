"""Benchmarks of the packed FFT / correlation hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c2|c1|c3|c4|c5]

Workloads (synthetic data, N(0,1) unless stated; all buffers stay resident in
HBM and are larger than the 126 MB L2, so no flush is needed between steps):

  c2 (default)  FP32 FFT size sweep: for every N = 2^6..2^20 a forward and an
                inverse (1/N) transform over a 1 GiB complex64 buffer (batch
                2^27/N), pack 8 split-complex, natural order, out of place.
  c1            N=1024, batch 64, forward then inverse (U[-1,1), seed 0).
  c3            fxcorr: 256 channels x 2^20 complex64 samples correlated in place
                with a 4096-tap kernel (sigma 1/64) by overlap-save, N_fft 16384.
  c4            tensor-core form: N in {256, 1024, 4096}, batch 4096, split-bf16
                and split-tf32 DFT-matrix stages vs the plain FP32 path, with
                rel L2 / max-abs / tone-bin error vs FP64 per N.
  c5            ragged batch: 10,000 FFTs, N log-uniform 2^8..2^18, plus 500
                correlations (S 2^12..2^20, K 64..8192), one persistent launch
                replayed from a CUDA graph, against per-size plain launches.

metric: algorithmic GB/s = 16 B per complex point per direction (c2, c1, c5)
or 16 B per signal sample (c3), divided by the device time of the step.
Multi-GPU (torchrun, one rank per GPU): every rank runs the same workload on
its own buffers (independent transforms, no collective: weak scaling); the
step time is the max over ranks.
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
B_PT = 16    # algorithmic bytes per complex point per direction (read + write complex64)


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
        self._proc = None
        self._t = None

    def _run(self):
        try:
            self._proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            for line in self._proc.stdout:
                self.samples.append([s.strip() for s in line.strip().split(",")])
        except Exception:
            pass

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        time.sleep(0.15)
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()
        if self._t is not None:
            self._t.join(timeout=5)

    def summary(self) -> dict:
        rows = [s for s in self.samples if len(s) >= 6 and s[0].replace(".", "").isdigit()]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in rows]
        mx = [float(s[1]) for s in rows if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in rows for i in range(4) if s[2 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


# --------------------------------------------------------------- workloads
def pipelined_e2e(torch, host_in, host_out, chunks, slot_reals, compute, reps=1, warmup=1):
    """Host -> device -> host through the library, chunk by chunk, with the
    copy of chunk c+1 in, the transform of chunk c and the copy of chunk c-1
    out in flight together on three streams (two device slots).
    chunks: (host offset in reals, reals, key); compute(slot_tensor, reals, key,
    stream) runs the library calls in place on the slot.  The slots and
    streams are set up once, `warmup` untimed passes over the chunks run
    first, then `reps` passes back to back are timed.  Returns ms per pass."""
    dev = torch.cuda.current_device()
    slots = [torch.empty(slot_reals, dtype=host_in.dtype, device=dev) for _ in range(2)]
    s_in, s_cmp, s_out = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    main = torch.cuda.current_stream()
    freed = [torch.cuda.Event(), torch.cuda.Event()]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def run(passes):
        for st in (s_in, s_cmp, s_out):
            st.wait_stream(main)
        work = [c for _ in range(passes) for c in chunks]
        for c, (off, n, key) in enumerate(work):
            k = c % 2
            buf = slots[k][:n]
            if c >= 2:
                s_in.wait_event(freed[k])
            with torch.cuda.stream(s_in):
                buf.copy_(host_in[off:off + n], non_blocking=True)
                landed = torch.cuda.Event()
                landed.record(s_in)
            s_cmp.wait_event(landed)
            with torch.cuda.stream(s_cmp):
                compute(buf, n, key, s_cmp)
                done = torch.cuda.Event()
                done.record(s_cmp)
            s_out.wait_event(done)
            with torch.cuda.stream(s_out):
                host_out[off:off + n].copy_(buf, non_blocking=True)
                freed[k].record(s_out)
        main.wait_stream(s_out)

    if warmup:
        run(warmup)
    torch.cuda.synchronize()
    e0.record(main)
    run(reps)
    e1.record(main)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


class C2Sweep:
    name = "c2"
    log_ns = list(range(6, 21))
    points = 1 << 27

    def config(self, world):
        return {"workload": "C2 FP32 FFT size sweep: N=2^6..2^20, 1 GiB complex64 per size (batch 2^27/N), "
                            "fwd+inv(1/N), pack 8 split-complex, natural order, out of place",
                "sizes": [1 << lg for lg in self.log_ns], "global_batch_points": self.points * world,
                "l2": "inputs 1 GiB > L2 (no flush needed)", "parallelism": f"independent shards x{world}"}

    def setup(self, dev, rank):
        import torch
        from packed_b200 import fft_unit
        g = torch.Generator(device=dev).manual_seed(1 + rank)
        self.x = torch.randn(2 * self.points, device=dev, generator=g)
        self.y = torch.empty_like(self.x)
        self.units = {lg: fft_unit(1 << lg) for lg in self.log_ns}
        # autotuner: time each size's forms on this batch, keep the fastest
        self.forms = {str(1 << lg): u.tune(self.points >> lg) for lg, u in self.units.items()
                      if self.tune and lg > 12}

    tune = True

    def bytes_per_step(self):
        return len(self.log_ns) * self.points * B_PT * 2

    def parts(self):
        return [str(1 << lg) for lg in self.log_ns]

    def run_part(self, key):
        lg = int(key).bit_length() - 1
        b = self.points >> lg
        self.units[lg].exec(self.y, self.x, batch=b, direction=0, check=False)
        self.units[lg].exec(self.x, self.y, batch=b, direction=1, check=False)

    def part_bytes(self, key):
        return self.points * B_PT * 2

    def part_work(self, key):
        """(transforms, 5 N log2 N flops) of one part: forward + inverse over the buffer."""
        lg = int(key).bit_length() - 1
        rows = self.points >> lg
        return 2 * rows, 2 * rows * 5 * (1 << lg) * lg

    def check_status(self):
        """Raise if a kernel gave up a bounded wait during the run (rows unwritten)."""
        for u in self.units.values():
            u.status()

    e2e_chunks = 8

    def e2e(self, torch, stream):
        host_in = torch.empty(2 * self.points, dtype=torch.float32).pin_memory()
        host_in.copy_(self.x.cpu())
        host_out = torch.empty_like(host_in).pin_memory()
        dev = torch.cuda.current_device()
        scratch = torch.empty((2 * self.points + self.e2e_chunks - 1) // self.e2e_chunks, device=dev)
        chunks = []
        for lg in self.log_ns:
            rows = self.points >> lg
            per = max(1, rows // self.e2e_chunks)
            for r0 in range(0, rows, per):
                nr = min(per, rows - r0)
                chunks.append((r0 * 2 << lg, nr * 2 << lg, lg))

        def compute(buf, n, lg, st):    # forward into scratch, inverse back: the exec calls themselves
            rows = n >> (lg + 1)
            u = self.units[lg]
            u.exec(scratch[:n], buf, batch=rows, direction=0, stream=st, check=False)
            u.exec(buf, scratch[:n], batch=rows, direction=1, stream=st, check=False)

        ms = pipelined_e2e(torch, host_in, host_out, chunks, scratch.numel(), compute)
        nb = 2 * self.points * 4 * len(self.log_ns)
        return {"value": self.bytes_per_step() / (ms / 1e3) / 1e9, "unit": "GB/s", "h2d_bytes_per_step": nb,
                "d2h_bytes_per_step": nb, "ms_per_step": ms}

    def launches(self):
        # per direction: one kernel (one pass, or the one-launch four-step), or
        # two per scratch chunk when the autotuner chose the chunked four-step
        total = 0
        for lg, u in self.units.items():
            f = u.form()
            if lg > 12 and f["form"] == "chunked four-step":
                rows = self.points >> lg
                per = max(1, f["chunk_bytes"] // ((1 << lg) * 8))
                total += 2 * 2 * ((rows + per - 1) // per)
            else:
                total += 2
        return total

    def cpu_reference(self, budget_s=12.0):
        import ctypes
        import oracle as O
        if not O.ref_available():
            return {"value": None, "unit": "GB/s", "cores": 0, "kind": "reference",
                    "sample": "unavailable: oracle/_ref/libpcx_ref.so not built"}
        threads = O.host_threads()
        fp = ctypes.POINTER(ctypes.c_float)
        per = budget_s / len(self.log_ns)
        tot_b, tot_t = 0.0, 0.0
        rng = np.random.default_rng(1)
        for lg in self.log_ns:
            n = 1 << lg
            rows = max(threads, min(self.points >> lg, (1 << 22) >> lg))
            data = rng.standard_normal(rows * 2 * n).astype(np.float32)
            ptr = data.ctypes.data_as(fp)
            t0 = time.perf_counter()
            O.ref().ref_fft_batch_f32(0, n, rows, ptr, 0, threads)
            O.ref().ref_fft_batch_f32(0, n, rows, ptr, 1, threads)
            reps = max(1, int(per / max(time.perf_counter() - t0, 1e-6)) - 1)
            t0 = time.perf_counter()
            for _ in range(reps):
                O.ref().ref_fft_batch_f32(0, n, rows, ptr, 0, threads)
                O.ref().ref_fft_batch_f32(0, n, rows, ptr, 1, threads)
            tot_t += time.perf_counter() - t0
            tot_b += reps * rows * n * B_PT * 2
        return {"value": tot_b / tot_t / 1e9, "unit": "GB/s", "cores": threads, "kind": "reference",
                "sample": f"reference fft_unit<float> (oracle/_ref) normal order fwd+inv on {threads} threads; "
                          f"per N in 2^{self.log_ns[0]}..2^{self.log_ns[-1]} a sample of max({threads}, 2^22/N) rows "
                          f"(2^22 points = 32 MiB of complex64, of the 2^{self.points.bit_length() - 1}-point "
                          f"workload) repeated for ~{per:.1f} s; GB/s in the bench's unit (16 B per point per "
                          f"direction)"}


class C1(C2Sweep):
    name = "c1"
    log_ns = [10]
    points = 1024 * 64

    def config(self, world):
        return {"workload": "C1: N=1024, batch 64, forward then inverse (1/N), pack 8, U[-1,1) seed 0; step = "
                            "CUDA-graph replay of the two exec calls (direct calls timed as 'direct:1024')",
                "global_batch_points": self.points * world, "l2": "1 MiB working set (L2 resident: latency-bound)",
                "parallelism": f"independent shards x{world}"}

    def setup(self, dev, rank):
        import torch
        from packed_b200 import fft_unit
        rng = np.random.default_rng(0)
        z = rng.uniform(-1, 1, (64, 1024)) + 1j * rng.uniform(-1, 1, (64, 1024))
        a = np.zeros((64, 128, 2, 8), np.float32)
        a[:, :, 0, :] = z.real.reshape(64, 128, 8)
        a[:, :, 1, :] = z.imag.reshape(64, 128, 8)
        self.x = torch.as_tensor(a.reshape(-1)).to(dev)
        self.y = torch.empty_like(self.x)
        self.units = {10: fft_unit(1024)}
        # the step is launch-bound (0.5 MB per exec): capture the forward and
        # inverse exec calls once in a CUDA graph and replay it; the direct
        # calls are timed beside it
        for _ in range(2):
            C2Sweep.run_part(self, "1024")
        torch.cuda.synchronize()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self.graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(self.graph, stream=s):
                C2Sweep.run_part(self, "1024")
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()

    def parts(self):
        return ["1024", "direct:1024"]

    def part_work(self, key):
        return C2Sweep.part_work(self, "1024")

    def run_part(self, key):
        if key == "1024":
            self.graph.replay()
        else:
            C2Sweep.run_part(self, "1024")

    def e2e(self, torch, stream):
        """Host -> device -> host per step: the copy in from pinned memory, the
        forward and inverse exec calls and the copy out, captured together in
        one CUDA graph (the step is launch-bound: 0.5 MB each way) and
        replayed back to back."""
        host_in = torch.empty(self.x.numel(), dtype=torch.float32).pin_memory()
        host_in.copy_(self.x.cpu())
        host_out = torch.empty_like(host_in).pin_memory()
        buf, tmp = torch.empty_like(self.x), torch.empty_like(self.x)
        u = self.units[10]
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())

        def step():
            buf.copy_(host_in, non_blocking=True)
            u.exec(tmp, buf, batch=64, direction=0, check=False)
            u.exec(buf, tmp, batch=64, direction=1, check=False)
            host_out.copy_(buf, non_blocking=True)

        with torch.cuda.stream(s):
            for _ in range(3):
                step()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=s):
                step()
            for _ in range(3):
                g.replay()
        torch.cuda.synchronize()
        reps = 500
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        with torch.cuda.stream(s):
            for _ in range(reps):
                g.replay()
        e1.record(s)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        nb = self.x.numel() * 4
        return {"value": self.bytes_per_step() / (ms / 1e3) / 1e9, "unit": "GB/s", "h2d_bytes_per_step": nb,
                "d2h_bytes_per_step": nb, "ms_per_step": ms, "form": "CUDA graph of copy in, exec x2, copy out"}

    def launches(self):
        return 4    # two kernels per form


class C3Fxcorr:
    name = "c3"
    channels, length, k, n_fft = 256, 1 << 20, 4096, 16384

    def config(self, world):
        return {"workload": "C3 fxcorr: 256 channels x 2^20 complex64 (N(0,1) seed 2), 4096-tap kernel "
                            "(N(0,1/4096) seed 3), overlap-save N_fft 16384 (step 12288), in place, pack 8",
                "global_batch_points": self.channels * self.length * world,
                "l2": "2 GiB signal > L2 (no flush needed)", "parallelism": f"independent shards x{world}"}

    def setup(self, dev, rank):
        import torch
        from packed_b200 import fxcorr_unit, vector
        g = torch.Generator(device=dev).manual_seed(2 + rank)
        self.x = torch.randn(self.channels * 2 * self.length, device=dev, generator=g)
        # the adjoint's inputs: an output cotangent (the gradient of the
        # weighted |y|^2 loss has this shape and distribution class)
        self.gy = torch.randn(self.channels * 2 * self.length, device=dev, generator=g)
        rng = np.random.default_rng(3)
        taps = (rng.standard_normal(self.k) + 1j * rng.standard_normal(self.k)) / 64
        self.unit = fxcorr_unit(vector.from_complex(taps, device=dev), self.n_fft)

    def bytes_per_step(self):
        return self.channels * self.length * B_PT

    def parts(self):
        # the forward correlator (the line's value) and the two halves of its
        # adjoint, timed beside it: the signal gradient (a convolution of gy
        # with the kernel) and the kernel gradient (block spectra of x and gy)
        return ["fxcorr", "vjp_x", "vjp_g"]

    def run_part(self, key):
        if key == "fxcorr":
            self.unit.exec(self.x, self.x, self.length, channels=self.channels, check=False)
        else:
            self.unit.vjp(self.gy, self.x, self.length, channels=self.channels, want_signal_grad=key == "vjp_x",
                          want_kernel_grad=key == "vjp_g")

    def check_status(self):
        self.unit.status()

    def part_work(self, key):
        """Two N_fft-point transforms per overlap-save block (forward and
        inverse; the kernel gradient: two forward, and one inverse in all)."""
        step = self.n_fft - self.k + 1
        blocks = self.channels * -(-self.length // step)
        lg = self.n_fft.bit_length() - 1
        tf = 2 * blocks + (1 if key == "vjp_g" else 0)
        return tf, tf * 5 * self.n_fft * lg

    def part_bytes(self, key):
        """16 B per signal sample: x in and y out; gy in and gx out; x and gy in."""
        return self.bytes_per_step()

    def e2e(self, torch, stream):
        host_in = torch.empty_like(self.x, device="cpu").pin_memory()
        host_in.copy_(self.x.cpu())
        host_out = torch.empty_like(host_in).pin_memory()
        group = max(1, self.channels // 8)    # channels per pipelined chunk
        per = 2 * self.length
        chunks = [(c0 * per, min(group, self.channels - c0) * per, None) for c0 in range(0, self.channels, group)]

        def compute(buf, n, _, st):    # the correlator call itself, in place
            self.unit.exec(buf, buf, self.length, channels=n // per, stream=st, check=False)

        ms = pipelined_e2e(torch, host_in, host_out, chunks, group * per, compute)
        nb = self.x.numel() * 4
        return {"value": self.bytes_per_step() / (ms / 1e3) / 1e9, "unit": "GB/s", "h2d_bytes_per_step": nb,
                "d2h_bytes_per_step": nb, "ms_per_step": ms}

    def launches(self):
        # forward: one kernel; signal gradient: one; kernel gradient: the
        # per-block spectra, their reduction, the inverse FFT and the repack
        return 1 + 1 + 4

    def cpu_reference(self, budget_s=12.0):
        import ctypes
        import oracle as O
        if not O.ref_available():
            return {"value": None, "unit": "GB/s", "cores": 0, "kind": "reference",
                    "sample": "unavailable: oracle/_ref/libpcx_ref.so not built"}
        threads = O.host_threads()
        fp = ctypes.POINTER(ctypes.c_float)
        rng = np.random.default_rng(3)
        taps = ((rng.standard_normal(self.k) + 1j * rng.standard_normal(self.k)) / 64).astype(np.complex64)
        g = O.pack(taps, 8)
        ch = max(threads, 8)
        sig = np.random.default_rng(2).standard_normal(ch * 2 * self.length).astype(np.float32)
        t0 = time.perf_counter()
        reps = 0
        while True:
            O.ref().ref_fxcorr_fixed_batch_f32(g.ctypes.data_as(fp), self.k, self.n_fft, sig.ctypes.data_as(fp),
                                               self.length, ch, threads)
            reps += 1
            if time.perf_counter() - t0 > budget_s / 2:
                break
        dt = time.perf_counter() - t0
        return {"value": reps * ch * self.length * B_PT / dt / 1e9, "unit": "GB/s", "cores": threads,
                "kind": "reference",
                "sample": f"reference fft_unit<float, unordered> overlap-save (offsets corrected) on {threads} "
                          f"threads, {ch} channels x 2^20 x {reps} repetitions"}


class C4TensorCore:
    """Tensor-core split-precision FFT against the plain FP32 path, batch 4096."""
    name = "c4"
    log_ns = [8, 10, 12, 14, 16]
    tc_max = 16    # the tensor-core form: one pass up to 4096, two passes for 16384 and 65536
    batch = 4096

    def config(self, world):
        return {"workload": "C4: N in {256, 1024, 4096, 16384, 65536}, batch 4096, complex64 N(0,1) + 1e-3 tone at "
                            "a seeded bin (seed 4); tensor-core split-bf16 (2 parts, 3 products), split-tf32 and "
                            "split-bf16 (3 parts, 6 products) forward vs plain FP32 "
                            "forward; each part replayed from a CUDA graph of its exec call",
                "global_batch_points": sum(self.batch << lg for lg in self.log_ns) * world,
                "l2": "inputs 8-128 MiB per size; timed steps back to back",
                "parallelism": f"independent shards x{world}"}

    def setup(self, dev, rank):
        import torch
        from packed_b200 import fft_unit
        self.units, self.x, self.y, self.z = {}, {}, {}, {}
        rng = np.random.default_rng(4)
        for lg in self.log_ns:
            n = 1 << lg
            # the first 16 rows (the accuracy sample) come from numpy; the rest,
            # same distribution, from the device generator
            rows = 16 if lg > 12 else self.batch
            z = rng.standard_normal((rows, n)) + 1j * rng.standard_normal((rows, n))
            k = rng.integers(0, n, rows)
            z += 1e-3 * np.exp(2j * np.pi * k[:, None] * np.arange(n)[None, :] / n)
            a = np.zeros((rows, n // 8, 2, 8), np.float32)
            a[:, :, 0, :] = z.real.reshape(rows, -1, 8)
            a[:, :, 1, :] = z.imag.reshape(rows, -1, 8)
            self.z[lg] = (z[:16], k[:16])
            if rows == self.batch:
                self.x[lg] = torch.as_tensor(a.reshape(-1)).to(dev)
            else:
                g = torch.Generator(device=dev).manual_seed(4)
                self.x[lg] = torch.randn(self.batch * 2 * n, device=dev, generator=g)
                self.x[lg][: rows * 2 * n] = torch.as_tensor(a.reshape(-1)).to(dev)
            self.y[lg] = torch.empty_like(self.x[lg])
            self.units[lg] = fft_unit(n)
            if lg > 12:
                self.units[lg].tune(self.batch)
        # each part is one exec call of 8-512 MB; the small ones take a few
        # microseconds on the GPU, less than the host needs to issue them, so
        # every part is captured once in a CUDA graph and replayed
        self.graphs = {}
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            for key in self.parts():
                for _ in range(2):
                    self._call(key)
                g = torch.cuda.CUDAGraph()
                try:
                    with torch.cuda.graph(g, stream=s):
                        self._call(key)
                    self.graphs[key] = g
                except RuntimeError:    # a form that cannot be captured runs directly
                    torch.cuda.synchronize()
                    self.graphs[key] = None
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()

    def forms_of(self, lg):
        return ("plain", "tc_bf16", "tc_tf32", "tc_bf16x6") if lg <= self.tc_max else ("plain",)

    def parts(self):
        return [f"{m}:{1 << lg}" for lg in self.log_ns for m in self.forms_of(lg)]

    def _split(self, key):
        m, n = key.split(":")
        return m, int(n).bit_length() - 1

    def _call(self, key):
        m, lg = self._split(key)
        u = self.units[lg]
        if m == "plain":
            u.exec(self.y[lg], self.x[lg], batch=self.batch, check=False)
        else:
            u.exec_tensor_core(self.y[lg], self.x[lg], batch=self.batch, precision=m[3:], check=False)

    def run_part(self, key):
        g = self.graphs[key]
        if g is None:
            self._call(key)
        else:
            g.replay()

    def part_bytes(self, key):
        _, lg = self._split(key)
        return (self.batch << lg) * B_PT

    def check_status(self):
        for u in self.units.values():
            u.status()

    def part_work(self, key):
        _, lg = self._split(key)
        return self.batch, self.batch * 5 * (1 << lg) * lg

    def bytes_per_step(self):
        return sum(self.part_bytes(p) for p in self.parts())

    def accuracy(self):
        """rel L2 / max-abs / tone-bin error vs FP64 per N and form (first 16 rows)."""
        import torch
        out = {}
        for lg in self.log_ns:
            n = 1 << lg
            z, k = self.z[lg]
            want = np.fft.fft(z, axis=-1)
            for m in self.forms_of(lg):
                self.run_part(f"{m}:{n}")
                torch.cuda.synchronize()
                a = self.y[lg][: 16 * 2 * n].cpu().numpy().astype(np.float64).reshape(16, -1, 2, 8)
                got = (a[:, :, 0, :] + 1j * a[:, :, 1, :]).reshape(16, n)
                rel = float(np.linalg.norm(got - want) / np.linalg.norm(want))
                mx = float(np.abs(got - want).max())
                tone = float(np.abs(got[np.arange(16), k] - want[np.arange(16), k]).max())
                out[f"{m}:{n}"] = {"rel_l2": rel, "max_abs": mx, "tone_bin_abs": tone}
        return out

    def e2e(self, torch, stream):
        return None

    def launches(self):
        total = 0
        for key in self.parts():
            m, lg = self._split(key)
            chunk = max(1, min(self.batch, (int(os.environ.get("PCX_SCRATCH_MB", "24")) << 20) // ((1 << lg) * 8)))
            chunks = (self.batch + chunk - 1) // chunk
            if m != "plain":
                total += 1 if lg <= 12 else 2 * chunks    # two-pass form: two launches per chunk
                continue
            f = self.units[lg].form() if lg > 12 else {"form": "default"}
            if f["form"] == "chunked four-step":
                chunk = max(1, f["chunk_bytes"] // ((1 << lg) * 8))
                total += 2 * ((self.batch + chunk - 1) // chunk)
            else:
                total += 1
        return total

    def cpu_reference(self, budget_s=12.0):
        c2 = C2Sweep()
        c2.log_ns = list(self.log_ns)
        return c2.cpu_reference(budget_s)


class C5Ragged:
    """Ragged batch: one persistent launch (graph) vs per-size plain launches."""
    name = "c5"
    n_fft, n_xc = 10000, 500

    def config(self, world):
        return {"workload": f"C5: {self.n_fft:,} complex64 FFTs, N log-uniform 2^8..2^18, plus {self.n_xc} correlations "
                            "(S log-uniform 2^12..2^20, K log-uniform 64..8192, N_fft per request from "
                            "correlation_fft_size(K)), "
                            "N(0,1) seed 5; one persistent launch from a device work queue replayed as a CUDA "
                            "graph, vs per-size plain launches",
                "global_batch_points": None, "parallelism": f"independent shards x{world}"}

    def setup(self, dev, rank):
        import torch
        from packed_b200 import correlation_fft_size, fft_unit, fxcorr_unit, ragged_batch, vector
        rng = np.random.default_rng(5)
        lgs = np.floor(rng.uniform(8, 19, self.n_fft)).astype(int)
        self.groups = {}
        for lg in sorted(set(lgs.tolist())):
            cnt = int((lgs == lg).sum())
            n = 1 << lg
            src = torch.randn(cnt * 2 * n, device=dev)
            self.groups[lg] = (cnt, src, torch.empty_like(src), fft_unit(n))
        ffts = []
        for lg, (cnt, src, dst, _) in self.groups.items():
            n = 1 << lg
            for i in range(cnt):
                ffts.append((dst[i * 2 * n:(i + 1) * 2 * n], src[i * 2 * n:(i + 1) * 2 * n], n))
        self.xcs, self.xunits = [], []
        s_all = np.floor(2 ** rng.uniform(12, 20, self.n_xc)).astype(int) // 8 * 8
        k_all = np.floor(2 ** rng.uniform(6, 13, self.n_xc)).astype(int)
        self.xc_points = int(s_all.sum())
        for s, k in zip(s_all, k_all):
            nf = correlation_fft_size(int(k))    # per request, from the transform-work model
            taps = vector.from_complex(rng.standard_normal(k) + 1j * rng.standard_normal(k), device=dev)
            x = torch.randn(2 * int(s), device=dev)
            y = torch.empty_like(x)
            self.xcs.append((y, x, int(s), taps, nf))
            self.xunits.append(fxcorr_unit(taps, nf))
        self.batch = ragged_batch(ffts, self.xcs)
        # the same batch with the transforms of 2^8..2^12 points in the
        # tensor-core form (bf16 x6, FP32-level accuracy), timed beside it
        self.batch_tc = ragged_batch(ffts, self.xcs, tensor_core="bf16x6")
        self.fft_points = sum(cnt << lg for lg, (cnt, _, _, _) in self.groups.items())
        self.fft_flops = sum(cnt * 5 * (lg << lg) for lg, (cnt, _, _, _) in self.groups.items())
        self.xc_ffts, self.xc_flops = 0, 0
        for (_, _, s, taps, nf) in self.xcs:
            blocks = -(-s // (nf - taps.size() + 1))
            self.xc_ffts += 2 * blocks
            self.xc_flops += 2 * blocks * 5 * nf * (nf.bit_length() - 1)

    def parts(self):
        return ["ragged_graph", "ragged_graph_tc", "plain_per_size"]

    def run_part(self, key):
        if key == "ragged_graph":
            self.batch()
        elif key == "ragged_graph_tc":
            self.batch_tc()
        else:
            for lg, (cnt, src, dst, u) in self.groups.items():
                u.exec(dst, src, batch=cnt, check=False)
            for (y, x, s, _, _), u in zip(self.xcs, self.xunits):
                u.exec(y, x, s, check=False)

    def part_bytes(self, key):
        return (self.fft_points + self.xc_points) * B_PT

    def part_work(self, key):
        t = sum(cnt for cnt, _, _, _ in self.groups.values()) + self.xc_ffts
        return t, self.fft_flops + self.xc_flops

    def check_status(self):
        self.batch.status()
        self.batch_tc.status()
        for _, _, _, u in self.groups.values():
            u.status()
        for u in self.xunits:
            u.status()

    def bytes_per_step(self):
        return self.part_bytes("ragged_graph")

    def accuracy(self):
        """Worst relative L2 error over every transform and every correlation of
        one ragged replay, against FP64 references computed on the device from
        the same FP32 inputs (torch.fft as the checker), outside the timed region."""
        import torch

        def rows(t, n):    # pack-8 rows -> complex128 [rows, n]
            v = t.reshape(-1, n // 8, 2, 8).double()
            return torch.complex(v[:, :, 0, :].reshape(-1, n), v[:, :, 1, :].reshape(-1, n))

        def rel(got, want):
            return torch.linalg.vector_norm(got - want, dim=-1) / torch.linalg.vector_norm(want, dim=-1)

        def worst_fft(lgs):
            w = 0.0
            for lg in lgs:
                cnt, src, dst, _ = self.groups[lg]
                n = 1 << lg
                for r0 in range(0, cnt, 128):
                    r1 = min(cnt, r0 + 128)
                    e = rel(rows(dst[r0 * 2 * n:r1 * 2 * n], n), torch.fft.fft(rows(src[r0 * 2 * n:r1 * 2 * n], n)))
                    w = max(w, float(e.max()))
            return w

        # the tensor-core batch first (same outputs), its transforms of 2^8..2^12
        self.batch_tc()
        torch.cuda.synchronize()
        self.batch_tc.status()
        w_tc = worst_fft([lg for lg in self.groups if 8 <= lg <= 12])
        self.batch()
        torch.cuda.synchronize()
        self.batch.status()
        w_xc = 0.0
        w_fft = worst_fft(list(self.groups))
        for y, x, s, taps, _ in self.xcs:
            k = taps.size()
            kp = (k + 7) // 8 * 8
            g = rows(taps.data[: 2 * kp], kp)[0, :k]
            L = 1 << int(np.ceil(np.log2(s + k)))
            want = torch.fft.ifft(torch.fft.fft(rows(x, s)[0], L) * torch.conj(torch.fft.fft(g, L)))[:s]
            w_xc = max(w_xc, float(rel(rows(y, s)[0], want)))
        return {"ragged_fft_max_rel_l2": w_fft, "ragged_xcorr_max_rel_l2": w_xc,
                "ragged_tc_bf16x6_fft_max_rel_l2": w_tc,
                "transforms": sum(c for c, _, _, _ in self.groups.values()), "correlations": len(self.xcs)}

    def e2e(self, torch, stream):
        return None

    def launches(self):
        # the ragged graph; the tensor-core graph (ragged launch + tensor-core
        # launch); per-size plain launches and one per correlation
        return 1 + 2 + len(self.groups) + self.n_xc

    def cpu_reference(self, budget_s=12.0):
        c2 = C2Sweep()
        c2.log_ns = list(range(8, 19))
        return c2.cpu_reference(budget_s)


WORKLOADS = {"c2": C2Sweep, "c1": C1, "c3": C3Fxcorr, "c4": C4TensorCore, "c5": C5Ragged}


# ----------------------------------------------------------------- driver
def max_over_ranks(torch, dist, value: float, device) -> float:
    """The slowest rank's step time: every rank transforms its own shard of
    the same size (weak scaling), and the job is done when the last one is."""
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_gbs(bytes_per_rank_step: float, world: int, ms_step: float) -> float:
    """Aggregate GB/s of all ranks: every rank moves bytes_per_rank_step per step."""
    return bytes_per_rank_step * world / (ms_step / 1e3) / 1e9


def run(args, wl, rank, world):
    import torch
    import torch.distributed as dist

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    wl.setup(dev, rank)
    stream = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        for p in wl.parts():
            wl.run_part(p)
    barrier()
    per = {p: [] for p in wl.parts()}
    with ClockSampler(dev.index) as clk:
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        ev = [{p: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for p in wl.parts()}
              for _ in range(args.steps)]
        barrier()
        t0.record(stream)
        for s in range(args.steps):
            for p in wl.parts():
                ev[s][p][0].record(stream)
                wl.run_part(p)
                ev[s][p][1].record(stream)
        t1.record(stream)
        barrier()
    wl.check_status()    # outside the timed region: a bounded wait that gave up fails the run
    ms = t0.elapsed_time(t1)
    for s in range(args.steps):
        for p in wl.parts():
            per[p].append(ev[s][p][0].elapsed_time(ev[s][p][1]))
    if world > 1:
        ms = max_over_ranks(torch, dist, ms, dev)
    e2e = wl.e2e(torch, stream) if rank == 0 else None
    return {"ms": ms, "per": per, "clocks": clk.summary(), "e2e": e2e}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="c2")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--points", type=int, default=None, help="log2 complex points per buffer (profiling captures)")
    ap.add_argument("--sizes", type=str, default=None, help="comma list of log2 N (profiling captures)")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner (built-in form choice)")
    ap.add_argument("--items", type=float, default=None,
                    help="c5: fraction of the 10,000 FFTs and 500 correlations (profiling captures)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    wl = WORKLOADS[args.workload]()
    if args.points is not None and hasattr(wl, "points"):
        wl.points = 1 << args.points
    if args.points is not None and hasattr(wl, "channels"):
        wl.channels = max(1, (1 << args.points) // wl.length)
    if args.sizes and hasattr(wl, "log_ns"):
        wl.log_ns = [int(v) for v in args.sizes.split(",")]
    if args.no_tune:
        wl.tune = False
    if args.items is not None and hasattr(wl, "n_xc"):
        wl.n_fft = max(1, int(round(wl.n_fft * args.items)))
        wl.n_xc = max(1, int(round(wl.n_xc * args.items)))
    config = wl.config(world)

    if args.impl == "reference":
        if rank != 0:
            return
        vals, cb = [], None
        for i in range(args.warmup + args.steps):
            cb = wl.cpu_reference(budget_s=max(3.0, 60.0 / max(1, args.warmup + args.steps)))
            if i >= args.warmup:
                vals.append(cb["value"])
        v = statistics.median(vals) if vals and vals[0] is not None else None
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "GB/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config,
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
    res = run(args, wl, rank, world)
    if isinstance(getattr(wl, "forms", None), dict):
        config["forms"] = wl.forms    # the autotuner's choice per four-step size
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank != 0:
        return
    pk = peaks()
    ms_step = res["ms"] / args.steps
    value = whole_job_gbs(wl.bytes_per_step(), world, ms_step)
    if wl.name in ("c1", "c3", "c4", "c5"):
        # the step runs several alternative forms of the same work, or work
        # beside the headline: report the headline form's own time (c5: the
        # ragged graph; c4: the fastest form; c3: the forward correlator)
        means = {p: statistics.mean(v) for p, v in res["per"].items()}
        if wl.name == "c5":
            ms_step = means["ragged_graph"]
            nbytes  = wl.bytes_per_step()
        elif wl.name == "c3":
            ms_step = means["fxcorr"]
            nbytes  = wl.bytes_per_step()
        elif wl.name == "c1":
            ms_step = means["1024"]
            nbytes  = wl.part_bytes("1024")
        else:
            # one transform of each size, in its fastest form
            ms_step = sum(min(means[f"{m}:{1 << lg}"] for m in wl.forms_of(lg)) for lg in wl.log_ns)
            nbytes  = sum(wl.part_bytes(f"plain:{1 << lg}") for lg in wl.log_ns)
        value = whole_job_gbs(nbytes, world, ms_step)
    mean = {p: statistics.mean(v) for p, v in res["per"].items()}
    per_part = {p: round(wl.part_bytes(p) / (mean[p] / 1e3) / 1e9, 1) for p in wl.parts()}
    # the parts `value` counts (for c1/c4/c5 only the headline form of each
    # piece of work); throughput in the other units, transforms/s and
    # 5 N log2 N GFLOP/s, is whole job (all ranks) over the same device time
    if wl.name in ("c1", "c3", "c4", "c5"):
        if wl.name == "c5":
            counted = ["ragged_graph"]
        elif wl.name == "c3":
            counted = ["fxcorr"]
        elif wl.name == "c1":
            counted = ["1024"]
        else:
            counted = [min((f"{m}:{1 << lg}" for m in wl.forms_of(lg)), key=lambda q: means[q]) for lg in wl.log_ns]
    else:
        counted = wl.parts()
    # roofline: the counted part with the largest share of the step
    top = max(counted, key=mean.get)
    ach = wl.part_bytes(top) / (mean[top] / 1e3) / 1e9
    work = [wl.part_work(p) for p in counted]
    n_tf, n_fl = sum(w[0] for w in work), sum(w[1] for w in work)
    per_part_tps = {p: round(wl.part_work(p)[0] / (mean[p] / 1e3), 1) for p in wl.parts()}
    per_part_gflops = {p: round(wl.part_work(p)[1] / (mean[p] / 1e3) / 1e9, 1) for p in wl.parts()}
    traffic = None
    tp = ROOT / "profiles" / "traffic.json"
    if tp.exists():
        traffic = json.loads(tp.read_text()).get(f"{wl.name}:{top}")
    line = {
        "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config,
        "pct_hbm": 100.0 * value / world / pk["hbm_gbs"],
        "transforms_per_s": n_tf * world / (ms_step / 1e3),
        "gflops_5nlogn": n_fl * world / (ms_step / 1e3) / 1e9,
        "per_part_gbs": per_part,
        "per_part_transforms_per_s": per_part_tps,
        "per_part_gflops_5nlogn": per_part_gflops,
        "roofline": {"bound": "hbm", "achieved": ach, "peak": pk["hbm_gbs"], "unit": "GB/s",
                     "frac": ach / pk["hbm_gbs"], "traffic": traffic, "peak_src": pk["src"],
                     "kernel": f"{wl.name}:{top}", "algorithmic_bytes": wl.part_bytes(top)},
        "clocks": res["clocks"], "e2e": res["e2e"], "gpu_launches": wl.launches() * args.steps,
    }
    if hasattr(wl, "accuracy"):
        line["accuracy_vs_fp64"] = wl.accuracy()
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = wl.cpu_reference()
    print(json.dumps(line))


if __name__ == "__main__":
    main()

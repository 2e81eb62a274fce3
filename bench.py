"""Benchmark of the fused-chunk path: chunk GB/s against the measured HBM peak.

Workload ("large fused chunks", float32, n = 2^28 per array, seeded synthetic data):
x ~ N(0,1), y ~ U[0.1, 10), z ~ U[-1, 1) with NaN injected at rate 1e-6. One step runs the six
operations a libsci user writes for it, each one kernel launch through the C ABI:

    stored = root(absolute(x)) * logarithm(y) + tanh(z)     16 B/element
    lower  = minimum(x, z)                                  12 B/element
    upper  = maximum(x, z)                                  12 B/element
    mean(exponential(-x * x))                                4 B/element
    maximum(sin(x) * cos(z))                                 8 B/element
    dot(x, z)                                                8 B/element

`value` = algorithmic bytes of a step (60 B/element) / device time of a step (CUDA events on the
library's stream, max over ranks). Inputs are 1 GiB each, far larger than the 126 MB L2, so no
flush is needed between steps. `e2e` runs the same step through the C ABI from pinned host buffers:
the three inputs are uploaded and the three stored outputs and three reductions downloaded inside
the timed region, the step streamed in pieces through the copy lanes so that uploads, kernels and
downloads overlap. `roofline` is the dominant kernel's achieved GB/s over the measured copy peak.
`cpu_baseline` times libsci's own CPU path (oracle/_ref/libsci_ref.so, all host cores) on a
2^24-element sample of the same workload.

`--impl reference` times only that CPU path (the reference arm), on rank 0.
With N > 1 GPUs (torchrun), every rank runs its own 2^28-element shard (weak scaling) and the
three reductions are combined across ranks each step (libsci_b200/shards.py: four small NCCL
all-reduces that keep the rule that a NaN on any rank wins).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

BYTES_PER_ELEMENT = {"stored": 16, "lower": 12, "upper": 12, "mean": 4, "peak": 8, "dot": 8}
STEP_BYTES_PER_ELEMENT = sum(BYTES_PER_ELEMENT.values())
METRIC = "chunk GB/s vs HBM peak"


def generate(count: int, seed: int = 0):
    """Seeded inputs of the large fused chunks: x ~ N(0,1), y ~ U[0.1,10), z ~ U[-1,1), NaN at 1e-6."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(count, dtype=np.float32)
    y = rng.uniform(0.1, 10.0, count).astype(np.float32)
    z = rng.uniform(-1.0, 1.0, count).astype(np.float32)
    holes = rng.choice(count, size=max(1, int(round(count * 1e-6))), replace=False)
    z[holes] = np.nan
    return x, y, z


def measured_traffic(section: str, step: str, elements: int):
    """DRAM bytes of one launch of `step` from the committed ncu figures (profiles/traffic.json,
    bytes per element of one capture, scaled to `elements`), or None."""
    path = ROOT / "profiles" / "traffic.json"
    if not path.exists():
        return None
    entry = json.loads(path.read_text()).get(section, {}).get(step)
    return entry["bytes_per_element"] * elements if entry else None


def measured_tensor_peak(sustained: bool = True):
    """The measured dense bf16 tensor peak in TFLOP/s (sustained for kernels inside a long step,
    burst for one timed alone) and where it came from."""
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        data = json.loads(path.read_text())
        key = "bf16_tflops_sustained" if sustained and "bf16_tflops_sustained" in data else "bf16_tflops"
        return float(data[key]), f"measured {key}"
    return (1400.0 if sustained else 1590.0), "fallback"


def measured_peaks():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        data = json.loads(path.read_text())
        return float(data["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """Samples SM clocks and throttle reasons through NVML while the timed region runs."""

    REASONS = {
        0x0000000000000008: "hw_slowdown",
        0x0000000000000040: "hw_thermal_slowdown",
        0x0000000000000020: "sw_thermal_slowdown",
        0x0000000000000004: "sw_power_cap",
        0x0000000000000080: "hw_power_brake_slowdown",
    }

    def __init__(self, index: int):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        try:
            import pynvml

            pynvml.nvmlInit()
            self.nvml = pynvml
            self.handle = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM)
        except Exception:  # NVML missing: clocks are reported as unknown
            self.nvml = None
        self.thread = threading.Thread(target=self._run, daemon=True)

    def _sample(self) -> bool:
        try:
            self.samples.append(self.nvml.nvmlDeviceGetClockInfo(self.handle, self.nvml.NVML_CLOCK_SM))
            mask = self.nvml.nvmlDeviceGetCurrentClocksEventReasons(self.handle)
        except Exception:
            return False
        for bit, name in self.REASONS.items():
            if mask & bit:
                self.reasons.add(name)
        return True

    def _run(self):
        # a fixed 5 ms period measured from the start, so a thread starved of the GIL for a while
        # resumes on the next tick instead of drifting
        start = time.perf_counter()
        tick = 1
        while not self._stop.wait(max(0.0, start + 0.005 * tick - time.perf_counter())):
            if not self._sample():
                break
            tick += 1

    def __enter__(self):
        if self.nvml:
            self._sample()  # one sample as the region starts, whatever the thread manages
            self.thread.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self.nvml:
            self.thread.join()

    def summary(self):
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def cpu_reference_sample(count: int, repeats: int):
    """libsci's own CPU path (oracle/_ref) on `count` elements: seconds per step, threads used."""
    from tests import _oracle

    lib = _oracle.reference()
    if lib is None:
        return None
    x, y, z = generate(count, seed=1)
    handle = lib.sci_ref_workload_create(x.ctypes.data, y.ctypes.data, z.ctypes.data, count)
    results = np.zeros(3, np.float64)
    lib.sci_ref_workload_step(handle, results.ctypes.data)  # warm-up (page faults, pool start)
    times = []
    for _ in range(repeats):
        start = time.perf_counter()
        lib.sci_ref_workload_step(handle, results.ctypes.data)
        times.append(time.perf_counter() - start)
    lib.sci_ref_workload_destroy(handle)
    return {"seconds": statistics.median(times), "threads": int(lib.sci_ref_threads()), "count": count,
            "times": times}


def run_reference_arm(args, rank: int) -> int:
    if rank != 0:
        return 0
    sample = 1 << 24
    from tests import _oracle

    lib = _oracle.reference()
    if lib is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libsci_ref.so was not built"}))
        return 0
    x, y, z = generate(sample, seed=1)
    handle = lib.sci_ref_workload_create(x.ctypes.data, y.ctypes.data, z.ctypes.data, sample)
    results = np.zeros(3, np.float64)
    for _ in range(args.warmup):
        lib.sci_ref_workload_step(handle, results.ctypes.data)
    start = time.perf_counter()
    for _ in range(args.steps):
        lib.sci_ref_workload_step(handle, results.ctypes.data)
    elapsed = time.perf_counter() - start
    lib.sci_ref_workload_destroy(handle)
    per_step = elapsed / args.steps
    value = STEP_BYTES_PER_ELEMENT * sample / per_step / 1e9
    threads = int(lib.sci_ref_threads())
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_step * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "large fused chunks (float32), libsci CPU path on a 2^24-element sample",
                   "elements": sample, "bytes_per_element": STEP_BYTES_PER_ELEMENT},
        "cpu_baseline": {"value": value, "unit": "GB/s", "cores": threads, "kind": "reference",
                         "sample": f"{sample} elements per step (2^24 of the 2^28 workload), libsci public API"},
        "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def run_plain(args, steps: int | None = None) -> dict:
    """The plain fused expression, float32, n = 2^20 per array: a = linspace(0, 1, n), b ~ U[-1, 1)
    (seed 0), c = ones; each step stores t = a*b + c*2.0f and e = exponential(t)*0.5f and reduces
    s = sum(sin(t)): three C-ABI calls, 28 B/element of algorithmic traffic (29.4 MB), so the cost
    is per-call latency, not HBM. Device-timed steps (inputs resident), an end-to-end step through
    the C ABI (b uploaded from pinned host memory, a and c made on the device with the creation
    entry points, t, e and s downloaded), the outputs checked against the oracle, and libsci's CPU
    path on the same workload (oracle/_ref, all host threads)."""
    import torch

    from libsci_b200 import chunk as C
    from libsci_b200.device import Device
    from libsci_b200.native import check, lib
    from tests import _oracle

    n = 1 << 20
    steps = steps or args.steps
    device = Device(0)
    stream = torch.cuda.ExternalStream(device.stream)
    b = np.random.default_rng(0).uniform(-1, 1, n).astype(np.float32)
    da, dc = device.linspace(0.0, 1.0, n), device.ones(n)
    db = device.array(b)
    dt, de = device.empty(n), device.empty(n)
    s_out = torch.zeros(1, dtype=torch.float64, device="cuda")
    t_chunk = C.record_output(da * db + dc * 2.0)
    e_chunk = C.record_output(C.unary("exponential", dt.expression()) * 0.5)
    s_chunk = C.record_reduce(C.unary("sin", dt.expression()))

    def step():
        device.execute(t_chunk, dt.pointer, n)
        device.execute(e_chunk, de.pointer, n)
        device.reduce_async(s_chunk, C.SUM, n, s_out.data_ptr())

    for _ in range(max(3, args.warmup)):
        step()
    device.jit_wait()
    step()
    device.synchronize()
    with ClockSampler(0) as clocks:
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(steps):
            step()
        stop.record(stream)
        stop.synchronize()
    ms = start.elapsed_time(stop) / steps
    bytes_per_step = 28.0 * n

    # end to end: b up, a and c made on the device, t, e and s down, every step
    hb = torch.from_numpy(b).pin_memory()
    ht, he = torch.empty(n, dtype=torch.float32).pin_memory(), torch.empty(n, dtype=torch.float32).pin_memory()
    hs = torch.zeros(1, dtype=torch.float64).pin_memory()

    def e2e_step():
        check(lib.sci_cuda_upload(device.handle, db.pointer, hb.data_ptr(), 4 * n), device.handle)
        check(lib.sci_cuda_linspace(device.handle, 0, da.pointer, n, 0.0, 1.0), device.handle)
        check(lib.sci_cuda_fill(device.handle, 0, dc.pointer, n, 1.0), device.handle)
        step()
        check(lib.sci_cuda_download(device.handle, ht.data_ptr(), dt.pointer, 4 * n), device.handle)
        check(lib.sci_cuda_download(device.handle, he.data_ptr(), de.pointer, 4 * n), device.handle)
        check(lib.sci_cuda_download(device.handle, hs.data_ptr(), s_out.data_ptr(), 8), device.handle)

    for _ in range(3):
        e2e_step()
    device.synchronize()
    e_start, e_stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    for _ in range(steps):
        e2e_step()
    e_stop.record(stream)
    e_stop.synchronize()
    e2e_ms = e_start.elapsed_time(e_stop) / steps

    # check: t and e bit for bit against the oracle, s within 1e-9 of its FP64 fold
    oracle = _oracle.port()
    a_host = da.numpy()
    hosts = {da.pointer: a_host, db.pointer: b, dc.pointer: np.ones(n, np.float32)}
    t_want = _oracle.execute(oracle, _oracle.on_host(t_chunk, hosts), n, np.float32)
    e_want = _oracle.execute(oracle, _oracle.on_host(e_chunk, {dt.pointer: t_want}), n, np.float32)
    s_want = _oracle.reduce(oracle, _oracle.on_host(s_chunk, {dt.pointer: t_want}), C.SUM, n)
    mismatches = int(_oracle.mismatches(ht.numpy(), t_want).size + _oracle.mismatches(he.numpy(), e_want).size)
    s_error = abs(float(hs[0]) - s_want) / abs(s_want)

    cpu = None
    ref = _oracle.reference()
    if ref is not None and not args.no_cpu:
        handle = ref.sci_ref_plain_create(b.ctypes.data, np.ones(n, np.float32).ctypes.data, n)
        for _ in range(3):
            ref.sci_ref_plain_step(handle)
        started = time.perf_counter()
        for _ in range(20):
            ref.sci_ref_plain_step(handle)
        seconds = (time.perf_counter() - started) / 20
        ref.sci_ref_plain_destroy(handle)
        cpu = {"value": bytes_per_step / seconds / 1e9, "unit": "GB/s", "cores": int(ref.sci_ref_threads()),
               "kind": "reference", "ms_per_step": seconds * 1e3,
               "sample": "the whole workload (2^20 elements), 20 steps after 3 warm-ups, libsci public API"}
    peak, peak_source = measured_peaks()
    value = bytes_per_step / (ms * 1e-3) / 1e9
    line = {"metric": "plain fused expression GB/s (t, e stored; sum(sin t))", "value": value, "unit": "GB/s",
            "n_gpus": 1, "steps": steps, "warmup": max(3, args.warmup), "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "plain fused expression, float32, n=2^20: t=a*b+c*2, e=exp(t)*0.5, s=sum(sin(t))",
                       "elements": n, "bytes_per_element": 28,
                       "l2": "29 MB per step fits in L2: latency-bound, no flush (the bound is per-call cost)"},
            "us_per_call": ms * 1e3 / 3,
            "check": {"t_e_mismatches_vs_oracle": mismatches, "s_rel_error_vs_fp64_fold": s_error},
            "roofline": {"bound": "launch latency", "achieved": value, "peak": peak, "unit": "GB/s",
                         "frac": value / peak, "traffic": None, "peak_source": f"{peak_source} hbm_gbs",
                         "note": "29 MB of traffic takes 4.5 us at the HBM peak; three launches cost more"},
            "e2e": {"value": bytes_per_step / (e2e_ms * 1e-3) / 1e9, "unit": "GB/s", "ms_per_step": e2e_ms,
                    "h2d_bytes_per_step": 4 * n, "d2h_bytes_per_step": 8 * n + 8},
            "cpu_baseline": cpu, "gpu_launches": 3 * steps, "clocks": clocks.summary()}
    device.close()
    return line


def run_product(args) -> dict:
    """linear::product at M = N = K (default 8192), float32 inputs ~ U[-1,1): every mode timed on the
    device (conversion to bf16 included), error against FP64 rows, reference CPU multiply sampled."""
    import torch

    from libsci_b200.device import Device
    from tests import _oracle

    size = args.size
    device = Device(0)
    stream = torch.cuda.ExternalStream(device.stream)
    rng = np.random.default_rng(0)
    a = rng.uniform(-1, 1, (size, size)).astype(np.float32)
    b = rng.uniform(-1, 1, (size, size)).astype(np.float32)
    da, db, dc = device.array(a.ravel()), device.array(b.ravel()), device.empty(size * size)
    flops = 2.0 * size ** 3
    peak = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["bf16_tflops"] if (ROOT / "MEASURED_PEAKS.json").exists() else 1590.0
    oracle = _oracle.port()
    sample_rows = np.sort(rng.choice(size, 64, replace=False))
    want = np.zeros((len(sample_rows), size))
    for i, r in enumerate(sample_rows):
        oracle.sci_oracle_product_rows(a.ctypes.data, b.ctypes.data, want[i].ctypes.data, size, size, size, int(r), int(r) + 1)
    modes = {}
    # |C - C64| <= (u_mode + k 2^-22) (|A| |B|) per element (tests/test_product_gpu.py)
    scale = np.abs(a[sample_rows].astype(np.float64)) @ np.abs(b.astype(np.float64))
    unit = {0: 2.0 ** -7, 1: 2.0 ** -14, 3: 2.0 ** -21, 2: 0.0}
    with ClockSampler(0) as clocks:
        for mode, name in ((0, "bf16"), (1, "split_bf16"), (3, "split3_bf16"), (2, "fp32")):
            for _ in range(args.warmup):
                device.product(da, db, size, size, size, mode=mode, out=dc)
            device.synchronize()
            start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            steps = args.steps if mode != 2 else max(1, args.steps // 4)
            start.record(stream)
            for _ in range(steps):
                device.product(da, db, size, size, size, mode=mode, out=dc)
            stop.record(stream)
            stop.synchronize()
            ms = start.elapsed_time(stop) / steps
            got = dc.numpy().reshape(size, size)[sample_rows]
            err = np.abs(got - want)
            bound = (unit[mode] + (2.0 ** -23 if mode == 2 else 2.0 ** -22) * size) * scale
            modes[name] = {"ms": ms, "TFLOP/s": flops / (ms * 1e-3) / 1e12,
                           "frac_of_bf16_peak": flops / (ms * 1e-3) / 1e12 / peak,
                           "tensor_TFLOP/s": {0: 1, 1: 3, 3: 6}.get(mode, 0) * flops / (ms * 1e-3) / 1e12 if mode != 2 else None,
                           "max_abs_err": float(err.max()), "rel_fro_err": float(np.linalg.norm(err) / np.linalg.norm(want)),
                           "within_bound": bool(np.all(err <= bound))}
    cpu = None
    ref = _oracle.reference()
    if ref is not None and not args.no_cpu:
        n = 2048
        x = rng.uniform(-1, 1, (n, n)).astype(np.float32)
        y = rng.uniform(-1, 1, (n, n)).astype(np.float32)
        z = np.empty((n, n), np.float32)
        t0 = time.perf_counter()
        ref.sci_ref_product(0, x.ctypes.data, y.ctypes.data, z.ctypes.data, n, n, n)
        seconds = time.perf_counter() - t0
        cpu = {"value": 2.0 * n ** 3 / seconds / 1e12, "unit": "TFLOP/s", "cores": int(ref.sci_ref_threads()),
               "kind": "reference", "sample": "libsci multiply (dispatch.cpp:171-224) at 2048^3, fp32, timed once"}
    best = modes["bf16"]
    line = {"metric": "product TFLOP/s", "value": best["TFLOP/s"], "unit": "TFLOP/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": best["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16 (fp32 accumulate)", "data": "synthetic",
            "config": {"workload": f"product M=N=K={size}, float32 ~ U[-1,1)", "modes": list(modes)},
            "modes": modes,
            "roofline": {"bound": "tensor", "achieved": best["TFLOP/s"], "peak": peak, "unit": "TFLOP/s",
                         "frac": best["TFLOP/s"] / peak, "traffic": None, "peak_source": "measured bf16_tflops (burst)"},
            "check": {name: {"within_bound": m["within_bound"], "rel_fro_err": m["rel_fro_err"]} for name, m in modes.items()},
            "cpu_baseline": cpu, "gpu_launches": 3 * args.steps,  # per bf16 product: two conversions + one GEMM
            "clocks": clocks.summary()}
    device.close()
    return line


def torch_solve(torch, a, b, args):
    """An external sanity point, not a product path: torch.linalg.solve in FP64 on the same GPU
    (cuSOLVER getrf + getrs), timed with events, with its normwise backward error."""
    ta, tb = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    for _ in range(args.warmup):
        torch.linalg.solve(ta, tb)
    torch.cuda.synchronize()
    times = []
    for _ in range(args.steps):
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        x = torch.linalg.solve(ta, tb)
        stop.record()
        stop.synchronize()
        times.append(start.elapsed_time(stop))
    x = x.cpu().numpy()
    r = np.abs(b - a @ x).max(axis=0)
    berr = r / (np.abs(a).sum(axis=1).max() * np.abs(x).max(axis=0) + np.abs(b).max(axis=0))
    del ta, tb
    torch.cuda.empty_cache()
    return {"ms": statistics.median(times), "backward_error": float(berr.max())}


def run_solve(args) -> dict:
    """linear::solve at n = 8192 with 16 right-hand sides ~ N(0,1), for A = G + n I and A = G
    (G ~ N(0,1)): FP32 LU + FP64 refinement against plain FP64 LU on the same GPU, both to a
    normwise backward error <= 1e-14; libsci's CPU solve<double> timed once on a 2048 sample."""
    import torch

    from libsci_b200.device import Device
    from tests import _oracle

    n, width = args.size, 16
    device = Device(0)
    stream = torch.cuda.ExternalStream(device.stream)
    flops = 2.0 / 3.0 * n ** 3 + 2.0 * n * n * width
    cases = {}
    clocks = ClockSampler(0)
    clocks.__enter__()
    for name, shift in (("G+nI", True), ("G", False)):
        rng = np.random.default_rng(17 + int(shift))
        a = rng.standard_normal((n, n)) + (n * np.eye(n) if shift else 0.0)
        b = rng.standard_normal((n, width))
        da, db, dx = device.array(a.ravel()), device.array(b.ravel()), device.empty(n * width, np.float64)
        result = {}
        for label, refine in (("fp32_lu_fp64_refine", True), ("fp64_lu", False)):
            for _ in range(args.warmup):  # workspaces, module loads
                device.solve(da, db, n, width, refine=refine, out=dx)
            times, berr, iterations = [], None, None
            for _ in range(args.steps):
                start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                start.record(stream)
                _, berr, iterations = device.solve(da, db, n, width, refine=refine, out=dx)
                stop.record(stream)
                stop.synchronize()
                times.append(start.elapsed_time(stop))
            ms = statistics.median(times)
            result[label] = {"ms": ms, "GFLOP/s": flops / (ms * 1e-3) / 1e9, "backward_error": berr,
                             "iterations": iterations}
        result["speedup_refined_vs_fp64"] = result["fp64_lu"]["ms"] / result["fp32_lu_fp64_refine"]["ms"]
        result["check"] = {"backward_error_le_1e-14": bool(result["fp32_lu_fp64_refine"]["backward_error"] <= 1e-14
                                                           and result["fp64_lu"]["backward_error"] <= 1e-14)}
        if not getattr(args, "compact", False):
            result["external_torch_linalg_solve_fp64"] = torch_solve(torch, a, b, args)
        cases[name] = result
        for arr in (da, db, dx):
            arr.free()
    cpu = None
    ref = _oracle.reference()
    if ref is not None and not args.no_cpu:
        m = 2048
        rng = np.random.default_rng(5)
        a = rng.standard_normal((m, m)) + m * np.eye(m)
        b = rng.standard_normal((m, width))
        x = np.empty((m, width))
        t0 = time.perf_counter()
        ref.sci_ref_solve_f64(a.ctypes.data, b.ctypes.data, x.ctypes.data, m, width)
        seconds = time.perf_counter() - t0
        cpu = {"value": (2.0 / 3.0 * m ** 3 + 2.0 * m * m * width) / seconds / 1e9, "unit": "GFLOP/s",
               "cores": int(ref.sci_ref_threads()), "kind": "reference",
               "sample": "libsci solve<double> (factor + substitute) at n=2048, 16 RHS, timed once"}
    clocks.__exit__(None, None, None)
    headline = cases["G+nI"]["fp32_lu_fp64_refine"]
    # The refined solve's work rate against what its arithmetic can reach: the FP32 trailing
    # updates run on the tensor cores as six bf16 products (split3), so the FP32-accurate tensor
    # rate is the measured bf16 peak / 6; the rest (panels, substitutions, FP64 residuals) is
    # latency-bound.
    tensor_peak = measured_tensor_peak()
    achieved = flops / (headline["ms"] * 1e-3) / 1e12
    line = {"metric": "solve speedup vs plain FP64 LU at equal backward error", "value": cases["G+nI"]["speedup_refined_vs_fp64"],
            "unit": "x", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": headline["ms"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 LU + f64 refinement",
            "data": "synthetic", "config": {"workload": f"solve n={n}, 16 RHS ~ N(0,1); A=G+nI and A=G"},
            "cases": cases, "cpu_baseline": cpu,
            "check": {name: case["check"] for name, case in cases.items()},
            "roofline": {"bound": "tensor (split3 trailing update) + latency (panel chain)", "achieved": achieved,
                         "peak": tensor_peak[0] / 6, "unit": "TFLOP/s", "frac": achieved / (tensor_peak[0] / 6),
                         "traffic": None, "peak_source": f"{tensor_peak[1]} / 6 (six bf16 products per FP32-accurate one)",
                         "work": "2/3 n^3 + 2 n^2 nrhs per factor + solve"},
            "clocks": clocks.summary()}
    device.close()
    return line


def run_gradient(args) -> dict:
    """sci::gradient workloads. Chunk: L = sum(exponential(-a*a)*sin(b) + logarithm(1+c*c)), float32,
    n = 2^26 per array, a,b,c ~ N(0,1): the recomputing adjoint against the temporary-storing one,
    each timed on the device (inputs 256 MiB each, above L2), gradients checked against the closed
    form in FP64. Solve: L = sum(solve(A, B)), A = G + 4096 I (4096^2, fp64), B 4096 x 64: the
    adjoint with FP32 LU + FP64 refinement (one factorisation for the forward and the transposed
    solve) against the plain FP64 form, both checked against numpy FP64."""
    import torch

    from libsci_b200 import chunk as C
    from libsci_b200.device import Device
    from libsci_b200.native import check, lib

    n = args.gradient_elements
    device = Device(0)
    stream = torch.cuda.ExternalStream(device.stream)
    rng = np.random.default_rng(0)
    hosts = [rng.standard_normal(n, dtype=np.float32) for _ in range(3)]
    arrays = [device.array(h) for h in hosts]
    grads = [device.empty(n) for _ in range(3)]
    expr = C.unary("exponential", -arrays[0].expression() * arrays[0].expression()) * C.unary("sin", arrays[1].expression()) \
        + C.unary("logarithm", 1 + arrays[2].expression() * arrays[2].expression())
    chunk = C.record_reduce(expr)
    slots = (ctypes.c_void_p * 3)(*[g.pointer for g in grads])
    peak, peak_source = measured_peaks()

    def time_form(form):
        for _ in range(args.warmup):
            check(lib.sci_cuda_gradient(device.handle, ctypes.byref(chunk), n, 1.0, slots, None, form), device.handle)
        device.jit_wait()
        check(lib.sci_cuda_gradient(device.handle, ctypes.byref(chunk), n, 1.0, slots, None, form), device.handle)
        device.synchronize()
        times = []
        for _ in range(args.steps):
            start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record(stream)
            check(lib.sci_cuda_gradient(device.handle, ctypes.byref(chunk), n, 1.0, slots, None, form), device.handle)
            stop.record(stream)
            stop.synchronize()
            times.append(start.elapsed_time(stop))
        return statistics.median(times)

    with ClockSampler(0) as clocks:
        ms_recompute = time_form(0)
        ms_stored = time_form(1)
    value = ctypes.c_double()
    check(lib.sci_cuda_gradient(device.handle, ctypes.byref(chunk), n, 1.0, slots, ctypes.byref(value), 0), device.handle)
    got = [g.numpy().astype(np.float64) for g in grads]
    a64, b64, c64 = (h.astype(np.float64) for h in hosts)
    e = np.exp(-a64 * a64)
    want = [-2.0 * a64 * e * np.sin(b64), e * np.cos(b64), 2.0 * c64 / (1.0 + c64 * c64)]
    errors = []
    for g, w in zip(got, want):
        scale = np.maximum(np.abs(w), 1e-3 * np.abs(w).max())
        errors.append(float((np.abs(g - w) / scale).max()))
    want_value = float(np.sum(e * np.sin(b64) + np.log1p(c64 * c64)))
    bytes_recompute = 24.0 * n  # read a, b, c; write three gradients
    nodes = 8
    bytes_stored = (12.0 + 4 * nodes + 4 * nodes + 12.0 + 12.0) * n  # forward + tape out, tape + inputs in, grads out
    chunk_result = {
        "elements": n,
        "recompute": {"ms": ms_recompute, "GB/s": bytes_recompute / (ms_recompute * 1e-3) / 1e9,
                      "frac_of_peak": bytes_recompute / (ms_recompute * 1e-3) / 1e9 / peak},
        "stored": {"ms": ms_stored, "GB/s_moved": bytes_stored / (ms_stored * 1e-3) / 1e9,
                   "bytes_per_element": bytes_stored / n},
        "speedup_recompute_vs_stored": ms_stored / ms_recompute,
        "max_rel_error_vs_fp64": max(errors),
        "value": value.value, "value_rel_error": abs(value.value - want_value) / abs(want_value),
    }
    for x in arrays + grads:
        x.free()

    # the solve adjoint
    m, width = 4096, 64
    rng = np.random.default_rng(1)
    a = rng.standard_normal((m, m)) + m * np.eye(m)
    b = rng.standard_normal((m, width))
    g = np.ones((m, width))
    da, db, dg = device.array(a.ravel()), device.array(b.ravel()), device.array(g.ravel())
    x_out, dA_out, dB_out = device.empty(m * width, np.float64), device.empty(m * m, np.float64), device.empty(m * width, np.float64)
    from libsci_b200.native import SolveReport

    def solve_adjoint(refine):
        report = SolveReport()
        check(lib.sci_cuda_solve_gradient(device.handle, 1, 1 if refine else 0, da.pointer, db.pointer, dg.pointer,
                                          x_out.pointer, dA_out.pointer, dB_out.pointer, m, width, ctypes.byref(report)),
              device.handle)
        return report

    solve_result = {}
    want_x = np.linalg.solve(a, b)
    want_l = np.linalg.solve(a.T, g)
    want_dA = -want_l @ want_x.T
    for label, refine in (("fp32_lu_fp64_refine", True), ("fp64_plain", False)):
        for _ in range(args.warmup):
            solve_adjoint(refine)
        times = []
        for _ in range(max(3, args.steps // 4)):
            start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record(stream)
            report = solve_adjoint(refine)
            stop.record(stream)
            stop.synchronize()
            times.append(start.elapsed_time(stop))
        dA = dA_out.numpy().reshape(m, m)
        dB = dB_out.numpy().reshape(m, width)
        solve_result[label] = {
            "ms": statistics.median(times), "backward_error": report.backward_error, "iterations": report.iterations,
            "dA_rel_error": float(np.abs(dA - want_dA).max() / np.abs(want_dA).max()),
            "dB_rel_error": float(np.abs(dB - want_l).max() / np.abs(want_l).max()),
        }
    solve_result["speedup_refined_vs_fp64"] = solve_result["fp64_plain"]["ms"] / solve_result["fp32_lu_fp64_refine"]["ms"]

    from tests import _oracle

    cpu = None
    ref = None if args.no_cpu else _oracle.reference()
    if ref is not None:
        # What the reference offers for gradients: central differences through its CPU path, two
        # Precision::wide evaluations of the chunk per input, on a 2^22-element sample.
        sample = 1 << 22
        base = [h[:sample].astype(np.float64) for h in hosts]
        start = time.perf_counter()
        for index in range(3):
            for sign in (1.0, -1.0):
                moved = [x.copy() for x in base]
                moved[index] += sign * 1e-5 * np.maximum(1.0, np.abs(base[index]))
                refs = [C.Reference(x.ctypes.data, sample, np.float64) for x in moved]
                wide = C.record_output(C.unary("exponential", -refs[0] * refs[0]) * C.unary("sin", refs[1])
                                       + C.unary("logarithm", 1 + refs[2] * refs[2]))
                _oracle.execute(ref, wide, sample, np.float64)
        seconds = time.perf_counter() - start
        cpu = {"value": sample / seconds, "unit": "gradient elements/s", "cores": int(ref.sci_ref_threads()),
               "kind": "reference", "sample": "central differences on libsci's CPU path: 6 Precision::wide chunk "
                                              "evaluations over 2^22 elements"}
    line = {"metric": "gradient speedup: recomputing adjoint vs temporary-storing adjoint", "unit": "x",
            "value": chunk_result["speedup_recompute_vs_stored"], "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_recompute, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (adjoints in f64)", "data": "synthetic",
            "config": {"workload": f"gradient of sum(exp(-a*a)*sin(b)+log(1+c*c)), n={n} float32; "
                                   "gradient of sum(solve(A,B)), A=G+4096I 4096^2 fp64, B 4096x64",
                       "l2": "inputs 256 MiB each, above L2"},
            "chunk": chunk_result, "solve": solve_result,
            "roofline": {"bound": "hbm", "achieved": chunk_result["recompute"]["GB/s"], "peak": peak, "unit": "GB/s",
                         "frac": chunk_result["recompute"]["frac_of_peak"], "traffic": None,
                         "peak_source": peak_source},
            "cpu_baseline": cpu, "gpu_launches": args.steps, "clocks": clocks.summary()}
    device.close()
    return line


def batch_chunk(C, precision=0):
    """t = a*b + c stored and tanh(t) reduced in one chunk: fuse(in0, in1, in2) -> T0; copy(T0) ->
    output; tanh(T0) -> T1; result T1."""
    chunk = C.Chunk(precision)
    chunk.arguments, chunk.temporaries, chunk.length = 3, 2, 3
    program = ((C.CODE["fuse"], C.TEMPORARY | 0, (0, 1, 2)),
               (C.CODE["copy"], C.OUTPUT, (C.TEMPORARY | 0, C.NONE, C.NONE)),
               (C.CODE["tanh"], C.TEMPORARY | 1, (C.TEMPORARY | 0, C.NONE, C.NONE)))
    for index, (code, target, sources) in enumerate(program):
        ins = chunk.instructions[index]
        ins.code, ins.target = code, target
        ins.sources[0], ins.sources[1], ins.sources[2] = sources
    chunk.result = C.TEMPORARY | 1
    return chunk


def run_batch(args) -> dict:
    """Batching: 8192 float32 instances of t = a*b + c, r = sum(tanh(t)), lengths log-uniform in
    [256, 2^20] (seeded), a, b, c ~ N(0,1), in one persistent launch replayed from a CUDA graph.
    Beside it: the plain form, a loop of single calls through the C ABI (execute t, reduce
    tanh(t), per item) on the same GPU, and libsci's CPU path on a sample of items."""
    import torch

    from libsci_b200 import chunk as C
    from libsci_b200.device import Device
    from libsci_b200.native import check, lib
    from tests import _oracle

    items = args.items
    rng = np.random.default_rng(0)
    counts = np.exp(rng.uniform(np.log(256), np.log(1 << 20), items)).astype(np.int64)
    offsets = np.concatenate([[0], np.cumsum((counts + 63) // 64 * 64)])
    total = int(offsets[-1])
    elements = int(counts.sum())
    device = Device(0)
    stream = torch.cuda.ExternalStream(device.stream)
    generator = torch.Generator(device="cuda").manual_seed(0)
    inputs = [torch.randn(total, generator=generator, device="cuda", dtype=torch.float32) for _ in range(3)]
    t_out = torch.empty(total, device="cuda", dtype=torch.float32)
    results = torch.zeros(items, device="cuda", dtype=torch.float64)
    pointers = np.array([[x.data_ptr() + 4 * int(o) for x in inputs] for o in offsets[:-1]], np.uint64)
    outputs = np.array([t_out.data_ptr() + 4 * int(o) for o in offsets[:-1]], np.uint64)

    class Results:  # the DeviceArray face of the torch buffer
        pointer = results.data_ptr()

    chunk = batch_chunk(C)
    torch.cuda.synchronize()
    created = time.perf_counter()
    batch = device.batch(chunk, C.SUM, pointers, counts, outputs, Results)
    created = time.perf_counter() - created
    spans, specialized = batch.spans()
    for _ in range(args.warmup):
        batch.launch()
    device.synchronize()
    times = []
    with ClockSampler(0) as clocks:
        for _ in range(args.steps):
            start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record(stream)
            batch.launch()
            stop.record(stream)
            stop.synchronize()
            times.append(start.elapsed_time(stop))
    ms = statistics.median(times)
    bytes_moved = 16.0 * elements  # read a, b, c; write t; r folds from registers
    peak, peak_source = measured_peaks()
    got = results.cpu().numpy()

    # the plain form: one execute and one reduce per item through the C ABI
    single_t = C.Chunk(0)
    single_r = C.Chunk(0)
    for ch, program, result in ((single_t, ((C.CODE["fuse"], C.OUTPUT, (0, 1, 2)),), C.OUTPUT),
                                (single_r, ((C.CODE["tanh"], C.TEMPORARY | 0, (0, C.NONE, C.NONE)),), C.TEMPORARY | 0)):
        ch.length, ch.temporaries = 1, (1 if ch is single_r else 0)
        ch.arguments = 3 if ch is single_t else 1
        ins = ch.instructions[0]
        ins.code, ins.target = program[0][0], program[0][1]
        ins.sources[0], ins.sources[1], ins.sources[2] = program[0][2]
        ch.result = result

    def loop():
        for k in range(items):
            for a in range(3):
                single_t.inputs[a] = int(pointers[k, a])
            check(lib.sci_cuda_execute(device.handle, ctypes.byref(single_t), int(outputs[k]), int(counts[k])), device.handle)
            single_r.inputs[0] = int(outputs[k])
            check(lib.sci_cuda_reduce_async(device.handle, ctypes.byref(single_r), C.SUM, int(counts[k]),
                                            results.data_ptr() + 8 * k), device.handle)

    loop()
    device.jit_wait()
    loop()
    device.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    loop()
    stop.record(stream)
    stop.synchronize()
    loop_ms = start.elapsed_time(stop)
    loop_results = results.cpu().numpy()

    # spot checks against libsci's CPU path on 16 items: t bit for bit, r to 1e-6 of sum |tanh t|
    ref = _oracle.reference()
    checked, t_mismatch, r_error = 0, 0, 0.0
    if ref is not None:
        t_host = t_out.cpu().numpy()
        host = [x.cpu().numpy() for x in inputs]
        for k in rng.choice(items, 16, replace=False):
            o, n = int(offsets[k]), int(counts[k])
            a, b, c = (np.ascontiguousarray(h[o:o + n]) for h in host)
            refs = [C.Reference(x.ctypes.data, n, np.float32) for x in (a, b, c)]
            t = _oracle.execute(ref, C.record_output(refs[0] * refs[1] + refs[2]), n, np.float32)
            values = _oracle.execute(ref, C.record_output(C.unary("tanh", C.Reference(t.ctypes.data, n, np.float32))), n,
                                     np.float32).astype(np.float64)
            t_mismatch += int(_oracle.mismatches(t_host[o:o + n], t).size)
            r_error = max(r_error, abs(got[k] - values.sum()) / np.abs(values).sum())
            checked += 1

    cpu = None
    if ref is not None and not args.no_cpu:
        sample = rng.choice(items, 256, replace=False)
        host = [x.cpu().numpy() for x in inputs]
        start_cpu = time.perf_counter()
        done = 0
        for k in sample:
            o, n = int(offsets[k]), int(counts[k])
            refs = [C.Reference(h[o:o + n].ctypes.data, n, np.float32) for h in host]
            t = _oracle.execute(ref, C.record_output(refs[0] * refs[1] + refs[2]), n, np.float32)
            _oracle.reduce(ref, C.record_reduce(C.unary("tanh", C.Reference(t.ctypes.data, n, np.float32))), C.SUM, n)
            done += n
        seconds = time.perf_counter() - start_cpu
        cpu = {"value": 16.0 * done / seconds / 1e9, "unit": "GB/s", "cores": int(ref.sci_ref_threads()),
               "kind": "reference", "sample": f"{len(sample)} of the {items} items ({done} elements): one assign and "
                                               "one reduce per item on libsci's CPU path"}
    line = {"metric": "batched chunk GB/s (one graph launch over all items)", "value": bytes_moved / (ms * 1e-3) / 1e9,
            "unit": "GB/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{items} instances of t=a*b+c, r=sum(tanh(t)), lengths log-uniform in [256, 2^20]",
                       "elements": elements, "bytes_per_element": 16, "l2": f"{16 * elements / 1e9:.1f} GB of operands, above L2"},
            "batch": {"spans": spans, "specialized": specialized, "create_s": created,
                      "plain_loop_ms": loop_ms, "speedup_vs_plain_loop": loop_ms / ms,
                      "loop_max_rel_diff": float(np.max(np.abs(loop_results - got) / np.maximum(np.abs(got), 1e-30))),
                      "checked_items": checked, "t_mismatches": t_mismatch, "r_rel_error": r_error},
            "roofline": {"bound": "hbm", "achieved": bytes_moved / (ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": bytes_moved / (ms * 1e-3) / 1e9 / peak, "traffic": None, "peak_source": peak_source},
            "cpu_baseline": cpu, "gpu_launches": args.steps, "clocks": clocks.summary()}
    batch.close()
    device.close()
    return line


def run_solves(args) -> dict:
    """Batching of solves: 4096 independent systems, n ~ U[8, 256] (seeded), A = G + n I (G ~ N(0,1)),
    one right-hand side ~ N(0,1), FP32 LU + FP64 refinement, one graph replay (block size tuned per
    order bucket). Beside it: a loop of single sci_cuda_solve calls (the plain form, sampled) and
    libsci's CPU solve<double> per system (sampled)."""
    import torch

    from libsci_b200.device import Device
    from libsci_b200.native import SolveReport, check, lib
    from tests import _oracle

    count = args.items if args.items != 8192 else 4096
    rng = np.random.default_rng(0)
    orders = rng.integers(8, 257, count)
    device = Device(0)
    stream = torch.cuda.ExternalStream(device.stream)
    mats = [rng.standard_normal((n, n)) + n * np.eye(n) for n in orders]
    rhs = [rng.standard_normal(n) for n in orders]
    offsets_a = np.concatenate([[0], np.cumsum(orders * orders)])
    offsets_b = np.concatenate([[0], np.cumsum(orders)])
    flat_a = device.array(np.concatenate([m.ravel() for m in mats]))
    flat_b = device.array(np.concatenate(rhs))
    flat_x = device.empty(int(offsets_b[-1]), np.float64)
    errors = device.empty(count, np.float64)
    iterations = device.empty(count, np.int32)
    pa = [flat_a.pointer + 8 * int(o) for o in offsets_a[:-1]]
    pb = [flat_b.pointer + 8 * int(o) for o in offsets_b[:-1]]
    px = [flat_x.pointer + 8 * int(o) for o in offsets_b[:-1]]
    created = time.perf_counter()
    batch = device.solve_batch(orders, pa, pb, px, errors, iterations)
    created = time.perf_counter() - created
    for _ in range(args.warmup):
        batch.launch()
    device.synchronize()
    times = []
    with ClockSampler(0) as clocks:
        for _ in range(args.steps):
            start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record(stream)
            batch.launch()
            stop.record(stream)
            stop.synchronize()
            times.append(start.elapsed_time(stop))
    ms = statistics.median(times)
    flops = float(np.sum(2.0 / 3.0 * orders.astype(np.float64) ** 3 + 2.0 * orders.astype(np.float64) ** 2))
    berr, its = errors.numpy(), iterations.numpy()
    x = flat_x.numpy()
    sample = rng.choice(count, 64, replace=False)
    mine = max(float(np.abs(rhs[k] - mats[k] @ x[offsets_b[k]:offsets_b[k + 1]]).max()
                     / (np.abs(mats[k]).sum(axis=1).max() * np.abs(x[offsets_b[k]:offsets_b[k + 1]]).max()
                        + np.abs(rhs[k]).max())) for k in sample)

    # the plain form: one sci_cuda_solve (FP32 LU + FP64 refinement) per system, sampled
    loop_sample = rng.choice(count, 128, replace=False)
    report = SolveReport()
    for k in loop_sample[:4]:
        check(lib.sci_cuda_solve(device.handle, 1, 1, pa[k], pb[k], px[k], int(orders[k]), 1, ctypes.byref(report)),
              device.handle)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for k in loop_sample:
        check(lib.sci_cuda_solve(device.handle, 1, 1, pa[k], pb[k], px[k], int(orders[k]), 1, ctypes.byref(report)),
              device.handle)
    stop.record(stream)
    stop.synchronize()
    loop_flops = float(np.sum(2.0 / 3.0 * orders[loop_sample].astype(np.float64) ** 3
                              + 2.0 * orders[loop_sample].astype(np.float64) ** 2))
    loop_gflops = loop_flops / (start.elapsed_time(stop) * 1e-3) / 1e9

    ref = None if args.no_cpu else _oracle.reference()
    cpu = None
    if ref is not None:
        cpu_sample = rng.choice(count, 256, replace=False)
        done = 0.0
        out = np.empty(257)
        started = time.perf_counter()
        for k in cpu_sample:
            n = int(orders[k])
            ref.sci_ref_solve_f64(mats[k].ctypes.data, rhs[k].ctypes.data, out.ctypes.data, n, 1)
            done += 2.0 / 3.0 * n ** 3 + 2.0 * n * n
        seconds = time.perf_counter() - started
        cpu = {"value": done / seconds / 1e9, "unit": "GFLOP/s", "cores": int(ref.sci_ref_threads()), "kind": "reference",
               "sample": "256 of the systems, one solve<double> call each on libsci's CPU path"}
    line = {"metric": "batched small solves GFLOP/s (one graph launch)", "value": flops / (ms * 1e-3) / 1e9,
            "unit": "GFLOP/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 LU + f64 refinement",
            "data": "synthetic",
            "config": {"workload": f"{count} solves, n ~ U[8,256], A = G + nI, 1 RHS", "flop": flops,
                       "matrix_bytes": int(offsets_a[-1]) * 8},
            "solves": {"threads_per_bucket": batch.shapes(), "create_s": created, "max_backward_error": float(np.nanmax(berr)),
                       "mean_iterations": float(its.mean()), "max_backward_error_numpy_sample": mine,
                       "plain_loop_GFLOP/s": loop_gflops,
                       "speedup_vs_plain_loop": (flops / (ms * 1e-3) / 1e9) / loop_gflops},
            "roofline": {"bound": "latency (per-column barriers)", "achieved": flops / (ms * 1e-3) / 1e12,
                         "peak": None, "unit": "TFLOP/s", "frac": None, "traffic": None,
                         "note": "A is read twice (FP32 copy + FP64 residuals from L2): "
                                 f"{2 * int(offsets_a[-1]) * 8 / (ms * 1e-3) / 1e9:.0f} GB/s of HBM for A"},
            "cpu_baseline": cpu, "gpu_launches": 4 * args.steps, "clocks": clocks.summary()}
    batch.close()
    device.close()
    return line


def run_creation(args) -> dict:
    """Arrays made on the device (include/operations/creation.hpp): full, linspace, range and eye of
    2^28 float32 elements (1 GiB each), grid of 16384 x 16384 (two 1 GiB outputs), and transpose
    (manipulations.hpp) of a 16384 x 16384 matrix; one step = all six. Bound by HBM: 4 B/element
    written, 8 for grid and for transpose (read + write). Beside them: the reference's own creation
    functions (libsci's host loops) on a 2^24-element sample."""
    import torch

    from libsci_b200.device import Device
    from libsci_b200.native import check, lib
    from tests import _oracle
    from tests.test_oracle import creation_functions

    count, side = 1 << 28, 1 << 14
    peak, peak_source = measured_peaks()
    device = Device(0)
    stream = torch.cuda.ExternalStream(device.stream)
    out = device.empty(count)
    second = device.empty(count)
    x, y = device.linspace(-1.0, 1.0, side), device.linspace(0.0, 5.0, side)
    extents = (ctypes.c_uint64 * 2)(side, side)
    steps = {
        "full": (lambda: check(lib.sci_cuda_fill(device.handle, 0, out.pointer, count, 2.5), device.handle), 4 * count),
        "linspace": (lambda: check(lib.sci_cuda_linspace(device.handle, 0, out.pointer, count, -3.0, 7.0), device.handle),
                     4 * count),
        "range": (lambda: check(lib.sci_cuda_range(device.handle, 0, out.pointer, count, -1.0, 0.25), device.handle),
                  4 * count),
        "eye": (lambda: check(lib.sci_cuda_eye(device.handle, 0, out.pointer, side, side), device.handle), 4 * count),
        "grid": (lambda: check(lib.sci_cuda_grid(device.handle, 0, x.pointer, side, y.pointer, side, out.pointer,
                                                 second.pointer), device.handle), 8 * count),
        # transpose (manipulations.hpp:33-62) of the 16384 x 16384 grid output: read + write
        "transpose": (lambda: check(lib.sci_cuda_transpose(device.handle, 0, out.pointer, 2, extents, second.pointer),
                                    device.handle), 8 * count),
    }
    for _ in range(args.warmup):
        for launch, _bytes in steps.values():
            launch()
    device.synchronize()
    kernels = {name: [] for name in steps}
    totals = []
    with ClockSampler(0) as clocks:
        for _ in range(args.steps):
            marks = [torch.cuda.Event(enable_timing=True) for _ in range(len(steps) + 1)]
            marks[0].record(stream)
            for index, (launch, _bytes) in enumerate(steps.values()):
                launch()
                marks[index + 1].record(stream)
            marks[-1].synchronize()
            for index, name in enumerate(steps):
                kernels[name].append(marks[index].elapsed_time(marks[index + 1]))
            totals.append(marks[0].elapsed_time(marks[-1]))
    ms = statistics.median(totals)
    moved = sum(b for _launch, b in steps.values())
    per = {name: {"ms": statistics.median(t), "GB/s": steps[name][1] / (statistics.median(t) * 1e-3) / 1e9,
                  "frac": steps[name][1] / (statistics.median(t) * 1e-3) / 1e9 / peak} for name, t in kernels.items()}
    top = max(per, key=lambda name: per[name]["ms"])

    ref = None if args.no_cpu else _oracle.reference()
    cpu = None
    if ref is not None:
        theirs = creation_functions(ref, "sci_ref")
        sample = 1 << 24
        host = np.empty(sample, np.float32)
        started = time.perf_counter()
        theirs["full"](0, host.ctypes.data, sample, 2.5)
        theirs["linspace"](0, host.ctypes.data, sample, -3.0, 7.0)
        theirs["range"](0, host.ctypes.data, sample, -1.0, -1.0 + 0.25 * sample, 0.25)
        theirs["eye"](0, host.ctypes.data, 1 << 12, 1 << 12)
        seconds = time.perf_counter() - started
        cpu = {"value": 4 * 4 * sample / seconds / 1e9, "unit": "GB/s", "cores": 1, "kind": "reference",
               "sample": "2^24 elements of full, linspace, range and eye each through libsci's own creation "
                         "functions (host loops, one thread)"}
    line = {"metric": "device creation GB/s written vs HBM peak", "value": moved / (ms * 1e-3) / 1e9, "unit": "GB/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "full, linspace, range, eye of 2^28 floats; grid and transpose 16384 x 16384",
                       "bytes_written": moved, "l2": "each output 1 GiB, above L2"},
            "kernels": per,
            "roofline": {"bound": "hbm", "achieved": per[top]["GB/s"], "peak": peak, "unit": "GB/s",
                         "frac": per[top]["frac"], "traffic": None, "kernel": top, "peak_source": peak_source},
            "cpu_baseline": cpu, "gpu_launches": len(steps) * args.steps, "clocks": clocks.summary()}
    device.close()
    return line


def run_elements(args) -> dict:
    """Integer-element chunks (sci_cuda_execute_elements / reduce_elements), the expressions libsci
    evaluates on the host for non-native element types (include/array/expression.hpp:178-184,
    203-220): int32 t = a*b + c, maximum(a, c) / b and sum(a*b) over 2^28 elements (1 GiB per
    array), int8 t = a*b + c over 2^30 and int64 t = a*b + c over 2^27 (1 GiB per array each); one
    step = all five. HBM-bound: bytes = inputs read + output written per element. Beside them: the
    reference's own host loop (array::calculate) for int32 a*b + c on a 2^24-element sample."""
    import torch

    from libsci_b200 import chunk as C
    from libsci_b200.device import Device
    from tests import _oracle

    peak, peak_source = measured_peaks()
    device = Device(0)
    stream = torch.cuda.ExternalStream(device.stream)

    def operands(dtype, count):
        # a 2^24-element hashed pattern per operand (no zeros, so b is a divisor), uploaded slice by
        # slice into 1 GiB device arrays
        piece = 1 << 24
        index = np.arange(piece, dtype=np.uint64)
        made = []
        for salt in (0x9E3779B97F4A7C15, 0xC2B2AE3D27D4EB4F, 0x165667B19E3779F9):
            values = ((index * np.uint64(salt)) >> np.uint64(40)).astype(dtype)
            values[values == 0] = 1
            array = device.empty(count, dtype)
            for start in range(0, count, piece):
                array.offset(start, piece).upload(values)
            made.append(array)
        return made

    steps, counts = {}, {}
    shrink = 2 if args.small else 0  # --small: a quarter of each size, for profiler captures
    for dtype, count in ((np.int32, 1 << (28 - shrink)), (np.int8, 1 << (30 - shrink)), (np.int64, 1 << (27 - shrink))):
        a, b, c = operands(dtype, count)
        out = device.empty(count, dtype)
        size = np.dtype(dtype).itemsize
        x, y, z = a.expression(), b.expression(), c.expression()
        name = np.dtype(dtype).name
        fused = C.record_output(x * y + z)
        counts.update({f"{name} a*b+c": count, f"{name} maximum(a,c)/b": count, f"{name} sum(a*b)": count})
        steps[f"{name} a*b+c"] = (lambda ch=fused, o=out, n=count, d=dtype: device.execute_elements(d, ch, o.pointer, n),
                                  4 * size * count)
        if dtype == np.int32:
            divided = C.record_output(C.binary("maximum", x, z) / y)
            steps[f"{name} maximum(a,c)/b"] = (
                lambda ch=divided, o=out, n=count, d=dtype: device.execute_elements(d, ch, o.pointer, n), 4 * size * count)
            summed = C.record_reduce(x * y)
            steps[f"{name} sum(a*b)"] = (lambda ch=summed, n=count, d=dtype: device.reduce_elements(d, ch, C.SUM, n),
                                         2 * size * count)
    for _ in range(args.warmup):
        for launch, _bytes in steps.values():
            launch()
    device.synchronize()
    kernels = {name: [] for name in steps}
    totals = []
    with ClockSampler(0) as clocks:
        for _ in range(args.steps):
            marks = [torch.cuda.Event(enable_timing=True) for _ in range(len(steps) + 1)]
            marks[0].record(stream)
            for index, (launch, _bytes) in enumerate(steps.values()):
                launch()
                marks[index + 1].record(stream)
            marks[-1].synchronize()
            for index, name in enumerate(steps):
                kernels[name].append(marks[index].elapsed_time(marks[index + 1]))
            totals.append(marks[0].elapsed_time(marks[-1]))
    ms = statistics.median(totals)
    moved = sum(b for _launch, b in steps.values())
    per = {name: {"ms": statistics.median(t), "GB/s": steps[name][1] / (statistics.median(t) * 1e-3) / 1e9,
                  "frac": steps[name][1] / (statistics.median(t) * 1e-3) / 1e9 / peak} for name, t in kernels.items()}
    top = max(per, key=lambda name: per[name]["ms"])
    top_elements = {name: n for name, n in counts.items()}[top]

    ref = None if args.no_cpu else _oracle.reference()
    cpu = None
    if ref is not None:
        sample = 1 << 24
        rng = np.random.default_rng(1)
        host = [rng.integers(-1000, 1000, sample, dtype=np.int32) for _ in range(3)]
        result = np.empty(sample, np.int32)
        started = time.perf_counter()
        ref.sci_ref_elements(0, C.ELEMENT[np.dtype(np.int32)], host[0].ctypes.data, host[1].ctypes.data,
                             host[2].ctypes.data, sample, result.ctypes.data)
        seconds = time.perf_counter() - started
        cpu = {"value": 16 * sample / seconds / 1e9, "unit": "GB/s", "cores": 1, "kind": "reference",
               "sample": "int32 a*b + c over 2^24 elements through libsci's own assign() host loop "
                         "(array::calculate, one thread)"}
    line = {"metric": "integer-element chunk GB/s vs HBM peak", "value": moved / (ms * 1e-3) / 1e9, "unit": "GB/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int8/int32/int64", "data": "synthetic",
            "config": {"workload": f"int32 a*b+c, maximum(a,c)/b, sum(a*b) over 2^{28 - shrink}; int8 a*b+c over "
                                   f"2^{30 - shrink}; int64 a*b+c over 2^{27 - shrink}", "bytes": moved,
                       "l2": "every array above L2"},
            "kernels": per,
            "roofline": {"bound": "hbm", "achieved": per[top]["GB/s"], "peak": peak, "unit": "GB/s",
                         "frac": per[top]["frac"], "traffic": measured_traffic("elements", top, top_elements),
                         "kernel": f"element_stream ({top})", "peak_source": peak_source},
            "cpu_baseline": cpu, "gpu_launches": (len(steps) + 1) * args.steps, "clocks": clocks.summary()}
    device.close()
    return line


def run_shapes(args) -> dict:
    """Broadcasting, the roadmap's elementwise functions and axis reductions (libsci's README.md:
    149-152, numpy's rules): over 16384 x 16384 float32 (1 GiB per full array), one step =
    (16384,1) + (1,16384); where((16384,1), x, y); clip(x, -1, 1); power(x, 2.5); floor(x); sum of
    x over axis 0 and over axis 1. HBM-bound: bytes = full operands read + output written (a
    broadcast operand is 64 KiB). Beside them: numpy on the host (one thread) on a 2048 x 16384
    sample of the same steps."""
    import torch

    from libsci_b200 import chunk as C
    from libsci_b200.device import Device
    from libsci_b200.native import check, lib

    side = 1 << (13 if args.small else 14)
    count = side * side
    peak, peak_source = measured_peaks()
    device = Device(0)
    stream = torch.cuda.ExternalStream(device.stream)
    full = (side, side)
    x = device.range(-2.0, -2.0 + count * (4.0 / count), 4.0 / count)
    y = device.full(count, 0.5)
    column = device.linspace(-1.0, 1.0, side)
    row = device.linspace(0.0, 3.0, side)
    out = device.empty(count)
    reduced = device.empty(side)
    scalars = {v: device.full(1, v) for v in (-1.0, 1.0, 2.5)}

    def apply(code, operands):
        # straight through the C ABI into a preallocated output: nothing allocates in the timed region
        number = C.EXTRA[code] if code in C.EXTRA else C.CODE[code]
        inputs = (ctypes.c_void_p * len(operands))(*[array.pointer for array, _ in operands])
        extents = (ctypes.c_uint64 * (2 * len(operands)))(*[e for _, shape in operands for e in shape])
        check(lib.sci_cuda_broadcast(device.handle, 0, number, 2, (ctypes.c_uint64 * 2)(*full), len(operands), inputs,
                                     extents, out.pointer), device.handle)

    def axis_sum(axis):
        check(lib.sci_cuda_reduce_axis(device.handle, 0, C.SUM, x.pointer, 2, (ctypes.c_uint64 * 2)(*full), axis,
                                       reduced.pointer), device.handle)

    one = (1, 1)
    steps = {
        "broadcast add (16384,1)+(1,16384)": (lambda: apply("add", [(column, (side, 1)), (row, (1, side))]), 4 * count),
        "where((16384,1), x, y)": (lambda: apply("where", [(column, (side, 1)), (x, full), (y, full)]), 12 * count),
        "clip(x, -1, 1)": (lambda: apply("clip", [(x, full), (scalars[-1.0], one), (scalars[1.0], one)]), 8 * count),
        "power(x, 2.5)": (lambda: apply("power", [(x, full), (scalars[2.5], one)]), 8 * count),
        "floor(x)": (lambda: apply("floor", [(x, full)]), 8 * count),
        "sum(x, axis=0)": (lambda: axis_sum(0), 4 * count),
        "sum(x, axis=1)": (lambda: axis_sum(1), 4 * count),
    }

    for _ in range(args.warmup):
        for launch, _bytes in steps.values():
            launch()
    device.synchronize()
    kernels = {name: [] for name in steps}
    totals = []
    with ClockSampler(0) as clocks:
        for _ in range(args.steps):
            marks = [torch.cuda.Event(enable_timing=True) for _ in range(len(steps) + 1)]
            marks[0].record(stream)
            for index, (launch, _bytes) in enumerate(steps.values()):
                launch()
                marks[index + 1].record(stream)
            marks[-1].synchronize()
            for index, name in enumerate(steps):
                kernels[name].append(marks[index].elapsed_time(marks[index + 1]))
            totals.append(marks[0].elapsed_time(marks[-1]))
    ms = statistics.median(totals)
    moved = sum(b for _launch, b in steps.values())
    per = {name: {"ms": statistics.median(t), "GB/s": steps[name][1] / (statistics.median(t) * 1e-3) / 1e9,
                  "frac": steps[name][1] / (statistics.median(t) * 1e-3) / 1e9 / peak} for name, t in kernels.items()}
    # power spends its time in the FP64 pipe (a double pow per element): the roofline names the
    # slowest HBM-bound step, power is reported beside it
    top = max((name for name in per if not name.startswith("power")), key=lambda name: per[name]["ms"])

    cpu = None
    if not args.no_cpu:
        rows = 2048
        hx = np.linspace(-2.0, 2.0, rows * side, dtype=np.float32).reshape(rows, side)
        hy = np.full((rows, side), 0.5, np.float32)
        hc = np.linspace(-1.0, 1.0, rows, dtype=np.float32).reshape(rows, 1)
        hr = np.linspace(0.0, 3.0, side, dtype=np.float32).reshape(1, side)
        started = time.perf_counter()
        with np.errstate(all="ignore"):
            _ = hc + hr
            _ = np.where(hc != 0, hx, hy)
            _ = np.clip(hx, np.float32(-1), np.float32(1))
            _ = np.power(hx, np.float32(2.5))
            _ = np.floor(hx)
            _ = hx.sum(axis=0, dtype=np.float64)
            _ = hx.sum(axis=1, dtype=np.float64)
        seconds = time.perf_counter() - started
        cpu = {"value": moved * rows / side / seconds / 1e9, "unit": "GB/s", "cores": 1, "kind": "port",
               "sample": "the seven steps over 2048 x 16384 floats in numpy on the host (the rules these "
                         "follow; libsci has no implementation of them)"}
    line = {"metric": "broadcast / roadmap elementwise / axis-reduction GB/s vs HBM peak",
            "value": moved / (ms * 1e-3) / 1e9, "unit": "GB/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{side} x {side} float32: broadcast add, where, clip, power, floor, sum over "
                                   "axis 0 and axis 1", "bytes": moved, "l2": "every full array above L2"},
            "kernels": per,
            "roofline": {"bound": "hbm", "achieved": per[top]["GB/s"], "peak": peak, "unit": "GB/s",
                         "frac": per[top]["frac"], "traffic": measured_traffic("shapes", top, count), "kernel": top,
                         "peak_source": peak_source},
            "fp64_bound": {"step": "power(x, 2.5)", "ms": per["power(x, 2.5)"]["ms"],
                           "note": "a double-precision pow per element; bound by the FP64 pipe, not HBM"},
            "cpu_baseline": cpu, "gpu_launches": 8 * args.steps, "clocks": clocks.summary()}
    device.close()
    return line


def main() -> int:
    parser = argparse.ArgumentParser()
    parser.add_argument("--workload", default="chunks",
                        choices=["chunks", "plain", "product", "solve", "gradient", "batch", "solves", "creation",
                                 "elements", "shapes"])
    parser.add_argument("--size", type=int, default=8192)
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=20)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", default="b200", choices=["b200", "reference"])
    parser.add_argument("--elements", type=int, default=1 << 28)
    parser.add_argument("--e2e-steps", type=int, default=3)
    parser.add_argument("--e2e-pieces", type=int, default=8,
                        help="pieces the end-to-end step streams through the copy lanes")
    parser.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    parser.add_argument("--no-extras", action="store_true",
                        help="default workload only: skip the other workloads' summaries in the line")
    parser.add_argument("--small", action="store_true",
                        help="elements / shapes workloads at a quarter size (for profiler captures)")
    parser.add_argument("--items", type=int, default=8192, help="batch workload: instances")
    parser.add_argument("--gradient-elements", type=int, default=1 << 26, help="gradient workload: elements per array")
    args = parser.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference_arm(args, rank)
    single = {"plain": run_plain, "product": run_product, "solve": run_solve, "gradient": run_gradient,
              "batch": run_batch, "elements": run_elements, "shapes": run_shapes, "creation": run_creation,
              "solves": run_solves}
    if args.workload in single:
        print(json.dumps(single[args.workload](args)))
        return 0

    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from libsci_b200 import chunk as C
    from libsci_b200.device import Device
    from libsci_b200.shards import combine

    n = args.elements
    device = Device(local)
    stream = torch.cuda.ExternalStream(device.stream, device=torch.device("cuda", local))

    x, y, z = generate(n, seed=rank)
    dx, dy, dz = device.array(x), device.array(y), device.array(z)
    stored, lower, upper = device.empty(n), device.empty(n), device.empty(n)
    results = torch.zeros(3, dtype=torch.float64, device=f"cuda:{local}")
    a, b, c = dx.expression(), dy.expression(), dz.expression()
    chunks = {
        "stored": (C.record_output(C.unary("root", C.unary("absolute", a)) * C.unary("logarithm", b) + C.unary("tanh", c)), stored),
        "lower": (C.record_output(C.binary("minimum", a, c)), lower),
        "upper": (C.record_output(C.binary("maximum", a, c)), upper),
        "mean": (C.record_reduce(C.unary("exponential", -a * a)), C.SUM),
        "peak": (C.record_reduce(C.unary("sin", a) * C.unary("cos", c)), C.MAXIMUM),
        "dot": (C.record_reduce(a * c), C.SUM),
    }
    names = list(chunks)

    def launch(name, slot):
        chunk, target = chunks[name]
        if name in ("stored", "lower", "upper"):
            device.execute(chunk, target.pointer, n)
        else:
            device.reduce_async(chunk, target, n, results.data_ptr() + 8 * slot)

    def step(events=None):
        for i, name in enumerate(names):
            if events is not None:
                events[i].record(stream)
            launch(name, max(0, i - 3))
        if events is not None:
            events[len(names)].record(stream)
        if dist is not None:
            with torch.cuda.stream(stream):
                results.copy_(combine(results, (C.SUM, C.MAXIMUM, C.SUM)))  # mean, peak, dot of the whole array

    # warm-up (also lets any specialised kernels compile and load)
    for _ in range(args.warmup):
        step()
    if hasattr(device, "jit_wait"):
        device.jit_wait()
    for _ in range(2):
        step()
    device.synchronize()

    # timed region: K steps, per-launch events on the library's stream
    per_kernel = {name: [] for name in names}
    step_events = [[torch.cuda.Event(enable_timing=True) for _ in range(len(names) + 1)] for _ in range(args.steps)]
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        start.record(stream)
        for k in range(args.steps):
            step(step_events[k])
        stop.record(stream)
        stop.synchronize()
    torch.cuda.synchronize()
    elapsed_ms = start.elapsed_time(stop)
    for k in range(args.steps):
        for i, name in enumerate(names):
            per_kernel[name].append(step_events[k][i].elapsed_time(step_events[k][i + 1]))
    if dist is not None:
        t = torch.tensor([elapsed_ms], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed_ms = float(t.item())
    ms_per_step = elapsed_ms / args.steps
    value = STEP_BYTES_PER_ELEMENT * n * world / (ms_per_step * 1e-3) / 1e9

    # the dominant kernel and its roofline
    mean_ms = {name: statistics.mean(v) for name, v in per_kernel.items()}
    dominant = max(mean_ms, key=mean_ms.get)
    peak_gbs, peak_kind = measured_peaks()
    achieved = BYTES_PER_ELEMENT[dominant] * n / (mean_ms[dominant] * 1e-3) / 1e9
    traffic = None
    traffic_file = ROOT / "profiles" / "traffic.json"
    if traffic_file.exists():
        known = json.loads(traffic_file.read_text())
        entry = known.get(dominant)
        if entry:
            traffic = entry["bytes_per_element"] * n
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak_gbs, "unit": "GB/s", "frac": achieved / peak_gbs,
                "traffic": traffic, "kernel": f"chunk_stream ({dominant})", "peak_source": f"{peak_kind} hbm_gbs",
                "traffic_source": "profiles/traffic.json: ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch "
                                  "at 2^28 elements (this size), scaled to the element count; the output's last ~20 MB "
                                  "are still in L2 when the kernel ends, so writes read slightly under 4 B/element"}
    kernels = {name: {"ms": mean_ms[name], "GB/s": BYTES_PER_ELEMENT[name] * n / (mean_ms[name] * 1e-3) / 1e9,
                      "frac": BYTES_PER_ELEMENT[name] * n / (mean_ms[name] * 1e-3) / 1e9 / peak_gbs}
               for name in names}

    # end to end through the C ABI from pinned host buffers
    hx = torch.from_numpy(x).pin_memory()
    hy = torch.from_numpy(y).pin_memory()
    hz = torch.from_numpy(z).pin_memory()
    outs = [torch.empty(n, dtype=torch.float32).pin_memory() for _ in range(3)]
    host_results = torch.zeros(3, dtype=torch.float64).pin_memory()
    from libsci_b200.native import check, lib

    # The step in pieces through the copy lanes: the upload of piece p+1, the six chunks over piece p
    # and the download of piece p-1 overlap (PCIe carries both directions at once). Each piece's
    # three reductions land in its own slots and are folded into `results` on the main stream.
    pieces = args.e2e_pieces if n % args.e2e_pieces == 0 else 1
    span = n // pieces
    piece_results = torch.zeros(pieces, 3, dtype=torch.float64, device=f"cuda:{local}")
    piece_chunks = []
    for p in range(pieces):
        o = p * span
        pa, pb, pc = (v.offset(o, span).expression() for v in (dx, dy, dz))
        piece_chunks.append([
            (C.record_output(C.unary("root", C.unary("absolute", pa)) * C.unary("logarithm", pb) + C.unary("tanh", pc)),
             stored.pointer + 4 * o),
            (C.record_output(C.binary("minimum", pa, pc)), lower.pointer + 4 * o),
            (C.record_output(C.binary("maximum", pa, pc)), upper.pointer + 4 * o),
            (C.record_reduce(C.unary("exponential", -pa * pa)), C.SUM),
            (C.record_reduce(C.unary("sin", pa) * C.unary("cos", pc)), C.MAXIMUM),
            (C.record_reduce(pa * pc), C.SUM),
        ])

    def e2e_step():
        check(lib.sci_cuda_join(device.handle), device.handle)  # lanes start after the main stream's work
        for p in range(pieces):
            o = p * span
            for host, dev in ((hx, dx), (hy, dy), (hz, dz)):
                check(lib.sci_cuda_upload_lane(device.handle, dev.pointer + 4 * o, host.data_ptr() + 4 * o, 4 * span),
                      device.handle)
            for i, (chunk, target) in enumerate(piece_chunks[p]):
                if i < 3:
                    device.execute(chunk, target, span)
                else:
                    device.reduce_async(chunk, target, span, piece_results.data_ptr() + 8 * (3 * p + i - 3))
            for host, dev in zip(outs, (stored, lower, upper)):
                check(lib.sci_cuda_download_lane(device.handle, host.data_ptr() + 4 * o, dev.pointer + 4 * o, 4 * span),
                      device.handle)
        with torch.cuda.stream(stream):
            results[0] = piece_results[:, 0].sum()
            results[1] = piece_results[:, 1].max()  # NaN propagates
            results[2] = piece_results[:, 2].sum()
            if dist is not None:
                results.copy_(combine(results, (C.SUM, C.MAXIMUM, C.SUM)))
        check(lib.sci_cuda_download_lane(device.handle, host_results.data_ptr(), results.data_ptr(), 24), device.handle)
        check(lib.sci_cuda_join(device.handle), device.handle)

    e2e_step()
    device.synchronize()
    e_start, e_stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist is not None:
        dist.barrier()
    e_start.record(stream)
    for _ in range(args.e2e_steps):
        e2e_step()
    e_stop.record(stream)
    e_stop.synchronize()
    e2e_ms = e_start.elapsed_time(e_stop) / args.e2e_steps
    if dist is not None:
        t = torch.tensor([e2e_ms], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = STEP_BYTES_PER_ELEMENT * n * world / (e2e_ms * 1e-3) / 1e9
    # the pieces reproduce the single-pass step: elementwise outputs bit for bit, reductions to FP64
    # rounding
    device.synchronize()
    piecewise = host_results.clone()
    step()
    device.synchronize()
    whole = results.cpu()
    for slot in range(3):
        a_, b_ = float(piecewise[slot]), float(whole[slot])
        if not ((math.isnan(a_) and math.isnan(b_)) or abs(a_ - b_) <= 1e-9 * max(abs(b_), 1e-300)):
            raise RuntimeError(f"pipelined reduction {slot} = {a_} differs from the single pass {b_}")

    # a correctness spot check of the step just run: the stored chunk against the CPU oracle
    cpu = None
    if rank == 0 and not args.no_cpu:
        sample = cpu_reference_sample(1 << 24, repeats=5)
        if sample:
            cpu = {"value": STEP_BYTES_PER_ELEMENT * sample["count"] / sample["seconds"] / 1e9, "unit": "GB/s",
                   "cores": sample["threads"], "kind": "reference",
                   "sample": f"{sample['count']} elements (2^24 of 2^28) per step, median of 5, libsci public API"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "large fused chunks (float32, n=2^28 per array per GPU, NaN rate 1e-6)",
                       "elements": n, "bytes_per_element": STEP_BYTES_PER_ELEMENT,
                       "chunks": names, "l2": "inputs 1 GiB each, larger than L2; no flush",
                       "parallelism": f"shard per GPU x{world}"},
            "roofline": roofline, "kernels": kernels, "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "GB/s", "h2d_bytes_per_step": 3 * n * 4,
                    "d2h_bytes_per_step": 3 * n * 4 + 24, "ms_per_step": e2e_ms},
            "gpu_launches": len(names) * args.steps,
            "clocks": clocks.summary(),
        }
    device.close()
    del dx, dy, dz, stored, lower, upper
    torch.cuda.empty_cache()
    if rank == 0:
        if world == 1 and not args.no_extras:
            line["configs"] = run_extras(args)
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


def compact(line: dict, *extra: str) -> dict:
    """The keys of a workload's line that the default run carries for it."""
    keys = ("metric", "value", "unit", "ms_per_step", "higher_is_better", "roofline", "check", "clocks", "e2e",
            "gpu_launches") + extra
    out = {k: line[k] for k in keys if k in line}
    if line.get("cpu_baseline"):
        out["cpu_baseline"] = {k: line["cpu_baseline"][k] for k in ("value", "unit", "cores", "kind", "sample")
                               if k in line["cpu_baseline"]}
    out["workload"] = line.get("config", {}).get("workload")
    return out


def run_extras(args) -> dict:
    """Every other workload of the benchmark at its full size, with fewer timed steps: the plain
    fused expression (n = 2^20), the product (8192^3, every mode), the solve (n = 8192, 16
    right-hand sides, both matrices), the gradients (2^26; 4096 x 64 solve) and both batches, each
    with its own device time, roofline, clocks and check against the oracle."""
    import copy

    import torch

    extra = copy.copy(args)
    extra.steps, extra.warmup, extra.compact = max(3, min(args.steps, 5)), 3, True
    out = {}
    for key, run, keep in (("plain_n2e20", run_plain, ("us_per_call",)),
                           ("product_8192", run_product, ("modes",)),
                           ("solve_8192", run_solve, ("cases",)),
                           ("gradient", run_gradient, ("chunk", "solve")),
                           ("batch_8192_items", run_batch, ("batch",)),
                           ("solves_4096", run_solves, ("solves",))):
        started = time.perf_counter()
        try:
            line = run(extra)
            out[key] = compact(line, *keep)
        except Exception as error:  # noqa: BLE001 - reported in the line, the headline stands
            out[key] = {"error": f"{type(error).__name__}: {error}"}
        out[key]["wall_s"] = time.perf_counter() - started
        torch.cuda.empty_cache()
    return out


if __name__ == "__main__":
    sys.exit(main())

#!/usr/bin/env python
"""Transform-pair throughput at T511 L40 x 5 fields on B200.

One step = the transform pair the sl_si dycore runs each 300 s step over one
batch of 200 planes (40 levels x 5 fields): grid -> spectral (forward) and
spectral -> grid (inverse) on the 768 x 1536 Gaussian grid at T511, through
the engine's public API (one C-ABI call each).  The headline path is the
split-FP16 tensor-core contraction; the plain FP32 path is timed beside it on
the same inputs, and both are checked against the FP64 path for the
relative spectral L2 error (<= 2e-6 is the bar).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun each rank owns one GPU and its own 200 planes (weak scaling,
no collective on the data path); rank 0 prints one JSON line.
``--impl reference`` times the CPU oracle (the numpy restatement of the
reference's dense float64 transform) on this host's cores instead.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path[:0] = [str(ROOT), str(ROOT / "gpuwm-global_b200")]

import numpy as np  # noqa: E402

METRIC = "Transform pairs/s at T511 L40: TC split-precision vs plain FP32 at ≤2e-6 err"
UNIT = "plane-pairs/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--truncation", type=int, default=511)
    ap.add_argument("--planes", type=int, default=200, help="planes per GPU (40 levels x 5 fields)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-planes", type=int, default=40,
                    help="planes of the CPU baseline sample inside the GPU run")
    ap.add_argument("--ref-planes", type=int, default=200,
                    help="planes per step of --impl reference (the configuration's 200)")
    ap.add_argument("--profile-only", action="store_true",
                    help="one plan, warmup + steps of the pair, no checks (small ncu case)")
    ap.add_argument("--precision", default="split16", choices=["split16", "float32", "float64"])
    ap.add_argument("--workload", default="pair", choices=["pair", "ensemble", "step", "sl_gather", "native"],
                    help="pair: the T511 L40 transform pair (default); ensemble: 32 members "
                         "at T126 + the T255 control as one batch; step: the full T511 "
                         "dycore-step transform set as one CUDA graph, with the "
                         "Rossby-Haurwitz wave's energy drift over --drift-steps steps")
    ap.add_argument("--drift-steps", type=int, default=100)
    ap.add_argument("--sl-fields", type=int, default=16, help="sl_gather: fields per call")
    ap.add_argument("--sl-levels", type=int, default=40, help="sl_gather: levels")
    return ap.parse_args()


def flops_per_plane(T, nlat):
    """Algorithmic Legendre flops per plane per direction on the folded
    triangle: nlat (T+1)(T+2)."""
    return nlat * (T + 1) * (T + 2)


def fft_bytes_per_plane(T, nlat, nlon):
    """Algorithmic bytes per plane per direction of a longitude FFT: the f32
    grid plus the c64 Fourier waist cut at m <= T."""
    return 4 * nlat * nlon + 8 * nlat * (T + 1)


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.device_index = device_index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            # nvidia-smi takes a moment to start: let its first sample land
            # before the timed work begins, so the samples cover it.
            t0 = time.time()
            while time.time() - t0 < 5.0 and os.path.getsize(self.path) == 0:
                time.sleep(0.02)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows),
                "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())
                if any(r[3].replace(".", "").isdigit() for r in rows) else None}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d["hbm_gbs"], "bf16_tflops": d["bf16_tflops"],
                "bf16_tflops_sustained": d.get("bf16_tflops_sustained", d["bf16_tflops"]),
                "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0,
            "source": "fallback"}


def ncu_traffic(kernel_kind, T):
    """DRAM bytes per plane of one kernel kind from the committed ncu summary
    (profiles/traffic.json), or None."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    d = json.loads(p.read_text())
    entry = d.get(f"T{T}", {}).get(kernel_kind)
    return None if entry is None else float(entry["dram_bytes_per_plane"])


def cpu_oracle_rate(T, planes, reps=2, ora=None):
    """Plane-pairs/s of the CPU oracle on `planes` planes (host cores)."""
    from b200sht.synthetic import red_spectrum
    from oracle.dense_sht import DenseSHT

    ora = ora if ora is not None else DenseSHT(T)
    coeff = red_spectrum(T, planes)
    grid = ora.inverse(coeff)
    best = math.inf
    for _ in range(reps):
        t0 = time.perf_counter()
        c = ora.forward(grid)
        grid = ora.inverse(c)
        best = min(best, time.perf_counter() - t0)
    return planes / best, best


def copy_floor(host_in, host_out, steps):
    """Milliseconds per step of the end-to-end leg's copies alone: the pinned
    grid host-to-device, the grid device-to-host, and both at once on two
    streams (the floor a host-streamed round trip can approach)."""
    import torch

    dev_in = torch.empty(host_in.shape, dtype=host_in.dtype, device="cuda")
    dev_out = torch.zeros_like(dev_in)
    cur = torch.cuda.current_stream()
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()

    def one(h2d, d2h):
        s_in.wait_stream(cur)
        s_out.wait_stream(cur)
        if h2d:
            with torch.cuda.stream(s_in):
                dev_in.copy_(host_in, non_blocking=True)
        if d2h:
            with torch.cuda.stream(s_out):
                host_out.copy_(dev_out, non_blocking=True)
        cur.wait_stream(s_in)
        cur.wait_stream(s_out)

    out = {}
    for name, h2d, d2h in (("h2d_only_ms", True, False), ("d2h_only_ms", False, True),
                           ("both_directions_ms", True, True)):
        one(h2d, d2h)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(steps):
            one(h2d, d2h)
        b.record()
        torch.cuda.synchronize()
        out[name] = a.elapsed_time(b) / steps
    del dev_in, dev_out
    return out


def cpu_sl_gather_rate():
    """Point-fields/s of the CPU oracle's cubic quasi-monotone gather on a
    bounded sample: one field of 4 levels on the 768 x 1536 grid."""
    import numpy as np

    from oracle import sl_gather as O

    nlev = 4
    lat = np.sort(np.arcsin(np.polynomial.legendre.leggauss(768)[0]))
    xi, phi, level = O.departure_sample(nlev, lat, 1536, 11, cells=1.0, dtype=np.float32)
    f = np.random.default_rng(5).standard_normal((nlev, 768, 1536)).astype(np.float32)
    t0 = time.perf_counter()
    O.gather([f], xi, phi, level, lat, 1536, dtype=np.float32)
    dt = time.perf_counter() - t0
    return {"value": nlev * 768 * 1536 / dt, "unit": "point-fields/s", "cores": 1,
            "kind": "port",
            "sample": f"1 field x 4 levels x 768 x 1536, cubic quasi-monotone, numpy ({dt:.1f} s)"}


def run_reference(args):
    ws, rank, _ = dist_setup()
    if rank != 0:
        return
    from b200sht.synthetic import red_spectrum
    from oracle.dense_sht import DenseSHT

    # The configuration's 200 planes per step (the oracle's dense GEMMs run
    # batched over the planes); a step takes seconds on the host, so at most
    # 10 timed steps and one warm-up step are run, whatever K and W ask for
    # (both counts are reported).
    T, P = args.truncation, args.ref_planes
    steps, warmup = max(1, min(args.steps, 10)), min(max(args.warmup, 0), 1)
    ora = DenseSHT(T)
    coeff = red_spectrum(T, P)
    grid = ora.inverse(coeff)
    for _ in range(warmup):
        grid = ora.inverse(ora.forward(grid))
    t0 = time.perf_counter()
    for _ in range(steps):
        grid = ora.inverse(ora.forward(grid))
    dt = (time.perf_counter() - t0) / steps
    value = P / dt
    cores = os.cpu_count()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "warmup": warmup, "steps_requested": args.steps,
        "warmup_requested": args.warmup, "ms_per_step": dt * 1e3,
        "higher_is_better": True, "impl": "reference", "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic red-spectrum (seeded)",
        "config": {"workload": f"T{T} L40 x 5 fields = {P} planes per GPU, {ora.nlat}x{ora.nlon} "
                               f"Gaussian grid, forward + inverse per step",
                   "truncation": T, "nlat": ora.nlat, "nlon": ora.nlon, "planes_per_gpu": P},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{P} planes of T{T} per step x {steps} steps, numpy float64 "
                                   f"dense oracle (the reference's dense transform restated)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload != "pair":
        from b200sht.workloads import run_workload

        line = run_workload(args, ClockSampler)
        if args.workload == "sl_gather" and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_sl_gather_rate()
        print(json.dumps(line), flush=True)
        return
    import torch
    import torch.distributed as dist

    from b200sht import SphericalHarmonicTransform
    from b200sht.synthetic import CONTROL_SEED, red_spectrum

    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if args.profile_only:
        sht = SphericalHarmonicTransform.create(args.truncation, precision=args.precision)
        c = torch.as_tensor(red_spectrum(args.truncation, args.planes)).to(dev, sht.backend.complex_dtype)
        g = sht.inverse(c)
        for _ in range(args.warmup + args.steps):
            g = sht.inverse(sht.forward(g))
        torch.cuda.synchronize()
        sht.check_device()
        print(json.dumps({"profile_only": True, "truncation": args.truncation,
                          "planes": args.planes, "precision": args.precision}))
        return
    if ws > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=dev)
    T, P = args.truncation, args.planes

    from b200sht import replicas

    def barrier():
        replicas.barrier(dev)

    def max_over_ranks(x):
        return replicas.max_over_ranks(x, dev)

    # Inputs: seeded red spectrum; grids are the FP64 synthesis cast to f32.
    coeff64 = torch.as_tensor(red_spectrum(T, P, CONTROL_SEED + rank)).to(dev)
    f64 = SphericalHarmonicTransform.create(T, precision="float64")
    grid64 = f64.inverse(coeff64)
    ref_coeff = f64.forward(grid64)
    nlat, nlon = f64.grid.shape
    grid32 = grid64.to(torch.float32).contiguous()
    coeff32 = coeff64.to(torch.complex64).contiguous()

    def errors(sht):
        c = sht.forward(grid32).to(torch.complex128)
        w = torch.ones(T + 1, dtype=torch.float64, device=dev)
        w[1:] = 2.0
        num = ((c - ref_coeff).abs() ** 2 * w).sum()
        den = (ref_coeff.abs() ** 2 * w).sum()
        g = sht.inverse(coeff32).to(torch.float64)
        gerr = (g - grid64).abs().max() / grid64.abs().max()
        rt = sht.transform_check(seed=7)
        return {"rel_spectral_l2": float(torch.sqrt(num / den)),
                "max_grid_rel": float(gerr),
                "roundtrip_relative_linf": rt["roundtrip_relative_linf"]}

    def timed_pairs(sht, steps, warmup, record_kernels=False):
        g = grid32
        for _ in range(warmup):
            c = sht.forward(g)
            g2 = sht.inverse(c)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        sht.plan.read_timing(reset=True)
        sht.plan.set_timing(record_kernels)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        for _ in range(steps):
            c = sht.forward(g)
            g2 = sht.inverse(c)
        stop.record()
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        sht.plan.set_timing(False)
        kern = sht.plan.read_timing(reset=True)
        ms = start.elapsed_time(stop) / steps
        return max_over_ranks(ms), kern

    split = SphericalHarmonicTransform.create(T, precision="split16")
    plain = SphericalHarmonicTransform.create(T, precision="float32")
    err_split = errors(split)
    err_plain = errors(plain)
    del f64

    def errors_vs_oracle(sht, ora, n=2):
        """Relative spectral L2 of forward and max grid error of inverse
        against the oracle's float64 transforms of the first n planes."""
        g64 = grid64[:n].cpu().numpy()
        c64 = coeff64[:n].cpu().numpy()
        ref_c = ora.forward(g64)
        ref_g = ora.inverse(c64)
        c = sht.forward(grid32[:n]).cpu().numpy().astype(np.complex128)
        g = sht.inverse(coeff32[:n]).cpu().numpy().astype(np.float64)
        w = np.where(np.arange(T + 1) == 0, 1.0, 2.0)
        rel = np.sqrt(np.sum(w * np.abs(c - ref_c) ** 2) / np.sum(w * np.abs(ref_c) ** 2))
        return {"rel_spectral_l2": float(rel),
                "max_grid_rel": float(np.max(np.abs(g - ref_g)) / np.max(np.abs(ref_g))),
                "planes": n}

    # Headline: the pair loop with no per-kernel events in it.  Kernel shares
    # and the roofline come from a second, instrumented run (CUDA events on
    # the library's stream around every launch).
    # Clocks are sampled over both timed loops (split, then plain).
    with ClockSampler(local) as clocks:
        ms_split, _ = timed_pairs(split, args.steps, args.warmup)
        ms_plain, _ = timed_pairs(plain, args.steps, args.warmup)
    clk = clocks.summary()
    k_inst = max(3, min(args.steps, 10))
    ms_split_inst, kern = timed_pairs(split, k_inst, 1, record_kernels=True)
    ms_plain_inst, kern_plain = timed_pairs(plain, k_inst, 1, record_kernels=True)
    # The split path with its double-buffered accumulator plan (one main
    # accumulator: faster, larger but still sub-2e-6 error), reported beside
    # the headline's three-segment plan.
    from b200sht.autotune import set_tuning

    set_tuning(split, accumulators=1)
    err_overlap = errors(split)
    ms_overlap, _ = timed_pairs(split, args.steps, args.warmup)
    set_tuning(split, accumulators=0)

    value = ws * P / (ms_split * 1e-3)
    value_plain = ws * P / (ms_plain * 1e-3)

    # Dominant kernel of the headline path and its roofline.
    peaks = measured_peaks()
    per_launch = {k: v["ms"] / v["timed"] for k, v in kern.items() if v["timed"]}
    share = {k: v["ms"] / sum(x["ms"] for x in kern.values()) for k, v in kern.items() if v["timed"]}
    dom = max(per_launch, key=lambda k: kern[k]["ms"])
    if dom.startswith("legendre"):
        flops = 3 * flops_per_plane(T, nlat) * P
        achieved = flops / (per_launch[dom] * 1e-3) / 1e12
        peak = peaks["bf16_tflops_sustained"]
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s"}
    else:
        if dom.startswith("fft"):
            byts = fft_bytes_per_plane(T, nlat, nlon) * P
        else:
            byts = 2 * 8 * (T + 1) * (T + 2) // 2 * P
        achieved = byts / (per_launch[dom] * 1e-3) / 1e9
        peak = peaks["hbm_gbs"]
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s"}
    roof["frac"] = roof["achieved"] / roof["peak"]
    # The plain FP32 path's Legendre kernels against the measured FFMA rate.
    from b200sht import _lib

    ffma = ctypes.c_double(0.0)
    _lib.call("sht_measure_fp32_peak", None, ctypes.byref(ffma))
    plain_leg = {}
    for k in ("legendre_analysis", "legendre_synthesis"):
        v = kern_plain.get(k)
        if v and v["timed"]:
            ms_l = v["ms"] / v["timed"]
            ach = flops_per_plane(T, nlat) * P / (ms_l * 1e-3) / 1e12
            plain_leg[k] = {"ms_per_launch": ms_l, "achieved_tflops": ach,
                            "frac_of_ffma_peak": ach / ffma.value}
    # The split path's Legendre kernels against the tensor-core peak: the
    # three FP16 products of the folded triangle, 3 nlat (T+1)(T+2) flops
    # per plane per direction.
    split_leg = {}
    for k in ("legendre_analysis", "legendre_synthesis"):
        if k in per_launch:
            ach = 3 * flops_per_plane(T, nlat) * P / (per_launch[k] * 1e-3) / 1e12
            split_leg[k] = {"ms_per_launch": per_launch[k], "achieved_tflops": ach,
                            "frac_of_bf16_peak_sustained": ach / peaks["bf16_tflops_sustained"]}
    traffic = ncu_traffic(dom, T)
    roof["traffic"] = None if traffic is None else traffic * P
    roof["kernel"] = dom
    roof["peak_source"] = peaks["source"] + (" sustained" if roof["bound"] == "tensor" else "")
    roof["ms_per_launch"] = per_launch[dom]

    # End to end through the public API with pinned host buffers: the
    # host-streamed round trip (grid in from host memory, forward + inverse,
    # grid out to host memory; the copies of neighbouring plane chunks overlap
    # each other and the transforms).  Each step is one synchronous call.
    g_split_dev_ref = split.inverse(split.forward(grid32)).cpu()  # the device calls' result
    host_in = torch.empty(grid32.shape, dtype=torch.float32, pin_memory=True)
    host_in.copy_(grid32)
    host_out = torch.empty(grid32.shape, dtype=torch.float32, pin_memory=True)
    e2e_steps = max(3, min(args.steps, 10))
    for _ in range(2):
        split.round_trip_host(host_in, out=host_out)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(e2e_steps):
        split.round_trip_host(host_in, out=host_out)
    b.record()
    torch.cuda.synchronize()
    barrier()
    e2e_ms = max_over_ranks(a.elapsed_time(b) / e2e_steps)
    e2e_err = float((host_out - g_split_dev_ref).abs().max() / g_split_dev_ref.abs().max())
    nbytes = grid32.numel() * 4
    del g_split_dev_ref
    copies = copy_floor(host_in, host_out, e2e_steps)
    # Launches of the headline loop: the instrumented run's count per pair
    # times the headline's pairs.
    gpu_launches = sum(v["launches"] for v in kern.values()) // k_inst * args.steps

    # The CPU oracle (rank 0, one GPU), built after every GPU timing (its ~10 GB
    # of host tables are allocated only now): the reported CPU baseline, and
    # the FP64 answer of a two-plane sample for the errors named "vs_oracle".
    cpu = None
    oracle_err = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        from oracle.dense_sht import DenseSHT

        ora = DenseSHT(T)
        oracle_err = {"split16": errors_vs_oracle(split, ora),
                      "float32": errors_vs_oracle(plain, ora)}
        rate, sec = cpu_oracle_rate(T, args.cpu_planes, ora=ora)
        cpu = {"value": rate, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
               "sample": f"{args.cpu_planes} planes of T{T} (768x1536), forward+inverse, "
                         f"numpy float64 dense oracle, best of 2 ({sec:.2f} s)"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_split, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f16x3-split (f32 accumulate)",
            "data": "synthetic seeded red spectrum, grids = FP64 synthesis cast to f32",
            "config": {
                "workload": f"T{T} L40 x 5 fields = {P} planes per GPU, {nlat}x{nlon} Gaussian "
                            f"grid, forward + inverse per step",
                "truncation": T, "nlat": nlat, "nlon": nlon, "planes_per_gpu": P,
                "parallelism": f"replicas x{ws} (planes sharded per GPU, no collective)",
                "l2": f"inputs larger than L2 ({grid32.numel() * 4 / 1e6:.0f} MB grid per step)",
                "sets_per_s": value / P,
                "plain_fp32": {"value": value_plain, "ms_per_step": ms_plain, **err_plain,
                               "legendre_vs_ffma_peak": plain_leg,
                               "ffma_peak_tflops_measured": ffma.value},
                "split16_overlapped_accumulators": {"value": ws * P / (ms_overlap * 1e-3),
                                                    "ms_per_step": ms_overlap, **err_overlap},
                "split16_legendre": split_leg,
                "split_over_plain": value / value_plain,
                "split_errors": err_split,
                "errors_measured_against": "this engine's FP64 plan on all planes (its FP64 "
                                           "transforms are pinned to the reference's outputs); "
                                           "errors_vs_oracle: the CPU float64 oracle on a "
                                           "plane sample",
                "errors_vs_oracle": oracle_err,
                "kernel_share": share,
                "kernel_share_run": {"pairs": k_inst, "ms_per_step_instrumented": ms_split_inst,
                                     "plain_ms_per_step_instrumented": ms_plain_inst},
                "headline_timing": "pair loop without per-kernel events",
            },
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": {"value": ws * P / (e2e_ms * 1e-3), "unit": UNIT,
                    "api": "SphericalHarmonicTransform.round_trip_host (sht_round_trip_host)",
                    "rel_diff_vs_device_calls": e2e_err,
                    "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
                    "ms_per_step": e2e_ms,
                    "copies_alone": copies,
                    "copies_alone_over_e2e": copies["both_directions_ms"] / e2e_ms},
            "gpu_launches": gpu_launches,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

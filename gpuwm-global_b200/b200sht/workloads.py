"""Timed workloads beside the headline transform pair (used by ``bench.py``).

``ensemble``: 32 LETKF members at T126 (192 x 384) and the control at T255
(384 x 768), 40 levels x 5 fields each, as one ``TransformBatch`` (one merged
Legendre launch per direction), eager and as a captured CUDA graph, against
the same plans run one after the other.  Inputs: the seeded red-spectrum
control plus per-member draws at 10 % amplitude, synthesised in FP64 on the
GPU and cast to f32.

``step``: the full T511 L40 dycore-step transform set (``DycoreTransformStep``)
as one CUDA graph per 300 s step, split16 and float32, with the
Rossby-Haurwitz wave-4 state plus 1 % red noise iterated for ``drift_steps``
steps and the wave's spectral energy drift reported against the FP64 path.
"""
from __future__ import annotations

import torch

from .autotune import tune
from .batch import TransformBatch
from .semi_implicit import VerticalModeOperator
from .step import DycoreTransformStep, rossby_haurwitz_state, wave_energy
from .synthetic import CONTROL_SEED, ensemble_member, red_spectrum, seeded_vertical_operator
from .transform import SphericalHarmonicTransform


def _time(fn, steps, warmup):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / steps


def _rel_l2(c, ref):
    t1 = ref.shape[-1]
    w = torch.ones(t1, dtype=torch.float64, device=ref.device)
    w[1:] = 2.0
    num = ((c.to(torch.complex128) - ref).abs() ** 2 * w).sum()
    den = (ref.abs() ** 2 * w).sum()
    return float(torch.sqrt(num / den))


def _graph(fn):
    """Capture ``fn`` (already warmed up) in a CUDA graph."""
    g = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side), torch.cuda.graph(g, stream=side):
        fn()
    torch.cuda.current_stream().wait_stream(side)
    return g


def ensemble(args, clock_sampler):
    dev = torch.device("cuda", torch.cuda.current_device())
    members, per = 32, 200
    specs = [(126, 192, 384, members * per), (255, 384, 768, per)]
    grids, refs = [], []
    for T, nl, no, planes in specs:
        f64 = SphericalHarmonicTransform.create(T, nlat=nl, nlon=no, precision="float64")
        control = red_spectrum(T, per, CONTROL_SEED)
        coeff = torch.empty((planes, T + 1, T + 1), dtype=torch.complex128, device=dev)
        if planes == per:
            coeff.copy_(torch.as_tensor(control))
        else:
            for k in range(members):
                coeff[k * per:(k + 1) * per].copy_(torch.as_tensor(ensemble_member(control, k)))
        g64 = f64.inverse(coeff)
        refs.append(f64.forward(g64))
        grids.append(g64.to(torch.float32).contiguous())
        del coeff, g64, f64
    total = sum(s[3] for s in specs)
    out = {"metric": "Batched ensemble transform pairs/s (32 x T126 + T255 control, L40 x 5)",
           "unit": "plane-pairs/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "higher_is_better": True, "data": "synthetic seeded red spectrum + 10% member draws",
           "config": {"workload": "32 members x 200 planes at T126 (192x384) + 200 planes at "
                                  "T255 (384x768), forward + inverse per step",
                      "planes": total, "l2": "inputs larger than L2"}}
    with clock_sampler(torch.cuda.current_device()) as clocks:
        for prec in ("split16", "float32"):
            plans = [SphericalHarmonicTransform.create(T, nlat=nl, nlon=no, precision=prec)
                     for T, nl, no, _ in specs]
            # The project autotuner picks each plan's settings for its plane count.
            tuned = [tune(pl, sp[3], repeats=3, warmup=1)["best"] for pl, sp in zip(plans, specs)]
            batch = TransformBatch(plans, [s[3] for s in specs])
            state = {}

            def pair():
                state["c"] = batch.forward(grids)
                state["g"] = batch.inverse(state["c"])

            def unbatched():
                for t, g in zip(plans, grids):
                    t.inverse(t.forward(g))

            ms_batch = _time(pair, args.steps, args.warmup)
            ms_single = _time(unbatched, args.steps, args.warmup)
            graph = _graph(pair)
            ms_graph = _time(graph.replay, args.steps, args.warmup)
            errs = [_rel_l2(c, r) for c, r in zip(state["c"], refs)]
            plans[0].check_device()
            out[prec] = {"plane_pairs_per_s_graph": total / (ms_graph * 1e-3),
                         "ms_graph": ms_graph, "ms_batch_eager": ms_batch,
                         "ms_per_plan_eager": ms_single,
                         "rel_spectral_l2": {"T126": errs[0], "T255": errs[1]},
                         "autotuned": {"T126": tuned[0], "T255": tuned[1]}}
            del graph, batch, plans, state
            torch.cuda.empty_cache()
    out["clocks"] = clocks.summary()
    out["value"] = out["split16"]["plane_pairs_per_s_graph"]
    out["ms_per_step"] = out["split16"]["ms_graph"]
    out["split_over_plain"] = out["float32"]["ms_graph"] / out["split16"]["ms_graph"]
    return out


def step(args, clock_sampler):
    T, nlev, n_scalar = 511, 40, 5
    b, c = seeded_vertical_operator(nlev)
    op = VerticalModeOperator(b, c)
    f64 = SphericalHarmonicTransform.create(T, precision="float64")
    state = rossby_haurwitz_state(f64, nlev, n_scalar=n_scalar, noise=0.01)
    n = int(args.drift_steps)
    out = {"metric": "T511 L40 dycore-step transform sets/s (one CUDA graph per step)",
           "unit": "steps/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "higher_is_better": True,
           "data": "Rossby-Haurwitz wave 4 (omega = K = 7.848e-6 1/s) + 1% seeded red noise; "
                   "seeded diagonally dominant 40x40 vertical structure",
           "config": {"workload": "per step: forward of 5 x 40 scalar planes + ln ps, vordiv "
                                  "from u,v (40 levels), Helmholtz solve, u,v from vordiv, "
                                  "gradients of theta (40) and ln ps, inverse of D (40)",
                      "truncation": T, "levels": nlev, "drift_steps": n}}
    z_end = {}
    with clock_sampler(torch.cuda.current_device()) as clocks:
        for prec in ("split16", "float32", "float64"):
            t = f64 if prec == "float64" else SphericalHarmonicTransform.create(T, precision=prec)
            st = DycoreTransformStep(t, op, n_scalar=n_scalar)
            st.load(*state)
            st.capture()
            res = {}
            if prec != "float64":
                st.load(*state)
                res["ms_eager"] = _time(st.run, args.steps, args.warmup)
                st.load(*state)
                res["ms_graph"] = _time(st.graph.replay, args.steps, args.warmup)
            st.load(*state)
            st.replay(1)
            torch.cuda.synchronize()
            z1 = st.vorticity.cpu().numpy()
            st.replay(n - 1)
            torch.cuda.synchronize()
            t.check_device()
            zn = st.vorticity.cpu().numpy()
            res["wave_energy_drift"] = wave_energy(zn, 5, 4, T) / wave_energy(z1, 5, 4, T) - 1.0
            res["solid_body_energy_drift"] = (wave_energy(zn, 1, 0, T) /
                                              wave_energy(z1, 1, 0, T) - 1.0)
            z_end[prec] = st.vorticity.to(torch.complex128)
            out[prec] = res
            del st
            torch.cuda.empty_cache()
    for prec in ("split16", "float32"):
        out[prec]["vorticity_rel_l2_vs_fp64_after_drift"] = _rel_l2(z_end[prec], z_end["float64"])
        out[prec]["wave_energy_drift_minus_fp64"] = (out[prec]["wave_energy_drift"] -
                                                     out["float64"]["wave_energy_drift"])
    out["clocks"] = clocks.summary()
    out["value"] = 1e3 / out["split16"]["ms_graph"]
    out["ms_per_step"] = out["split16"]["ms_graph"]
    out["split_over_plain"] = out["float32"]["ms_graph"] / out["split16"]["ms_graph"]
    return out


def run_workload(args, clock_sampler):
    torch.cuda.set_device(0)
    return {"ensemble": ensemble, "step": step}[args.workload](args, clock_sampler)

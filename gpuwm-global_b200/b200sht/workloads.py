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

``native``: forward + inverse at T767 and T1534 on their native grids with
resident tables (plan build time, memory, pair time, round-trip error).

``sl_gather``: the semi-Lagrangian gather of 16 fields at T511 L40 (cubic
quasi-monotone headline, cubic and quintic unlimited, trilinear) at the
departure points of a solid-body rotation across both poles.
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


def rotation_departures(lat, nlon, nlev, *, speed=80.0, dt=300.0, radius=6371220.0,
                        dtype=torch.float32, device=None):
    """Departure coordinates of a solid-body rotation about the axis
    through (0 N, 0 E), whose flow crosses both poles: every arrival point
    rotated back by speed * dt / radius radians (0.94 equatorial cells at
    T511), the angle varied by +-20 % over the levels, and the departure
    level k - 0.6 sin(2 lambda) cos(phi), which reaches both half layers."""
    dev = device or torch.device("cuda", torch.cuda.current_device())
    lat = torch.as_tensor(lat, dtype=torch.float64, device=dev)
    lon = torch.arange(nlon, dtype=torch.float64, device=dev) * (2 * torch.pi / nlon)
    k = torch.arange(nlev, dtype=torch.float64, device=dev)
    th = -(speed * dt / radius) * (1.0 + 0.2 * torch.cos(torch.pi * k / max(nlev - 1, 1)))
    cl, sl = torch.cos(lat)[None, :, None], torch.sin(lat)[None, :, None]
    x = cl * torch.cos(lon)[None, None, :]
    y = cl * torch.sin(lon)[None, None, :]
    c, s = torch.cos(th)[:, None, None], torch.sin(th)[:, None, None]
    y2, z2 = y * c - sl * s, y * s + sl * c
    x2 = x.expand_as(y2)
    phi = torch.atan2(z2, torch.sqrt(x2 * x2 + y2 * y2))
    lam = torch.remainder(torch.atan2(y2, x2), 2 * torch.pi)
    xi = lam * (nlon / (2 * torch.pi))
    level = k[:, None, None] - 0.6 * torch.sin(2 * lon)[None, None, :] * cl
    level = level.expand_as(xi)
    return (xi.to(dtype).contiguous(), phi.to(dtype).contiguous(),
            level.to(dtype).contiguous())


def _rhs_timings(args, shape, peak):
    """The fused RHS kernels at the gather's grid (float32; 8 tracers for
    the flux, tendency and vertical flux divergence), with the bytes each
    must move and the fraction of the measured HBM copy rate they reach."""
    from . import rhs

    dev = torch.device("cuda", torch.cuda.current_device())
    g = torch.Generator(device=dev).manual_seed(7)
    rnd = lambda *sh: torch.randn(sh, generator=g, device=dev, dtype=torch.float32)
    nlev, nlat, nlon = shape
    ntr = 8
    n = nlev * nlat * nlon
    res = {}

    def rec(name, fn, nbytes):
        ms = _time(fn, args.steps, args.warmup)
        gbs = nbytes / (ms * 1e-3) / 1e9
        res[name] = {"ms": ms, "gb_per_s": gbs, "frac_of_hbm": gbs / peak}

    three = [rnd(*shape) for _ in range(8)]
    two = [rnd(nlat, nlon) for _ in range(3)]
    zeta, u, v, wu, wv, tv, pg, phi = three
    cor, ge, gn = two
    rec("momentum_bernoulli",
        lambda: rhs.momentum_bernoulli(zeta, cor, u, v, wu, wv, tv, pg, ge, gn, phi, 287.04),
        4 * n * (8 + 3))
    del three
    s = rnd(ntr, *shape)
    dp = rnd(*shape).abs_() + 1.0
    flux = torch.empty((2, ntr, *shape), device=dev)
    rec("tracer_flux_8", lambda: rhs.tracer_flux(dp, s, u, v, out=flux), 4 * n * (3 + 3 * ntr))
    del flux
    h, vert = rnd(ntr, *shape), rnd(ntr, *shape)
    rec("scalar_tendency_8", lambda: rhs.scalar_tendency(h, vert, s, u, dp),
        4 * n * (2 + 4 * ntr))
    del h, vert
    w = rnd(nlev + 1, nlat, nlon)
    ph = torch.cumsum(torch.rand((nlev + 1, nlat, nlon), device=dev) + 0.5, dim=0)
    pf = 0.5 * (ph[:-1] + ph[1:])
    rec("vertical_flux_divergence_8", lambda: rhs.vertical_flux_divergence(s, w, pf, ph),
        4 * n * (3 + 2 * ntr))
    return res


def _sampling_timings(args):
    """Point sampling at T511 in FP64: 4 fields at 16 384 random points,
    scalar and gradient (the verification harness's regular-grid export)."""
    from .sampling import sample_into

    dev = torch.device("cuda", torch.cuda.current_device())
    g = torch.Generator(device=dev).manual_seed(9)
    T, nf, npts = 511, 4, 16384
    c = torch.randn((nf, T + 1, T + 1), generator=g, device=dev, dtype=torch.complex128)
    lat = (torch.rand(npts, generator=g, device=dev, dtype=torch.float64) - 0.5) * 3.0
    lon = torch.rand(npts, generator=g, device=dev, dtype=torch.float64) * 6.283
    o0 = torch.empty((nf, npts), dtype=torch.float64, device=dev)
    o1 = torch.empty_like(o0)
    steps, warm = max(2, args.steps // 10), max(1, args.warmup // 3)
    ms_s = _time(lambda: sample_into(T, c, lat, lon, 6371220.0, o0), steps, warm)
    ms_g = _time(lambda: sample_into(T, c, lat, lon, 6371220.0, o0, o1), steps, warm)
    terms = nf * npts * (T + 1) * (T + 2) / 2
    return {"truncation": T, "fields": nf, "points": npts,
            "scalar_ms": ms_s, "gradient_ms": ms_g,
            "scalar_point_fields_per_s": nf * npts / (ms_s * 1e-3),
            "scalar_terms_per_s": terms / (ms_s * 1e-3)}


def sl_gather(args, clock_sampler):
    """The semi-Lagrangian gather of 16 fields (the reference's batch) at
    T511 L40 on the 768 x 1536 grid, float32: cubic quasi-monotone (the
    limited species, headline), cubic unlimited, quintic unlimited (the
    dynamical bundle) and the trilinear value."""
    from .grid import GaussianGrid
    from .semilag import (CartesianWind, SphericalGridTables, Stencil, gather_batch,
                          gather_linear_batch, lipschitz, search_into)

    nlev, nfield = getattr(args, "sl_levels", 40), getattr(args, "sl_fields", 16)
    grid = GaussianGrid.create(511, nlat=768, nlon=1536)
    dev = torch.device("cuda", torch.cuda.current_device())
    tables = SphericalGridTables.create(grid, dtype=torch.float32)
    xi, phi, level = rotation_departures(grid.lat_rad, grid.nlon, nlev)
    st = Stencil(xi=xi, phi=phi, level=level, tables=tables)
    gen = torch.Generator(device=dev).manual_seed(20261203)
    src = torch.randn((nfield, nlev, grid.nlat, grid.nlon), generator=gen, device=dev,
                      dtype=torch.float32)
    fields = list(src)
    npts = nlev * grid.nlat * grid.nlon
    cases = {"cubic_quasi_monotone": dict(monotone=True, order=4),
             "cubic_none": dict(monotone=False, order=4),
             "quintic_none": dict(monotone=False, order=6)}
    out = {"metric": f"Semi-Lagrangian gather point-fields/s (T511 L{nlev}, {nfield} fields, "
                     "cubic quasi-monotone)",
           "unit": "point-fields/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "higher_is_better": True, "dtype": "f32",
           "data": "synthetic: seeded normal fields; departure points of a solid-body rotation "
                   "across both poles (0.94 equatorial cells) and +-0.6 levels",
           "config": {"workload": f"{nfield} fields x {nlev} levels x 768 x 1536, one gather "
                                  "call of 16 fields per step",
                      "points": npts, "fields": nfield,
                      "l2": f"inputs larger than L2 ({npts * nfield * 4 / 1e9:.1f} GB of "
                            "source fields)"}}
    peak = None
    try:
        import json
        from pathlib import Path

        mp = Path(__file__).resolve().parents[2] / "MEASURED_PEAKS.json"
        peak = float(json.loads(mp.read_text())["hbm_gbs"]) if mp.exists() else 6650.0
    except Exception:
        peak = 6650.0
    with clock_sampler(torch.cuda.current_device()) as clocks:
        for name, kw in cases.items():
            ms = _time(lambda: gather_batch(fields, st, batch=nfield, **kw), args.steps,
                       args.warmup)
            byts = npts * (3 * 4 + nfield * 8)
            out[name] = {"ms": ms, "point_fields_per_s": npts * nfield / (ms * 1e-3),
                         "algorithmic_gb_per_s": byts / (ms * 1e-3) / 1e9}
        ms = _time(lambda: gather_linear_batch(fields, st, batch=nfield), args.steps, args.warmup)
        out["trilinear"] = {"ms": ms, "point_fields_per_s": npts * nfield / (ms * 1e-3)}
        # the fixed-point departure search, 3 iterations, on the rotation's
        # wind as Cartesian components (80 m/s) and a +-1.5e-3 levels/s rate
        lat = torch.as_tensor(grid.lat_rad, dtype=torch.float64, device=dev)[None, :, None]
        lon = torch.as_tensor(grid.lon_rad, dtype=torch.float64, device=dev)[None, None, :]
        shape = (nlev, grid.nlat, grid.nlon)
        vz_ = (80.0 * torch.cos(lat) * torch.sin(lon)).expand(shape)
        vy_ = (-80.0 * torch.sin(lat)).expand(shape)
        wind = [torch.zeros(shape, dtype=torch.float32, device=dev), vy_.float().contiguous(),
                vz_.float().contiguous(),
                (1.5e-3 * torch.sin(2 * lon) * torch.cos(lat)).expand(shape).float().contiguous()]
        dep = [torch.empty(shape, dtype=torch.float32, device=dev) for _ in range(5)]
        ms = _time(lambda: search_into(tables, wind + wind, 3, 300.0, dep), args.steps,
                   args.warmup)
        out["departure_search_3_iterations"] = {"ms": ms, "points_per_s": npts / (ms * 1e-3)}
        ms = _time(lambda: search_into(tables, wind + wind, 3, 300.0, dep, solver="newton"),
                   args.steps, args.warmup)
        out["departure_newton_3_iterations"] = {"ms": ms, "points_per_s": npts / (ms * 1e-3)}
        ms = _time(lambda: search_into(tables, wind + wind, 3, 300.0, dep, solver="newton_ls"),
                   args.steps, args.warmup)
        out["departure_newton_ls_3_iterations"] = {"ms": ms, "points_per_s": npts / (ms * 1e-3)}
        # the trajectory gate's deformation diagnostic on the same wind, the
        # arrival side reading an extrapolated wind (the same arrays): norms
        # and both fold determinants, reduced to the host each call
        flow = CartesianWind(*wind)
        ms = _time(lambda: lipschitz(flow, tables, 300.0, extrapolated=flow), args.steps,
                   args.warmup)
        out["deformation_diagnostic"] = {"ms": ms, "points_per_s": npts / (ms * 1e-3),
                                         "algorithmic_gb_per_s": npts * 32 / (ms * 1e-3) / 1e9,
                                         "algorithmic_bytes_per_point": 32}
        del wind, dep, flow
        out["rhs_kernels"] = _rhs_timings(args, (nlev, grid.nlat, grid.nlon), peak)
        out["point_sampling"] = _sampling_timings(args)
    head = out["cubic_quasi_monotone"]
    out["clocks"] = clocks.summary()
    out["value"] = head["point_fields_per_s"]
    out["ms_per_step"] = head["ms"]
    out["gpu_launches"] = (len(cases) + 3 + 4 + 2) * args.steps
    out["roofline"] = {"bound": "hbm", "achieved": head["algorithmic_gb_per_s"], "peak": peak,
                       "unit": "GB/s", "frac": head["algorithmic_gb_per_s"] / peak,
                       "traffic": None, "kernel": "sl_gather_kernel<float, 4, qm>",
                       "algorithmic_bytes_per_point": 3 * 4 + nfield * 8}
    return out


def native_grids(args, clock_sampler):
    """Analysis and synthesis on the verification harness's native grids,
    T767 (1152 x 2304) and T1534 (1536 x 3072, the GFS grid), with every
    table resident (the reference streams them from the recurrence because
    a 16 GB card cannot hold them): plan build time, device memory, the
    split16 pair's time at 8 planes and the round-trip error of a seeded
    red spectrum."""
    import time as _t

    out = {"metric": "Native-grid transform pair (T767 and T1534, split16), ms per 8-plane pair",
           "unit": "ms", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "higher_is_better": False, "data": "synthetic seeded red spectrum", "cases": []}
    dev = torch.device("cuda", torch.cuda.current_device())
    with clock_sampler(torch.cuda.current_device()) as clocks:
        # T767 on its quadratic grid, T1534 on the linear GFS grid
        for T, nl, no, dealias in ((767, 1152, 2304, 1.5), (1534, 1536, 3072, 1.0)):
            torch.cuda.synchronize()
            free0 = torch.cuda.mem_get_info()[0]
            t0 = _t.perf_counter()
            t = SphericalHarmonicTransform.create(T, nlat=nl, nlon=no, dealias_factor=dealias,
                                                  precision="split16")
            c = torch.as_tensor(red_spectrum(T, 8, CONTROL_SEED), device=dev)
            c = c.to(t.backend.complex_dtype)
            t.inverse(c)
            torch.cuda.synchronize()
            build_s = _t.perf_counter() - t0
            used = (free0 - torch.cuda.mem_get_info()[0]) / 2**30
            state = {}

            def pair():
                state["c"] = t.forward(t.inverse(c))

            ms = _time(pair, max(2, args.steps // 20), max(1, args.warmup))
            c2 = t.forward(t.inverse(c)).to(torch.complex128)
            c1 = c.to(torch.complex128)
            err = _rel_l2(c2, c1)
            err_max = float((c2 - c1).abs().max() / c1.abs().max())
            out["cases"].append({"truncation": T, "grid": [nl, no], "precision": "split16",
                                 "plan_build_s": build_s, "device_gib": used,
                                 "ms_per_pair_8_planes": ms, "roundtrip_rel_spectral_l2": err,
                                 "roundtrip_rel_max": err_max})
            del t, c, state
            torch.cuda.empty_cache()
    out["clocks"] = clocks.summary()
    out["value"] = out["cases"][-1]["ms_per_pair_8_planes"]
    out["ms_per_step"] = out["value"]
    return out


def run_workload(args, clock_sampler):
    torch.cuda.set_device(0)
    return {"ensemble": ensemble, "step": step, "sl_gather": sl_gather,
            "native": native_grids}[args.workload](args, clock_sampler)

"""The semi-implicit maps on the GPU against the reference's outputs.

``solve_shifted``, ``apply`` and ``half_apply`` (off-centring 0.5 and 0.55,
divergence weight 1 and 0.9) called the reference's way, with the vertical
coordinate as the third argument, against the reference's recorded outputs
and max divergence increments (tests/golden/make_golden_semi.py): FP64 within
1e-11 of the largest value, FP32 within 1e-5.  Also: two half maps compose
to the full map, the fused solve-and-synthesis equals the solve followed by
the synthesis bit for bit, and the inactive solver is the identity.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_golden
from semi_fixtures import RecordedCoordinate, State

pytestmark = pytest.mark.gpu

CASES = ["semi_t7_l6.npz", "semi_t21_l40.npz"]


def _close(a, b, tol):
    a = np.asarray(a)
    scale = max(float(np.max(np.abs(b))), 1e-300)
    assert float(np.max(np.abs(a - b))) <= tol * scale


def _setup(case, precision):
    from b200sht import SphericalHarmonicTransform, build

    build.build()
    g = load_golden(case)
    sht = SphericalHarmonicTransform.create(int(g["truncation"]), precision=precision)
    return g, sht, RecordedCoordinate(g)


@pytest.mark.parametrize("precision", ["float64", "float32"])
@pytest.mark.parametrize("case", CASES)
def test_linear_tendencies_match_reference(case, precision):
    from b200sht import VerticalModeSemiImplicit

    g, sht, vertical = _setup(case, precision)
    tol = 1e-12 if precision == "float64" else 2e-6
    np_ = sht.backend.to_numpy
    state = State.from_golden(g)
    for key, semi in (("linear", VerticalModeSemiImplicit()),
                      ("linear90", VerticalModeSemiImplicit(off_centring_weight=0.55,
                                                            divergence_weight=0.9))):
        lin = semi.linear_tendencies(state, sht, vertical)
        _close(np_(lin.divergence), g[f"{key}_divergence"], tol)
        _close(np_(lin.theta), g[f"{key}_theta"], tol)
        _close(np_(lin.log_surface_pressure), g[f"{key}_lnps"], tol)
        # projected: zero above the triangle, real at m = 0
        d = np_(lin.divergence)
        assert not np.any(np.triu(np.ones(d.shape[-2:], dtype=bool), 1) & (d != 0))
        assert not np.any(d[..., :, 0].imag)
    assert VerticalModeSemiImplicit(enabled=False).linear_tendencies(state, sht, vertical) is None
    sht.check_device()


@pytest.mark.parametrize("precision", ["float64", "float32"])
@pytest.mark.parametrize("case", CASES)
def test_semi_implicit_maps_match_reference(case, precision):
    from b200sht import VerticalModeSemiImplicit

    g, sht, vertical = _setup(case, precision)
    tol = 1e-11 if precision == "float64" else 1e-5
    np_ = sht.backend.to_numpy
    state = State.from_golden(g)
    semi = VerticalModeSemiImplicit()
    solved = semi.solve_shifted(state, sht, vertical, float(g["tau_s"]))
    _close(np_(solved.divergence), g["solve_divergence"], tol)
    _close(np_(solved.theta), g["solve_theta"], tol)
    _close(np_(solved.log_surface_pressure), g["solve_lnps"], tol)
    for key, semi in (("apply", VerticalModeSemiImplicit()),
                      ("apply55", VerticalModeSemiImplicit(off_centring_weight=0.55,
                                                           divergence_weight=0.9))):
        out, metrics = semi.apply(state, sht, vertical, float(g["dt_s"]))
        _close(np_(out.divergence), g[f"{key}_divergence"], tol)
        _close(np_(out.theta), g[f"{key}_theta"], tol)
        _close(np_(out.log_surface_pressure), g[f"{key}_lnps"], tol)
        m = metrics["semi_implicit_max_divergence_increment_s1"]
        assert abs(m - float(g[f"{key}_metric"])) <= tol * float(g[f"{key}_metric"]) * 10
    for key, semi in (("half", VerticalModeSemiImplicit()),
                      ("half55", VerticalModeSemiImplicit(off_centring_weight=0.55,
                                                          divergence_weight=0.9))):
        out, metrics = semi.half_apply(state, sht, vertical, float(g["dt_s"]))
        _close(np_(out.divergence), g[f"{key}_divergence"], tol)
        _close(np_(out.theta), g[f"{key}_theta"], tol)
        _close(np_(out.log_surface_pressure), g[f"{key}_lnps"], tol)
        m = metrics["semi_implicit_max_divergence_increment_s1"]
        assert abs(m - float(g[f"{key}_metric"])) <= tol * float(g[f"{key}_metric"]) * 10
        pre, _ = semi.pre_apply(state, sht, vertical, float(g["dt_s"]))
        _close(np_(pre.divergence), g[f"{key}_divergence"], tol)
    sht.check_device()


def test_two_half_maps_compose_to_the_full_map():
    from b200sht import VerticalModeSemiImplicit

    g, sht, vertical = _setup("semi_t21_l40.npz", "float64")
    semi = VerticalModeSemiImplicit()
    state = State.from_golden(g)
    once, _ = semi.half_apply(state, sht, vertical, float(g["dt_s"]))
    twice, _ = semi.half_apply(once, sht, vertical, float(g["dt_s"]))
    full, _ = semi.apply(state, sht, vertical, float(g["dt_s"]))
    np_ = sht.backend.to_numpy
    for a, b in ((twice.divergence, full.divergence), (twice.theta, full.theta),
                 (twice.log_surface_pressure, full.log_surface_pressure)):
        _close(np_(a), np_(b), 1e-10)


@pytest.mark.parametrize("precision", ["float64", "float32", "split16"])
def test_fused_solve_and_synthesis_equals_solve_then_inverse(precision):
    import torch

    from b200sht import VerticalModeSemiImplicit

    g, sht, vertical = _setup("semi_t21_l40.npz", precision)
    semi = VerticalModeSemiImplicit()
    op = semi.operator(vertical)
    dev, cd = sht.backend.device, sht.backend.complex_dtype
    d = torch.as_tensor(g["divergence"]).to(dev, cd)
    th = torch.as_tensor(g["theta"]).to(dev, cd)
    lp = torch.as_tensor(g["lnps"]).to(dev, cd)
    outs = [torch.empty_like(d), torch.empty_like(th), torch.empty_like(lp)]
    semi.solve_into(sht, op, float(g["tau_s"]), d, th, lp, *outs)
    grid_ref = sht.inverse(outs[0])
    fused = [torch.empty_like(d), torch.empty_like(th), torch.empty_like(lp)]
    grid = torch.empty_like(grid_ref)
    semi.solve_and_synthesize_into(sht, op, float(g["tau_s"]), d, th, lp, *fused, grid)
    for a, b in zip(fused, outs):
        assert torch.equal(a, b)
    assert torch.equal(grid, grid_ref)
    sht.check_device()


def test_inactive_solver_is_identity():
    from b200sht import VerticalModeSemiImplicit

    g, sht, vertical = _setup("semi_t7_l6.npz", "float64")
    state = State.from_golden(g)
    semi = VerticalModeSemiImplicit(enabled=False)
    assert semi.solve_shifted(state, sht, vertical, 300.0) is state
    out, metrics = semi.apply(state, sht, vertical, 300.0)
    assert out is state and metrics["semi_implicit_max_divergence_increment_s1"] == 0.0

"""The semi-implicit operator build and the oracle's maps, on the CPU.

The product's host build of the vertical operator from a hybrid coordinate
(``VerticalModeOperator.from_coordinate``) and the oracle's
``solve_shifted`` / ``apply_crank_nicolson`` / ``half_apply`` against the
reference's recorded operator and outputs (tests/golden/make_golden_semi.py).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_golden
from oracle.dense_sht import apply_crank_nicolson, half_apply, linear_tendencies, solve_shifted
from semi_fixtures import RecordedCoordinate

CASES = ["semi_t7_l6.npz", "semi_t21_l40.npz"]


def _close(a, b, tol):
    scale = max(float(np.max(np.abs(b))), 1e-300)
    assert float(np.max(np.abs(np.asarray(a) - np.asarray(b)))) <= tol * scale


@pytest.mark.parametrize("case", CASES)
def test_operator_build_matches_reference(case):
    from b200sht.semi_implicit import VerticalModeOperator

    g = load_golden(case)
    op = VerticalModeOperator.from_coordinate(RecordedCoordinate(g),
                                              float(g["reference_temperature_k"]),
                                              float(g["reference_surface_pressure_pa"]))
    _close(op.b_matrix, g["b_matrix"], 1e-13)
    _close(op.c_matrix, g["c_matrix"], 1e-13)
    _close(op.eigenvalues, g["eigenvalues"], 1e-12)
    _close(np.sort(op.x_eigenvalues), np.sort(g["x_eigenvalues"]), 1e-12)
    assert np.all(op.eigenvalues > 0) and np.max(op.x_eigenvalues) <= 0


@pytest.mark.parametrize("case", CASES)
def test_oracle_maps_match_reference(case):
    g = load_golden(case)
    args = (g["divergence"], g["theta"], g["lnps"], g["b_matrix"], g["c_matrix"],
            g["eigenvalues"], g["eigenvectors"])
    a = float(g["radius_m"])
    d, th, lp = solve_shifted(*args, float(g["tau_s"]), radius_m=a)
    _close(d, g["solve_divergence"], 1e-12)
    _close(th, g["solve_theta"], 1e-12)
    _close(lp, g["solve_lnps"], 1e-12)
    for key, alpha, weight in (("apply", 0.5, 1.0), ("apply55", 0.55, 0.9)):
        d, th, lp, metric = apply_crank_nicolson(*args, float(g["dt_s"]) * weight, alpha,
                                                 radius_m=a)
        _close(d, g[f"{key}_divergence"], 1e-12)
        _close(th, g[f"{key}_theta"], 1e-12)
        _close(lp, g[f"{key}_lnps"], 1e-12)
        assert abs(metric - float(g[f"{key}_metric"])) <= 1e-12 * float(g[f"{key}_metric"])
    for key, alpha, weight in (("half", 0.5, 1.0), ("half55", 0.55, 0.9)):
        d, th, lp, metric = half_apply(*args, g["x_eigenvalues"], g["x_eigenvectors"],
                                       float(g["dt_s"]) * weight, alpha, radius_m=a)
        _close(d, g[f"{key}_divergence"], 1e-12)
        _close(th, g[f"{key}_theta"], 1e-12)
        _close(lp, g[f"{key}_lnps"], 1e-12)
        assert abs(metric - float(g[f"{key}_metric"])) <= 1e-12 * float(g[f"{key}_metric"])


@pytest.mark.parametrize("case", CASES)
def test_oracle_linear_tendencies_and_mode_report_match_reference(case):
    from b200sht.semi_implicit import VerticalModeSemiImplicit

    g = load_golden(case)
    for key, weight in (("linear", 1.0), ("linear90", 0.9)):
        d, th, lp = linear_tendencies(g["divergence"], g["theta"], g["lnps"], g["b_matrix"],
                                      g["c_matrix"], weight, radius_m=float(g["radius_m"]))
        _close(d, g[f"{key}_divergence"], 1e-13)
        _close(th, g[f"{key}_theta"], 1e-13)
        _close(lp, g[f"{key}_lnps"], 1e-13)
    # the host-side report of the operator's modes and the explicit budget
    vertical = RecordedCoordinate(g)
    semi = VerticalModeSemiImplicit()
    semi90 = VerticalModeSemiImplicit(off_centring_weight=0.55, divergence_weight=0.9)
    report = semi.describe(vertical)
    assert report["scheme"] == "vertical_modes" and report["nlev"] == int(g["nlev"])
    assert report["reference_temperature_k"] == float(g["reference_temperature_k"])
    _close(report["phase_speeds_m_s"], g["phase_speeds_m_s"], 1e-12)
    _close(report["equivalent_depths_m"], g["equivalent_depths_m"], 1e-12)
    assert semi.explicit_wave_speed_m_s(vertical) == float(g["explicit_wave_speed_m_s"]) == 0.0
    _close(semi90.explicit_wave_speed_m_s(vertical), g["explicit90_wave_speed_m_s"], 1e-12)


def test_semi_implicit_refusals_match_reference():
    from b200sht.semi_implicit import VerticalModeSemiImplicit

    with pytest.raises(ValueError, match="off_centring_weight must lie in"):
        VerticalModeSemiImplicit(off_centring_weight=0.4)
    with pytest.raises(ValueError, match="reference_temperature_k must lie in"):
        VerticalModeSemiImplicit(reference_temperature_k=500.0)
    with pytest.raises(ValueError, match="reference_surface_pressure_pa must lie in"):
        VerticalModeSemiImplicit(reference_surface_pressure_pa=10.0)
    with pytest.raises(ValueError, match="divergence_weight must lie in"):
        VerticalModeSemiImplicit(divergence_weight=1.5)
    assert not VerticalModeSemiImplicit(divergence_weight=0.0).active

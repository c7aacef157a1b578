"""The trajectory gate on the CPU: the oracle of the deformation diagnostic
against the reference's recorded outputs, and the product's host-side gate
logic (``refuse_trajectory_fold``, ``convergence``,
``level_rate_from_mass_flux``) against the reference's messages and numbers
(tests/golden/make_golden_lipschitz.py)."""
from __future__ import annotations

import json

import numpy as np
import pytest

from conftest import load_golden
from oracle import sl_lipschitz as O

TAGS = ["f64", "f32"]


def _cases(g):
    nlat = len(g["lat_ext"]) - 4
    whole = (0, nlat)
    return {
        "whole_long": dict(dt=float(g["dt_long"]), src=whole, arr=whole),
        "whole_long_ex": dict(dt=float(g["dt_long"]), src=whole, arr=whole, ex=True),
        "whole_short_ex": dict(dt=float(g["dt_short"]), src=whole, arr=whole, ex=True),
        "whole_chunk2": dict(dt=float(g["dt_long"]), src=whole, arr=whole),
        "whole_lref": dict(dt=float(g["dt_short"]), src=whole, arr=whole, lref=25_000.0),
        "band_south": dict(dt=float(g["dt_long"]), src=(0, 11), arr=(0, 8)),
        "band_south_ex": dict(dt=float(g["dt_long"]), src=(0, 11), arr=(0, 8), ex=True),
        "band_mid": dict(dt=float(g["dt_long"]), src=(9, 23), arr=(12, 20)),
        "band_mid_ex": dict(dt=float(g["dt_long"]), src=(9, 23), arr=(12, 20), ex=True),
    }


def _ex_rows(spec, nlat):
    a0, a1 = spec["arr"]
    if spec["src"] == (0, nlat):
        return (0, nlat)
    return (max(a0 - 1, 0), min(a1 + 1, nlat))


@pytest.mark.parametrize("tag", TAGS)
def test_oracle_matches_the_reference_bit_for_bit(tag):
    g = load_golden(f"lipschitz_{tag}.npz")
    want_all = json.loads(str(g["cases"]))
    nlon, radius, lat_ext = int(g["nlon"]), float(g["radius_m"]), g["lat_ext"]
    nlat = len(lat_ext) - 4
    for name, spec in _cases(g).items():
        s0, s1 = spec["src"]
        wind = [f[:, s0:s1] for f in g["wind"]]
        kw = {}
        if spec.get("ex"):
            e0, e1 = _ex_rows(spec, nlat)
            kw = dict(extrapolated=[f[:, e0:e1] for f in g["wind_ex"]],
                      extrapolated_held=(e0, e1))
        got = O.lipschitz(wind, lat_ext, nlon, radius, spec["dt"],
                          reference_length_m=spec.get("lref"), held=spec["src"],
                          arrival=spec["arr"], **kw)
        want = want_all[name]
        assert got["spectral"] == want["semilag_jacobian_spectral_s"], name
        assert got["frobenius"] == want["semilag_jacobian_frobenius_s"], name
        assert got["horizontal"] == want["semilag_jacobian_horizontal_s"], name
        assert got["vertical"] == want["semilag_jacobian_vertical_s"], name
        assert got["balanced"] == want["semilag_jacobian_balanced_s"], name
        assert min(1.0, got["fold_departure"]) == want["semilag_fold_determinant_departure"]
        assert min(1.0, got["fold_arrival"]) == want["semilag_fold_determinant_arrival"]
        a0 = spec["arr"][0]
        assert O.where_text(got["where_departure"], got["shape"], lat_ext, nlon, a0) == \
            want["fold_where_departure"]
        assert O.where_text(got["where_arrival"], got["shape"], lat_ext, nlon, a0) == \
            want["fold_where_arrival"]


@pytest.mark.parametrize("tag", TAGS)
def test_level_rate_matches_the_reference(tag):
    from b200sht.semilag import level_rate_from_mass_flux

    g = load_golden(f"lipschitz_{tag}.npz")
    want = g["level_rate"]
    assert np.array_equal(O.level_rate_from_mass_flux(g["omega_half"], g["p_full"]), want)
    got = level_rate_from_mass_flux(g["omega_half"], p_full=g["p_full"])
    assert got.dtype == want.dtype and np.array_equal(got, want)
    with pytest.raises(ValueError, match="interfaces"):
        level_rate_from_mass_flux(g["omega_half"][:-1], p_full=g["p_full"])


def _diagnostics(rec):
    from b200sht.semilag import LipschitzDiagnostics

    return LipschitzDiagnostics(
        dt_s=rec["semilag_lipschitz_dt_s"],
        reference_length_m=rec["semilag_lipschitz_reference_length_m"],
        lipschitz=rec["semilag_lipschitz"],
        lipschitz_frobenius=rec["semilag_lipschitz_frobenius"],
        lipschitz_horizontal=rec["semilag_lipschitz_horizontal"],
        jacobian_spectral_s=rec["semilag_jacobian_spectral_s"],
        jacobian_frobenius_s=rec["semilag_jacobian_frobenius_s"],
        jacobian_horizontal_s=rec["semilag_jacobian_horizontal_s"],
        lipschitz_vertical=rec["semilag_lipschitz_vertical"],
        jacobian_vertical_s=rec["semilag_jacobian_vertical_s"],
        lipschitz_mixed=rec["semilag_lipschitz_mixed"],
        lipschitz_balanced=rec["semilag_lipschitz_balanced"],
        jacobian_balanced_s=rec["semilag_jacobian_balanced_s"],
        fold_determinant_arrival=rec["semilag_fold_determinant_arrival"],
        fold_determinant_departure=rec["semilag_fold_determinant_departure"],
        fold_where_arrival=rec["fold_where_arrival"],
        fold_where_departure=rec["fold_where_departure"])


def test_fold_refusal_is_the_reference_s():
    from b200sht.semilag import refuse_trajectory_fold

    g = load_golden("lipschitz_f64.npz")
    cases = json.loads(str(g["cases"]))
    d = _diagnostics(cases["whole_long_ex"])
    keys = {k: v for k, v in cases["whole_long_ex"].items() if k.startswith("semilag_")}
    assert d.as_dict() == keys
    with pytest.raises(ValueError) as err:
        refuse_trajectory_fold(d, float(g["refusal_floor"]))
    assert str(err.value) == str(g["refusal"])
    refuse_trajectory_fold(_diagnostics(cases["whole_short_ex"]), 0.2)
    with pytest.raises(ValueError, match="must lie in"):
        refuse_trajectory_fold(d, 1.0)
    assert d.fold_side == "arrival" and d.binding_direction in ("horizontal", "coupling")


def test_convergence_refusal():
    from b200sht.semilag import TrajectoryDiagnostics, convergence

    diag = TrajectoryDiagnostics(3, 300.0, 120.0, 0.02, 0.0, 1e4, 1.0, 0.5)
    convergence(diag, 0.05)
    with pytest.raises(ValueError, match="did not converge: the last of 3 iterations"):
        convergence(diag, 0.01)

"""The deformation diagnostic of the trajectory on the GPU (sht_sl_lipschitz).

Against the reference's recorded diagnostics (tests/golden/make_golden_lipschitz.py:
whole grid with and without an extrapolated wind, two time steps, a reference
length, two latitude bands with their extrapolated band windows) and against
the oracle on a larger seeded grid.  The kernel evaluates the reference's
expressions without fused multiply-adds, so the numbers differ from the
reference's only through the last bits of sin, cos and acos: FP64 within
1e-12, FP32 within 2e-6 relative; the location of each minimum is the
reference's.  The fold refusal built from the GPU's numbers is the
reference's message word for word.
"""
from __future__ import annotations

import json

import numpy as np
import pytest
import torch

from conftest import load_golden

pytestmark = pytest.mark.gpu

TAGS = ["f64", "f32"]


class _Grid:
    def __init__(self, lat, nlon, radius):
        self.nlat, self.nlon = len(lat), int(nlon)
        self.lat_rad = lat
        self.lon_rad = np.arange(nlon) * 2 * np.pi / nlon
        self.radius_m = radius


def _setup(tag):
    from b200sht.semilag import SphericalGridTables

    g = load_golden(f"lipschitz_{tag}.npz")
    dtype = torch.float64 if tag == "f64" else torch.float32
    tables = SphericalGridTables.create(_Grid(g["lat"], int(g["nlon"]), float(g["radius_m"])),
                                        dtype=dtype)
    return g, tables, dtype


def _flow(arrs, rows, dtype):
    from b200sht.semilag import CartesianWind

    s0, s1 = rows
    return CartesianWind(*(torch.as_tensor(np.ascontiguousarray(f[:, s0:s1]), dtype=dtype,
                                           device="cuda") for f in arrs))


def _rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


@pytest.mark.parametrize("tag", TAGS)
def test_diagnostics_match_the_reference(tag):
    from b200sht.semilag import lipschitz, refuse_trajectory_fold

    g, tables, dtype = _setup(tag)
    want_all = json.loads(str(g["cases"]))
    nlat = tables.nlat
    tol = 1e-12 if tag == "f64" else 2e-6
    whole = (0, nlat)
    specs = {
        "whole_long": (float(g["dt_long"]), whole, whole, False, None),
        "whole_long_ex": (float(g["dt_long"]), whole, whole, True, None),
        "whole_short_ex": (float(g["dt_short"]), whole, whole, True, None),
        "whole_chunk2": (float(g["dt_long"]), whole, whole, False, None),
        "whole_lref": (float(g["dt_short"]), whole, whole, False, 25_000.0),
        "band_south": (float(g["dt_long"]), (0, 11), (0, 8), False, None),
        "band_south_ex": (float(g["dt_long"]), (0, 11), (0, 8), True, None),
        "band_mid": (float(g["dt_long"]), (9, 23), (12, 20), False, None),
        "band_mid_ex": (float(g["dt_long"]), (9, 23), (12, 20), True, None),
    }
    got_all = {}
    for name, (dt, src, arr, has_ex, lref) in specs.items():
        kw = {}
        if src != whole:
            kw["window"] = tables.window(slice(*src), slice(*arr))
        if has_ex:
            ex_rows = whole if src == whole else (max(arr[0] - 1, 0), min(arr[1] + 1, nlat))
            kw["extrapolated"] = _flow(g["wind_ex"], ex_rows, dtype)
            if src != whole:
                kw["extrapolated_window"] = tables.window(slice(*ex_rows), slice(*arr))
        d = lipschitz(_flow(g["wind"], src, dtype), tables, dt, reference_length_m=lref,
                      level_chunk=2 if name == "whole_chunk2" else 8, **kw)
        got_all[name] = d
        want = want_all[name]
        for key, value in d.as_dict().items():
            assert _rel(value, want[key]) <= tol, (name, key, value, want[key])
        assert d.fold_where_departure == want["fold_where_departure"], name
        assert d.fold_where_arrival == want["fold_where_arrival"], name
    with pytest.raises(ValueError) as err:
        refuse_trajectory_fold(got_all["whole_long_ex"], float(g["refusal_floor"]))
    assert str(err.value) == str(g["refusal"])
    refuse_trajectory_fold(got_all["whole_short_ex"], 0.2)


@pytest.mark.parametrize("tag", TAGS)
def test_diagnostics_match_the_oracle_on_a_larger_grid(tag):
    from b200sht.semilag import CartesianWind, SphericalGridTables, lipschitz
    from oracle import sl_lipschitz as O

    nlat, nlon, nlev = 96, 192, 10
    lat = np.arcsin(np.polynomial.legendre.leggauss(nlat)[0])
    dtype_np = np.float64 if tag == "f64" else np.float32
    dtype = torch.float64 if tag == "f64" else torch.float32
    tables = SphericalGridTables.create(_Grid(lat, nlon, 6371220.0), dtype=dtype)
    lat_ext = tables.host_tables(4)["lat_ext"]
    wind = O.deforming_wind(lat, nlon, nlev, speed=30.0, noise=200.0, seed=21, dtype=dtype_np)
    ex = O.deforming_wind(lat, nlon, nlev, speed=35.0, noise=260.0, seed=22, dtype=dtype_np)
    tol = 1e-12 if tag == "f64" else 2e-6
    for dt in (900.0, 10800.0):
        want = O.lipschitz(wind, lat_ext, nlon, 6371220.0, dt, extrapolated=ex)
        d = lipschitz(CartesianWind(*(torch.as_tensor(f, device="cuda") for f in wind)), tables,
                      dt, extrapolated=CartesianWind(*(torch.as_tensor(f, device="cuda")
                                                       for f in ex)))
        assert _rel(d.jacobian_spectral_s, want["spectral"]) <= tol
        assert _rel(d.jacobian_frobenius_s, want["frobenius"]) <= tol
        assert _rel(d.jacobian_horizontal_s, want["horizontal"]) <= tol
        assert _rel(d.jacobian_vertical_s, want["vertical"]) <= tol
        assert _rel(d.jacobian_balanced_s, want["balanced"]) <= tol
        assert _rel(d.fold_determinant_departure, min(1.0, want["fold_departure"])) <= tol
        assert _rel(d.fold_determinant_arrival, min(1.0, want["fold_arrival"])) <= tol
        shape = want["shape"]
        assert d.fold_where_departure == O.where_text(want["where_departure"], shape, lat_ext,
                                                      nlon)
        assert d.fold_where_arrival == O.where_text(want["where_arrival"], shape, lat_ext, nlon)


def test_band_halo_escape_and_argument_checks():
    from b200sht.semilag import HaloEscape, lipschitz

    g, tables, dtype = _setup("f64")
    nlat = tables.nlat
    win = tables.window(slice(12, 20), slice(12, 20))  # no row either side of the band
    with pytest.raises(HaloEscape, match="outside the rows"):
        lipschitz(_flow(g["wind"], (12, 20), dtype), tables, 600.0, window=win)
    whole = _flow(g["wind"], (0, nlat), dtype)
    with pytest.raises(ValueError, match="rows were expected"):
        lipschitz(_flow(g["wind"], (0, nlat - 1), dtype), tables, 600.0)
    with pytest.raises(ValueError, match="reference_length_m"):
        lipschitz(whole, tables, 600.0, reference_length_m=-1.0)
    band = tables.window(slice(9, 23), slice(12, 20))
    with pytest.raises(ValueError, match="needs the window"):
        lipschitz(_flow(g["wind"], (9, 23), dtype), tables, 600.0, window=band,
                  extrapolated=_flow(g["wind_ex"], (11, 21), dtype))


def test_level_rate_on_the_device():
    from b200sht.semilag import level_rate_from_mass_flux

    g = load_golden("lipschitz_f64.npz")
    omega = torch.as_tensor(g["omega_half"], device="cuda")
    p_full = torch.as_tensor(g["p_full"], device="cuda")
    got = level_rate_from_mass_flux(omega, p_full=p_full)
    assert got.is_cuda and np.array_equal(got.cpu().numpy(), g["level_rate"])


def test_converged_departure_points_retries_then_refuses():
    from b200sht.semilag import (CartesianWind, MAXIMUM_TRAJECTORY_ITERATIONS,
                                 SphericalGridTables, converged_departure_points,
                                 departure_points)
    from oracle import sl_lipschitz as O

    nlat, nlon, nlev = 32, 64, 6
    lat = np.arcsin(np.polynomial.legendre.leggauss(nlat)[0])
    tables = SphericalGridTables.create(_Grid(lat, nlon, 6371220.0), dtype=torch.float64)
    wind = CartesianWind(*(torch.as_tensor(f, device="cuda") for f in
                           O.deforming_wind(lat, nlon, nlev, speed=40.0, noise=120.0, seed=3)))
    one, diag1 = departure_points(wind, tables, 3600.0, iterations=1)
    limit = 0.5 * diag1.move_max_cells  # the one-pass search misses it
    st, diag = converged_departure_points(wind, tables, 3600.0, iterations=1, limit_cells=limit)
    assert diag.iterations == MAXIMUM_TRAJECTORY_ITERATIONS and diag.move_max_cells <= limit
    ref, _ = departure_points(wind, tables, 3600.0, iterations=MAXIMUM_TRAJECTORY_ITERATIONS)
    assert torch.equal(st.phi, ref.phi) and torch.equal(st.xi, ref.xi)
    # converged at the configured count: the plain search's bits
    st3, d3 = converged_departure_points(wind, tables, 3600.0, iterations=1,
                                         limit_cells=2 * diag1.move_max_cells)
    assert d3.iterations == 1 and torch.equal(st3.phi, one.phi)
    with pytest.raises(ValueError, match="did not converge"):
        converged_departure_points(wind, tables, 3600.0, iterations=1, limit_cells=0.0)


@pytest.mark.parametrize("tag", TAGS)
def test_north_pole_band_against_the_oracle(tag):
    """A band that ends at the north pole (its rows beyond the pole are the
    pole row half a turn round), with an extrapolated band window, against
    the oracle; and a whole-grid call with a two-level grid (the vertical
    differences one-sided at both ends)."""
    from b200sht.semilag import lipschitz
    from oracle import sl_lipschitz as O

    g, tables, dtype = _setup(tag)
    nlat, nlon = tables.nlat, tables.nlon
    lat_ext = tables.host_tables(4)["lat_ext"]
    tol = 1e-12 if tag == "f64" else 2e-6
    src, arr, ex_rows = (21, nlat), (24, nlat), (23, nlat)
    wind = [f[:, src[0]:src[1]] for f in g["wind"]]
    ex = [f[:, ex_rows[0]:ex_rows[1]] for f in g["wind_ex"]]
    want = O.lipschitz(wind, lat_ext, nlon, float(g["radius_m"]), float(g["dt_long"]),
                       extrapolated=ex, held=src, arrival=arr, extrapolated_held=ex_rows)
    d = lipschitz(_flow(g["wind"], src, dtype), tables, float(g["dt_long"]),
                  window=tables.window(slice(*src), slice(*arr)),
                  extrapolated=_flow(g["wind_ex"], ex_rows, dtype),
                  extrapolated_window=tables.window(slice(*ex_rows), slice(*arr)))
    assert _rel(d.jacobian_spectral_s, want["spectral"]) <= tol
    assert _rel(d.jacobian_balanced_s, want["balanced"]) <= tol
    assert _rel(d.jacobian_vertical_s, want["vertical"]) <= tol
    assert _rel(d.fold_determinant_departure, min(1.0, want["fold_departure"])) <= tol
    assert _rel(d.fold_determinant_arrival, min(1.0, want["fold_arrival"])) <= tol
    assert d.fold_where_arrival == O.where_text(want["where_arrival"], want["shape"], lat_ext,
                                                nlon, arr[0])
    two = [f[:2] for f in g["wind"]]
    want2 = O.lipschitz(two, lat_ext, nlon, float(g["radius_m"]), 600.0)
    from b200sht.semilag import CartesianWind

    d2 = lipschitz(CartesianWind(*(torch.as_tensor(np.ascontiguousarray(f), dtype=dtype,
                                                   device="cuda") for f in two)), tables, 600.0)
    assert _rel(d2.jacobian_vertical_s, want2["vertical"]) <= tol
    assert _rel(d2.fold_determinant_departure, min(1.0, want2["fold_departure"])) <= tol

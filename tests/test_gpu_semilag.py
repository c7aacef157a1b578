"""The semi-Lagrangian gathers on the GPU (sht_sl_gather, sht_sl_gather_linear)
against the reference's recorded outputs and against the oracle.

Tolerances: float64 1e-12 of the field's range; float32 4e-6 of it (the
kernel contracts a*b+c into FMAs where numpy rounds twice, and the
meridional weights' normalisation is a reciprocal multiply against numpy's
division)."""
from __future__ import annotations

import types

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

CASES = [("cubic_qm", 4, "quasi_monotone", False), ("cubic_qm_deficit", 4, "quasi_monotone", True),
         ("cubic_none", 4, "none", False), ("quintic_qm", 6, "quasi_monotone", False),
         ("quintic_none", 6, "none", False)]
TOL = {"f64": 1e-12, "f32": 4e-6}
DT = {"f64": torch.float64, "f32": torch.float32}


def _grid(lat, nlon):
    lat = np.asarray(lat, np.float64)
    return types.SimpleNamespace(nlat=lat.shape[0], nlon=int(nlon), lat_rad=lat,
                                 lon_rad=np.arange(nlon) * 2 * np.pi / nlon, radius_m=6371220.0)


def _setup(g, tag):
    from b200sht.semilag import SphericalGridTables, Stencil

    tables = SphericalGridTables.create(_grid(g["lat"], g["nlon"]), dtype=DT[tag])
    dev = lambda a: torch.as_tensor(a, device="cuda")
    st = Stencil(xi=dev(g["xi"]), phi=dev(g["phi"]), level=dev(g["level"]), tables=tables)
    fields = [dev(f) for f in g["fields"]]
    return tables, st, fields


def _close(got, want, tag, scale=None):
    """max |got - want| within TOL of the range of `scale` (default: want)."""
    got = got.cpu().numpy() if isinstance(got, torch.Tensor) else got
    ref = want if scale is None else scale
    rng = max(float(np.max(ref) - np.min(ref)), 1e-300)
    err = float(np.max(np.abs(got - want))) / rng
    assert err <= TOL[tag], err


@pytest.mark.parametrize("tag", ["f64", "f32"])
@pytest.mark.parametrize("order", [4, 6])
def test_tables_match_reference(golden, tag, order):
    g = golden(f"sl_gather_{tag}.npz")
    tables, _, _ = _setup(g, tag)
    t = tables.host_tables(order)
    for key in ("lat_ext", "mrden", "rowoff", "rowshift", "mlut"):
        np.testing.assert_array_equal(t[key], g[f"{key}{order}"].reshape(t[key].shape))


@pytest.mark.parametrize("tag", ["f64", "f32"])
@pytest.mark.parametrize("name,order,limiter,deficit", CASES)
def test_gather_matches_reference(golden, tag, name, order, limiter, deficit):
    from b200sht.semilag import gather_batch

    g = golden(f"sl_gather_{tag}.npz")
    _, st, fields = _setup(g, tag)
    out = gather_batch(fields, st, monotone=limiter, deficit=deficit, order=order)
    torch.cuda.synchronize()
    for i, item in enumerate(out):
        if deficit:
            _close(item[0], g[name][i], tag)
            # the deficit to the same absolute accuracy as the values
            _close(item[1], g[name + "_cut"][i], tag, scale=g[name][i])
        else:
            _close(item, g[name][i], tag)


@pytest.mark.parametrize("tag", ["f64", "f32"])
def test_linear_matches_reference(golden, tag):
    from b200sht.semilag import gather_linear_batch

    g = golden(f"sl_gather_{tag}.npz")
    _, st, fields = _setup(g, tag)
    for i, v in enumerate(gather_linear_batch(fields, st)):
        _close(v, g["linear"][i], tag)


@pytest.mark.parametrize("tag", ["f64", "f32"])
@pytest.mark.parametrize("order", [4, 6])
@pytest.mark.parametrize("limiter", ["quasi_monotone", "none"])
def test_larger_grid_against_oracle(tag, order, limiter):
    """A 48 x 96 grid, 8 levels, 3 fields, departure points up to 3 cells
    away (past both poles and into both half layers), against the oracle."""
    from b200sht.semilag import SphericalGridTables, Stencil, gather_batch
    from oracle import sl_gather as O

    nlat, nlon, nlev = 48, 96, 8
    lat = np.sort(np.arcsin(np.polynomial.legendre.leggauss(nlat)[0]))
    dtype = np.float64 if tag == "f64" else np.float32
    xi, phi, level = O.departure_sample(nlev, lat, nlon, 7, cells=3.0, dtype=dtype)
    rng = np.random.default_rng(3)
    fields = [rng.standard_normal((nlev, nlat, nlon)).astype(dtype) for _ in range(3)]
    tables = SphericalGridTables.create(_grid(lat, nlon), dtype=DT[tag])
    dev = lambda a: torch.as_tensor(a, device="cuda")
    st = Stencil(xi=dev(xi), phi=dev(phi), level=dev(level), tables=tables)
    got = gather_batch([dev(f) for f in fields], st, monotone=limiter, order=order, batch=2)
    want = O.gather(fields, xi, phi, level, lat, nlon, order=order, limiter=limiter, dtype=dtype)
    for a, b in zip(got, want):
        _close(a, b, tag)


@pytest.mark.parametrize("tag", ["f64", "f32"])
@pytest.mark.parametrize("order", [4, 6])
@pytest.mark.parametrize("limiter", ["quasi_monotone", "none"])
def test_zero_displacement_is_the_identity(tag, order, limiter):
    """Every weight set is normalised, so a point that departs from itself
    reads its own value exactly, polar rows and boundary levels included."""
    from b200sht.semilag import SphericalGridTables, gather, gather_linear_batch, zero_stencil

    nlat, nlon, nlev = 16, 32, 6
    lat = np.sort(np.arcsin(np.polynomial.legendre.leggauss(nlat)[0]))
    tables = SphericalGridTables.create(_grid(lat, nlon), dtype=DT[tag])
    st = zero_stencil(tables, nlev)
    f = torch.randn((nlev, nlat, nlon), dtype=DT[tag], device="cuda")
    assert torch.equal(gather(f, st, monotone=limiter, order=order), f)
    assert torch.equal(gather_linear_batch([f], st)[0], f)


def test_batches_and_single_fields_agree(golden):
    from b200sht.semilag import gather, gather_batch

    g = golden("sl_gather_f64.npz")
    _, st, fields = _setup(g, "f64")
    many = gather_batch(fields * 3, st, batch=4)
    one = [gather(f, st) for f in fields * 3]
    for a, b in zip(many, one):
        assert torch.equal(a, b)


def test_errors_name_the_reason(golden):
    from b200sht.semilag import SphericalGridTables, Stencil, gather_batch

    g = golden("sl_gather_f64.npz")
    tables, st, fields = _setup(g, "f64")
    with pytest.raises(ValueError, match="limiter must be one of"):
        gather_batch(fields, st, monotone="positive_definite")
    with pytest.raises(ValueError, match="horizontal order must be one of"):
        gather_batch(fields, st, order=5)
    with pytest.raises(ValueError, match="unlimited gather has none"):
        gather_batch(fields, st, monotone=False, deficit=True)
    with pytest.raises(ValueError, match="cubic gather only"):
        gather_batch(fields, st, deficit=True, order=6)
    with pytest.raises(ValueError, match="where the stencil reads"):
        gather_batch([fields[0][:, :, :-2]], st)
    with pytest.raises(ValueError, match="mixed-precision"):
        gather_batch([fields[0].float()], st)
    with pytest.raises(ValueError, match="nlev >= 4"):
        Stencil(xi=st.xi[:3], phi=st.phi[:3], level=st.level[:3], tables=tables)
    with pytest.raises(ValueError, match="nlon must be even"):
        SphericalGridTables.create(_grid(g["lat"], 25))
    with pytest.raises(ValueError, match="strictly ascending"):
        SphericalGridTables.create(_grid(g["lat"][::-1], 24))


@pytest.mark.parametrize("tag", ["f64", "f32"])
def test_departure_search_matches_reference(golden, tag):
    """The fixed-point search (3 iterations, a rotation across both poles)
    against the reference's recorded departure points and diagnostics."""
    from b200sht.semilag import CartesianWind, departure_points

    g = golden(f"sl_gather_{tag}.npz")
    tables, _, _ = _setup(g, tag)
    dev = lambda a: torch.as_tensor(a, device="cuda")
    st, diag = departure_points(CartesianWind(*[dev(w) for w in g["wind"]]), tables,
                                float(g["dt"]), iterations=3,
                                extrapolated=CartesianWind(*[dev(w) for w in g["wind_ex"]]))
    tol = 1e-12 if tag == "f64" else 2e-6
    # positions: radians of latitude, zonal index (2 pi / 24 radians each), levels
    assert np.max(np.abs(st.phi.cpu().numpy() - g["dep_phi"])) < tol * 4
    dxi = np.abs(st.xi.cpu().numpy() - g["dep_xi"])
    assert np.max(np.minimum(dxi, 24 - dxi)) < tol * 24
    assert np.max(np.abs(st.level.cpu().numpy() - g["dep_level"])) < tol * 8
    got = np.array([diag.move_max_m, diag.move_max_cells, diag.move_max_levels,
                    diag.displacement_max_m, diag.displacement_max_cells,
                    diag.displacement_max_levels])
    # the last move is a small difference of unit vectors: loose in float32
    rel = 1e-9 if tag == "f64" else 5e-2
    np.testing.assert_allclose(got[3:], g["dep_diag"][3:], rtol=1e-9 if tag == "f64" else 1e-5)
    np.testing.assert_allclose(got[:3], g["dep_diag"][:3], rtol=rel)


@pytest.mark.parametrize("tag", ["f64", "f32"])
def test_departure_search_against_oracle_and_gather(tag):
    """48 x 96 x 8 against the oracle, then the gather reads the result."""
    from b200sht.semilag import (CartesianWind, SphericalGridTables, departure_points,
                                 gather_batch)
    from oracle import sl_gather as O

    nlat, nlon, nlev = 48, 96, 8
    lat = np.sort(np.arcsin(np.polynomial.legendre.leggauss(nlat)[0]))
    dtype = np.float64 if tag == "f64" else np.float32
    wind = O.rotation_wind(lat, nlon, nlev, speed=60.0, seed=4, dtype=dtype)
    tables = SphericalGridTables.create(_grid(lat, nlon), dtype=DT[tag])
    dev = lambda a: torch.as_tensor(a, device="cuda")
    st, diag = departure_points(CartesianWind(*[dev(w) for w in wind]), tables, 900.0,
                                iterations=4)
    xi, phi, lev, _, _ = O.departure(wind, lat, nlon, 900.0, iterations=4, dtype=dtype)
    tol = 1e-12 if tag == "f64" else 2e-6
    assert np.max(np.abs(st.phi.cpu().numpy() - phi)) < tol * 4
    dxi = np.abs(st.xi.cpu().numpy() - xi)
    assert np.max(np.minimum(dxi, nlon - dxi)) < tol * nlon
    assert np.max(np.abs(st.level.cpu().numpy() - lev)) < tol * nlev
    assert diag.move_max_cells < 1e-3 and diag.displacement_max_cells > 0.1
    f = torch.randn((nlev, nlat, nlon), dtype=DT[tag], device="cuda")
    assert torch.isfinite(gather_batch([f], st)[0]).all()


def test_departure_errors_and_rest_state():
    from b200sht.semilag import CartesianWind, SphericalGridTables, departure_points

    nlat, nlon, nlev = 16, 32, 5
    lat = np.sort(np.arcsin(np.polynomial.legendre.leggauss(nlat)[0]))
    tables = SphericalGridTables.create(_grid(lat, nlon), dtype=torch.float64)
    zero = torch.zeros((nlev, nlat, nlon), dtype=torch.float64, device="cuda")
    wind = CartesianWind(zero, zero, zero, zero)
    st, diag = departure_points(wind, tables, 300.0)
    # a resting atmosphere departs from its arrival point
    assert torch.max(torch.abs(st.phi - torch.as_tensor(lat, device="cuda")[None, :, None])) < 1e-14
    xi = st.xi.cpu().numpy() % nlon
    dxi = np.abs(xi - np.arange(nlon)[None, None, :])
    assert np.max(np.minimum(dxi, nlon - dxi)) < 1e-12
    assert diag.displacement_max_m < 1e-6 and diag.move_max_m == 0.0
    with pytest.raises(ValueError, match="at least one iteration"):
        departure_points(wind, tables, 300.0, iterations=0)
    with pytest.raises(ValueError, match="must be one of"):
        departure_points(wind, tables, 300.0, solver="rk4")
    with pytest.raises(ValueError, match="must all be"):
        departure_points(wind, tables, 300.0,
                         extrapolated=CartesianWind(zero[:4], zero, zero, zero))


@pytest.mark.parametrize("tag", ["f64", "f32"])
def test_newton_search_reaches_the_fixed_point(tag):
    """Newton's method and the fixed-point pass solve one equation: a long
    fixed-point run and a short Newton run on a rotation across both poles
    (900 s steps, 48 x 96 x 8) agree, and Newton's last move is small."""
    from b200sht.semilag import CartesianWind, SphericalGridTables, departure_points
    from oracle import sl_gather as O

    nlat, nlon, nlev = 48, 96, 8
    lat = np.sort(np.arcsin(np.polynomial.legendre.leggauss(nlat)[0]))
    dtype = np.float64 if tag == "f64" else np.float32
    wind = O.rotation_wind(lat, nlon, nlev, speed=60.0, seed=4, dtype=dtype)
    tables = SphericalGridTables.create(_grid(lat, nlon), dtype=DT[tag])
    w = CartesianWind(*[torch.as_tensor(a, device="cuda") for a in wind])
    fp, _ = departure_points(w, tables, 900.0, iterations=30)
    nt, diag = departure_points(w, tables, 900.0, iterations=6, solver="newton")
    tol = 1e-9 if tag == "f64" else 2e-5
    assert float((nt.phi - fp.phi).abs().max()) < tol
    dxi = (nt.xi - fp.xi).abs().cpu().numpy()
    assert np.max(np.minimum(dxi, nlon - dxi)) < tol * nlon
    assert float((nt.level - fp.level).abs().max()) < tol * nlev
    assert diag.move_max_cells < (1e-6 if tag == "f64" else 1e-3)


@pytest.mark.parametrize("tag", ["f64", "f32"])
def test_line_search_newton_reaches_the_fixed_point(tag):
    """The line-search Newton form solves the same equation: on the rotation
    across both poles (900 s, 48 x 96 x 8) six iterations land on the point
    thirty fixed-point iterations reach, to within its own stopping gate (a
    residual of 1e-4 meridional grid lengths), and its reported step at the
    returned point is below the gate as well."""
    from b200sht.semilag import CartesianWind, SphericalGridTables, departure_points
    from oracle import sl_gather as O

    nlat, nlon, nlev = 48, 96, 8
    lat = np.sort(np.arcsin(np.polynomial.legendre.leggauss(nlat)[0]))
    dtype = np.float64 if tag == "f64" else np.float32
    wind = O.rotation_wind(lat, nlon, nlev, speed=60.0, seed=4, dtype=dtype)
    tables = SphericalGridTables.create(_grid(lat, nlon), dtype=DT[tag])
    w = CartesianWind(*[torch.as_tensor(a, device="cuda") for a in wind])
    fp, _ = departure_points(w, tables, 900.0, iterations=30)
    ls, diag = departure_points(w, tables, 900.0, iterations=6, solver="newton_ls")
    gate = 1e-4 * np.pi / nlat  # the stopping residual, radians
    tol = 2 * gate if tag == "f64" else 2 * gate + 2e-5
    def unit(st):
        lam = st.xi.double() * (2 * np.pi / nlon)
        ph = st.phi.double()
        return torch.stack([ph.cos() * lam.cos(), ph.cos() * lam.sin(), ph.sin()])

    # the great-circle distance between the two answers (chord ~ arc here)
    assert float((unit(ls) - unit(fp)).norm(dim=0).max()) < tol
    assert float((ls.level - fp.level).abs().max()) < (2e-4 if tag == "f64" else 1e-3)
    assert diag.move_max_cells < (2e-4 if tag == "f64" else 1e-3)


def test_line_search_newton_on_a_strongly_deforming_flow():
    """Where (dt/2)|J| nears one (a rough 150 m/s flow at a 3600 s step on a
    coarse grid) the fixed-point pass stops contracting and the full Newton
    step cycles between cells; the line-search form keeps the residual of
    the departure equation falling.  Measured independently of the search
    kernels (the oracle's float64 residual |G(q) - q| at the returned
    points), after the same four iterations: the line-search form's mean
    residual is below both others', and its 90th percentile too."""
    from b200sht.semilag import CartesianWind, SphericalGridTables, departure_points
    from oracle import sl_gather as O

    nlat, nlon, nlev = 32, 64, 6
    lat = np.sort(np.arcsin(np.polynomial.legendre.leggauss(nlat)[0]))
    rng = np.random.default_rng(8)
    base = O.rotation_wind(lat, nlon, nlev, speed=60.0, seed=3)
    wind = [base[i] + 150.0 * rng.standard_normal(base[i].shape) for i in range(3)]
    wind.append(base[3] + 2e-4 * rng.standard_normal(base[3].shape))
    tables = SphericalGridTables.create(_grid(lat, nlon), dtype=torch.float64)
    w = CartesianWind(*[torch.as_tensor(a, device="cuda") for a in wind])
    stats = {}
    for solver in ("fixed_point", "newton", "newton_ls"):
        st, _ = departure_points(w, tables, 3600.0, iterations=4, solver=solver)
        cells, levels = O.departure_residual(wind, lat, nlon, 3600.0, st.xi.cpu().numpy(),
                                             st.phi.cpu().numpy(), st.level.cpu().numpy())
        r = np.sqrt(cells ** 2 + levels ** 2).ravel()
        stats[solver] = (float(np.mean(r)), float(np.percentile(r, 90)))
    ls = stats["newton_ls"]
    for other in ("fixed_point", "newton"):
        assert ls[0] < stats[other][0], stats
        assert ls[1] < stats[other][1], stats


def _band_case(tag, seed=5):
    from b200sht.semilag import SphericalGridTables, Stencil
    from oracle import sl_gather as O

    nlat, nlon, nlev = 32, 64, 6
    lat = np.sort(np.arcsin(np.polynomial.legendre.leggauss(nlat)[0]))
    dtype = np.float64 if tag == "f64" else np.float32
    xi, phi, level = O.departure_sample(nlev, lat, nlon, seed, cells=1.5, dtype=dtype)
    tables = SphericalGridTables.create(_grid(lat, nlon), dtype=DT[tag])
    dev = lambda a: torch.as_tensor(a, device="cuda")
    whole = Stencil(xi=dev(xi), phi=dev(phi), level=dev(level), tables=tables)
    f = [torch.randn((nlev, nlat, nlon), dtype=DT[tag], device="cuda") for _ in range(3)]
    return tables, whole, f


@pytest.mark.parametrize("tag", ["f64", "f32"])
@pytest.mark.parametrize("order", [4, 6])
@pytest.mark.parametrize("rows", [(0, 8), (12, 20), (26, 32)])
def test_band_gather_is_the_whole_grid_gather(tag, order, rows):
    """A band's gather from fields holding only the band and a 5-row halo
    returns the whole-grid values of its rows bit for bit (poles included)."""
    from b200sht.semilag import Stencil, gather_batch

    tables, whole, f = _band_case(tag)
    a0, a1 = rows
    s0, s1 = max(0, a0 - 5), min(32, a1 + 5)
    win = tables.window(slice(s0, s1), slice(a0, a1))
    band = Stencil(xi=whole.xi[:, a0:a1].contiguous(), phi=whole.phi[:, a0:a1].contiguous(),
                   level=whole.level[:, a0:a1].contiguous(), tables=tables, window=win)
    want = gather_batch(f, whole, order=order, deficit=order == 4)
    got = gather_batch([x[:, s0:s1].contiguous() for x in f], band, order=order,
                       deficit=order == 4)
    for g, w in zip(got, want):
        if order == 4:
            assert torch.equal(g[0], w[0][:, a0:a1]) and torch.equal(g[1], w[1][:, a0:a1])
        else:
            assert torch.equal(g, w[:, a0:a1])


def test_band_escape_is_refused_by_name():
    from b200sht.semilag import HaloEscape, Stencil, gather_batch, gather_linear_batch

    tables, whole, f = _band_case("f64")
    win = tables.window(slice(12, 20), slice(12, 20))  # no halo: stencils leave the band
    band = Stencil(xi=whole.xi[:, 12:20].contiguous(), phi=whole.phi[:, 12:20].contiguous(),
                   level=whole.level[:, 12:20].contiguous(), tables=tables, window=win)
    src = [x[:, 12:20].contiguous() for x in f]
    with pytest.raises(HaloEscape, match="outside the rows 12..20"):
        gather_batch(src, band)
    gather_batch(src, band, defer_escape=True)  # the flag is left for the caller
    with pytest.raises(HaloEscape):
        win.raise_if_escaped("gather")
    win.clear_escape()
    win.raise_if_escaped("gather")
    with pytest.raises(ValueError, match="whole stencil"):
        gather_linear_batch(src, band)
    with pytest.raises(ValueError, match="computed rows must lie inside"):
        tables.window(slice(4, 10), slice(2, 8))


@pytest.mark.parametrize("tag", ["f64", "f32"])
@pytest.mark.parametrize("solver", ["fixed_point", "newton", "newton_ls"])
def test_band_departure_search_is_the_whole_grid_search(tag, solver):
    from b200sht.semilag import CartesianWind, SphericalGridTables, departure_points
    from oracle import sl_gather as O

    nlat, nlon, nlev = 32, 64, 6
    lat = np.sort(np.arcsin(np.polynomial.legendre.leggauss(nlat)[0]))
    dtype = np.float64 if tag == "f64" else np.float32
    wind = [torch.as_tensor(a, device="cuda")
            for a in O.rotation_wind(lat, nlon, nlev, speed=60.0, seed=2, dtype=dtype)]
    tables = SphericalGridTables.create(_grid(lat, nlon), dtype=DT[tag])
    whole, _ = departure_points(CartesianWind(*wind), tables, 900.0, solver=solver)
    for a0, a1 in ((0, 6), (13, 19), (27, 32)):
        s0, s1 = max(0, a0 - 4), min(nlat, a1 + 4)
        win = tables.window(slice(s0, s1), slice(a0, a1))
        band, diag = departure_points(CartesianWind(*[w[:, s0:s1].contiguous() for w in wind]),
                                      tables, 900.0, window=win, solver=solver)
        assert band.shape == (nlev, a1 - a0, nlon) and band.window is win
        for x, y in ((band.xi, whole.xi), (band.phi, whole.phi), (band.level, whole.level)):
            assert torch.equal(x, y[:, a0:a1])
        assert np.isfinite(diag.displacement_max_m)

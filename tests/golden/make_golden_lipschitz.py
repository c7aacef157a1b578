"""Record the reference's trajectory deformation diagnostics.

Run in the build container, where the reference source tree is mounted:

    python tests/golden/make_golden_lipschitz.py <reference checkout>

It builds the reference's grid tables (``semilag.tables.SphericalGridTables``)
on the numpy backend and runs ``semilag.trajectory.lipschitz`` on seeded
winds of a 32 x 64 Gaussian grid with 6 levels, float64 and float32:

* a strongly deforming wind alone and with an extrapolated wind (the arrival
  side reading it), at a six-hour step whose determinants come down to 0.24
  (``refuse_trajectory_fold`` with a floor of 0.3 refuses it, and the
  message is recorded), and at a short step that the default floor passes;
* two latitude bands (one touching the south pole, one interior) with
  their halo windows, and the extrapolated band window holding one row
  either side;
* a chunk of two levels (``level_chunk = 2``), which must not change the
  numbers;

and ``level_rate_from_mass_flux`` on a seeded interface mass flux.  It
writes ``lipschitz_f64.npz`` / ``lipschitz_f32.npz``: the inputs, the
grid's extended latitudes and each case's diagnostics (``as_dict`` plus the
two ``fold_where`` strings).
"""
from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

NLAT, NLON, NLEV = 32, 64, 6
DT_LONG, DT_SHORT = 21600.0, 600.0
REFUSAL_FLOOR = 0.3  # above the long step's smallest determinant (0.24)


def _record(d):
    out = {k: float(v) for k, v in d.as_dict().items()}
    out["fold_where_arrival"] = d.fold_where_arrival
    out["fold_where_departure"] = d.fold_where_departure
    return out


def main(ref_root: str) -> None:
    os.environ.setdefault("ARWEN_GLOBAL_LEGENDRE_CACHE", "off")
    sys.path.insert(0, str(Path(ref_root) / "src"))
    from arwen_global.semilag.tables import SphericalGridTables
    from arwen_global.semilag.trajectory import (
        CartesianWind, level_rate_from_mass_flux, lipschitz, refuse_trajectory_fold)
    from arwen_global.spectral.grid import GaussianGrid

    from oracle.sl_lipschitz import deforming_wind

    grid = GaussianGrid.create(20, nlat=NLAT, nlon=NLON)
    lat = np.asarray(grid.lat_rad, dtype=np.float64)
    for dtype, tag in ((np.float64, "f64"), (np.float32, "f32")):
        tables = SphericalGridTables.create(grid, xp=np, dtype=dtype)
        wind = deforming_wind(lat, NLON, NLEV, seed=5, dtype=dtype)
        ex = deforming_wind(lat, NLON, NLEV, speed=55.0, noise=150.0, seed=6, dtype=dtype)
        cases = {}
        cases["whole_long"] = lipschitz(CartesianWind(*wind), tables, DT_LONG)
        cases["whole_long_ex"] = lipschitz(CartesianWind(*wind), tables, DT_LONG,
                                           extrapolated=CartesianWind(*ex))
        cases["whole_short_ex"] = lipschitz(CartesianWind(*wind), tables, DT_SHORT,
                                            extrapolated=CartesianWind(*ex))
        cases["whole_chunk2"] = lipschitz(CartesianWind(*wind), tables, DT_LONG,
                                          level_chunk=2)
        cases["whole_lref"] = lipschitz(CartesianWind(*wind), tables, DT_SHORT,
                                        reference_length_m=25_000.0)
        bands = {"band_south": (slice(0, 11), slice(0, 8)),
                 "band_mid": (slice(9, 23), slice(12, 20))}
        for name, (source, arrival) in bands.items():
            win = tables.window(source, arrival)
            held = CartesianWind(*(f[:, source] for f in wind))
            ex_src = slice(max(arrival.start - 1, 0), min(arrival.stop + 1, NLAT))
            ex_win = tables.window(ex_src, arrival)
            ex_held = CartesianWind(*(f[:, ex_src] for f in ex))
            cases[name] = lipschitz(held, tables, DT_LONG, window=win)
            cases[name + "_ex"] = lipschitz(held, tables, DT_LONG, window=win,
                                            extrapolated=ex_held, extrapolated_window=ex_win)
        refusal = ""
        try:
            refuse_trajectory_fold(cases["whole_long_ex"], REFUSAL_FLOOR)
        except ValueError as exc:
            refusal = str(exc)
        refuse_trajectory_fold(cases["whole_short_ex"], 0.2)  # passes
        rng = np.random.default_rng(8)
        p_half = np.sort(rng.uniform(100.0, 100_000.0, (NLEV + 1, 4, 5)), axis=0)
        p_full = np.sqrt(p_half[:-1] * p_half[1:])  # (nlev, 4, 5): a pressure per column
        omega = rng.standard_normal((NLEV + 1, 4, 5)) * 0.5
        omega[0] = omega[-1] = 0.0
        rate = level_rate_from_mass_flux(omega.astype(dtype), p_full=p_full.astype(dtype))
        np.savez_compressed(
            HERE / f"lipschitz_{tag}.npz",
            lat=lat, lat_ext=tables.lat_ext_host, nlon=np.int64(NLON),
            radius_m=np.float64(tables.radius_m), dt_long=np.float64(DT_LONG),
            dt_short=np.float64(DT_SHORT), wind=np.stack(wind), wind_ex=np.stack(ex),
            cases=json.dumps({k: _record(v) for k, v in cases.items()}),
            refusal=refusal, refusal_floor=np.float64(REFUSAL_FLOOR),
            omega_half=omega.astype(dtype), p_full=p_full.astype(dtype),
            level_rate=rate)
        print("wrote", HERE / f"lipschitz_{tag}.npz")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path to the reference checkout>")
    main(sys.argv[1])

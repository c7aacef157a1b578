"""Record golden vectors of the semi-Lagrangian gathers from the reference.

Run in the build container, where the reference source tree is mounted:

    python tests/golden/make_golden_sl.py <reference checkout>

It builds the reference's own grid tables
(``arwen_global.semilag.tables.SphericalGridTables``) and runs its
``gather_batch`` and ``gather_linear_batch``
(``arwen_global.semilag.interpolate``) on the numpy backend -- the numpy
specification the reference grades its CUDA gather against -- on seeded
departure points of a small Gaussian grid, and writes
``tests/golden/sl_gather_f64.npz`` and ``sl_gather_f32.npz``: the inputs,
every table of both stencil widths and the outputs of each (order, limiter,
deficit) case; and ``trajectory.departure_points`` (fixed point, three
iterations) on a solid-body rotation across both poles, with its
diagnostics.  The departure points reach past both poles (rows next to a
pole displaced by up to 1.5 rows) and into the half layers above the top
and below the bottom full level.
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

NLAT, NLON, NLEV, SEED = 12, 24, 5, 20261203
DT = 1800.0  # s: the rotation moves about 0.6 cells per step on this grid

#: (name, order, limiter, deficit)
CASES = [
    ("cubic_qm", 4, "quasi_monotone", False),
    ("cubic_qm_deficit", 4, "quasi_monotone", True),
    ("cubic_none", 4, "none", False),
    ("quintic_qm", 6, "quasi_monotone", False),
    ("quintic_none", 6, "none", False),
]


def main(ref_root: str) -> None:
    os.environ.setdefault("ARWEN_GLOBAL_LEGENDRE_CACHE", "off")
    sys.path.insert(0, str(Path(ref_root) / "src"))
    from arwen_global.semilag.interpolate import Stencil, gather_batch, gather_linear_batch
    from arwen_global.semilag.tables import SphericalGridTables
    from arwen_global.semilag.trajectory import CartesianWind, departure_points
    from arwen_global.spectral.grid import GaussianGrid

    from oracle.sl_gather import departure_sample, rotation_wind

    grid = GaussianGrid.create(7, nlat=NLAT, nlon=NLON)
    lat = np.asarray(grid.lat_rad, dtype=np.float64)
    rng = np.random.default_rng(SEED + 1)
    shape = (NLEV, NLAT, NLON)
    lon = np.arange(NLON) * 2 * np.pi / NLON
    smooth = (np.cos(lat)[None, :, None] * np.sin(3 * lon)[None, None, :]
              + 0.3 * np.arange(NLEV)[:, None, None])
    fields = [smooth + 0.2 * rng.standard_normal(shape), np.abs(rng.standard_normal(shape))]
    for dtype, tag in ((np.float64, "f64"), (np.float32, "f32")):
        tables = SphericalGridTables.create(grid, xp=np, dtype=dtype)
        xi, phi, level = departure_sample(NLEV, lat, NLON, SEED, dtype=dtype)
        st = Stencil(xi=xi, phi=phi, level=level, tables=tables)
        src = [f.astype(dtype) for f in fields]
        rec = {"lat": lat, "xi": xi, "phi": phi, "level": level,
               "fields": np.stack(src), "nlon": np.int64(NLON)}
        rec.update({
            "lat_ext4": tables.lat_ext_host, "mrden4": tables.mrden_host,
            "rowoff4": tables.rowoff_host, "rowshift4": tables.rowshift_host,
            "mlut4": np.asarray(tables.mlut), "lat_ext6": tables.lat_ext6_host,
            "mrden6": tables.mrden6_host, "rowoff6": tables.rowoff6_host,
            "rowshift6": tables.rowshift6_host, "mlut6": np.asarray(tables.mlut6),
        })
        for name, order, limiter, deficit in CASES:
            out = gather_batch(src, st, monotone=limiter, deficit=deficit, order=order)
            if deficit:
                rec[name] = np.stack([v for v, _ in out])
                rec[name + "_cut"] = np.stack([c for _, c in out])
            else:
                rec[name] = np.stack(out)
        rec["linear"] = np.stack(gather_linear_batch(src, st))
        # the fixed-point departure search on a rotation across both poles
        wind = rotation_wind(lat, NLON, NLEV, seed=SEED + 2, dtype=dtype)
        ex = rotation_wind(lat, NLON, NLEV, speed=45.0, seed=SEED + 3, dtype=dtype)
        dst, diag = departure_points(CartesianWind(*wind), tables, DT, iterations=3,
                                     extrapolated=CartesianWind(*ex))
        rec.update({"wind": np.stack(wind), "wind_ex": np.stack(ex), "dt": np.float64(DT),
                    "dep_xi": np.asarray(dst.xi), "dep_phi": np.asarray(dst.phi),
                    "dep_level": np.asarray(dst.level),
                    "dep_diag": np.array([diag.move_max_m, diag.move_max_cells,
                                          diag.move_max_levels, diag.displacement_max_m,
                                          diag.displacement_max_cells,
                                          diag.displacement_max_levels])})
        np.savez_compressed(HERE / f"sl_gather_{tag}.npz", **rec)
        print("wrote", HERE / f"sl_gather_{tag}.npz")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path to the reference checkout>")
    main(sys.argv[1])

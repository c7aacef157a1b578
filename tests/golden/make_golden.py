"""Record golden input/output vectors from the reference implementation.

Run in the build container, where the reference source tree is mounted:

    python tests/golden/make_golden.py <reference checkout>

It imports the reference's own numpy float64 transform
(``arwen_global.spectral.transform.SphericalHarmonicTransform`` and
``arwen_global.spectral.vector.VorticityDivergenceOperator``), its frozen dense
oracle (``tests/global_spectral_dense_reference.py``) and its semi-implicit
solver (``arwen_global.semi_implicit.VerticalModeSemiImplicit``), runs them on
seeded inputs at small truncations and writes ``tests/golden/*.npz``.  The
reference cannot travel to the GPU host, so these fixtures are how the oracle
and the CUDA path are pinned to it there.  It also copies the reference's
pinned SciPy ``Y_nm`` values (``tests/data/sph_harm_reference_scipy115.json``)
and adds an independent SciPy table when SciPy >= 1.15 is importable.
"""
from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

#: (name, truncation, create kwargs, lead shape).  T9 has an odd latitude
#: count (15), so the equator row is covered; T62 is the 94x192 grid the
#: reference's default rule refuses without ``dealias_factor=1.49``.
CASES = [
    ("t9", 9, {}, (2,)),
    ("t21", 21, {}, (3,)),
    ("t31_wide", 31, {"nlat": 50, "nlon": 100}, (2,)),
    ("t62", 62, {"nlat": 94, "nlon": 192, "dealias_factor": 1.49}, (2,)),
]


def _red_triangle(rng, lead, t):
    n = np.arange(t + 1, dtype=np.float64)
    sigma = np.zeros(t + 1)
    sigma[1:] = (n[1:] * (n[1:] + 1.0)) ** -1.5
    c = sigma[:, None] * (rng.standard_normal((*lead, t + 1, t + 1))
                          + 1j * rng.standard_normal((*lead, t + 1, t + 1)))
    c *= np.tri(t + 1, dtype=bool)
    c[..., :, 0] = c[..., :, 0].real
    c[..., 0, 0] = 0.0
    return c


def record_transforms(ref_root: Path) -> None:
    from arwen_global.spectral.transform import SphericalHarmonicTransform
    from arwen_global.spectral.vector import VorticityDivergenceOperator
    import global_spectral_dense_reference as dense

    for name, t, kw, lead in CASES:
        rng = np.random.default_rng(20261203 + t)
        live = SphericalHarmonicTransform.create(t, precision="float64", **kw)
        frozen = dense.SphericalHarmonicTransform.create(t, precision="float64", **kw)
        vec = VorticityDivergenceOperator(live)
        nlat, nlon = live.grid.shape
        coeff = _red_triangle(rng, lead, t)
        coeff2 = _red_triangle(rng, lead, t)
        grid = live.inverse(coeff) + 0.05 * rng.standard_normal((*lead, nlat, nlon))
        u = rng.standard_normal((*lead, nlat, nlon))
        v = rng.standard_normal((*lead, nlat, nlon))
        east, north = live.gradient(coeff)
        wu, wv = vec.wind_from_vordiv(coeff, coeff2)
        zeta, div = vec.vordiv_from_wind(u, v)
        out = {
            "truncation": t, "nlat": nlat, "nlon": nlon,
            "radius_m": live.grid.radius_m,
            "dealias_factor": kw.get("dealias_factor", 1.5),
            "mu": live.grid.sin_lat, "weights": live.grid.quadrature_weights,
            "coeff": coeff, "coeff2": coeff2, "grid": grid, "u": u, "v": v,
            "forward": live.forward(grid),
            "forward_frozen": frozen.forward(grid),
            "inverse": live.inverse(coeff),
            "zonal": live.inverse_zonal_derivative(coeff),
            "meridional": live.inverse_meridional_derivative(coeff),
            "east": east, "north": north,
            "laplacian": live.laplacian(coeff),
            "inverse_laplacian": live.inverse_laplacian(coeff),
            "project_in": rng.standard_normal((*lead, t + 1, t + 1))
            + 1j * rng.standard_normal((*lead, t + 1, t + 1)),
            "wind_u": wu, "wind_v": wv, "vort": zeta, "div": div,
        }
        out["project_out"] = live.project(out["project_in"])
        check = live.transform_check(seed=19)
        out["check_roundtrip"] = check["roundtrip_relative_linf"]
        out["check_parseval"] = check["parseval_relative_error"]
        np.savez_compressed(HERE / f"sht_{name}.npz", **out)
        print("wrote", name, nlat, nlon)


class _State:
    """The four fields ``solve_shifted`` reads, plus ``with_fields``."""

    def __init__(self, vorticity, divergence, theta, lnps):
        self.vorticity = vorticity
        self.divergence = divergence
        self.theta = theta
        self.log_surface_pressure = lnps
        self.qv = np.zeros_like(theta)
        self.qc = self.qr = self.qi = self.qs = self.qg = None

    def with_fields(self, fields):
        f = tuple(fields)
        return _State(f[0], f[1], f[2], f[3])


def record_helmholtz() -> None:
    from arwen_global.semi_implicit import VerticalModeSemiImplicit
    from arwen_global.spectral.transform import SphericalHarmonicTransform
    from arwen_global.vertical import HybridCoordinate

    for name, t, nlev, tau in [("t7_l6", 7, 6, 1800.0), ("t21_l40", 21, 40, 300.0)]:
        rng = np.random.default_rng(7 + nlev)
        transform = SphericalHarmonicTransform.create(t, precision="float64")
        vertical = HybridCoordinate.pressure_blend(nlev, 100.0)
        semi = VerticalModeSemiImplicit()
        op = semi.operator(vertical)

        def field(shape, scale):
            return transform.project(scale * (rng.standard_normal(shape)
                                              + 1j * rng.standard_normal(shape)))

        shape = (nlev, t + 1, t + 1)
        state = _State(field(shape, 1e-5), field(shape, 1e-5), field(shape, 1.0),
                       field((t + 1, t + 1), 1e-3))
        solved = semi.solve_shifted(state, transform, vertical, tau)
        np.savez_compressed(
            HERE / f"helmholtz_{name}.npz",
            truncation=t, nlev=nlev, tau_s=tau, weight=semi.divergence_weight,
            radius_m=transform.grid.radius_m,
            b_matrix=op.b_matrix, c_matrix=op.c_matrix,
            eigenvalues=op.eigenvalues, eigenvectors=op.eigenvectors,
            divergence=state.divergence, theta=state.theta,
            lnps=state.log_surface_pressure,
            out_divergence=solved.divergence, out_theta=solved.theta,
            out_lnps=solved.log_surface_pressure,
        )
        print("wrote helmholtz", name)


def record_ynm(ref_root: Path) -> None:
    src = ref_root / "tests" / "data" / "sph_harm_reference_scipy115.json"
    data = json.loads(src.read_text(encoding="utf-8"))
    keep = {k: data[k] for k in ("convention", "latitude_deg", "longitude_deg", "values")}
    try:
        from scipy.special import sph_harm_y
    except ImportError:
        sph_harm_y = None
    if sph_harm_y is not None:
        lat = np.linspace(-85.0, 85.0, 9)
        lon = np.linspace(0.0, 350.0, 9)
        values = {}
        for n in range(0, 13):
            for m in range(0, n + 1, 3):
                y = sph_harm_y(n, m, np.pi / 2 - np.deg2rad(lat), np.deg2rad(lon))
                values[f"{n},{m}"] = {"real": y.real.tolist(), "imag": y.imag.tolist()}
        keep["scipy_extra"] = {"latitude_deg": lat.tolist(), "longitude_deg": lon.tolist(),
                               "values": values}
    (HERE / "ynm_reference.json").write_text(json.dumps(keep, indent=1, sort_keys=True))
    print("wrote ynm_reference.json")


def record_gauss_exact() -> None:
    """Gauss-Legendre nodes/weights to 40 digits (mpmath Newton on P_n),
    rounded to float64: the accuracy yardstick for the device geometry."""
    import mpmath

    mpmath.mp.dps = 40
    out = {}
    for n in (15, 33, 50, 94, 768):
        xs, ws = [], []
        for k in range(n // 2):
            x = mpmath.cos(mpmath.pi * (k + mpmath.mpf("0.75")) / (n + mpmath.mpf("0.5")))
            for _ in range(60):
                p = mpmath.legendre(n, x)
                dp = n * (x * p - mpmath.legendre(n - 1, x)) / (x * x - 1)
                step = p / dp
                x -= step
                if abs(step) < mpmath.mpf(10) ** -38:
                    break
            dp = n * (x * mpmath.legendre(n, x) - mpmath.legendre(n - 1, x)) / (x * x - 1)
            xs.append(float(x))
            ws.append(float(2 / ((1 - x * x) * dp * dp)))
        mu = np.array([-v for v in xs] + ([0.0] if n % 2 else []) + xs[::-1])
        w_mid = []
        if n % 2:
            x = mpmath.mpf(0)
            dp = n * (x * mpmath.legendre(n, x) - mpmath.legendre(n - 1, x)) / (x * x - 1)
            w_mid = [float(2 / dp ** 2)]
        w = np.array(ws + w_mid + ws[::-1])
        out[f"mu_{n}"] = mu
        out[f"w_{n}"] = w
    np.savez_compressed(HERE / "gauss_exact.npz", **out)
    print("wrote gauss_exact.npz")


def record_fp32_errors() -> None:
    """The reference's own float32 accuracy on the config grids: relative
    spectral L2 of vordiv_from_wind (float32 inputs) and of forward against
    its float64 path, on the seeded red-spectrum inputs the GPU tests use.
    The integration-by-parts vector analysis loses digits to cancellation
    in float32, so its bar is set from the reference rather than 2e-6."""
    from arwen_global.spectral.transform import SphericalHarmonicTransform
    from arwen_global.spectral.vector import VorticityDivergenceOperator

    sys.path.insert(0, str(HERE.parents[1] / "gpuwm-global_b200"))
    from b200sht.synthetic import red_spectrum

    def rel_l2(a, b):
        w = np.where(np.arange(a.shape[-1]) == 0, 1.0, 2.0)[None, :]
        return float(np.sqrt(np.sum(w * np.abs(a - b) ** 2) / np.sum(w * np.abs(b) ** 2)))

    out = {}
    for t, kw in [(62, {"nlat": 94, "nlon": 192, "dealias_factor": 1.49}),
                  (126, {"nlat": 192, "nlon": 384}), (255, {}), (511, {})]:
        r64 = SphericalHarmonicTransform.create(t, precision="float64", **kw)
        r32 = SphericalHarmonicTransform.create(t, precision="float32", **kw)
        v64, v32 = VorticityDivergenceOperator(r64), VorticityDivergenceOperator(r32)
        c = red_spectrum(t, 3)
        u, v = v64.wind_from_vordiv(c, c[::-1].copy())
        z, d = v64.vordiv_from_wind(u, v)
        z2, d2 = v32.vordiv_from_wind(u.astype(np.float32), v.astype(np.float32))
        g = r64.inverse(c)
        f2 = r32.forward(g.astype(np.float32))
        out[str(t)] = {"vordiv": max(rel_l2(z2, z), rel_l2(d2, d)),
                       "forward": rel_l2(f2, r64.forward(g))}
        print("fp32 errors", t, out[str(t)], flush=True)
    (HERE / "reference_fp32_errors.json").write_text(json.dumps(out, indent=1, sort_keys=True))


def main() -> None:
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path to the reference checkout>")
    ref_root = Path(sys.argv[1])
    os.environ.setdefault("ARWEN_GLOBAL_LEGENDRE_CACHE", "off")
    sys.path[:0] = [str(ref_root / "src"), str(ref_root / "tests")]
    record_transforms(ref_root)
    record_helmholtz()
    record_ynm(ref_root)
    record_gauss_exact()
    record_fp32_errors()


if __name__ == "__main__":
    main()

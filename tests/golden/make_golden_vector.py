"""Record the reference's vector-waist outputs and its contraction census.

Run in the build container, where the reference source tree is mounted:

    python tests/golden/make_golden_vector.py <reference checkout>

It imports the reference's numpy float64 ``SphericalHarmonicTransform`` and
``VorticityDivergenceOperator`` and writes:

* ``vector_waist_t21.npz``, ``vector_waist_t62.npz``: a seeded wind pair, the
  reference's ``vordiv_from_wind_waist`` of its ``_wind_fourier`` waist,
  ``_vordiv_from_fourier`` of the raw full-width zonal spectrum
  (``numpy.fft.rfft / nlon`` of the pair, cut inside the method; the test
  recomputes that spectrum with the same numpy call), and
  ``divergence_from_fourier`` of the same waist;
* ``census.json``: every ``_batched_contract`` call the reference's public
  methods make, recorded by replacing that method exactly as the reference's
  census tool does (tools/arwen_global_transform_census.py:64-140): per
  method, the sequence of (table, transposed, leading planes).
"""
from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

CASES = [
    ("t21", 21, {}, (3,)),
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


def record_vector_waists() -> None:
    from arwen_global.spectral.transform import SphericalHarmonicTransform
    from arwen_global.spectral.vector import VorticityDivergenceOperator

    for name, t, kw, lead in CASES:
        rng = np.random.default_rng(20261203 + 500 + t)
        live = SphericalHarmonicTransform.create(t, precision="float64", **kw)
        vec = VorticityDivergenceOperator(live)
        nlat, nlon = live.grid.shape
        # A smooth wind (the synthesis of a red spectrum) plus grid noise.
        u = live.inverse(_red_triangle(rng, lead, t)) + 0.01 * rng.standard_normal((*lead, nlat, nlon))
        v = live.inverse(_red_triangle(rng, lead, t)) + 0.01 * rng.standard_normal((*lead, nlat, nlon))
        pair = np.stack([u, v])
        waist = vec._wind_fourier(pair)
        waist_values = np.array(waist.values)
        zeta_w, div_w = vec.vordiv_from_wind_waist(vec._wind_fourier(pair))
        raw = np.fft.rfft(pair, axis=-1) / nlon
        zeta_r, div_r = vec._vordiv_from_fourier(raw)
        div_only = vec.divergence_from_fourier(vec._wind_fourier(pair))
        zeta, div = vec.vordiv_from_wind(u, v)
        np.savez_compressed(
            HERE / f"vector_waist_{name}.npz",
            truncation=t, nlat=nlat, nlon=nlon, dealias_factor=kw.get("dealias_factor", 1.5),
            u=u, v=v, waist=waist_values, zeta_waist=zeta_w, div_waist=div_w,
            zeta_raw=zeta_r, div_raw=div_r, div_only=div_only, zeta=zeta, div=div)
        print("wrote vector_waist", name)


def record_census() -> None:
    from arwen_global.spectral import transform as T
    from arwen_global.spectral.vector import VorticityDivergenceOperator

    t = 21
    live = T.SphericalHarmonicTransform.create(t, precision="float64")
    vec = VorticityDivergenceOperator(live)
    rng = np.random.default_rng(11)
    lead = (2, 3)
    nlat, nlon = live.grid.shape
    coeff = _red_triangle(rng, lead, t)
    grid = rng.standard_normal((*lead, nlat, nlon))
    records: list = []
    names = {id(live._analysis): "analysis", id(live._basis): "basis",
             id(live._derivative_basis): "derivative_basis"}
    contract = T.SphericalHarmonicTransform._batched_contract

    def hook(self, values, table, *, transposed=False, **keywords):
        planes = 1
        for extent in values.shape[:-2]:
            planes *= int(extent)
        records.append([names.get(id(table), "other"), bool(transposed), planes])
        return contract(self, values, table, transposed=transposed, **keywords)

    calls = {
        "forward": lambda: live.forward(grid),
        "inverse": lambda: live.inverse(coeff),
        "inverse_zonal_derivative": lambda: live.inverse_zonal_derivative(coeff),
        "inverse_meridional_derivative": lambda: live.inverse_meridional_derivative(coeff),
        "gradient": lambda: live.gradient(coeff),
        "contract_waist": lambda: live.contract_waist(live.fourier_waist(grid)),
        "contract_to_waist": lambda: live.contract_to_waist(coeff),
        "gradient_waists": lambda: live.gradient_waists(coeff),
        "wind_from_vordiv": lambda: vec.wind_from_vordiv(coeff, coeff),
        "vordiv_from_wind": lambda: vec.vordiv_from_wind(grid, grid),
        "vordiv_from_wind_waist": lambda: vec.vordiv_from_wind_waist(
            vec._wind_fourier(np.stack([grid, grid]))),
        "divergence_from_fourier": lambda: vec.divergence_from_fourier(
            vec._wind_fourier(np.stack([grid, grid]))),
    }
    out = {"truncation": t, "lead": list(lead), "calls": {}}
    T.SphericalHarmonicTransform._batched_contract = hook
    try:
        for name, fn in calls.items():
            records.clear()
            fn()
            out["calls"][name] = [list(r) for r in records]
    finally:
        T.SphericalHarmonicTransform._batched_contract = contract
    (HERE / "census.json").write_text(json.dumps(out, indent=1) + "\n")
    print("wrote census.json")


def main(ref_root: str) -> None:
    root = Path(ref_root)
    os.environ.setdefault("ARWEN_GLOBAL_LEGENDRE_CACHE", "off")
    sys.path[:0] = [str(root / "src"), str(root / "tests")]
    record_vector_waists()
    record_census()


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path to the reference checkout>")
    main(sys.argv[1])

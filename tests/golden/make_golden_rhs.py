"""Record golden vectors of the van Leer vertical flux divergence from the
reference.

Run in the build container, where the reference source tree is mounted:

    python tests/golden/make_golden_rhs.py <reference checkout>

It calls the reference's own numpy specification,
``arwen_global.dynamics.MoistHybridModel._vertical_scalar_flux_divergence``
(the method its fused CuPy kernel replaces), on seeded columns
(``oracle.rhs.column_state``: 12 levels, 6 x 10 columns, 3 tracers, float64
and float32) through a minimal stand-in for the model object (the method
reads only ``nlev`` and the transform's backend), and writes
``tests/golden/rhs_vertical_flux.npz``.

It also calls the reference's numpy specifications of the three elementwise
chains -- ``momentum_bernoulli_reference``, ``tracer_flux_reference`` and
``scalar_tendency_reference`` in ``tools/gpu_selftest_rhs.py``, the functions
the reference proves its fused kernel bodies bit-identical to -- on seeded
fields (8 levels x 6 x 10, 3 tracers, a sub-pascal layer, float64 and
float32) and writes ``tests/golden/rhs_elementwise.npz``.  That tool imports
a local-GPU guard module that is not part of the reference checkout; a
stand-in module with the two names it imports is installed first (neither
is called by the specification functions).
"""
from __future__ import annotations

import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))


def main(ref_root: str) -> None:
    os.environ.setdefault("ARWEN_GLOBAL_LEGENDRE_CACHE", "off")
    sys.path.insert(0, str(Path(ref_root) / "src"))
    from arwen_global.dynamics import MoistHybridModel

    from oracle.rhs import column_state

    rec = {}
    for dtype, tag in ((np.float64, "f64"), (np.float32, "f32")):
        s, w, pf, ph = column_state(12, 6, 10, 3, 20261203, dtype=dtype)
        backend = types.SimpleNamespace(xp=np, name="numpy", float_dtype=dtype)
        model = types.SimpleNamespace(nlev=12, transform=types.SimpleNamespace(backend=backend))
        out = MoistHybridModel._vertical_scalar_flux_divergence(model, s, w, pf, ph)
        rec.update({f"s_{tag}": s, f"w_{tag}": w, f"pf_{tag}": pf, f"ph_{tag}": ph,
                    f"out_{tag}": np.asarray(out)})
    np.savez_compressed(HERE / "rhs_vertical_flux.npz", **rec)
    print("wrote", HERE / "rhs_vertical_flux.npz")
    record_elementwise(ref_root)


def record_elementwise(ref_root: str) -> None:
    guard = types.ModuleType("gpuwm.local_gpu")
    guard.NO_LOCAL_GPU_ENV = "GPUWM_NO_LOCAL_GPU"
    guard.no_local_gpu = lambda *a, **k: False
    pkg = types.ModuleType("gpuwm")
    pkg.local_gpu = guard
    sys.modules.setdefault("gpuwm", pkg)
    sys.modules.setdefault("gpuwm.local_gpu", guard)
    sys.path.insert(0, str(Path(ref_root)))
    from tools.gpu_selftest_rhs import (momentum_bernoulli_reference, scalar_tendency_reference,
                                        tracer_flux_reference)

    nlev, nlat, nlon, ntr = 8, 6, 10, 3
    rec = {}
    for dtype, tag in ((np.float64, "f64"), (np.float32, "f32")):
        r = np.random.default_rng(20261204)
        shape = (nlev, nlat, nlon)
        lat = np.linspace(-1.3, 1.3, nlat)
        f = {
            "zeta": r.normal(0.0, 1.0e-5, shape),
            "cor": np.broadcast_to((1.4584e-4 * np.sin(lat))[:, None], (nlat, nlon)),
            "u": r.uniform(-70.0, 70.0, shape),
            "v": r.uniform(-70.0, 70.0, shape),
            "wu": r.normal(0.0, 1.0e-3, shape),
            "wv": r.normal(0.0, 1.0e-3, shape),
            "tv": r.uniform(190.0, 310.0, shape),
            "pg": np.broadcast_to(np.linspace(0.05, 1.0, nlev)[:, None, None], shape),
            "ge": r.normal(0.0, 1.0e-5, (nlat, nlon)),
            "gn": r.normal(0.0, 1.0e-5, (nlat, nlon)),
            "phi": r.uniform(0.0, 2.5e5, shape),
            "dp": r.uniform(40.0, 4000.0, shape),
            "s": r.uniform(-1.0e-4, 0.02, (ntr,) + shape),
            "h": r.normal(0.0, 1.0e-3, (ntr,) + shape),
            "vert": r.normal(0.0, 1.0e-3, (ntr,) + shape),
            "dpt": r.normal(0.0, 1.0e-2, shape),
        }
        f = {k: np.ascontiguousarray(v, dtype=dtype) for k, v in f.items()}
        f["dp"][0] = dtype(2.0e-3)  # a sub-pascal top layer: the division is not floored
        f["s"][1, 3] = 0.0          # a tracer-free level
        mu, mv, bern = momentum_bernoulli_reference(
            f["zeta"], f["cor"], f["u"], f["v"], f["wu"], f["wv"], f["tv"], f["pg"], f["ge"],
            f["gn"], f["phi"], dtype(287.0528))
        fx, fy = tracer_flux_reference(f["dp"], f["s"], f["u"], f["v"])
        st = scalar_tendency_reference(f["h"], f["vert"], f["s"], f["dpt"], f["dp"])
        for k, v in f.items():
            rec[f"{k}_{tag}"] = v
        for k, v in (("mu", mu), ("mv", mv), ("bern", bern), ("fx", fx), ("fy", fy), ("st", st)):
            rec[f"{k}_{tag}"] = np.asarray(v)
    np.savez_compressed(HERE / "rhs_elementwise.npz", **rec)
    print("wrote", HERE / "rhs_elementwise.npz")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path to the reference checkout>")
    main(sys.argv[1])

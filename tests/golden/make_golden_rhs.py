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


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path to the reference checkout>")
    main(sys.argv[1])

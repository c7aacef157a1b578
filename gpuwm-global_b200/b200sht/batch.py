"""Several transforms (truncations) run as one batched call.

The ensemble workload holds 32 LETKF members at T126 and one control at
T255, 40 levels x 5 fields each.  The reference transforms every member and
every truncation through its own ``SphericalHarmonicTransform`` object
(src/arwen_global/spectral/transform.py:1435-1490 and 1629-1746 per call).
Here members of one truncation are simply more planes of one plan, and a
``TransformBatch`` runs up to four plans together: the Legendre contractions
of all of them go to ONE launch per direction (on split16 plans, the
persistent tensor-core kernel over the merged work list sorted by the
triangular per-order cost), between per-plan FFT and pack/unpack launches.
"""
from __future__ import annotations

import ctypes
from typing import Sequence

from . import _lib
from .transform import SphericalHarmonicTransform, _stream


class TransformBatch:
    def __init__(self, transforms: Sequence[SphericalHarmonicTransform], planes: Sequence[int]):
        if len(transforms) != len(planes):
            raise ValueError("one plane count per transform")
        self.transforms = list(transforms)
        self.planes = [int(p) for p in planes]
        self._lib = _lib.load()
        n = len(self.transforms)
        handles = (ctypes.c_void_p * max(n, 1))(*[t.plan.handle.value for t in self.transforms])
        counts = (ctypes.c_int64 * max(n, 1))(*self.planes)
        out = ctypes.c_void_p()
        _lib.check(self._lib.sht_batch_create(n, handles, counts, ctypes.byref(out)))
        self.handle = out

    def _inputs(self, arrays, shape_of, dtype_of):
        if len(arrays) != len(self.transforms):
            raise ValueError(f"expected {len(self.transforms)} arrays, got {len(arrays)}")
        ins = []
        for t, p, a in zip(self.transforms, self.planes, arrays):
            x = t.backend.asarray(a, dtype=dtype_of(t)).contiguous()
            if tuple(x.shape[-2:]) != shape_of(t) or t._planes(x) != p:
                raise ValueError(f"batch array of shape {tuple(x.shape)} does not hold {p} planes "
                                 f"of {shape_of(t)}")
            ins.append(x)
        return ins

    def forward(self, grids):
        """grid -> spectral for every plan; one coefficient array per plan."""
        ins = self._inputs(grids, lambda t: t.grid.shape, lambda t: t.backend.float_dtype)
        outs = [t._empty_spec(x.shape[:-2]) for t, x in zip(self.transforms, ins)]
        self._call("sht_batch_forward", ins, outs)
        return outs

    def inverse(self, coeffs):
        """spectral -> grid for every plan; one grid array per plan."""
        ins = self._inputs(coeffs, lambda t: t.spectral_shape, lambda t: t.backend.complex_dtype)
        outs = [t._empty_grid(x.shape[:-2]) for t, x in zip(self.transforms, ins)]
        self._call("sht_batch_inverse", ins, outs)
        return outs

    def _call(self, name, ins, outs):
        n = len(ins)
        pin = (ctypes.c_void_p * n)(*[x.data_ptr() for x in ins])
        pout = (ctypes.c_void_p * n)(*[y.data_ptr() for y in outs])
        _lib.call(name, self.handle, pin, pout, _stream())

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self._lib.sht_batch_destroy(h)
            except Exception:
                pass
            self.handle = None


def ensemble_batch(members: int = 32, levels: int = 40, fields: int = 5, *,
                   precision: str = "split16", member_truncation: int = 126,
                   control_truncation: int = 255):
    """The ensemble workload's batch: ``members`` x levels x fields planes at
    T126 on 192 x 384 and the control's levels x fields planes at T255 on
    384 x 768, as two plans of one batch."""
    lo = SphericalHarmonicTransform.create(member_truncation, nlat=192, nlon=384,
                                           precision=precision)
    hi = SphericalHarmonicTransform.create(control_truncation, nlat=384, nlon=768,
                                           precision=precision)
    per = levels * fields
    return TransformBatch([lo, hi], [members * per, per])

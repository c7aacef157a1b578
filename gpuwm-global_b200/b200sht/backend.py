"""Device-array backend of the B200 engine.

The reference's ``Backend`` (src/arwen_global/spectral/backend.py:14-71)
switches numpy/cupy; here the arrays are torch CUDA tensors (torch is only
the device-memory and stream plumbing; every transform kernel is the
library's own CUDA).  ``precision`` is ``"float64"``, ``"float32"`` or
``"split16"``; the last two share float32/complex64 arrays.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Any

import numpy as np
import torch

PRECISIONS = ("float64", "float32", "split16")


@dataclass(frozen=True)
class Backend:
    name: str
    xp: Any
    float_dtype: Any
    complex_dtype: Any
    precision: str
    device: torch.device

    def asarray(self, value, *, dtype=None):
        dtype = dtype or (self.complex_dtype if _is_complex(value) else self.float_dtype)
        if isinstance(value, torch.Tensor):
            return value.to(device=self.device, dtype=dtype)
        arr = np.asarray(value)
        return torch.as_tensor(arr).to(device=self.device, dtype=dtype)

    def to_numpy(self, value) -> np.ndarray:
        if isinstance(value, torch.Tensor):
            return value.detach().cpu().numpy()
        return np.asarray(value)

    def synchronize(self) -> None:
        torch.cuda.synchronize(self.device)

    @property
    def numpy_float(self):
        return np.float64 if self.float_dtype == torch.float64 else np.float32

    @property
    def numpy_complex(self):
        return np.complex128 if self.float_dtype == torch.float64 else np.complex64


def _is_complex(value) -> bool:
    if isinstance(value, torch.Tensor):
        return value.is_complex()
    return np.iscomplexobj(value)


def get_backend(name: str = "b200", precision: str = "float32", device=None) -> Backend:
    key = str(name).strip().lower()
    prec = str(precision).strip().lower()
    if key != "b200":
        raise ValueError(f"backend must be 'b200', got {name!r}")
    if prec not in PRECISIONS:
        raise ValueError(f"precision must be one of {PRECISIONS}, got {precision!r}")
    if not torch.cuda.is_available():
        raise RuntimeError("backend='b200' needs a CUDA device; there is no CPU fallback")
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    if prec == "float64":
        return Backend(key, torch, torch.float64, torch.complex128, prec, dev)
    return Backend(key, torch, torch.float32, torch.complex64, prec, dev)

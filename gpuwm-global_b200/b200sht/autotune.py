"""Project autotuner: picks a plan's contraction engine, FFT kernel and
tensor-core tile order for the caller's plane count by timing them.

The reference fixes its Legendre band width and GEMM shapes in code (its
``legendre_band`` knob, transform.py:953-1023, is a memory setting for
small cards).  Here the variants that exist at run time are timed on the
plan itself: ``tune(transform, planes)`` runs the forward + inverse pair on
seeded red-spectrum planes for every combination of

* contraction: the plan's own (split-FP16 tensor cores on a split16 plan)
  or FP32 SIMT (split16 plans only: both meet the 2e-6 bar);
* FFT: register-resident (where the grid allows) or shared-memory Stockham;
* tensor-core tile order among equal-cost tiles: a column tile's row blocks
  adjacent (table-image reuse) or a row block's column tiles adjacent
  (converted-data reuse);
* the FP32 SIMT contraction's tile shape: 128 x 128 or 64 x 128 (columns x
  rows; the narrow shape pads the ragged analysis blocks less);

keeps the fastest on the plan (``sht_plan_set_tuning``) and returns the
timings.  Results can be cached in a JSON file keyed by device, grid,
truncation, precision and plane count, so a run tunes once.
"""
from __future__ import annotations

import ctypes
import itertools
import json
import os
from pathlib import Path

import torch

from . import _lib

KEYS = {"contraction": _lib.SHT_TUNE_CONTRACTION, "fft": _lib.SHT_TUNE_FFT,
        "tile_order": _lib.SHT_TUNE_TILE_ORDER, "tc_ctas": _lib.SHT_TUNE_TC_CTAS,
        "accumulators": _lib.SHT_TUNE_ACCUMULATORS, "simt_tile": _lib.SHT_TUNE_SIMT_TILE}


def get_tuning(transform) -> dict:
    out = {}
    for name, key in KEYS.items():
        v = ctypes.c_int()
        _lib.call("sht_plan_get_tuning", transform.plan.handle, key, ctypes.byref(v))
        out[name] = v.value
    return out


def set_tuning(transform, **settings) -> None:
    for name, value in settings.items():
        if name not in KEYS:
            raise ValueError(f"unknown tuning setting {name!r}; known: {sorted(KEYS)}")
        _lib.call("sht_plan_set_tuning", transform.plan.handle, KEYS[name], int(value))


def _candidates(transform) -> list[dict]:
    current = get_tuning(transform)
    split = transform.precision == "split16"
    ffts = [current["fft"]]
    try:  # the register-resident FFT exists for this grid?
        set_tuning(transform, fft=0)
        ffts = [0, 1]
    except ValueError:
        pass
    finally:
        set_tuning(transform, fft=current["fft"])
    fp32 = transform.precision != "float64"
    out = []
    for contraction, fft, order, simt_tile in itertools.product(
            [0, 1] if split else [0], ffts, [0, 1] if split else [0], [0, 1] if fp32 else [0]):
        if contraction == 1 and order == 1:
            continue  # the tile order only steers the tensor-core kernel
        if split and contraction == 0 and simt_tile == 1:
            continue  # the SIMT tile shape only steers the SIMT contraction
        out.append({"contraction": contraction, "fft": fft, "tile_order": order, "tc_ctas": 0,
                    "accumulators": current["accumulators"], "simt_tile": simt_tile})
    return out


def _cache_key(transform, planes) -> str:
    name = torch.cuda.get_device_name(transform.backend.device)
    g = transform.grid
    return f"{name}|T{transform.truncation}|{g.nlat}x{g.nlon}|{transform.precision}|P{int(planes)}"


def tune(transform, planes: int, *, repeats: int = 5, warmup: int = 2,
         cache: str | os.PathLike | None = None) -> dict:
    """Time every candidate setting on ``planes`` planes, keep the fastest on
    the plan, and return ``{"best": settings, "ms": {...}, "cached": bool}``."""
    from .synthetic import red_spectrum

    key = _cache_key(transform, planes)
    path = Path(cache) if cache else None
    if path is not None and path.exists():
        table = json.loads(path.read_text())
        if key in table:
            set_tuning(transform, **table[key]["best"])
            return {**table[key], "cached": True}
    coeff = torch.as_tensor(red_spectrum(transform.truncation, int(planes))).to(
        transform.backend.device, transform.backend.complex_dtype)
    grid = transform.inverse(coeff)
    timings = {}
    for cand in _candidates(transform):
        set_tuning(transform, **cand)
        for _ in range(warmup):
            transform.inverse(transform.forward(grid))
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(repeats):
            transform.inverse(transform.forward(grid))
        b.record()
        torch.cuda.synchronize()
        transform.check_device()
        timings[json.dumps(cand, sort_keys=True)] = a.elapsed_time(b) / repeats
    best_key = min(timings, key=timings.get)
    best = json.loads(best_key)
    set_tuning(transform, **best)
    result = {"best": best, "ms": timings, "cached": False}
    if path is not None:
        table = json.loads(path.read_text()) if path.exists() else {}
        table[key] = {"best": best, "ms": timings}
        path.write_text(json.dumps(table, indent=1, sort_keys=True))
    return result

"""ctypes binding of ``libb200sht.so`` (the C ABI in ``include/b200sht.h``).

There is no CPU fallback: if the library is missing or fails to load, every
call raises.  Loading does not touch the GPU; the first plan does.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parents[1] / "lib" / "libb200sht.so"

SHT_ABI_VERSION = 1
SHT_PREC_F64 = 0
SHT_PREC_F32 = 1
SHT_PREC_SPLIT16 = 2
SHT_FLAG_GEOMETRY_ONLY = 1
SHT_FLAG_GENERIC_FFT = 2
SHT_WAIST_BASIS = 0
SHT_WAIST_DBASIS = 1
SHT_WAIST_ZONAL = 2
SHT_TABLE_BASIS = 0
SHT_TABLE_DBASIS = 1
SHT_TABLE_ANALYSIS = 2
SHT_TABLE_ROTATION = 3
SHT_TABLE_SHEAR = 4
SHT_TUNE_CONTRACTION = 0
SHT_TUNE_FFT = 1
SHT_TUNE_TILE_ORDER = 2
SHT_TUNE_TC_CTAS = 3
SHT_TUNE_ACCUMULATORS = 4
SHT_TUNE_SIMT_TILE = 5
SHT_OK = 0
SHT_ERR_ARG = 1
SHT_ERR_CUDA = 2
SHT_ERR_DEVICE = 3
SHT_ERR_STATE = 4
SHT_SL_NONE = 0
SHT_SL_QUASI_MONOTONE = 1
SHT_SEMI_SOLVE_SHIFTED = 0
SHT_SEMI_APPLY = 1
SHT_SEMI_HALF_APPLY = 2
SHT_SEMI_LINEAR_TENDENCIES = 3
#: Kernel kinds of sht_plan_read_timing, in order.
KERNEL_KINDS = ("fft_forward", "fft_inverse", "legendre_analysis", "legendre_synthesis", "pack",
                "unpack", "elementwise", "helmholtz")

#: Every symbol ``include/b200sht.h`` declares, with its ctypes signature.
_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_D = ctypes.c_double
_DP = ctypes.POINTER(ctypes.c_double)
_I32P = ctypes.POINTER(ctypes.c_int32)
SIGNATURES = {
    "sht_abi_version": (ctypes.c_int, []),
    "sht_last_error": (ctypes.c_char_p, []),
    "sht_plan_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _D, ctypes.c_int,
                                       ctypes.c_int, ctypes.POINTER(_P)]),
    "sht_plan_destroy": (ctypes.c_int, [_P]),
    "sht_plan_reserve": (ctypes.c_int, [_P, _I64]),
    "sht_plan_geometry": (ctypes.c_int, [_P, _DP, _DP, _DP]),
    "sht_plan_check": (ctypes.c_int, [_P]),
    "sht_plan_table_bytes": (ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(_I64)]),
    "sht_plan_read_table": (ctypes.c_int, [_P, ctypes.c_int, _P]),
    "sht_plan_set_timing": (ctypes.c_int, [_P, ctypes.c_int]),
    "sht_plan_read_timing": (ctypes.c_int, [_P, _DP, ctypes.POINTER(_I64), ctypes.POINTER(_I64),
                                            ctypes.c_int, ctypes.c_int]),
    "sht_measure_fp32_peak": (ctypes.c_int, [_P, _DP]),
    "sht_forward": (ctypes.c_int, [_P, _P, _I64, _P, _P]),
    "sht_forward_static_scratch": (ctypes.c_int, [_P, _P, _I64, _P, _P]),
    "sht_forward_host": (ctypes.c_int, [_P, _P, _I64, _P, _I64]),
    "sht_inverse_host": (ctypes.c_int, [_P, _P, _I64, _P, _I64]),
    "sht_round_trip_host": (ctypes.c_int, [_P, _P, _I64, _P, _I64]),
    "sht_inverse": (ctypes.c_int, [_P, _P, _I64, _P, _P]),
    "sht_inverse_meridional_derivative": (ctypes.c_int, [_P, _P, _I64, _P, _P]),
    "sht_inverse_zonal_derivative": (ctypes.c_int, [_P, _P, _I64, _P, _P]),
    "sht_gradient": (ctypes.c_int, [_P, _P, _I64, _P, _P, _P]),
    "sht_wind_from_vordiv": (ctypes.c_int, [_P, _P, _P, _I64, _P, _P, _P]),
    "sht_vordiv_from_wind": (ctypes.c_int, [_P, _P, _P, _I64, _P, _P, _P]),
    "sht_vordiv_from_waist": (ctypes.c_int, [_P, _P, _I64, _P, _P, _P]),
    "sht_vertical_create_modes": (ctypes.c_int, [_P, ctypes.c_int] + [_DP] * 8
                                  + [ctypes.POINTER(_P)]),
    "sht_semi_implicit_map": (ctypes.c_int, [_P, _P, ctypes.c_int, ctypes.c_double,
                                             ctypes.c_double] + [_P] * 7),
    "sht_semi_implicit_metric": (ctypes.c_int, [_P, _DP, _P]),
    "sht_helmholtz_synthesis": (ctypes.c_int, [_P, _P, ctypes.c_double] + [_P] * 8),
    "sht_divergence_from_waist": (ctypes.c_int, [_P, _P, _I64, _P, _P]),
    "sht_project": (ctypes.c_int, [_P, _P, _I64, _P, _P]),
    "sht_laplacian": (ctypes.c_int, [_P, _P, _I64, _P, _P]),
    "sht_inverse_laplacian": (ctypes.c_int, [_P, _P, _I64, _P, _P]),
    "sht_helmholtz_solve": (ctypes.c_int, [_P, ctypes.c_int, _DP, _DP, _DP, _DP, _DP, _D,
                                           _P, _P, _P, _P, _P, _P, _P]),
    "sht_vertical_create": (ctypes.c_int, [_P, ctypes.c_int, _DP, _DP, _DP, _DP, _DP,
                                           ctypes.POINTER(_P)]),
    "sht_vertical_destroy": (ctypes.c_int, [_P]),
    "sht_helmholtz_apply": (ctypes.c_int, [_P, _P, _D, _P, _P, _P, _P, _P, _P, _P]),
    "sht_plan_set_tuning": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int]),
    "sht_plan_get_tuning": (ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    "sht_fourier_waist": (ctypes.c_int, [_P, _P, _I64, _P, _P]),
    "sht_contract_waist": (ctypes.c_int, [_P, _P, _I64, _P, _P]),
    "sht_contract_to_waist": (ctypes.c_int, [_P, _P, _I64, ctypes.c_int, _P, _P]),
    "sht_waist_to_grid": (ctypes.c_int, [_P, _P, _I64, _P, _P]),
    "sht_batch_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_P), ctypes.POINTER(_I64),
                                        ctypes.POINTER(_P)]),
    "sht_batch_destroy": (ctypes.c_int, [_P]),
    "sht_batch_forward": (ctypes.c_int, [_P, ctypes.POINTER(_P), ctypes.POINTER(_P), _P]),
    "sht_batch_inverse": (ctypes.c_int, [_P, ctypes.POINTER(_P), ctypes.POINTER(_P), _P]),
    "sht_sl_tables_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _DP, _DP, ctypes.c_int,
                                            ctypes.POINTER(_P)]),
    "sht_sl_tables_destroy": (ctypes.c_int, [_P]),
    "sht_sl_tables_read": (ctypes.c_int, [_P, ctypes.c_int, _DP, _DP, _I32P, _I32P, _I32P,
                                          ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_int), _DP]),
    "sht_sl_gather": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, _I64,
                                     ctypes.c_int, _P, _P, _P, _P, _P, _P]),
    "sht_sl_gather_linear": (ctypes.c_int, [_P, _P, _I64, ctypes.c_int, _P, _P, _P, _P, _P]),
    "sht_sl_departure": (ctypes.c_int, [_P, ctypes.c_int, _P, _P, _P, _P, _P, _P, _P, _P,
                                        ctypes.c_int, _D, _D, _P, _P, _P, _P, _P, _P]),
    "sht_sl_departure_newton": (ctypes.c_int, [_P, ctypes.c_int, _P, _P, _P, _P, _P, _P, _P, _P,
                                               ctypes.c_int, _D, _D, _P, _P, _P, _P, _P, _P]),
    "sht_sl_departure_newton_ls": (ctypes.c_int, [_P, ctypes.c_int, _P, _P, _P, _P, _P, _P, _P,
                                                  _P, ctypes.c_int, _D, _D, _P, _P, _P, _P, _P,
                                                  _P]),
    "sht_sl_lipschitz": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, _P, _P,
                                        _P, ctypes.c_int, ctypes.c_int, _P, _P, _P, _P,
                                        ctypes.c_int, ctypes.c_int, _D, _D, _D, _DP, _DP,
                                        ctypes.POINTER(_I64), _P]),
    "sht_sl_window_create": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int, ctypes.POINTER(_P)]),
    "sht_sl_window_destroy": (ctypes.c_int, [_P]),
    "sht_sl_window_escape": (ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(ctypes.c_int), _P]),
    "sht_sl_gather_band": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, _I64,
                                          ctypes.c_int, _P, _P, _P, _P, _P, _P]),
    "sht_sl_departure_band": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int, _P, _P, _P, _P, _P,
                                             _P, _P, _P, ctypes.c_int, _D, _D, _P, _P, _P, _P,
                                             _P, _P]),
    "sht_rhs_momentum_bernoulli": (ctypes.c_int, [ctypes.c_int, _I64, _I64] + [_P] * 11
                                   + [_D, _P, _P, _P, _P]),
    "sht_rhs_tracer_flux": (ctypes.c_int, [ctypes.c_int, _I64, _I64, _I64] + [_P] * 7),
    "sht_rhs_scalar_tendency": (ctypes.c_int, [ctypes.c_int, _I64, _I64, _I64] + [_P] * 7),
    "sht_rhs_vertical_flux_divergence": (ctypes.c_int, [ctypes.c_int, _I64, _I64, _I64]
                                         + [_P] * 6),
    "sht_sampler_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_P)]),
    "sht_sampler_destroy": (ctypes.c_int, [_P]),
    "sht_sample": (ctypes.c_int, [_P, _P, _I64, _I64, _P, _P, ctypes.c_int, _D, _P, _P, _P]),
    "sht_sample_packed_basis": (ctypes.c_int, [_P, _I64, _P, _P, ctypes.c_int, ctypes.c_int, _P,
                                               _P, _P]),
}

_lib = None


class ShtError(RuntimeError):
    """A failing library call (status and message from ``sht_last_error``)."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


def load(path: Path | None = None):
    """Load the library once and bind every declared symbol."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(
            f"b200sht CUDA library not built ({p}); run "
            "`python gpuwm-global_b200/b200sht/build.py` or __graft_entry__.build()")
    lib = ctypes.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.sht_abi_version() != SHT_ABI_VERSION:
        raise ImportError(f"{p}: ABI version {lib.sht_abi_version()} != {SHT_ABI_VERSION}")
    _lib = lib
    return lib


def check(status: int) -> None:
    """Raise for a non-zero status: ValueError for argument errors (the
    reference raises ValueError for bad shapes), ShtError otherwise."""
    if status == SHT_OK:
        return
    msg = (load().sht_last_error() or b"").decode()
    if status == SHT_ERR_ARG:
        raise ValueError(msg)
    raise ShtError(status, msg)


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args))

"""Triangular spherical-harmonic transform pair on a Gaussian grid, on a B200.

Drop-in for the reference's ``SphericalHarmonicTransform``
(src/arwen_global/spectral/transform.py:632-1863): the same ``create``
signature, entry points, coefficient layout ``(*lead, T+1, T+1)`` indexed
``[n, m]`` (zero above the triangle, real at ``m = 0``), grid layout
``(*lead, nlat, nlon)`` with row 0 southernmost, and the same error messages
for shape mismatches.  Each call is one C-ABI call into ``libb200sht.so`` on
the current torch stream; arrays are torch CUDA tensors (numpy inputs are
copied to the device).

Precision: ``"float64"`` (FP64 SIMT contractions; the parity path),
``"float32"`` (plain FP32 FFMA contractions) and ``"split16"`` (FP16 hi/lo
split contractions on tcgen05 tensor cores with FP32 accumulation).  The
reference's ``tensor_core_contractions=True`` (its TF32 opt-in) selects
``"split16"`` on a float32 transform.

The reference's memory-layout knobs (``legendre_band``, ``streaming``,
``latitude_bands``) are accepted and validated but change nothing here: the
tables are resident in HBM and the contraction walks the triangle directly
(``forward_streaming`` / ``inverse_streaming`` return the resident bits).
``order_partition`` (a table built for some orders only) is refused: every
order's table is resident; an order exchange's collective is honoured
(``forward_orders`` / ``inverse_orders``).
"""
from __future__ import annotations

import contextlib
import ctypes
import hashlib
import json
import math
import weakref
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .backend import Backend, get_backend
from .grid import EARTH_RADIUS_M, GaussianGrid, shape_for

_PREC_CODE = {"float64": _lib.SHT_PREC_F64, "float32": _lib.SHT_PREC_F32,
              "split16": _lib.SHT_PREC_SPLIT16}


class Plan:
    """Owns one ``sht_plan`` handle."""

    def __init__(self, truncation, nlat, nlon, radius_m, precision, flags=0):
        self._lib = _lib.load()
        handle = ctypes.c_void_p()
        _lib.check(self._lib.sht_plan_create(int(truncation), int(nlat), int(nlon),
                                             float(radius_m), _PREC_CODE[precision], int(flags),
                                             ctypes.byref(handle)))
        self.handle = handle

    def geometry(self, nlat):
        mu, w, cl = (np.zeros(nlat) for _ in range(3))
        dp = ctypes.POINTER(ctypes.c_double)
        _lib.check(self._lib.sht_plan_geometry(self.handle, mu.ctypes.data_as(dp),
                                               w.ctypes.data_as(dp), cl.ctypes.data_as(dp)))
        return mu, w, cl

    def reserve(self, planes):
        _lib.check(self._lib.sht_plan_reserve(self.handle, int(planes)))

    def check(self):
        _lib.check(self._lib.sht_plan_check(self.handle))

    def table_bytes(self, code: int) -> int:
        out = ctypes.c_int64()
        _lib.check(self._lib.sht_plan_table_bytes(self.handle, int(code), ctypes.byref(out)))
        return int(out.value)

    def read_table(self, code: int, shape, dtype) -> np.ndarray:
        out = np.empty(shape, dtype=dtype)
        _lib.check(self._lib.sht_plan_read_table(self.handle, int(code),
                                                 ctypes.c_void_p(out.ctypes.data)))
        return out

    def set_timing(self, enable: bool):
        _lib.check(self._lib.sht_plan_set_timing(self.handle, 1 if enable else 0))

    def read_timing(self, reset: bool = False) -> dict:
        """``{kind: {"ms": total, "launches": n, "timed": n}}`` per kernel kind."""
        k = len(_lib.KERNEL_KINDS)
        ms = (ctypes.c_double * k)()
        launches = (ctypes.c_int64 * k)()
        timed = (ctypes.c_int64 * k)()
        _lib.check(self._lib.sht_plan_read_timing(self.handle, ms, launches, timed, k,
                                                  1 if reset else 0))
        return {name: {"ms": ms[i], "launches": launches[i], "timed": timed[i]}
                for i, name in enumerate(_lib.KERNEL_KINDS)}

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self._lib.sht_plan_destroy(h)
            except Exception:
                pass
            self.handle = None


class LegendreTable(str):
    """One of a transform's resident Legendre tables, as its contraction seam
    names it.

    Equal to (and hashing as) its name, ``"basis"``, ``"derivative_basis"`` or
    ``"analysis"``, which is what ``_batched_contract`` dispatches on; the
    object itself is the transform's one instance per table, so a census hook
    that tells tables apart by identity (the reference's
    tools/arwen_global_transform_census.py:64-140) sees three distinct
    tables.  ``dense()`` is the reference's BandedLegendreTable.dense()
    (src/arwen_global/spectral/transform.py:214-216): the whole table in the
    dense layout, in host numpy, assembled from the device table
    (``sht_plan_read_table``); tests and inspection only."""

    _CODES = {"basis": _lib.SHT_TABLE_BASIS, "derivative_basis": _lib.SHT_TABLE_DBASIS,
              "analysis": _lib.SHT_TABLE_ANALYSIS}

    def __new__(cls, name: str, owner: "SphericalHarmonicTransform"):
        table = super().__new__(cls, name)
        table.name = name
        table.layout = "jn" if name == "analysis" else "nj"
        table._owner_ref = weakref.ref(owner)
        return table

    @property
    def _owner(self) -> "SphericalHarmonicTransform":
        owner = self._owner_ref()
        if owner is None:
            raise RuntimeError(f"the transform that held the {self.name} table is gone")
        return owner

    @property
    def code(self) -> int:
        return self._CODES[self.name]

    @property
    def nbytes(self) -> int:
        """Resident device bytes (the folded table; on a split16 transform
        also its FP16 hi/lo tile image)."""
        return self._owner.plan.table_bytes(self.code)

    def dense(self) -> np.ndarray:
        """``(T+1, T+1, nlat)`` indexed ``[m, n, j]`` (basis, derivative
        basis) or ``(T+1, nlat, T+1)`` indexed ``[m, j, n]`` (analysis), in the
        transform's float dtype, latitude row 0 southernmost, zero above the
        triangle."""
        t = self._owner
        t1, nlat = t.truncation + 1, t.grid.nlat
        shape = (t1, nlat, t1) if self.layout == "jn" else (t1, t1, nlat)
        dtype = np.float64 if t.precision == "float64" else np.float32
        return t.plan.read_table(self.code, shape, dtype)

    def __reduce__(self):
        return (str, (str(self),))


def _ptr(t: torch.Tensor):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class _FusedJob:
    """One fused library call that performs several Legendre contractions
    (and the FFTs and layout passes around them); run once, on first demand."""

    def __init__(self, run):
        self._run = run
        self._out = None

    def output(self, index: int):
        if self._out is None:
            self._out = self._run()
            self._run = None
        return self._out[index]


class FusedOperand:
    """The operand of one Legendre contraction that runs inside a fused
    library call.

    The reference routes every contraction through
    ``SphericalHarmonicTransform._batched_contract`` (transform.py:1178-1274),
    and its census tool (tools/arwen_global_transform_census.py:64-140)
    counts the calls by replacing that method and reading
    ``values.shape[:-2]``.  Here a contraction runs inside one C-ABI call
    together with its FFT and layout passes, so each public method hands the
    seam one ``FusedOperand`` per contraction the reference performs, shaped
    like the reference's operand (``(*lead, nlat, T+1)`` for an analysis,
    ``(*lead, T+1, T+1)`` for a synthesis).  The first operand of a call
    runs the library call; each returns its own output of it."""

    def __init__(self, shape, job: _FusedJob, index: int = 0):
        self.shape = tuple(int(v) for v in shape)
        self.ndim = len(self.shape)
        self._job = job
        self._index = int(index)

    def result(self):
        return self._job.output(self._index)


def fused_operands(shapes, run):
    """``FusedOperand`` objects of the given shapes over one call ``run()``
    (which returns a tuple of as many outputs)."""
    job = _FusedJob(run)
    return [FusedOperand(sh, job, i) for i, sh in enumerate(shapes)]


@dataclass
class SphericalHarmonicTransform:
    #: The multi-card row exchange, or None (transform.py:632-640).  Not a
    #: dataclass field and in no identity.  The reference sets it at run
    #: start on a multi-card run; its ``agree_once`` hook is called on each
    #: contraction output here as there (``_agree_across_cards``) and its
    #: ``fill_rows`` completes a band-filled waist (``FourierWaist.close``).
    row_exchange = None
    #: The multi-card order exchange, or None (transform.py:641-647).  With
    #: more than one rank, forward and inverse run on the order axis
    #: (``forward_orders`` / ``inverse_orders``): the whole contraction on this
    #: GPU, this rank's order columns gathered with the others' through the
    #: exchange's ``gather_columns``.
    order_exchange = None

    grid: GaussianGrid
    backend: Backend
    plan: Plan = field(repr=False)
    tensor_core_contractions: bool = False
    legendre_band: int = 32
    streaming: bool = False
    latitude_bands: int = 1
    #: Legendre contractions issued through ``_batched_contract``.
    contraction_count: int = 0

    @classmethod
    def create(cls, truncation, *, nlat=None, nlon=None, dealias_factor=1.5, radius_m=None,
               grid=None, backend="b200", precision="float32",
               tensor_core_contractions=False, legendre_band=32, streaming=False,
               latitude_bands=1, order_partition=(), device=None, plan_flags=0):
        if tuple(order_partition or ()):
            raise ValueError("order_partition (the multi-card order axis) is not built by the "
                             "B200 engine: the whole table is resident on one GPU")
        if int(legendre_band) < 1:
            raise ValueError(f"legendre_band must be >= 1, got {legendre_band}")
        if int(latitude_bands) < 1:
            raise ValueError(f"latitude_bands must be >= 1, got {latitude_bands}")
        prec = str(precision).strip().lower()
        if tensor_core_contractions:
            if prec not in ("float32", "split16"):
                raise ValueError("tensor_core_contractions=True requires precision='float32'")
            prec = "split16"
        be = get_backend(backend, prec, device)
        if grid is not None:
            if nlat is not None or nlon is not None or radius_m is not None or dealias_factor != 1.5:
                raise ValueError("grid= carries its own shape and radius: nlat, nlon, "
                                 "dealias_factor and radius_m cannot be combined with it")
            g = grid.truncated_to(truncation)
            nl, no, rad = g.nlat, g.nlon, g.radius_m
            t = int(truncation)
        else:
            nl, no = shape_for(truncation, nlat=nlat, nlon=nlon, dealias_factor=dealias_factor)
            rad = EARTH_RADIUS_M if radius_m is None else float(radius_m)
            if not math.isfinite(rad) or rad <= 0:
                raise ValueError("radius_m must be finite and positive")
            t = int(truncation)
        with torch.cuda.device(be.device):
            plan = Plan(t, nl, no, rad, prec, plan_flags)
            mu, w, cl = plan.geometry(nl)
        g = GaussianGrid.from_geometry(t, nl, no, mu, w, cl, rad)
        return cls(g, be, plan, bool(tensor_core_contractions or prec == "split16"),
                   int(legendre_band), bool(streaming), int(latitude_bands))

    # ------------------------------------------------------------- shape
    @property
    def truncation(self) -> int:
        return self.grid.truncation

    @property
    def spectral_shape(self):
        n = self.truncation + 1
        return n, n

    @property
    def precision(self) -> str:
        return self.backend.precision

    @property
    def geometry_identity(self) -> dict:
        return {
            "truncation": int(self.truncation),
            "nlat": int(self.grid.nlat),
            "nlon": int(self.grid.nlon),
            "radius_m": float(self.grid.radius_m),
            "normalization": "complex-orthonormal-condon-shortley",
            "latitude_grid": "gauss-legendre-in-sin-latitude",
        }

    @property
    def geometry_hash(self) -> str:
        raw = json.dumps(self.geometry_identity, sort_keys=True, separators=(",", ":")).encode()
        return hashlib.sha256(raw).hexdigest()

    @property
    def identity(self) -> dict:
        payload = {
            **self.geometry_identity,
            "backend": self.backend.name,
            "float_dtype": str(self.backend.float_dtype).replace("torch.", ""),
        }
        if self.precision == "split16":
            # Different arithmetic from the float32 path: never share its hash.
            payload["tensor_core_contractions"] = "split-fp16-tcgen05"
        return payload

    @property
    def identity_hash(self) -> str:
        raw = json.dumps(self.identity, sort_keys=True, separators=(",", ":")).encode()
        return hashlib.sha256(raw).hexdigest()

    # ------------------------------------------------------------ tables
    def _table(self, name: str) -> LegendreTable:
        tables = self.__dict__.setdefault("_legendre_tables", {})
        if name not in tables:
            tables[name] = LegendreTable(name, self)
        return tables[name]

    @property
    def _basis(self) -> LegendreTable:
        """P_nm (transform.py:888-899)."""
        return self._table("basis")

    @property
    def _analysis(self) -> LegendreTable:
        """The Gram-corrected analysis rows (transform.py:97-119)."""
        return self._table("analysis")

    @property
    def _derivative_basis(self) -> LegendreTable:
        """dP_nm/dphi (transform.py:901-933)."""
        return self._table("derivative_basis")

    @property
    def _dbasis(self) -> LegendreTable:
        """The derivative table.  The reference builds it on the first
        gradient and holds None until then (transform.py:905-933); the plan
        here computes dP/dphi in the same recurrence pass as P when it is
        created, so the table is always resident."""
        return self._derivative_basis

    @property
    def legendre_table_nbytes(self) -> dict[str, int]:
        """Resident table bytes by name (transform.py:936-954).  ``rotation``
        and ``shear`` are the vector analysis's weighted tables, which the
        reference forms per call; ``scratch`` is 0: the contraction reads the
        folded tables directly and expands nothing."""
        plan = self.plan
        return {
            "basis": plan.table_bytes(_lib.SHT_TABLE_BASIS),
            "analysis": plan.table_bytes(_lib.SHT_TABLE_ANALYSIS),
            "derivative": plan.table_bytes(_lib.SHT_TABLE_DBASIS),
            "rotation": plan.table_bytes(_lib.SHT_TABLE_ROTATION),
            "shear": plan.table_bytes(_lib.SHT_TABLE_SHEAR),
            "scratch": 0,
        }

    def zeros(self, *leading):
        return torch.zeros((*leading, *self.spectral_shape), dtype=self.backend.complex_dtype,
                           device=self.backend.device)

    # --------------------------------------------------------- validation
    def _validate_grid(self, f) -> None:
        if tuple(f.shape[-2:]) != self.grid.shape:
            raise ValueError(
                f"grid field has trailing shape {tuple(f.shape[-2:])}, expected {self.grid.shape}")

    def _validate_spectral(self, c) -> None:
        if tuple(c.shape[-2:]) != self.spectral_shape:
            raise ValueError(
                f"spectral field has trailing shape {tuple(c.shape[-2:])}, "
                f"expected {self.spectral_shape}")

    def _grid_in(self, field):
        f = self.backend.asarray(field, dtype=self.backend.float_dtype)
        self._validate_grid(f)
        return f.contiguous()

    def _spec_in(self, coeff):
        c = self.backend.asarray(coeff, dtype=self.backend.complex_dtype)
        self._validate_spectral(c)
        return c.contiguous()

    @staticmethod
    def _planes(t: torch.Tensor) -> int:
        return int(np.prod(t.shape[:-2], dtype=np.int64)) if t.dim() > 2 else 1

    def _empty_grid(self, lead):
        return torch.empty((*lead, *self.grid.shape), dtype=self.backend.float_dtype,
                           device=self.backend.device)

    def _empty_spec(self, lead):
        return torch.empty((*lead, *self.spectral_shape), dtype=self.backend.complex_dtype,
                           device=self.backend.device)

    # ------------------------------------------------------ contraction seam
    def _contraction_scope(self):
        """The reference scopes its TF32 compute type around each contraction
        (transform.py:1146-1176) because CuPy's compute type is process-global.
        Here the arithmetic is a property of the plan, so there is nothing to
        scope."""
        return contextlib.nullcontext()

    def _batched_contract(self, values, table, *, transposed=False, realify=False):
        """The Legendre contraction seam (transform.py:1178-1274): every
        contraction of this transform passes through here, once per
        contraction the reference performs, so a caller that replaces this
        method (the reference's census tool) counts the same calls and planes.

        ``values`` is a ``FusedOperand`` (the contraction runs inside a fused
        library call; its output is returned) or a device array:
        ``table`` analysis with ``(*lead, nlat, T+1)`` waist values gives the
        ``(*lead, T+1, T+1)`` coefficients (``sht_contract_waist``; the m = 0
        imaginary parts are stored 0, what the reference's callers store after
        it with ``realify``); ``table`` basis or derivative basis with
        ``(*lead, T+1, T+1)`` coefficients gives the ``(*lead, nlat, T+1)``
        waist (``sht_contract_to_waist``).  A transposed contraction of an
        arbitrary weighted waist is not a library operation: the vector
        analysis runs it fused (``VorticityDivergenceOperator``)."""
        self.contraction_count += 1
        if isinstance(values, FusedOperand):
            return values.result()
        from .waist import ANALYSIS, BASIS, DERIVATIVE_BASIS

        if transposed:
            raise NotImplementedError(
                "a transposed contraction of caller-weighted waist values is not a library "
                "operation here; VorticityDivergenceOperator runs the vector analysis fused")
        if table == ANALYSIS:
            v = self.backend.asarray(values, dtype=self.backend.complex_dtype).contiguous()
            if tuple(v.shape[-2:]) != (self.grid.nlat, self.truncation + 1):
                raise ValueError(f"waist values have trailing shape {tuple(v.shape[-2:])}, "
                                 f"expected {(self.grid.nlat, self.truncation + 1)}")
            out = self._empty_spec(v.shape[:-2])
            _lib.call("sht_contract_waist", self.plan.handle, _ptr(v), self._planes(v),
                      _ptr(out), _stream())
            return out
        if table in (BASIS, DERIVATIVE_BASIS):
            c = self._spec_in(values)
            out = torch.empty((*c.shape[:-2], self.grid.nlat, self.truncation + 1),
                              dtype=self.backend.complex_dtype, device=self.backend.device)
            code = _lib.SHT_WAIST_DBASIS if table == DERIVATIVE_BASIS else _lib.SHT_WAIST_BASIS
            _lib.call("sht_contract_to_waist", self.plan.handle, _ptr(c), self._planes(c),
                      int(code), _ptr(out), _stream())
            return out
        raise ValueError(f"unknown table {table!r}: expected the transform's _analysis, _basis "
                         "or _derivative_basis")

    def _agree_across_cards(self, direction: str, table, array) -> None:
        """Hand a contraction's output to the row exchange's ``agree_once``
        hook (transform.py:1405-1433); one attribute read on a one-card run."""
        exchange = self.row_exchange
        hook = getattr(exchange, "agree_once", None)
        if hook is None or int(getattr(exchange, "world", 1)) <= 1:
            return
        name = table if isinstance(table, str) else getattr(table, "name", None) or f"table@{id(table):x}"
        hook(self.backend.xp,
             (direction, name, tuple(int(v) for v in array.shape), str(array.dtype)), array)

    # ------------------------------------------------- the order axis
    @property
    def owned_order_range(self) -> tuple[int, int]:
        """``(m_lo, m_hi)`` orders this transform holds a table for
        (transform.py:828-836): every order, since one GPU holds the whole
        table (``order_partition`` is refused at ``create``)."""
        return (0, self.truncation + 1)

    def _exchange_range(self, exchange) -> tuple[int, int]:
        """The order range this rank owns, from the exchange or the table
        (transform.py:1580-1584)."""
        if exchange is not None and hasattr(exchange, "owned_order_range"):
            m_lo, m_hi = (int(v) for v in exchange.owned_order_range)
            if not 0 <= m_lo < m_hi <= self.truncation + 1:
                raise ValueError(f"the exchange's owned_order_range {(m_lo, m_hi)} is not a "
                                 f"non-empty range of orders in [0, {self.truncation + 1}]")
            return m_lo, m_hi
        return self.owned_order_range

    def _contract_orders(self, values, table, m_lo, m_hi, *, transposed=False):
        """Only orders ``[m_lo, m_hi)`` of a contraction, compactly
        (transform.py:1491-1530): the analysis of waist values gives
        ``(*lead, T+1, m_hi-m_lo)`` coefficient columns, a synthesis of
        coefficients ``(*lead, nlat, m_hi-m_lo)`` waist columns.  The whole
        table is resident, so these are the whole contraction's columns
        there, bit for bit."""
        m_lo, m_hi = int(m_lo), int(m_hi)
        if not 0 <= m_lo < m_hi <= self.truncation + 1:
            raise ValueError(f"orders [{m_lo}, {m_hi}) are not a non-empty range in "
                             f"[0, {self.truncation + 1}]")
        with self._contraction_scope():
            whole = self._batched_contract(values, table, transposed=transposed,
                                           realify=table == "analysis")
        return whole[..., m_lo:m_hi].contiguous()

    def _analyze(self, field, table=None, *, bands=None):
        """grid -> spectral through the waist (transform.py:1474-1484)."""
        return self.contract_waist(self.fourier_waist(field, bands=bands), table)

    def _synthesize(self, coeff, table=None, *, bands=None):
        """spectral -> grid through the waist (transform.py:1736-1739)."""
        return self.waist_to_grid(self.contract_to_waist(coeff, table, bands=bands))

    def _gather_order_columns(self, exchange, compact, width, *, name):
        """The whole ``(*lead, X, width)`` from every rank's columns through
        the exchange's ``gather_columns`` (transform.py:1586-1599); with no
        exchange, or a world of one, the columns are already whole."""
        if exchange is None or int(getattr(exchange, "world", 1)) <= 1:
            return compact
        full = exchange.gather_columns(self.backend.xp, compact, int(width), name=name)
        full = self.backend.asarray(full, dtype=self.backend.complex_dtype).contiguous()
        if tuple(full.shape) != (*compact.shape[:-1], int(width)):
            raise ValueError(f"gather_columns returned shape {tuple(full.shape)}, expected "
                             f"{(*compact.shape[:-1], int(width))}")
        return full

    @staticmethod
    def _multi_card(exchange) -> bool:
        return exchange is not None and int(getattr(exchange, "world", 1)) > 1

    def forward_orders(self, field, exchange=None):
        """Analysis on the order axis (transform.py:1532-1557).

        The reference's rank contracts only its own orders and the ranks
        all-gather the coefficient columns.  Here every order's table is
        resident, so the contraction runs whole on this GPU; this rank's
        owned columns still go through the exchange's ``gather_columns`` (so
        every rank takes the reference's collective step, named
        ``"analysis_orders"``) and the gathered spectrum, disjoint column
        ranges placed side by side, is the single-card spectrum bit for bit.
        With no exchange, or a world of one, this is :meth:`forward`."""
        exchange = self.order_exchange if exchange is None else exchange
        whole = self._analyze_whole(field)
        if not self._multi_card(exchange):
            return whole
        m_lo, m_hi = self._exchange_range(exchange)
        full = self._gather_order_columns(exchange, whole[..., m_lo:m_hi].contiguous(),
                                          self.truncation + 1, name="analysis_orders")
        full[..., :, 0].imag.zero_()
        return full

    def inverse_orders(self, coeff, exchange=None):
        """Synthesis on the order axis (transform.py:1559-1578): the waist
        columns of this rank's orders are gathered with every rank's
        (``"synthesis_orders"``), then the whole waist goes through the
        inverse FFT.  The contraction runs whole on this GPU (every order's
        table is resident), so the result is this engine's waist-path
        synthesis (``waist_to_grid(contract_to_waist(c))``) bit for bit.
        With no exchange, or a world of one, this is :meth:`inverse`."""
        exchange = self.order_exchange if exchange is None else exchange
        if not self._multi_card(exchange):
            return self._synth("sht_inverse", coeff)
        from .waist import FourierWaist, latitude_band_edges

        m_lo, m_hi = self._exchange_range(exchange)
        values = self.contract_to_waist(coeff).take()
        full = self._gather_order_columns(exchange, values[..., m_lo:m_hi].contiguous(),
                                          self.truncation + 1, name="synthesis_orders")
        waist = FourierWaist(self, full, latitude_band_edges(self.grid.nlat,
                                                             self.latitude_bands))
        return self.waist_to_grid(waist)

    # ------------------------------------------------- the streamed forms
    @staticmethod
    def _check_order_chunk(order_chunk) -> None:
        if order_chunk is not None and int(order_chunk) < 1:
            raise ValueError(f"order_chunk must be >= 1, got {order_chunk}")

    def forward_streaming(self, field, *, order_chunk: int | None = None):
        """:meth:`forward` without a resident table in the reference
        (transform.py:1603-1618), whose contract is the resident table's
        bits in O(order_chunk x (T+1) x nlat) host memory.  The plan here
        keeps its tables resident in HBM (T1534's few GB on a 180 GB part),
        so the streamed form is the resident contraction: the same bits,
        and no per-chunk table."""
        self._check_order_chunk(order_chunk)
        return self.forward(field)

    def inverse_streaming(self, coeff, *, order_chunk: int | None = None):
        """:meth:`inverse`; see :meth:`forward_streaming`
        (transform.py:1620-1627)."""
        self._check_order_chunk(order_chunk)
        return self.inverse(coeff)

    def streaming_working_bytes(self, order_chunk: int | None = None) -> dict[str, int]:
        """Bytes one streamed contraction holds for a chunk of orders
        (transform.py:1025-1045): none here, since the streamed forms run on
        the resident tables (``legendre_table_nbytes``) and allocate no
        per-chunk block."""
        self._check_order_chunk(order_chunk)
        return {"recurrence": 0, "analysis": 0, "device": 0, "scratch": 0}

    # ---------------------------------------------------------- transforms
    def forward(self, field):
        """grid -> spectral (transform.py:1486); on the order axis
        (:meth:`forward_orders`) when a multi-card order exchange is set."""
        if self._multi_card(self.order_exchange):
            return self.forward_orders(field)
        return self._analyze_whole(field)

    def _analyze_whole(self, field):
        f = self._grid_in(field)
        lead = tuple(f.shape[:-2])

        def run():
            out = self._empty_spec(lead)
            _lib.call("sht_forward", self.plan.handle, _ptr(f), self._planes(f), _ptr(out),
                      _stream())
            return (out,)

        (op,) = fused_operands([(*lead, self.grid.nlat, self.truncation + 1)], run)
        with self._contraction_scope():
            out = self._batched_contract(op, self._analysis, realify=True)
        self._agree_across_cards("analysis", self._analysis, out)
        return out

    def _synth(self, name, coeff, table=None):
        c = self._spec_in(coeff)
        lead = tuple(c.shape[:-2])

        def run():
            out = self._empty_grid(lead)
            _lib.call(name, self.plan.handle, _ptr(c), self._planes(c), _ptr(out), _stream())
            return (out,)

        (op,) = fused_operands([tuple(c.shape)], run)
        with self._contraction_scope():
            return self._batched_contract(op, self._basis if table is None else table)

    def inverse(self, coeff):
        """spectral -> grid (transform.py:1742); on the order axis
        (:meth:`inverse_orders`) when a multi-card order exchange is set."""
        if self._multi_card(self.order_exchange):
            return self.inverse_orders(coeff)
        return self._synth("sht_inverse", coeff)

    # ------------------------------------------------- host-resident batches
    def _host_call(self, name, src, in_dtype, in_tail, out_tail, out_dtype, out, chunk):
        """One host-streamed C-ABI call: host input, host output."""
        x = torch.as_tensor(src)
        if x.device.type != "cpu":
            raise ValueError("host-streamed calls take host (CPU) arrays")
        if x.dtype != in_dtype:
            x = x.to(in_dtype)
        x = x.contiguous()
        if tuple(x.shape[-2:]) != in_tail:
            raise ValueError(f"input has trailing shape {tuple(x.shape[-2:])}, expected {in_tail}")
        lead = tuple(x.shape[:-2])
        if out is None:
            out = torch.empty((*lead, *out_tail), dtype=out_dtype, pin_memory=True)
        elif (out.device.type != "cpu" or out.dtype != out_dtype or not out.is_contiguous()
              or tuple(out.shape) != (*lead, *out_tail)):
            raise ValueError("out must be a contiguous host tensor of shape "
                             f"{(*lead, *out_tail)} and dtype {out_dtype}")
        _lib.call(name, self.plan.handle, x.data_ptr(), self._planes(x), out.data_ptr(), int(chunk))
        return out

    def forward_host(self, field, *, out=None, chunk: int = 0):
        """grid -> spectral for host-resident fields, copies pipelined with the
        transforms in chunks of planes (sht_forward_host); returns a host
        tensor (page-locked when allocated here)."""
        return self._host_call("sht_forward_host", field, self.backend.float_dtype,
                               self.grid.shape, self.spectral_shape, self.backend.complex_dtype,
                               out, chunk)

    def inverse_host(self, coeff, *, out=None, chunk: int = 0):
        """spectral -> grid for host-resident coefficients (sht_inverse_host)."""
        return self._host_call("sht_inverse_host", coeff, self.backend.complex_dtype,
                               self.spectral_shape, self.grid.shape, self.backend.float_dtype,
                               out, chunk)

    def round_trip_host(self, field, *, out=None, chunk: int = 0):
        """inverse(forward(field)) for host-resident fields (sht_round_trip_host):
        grid in, grid out, the coefficients stay on the device."""
        return self._host_call("sht_round_trip_host", field, self.backend.float_dtype,
                               self.grid.shape, self.grid.shape, self.backend.float_dtype,
                               out, chunk)

    def inverse_meridional_derivative(self, coeff):
        """d field / d latitude in grid space (transform.py:1748)."""
        return self._synth("sht_inverse_meridional_derivative", coeff, self._derivative_basis)

    def inverse_zonal_derivative(self, coeff):
        """d field / d longitude in grid space (transform.py:1752)."""
        return self._synth("sht_inverse_zonal_derivative", coeff)

    def gradient(self, coeff):
        """Physical (east, north) derivatives per metre (transform.py:1762):
        both syntheses in one library call, two contractions at the seam."""
        c = self._spec_in(coeff)
        lead = tuple(c.shape[:-2])

        def run():
            east = self._empty_grid(lead)
            north = self._empty_grid(lead)
            _lib.call("sht_gradient", self.plan.handle, _ptr(c), self._planes(c), _ptr(east),
                      _ptr(north), _stream())
            return east, north

        op_e, op_n = fused_operands([tuple(c.shape)] * 2, run)
        with self._contraction_scope():
            east = self._batched_contract(op_e, self._basis)
            north = self._batched_contract(op_n, self._derivative_basis)
        return east, north

    def _elementwise(self, name, coeff):
        c = self._spec_in(coeff)
        out = self._empty_spec(c.shape[:-2])
        _lib.call(name, self.plan.handle, _ptr(c), self._planes(c), _ptr(out), _stream())
        return out

    def project(self, coeff):
        """Triangle mask and real m = 0 column (transform.py:1124-1144)."""
        return self._elementwise("sht_project", coeff)

    def laplacian(self, coeff):
        return self._elementwise("sht_laplacian", coeff)

    def inverse_laplacian(self, coeff):
        return self._elementwise("sht_inverse_laplacian", coeff)

    # ---------------------------------------------------------- diagnostics
    def spectral_mean_square(self, coeff) -> float:
        c = self.backend.to_numpy(coeff)
        self._validate_spectral(c)
        weight = np.ones(self.truncation + 1)
        weight[1:] = 2.0
        total = np.sum(np.abs(c) ** 2 * weight[None, :], axis=(-2, -1))
        return float(np.asarray(total).mean() / (4.0 * np.pi))

    def power_by_degree(self, coeff) -> np.ndarray:
        c = self.backend.to_numpy(coeff)
        weight = np.ones(self.truncation + 1)
        weight[1:] = 2.0
        return np.sum(np.abs(c) ** 2 * weight[None, :], axis=-1)

    def constant_coeff(self, value: float):
        out = self.zeros()
        out[0, 0] = float(value) * math.sqrt(4.0 * math.pi)
        return out

    def add_grid_constant(self, coeff, value: float):
        out = self.backend.asarray(coeff).clone()
        out[..., 0, 0] += float(value) * math.sqrt(4.0 * math.pi)
        return out

    def transform_check(self, *, seed: int = 0, max_degree=None) -> dict:
        """Round trip and Parseval KAT (transform.py:1837-1863)."""
        rng = np.random.default_rng(seed)
        t = self.truncation if max_degree is None else min(self.truncation, int(max_degree))
        coeff = np.zeros(self.spectral_shape, dtype=np.complex128)
        for n in range(t + 1):
            for m in range(n + 1):
                coeff[n, m] = rng.normal() + (0.0j if m == 0 else 1j * rng.normal())
        grid = self.inverse(coeff)
        back = self.backend.to_numpy(self.forward(grid))
        scale = max(1.0, float(np.max(np.abs(coeff))))
        error = float(np.max(np.abs(back - coeff)) / scale)
        spatial_ms = self.grid.global_mean(self.backend.to_numpy(grid) ** 2)
        spectral_ms = float(np.sum(np.abs(coeff) ** 2 * np.where(
            np.arange(self.truncation + 1)[None, :] == 0, 1.0, 2.0)) / (4.0 * np.pi))
        parseval = abs(spatial_ms - spectral_ms) / max(1.0, abs(spectral_ms))
        return {"truncation": self.truncation, "nlat": self.grid.nlat, "nlon": self.grid.nlon,
                "roundtrip_relative_linf": error, "parseval_relative_error": float(parseval)}

    def check_device(self) -> None:
        """Raise if a kernel of this plan reported a device error word."""
        self.plan.check()

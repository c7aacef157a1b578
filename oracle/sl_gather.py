"""CPU oracle of the semi-Lagrangian gathers -- TEST INFRASTRUCTURE ONLY.

Imported by ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU
legs as the checker; the product path (``b200sht.semilag``) never imports
it.  A numpy restatement, in float64 or the tables' float32, of:

* the pole-extended geometry tables of the four- and six-point meridional
  stencils (the reference's ``semilag/tables.py:51-95`` and ``:136-217``);
* the tricubic / quintic-horizontal gather with the quasi-monotone limiter,
  its clip deficit and the half-layer hold at the vertical boundaries
  (``semilag/interpolate.py:536-669``, the numpy specification the
  reference grades its kernel against);
* the trilinear gather inside the limiter's cell
  (``semilag/interpolate.py:672-725``);
* the fixed-point departure-point search and its trilinear wind read
  (``semilag/trajectory.py:493-618``).

Pinned against ``tests/golden/sl_gather_*.npz``, outputs of the reference's
own ``gather_batch`` / ``gather_linear_batch`` / ``departure_points`` (numpy
backend) recorded by
``tests/golden/make_golden_sl.py``.
"""
from __future__ import annotations

import math

import numpy as np

BINS_PER_ROW = 4


def build_tables(lat: np.ndarray, nlon: int, order: int = 4) -> dict:
    """Extended latitudes, row offsets/shifts, reciprocal Lagrange
    denominators and the bracket lookup of one stencil width
    (tables.py:164-196 for order 4, :51-95 for order 6)."""
    lat = np.asarray(lat, dtype=np.float64)
    nlat = lat.shape[0]
    ghost = order // 2
    rows = nlat + 2 * ghost
    lat_ext = np.empty(rows)
    for g in range(ghost):
        lat_ext[ghost - 1 - g] = -math.pi - lat[g]
        lat_ext[nlat + ghost + g] = math.pi - lat[nlat - 1 - g]
    lat_ext[ghost:nlat + ghost] = lat
    row = np.arange(rows) - ghost
    data = np.where(row < 0, -1 - row, np.where(row >= nlat, 2 * nlat - 1 - row, row))
    rowoff = (data * nlon).astype(np.int32)
    rowshift = np.where((row < 0) | (row >= nlat), nlon // 2, 0).astype(np.int32)
    nodes = lat_ext[np.arange(nlat + 1)[:, None] + np.arange(order)[None, :]]
    mrden = np.empty((nlat + 1, order))
    for m in range(order):
        den = np.ones(nlat + 1)
        for q in range(order):
            if q != m:
                den = den * (nodes[:, m] - nodes[:, q])
        mrden[:, m] = 1.0 / den
    bins = BINS_PER_ROW * rows
    scale = bins / math.pi
    centres = -0.5 * math.pi + (np.arange(bins) + 0.5) / scale
    mlut = np.clip(np.searchsorted(lat_ext, centres, side="right") - 1,
                   ghost - 1, nlat + ghost - 1).astype(np.int32)
    return dict(lat_ext=lat_ext, rowoff=rowoff, rowshift=rowshift, mrden=mrden, mlut=mlut,
                bins=bins, lut_scale=scale, ghost=ghost)


def _equispaced(t: np.ndarray, n: int) -> np.ndarray:
    """Normalised Lagrange weights on the nodes 0 .. n-1 at t."""
    cols = []
    for m in range(n):
        num = np.ones_like(t)
        den = 1.0
        for q in range(n):
            if q != m:
                num = num * (t - q)
                den *= (m - q)
        cols.append(num / den)
    w = np.stack(cols, axis=-1)
    return w / w.sum(axis=-1, keepdims=True)


def gather(fields, xi, phi, level, lat, nlon, *, order=4, limiter="quasi_monotone",
           deficit=False, dtype=np.float64):
    """Every field (nlev, nlat, nlon) read at the departure coordinates
    (interpolate.py:536-669).  Returns values, or (values, deficits)."""
    dtype = np.dtype(dtype)
    sc = dtype.type
    tab = build_tables(lat, nlon, order)
    lat_ext = tab["lat_ext"].astype(dtype)
    mrden = tab["mrden"].astype(dtype)
    nh, ghost = order, order // 2 - 1
    mid = nh // 2 - 1
    nlev, nlat, _ = np.shape(xi)
    plane = nlat * nlon
    flat = [np.ascontiguousarray(f, dtype=dtype).reshape(-1) for f in fields]
    outs = [np.empty((nlev, plane), dtype) for _ in fields]
    cuts = [np.zeros((nlev, plane), dtype) for _ in fields]
    half_pi = sc(np.pi / 2.0)
    for k in range(nlev):
        p = np.clip(np.asarray(phi[k], dtype).reshape(-1), -half_pi, half_pi)
        xk = np.clip(np.asarray(level[k], dtype).reshape(-1), sc(-0.5), sc(nlev - 0.5))
        below = xk < 0
        outside = below | (xk > sc(nlev - 1))
        c_edge = np.where(below, 0, 3)
        c_next = np.where(below, 1, 2)
        x = np.asarray(xi[k], dtype).reshape(-1)
        fx = np.floor(x)
        i0 = fx.astype(np.int64) - ghost
        wx = _equispaced(x - i0.astype(dtype), nh).astype(dtype)
        cols = (i0[:, None] + np.arange(nh)) % nlon
        colh = (cols + nlon // 2) % nlon
        m0 = np.clip(np.searchsorted(lat_ext.astype(np.float64), p.astype(np.float64),
                                     side="right") - 1, ghost, nlat + ghost)
        sst = m0 - ghost
        nodes = lat_ext[sst[:, None] + np.arange(nh)]
        d = p[:, None] - nodes
        wy = np.stack([np.prod(np.delete(d, m, axis=1), axis=1) for m in range(nh)], axis=-1)
        wy = wy * mrden[sst]
        wy = wy / wy.sum(axis=-1, keepdims=True)
        kb = np.clip(np.floor(xk).astype(np.int64), 0, nlev - 2)
        k0 = np.clip(kb - 1, 0, nlev - 4)
        kbox = kb - k0
        wz = _equispaced(xk - k0.astype(dtype), 4).astype(dtype)
        ridx = sst[:, None] + np.arange(nh)
        shifted = tab["rowshift"][ridx] > 0
        adr = (tab["rowoff"][ridx][:, :, None]
               + np.where(shifted[:, :, None], colh[:, None, :], cols[:, None, :]))
        cx = np.where(x - fx >= sc(0.5), mid + 1, mid)
        cy = np.where(p - nodes[:, mid] >= nodes[:, mid + 1] - p, mid + 1, mid)
        kn = np.clip(np.floor(xk + sc(0.5)).astype(np.int64), 0, nlev - 1)
        pts = np.arange(p.shape[0])
        centre = kn * plane + adr[pts, cy, cx]
        for fi, f in enumerate(flat):
            base = f[centre]
            acc = np.zeros(p.shape, dtype)
            lo = np.full(p.shape, np.inf, dtype)
            hi = np.full(p.shape, -np.inf, dtype)
            f_edge = np.zeros(p.shape, dtype)
            f_next = np.zeros(p.shape, dtype)
            for c in range(4):
                v = f[(k0 + c)[:, None, None] * plane + adr]
                inner = np.einsum("pa,pra,pr->p", wx, v - base[:, None, None], wy)
                acc = acc + wz[:, c] * inner
                f_edge = np.where(c_edge == c, inner, f_edge)
                f_next = np.where(c_next == c, inner, f_next)
                if limiter != "none":
                    inbox = (c == kbox) | (c == kbox + 1)
                    box = v[:, mid:mid + 2, mid:mid + 2].reshape(-1, 4)
                    lo = np.where(inbox, np.minimum(lo, box.min(axis=1)), lo)
                    hi = np.where(inbox, np.maximum(hi, box.max(axis=1)), hi)
            if limiter == "none":
                face = f_edge + sc(0.5) * (f_edge - f_next)
                held = np.minimum(np.maximum(acc, np.minimum(f_edge, face)),
                                  np.maximum(f_edge, face))
                acc = np.where(outside, held, acc)
            acc = acc + base
            kept = np.minimum(np.maximum(acc, lo), hi) if limiter != "none" else acc
            outs[fi][k] = kept
            if deficit:
                cuts[fi][k] = acc - kept
    shape = np.shape(xi)
    values = [o.reshape(shape) for o in outs]
    if not deficit:
        return values
    return list(zip(values, [c.reshape(shape) for c in cuts]))


def gather_linear(fields, xi, phi, level, lat, nlon, *, dtype=np.float64):
    """Trilinear value inside the limiter's cell (interpolate.py:672-725)."""
    dtype = np.dtype(dtype)
    sc = dtype.type
    tab = build_tables(lat, nlon, 4)
    lat_ext = tab["lat_ext"].astype(dtype)
    nlev, nlat, _ = np.shape(xi)
    plane = nlat * nlon
    flat = [np.ascontiguousarray(f, dtype=dtype).reshape(-1) for f in fields]
    outs = [np.empty((nlev, plane), dtype) for _ in fields]
    half_pi = sc(np.pi / 2.0)
    for k in range(nlev):
        p = np.clip(np.asarray(phi[k], dtype).reshape(-1), -half_pi, half_pi)
        xk = np.clip(np.asarray(level[k], dtype).reshape(-1), sc(0.0), sc(nlev - 1))
        x = np.asarray(xi[k], dtype).reshape(-1)
        fx = np.floor(x)
        ax = x - fx
        c0 = fx.astype(np.int64) % nlon
        c1 = (c0 + 1) % nlon
        h0 = (c0 + nlon // 2) % nlon
        h1 = (c1 + nlon // 2) % nlon
        m0 = np.clip(np.searchsorted(lat_ext.astype(np.float64), p.astype(np.float64),
                                     side="right") - 1, 1, nlat + 1)
        la, lb = lat_ext[m0], lat_ext[m0 + 1]
        ay = np.clip((p - la) / (lb - la), sc(0.0), sc(1.0))
        r0, r1 = tab["rowoff"][m0], tab["rowoff"][m0 + 1]
        s0, s1 = tab["rowshift"][m0] > 0, tab["rowshift"][m0 + 1] > 0
        i00 = r0 + np.where(s0, h0, c0)
        i01 = r0 + np.where(s0, h1, c1)
        i10 = r1 + np.where(s1, h0, c0)
        i11 = r1 + np.where(s1, h1, c1)
        kb = np.clip(np.floor(xk).astype(np.int64), 0, nlev - 2)
        az = xk - kb.astype(dtype)
        o0 = kb * plane
        o1 = o0 + plane
        bx, by, bz = 1 - ax, 1 - ay, 1 - az
        for fi, f in enumerate(flat):
            t0 = by * (bx * f[o0 + i00] + ax * f[o0 + i01]) + ay * (bx * f[o0 + i10] + ax * f[o0 + i11])
            t1 = by * (bx * f[o1 + i00] + ax * f[o1 + i01]) + ay * (bx * f[o1 + i10] + ax * f[o1 + i11])
            outs[fi][k] = bz * t0 + az * t1
    return [o.reshape(np.shape(xi)) for o in outs]


def departure_sample(nlev, lat, nlon, seed, *, cells=1.5, dtype=np.float64):
    """Seeded departure coordinates: every arrival point displaced by up to
    `cells` grid cells zonally and meridionally (the meridional offset in
    radians of one equatorial cell, so rows next to a pole reach past it)
    and up to one level vertically, reaching the half layers."""
    rng = np.random.default_rng(seed)
    lat = np.asarray(lat, dtype=np.float64)
    nlat = lat.shape[0]
    shape = (nlev, nlat, nlon)
    dlat = math.pi / nlat
    xi = np.arange(nlon)[None, None, :] + rng.uniform(-cells, cells, shape)
    phi = lat[None, :, None] + rng.uniform(-cells, cells, shape) * dlat
    level = np.arange(nlev)[:, None, None] + rng.uniform(-1.0, 1.0, shape)
    return xi.astype(dtype), phi.astype(dtype), level.astype(dtype)


def _trilinear_at(fields, lam, phi, lev, tab, nlat, nlon, dtype):
    """The search's trilinear read at (longitude, latitude, level)
    (trajectory.py:493-550): the cubic gather's cell, no clamp on the
    meridional fraction, the level held in [0, nlev - 1]."""
    sc = dtype.type
    nlev = fields[0].shape[0]
    lat_ext = tab["lat_ext"].astype(dtype)
    half_pi = sc(np.pi / 2.0)
    p = np.clip(phi, -half_pi, half_pi)
    xk = np.clip(lev, sc(0.0), sc(nlev - 1))
    x = lam * sc(1.0 / (2.0 * math.pi / nlon))
    fx = np.floor(x)
    ax = (x - fx).astype(dtype)
    c0 = fx.astype(np.int64) % nlon
    c1 = (c0 + 1) % nlon
    h0, h1 = (c0 + nlon // 2) % nlon, (c1 + nlon // 2) % nlon
    m0 = np.clip(np.searchsorted(lat_ext.astype(np.float64), p.astype(np.float64),
                                 side="right") - 1, 1, nlat + 1)
    la, lb = lat_ext[m0], lat_ext[m0 + 1]
    ay = ((p - la) / (lb - la)).astype(dtype)
    r0, r1 = tab["rowoff"][m0], tab["rowoff"][m0 + 1]
    s0, s1 = tab["rowshift"][m0] > 0, tab["rowshift"][m0 + 1] > 0
    i00, i01 = r0 + np.where(s0, h0, c0), r0 + np.where(s0, h1, c1)
    i10, i11 = r1 + np.where(s1, h0, c0), r1 + np.where(s1, h1, c1)
    k0 = np.clip(np.floor(xk).astype(np.int64), 0, nlev - 2)
    az = (xk - k0).astype(dtype)
    plane = nlat * nlon
    bx, by, bz = 1.0 - ax, 1.0 - ay, 1.0 - az
    out = []
    for f in fields:
        flat = np.ascontiguousarray(f).reshape(-1)
        b0 = k0 * plane
        b1 = b0 + plane
        t0 = by * (bx * flat[b0 + i00] + ax * flat[b0 + i01]) + ay * (bx * flat[b0 + i10] + ax * flat[b0 + i11])
        t1 = by * (bx * flat[b1 + i00] + ax * flat[b1 + i01]) + ay * (bx * flat[b1 + i10] + ax * flat[b1 + i11])
        out.append((bz * t0 + az * t1).astype(dtype))
    return out


def departure(wind, lat, nlon, dt, *, iterations=3, extrapolated=None, radius=6371220.0,
              dtype=np.float64):
    """The fixed-point departure-point search (trajectory.py:553-618):
    wind = (vx, vy, vz, level_rate), each (nlev, nlat, nlon).  Returns
    xi, phi, level, move_m, move_k."""
    dtype = np.dtype(dtype)
    sc = dtype.type
    tab = build_tables(lat, nlon, 4)
    vx, vy, vz, sv = [np.asarray(w, dtype) for w in wind]
    ex = [np.asarray(w, dtype) for w in (extrapolated or wind)]
    nlev, nlat, _ = vx.shape
    shape = vx.shape
    latd = tab["lat_ext"][2:nlat + 2].astype(dtype)
    lon = (np.arange(nlon) * (2.0 * math.pi / nlon)).astype(dtype)
    sph, cph = np.sin(latd)[None, :, None], np.cos(latd)[None, :, None]
    sla, cla = np.sin(lon)[None, None, :], np.cos(lon)[None, None, :]
    ax = np.broadcast_to(cph * cla, shape).astype(dtype)
    ay = np.broadcast_to(cph * sla, shape).astype(dtype)
    az = np.broadcast_to(sph + 0.0 * cla, shape).astype(dtype)
    ak = np.broadcast_to(np.arange(nlev, dtype=dtype)[:, None, None], shape).astype(dtype)
    r = sc(radius)
    inv_r = sc(1.0) / r
    dts = sc(dt)
    hdt = sc(0.5) * dts
    qx, qy, qz = ax - dts * vx * inv_r, ay - dts * vy * inv_r, az - dts * vz * inv_r
    nrm = np.sqrt(qx * qx + qy * qy + qz * qz)
    qx, qy, qz = qx / nrm, qy / nrm, qz / nrm
    klo, khi = sc(-0.5), sc(nlev - 0.5)
    qk = np.clip(ak - dts * sv, klo, khi)
    move_m = np.zeros(shape, dtype)
    move_k = np.zeros(shape, dtype)
    for _ in range(iterations):
        lam = np.arctan2(qy, qx)
        phi = np.arctan2(qz, np.sqrt(qx * qx + qy * qy))
        w = _trilinear_at([vx, vy, vz, sv], lam, phi, qk, tab, nlat, nlon, dtype)
        px = ax - hdt * (ex[0] + w[0]) * inv_r
        py = ay - hdt * (ex[1] + w[1]) * inv_r
        pz = az - hdt * (ex[2] + w[2]) * inv_r
        nrm = np.sqrt(px * px + py * py + pz * pz)
        px, py, pz = px / nrm, py / nrm, pz / nrm
        pk = np.clip(ak - hdt * (ex[3] + w[3]), klo, khi)
        chord = np.sqrt((px - qx) ** 2 + (py - qy) ** 2 + (pz - qz) ** 2)
        move_m = r * 2.0 * np.arcsin(np.clip(0.5 * chord, sc(0.0), sc(1.0)))
        move_k = np.abs(pk - qk)
        qx, qy, qz, qk = px, py, pz, pk
    xi = (np.arctan2(qy, qx) * sc(1.0 / (2.0 * math.pi / nlon))).astype(dtype)
    phi = np.arctan2(qz, np.sqrt(qx * qx + qy * qy)).astype(dtype)
    return xi, phi, qk.astype(dtype), move_m.astype(dtype), move_k.astype(dtype)


def departure_residual(wind, lat, nlon, dt, xi, phi, level, *, extrapolated=None,
                       radius=6371220.0):
    """How far given departure points are from solving the departure
    equation: |G(q) - q| for the fixed-point map G of ``departure`` above,
    in float64, the horizontal part in meridional grid lengths (the arc over
    pi / nlat) and the level part in levels.  Returns (cells, levels)."""
    tab = build_tables(lat, nlon, 4)
    vx, vy, vz, sv = [np.asarray(w, np.float64) for w in wind]
    ex = [np.asarray(w, np.float64) for w in (extrapolated or wind)]
    nlev, nlat, _ = vx.shape
    shape = vx.shape
    latd = tab["lat_ext"][2:nlat + 2]
    lon = np.arange(nlon) * (2.0 * math.pi / nlon)
    ax = np.broadcast_to(np.cos(latd)[None, :, None] * np.cos(lon)[None, None, :], shape)
    ay = np.broadcast_to(np.cos(latd)[None, :, None] * np.sin(lon)[None, None, :], shape)
    az = np.broadcast_to(np.sin(latd)[None, :, None] + 0.0 * lon[None, None, :], shape)
    ak = np.broadcast_to(np.arange(nlev, dtype=np.float64)[:, None, None], shape)
    lam = np.asarray(xi, np.float64) * (2.0 * math.pi / nlon)
    ph = np.asarray(phi, np.float64)
    qk = np.asarray(level, np.float64)
    qx, qy, qz = np.cos(ph) * np.cos(lam), np.cos(ph) * np.sin(lam), np.sin(ph)
    w = _trilinear_at([vx, vy, vz, sv], lam, ph, qk, tab, nlat, nlon, np.dtype(np.float64))
    hdt = 0.5 * dt
    px = ax - hdt * (ex[0] + w[0]) / radius
    py = ay - hdt * (ex[1] + w[1]) / radius
    pz = az - hdt * (ex[2] + w[2]) / radius
    nrm = np.sqrt(px * px + py * py + pz * pz)
    px, py, pz = px / nrm, py / nrm, pz / nrm
    pk = np.clip(ak - hdt * (ex[3] + w[3]), -0.5, nlev - 0.5)
    chord = np.sqrt((px - qx) ** 2 + (py - qy) ** 2 + (pz - qz) ** 2)
    arc = 2.0 * np.arcsin(np.clip(0.5 * chord, 0.0, 1.0))
    return arc * nlat / math.pi, np.abs(pk - qk)


def rotation_wind(lat, nlon, nlev, *, speed=40.0, seed=0, dtype=np.float64):
    """Seeded advecting flow: a solid-body rotation about the axis through
    (0 N, 0 E) (its flow crosses both poles) as Cartesian components, plus
    a little noise, and a level rate reaching the half layers in one 300 s
    step."""
    rng = np.random.default_rng(seed)
    lat = np.asarray(lat, np.float64)
    nlat = lat.shape[0]
    lon = np.arange(nlon) * 2 * math.pi / nlon
    x = np.cos(lat)[:, None] * np.cos(lon)[None, :]
    y = np.cos(lat)[:, None] * np.sin(lon)[None, :]
    z = np.sin(lat)[:, None] * np.ones(nlon)[None, :]
    om = speed / 6371220.0
    # V = omega x r with omega along the x axis: (0, -om z, om y) * radius
    shape = (nlev, nlat, nlon)
    scale = 1.0 + 0.1 * np.arange(nlev)[:, None, None] / nlev
    vx = np.zeros(shape) + 0.5 * rng.standard_normal(shape)
    vy = -om * z[None] * 6371220.0 * scale + 0.5 * rng.standard_normal(shape)
    vz = om * y[None] * 6371220.0 * scale + 0.5 * rng.standard_normal(shape)
    sv = 1.5e-3 * np.sin(2 * lon)[None, None, :] * np.cos(lat)[None, :, None] * np.ones(shape)
    return [a.astype(dtype) for a in (vx, vy, vz, sv)]

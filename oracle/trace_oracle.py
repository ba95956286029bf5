"""CPU oracle for field-line tracing and Q maps (TEST INFRASTRUCTURE ONLY).

The checker for the B200 tracer (``nfgs_trace_field_lines`` /
``nfgs_qmap_plane``), never the product: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU legs may import it.  FP64
NumPy, vectorised over seeds, a Python loop over steps.

The reference computes its topology maps with FastQSL (CuPy-launched CUDA,
``nfgs/_backend/util/fastqsl_plane.py:203-506``), which cannot run here (no
CuPy) and whose source is not used: this restates the published definitions
instead, the same ones the kernel implements:

* field line dr/ds = B/|B| in grid-index units, B trilinear between nodes,
  classical RK4 with a fixed step; the step that leaves the box is cut where
  its chord meets the first face (ties: x before y before z) and the end is
  snapped onto that face;
* the squashing factor Q = ||D||^2 / |det D| of the footpoint map D (Titov,
  Hornig & Demoulin 2002; Titov 2007), evaluated from a seed plane with
  in-plane unit axes u, v:
  Q = [|a+|^2 |b-|^2 + |b+|^2 |a-|^2 - 2 (a+.b+)(a-.b-)] |Bn+ Bn-| / Bn0^2,
  a = dr/du, b = dr/dv of the two end points (central differences), using
  flux conservation |det dr/d(u,v)| = |Bn0 / Bn|.

Parity with FastQSL itself is unpinned (it cannot run here); the oracle is
pinned by known answers instead: a uniform field (Q = 2) and the linear
hyperbolic field B = ((x-xc)/L, -(y-yc)/L, 1), whose footpoint map between
z = 0 and z = H is diag(e^{H/L}, e^{-H/L}), so Q = 2 cosh(2H/L).
"""

from __future__ import annotations

import numpy as np


def interp(pk, pts):
    """Trilinear B at points (m, 3) xyz, clamped into the box; pk (nz, ny, nx, 3)."""
    nz, ny, nx, _ = pk.shape
    x = np.clip(pts[:, 0], 0.0, nx - 1.0)
    y = np.clip(pts[:, 1], 0.0, ny - 1.0)
    z = np.clip(pts[:, 2], 0.0, nz - 1.0)
    i = np.minimum(np.floor(x).astype(np.int64), nx - 2)
    j = np.minimum(np.floor(y).astype(np.int64), ny - 2)
    k = np.minimum(np.floor(z).astype(np.int64), nz - 2)
    fx, fy, fz = (x - i)[:, None], (y - j)[:, None], (z - k)[:, None]
    c = [[[pk[k + dz, j + dy, i + dx] for dx in (0, 1)] for dy in (0, 1)] for dz in (0, 1)]
    x00 = c[0][0][0] + fx * (c[0][0][1] - c[0][0][0])
    x10 = c[0][1][0] + fx * (c[0][1][1] - c[0][1][0])
    x01 = c[1][0][0] + fx * (c[1][0][1] - c[1][0][0])
    x11 = c[1][1][0] + fx * (c[1][1][1] - c[1][1][0])
    y0 = x00 + fy * (x10 - x00)
    y1 = x01 + fy * (x11 - x01)
    return y0 + fz * (y1 - y0)


def curl_grid(b):
    """J = curl B in grid units with second-order differences (centred inside,
    three-point one-sided at the walls), b (3, nz, ny, nx); the reference's
    include_twist current (fastqsl_plane.py:287-305)."""
    g = [[np.gradient(b[c], axis=a, edge_order=2) for a in range(3)] for c in range(3)]  # g[c][axis z,y,x]
    return np.stack([g[2][1] - g[1][0], g[0][0] - g[2][2], g[1][2] - g[0][1]])


def trace(b, seeds, normal, step, max_steps, twist=False):
    """Trace every seed along +B and -B.  b (3, nz, ny, nx); seeds (n, 3).
    Returns ends (2, n, 3), flags (2, n), bn (3, n), length (2, n) with the
    layout and codes of nfgs_trace_field_lines; with twist=True also the
    twist of each half (2, n): J.B / (4 pi |B|^2) integrated with the RK4
    stages of the line (a cut last step contributes its fraction)."""
    b = np.asarray(b, dtype=np.float64)
    pk = np.ascontiguousarray(np.moveaxis(b, 0, -1))
    pj = np.ascontiguousarray(np.moveaxis(curl_grid(b), 0, -1)) if twist else None
    nz, ny, nx, _ = pk.shape
    hi = np.array([nx - 1.0, ny - 1.0, nz - 1.0])
    seeds = np.clip(np.asarray(seeds, dtype=np.float64).reshape(-1, 3), 0.0, hi)
    n = seeds.shape[0]
    bseed = interp(pk, seeds)
    bn = np.full((3, n), np.nan)
    bn[0] = bseed @ np.asarray(normal, dtype=np.float64)
    p = np.concatenate([seeds, seeds])
    sgn = np.concatenate([np.ones(n), -np.ones(n)])[:, None]
    flags = np.zeros(2 * n, dtype=np.int32)
    length = np.zeros(2 * n)
    tw = np.zeros(2 * n)
    act = np.arange(2 * n)

    def direction(q, s):
        v = interp(pk, q)
        m2 = (v * v).sum(axis=1)
        m = np.sqrt(m2)
        ok = m > 0
        with np.errstate(invalid="ignore", divide="ignore"):
            d = v * (s / m[:, None])
            f = (interp(pj, q) * v).sum(axis=1) / (4.0 * np.pi * m2) if twist else np.zeros(len(q))
        d[~ok] = 0.0  # the line stops there; keep later stages finite
        return d, ok, f

    for _ in range(max_steps):
        if act.size == 0:
            break
        pa, s = p[act], sgn[act]
        k1, o1, f1 = direction(pa, s)
        k2, o2, f2 = direction(pa + 0.5 * step * k1, s)
        k3, o3, f3 = direction(pa + 0.5 * step * k2, s)
        k4, o4, f4 = direction(pa + step * k3, s)
        ok = o1 & o2 & o3 & o4
        flags[act[~ok]] = -1
        q = pa + (step / 6.0) * (k1 + 2.0 * k2 + 2.0 * k3 + k4)
        dtw = (step / 6.0) * (f1 + 2.0 * f2 + 2.0 * f3 + f4)
        inside = np.all((q >= 0.0) & (q <= hi), axis=1) & ok
        p[act[inside]] = q[inside]
        length[act[inside]] += step
        tw[act[inside]] += dtw[inside]
        out = ok & ~inside
        if out.any():
            po, qo, ids = pa[out], q[out], act[out]
            t = np.full(ids.size, 2.0)
            face = np.zeros(ids.size, dtype=np.int32)
            for d in range(3):
                with np.errstate(invalid="ignore", divide="ignore"):
                    lo_t = (0.0 - po[:, d]) / (qo[:, d] - po[:, d])
                    hi_t = (hi[d] - po[:, d]) / (qo[:, d] - po[:, d])
                m_lo = (qo[:, d] < 0.0) & (lo_t < t)
                t[m_lo], face[m_lo] = lo_t[m_lo], 2 * d + 1
                m_hi = (qo[:, d] > hi[d]) & ~(qo[:, d] < 0.0) & (hi_t < t)
                t[m_hi], face[m_hi] = hi_t[m_hi], 2 * d + 2
            e = po + t[:, None] * (qo - po)
            fd = (face - 1) // 2
            e[np.arange(ids.size), fd] = np.where(face % 2 == 1, 0.0, hi[fd])
            p[ids] = e
            length[ids] += t * step
            tw[ids] += t * dtw[out]
            flags[ids] = face
        act = act[inside]
    ends = p.reshape(2, n, 3)
    flags = flags.reshape(2, n)
    for d in range(2):
        f = flags[d]
        okf = f > 0
        if okf.any():
            bv = interp(pk, ends[d][okf])
            bn[1 + d, okf] = np.abs(bv[np.arange(bv.shape[0]), (f[okf] - 1) // 2])
    if twist:
        return ends, flags, bn, length.reshape(2, n), tw.reshape(2, n)
    return ends, flags, bn, length.reshape(2, n)


def qmap(nu, nv, ends, flags, bn):
    """Q on the regular nv x nu seed plane (seed iu + nu iv); NaN on the
    border and where the five lines of a direction end on different faces."""
    q = np.full((nv, nu), np.nan)
    if nu < 3 or nv < 3:
        return q
    E = ends.reshape(2, nv, nu, 3)
    F = flags.reshape(2, nv, nu)
    c = (slice(1, -1), slice(1, -1))
    ok = np.ones((nv - 2, nu - 2), dtype=bool)
    for d in range(2):
        f = F[d]
        fc = f[c]
        ok &= (fc > 0) & (f[1:-1, 2:] == fc) & (f[1:-1, :-2] == fc) & (f[2:, 1:-1] == fc) & (f[:-2, 1:-1] == fc)
    a = [(E[d][1:-1, 2:] - E[d][1:-1, :-2]) * 0.5 for d in range(2)]
    b = [(E[d][2:, 1:-1] - E[d][:-2, 1:-1]) * 0.5 for d in range(2)]

    def dot(u, v):
        return (u * v).sum(axis=-1)

    br = dot(a[0], a[0]) * dot(b[1], b[1]) + dot(b[0], b[0]) * dot(a[1], a[1]) - 2.0 * dot(a[0], b[0]) * dot(a[1], b[1])
    B = bn.reshape(3, nv, nu)
    with np.errstate(invalid="ignore", divide="ignore"):
        val = br * np.abs(B[1][c] * B[2][c]) / (B[0][c] * B[0][c])
    q[c] = np.where(ok, val, np.nan)
    return q


def hyperbolic_field(nx, ny, nz, scale):
    """B = ((x - xc)/L, -(y - yc)/L, 1) on the nodes, (3, nz, ny, nx)."""
    z, y, x = np.meshgrid(np.arange(nz, dtype=np.float64), np.arange(ny, dtype=np.float64),
                          np.arange(nx, dtype=np.float64), indexing="ij")
    xc, yc = 0.5 * (nx - 1), 0.5 * (ny - 1)
    return np.stack([(x - xc) / scale, -(y - yc) / scale, np.ones_like(z)])


def dipole_field(nx, ny, nz, depth=6.0, tilt=0.4):
    """Field of a point dipole buried `depth` cells below the centre of the
    bottom face, moment tilted by `tilt` rad from vertical in x-z: a smooth
    closed-loop test field (3, nz, ny, nx)."""
    z, y, x = np.meshgrid(np.arange(nz, dtype=np.float64), np.arange(ny, dtype=np.float64),
                          np.arange(nx, dtype=np.float64), indexing="ij")
    r = np.stack([x - 0.5 * (nx - 1), y - 0.5 * (ny - 1), z + depth])
    m = np.array([np.sin(tilt), 0.0, np.cos(tilt)])
    rr = np.sqrt((r * r).sum(axis=0))
    mr = (m[:, None, None, None] * r).sum(axis=0)
    return (3.0 * mr * r / rr ** 5 - m[:, None, None, None] / rr ** 3) * depth ** 3


def perp_frame(B):
    """Unit vectors e1, e2 perpendicular to B (m, 3): e1 = unit(b x a) with a
    the coordinate axis least aligned with b, e2 = b x e1; |B| (m,)."""
    bm = np.sqrt((B * B).sum(axis=1))
    with np.errstate(invalid="ignore", divide="ignore"):
        b = B / bm[:, None]
    ax = np.argmin(np.abs(b), axis=1)  # first minimum: x before y before z
    a = np.eye(3)[ax]
    c = np.cross(b, a)
    with np.errstate(invalid="ignore", divide="ignore"):
        e1 = c / np.sqrt((c * c).sum(axis=1))[:, None]
    e2 = np.cross(b, e1)
    return bm, e1, e2


def qperp(b, seeds, delta, step, max_steps):
    """Q_perp (Titov 2007) at each seed from five lines traced both ways (the
    seed and seed +- delta e1, +- delta e2); returns q (n,) and the central
    line's (ends, flags, bn = (|B0|, |Bn+|, |Bn-|), length)."""
    b = np.asarray(b, dtype=np.float64)
    pk = np.ascontiguousarray(np.moveaxis(b, 0, -1))
    nz, ny, nx, _ = pk.shape
    hi = np.array([nx - 1.0, ny - 1.0, nz - 1.0])
    s0 = np.clip(np.asarray(seeds, dtype=np.float64).reshape(-1, 3), 0.0, hi)
    n = s0.shape[0]
    bm, e1, e2 = perp_frame(interp(pk, s0))
    ok = bm > 0
    e1[~ok] = 0.0
    e2[~ok] = 0.0
    aux = [s0, s0 + delta * e1, s0 - delta * e1, s0 + delta * e2, s0 - delta * e2]
    allseeds = np.clip(np.concatenate(aux), 0.0, hi)
    ends, flags, bnx, length = trace(b, allseeds, (0.0, 0.0, 1.0), step, max_steps)
    E = ends.reshape(2, 5, n, 3)
    F = flags.reshape(2, 5, n)
    F[:, :, ~ok] = -1
    good = np.ones(n, dtype=bool)
    for d in range(2):
        good &= (F[d, 0] > 0) & np.all(F[d] == F[d, 0][None], axis=0)
    a = [(E[d, 1] - E[d, 2]) / (2.0 * delta) for d in range(2)]
    bb = [(E[d, 3] - E[d, 4]) / (2.0 * delta) for d in range(2)]

    def dot(u, v):
        return (u * v).sum(axis=-1)

    br = dot(a[0], a[0]) * dot(bb[1], bb[1]) + dot(bb[0], bb[0]) * dot(a[1], a[1]) - 2.0 * dot(a[0], bb[0]) * dot(a[1], bb[1])
    bne = bnx[1:].reshape(2, 5, n)[:, 0]
    with np.errstate(invalid="ignore", divide="ignore"):
        q = np.where(good & ok, br * np.abs(bne[0] * bne[1]) / (bm * bm), np.nan)
    bn = np.stack([np.where(ok, bm, 0.0), bne[0], bne[1]])
    return q, E[:, 0], F[:, 0], bn, length.reshape(2, 5, n)[:, 0]

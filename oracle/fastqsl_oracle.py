"""CPU restatement of the reference's FastQSL tracing and Q (test
infrastructure: only the tests use it, as the checker).

The reference's topology maps (nfgs/_backend/util/fastqsl_plane.py:203-506)
trace with the vendored FastQSL adaptive tracer (TraceAllBline,
third_party/FastQSL/fastqslpy/cu/TraceBlineAdaptive.cu:333-512) and form Q
with QCalcPlane (fastqslpy/FastQSL.py:65-122).  ``trace_seed`` follows the
tracer in FP32 scalar arithmetic with the double-precision steps where the
reference has them (one seed at a time: slow, for a handful of seeds);
``qcalc_plane`` is the plane formula on NumPy arrays.
"""

from __future__ import annotations

import math

import numpy as np

F = np.float32
TOL0 = 1e-3
PI_REF = 3.14159265

# Fehlberg 4(5) (Fehlberg 1969) as single-precision constants
A = {k: F(v) for k, v in dict(
    a21=1 / 4, a31=3 / 32, a32=9 / 32, a41=1932 / 2197, a42=-7200 / 2197, a43=7296 / 2197,
    a51=439 / 216, a52=-8.0, a53=3680 / 513, a54=-845 / 4104,
    a61=-8 / 27, a62=2.0, a63=-3544 / 2565, a64=1859 / 4104, a65=-11 / 40,
    b1=16 / 135, b3=6656 / 12825, b4=28561 / 56430, b5=-9 / 50, b6=2 / 55,
    e1=1 / 360, e3=-128 / 4275, e4=-2197 / 75240, e5=1 / 50, e6=2 / 55).items()}


def _v(x, y, z):
    return np.array([x, y, z], dtype=F)


def interp_dir(b, p, norm=True):
    """Trilinear vector of b (3, nz, ny, nx) at p = (x, y, z) with the faces'
    outermost cell, weights in double (TraceBlineAdaptive.cu:101-200)."""
    _, nz, ny, nx = b.shape
    n = (nx, ny, nz)
    r = [F(p[d] - np.floor(p[d])) for d in range(3)]
    idx = [int(np.floor(p[d])) if np.isfinite(p[d]) else 0 for d in range(3)]
    for d in range(3):
        if p[d] <= 0:
            r[d], idx[d] = F(0), 0
        if p[d] >= n[d] - 1:
            r[d], idx[d] = F(1), n[d] - 2
        if not 0 <= idx[d] <= n[d] - 2:
            idx[d] = 0
    i, j, k = idx
    rx, ry, rz = (float(v) for v in r)
    ux, uy, uz = 1.0 - rx, 1.0 - ry, 1.0 - rz
    w = [F(ux * uy * uz), F(ux * uy * rz), F(ux * ry * uz), F(ux * ry * rz),
         F(rx * uy * uz), F(rx * uy * rz), F(rx * ry * uz), F(rx * ry * rz)]
    corners = [(i, j, k), (i, j, k + 1), (i, j + 1, k), (i, j + 1, k + 1),
               (i + 1, j, k), (i + 1, j, k + 1), (i + 1, j + 1, k), (i + 1, j + 1, k + 1)]
    out = np.zeros(3, dtype=F)
    for c in range(3):
        acc = F(0)
        for q, (a, bb, cc) in enumerate(corners):
            acc = F(acc + F(b[c, cc, bb, a] * w[q]))
        out[c] = acc
    if norm:
        m = F(np.sqrt(F(F(out[0] * out[0] + out[1] * out[1]) + out[2] * out[2])))
        out = (out / m).astype(F)
    return out


def interp_sample(b, p):
    """Trilinear sample in double inside [1e-4, N - 1 - 1e-4]
    (TraceBlineAdaptive.cu:46-99)."""
    _, nz, ny, nx = b.shape
    n = (nx, ny, nz)
    q = [F(p[d]) for d in range(3)]
    for d in range(3):
        q[d] = q[d] if q[d] > 0 else F(0.0001)
        q[d] = q[d] if q[d] < n[d] - 1 else F(float(F(n[d]) - F(1)) - 0.0001)
    r = [float(F(q[d] - np.floor(q[d]))) for d in range(3)]
    i, j, k = (min(max(int(np.floor(q[d])), 0), n[d] - 2) for d in range(3))
    rx, ry, rz = r
    out = np.zeros(3, dtype=F)
    for c in range(3):
        a = b[c]
        v = (float(a[k, j, i]) * (1 - rx) * (1 - ry) * (1 - rz) + float(a[k + 1, j, i]) * (1 - rx) * (1 - ry) * rz
             + float(a[k, j + 1, i]) * (1 - rx) * ry * (1 - rz) + float(a[k + 1, j + 1, i]) * (1 - rx) * ry * rz
             + float(a[k, j, i + 1]) * rx * (1 - ry) * (1 - rz) + float(a[k + 1, j, i + 1]) * rx * (1 - ry) * rz
             + float(a[k, j + 1, i + 1]) * rx * ry * (1 - rz) + float(a[k + 1, j + 1, i + 1]) * rx * ry * rz)
        out[c] = F(v)
    return out


def rkf45(b, p, h):
    """One Fehlberg step (TraceBlineAdaptive.cu:215-251): the fifth-order end
    point and the error norm."""
    g = lambda q: (h * interp_dir(b, q)).astype(F)  # noqa: E731
    k1 = g(p)
    k2 = g(p + A["a21"] * k1)
    k3 = g(p + (A["a31"] * k1 + A["a32"] * k2))
    k4 = g(p + (A["a41"] * k1 + A["a42"] * k2 + A["a43"] * k3))
    k5 = g(p + (A["a51"] * k1 + A["a52"] * k2 + A["a53"] * k3 + A["a54"] * k4))
    k6 = g(p + (A["a61"] * k1 + A["a62"] * k2 + A["a63"] * k3 + A["a64"] * k4 + A["a65"] * k5))
    e = A["e1"] * k1 + A["e3"] * k3 + A["e4"] * k4 + A["e5"] * k5 + A["e6"] * k6
    err = F(np.sqrt(F(F(e[0] * e[0] + e[1] * e[1]) + e[2] * e[2])))
    return (p + (A["b1"] * k1 + A["b3"] * k3 + A["b4"] * k4 + A["b5"] * k5 + A["b6"] * k6)).astype(F), err


def rk4_face(b, p, s, d):
    """Runge-Kutta step of length s in coordinate d (TraceBlineAdaptive.cu:
    282-306)."""
    def k(q):
        u = interp_dir(b, q)
        return (u / u[d]).astype(F)
    s = F(s)
    k1 = k(p)
    k2 = k(p + (s * k1) / F(2))
    k3 = k(p + (s * k2) / F(2))
    k4 = k(p + s * k3)
    return (p + F((1.0 / 6.0) * float(s)) * (k1 + F(2) * k2 + F(2) * k3 + k4)).astype(F)


def face_code(shape_xyz, p):
    """0 inside, 1..6 through one face, 42 otherwise (TraceBlineAdaptive.cu:
    308-331; y exactly 0 counts as outside)."""
    X, Y, Z = (n - 1 for n in shape_xyz)
    x, y, z = (float(v) for v in p)
    if x >= 0 and y > 0 and z >= 0 and x <= X and y <= Y and z <= Z:
        return 0
    c = 42
    lx, ly, lz = x < X, y < Y, z < Z
    if x < 0 and y >= 0 and z >= 0 and lx and ly and lz:
        c = 1
    if x >= 0 and y >= 0 and z >= 0 and not lx and ly and lz:
        c = 2
    if x >= 0 and y < 0 and z >= 0 and lx and ly and lz:
        c = 3
    if x >= 0 and y >= 0 and z >= 0 and lx and not ly and lz:
        c = 4
    if x >= 0 and y >= 0 and z < 0 and lx and ly and lz:
        c = 5
    if x >= 0 and y >= 0 and z >= 0 and lx and ly and not lz:
        c = 6
    return c


def trace_line(b, p0, normal, h, tol_coef, direction, cur=None):
    """One line (TraceBlineAdaptive.cu:333-427): returns (code, end point,
    path length, twist)."""
    _, nz, ny, nx = b.shape
    shp = (nx, ny, nz)
    len_lim = 3.0 * (nx + ny + nz)
    n0 = np.asarray(normal, dtype=F)
    u0 = interp_dir(b, p0)
    bn = abs(F(F(F(u0[0] * n0[0]) + F(u0[1] * n0[1])) + F(u0[2] * n0[2])))
    tol = F(TOL0 / 8e3) if float(bn) <= 0.05 else F(TOL0 * float(F(np.power(bn, F(1.5)))))
    tol = F(tol * F(tol_coef))
    h = F(h)
    p1 = np.asarray(p0, dtype=F)
    pout = p1.copy()
    length, tw, code, steps = 0.0, 0.0, 0, 0
    while code == 0 and length < len_lim and steps < 500000:
        p2, err = rkf45(b, p1, F(h * F(direction)))
        with np.errstate(divide="ignore", invalid="ignore"):  # err = 0 gives an infinite factor, as on the device
            scale = F(np.power(F(float(F(tol / err)) / 11.09), F(0.2)))
        if float(scale) < 0.618:
            h = F(float(h) * 0.618)
            continue
        h = F(h * scale)
        if float(h) > 100.0:
            h = F(100.0)
        if float(h) < 0.1:
            h = F(0.1)
        dv = p1 - p2
        dl = F(np.sqrt(F(F(dv[0] * dv[0] + dv[1] * dv[1]) + dv[2] * dv[2])))
        length += float(dl)
        dtw = 0.0
        if cur is not None:
            c1 = interp_dir(cur, p1, norm=False)
            b1 = interp_dir(b, p1, norm=False)
            num = F(F(F(c1[0] * b1[0]) + F(c1[1] * b1[1])) + F(c1[2] * b1[2]))
            den = F(F(F(b1[0] * b1[0]) + F(b1[1] * b1[1])) + F(b1[2] * b1[2]))
            dtw = float(F(num / den)) / 4.0 / PI_REF * float(dl)
            tw += dtw
        code = face_code(shp, p2)
        if code > 0:
            length -= float(dl)
            tw -= dtw
            if code <= 6:
                d = (code - 1) // 2
                q1, q2 = p1[d], p2[d]
                if abs(float(F(q1 - q2))) > 1e-3:
                    qm = F(0) if code % 2 == 1 else F(shp[d])
                    u1, u2 = interp_dir(b, p1), interp_dir(b, p2)
                    if abs(float(u1[d])) < 0.2 or abs(float(u2[d])) < 0.2:
                        pout = ((p1 * F(q2 - qm) + p2 * F(qm - q1)) / F(q2 - q1)).astype(F)
                    else:
                        p2 = rk4_face(b, p1, F(qm - q1), d)
                        pout = p2
                    length += float(abs(F(qm - q1))) / (1e-4 + abs(float(u1[d])))
                else:
                    pout = p1
            else:
                pout = p2
        p1 = p2
        steps += 1
    if code == 0:
        pout = p1
    return code, pout, length, tw


def trace_seed(b, seed, normal, step_len=1.0 / 8.0, tol=0.1, cur=None):
    """TraceAllBline for one seed (TraceBlineAdaptive.cu:429-512): the end
    along +B, the start along -B, B at the seed and both ends, the summed
    path length and twist."""
    p0 = np.asarray(seed, dtype=F)
    ce, pe, le, te = trace_line(b, p0, normal, step_len, tol, 1.0, cur)
    cs, ps, ls, ts = trace_line(b, p0, normal, step_len, tol, -1.0, cur)
    return {"flag_end": ce, "end": pe, "flag_start": cs, "start": ps, "length": le + ls, "twist": te + ts,
            "b_inp": interp_sample(b, p0), "b_end": interp_sample(b, pe), "b_start": interp_sample(b, ps)}


def _face_xy(x, y, z, flags):
    X = np.zeros(flags.shape, dtype=F)
    Y = np.zeros(flags.shape, dtype=F)
    d = (flags - 1) // 2
    X[d == 2], Y[d == 2] = x[d == 2], y[d == 2]
    X[d == 1], Y[d == 1] = z[d == 1], x[d == 1]
    X[d == 0], Y[d == 0] = y[d == 0], z[d == 0]
    return X, Y


def qcalc_plane(end_xyz, flag_end, start_xyz, flag_start, bz_start, bz_end, b_inp, normal, stride=1.0):
    """QCalcPlane (fastqslpy/FastQSL.py:65-122) on (nv, nu) plane arrays:
    end/start (nv, nu, 3), flags (nv, nu), b_inp (nv, nu, 3).  The border is
    NaN, as fastqsl_plane.py:345-347 pads it."""
    X2, Y2 = _face_xy(end_xyz[..., 0], end_xyz[..., 1], end_xyz[..., 2], flag_end)
    X1, Y1 = _face_xy(start_xyz[..., 0], start_xyz[..., 1], start_xyz[..., 2], flag_start)
    c = (slice(1, -1), slice(1, -1))
    mism = np.zeros(flag_end.shape, dtype=np.int64)[c]
    for f in (flag_start, flag_end):
        for sl in ((slice(2, None), slice(1, -1)), (slice(0, -2), slice(1, -1)),
                   (slice(1, -1), slice(2, None)), (slice(1, -1), slice(0, -2))):
            mism = mism + np.abs(f[sl].astype(np.int64) - f[c])
    dx = lambda A: A[2:, 1:-1] - A[:-2, 1:-1]  # noqa: E731
    dy = lambda A: A[1:-1, 2:] - A[1:-1, :-2]  # noqa: E731
    a = dx(X2) * dy(Y1) - dy(X2) * dx(Y1)
    b = dy(X2) * dx(X1) - dx(X2) * dy(X1)
    cc = dx(Y2) * dy(Y1) - dy(Y2) * dx(Y1)
    d = dy(Y2) * dx(X1) - dx(Y2) * dy(X1)
    n = np.asarray(normal, dtype=F)
    bnorm = (b_inp[..., 0] * n[0] + b_inp[..., 1] * n[1] + b_inp[..., 2] * n[2]).astype(F)
    sc = F(1.0) / (F(2.0) * F(stride))
    with np.errstate(divide="ignore", invalid="ignore"):
        bnr = np.abs(bz_start[c]) / np.abs(bnorm[c]) ** 2 * np.abs(bz_end[c]) * sc ** 4
        q = (a ** 2 + b ** 2 + cc ** 2 + d ** 2) * bnr
    q = q.astype(F)
    q[q < 1.0] = 1.0
    q[mism > 0] = np.nan
    out = np.full(flag_end.shape, np.nan, dtype=F)
    out[c] = q
    return out

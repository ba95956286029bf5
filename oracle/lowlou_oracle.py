"""Low & Lou (1990) analytic force-free field (test infrastructure).

The reference builds its config-1 boundary and its "analytic interior" with
``get_analytic_b_field`` (nfgs/_backend/util/lnl_io.py:97-153), which
evaluates the published Low & Lou separable solution from the eigenfunction
P(mu) of the angular ODE

    (1 - mu^2) P'' + n (n + 1) P + a^2 (1 + n) / n P |P|^(2/n) = 0,
    P(-1) = P(1) = 0,  P'(-1) = 10,

solved by SciPy's collocation BVP solver (lnl_io.py:45-94).  The boundary
value problem itself is not restated here: the piecewise-cubic interpolant
the solver returns (breakpoints and coefficients) and the eigenvalue a^2
are recorded from the reference by tests/golden/make_fp32_golden.py, and
this module rebuilds that same interpolant and evaluates the field:

    A = P(mu) / r^n,  Q = a A |A|^(1/n),
    B_r = (1 / (r^2 sin t)) dA/dt,  B_t = -(1 / (r sin t)) dA/dr,
    B_p = Q / (r sin t)

in a frame tilted by psi about y and shifted by l below the surface, then
rotated back to Cartesian (x, y, z).  Only tests import this module.
"""

from __future__ import annotations

import numpy as np
from scipy.interpolate import PPoly


def profile(breaks, coeffs):
    """The cubic interpolant of the BVP solution: mu -> (P, dP/dmu)."""
    pp = PPoly(np.asarray(coeffs, dtype=np.float64), np.asarray(breaks, dtype=np.float64))
    return lambda mu: np.moveaxis(pp(mu), -1, 0)


def lowlou_field(breaks, coeffs, a2, *, n=1, l=0.3, psi=np.pi / 4, resolution=(64, 64, 64),
                 bounds=(-1.0, 1.0, -1.0, 1.0, 0.0, 2.0), dtype=np.float64, eps=1e-12):
    """(Nx, Ny, Nz, 3) field on the node lattice of ``bounds`` (lnl_io.py:97-153)."""
    dt = np.dtype(dtype)
    nx, ny, nz = resolution
    xs = np.linspace(bounds[0], bounds[1], nx, dtype=dt)
    ys = np.linspace(bounds[2], bounds[3], ny, dtype=dt)
    zs = np.linspace(bounds[4], bounds[5], nz, dtype=dt)
    x, y, z = np.meshgrid(xs, ys, zs, indexing="ij")
    c, s = np.cos(psi), np.sin(psi)
    # tilted frame: (X, Y, Z) = R_psi (x, y, z + l)
    X = x * c - (z + l) * s
    Y = y
    Z = x * s + (z + l) * c
    rho2 = X * X + Y * Y
    r = np.sqrt(rho2 + Z * Z + eps)
    t = np.arctan2(np.sqrt(rho2), Z)
    ph = np.arctan2(Y, X)
    st, ct = np.sin(t), np.cos(t)
    P, dP = profile(breaks, coeffs)(ct)
    rn = r ** n
    A = P / rn
    dA_dt = -st / rn * dP
    dA_dr = P * (-n * r ** (-n - 1))
    Q = np.sqrt(a2) * A * np.abs(A) ** (1.0 / n)
    br = dA_dt / (r * r * st + eps)
    bt = -dA_dr / (r * st + eps)
    bp = Q / (r * st + eps)
    cp, sp = np.cos(ph), np.sin(ph)
    BX = br * st * cp + bt * ct * cp - bp * sp
    BY = br * st * sp + bt * ct * sp + bp * cp
    BZ = br * ct - bt * st
    out = np.stack([BX * c + BZ * s, BY, -BX * s + BZ * c], axis=-1)
    return np.real(out).astype(dt, copy=False)


def zyx_components(field_xyz3):
    """(Nx, Ny, Nz, 3) -> three (Nz, Ny, Nx) volumes, the solver's layout."""
    return [np.ascontiguousarray(np.transpose(field_xyz3[..., i], (2, 1, 0))) for i in range(3)]

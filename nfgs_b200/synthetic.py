"""Seeded synthetic boundaries for benchmarks and tests.

* ``td_bottom``: a Titov-Demoulin-type flux rope (Titov & Demoulin 1999,
  A&A 351, 707): a ring current of major radius R and minor radius a whose
  centre lies at depth d, two magnetic charges +-q at (+-L, 0, -d) on the
  ring's symmetry axis, and a line current I0 along that axis giving the
  toroidal field.  The ring's vector potential is the standard circular
  loop potential with complete elliptic integrals outside the tube and its
  first-order continuation in k inside the tube; B = curl A is taken with
  centred differences.  The ring current I takes the equilibrium value of
  the published model.  Only the z = 0 plane is returned; ``td_volume``
  returns the 3-D field for metric checks.
* ``sunspot_magnetogram``: 2-6 Gaussian spots with random twist, net flux
  balanced to zero.
* ``quadrupole_magnetogram``: four Gaussian poles with random shear.

All units are the model's own; grids are (ny, nx) maps in zyx order.
"""

from __future__ import annotations

import numpy as np
from scipy import special

__all__ = ["td_params", "td_bottom", "td_volume", "sunspot_magnetogram", "quadrupole_magnetogram",
           "bipolar_boundary"]


def td_params(seed: int, R=3.0, a=1.0, d=1.5, L=2.0, q=None, twist=None) -> dict:
    """Seeded TD parameters: q in [0.5, 2], I0 = -sign * I_eq * U(0.8, 1.2)."""
    rng = np.random.default_rng(seed)
    q = float(rng.uniform(0.5, 2.0)) if q is None else float(q)
    l_i = 0.5
    I_eq = 8.0 * np.pi * q * L * R * (R * R + L * L) ** -1.5 / (np.log(8.0 * R / a) - 1.5 + l_i / 2.0)
    f = float(rng.uniform(0.8, 1.2)) if twist is None else float(twist)
    return {"R": R, "a": a, "d": d, "L": L, "q": q, "I": I_eq, "I0": -f * I_eq}


def _ring_potential(x, y, z, R, a, d, I):
    """theta-component of the ring-current vector potential (mu = 1)."""
    rp = np.sqrt(y * y + (z + d) ** 2)
    rp = np.maximum(rp, 1e-12)
    rho = np.sqrt(x * x + (rp - R) ** 2)

    def A_of_k(k):
        m = np.clip(k * k, 0.0, 1.0 - 1e-15)
        K = special.ellipk(m)
        E = special.ellipe(m)
        return ((2.0 - m) * K - 2.0 * E) / np.maximum(k, 1e-15)

    k = 2.0 * np.sqrt(rp * R / ((rp + R) ** 2 + x * x))
    outside = (I / (2.0 * np.pi)) * np.sqrt(R / rp) * A_of_k(k)
    # inside the tube: first-order continuation from the tube surface
    ka = 2.0 * np.sqrt(rp * R / (4.0 * rp * R + a * a))
    h = 1e-6
    dA = (A_of_k(ka + h) - A_of_k(ka - h)) / (2.0 * h)
    inside = (I / (2.0 * np.pi)) * np.sqrt(R / rp) * (A_of_k(ka) + dA * (k - ka))
    return np.where(rho < a, inside, outside), rp


def _td_B(x, y, z, p, h=1e-4):
    R, a, d, L, q, I, I0 = p["R"], p["a"], p["d"], p["L"], p["q"], p["I"], p["I0"]
    # charges
    B = np.zeros((3,) + x.shape)
    for sgn, xc in ((1.0, L), (-1.0, -L)):
        rx, ry, rz = x - xc, y, z + d
        r3 = np.maximum((rx * rx + ry * ry + rz * rz) ** 1.5, 1e-12)
        B[0] += sgn * q * rx / r3
        B[1] += sgn * q * ry / r3
        B[2] += sgn * q * rz / r3

    # ring current: A = A_theta theta_hat, theta_hat = (0, -(z+d)/rp, y/rp)
    def A_vec(xx, yy, zz):
        At, rp = _ring_potential(xx, yy, zz, R, a, d, I)
        return np.zeros_like(At), -At * (zz + d) / rp, At * yy / rp

    def dA(axis):
        e = [0.0, 0.0, 0.0]
        e[axis] = h
        ap = A_vec(x + e[0], y + e[1], z + e[2])
        am = A_vec(x - e[0], y - e[1], z - e[2])
        return [(ap[c] - am[c]) / (2 * h) for c in range(3)]

    dx_, dy_, dz_ = dA(0), dA(1), dA(2)
    B[0] += dy_[2] - dz_[1]
    B[1] += dz_[0] - dx_[2]
    B[2] += dx_[1] - dy_[0]
    # line current along the symmetry axis: B = I0 / (2 pi rp) theta_hat,
    # confined by a smooth cut-off to the flux-rope neighbourhood
    rp = np.maximum(np.sqrt(y * y + (z + d) ** 2), 1e-12)
    rho = np.sqrt(x * x + (rp - R) ** 2)
    inside = np.exp(-(rho / a) ** 4)
    bt = I0 / (2.0 * np.pi * rp) * (R / a) * inside
    B[1] += -bt * (z + d) / rp
    B[2] += bt * y / rp
    return B


def td_bottom(nx: int, ny: int, seed: int = 0, extent: float = 8.0, **kw):
    """Bottom maps (Bx, By, Bz), each (ny, nx), of a TD-type rope on [-extent, extent]^2."""
    p = td_params(seed, **kw)
    xs = np.linspace(-extent, extent, nx)
    ys = np.linspace(-extent, extent, ny)
    y, x = np.meshgrid(ys, xs, indexing="ij")
    B = _td_B(x, y, np.zeros_like(x), p)
    return B[0], B[1], B[2]


def td_volume(nx: int, ny: int, nz: int, seed: int = 0, extent: float = 8.0, **kw):
    """(3, nz, ny, nx) field on [-extent, extent]^2 x [0, extent]."""
    p = td_params(seed, **kw)
    xs = np.linspace(-extent, extent, nx)
    ys = np.linspace(-extent, extent, ny)
    zs = np.linspace(0.0, extent, nz)
    z, y, x = np.meshgrid(zs, ys, xs, indexing="ij")
    return _td_B(x, y, z, p)


def sunspot_magnetogram(n: int, seed: int, ny: int | None = None):
    """2-6 Gaussian spots (sigma 4-16 cells, |Bz| <= 1), random twist, zero net flux."""
    ny = n if ny is None else ny
    rng = np.random.default_rng(seed)
    y, x = np.meshgrid(np.arange(ny, dtype=np.float64), np.arange(n, dtype=np.float64), indexing="ij")
    ns = int(rng.integers(2, 7))
    bz = np.zeros_like(x)
    bx = np.zeros_like(x)
    by = np.zeros_like(x)
    support = np.zeros_like(x, dtype=bool)
    for s in range(ns):
        cx, cy = rng.uniform(0.25 * n, 0.75 * n), rng.uniform(0.25 * ny, 0.75 * ny)
        sig = rng.uniform(4.0, 16.0)
        amp = rng.uniform(0.3, 1.0) * (1 if s % 2 == 0 else -1)
        g = np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * sig * sig))
        bz += amp * g
        tw = rng.uniform(-1.0, 1.0)
        bx += -tw * amp * (y - cy) / sig * g
        by += tw * amp * (x - cx) / sig * g
        support |= g > 1e-3
    bz[support] -= bz[support].mean()
    m = np.abs(bz).max()
    if m > 1.0:
        bz, bx, by = bz / m, bx / m, by / m
    return bx, by, bz


def quadrupole_magnetogram(n: int, seed: int, sigma: float = 24.0):
    """Four Gaussian poles (sigma cells) with random shear."""
    rng = np.random.default_rng(seed)
    y, x = np.meshgrid(np.arange(n, dtype=np.float64), np.arange(n, dtype=np.float64), indexing="ij")
    c = (n - 1) / 2.0
    off = n / 6.0
    bz = np.zeros_like(x)
    bx = np.zeros_like(x)
    by = np.zeros_like(x)
    for (sx, sy, sg) in ((1, 1, 1), (-1, 1, -1), (-1, -1, 1), (1, -1, -1)):
        cx, cy = c + sx * off + rng.uniform(-4, 4), c + sy * off + rng.uniform(-4, 4)
        g = np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * sigma * sigma))
        bz += sg * g
        sh = rng.uniform(-0.6, 0.6)
        bx += sh * sg * (y - cy) / sigma * g
        by += -sh * sg * (x - cx) / sigma * g
    return bx, by, bz


def bipolar_boundary(ny: int, nx: int, seed: int):
    """Small sheared bipolar region used by the parity tests."""
    rng = np.random.default_rng(seed)
    y, x = np.meshgrid(np.arange(ny, dtype=np.float64), np.arange(nx, dtype=np.float64), indexing="ij")
    cx, cy = (nx - 1) / 2 + rng.uniform(-1, 1), (ny - 1) / 2 + rng.uniform(-1, 1)
    s = min(nx, ny) / 6.0
    sep = min(nx, ny) / 5.0
    g1 = np.exp(-((x - cx - sep) ** 2 + (y - cy) ** 2) / (2 * s * s))
    g2 = np.exp(-((x - cx + sep) ** 2 + (y - cy) ** 2) / (2 * s * s))
    shear = rng.uniform(0.2, 0.5)
    return (-shear * (y - cy) / s * (g1 + g2) + 0.05, shear * (x - cx) / s * (g1 - g2) - 0.03, g1 - 0.9 * g2)

"""Seeded synthetic boundaries for benchmarks and tests.

* ``td_bottom`` / ``td_volume``: the Titov-Demoulin flux rope (Titov &
  Demoulin 1999, A&A 351, 707) as the reference generates it
  (``generate_td_model``, nfgs/_backend/td.py:370-581): two magnetic
  charges +-q at (+-L, 0, -d); a ring current of major radius R and minor
  radius a centred at depth d whose vector potential is the circular-loop
  potential with complete elliptic integrals outside the tube and its
  first-order continuation in k inside, differentiated exactly (chain rule
  in k); a line current I0 along the ring's symmetry axis whose toroidal
  field is the model's sqrt(1/R^2 + 2 chi (1 - rho^2/a^2) I^2/(a^2 I0^2)) +
  1/r - 1/R profile; the ring current I at the model's equilibrium value.
  Only the z = 0 plane is returned by ``td_bottom``.
* ``sunspot_magnetogram``: 2-6 Gaussian spots with random twist, net flux
  balanced to zero.
* ``quadrupole_magnetogram``: four Gaussian poles with random shear.

All units are the model's own; grids are (ny, nx) maps in zyx order.
"""

from __future__ import annotations

import numpy as np

__all__ = ["td_params", "td_bottom", "td_volume", "sunspot_magnetogram", "quadrupole_magnetogram",
           "bipolar_boundary"]


MU0_TD = 4.0 * np.pi * 1e-1  # the reference generator's permeability (td.py:385)


def td_params(seed: int, R=3.0, a=1.0, d=1.5, L=2.0, q=None, twist=None, l_i=0.5) -> dict:
    """Seeded TD parameters: q ~ U(0.5, 2); I0 = -f I_eq with f ~ U(0.8, 1.2).

    I_eq is the equilibrium ring current of the model (td.py:401-403); the
    minus sign is the reference generator's internal I0 convention, opposite
    to the published table (nfgs/_backend/scripts/run_analytic_validation.py:670)."""
    rng = np.random.default_rng(seed)
    q = float(rng.uniform(0.5, 2.0)) if q is None else float(q)
    I_eq = td_ring_current(q, R, a, L, l_i)
    f = float(rng.uniform(0.8, 1.2)) if twist is None else float(twist)
    return {"R": R, "a": a, "d": d, "L": L, "q": q, "I": I_eq, "I0": -f * I_eq, "l_i": l_i}


def td_ring_current(q, R, a, L, l_i=0.5, mu0=MU0_TD):
    """Equilibrium ring current of the TD model (td.py:401-403)."""
    return (8.0 * np.pi * q * L * R * (R * R + L * L) ** -1.5 / mu0) / (np.log(8.0 * R / a) - 1.5 + l_i / 2.0)


def _loop_kernel(k, K, E, eps):
    """A(k) = ((2 - k^2) K - 2 E) / k of the circular-loop potential and its
    first k-derivative, with the reference's guards near k = 0 and k = 1."""
    k2 = k * k
    omk2 = np.maximum(1.0 - k2, eps)
    A = ((2.0 - k2) * K - 2.0 * E) / np.where(k == 0.0, 1e-30, k)
    dA = ((2.0 - k2) * E - 2.0 * omk2 * K) / (np.maximum(k2, eps) * omk2)
    dA = np.where(k2 < max(eps, 1e-30), 0.0, dA)
    return A, dA, omk2


def td99_field(x, y, z, *, R, a, d, L, q, I0, l_i=0.5, mu0=MU0_TD, p_bt=1.0, k_eps=1e-12):
    """(Bx, By, Bz) of the TD model at points x, y, z (any equal shapes)."""
    from scipy import special as sp

    x, y, z = (np.asarray(v, dtype=np.float64) for v in (x, y, z))
    I = td_ring_current(q, R, a, L, l_i, mu0)
    zd = z + d
    r = np.sqrt(y * y + zd * zd)
    rho = np.sqrt(x * x + (r - R) ** 2)
    inside = (a - rho > 0).astype(np.float64)
    rs = np.where(r == 0.0, 1e-30, r)
    # magnetic charges
    bx = np.zeros_like(x)
    by = np.zeros_like(x)
    bz = np.zeros_like(x)
    for sgn, xc in ((1.0, L), (-1.0, -L)):
        rx = x - xc
        r3 = (rx * rx + y * y + zd * zd) ** 1.5
        bx += sgn * q * rx / r3
        by += sgn * q * y / r3
        bz += sgn * q * zd / r3
    # toroidal field of the axial line current, along theta = (0, -(z+d), y)/r
    prof = np.maximum(0.0, 1.0 - rho * rho / (a * a)) * float(p_bt)
    root = np.sqrt(np.maximum(1.0 / (R * R) + 2.0 * inside / (a * a) * (I * I / (I0 * I0)) * prof, 0.0))
    bt = (mu0 * I0 / (2.0 * np.pi)) * (root + 1.0 / r - 1.0 / R)
    by += -bt * zd / r
    bz += bt * y / r
    # poloidal field of the ring current from its exact potential derivatives
    s2 = (r + R) ** 2 + x * x
    k = 2.0 * np.sqrt(r * R) / np.sqrt(s2)
    ka = 2.0 * np.sqrt(r * R) / np.sqrt(4.0 * r * R + a * a)
    if k_eps > 0.0:
        k = np.clip(k, 0.0, 1.0 - k_eps)
        ka = np.clip(ka, 0.0, 1.0 - k_eps)
    dk_dx = -x * k / s2
    dk_dr = k * (R * R + x * x - r * r) / (2.0 * rs * s2)
    dka_dr = ka * a * a / (2.0 * rs * (a * a + 4.0 * R * r))
    A_k, dA_k, _ = _loop_kernel(k, sp.ellipk(k * k), sp.ellipe(k * k), k_eps)
    Ka, Ea = sp.ellipk(ka * ka), sp.ellipe(ka * ka)
    A_a, dA_a, omka2 = _loop_kernel(ka, Ka, Ea, k_eps)
    ka2 = ka * ka
    kas = np.where(ka == 0.0, 1e-30, ka)
    d2A_a = ((7.0 * ka2 - 4.0 - ka2 * ka2) * (Ea / omka2) + (4.0 - 5.0 * ka2) * Ka) / (kas ** 3 * omka2)
    d2A_a = np.where(ka2 < max(k_eps, 1e-30), 0.0, d2A_a)
    pre = (mu0 * I / (2.0 * np.pi)) * np.sqrt(R / rs)
    A_out = pre * A_k
    A_in = pre * (A_a + dA_a * (k - ka))
    dAdx = np.where(inside > 0, pre * dA_a * dk_dx, pre * dA_k * dk_dx)
    dAdr = np.where(inside > 0, pre * (dA_a * dk_dr + d2A_a * dka_dr * (k - ka)) - A_in * 0.5 / rs,
                    pre * dA_k * dk_dr - A_out * 0.5 / rs)
    A_I = np.where(inside > 0, A_in, A_out)
    bperp = -dAdx
    bx += dAdr + A_I / rs
    by += bperp * (y / rs)
    bz += bperp * (zd / rs)
    return bx, by, bz


def td_bottom(nx: int, ny: int, seed: int = 0, extent: float = 8.0, **kw):
    """Bottom maps (Bx, By, Bz), each (ny, nx), of the TD rope on [-extent, extent]^2."""
    p = td_params(seed, **kw)
    xs = np.linspace(-extent, extent, nx)
    ys = np.linspace(-extent, extent, ny)
    y, x = np.meshgrid(ys, xs, indexing="ij")
    return td99_field(x, y, np.zeros_like(x), **{k: p[k] for k in ("R", "a", "d", "L", "q", "I0", "l_i")})


def td_volume(nx: int, ny: int, nz: int, seed: int = 0, extent: float = 8.0, **kw):
    """(3, nz, ny, nx) field on [-extent, extent]^2 x [0, extent]."""
    p = td_params(seed, **kw)
    xs = np.linspace(-extent, extent, nx)
    ys = np.linspace(-extent, extent, ny)
    zs = np.linspace(0.0, extent, nz)
    z, y, x = np.meshgrid(zs, ys, xs, indexing="ij")
    return np.stack(td99_field(x, y, z, **{k: p[k] for k in ("R", "a", "d", "L", "q", "I0", "l_i")}))


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

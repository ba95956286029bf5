"""CPU oracle for the soft_cfcf start (TEST INFRASTRUCTURE ONLY).

The checker for the B200 soft_cfcf kernel, never the product: only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU legs may
import it.  FP64 NumPy, vectorised over a batch of horizontal modes, loops
over heights.

What it restates (``nfgs_solver.py`` of spaceprod/NFGS):

* ``_soft_constrained_profile`` (nfgs_solver.py:6234-6270): the z profile of
  one horizontal mode as an affine function of free unknowns, with the bottom
  value (and, for Phi, the bottom Neumann row ``D_z p(0) = k p(0)``) and the
  transparent top Robin row ``(3u_N - 4u_{N-1} + u_{N-2})/(2dz) + k u_N = 0``
  eliminated exactly;
* the modal quadratic (nfgs_solver.py:6321-6405): rows ``|D_z L_k Phi|^2 +
  (k^2+eps)|L_k Phi|^2`` over interior heights for Phi, ``|L_k A|^2 +
  eps(|D_z A|^2 + k^2|A|^2)`` for A_z, with ``L_k = D_zz - k^2``, assembled
  into banded normal equations, optional diagonal ridge;
* the banded Cholesky solve with its pivot floor (nfgs_solver.py:6272-6319);
* the modal energies (nfgs_solver.py:6486-6540).

The arithmetic follows the reference's operation order (affine sums term by
term, rows in height order, keys ascending within a row, no fused
multiply-add), so the CUDA kernel, which follows the same order, can be
compared with it exactly.
"""

from __future__ import annotations

import numpy as np

_EPS64 = float(np.finfo(np.float64).eps)


class Expr:
    """Affine expression sum_i c_i u_i + const over a modal batch: `coef`
    maps an unknown index to a batch array (keys in insertion order)."""

    __slots__ = ("coef", "const")

    def __init__(self, coef, const):
        self.coef = coef
        self.const = const


def combine(terms, batch):
    """sum_t scale_t * expr_t, keys merged in order of first appearance
    (nfgs_solver.py:6151-6170)."""
    coef: dict[int, np.ndarray] = {}
    const = np.zeros(batch)
    for scale, e in terms:
        s = np.broadcast_to(np.asarray(scale, dtype=np.float64), (batch,))
        const = const + s * e.const
        for idx, c in e.coef.items():
            v = s * c
            coef[idx] = (coef[idx] + v) if idx in coef else (0.0 + v)
    return Expr(coef, const)


def profile_exprs(k, bottom, kind, nz, dz):
    """The nz affine plane values of each mode and the unknown count
    (nfgs_solver.py:6234-6270)."""
    batch = k.shape[0]
    zero = np.zeros(batch)
    one = np.ones(batch)
    denom = 3.0 + (2.0 * dz) * k
    f = [None] * nz
    f[0] = Expr({}, bottom)
    if kind == "phi":
        n = nz - 3
        f[1] = Expr({0: 0.25 * one}, (0.75 + (0.5 * dz) * k) * bottom)
        for z in range(2, nz - 1):
            f[z] = Expr({z - 2: one}, zero)
    elif kind == "az":
        n = nz - 2
        for z in range(1, nz - 1):
            f[z] = Expr({z - 1: one}, zero)
    else:
        raise ValueError("kind must be 'phi' or 'az'")
    f[nz - 1] = combine([(4.0 / denom, f[nz - 2]), (-1.0 / denom, f[nz - 3])], batch)
    return f, n


def _lap(f, z, k2, dz, batch):
    """L_k at an interior height: D_zz (centred) minus k^2
    (nfgs_solver.py:6204-6219, 6329-6335)."""
    i2 = 1.0 / (dz ** 2)
    d2 = combine([(i2, f[z - 1]), (-2.0 * i2, f[z]), (i2, f[z + 1])], batch)
    return combine([(1.0, d2), (-k2, f[z])], batch)


def _d1(seq, j, dz, batch):
    """Second-order first derivative of a list of expressions at j
    (nfgs_solver.py:6172-6199)."""
    h = 1.0 / (2.0 * dz)
    m = len(seq)
    if j == 0:
        return combine([(-3.0 * h, seq[0]), (4.0 * h, seq[1]), (-h, seq[2])], batch)
    if j == m - 1:
        return combine([(3.0 * h, seq[m - 1]), (-4.0 * h, seq[m - 2]), (h, seq[m - 3])], batch)
    return combine([(-h, seq[j - 1]), (h, seq[j + 1])], batch)


def quadratic_rows(f, k, kind, nz, dz, epsilon, batch):
    """(expression, weight) rows of the modal functional
    (nfgs_solver.py:6337-6359)."""
    k2 = k * k
    rows = []
    if kind == "phi":
        lap = [_lap(f, z, k2, dz, batch) for z in range(1, nz - 1)]
        for j in range(nz - 2):
            rows.append((_d1(lap, j, dz, batch), 1.0))
            rows.append((lap[j], 1.0 * (k2 + epsilon)))
    else:
        for z in range(1, nz - 1):
            rows.append((_lap(f, z, k2, dz, batch), 1.0))
            if epsilon > 0.0:
                rows.append((_d1(f, z, dz, batch), 1.0 * epsilon))
                rows.append((f[z], (1.0 * epsilon) * k2))
    return rows


def normal_equations(rows, n, batch, ridge):
    """Banded normal matrix lower[d, b, i] = H[b, i, i-d] and gradient
    (nfgs_solver.py:6361-6389)."""
    bw = 0
    for e, _w in rows:
        if e.coef:
            bw = max(bw, max(e.coef) - min(e.coef))
    lower = np.zeros((bw + 1, batch, n))
    grad = np.zeros((batch, n))
    for e, w in rows:
        items = sorted(e.coef.items())
        for i, ci in items:
            wci = w * ci
            grad[:, i] += wci * e.const
            for j, cj in items:
                if j > i:
                    break
                lower[i - j, :, i] += wci * cj
    dscale = np.maximum(np.abs(lower[0]).max(axis=-1), 1.0)
    lower[0] += ridge * dscale[:, None]
    return lower, grad


def banded_cholesky_solve(lower, rhs):
    """Batched banded SPD solve with the pivot floor eps * max(1, max|diag|)
    (nfgs_solver.py:6272-6319)."""
    bw = lower.shape[0] - 1
    batch, n = rhs.shape
    fac = lower.copy()
    floor = _EPS64 * np.maximum(np.abs(lower[0]).max(axis=-1), 1.0)
    for i in range(n):
        dg = lower[0, :, i].copy()
        for o in range(1, min(bw, i) + 1):
            dg -= fac[o, :, i] * fac[o, :, i]
        fac[0, :, i] = np.sqrt(np.maximum(dg, floor))
        for r in range(i + 1, min(n, i + bw + 1)):
            v = lower[r - i, :, r].copy()
            for c in range(max(0, i - bw, r - bw), i):
                v -= fac[r - c, :, r] * fac[i - c, :, i]
            fac[r - i, :, r] = v / fac[0, :, i]
    y = np.empty_like(rhs)
    for i in range(n):
        v = rhs[:, i].copy()
        for o in range(1, min(bw, i) + 1):
            v -= fac[o, :, i] * y[:, i - o]
        y[:, i] = v / fac[0, :, i]
    x = np.empty_like(rhs)
    for i in range(n - 1, -1, -1):
        v = y[:, i].copy()
        for r in range(i + 1, min(n, i + bw + 1)):
            v -= fac[r - i, :, r] * x[:, r]
        x[:, i] = v / fac[0, :, i]
    return x


def modal_profiles(k, bottom, kind, nz, dz, epsilon, ridge):
    """(nz, batch) FP64 profiles of the modes with k > 0; zero where k <= 0
    (nfgs_solver.py:6321-6425)."""
    k = np.asarray(k, dtype=np.float64).reshape(-1)
    bottom = np.asarray(bottom, dtype=np.float64).reshape(-1)
    out = np.zeros((nz, k.size))
    act = np.nonzero(k > 0.0)[0]
    if act.size == 0:
        return out
    ka, ba = k[act], bottom[act]
    batch = act.size
    f, n = profile_exprs(ka, ba, kind, nz, dz)
    rows = quadratic_rows(f, ka, kind, nz, dz, float(epsilon), batch)
    lower, grad = normal_equations(rows, n, batch, float(ridge))
    u = banded_cholesky_solve(lower, -grad)
    if not np.isfinite(u).all():
        raise RuntimeError("soft_cfcf modal normal solve produced non-finite values")
    prof = np.empty((nz, batch))
    for z, e in enumerate(f):
        v = e.const.copy()
        for idx, c in e.coef.items():
            v += c * u[:, idx]
        prof[z] = v
    out[:, act] = prof
    return out


def modal_energies(phi_hat, k_phi, az_hat, k_az, nx, ny, dx, dy, dz):
    """curl-current and current energies of the modal profiles
    (nfgs_solver.py:6486-6540): phi_hat (nz, ny, nx) DCT-I modes, az_hat
    (nz, ny-2, nx-2) DST-I modes."""
    phi = np.asarray(phi_hat, dtype=np.float64)
    kp2 = np.asarray(k_phi, dtype=np.float64) ** 2
    q = (phi[2:] - 2.0 * phi[1:-1] + phi[:-2]) / (dz * dz) - kp2[None] * phi[1:-1]
    dq = np.empty_like(q)
    dq[0] = (-3.0 * q[0] + 4.0 * q[1] - q[2]) / (2.0 * dz)
    dq[1:-1] = (q[2:] - q[:-2]) / (2.0 * dz)
    dq[-1] = (3.0 * q[-1] - 4.0 * q[-2] + q[-3]) / (2.0 * dz)
    phi_cur = kp2 * (q * q).sum(axis=0)
    phi_curl = kp2 * (dq * dq + kp2[None] * q * q).sum(axis=0)
    az = np.asarray(az_hat, dtype=np.float64)
    ka2 = np.asarray(k_az, dtype=np.float64) ** 2
    qa = (az[2:] - 2.0 * az[1:-1] + az[:-2]) / (dz * dz) - ka2[None] * az[1:-1]
    da = (az[2:] - az[:-2]) / (2.0 * dz)
    az_cur = ka2 * (da * da + ka2[None] * az[1:-1] ** 2).sum(axis=0)
    az_curl = ka2 * (qa * qa).sum(axis=0)
    wx = np.ones(nx)
    wy = np.ones(ny)
    wx[[0, -1]] = 0.5
    wy[[0, -1]] = 0.5
    w = wy[:, None] * wx[None, :]
    fac = dx * dy * dz / (4.0 * (nx - 1) * (ny - 1))
    return {"curl_current_energy": float(fac * ((w * phi_curl).sum() + az_curl.sum())),
            "current_energy": float(fac * ((w * phi_cur).sum() + az_cur.sum()))}

"""CPU oracle of the evaluation metrics (test infrastructure).

A plain NumPy (FP64) restatement of the reference's solution metrics, which
the CUDA pass nfgs_field_metrics computes in one sweep.  Only tests and the
bench's CPU leg use it.  It follows:

* the second-order derivative, curl and divergence of
  nfgs/diagnostics/common_fd2.py:21-56 (central interior, three-point
  one-sided ends, full volume first, then the region of interest);
* the common-FD2 sigma_J of common_fd2.py:59-78;
* the reference-field metrics of nfgs/_backend/util/metrics.py:123-178 and
  nfgs/_backend/scripts/recompute_td_referee_diagnostics.py:344-400
  (C_vec, C_CS, E'_n, E'_m, epsilon, sigma_J on the solver's own current,
  divB normalised by 6 mean|B| / h_eff, h_eff = 3 / (1/dx + 1/dy + 1/dz) as in
  nfgs/controlled.py:84-87);
* the region helpers of metrics.py:9-54 and the Fortran CWsin box of
  metrics.py:89-120.

Pinned against outputs of the reference's own functions on seeded fields
(tests/golden/metrics_golden.npz, made by tests/golden/make_metrics_golden.py).
"""

from __future__ import annotations

import math

import numpy as np

B_FLOOR = 1.0e-10


def derivative(f, h, axis):
    """common_fd2.py:21-37."""
    m = np.moveaxis(np.asarray(f, dtype=np.float64), axis, 0)
    out = np.empty_like(m)
    n = m.shape[0]
    if n == 1:
        out[...] = 0.0
    elif n == 2:
        out[0] = (m[1] - m[0]) / h
        out[1] = out[0]
    else:
        out[1:-1] = (m[2:] - m[:-2]) / (2.0 * h)
        out[0] = (-3.0 * m[0] + 4.0 * m[1] - m[2]) / (2.0 * h)
        out[-1] = (3.0 * m[-1] - 4.0 * m[-2] + m[-3]) / (2.0 * h)
    return np.moveaxis(out, 0, axis)


def curl(b, spacing):
    """(Bx, By, Bz) z-y-x volumes -> (Jx, Jy, Jz); common_fd2.py:40-48."""
    dx, dy, dz = spacing
    bx, by, bz = b
    return (derivative(bz, dy, 1) - derivative(by, dz, 0),
            derivative(bx, dz, 0) - derivative(bz, dx, 2),
            derivative(by, dx, 2) - derivative(bx, dy, 1))


def divergence(b, spacing):
    """common_fd2.py:51-56."""
    dx, dy, dz = spacing
    return derivative(b[0], dx, 2) + derivative(b[1], dy, 1) + derivative(b[2], dz, 0)


def _cwsin_sums(j, b):
    bn = np.sqrt(np.sum(b * b, axis=0))
    jxb = np.cross(np.moveaxis(j, 0, -1), np.moveaxis(b, 0, -1), axis=-1)
    return float(np.sum(np.linalg.norm(jxb, axis=-1) / np.maximum(bn, B_FLOOR))), float(
        np.sum(np.sqrt(np.sum(j * j, axis=0))))


def field_metrics(ref, sol, cur, spacing, roi):
    """All metrics of one region.

    ref, sol, cur: (3, nz, ny, nx) arrays (ref or cur may be None);
    roi: (z0, z1, y0, y1, x0, x1), half-open.  Returns a dict with the keys
    of nfgs_b200.metrics.METRIC_NAMES."""
    sol = np.asarray(sol, dtype=np.float64)
    z0, z1, y0, y1, x0, x1 = roi
    s = (slice(None), slice(z0, z1), slice(y0, y1), slice(x0, x1))
    b = sol[s]
    count = b[0].size
    out = dict.fromkeys(("C_vec", "C_CS", "Eprime_n", "Eprime_m", "epsilon", "sigma_J"), math.nan)
    if ref is not None:
        B = np.asarray(ref, dtype=np.float64)[s]
        Bn = np.sqrt(np.sum(B * B, axis=0))
        bn = np.sqrt(np.sum(b * b, axis=0))
        dot = np.sum(B * b, axis=0)
        diff = np.sqrt(np.sum((b - B) ** 2, axis=0))
        ref2, sol2 = float(np.sum(B * B)), float(np.sum(b * b))
        out["C_vec"] = float(np.sum(dot)) / (math.sqrt(ref2 * sol2) + 1.0e-12)
        out["C_CS"] = float(np.sum(dot / (Bn * bn + 1.0e-12))) / max(count, 1)
        out["Eprime_n"] = 1.0 - float(np.sum(diff)) / (float(np.sum(Bn)) + 1.0e-12)
        out["Eprime_m"] = 1.0 - float(np.sum(diff / (Bn + 1.0e-12))) / max(count, 1)
        out["epsilon"] = sol2 / (ref2 + 1.0e-12)
    if cur is not None:
        num, den = _cwsin_sums(np.asarray(cur, dtype=np.float64)[s], b)
        out["sigma_J"] = num / max(den, 1.0e-30)
    jf = np.stack(curl(sol, spacing))[s]
    num, den = _cwsin_sums(jf, b)
    out["sigma_J_common_fd2"] = num / max(den, 1.0e-30)
    div = divergence(sol, spacing)[s[1:]]
    h_eff = 3.0 / sum(1.0 / h for h in spacing)
    mean_div = float(np.sum(np.abs(div))) / max(count, 1)
    mean_b = float(np.sum(np.sqrt(np.sum(b * b, axis=0)))) / max(count, 1)
    out["divB_normalized"] = mean_div / (6.0 * mean_b / h_eff + 1.0e-12)
    out["cells"] = float(count)
    out["sum_b2"] = float(np.sum(b * b))
    out["sum_ref2"] = float(np.sum(np.asarray(ref, dtype=np.float64)[s] ** 2)) if ref is not None else math.nan
    return out


def flux_rope_center_from_bottom_jz(jz):
    """metrics.py:9-20."""
    w = np.abs(np.asarray(jz, dtype=np.float64))
    tot = float(w.sum()) + 1e-30
    ny, nx = w.shape
    jj, ii = np.meshgrid(np.arange(ny, dtype=np.float64), np.arange(nx, dtype=np.float64), indexing="ij")
    return (int(np.clip(np.round(np.sum(w * jj) / tot), 0, ny - 1)),
            int(np.clip(np.round(np.sum(w * ii) / tot), 0, nx - 1)))


def fortran_box(nz, ny, nx):
    """Region of the Fortran CWsin check, metrics.py:107-113, as (z0,z1,y0,y1,x0,x1)."""
    ax, ay, az = nx // 8, ny // 8, nz // 4
    return (1, max(1, nz - az), ay, min(ny, max(ay + 1, ny - ay + 1)), ax, min(nx, max(ax + 1, nx - ax + 1)))

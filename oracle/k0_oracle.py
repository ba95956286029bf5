"""FP64 NumPy restatement of the NFGS k_h=0 closures (test infrastructure).

This module is part of the oracle: only the tests, the smoke check and the
CPU legs of the benchmark use it, as the checker.  The product computes the
closures on the GPU.

The horizontally uniform part of the field, H(z) = (H_x(z), H_y(z)), is
carried outside the DCT/DST scalars of the NFGS solver.  Two closures make
it a per-height unknown driven by the horizontal mean of the parallel
current:

* ``coupled_k0`` (nfgs_solver.py:5058-5067, 5262-5431): a least-squares fit
  of dH/dz to the target mean current with H(0) fixed, on vertical faces
  ("staggered_face_D1_true_three_point_curvature") or on planes
  ("legacy_plane_centred"), with an optional curvature penalty;
* ``constrained_spline_harmonic`` (nfgs_solver.py:5099-5260): H is a clamped
  cubic B-spline whose coefficients solve the same face fit under two exact
  constraints, H(0) = observed and a one-sided FD2 dH/dz = 0 at the top.

The per-step update (nfgs_solver.py:5952-6067) fits H_x to the mean of J_y
and H_y to minus the mean of J_x, with the current's mean taken as the DCT-I
zero mode of each plane (nfgs_solver.py:4466-4468).
"""

from __future__ import annotations

import math

import numpy as np


def open_uniform_cubic_bspline(n_points: int, n_basis: int) -> np.ndarray:
    """Clamped open-uniform cubic B-spline collocation matrix (n_points x
    n_basis) on t = linspace(0, 1, n_points), built by the Cox-de Boor
    recursion (nfgs_solver.py:5099-5147)."""
    degree = 3
    inner = n_basis - degree - 1
    knots = [0.0] * (degree + 1) + [i / (inner + 1) for i in range(1, inner + 1)] + [1.0] * (degree + 1)
    kn = np.asarray(knots, dtype=np.float64)
    t = np.linspace(0.0, 1.0, n_points)
    width = kn.size - 1
    cur = np.zeros((n_points, width))
    for i in range(width):
        cur[:, i] = ((t >= kn[i]) & (t < kn[i + 1])).astype(np.float64)
    cur[-1, -1] = 1.0
    for order in range(1, degree + 1):
        nxt = np.zeros((n_points, width - 1))
        for i in range(width - 1):
            left = kn[i + order] - kn[i]
            right = kn[i + order + 1] - kn[i + 1]
            if left > 0.0:
                nxt[:, i] += (t - kn[i]) / left * cur[:, i]
            if right > 0.0:
                nxt[:, i] += (kn[i + order + 1] - t) / right * cur[:, i + 1]
        cur = nxt
        width -= 1
        cur[-1] = 0.0
        cur[-1, -1] = 1.0
    if cur.shape != (n_points, n_basis):
        raise RuntimeError(f"unexpected B-spline basis shape {cur.shape}")
    return cur


def face_difference(nz: int, dz: float) -> np.ndarray:
    """(nz-1) x nz forward difference onto vertical faces."""
    d = np.zeros((max(nz - 1, 0), nz))
    for r in range(nz - 1):
        d[r, r] = -1.0 / dz
        d[r, r + 1] = 1.0 / dz
    return d


def three_point_curvature(nz: int, dz: float) -> np.ndarray:
    """(nz-2) x nz matrix of dz * d2/dz2 (three-point)."""
    c = np.zeros((max(nz - 2, 0), nz))
    for r in range(nz - 2):
        c[r, r] = 1.0 / dz
        c[r, r + 1] = -2.0 / dz
        c[r, r + 2] = 1.0 / dz
    return c


def centred_difference(nz: int, dz: float) -> np.ndarray:
    """nz x nz plane-centred derivative with one-sided FD2 ends (the legacy
    discretization, nfgs_solver.py:5312-5333)."""
    d = np.zeros((nz, nz))
    if nz >= 3:
        for r in range(1, nz - 1):
            d[r, r - 1] = -0.5 / dz
            d[r, r + 1] = 0.5 / dz
        d[0, :3] = [-1.5 / dz, 2.0 / dz, -0.5 / dz]
        d[nz - 1, nz - 3:] = [0.5 / dz, -2.0 / dz, 1.5 / dz]
    elif nz == 2:
        d[:] = [[-1.0 / dz, 1.0 / dz], [-1.0 / dz, 1.0 / dz]]
    return d


class CoupledK0:
    """Least-squares H(z) with H(0) fixed (nfgs_solver.py:5262-5419)."""

    def __init__(self, nz: int, dz: float, smoothness: float, legacy: bool):
        self.nz, self.dz, self.legacy = nz, float(dz), bool(legacy)
        self.root = math.sqrt(smoothness)
        if legacy:
            self.D = centred_difference(nz, dz)
            self.C = self.D @ self.D
            blocks = [self.D[1:, 1:]]
            if self.root > 0.0 and nz >= 2:
                blocks.append(self.root * self.C[1:, 1:])
        else:
            self.D = face_difference(nz, dz)
            self.C = three_point_curvature(nz, dz)
            blocks = [self.D[:, 1:]]
            if self.C.shape[0] > 0 and self.root > 0.0:
                blocks.append(self.root * self.C[:, 1:])
        self.A = np.concatenate(blocks, axis=0)
        self.L = np.linalg.cholesky(self.A.T @ self.A)

    def solve(self, q: np.ndarray, h0: float) -> np.ndarray:
        q = np.asarray(q, dtype=np.float64)
        if self.legacy:
            rhs = [q[1:] - self.D[1:, 0] * h0]
            if self.root > 0.0:
                rhs.append(-self.root * self.C[1:, 0] * h0)
        else:
            qf = 0.5 * (q[:-1] + q[1:])
            rhs = [qf - self.D[:, 0] * h0]
            if self.C.shape[0] > 0 and self.root > 0.0:
                rhs.append(-self.root * self.C[:, 0] * h0)
        b = self.A.T @ np.concatenate(rhs)
        y = np.linalg.solve(self.L, b)
        x = np.linalg.solve(self.L.T, y)
        return np.concatenate([[h0], x])

    def centre_derivative(self, prof: np.ndarray) -> np.ndarray:
        """dH/dz at the planes (nfgs_solver.py:5406-5432)."""
        if self.legacy:
            return (self.D @ prof.T).T
        return centre_derivative_fd2(prof, self.dz)


def centre_derivative_fd2(prof: np.ndarray, dz: float) -> np.ndarray:
    """Face differences averaged to the planes, one-sided FD2 at both ends
    (nfgs_solver.py:5413-5432)."""
    nz = prof.shape[1]
    out = np.zeros_like(prof)
    if nz < 2:
        return out
    face = (prof[:, 1:] - prof[:, :-1]) / dz
    if nz == 2:
        out[:, 0] = face[:, 0]
        out[:, 1] = face[:, 0]
        return out
    out[:, 1:-1] = 0.5 * (face[:, :-1] + face[:, 1:])
    out[:, 0] = (-3.0 * prof[:, 0] + 4.0 * prof[:, 1] - prof[:, 2]) / (2.0 * dz)
    out[:, -1] = (3.0 * prof[:, -1] - 4.0 * prof[:, -2] + prof[:, -3]) / (2.0 * dz)
    return out


class SplineK0:
    """Constrained cubic B-spline H(z) (nfgs_solver.py:5149-5260): least
    squares of the face derivative against the target plus a curvature
    penalty, a 1e-12 relative ridge, and exact H(0) and top FD2 H' = 0 rows
    through a KKT system."""

    def __init__(self, nz: int, dz: float, n_basis: int, smoothness: float):
        self.nz, self.dz, self.nb = nz, float(dz), int(n_basis)
        self.smoothness = float(smoothness)
        self.basis = open_uniform_cubic_bspline(nz, self.nb)
        self.D = face_difference(nz, dz)
        self.C = three_point_curvature(nz, dz)
        blocks = [self.D @ self.basis]
        if self.smoothness > 0.0 and self.C.shape[0] > 0:
            blocks.append(math.sqrt(self.smoothness) * (self.C @ self.basis))
        self.design = np.concatenate(blocks, axis=0)
        normal = self.design.T @ self.design
        ridge = max(float(np.abs(np.diag(normal)).max()), 1.0) * 1.0e-12
        normal = normal + ridge * np.eye(self.nb)
        top = np.zeros(nz)
        top[-1] = 3.0 / (2.0 * dz)
        top[-2] = -4.0 / (2.0 * dz)
        top[-3] = 1.0 / (2.0 * dz)
        self.constraints = np.stack([self.basis[0], top @ self.basis])
        self.kkt = np.block([[normal, self.constraints.T], [self.constraints, np.zeros((2, 2))]])

    def solve(self, q: np.ndarray, h0: float) -> np.ndarray:
        q = np.asarray(q, dtype=np.float64)
        qf = 0.5 * (q[:-1] + q[1:])
        rhs = [qf]
        if self.smoothness > 0.0 and self.C.shape[0] > 0:
            rhs.append(np.zeros(self.C.shape[0]))
        nrhs = self.design.T @ np.concatenate(rhs)
        sol = np.linalg.solve(self.kkt, np.concatenate([nrhs, [h0, 0.0]]))
        return self.basis @ sol[: self.nb]

    def centre_derivative(self, prof: np.ndarray) -> np.ndarray:
        return centre_derivative_fd2(prof, self.dz)


def fit_diagnostics(closure, prof: np.ndarray, desired: np.ndarray, history: list) -> dict:
    """The per-update closure diagnostics (nfgs_solver.py:5965-6009,
    6024-6065).  ``desired`` = (mean Jx, mean Jy) target by height; the fit
    is H_x' = desired_y, H_y' = -desired_x."""
    dz = closure.dz
    der = closure.centre_derivative(prof)
    actual = np.stack([-der[1], der[0]])
    res = actual - desired
    res_rms = float(np.sqrt(np.mean(res ** 2)))
    des_rms = float(np.sqrt(np.mean(desired ** 2)))
    rel = res_rms / max(des_rms, 1e-30)
    history.append(rel)
    face = (prof[:, 1:] - prof[:, :-1]) / dz
    dface = np.stack([0.5 * (desired[1, :-1] + desired[1, 1:]), -0.5 * (desired[0, :-1] + desired[0, 1:])])
    fres = face - dface
    fres_rms = float(np.sqrt(np.mean(fres ** 2)))
    ftgt_rms = float(np.sqrt(np.mean(dface ** 2)))
    if prof.shape[1] >= 3:
        grid = prof[:, 1:-1] - 0.25 * (prof[:, :-2] + 2.0 * prof[:, 1:-1] + prof[:, 2:])
        grid_rms = float(np.sqrt(np.mean(grid ** 2)))
    else:
        grid_rms = 0.0
    prof_rms = float(np.sqrt(np.mean(prof ** 2)))
    return {
        "ode_residual_rms": res_rms,
        "ode_residual_relative": rel,
        "ode_residual_relative_max": max(history),
        "face_ode_residual_rms": fres_rms,
        "face_ode_residual_relative": fres_rms / max(ftgt_rms, 1e-30),
        "gridscale_profile_rms": grid_rms,
        "gridscale_profile_relative": grid_rms / max(prof_rms, 1e-30),
        "top_derivative": [float(v) for v in closure.centre_derivative(prof)[:, -1]],
        "profile_max_abs": float(np.abs(prof).max()),
        "profile_top": [float(v) for v in prof[:, -1]],
        "desired_mean_current_rms": des_rms,
    }

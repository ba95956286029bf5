"""CPU oracle for the NFGS reconstruction path (TEST INFRASTRUCTURE ONLY).

This module is the checker, never the product.  It is a plain NumPy/SciPy
FP64 restatement of the reference NFGS solver's production path
(``nfgs_solver.py`` in spaceprod/NFGS, class ``NFGSSolverGPU``), written so
that every step can be compared element-wise with the CUDA path.  Only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
may import it.  The product package (``nfgs_b200``) never imports it and has
no CPU fallback.

Citations are ``nfgs_solver.py:<line>`` in the reference repository.

Parity pinning: the restatement is pinned against golden tensors produced by
running the reference solver itself (``tests/golden/make_golden.py``), at
several grids, for the boundary set-up products, the ``gs_cfcf`` initial
state, individual NFPT iterations and complete ``iterate`` histories.

Transforms: the reference builds DCT-I / DST-I by mirroring and
``torch.fft.rfft`` (``nfgs_solver.py:1019-1081``).  SciPy's unnormalised
``dct(type=1)`` / ``dst(type=1)`` are the same linear maps and are used here.
"""

from __future__ import annotations

import math
import warnings
from typing import Callable, Optional

import numpy as np
from scipy import fft as _sfft

from .k0_oracle import CoupledK0, SplineK0, centre_derivative_fd2, fit_diagnostics

# SciPy FFT worker threads (batch-parallel transforms give identical results)
_WORKERS = -1

__all__ = [
    "mudpack_axis_size",
    "fortran_grid",
    "OracleNFGS",
    "dct1",
    "idct1",
    "dst1",
    "idst1",
]


# ---------------------------------------------------------------------------
# Grid sizing (nfgs_solver.py:73-177)
# ---------------------------------------------------------------------------
def mudpack_axis_size(n_obs: int) -> int:
    """MUDPACK-friendly padded axis size (nfgs_solver.py:73-84)."""
    n_obs = int(n_obs)
    if n_obs < 2:
        return max(1, n_obs)
    n_real = float(n_obs)
    exp2 = math.ceil(math.log((n_real - 1.0) / 2.0) / math.log(2.0)) + 1
    exp3 = math.ceil(math.log((n_real - 1.0) / 3.0) / math.log(2.0)) + 1
    n2 = int(2 * (2 ** (exp2 - 1)) + 1)
    n3 = int(3 * (2 ** (exp3 - 1)) + 1)
    return min(n2, n3)


def _even_xy_pad_size(n_calc: int, n_obs: int) -> int:
    """nfgs_solver.py:87-103."""
    if n_calc < n_obs:
        raise ValueError(f"calculation size {n_calc} is smaller than observed size {n_obs}")
    return n_calc + 1 if (n_calc - n_obs) % 2 == 1 else n_calc


def fortran_grid(nxo: int, nyo: int, nzo: int, symmetric_xy: bool = False):
    """(nx, ny, nz, bfx, bfy, bfz) of nfpt_fortran_grid (nfgs_solver.py:105-177)."""
    nx, ny, nz = mudpack_axis_size(nxo), mudpack_axis_size(nyo), mudpack_axis_size(nzo)
    if symmetric_xy:
        nx = _even_xy_pad_size(nx, nxo)
        ny = _even_xy_pad_size(ny, nyo)
    return nx, ny, nz, (nx - nxo) // 2, (ny - nyo) // 2, nz - nzo


# ---------------------------------------------------------------------------
# Transforms (nfgs_solver.py:1019-1081) and 2-D helpers
# ---------------------------------------------------------------------------
def dct1(x: np.ndarray, axis: int) -> np.ndarray:
    """Unnormalised DCT-I along ``axis`` (nfgs_solver.py:1052-1074)."""
    if x.shape[axis] == 1:
        return x.copy()
    return _sfft.dct(x, type=1, axis=axis, workers=_WORKERS)


def idct1(x: np.ndarray, axis: int) -> np.ndarray:
    """Inverse DCT-I (nfgs_solver.py:1076-1081)."""
    n = x.shape[axis]
    if n == 1:
        return x.copy()
    return dct1(x, axis) / (2.0 * (n - 1))


def dst1(x: np.ndarray, axis: int) -> np.ndarray:
    """Unnormalised DST-I along ``axis`` (nfgs_solver.py:1019-1045)."""
    return _sfft.dst(x, type=1, axis=axis, workers=_WORKERS)


def idst1(x: np.ndarray, axis: int) -> np.ndarray:
    """Inverse DST-I (nfgs_solver.py:1047-1050)."""
    return dst1(x, axis) / (2.0 * (x.shape[axis] + 1))


def dct2(v):
    """x then y DCT-I (nfgs_solver.py:4354-4355)."""
    return dct1(dct1(v, -1), -2)


def idct2(v):
    """nfgs_solver.py:4445-4446."""
    return idct1(idct1(v, -1), -2)


def dst2(v):
    return dst1(dst1(v, -1), -2)


def idst2(v):
    return idst1(idst1(v, -1), -2)


# ---------------------------------------------------------------------------
# Second-order finite differences (nfgs_solver.py:1361-1469, 1711-1749)
# ---------------------------------------------------------------------------
def _d_axis(f: np.ndarray, h: float, axis: int) -> np.ndarray:
    """Central interior, one-sided 3-point ends (nfgs_solver.py:1361-1419)."""
    out = np.zeros_like(f)
    n = f.shape[axis]
    if n < 2:
        return out
    f = np.moveaxis(f, axis, 0)
    o = np.moveaxis(out, axis, 0)
    if n >= 3:
        o[1:-1] = (f[2:] - f[:-2]) / (2.0 * h)
        o[0] = (-3.0 * f[0] + 4.0 * f[1] - f[2]) / (2.0 * h)
        o[-1] = (3.0 * f[-1] - 4.0 * f[-2] + f[-3]) / (2.0 * h)
    else:
        o[0] = (f[1] - f[0]) / h
        o[-1] = (f[-1] - f[-2]) / h
    return out


def d_dx(f, dx):
    return _d_axis(f, dx, -1)


def d_dy(f, dy):
    return _d_axis(f, dy, -2)


def d_dz(f, dz):
    return _d_axis(f, dz, 0)


def lap_xy(f, dx, dy):
    """Mirrored-Neumann horizontal Laplacian (nfgs_solver.py:1741-1749)."""
    lap = np.zeros_like(f)
    lap[..., 1:-1] += (f[..., 2:] - 2 * f[..., 1:-1] + f[..., :-2]) / dx**2
    lap[..., 1:-1, :] += (f[..., 2:, :] - 2 * f[..., 1:-1, :] + f[..., :-2, :]) / dy**2
    lap[..., 0, :] += (2 * f[..., 1, :] - 2 * f[..., 0, :]) / dy**2
    lap[..., -1, :] += (2 * f[..., -2, :] - 2 * f[..., -1, :]) / dy**2
    lap[..., 0] += (2 * f[..., 1] - 2 * f[..., 0]) / dx**2
    lap[..., -1] += (2 * f[..., -2] - 2 * f[..., -1]) / dx**2
    return lap


def d2_dxdz(f, dx, dz):
    """Interior-only mixed derivative (nfgs_solver.py:1729-1733)."""
    d2 = np.zeros_like(f)
    if f.shape[0] < 3 or f.shape[2] < 3:
        return d2
    d2[1:-1, :, 1:-1] = (f[2:, :, 2:] - f[:-2, :, 2:] - f[2:, :, :-2] + f[:-2, :, :-2]) / (4.0 * dx * dz)
    return d2


def d2_dydz(f, dy, dz):
    """nfgs_solver.py:1735-1739."""
    d2 = np.zeros_like(f)
    if f.shape[0] < 3 or f.shape[1] < 3:
        return d2
    d2[1:-1, 1:-1, :] = (f[2:, 2:, :] - f[:-2, 2:, :] - f[2:, :-2, :] + f[:-2, :-2, :]) / (4.0 * dy * dz)
    return d2


def _rms(v) -> float:
    return float(np.sqrt(np.mean(np.asarray(v, dtype=np.float64) ** 2)))


def _pad_or_crop_center_2d(a2: np.ndarray, ty: int, tx: int):
    """nfgs_solver.py:1593-1609."""
    ny, nx = a2.shape
    out = np.zeros((ty, tx), dtype=np.float64)
    sy0, sx0 = max(0, (ny - ty) // 2), max(0, (nx - tx) // 2)
    sy1, sx1 = sy0 + min(ny, ty), sx0 + min(nx, tx)
    dy0, dx0 = max(0, (ty - ny) // 2), max(0, (tx - nx) // 2)
    dy1, dx1 = dy0 + (sy1 - sy0), dx0 + (sx1 - sx0)
    out[dy0:dy1, dx0:dx1] = a2[sy0:sy1, sx0:sx1]
    return out, (slice(dy0, dy1), slice(dx0, dx1))


def _smooth_bottom_2d(a2: np.ndarray, n: int) -> np.ndarray:
    """3x3 binomial smoothing with reflect padding (nfgs_solver.py:1471-1483)."""
    if n <= 0 or a2.shape[0] < 3 or a2.shape[1] < 3:
        return a2
    k = np.array([[1.0, 2.0, 1.0], [2.0, 4.0, 2.0], [1.0, 2.0, 1.0]]) / 16.0
    x = a2
    for _ in range(n):
        p = np.pad(x, 1, mode="reflect")
        y = np.zeros_like(x)
        for a in range(3):
            for b in range(3):
                y += k[a, b] * p[a:a + x.shape[0], b:b + x.shape[1]]
        x = y
    return x


def _balance_jz(jzb: np.ndarray, mode: int) -> np.ndarray:
    """botbal sign-separated balancing (nfgs_solver.py:1527-1558)."""
    if mode < 2 or jzb.shape[0] < 3 or jzb.shape[1] < 3:
        return jzb
    jzp = np.where(jzb >= 0.0, jzb, 0.0)
    jzn = np.where(jzb < 0.0, jzb, 0.0)

    def cell_sum(a):
        return 0.25 * (a[1:-1, 2:].sum() + a[2:, 1:-1].sum() + a[1:-1, 1:-1].sum() + a[2:, 2:].sum())

    jzsum, jzpsum, jznsum = cell_sum(jzb), cell_sum(jzp), cell_sum(jzn)
    if mode == 2:
        cor = jzpsum - 0.5 * jzsum
    elif mode == 3:
        cor = max(jzpsum, abs(jznsum))
    elif mode == 4:
        cor = min(jzpsum, abs(jznsum))
    else:
        return jzb
    pos = jzb >= 0.0
    if abs(jzpsum) > 0.0:
        jzb = np.where(pos, (cor / jzpsum) * jzb, jzb)
    if abs(jznsum) > 0.0:
        jzb = np.where(~pos, (cor / abs(jznsum)) * jzb, jzb)
    return jzb


def derive_bottom_jz_legacy(bx, by, nz, dx, dy, ijzbcor):
    """Helper-grid bottom Jz (nfgs_solver.py:1498-1567).

    The calculation-grid maps are embedded once more in the MUDPACK grid of
    their own size, the centred curl is taken there, balanced, the helper
    grid's outer nodes zeroed and the calculation window cropped back out.
    """
    nyo, nxo = bx.shape
    nx, ny, _nz, bfx, bfy, _ = fortran_grid(nxo, nyo, max(2, int(nz)))
    bxb = np.zeros((ny, nx))
    byb = np.zeros((ny, nx))
    y1, x1 = bfy + nyo, bfx + nxo
    bxb[bfy:y1, bfx:x1] = bx
    byb[bfy:y1, bfx:x1] = by
    jzb = np.zeros((ny, nx))
    if nx >= 3 and ny >= 3:
        jzb[1:-1, 1:-1] = (byb[1:-1, 2:] - byb[1:-1, :-2]) / (2.0 * dx) - (bxb[2:, 1:-1] - bxb[:-2, 1:-1]) / (2.0 * dy)
        jzb = _balance_jz(jzb, int(ijzbcor))
    jzb[0, :] = 0.0
    jzb[-1, :] = 0.0
    jzb[:, 0] = 0.0
    jzb[:, -1] = 0.0
    return jzb[bfy:y1, bfx:x1].copy()


def derive_bottom_jz_calc(bx, by, dx, dy, ijzbcor):
    """Unpadded-domain bottom Jz on the calculation grid (nfgs_solver.py:4515-4546)."""
    ny, nx = bx.shape
    jz = np.zeros_like(bx)
    if nx >= 3 and ny >= 3:
        jz[1:-1, 1:-1] = (by[1:-1, 2:] - by[1:-1, :-2]) / (2 * dx) - (bx[2:, 1:-1] - bx[:-2, 1:-1]) / (2 * dy)
    mode = int(ijzbcor)
    if mode >= 2 and nx >= 3 and ny >= 3:
        pos_a = np.maximum(jz, 0.0)
        neg_a = np.minimum(jz, 0.0)

        def cell_sum(a):
            return 0.25 * (a[1:-1, 2:].sum() + a[2:, 1:-1].sum() + a[1:-1, 1:-1].sum() + a[2:, 2:].sum())

        total, pos, neg = cell_sum(jz), cell_sum(pos_a), cell_sum(neg_a)
        if mode == 2:
            target = pos - 0.5 * total
        elif mode == 3:
            target = max(pos, abs(neg))
        elif mode == 4:
            target = min(pos, abs(neg))
        else:
            target = None
        if target is not None:
            fp = target / pos if abs(pos) > 0 else 1.0
            fn = target / abs(neg) if abs(neg) > 0 else 1.0
            jz = np.where(jz >= 0, fp * jz, fn * jz)
    return jz


# ---------------------------------------------------------------------------
# The solver restatement
# ---------------------------------------------------------------------------
_PROD_POLICIES = dict(
    horizontal_zero_mode_policy={"omit", "frozen_linear_harmonic", "external_potential", "user_supplied",
                                 "coupled_k0", "constrained_spline_harmonic"},
    mean_bz_policy={"uniform_open", "require_balanced", "external_potential", "user_supplied"},
)


class OracleNFGS:
    """FP64 restatement of ``NFGSSolverGPU`` (nfgs_solver.py:3905-7196).

    Supported: gaussian_separated partition, staggered_face current,
    direct poloidal update, gs_cfcf and soft_cfcf starts, sigma_best stop (with optional
    adaptive_mu rollback), mixed bottom Robin weight rho in [0, 1] or the
    bottom-divergence projection, frozen/omitted/external/user horizontal
    zero modes.
    """

    def __init__(self, Nx, Ny, Nz, dx, dy, dz, *, pad_calculation_domain=True,
                 calculation_domain_mode="mudpack", buffer_thickness=None,
                 buffer_xy_only=False, padded_buffer_zone=True,
                 bottom_divergence_robin_weight=0.0,
                 bottom_divergence_projection_weight=0.0,
                 horizontal_zero_mode_policy="frozen_linear_harmonic",
                 mean_bz_policy="uniform_open", d0_zero_mode_policy="error",
                 source_zero_mode_policy="error", harmonic_residual_policy="diagnose",
                 mean_mode_tolerance=1e-6, source_zero_mode_tolerance=1e-2,
                 alpha_clip_scale=None, alpha_limit_factor=1.0,
                 weak_field_floor_b2=1e-20, gaussian_horizontal_operator="spectral",
                 bottom_parallel_current_mode="observed_full",
                 user_supplied_open_bz=None, user_supplied_horizontal_field=None,
                 external_potential_field=None, soft_cfcf_epsilon=None, soft_cfcf_normal_ridge=0.0,
                 lateral_wall="paper_bc1", record_iteration_diagnostics=False,
                 k0_ode_smoothness=1.0e-3,
                 coupled_k0_discretization="staggered_face_D1_true_three_point_curvature",
                 k0_update_mu=None, k0_spline_basis_size=8, k0_current_target_placement=None):
        ix, iy, iz = int(Nx), int(Ny), int(Nz)
        # the wall condition of the Stable-NFPT field behind the cfcf start
        # (nfgs_solver.py:845-853, 2161-2170)
        self.lateral_bc1 = str(lateral_wall).lower().replace("-", "_") in ("bc1", "paper_bc1", "paper")
        self.record_iteration_diagnostics = bool(record_iteration_diagnostics)
        self.last_iteration_diagnostics = {}
        mode = str(calculation_domain_mode).lower().replace("-", "_")
        # nfgs_solver.py:771-819
        if pad_calculation_domain:
            if mode in ("mudpack", "mudpack_legacy"):
                nx, ny, nz, bfx, bfy, _ = fortran_grid(ix, iy, iz, symmetric_xy=(mode == "mudpack"))
                pad_xy = (bfx, bfy)
            elif mode == "bottom_padding":
                bp = (ix + iy) // 6
                nx, ny = ix + 2 * bp, iy + 2 * bp
                nz = min(nx, ny)
                if nz < iz:
                    raise ValueError("bottom_padding calculation height cannot contain the input z domain")
                pad_xy = (bp, bp)
            else:
                raise ValueError(f"bad calculation_domain_mode {calculation_domain_mode!r}")
        else:
            nx, ny, nz = ix, iy, iz
            pad_xy = (0, 0)
        self.input_shape_zyx = (iz, iy, ix)
        self.calculation_pad_xy = pad_xy
        self.Nx, self.Ny, self.Nz = nx, ny, nz
        self.dx, self.dy, self.dz = float(dx), float(dy), float(dz)
        if self.Nz < 3:
            raise ValueError("NFGS requires Nz >= 3")
        self.buffer_thickness = 0 if buffer_thickness is None else int(buffer_thickness)
        self.buffer_xy_only = bool(buffer_xy_only)
        self.padded_buffer_zone = bool(padded_buffer_zone)
        self.rho = float(bottom_divergence_robin_weight)
        self.proj_w = float(bottom_divergence_projection_weight)
        if not 0.0 <= self.rho <= 1.0 or not 0.0 <= self.proj_w <= 1.0:
            raise ValueError("bottom-divergence weights must be between 0 and 1")
        if self.rho > 0 and self.proj_w > 0:
            raise ValueError("Bottom-divergence projection and mixed Robin controls are mutually exclusive")
        self.hzm = str(horizontal_zero_mode_policy).lower()
        self.mean_bz_policy = str(mean_bz_policy).lower()
        if self.hzm not in _PROD_POLICIES["horizontal_zero_mode_policy"]:
            raise NotImplementedError(self.hzm)
        # k_h=0 closure settings (nfgs_solver.py:3966-3976, 4120-4170, 4252-4270)
        self.k0_smoothness = float(k0_ode_smoothness)
        self.k0_legacy = str(coupled_k0_discretization).lower().replace("-", "_") == "legacy_plane_centred"
        if k0_update_mu is None and self.hzm == "constrained_spline_harmonic":
            k0_update_mu = 0.2
        self.k0_update_mu = None if k0_update_mu is None else float(k0_update_mu)
        self.k0_basis = int(k0_spline_basis_size)
        place = "cell" if k0_current_target_placement is None else str(k0_current_target_placement).lower()
        self.k0_face_target = place.replace("-", "_") == "face"
        self.k0 = None
        self.k0_diagnostics = {}
        self.k0_history: list[float] = []
        if self.mean_bz_policy not in _PROD_POLICIES["mean_bz_policy"]:
            raise ValueError(self.mean_bz_policy)
        self.d0_policy = str(d0_zero_mode_policy).lower()
        self.src_policy = str(source_zero_mode_policy).lower()
        self.harm_policy = str(harmonic_residual_policy).lower()
        self.mean_mode_tolerance = float(mean_mode_tolerance)
        self.source_zero_mode_tolerance = float(source_zero_mode_tolerance)
        factor = float(alpha_clip_scale) if alpha_clip_scale is not None else alpha_limit_factor
        self.alpha_limit_factor = None if factor is None else float(factor)
        self.weak_floor = float(weak_field_floor_b2)
        self.ghop = str(gaussian_horizontal_operator).lower()
        self.bpcm = str(bottom_parallel_current_mode).lower().replace("-", "_")
        self.user_open_bz = user_supplied_open_bz
        self.user_h = user_supplied_horizontal_field
        self.external = external_potential_field
        # nfgs_solver.py:4299-4305
        gs = min(self.dx, self.dy, self.dz)
        self.soft_cfcf_epsilon = 1.0e-4 / (gs * gs) if soft_cfcf_epsilon is None else float(soft_cfcf_epsilon)
        self.soft_cfcf_normal_ridge = float(soft_cfcf_normal_ridge)
        self.soft_cfcf_diagnostics = None
        self.source_zero_mode_history: list[float] = []
        self.last_source_zero_mode_by_height: list[float] = []
        self.projection_history: list[dict] = []
        self._B = self._J = self._Phi_c = self._Az = None

    # ------------------------------------------------------------- tables
    def alpha_max(self):
        """nfgs_solver.py:2970-2975."""
        if self.alpha_limit_factor is None:
            return None
        return self.alpha_limit_factor / min(self.dx, self.dy, self.dz)

    def lam_neumann(self):
        """nfgs_solver.py:1098-1109."""
        kx = np.arange(self.Nx, dtype=np.float64)
        ky = np.arange(self.Ny, dtype=np.float64)
        lx = -4.0 * np.sin(np.pi * kx / (2.0 * max(self.Nx - 1, 1))) ** 2 / self.dx**2
        ly = -4.0 * np.sin(np.pi * ky / (2.0 * max(self.Ny - 1, 1))) ** 2 / self.dy**2
        return ly[:, None] + lx[None, :]

    def lam_dirichlet(self):
        """nfgs_solver.py:1083-1096."""
        nxi, nyi = self.Nx - 2, self.Ny - 2
        kx = np.arange(1, nxi + 1, dtype=np.float64)
        ky = np.arange(1, nyi + 1, dtype=np.float64)
        lx = -4.0 * np.sin(np.pi * kx / (2.0 * (nxi + 1))) ** 2 / self.dx**2
        ly = -4.0 * np.sin(np.pi * ky / (2.0 * (nyi + 1))) ** 2 / self.dy**2
        return ly[:, None] + lx[None, :]

    def alpha_x(self):
        """nfgs_solver.py:4357-4369."""
        kx = np.arange(self.Nx, dtype=np.float64)
        return 2.0 * np.sin(np.pi * kx / (2.0 * max(self.Nx - 1, 1))) / self.dx

    def alpha_y(self):
        ky = np.arange(self.Ny, dtype=np.float64)
        return 2.0 * np.sin(np.pi * ky / (2.0 * max(self.Ny - 1, 1))) / self.dy

    def buffer_window(self):
        """nfgs_solver.py:1569-1591 (None when the window is identically one)."""
        t = self.buffer_thickness
        if t <= 0:
            return None

        def bell(n):
            tt = min(t, max(1, (n - 1) // 2))
            idx = np.arange(n, dtype=np.float64)
            dist = np.minimum(idx, (n - 1) - idx)
            return np.where(dist >= tt, 1.0, 0.5 * (1.0 - np.cos(np.pi * dist / tt)))

        wx, wy = bell(self.Nx), bell(self.Ny)
        if self.buffer_xy_only:
            wz = np.ones(self.Nz)
        else:
            tz = min(t, max(1, self.Nz - 1))
            k = np.arange(self.Nz, dtype=np.float64)
            dist_top = (self.Nz - 1) - k
            wz = np.where(dist_top >= tz, 1.0, 0.5 * (1.0 - np.cos(np.pi * dist_top / tz)))
            wz[0] = 1.0
        return wz[:, None, None] * wy[None, :, None] * wx[None, None, :]

    # --------------------------------------------------------- 2-D Poisson
    def poisson2d_dirichlet(self, source):
        """Endpoint-Dirichlet 2-D Poisson (nfgs_solver.py:1132-1144)."""
        out = np.zeros_like(source)
        if self.Nx < 3 or self.Ny < 3:
            return out
        hat = dst2(source[..., 1:-1, 1:-1]) / self.lam_dirichlet()
        out[..., 1:-1, 1:-1] = idst2(hat)
        return out

    def poisson2d_neumann(self, source):
        """Endpoint-Neumann 2-D Poisson, no flux maps (nfgs_solver.py:1146-1179)."""
        lam = self.lam_neumann().copy()
        lam[0, 0] = 1.0
        hat = dct2(source) / lam
        hat[..., 0, 0] = 0.0
        return idct2(hat)

    def spectral_dx_2d(self, v):
        """nfgs_solver.py:4385-4393."""
        sine_hat = -self.alpha_x() * dct2(v)
        tmp = idct1(sine_hat, -2)
        out = np.zeros_like(v)
        if v.shape[-1] >= 3:
            out[..., 1:-1] = idst1(tmp[..., 1:-1], -1)
        return out

    def spectral_dy_2d(self, v):
        """nfgs_solver.py:4395-4403."""
        sine_hat = -self.alpha_y()[:, None] * dct2(v)
        tmp = idct1(sine_hat, -1)
        out = np.zeros_like(v)
        if v.shape[-2] >= 3:
            out[..., 1:-1, :] = idst1(tmp[..., 1:-1, :], -2)
        return out

    def dstx_dcty_hat(self, bx):
        """nfgs_solver.py:4408-4415."""
        out = np.zeros_like(bx)
        if bx.shape[-1] < 3:
            return out
        tmp = dct1(bx, -2)
        out[..., 1:-1] = dst1(tmp[..., 1:-1], -1)
        return out

    def dctx_dsty_hat(self, by):
        """nfgs_solver.py:4417-4424."""
        out = np.zeros_like(by)
        if by.shape[-2] < 3:
            return out
        tmp = dct1(by, -1)
        out[..., 1:-1, :] = dst1(tmp[..., 1:-1, :], -2)
        return out

    def spectral_div_xy_hat(self, bx, by):
        """nfgs_solver.py:4436-4443."""
        return self.alpha_x() * self.dstx_dcty_hat(bx) + self.alpha_y()[:, None] * self.dctx_dsty_hat(by)

    def horizontal_grad(self, v):
        """nfgs_solver.py:4445-4452."""
        if self.ghop == "spectral":
            return self.spectral_dx_2d(v), self.spectral_dy_2d(v)
        return d_dx(v, self.dx), d_dy(v, self.dy)

    def horizontal_div(self, bx, by):
        if self.ghop == "spectral":
            return idct2(self.spectral_div_xy_hat(bx, by))
        return d_dx(bx, self.dx) + d_dy(by, self.dy)

    def const_mode(self, hat):
        """nfgs_solver.py:4462-4468."""
        return hat[..., 0, 0] / (4.0 * max(self.Nx - 1, 1) * max(self.Ny - 1, 1))

    @staticmethod
    def _policy(ratio, tol, policy, message):
        """nfgs_solver.py:4477-4487."""
        if ratio <= tol:
            return
        detail = f"{message} ratio={ratio:.6e} exceeds tolerance={tol:.6e}."
        if policy == "error":
            raise ValueError(detail)
        if policy == "warn_project":
            warnings.warn(detail + " The incompatible zero mode will be projected out.", RuntimeWarning, stacklevel=3)

    # ------------------------------------------------------ boundary set-up
    def _bottom_plane(self, a):
        a = np.asarray(a, dtype=np.float64)
        if a.ndim == 3:
            if a.shape[0] != self.Nz:
                raise ValueError(f"3D input must be in (Nz, Ny, Nx) order with Nz={self.Nz}")
            return a[0]
        if a.ndim != 2:
            raise ValueError("bottom maps must be 2D (Ny, Nx) or 3D (Nz, Ny, Nx)")
        return a

    def set_bottom_vector_boundary(self, Bx_obs, By_obs, Bz_obs, zero_net_current=None,
                                   smooth_passes=None, padded_buffer_zone=None, ijzbcor=3, Jz_obs=None):
        """nfgs_solver.py:4548-4596 -> 3024-3057 -> 2000-2113, then 4671-4919."""
        bz = self._bottom_plane(Bz_obs)
        bx = self._bottom_plane(Bx_obs)
        by = self._bottom_plane(By_obs)
        derived = Jz_obs is None
        jz = None if derived else self._bottom_plane(Jz_obs)
        if zero_net_current is None:
            zero_net_current = not derived
        if smooth_passes is None:
            smooth_passes = 0 if derived else 3
        if bx.shape != bz.shape or by.shape != bz.shape:
            raise ValueError("Bx_obs/By_obs must have the same observed-FOV shape as Bz_obs.")
        use_pad = self.padded_buffer_zone if padded_buffer_zone is None else bool(padded_buffer_zone)
        if bz.shape != (self.Ny, self.Nx):
            if not use_pad:
                raise ValueError(f"Bz_obs/Jz_obs must have shape ({self.Ny}, {self.Nx}); got {bz.shape}.")
            oy, ox = bz.shape
            bz, fov = _pad_or_crop_center_2d(bz, self.Ny, self.Nx)
            bx, _ = _pad_or_crop_center_2d(bx, self.Ny, self.Nx)
            by, _ = _pad_or_crop_center_2d(by, self.Ny, self.Nx)
            if jz is not None:
                jz, _ = _pad_or_crop_center_2d(jz, self.Ny, self.Nx)
            self.fov = fov
            self.observed_shape = (min(self.Nz, self.input_shape_zyx[0]), oy, ox)
        else:
            self.fov = (slice(0, self.Ny), slice(0, self.Nx))
            self.observed_shape = (self.Nz, self.Ny, self.Nx)
        if derived:
            calc = (self.Nz, self.Ny, self.Nx)
            padded = any(c > o for c, o in zip(calc, self.input_shape_zyx)) or \
                any(c > o for c, o in zip(calc, self.observed_shape)) or any(p > 0 for p in self.calculation_pad_xy)
            if padded:
                self.bottom_current_grid_mode = "legacy_helper"
                jz = derive_bottom_jz_legacy(bx, by, self.Nz, self.dx, self.dy, ijzbcor)
            else:
                self.bottom_current_grid_mode = "calculation_grid"
                jz = derive_bottom_jz_calc(bx, by, self.dx, self.dy, ijzbcor)
        else:
            self.bottom_current_grid_mode = "provided"
        # the Stable-NFPT solver behind the cfcf start derives its own bottom
        # current, always on the legacy helper grid (nfgs_solver.py:2071-2072,
        # 1498-1567), from the same maps
        jz_st = jz if self.bottom_current_grid_mode == "legacy_helper" else \
            derive_bottom_jz_legacy(bx, by, self.Nz, self.dx, self.dy, ijzbcor)
        if int(smooth_passes) > 0:
            bz = _smooth_bottom_2d(bz, smooth_passes)
            jz = _smooth_bottom_2d(jz, smooth_passes)
            jz_st = _smooth_bottom_2d(jz_st, smooth_passes)
            bx = _smooth_bottom_2d(bx, smooth_passes)
            by = _smooth_bottom_2d(by, smooth_passes)
        if zero_net_current:
            jz = jz - jz.mean()
            jz_st = jz_st - jz_st.mean()
        self.Jz_stable = jz_st.copy()
        self.Bz_obs, self.Jz_obs, self.Bx_obs, self.By_obs = bz.copy(), jz.copy(), bx.copy(), by.copy()
        # nfgs_solver.py:2105 and 3039-3057
        self.Az_bottom = self.poisson2d_dirichlet(-self.Jz_obs)
        jzt = -lap_xy(self.Az_bottom[None], self.dx, self.dy)[0]
        jzt[:, 0] = 0.0
        jzt[:, -1] = 0.0
        jzt[0, :] = 0.0
        jzt[-1, :] = 0.0
        self.Jz_T = jzt
        self.toroidal_boundary_diagnostics = {
            "t_source": "jz",
            "t_filter_scale": 0.0,
            "raw_jz_rms": _rms(self.Jz_obs),
            "t_implied_jz_rms": _rms(jzt),
            "raw_vs_t_implied_jz_rms": _rms(self.Jz_obs - jzt),
        }
        self._configure_gaussian_background()
        self._B = self._J = self._Phi_c = self._Az = None
        self.source_zero_mode_history = []
        self.last_source_zero_mode_by_height = []
        self.projection_history = []

    def _configure_gaussian_background(self):
        """Gaussian separation (nfgs_solver.py:4671-4919)."""
        nz, ny, nx = self.Nz, self.Ny, self.Nx
        bx_hat, by_hat, bz_hat = dct2(self.Bx_obs), dct2(self.By_obs), dct2(self.Bz_obs)
        self.B_mean = np.array([self.const_mode(bx_hat), self.const_mode(by_hat), self.const_mode(bz_hat)])
        use_external = self.mean_bz_policy == "external_potential" or self.hzm == "external_potential"
        external = np.zeros((3, nz, ny, nx))
        if use_external:
            if self.external is None:
                raise ValueError("external_potential_field is required when an external_potential mean-mode policy is selected")
            external = np.array(self.external, dtype=np.float64)
            if external.shape != (3, nz, ny, nx):
                raise ValueError("external_potential_field has the wrong shape")
        elif self.external is not None:
            raise ValueError("external_potential_field was supplied but neither mean-mode policy selects 'external_potential'")
        user_h = np.zeros_like(external)
        if self.hzm == "user_supplied":
            if self.user_h is None:
                raise ValueError("user_supplied_horizontal_field is required")
            s = np.asarray(self.user_h, dtype=np.float64)
            if s.shape == (2,):
                user_h[:2] = s[:, None, None, None]
            elif s.shape == (2, nz, ny, nx):
                user_h[:2] = s
            else:
                raise ValueError("user_supplied_horizontal_field has the wrong shape")
        supplemental = external + user_h
        bx_res = self.Bx_obs - supplemental[0, 0]
        by_res = self.By_obs - supplemental[1, 0]
        bz_res = self.Bz_obs - supplemental[2, 0]
        res_bz_hat = dct2(bz_res)
        res_mean = self.const_mode(res_bz_hat)
        res_scale = max(_rms(bz_res), 1e-30)
        flux_imb = float(abs(bz_res.sum()) / max(np.abs(bz_res).sum(), 1e-30))
        if self.mean_bz_policy in ("uniform_open", "require_balanced"):
            if self.mean_bz_policy == "require_balanced" and flux_imb > self.mean_mode_tolerance:
                raise ValueError(f"The residual bottom Bz is not flux balanced: fraction={flux_imb:.6e}, "
                                 f"tolerance={self.mean_mode_tolerance:.6e}.")
            self.Bz_open_mean = float(res_mean)
        elif self.mean_bz_policy == "external_potential":
            if abs(res_mean) / res_scale > self.mean_mode_tolerance:
                raise ValueError("external_potential_field does not carry the observed Bz zero mode")
            self.Bz_open_mean = 0.0
        else:
            if self.user_open_bz is None:
                raise ValueError("user_supplied_open_bz is required for mean_bz_policy='user_supplied'")
            self.Bz_open_mean = float(np.asarray(self.user_open_bz).reshape(()))
            if abs(res_mean - self.Bz_open_mean) / res_scale > self.mean_mode_tolerance:
                raise ValueError("user_supplied_open_bz does not match the residual Bz zero mode")
        bz_nonmean_hat = res_bz_hat.copy()
        bz_nonmean_hat[0, 0] = 0.0
        if self.ghop == "spectral":
            d_hat = self.spectral_div_xy_hat(bx_res, by_res)
            self.D0 = idct2(d_hat)
        else:
            self.D0 = d_dx(bx_res, self.dx) + d_dy(by_res, self.dy)
            d_hat = dct2(self.D0)
        d0_mean = float(self.const_mode(d_hat))
        d0_ratio = float(abs(d0_mean) / max(_rms(self.D0), 1e-30))
        self._policy(d0_ratio, self.mean_mode_tolerance, self.d0_policy,
                     "The bottom vector field is incompatible with the zero-mean endpoint-Neumann GS model")
        d_hat[0, 0] = 0.0
        lam = self.lam_neumann()
        k = np.sqrt(np.maximum(-lam, 0.0))
        k_safe = k.copy()
        k_safe[0, 0] = 1.0
        lam_safe = lam.copy()
        lam_safe[0, 0] = 1.0
        self.k = k
        dphi_total_hat = -d_hat / lam_safe
        dphi_total_hat[0, 0] = 0.0
        bz_below_hat = 0.5 * (bz_nonmean_hat + d_hat / k_safe)
        bz_above_hat = 0.5 * (bz_nonmean_hat - d_hat / k_safe)
        bz_below_hat[0, 0] = 0.0
        bz_above_hat[0, 0] = 0.0
        phi_below_hat = bz_below_hat / lam_safe
        phi_above_hat = bz_above_hat / lam_safe
        phi_below_hat[0, 0] = 0.0
        phi_above_hat[0, 0] = 0.0
        self.phi_below_hat, self.phi_above_hat = phi_below_hat, phi_above_hat
        self.Bz_below = idct2(bz_below_hat)
        self.Bz_above = idct2(bz_above_hat)
        self.Phi_below_bottom = idct2(phi_below_hat)
        self.Phi_above_bottom = idct2(phi_above_hat)
        z = np.arange(nz, dtype=np.float64) * self.dz
        decay = np.exp(-z[:, None, None] * k[None])
        phi_below = idct2(decay * phi_below_hat[None])
        bz_below = idct2(decay * bz_below_hat[None])
        if self.ghop == "spectral":
            dphi_dz = idct2((-k)[None] * decay * phi_below_hat[None])
            gx, gy = self.spectral_dx_2d(dphi_dz), self.spectral_dy_2d(dphi_dz)
            bx_below, by_below = -gx, -gy
        else:
            dpz = d_dz(phi_below, self.dz)
            bx_below, by_below = -d_dx(dpz, self.dx), -d_dy(dpz, self.dy)
        self.B_below = np.stack([bx_below, by_below, bz_below])
        B_open = np.zeros_like(self.B_below)
        B_open[2] = self.Bz_open_mean
        self.B_external_harmonic = supplemental.copy()
        self.B_background = self.B_below + B_open + self.B_external_harmonic
        self.Phi_pot = phi_below
        self.bottom_dphi_c_target = idct2(dphi_total_hat) - d_dz(phi_below, self.dz)[0]
        recon = self.B_background[2, 0] + self.Bz_above - self.Bz_obs
        b_from_phi = np.stack([bx_below, by_below, lap_xy(phi_below, self.dx, self.dy)])
        inv = b_from_phi + B_open + self.B_external_harmonic - self.B_background
        self.gaussian_separation_diagnostics = {
            "bottom_reconstruction_rms": _rms(recon),
            "bottom_reconstruction_max": float(np.abs(recon).max()),
            "mean_field": [float(v) for v in self.B_mean],
            "dct_zero_mode_Bx": float(self.B_mean[0]),
            "dct_zero_mode_By": float(self.B_mean[1]),
            "dct_zero_mode_Bz": float(self.B_mean[2]),
            "arithmetic_mean_B": [float(self.Bx_obs.mean()), float(self.By_obs.mean()), float(self.Bz_obs.mean())],
            "mean_bz_policy": self.mean_bz_policy,
            "horizontal_zero_mode_policy": self.hzm,
            "gaussian_horizontal_operator": self.ghop,
            "Bz_open_mean": float(self.Bz_open_mean),
            "Bh_mean_bottom": [float(self.B_mean[0]), float(self.B_mean[1])],
            "flux_imbalance_fraction": flux_imb,
            "D0_zero_mode": d0_mean,
            "D0_zero_mode_ratio": d0_ratio,
            "d0_removed_constant_mode": d0_mean,
            "background_scalar_plus_explicit_rms": _rms(inv),
        }
        self.gaussian_separation_diagnostics.update(self._bottom_harmonic_diagnostics())
        self._init_k0()

    def _init_k0(self):
        """H(z) start and closure operators (nfgs_solver.py:4911-4919,
        5058-5097, 5149-5225, 5262-5360)."""
        nz = self.Nz
        tgt = [float(v) for v in self.H_bottom_target]
        self.k0 = None
        self.k0_history = []
        if self.hzm == "frozen_linear_harmonic":
            self.H = np.repeat(self.H_bottom_target[:, None], nz, axis=1)
            self.k0_diagnostics = {"enabled": True, "closure": "frozen_linear_harmonic",
                                   "representation": "analytic_Az_linear_lift", "bottom_target": tgt,
                                   "current_free": True, "open_side_current": False, "top_derivative": [0.0, 0.0],
                                   "profile_max_abs": float(np.abs(self.H).max())}
        elif self.hzm == "coupled_k0":
            self.H = np.repeat(self.H_bottom_target[:, None], nz, axis=1)
            self.k0 = CoupledK0(nz, self.dz, self.k0_smoothness, self.k0_legacy)
            self.k0_diagnostics = {"enabled": True, "smoothness": self.k0_smoothness,
                                   "discretization": ("legacy_plane_centred" if self.k0_legacy else
                                                      "staggered_face_D1_true_three_point_curvature"),
                                   "bottom_target": tgt, "open_side_current": True}
            if self.k0_legacy:
                self.k0_diagnostics["diagnosis_only"] = True
        elif self.hzm == "constrained_spline_harmonic":
            self.H = np.repeat(self.H_bottom_target[:, None], nz, axis=1)
            self.k0 = SplineK0(nz, self.dz, self.k0_basis, self.k0_smoothness)
            self.k0_diagnostics = {"enabled": True, "closure": "constrained_spline_harmonic",
                                   "representation": "cubic_bspline_explicit_linear_harmonic_lift",
                                   "basis_size": self.k0_basis, "smoothness": self.k0_smoothness,
                                   "update_mu": self.k0_update_mu, "bottom_target": tgt,
                                   "bottom_constraint": "exact",
                                   "top_constraint": "discrete_second_order_Hprime_zero",
                                   "lateral_current_contract": "open_harmonic_plus_closed_PT",
                                   "open_side_current": True, "top_derivative": [0.0, 0.0],
                                   "kkt_condition_number": float(np.linalg.cond(self.k0.kkt))}
        else:
            self.H = None
            self.k0_diagnostics = {}

    def k0_field_and_current(self, prof):
        """Uniform field H and current (-dH_y/dz, dH_x/dz, 0) by plane
        (nfgs_solver.py:5434-5455)."""
        if self.k0 is not None:
            der = self.k0.centre_derivative(prof)
        else:
            der = centre_derivative_fd2(prof, self.dz)
        return prof, np.stack([-der[1], der[0]])

    def _bottom_harmonic_diagnostics(self):
        """nfgs_solver.py:4962-5029."""
        dphi = idct2(self.k * (self.phi_above_hat - self.phi_below_hat))
        gx, gy = self.horizontal_grad(dphi)
        bt_x = d_dy(self.Az_bottom, self.dy)
        bt_y = -d_dx(self.Az_bottom, self.dx)
        rec = np.stack([-gx + bt_x, -gy + bt_y]) + self.B_external_harmonic[:2, 0]
        obs = np.stack([self.Bx_obs, self.By_obs])
        res = obs - rec
        const = np.array([self.const_mode(dct2(res[0])), self.const_mode(dct2(res[1]))])
        self.H_bottom_target = const.copy()
        nonconst = res - const[:, None, None]
        div = self.horizontal_div(res[0], res[1])
        curl = d_dx(res[1], self.dx) - d_dy(res[0], self.dy)
        res_rms, obs_rms = _rms(res), _rms(obs)
        ratio = res_rms / max(obs_rms, 1e-30)
        if ratio > self.mean_mode_tolerance:
            msg = (f"Bottom horizontal reconstruction leaves a finite-domain harmonic residual "
                   f"ratio={ratio:.6e}, tolerance={self.mean_mode_tolerance:.6e}.")
            if self.harm_policy == "error":
                raise ValueError(msg)
            if self.harm_policy == "warn":
                warnings.warn(msg, RuntimeWarning, stacklevel=3)
        return {
            "bottom_horizontal_reconstruction_rms": res_rms,
            "bottom_horizontal_reconstruction_ratio": ratio,
            "harmonic_residual_constant": [float(v) for v in const],
            "harmonic_residual_constant_rms": _rms(const),
            "harmonic_residual_nonconstant_rms": _rms(nonconst),
            "harmonic_residual_divergence_rms": _rms(div),
            "harmonic_residual_curl_rms": _rms(curl),
        }

    def gaussian_above_bottom_field(self):
        """nfgs_solver.py:4921-4946."""
        dphi = idct2(self.k * self.phi_above_hat)
        gx, gy = self.horizontal_grad(dphi)
        return np.stack([-gx, -gy, self.Bz_above])

    # ------------------------------------------------------------ solves
    def _diagnose_source_zero_mode(self, source, context):
        """nfgs_solver.py:5457-5476."""
        mean_by_height = self.const_mode(dct2(source))
        ratio = float(np.sqrt(np.mean(mean_by_height**2)) / max(_rms(source), 1e-30))
        self.last_source_zero_mode_by_height = [float(v) for v in mean_by_height]
        self.source_zero_mode_history.append(ratio)
        self._policy(ratio, self.source_zero_mode_tolerance, self.src_policy,
                     f"The {context} nonlinear source has an incompatible zero mode")

    def modal_robin(self, source_hat, bottom_hat, derivative_hat=None, rho=0.0, top_robin_hat=None):
        """Modal top-Robin / mixed-bottom tridiagonal solve (nfgs_solver.py:5512-5625)."""
        source_hat = source_hat.copy()
        bottom_hat = bottom_hat.copy()
        source_hat[:, 0, 0] = 0.0
        bottom_hat[0, 0] = 0.0
        top = np.zeros_like(bottom_hat) if top_robin_hat is None else np.array(top_robin_hat, dtype=np.float64)
        top[0, 0] = 0.0
        if rho > 0:
            derivative_hat = derivative_hat.copy()
            derivative_hat[0, 0] = 0.0
        lam = self.lam_neumann()
        k = self.k
        dz = self.dz
        dz2 = dz * dz
        low, up = 1.0 / dz2, 1.0 / dz2
        diag = lam - 2.0 / dz2
        n = self.Nz - 1
        c = np.empty((n,) + lam.shape)
        d = np.empty_like(c)
        if rho > 0:
            known_bottom = (1.0 + 0.5 * rho) / dz2
            fdiag = (1.0 - rho) * lam - 2.0 / dz2
            fup = (1.0 - 0.5 * rho) / dz2
            frhs = (1.0 - rho) * source_hat[1] - rho * derivative_hat / dz
            rhs0 = frhs - known_bottom * bottom_hat
        else:
            fdiag, fup = diag, up
            rhs0 = source_hat[1] - low * bottom_hat
        c[0] = fup / fdiag
        d[0] = rhs0 / fdiag
        for r in range(1, n - 1):
            den = diag - low * c[r - 1]
            c[r] = up / den
            d[r] = (source_hat[r + 1] - low * d[r - 1]) / den
        rl = -lam * dz2 - 2.0
        rd = 2.0 + 2.0 * dz * k
        rr = 2.0 * dz * top - source_hat[-2] * dz2
        last = n - 1
        den = rd - rl * c[last - 1]
        c[last] = 0.0
        d[last] = (rr - rl * d[last - 1]) / den
        sol = np.empty_like(source_hat)
        sol[0] = bottom_hat
        sol[-1] = d[last]
        for r in range(last - 1, -1, -1):
            sol[r + 1] = d[r] - c[r] * sol[r + 2]
        sol[:, 0, 0] = 0.0
        return idct2(sol)

    def solve_phi_c(self, source_bcz, bottom_phi):
        """nfgs_solver.py:5627-5672."""
        lam = self.lam_neumann().copy()
        lam[0, 0] = 1.0
        self._diagnose_source_zero_mode(source_bcz, "Phi_c")
        source_hat = dct2(source_bcz) / lam[None]
        source_hat[:, 0, 0] = 0.0
        bottom_hat = dct2(bottom_phi)
        bottom_hat[0, 0] = 0.0
        deriv = None
        if self.rho > 0:
            deriv = dct2(self.bottom_dphi_c_target)
            deriv[0, 0] = 0.0
        phi = self.modal_robin(source_hat, bottom_hat, deriv, self.rho)
        if self.rho > 0:
            phi[0] = bottom_phi
        return phi

    def thomas_dirichlet(self, rhs_hat, u0, lam, u_top):
        """Dirichlet-Dirichlet Thomas along z (nfgs_solver.py:536-608)."""
        nz = rhs_hat.shape[0]
        dz2 = self.dz * self.dz
        a = c = 1.0 / dz2
        b = lam - 2.0 / dz2
        n = nz - 2
        u = np.zeros_like(rhs_hat)
        u[0] = u0
        u[nz - 1] = u_top
        if n <= 0:
            return u
        cs = np.empty((n,) + b.shape)
        ds = np.empty_like(cs)
        d0 = rhs_hat[1] - a * u0
        if n == 1:
            d0 = d0 - c * u_top
            cs[0] = 0.0
            ds[0] = d0 / b
        else:
            cs[0] = c / b
            ds[0] = d0 / b
            for i in range(1, n):
                dd = rhs_hat[i + 1]
                ce = c
                if i == n - 1:
                    dd = dd - c * u_top
                    ce = 0.0
                den = b - a * cs[i - 1]
                cs[i] = ce / den
                ds[i] = (dd - a * ds[i - 1]) / den
        for i in range(n - 2, -1, -1):
            ds[i] = ds[i] - cs[i] * ds[i + 1]
        u[1:1 + n] = ds
        return u

    def solve_az(self, source_jz):
        """Toroidal chain (nfgs_solver.py:3263-3306)."""
        az = np.zeros_like(source_jz)
        az[0] = self.Az_bottom
        az[-1] = 0.0
        if self.Nx < 3 or self.Ny < 3:
            return az
        lam = self.lam_dirichlet()
        rhs_hat = -dst2(source_jz[:, 1:-1, 1:-1]) / lam
        bottom_hat = dst2(self.Az_bottom[1:-1, 1:-1])
        top_hat = np.zeros_like(bottom_hat)
        az_hat = self.thomas_dirichlet(rhs_hat, bottom_hat, lam, top_hat)
        az[:, 1:-1, 1:-1] = idst2(az_hat)
        az[0] = self.Az_bottom
        az[-1] = 0.0
        self._az_walls_zero(az)
        return az

    @staticmethod
    def _az_walls_zero(az):
        """nfgs_solver.py:2150-2152."""
        az[:, :, 0] = 0.0
        az[:, :, -1] = 0.0
        az[:, 0, :] = 0.0
        az[:, -1, :] = 0.0

    def apply_projection(self, phi):
        """Bottom-divergence projection (nfgs_solver.py:4948-4988)."""
        w = self.proj_w
        if w == 0.0:
            return phi
        cur = (-3.0 * phi[0] + 4.0 * phi[1] - phi[2]) / (2.0 * self.dz)
        res = self.bottom_dphi_c_target - cur
        out = phi.copy()
        out[1] += (8.0 * self.dz / 17.0) * w * res
        out[2] -= (2.0 * self.dz / 17.0) * w * res
        out[0] = self.Phi_above_bottom
        post = (-3.0 * out[0] + 4.0 * out[1] - out[2]) / (2.0 * self.dz)
        self.projection_history.append({
            "pre_derivative_rms": _rms(res),
            "post_derivative_rms": _rms(self.bottom_dphi_c_target - post),
            "increment_rms": _rms(out - phi),
        })
        return out

    # ------------------------------------------------ state reconstruction
    def face_state(self, B, Jz_center):
        """Vertical-face B and carrier curl (nfgs_solver.py:5738-5778)."""
        Bf = 0.5 * (B[:, 1:] + B[:, :-1])
        car = B - self.B_background
        carf = 0.5 * (car[:, 1:] + car[:, :-1])
        dbx = (car[0, 1:] - car[0, :-1]) / self.dz
        dby = (car[1, 1:] - car[1, :-1]) / self.dz
        jxf = d_dy(carf[2], self.dy) - dby
        jyf = dbx - d_dx(carf[2], self.dx)
        jzf = 0.5 * (Jz_center[1:] + Jz_center[:-1])
        return Bf, np.stack([jxf, jyf, jzf])

    @staticmethod
    def faces_to_centres(v):
        """nfgs_solver.py:5780-5794."""
        nzf = v.shape[1]
        out = np.empty((v.shape[0], nzf + 1) + v.shape[2:])
        out[:, 0] = v[:, 0]
        out[:, -1] = v[:, -1]
        if nzf + 1 > 2:
            out[:, 1:-1] = 0.5 * (v[:, :-1] + v[:, 1:])
        return out

    def _zero_j_walls(self, J):
        """nfgs_solver.py:6069-6078."""
        J[:, :, :, 0] = 0.0
        J[:, :, :, -1] = 0.0
        J[:, :, 0, :] = 0.0
        J[:, :, -1, :] = 0.0
        J[:, -1] = 0.0

    def reconstruct(self, phi_c, az, bc_z):
        """nfgs_solver.py:5901-5942 -> 3311-3341."""
        dpz = d_dz(phi_c, self.dz)
        bcx = -d_dx(dpz, self.dx) + d_dy(az, self.dy)
        bcy = -d_dy(dpz, self.dy) - d_dx(az, self.dx)
        jz = -lap_xy(az, self.dx, self.dy)
        Bc = np.stack([bcx, bcy, bc_z])
        B = self.B_background + Bc
        J = np.stack([np.zeros_like(jz), np.zeros_like(jz), jz])
        self._zero_j_walls(J)
        B[2, 0] = self.Bz_obs
        J[2, 0] = self.Jz_T
        jh = None
        if self.H is not None:
            hb, jh = self.k0_field_and_current(self.H)
            B[0] = B[0] + hb[0][:, None, None]
            B[1] = B[1] + hb[1][:, None, None]
            J[0] = J[0] + jh[0][:, None, None]
            J[1] = J[1] + jh[1][:, None, None]
            B[2, 0] = self.Bz_obs
            J[2, 0] = self.Jz_T
            J[:, -1] = 0.0
        _bf, jf = self.face_state(B, J[2])
        Js = self.faces_to_centres(jf)
        if self.hzm == "constrained_spline_harmonic":
            # the closed PT current gets zero walls, the explicit harmonic
            # current stays open on them (nfgs_solver.py:5920-5933); all
            # three components come from the face current, so J_z is the
            # face average of J_z mapped back to the planes
            jt = Js.copy()
            jt[0] -= jh[0][:, None, None]
            jt[1] -= jh[1][:, None, None]
            self._zero_j_walls(jt)
            jt[0] += jh[0][:, None, None]
            jt[1] += jh[1][:, None, None]
            J = jt
            J[:, -1] = 0.0
        else:
            J[:2] = Js[:2]
            self._zero_j_walls(J)
        J[2, 0] = self.Jz_T
        return B, J, Bc

    def pt_current_xy(self, phi_c, az, bc_z):
        """Horizontal current of the PT scalars alone (ccu_pure_current,
        nfgs_solver.py:3311-3341 with 1760-1768), walls and top zero
        (nfgs_solver.py:6069-6078)."""
        dazdz = d_dz(az, self.dz)
        lphi = bc_z + self.d2dz2(phi_c)
        jx = d_dx(dazdz, self.dx) + d_dy(lphi, self.dy)
        jy = d_dy(dazdz, self.dy) - d_dx(lphi, self.dx)
        J = np.stack([jx, jy, np.zeros_like(jx)])
        self._zero_j_walls(J)
        return J[:2]

    def plane_means(self, f):
        """DCT-I zero mode of each plane (nfgs_solver.py:5944-5950)."""
        return np.stack([self.const_mode(dct2(f[0])), self.const_mode(dct2(f[1]))])

    def k0_target(self, jp, B, J):
        """Target mean current of the H(z) fit (nfgs_solver.py:5859-5880,
        6718-6724): the cell parallel current, or the face-aligned current's
        plain plane means mapped to the planes."""
        if not self.k0_face_target:
            return jp
        Bf, Jf = self.face_state(B, J[2])
        b2 = np.maximum((Bf * Bf).sum(0), self.weak_floor)
        alpha = (Jf * Bf).sum(0) / b2
        am = self.alpha_max()
        if am is not None and math.isfinite(am):
            alpha = np.clip(alpha, -am, am)
        mf = (alpha[None] * Bf).mean(axis=(-2, -1))
        mc = np.empty((3, self.Nz))
        mc[:, 0] = mf[:, 0]
        mc[:, -1] = mf[:, -1]
        mc[:, 1:-1] = 0.5 * (mf[:, :-1] + mf[:, 1:])
        out = np.broadcast_to(mc[:, :, None, None], jp.shape).copy()
        w = self.buffer_window()
        if w is not None:
            out = out * w
        return out

    def k0_update(self, jpk0, phi_s, az_s):
        """H* from the mean-current fit (nfgs_solver.py:5952-6067)."""
        jpt = self.pt_current_xy(phi_s, az_s, lap_xy(phi_s, self.dx, self.dy))
        desired = self.plane_means(jpk0) - self.plane_means(jpt)
        hx = self.k0.solve(desired[1], float(self.H_bottom_target[0]))
        hy = self.k0.solve(-desired[0], float(self.H_bottom_target[1]))
        prof = np.stack([hx, hy])
        self.k0_diagnostics.update(fit_diagnostics(self.k0, prof, desired, self.k0_history))
        return prof

    def recover_h(self, B, Bc):
        """H of a stored state: plane means of B - B_background - B_c with the
        bottom target (nfgs_solver.py:6685-6693, 6991-7004)."""
        h = (B[:2] - self.B_background[:2] - Bc[:2]).mean(axis=(-2, -1))
        h[:, 0] = self.H_bottom_target
        return h

    # -------------------------------------------------------- diagnostics
    def cwsin_slices(self, nz_faces):
        """nfgs_solver.py:2656-2676 applied to the face grid."""
        nzo, nyo, nxo = self.observed_shape
        sy_fov, sx_fov = self.fov
        bfx, bfy = int(sx_fov.start or 0), int(sy_fov.start or 0)
        nz, ny, nx = nz_faces, self.Ny, self.Nx
        bfz = max(0, nz - int(nzo))
        ax = int(nxo) // 8 + bfx
        ay = int(nyo) // 8 + bfy
        az = int(nzo) // 4 + bfz
        sz = slice(1, max(1, nz - 1 - az + 1))
        sy = slice(ay, max(ay + 1, ny - 1 - ay + 1))
        sx = slice(ax, max(ax + 1, nx - 1 - ax + 1))
        return sz, sy, sx

    def compute_sigma(self, B, J):
        """Face sigma_J over the cwsin box (nfgs_solver.py:5882-5895)."""
        Bf, Jf = self.face_state(B, J[2])
        sz, sy, sx = self.cwsin_slices(Bf.shape[1])
        b = Bf[:, sz, sy, sx]
        j = Jf[:, sz, sy, sx]
        bn = np.maximum(np.sqrt((b * b).sum(0)), 1e-10)
        jn = np.sqrt((j * j).sum(0))
        jxb = np.cross(np.moveaxis(j, 0, -1), np.moveaxis(b, 0, -1))
        num = (np.sqrt((jxb * jxb).sum(-1)) / bn).sum()
        return float(num / max(jn.sum(), 1e-30))

    def compute_divB(self, B):
        """nfgs_solver.py:2689-2693."""
        div = d_dx(B[0], self.dx) + d_dy(B[1], self.dy) + d_dz(B[2], self.dz)
        bm = np.sqrt(B[0] ** 2 + B[1] ** 2 + B[2] ** 2)
        delta = min(self.dx, self.dy, self.dz)
        return float(np.abs(div).mean() / (6.0 * bm.mean() / delta + 1e-12))

    def compute_energy(self, B):
        """nfgs_solver.py:2695-2697."""
        return float((B[0] ** 2 + B[1] ** 2 + B[2] ** 2).sum() * self.dx * self.dy * self.dz / 2.0)

    # ----------------------------------------------------------- iteration
    def parallel_current(self, J, B):
        """Face-aligned current mapped to centres (nfgs_solver.py:5811-5853)."""
        Bf, Jf = self.face_state(B, J[2])
        b2 = np.maximum((Bf * Bf).sum(0), self.weak_floor)
        alpha = (Jf * Bf).sum(0) / b2
        am = self.alpha_max()
        if am is not None and math.isfinite(am):
            alpha = np.clip(alpha, -am, am)
        return self.faces_to_centres(alpha[None] * Bf)

    def compute_initial_conditions(self, init_mode="gs_cfcf"):
        """gs_cfcf start (nfgs_solver.py:6613-6645); soft_cfcf dispatches to
        soft_cfcf_initial_state."""
        mode = str(init_mode).lower().replace("-", "_")
        if mode in ("soft_cfcf", "yi_soft"):
            return self.soft_cfcf_initial_state()
        if mode in ("cfcf", "curl_free_current"):
            return self.cfcf_initial_state(lateral_bc1=getattr(self, "lateral_bc1", True))
        if mode != "gs_cfcf":
            raise NotImplementedError("the oracle restates the gs_cfcf, cfcf and soft_cfcf starts")
        zeros = np.zeros((self.Nz, self.Ny, self.Nx))
        phi = self.solve_phi_c(zeros, self.Phi_above_bottom)
        phi = self.apply_projection(phi)
        bcz = lap_xy(phi, self.dx, self.dy)
        az = self.solve_az(zeros)
        B, J, Bc = self.reconstruct(phi, az, bcz)
        return B, J, phi, az, Bc

    def harmonic_modal(self, u0_hat, lam, top_dirichlet):
        """Zero-source modal Thomas solve along z with Dirichlet bottom u0_hat
        and a Dirichlet (zero) or mirrored-ghost Neumann top
        (_thomas_solve_batched_lowmem, nfgs_solver.py:536-608)."""
        nz = self.Nz
        dz2 = self.dz * self.dz
        a = c = 1.0 / dz2
        b = lam - 2.0 / dz2
        n = nz - 2 if top_dirichlet else nz - 1
        u = np.zeros((nz,) + lam.shape)
        u[0] = u0_hat
        if n <= 0:
            return u
        cs = np.empty((n,) + lam.shape)
        ds = np.empty_like(cs)
        bottom_a = 2.0 * a if (n == 1 and not top_dirichlet) else a
        d0 = 0.0 - bottom_a * u0_hat
        if n == 1:
            cs[0] = 0.0
            ds[0] = d0 / b
        else:
            cs[0] = c / b
            ds[0] = d0 / b
            for i in range(1, n):
                ae, ce = a, c
                if i == n - 1:
                    ce = 0.0
                    if not top_dirichlet:
                        ae = 2.0 * a
                den = b - ae * cs[i - 1]
                cs[i] = ce / den
                ds[i] = (0.0 - ae * ds[i - 1]) / den
        for i in range(n - 2, -1, -1):
            ds[i] = ds[i] - cs[i] * ds[i + 1]
        u[1:1 + n] = ds
        return u

    def cfcf_initial_state(self, lateral_bc1=True):
        """cfcf start (nfgs_solver.py:6080-6147): the Stable-NFPT
        curl-free-current state (nfgs_solver.py:2331-2376, 3343-3405) projected
        into the NFGS scalars.  Its A_z is the zero-source Dirichlet extension
        of the stable solver's T = Poisson2D(-Jz) (nfgs_solver.py:2331-2351,
        1305-1333, 3394-3398); its B_z is the potential field's, the harmonic extension of
        Bz_obs with a Neumann top (nfgs_solver.py:1611-1627), with the BC1
        wall and top copies (nfgs_solver.py:2138-2156) and Bz_obs on the bottom
        plane.  Phi_c solves lap_xy Phi_c = B_z - B_background,z plane by plane
        above the bottom (mean mode dropped, nfgs_solver.py:1120-1130,
        1146-1181), Phi_c(0) = Phi^>.  Returns (B, J, Phi_c, A_z, B_c) and sets
        cfcf_diagnostics (the mean B_c,z per height)."""
        nz, ny, nx = self.Nz, self.Ny, self.Nx
        lamN = self.lam_neumann()
        bz_hat = dct2(self.Bz_obs)
        bzp = idct2(self.harmonic_modal(bz_hat, lamN, top_dirichlet=False))
        if lateral_bc1:
            if nx > 1:
                bzp[:, 1:-1, 0] = bzp[:, 1:-1, 1]
                bzp[:, 1:-1, -1] = bzp[:, 1:-1, -2]
            if ny > 1:
                bzp[:, 0, :] = bzp[:, 1, :]
                bzp[:, -1, :] = bzp[:, -2, :]
            if nz > 1:
                bzp[-1] = bzp[-2]
        bzp[0] = self.Bz_obs
        bcz = bzp - self.B_background[2]
        hat = dct2(bcz)
        norm = 4.0 * max(nx - 1, 1) * max(ny - 1, 1)
        mean_by_height = hat[:, 0, 0] / norm
        lam = lamN.copy()
        lam[0, 0] = 1.0
        ph = hat / lam[None]
        ph[:, 0, 0] = 0.0
        phi = idct2(ph)
        phi[0] = self.Phi_above_bottom
        if self.bottom_current_grid_mode == "legacy_helper":
            t_st = self.Az_bottom
        else:
            t_st = self.poisson2d_dirichlet(-self.Jz_stable)
        az = np.zeros((nz, ny, nx))
        if nx >= 3 and ny >= 3:
            lamD = self.lam_dirichlet()
            az[:, 1:-1, 1:-1] = idst2(self.harmonic_modal(dst2(t_st[1:-1, 1:-1]), lamD, top_dirichlet=True))
        az[0] = t_st
        az[-1] = 0.0
        self._az_walls_zero(az)
        self.cfcf_diagnostics = {"stable_cfcf_mean_bcz_by_height": [float(v) for v in mean_by_height]}
        B, J, Bc = self.reconstruct(phi, az, lap_xy(phi, self.dx, self.dy))
        return B, J, phi, az, Bc

    def soft_cfcf_initial_state(self):
        """soft_cfcf start (nfgs_solver.py:6427-6484): per horizontal mode the
        z profile minimising the modal curl(J) functional with the bottom and
        transparent-top rows exact; Phi_c and A_z from the inverse transforms,
        bottom planes restored, A_z walls zero."""
        from . import soft_cfcf_oracle as SO

        if self.Nz < 5:
            raise ValueError("soft_cfcf requires Nz >= 5")
        if self.Nx < 3 or self.Ny < 3:
            raise ValueError("soft_cfcf requires Nx, Ny >= 3")
        nz, ny, nx = self.Nz, self.Ny, self.Nx
        eps, ridge = self.soft_cfcf_epsilon, self.soft_cfcf_normal_ridge
        k_phi = np.sqrt(np.maximum(-self.lam_neumann(), 0.0))
        pb = dct2(self.Phi_above_bottom)
        pb[0, 0] = 0.0
        phi_hat = SO.modal_profiles(k_phi, pb, "phi", nz, self.dz, eps, ridge).reshape(nz, ny, nx)
        phi = idct2(phi_hat)
        phi[0] = self.Phi_above_bottom
        k_az = np.sqrt(np.maximum(-self.lam_dirichlet(), 0.0))
        ab = dst2(self.Az_bottom[1:-1, 1:-1])
        az_hat = SO.modal_profiles(k_az, ab, "az", nz, self.dz, eps, ridge).reshape(nz, ny - 2, nx - 2)
        az = np.zeros((nz, ny, nx))
        az[:, 1:-1, 1:-1] = idst2(az_hat)
        az[0] = self.Az_bottom
        self._az_walls_zero(az)
        en = SO.modal_energies(phi_hat, k_phi, az_hat, k_az, nx, ny, self.dx, self.dy, self.dz)
        en["objective"] = en["curl_current_energy"] + eps * en["current_energy"]
        self.soft_cfcf_diagnostics = en
        bcz = lap_xy(phi, self.dx, self.dy)
        B, J, Bc = self.reconstruct(phi, az, bcz)
        return B, J, phi, az, Bc

    def face_fractions(self, B, J):
        """Weak-field and alpha-clip fractions of the face state
        (nfgs_solver.py:6660-6681): means over every vertical face."""
        Bf, Jf = self.face_state(B, J[2])
        b2 = (Bf * Bf).sum(0)
        weak = float(np.mean(b2 <= self.weak_floor))
        alpha = (Jf * Bf).sum(0) / np.maximum(b2, self.weak_floor)
        am = self.alpha_max()
        clip = float(np.mean(np.abs(alpha) > am)) if am is not None else 0.0
        return clip, weak

    @staticmethod
    def _rms(v):
        return float(np.sqrt(np.mean(np.asarray(v, dtype=np.float64) ** 2)))

    def d2dz2(self, f):
        """nfgs_solver.py:1717-1727."""
        dz2 = self.dz ** 2
        d2 = np.zeros_like(f)
        if f.shape[0] >= 3:
            d2[1:-1] = (f[2:] - 2 * f[1:-1] + f[:-2]) / dz2
        if f.shape[0] >= 2:
            if f.shape[0] >= 4:
                d2[0] = (2.0 * f[0] - 5.0 * f[1] + 4.0 * f[2] - f[3]) / dz2
            else:
                d2[0] = (f[1] - f[0]) / dz2
            d2[-1] = (-2.0 * f[-1] + 2.0 * f[-2]) / dz2
        return d2

    def step_diagnostics(self, phi, az, phi_s, az_s, s_b, s_j, phi_n, az_n, Bn, Jn, clip, weak,
                         h_before=None, h_star=None):
        """The per-step diagnostics of record_iteration_diagnostics
        (nfgs_solver.py:6806-6929) for one attempted candidate."""
        rms = self._rms

        def rel(delta, scale):
            return rms(delta) / max(rms(scale), 1e-30)

        def rel_op(residual, *terms):
            return rms(residual) / max(max(rms(t) for t in terms), 1e-30)

        nz = self.Nz
        lx = lambda f: lap_xy(f, self.dx, self.dy)  # noqa: E731
        bcz_s = lx(phi_s)
        bcz_res = self.d2dz2(bcz_s) + lx(bcz_s) - s_b
        jz_s = -lx(az_s)
        jz_res = self.d2dz2(jz_s) + lx(jz_s) - s_j
        bi = slice(2, -1) if nz > 4 else slice(1, -1)
        lam = self.lam_neumann().copy()
        lam[0, 0] = 1.0
        sp_hat = dct2(s_b) / lam[None]
        sp_hat[:, 0, 0] = 0.0
        source_phi = idct2(sp_hat)
        d2p, lxp = self.d2dz2(phi_s), lx(phi_s)
        phi_res = d2p + lxp - source_phi
        source_az = np.zeros_like(az_s)
        source_az[:, 1:-1, 1:-1] = idst2(-dst2(s_j[:, 1:-1, 1:-1]) / self.lam_dirichlet()[None])
        d2a, lxa = self.d2dz2(az_s), lx(az_s)
        az_res = d2a + lxa - source_az
        dphi_bottom = (-3.0 * phi_s[0] + 4.0 * phi_s[1] - phi_s[2]) / (2.0 * self.dz)
        target = self.bottom_dphi_c_target if self.bottom_dphi_c_target is not None else np.zeros_like(dphi_bottom)
        mixed_pde = (1.0 - self.rho) * phi_res[1]
        mixed_der = -self.rho * (dphi_bottom - target) / self.dz
        obs = np.stack([self.Bx_obs, self.By_obs, self.Bz_obs])
        ii = (slice(1, -1), slice(1, -1), slice(1, -1))
        return {
            "phi_update_relative": rel(phi_n - phi, phi),
            "az_update_relative": rel(az_n - az, az),
            "phi_map_residual_relative": rel(phi_s - phi, phi),
            "az_map_residual_relative": rel(az_s - az, az),
            "h_k0_update_relative": (rel(self.H - h_before, h_before)
                                     if h_before is not None and self.H is not None else 0.0),
            "h_k0_map_residual_relative": (rel(h_star - h_before, h_before)
                                           if h_star is not None and h_before is not None else 0.0),
            "bcz_pde_residual_relative": rel(bcz_res[bi], s_b[bi]),
            "jz_pde_residual_relative": rel(jz_res[1:-1], s_j[1:-1]),
            "poloidal_pde_residual_relative": rel_op(phi_res[bi], d2p[bi], lxp[bi], source_phi[bi]),
            "toroidal_pde_residual_relative": rel_op(az_res[ii], d2a[ii], lxa[ii], source_az[ii]),
            "mixed_row_residual_relative": rel_op(mixed_pde + mixed_der, mixed_pde, mixed_der, source_phi[1]),
            "bottom_field_imprint_relative": rel(Bn[:, 0] - obs, obs),
            "bottom_jz_imprint_relative": rel(Jn[2, 0] - self.Jz_T, self.Jz_T),
            "alpha_clip_fraction": clip,
            "weak_field_floor_fraction": weak,
        }

    def iteration_step(self, B, J, phi, az, Bc, mu=1.0, polarity_mask="both"):
        """NFGS NFPT update (nfgs_solver.py:6647-6935, production branch)."""
        h_before = self.H.copy() if (self.record_iteration_diagnostics and self.H is not None) else None
        if self.record_iteration_diagnostics:
            clip, weak = self.face_fractions(B, J)
        if self.k0 is not None:
            self.H = self.recover_h(B, Bc)
        jp = self.parallel_current(J, B)
        if polarity_mask == "positive":
            jp[:, 0] = J[:, 0] * (self.Bz_obs > 0)
        elif polarity_mask == "negative":
            jp[:, 0] = J[:, 0] * (self.Bz_obs < 0)
        elif polarity_mask == "both":
            if self.bpcm == "face_parallel_exact_jz":
                jp[2, 0] = self.Jz_T
            else:
                jp[:, 0] = J[:, 0]
        else:
            raise ValueError("polarity_mask must be 'positive', 'negative', or 'both'")
        w = self.buffer_window()
        if w is not None:
            jp = jp * w
        jpk0 = self.k0_target(jp, B, J) if self.k0 is not None else None
        s_b = d_dy(jp[0], self.dy) - d_dx(jp[1], self.dx)
        phi_s = self.solve_phi_c(s_b, self.Phi_above_bottom)
        s_j = lap_xy(jp[2], self.dx, self.dy) - d2_dxdz(jp[0], self.dx, self.dz) - d2_dydz(jp[1], self.dy, self.dz)
        az_s = self.solve_az(s_j)
        phi_s[0] = self.Phi_above_bottom
        phi_s = self.apply_projection(phi_s)
        az_s[0] = self.Az_bottom
        az_s[-1] = 0.0
        self._az_walls_zero(az_s)
        h_star = None
        if self.k0 is not None:
            h_star = self.k0_update(jpk0, phi_s, az_s)
            mu_k0 = self.k0_update_mu if self.k0_update_mu is not None else float(mu)
            self.H = mu_k0 * h_star + (1.0 - mu_k0) * self.H if mu_k0 < 1.0 else h_star
        if mu < 1.0:
            phi_n = mu * phi_s + (1.0 - mu) * phi
            az_n = mu * az_s + (1.0 - mu) * az
        else:
            phi_n, az_n = phi_s, az_s
        phi_n[0] = self.Phi_above_bottom
        bcz = lap_xy(phi_n, self.dx, self.dy)
        az_n[0] = self.Az_bottom
        az_n[-1] = 0.0
        self._az_walls_zero(az_n)
        Bn, Jn, Bcn = self.reconstruct(phi_n, az_n, bcz)
        if self.record_iteration_diagnostics:
            self.last_iteration_diagnostics = self.step_diagnostics(
                phi, az, phi_s, az_s, s_b, s_j, phi_n, az_n, Bn, Jn, clip, weak, h_before, h_star)
        return Bn, Jn, phi_n, az_n, Bcn

    def iterate(self, max_iter=200, tol=1e-5, mu=1.0, patience=1, verbose=False,
                polarity_mask="both", init_mode="gs_cfcf", sigma_improvement_tol=1e-5,
                per_step_callback: Optional[Callable] = None, *, adaptive_mu=False,
                mu_min=0.02, mu_max=1.0, mu_backoff=0.5, mu_growth=1.1, growth_streak=5,
                divergence_factor=2.0, max_rollbacks=12, stop_mode="sigma_best",
                fixed_point_update_tol=None, fixed_point_pde_tol=1.0e-8, fixed_point_observable_tol=None,
                fixed_point_patience=10, **_ignored):
        """Stable driver (nfgs_solver.py:3522-3850) with the NFGS wrapper (6937-7009),
        including the fixed-point stop (nfgs_solver.py:3572-3584, 3707-3776) and the
        per-step diagnostics history (nfgs_solver.py:6962-6990)."""
        if str(init_mode).lower().replace("-", "_") not in ("gs_cfcf", "soft_cfcf", "yi_soft", "cfcf", "curl_free_current"):
            raise NotImplementedError("the oracle restates the gs_cfcf and soft_cfcf starts")
        stop_mode = str(stop_mode).lower().replace("-", "_")
        if stop_mode not in ("sigma_best", "fixed_point"):
            raise ValueError("stop_mode must be 'sigma_best' or 'fixed_point'")
        if stop_mode == "fixed_point" and not self.record_iteration_diagnostics:
            raise ValueError("stop_mode='fixed_point' requires record_iteration_diagnostics=True")
        update_tol = float(tol if fixed_point_update_tol is None else fixed_point_update_tol)
        pde_tol = float(fixed_point_pde_tol)
        observable_tol = float(tol if fixed_point_observable_tol is None else fixed_point_observable_tol)
        fixed_required = int(fixed_point_patience)
        fp_streak = 0
        fp_converged = False
        diag_rows = []
        B, J, phi, az, Bc = self.compute_initial_conditions(init_mode)
        sigma0, divb0, e0 = self.compute_sigma(B, J), self.compute_divB(B), self.compute_energy(B)
        hist = {k: [] for k in ("sigma", "divB", "energy", "mu", "rollback", "sigma_relative_change",
                                "energy_relative_change", "fixed_point_criteria_met")}
        best_sigma, best_iter = sigma0, 0
        best = (B.copy(), J.copy(), phi.copy(), az.copy(), Bc.copy())
        stall = flat = streak = rollbacks = 0
        flat_req = max(int(patience), 1)
        mu_cur = float(mu)
        prev = sigma0
        use_imp = sigma_improvement_tol is not None and float(sigma_improvement_tol) > 0
        eps = float(sigma_improvement_tol) if use_imp else 0.0
        last_imp = None
        stop = "max_iter"
        final_iter = 0
        for n in range(1, max_iter + 1):
            Bn, Jn, phin, azn, Bcn = self.iteration_step(B, J, phi, az, Bc, mu=mu_cur, polarity_mask=polarity_mask)
            if self.record_iteration_diagnostics:
                diag_rows.append(dict(self.last_iteration_diagnostics))
            sigma = self.compute_sigma(Bn, Jn)
            diverged = (not math.isfinite(sigma)) or sigma > divergence_factor * max(best_sigma, 1e-30)
            if adaptive_mu and diverged:
                rollbacks += 1
                mu_cur = max(mu_cur * mu_backoff, mu_min)
                B, J, phi, az, Bc = (s.copy() for s in best)
                streak = 0
                hist["sigma"].append(sigma)
                hist["divB"].append(float("nan"))
                hist["energy"].append(float("nan"))
                hist["mu"].append(mu_cur)
                hist["rollback"].append(1)
                hist["sigma_relative_change"].append(float("nan"))
                hist["energy_relative_change"].append(float("nan"))
                hist["fixed_point_criteria_met"].append(0)
                fp_streak = 0
                if rollbacks >= max_rollbacks:
                    stop = "max_rollbacks"
                    break
                continue
            B, J, phi, az, Bc = Bn, Jn, phin, azn, Bcn
            divb, energy = self.compute_divB(B), self.compute_energy(B)
            src = abs(sigma - prev) / max(abs(prev), 1e-30)
            pe = hist["energy"][-1] if hist["energy"] else e0
            erc = abs(energy - pe) / max(abs(pe), 1e-30)
            hist["sigma"].append(sigma)
            hist["divB"].append(divb)
            hist["energy"].append(energy)
            hist["mu"].append(mu_cur)
            hist["rollback"].append(0)
            hist["sigma_relative_change"].append(src)
            hist["energy_relative_change"].append(erc)
            d = self.last_iteration_diagnostics if self.record_iteration_diagnostics else {}
            map_res = max(d.get("phi_map_residual_relative", math.inf), d.get("az_map_residual_relative", math.inf),
                          d.get("h_k0_map_residual_relative", 0.0))
            pde_res = max(d.get("poloidal_pde_residual_relative", math.inf),
                          d.get("toroidal_pde_residual_relative", math.inf), d.get("mixed_row_residual_relative", 0.0))
            met = (stop_mode == "fixed_point" and math.isfinite(map_res) and math.isfinite(pde_res)
                   and map_res <= update_tol and pde_res <= pde_tol and src <= observable_tol
                   and erc <= observable_tol)
            hist["fixed_point_criteria_met"].append(int(met))
            fp_streak = fp_streak + 1 if met else 0
            final_iter = n
            if per_step_callback is not None:
                per_step_callback(n, sigma, B, J)
            imp = prev - sigma
            last_imp = imp
            prev = sigma
            flat = flat + 1 if imp < eps else 0
            if sigma < best_sigma:
                best_sigma, best_iter = sigma, n
                best = (B.copy(), J.copy(), phi.copy(), az.copy(), Bc.copy())
                stall = 0
                streak += 1
                if adaptive_mu and streak >= growth_streak:
                    mu_cur = min(mu_cur * mu_growth, mu_max)
                    streak = 0
            else:
                stall += 1
                streak = 0
            if stop_mode == "fixed_point" and fp_streak >= fixed_required:
                stop = "fixed_point"
                fp_converged = True
                break
            if stop_mode == "sigma_best" and sigma < tol:
                stop = "tol"
                break
            if stop_mode == "sigma_best" and use_imp and flat >= flat_req:
                stop = "sigma_improvement_tol"
                break
            if stop_mode == "sigma_best" and patience > 0 and stall >= patience:
                stop = "sigma_stall"
                break
        final = (B, J, phi, az, Bc)
        sel = final if stop_mode == "fixed_point" else best
        self._B, self._J, self._Phi_c, self._Az = sel[0], sel[1], sel[2], sel[3]
        if self.k0 is not None:
            self.H = self.recover_h(sel[0], sel[4])
        fvb = math.sqrt(np.mean((final[0] - best[0]) ** 2)) / max(math.sqrt(np.mean(best[0] ** 2)), 1e-30)
        hist.update({
            "best_sigma": best_sigma, "best_iter": best_iter, "rollbacks": rollbacks,
            "stop_reason": stop, "stop_mode": stop_mode,
            "selected_state": "final_accepted_iterate" if stop_mode == "fixed_point" else "best_sigma",
            "final_iter": final_iter, "final_sigma": self.compute_sigma(final[0], final[1]),
            "final_vs_best_B_relative": fvb, "fixed_point_converged": fp_converged,
            "fixed_point_streak": fp_streak,
            "sigma_improvement_tol": eps if use_imp else None,
            "auto_rbsl_improvement_grace": 0, "last_sigma_improvement": last_imp,
            "source_partition_mode": "gaussian_separated",
            "bottom_current_grid_mode": self.bottom_current_grid_mode,
            "vertical_current_operator": "staggered_face",
            "sigma_placement": "vertical_faces",
            "initial_sigma": sigma0, "initial_divB": divb0, "initial_energy": e0,
        })
        if self.record_iteration_diagnostics:
            rows = diag_rows[:len(hist["sigma"])]
            for key in (sorted(rows[0]) if rows else []):
                hist[key] = [float(r[key]) for r in rows]
        hist["source_diagnostics"] = self.compute_source_diagnostics()
        return hist

    def compute_source_diagnostics(self):
        """Post-solve Robin/zero-mode diagnostics (nfgs_solver.py:7014-7196, scalar keys)."""
        B = self._B
        bcz = B[2] - self.B_background[2]
        recon = self.B_background[2, 0] + self.Bz_above - self.Bz_obs
        corr = bcz[0] - self.Bz_above
        dz = self.dz
        bc_hat = dct2(bcz)
        dh = (3.0 * bc_hat[-1] - 4.0 * bc_hat[-2] + bc_hat[-3]) / (2.0 * dz)
        rh = dh + self.k * bc_hat[-1]
        rh[0, 0] = 0.0
        phi = np.empty_like(bcz)
        phi[0] = self.Phi_above_bottom
        phi[1:] = self.poisson2d_neumann(bcz[1:])
        ph = dct2(phi)
        pdh = (3.0 * ph[-1] - 4.0 * ph[-2] + ph[-3]) / (2.0 * dz)
        prh = pdh + self.k * ph[-1]
        prh[0, 0] = 0.0
        ks = self.k.copy()
        ks[0, 0] = 1.0
        uh = 0.5 * (bc_hat[-1] + dh / ks)
        uh[0, 0] = 0.0
        up = idct2(uh)
        bdiv = d_dx(B[0, 0], self.dx) + d_dy(B[1, 0], self.dy)
        derr = bdiv - self.D0
        dphi_b = (-3.0 * phi[0] + 4.0 * phi[1] - phi[2]) / (2.0 * dz)
        return {
            "bottom_reconstruction_rms": _rms(recon),
            "bottom_reconstruction_max": float(np.abs(recon).max()),
            "correction_bottom_rms": _rms(corr),
            "top_robin_rms": _rms(idct2(rh)),
            "top_phi_robin_rms": _rms(idct2(prh)),
            "top_upward_source_rms": _rms(up),
            "top_upward_source_ratio": _rms(up) / max(_rms(bcz[-1]), 1e-30),
            "source_zero_mode_ratio_last": self.source_zero_mode_history[-1] if self.source_zero_mode_history else 0.0,
            "source_zero_mode_ratio_max": max(self.source_zero_mode_history) if self.source_zero_mode_history else 0.0,
            "bottom_divergence_rms": _rms(derr),
            "bottom_divergence_relative": _rms(derr) / max(_rms(self.D0), 1e-30),
            "bottom_dphi_residual_rms": _rms(dphi_b - self.bottom_dphi_c_target),
            **self.k0_source_diagnostics(),
        }

    def k0_source_diagnostics(self):
        """The closure's block with the selected state's H by height
        (nfgs_solver.py:7171-7196)."""
        if self.hzm not in ("coupled_k0", "frozen_linear_harmonic", "constrained_spline_harmonic"):
            return {}
        d = dict(self.k0_diagnostics)
        if self.H is not None:
            d["profile_by_height"] = [[float(v) for v in comp] for comp in self.H]
        return {self.hzm: d}

    def fields_to_numpy(self, crop_to_observed_fov=True):
        """nfgs_solver.py:2881-2903."""
        if self._B is None or self._J is None:
            raise RuntimeError("No solution stored; call iterate() first.")
        B, J = self._B, self._J
        if crop_to_observed_fov:
            nzo = self.observed_shape[0]
            sy, sx = self.fov
            B = B[:, :nzo, sy, sx]
            J = J[:, :nzo, sy, sx]
        return {"Bx": B[0].copy(), "By": B[1].copy(), "Bz": B[2].copy(),
                "Jx": J[0].copy(), "Jy": J[1].copy(), "Jz": J[2].copy()}

"""``NFGSSolverGPU``: drop-in host class for the NFGS reconstruction path.

Mirrors the public API of the reference ``nfgs_solver.NFGSSolverGPU``
(nfgs_solver.py:3905-7196 in spaceprod/NFGS): the constructor with its
policy keywords, ``set_bottom_vector_boundary`` / ``set_bottom_boundary``,
``iterate`` (gs_cfcf, cfcf or soft_cfcf start, sigma_best stop, optional adaptive mu) and
``fields_to_numpy``.  All numerical work runs in libnfgs_b200.so on the
GPU; this module only validates options, sizes the grid, places the
observed maps and assembles the ``history`` dictionary.

Options that select the reference's ablation branches (coupled k=0 modes,
two-stage poloidal update, collocated current, fixed-point stop mode with
per-iteration diagnostics) raise ``NotImplementedError``.
"""

from __future__ import annotations

import math
import warnings
from typing import Callable, Optional

import numpy as np

from . import _lib as L
from .grid import calculation_grid, pad_or_crop_center

__all__ = ["NFGSSolverGPU"]

_VALID_PROJECTION = {"error": 0, "warn_project": 1, "project": 2}
_VALID_HARMONIC = {"diagnose": 0, "warn": 1, "error": 2}
_POLARITY = {"both": 0, "positive": 1, "negative": 2}

# diag_out layout of nfgs_set_boundary (indices into the returned vector)
_DIAG = dict(mean_x=0, mean_y=1, mean_z=2, amean_x=3, amean_y=4, amean_z=5, open_bz=6, flux_imbalance=7,
             d0_mode=8, d0_ratio=9, recon_rms=10, recon_max=11, invariant_rms=12, harm_rms=13, harm_ratio=14,
             harm_cx=15, harm_cy=16, harm_const_rms=17, harm_nonconst_rms=18, harm_div_rms=19, harm_curl_rms=20,
             raw_jz_rms=21, t_jz_rms=22, raw_vs_t_rms=23, jz_mode=24, d0_warn=30, harm_warn=31)


def _dtype_code(dtype) -> tuple[int, np.dtype]:
    name = str(dtype).replace("torch.", "").lower()
    if name in ("float32", "float", "f4", "<f4", "single"):
        return L.NFGS_F32, np.dtype(np.float32)
    if name in ("float64", "double", "f8", "<f8"):
        return L.NFGS_F64, np.dtype(np.float64)
    raise ValueError(f"dtype must be float32 or float64; got {dtype!r}")


def _check_device(device) -> None:
    if hasattr(device, "type") and hasattr(device, "index"):  # torch.device
        device = f"{device.type}:{device.index}" if device.index is not None else device.type
    name = str(device)
    if not name.startswith("cuda"):
        raise ValueError(
            f"NFGSSolverGPU (B200 build) runs on CUDA only; got device={device!r}. There is no CPU path."
        )


def _as_plane(a, nz: int, name: str) -> np.ndarray:
    """Bottom map from a (Ny, Nx) map or an (Nz, Ny, Nx) volume (nfgs_solver.py:1485-1496)."""
    if hasattr(a, "detach"):
        a = a.detach().cpu().numpy()
    a = np.asarray(a)
    if a.ndim == 2:
        return a
    if a.ndim == 3:
        if int(a.shape[0]) != nz:
            raise ValueError(f"{name} 3D input must be in (Nz, Ny, Nx) order with Nz={nz}; got {tuple(a.shape)}.")
        return a[0]
    raise ValueError(f"{name} must be 2D (Ny, Nx) or 3D (Nz, Ny, Nx); got {tuple(a.shape)}.")


class NFGSSolverGPU:
    """Gaussian-separated NFPT solver on one B200 (reference nfgs_solver.py:3905)."""

    def __init__(self, Nx, Ny, Nz, dx, dy, dz, device="cuda", *, dtype="float64", **kwargs):
        _check_device(device)
        kw = dict(kwargs)
        pop = kw.pop
        # --- NFGS policy keywords (nfgs_solver.py:3925-4349)
        source_partition_mode = str(pop("source_partition_mode", "gaussian_separated")).lower().replace("-", "_")
        weak_floor = float(pop("weak_field_floor_b2", 1.0e-20))
        alpha_clip_scale = pop("alpha_clip_scale", None)
        if alpha_clip_scale is not None:
            alpha_clip_scale = float(alpha_clip_scale)
            if "alpha_limit_factor" in kw and float(kw["alpha_limit_factor"]) != alpha_clip_scale:
                raise ValueError("alpha_clip_scale and alpha_limit_factor specify different values")
            kw["alpha_limit_factor"] = alpha_clip_scale
        mean_bz_policy = str(pop("mean_bz_policy", "uniform_open")).lower()
        hzm = str(pop("horizontal_zero_mode_policy", "frozen_linear_harmonic")).lower()
        d0_policy = str(pop("d0_zero_mode_policy", "error")).lower()
        harm_policy = str(pop("harmonic_residual_policy", "diagnose")).lower()
        src_policy = str(pop("source_zero_mode_policy", "error")).lower()
        handoff = str(pop("handoff_projection_policy", "project")).lower()
        mean_tol = float(pop("mean_mode_tolerance", 1.0e-6))
        src_tol = float(pop("source_zero_mode_tolerance", 1.0e-2))
        k0_smooth = float(pop("k0_ode_smoothness", 1.0e-3))
        k0_disc = str(pop("coupled_k0_discretization", "staggered_face_D1_true_three_point_curvature")).lower().replace("-", "_")
        k0_mu = pop("k0_update_mu", None)
        k0_basis = int(pop("k0_spline_basis_size", 8))
        k0_place = pop("k0_current_target_placement", None)
        bpcm = str(pop("bottom_parallel_current_mode", "observed_full")).lower().replace("-", "_")
        handoff_tol = float(pop("handoff_projection_tolerance", 1.0e-6))
        proj_w = float(pop("bottom_divergence_projection_weight", 0.0))
        rho = float(pop("bottom_divergence_robin_weight", 0.0))
        pum = str(pop("poloidal_update_mode", "direct")).lower().replace("-", "_")
        record = bool(pop("record_iteration_diagnostics", False))
        soft_eps = pop("soft_cfcf_epsilon", None)
        soft_bs = int(pop("soft_cfcf_mode_batch_size", 1024))
        soft_ridge = float(pop("soft_cfcf_normal_ridge", 0.0))
        user_open = pop("user_supplied_open_bz", None)
        user_h = pop("user_supplied_horizontal_field", None)
        external = pop("external_potential_field", None)
        pzo = int(pop("poisson_z_order", 2))
        pzb = str(pop("poisson_z_backend", "thomas")).lower()
        ccu = bool(pop("ccu_pure_current", True))
        t_source = str(pop("t_source", "jz")).lower()
        toroidal = bool(pop("toroidal_boundary", True))
        mudpack_like = bool(pop("poisson_mudpack_like", True))
        pxo = int(pop("poisson_xy_order", 2))
        bjt00 = bool(pop("fortran_bjt00", False))
        phi_total = bool(pop("fortran_phi_total_solve", False))
        ghop = str(pop("gaussian_horizontal_operator", "spectral")).lower()
        vco = str(pop("vertical_current_operator", "staggered_face")).lower().replace("-", "_")
        if pzo != 2:
            raise ValueError("NFGS v1 supports only poisson_z_order=2 for the top Robin solve")
        if pzb != "thomas":
            raise ValueError("NFGS v1 supports only poisson_z_backend='thomas'")
        if pxo != 2:
            raise ValueError("NFGS v1 supports only poisson_xy_order=2")
        if not mudpack_like:
            raise ValueError("NFGS requires poisson_mudpack_like=True so separation and 2-D Poisson use the same "
                             "endpoint-Neumann spectrum")
        if not ccu:
            raise ValueError("NFGS requires ccu_pure_current=True")
        if t_source != "jz":
            raise ValueError("NFGS v1 supports only t_source='jz'")
        if not toroidal:
            raise ValueError("NFGS v1 requires toroidal_boundary=True")
        if bjt00:
            raise ValueError("NFGS requires fortran_bjt00=False to preserve explicit mean modes")
        if phi_total:
            raise ValueError("NFGS requires fortran_phi_total_solve=False")
        valid_mean = {"uniform_open", "require_balanced", "external_potential", "user_supplied"}
        valid_h = {"omit", "frozen_linear_harmonic", "constrained_spline_harmonic", "coupled_k0",
                   "external_potential", "user_supplied"}
        if source_partition_mode not in {"gaussian_separated", "legacy_single_field"}:
            raise ValueError("source_partition_mode must be 'gaussian_separated' or 'legacy_single_field'")
        if weak_floor <= 0.0 or not math.isfinite(weak_floor):
            raise ValueError("weak_field_floor_b2 must be finite and positive")
        if mean_bz_policy not in valid_mean:
            raise ValueError(f"mean_bz_policy must be one of {sorted(valid_mean)}")
        if hzm not in valid_h:
            raise ValueError(f"horizontal_zero_mode_policy must be one of {sorted(valid_h)}")
        if d0_policy not in _VALID_PROJECTION:
            raise ValueError(f"d0_zero_mode_policy must be one of {sorted(_VALID_PROJECTION)}")
        if src_policy not in _VALID_PROJECTION:
            raise ValueError(f"source_zero_mode_policy must be one of {sorted(_VALID_PROJECTION)}")
        if harm_policy not in _VALID_HARMONIC:
            raise ValueError("harmonic_residual_policy must be 'diagnose', 'warn', or 'error'")
        if handoff not in {"project", "error"}:
            raise ValueError("handoff_projection_policy must be 'project' or 'error'")
        if mean_tol <= 0.0 or src_tol <= 0.0:
            raise ValueError("zero-mode tolerances must be positive")
        if k0_smooth < 0.0:
            raise ValueError("k0_ode_smoothness must be non-negative")
        if k0_disc not in {"staggered_face_d1_true_three_point_curvature", "legacy_plane_centred"}:
            raise ValueError("coupled_k0_discretization is not recognised")
        if k0_mu is not None and not 0.0 < float(k0_mu) <= 1.0:
            raise ValueError("k0_update_mu must be in (0, 1]")
        if k0_basis < 4:
            raise ValueError("k0_spline_basis_size must be >= 4")
        if k0_mu is None and hzm == "constrained_spline_harmonic":
            k0_mu = 0.2  # the closure's own conservative default (nfgs_solver.py:4141-4146)
        k0_place = "cell" if k0_place is None else str(k0_place).lower().replace("-", "_")
        if k0_place not in {"face", "cell"}:
            raise ValueError("k0_current_target_placement must be 'face' or 'cell'")
        if k0_place == "face" and vco != "staggered_face":
            raise ValueError("k0_current_target_placement='face' requires vertical_current_operator='staggered_face'")
        if bpcm not in {"observed_full", "face_parallel_exact_jz"}:
            raise ValueError("bottom_parallel_current_mode must be one of ['face_parallel_exact_jz', 'observed_full']")
        if handoff_tol <= 0.0:
            raise ValueError("handoff_projection_tolerance must be positive")
        if not 0.0 <= proj_w <= 1.0:
            raise ValueError("bottom_divergence_projection_weight must be between 0 and 1")
        if not 0.0 <= rho <= 1.0:
            raise ValueError("bottom_divergence_robin_weight must be between 0 and 1")
        if proj_w > 0.0 and rho > 0.0:
            raise ValueError("Bottom-divergence projection and mixed Robin controls are mutually exclusive")
        if pum not in {"direct", "two_stage"}:
            raise ValueError("poloidal_update_mode must be 'direct' or 'two_stage'")
        if soft_eps is not None and float(soft_eps) < 0.0:
            raise ValueError("soft_cfcf_epsilon must be non-negative")
        if soft_bs <= 0:
            raise ValueError("soft_cfcf_mode_batch_size must be positive")
        if soft_ridge < 0.0:
            raise ValueError("soft_cfcf_normal_ridge must be non-negative")
        if ghop not in {"fd", "spectral"}:
            raise ValueError("gaussian_horizontal_operator must be one of ['fd', 'spectral']")
        if vco not in {"staggered_face", "collocated_centered"}:
            raise ValueError("vertical_current_operator must be one of ['collocated_centered', 'staggered_face']")
        # branches outside the production NFGS path
        unsupported = []
        if source_partition_mode != "gaussian_separated":
            unsupported.append("source_partition_mode='legacy_single_field'")
        if hzm not in {"omit", "frozen_linear_harmonic", "coupled_k0", "constrained_spline_harmonic"}:
            unsupported.append(f"horizontal_zero_mode_policy={hzm!r}")
        if mean_bz_policy == "external_potential" or external is not None:
            unsupported.append("external_potential_field")
        if user_h is not None:
            unsupported.append("user_supplied_horizontal_field")
        if pum != "direct":
            unsupported.append("poloidal_update_mode='two_stage'")
        if vco != "staggered_face":
            unsupported.append("vertical_current_operator='collocated_centered'")
        # --- Stable-NFPT / base keywords (nfgs_solver.py:2910-2965, 736-937)
        alpha_limit_factor = kw.pop("alpha_limit_factor", 1.0)
        bottom_jperp_zero = bool(kw.pop("bottom_jperp_zero", True))
        relax_scalars = bool(kw.pop("relax_scalars", True))
        t_filter = float(kw.pop("t_filter_scale", 0.0))
        imprint = float(kw.pop("bottom_imprint_robin_weight", 0.0))
        buffer_thickness = kw.pop("buffer_thickness", None)
        pin = bool(kw.pop("pin_potential_boundaries", False))
        lateral_wall = str(kw.pop("lateral_wall", "paper_bc1")).lower().replace("-", "_")
        padded_buffer_zone = bool(kw.pop("padded_buffer_zone", True))
        pad_calc = kw.pop("pad_calculation_domain", True)
        calc_mode = str(kw.pop("calculation_domain_mode", "mudpack")).lower().replace("-", "_")
        buffer_xy_only = bool(kw.pop("buffer_xy_only", False))
        rhs_lap = str(kw.pop("rhs_lap_xy", "fd")).lower()
        rhs_ext = str(kw.pop("rhs_lap_xy_spectral_ext", "neumann")).lower()
        rhs_div_chain = bool(kw.pop("rhs_jz_div_chain", False))
        kw.pop("lap_phi_z_boundary_mean", False)
        fdo = int(kw.pop("finite_difference_order", 2))
        for key in ("poisson_2d_interior_rhs_only", "poisson_2d_endpoint_dirichlet",
                    "poisson_3d_endpoint_neumann_xy", "poisson_3d_top_neumann_one_sided",
                    "fortran_iphiws3_potential"):
            kw.pop(key, None)
        if kw:
            raise TypeError(f"unexpected keyword arguments: {sorted(kw)}")
        if fdo not in (2, 4):
            raise ValueError("finite_difference_order must be 2 or 4")
        if lateral_wall not in {"bc1", "paper_bc1", "paper", "potential_pin", "legacy_potential_pin",
                                "potentialpin", "pin", "legacy"}:
            raise ValueError("lateral_wall must be one of: 'potential_pin', 'legacy_potential_pin', 'BC1', "
                             f"'paper_bc1', 'paper'; got {lateral_wall!r}")
        # wall condition of the Stable-NFPT field behind the cfcf start
        self._lateral_bc1 = lateral_wall in {"bc1", "paper_bc1", "paper"}
        self.handoff_projection_policy = handoff
        self.handoff_projection_tolerance = handoff_tol
        if rhs_lap not in ("fd", "spectral"):
            raise ValueError("rhs_lap_xy must be 'fd' or 'spectral'")
        if rhs_ext not in ("neumann", "dirichlet"):
            raise ValueError("rhs_lap_xy_spectral_ext must be 'neumann' or 'dirichlet'")
        if not 0.0 <= imprint <= 1.0:
            raise ValueError("bottom_imprint_robin_weight must be between 0 and 1")
        # k_h=0 closure checks that follow the base initialiser (nfgs_solver.py:4252-4270)
        if hzm in {"coupled_k0", "constrained_spline_harmonic"} and not relax_scalars:
            raise ValueError("coupled horizontal harmonic modes require relax_scalars=True")
        if hzm == "constrained_spline_harmonic" and vco != "staggered_face":
            raise ValueError("constrained_spline_harmonic requires vertical_current_operator='staggered_face'")
        if fdo != 2:
            unsupported.append("finite_difference_order=4")
        if rhs_lap != "fd":
            unsupported.append("rhs_lap_xy='spectral'")
        if rhs_div_chain:
            unsupported.append("rhs_jz_div_chain=True")
        if not bottom_jperp_zero:
            unsupported.append("bottom_jperp_zero=False")
        if not relax_scalars:
            unsupported.append("relax_scalars=False")
        if t_filter > 0.0:
            unsupported.append("t_filter_scale > 0")
        if imprint > 0.0:
            unsupported.append("bottom_imprint_robin_weight > 0")
        if unsupported:
            raise NotImplementedError(
                "outside the production NFGS branch built for B200: " + ", ".join(unsupported))
        del pin
        # --- grid (nfgs_solver.py:771-819)
        g = calculation_grid(int(Nx), int(Ny), int(Nz), pad_calculation_domain=pad_calc,
                             calculation_domain_mode=calc_mode, padded_buffer_zone=padded_buffer_zone)
        self.Nx, self.Ny, self.Nz = g["nx"], g["ny"], g["nz"]
        self._input_shape_zyx = (int(Nz), int(Ny), int(Nx))
        self._calculation_pad_xy = g["pad_xy"]
        self._calculation_domain_mode = calc_mode
        self.dx, self.dy, self.dz = float(dx), float(dy), float(dz)
        if self.Nz < 3:
            raise ValueError("NFGS requires Nz >= 3")
        if hzm == "constrained_spline_harmonic" and k0_basis > self.Nz:
            raise ValueError("k0_spline_basis_size must not exceed Nz")
        if hzm == "constrained_spline_harmonic" and k0_disc == "legacy_plane_centred":
            # the reference's centre derivative of this combination has no
            # operator (nfgs_solver.py:5406-5411)
            raise RuntimeError("legacy coupled_k0 operator is not initialized")
        self.k0_ode_smoothness = k0_smooth
        self.coupled_k0_discretization = ("staggered_face_D1_true_three_point_curvature"
                                          if k0_disc == "staggered_face_d1_true_three_point_curvature" else k0_disc)
        self.k0_update_mu = None if k0_mu is None else float(k0_mu)
        self.k0_spline_basis_size = k0_basis
        self.k0_current_target_placement = k0_place
        self.device = str(device)
        self._dtype_code, self._np_dtype = _dtype_code(dtype)
        self.dtype = dtype
        self._padded_buffer_zone = padded_buffer_zone
        self._alpha_limit_factor = None if alpha_limit_factor is None else float(alpha_limit_factor)
        self.alpha_clip_scale = self._alpha_limit_factor
        self.bottom_divergence_robin_weight = rho
        self.bottom_divergence_projection_weight = proj_w
        self.horizontal_zero_mode_policy = hzm
        self.mean_bz_policy = mean_bz_policy
        self.d0_zero_mode_policy = d0_policy
        self.source_zero_mode_policy = src_policy
        self.harmonic_residual_policy = harm_policy
        self.mean_mode_tolerance = mean_tol
        self.source_zero_mode_tolerance = src_tol
        self.weak_field_floor_b2 = weak_floor
        self.gaussian_horizontal_operator = ghop
        self.vertical_current_operator = vco
        self.source_partition_mode = source_partition_mode
        self.bottom_parallel_current_mode = bpcm
        self.poloidal_update_mode = pum
        self.record_iteration_diagnostics = record
        self.buffer_thickness = 0 if buffer_thickness is None else int(buffer_thickness)
        # nfgs_solver.py:4299-4305 (the batch size is recorded only: the
        # device solves every mode in one pass)
        grid_scale = min(self.dx, self.dy, self.dz)
        self.soft_cfcf_epsilon = 1.0e-4 / (grid_scale * grid_scale) if soft_eps is None else float(soft_eps)
        self.soft_cfcf_mode_batch_size = soft_bs
        self.soft_cfcf_normal_ridge = soft_ridge
        self._init_diagnostics = None
        self.fov_slice_yx = None
        self._observed_shape_zyx = None
        self._bottom_current_grid_mode = None
        self.gaussian_separation_diagnostics = None
        self.toroidal_boundary_diagnostics = None
        self._source_zero_mode_history: list[float] = []
        self._have_solution = False
        self._lib = L.lib()
        am = self.alpha_max()
        dev = str(device)
        self._device_index = int(dev.split(":")[1]) if ":" in dev else 0
        geom = L.NfgsGeom(self.Nx, self.Ny, self.Nz, self.dx, self.dy, self.dz, int(Nx), int(Ny), int(Nz),
                          g["pad_xy"][0], g["pad_xy"][1], self._dtype_code, self._device_index)
        prm = L.NfgsParams(
            robin_weight=rho, projection_weight=proj_w,
            alpha_max=(am if (am is not None and math.isfinite(am)) else -1.0),
            weak_field_floor_b2=weak_floor, mean_mode_tolerance=mean_tol,
            source_zero_mode_tolerance=src_tol,
            user_open_bz=float(np.asarray(user_open).reshape(())) if user_open is not None else 0.0,
            horizontal_zero_mode={"frozen_linear_harmonic": 1, "coupled_k0": 2,
                                  "constrained_spline_harmonic": 3}.get(hzm, 0),
            mean_bz_policy={"uniform_open": 0, "require_balanced": 1, "user_supplied": 2}[mean_bz_policy],
            d0_policy=_VALID_PROJECTION[d0_policy], source_policy=_VALID_PROJECTION[src_policy],
            harmonic_policy=_VALID_HARMONIC[harm_policy], gaussian_spectral=1 if ghop == "spectral" else 0,
            face_parallel_exact_jz=1 if bpcm == "face_parallel_exact_jz" else 0,
            buffer_thickness=self.buffer_thickness, buffer_xy_only=int(buffer_xy_only),
            k0_smoothness=k0_smooth, k0_update_mu=(-1.0 if k0_mu is None else float(k0_mu)),
            k0_spline_basis=k0_basis, k0_legacy=int(k0_disc == "legacy_plane_centred"),
            k0_face_target=int(k0_place == "face"))
        if mean_bz_policy == "user_supplied" and user_open is None:
            self._user_open_missing = True
        else:
            self._user_open_missing = False
        h = L.C.c_void_p()
        L.check(self._lib.nfgs_create(L.C.byref(geom), L.C.byref(prm), L.C.byref(h)))
        self._h = h

    # ------------------------------------------------------------------
    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._lib.nfgs_destroy(h)
            except Exception:
                pass
            self._h = None

    def alpha_max(self) -> Optional[float]:
        """|alpha| bound alpha_limit_factor / min(dx, dy, dz) (nfgs_solver.py:2970-2975)."""
        if self._alpha_limit_factor is None:
            return None
        return self._alpha_limit_factor / min(self.dx, self.dy, self.dz)

    # ------------------------------------------------------------------
    # Boundary (nfgs_solver.py:4548-4596, 4661)
    # ------------------------------------------------------------------
    def set_bottom_vector_boundary(self, Bx_obs, By_obs, Bz_obs, **kwargs):
        """Set NFGS from vector magnetogram maps in (Ny, Nx) order."""
        return self.set_bottom_boundary(Bz_obs=Bz_obs, Jz_obs=None, Bx_obs=Bx_obs, By_obs=By_obs, **kwargs)

    def set_bottom_boundary(self, Bz_obs, Jz_obs=None, zero_net_current=None, *, Bx_obs=None, By_obs=None,
                            smooth_passes=None, padded_buffer_zone=None, ijzbcor: int = 3):
        if Bx_obs is None or By_obs is None:
            raise ValueError("NFGS requires Bx_obs and By_obs; use set_bottom_vector_boundary() "
                             "or pass both tangential components to set_bottom_boundary().")
        if self._user_open_missing:
            raise ValueError("user_supplied_open_bz is required for mean_bz_policy='user_supplied'")
        bz = _as_plane(Bz_obs, self.Nz, "Bz_obs")
        bx = _as_plane(Bx_obs, self.Nz, "Bx_obs")
        by = _as_plane(By_obs, self.Nz, "By_obs")
        derived = Jz_obs is None
        jz = None if derived else _as_plane(Jz_obs, self.Nz, "Jz_obs")
        if zero_net_current is None:
            zero_net_current = not derived
        if smooth_passes is None:
            smooth_passes = 0 if derived else 3
        if bz.ndim != 2 or (jz is not None and jz.ndim != 2):
            raise ValueError("Bz_obs/Jz_obs must be 2D.")
        if bx.shape != bz.shape or by.shape != bz.shape:
            raise ValueError("Bx_obs/By_obs must have the same observed-FOV shape as Bz_obs. "
                             f"Got Bx={bx.shape}, By={by.shape}, Bz={bz.shape}.")
        if jz is not None and jz.shape != bz.shape:
            raise ValueError("Jz_obs must have the same shape as Bz_obs")
        use_pad = self._padded_buffer_zone if padded_buffer_zone is None else bool(padded_buffer_zone)
        oy, ox = int(bz.shape[0]), int(bz.shape[1])
        if (oy, ox) != (self.Ny, self.Nx):
            if not use_pad:
                raise ValueError(f"Bz_obs/Jz_obs must have shape ({self.Ny}, {self.Nx}); got {bz.shape}.")
            place = pad_or_crop_center(oy, ox, self.Ny, self.Nx)
            self.fov_slice_yx = (slice(place["dy0"], place["dy0"] + place["cny"]),
                                 slice(place["dx0"], place["dx0"] + place["cnx"]))
            self._observed_shape_zyx = (min(self.Nz, self._input_shape_zyx[0]), oy, ox)
        else:
            place = dict(dy0=0, dx0=0, sy0=0, sx0=0, cny=self.Ny, cnx=self.Nx)
            self.fov_slice_yx = (slice(0, self.Ny), slice(0, self.Nx))
            self._observed_shape_zyx = (self.Nz, self.Ny, self.Nx)
        if derived:
            calc = (self.Nz, self.Ny, self.Nx)
            padded = any(c > o for c, o in zip(calc, self._input_shape_zyx)) or \
                any(c > o for c, o in zip(calc, self._observed_shape_zyx)) or \
                any(p > 0 for p in self._calculation_pad_xy)
            jz_mode = 0 if padded else 1
            self._bottom_current_grid_mode = "legacy_helper" if padded else "calculation_grid"
        else:
            jz_mode = 2
            self._bottom_current_grid_mode = "provided"
        opts = L.NfgsBoundaryOpts(
            ny_obs=oy, nx_obs=ox, zero_net_current=int(bool(zero_net_current)), smooth_passes=int(smooth_passes),
            ijzbcor=int(ijzbcor), jz_mode=jz_mode, nzo=int(self._observed_shape_zyx[0]),
            fov_y0=place["dy0"], fov_x0=place["dx0"], src_y0=place["sy0"], src_x0=place["sx0"],
            copy_ny=place["cny"], copy_nx=place["cnx"])
        arrs = [np.ascontiguousarray(np.asarray(a, dtype=np.float64)) for a in (bx, by, bz)]
        jza = np.ascontiguousarray(np.asarray(jz, dtype=np.float64)) if jz is not None else None
        diag = np.zeros(L.NFGS_NDIAG)
        self._have_solution = False
        L.check(self._lib.nfgs_set_boundary(self._h, L.dptr(arrs[0]), L.dptr(arrs[1]), L.dptr(arrs[2]),
                                            L.dptr(jza) if jza is not None else None, L.C.byref(opts),
                                            L.dptr(diag)))
        self._diag = diag
        d = _DIAG
        if diag[d["d0_warn"]]:
            warnings.warn(
                "The bottom vector field is incompatible with the zero-mean endpoint-Neumann GS model "
                f"ratio={diag[d['d0_ratio']]:.6e} exceeds tolerance={self.mean_mode_tolerance:.6e}. "
                "The incompatible zero mode will be projected out.", RuntimeWarning, stacklevel=2)
        if diag[d["harm_warn"]]:
            warnings.warn(
                "Bottom horizontal reconstruction leaves a finite-domain harmonic residual "
                f"ratio={diag[d['harm_ratio']]:.6e}, tolerance={self.mean_mode_tolerance:.6e}.",
                RuntimeWarning, stacklevel=2)
        self.toroidal_boundary_diagnostics = {
            "t_source": "jz", "t_filter_scale": 0.0, "raw_jz_rms": float(diag[d["raw_jz_rms"]]),
            "t_implied_jz_rms": float(diag[d["t_jz_rms"]]), "raw_vs_t_implied_jz_rms": float(diag[d["raw_vs_t_rms"]]),
        }
        mean = [float(diag[d["mean_x"]]), float(diag[d["mean_y"]]), float(diag[d["mean_z"]])]
        gsd = {
            "bottom_reconstruction_rms": float(diag[d["recon_rms"]]),
            "bottom_reconstruction_max": float(diag[d["recon_max"]]),
            "mean_field": mean,
            "dct_zero_mode_Bx": mean[0], "dct_zero_mode_By": mean[1], "dct_zero_mode_Bz": mean[2],
            "arithmetic_mean_B": [float(diag[d["amean_x"]]), float(diag[d["amean_y"]]), float(diag[d["amean_z"]])],
            "mean_bz_policy": self.mean_bz_policy,
            "horizontal_zero_mode_policy": self.horizontal_zero_mode_policy,
            "gaussian_horizontal_operator": self.gaussian_horizontal_operator,
            "Bz_open_mean": float(diag[d["open_bz"]]),
            "Bh_mean_bottom": mean[:2],
            "flux_imbalance_fraction": float(diag[d["flux_imbalance"]]),
            "D0_zero_mode": float(diag[d["d0_mode"]]),
            "D0_zero_mode_ratio": float(diag[d["d0_ratio"]]),
            "d0_removed_constant_mode": float(diag[d["d0_mode"]]),
            "background_scalar_plus_explicit_rms": float(diag[d["invariant_rms"]]),
            "bottom_horizontal_reconstruction_rms": float(diag[d["harm_rms"]]),
            "bottom_horizontal_reconstruction_ratio": float(diag[d["harm_ratio"]]),
            "harmonic_residual_constant": [float(diag[d["harm_cx"]]), float(diag[d["harm_cy"]])],
            "harmonic_residual_constant_rms": float(diag[d["harm_const_rms"]]),
            "harmonic_residual_nonconstant_rms": float(diag[d["harm_nonconst_rms"]]),
            "harmonic_residual_divergence_rms": float(diag[d["harm_div_rms"]]),
            "harmonic_residual_curl_rms": float(diag[d["harm_curl_rms"]]),
        }
        self.gaussian_separation_diagnostics = gsd
        target = [float(v) for v in gsd["harmonic_residual_constant"]]
        hzm = self.horizontal_zero_mode_policy
        if hzm == "frozen_linear_harmonic":
            self._k0_diagnostics = {
                "enabled": True, "closure": "frozen_linear_harmonic",
                "representation": "analytic_Az_linear_lift", "bottom_target": list(target),
                "current_free": True, "open_side_current": False, "top_derivative": [0.0, 0.0],
                "profile_max_abs": float(max(abs(target[0]), abs(target[1]))),
            }
        elif hzm == "coupled_k0":
            # nfgs_solver.py:5296-5310, 5347-5358
            legacy = self.coupled_k0_discretization == "legacy_plane_centred"
            self._k0_diagnostics = {"enabled": True, "smoothness": self.k0_ode_smoothness,
                                    "discretization": self.coupled_k0_discretization,
                                    "bottom_target": list(target), "open_side_current": True}
            if legacy:
                self._k0_diagnostics["diagnosis_only"] = True
        elif hzm == "constrained_spline_harmonic":
            # nfgs_solver.py:5209-5225
            st = self._k0_state()
            self._k0_diagnostics = {
                "enabled": True, "closure": "constrained_spline_harmonic",
                "representation": "cubic_bspline_explicit_linear_harmonic_lift",
                "basis_size": self.k0_spline_basis_size, "smoothness": self.k0_ode_smoothness,
                "update_mu": self.k0_update_mu, "bottom_target": list(target), "bottom_constraint": "exact",
                "top_constraint": "discrete_second_order_Hprime_zero",
                "lateral_current_contract": "open_harmonic_plus_closed_PT", "open_side_current": True,
                "top_derivative": [0.0, 0.0], "kkt_condition_number": st["kkt_condition_number"]}
        else:
            self._k0_diagnostics = {}
        self._source_zero_mode_history = []
        return None

    # ------------------------------------------------------------------
    # Boundary products (device -> host copies on demand)
    # ------------------------------------------------------------------
    def _plane(self, which: int) -> np.ndarray:
        out = np.empty((self.Ny, self.Nx))
        L.check(self._lib.nfgs_get_plane(self._h, which, L.dptr(out)))
        return out

    @property
    def Bz_obs(self):
        return self._plane(0)

    @property
    def Bx_obs(self):
        return self._plane(1)

    @property
    def By_obs(self):
        return self._plane(2)

    @property
    def Jz_obs(self):
        return self._plane(3)

    @property
    def Az_bottom(self):
        return self._plane(4)

    @property
    def Jz_toroidal_boundary(self):
        return self._plane(5)

    @property
    def Phi_above_bottom(self):
        return self._plane(6)

    @property
    def Bz_above(self):
        return self._plane(7)

    @property
    def D0(self):
        return self._plane(8)

    @property
    def bottom_dphi_c_target(self):
        return self._plane(9)

    @property
    def B_background(self):
        out = np.empty((3, self.Nz, self.Ny, self.Nx))
        L.check(self._lib.nfgs_get_background(self._h, L.dptr(out)))
        return out

    @property
    def _H_k0_bottom_target(self):
        d = _DIAG
        return np.array([self._diag[d["harm_cx"]], self._diag[d["harm_cy"]]])

    def gaussian_above_bottom_field(self) -> np.ndarray:
        """B^> on z = 0, shape (3, Ny, Nx) (nfgs_solver.py:4921-4946)."""
        out = np.empty((3, self.Ny, self.Nx))
        L.check(self._lib.nfgs_gaussian_above(self._h, L.dptr(out)))
        return out

    # ------------------------------------------------------------------
    # Iteration (nfgs_solver.py:6937-7009 -> 3522-3850)
    # ------------------------------------------------------------------
    def compute_initial_conditions(self, *, init_mode="gs_cfcf", **_unused):
        """The start state of `init_mode` (gs_cfcf, nfgs_solver.py:6613-6645;
        cfcf, 6080-6147; soft_cfcf, 6427-6484) as host arrays (B, J, Phi_c, A_z, B_c) on the
        calculation grid, B_c = B - B_background.  It is built on the device
        as iterate() builds it; until the next iterate(), fields_to_numpy()
        returns this state."""
        mode = str(init_mode).lower().replace("-", "_")
        if mode == "learned":
            raise ValueError("NFGS supports init_mode='gs_cfcf', 'cfcf', or 'soft_cfcf'")
        ctx = self._iterate_begin(max_iter=0, verbose=False, init_mode=init_mode)
        self._iterate_finish(ctx)  # no step: the start is the current and the selected state
        B, J = self._state_fields(which=1)
        phi, az, _ = self._get_state(1)
        dt = self._np_dtype
        return B, J, phi.astype(dt), az.astype(dt), (B - self.B_background).astype(dt)

    def iterate(self, max_iter=200, tol=1e-5, mu=1.0, patience=1, verbose=True, polarity_mask="both", *,
                init_mode="gs_cfcf", sigma_improvement_tol: Optional[float] = 1e-5,
                per_step_callback: Optional[Callable] = None, adaptive_mu: bool = False, mu_min: float = 0.02,
                mu_max: float = 1.0, mu_backoff: float = 0.5, mu_growth: float = 1.1, growth_streak: int = 5,
                divergence_factor: float = 2.0, max_rollbacks: int = 12, stop_mode: str = "sigma_best",
                fixed_point_update_tol=None, fixed_point_pde_tol: float = 1.0e-8,
                fixed_point_observable_tol=None, fixed_point_patience: int = 10,
                auto_rbsl_improvement_grace: int = 20, check_every: int = 32, use_graph: bool = True,
                warm_start=None, **_auto_rbsl_kwargs):
        """Run the NFGS iteration to its stop rule (nfgs_solver.py:6937-7009 ->
        3522-3850) and return the reference's history dict."""
        ctx = self._iterate_begin(
            max_iter=max_iter, tol=tol, mu=mu, patience=patience, verbose=verbose, polarity_mask=polarity_mask,
            init_mode=init_mode, sigma_improvement_tol=sigma_improvement_tol, per_step_callback=per_step_callback,
            adaptive_mu=adaptive_mu, mu_min=mu_min, mu_max=mu_max, mu_backoff=mu_backoff, mu_growth=mu_growth,
            growth_streak=growth_streak, divergence_factor=divergence_factor, max_rollbacks=max_rollbacks,
            stop_mode=stop_mode, fixed_point_update_tol=fixed_point_update_tol,
            fixed_point_pde_tol=fixed_point_pde_tol, fixed_point_observable_tol=fixed_point_observable_tol,
            fixed_point_patience=fixed_point_patience, auto_rbsl_improvement_grace=auto_rbsl_improvement_grace,
            check_every=check_every, use_graph=use_graph, warm_start=warm_start, **_auto_rbsl_kwargs)
        self._iterate_loop(ctx)
        return self._iterate_finish(ctx)

    def _iterate_begin(self, max_iter=200, tol=1e-5, mu=1.0, patience=1, verbose=True, polarity_mask="both", *,
                init_mode="gs_cfcf", sigma_improvement_tol: Optional[float] = 1e-5,
                per_step_callback: Optional[Callable] = None, adaptive_mu: bool = False, mu_min: float = 0.02,
                mu_max: float = 1.0, mu_backoff: float = 0.5, mu_growth: float = 1.1, growth_streak: int = 5,
                divergence_factor: float = 2.0, max_rollbacks: int = 12, stop_mode: str = "sigma_best",
                fixed_point_update_tol=None, fixed_point_pde_tol: float = 1.0e-8,
                fixed_point_observable_tol=None, fixed_point_patience: int = 10,
                auto_rbsl_improvement_grace: int = 20, check_every: int = 32, use_graph: bool = True,
                warm_start=None, **_auto_rbsl_kwargs):
        mode = str(init_mode).lower().replace("-", "_")
        if mode == "yi_soft":
            mode = "soft_cfcf"
        if mode not in ("gs_cfcf", "cfcf", "curl_free_current", "soft_cfcf", "learned"):
            raise ValueError("NFGS supports init_mode='gs_cfcf', 'cfcf', or 'soft_cfcf'")
        if mode == "learned" and warm_start is None:
            raise ValueError("init_mode='learned' needs warm_start (a learned.NeuralOperator or a callable)")
        stop_mode = str(stop_mode).lower().replace("-", "_")
        if stop_mode == "fixed_point" and not self.record_iteration_diagnostics:
            raise ValueError("stop_mode='fixed_point' requires record_iteration_diagnostics=True")
        if stop_mode not in {"sigma_best", "fixed_point"}:
            raise ValueError("stop_mode must be 'sigma_best' or 'fixed_point'")
        update_tol = float(tol if fixed_point_update_tol is None else fixed_point_update_tol)
        observable_tol = float(tol if fixed_point_observable_tol is None else fixed_point_observable_tol)
        if update_tol <= 0.0 or float(fixed_point_pde_tol) <= 0.0 or observable_tol <= 0.0:
            raise ValueError("fixed-point tolerances must be positive")
        if int(fixed_point_patience) < 1:
            raise ValueError("fixed_point_patience must be >= 1")
        if mode == "curl_free_current":
            mode = "cfcf"
        if mode == "cfcf" and self.handoff_projection_policy == "error":
            raise NotImplementedError(
                "handoff_projection_policy='error' needs the Stable-NFPT field's projection errors "
                "(its Fortran-compatible bjt00 reconstruction), which this build does not form; "
                "the cfcf start runs with handoff_projection_policy='project'")
        if mode == "soft_cfcf" and self.Nz < 5:
            raise ValueError("soft_cfcf requires Nz >= 5")
        if mode == "soft_cfcf" and (self.Nx < 3 or self.Ny < 3):
            raise ValueError("soft_cfcf requires Nx, Ny >= 3")
        if polarity_mask not in _POLARITY:
            raise ValueError("polarity_mask must be 'positive', 'negative', or 'both'")
        if self.gaussian_separation_diagnostics is None:
            raise RuntimeError("NFGS boundary is not set. Call set_bottom_vector_boundary() first.")
        max_iter = int(max_iter)
        use_imp = sigma_improvement_tol is not None and float(sigma_improvement_tol) > 0.0
        eps = float(sigma_improvement_tol) if use_imp else 0.0
        record = bool(self.record_iteration_diagnostics)
        fixed = stop_mode == "fixed_point"
        step_by_step = per_step_callback is not None or verbose or record
        # the fixed-point mode replaces the sigma_best stop rules (nfgs_solver.py:3777-3812):
        # on the device only max_iter and the rollback limit remain
        stop = L.NfgsStop(
            max_iter=max_iter, patience=0 if fixed else int(patience), tol=-1.0 if fixed else float(tol),
            mu=float(mu),
            sigma_improvement_tol=eps if (use_imp and not fixed) else -1.0, polarity_mask=_POLARITY[polarity_mask],
            adaptive_mu=int(bool(adaptive_mu)), mu_min=float(mu_min), mu_max=float(mu_max),
            mu_backoff=float(mu_backoff), mu_growth=float(mu_growth), growth_streak=int(growth_streak),
            max_rollbacks=int(max_rollbacks), divergence_factor=float(divergence_factor),
            check_every=1 if (per_step_callback is not None or record) else max(1, int(check_every)),
            use_graph=int(bool(use_graph)))
        lib = self._lib
        L.check(lib.nfgs_iterate_begin(self._h, L.C.byref(stop)))
        if fixed:
            L.check(lib.nfgs_iterate_fixed_point(self._h, 0))
        self._init_diagnostics = {"init_mode": "gs_cfcf", "mfr_count": 0,
                                  "gaussian_separation": self.gaussian_separation_diagnostics,
                                  "coupled_k0": self._k0_diagnostics}
        if mode == "soft_cfcf":
            self._init_diagnostics = self._soft_cfcf_start()
        if mode == "cfcf":
            self._init_diagnostics = self._cfcf_start()
        self.learned_start_info = None
        if mode == "learned":
            from . import learned as _learned

            self.learned_start_info = _learned.learned_start(self, warm_start, fallback=True)
        if verbose:
            sc = np.zeros(3)
            L.check(lib.nfgs_iterate_initial(self._h, L.dptr(sc)))
            am = self.alpha_max()
            am_text = f"{am:.3e}" if am is not None else "off"
            print(f"Initial  sigma={sc[0]:.4e}  divB={sc[1]:.4e}  E={sc[2]:.4e} "
                  f"(mu0={mu}, adaptive={adaptive_mu}, alpha_max={am_text}, toroidal_bc=True)")
        return dict(lib=lib, mode=mode, verbose=verbose, per_step_callback=per_step_callback, step_by_step=step_by_step,
                    record=record, diag_rows=[], fp_met=[], fp_streak=0, fp_converged=False,
                    check_every=check_every, max_iter=max_iter, stop_mode=stop_mode, update_tol=update_tol,
                    observable_tol=observable_tol, fixed_point_pde_tol=fixed_point_pde_tol,
                    fixed_point_patience=fixed_point_patience, eps=eps, use_imp=use_imp)

    def _cfcf_start(self):
        """cfcf start on the device (nfgs_solver.py:6080-6147), after
        nfgs_iterate_begin: the Stable-NFPT curl-free-current state projected
        into the NFGS scalars replaces the gs_cfcf start.  The projection's
        field and current RMS differences (diagnostics of the stable solver's
        own Fortran-compatible field) are not formed: those keys are None."""
        mean = np.zeros(self.Nz)
        out = np.zeros(2)
        L.check(self._lib.nfgs_iterate_cfcf_start(self._h, int(self._lateral_bc1), L.dptr(mean), L.dptr(out)))
        return {"init_mode": "cfcf", "mfr_count": 0, "stable_cfcf_handoff": True,
                "stable_cfcf_handoff_projected": True,
                "stable_cfcf_field_rms_difference": None, "stable_cfcf_current_rms_difference": None,
                "stable_cfcf_field_relative_difference": None, "stable_cfcf_current_relative_difference": None,
                "stable_cfcf_mean_bcz_by_height": [float(v) for v in mean],
                "stable_cfcf_own_az": bool(out[1]),
                "gaussian_separation": self.gaussian_separation_diagnostics,
                "coupled_k0": self._k0_diagnostics}

    def _soft_cfcf_start(self):
        """soft_cfcf start on the device (nfgs_solver.py:6427-6484), after
        nfgs_iterate_begin: replaces the gs_cfcf start; returns the init
        diagnostics with the modal energies (nfgs_solver.py:6473-6483)."""
        out = np.zeros(4)
        L.check(self._lib.nfgs_iterate_soft_cfcf_start(self._h, float(self.soft_cfcf_epsilon),
                                                       float(self.soft_cfcf_normal_ridge), L.dptr(out)))
        return {"init_mode": "soft_cfcf", "mfr_count": 0, "soft_cfcf_epsilon": self.soft_cfcf_epsilon,
                "soft_cfcf_mode_batch_size": self.soft_cfcf_mode_batch_size,
                "soft_cfcf_normal_ridge": self.soft_cfcf_normal_ridge,
                "soft_cfcf": {"curl_current_energy": float(out[0]), "current_energy": float(out[1]),
                              "objective": float(out[2])},
                "gaussian_separation": self.gaussian_separation_diagnostics,
                "coupled_k0": self._k0_diagnostics}

    def _iterate_loop(self, ctx):
        lib, per_step_callback, check_every = ctx["lib"], ctx["per_step_callback"], ctx["check_every"]
        step_by_step, verbose = ctx["step_by_step"], ctx["verbose"]
        rows_seen = 0
        reason = L.C.c_int32(0)
        ndone = L.C.c_int32(0)
        record = ctx.get("record", False)
        while True:
            steps = 1 if (per_step_callback is not None or record) else max(1, int(check_every))
            L.check(lib.nfgs_iterate_advance(self._h, steps, L.C.byref(reason), L.C.byref(ndone)))
            if record:
                tot = L.C.c_int32(0)
                L.check(lib.nfgs_get_history(self._h, 0, 0, None, L.C.byref(tot)))
                if tot.value > len(ctx["diag_rows"]):
                    if self._record_step(ctx, tot.value):
                        break
            if step_by_step:
                tot = L.C.c_int32(0)
                L.check(lib.nfgs_get_history(self._h, 0, 0, None, L.C.byref(tot)))
                if tot.value > rows_seen:
                    buf = np.zeros((tot.value - rows_seen, L.NFGS_HIST_COLS))
                    L.check(lib.nfgs_get_history(self._h, rows_seen, tot.value - rows_seen, L.dptr(buf),
                                                 L.C.byref(tot)))
                    for r in buf:
                        rows_seen += 1
                        n = rows_seen
                        if r[4] == 0 and per_step_callback is not None:
                            B, J = self._state_fields(which=1)
                            per_step_callback(n, float(r[0]), B, J)
                        if verbose and r[4] == 0 and (n == 1 or n % 10 == 0):
                            print(f"Iter {n:4d} | sigma={r[0]:.4e} | divB={r[1]:.4e} | E={r[2]:.4e} | "
                                  f"mu={r[3]:.3f}")
                        elif verbose and r[4] == 1:
                            print(f"Iter {n:4d} | sigma={r[0]:.4e} DIVERGED -> rollback, mu={r[3]:.3f}")
            if reason.value != 0:
                break

    _DIAG_KEYS = ("phi_update_relative", "az_update_relative", "phi_map_residual_relative",
                  "az_map_residual_relative", "h_k0_update_relative", "h_k0_map_residual_relative",
                  "bcz_pde_residual_relative", "jz_pde_residual_relative", "poloidal_pde_residual_relative",
                  "toroidal_pde_residual_relative", "mixed_row_residual_relative", "bottom_field_imprint_relative",
                  "bottom_jz_imprint_relative", "alpha_clip_fraction", "weak_field_floor_fraction")

    def _record_step(self, ctx, rows):
        """One step of record_iteration_diagnostics: the device diagnostics of
        the attempted candidate (nfgs_solver.py:6806-6933) and the fixed-point
        criteria of an accepted step (nfgs_solver.py:3707-3735, 3764-3776).
        Returns True when the fixed-point stop is reached."""
        out = np.zeros(L.NFGS_NSTEPDIAG)
        L.check(self._lib.nfgs_step_diagnostics(self._h, L.dptr(out)))
        d = {k: float(v) for k, v in zip(self._DIAG_KEYS, out)}
        ctx["diag_rows"].append(d)
        row = np.zeros((1, L.NFGS_HIST_COLS))
        tot = L.C.c_int32(0)
        L.check(self._lib.nfgs_get_history(self._h, rows - 1, 1, L.dptr(row), L.C.byref(tot)))
        src, erc, rollback = float(row[0, 5]), float(row[0, 6]), int(row[0, 4])
        if rollback:
            ctx["fp_met"].append(0)
            ctx["fp_streak"] = 0
            return False
        map_res = max(d["phi_map_residual_relative"], d["az_map_residual_relative"], d["h_k0_map_residual_relative"])
        pde_res = max(d["poloidal_pde_residual_relative"], d["toroidal_pde_residual_relative"],
                      d["mixed_row_residual_relative"])
        met = (ctx["stop_mode"] == "fixed_point" and math.isfinite(map_res) and math.isfinite(pde_res)
               and map_res <= ctx["update_tol"] and pde_res <= float(ctx["fixed_point_pde_tol"])
               and src <= ctx["observable_tol"] and erc <= ctx["observable_tol"])
        ctx["fp_met"].append(int(met))
        ctx["fp_streak"] = ctx["fp_streak"] + 1 if met else 0
        if ctx["stop_mode"] == "fixed_point" and ctx["fp_streak"] >= int(ctx["fixed_point_patience"]):
            ctx["fp_converged"] = True
            L.check(self._lib.nfgs_iterate_fixed_point(self._h, 1))
            return True
        return False

    def _iterate_finish(self, ctx):
        lib, verbose, max_iter, stop_mode = ctx["lib"], ctx["verbose"], ctx["max_iter"], ctx["stop_mode"]
        update_tol, observable_tol = ctx["update_tol"], ctx["observable_tol"]
        fixed_point_pde_tol, fixed_point_patience = ctx["fixed_point_pde_tol"], ctx["fixed_point_patience"]
        eps, use_imp = ctx["eps"], ctx["use_imp"]
        res = L.NfgsIterResult()
        hist = np.zeros((max(max_iter, 0) + 1, L.NFGS_HIST_COLS))
        code = lib.nfgs_iterate_end(self._h, L.C.byref(res), L.dptr(hist), hist.shape[0])
        n = int(res.n_hist)
        hist = hist[:n]
        # the gs_cfcf start's zero-source solve records a 0.0 ratio first; the
        # soft_cfcf start runs no source solve (nfgs_solver.py:5457-5476)
        zr = ([] if ctx.get("mode") == "soft_cfcf" else [0.0]) + [float(v) for v in hist[:, 7]]
        if code == L.NFGS_EPOLICY:
            # the failing source of the next step is the last recorded ratio
            self._source_zero_mode_history = zr
            L.check(code)
        L.check(code)
        self._source_zero_mode_history = zr
        if self.source_zero_mode_policy == "warn_project":
            for v in zr:
                if v > self.source_zero_mode_tolerance:
                    warnings.warn(f"The Phi_c nonlinear source has an incompatible zero mode ratio={v:.6e} "
                                  f"exceeds tolerance={self.source_zero_mode_tolerance:.6e}. The incompatible "
                                  "zero mode will be projected out.", RuntimeWarning, stacklevel=2)
        stop_reason = L.STOP_REASONS[int(res.stop_reason)]
        if verbose:
            if stop_reason == "tol":
                print(f"Converged at iteration {res.final_iter}")
            elif stop_reason in ("sigma_improvement_tol", "sigma_stall"):
                print(f"Early stop at iter {res.final_iter}: {stop_reason} "
                      f"(best sigma={res.best_sigma:.4e} at iter {res.best_iter})")
        self._have_solution = True
        self._last_result = res
        if self.horizontal_zero_mode_policy in ("coupled_k0", "constrained_spline_harmonic"):
            self._k0_update_diagnostics()
        history = {
            "sigma": [float(v) for v in hist[:, 0]],
            "divB": [float(v) for v in hist[:, 1]],
            "energy": [float(v) for v in hist[:, 2]],
            "mu": [float(v) for v in hist[:, 3]],
            "rollback": [int(v) for v in hist[:, 4]],
            "sigma_relative_change": [float(v) for v in hist[:, 5]],
            "energy_relative_change": [float(v) for v in hist[:, 6]],
            "fixed_point_criteria_met": (list(ctx["fp_met"][:n]) + [0] * max(0, n - len(ctx["fp_met"]))
                                         if ctx.get("record") else [0] * n),
            "best_sigma": float(res.best_sigma),
            "best_iter": int(res.best_iter),
            "rollbacks": int(res.rollbacks),
            "stop_reason": stop_reason,
            "stop_mode": stop_mode,
            "selected_state": "final_accepted_iterate" if stop_mode == "fixed_point" else "best_sigma",
            "final_iter": int(res.final_iter),
            "final_sigma": float(res.final_sigma),
            "final_vs_best_B_relative": float(res.final_vs_best_B_relative),
            "fixed_point_converged": bool(ctx.get("fp_converged", False)),
            "fixed_point_streak": int(ctx.get("fp_streak", 0)),
            "fixed_point_tolerances": {"update": update_tol, "pde": float(fixed_point_pde_tol),
                                       "observable": observable_tol, "patience": int(fixed_point_patience)},
            "sigma_improvement_tol": eps if use_imp else None,
            "auto_rbsl_improvement_grace": 0,
            "last_sigma_improvement": None if math.isnan(res.last_sigma_improvement)
            else float(res.last_sigma_improvement),
            "init_diagnostics": dict(self._init_diagnostics),
            "source_partition_mode": self.source_partition_mode,
            "bottom_current_grid_mode": self._bottom_current_grid_mode,
            "vertical_current_operator": self.vertical_current_operator,
            "sigma_placement": "vertical_faces",
            # B200 build extras (not in the reference history)
            "initial_sigma": float(res.sigma0), "initial_divB": float(res.divB0),
            "initial_energy": float(res.energy0),
            "device_ms": float(res.device_ms), "kernel_launches": int(res.kernel_launches),
            "learned_start": self.learned_start_info,
        }
        if ctx.get("record"):
            rows = ctx["diag_rows"][:n]
            for key in (sorted(rows[0]) if rows else []):
                history[key] = [float(r[key]) for r in rows]
            history["iteration_diagnostics_definition"] = {
                "state": "the candidate each step proposed (before acceptance); history.rollback marks rejected ones",
                "map_residual": "RMS of the unrelaxed map T(x_n) - x_n over the RMS of x_n",
                "pde_scope": "interior rows of the scalar poloidal / toroidal equations; the mixed first interior "
                             "row on its own",
                "relative_norm": "RMS residual over the largest RMS of the operator and source terms",
                "weak_field_floor_B2": self.weak_field_floor_b2,
                "alpha_clip_scale": self.alpha_clip_scale,
            }
        history["source_diagnostics"] = self.compute_source_diagnostics()
        return history

    def _state_fields(self, which: int):
        """B, J (3, Nz, Ny, Nx) of a device state as host arrays."""
        out = np.empty(6 * self.Nz * self.Ny * self.Nx)
        dims = (L.C.c_int32 * 3)()
        L.check(self._lib.nfgs_fields(self._h, which, 0, L.dptr(out), dims))
        f = out.reshape(6, self.Nz, self.Ny, self.Nx).astype(self._np_dtype)
        return f[:3], f[3:]

    # ------------------------------------------------------------------
    def fields_to_numpy(self, *, crop_to_observed_fov: bool = True):
        """Cropped host copies of B and J (nfgs_solver.py:2881-2903)."""
        if not self._have_solution:
            raise RuntimeError("No solution stored; call iterate() first.")
        nzo, _, _ = self._observed_shape_zyx
        sy, sx = self.fov_slice_yx
        if crop_to_observed_fov:
            shape = (nzo, sy.stop - sy.start, sx.stop - sx.start)
        else:
            shape = (self.Nz, self.Ny, self.Nx)
        # a reused page-locked block when one is free (the device copy lands
        # in it directly), else pageable memory
        from .hostmem import POOL

        n = 6 * int(np.prod(shape))
        out = POOL.empty(n, self._np_dtype)
        if out is None:
            out = np.empty(n, dtype=self._np_dtype)
        dims = (L.C.c_int32 * 3)()
        code = L.NFGS_F32 if out.dtype == np.float32 else L.NFGS_F64
        L.check(self._lib.nfgs_fields_into(self._h, 0, int(bool(crop_to_observed_fov)),
                                           out.ctypes.data_as(L.C.c_void_p), code, dims))
        f = out.reshape((6,) + shape)
        return {"Bx": f[0], "By": f[1], "Bz": f[2], "Jx": f[3], "Jy": f[4], "Jz": f[5]}

    def fields_to_torch(self, *, crop_to_observed_fov: bool = True):
        """The fields of fields_to_numpy as one CUDA tensor (6, nz, ny, nx) of
        the solver dtype -- Bx, By, Bz, Jx, Jy, Jz -- gathered on the device
        (nfgs_fields_device); nothing is copied to the host."""
        import torch

        if not self._have_solution:
            raise RuntimeError("No solution stored; call iterate() first.")
        dims = (L.C.c_int32 * 3)()
        crop = int(bool(crop_to_observed_fov))
        code = L.NFGS_F32 if self._np_dtype == np.float32 else L.NFGS_F64
        L.check(self._lib.nfgs_fields_device(self._h, 0, crop, None, code, dims))
        dt = torch.float32 if code == L.NFGS_F32 else torch.float64
        out = torch.empty((6, dims[0], dims[1], dims[2]), dtype=dt, device=f"cuda:{self._device_index}")
        torch.cuda.current_stream(out.device).synchronize()  # the solver writes it on its own stream
        L.check(self._lib.nfgs_fields_device(self._h, 0, crop, L.C.c_void_p(out.data_ptr()), code, dims))
        return out

    def compute_source_diagnostics(self) -> dict:
        """Source-attribution diagnostics of the stored solution (nfgs_solver.py:7014-7196)."""
        if self.gaussian_separation_diagnostics is None:
            raise RuntimeError("NFGS boundary is not configured")
        v = np.zeros(L.NFGS_NSRCDIAG)
        L.check(self._lib.nfgs_source_diagnostics(self._h, L.dptr(v)))
        hist = self._source_zero_mode_history
        diag = {
            "source_partition_mode": self.source_partition_mode,
            "weak_field_floor_B2": self.weak_field_floor_b2,
            "alpha_clip_scale": self.alpha_clip_scale,
            "bottom_reconstruction_rms": float(v[0]),
            "bottom_reconstruction_max": float(v[1]),
            "correction_bottom_rms": float(v[2]),
            "top_robin_rms": float(v[3]),
            "top_phi_robin_rms": float(v[4]),
            "top_upward_source_rms": float(v[5]),
            "top_upward_source_ratio": float(v[6]),
            "source_zero_mode_ratio_last": hist[-1] if hist else 0.0,
            "source_zero_mode_ratio_max": max(hist) if hist else 0.0,
            "source_zero_mode_tolerance": self.source_zero_mode_tolerance,
            "source_zero_mode_policy": self.source_zero_mode_policy,
            "bottom_divergence_projection_weight": self.bottom_divergence_projection_weight,
            "bottom_divergence_robin_weight": self.bottom_divergence_robin_weight,
            "poloidal_update_mode": self.poloidal_update_mode,
            "vertical_current_operator": self.vertical_current_operator,
            "bottom_current_grid_mode": self._bottom_current_grid_mode,
            "bottom_divergence_control_mode": (
                "projection" if self.bottom_divergence_projection_weight > 0.0
                else ("mixed_robin" if self.bottom_divergence_robin_weight > 0.0 else "none")),
            "bottom_divergence_rms": float(v[9]),
            "bottom_divergence_relative": float(v[10]),
            "bottom_dphi_residual_rms": float(v[11]),
        }
        tor = self.toroidal_boundary_diagnostics or {}
        raw = float(tor.get("raw_jz_rms", 0.0) or 0.0)
        proj = float(tor.get("raw_vs_t_implied_jz_rms", 0.0) or 0.0)
        diag.update({
            "Jz_projected_out_rms": proj,
            "Jz_projected_out_over_Jz_rms": proj / max(raw, 1.0e-30),
            "B_harm_over_Bobs_rms": float((self.gaussian_separation_diagnostics or {}).get(
                "bottom_horizontal_reconstruction_ratio", 0.0)),
        })
        diag.update(self.gaussian_separation_diagnostics or {})
        if self.horizontal_zero_mode_policy == "frozen_linear_harmonic":
            fr = dict(self._k0_diagnostics)
            t = fr.get("bottom_target", [0.0, 0.0])
            fr["profile_by_height"] = [[float(t[0])] * self.Nz, [float(t[1])] * self.Nz]
            diag["frozen_linear_harmonic"] = fr
        elif self.horizontal_zero_mode_policy in ("coupled_k0", "constrained_spline_harmonic"):
            # nfgs_solver.py:7171-7196: the closure's block with the selected
            # state's profile by height
            fr = dict(self._k0_diagnostics)
            fr["profile_by_height"] = [[float(v) for v in comp] for comp in self._k0_state()["profile"]]
            diag[self.horizontal_zero_mode_policy] = fr
        return diag

    def _k0_state(self):
        """The device's k_h=0 closure state (nfgs_k0_state)."""
        nz = self.Nz
        out = np.zeros(6 * nz + 3)
        L.check(self._lib.nfgs_k0_state(self._h, L.dptr(out), out.size))
        return {"profile": out[:2 * nz].reshape(2, nz), "fit": out[2 * nz:4 * nz].reshape(2, nz),
                "target": out[4 * nz:6 * nz].reshape(2, nz), "residual_relative_max": float(out[6 * nz]),
                "kkt_condition_number": float(out[6 * nz + 1]), "updates": int(out[6 * nz + 2])}

    def _k0_update_diagnostics(self):
        """The closure's fit diagnostics of the last update
        (nfgs_solver.py:5965-6009, 6024-6065), from the device's last fitted
        profile H* and target mean current q: the fitted current is
        (-dH_y/dz, dH_x/dz) at the planes, the face fit H_x' = avg q_y,
        H_y' = -avg q_x."""
        st = self._k0_state()
        if st["updates"] <= 0:
            return
        prof, desired, dz = st["fit"], st["target"], float(self.dz)
        face = (prof[:, 1:] - prof[:, :-1]) / dz
        der = np.zeros_like(prof)
        der[:, 1:-1] = 0.5 * (face[:, :-1] + face[:, 1:])
        der[:, 0] = (-3.0 * prof[:, 0] + 4.0 * prof[:, 1] - prof[:, 2]) / (2.0 * dz)
        der[:, -1] = (3.0 * prof[:, -1] - 4.0 * prof[:, -2] + prof[:, -3]) / (2.0 * dz)
        rms = lambda a: float(np.sqrt(np.mean(np.square(a))))  # noqa: E731
        res = np.stack([-der[1], der[0]]) - desired
        des_rms = rms(desired)
        dface = np.stack([0.5 * (desired[1, :-1] + desired[1, 1:]), -0.5 * (desired[0, :-1] + desired[0, 1:])])
        grid = prof[:, 1:-1] - 0.25 * (prof[:, :-2] + 2.0 * prof[:, 1:-1] + prof[:, 2:])
        prof_rms = rms(prof)
        self._k0_diagnostics.update({
            "ode_residual_rms": rms(res),
            "ode_residual_relative": rms(res) / max(des_rms, 1e-30),
            "ode_residual_relative_max": st["residual_relative_max"],
            "face_ode_residual_rms": rms(face - dface),
            "face_ode_residual_relative": rms(face - dface) / max(rms(dface), 1e-30),
            "gridscale_profile_rms": rms(grid),
            "gridscale_profile_relative": rms(grid) / max(prof_rms, 1e-30),
            "top_derivative": [float(v) for v in der[:, -1]],
            "profile_max_abs": float(np.abs(prof).max()),
            "profile_top": [float(v) for v in prof[:, -1]],
            "desired_mean_current_rms": des_rms,
        })

    # ------------------------------------------------------------------
    # Step-level access (used by parity tests; not in the reference API)
    # ------------------------------------------------------------------
    def _get_state(self, which: int = 1):
        V = self.Nz * self.Ny * self.Nx
        phi = np.empty(V)
        az = np.empty(V)
        sc = np.zeros(3)
        L.check(self._lib.nfgs_get_scalars_state(self._h, which, L.dptr(phi), L.dptr(az), L.dptr(sc)))
        s = (self.Nz, self.Ny, self.Nx)
        return phi.reshape(s), az.reshape(s), sc

    def _step(self, mu: float = 1.0, polarity_mask: str = "both"):
        L.check(self._lib.nfgs_step(self._h, float(mu), _POLARITY[polarity_mask]))

    def _time_phases(self, n_iters: int) -> np.ndarray:
        """Device ms per phase over n_iters iterations (see nfgs_time_phases)."""
        ms = np.zeros(5)
        L.check(self._lib.nfgs_time_phases(self._h, int(n_iters), L.dptr(ms)))
        return ms

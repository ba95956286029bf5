"""Generate the golden fixtures in this directory by running the REFERENCE solver.

Run in a container where the reference repository is mounted (default
``/root/reference``, override with ``NFGS_REFERENCE``):

    python tests/golden/make_golden.py

It imports ``nfgs_solver.NFGSSolverGPU`` (the reference implementation,
FP64 on CPU) and records, for a few small grids: the boundary set-up
products, the ``gs_cfcf`` initial state, single NFPT steps (mu = 1 and
mu < 1), and a full ``iterate`` history with the final cropped fields.
The fixtures are committed; the tests never import the reference.
"""

from __future__ import annotations

import json
import math
import os
import sys
from pathlib import Path

import numpy as np

REF = os.environ.get("NFGS_REFERENCE", "/root/reference")
sys.path.insert(0, REF)

import torch  # noqa: E402
from nfgs_solver import NFGSSolverGPU  # noqa: E402

OUT = Path(__file__).resolve().parent


def analytic_boundary(ny, nx):
    """The analytic boundary used by the reference's own padding tests."""
    y, x = np.meshgrid(np.arange(ny, dtype=np.float64), np.arange(nx, dtype=np.float64), indexing="ij")
    return 0.2 * y**2, np.sin(x) * (1 + y), 2 + np.cos(x) * np.cos(y)


def bipolar_boundary(ny, nx, seed):
    """Smooth sheared bipolar region with a net-flux offset (seeded)."""
    rng = np.random.default_rng(seed)
    y, x = np.meshgrid(np.arange(ny, dtype=np.float64), np.arange(nx, dtype=np.float64), indexing="ij")
    cx, cy = (nx - 1) / 2 + rng.uniform(-1, 1), (ny - 1) / 2 + rng.uniform(-1, 1)
    s = min(nx, ny) / 6.0
    sep = min(nx, ny) / 5.0
    g1 = np.exp(-((x - cx - sep) ** 2 + (y - cy) ** 2) / (2 * s * s))
    g2 = np.exp(-((x - cx + sep) ** 2 + (y - cy) ** 2) / (2 * s * s))
    bz = g1 - 0.9 * g2
    shear = rng.uniform(0.2, 0.5)
    bx = -shear * (y - cy) / s * (g1 + g2) + 0.05
    by = shear * (x - cx) / s * (g1 - g2) - 0.03
    return bx, by, bz


def lowlou_boundary(n):
    from nfgs._backend.util.lnl_io import get_analytic_b_field

    b = get_analytic_b_field(n=1, m=1, l=0.3, psi=math.pi / 4, resolution=(n, n, n), dtype=np.float64)
    ref = [np.transpose(b[..., i], (2, 1, 0)).copy() for i in range(3)]
    return ref[0][0], ref[1][0], ref[2][0]


CASES = {
    "tiny_rho05": dict(
        shape=(11, 9, 7), spacing=(1.0, 1.0, 1.0), boundary=("analytic", None),
        ctor=dict(buffer_thickness=0, bottom_divergence_robin_weight=0.5),
        bnd=dict(smooth_passes=0), iters=12, patience=40, mu2=0.7,
    ),
    "tiny_rho0_legacy": dict(
        shape=(11, 9, 7), spacing=(1.0, 1.0, 1.0), boundary=("analytic", None),
        ctor=dict(buffer_thickness=0, bottom_divergence_robin_weight=0.0, calculation_domain_mode="mudpack_legacy"),
        bnd=dict(smooth_passes=0), iters=10, patience=40, mu2=0.3,
    ),
    "small_rho03_buffer": dict(
        shape=(16, 14, 10), spacing=(0.5, 0.5, 0.5), boundary=("bipolar", 7),
        ctor=dict(buffer_thickness=2, bottom_divergence_robin_weight=0.3),
        bnd=dict(smooth_passes=0), iters=15, patience=5, mu2=0.6, store="small",
    ),
    "small_rho1_unpadded": dict(
        shape=(15, 13, 9), spacing=(1.0, 0.8, 0.9), boundary=("bipolar", 11),
        ctor=dict(bottom_divergence_robin_weight=1.0, pad_calculation_domain=False,
                  alpha_clip_scale=0.5),
        bnd=dict(smooth_passes=1), iters=12, patience=40, mu2=1.0, store="small",
    ),
    "small_projection_omit": dict(
        shape=(16, 14, 10), spacing=(1.0, 1.0, 1.0), boundary=("bipolar", 3),
        ctor=dict(bottom_divergence_projection_weight=0.6, horizontal_zero_mode_policy="omit",
                  gaussian_horizontal_operator="fd", bottom_parallel_current_mode="face_parallel_exact_jz"),
        bnd=dict(smooth_passes=0), iters=10, patience=40, mu2=1.0, store="small",
    ),
    "lowlou32_rho05": dict(
        shape=(32, 32, 32), spacing=(1.0, 1.0, 1.0), boundary=("lowlou", 32),
        ctor=dict(bottom_divergence_robin_weight=0.5),
        bnd=dict(smooth_passes=0), iters=200, patience=40, mu2=1.0, store="history",
    ),
}

POLICIES = dict(d0_zero_mode_policy="project", source_zero_mode_policy="project",
                horizontal_zero_mode_policy="frozen_linear_harmonic",
                vertical_current_operator="staggered_face")


def t2n(t):
    return t.detach().cpu().numpy().astype(np.float64)


def run_case(name, spec):
    nx, ny, nz = spec["shape"]
    kind, arg = spec["boundary"]
    if kind == "analytic":
        bx, by, bz = analytic_boundary(ny, nx)
    elif kind == "bipolar":
        bx, by, bz = bipolar_boundary(ny, nx, arg)
    else:
        bx, by, bz = lowlou_boundary(arg)
    ctor = dict(POLICIES)
    ctor.update(spec["ctor"])
    dx, dy, dz = spec["spacing"]

    def make():
        s = NFGSSolverGPU(nx, ny, nz, dx, dy, dz, device="cpu", dtype=torch.float64, **ctor)
        s.set_bottom_vector_boundary(bx, by, bz, zero_net_current=False, ijzbcor=3, **spec["bnd"])
        return s

    out = {"bx_in": bx, "by_in": by, "bz_in": bz}
    with torch.inference_mode():
        s = make()
        out.update({
            "Bz_obs": t2n(s.Bz_obs), "Bx_obs": t2n(s.Bx_obs), "By_obs": t2n(s.By_obs),
            "Jz_obs": t2n(s.Jz_obs), "Az_bottom": t2n(s.Az_bottom),
            "Jz_T": t2n(s.Jz_toroidal_boundary), "B_background": t2n(s.B_background),
            "Phi_above_bottom": t2n(s.Phi_above_bottom), "Bz_above": t2n(s.Bz_above),
            "bottom_dphi_c_target": t2n(s._bottom_dphi_c_target), "D0": t2n(s.D0),
            "H_bottom": t2n(s._H_k0_bottom_target) if s._H_k0_bottom_target is not None else np.zeros(2),
            "gaussian_above": t2n(s.gaussian_above_bottom_field()),
        })
        st = s.compute_initial_conditions(init_mode="gs_cfcf")
        B, J, phi, az, bc = st
        out.update({"init_B": t2n(B), "init_J": t2n(J), "init_phi": t2n(phi), "init_az": t2n(az)})
        out["init_scalars"] = np.array([s.compute_sigma(B, J), s.compute_divB(B), s.compute_energy(B)])
        st1 = s.iteration_step(*st, mu=1.0)
        out.update({"step1_B": t2n(st1[0]), "step1_J": t2n(st1[1]), "step1_phi": t2n(st1[2]), "step1_az": t2n(st1[3])})
        st2 = s.iteration_step(*st1, mu=spec["mu2"])
        out.update({"step2_B": t2n(st2[0]), "step2_J": t2n(st2[1]), "step2_phi": t2n(st2[2]), "step2_az": t2n(st2[3])})
        out["step_scalars"] = np.array([
            s.compute_sigma(st1[0], st1[1]), s.compute_divB(st1[0]), s.compute_energy(st1[0]),
            s.compute_sigma(st2[0], st2[1]), s.compute_divB(st2[0]), s.compute_energy(st2[0]),
        ])

        s = make()
        h = s.iterate(init_mode="gs_cfcf", max_iter=spec["iters"], tol=1e-5, mu=1.0, patience=spec["patience"],
                      sigma_improvement_tol=1e-5, stop_mode="sigma_best", verbose=False)
        f = s.fields_to_numpy(crop_to_observed_fov=True)
    store = spec.get("store", "full")
    if store == "full":
        for k in ("Bx", "By", "Bz", "Jx", "Jy", "Jz"):
            out["final_" + k] = f[k].astype(np.float64)
    else:
        for k in ("step1_B", "step1_J", "step2_B", "step2_J"):
            out.pop(k)
        if store == "history":
            for k in [k for k in out if k.startswith(("init_", "step1_", "step2_"))
                      and k not in ("init_scalars", "step_scalars", "init_phi", "init_az")]:
                out.pop(k)
            out.pop("B_background")
            for k in ("Bx", "By", "Bz", "Jx", "Jy", "Jz"):
                out["final_" + k + "_s2"] = f[k][::2, ::2, ::2].astype(np.float32)
                out["final_" + k + "_norm"] = np.array([np.sqrt(np.sum(f[k].astype(np.float64) ** 2))])
        else:
            for k in ("Bx", "By", "Bz", "Jx", "Jy", "Jz"):
                out["final_" + k] = f[k].astype(np.float64)
    out["hist_sigma"] = np.array(h["sigma"])
    out["hist_divB"] = np.array(h["divB"])
    out["hist_energy"] = np.array(h["energy"])
    meta = {
        "name": name, "store": spec.get("store", "full"), "shape": spec["shape"], "spacing": spec["spacing"], "ctor": ctor,
        "bnd": spec["bnd"], "iters": spec["iters"], "patience": spec["patience"], "mu2": spec["mu2"],
        "calc_grid": [s.Nx, s.Ny, s.Nz],
        "fov": [s.fov_slice_yx[0].start, s.fov_slice_yx[0].stop, s.fov_slice_yx[1].start, s.fov_slice_yx[1].stop],
        "observed_shape_zyx": list(s._observed_shape_zyx),
        "bottom_current_grid_mode": s._bottom_current_grid_mode,
        "best_iter": h["best_iter"], "best_sigma": h["best_sigma"], "stop_reason": h["stop_reason"],
        "final_iter": h["final_iter"], "final_sigma": h["final_sigma"],
        "final_vs_best_B_relative": h["final_vs_best_B_relative"],
        "source_diagnostics": {k: v for k, v in h["source_diagnostics"].items()
                               if isinstance(v, float)},
        "gaussian_separation_diagnostics": {k: v for k, v in (s.gaussian_separation_diagnostics or {}).items()
                                            if isinstance(v, float)},
    }
    np.savez_compressed(OUT / f"{name}.npz", **out)
    (OUT / f"{name}.json").write_text(json.dumps(meta, indent=1, sort_keys=True) + "\n")
    print(name, meta["calc_grid"], meta["stop_reason"], meta["best_iter"], f"{meta['best_sigma']:.6e}")


if __name__ == "__main__":
    torch.set_num_threads(int(os.environ.get("NFGS_THREADS", "8")))
    only = set(sys.argv[1:])
    for name, spec in CASES.items():
        if not only or name in only:
            run_case(name, spec)

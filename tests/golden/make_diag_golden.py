"""Generate the per-iteration diagnostics fixtures in tests/golden/diag/ by
running the REFERENCE with record_iteration_diagnostics=True.

Run where the reference repository is importable (default /root/reference,
override with NFGS_REFERENCE):

    python tests/golden/make_diag_golden.py

For a few of the golden cases it records the reference's per-step
diagnostics history (nfgs_solver.py:6806-6933: map residuals, PDE
residuals, bottom imprints, alpha-clip and weak-field fractions), the
fixed_point_criteria_met column and the stop of the sigma_best and
fixed_point modes (nfgs_solver.py:3707-3776), with the selected state's
cropped fields.  The tests never import the reference.
"""

from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np

REF = os.environ.get("NFGS_REFERENCE", "/root/reference")
sys.path.insert(0, REF)
sys.path.insert(0, str(Path(__file__).resolve().parent))

import torch  # noqa: E402
from make_golden import CASES, POLICIES, analytic_boundary, bipolar_boundary, lowlou_boundary  # noqa: E402
from nfgs_solver import NFGSSolverGPU  # noqa: E402

OUT = Path(__file__).resolve().parent / "diag"
DIAG_KEYS = ("alpha_clip_fraction", "az_map_residual_relative", "az_update_relative", "bcz_pde_residual_relative",
             "bottom_field_imprint_relative", "bottom_jz_imprint_relative", "h_k0_map_residual_relative",
             "h_k0_update_relative", "jz_pde_residual_relative", "mixed_row_residual_relative",
             "phi_map_residual_relative", "phi_update_relative", "poloidal_pde_residual_relative",
             "toroidal_pde_residual_relative", "weak_field_floor_fraction")
NAMES = {
    "tiny_sigma_best": dict(base="tiny_rho05", it=dict(max_iter=10, patience=40)),
    "buffer_fixed_point": dict(base="small_rho03_buffer",
                               it=dict(max_iter=40, patience=40, stop_mode="fixed_point", tol=2e-2,
                                       fixed_point_pde_tol=5e-2, fixed_point_patience=3)),
    "unpadded_clip_mu": dict(base="small_rho1_unpadded", it=dict(max_iter=8, patience=40, mu=0.7)),
    "lowlou32_fixed_point": dict(base="lowlou32_rho05",
                                 it=dict(max_iter=60, patience=40, stop_mode="fixed_point", tol=1e-3,
                                         fixed_point_pde_tol=1e-1, fixed_point_patience=2)),
}


def run(name, spec):
    base = CASES[spec["base"]]
    nx, ny, nz = base["shape"]
    kind, arg = base["boundary"]
    if kind == "analytic":
        bx, by, bz = analytic_boundary(ny, nx)
    elif kind == "bipolar":
        bx, by, bz = bipolar_boundary(ny, nx, arg)
    else:
        bx, by, bz = lowlou_boundary(arg)
    ctor = dict(POLICIES)
    ctor.update(base["ctor"])
    ctor["record_iteration_diagnostics"] = True
    dx, dy, dz = base["spacing"]
    it = dict(tol=1e-5, mu=1.0, sigma_improvement_tol=1e-5, stop_mode="sigma_best")
    it.update(spec["it"])
    with torch.inference_mode():
        s = NFGSSolverGPU(nx, ny, nz, dx, dy, dz, device="cpu", dtype=torch.float64, **ctor)
        s.set_bottom_vector_boundary(bx, by, bz, zero_net_current=False, ijzbcor=3, **base["bnd"])
        h = s.iterate(init_mode="gs_cfcf", verbose=False, **it)
        f = s.fields_to_numpy(crop_to_observed_fov=True)
    out = {"bx_in": bx, "by_in": by, "bz_in": bz, "hist_sigma": np.array(h["sigma"]),
           "hist_energy": np.array(h["energy"]), "hist_mu": np.array(h["mu"]),
           "fixed_point_criteria_met": np.array(h["fixed_point_criteria_met"])}
    for k in DIAG_KEYS:
        out["diag_" + k] = np.array(h[k])
    if nx * ny * nz < 20000:
        for k in ("Bx", "By", "Bz", "Jx", "Jy", "Jz"):
            out["final_" + k] = f[k].astype(np.float64)
    meta = {"name": name, "base": spec["base"], "shape": base["shape"], "spacing": base["spacing"], "ctor": ctor,
            "bnd": base["bnd"], "iterate": it, "best_iter": h["best_iter"], "best_sigma": h["best_sigma"],
            "stop_reason": h["stop_reason"], "final_iter": h["final_iter"], "selected_state": h["selected_state"],
            "fixed_point_converged": h["fixed_point_converged"], "fixed_point_streak": h["fixed_point_streak"]}
    OUT.mkdir(exist_ok=True)
    np.savez_compressed(OUT / f"{name}.npz", **out)
    (OUT / f"{name}.json").write_text(json.dumps(meta, indent=1, sort_keys=True) + "\n")
    print(name, meta["stop_reason"], meta["best_iter"], meta["final_iter"], len(h["sigma"]),
          {k: round(float(h[k][-1]), 6) for k in ("phi_map_residual_relative", "poloidal_pde_residual_relative",
                                                  "alpha_clip_fraction", "weak_field_floor_fraction")})


if __name__ == "__main__":
    torch.set_num_threads(int(os.environ.get("NFGS_THREADS", "8")))
    only = set(sys.argv[1:])
    for name, spec in NAMES.items():
        if not only or name in only:
            run(name, spec)

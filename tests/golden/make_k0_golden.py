"""Generate the k_h=0 closure fixtures in tests/golden/k0/ by running the
REFERENCE with horizontal_zero_mode_policy 'coupled_k0' and
'constrained_spline_harmonic'.

Run where the reference repository is importable (default /root/reference,
override with NFGS_REFERENCE):

    python tests/golden/make_k0_golden.py

For each case it records the reference's history (sigma, energy, divB, mu),
the stop, the selected state's cropped fields, the horizontal-mean profile
H(z) of the selected state and the closure's diagnostics
(nfgs_solver.py:5058-5431, 5952-6067, 7171-7196), and, where the case asks
for it, the per-step h_k0 diagnostics (nfgs_solver.py:6884-6893).  The
tests never import the reference.
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

OUT = Path(__file__).resolve().parent / "k0"
DIAG_KEYS = ("h_k0_map_residual_relative", "h_k0_update_relative", "phi_map_residual_relative",
             "az_map_residual_relative", "bottom_field_imprint_relative")
NAMES = {
    "coupled_tiny": dict(base="tiny_rho05", ctor=dict(horizontal_zero_mode_policy="coupled_k0"),
                         it=dict(max_iter=12, patience=40), diag=True),
    "coupled_legacy_mu": dict(base="small_rho03_buffer",
                              ctor=dict(horizontal_zero_mode_policy="coupled_k0",
                                        coupled_k0_discretization="legacy_plane_centred", k0_update_mu=0.5,
                                        k0_ode_smoothness=1e-2),
                              it=dict(max_iter=10, patience=40, mu=0.7)),
    "coupled_face_unpadded": dict(base="small_rho1_unpadded",
                                  ctor=dict(horizontal_zero_mode_policy="coupled_k0",
                                            k0_current_target_placement="face", k0_ode_smoothness=0.0),
                                  it=dict(max_iter=10, patience=40)),
    "spline_tiny": dict(base="tiny_rho05", ctor=dict(horizontal_zero_mode_policy="constrained_spline_harmonic",
                                                  k0_spline_basis_size=5),
                        it=dict(max_iter=12, patience=40), diag=True),
    "spline_buffer_face": dict(base="small_rho03_buffer",
                               ctor=dict(horizontal_zero_mode_policy="constrained_spline_harmonic",
                                         k0_current_target_placement="face", k0_spline_basis_size=6,
                                         k0_ode_smoothness=1e-2, k0_update_mu=0.6),
                               it=dict(max_iter=10, patience=40, mu=0.8)),
    "spline_unpadded": dict(base="small_rho1_unpadded",
                            ctor=dict(horizontal_zero_mode_policy="constrained_spline_harmonic",
                                      k0_spline_basis_size=5),
                            it=dict(max_iter=10, patience=40)),
    "lowlou32_coupled": dict(base="lowlou32_rho05", ctor=dict(horizontal_zero_mode_policy="coupled_k0"),
                             it=dict(max_iter=200, patience=40)),
    "lowlou32_spline": dict(base="lowlou32_rho05",
                            ctor=dict(horizontal_zero_mode_policy="constrained_spline_harmonic"),
                            it=dict(max_iter=200, patience=40)),
}


def _scalars(d):
    out = {}
    for k, v in d.items():
        if isinstance(v, bool):
            out[k] = v
        elif isinstance(v, (int, float)):
            out[k] = float(v)
        elif isinstance(v, str):
            out[k] = v
        elif isinstance(v, list) and all(isinstance(x, (int, float)) for x in v):
            out[k] = [float(x) for x in v]
    return out


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
    ctor.update(spec["ctor"])
    if spec.get("diag"):
        ctor["record_iteration_diagnostics"] = True
    dx, dy, dz = base["spacing"]
    it = dict(tol=1e-5, mu=1.0, sigma_improvement_tol=1e-5)
    it.update(spec["it"])
    with torch.inference_mode():
        s = NFGSSolverGPU(nx, ny, nz, dx, dy, dz, device="cpu", dtype=torch.float64, **ctor)
        s.set_bottom_vector_boundary(bx, by, bz, zero_net_current=False, ijzbcor=3, **base["bnd"])
        init_diag = _scalars(dict(s._k0_diagnostics))
        h = s.iterate(init_mode="gs_cfcf", verbose=False, **it)
        f = s.fields_to_numpy(crop_to_observed_fov=True)
    policy = ctor["horizontal_zero_mode_policy"]
    sd = h["source_diagnostics"][policy]
    out = {"bx_in": bx, "by_in": by, "bz_in": bz, "hist_sigma": np.array(h["sigma"]),
           "hist_energy": np.array(h["energy"]), "hist_divB": np.array(h["divB"]), "hist_mu": np.array(h["mu"]),
           "profile": np.array(sd["profile_by_height"], dtype=np.float64)}
    if spec.get("diag"):
        for k in DIAG_KEYS:
            out["diag_" + k] = np.array(h[k])
    if base.get("store") != "history":
        for k in ("Bx", "By", "Bz", "Jx", "Jy", "Jz"):
            out["final_" + k] = f[k].astype(np.float64)
    meta = {"name": name, "base": spec["base"], "shape": base["shape"], "spacing": base["spacing"], "ctor": ctor,
            "bnd": base["bnd"], "iterate": it, "best_iter": h["best_iter"], "best_sigma": h["best_sigma"],
            "stop_reason": h["stop_reason"], "final_iter": h["final_iter"],
            "k0_init": init_diag, "k0_final": _scalars(sd)}
    OUT.mkdir(exist_ok=True)
    np.savez_compressed(OUT / f"{name}.npz", **out)
    (OUT / f"{name}.json").write_text(json.dumps(meta, indent=1, sort_keys=True) + "\n")
    print(name, meta["stop_reason"], meta["best_iter"], meta["final_iter"], round(h["best_sigma"], 6),
          np.abs(out["profile"]).max())


if __name__ == "__main__":
    torch.set_num_threads(int(os.environ.get("NFGS_THREADS", "8")))
    only = set(sys.argv[1:])
    for name, spec in NAMES.items():
        if not only or name in only:
            run(name, spec)

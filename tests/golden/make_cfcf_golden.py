"""Generate the cfcf-start fixtures in tests/golden/cfcf/ by running the REFERENCE.

Run where the reference repository is importable (default /root/reference,
override with NFGS_REFERENCE):

    python tests/golden/make_cfcf_golden.py

For a few of the golden cases it runs the reference NFGSSolverGPU (FP64,
CPU) with init_mode="cfcf" (nfgs_solver.py:6080-6147): the projected start
state (Phi_c, A_z, B, J), the start's sigma_J / divB / energy, the mean
B_c,z per height it reports, and the iterate history from that start.
The tests never import the reference.
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

OUT = Path(__file__).resolve().parent / "cfcf"
NAMES = {
    "tiny_rho05": dict(iters=12, patience=40),
    "small_rho1_unpadded": dict(iters=12, patience=40),
    "small_rho03_buffer": dict(iters=15, patience=5),
    "lowlou32_rho05": dict(iters=200, patience=40),
    "lowlou32_pin": dict(base="lowlou32_rho05", iters=60, patience=40, ctor=dict(lateral_wall="legacy_potential_pin"),
                         store="scalars"),
}


def t2n(t):
    return t.detach().cpu().numpy().astype(np.float64)


def run(name, spec):
    base = CASES[spec.get("base", name)]
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
    ctor.update(spec.get("ctor", {}))
    dx, dy, dz = base["spacing"]

    def make():
        s = NFGSSolverGPU(nx, ny, nz, dx, dy, dz, device="cpu", dtype=torch.float64, **ctor)
        s.set_bottom_vector_boundary(bx, by, bz, zero_net_current=False, ijzbcor=3, **base["bnd"])
        return s

    out = {"bx_in": bx, "by_in": by, "bz_in": bz}
    with torch.inference_mode():
        s = make()
        B, J, phi, az, bc = s.compute_initial_conditions(init_mode="cfcf")
        diag = dict(s._init_diagnostics)
        store = spec.get("store", "fields" if nx * ny * nz < 20000 else "state")
        if store == "fields":
            out.update({"init_B": t2n(B), "init_J": t2n(J)})
        if store in ("fields", "state"):
            out.update({"init_phi": t2n(phi), "init_az": t2n(az)})
        out["init_scalars"] = np.array([s.compute_sigma(B, J), s.compute_divB(B), s.compute_energy(B)])
        out["mean_bcz_by_height"] = np.array(diag["stable_cfcf_mean_bcz_by_height"])
        s = make()
        h = s.iterate(init_mode="cfcf", max_iter=spec["iters"], tol=1e-5, mu=1.0, patience=spec["patience"],
                      sigma_improvement_tol=1e-5, stop_mode="sigma_best", verbose=False)
    out["hist_sigma"] = np.array(h["sigma"])
    out["hist_energy"] = np.array(h["energy"])
    out["hist_divB"] = np.array(h["divB"])
    meta = {"name": name, "store": store, "shape": base["shape"], "spacing": base["spacing"], "ctor": ctor, "bnd": base["bnd"],
            "iters": spec["iters"], "patience": spec["patience"], "calc_grid": [s.Nx, s.Ny, s.Nz],
            "best_iter": h["best_iter"], "best_sigma": h["best_sigma"], "stop_reason": h["stop_reason"],
            "final_iter": h["final_iter"],
            "diagnostics": {k: v for k, v in diag.items() if isinstance(v, (float, bool, int, str))}}
    OUT.mkdir(exist_ok=True)
    np.savez_compressed(OUT / f"{name}.npz", **out)
    (OUT / f"{name}.json").write_text(json.dumps(meta, indent=1, sort_keys=True) + "\n")
    print(name, meta["calc_grid"], meta["stop_reason"], meta["best_iter"], f"{meta['best_sigma']:.6e}")


if __name__ == "__main__":
    torch.set_num_threads(int(os.environ.get("NFGS_THREADS", "8")))
    only = set(sys.argv[1:])
    for name, spec in NAMES.items():
        if not only or name in only:
            run(name, spec)

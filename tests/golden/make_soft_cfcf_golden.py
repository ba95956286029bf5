"""Generate the soft_cfcf golden fixtures (tests/golden/soft_cfcf/) by running
the REFERENCE solver.

Run where the reference repository is mounted (default ``/root/reference``,
override with ``NFGS_REFERENCE``):

    python tests/golden/make_soft_cfcf_golden.py

For each case it records, from the reference ``NFGSSolverGPU`` in FP64 on
CPU: the modal profiles of the Phi and A_z modes (``_solve_soft_cfcf_modes``),
the soft_cfcf initial state and its diagnostics, and a complete
``iterate(init_mode="soft_cfcf")`` history.  The tests never import the
reference.
"""

from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF = os.environ.get("NFGS_REFERENCE", "/root/reference")
sys.path.insert(0, REF)
sys.path.insert(0, str(HERE))

import torch  # noqa: E402
from make_golden import POLICIES, analytic_boundary, bipolar_boundary, lowlou_boundary  # noqa: E402
from nfgs_solver import NFGSSolverGPU  # noqa: E402

OUT = HERE / "soft_cfcf"

CASES = {
    "tiny_default": dict(
        shape=(11, 9, 7), spacing=(1.0, 1.0, 1.0), boundary=("analytic", None),
        ctor=dict(buffer_thickness=0, bottom_divergence_robin_weight=0.5), bnd=dict(smooth_passes=0),
        iters=12, patience=40,
    ),
    "small_eps_ridge": dict(
        shape=(16, 14, 10), spacing=(0.5, 0.5, 0.5), boundary=("bipolar", 7),
        ctor=dict(buffer_thickness=2, bottom_divergence_robin_weight=0.3, soft_cfcf_epsilon=0.05,
                  soft_cfcf_normal_ridge=1e-7),
        bnd=dict(smooth_passes=0), iters=15, patience=5,
    ),
    "small_eps0_unpadded": dict(
        shape=(15, 13, 9), spacing=(1.0, 0.8, 0.9), boundary=("bipolar", 11),
        ctor=dict(bottom_divergence_robin_weight=1.0, pad_calculation_domain=False, alpha_clip_scale=0.5,
                  soft_cfcf_epsilon=0.0),
        bnd=dict(smooth_passes=1), iters=12, patience=40,
    ),
    "lowlou32_default": dict(
        shape=(32, 32, 32), spacing=(1.0, 1.0, 1.0), boundary=("lowlou", 32),
        ctor=dict(bottom_divergence_robin_weight=0.5), bnd=dict(smooth_passes=0),
        iters=200, patience=40,
    ),
}


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
        pb = s._dct2(s.Phi_above_bottom)
        pb[0, 0] = 0.0
        out["phi_hat"] = t2n(s._solve_soft_cfcf_modes(s._nfgs_k, pb, kind="phi"))
        ab = s._dst1(s._dst1(s.Az_bottom[1:-1, 1:-1], -1), -2)
        az_k = torch.sqrt(torch.clamp(-s._dirichlet_lam_xy_interior(), min=0.0))
        out["az_hat"] = t2n(s._solve_soft_cfcf_modes(az_k, ab, kind="az"))
        B, J, phi, az, _bc = s.compute_initial_conditions(init_mode="soft_cfcf")
        out.update({"init_B": t2n(B), "init_J": t2n(J), "init_phi": t2n(phi), "init_az": t2n(az)})
        out["init_scalars"] = np.array([s.compute_sigma(B, J), s.compute_divB(B), s.compute_energy(B)])
        diag = {k: float(v) for k, v in s._init_diagnostics["soft_cfcf"].items()}
        s = make()
        h = s.iterate(init_mode="soft_cfcf", max_iter=spec["iters"], tol=1e-5, mu=1.0, patience=spec["patience"],
                      sigma_improvement_tol=1e-5, stop_mode="sigma_best", verbose=False)
    if spec["shape"][0] >= 32:
        for k in ("init_B", "init_J"):
            out.pop(k)
    out["hist_sigma"] = np.array(h["sigma"])
    out["hist_divB"] = np.array(h["divB"])
    out["hist_energy"] = np.array(h["energy"])
    meta = {
        "name": name, "shape": spec["shape"], "spacing": spec["spacing"], "ctor": ctor, "bnd": spec["bnd"],
        "iters": spec["iters"], "patience": spec["patience"], "calc_grid": [s.Nx, s.Ny, s.Nz],
        "soft_cfcf_epsilon": s.soft_cfcf_epsilon, "soft_cfcf_normal_ridge": s.soft_cfcf_normal_ridge,
        "soft_cfcf": diag, "best_iter": h["best_iter"], "best_sigma": h["best_sigma"],
        "stop_reason": h["stop_reason"], "final_iter": h["final_iter"],
        "source_zero_mode_history_length": len(s._source_zero_mode_history),
    }
    OUT.mkdir(exist_ok=True)
    np.savez_compressed(OUT / f"{name}.npz", **out)
    (OUT / f"{name}.json").write_text(json.dumps(meta, indent=1, sort_keys=True) + "\n")
    print(name, meta["calc_grid"], meta["stop_reason"], meta["best_iter"], f"{meta['best_sigma']:.6e}")


if __name__ == "__main__":
    torch.set_num_threads(int(os.environ.get("NFGS_THREADS", "8")))
    only = set(sys.argv[1:])
    for name, spec in CASES.items():
        if not only or name in only:
            run_case(name, spec)

"""Generate the FP32-parity fixtures in tests/golden/fp32/ by running the REFERENCE.

Run in a container where the reference repository is importable (default
``/root/reference``, override with ``NFGS_REFERENCE``):

    python tests/golden/make_fp32_golden.py [case ...]

For each configuration of record it runs the reference ``NFGSSolverGPU``
on the CPU twice, in FP64 and in FP32 (its production dtype), from the
same boundary, and records:

* the boundary maps handed to ``set_bottom_vector_boundary``;
* both runs' gs_cfcf start (sigma_J, divB, energy) and first NFPT step;
* the reference's own FP32-vs-FP64 deviation (relative L2) of the start
  state (Phi_c, A_z, B, J), of the first step (B, J) and of the final
  cropped fields after the sigma_best stop;
* both runs' histories, best / final iterations, stop reasons and source
  diagnostics; the FP64 final fields, every 4th cell of each axis;
* the solution metrics of the FP32 result against the FP64 result with the
  reference's own metric function (``compute_reference_metrics``,
  nfgs/_backend/util/metrics.py:123-178) on the whole cropped volume:
  C_vec, C_CS, E'_n, E'_m, epsilon (energy ratio), sigma_J, and the
  reference's div-B fraction (``compute_divB``) of each result;
* config 1 only: the metrics of both results against the analytic Low-Lou
  interior, and the Low-Lou profile interpolant (breakpoints, coefficients,
  eigenvalue) from which ``oracle/lowlou_oracle.py`` rebuilds that interior,
  with reference field samples that pin the rebuild.

The tests never import the reference; they compare the CUDA path, FP32 and
FP64, with these numbers.  A second file, ``td99_points.npz``, holds the
reference TD generator (``generate_td_model``, nfgs/_backend/td.py:370-581)
evaluated on a small lattice with the benchmark's parameters, which pins
``nfgs_b200.synthetic.td99_field``.
"""

from __future__ import annotations

import json
import math
import os
import sys
import time
from pathlib import Path

import numpy as np

REF = os.environ.get("NFGS_REFERENCE", "/root/reference")
sys.path.insert(0, REF)
ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import torch  # noqa: E402
from nfgs_solver import NFGSSolverGPU  # noqa: E402
from nfgs._backend.util.metrics import compute_reference_metrics  # noqa: E402

OUT = Path(__file__).resolve().parent / "fp32"

POLICIES = dict(d0_zero_mode_policy="project", source_zero_mode_policy="project",
                horizontal_zero_mode_policy="frozen_linear_harmonic",
                vertical_current_operator="staggered_face", bottom_divergence_robin_weight=0.5)
STOP = dict(tol=1e-5, mu=1.0, patience=40, sigma_improvement_tol=1e-5, stop_mode="sigma_best")


def lowlou_case():
    from nfgs._backend.util.lnl_io import get_analytic_b_field, solve_low_lou_profile

    sol, a2 = solve_low_lou_profile(n=1, m=1)
    b = get_analytic_b_field(n=1, m=1, l=0.3, psi=math.pi / 4, resolution=(64, 64, 64),
                             bounds=(-1, 1, -1, 1, 0, 2), dtype=np.float64)
    zyx = [np.ascontiguousarray(np.transpose(b[..., i], (2, 1, 0))) for i in range(3)]
    rng = np.random.default_rng(0)
    idx = np.stack([rng.integers(0, 64, 256) for _ in range(3)])
    extra = {"lowlou_breaks": np.asarray(sol.x), "lowlou_coeffs": np.asarray(sol.c),
             "lowlou_a2": np.array([a2]), "analytic_sample_idx": idx,
             "analytic_sample": b[idx[0], idx[1], idx[2], :]}
    meta = {"analytic": {"n": 1, "m": 1, "l": 0.3, "psi": math.pi / 4, "resolution": [64, 64, 64],
                         "bounds": [-1, 1, -1, 1, 0, 2]}}
    return (zyx[0][0], zyx[1][0], zyx[2][0]), (1.0, 1.0, 1.0), (64, 64, 64), 500, zyx, extra, meta


def td_case():
    from nfgs_b200.synthetic import td_params
    from nfgs._backend.td import generate_td_model

    n, nz, ext = 96, 48, 8.0
    p = td_params(1)
    xs = np.linspace(-ext, ext, n)
    x, y = np.meshgrid(xs, xs, indexing="ij")
    bx, by, bz = generate_td_model(x[..., None], y[..., None], np.zeros_like(x)[..., None], R=p["R"], a=p["a"],
                                   L=p["L"], d=p["d"], q=p["q"], I_0=p["I0"], l_i=p["l_i"])
    bnd = tuple(np.ascontiguousarray(v[..., 0].T) for v in (bx, by, bz))
    h = 2 * ext / (n - 1)
    meta = {"td": {k: float(v) for k, v in p.items()}, "extent": ext, "seed": 1}
    return bnd, (h, h, h), (n, n, nz), 3000, None, {}, meta


CASES = {"lowlou64_rho05": lowlou_case, "td99_96_rho05": td_case}


def t2n(t):
    return t.detach().cpu().numpy().astype(np.float64)


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - np.asarray(b, np.float64)) /
                 max(np.linalg.norm(np.asarray(b, np.float64)), 1e-300))


def run(dtype, bnd, spacing, shape, max_iter):
    nx, ny, nz = shape
    dx, dy, dz = spacing
    s = NFGSSolverGPU(nx, ny, nz, dx, dy, dz, device="cpu", dtype=dtype, **POLICIES)
    s.set_bottom_vector_boundary(*bnd, zero_net_current=False, smooth_passes=0, ijzbcor=3)
    with torch.inference_mode():
        st = s.compute_initial_conditions(init_mode="gs_cfcf")
        init = {k: t2n(v) for k, v in zip(("B", "J", "phi", "az"), st[:4])}
        init_sc = [float(s.compute_sigma(st[0], st[1])), float(s.compute_divB(st[0])), float(s.compute_energy(st[0]))]
        st1 = s.iteration_step(*st, mu=1.0)
        step1 = {"B": t2n(st1[0]), "J": t2n(st1[1])}
        step_sc = [float(s.compute_sigma(st1[0], st1[1])), float(s.compute_divB(st1[0])),
                   float(s.compute_energy(st1[0]))]
        t0 = time.perf_counter()
        h = s.iterate(init_mode="gs_cfcf", max_iter=max_iter, verbose=False, **STOP)
        wall = time.perf_counter() - t0
        f = {k: v.astype(np.float64) for k, v in s.fields_to_numpy(crop_to_observed_fov=True).items()}
        Bt = torch.as_tensor(np.stack([f["Bx"], f["By"], f["Bz"]]), dtype=torch.float64)
        divb = float(s.compute_divB(Bt.to(s.dtype)))
    return {"init": init, "init_sc": init_sc, "step1": step1, "step_sc": step_sc, "h": h, "fields": f,
            "wall": wall, "divB_final": divb, "calc": [s.Nx, s.Ny, s.Nz]}


def summary(r):
    h = r["h"]
    return {"best_iter": h["best_iter"], "best_sigma": h["best_sigma"], "stop_reason": h["stop_reason"],
            "final_iter": h["final_iter"], "final_sigma": h["final_sigma"], "iterations": len(h["sigma"]),
            "init_scalars": r["init_sc"], "step1_scalars": r["step_sc"], "wall_s": r["wall"],
            "divB_fraction_final": r["divB_final"],
            "source_diagnostics": {k: v for k, v in h["source_diagnostics"].items() if isinstance(v, float)}}


def run_case(name):
    bnd, spacing, shape, max_iter, analytic, extra, meta = CASES[name]()
    r64 = run(torch.float64, bnd, spacing, shape, max_iter)
    r32 = run(torch.float32, bnd, spacing, shape, max_iter)
    f64, f32 = r64["fields"], r32["fields"]
    dev = {
        "init_phi": rel(r32["init"]["phi"], r64["init"]["phi"]), "init_az": rel(r32["init"]["az"], r64["init"]["az"]),
        "init_B": rel(r32["init"]["B"], r64["init"]["B"]), "init_J": rel(r32["init"]["J"], r64["init"]["J"]),
        "step1_B": rel(r32["step1"]["B"], r64["step1"]["B"]), "step1_J": rel(r32["step1"]["J"], r64["step1"]["J"]),
        "final_B": rel(np.stack([f32[k] for k in ("Bx", "By", "Bz")]), np.stack([f64[k] for k in ("Bx", "By", "Bz")])),
        "final_J": rel(np.stack([f32[k] for k in ("Jx", "Jy", "Jz")]), np.stack([f64[k] for k in ("Jx", "Jy", "Jz")])),
    }
    roi = (slice(None), slice(None), slice(None))
    m32_vs_64 = compute_reference_metrics(f64, f32, roi)
    m64_self = compute_reference_metrics(f64, f64, roi)
    meta.update({
        "name": name, "shape": list(shape), "spacing": list(spacing), "ctor": POLICIES, "stop": STOP,
        "max_iter": max_iter, "calc_grid": r64["calc"],
        "fp64": summary(r64), "fp32": summary(r32), "fp32_vs_fp64_deviation": dev,
        "fp32_vs_fp64_metrics": m32_vs_64, "fp64_sigma_J_roi": m64_self["sigma_J"],
        "roi": "whole cropped (observed) volume",
    })
    out = {"bx_in": bnd[0], "by_in": bnd[1], "bz_in": bnd[2],
           "hist_sigma_fp64": np.array(r64["h"]["sigma"]), "hist_energy_fp64": np.array(r64["h"]["energy"]),
           "hist_divB_fp64": np.array(r64["h"]["divB"]), "hist_sigma_fp32": np.array(r32["h"]["sigma"]),
           "hist_energy_fp32": np.array(r32["h"]["energy"])}
    for k in ("Bx", "By", "Bz", "Jx", "Jy", "Jz"):
        out["final64_" + k + "_s4"] = f64[k][::4, ::4, ::4].astype(np.float32)
        out["final64_" + k + "_norm"] = np.array([np.linalg.norm(f64[k])])
    if analytic is not None:
        ref = {"Bx": analytic[0], "By": analytic[1], "Bz": analytic[2]}
        nzo = f64["Bx"].shape[0]
        ref = {k: v[:nzo] for k, v in ref.items()}
        meta["fp64_vs_analytic"] = compute_reference_metrics(ref, f64, roi)
        meta["fp32_vs_analytic"] = compute_reference_metrics(ref, f32, roi)
    out.update(extra)
    OUT.mkdir(exist_ok=True)
    np.savez_compressed(OUT / f"{name}.npz", **out)
    (OUT / f"{name}.json").write_text(json.dumps(meta, indent=1, sort_keys=True, default=float) + "\n")
    print(name, r64["calc"], "fp64", summary(r64)["stop_reason"], summary(r64)["best_iter"],
          f"{summary(r64)['best_sigma']:.6e}", "fp32", summary(r32)["stop_reason"], summary(r32)["best_iter"],
          f"{summary(r32)['best_sigma']:.6e}", json.dumps(dev), flush=True)


def td_points():
    """The reference TD generator on a small lattice with the benchmark's parameters."""
    from nfgs_b200.synthetic import td_params
    from nfgs._backend.td import generate_td_model

    out = {}
    for seed in (1, 5):
        p = td_params(seed)
        xs, ys, zs = np.linspace(-4, 4, 17), np.linspace(-4.5, 4.5, 15), np.linspace(0, 3, 7)
        X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
        b = generate_td_model(X, Y, Z, R=p["R"], a=p["a"], L=p["L"], d=p["d"], q=p["q"], I_0=p["I0"],
                              l_i=p["l_i"])
        out[f"seed{seed}_B"] = np.stack(b)
        out[f"seed{seed}_params"] = np.array([p[k] for k in ("R", "a", "d", "L", "q", "I0", "l_i")])
    out["grid"] = np.array([-4, 4, 17, -4.5, 4.5, 15, 0, 3, 7], dtype=np.float64)
    np.savez_compressed(Path(__file__).resolve().parent / "td99_points.npz", **out)


if __name__ == "__main__":
    torch.set_num_threads(int(os.environ.get("NFGS_THREADS", "8")))
    only = sys.argv[1:]
    if not only or "td99_points" in only:
        td_points()
    for name in CASES:
        if not only or name in only:
            run_case(name)

"""Large single solve: a quadrupolar magnetogram at 512 x 512 x 256 (calc
514 x 514 x 257), FP32, timed per phase and to the sigma_best stop, and
(--fp64) scored against an FP64 solve of the same boundary with the GPU
evaluation metrics (energy ratio, C_vec, E'_n, sigma_J, divB on the
observed box), fields compared on the device.

    python -m nfgs_b200.large_solve --fp64 --report large.json

The transforms (256 pairs per axis) run on the SIMT contractions by
default; NFGS_TC_WIDE=1 in the environment runs them on the four-role
tensor-core kernel (3x faster, but FP32 solves through it end twice as far
from the FP64 solve).  --soft also solves from the soft_cfcf start and
times both starts (iterate_begin with the start's evaluation, CUDA-synchronised
wall time, best of three).
"""

from __future__ import annotations

import argparse
import json
import os
import time

KW = dict(bottom_divergence_robin_weight=0.5, horizontal_zero_mode_policy="frozen_linear_harmonic",
          vertical_current_operator="staggered_face", d0_zero_mode_policy="project",
          source_zero_mode_policy="project")
STOP = dict(tol=1e-5, patience=40, sigma_improvement_tol=1e-5)


def _solver(n, nz, seed, dtype):
    from .solver import NFGSSolverGPU
    from .synthetic import quadrupole_magnetogram

    bx, by, bz = quadrupole_magnetogram(n, seed=seed)
    s = NFGSSolverGPU(n, n, nz, 1.0, 1.0, 1.0, dtype=dtype, **KW)
    s.set_bottom_vector_boundary(bx, by, bz, zero_net_current=False, smooth_passes=0, ijzbcor=3)
    return s


def _solve(s, max_iter, init_mode="gs_cfcf"):
    import torch

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    h = s.iterate(max_iter=max_iter, verbose=False, init_mode=init_mode, **STOP)
    torch.cuda.synchronize()
    return h, time.perf_counter() - t0


def _start_seconds(s, init_mode, reps=3):
    """Best wall time of a begun-and-ended iteration (the start state, its
    sigma_J, divB and energy), synchronised."""
    import torch

    best = float("inf")
    for _ in range(reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.iterate(max_iter=0, verbose=False, init_mode=init_mode, **STOP)
        torch.cuda.synchronize()
        best = min(best, time.perf_counter() - t0)
    return best


def main(argv=None):
    import torch

    from . import metrics as M

    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--nz", type=int, default=256)
    ap.add_argument("--seed", type=int, default=5)
    ap.add_argument("--max-iter", type=int, default=3000)
    ap.add_argument("--phase-iters", type=int, default=5)
    ap.add_argument("--fp64", action="store_true", help="also solve in FP64 and score the FP32 result against it")
    ap.add_argument("--soft", action="store_true", help="also solve from the soft_cfcf start and time both starts")
    ap.add_argument("--report", default=None)
    args = ap.parse_args(argv)

    out = {"grid": [args.n, args.n, args.nz], "seed": args.seed,
           "transforms": None}
    s = _solver(args.n, args.nz, args.seed, "float32")
    out["calc_grid"] = [s.Nx, s.Ny, s.Nz]
    wide = max(s.Nx, s.Ny) - 2 > 2 * 128
    tc = not os.environ.get("NFGS_DISABLE_TC") and (not wide or bool(os.environ.get("NFGS_TC_WIDE")))
    out["transforms"] = ("tcgen05 four-role" if wide else "tcgen05") if tc else "simt"
    cells = s.Nx * s.Ny * s.Nz
    s.iterate(max_iter=0, verbose=False)
    s._time_phases(2)
    ph = s._time_phases(args.phase_iters) / args.phase_iters
    out["phase_ms"] = dict(zip(("stencil", "forward_transforms", "z_solves", "inverse_transforms", "finalize"),
                               (float(v) for v in ph)))
    out["iteration_ms"] = float(ph.sum())
    out["gcell_iter_per_s"] = cells / (ph.sum() * 1e-3) / 1e9
    h, t = _solve(s, args.max_iter)
    out["fp32"] = {"iterations": len(h["sigma"]), "best_iter": h["best_iter"], "best_sigma": h["best_sigma"],
                   "stop_reason": h["stop_reason"], "seconds": t, "initial_sigma": h["initial_sigma"]}
    if args.soft:
        out["start_seconds"] = {m: _start_seconds(s, m) for m in ("gs_cfcf", "soft_cfcf")}
        hs, ts = _solve(s, args.max_iter, "soft_cfcf")
        out["fp32_soft_cfcf"] = {"iterations": len(hs["sigma"]), "best_iter": hs["best_iter"],
                                 "best_sigma": hs["best_sigma"], "stop_reason": hs["stop_reason"], "seconds": ts,
                                 "initial_sigma": hs["initial_sigma"],
                                 "soft_cfcf": hs["init_diagnostics"]["soft_cfcf"]}
    if args.fp64:
        s64 = _solver(args.n, args.nz, args.seed, "float64")
        h64, t64 = _solve(s64, args.max_iter)
        out["fp64"] = {"iterations": len(h64["sigma"]), "best_iter": h64["best_iter"],
                       "best_sigma": h64["best_sigma"], "stop_reason": h64["stop_reason"], "seconds": t64}
        f32 = s.fields_to_torch()
        f64 = s64.fields_to_torch()
        nz, ny, nx = (int(v) for v in f32.shape[1:])
        full = (slice(0, nz), slice(0, ny), slice(0, nx))
        m = M.field_metrics(f64[0:3], f32[0:3].double(), f32[3:6].double(), (s.dx, s.dy, s.dz), full)
        m64 = M.field_metrics(None, f64[0:3], f64[3:6], (s.dx, s.dy, s.dz), full)
        out["fp32_vs_fp64"] = {k: m[k] for k in ("C_vec", "C_CS", "Eprime_n", "Eprime_m", "epsilon", "sigma_J",
                                                   "sigma_J_common_fd2", "divB_normalized")}
        out["fp64_metrics"] = {k: m64[k] for k in ("sigma_J", "sigma_J_common_fd2", "divB_normalized")}
        del f32, f64, s64
        torch.cuda.empty_cache()
    print(json.dumps(out), flush=True)
    if args.report:
        with open(args.report, "w") as f:
            json.dump(out, f, indent=1)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())

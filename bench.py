#!/usr/bin/env python3
"""Benchmark of the NFGS reconstruction hot path on B200.

Workload (one GPU): the Titov-Demoulin flux rope of the reference's own
generator model (R=3, a=1, d=1.5, L=2; q and I0 from seed 1) on a
256x256x128 grid (calculation grid 258x258x129), rho = 0.5, FP32 storage,
gs_cfcf start.  One *step* is one NFGSSolverGPU.iterate() call of ITERS NFPT
iterations with the stop rule disabled, on a boundary that is already
resident on the device.  The metric is Gcell-iter/s on the calculation
grid (cells x iterations / device seconds, CUDA events on the solver's
stream, max over ranks).

  python bench.py [--gpus N --steps K --warmup W]            # B200 path
  python bench.py --impl reference [--steps K --warmup W]    # CPU reference arm

The reference arm runs the reference's own solver (nfgs_solver.NFGSSolverGPU
as installed in baseline/_ref by baseline/install_reference.sh) on the host
cores in FP32, one NFPT iteration (with its sigma_J / divB / energy) per
step; where that install is absent it times the CPU restatement of the
algorithm (the oracle, FP64) and says so.  The B200 line also carries the
reference's PyTorch CUDA path on the same GPU (``reference_torch_cuda``).
Under torchrun (N > 1) every rank solves its own replica (the path does
not shard); rank 0 prints the line.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import tempfile
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Gcell-iter/s (NFGS NFPT iterations, calc grid 258x258x129, TD99 flux rope 256x256x128)"
WORKLOAD = ("td99 flux rope (reference generator model, seed 1) 256x256x128 -> calc 258x258x129, rho=0.5, "
            "FP32, gs_cfcf start, NFPT iterations with sigma_J / divB / energy every iteration")
NX, NY, NZ = 256, 256, 128
EXTENT = 8.0
RHO = 0.5
# per calculation-grid cell and iteration: 19 volume passes x 4 B on the
# minimal data flow (stencil 5R+2W, forward 2R+2W, z-solves 2R+2W,
# inverse 2R+2W)
ALG_BYTES_PER_CELL_ITER = 76.0
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one launch of
# the dominant kernels on this workload, from one ncu capture each
KERNEL_TRAFFIC = {"stencil": 172.62e6 + 56.69e6}
REF_DIR = ROOT / "baseline" / "_ref"


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    return 6650.0, 1590.0, "fallback"


def boundary():
    from nfgs_b200.synthetic import td_bottom

    return td_bottom(NX, NY, seed=1, extent=EXTENT)


def solver_kwargs():
    return dict(bottom_divergence_robin_weight=RHO, horizontal_zero_mode_policy="frozen_linear_harmonic",
                vertical_current_operator="staggered_face", d0_zero_mode_policy="project",
                source_zero_mode_policy="project")


def spacing():
    h = 2 * EXTENT / (NX - 1)
    return h, h, h


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        # the raw samples (the JSON line carries their summary); NFGS_CLOCKS_DIR keeps them
        self.path = Path(os.environ.get("NFGS_CLOCKS_DIR", tempfile.gettempdir())) / f"nfgs_clocks_{index}.csv"

    def start(self):
        try:
            self.path.parent.mkdir(exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        for line in self.path.read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for n, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(rows)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta

        # one replica per GPU over NCCL; gloo where no GPU is visible (the
        # host-side logic of the replicas, tested on CPU)
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def barrier_sync(pg, local):
    import torch

    cuda = torch.cuda.is_available()
    if cuda:
        torch.cuda.synchronize(local)
    if pg is not None:
        pg.barrier()
        if cuda:
            torch.cuda.synchronize(local)


def max_over_ranks(pg, value: float, local: int) -> float:
    """The slowest replica's time: every rank gets the maximum."""
    if pg is None:
        return value
    import torch

    dev = f"cuda:{local}" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def reference_module():
    """The reference's own solver module as installed in baseline/_ref, or None."""
    if not (REF_DIR / "nfgs_solver.py").exists():
        return None
    if str(REF_DIR) not in sys.path:
        sys.path.insert(0, str(REF_DIR))
    import nfgs_solver

    return nfgs_solver


def _ref_cpu_solver(mod):
    import torch

    torch.set_num_threads(os.cpu_count() or 1)
    bx, by, bz = boundary()
    dx, dy, dz = spacing()
    s = mod.NFGSSolverGPU(NX, NY, NZ, dx, dy, dz, device="cpu", dtype=torch.float32, calculation_domain_mode="mudpack",
                          record_iteration_diagnostics=False, **solver_kwargs())
    s.set_bottom_vector_boundary(bx, by, bz, zero_net_current=False, smooth_passes=0, ijzbcor=3)
    return s


def _ref_step(s, st):
    """One NFPT iteration of the reference with the diagnostics its iterate
    takes every iteration (nfgs_solver.py:3656-3679)."""
    st = s.iteration_step(*st, mu=1.0)
    s.compute_sigma(st[0], st[1])
    s.compute_divB(st[0])
    s.compute_energy(st[0])
    return st


def cpu_reference_rate(max_iters: int = 10, budget_s: float = 25.0) -> dict:
    """Reference CPU Gcell-iter/s on this workload: the reference's own FP32
    code on all host threads (one warm-up iteration, then up to max_iters
    timed iterations within budget_s, at least 3); the FP64 oracle port when
    the reference install is absent."""
    mod = reference_module()
    if mod is None:
        return cpu_port_rate(iters=2)
    import torch

    s = _ref_cpu_solver(mod)
    with torch.inference_mode():
        st = s.compute_initial_conditions(init_mode="gs_cfcf")
        st = _ref_step(s, st)
        n, t0 = 0, time.perf_counter()
        while n < max_iters and (n < 3 or time.perf_counter() - t0 < budget_s):
            st = _ref_step(s, st)
            n += 1
        dt = time.perf_counter() - t0
    cells = s.Nx * s.Ny * s.Nz
    return {"value": cells * n / dt / 1e9, "unit": "Gcell-iter/s", "cores": torch.get_num_threads(),
            "kind": "reference",
            "sample": f"{n} NFPT iterations (iteration_step + sigma_J/divB/energy) of the reference nfgs_solver "
                      f"(torch CPU, FP32) on the same {s.Nx}x{s.Ny}x{s.Nz} workload after its gs_cfcf start and one "
                      f"warm-up iteration; {dt:.1f} s on {torch.get_num_threads()} threads"}


def cpu_port_rate(iters: int = 2) -> dict:
    """Oracle (CPU restatement of the reference, FP64) Gcell-iter/s on this workload."""
    from oracle.nfgs_oracle import OracleNFGS

    bx, by, bz = boundary()
    dx, dy, dz = spacing()
    o = OracleNFGS(NX, NY, NZ, dx, dy, dz, **{k: v for k, v in solver_kwargs().items()
                                               if k != "vertical_current_operator"})
    o.set_bottom_vector_boundary(bx, by, bz, zero_net_current=False, smooth_passes=0, ijzbcor=3)
    st = o.compute_initial_conditions()
    t0 = time.perf_counter()
    for _ in range(iters):
        st = o.iteration_step(*st)
        o.compute_sigma(st[0], st[1])
        o.compute_divB(st[0])
        o.compute_energy(st[0])
    dt = time.perf_counter() - t0
    cells = o.Nx * o.Ny * o.Nz
    return {"value": cells * iters / dt / 1e9, "unit": "Gcell-iter/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"{iters} NFPT iterations (+ sigma/divB/energy) of the FP64 NumPy/SciPy oracle on the "
                      f"same {o.Nx}x{o.Ny}x{o.Nz} workload after its gs_cfcf start; {dt:.1f} s; transforms on "
                      f"{os.cpu_count()} threads, element-wise work on one (reference install absent)"}


def run_reference(args):
    world, rank = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    mod = reference_module()
    if mod is None:
        return run_reference_port(args, world)
    import torch

    s = _ref_cpu_solver(mod)
    cells = s.Nx * s.Ny * s.Nz
    with torch.inference_mode():
        st = s.compute_initial_conditions(init_mode="gs_cfcf")
        for _ in range(args.warmup):
            st = _ref_step(s, st)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            st = _ref_step(s, st)
        dt = time.perf_counter() - t0
    value = cells * args.steps / dt / 1e9
    threads = torch.get_num_threads()
    line = {
        "metric": METRIC, "value": value, "unit": "Gcell-iter/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (TD99 flux rope of the reference generator model, seed 1)",
        "config": {"workload": WORKLOAD, "grid": [NX, NY, NZ], "calc_grid": [s.Nx, s.Ny, s.Nz], "iters_per_step": 1},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "Gcell-iter/s", "cores": threads, "kind": "reference",
                         "sample": f"{args.steps} timed NFPT iterations (iteration_step + sigma_J/divB/energy) of the "
                                   f"reference nfgs_solver, torch CPU FP32 on {threads} threads, after its gs_cfcf "
                                   f"start and {args.warmup} warm-up iterations"},
        "e2e": {"value": value, "unit": "Gcell-iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_reference_port(args, world):
    from oracle.nfgs_oracle import OracleNFGS

    bx, by, bz = boundary()
    dx, dy, dz = spacing()
    o = OracleNFGS(NX, NY, NZ, dx, dy, dz, **{k: v for k, v in solver_kwargs().items()
                                               if k != "vertical_current_operator"})
    o.set_bottom_vector_boundary(bx, by, bz, zero_net_current=False, smooth_passes=0, ijzbcor=3)
    st = o.compute_initial_conditions()
    cells = o.Nx * o.Ny * o.Nz
    for _ in range(args.warmup):
        st = o.iteration_step(*st)
        o.compute_sigma(st[0], st[1])
    t0 = time.perf_counter()
    for _ in range(args.steps):
        st = o.iteration_step(*st)
        o.compute_sigma(st[0], st[1])
        o.compute_divB(st[0])
        o.compute_energy(st[0])
    dt = time.perf_counter() - t0
    value = cells * args.steps / dt / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "Gcell-iter/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (TD99 flux rope of the reference generator model, seed 1)",
        "config": {"workload": WORKLOAD, "grid": [NX, NY, NZ], "calc_grid": [o.Nx, o.Ny, o.Nz], "iters_per_step": 1},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "Gcell-iter/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": f"{args.steps} timed NFPT iterations of the FP64 NumPy/SciPy restatement of the "
                                   f"reference algorithm (reference install absent); transforms on {os.cpu_count()} "
                                   f"threads"},
        "e2e": {"value": value, "unit": "Gcell-iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def reference_torch_cuda(dev: str, iters: int, mine: dict) -> dict | None:
    """The reference's PyTorch CUDA path on the same GPU, same boundary and
    FP32 production kwargs (examples/reconstruct_npz.py:31-40 plus the
    projection policies): Gcell-iter/s of iterate() with the stop rule off
    (init included, as in this bench's own steps), and its time to the
    production sigma_J stop, beside this build's figures."""
    mod = reference_module()
    if mod is None:
        return {"unavailable": "reference install (baseline/_ref) absent"}
    import torch

    bx, by, bz = boundary()
    dx, dy, dz = spacing()
    s = mod.NFGSSolverGPU(NX, NY, NZ, dx, dy, dz, device=dev, dtype=torch.float32, calculation_domain_mode="mudpack",
                          record_iteration_diagnostics=False, **solver_kwargs())
    s.set_bottom_vector_boundary(bx, by, bz, zero_net_current=False, smooth_passes=0, ijzbcor=3)
    cells = s.Nx * s.Ny * s.Nz
    off = dict(tol=1e-30, mu=1.0, patience=0, sigma_improvement_tol=None, verbose=False, init_mode="gs_cfcf")
    with torch.inference_mode():
        s.iterate(max_iter=2, **off)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        s.iterate(max_iter=iters, **off)
        torch.cuda.synchronize(dev)
        dt = time.perf_counter() - t0
        t1 = time.perf_counter()
        h = s.iterate(max_iter=3000, tol=1e-5, mu=1.0, patience=40, sigma_improvement_tol=1e-5, verbose=False,
                      init_mode="gs_cfcf", stop_mode="sigma_best")
        torch.cuda.synchronize(dev)
        dstop = time.perf_counter() - t1
    rate = cells * iters / dt / 1e9
    out = {"value": rate, "unit": "Gcell-iter/s", "iters": iters, "seconds": dt,
           "plain_over_reference": mine["value"] / rate,
           "time_to_sigma_stop": {"seconds": dstop, "iterations": len(h["sigma"]), "best_iter": h["best_iter"],
                                  "best_sigma": h["best_sigma"], "stop_reason": h["stop_reason"]},
           "note": "reference nfgs_solver.NFGSSolverGPU on the same B200, torch CUDA FP32, wall time with "
                   "torch.cuda.synchronize brackets; iterate() of the stop-rule-off workload includes its gs_cfcf "
                   "start like this bench's steps"}
    if mine.get("stop"):
        out["time_to_sigma_stop"]["plain_over_reference"] = dstop / mine["stop"]["seconds"]
    del s
    torch.cuda.empty_cache()
    return out


def learned_vs_plain(seeds=(1_000_000, 1_000_001, 1_000_002), eps=1e-3):
    """Time to sigma* (1 + eps) from the gs_cfcf start and from the learned
    start on held-out sunspot magnetograms at 256x256x128 (the network was
    trained at 128x128x64); sigma* is the plain run's best sigma_J."""
    from nfgs_b200 import learned as LN
    from nfgs_b200 import warmstart_train as W

    model = LN.NeuralOperator.load(ROOT / "nfgs_b200" / "weights" / "warmstart_sunspots_130x130x65.npz")
    rows = W.evaluate(model, list(seeds), 256, 128, eps=(eps,), log=lambda m: None)
    tag = f"eps{eps:g}"
    tp = sum(r[tag]["plain_s"] for r in rows)
    tl = sum(r[tag]["learned_s"] for r in rows)
    return {"workload": "held-out seeded sunspot magnetograms 256x256x128 (calc 258x258x129), FP32, rho=0.5",
            "target": f"sigma <= sigma_plain_best * (1 + {eps:g}), same stop rule",
            "plain_s": tp, "learned_s": tl, "speedup": tp / tl if tl > 0 else None,
            "accepted": sum(int(r[tag]["learned_accepted"]) for r in rows), "solves": len(rows),
            "rows": [{"seed": r["seed"], "plain_s": r[tag]["plain_s"], "plain_iterations": r[tag]["plain_iterations"],
                      "learned_s": r[tag]["learned_s"], "learned_iterations": r[tag]["learned_iterations"],
                      "accepted": r[tag]["learned_accepted"]} for r in rows]}


def run_b200(args):
    world, rank, local, pg = dist_setup()
    import torch  # noqa: F401  (device plumbing and synchronisation only)

    from nfgs_b200 import NFGSSolverGPU

    bx, by, bz = boundary()
    dx, dy, dz = spacing()
    dev = f"cuda:{local}"
    s = NFGSSolverGPU(NX, NY, NZ, dx, dy, dz, device=dev, dtype="float32", **solver_kwargs())
    cells = s.Nx * s.Ny * s.Nz
    s.set_bottom_vector_boundary(bx, by, bz, zero_net_current=False, smooth_passes=0, ijzbcor=3)
    it_kw = dict(max_iter=args.iters, tol=1e-30, patience=0, sigma_improvement_tol=None, verbose=False,
                 check_every=args.check_every)
    for _ in range(args.warmup):
        s.iterate(**it_kw)
    clocks = Clocks(local)
    barrier_sync(pg, local)
    clocks.start()
    dev_ms = 0.0
    launches = 0
    for _ in range(args.steps):
        h = s.iterate(**it_kw)
        dev_ms += h["device_ms"]
        launches += h["kernel_launches"]
    barrier_sync(pg, local)
    ck = clocks.stop()
    dev_ms = max_over_ranks(pg, dev_ms, local)
    total_iters = args.iters * args.steps
    value = cells * total_iters * world / (dev_ms / 1e3) / 1e9

    # end to end through the public API with host buffers: boundary H2D,
    # set-up, iterate, fields D2H, every step
    # (one untimed step first, as a caller reconstructing one magnetogram
    # after another sees it: the host block of the exported fields is
    # page-locked once and reused once the previous result is dropped)
    e2e_times = []
    fields_bytes = 0
    for step in range(1 + max(1, min(args.steps, 3))):
        barrier_sync(pg, local)
        t0 = time.perf_counter()
        s2 = NFGSSolverGPU(NX, NY, NZ, dx, dy, dz, device=dev, dtype="float32", **solver_kwargs())
        s2.set_bottom_vector_boundary(bx, by, bz, zero_net_current=False, smooth_passes=0, ijzbcor=3)
        s2.iterate(**it_kw)
        f = s2.fields_to_numpy()
        barrier_sync(pg, local)
        if step > 0:
            e2e_times.append(time.perf_counter() - t0)
        fields_bytes = 6 * f["Bx"].size * f["Bx"].itemsize
        del s2, f
    e2e_s = max_over_ranks(pg, statistics.median(e2e_times), local)
    e2e_value = cells * args.iters * world / e2e_s / 1e9

    # phase breakdown of the iteration (CUDA events on the solver stream)
    s.iterate(max_iter=0, verbose=False)
    ph = s._time_phases(args.phase_iters)
    ph_ms = ph / args.phase_iters
    names = ["stencil", "forward_transforms", "z_solves", "inverse_transforms", "finalize"]
    dom = int(np.argmax(ph_ms))
    hbm_gbs, bf16_tf, peak_src = load_peaks()
    # algorithmic bytes / flops per launch group (per iteration)
    alg_bytes = {"stencil": 28.0 * cells, "forward_transforms": 16.0 * cells, "z_solves": 16.0 * cells,
                 "inverse_transforms": 16.0 * cells, "finalize": 4.0 * s.Nx * s.Ny}
    tr_flops = 2.0 * cells * (s.Nx + s.Ny) * 2  # two chains x (x and y) x 2N per output element
    dname = names[dom]
    if dname in ("forward_transforms", "inverse_transforms"):
        achieved = tr_flops / (ph_ms[dom] / 1e3) / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": bf16_tf, "unit": "TFLOP/s",
                "frac": achieved / bf16_tf, "traffic": None, "kernel": dname,
                "note": f"peak = {peak_src} bf16 dense; dense FP32-equivalent transform flops"}
    else:
        achieved = alg_bytes[dname] / (ph_ms[dom] / 1e3) / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": hbm_gbs, "unit": "GB/s", "frac": achieved / hbm_gbs,
                "traffic": KERNEL_TRAFFIC.get(dname), "algorithmic_bytes": alg_bytes[dname], "kernel": dname,
                "note": f"peak = {peak_src} HBM copy bandwidth; traffic = ncu DRAM bytes of one launch"}
    iter_ms = float(ph_ms.sum())
    whole = {"achieved_gbs": ALG_BYTES_PER_CELL_ITER * cells / (iter_ms / 1e3) / 1e9,
             "frac_of_hbm": ALG_BYTES_PER_CELL_ITER * cells / (iter_ms / 1e3) / 1e9 / hbm_gbs,
             "iteration_ms": iter_ms, "phase_ms": {n: float(v) for n, v in zip(names, ph_ms)}}

    # time to the sigma_J stop with the production stop rule
    t_stop = None
    if args.stop_run:
        h = s.iterate(max_iter=3000, tol=1e-5, patience=40, sigma_improvement_tol=1e-5, verbose=False,
                      check_every=args.check_every)
        t_stop = {"seconds": h["device_ms"] / 1e3, "iterations": len(h["sigma"]), "best_iter": h["best_iter"],
                  "best_sigma": h["best_sigma"], "stop_reason": h["stop_reason"]}
    lvp = None
    if world == 1 and args.learned:
        lvp = learned_vs_plain()
    ref_cuda = None
    if rank == 0 and world == 1 and args.ref_cuda:
        ref_cuda = reference_torch_cuda(dev, args.ref_cuda_iters, {"value": value, "stop": t_stop})
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_reference_rate(max_iters=args.cpu_iters)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Gcell-iter/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (TD99 flux rope of the reference generator model, seed 1)",
            "config": {"workload": WORKLOAD, "grid": [NX, NY, NZ], "calc_grid": [s.Nx, s.Ny, s.Nz],
                       "iters_per_step": args.iters, "stop_rule": "off (one iterate() call of iters_per_step)",
                       "parallelism": f"replicas x{world}",
                       "l2": "working set > L2: each iteration streams phi, A_z and the 103 MB background"},
            "e2e": {"value": e2e_value, "unit": "Gcell-iter/s", "h2d_bytes_per_step": 3 * NX * NY * 8,
                    "d2h_bytes_per_step": fields_bytes, "seconds_per_step": e2e_s},
            "roofline": roof,
            "iteration_roofline": whole,
            "gpu_launches": launches,
            "clocks": ck,
            "time_to_sigma_stop": t_stop,
            "learned_vs_plain": lvp,
            "reference_torch_cuda": ref_cuda,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def run_window(args):
    import torch

    from nfgs_b200 import NFGSSolverGPU

    bx, by, bz = boundary()
    dx, dy, dz = spacing()
    s = NFGSSolverGPU(NX, NY, NZ, dx, dy, dz, device="cuda:0", dtype="float32", **solver_kwargs())
    s.set_bottom_vector_boundary(bx, by, bz, zero_net_current=False, smooth_passes=0, ijzbcor=3)
    s.iterate(max_iter=0, verbose=False)
    s._time_phases(1)
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    ms = s._time_phases(args.phase_iters)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    print(json.dumps({"phase_ms_per_iter": (ms / args.phase_iters).tolist()}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--iters", type=int, default=100)
    ap.add_argument("--check-every", type=int, default=50)
    ap.add_argument("--phase-iters", type=int, default=10)
    ap.add_argument("--cpu-iters", type=int, default=10)
    ap.add_argument("--ref-cuda-iters", type=int, default=20)
    ap.add_argument("--no-ref-cuda", dest="ref_cuda", action="store_false",
                    help="skip the reference PyTorch CUDA leg")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-stop-run", dest="stop_run", action="store_false")
    ap.add_argument("--no-learned", dest="learned", action="store_false",
                    help="skip the learned-vs-plain time-to-sigma measurement")
    ap.add_argument("--ncu-window", action="store_true",
                    help="profile window only: set-up, then --phase-iters iterations between "
                         "cudaProfilerStart/Stop (for ncu --profile-from-start off)")
    args = ap.parse_args()
    if args.ncu_window:
        return run_window(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())

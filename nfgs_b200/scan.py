"""Batched weight x rho scan: many NFGS solves advanced together.

The reference runs its TD weight x rho sweeps as a serial loop of solves
(run_nfgs_td_robin_weight_sweep.py:510-660).  Here every solve of the scan is
begun on its own handle (gs_cfcf start, per-iteration CUDA graph captured),
and one CUDA graph holding `iters` iterations of every solve -- independent
chains, so solves of different sizes fill the GPU together -- is launched
until every solve has met its stop rule.  Solves that stopped skip their work
on the device, and the graph is rebuilt from the running solves whenever
half have stopped; the results are those of the same solves run one by one.
The solvers are set up by a thread pool (the first of each grid shape alone,
so that the fused stencil's per-shape z-segment tuning runs on a quiet GPU);
run_scan_overlapped starts launching with those first solves and joins the
others to the running scan between launches as the threads finish them.

    python -m nfgs_b200.scan --boundaries 33 --overlap --serial --report scan.json

Under torchrun (one process per GPU) the solves are dealt round-robin to the
ranks, each rank runs its share as one batched scan, and rank 0 reports the
gathered results (replicas: no data crosses GPUs).
"""

from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import time

import numpy as np

from . import _lib as L
from .solver import NFGSSolverGPU
from .synthetic import td_bottom

GRIDS = ((128, 64), (160, 80), (192, 96), (224, 112), (256, 128))
RHOS = (0.0, 0.3, 0.5, 0.7, 1.0)
KW = dict(dtype="float32", horizontal_zero_mode_policy="frozen_linear_harmonic",
          vertical_current_operator="staggered_face", d0_zero_mode_policy="project",
          source_zero_mode_policy="project")
STOP = dict(tol=1e-5, patience=40, sigma_improvement_tol=1e-5)


def td_scan_cases(n_boundaries: int = 33, rhos=RHOS, seed: int = 0, grids=GRIDS, extent: float = 8.0):
    """Seeded TD-type boundaries (R in [2,4], a in [0.6,1.2], d in [1,2],
    twist from the seeded current) on grids drawn from `grids`, each at
    every rho."""
    rng = np.random.default_rng(seed)
    cases = []
    for b in range(n_boundaries):
        R, a, d = rng.uniform(2.0, 4.0), rng.uniform(0.6, 1.2), rng.uniform(1.0, 2.0)
        n, nz = grids[int(rng.integers(len(grids)))]
        bx, by, bz = td_bottom(n, n, seed=seed * 1000 + b, extent=extent, R=R, a=a, d=d)
        h = 2 * extent / (n - 1)
        for rho in rhos:
            cases.append(dict(boundary=b, n=n, nz=nz, rho=float(rho), R=R, a=a, d=d, h=h, bx=bx, by=by, bz=bz))
    return cases


def _solver(case):
    s = NFGSSolverGPU(case["n"], case["n"], case["nz"], case["h"], case["h"], case["h"],
                      bottom_divergence_robin_weight=case["rho"], **KW)
    s.set_bottom_vector_boundary(case["bx"], case["by"], case["bz"], zero_net_current=False, smooth_passes=0,
                                 ijzbcor=3)
    return s


def run_scan(cases, iters: int = 8, max_iter: int = 3000, stop=STOP, workers: int = 8):
    """All cases in one batched run; returns (histories, timings).  The
    solvers are set up (created, boundary, gs_cfcf start) by `workers`
    threads: each handle has its own stream and the library's shared state
    is locked, and the set-up is mostly host work and synchronous copies."""
    import torch
    from concurrent.futures import ThreadPoolExecutor

    def begin(c):
        s = _solver(c)
        return s, s._iterate_begin(max_iter=max_iter, verbose=False, use_graph=True, **stop)

    t0 = time.perf_counter()
    # the first solve of each grid shape alone (its stencil tuning runs on a
    # quiet GPU), then the rest concurrently
    firsts, seen = [], set()
    for q, c in enumerate(cases):
        if (c["n"], c["nz"]) not in seen:
            seen.add((c["n"], c["nz"]))
            firsts.append(q)
    pairs = [None] * len(cases)
    for q in firsts:
        pairs[q] = begin(cases[q])
    rest = [q for q in range(len(cases)) if pairs[q] is None]
    if workers > 1:
        with ThreadPoolExecutor(max_workers=workers) as ex:
            for q, pr in zip(rest, ex.map(lambda q: begin(cases[q]), rest)):
                pairs[q] = pr
    else:
        for q in rest:
            pairs[q] = begin(cases[q])
    solvers = [p[0] for p in pairs]
    ctxs = [p[1] for p in pairs]
    lib = L.lib()
    arr = (C.c_void_p * len(solvers))(*[s._h.value if isinstance(s._h, C.c_void_p) else s._h for s in solvers])
    scan = C.c_void_p()
    L.check(lib.nfgs_scan_create(arr, len(solvers), iters, C.byref(scan)))
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    launches = 0
    active = C.c_int32(len(solvers))
    try:
        while active.value > 0 and launches * iters < max_iter + iters:
            L.check(lib.nfgs_scan_launch(scan, C.byref(active)))
            launches += 1
    finally:
        t2 = time.perf_counter()
        L.check(lib.nfgs_scan_destroy(scan))
    hists = [s._iterate_finish(ctx) for s, ctx in zip(solvers, ctxs)]
    cells_iters = sum(s.Nx * s.Ny * s.Nz * len(h["sigma"]) for s, h in zip(solvers, hists))
    timing = dict(setup_s=t1 - t0, scan_s=t2 - t1, graph_launches=launches, iters_per_launch=iters,
                  cell_iterations=cells_iters, gcell_iter_per_s=cells_iters / (t2 - t1) / 1e9)
    del solvers
    return hists, timing


def run_scan_overlapped(cases, iters: int = 8, max_iter: int = 3000, stop=STOP, workers: int = 8):
    """All cases in one batched run whose launches start while the solves
    are still being set up: the first solve of each grid shape is begun
    alone (its stencil tuning on a quiet GPU) and starts the scan; the
    others are begun by `workers` threads and joined to the scan between
    launches (nfgs_scan_add).  Returns (histories, timings); the wall time
    counts set-up and iterations together."""
    import torch
    from concurrent.futures import FIRST_COMPLETED, ThreadPoolExecutor, wait

    def begin(q):
        s = _solver(cases[q])
        return q, s, s._iterate_begin(max_iter=max_iter, verbose=False, use_graph=True, **stop)

    def hptr(s):
        return s._h.value if isinstance(s._h, C.c_void_p) else s._h

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    firsts, seen = [], set()
    for q, c in enumerate(cases):
        if (c["n"], c["nz"]) not in seen:
            seen.add((c["n"], c["nz"]))
            firsts.append(q)
    pairs = [None] * len(cases)
    for q in firsts:
        _, s, ctx = begin(q)
        pairs[q] = (s, ctx)
    lib = L.lib()
    arr = (C.c_void_p * len(firsts))(*[hptr(pairs[q][0]) for q in firsts])
    scan = C.c_void_p()
    L.check(lib.nfgs_scan_create(arr, len(firsts), iters, C.byref(scan)))
    launches, joins = 0, 0
    active = C.c_int32(len(firsts))
    ex = ThreadPoolExecutor(max_workers=workers)
    try:
        pending = {ex.submit(begin, q) for q in range(len(cases)) if pairs[q] is None}
        while pending or active.value > 0:
            if pending:
                # join what is ready; wait for one only when nothing else runs
                done, pending = wait(pending, timeout=None if active.value == 0 else 0,
                                     return_when=FIRST_COMPLETED)
                ready = [f.result() for f in done]
                if ready:
                    for q, s, ctx in ready:
                        pairs[q] = (s, ctx)
                    add = (C.c_void_p * len(ready))(*[hptr(s) for _, s, _ in ready])
                    L.check(lib.nfgs_scan_add(scan, add, len(ready)))
                    active.value += len(ready)
                    joins += 1
            if active.value > 0:
                L.check(lib.nfgs_scan_launch(scan, C.byref(active)))
                launches += 1
    finally:
        ex.shutdown(wait=True)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        L.check(lib.nfgs_scan_destroy(scan))
    solvers = [p[0] for p in pairs]
    hists = [s._iterate_finish(ctx) for s, (_, ctx) in zip(solvers, pairs)]
    cells_iters = sum(s.Nx * s.Ny * s.Nz * len(h["sigma"]) for s, h in zip(solvers, hists))
    timing = dict(wall_s=t1 - t0, graph_launches=launches, joins=joins, iters_per_launch=iters,
                  cell_iterations=cells_iters, gcell_iter_per_s=cells_iters / (t1 - t0) / 1e9)
    del solvers
    return hists, timing


def run_serial(cases, max_iter: int = 3000, stop=STOP):
    """The same solves one after another (each its own iterate call)."""
    import torch

    hists, t_iter = [], 0.0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for c in cases:
        s = _solver(c)
        torch.cuda.synchronize()
        t = time.perf_counter()
        hists.append(s.iterate(max_iter=max_iter, verbose=False, **stop))
        torch.cuda.synchronize()
        t_iter += time.perf_counter() - t
        del s
    torch.cuda.synchronize()
    return hists, dict(serial_iterate_s=t_iter, serial_total_s=time.perf_counter() - t0)


def shard_cases(cases, rank: int, world: int):
    """Indices of the cases of one replica: round-robin over the list, which
    mixes the grid sizes of every boundary across the ranks."""
    return list(range(rank, len(cases), world))


def distributed_scan(cases, pg, rank: int, world: int, runner=None, **kw):
    """Under torchrun: each rank runs its share of the solves as one batched
    scan on its GPU (the solves are independent; no data crosses ranks), then
    the per-solve results and timings are gathered to every rank.  Returns
    (results in case order, timing); timing's scan_s is the slowest rank's."""
    runner = run_scan if runner is None else runner
    mine = shard_cases(cases, rank, world)
    hists, timing = runner([cases[i] for i in mine], **kw)
    slim = [dict(best_sigma=h["best_sigma"], best_iter=h["best_iter"], iterations=len(h["sigma"]),
                 stop_reason=h["stop_reason"], sigma=list(h["sigma"])) for h in hists]
    parts = [None] * world
    pg.all_gather_object(parts, (mine, slim, timing))
    results = [None] * len(cases)
    for idx, res, _t in parts:
        for i, r in zip(idx, res):
            results[i] = r
    cells = sum(t["cell_iterations"] for _, _, t in parts)
    scan_s = max(t["scan_s"] for _, _, t in parts)
    timing = dict(setup_s=max(t["setup_s"] for _, _, t in parts), scan_s=scan_s, ranks=world,
                  cell_iterations=cells, gcell_iter_per_s=cells / scan_s / 1e9,
                  per_rank=[t for _, _, t in parts])
    return results, timing


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--boundaries", type=int, default=33)
    ap.add_argument("--iters", type=int, default=8)
    ap.add_argument("--max-iter", type=int, default=3000)
    ap.add_argument("--serial", action="store_true", help="also run the solves one by one and compare")
    ap.add_argument("--overlap", action="store_true",
                    help="also run the batch with set-up overlapped by the launches (wall time counts both)")
    ap.add_argument("--report", default=None)
    args = ap.parse_args(argv)
    cases = td_scan_cases(args.boundaries)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1:
        # replicas: one GPU per rank, each with its share of the solves
        import torch
        import torch.distributed as dist
        from datetime import timedelta

        rank, local = int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
        try:
            results, timing = distributed_scan(cases, dist, rank, world, iters=args.iters, max_iter=args.max_iter)
        finally:
            dist.destroy_process_group()
        if rank == 0:
            out = dict(solves=len(cases), timing=timing,
                       results=[dict(boundary=c["boundary"], n=c["n"], nz=c["nz"], rho=c["rho"],
                                     **{k: r[k] for k in ("best_sigma", "best_iter", "iterations", "stop_reason")})
                                for c, r in zip(cases, results)])
            print(json.dumps({k: v for k, v in out.items() if k != "results"}), flush=True)
            if args.report:
                with open(args.report, "w") as f:
                    json.dump(out, f, indent=1)
        return 0
    hists, timing = run_scan(cases, args.iters, args.max_iter)
    out = dict(solves=len(cases), timing=timing,
               results=[dict(boundary=c["boundary"], n=c["n"], nz=c["nz"], rho=c["rho"],
                             best_sigma=h["best_sigma"], best_iter=h["best_iter"], iterations=len(h["sigma"]),
                             stop_reason=h["stop_reason"]) for c, h in zip(cases, hists)])
    if args.overlap:
        oh, ot = run_scan_overlapped(cases, args.iters, args.max_iter)
        out["overlapped"] = ot
        out["overlapped_identical_histories"] = all(a["sigma"] == b["sigma"] for a, b in zip(hists, oh))
    if args.serial:
        sh, st = run_serial(cases, args.max_iter)
        out["serial"] = st
        out["identical_histories"] = all(a["sigma"] == b["sigma"] for a, b in zip(hists, sh))
        out["speedup_vs_serial_iterate"] = st["serial_iterate_s"] / timing["scan_s"]
        if args.overlap:
            out["overlapped_speedup_vs_serial_total"] = st["serial_total_s"] / out["overlapped"]["wall_s"]
    print(json.dumps({k: v for k, v in out.items() if k != "results"}), flush=True)
    if args.report:
        with open(args.report, "w") as f:
            json.dump(out, f, indent=1)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())

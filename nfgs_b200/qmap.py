"""Field-line tracing and squashing-factor (Q) maps on the GPU.

Drop-in for the reference's topology-map helpers
``compute_y0_qmap`` / ``compute_bottom_qmap``
(nfgs/_backend/util/fastqsl_plane.py:203-506), which trace every seed of a
plane with FastQSL through CuPy and evaluate Q with its QCalcPlane.  Here,
by default (``q_method="fastqsl"``), the library restates both on device
tensors: ``nfgs_trace_fastqsl`` traces every seed with FastQSL's adaptive
RKF4(5) step control, face handling and limits in FP32, and
``nfgs_qcalc_plane`` forms QCalcPlane's Q; flags are FastQSL's face codes
(1..6 for x min, x max, y min, y max, z min, z max, 0 stopped inside, 42
through an edge or corner).  Nothing of the field goes through the host when
it is passed as a CUDA tensor, e.g. from ``NFGSSolverGPU.fields_to_torch()``.
``block_x`` and ``trace_chunk_seeds`` are recorded only (every seed is
launched at once) and ``fastqsl_root`` is ignored.  ``include_twist=True``
integrates J.B / (4 pi |B|^2) along both halves of each line, J the centred
grid curl (fastqsl_plane.py:287-305).

Two other methods use the library's fixed-step RK4 tracer
(``nfgs_trace_field_lines``: trilinear B, ends snapped onto the face a line
leaves through; flags 1..6 for x=0, x=nx-1, y=0, y=ny-1, z=0, z=nz-1, 0
unfinished, -1 zero field): ``q_method="perp"``, Titov's (2007) Q_perp from
four more lines offset by +-delta perpendicular to B (``nfgs_trace_qperp``),
which is defined also where B lies in the seed plane (By = 0 on the y = 0
midplane of a symmetric rope, where the seed-plane forms divide by
Bn0 = 0), and ``q_method="plane"``, Q = ||D||^2/|det D| of the footpoint map
from central differences over the seed grid (``nfgs_qmap_plane``).

    python -m nfgs_b200.qmap --n 256 --nz 128 --report qmap.json
"""

from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import time

import numpy as np

from . import _lib as L

Y0_PLANE_COORDINATE_CONTRACT = "physical_midplane_fractional_index_v2"


def _torch():
    import torch

    return torch


def physical_midplane_grid_index(n_nodes: int) -> float:
    """Grid coordinate of the physical midpoint of a node axis
    (fastqsl_plane.py:49-54)."""
    n = int(n_nodes)
    if n < 1:
        raise ValueError(f"n_nodes must be positive, got {n_nodes}")
    return 0.5 * float(n - 1)


def _volume(bx, by, bz, dtype):
    """(3, nz, ny, nx) contiguous CUDA tensor of dtype from three arrays or tensors."""
    torch = _torch()
    comps = []
    for a in (bx, by, bz):
        t = a if isinstance(a, torch.Tensor) else torch.as_tensor(np.asarray(a))
        comps.append(t.to(device="cuda", dtype=dtype))
    if comps[0].ndim != 3 or comps[0].shape != comps[1].shape or comps[0].shape != comps[2].shape:
        raise ValueError("bx, by, and bz must have the same (nz,ny,nx) shape")
    return torch.stack(comps).contiguous()


def spectral_gaussian_lowpass(b, sigma_cells: float):
    """Isotropic Gaussian low-pass of each component in Fourier space, sigma in
    cells (fastqsl_plane.py:82-101), on the device; b (3, nz, ny, nx)."""
    torch = _torch()
    sigma = float(sigma_cells)
    if sigma <= 0.0:
        return b
    if not bool(torch.isfinite(b).all()):
        raise ValueError("field must be finite for spectral filtering")
    shape = b.shape[1:]
    k2 = None
    for ax, n in enumerate(shape):
        f = torch.fft.fftfreq(n, dtype=torch.float64, device=b.device) ** 2
        view = [1, 1, 1]
        view[ax] = n
        f = f.view(view)
        k2 = f if k2 is None else k2 + f
    transfer = torch.exp(-0.5 * ((2.0 * math.pi * sigma) ** 2) * k2)
    out = torch.fft.ifftn(torch.fft.fftn(b.double(), dim=(1, 2, 3)) * transfer, dim=(1, 2, 3)).real
    return out.to(torch.float32).to(b.dtype).contiguous()


def trace_field_lines(b, seeds, *, normal=(0.0, 0.0, 1.0), step_len: float = 1.0 / 8.0, max_steps=None,
                      twist: bool = False):
    """Trace seeds (n, 3 xyz grid units) through b (3, nz, ny, nx CUDA
    tensor, float32 or float64) along +B and -B.  Returns device tensors:
    ends (2, n, 3), flags (2, n) int32, bn (3, n), length (2, n), and with
    twist=True the twist of each half (2, n)."""
    torch = _torch()
    if b.dtype not in (torch.float32, torch.float64) or b.device.type != "cuda" or b.ndim != 4 or b.shape[0] != 3:
        raise ValueError("b must be a (3, nz, ny, nx) float32/float64 CUDA tensor")
    b = b.contiguous()
    _, nz, ny, nx = (int(v) for v in b.shape)
    seeds = seeds.to(device=b.device, dtype=b.dtype).reshape(-1, 3).contiguous()
    n = int(seeds.shape[0])
    if max_steps is None:
        max_steps = int(math.ceil(4.0 * (nx + ny + nz) / float(step_len)))
    ends = torch.empty((2, n, 3), dtype=b.dtype, device=b.device)
    flags = torch.empty((2, n), dtype=torch.int32, device=b.device)
    bn = torch.empty((3, n), dtype=b.dtype, device=b.device)
    length = torch.empty((2, n), dtype=b.dtype, device=b.device)
    tw = torch.empty((2, n), dtype=b.dtype, device=b.device) if twist else None
    nrm = np.asarray(normal, dtype=np.float64)
    code = L.NFGS_F32 if b.dtype == torch.float32 else L.NFGS_F64
    stream = torch.cuda.current_stream(b.device)
    L.check(L.lib().nfgs_trace_field_lines(
        C.c_void_p(b.data_ptr()), code, nz, ny, nx, C.c_void_p(seeds.data_ptr()), n, L.dptr(nrm),
        float(step_len), int(max_steps), C.c_void_p(ends.data_ptr()), C.c_void_p(flags.data_ptr()),
        C.c_void_p(bn.data_ptr()), C.c_void_p(length.data_ptr()), C.c_void_p(tw.data_ptr() if twist else None),
        C.c_void_p(stream.cuda_stream)))
    out = {"ends": ends, "flags": flags, "bn": bn, "length": length, "max_steps": max_steps}
    if twist:
        out["twist"] = tw
    return out


def trace_qperp(b, seeds, *, delta: float = 0.25, step_len: float = 1.0 / 8.0, max_steps=None,
                twist: bool = False):
    """Q_perp (Titov 2007) at each seed: five lines per seed (the seed and
    +-delta along two unit vectors perpendicular to B), traced both ways.
    Returns device tensors q (n,), ends (2, n, 3), flags (2, n) int32,
    bn (3, n) = |B0|, |Bn+|, |Bn-|, length (2, n) of the central line, and
    with twist=True its twist per half (2, n)."""
    torch = _torch()
    if b.dtype not in (torch.float32, torch.float64) or b.device.type != "cuda" or b.ndim != 4 or b.shape[0] != 3:
        raise ValueError("b must be a (3, nz, ny, nx) float32/float64 CUDA tensor")
    b = b.contiguous()
    _, nz, ny, nx = (int(v) for v in b.shape)
    seeds = seeds.to(device=b.device, dtype=b.dtype).reshape(-1, 3).contiguous()
    n = int(seeds.shape[0])
    if max_steps is None:
        max_steps = int(math.ceil(4.0 * (nx + ny + nz) / float(step_len)))
    out = {"q": torch.empty((n,), dtype=b.dtype, device=b.device),
           "ends": torch.empty((2, n, 3), dtype=b.dtype, device=b.device),
           "flags": torch.empty((2, n), dtype=torch.int32, device=b.device),
           "bn": torch.empty((3, n), dtype=b.dtype, device=b.device),
           "length": torch.empty((2, n), dtype=b.dtype, device=b.device)}
    if twist:
        out["twist"] = torch.empty((2, n), dtype=b.dtype, device=b.device)
    code = L.NFGS_F32 if b.dtype == torch.float32 else L.NFGS_F64
    stream = torch.cuda.current_stream(b.device)
    L.check(L.lib().nfgs_trace_qperp(
        C.c_void_p(b.data_ptr()), code, nz, ny, nx, C.c_void_p(seeds.data_ptr()), n, float(delta), float(step_len),
        int(max_steps), C.c_void_p(out["ends"].data_ptr()), C.c_void_p(out["flags"].data_ptr()),
        C.c_void_p(out["bn"].data_ptr()), C.c_void_p(out["length"].data_ptr()), C.c_void_p(out["q"].data_ptr()),
        C.c_void_p(out["twist"].data_ptr() if twist else None), C.c_void_p(stream.cuda_stream)))
    out["max_steps"] = max_steps
    return out


def trace_fastqsl(b, seeds, *, normal=(0.0, 0.0, 1.0), step_len: float = 1.0 / 8.0, tol: float = 0.1,
                  twist: bool = False):
    """FastQSL's adaptive trace of every seed (``nfgs_trace_fastqsl``: the
    reference's RKF4(5) step control, face handling and limits in FP32).
    b (3, nz, ny, nx) CUDA tensor (cast to float32, as the reference does);
    seeds (n, 3) xyz grid coordinates.  Returns device tensors ends (2, n, 3)
    ([0] end along +B, [1] start along -B), flags (2, n) int32, bsamp
    (3, 3, n) (B components at the seed, end and start), bflag (n,) int32,
    length (n,) float64 (both halves) and with twist=True twist (n,)."""
    torch = _torch()
    if b.device.type != "cuda" or b.ndim != 4 or b.shape[0] != 3:
        raise ValueError("b must be a (3, nz, ny, nx) CUDA tensor")
    b = b.to(torch.float32).contiguous()
    _, nz, ny, nx = (int(v) for v in b.shape)
    seeds = seeds.to(device=b.device, dtype=torch.float32).reshape(-1, 3).contiguous()
    n = int(seeds.shape[0])
    dev = b.device
    out = {"ends": torch.empty((2, n, 3), dtype=torch.float32, device=dev),
           "flags": torch.empty((2, n), dtype=torch.int32, device=dev),
           "bsamp": torch.empty((3, 3, n), dtype=torch.float32, device=dev),
           "bflag": torch.empty((n,), dtype=torch.int32, device=dev),
           "length": torch.empty((n,), dtype=torch.float64, device=dev)}
    if twist:
        out["twist"] = torch.empty((n,), dtype=torch.float64, device=dev)
    nrm = np.asarray(normal, dtype=np.float64)
    stream = torch.cuda.current_stream(dev)
    ptr = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    L.check(L.lib().nfgs_trace_fastqsl(
        ptr(b), nz, ny, nx, ptr(seeds), n, L.dptr(nrm), float(step_len), float(tol), int(bool(twist)),
        ptr(out["ends"]), ptr(out["flags"]), ptr(out["bsamp"]), ptr(out["bflag"]), ptr(out["length"]),
        C.c_void_p(out["twist"].data_ptr() if twist else None), C.c_void_p(stream.cuda_stream)))
    return out


def qcalc_plane(tr, nu: int, nv: int, normal, stride: float = 1.0):
    """QCalcPlane's Q (nv, nu) on the device from a trace_fastqsl of an
    nv x nu seed grid (``nfgs_qcalc_plane``)."""
    torch = _torch()
    q = torch.empty((nv, nu), dtype=torch.float32, device=tr["ends"].device)
    nrm = np.asarray(normal, dtype=np.float64)
    stream = torch.cuda.current_stream(q.device)
    L.check(L.lib().nfgs_qcalc_plane(int(nu), int(nv), C.c_void_p(tr["ends"].data_ptr()),
                                     C.c_void_p(tr["flags"].data_ptr()), C.c_void_p(tr["bsamp"].data_ptr()),
                                     L.dptr(nrm), float(stride), C.c_void_p(q.data_ptr()),
                                     C.c_void_p(stream.cuda_stream)))
    return q


def _plane_q(b, seeds, nu, nv, normal, q_method, step_len, max_steps, delta, twist=False, tol=0.1):
    """Trace the nv x nu seed grid and evaluate Q by the chosen method; the
    plane's border is NaN either way (the reference keeps only the interior)."""
    if q_method == "fastqsl":
        tr = trace_fastqsl(b, seeds, normal=normal, step_len=step_len, tol=tol, twist=twist)
        tr["max_steps"] = None
        return tr, qcalc_plane(tr, nu, nv, normal)
    if q_method == "perp":
        tr = trace_qperp(b, seeds, delta=delta, step_len=step_len, max_steps=max_steps, twist=twist)
        q = tr["q"].reshape(nv, nu).clone()
        q[0, :] = float("nan")
        q[-1, :] = float("nan")
        q[:, 0] = float("nan")
        q[:, -1] = float("nan")
        return tr, q
    if q_method == "plane":
        tr = trace_field_lines(b, seeds, normal=normal, step_len=step_len, max_steps=max_steps, twist=twist)
        return tr, q_on_plane(tr, nu, nv)
    raise ValueError("q_method must be 'fastqsl', 'perp' or 'plane'")


def q_on_plane(tr, nu: int, nv: int):
    """Q (nv, nu) on the device from a trace of an nv x nu unit-spacing seed grid."""
    torch = _torch()
    q = torch.empty((nv, nu), dtype=tr["ends"].dtype, device=tr["ends"].device)
    code = L.NFGS_F32 if q.dtype == torch.float32 else L.NFGS_F64
    stream = torch.cuda.current_stream(q.device)
    L.check(L.lib().nfgs_qmap_plane(code, int(nu), int(nv), C.c_void_p(tr["ends"].data_ptr()),
                                    C.c_void_p(tr["flags"].data_ptr()), C.c_void_p(tr["bn"].data_ptr()),
                                    C.c_void_p(q.data_ptr()), C.c_void_p(stream.cuda_stream)))
    return q


def _bundle(tr, q, plane_shape, meta):
    nv, nu = plane_shape
    ends = tr["ends"].float().cpu().numpy()
    flags = tr["flags"].cpu().numpy()
    both = tr["length"].ndim == 1  # the FastQSL trace sums the halves itself
    length = (tr["length"] if both else tr["length"][0] + tr["length"][1]).float().cpu().numpy()
    extra = {}
    if "twist" in tr:
        tw = tr["twist"] if both else tr["twist"][0] + tr["twist"][1]
        extra["twist"] = tw.double().cpu().numpy().reshape(nv, nu)
    return {**extra,
        "q": q.float().cpu().numpy(),
        "flag_start": flags[1].reshape(nv, nu).astype(np.int32),
        "flag_end": flags[0].reshape(nv, nu).astype(np.int32),
        "start_xyz": ends[1].reshape(nv, nu, 3).astype(np.float32),
        "end_xyz": ends[0].reshape(nv, nu, 3).astype(np.float32),
        "line_len": length.reshape(nv, nu).astype(np.float32),
        "metadata": meta,
    }


def compute_y0_qmap(bx, by, bz, *, fastqsl_root=None, y_index=None, step_len: float = 1.0 / 8.0, tol: float = 0.1,
                    block_x: int = 128, trace_chunk_seeds: int = 8192, b_smooth_sigma_cells: float = 0.0,
                    include_twist: bool = False, dtype: str = "float32", max_steps=None,
                    q_method: str = "fastqsl", delta: float = 0.25):
    """Q on the x-z plane at y = y_index (default the physical midplane),
    shape (nz, nx), seeds at every x-z node (fastqsl_plane.py:203-383).
    q_method "fastqsl" (default): the reference's FastQSL adaptive trace and
    QCalcPlane in FP32; "perp": Q_perp from RK4 lines offset perpendicular to
    B by +-delta, defined where B lies in the plane (By = 0 on the midplane of
    a symmetric field); "plane": RK4 lines and central differences over the
    seed grid."""
    torch = _torch()
    dt = torch.float64 if str(dtype) in ("float64", "torch.float64") else torch.float32
    b = spectral_gaussian_lowpass(_volume(bx, by, bz, dt), b_smooth_sigma_cells)
    _, nz, ny, nx = (int(v) for v in b.shape)
    iy = physical_midplane_grid_index(ny) if y_index is None else float(y_index)
    if not 0.0 <= iy <= float(ny - 1):
        raise ValueError(f"y_index={iy} is outside [0,{ny - 1}]")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    z, x = torch.meshgrid(torch.arange(nz, dtype=dt, device=b.device), torch.arange(nx, dtype=dt, device=b.device),
                          indexing="ij")
    seeds = torch.stack([x.reshape(-1), torch.full_like(x.reshape(-1), iy), z.reshape(-1)], dim=1)
    tr, q = _plane_q(b, seeds, nx, nz, (0.0, 1.0, 0.0), q_method, step_len, max_steps, delta,
                     twist=bool(include_twist), tol=tol)
    torch.cuda.synchronize()
    algo = "FastQSL QCalcPlane on y=0" if q_method == "fastqsl" else f"B200 RK4 tracer + Q ({q_method}) on y=0"
    meta = {"algorithm": algo, "q_method": q_method, "delta": float(delta),
            "shape_zyx": [nz, ny, nx],
            "plane_y_index": iy, "plane_coordinate_contract": Y0_PLANE_COORDINATE_CONTRACT,
            "plane_is_fractional": bool(not float(iy).is_integer()), "plane_shape_zx": [nz, nx],
            "step_len_grid": float(step_len), "tolerance": float(tol), "max_steps": tr["max_steps"],
            "block": [int(block_x), 1, 1], "trace_chunk_seeds": int(trace_chunk_seeds), "trace_n_chunks": 1,
            "downsample": 1, "qmap_b_smooth_sigma_cells": float(b_smooth_sigma_cells),
            "elapsed_s": time.perf_counter() - t0, "twist_included": bool(include_twist),
            "dtype": "float64" if dt == torch.float64 else "float32"}
    return _bundle(tr, q, (nz, nx), meta)


def compute_bottom_qmap(bx, by, bz, *, fastqsl_root=None, z_index=None, step_len: float = 1.0 / 8.0,
                        tol: float = 0.1, block_x: int = 128, trace_chunk_seeds: int = 8192,
                        b_smooth_sigma_cells: float = 0.0, dtype: str = "float32", max_steps=None,
                        q_method: str = "fastqsl", delta: float = 0.25):
    """Q on the bottom x-y plane, shape (ny, nx); seeds half a cell above the
    bottom face by default (z = 0.5), normal +z (fastqsl_plane.py:385-506).
    q_method as compute_y0_qmap."""
    torch = _torch()
    dt = torch.float64 if str(dtype) in ("float64", "torch.float64") else torch.float32
    b = spectral_gaussian_lowpass(_volume(bx, by, bz, dt), b_smooth_sigma_cells)
    _, nz, ny, nx = (int(v) for v in b.shape)
    iz = 0.5 if z_index is None else float(z_index)
    if not 0.0 <= iz <= float(nz - 1):
        raise ValueError(f"z_index={iz} is outside [0,{nz - 1}]")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    y, x = torch.meshgrid(torch.arange(ny, dtype=dt, device=b.device), torch.arange(nx, dtype=dt, device=b.device),
                          indexing="ij")
    seeds = torch.stack([x.reshape(-1), y.reshape(-1), torch.full_like(x.reshape(-1), iz)], dim=1)
    tr, q = _plane_q(b, seeds, nx, ny, (0.0, 0.0, 1.0), q_method, step_len, max_steps, delta, tol=tol)
    torch.cuda.synchronize()
    algo = ("FastQSL QCalcPlane on the bottom plane" if q_method == "fastqsl"
            else f"B200 RK4 tracer + Q ({q_method}) on the bottom plane")
    meta = {"algorithm": algo, "q_method": q_method,
            "delta": float(delta), "shape_zyx": [nz, ny, nx],
            "plane_z_index": iz, "plane_shape_yx": [ny, nx], "step_len_grid": float(step_len),
            "tolerance": float(tol), "max_steps": tr["max_steps"], "block": [int(block_x), 1, 1],
            "trace_chunk_seeds": int(trace_chunk_seeds), "trace_n_chunks": 1, "downsample": 1,
            "qmap_b_smooth_sigma_cells": float(b_smooth_sigma_cells), "elapsed_s": time.perf_counter() - t0,
            "dtype": "float64" if dt == torch.float64 else "float32"}
    return _bundle(tr, q, (ny, nx), meta)


def main(argv=None):
    """Time the y=0 and bottom Q maps of a solved TD-type rope (--field solve)
    or of the analytic TD field itself (--field td)."""
    import torch

    from .scan import KW, STOP
    from .solver import NFGSSolverGPU
    from .synthetic import td_bottom, td_volume

    ap = argparse.ArgumentParser(description="Q maps of a TD-type flux rope")
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--nz", type=int, default=128)
    ap.add_argument("--field", choices=["solve", "td"], default="solve")
    ap.add_argument("--iters", type=int, default=400)
    ap.add_argument("--report", default=None)
    ap.add_argument("--q-method", default="fastqsl", choices=["fastqsl", "perp", "plane"])
    args = ap.parse_args(argv)
    if args.field == "solve":
        h = 16.0 / (args.n - 1)
        bx, by, bz = td_bottom(args.n, args.n, seed=1, extent=8.0)
        s = NFGSSolverGPU(args.n, args.n, args.nz, h, h, h, bottom_divergence_robin_weight=0.5, **KW)
        s.set_bottom_vector_boundary(bx, by, bz, zero_net_current=False, smooth_passes=0, ijzbcor=3)
        hist = s.iterate(max_iter=args.iters, verbose=False, **STOP)
        f = s.fields_to_torch()
        out = {"field": "NFGS solution", "grid_zyx": [int(v) for v in f.shape[1:]], "best_sigma": hist["best_sigma"]}
    else:
        f = torch.as_tensor(td_volume(args.n, args.n, args.nz, seed=1, extent=8.0), dtype=torch.float32,
                            device="cuda")
        out = {"field": "analytic TD (td_volume seed 1)", "grid_zyx": [int(v) for v in f.shape[1:]]}
    for name, fn in (("y0", compute_y0_qmap), ("bottom", compute_bottom_qmap)):
        fn(f[0], f[1], f[2], q_method=args.q_method)  # warm-up
        r = fn(f[0], f[1], f[2], q_method=args.q_method)
        lens = r["line_len"]
        qv = r["q"][np.isfinite(r["q"])]
        seeds = r["q"].size
        out[name] = {"seeds": seeds, "seconds": r["metadata"]["elapsed_s"], "q_method": r["metadata"]["q_method"],
                     "lines_per_s": (10 if r["metadata"]["q_method"] == "perp" else 2) * seeds
                     / r["metadata"]["elapsed_s"],
                     "mean_line_len": float(np.mean(lens)),
                     "cells_traced_per_s": float(np.sum(lens)) / r["metadata"]["elapsed_s"],
                     "q_valid": int(qv.size), "q_median": float(np.median(qv)) if qv.size else None,
                     "log10_q_p99": float(np.log10(np.percentile(qv, 99))) if qv.size else None}
    torch.cuda.synchronize()
    print(json.dumps(out), flush=True)
    if args.report:
        with open(args.report, "w") as fh:
            json.dump(out, fh, indent=1)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())

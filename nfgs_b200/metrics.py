"""Evaluation metrics of a reconstruction, computed on the GPU.

The reference evaluates its solutions with NumPy on host copies of the
fields; here one CUDA pass (nfgs_field_metrics) computes every metric of a
region of interest from device-resident volumes:

* compute_reference_metrics   nfgs/_backend/util/metrics.py:123-178
* compute_metrics             nfgs/_backend/scripts/recompute_td_referee_diagnostics.py:344-400
* roi_cwsin, fortran_cwsin    nfgs/_backend/util/metrics.py:64-120
* common_fd2_sigma_j          nfgs/diagnostics/common_fd2.py:59-78 (second-order
                              curl of the full volume, then the region)
* the region helpers          nfgs/_backend/util/metrics.py:9-54

Inputs may be NumPy arrays (copied to the device) or CUDA tensors, as dicts
of z-y-x volumes ("Bx", "By", "Bz", "Jx", "Jy", "Jz") like the reference's.
Sums are FP64 and in a fixed order (repeatable to the bit); an FP32 field
is differentiated in FP64, where the reference differentiates in the array's
own dtype, so FP32 results agree with it to FP32 rounding.

solution_metrics(solver, ...) evaluates a solver's stored solution without
copying its fields to the host.
"""

from __future__ import annotations

import ctypes as C
import math
from typing import Dict, Optional, Sequence, Tuple

import numpy as np

from . import _lib as L

METRIC_NAMES = ("C_vec", "C_CS", "Eprime_n", "Eprime_m", "epsilon", "sigma_J", "sigma_J_common_fd2",
                "divB_normalized", "cells", "sum_b2", "sum_ref2", "nonfinite_B", "nonfinite_J")
B_KEYS = ("Bx", "By", "Bz")
J_KEYS = ("Jx", "Jy", "Jz")


def _torch():
    import torch

    return torch


# ---------------------------------------------------------------- regions
def flux_rope_center_from_bottom_jz(Jz_bottom) -> Tuple[int, int]:
    """(iy, ix) of the |Jz| centroid on the bottom plane (metrics.py:9-20)."""
    w = np.abs(np.asarray(Jz_bottom, dtype=np.float64))
    tot = float(w.sum()) + 1e-30
    ny, nx = w.shape
    iy = float(np.sum(w.sum(axis=1) * np.arange(ny))) / tot
    ix = float(np.sum(w.sum(axis=0) * np.arange(nx))) / tot
    return int(np.clip(np.round(iy), 0, ny - 1)), int(np.clip(np.round(ix), 0, nx - 1))


def metric_roi_slices_zyx(nz: int, ny: int, nx: int, pad: int) -> Tuple[slice, slice, slice]:
    """Interior slices without a pad-cell border (metrics.py:23-32)."""
    pad = int(pad)
    if pad <= 0:
        return slice(None), slice(None), slice(None)
    return (slice(0, nz - pad) if nz > pad else slice(None),
            slice(pad, ny - pad) if ny > 2 * pad else slice(None),
            slice(pad, nx - pad) if nx > 2 * pad else slice(None))


def test_domain_slices_zyx(nz, ny, nx, iy_c, ix_c, n_test_x, n_test_y, n_test_z) -> Tuple[slice, slice, slice]:
    """Analysis box centred on a photospheric feature (metrics.py:35-54)."""
    n_test_x, n_test_y, n_test_z = min(int(n_test_x), nx), min(int(n_test_y), ny), min(int(n_test_z), nz)
    y0 = int(np.clip(iy_c - n_test_y // 2, 0, ny - n_test_y))
    x0 = int(np.clip(ix_c - n_test_x // 2, 0, nx - n_test_x))
    return slice(0, n_test_z), slice(y0, y0 + n_test_y), slice(x0, x0 + n_test_x)


test_domain_slices_zyx.__test__ = False  # a library function, not a pytest test


def fortran_box(nz: int, ny: int, nx: int) -> Tuple[slice, slice, slice]:
    """Region of the NFPT Fortran CWsin check (metrics.py:107-113): z from
    plane 1 without the upper quarter, x/y without an eighth on each side."""
    ax, ay, az = nx // 8, ny // 8, nz // 4
    return slice(1, max(1, nz - az)), slice(ay, max(ay + 1, ny - ay + 1)), slice(ax, max(ax + 1, nx - ax + 1))


def _roi(slices, shape) -> np.ndarray:
    out = []
    for s, n in zip(slices, shape):
        if not isinstance(s, slice):
            raise ValueError("metric slices must be three slice objects (z, y, x)")
        lo, hi, step = s.indices(n)
        if step != 1:
            raise ValueError("Scoring box is outside the field or is strided")
        out += [lo, hi]
    if any(out[2 * d] >= out[2 * d + 1] for d in range(3)):
        raise ValueError("Scoring box is outside the field or is empty")
    return np.asarray(out, dtype=np.int32)


def _spacing(spacing) -> Tuple[float, float, float]:
    """A scalar or (dx, dy, dz), positive (common_fd2.py:10-18)."""
    if np.isscalar(spacing):
        v = (float(spacing),) * 3
    else:
        v = tuple(float(x) for x in spacing)
    if len(v) != 3 or any(not math.isfinite(x) or x <= 0 for x in v):
        raise ValueError("spacing must be positive: a scalar or (dx, dy, dz)")
    return v


# ---------------------------------------------------------------- the pass
def _stack3(fields, keys, dtype, device):
    """(3, nz, ny, nx) contiguous CUDA tensor from a dict of volumes or a stacked array."""
    torch = _torch()
    if fields is None:
        return None
    if isinstance(fields, torch.Tensor) and fields.dim() == 4 and fields.shape[0] == 3:
        return fields.to(device=device, dtype=dtype).contiguous()
    if isinstance(fields, dict):
        parts = [fields[k] for k in keys]
    else:
        parts = [fields[i] for i in range(3)]
    ts = [p if isinstance(p, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(p)) for p in parts]
    return torch.stack([t.to(device=device, dtype=dtype) for t in ts]).contiguous()


def _dtype_of(*fields):
    torch = _torch()
    for f in fields:
        if f is None:
            continue
        vals = f.values() if isinstance(f, dict) else [f]
        for v in vals:
            if v.dtype in (np.float64, torch.float64):
                return torch.float64
    return torch.float32


def field_metrics(ref, sol, cur, spacing, slices) -> Dict[str, float]:
    """Every metric of one region.

    ref, sol, cur: dicts of z-y-x volumes (B_KEYS for ref and sol, J_KEYS or
    B-named current for cur) or stacked (3, nz, ny, nx) arrays / tensors;
    ref and cur may be None.  Arrays are evaluated in FP64 when any input is
    FP64, else FP32 (the storage type; sums are FP64 either way)."""
    torch = _torch()
    if not torch.cuda.is_available():
        raise RuntimeError("nfgs_b200.metrics needs a CUDA device")
    dev = torch.device("cuda", torch.cuda.current_device())
    dt = _dtype_of(ref, sol, cur)
    s = _stack3(sol, B_KEYS, dt, dev)
    r = _stack3(ref, B_KEYS, dt, dev)
    j = _stack3(cur, J_KEYS if isinstance(cur, dict) and "Jx" in cur else B_KEYS, dt, dev)
    shape = tuple(s.shape[1:])
    for t in (r, j):
        if t is not None and tuple(t.shape[1:]) != shape:
            raise ValueError(f"B_vec/J_vec must both have shape (3, Nz, Ny, Nx); got {tuple(s.shape)}, "
                             f"{tuple(t.shape)}")
    roi = _roi(slices, shape)
    sp = np.asarray(_spacing(spacing), dtype=np.float64)
    out = np.zeros(len(METRIC_NAMES))
    stream = torch.cuda.current_stream(dev).cuda_stream
    L.check(L.lib().nfgs_field_metrics(
        C.c_void_p(r.data_ptr()) if r is not None else None, C.c_void_p(s.data_ptr()),
        C.c_void_p(j.data_ptr()) if j is not None else None, L.NFGS_F64 if dt == torch.float64 else L.NFGS_F32,
        shape[0], shape[1], shape[2], L.dptr(sp), roi.ctypes.data_as(C.POINTER(C.c_int32)), L.dptr(out),
        C.c_void_p(stream)))
    return dict(zip(METRIC_NAMES, (float(v) for v in out)))


# ------------------------------------------------- the reference's functions
def compute_reference_metrics(ref_fields, fields, metric_slices) -> Dict[str, float]:
    """Reference-field agreement and force-freeness on a z-y-x region
    (metrics.py:123-178).  fields holds Bx..Bz and Jx..Jz."""
    m = field_metrics(ref_fields, fields, {k: fields[k] for k in J_KEYS}, 1.0, metric_slices)
    if m["nonfinite_B"] > 0:
        raise RuntimeError("Non-finite values in B fields for metrics.")
    if m["nonfinite_J"] > 0:
        raise RuntimeError("Non-finite values in J for sigma_J.")
    return {"C_vec": m["C_vec"], "C_CS": m["C_CS"], "En": 1.0 - m["Eprime_n"], "Em": 1.0 - m["Eprime_m"],
            "Eprime_n": m["Eprime_n"], "Eprime_m": m["Eprime_m"], "epsilon": m["epsilon"], "sigma_J": m["sigma_J"]}


def compute_metrics(reference, candidate, current, slices, spacing) -> Dict[str, float]:
    """recompute_td_referee_diagnostics.py:344-400: the same metrics plus
    divB normalised by 6 mean|B| / spacing.  current is the solution's
    current (Jx..Jz), or None for the second-order curl of the candidate;
    the divergence is always the second-order one of the candidate."""
    m = field_metrics(reference, candidate, current, spacing, slices)
    sj = m["sigma_J"] if current is not None else m["sigma_J_common_fd2"]
    return {"C_vec": m["C_vec"], "C_CS": m["C_CS"], "Eprime_n": m["Eprime_n"], "Eprime_m": m["Eprime_m"],
            "epsilon": m["epsilon"], "sigma_J": sj, "divB_normalized": m["divB_normalized"]}


def common_fd2_sigma_j(fields, spacing, slices) -> float:
    """sigma_J on the second-order curl of B (common_fd2.py:59-78)."""
    return field_metrics(None, fields, None, spacing, slices)["sigma_J_common_fd2"]


def roi_cwsin(B_vec, J_vec, *, b2min: float = 1e-10) -> float:
    """sum |J x B| / max(|B|, 1e-10) / sum |J| on pre-sliced (3, nz, ny, nx) volumes (metrics.py:64-86)."""
    if b2min != 1e-10:
        raise NotImplementedError("only the reference's floor |B| >= 1e-10 is built")
    nz, ny, nx = tuple(B_vec.shape[1:])
    return field_metrics(None, B_vec, J_vec, 1.0, (slice(0, nz), slice(0, ny), slice(0, nx)))["sigma_J"]


def fortran_cwsin(B_vec, J_vec, *, b2min: float = 1e-20) -> float:
    """The NFPT Fortran CWsin on its interior box (metrics.py:89-120)."""
    if b2min != 1e-20:
        raise NotImplementedError("only the reference's floor |B| >= sqrt(1e-20) is built")
    nz, ny, nx = tuple(B_vec.shape[1:])
    return field_metrics(None, B_vec, J_vec, 1.0, fortran_box(nz, ny, nx))["sigma_J"]


# ---------------------------------------------------------- solver fields
def solution_metrics(solver, reference: Optional[dict] = None, slices: Optional[Sequence[slice]] = None,
                     crop_to_observed_fov: bool = True) -> Dict[str, float]:
    """Metrics of the solver's stored solution, evaluated on the device.

    reference: optional dict of reference Bx/By/Bz volumes on the exported
    grid; slices: region (default: the whole exported grid).  Adds
    "sigma_J_fortran_box" (the solver current on the Fortran CWsin box)."""
    f = solver.fields_to_torch(crop_to_observed_fov=crop_to_observed_fov)
    nz, ny, nx = tuple(f.shape[1:])
    if slices is None:
        slices = (slice(0, nz), slice(0, ny), slice(0, nx))
    sp = (float(solver.dx), float(solver.dy), float(solver.dz))
    ref = None
    if reference is not None:
        ref = _stack3(reference, B_KEYS, f.dtype, f.device)
        if tuple(ref.shape[1:]) != (nz, ny, nx):
            raise ValueError(f"reference shape {tuple(ref.shape[1:])} != solution shape {(nz, ny, nx)}")
    m = field_metrics(ref, f[0:3], f[3:6], sp, slices)
    m["sigma_J_fortran_box"] = field_metrics(None, f[0:3], f[3:6], sp, fortran_box(nz, ny, nx))["sigma_J"]
    return m


def main(argv=None):
    """Time field_metrics on seeded FP32 volumes (all three inputs, whole
    volume as the region) and report effective bandwidth: 36 algorithmic
    bytes per cell (reference, solution and current, 3 components x 4 B)."""
    import argparse
    import json
    import time

    torch = _torch()
    ap = argparse.ArgumentParser(description="time the GPU evaluation metrics")
    ap.add_argument("--shape", default="128,256,256", help="nz,ny,nx of the evaluated volumes")
    ap.add_argument("--iters", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    args = ap.parse_args(argv)
    nz, ny, nx = (int(v) for v in args.shape.split(","))
    g = torch.Generator(device="cuda").manual_seed(0)
    ref = torch.randn((3, nz, ny, nx), device="cuda", generator=g)
    sol = ref + 0.1 * torch.randn((3, nz, ny, nx), device="cuda", generator=g)
    cur = torch.randn((3, nz, ny, nx), device="cuda", generator=g)
    sl = (slice(0, nz), slice(0, ny), slice(0, nx))
    for _ in range(args.warmup):
        m = field_metrics(ref, sol, cur, 1.0, sl)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.iters):
        m = field_metrics(ref, sol, cur, 1.0, sl)
    dt = (time.perf_counter() - t0) / args.iters
    cells = nz * ny * nx
    print(json.dumps({"shape": [nz, ny, nx], "cells": cells, "ms_per_call": dt * 1e3,
                      "algorithmic_bytes": 36 * cells, "gbs": 36 * cells / dt / 1e9,
                      "sigma_J_common_fd2": m["sigma_J_common_fd2"]}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())

"""Generate the FastQSL tracing fixtures in tests/golden/fastqsl/ from the
REFERENCE's own adaptive tracer and Q formula, in two phases.

Phase ``trace`` (on a GPU box): the reference's vendored FastQSL kernel
``TraceAllBline`` of TraceBlineAdaptive.cu, compiled unmodified by
oracle/build_ref.sh into oracle/_ref/libfastqsl_ref.so (CuPy, through which
fastqsl_plane.py drives it, is not in this image), traces every seed of a
plane of a TD99 flux-rope field with the arguments of
nfgs/_backend/util/fastqsl_plane.py:203-383 / 386-506 (step 1/8, tol 0.1,
block 128; the twist case with the centred grid curl of :287-305).  It writes
the raw per-seed outputs (end points, flags, B samples, line lengths, twist):

    bash oracle/build_ref.sh                          # where the reference is
    python tests/golden/make_fastqsl_golden.py trace  # on the GPU box

Phase ``q`` (where the reference is importable): the reference's own
``FastQSL.QCalcPlane`` and ``ResReshape`` (fastqslpy/FastQSL.py), run with
NumPy standing in for CuPy (the function uses only the array calls NumPy
shares with CuPy), turn those outputs into the Q map exactly as
fastqsl_plane.py:340-348 does, and add it to each fixture:

    python tests/golden/make_fastqsl_golden.py q

The fields are regenerated by the tests from nfgs_b200.synthetic.td_volume
(a checksum in each fixture guards that); the tests never import the
reference.
"""

from __future__ import annotations

import ctypes
import json
import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
OUT = Path(os.environ.get("FASTQSL_GOLDEN_OUT", HERE / "fastqsl"))  # the trace phase may write elsewhere
sys.path.insert(0, str(ROOT))

# (nx, ny, nz, td seed, plane, twist)
CASES = {
    "td1_y0": dict(shape=(48, 48, 40), seed=1, plane="y0", twist=True),
    "td1_bottom": dict(shape=(48, 48, 40), seed=1, plane="bottom", twist=False),
    "td2_y0": dict(shape=(56, 40, 36), seed=2, plane="y0", twist=False),
}
STEP, TOL, BLOCK = 1.0 / 8.0, 0.1, 128


def field(spec):
    """float32 (3, nz, ny, nx) TD99 rope field of a case and its checksum."""
    from nfgs_b200.synthetic import td_volume

    nx, ny, nz = spec["shape"]
    b = td_volume(nx, ny, nz, seed=spec["seed"]).astype(np.float32)
    return b, float(np.abs(b.astype(np.float64)).sum())


def seeds(spec):
    """Seed coordinates (x, y, z) of the plane and the plane's shape and
    normal (fastqsl_plane.py:243-252, 436-446)."""
    nx, ny, nz = spec["shape"]
    if spec["plane"] == "y0":
        x, z = np.meshgrid(np.arange(nx, dtype=np.float32), np.arange(nz, dtype=np.float32), indexing="xy")
        y = np.full(x.shape, 0.5 * (ny - 1), dtype=np.float32)
        normal = np.array([0.0, 1.0, 0.0], np.float32)
    else:
        x, y = np.meshgrid(np.arange(nx, dtype=np.float32), np.arange(ny, dtype=np.float32), indexing="xy")
        z = np.full(x.shape, 0.5, dtype=np.float32)
        normal = np.array([0.0, 0.0, 1.0], np.float32)
    return x.ravel(), y.ravel(), z.ravel(), x.shape, normal


def grid_curl(b):
    """Centred curl with second-order one-sided edges in grid units
    (fastqsl_plane.py:287-305; arrays (z, y, x))."""
    bx, by, bz = b
    g = lambda a, ax: np.gradient(a, axis=ax, edge_order=2).astype(np.float32)  # noqa: E731
    return g(bz, 1) - g(by, 0), g(bx, 0) - g(bz, 2), g(by, 2) - g(bx, 1)


def trace_case(name, spec, lib):
    import torch

    dev = torch.device("cuda")
    b, checksum = field(spec)
    nx, ny, nz = spec["shape"]
    sx, sy, sz, shape, normal = seeds(spec)
    n = sx.size
    f32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device=dev)  # noqa: E731
    bxg, byg, bzg = (f32(c) for c in b)
    if spec["twist"]:
        cx, cy, cz = (f32(c) for c in grid_curl(b))
        twist = torch.zeros(n, dtype=torch.float64, device=dev)
    else:
        cx = cy = cz = torch.zeros((1, 1), dtype=torch.float32, device=dev)
        twist = torch.zeros((1, 1), dtype=torch.float32, device=dev)
    cur_flag = torch.tensor([bool(spec["twist"])], dtype=torch.bool, device=dev)
    bshape = torch.tensor([nx, ny, nz], dtype=torch.int32, device=dev)
    inp = [f32(sx), f32(sy), f32(sz)]
    nrm = f32(normal)
    outf = {k: torch.zeros(n, dtype=torch.float32, device=dev) for k in (
        "x_start", "y_start", "z_start", "x_end", "y_end", "z_end", "bx_start", "by_start", "bz_start",
        "bx_end", "by_end", "bz_end", "bx_inp", "by_inp", "bz_inp")}
    outi = {k: torch.zeros(n, dtype=torch.int32, device=dev) for k in ("flag_start", "flag_end", "b_flag")}
    line_len = torch.zeros(n, dtype=torch.float64, device=dev)
    step = torch.tensor([STEP], dtype=torch.float32, device=dev)
    tol = torch.tensor([TOL], dtype=torch.float32, device=dev)
    ntr = torch.tensor([n], dtype=torch.int64, device=dev)  # unsigned long long on the device
    P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    args = [P(bxg), P(byg), P(bzg), P(bshape), P(cx), P(cy), P(cz), P(twist), P(cur_flag), *map(P, inp), P(nrm),
            P(outf["x_start"]), P(outf["y_start"]), P(outf["z_start"]), P(outi["flag_start"]),
            P(outf["x_end"]), P(outf["y_end"]), P(outf["z_end"]), P(outi["flag_end"]),
            P(outf["bx_inp"]), P(outf["by_inp"]), P(outf["bz_inp"]), P(outi["b_flag"]),
            P(outf["bx_start"]), P(outf["by_start"]), P(outf["bz_start"]),
            P(outf["bx_end"]), P(outf["by_end"]), P(outf["bz_end"]),
            P(step), P(ntr), P(line_len), P(tol), ctypes.c_longlong(n), ctypes.c_int(BLOCK),
            ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)]
    rc = lib.fq_ref_trace_all(*args)
    torch.cuda.synchronize()
    if rc != 0:
        raise RuntimeError(f"reference trace launch failed: {rc}")
    out = {k: v.cpu().numpy() for k, v in outf.items()}
    out.update({k: v.cpu().numpy() for k, v in outi.items()})
    out["line_len"] = line_len.cpu().numpy()
    if spec["twist"]:
        out["twist"] = twist.cpu().numpy()
    out["seeds"] = np.stack([sx, sy, sz], axis=-1)
    meta = dict(spec, name=name, plane_shape=list(shape), normal=normal.tolist(), step_len=STEP, tol=TOL,
                block_x=BLOCK, field_checksum=checksum, n_seeds=int(n))
    OUT.mkdir(exist_ok=True)
    np.savez_compressed(OUT / f"{name}.npz", **out)
    (OUT / f"{name}.json").write_text(json.dumps(meta, indent=1, sort_keys=True) + "\n")
    print(name, n, "flags", np.bincount(out["flag_end"].clip(0, 50)).nonzero()[0].tolist(),
          "len", float(out["line_len"].mean()))


def qcalc_case(name):
    """Q of a traced case by the reference's QCalcPlane with NumPy as CuPy."""
    ref = Path(os.environ.get("NFGS_REFERENCE", "/root/reference")) / "third_party" / "FastQSL" / "fastqslpy"
    shim = types.ModuleType("cupy")
    for k in ("zeros", "abs", "where", "asarray", "float32", "nan", "full"):
        setattr(shim, k, getattr(np, k))
    sys.modules["cupy"] = shim
    sys.path.insert(0, str(ref))
    import FastQSL  # noqa: E402  (the reference's module)

    meta = json.loads((OUT / f"{name}.json").read_text())
    z = dict(np.load(OUT / f"{name}.npz"))
    shape = tuple(meta["plane_shape"])
    result = FastQSL.ResReshape(shape, *(z[k] for k in (
        "x_end", "y_end", "z_end", "flag_end", "x_start", "y_start", "z_start", "flag_start",
        "bx_start", "by_start", "bz_start", "bx_end", "by_end", "bz_end", "bx_inp", "by_inp", "bz_inp",
        "b_flag")))
    normal = np.asarray(meta["normal"], dtype=np.float32)
    q_inner = FastQSL.QCalcPlane(*result[:-1], result[-1], np.float32(1.0), normal)
    q = np.full(shape, np.nan, dtype=np.float32)
    q[1:-1, 1:-1] = q_inner
    z["q"] = q
    np.savez_compressed(OUT / f"{name}.npz", **z)
    print(name, "q finite", int(np.isfinite(q).sum()), "median", float(np.nanmedian(q)))


def time_against_reference(path, reps=5):
    """Phase ``time`` (GPU box): the reference kernel, in one launch and in
    the 8192-seed chunks of fastqsl_plane.py:221-338, against the library's
    nfgs_trace_fastqsl on the TD99 field at 256 x 256 x 128 (y = 0 midplane and
    bottom seed planes), CUDA-event times and a bitwise comparison."""
    import torch

    from nfgs_b200 import qmap
    from nfgs_b200.synthetic import td_volume

    lib = ctypes.CDLL(str(ROOT / "oracle" / "_ref" / "libfastqsl_ref.so"))
    lib.fq_ref_trace_all.restype = ctypes.c_int
    dev = torch.device("cuda")
    b = torch.as_tensor(td_volume(256, 256, 128, seed=1).astype(np.float32), device=dev)
    nz, ny, nx = b.shape[1:]
    out = {}

    def ref(sx, sy, sz, normal, chunk):
        n = sx.numel()
        z = lambda dt: torch.zeros(n, dtype=dt, device=dev)  # noqa: E731
        o = [z(torch.float32) for _ in range(15)]
        oi = [z(torch.int32) for _ in range(3)]
        ll = z(torch.float64)
        dummy = torch.zeros((1, 1), dtype=torch.float32, device=dev)
        consts = [torch.tensor([nx, ny, nz], dtype=torch.int32, device=dev), torch.tensor([False], device=dev),
                  torch.tensor(normal, dtype=torch.float32, device=dev),
                  torch.tensor([STEP], dtype=torch.float32, device=dev),
                  torch.tensor([TOL], dtype=torch.float32, device=dev)]
        P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
        comps = [b[c].contiguous() for c in range(3)]
        for s0 in range(0, n, chunk):
            s1 = min(n, s0 + chunk)
            sl = lambda t: t[s0:s1]  # noqa: E731
            ntr = torch.tensor([s1 - s0], dtype=torch.int64, device=dev)
            rc = lib.fq_ref_trace_all(
                *map(P, comps), P(consts[0]), P(dummy), P(dummy), P(dummy), P(dummy), P(consts[1]),
                P(sl(sx)), P(sl(sy)), P(sl(sz)), P(consts[2]),
                *(P(sl(o[k])) for k in (0, 1, 2)), P(sl(oi[0])), *(P(sl(o[k])) for k in (3, 4, 5)), P(sl(oi[1])),
                *(P(sl(o[k])) for k in (6, 7, 8)), P(sl(oi[2])), *(P(sl(o[k])) for k in (9, 10, 11, 12, 13, 14)),
                P(consts[3]), P(ntr), P(sl(ll)), P(consts[4]), ctypes.c_longlong(s1 - s0), ctypes.c_int(BLOCK),
                ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
            if rc != 0:
                raise RuntimeError(f"reference trace launch failed: {rc}")
        return o, oi, ll

    def timed(fn):
        r = fn()
        torch.cuda.synchronize()
        ms = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            r = fn()
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        return float(np.median(ms)), r

    for plane in ("y0", "bottom"):
        ar = lambda n: torch.arange(n, dtype=torch.float32, device=dev)  # noqa: E731
        if plane == "y0":
            x, zz = torch.meshgrid(ar(nx), ar(nz), indexing="xy")
            sx, sz = x.reshape(-1), zz.reshape(-1)
            sy = torch.full_like(sx, 0.5 * (ny - 1))
            normal = [0.0, 1.0, 0.0]
        else:
            x, y = torch.meshgrid(ar(nx), ar(ny), indexing="xy")
            sx, sy = x.reshape(-1), y.reshape(-1)
            sz = torch.full_like(sx, 0.5)
            normal = [0.0, 0.0, 1.0]
        seeds = torch.stack([sx, sy, sz], 1).contiguous()
        t_chunk, _ = timed(lambda: ref(sx, sy, sz, normal, 8192))
        t_one, (o, oi, ll) = timed(lambda: ref(sx, sy, sz, normal, sx.numel()))
        t_lib, tr = timed(lambda: qmap.trace_fastqsl(b, seeds, normal=normal, step_len=STEP, tol=TOL))
        same = (torch.equal(tr["ends"][0], torch.stack(o[3:6], 1)) and torch.equal(tr["ends"][1], torch.stack(o[0:3], 1))
                and torch.equal(tr["flags"][0], oi[1]) and torch.equal(tr["flags"][1], oi[0])
                and torch.equal(tr["length"], ll))
        out[plane] = {"seeds": int(sx.numel()), "reference_chunked_8192_ms": t_chunk, "reference_one_launch_ms": t_one,
                      "library_ms": t_lib, "bitwise_identical": bool(same),
                      "mean_line_len_cells": float(ll.mean())}
        print(plane, out[plane], flush=True)
    Path(path).write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    phase = sys.argv[1] if len(sys.argv) > 1 else "trace"
    only = set(sys.argv[2:])
    if phase == "trace":
        lib = ctypes.CDLL(str(ROOT / "oracle" / "_ref" / "libfastqsl_ref.so"))
        lib.fq_ref_trace_all.restype = ctypes.c_int
        for name, spec in CASES.items():
            if not only or name in only:
                trace_case(name, spec, lib)
    elif phase == "time":
        time_against_reference(sys.argv[2] if len(sys.argv) > 2 else "fastqsl_time.json")
    elif phase == "q":
        for name in CASES:
            if not only or name in only:
                qcalc_case(name)
    else:
        raise SystemExit("phase must be 'trace', 'q' or 'time'")

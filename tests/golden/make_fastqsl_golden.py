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


if __name__ == "__main__":
    phase = sys.argv[1] if len(sys.argv) > 1 else "trace"
    only = set(sys.argv[2:])
    if phase == "trace":
        lib = ctypes.CDLL(str(ROOT / "oracle" / "_ref" / "libfastqsl_ref.so"))
        lib.fq_ref_trace_all.restype = ctypes.c_int
        for name, spec in CASES.items():
            if not only or name in only:
                trace_case(name, spec, lib)
    elif phase == "q":
        for name in CASES:
            if not only or name in only:
                qcalc_case(name)
    else:
        raise SystemExit("phase must be 'trace' or 'q'")

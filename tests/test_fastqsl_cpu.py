"""FastQSL tracing and Q on the CPU: the oracle restatement
(oracle/fastqsl_oracle.py) against fixtures the reference's own FastQSL tracer
and QCalcPlane wrote (tests/golden/make_fastqsl_golden.py), and the C-ABI
exports of the library's FastQSL-compatible entry points.

QCalcPlane's restatement reproduces the reference's Q bit for bit from the
reference's traces.  The tracer's restatement runs in FP32 scalar NumPy
arithmetic, which cannot reproduce the device's fused multiply-adds, so its
lines are held to the same faces and to end points within 2e-2 cells on a
sample of seeds (the GPU tests hold the library's tracer to identity).
"""

import json
import sys
from pathlib import Path

import numpy as np
import pytest

GOLD = Path(__file__).resolve().parent / "golden" / "fastqsl"
CASES = sorted(p.stem for p in GOLD.glob("*.json"))


def load(name, with_field=False):
    meta = json.loads((GOLD / f"{name}.json").read_text())
    z = dict(np.load(GOLD / f"{name}.npz"))
    if not with_field:
        return meta, z, None
    sys.path.insert(0, str(GOLD.parent))
    import make_fastqsl_golden as M

    b, checksum = M.field(meta)
    assert checksum == meta["field_checksum"], "the TD field generator changed"
    return meta, z, b


@pytest.mark.parametrize("name", CASES)
def test_qcalc_plane_restatement_is_exact(name):
    from oracle import fastqsl_oracle as FO

    meta, z, _ = load(name)
    sh = tuple(meta["plane_shape"])
    r = lambda k: z[k].reshape(sh)  # noqa: E731
    q = FO.qcalc_plane(np.stack([r("x_end"), r("y_end"), r("z_end")], -1), r("flag_end"),
                       np.stack([r("x_start"), r("y_start"), r("z_start")], -1), r("flag_start"),
                       r("bz_start"), r("bz_end"), np.stack([r("bx_inp"), r("by_inp"), r("bz_inp")], -1),
                       meta["normal"])
    np.testing.assert_array_equal(q, z["q"])


@pytest.mark.parametrize("name", CASES)
def test_tracer_restatement_follows_reference(name):
    from oracle import fastqsl_oracle as FO

    meta, z, b = load(name, with_field=True)
    cur = None
    if meta["twist"]:
        import make_fastqsl_golden as M

        cur = np.stack(M.grid_curl(b))
    idx = np.random.default_rng(7).choice(meta["n_seeds"], 8, replace=False)
    dev = []
    for i in idx:
        o = FO.trace_seed(b, z["seeds"][i], meta["normal"], meta["step_len"], meta["tol"], cur)
        assert o["flag_end"] == z["flag_end"][i] and o["flag_start"] == z["flag_start"][i]
        dev.append(max(np.abs(o["end"] - [z["x_end"][i], z["y_end"][i], z["z_end"][i]]).max(),
                       np.abs(o["start"] - [z["x_start"][i], z["y_start"][i], z["z_start"][i]]).max()))
    assert np.median(dev) < 2e-2
    assert np.mean(np.array(dev) < 2e-2) >= 0.75


def test_fastqsl_entry_points_exported():
    from nfgs_b200 import _lib as L

    lib = L.lib()
    for sym in ("nfgs_trace_fastqsl", "nfgs_qcalc_plane"):
        assert hasattr(lib, sym)

"""FastQSL-compatible tracing and Q on the GPU (nfgs_trace_fastqsl,
nfgs_qcalc_plane, and the compute_y0_qmap / compute_bottom_qmap helpers)
against fixtures the reference's own FastQSL tracer and QCalcPlane wrote
(tests/golden/fastqsl/, tests/golden/make_fastqsl_golden.py) on TD99
flux-rope fields: seed planes at y = 0 (with the twist) and at the bottom.

The bar is identity: every seed's flags, end and start points, the B samples
at the seed and both ends, the B.n flag and the path length equal the
reference's bit for bit, the path length to 1e-12, the twist (a double sum
whose last bits may differ) to 1e-6 of its largest value, and Q (value and
NaN pattern) bit for bit.
"""

import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden" / "fastqsl"
CASES = sorted(p.stem for p in GOLD.glob("*.json"))


def load(name):
    import sys

    sys.path.insert(0, str(GOLD.parent))
    import make_fastqsl_golden as M

    meta = json.loads((GOLD / f"{name}.json").read_text())
    z = dict(np.load(GOLD / f"{name}.npz"))
    b, checksum = M.field(meta)
    assert checksum == meta["field_checksum"], "the TD field generator changed"
    return meta, z, b


def trace(meta, z, b):
    import torch

    from nfgs_b200 import qmap

    return qmap.trace_fastqsl(torch.as_tensor(b, device="cuda"), torch.as_tensor(z["seeds"], device="cuda"),
                              normal=meta["normal"], step_len=meta["step_len"], tol=meta["tol"],
                              twist=meta["twist"])


@pytest.mark.parametrize("name", CASES)
def test_traces_equal_reference(name):
    meta, z, b = load(name)
    tr = {k: v.cpu().numpy() for k, v in trace(meta, z, b).items()}
    np.testing.assert_array_equal(tr["flags"][0], z["flag_end"])
    np.testing.assert_array_equal(tr["flags"][1], z["flag_start"])
    np.testing.assert_array_equal(tr["ends"][0], np.stack([z["x_end"], z["y_end"], z["z_end"]], -1))
    np.testing.assert_array_equal(tr["ends"][1], np.stack([z["x_start"], z["y_start"], z["z_start"]], -1))
    for c, ax in enumerate("xyz"):
        np.testing.assert_array_equal(tr["bsamp"][c, 0], z[f"b{ax}_inp"])
        np.testing.assert_array_equal(tr["bsamp"][c, 1], z[f"b{ax}_end"])
        np.testing.assert_array_equal(tr["bsamp"][c, 2], z[f"b{ax}_start"])
    np.testing.assert_array_equal(tr["bflag"], z["b_flag"])
    np.testing.assert_allclose(tr["length"], z["line_len"], rtol=1e-12, atol=0)
    if meta["twist"]:
        np.testing.assert_allclose(tr["twist"], z["twist"], rtol=0, atol=1e-6 * np.abs(z["twist"]).max())
    codes = set(np.unique(np.concatenate([z["flag_end"], z["flag_start"]])).tolist())
    assert len(codes & {1, 2, 3, 4, 5, 6}) >= 3 and 42 in codes  # several faces and the edge code


@pytest.mark.parametrize("name", CASES)
def test_q_equals_reference(name):
    from nfgs_b200 import qmap

    meta, z, b = load(name)
    nv, nu = meta["plane_shape"]
    q = qmap.qcalc_plane(trace(meta, z, b), nu, nv, meta["normal"]).cpu().numpy()
    np.testing.assert_array_equal(q, z["q"])  # NaN positions equal as well


@pytest.mark.parametrize("name", CASES)
def test_qcalc_kernel_on_the_reference_traces(name):
    """The Q kernel alone, fed the reference tracer's own outputs."""
    import torch

    from nfgs_b200 import qmap

    meta, z, _ = load(name)
    nv, nu = meta["plane_shape"]
    dev = "cuda"
    tr = {"ends": torch.as_tensor(np.stack([np.stack([z["x_end"], z["y_end"], z["z_end"]], -1),
                                            np.stack([z["x_start"], z["y_start"], z["z_start"]], -1)]),
                                  device=dev).contiguous(),
          "flags": torch.as_tensor(np.stack([z["flag_end"], z["flag_start"]]), device=dev).contiguous(),
          "bsamp": torch.as_tensor(np.stack([np.stack([z[f"b{a}_inp"], z[f"b{a}_end"], z[f"b{a}_start"]])
                                             for a in "xyz"]), device=dev).contiguous()}
    q = qmap.qcalc_plane(tr, nu, nv, meta["normal"]).cpu().numpy()
    np.testing.assert_array_equal(q, z["q"])


def test_reference_helpers_reproduce_the_reference_maps():
    """compute_y0_qmap / compute_bottom_qmap with the reference's defaults
    give the reference's Q maps, flags, end points and twist."""
    from nfgs_b200 import qmap

    meta, z, b = load("td1_y0")
    r = qmap.compute_y0_qmap(b[0], b[1], b[2], include_twist=True)
    shape = tuple(meta["plane_shape"])
    np.testing.assert_array_equal(r["q"], z["q"])
    np.testing.assert_array_equal(r["flag_start"], z["flag_start"].reshape(shape))
    np.testing.assert_array_equal(r["end_xyz"], np.stack([z["x_end"], z["y_end"], z["z_end"]], -1).reshape(*shape, 3))
    np.testing.assert_allclose(r["twist"], z["twist"].reshape(shape), rtol=0, atol=1e-6 * np.abs(z["twist"]).max())
    meta, z, b = load("td1_bottom")
    r = qmap.compute_bottom_qmap(b[0], b[1], b[2])
    np.testing.assert_array_equal(r["q"], z["q"])
    np.testing.assert_array_equal(r["flag_end"], z["flag_end"].reshape(tuple(meta["plane_shape"])))

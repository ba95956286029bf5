"""record_iteration_diagnostics and stop_mode="fixed_point" on the GPU
(nfgs_step_diagnostics, nfgs_iterate_fixed_point) against fixtures from the
reference itself (tests/golden/diag/, written by
tests/golden/make_diag_golden.py; the oracle is pinned to the same fixtures
in tests/test_diag_cpu.py).

FP64 storage: every per-step diagnostic to 1e-7 relative (the ones whose
reference values are round-off of exact identities to 1e-9 absolute), the
fixed_point_criteria_met column exactly, the stop reason, best and final
iteration, the selected state (the final accepted iterate in fixed-point
mode) and its fields.  FP32 storage: the fixed-point run stops and its
diagnostics follow FP64's.
"""

import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden" / "diag"
CASES = sorted(p.stem for p in GOLD.glob("*.json"))
ROUNDOFF = ("poloidal_pde_residual_relative", "toroidal_pde_residual_relative", "h_k0_map_residual_relative",
            "h_k0_update_relative", "bottom_jz_imprint_relative")


def load(name):
    return json.loads((GOLD / f"{name}.json").read_text()), dict(np.load(GOLD / f"{name}.npz"))


def run(name, dtype):
    from nfgs_b200 import NFGSSolverGPU

    meta, data = load(name)
    nx, ny, nz = meta["shape"]
    s = NFGSSolverGPU(nx, ny, nz, *meta["spacing"], device="cuda", dtype=dtype, **meta["ctor"])
    s.set_bottom_vector_boundary(data["bx_in"], data["by_in"], data["bz_in"], zero_net_current=False, ijzbcor=3,
                                 **meta["bnd"])
    h = s.iterate(init_mode="gs_cfcf", verbose=False, **meta["iterate"])
    return meta, data, s, h


@pytest.mark.parametrize("name", CASES)
def test_step_diagnostics_fp64(name):
    meta, data, s, h = run(name, "float64")
    assert h["stop_reason"] == meta["stop_reason"]
    assert h["best_iter"] == meta["best_iter"]
    assert h["final_iter"] == meta["final_iter"]
    assert h["selected_state"] == meta["selected_state"]
    assert h["fixed_point_converged"] == meta["fixed_point_converged"]
    np.testing.assert_allclose(h["sigma"], data["hist_sigma"], rtol=1e-7)
    np.testing.assert_array_equal(h["fixed_point_criteria_met"], data["fixed_point_criteria_met"])
    for key in [k[5:] for k in data if k.startswith("diag_")]:
        want = data["diag_" + key]
        assert len(h[key]) == len(want), key
        if key in ROUNDOFF:
            assert np.max(np.abs(np.asarray(h[key]) - want)) < 1e-9, key
        else:
            np.testing.assert_allclose(h[key], want, rtol=1e-7, atol=1e-13, err_msg=key)
    if "final_Bx" in data:
        f = s.fields_to_numpy()
        for k in ("Bx", "By", "Bz", "Jx", "Jy", "Jz"):
            assert np.linalg.norm(f[k] - data["final_" + k]) <= 1e-7 * np.linalg.norm(data["final_" + k]), k


def test_fixed_point_fp32():
    meta, data, s, h = run("lowlou32_fixed_point", "float32")
    assert h["stop_reason"] == "fixed_point"
    assert abs(h["final_iter"] - meta["final_iter"]) <= 3
    n = min(len(h["phi_map_residual_relative"]), len(data["diag_phi_map_residual_relative"]))
    np.testing.assert_allclose(h["phi_map_residual_relative"][:n], data["diag_phi_map_residual_relative"][:n],
                               rtol=5e-2)
    np.testing.assert_allclose(h["alpha_clip_fraction"][:n], data["diag_alpha_clip_fraction"][:n], atol=2e-3)


def test_fixed_point_needs_diagnostics():
    from nfgs_b200 import NFGSSolverGPU

    meta, data = load("tiny_sigma_best")
    nx, ny, nz = meta["shape"]
    ctor = dict(meta["ctor"])
    ctor["record_iteration_diagnostics"] = False
    s = NFGSSolverGPU(nx, ny, nz, *meta["spacing"], device="cuda", dtype="float64", **ctor)
    s.set_bottom_vector_boundary(data["bx_in"], data["by_in"], data["bz_in"], zero_net_current=False, ijzbcor=3,
                                 **meta["bnd"])
    with pytest.raises(ValueError):
        s.iterate(max_iter=3, stop_mode="fixed_point", verbose=False)

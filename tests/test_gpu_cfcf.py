"""The cfcf start on the GPU (nfgs_iterate_cfcf_start, iterate(init_mode="cfcf"))
against fixtures from the reference itself (tests/golden/cfcf/, written by
tests/golden/make_cfcf_golden.py; the oracle is pinned to the same fixtures
in tests/test_cfcf_cpu.py).

FP64 storage must equal the reference's FP64 run to round-off: start state
(Phi_c, A_z, B, J) 1e-10 relative L2, start sigma_J / divB / energy 1e-9, the
mean B_c,z per height 1e-9, and the iterate history from the cfcf start
(stop reason, best iteration, sigma 1e-7).  FP32 storage: start state 2e-5
relative L2 and the start sigma_J within 1e-4.
"""

import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden" / "cfcf"
CASES = sorted(p.stem for p in GOLD.glob("*.json"))


def load(name):
    return json.loads((GOLD / f"{name}.json").read_text()), dict(np.load(GOLD / f"{name}.npz"))


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def solver(meta, data, dtype):
    from nfgs_b200 import NFGSSolverGPU

    nx, ny, nz = meta["shape"]
    s = NFGSSolverGPU(nx, ny, nz, *meta["spacing"], device="cuda", dtype=dtype, **meta["ctor"])
    s.set_bottom_vector_boundary(data["bx_in"], data["by_in"], data["bz_in"], zero_net_current=False, ijzbcor=3,
                                 **meta["bnd"])
    return s


@pytest.mark.parametrize("name", CASES)
def test_cfcf_start_fp64(name):
    meta, data = load(name)
    s = solver(meta, data, "float64")
    B, J, phi, az, _ = s.compute_initial_conditions(init_mode="cfcf")
    d = s._init_diagnostics
    assert d["init_mode"] == "cfcf"
    np.testing.assert_allclose(d["stable_cfcf_mean_bcz_by_height"], data["mean_bcz_by_height"], rtol=1e-9,
                               atol=1e-13)
    if "init_phi" in data:
        assert rel(phi, data["init_phi"]) < 1e-10
        assert rel(az, data["init_az"]) < 1e-10
    if "init_B" in data:
        assert rel(B, data["init_B"]) < 1e-10
        assert rel(J, data["init_J"]) < 1e-10
    h = s.iterate(init_mode="cfcf", max_iter=0, verbose=False)
    np.testing.assert_allclose([h["initial_sigma"], h["initial_divB"], h["initial_energy"]], data["init_scalars"],
                               rtol=1e-9)


@pytest.mark.parametrize("name", CASES)
def test_iterate_from_cfcf_fp64(name):
    meta, data = load(name)
    s = solver(meta, data, "float64")
    h = s.iterate(init_mode="cfcf", max_iter=meta["iters"], tol=1e-5, mu=1.0, patience=meta["patience"],
                  sigma_improvement_tol=1e-5, verbose=False)
    assert h["stop_reason"] == meta["stop_reason"]
    assert h["best_iter"] == meta["best_iter"]
    np.testing.assert_allclose(h["sigma"], data["hist_sigma"], rtol=1e-7)
    np.testing.assert_allclose(h["energy"], data["hist_energy"], rtol=1e-8)
    assert h["init_diagnostics"]["init_mode"] == "cfcf"


@pytest.mark.parametrize("name", ["small_rho1_unpadded", "lowlou32_rho05"])
def test_cfcf_start_fp32(name):
    meta, data = load(name)
    s = solver(meta, data, "float32")
    B, J, phi, az, _ = s.compute_initial_conditions(init_mode="cfcf")
    if "init_phi" in data:
        assert rel(phi, data["init_phi"]) < 2e-5
        assert rel(az, data["init_az"]) < 2e-5
    h = s.iterate(init_mode="cfcf", max_iter=5, patience=40, verbose=False)
    assert h["initial_sigma"] == pytest.approx(data["init_scalars"][0], rel=1e-4)
    assert np.isfinite(h["sigma"]).all()


def test_cfcf_handoff_error_policy_is_not_built():
    meta, data = load("tiny_rho05")
    from nfgs_b200 import NFGSSolverGPU

    nx, ny, nz = meta["shape"]
    s = NFGSSolverGPU(nx, ny, nz, *meta["spacing"], device="cuda", dtype="float64",
                      handoff_projection_policy="error", **meta["ctor"])
    s.set_bottom_vector_boundary(data["bx_in"], data["by_in"], data["bz_in"], zero_net_current=False, ijzbcor=3,
                                 **meta["bnd"])
    with pytest.raises(NotImplementedError):
        s.iterate(init_mode="cfcf", max_iter=2, verbose=False)

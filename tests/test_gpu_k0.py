"""k_h=0 closures on the GPU (horizontal_zero_mode_policy "coupled_k0" and
"constrained_spline_harmonic") against fixtures the reference wrote
(tests/golden/k0/, tests/golden/make_k0_golden.py; the oracle is pinned to
the same fixtures in tests/test_k0_cpu.py) and against the oracle.

FP64 storage: histories to 1e-9, the stop and best iteration exactly, the
selected state's H(z) to 1e-9 and its cropped fields to 1e-7, the closure's
diagnostics to 1e-6 (round-off quantities to an absolute floor), the per-step
h_k0 diagnostics to 1e-7.  FP32 storage: Low-Lou at 32^3 to the sigma stop
follows the FP64 solve.
"""

import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden" / "k0"
CASES = sorted(p.stem for p in GOLD.glob("*.json"))


def load(name):
    return json.loads((GOLD / f"{name}.json").read_text()), dict(np.load(GOLD / f"{name}.npz"))


def solver(meta, data, dtype):
    from nfgs_b200 import NFGSSolverGPU

    nx, ny, nz = meta["shape"]
    s = NFGSSolverGPU(nx, ny, nz, *meta["spacing"], device="cuda", dtype=dtype, **meta["ctor"])
    s.set_bottom_vector_boundary(data["bx_in"], data["by_in"], data["bz_in"], zero_net_current=False, ijzbcor=3,
                                 **meta["bnd"])
    return s


def rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("name", CASES)
def test_closure_fp64_matches_reference(name):
    meta, data = load(name)
    s = solver(meta, data, "float64")
    h = s.iterate(init_mode="gs_cfcf", verbose=False, **meta["iterate"])
    assert h["stop_reason"] == meta["stop_reason"]
    assert h["best_iter"] == meta["best_iter"]
    assert h["final_iter"] == meta["final_iter"]
    assert rel(h["sigma"], data["hist_sigma"]) < 1e-9
    assert rel(h["energy"], data["hist_energy"]) < 1e-9
    assert rel(h["divB"], data["hist_divB"]) < 1e-7
    policy = meta["ctor"]["horizontal_zero_mode_policy"]
    sd = h["source_diagnostics"][policy]
    assert rel(sd["profile_by_height"], data["profile"]) < 1e-9
    for key, want in meta["k0_final"].items():
        got = sd[key]
        if isinstance(want, (str, bool)):
            assert got == want, key
        elif key == "kkt_condition_number":
            assert got == pytest.approx(want, rel=1e-6)
        else:
            np.testing.assert_allclose(got, want, rtol=1e-6, atol=1e-10, err_msg=key)
    if "final_Bx" in data:
        f = s.fields_to_numpy()
        for k in ("Bx", "By", "Bz", "Jx", "Jy", "Jz"):
            assert np.linalg.norm(f[k] - data["final_" + k]) <= 1e-7 * np.linalg.norm(data["final_" + k]), k
    for k in data:
        if k.startswith("diag_"):
            np.testing.assert_allclose(h[k[5:]], data[k], rtol=1e-7, atol=1e-12, err_msg=k)


def test_closure_fp32_follows_fp64():
    meta, data = load("lowlou32_coupled")
    h32 = solver(meta, data, "float32").iterate(init_mode="gs_cfcf", verbose=False, **meta["iterate"])
    h64 = solver(meta, data, "float64").iterate(init_mode="gs_cfcf", verbose=False, **meta["iterate"])
    n = min(len(h32["sigma"]), len(h64["sigma"]), 60)
    np.testing.assert_allclose(h32["sigma"][:n], h64["sigma"][:n], rtol=2e-3)
    assert abs(h32["best_sigma"] - h64["best_sigma"]) <= 2e-2 * h64["best_sigma"]
    p32 = np.array(h32["source_diagnostics"]["coupled_k0"]["profile_by_height"])
    p64 = np.array(h64["source_diagnostics"]["coupled_k0"]["profile_by_height"])
    assert np.abs(p32 - p64).max() <= 2e-2 * np.abs(p64).max()


@pytest.mark.parametrize("name,init", [("spline_unpadded", "soft_cfcf"), ("coupled_tiny", "soft_cfcf"),
                                       ("coupled_legacy_mu", "gs_cfcf")])
def test_closure_repeat_and_starts_match_oracle(name, init):
    """A second iterate starts from the first solve's H(z) (the reference
    reconstructs every start with its running H_k0), and the soft_cfcf start
    carries H(z) too: GPU FP64 against the oracle."""
    from oracle.nfgs_oracle import OracleNFGS

    meta, data = load(name)
    s = solver(meta, data, "float64")
    nx, ny, nz = meta["shape"]
    ctor = {k: v for k, v in meta["ctor"].items() if k != "vertical_current_operator"}
    o = OracleNFGS(nx, ny, nz, *meta["spacing"], **ctor)
    o.set_bottom_vector_boundary(data["bx_in"], data["by_in"], data["bz_in"], zero_net_current=False, ijzbcor=3,
                                 **meta["bnd"])
    it = dict(meta["iterate"], max_iter=5)
    for _ in range(2):
        h = s.iterate(init_mode=init, verbose=False, **it)
        ho = o.iterate(init_mode=init, **it)
        assert rel(h["sigma"], ho["sigma"]) < 1e-9
        assert h["initial_sigma"] == pytest.approx(ho["initial_sigma"], rel=1e-9)
        pol = meta["ctor"]["horizontal_zero_mode_policy"]
        assert rel(h["source_diagnostics"][pol]["profile_by_height"],
                   ho["source_diagnostics"][pol]["profile_by_height"]) < 1e-9
        assert h["source_diagnostics"][pol]["ode_residual_relative_max"] == pytest.approx(
            ho["source_diagnostics"][pol]["ode_residual_relative_max"], rel=1e-7)


def test_closure_adaptive_mu_rollback_matches_oracle():
    """Rollbacks restore the best state's H(z) with its scalars."""
    from oracle.nfgs_oracle import OracleNFGS

    meta, data = load("coupled_face_unpadded")
    s = solver(meta, data, "float64")
    nx, ny, nz = meta["shape"]
    ctor = {k: v for k, v in meta["ctor"].items() if k != "vertical_current_operator"}
    o = OracleNFGS(nx, ny, nz, *meta["spacing"], **ctor)
    o.set_bottom_vector_boundary(data["bx_in"], data["by_in"], data["bz_in"], zero_net_current=False, ijzbcor=3,
                                 **meta["bnd"])
    it = dict(max_iter=25, patience=40, tol=1e-6, mu=1.0, sigma_improvement_tol=None, adaptive_mu=True,
              divergence_factor=0.995, mu_backoff=0.5)
    h = s.iterate(verbose=False, **it)
    ho = o.iterate(**it)
    assert h["rollback"] == ho["rollback"]
    assert sum(ho["rollback"]) >= 1
    m = np.isfinite(ho["sigma"])
    assert rel(np.array(h["sigma"])[m], np.array(ho["sigma"])[m]) < 1e-9
    assert rel(h["source_diagnostics"]["coupled_k0"]["profile_by_height"],
               ho["source_diagnostics"]["coupled_k0"]["profile_by_height"]) < 1e-9

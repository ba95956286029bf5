"""Pin the soft_cfcf oracle against fixtures produced by the reference solver.

``tests/golden/soft_cfcf/*`` were written by
``tests/golden/make_soft_cfcf_golden.py`` running the reference
``NFGSSolverGPU`` in FP64 on CPU: modal profiles, the soft_cfcf initial
state, its diagnostics and an ``iterate(init_mode="soft_cfcf")`` history.
The oracle is FP64 too; the modal normal matrices square the conditioning of
fourth-order rows, so round-off of the bottom transform (SciPy vs torch FFT)
reaches the profiles at ~1e-14 relative.
"""

import json
from pathlib import Path

import numpy as np
import pytest

from oracle import soft_cfcf_oracle as SO
from oracle.nfgs_oracle import OracleNFGS, dct2, dst2

GOLD = Path(__file__).resolve().parent / "golden" / "soft_cfcf"
CASES = sorted(p.stem for p in GOLD.glob("*.json"))


def load(name):
    return json.loads((GOLD / f"{name}.json").read_text()), dict(np.load(GOLD / f"{name}.npz"))


def oracle(meta, data):
    ctor = {k: v for k, v in meta["ctor"].items() if k != "vertical_current_operator"}
    nx, ny, nz = meta["shape"]
    dx, dy, dz = meta["spacing"]
    o = OracleNFGS(nx, ny, nz, dx, dy, dz, **ctor)
    o.set_bottom_vector_boundary(data["bx_in"], data["by_in"], data["bz_in"], zero_net_current=False, ijzbcor=3,
                                 **meta["bnd"])
    return o


def rel_max(a, b):
    return float(np.abs(np.asarray(a) - b).max() / max(np.abs(b).max(), 1e-300))


def test_cases_present():
    assert len(CASES) == 4


@pytest.mark.parametrize("name", CASES)
def test_modal_profiles(name):
    meta, data = load(name)
    o = oracle(meta, data)
    assert [o.Nx, o.Ny, o.Nz] == meta["calc_grid"]
    assert o.soft_cfcf_epsilon == pytest.approx(meta["soft_cfcf_epsilon"], rel=0, abs=0)
    k = np.sqrt(np.maximum(-o.lam_neumann(), 0.0))
    pb = dct2(o.Phi_above_bottom)
    pb[0, 0] = 0.0
    ph = SO.modal_profiles(k, pb, "phi", o.Nz, o.dz, o.soft_cfcf_epsilon, o.soft_cfcf_normal_ridge)
    assert rel_max(ph.reshape(data["phi_hat"].shape), data["phi_hat"]) < 1e-12
    ka = np.sqrt(np.maximum(-o.lam_dirichlet(), 0.0))
    ab = dst2(o.Az_bottom[1:-1, 1:-1])
    ah = SO.modal_profiles(ka, ab, "az", o.Nz, o.dz, o.soft_cfcf_epsilon, o.soft_cfcf_normal_ridge)
    assert rel_max(ah.reshape(data["az_hat"].shape), data["az_hat"]) < 1e-13
    # the (0,0) Phi mode is not solved: zero at every height
    assert np.all(ph[:, 0] == 0.0)


@pytest.mark.parametrize("name", CASES)
def test_initial_state_and_diagnostics(name):
    meta, data = load(name)
    o = oracle(meta, data)
    B, J, phi, az, _bc = o.compute_initial_conditions("soft_cfcf")
    assert rel_max(phi, data["init_phi"]) < 1e-12
    assert rel_max(az, data["init_az"]) < 1e-13
    if "init_B" in data:
        assert rel_max(B, data["init_B"]) < 1e-12
        assert rel_max(J, data["init_J"]) < 1e-11
    np.testing.assert_allclose([o.compute_sigma(B, J), o.compute_divB(B), o.compute_energy(B)],
                               data["init_scalars"], rtol=1e-12)
    for key in ("curl_current_energy", "current_energy", "objective"):
        assert o.soft_cfcf_diagnostics[key] == pytest.approx(meta["soft_cfcf"][key], rel=1e-12), key
    # exact constraints: bottom planes, zero A_z walls, transparent tops
    np.testing.assert_array_equal(phi[0], o.Phi_above_bottom)
    assert np.all(az[:, 0, :] == 0.0) and np.all(az[:, :, -1] == 0.0)
    assert abs(meta["soft_cfcf"]["top_phi_transparent_rms"]) < 1e-12


@pytest.mark.parametrize("name", CASES)
def test_iterate_history(name):
    meta, data = load(name)
    o = oracle(meta, data)
    h = o.iterate(init_mode="soft_cfcf", max_iter=meta["iters"], tol=1e-5, mu=1.0, patience=meta["patience"],
                  sigma_improvement_tol=1e-5)
    np.testing.assert_allclose(h["sigma"], data["hist_sigma"], rtol=1e-11)
    np.testing.assert_allclose(h["energy"], data["hist_energy"], rtol=1e-11)
    assert h["best_iter"] == meta["best_iter"]
    assert h["stop_reason"] == meta["stop_reason"]
    # no zero-source solve at the start: one ratio per iteration
    assert len(o.source_zero_mode_history) == meta["source_zero_mode_history_length"]


def test_banded_cholesky_matches_dense():
    """The banded solve with its floor equals a dense SPD solve."""
    rng = np.random.default_rng(3)
    n, bw, batch = 23, 3, 5
    A = np.zeros((batch, n, n))
    for b in range(batch):
        M = np.zeros((n + bw, n))
        for i in range(n + bw):
            lo = max(0, i - bw)
            M[i, lo:min(n, i + 1)] = rng.normal(size=min(n, i + 1) - lo)
        A[b] = M.T @ M + np.eye(n)
    lower = np.zeros((bw + 1, batch, n))
    for d in range(bw + 1):
        for i in range(d, n):
            lower[d, :, i] = A[:, i, i - d]
    rhs = rng.normal(size=(batch, n))
    x = SO.banded_cholesky_solve(lower, rhs)
    ref = np.linalg.solve(A, rhs[..., None])[..., 0]
    np.testing.assert_allclose(x, ref, rtol=1e-10, atol=1e-12)


def test_profiles_are_linear_in_the_bottom_value():
    """Every constant of the modal rows is proportional to the bottom value,
    so the profile of bottom b is b times the profile of bottom 1."""
    k = np.linspace(0.05, 2.0, 17)
    one = SO.modal_profiles(k, np.ones_like(k), "phi", 12, 0.7, 2e-3, 0.0)
    b = np.linspace(-3.0, 5.0, 17)
    prof = SO.modal_profiles(k, b, "phi", 12, 0.7, 2e-3, 0.0)
    np.testing.assert_allclose(prof, one * b[None], rtol=1e-12, atol=1e-14)
    # top transparent row: (3u_N - 4u_{N-1} + u_{N-2})/(2dz) + k u_N = 0
    for kind in ("phi", "az"):
        p = SO.modal_profiles(k, b, kind, 12, 0.7, 2e-3, 1e-9)
        top = (3 * p[-1] - 4 * p[-2] + p[-3]) / (2 * 0.7) + k * p[-1]
        assert np.abs(top).max() < 1e-12 * max(np.abs(p).max(), 1.0)
    # bottom Neumann row of Phi: (-3p_0 + 4p_1 - p_2)/(2dz) = k p_0
    bot = (-3 * prof[0] + 4 * prof[1] - prof[2]) / (2 * 0.7) - k * prof[0]
    assert np.abs(bot).max() < 1e-12 * np.abs(prof).max()

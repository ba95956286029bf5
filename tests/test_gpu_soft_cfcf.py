"""soft_cfcf start on the GPU (nfgs_iterate_soft_cfcf_start) against the oracle
and the reference fixtures.

FP64 storage: the modal solve is FP64 in both and follows the same operation
order; the device transforms are dense contractions, the oracle's SciPy FFTs,
so start states agree to ~1e-13 and histories to round-off.  FP32 storage
solves the modes in FP64 and stores FP32 profiles; the FP32 bar is stated
per comparison.
"""

import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden" / "soft_cfcf"
CASES = sorted(p.stem for p in GOLD.glob("*.json"))
STOP = dict(tol=1e-5, mu=1.0, sigma_improvement_tol=1e-5)


def load(name):
    return json.loads((GOLD / f"{name}.json").read_text()), dict(np.load(GOLD / f"{name}.npz"))


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def solver(meta, data, dtype):
    from nfgs_b200 import NFGSSolverGPU

    nx, ny, nz = meta["shape"]
    dx, dy, dz = meta["spacing"]
    s = NFGSSolverGPU(nx, ny, nz, dx, dy, dz, device="cuda", dtype=dtype, **meta["ctor"])
    s.set_bottom_vector_boundary(data["bx_in"], data["by_in"], data["bz_in"], zero_net_current=False, ijzbcor=3,
                                 **meta["bnd"])
    return s


def start_state(s, **kw):
    """Begin an iteration with the soft_cfcf start; (phi, az, initial sigma/divB/E)."""
    from nfgs_b200 import _lib as L
    from nfgs_b200.learned import start_state_views

    s._iterate_begin(max_iter=10, verbose=False, init_mode="soft_cfcf", **kw)
    phi, az = start_state_views(s)
    sc = np.zeros(3)
    L.check(s._lib.nfgs_iterate_initial(s._h, L.dptr(sc)))
    return phi.cpu().numpy().astype(np.float64), az.cpu().numpy().astype(np.float64), sc


@pytest.mark.parametrize("name", CASES)
def test_start_state_fp64(name):
    meta, data = load(name)
    s = solver(meta, data, "float64")
    assert [s.Nx, s.Ny, s.Nz] == meta["calc_grid"]
    phi, az, sc = start_state(s)
    assert rel(phi, data["init_phi"]) < 1e-11
    assert rel(az, data["init_az"]) < 1e-11
    np.testing.assert_array_equal(phi[0], s.Phi_above_bottom)
    np.testing.assert_allclose(sc, data["init_scalars"], rtol=1e-10)
    diag = s._init_diagnostics
    assert diag["init_mode"] == "soft_cfcf"
    assert diag["soft_cfcf_epsilon"] == meta["soft_cfcf_epsilon"]
    for key in ("curl_current_energy", "current_energy", "objective"):
        assert diag["soft_cfcf"][key] == pytest.approx(meta["soft_cfcf"][key], rel=1e-10), key


@pytest.mark.parametrize("name", CASES)
def test_history_fp64(name):
    meta, data = load(name)
    s = solver(meta, data, "float64")
    h = s.iterate(init_mode="soft_cfcf", max_iter=meta["iters"], patience=meta["patience"], verbose=False, **STOP)
    np.testing.assert_allclose(h["sigma"], data["hist_sigma"], rtol=1e-9)
    np.testing.assert_allclose(h["energy"], data["hist_energy"], rtol=1e-9)
    assert h["best_iter"] == meta["best_iter"]
    assert h["stop_reason"] == meta["stop_reason"]
    assert h["init_diagnostics"]["init_mode"] == "soft_cfcf"
    assert len(s._source_zero_mode_history) == meta["source_zero_mode_history_length"]


@pytest.mark.parametrize("name", CASES)
def test_fp32(name):
    """FP32 storage: start state within 2e-6 of the reference (FP32 profiles
    and transforms); the sigma history within 1e-3 over the first iterations
    (the same bar as the gs_cfcf FP32 path on these cases)."""
    meta, data = load(name)
    s = solver(meta, data, "float32")
    phi, az, sc = start_state(s)
    assert rel(phi, data["init_phi"]) < 2e-6
    assert rel(az, data["init_az"]) < 2e-6
    np.testing.assert_allclose(sc[0], data["init_scalars"][0], rtol=2e-5)
    s = solver(meta, data, "float32")
    h = s.iterate(init_mode="soft_cfcf", max_iter=meta["iters"], patience=meta["patience"], verbose=False, **STOP)
    n = min(6, len(h["sigma"]))
    np.testing.assert_allclose(h["sigma"][:n], data["hist_sigma"][:n], rtol=1e-3)


def test_matches_oracle_at_130():
    """A 128 x 128 x 64 TD-type boundary (calc 130^2 x 65: 16,900 Phi modes,
    16,384 A_z modes): FP64 start state and first steps against the oracle."""
    from nfgs_b200 import NFGSSolverGPU
    from nfgs_b200.synthetic import td_bottom
    from oracle.nfgs_oracle import OracleNFGS

    n, nz = 128, 64
    bx, by, bz = td_bottom(n, n, seed=4, extent=8.0)
    h = 16.0 / (n - 1)
    kw = dict(bottom_divergence_robin_weight=0.5, horizontal_zero_mode_policy="frozen_linear_harmonic",
              d0_zero_mode_policy="project", source_zero_mode_policy="project", soft_cfcf_epsilon=0.3)
    s = NFGSSolverGPU(n, n, nz, h, h, h, device="cuda", dtype="float64", vertical_current_operator="staggered_face",
                      **kw)
    s.set_bottom_vector_boundary(bx, by, bz, zero_net_current=False, smooth_passes=0, ijzbcor=3)
    o = OracleNFGS(n, n, nz, h, h, h, **kw)
    o.set_bottom_vector_boundary(bx, by, bz, zero_net_current=False, smooth_passes=0, ijzbcor=3)
    phi, az, sc = start_state(s)
    B, J, ophi, oaz, _ = o.compute_initial_conditions("soft_cfcf")
    assert rel(phi, ophi) < 1e-11
    assert rel(az, oaz) < 1e-11
    np.testing.assert_allclose(sc, [o.compute_sigma(B, J), o.compute_divB(B), o.compute_energy(B)], rtol=1e-10)
    for key in ("curl_current_energy", "current_energy", "objective"):
        assert s._init_diagnostics["soft_cfcf"][key] == pytest.approx(o.soft_cfcf_diagnostics[key], rel=1e-10)
    s2 = NFGSSolverGPU(n, n, nz, h, h, h, device="cuda", dtype="float64", vertical_current_operator="staggered_face",
                       **kw)
    s2.set_bottom_vector_boundary(bx, by, bz, zero_net_current=False, smooth_passes=0, ijzbcor=3)
    hg = s2.iterate(init_mode="soft_cfcf", max_iter=4, patience=40, verbose=False, **STOP)
    ho = o.iterate(init_mode="soft_cfcf", max_iter=4, patience=40, **STOP)
    np.testing.assert_allclose(hg["sigma"], ho["sigma"], rtol=1e-9)


def test_start_is_replaced_only_before_advance():
    from nfgs_b200 import NFGSSolverGPU
    from nfgs_b200 import _lib as L

    meta, data = load(CASES[0])
    s = solver(meta, data, "float64")
    s.iterate(max_iter=2, verbose=False)
    out = np.zeros(4)
    code = s._lib.nfgs_iterate_soft_cfcf_start(s._h, 1e-3, 0.0, L.dptr(out))
    assert code == L.NFGS_ESTATE
    s._iterate_begin(max_iter=5, verbose=False)
    assert s._lib.nfgs_iterate_soft_cfcf_start(s._h, -1.0, 0.0, L.dptr(out)) == L.NFGS_EINVAL
    ctor = {k: v for k, v in meta["ctor"].items() if k != "buffer_thickness"}
    t = NFGSSolverGPU(12, 12, 4, 1.0, 1.0, 1.0, device="cuda", pad_calculation_domain=False, **ctor)
    rng = np.random.default_rng(0)
    t.set_bottom_vector_boundary(rng.normal(size=(12, 12)) * 0.1, rng.normal(size=(12, 12)) * 0.1,
                                 rng.normal(size=(12, 12)), zero_net_current=False)
    assert t.Nz == 4
    with pytest.raises(ValueError, match="Nz >= 5"):
        t.iterate(init_mode="soft_cfcf", max_iter=2, verbose=False)


@pytest.mark.parametrize("mode", ["gs_cfcf", "soft_cfcf"])
def test_compute_initial_conditions(mode):
    """NFGSSolverGPU.compute_initial_conditions returns the reference's start
    state (B, J, Phi_c, A_z, B_c) for both built start modes (FP64)."""
    if mode == "soft_cfcf":
        meta, data = load("small_eps_ridge")
    else:
        gold = Path(__file__).resolve().parent / "golden"
        meta = json.loads((gold / "small_rho03_buffer.json").read_text())
        data = dict(np.load(gold / "small_rho03_buffer.npz"))
    s = solver(meta, data, "float64")
    B, J, phi, az, bc = s.compute_initial_conditions(init_mode=mode)
    assert B.shape == (3, s.Nz, s.Ny, s.Nx) and phi.shape == (s.Nz, s.Ny, s.Nx)
    assert rel(phi, data["init_phi"]) < 1e-10
    assert rel(az, data["init_az"]) < 1e-10
    if "init_B" in data:
        assert rel(B, data["init_B"]) < 1e-10
        assert rel(J, data["init_J"]) < 1e-9
    np.testing.assert_allclose(bc, B - s.B_background, rtol=0, atol=1e-12)

"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

FP64 storage runs the same kernels as FP32 with double precision
everywhere, so it must agree with the FP64 oracle to round-off: this pins
the kernel logic.  FP32 storage is then checked against the same oracle
with FP32 tolerances stated per comparison.
"""

import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden"
CASES = sorted(p.stem for p in GOLD.glob("*.json"))


def load(name):
    meta = json.loads((GOLD / f"{name}.json").read_text())
    return meta, dict(np.load(GOLD / f"{name}.npz"))


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def build(meta, data, dtype):
    from nfgs_b200 import NFGSSolverGPU
    from oracle.nfgs_oracle import OracleNFGS

    ctor = dict(meta["ctor"])
    nx, ny, nz = meta["shape"]
    dx, dy, dz = meta["spacing"]
    s = NFGSSolverGPU(nx, ny, nz, dx, dy, dz, device="cuda", dtype=dtype, **ctor)
    s.set_bottom_vector_boundary(data["bx_in"], data["by_in"], data["bz_in"], zero_net_current=False, ijzbcor=3,
                                 **meta["bnd"])
    octor = {k: v for k, v in ctor.items() if k != "vertical_current_operator"}
    o = OracleNFGS(nx, ny, nz, dx, dy, dz, **octor)
    o.set_bottom_vector_boundary(data["bx_in"], data["by_in"], data["bz_in"], zero_net_current=False, ijzbcor=3,
                                 **meta["bnd"])
    return s, o


@pytest.mark.parametrize("name", CASES)
def test_setup_fp64(name):
    meta, data = load(name)
    s, o = build(meta, data, "float64")
    assert [s.Nx, s.Ny, s.Nz] == meta["calc_grid"]
    assert s._bottom_current_grid_mode == meta["bottom_current_grid_mode"]
    for key, ref in [("Bz_obs", o.Bz_obs), ("Bx_obs", o.Bx_obs), ("By_obs", o.By_obs), ("Jz_obs", o.Jz_obs),
                     ("Az_bottom", o.Az_bottom), ("Jz_toroidal_boundary", o.Jz_T),
                     ("Phi_above_bottom", o.Phi_above_bottom), ("Bz_above", o.Bz_above), ("D0", o.D0),
                     ("bottom_dphi_c_target", o.bottom_dphi_c_target)]:
        assert rel(getattr(s, key), ref) < 1e-11, key
    assert rel(s.B_background, o.B_background) < 1e-11
    assert rel(s.gaussian_above_bottom_field(), o.gaussian_above_bottom_field()) < 1e-11
    if o.H is not None:
        np.testing.assert_allclose(s._H_k0_bottom_target, o.H[:, 0], rtol=1e-9, atol=1e-13)
    for k, v in o.gaussian_separation_diagnostics.items():
        if isinstance(v, float):
            assert abs(s.gaussian_separation_diagnostics[k] - v) <= 1e-8 * abs(v) + 1e-11, k


@pytest.mark.parametrize("name", CASES)
def test_init_and_steps_fp64(name):
    meta, data = load(name)
    s, o = build(meta, data, "float64")
    s.iterate(max_iter=0, verbose=False)
    phi, az, sc = s._get_state(1)
    B, J, ophi, oaz, Bc = o.compute_initial_conditions()
    assert rel(phi, ophi) < 1e-10
    assert rel(az, oaz) < 1e-10
    np.testing.assert_allclose(sc, [o.compute_sigma(B, J), o.compute_divB(B), o.compute_energy(B)], rtol=1e-9)
    st = (B, J, ophi, oaz, Bc)
    for mu in (1.0, meta["mu2"]):
        s._step(mu)
        st = o.iteration_step(*st, mu=mu)
        phi, az, sc = s._get_state(1)
        assert rel(phi, st[2]) < 1e-9, mu
        assert rel(az, st[3]) < 1e-9, mu
        np.testing.assert_allclose(sc, [o.compute_sigma(st[0], st[1]), o.compute_divB(st[0]),
                                        o.compute_energy(st[0])], rtol=1e-8)


@pytest.mark.parametrize("name", CASES)
def test_iterate_fp64_matches_reference_history(name):
    meta, data = load(name)
    s, o = build(meta, data, "float64")
    h = s.iterate(max_iter=meta["iters"], tol=1e-5, mu=1.0, patience=meta["patience"],
                  sigma_improvement_tol=1e-5, verbose=False, check_every=4)
    assert h["stop_reason"] == meta["stop_reason"]
    assert h["best_iter"] == meta["best_iter"]
    assert h["final_iter"] == meta["final_iter"]
    np.testing.assert_allclose(h["sigma"], data["hist_sigma"], rtol=1e-7)
    np.testing.assert_allclose(h["energy"], data["hist_energy"], rtol=1e-8)
    np.testing.assert_allclose(h["divB"], data["hist_divB"], rtol=1e-6)
    assert abs(h["best_sigma"] - meta["best_sigma"]) < 1e-8 * meta["best_sigma"]
    assert abs(h["final_vs_best_B_relative"] - meta["final_vs_best_B_relative"]) <= \
        1e-6 * meta["final_vs_best_B_relative"] + 1e-12
    f = s.fields_to_numpy()
    for k in ("Bx", "By", "Bz", "Jx", "Jy", "Jz"):
        if "final_" + k in data:
            assert rel(f[k], data["final_" + k]) < 1e-7, k
        else:
            assert rel(f[k][::2, ::2, ::2], data["final_" + k + "_s2"]) < 1e-6, k
    sd = meta["source_diagnostics"]
    got = h["source_diagnostics"]
    for k in ("bottom_reconstruction_rms", "correction_bottom_rms", "top_robin_rms", "top_phi_robin_rms",
              "top_upward_source_rms", "top_upward_source_ratio", "bottom_divergence_rms",
              "bottom_divergence_relative", "bottom_dphi_residual_rms", "source_zero_mode_ratio_last",
              "source_zero_mode_ratio_max"):
        assert abs(got[k] - sd[k]) <= 1e-6 * abs(sd[k]) + 1e-10, k


@pytest.mark.parametrize("name", CASES)
def test_iterate_fp32_against_fp64_oracle(name):
    """FP32 storage (the production dtype) against the FP64 oracle.

    Tolerances: gs_cfcf state 2e-5 relative L2, first-step sigma 1e-4
    relative; the full history agrees to 2e-3 relative while the stop
    iteration and best iteration match the FP64 run.
    """
    meta, data = load(name)
    s, o = build(meta, data, "float32")
    s.iterate(max_iter=0, verbose=False)
    phi, az, sc = s._get_state(1)
    B, J, ophi, oaz, Bc = o.compute_initial_conditions()
    assert rel(phi, ophi) < 2e-5
    assert rel(az, oaz) < 2e-5
    np.testing.assert_allclose(sc[0], o.compute_sigma(B, J), rtol=1e-4)
    h = s.iterate(max_iter=meta["iters"], tol=1e-5, mu=1.0, patience=meta["patience"],
                  sigma_improvement_tol=1e-5, verbose=False)
    n = min(len(h["sigma"]), len(data["hist_sigma"]))
    np.testing.assert_allclose(h["sigma"][:n], data["hist_sigma"][:n], rtol=2e-3)
    f = s.fields_to_numpy()
    assert f["Bx"].dtype == np.float32


def test_per_step_callback_and_verbose(capsys):
    meta, data = load("tiny_rho05")
    s, o = build(meta, data, "float64")
    seen = []

    def cb(n, sigma, B, J):
        seen.append((n, sigma, B.shape, J.shape))

    h = s.iterate(max_iter=5, patience=40, verbose=True, per_step_callback=cb)
    assert [x[0] for x in seen] == list(range(1, 6))
    np.testing.assert_allclose([x[1] for x in seen], h["sigma"], rtol=0)
    assert seen[0][2] == (3, s.Nz, s.Ny, s.Nx)
    out = capsys.readouterr().out
    assert "Initial  sigma=" in out and "Iter    1 |" in out


def test_wrong_call_order_raises():
    from nfgs_b200 import NFGSSolverGPU

    s = NFGSSolverGPU(16, 14, 10, 1.0, 1.0, 1.0, dtype="float32")
    with pytest.raises(RuntimeError):
        s.fields_to_numpy()
    with pytest.raises(RuntimeError):
        s.iterate(max_iter=3, verbose=False)


def test_deterministic_reductions():
    meta, data = load("small_rho03_buffer")
    s1, _ = build(meta, data, "float32")
    s2, _ = build(meta, data, "float32")
    h1 = s1.iterate(max_iter=8, patience=40, verbose=False)
    h2 = s2.iterate(max_iter=8, patience=40, verbose=False)
    assert h1["sigma"] == h2["sigma"]
    assert h1["energy"] == h2["energy"]


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_fields_into_matches_fp64_export(dtype):
    """nfgs_fields_into (solver dtype, pinned chunked copy) returns exactly
    the FP64 export of nfgs_fields rounded to the solver dtype, cropped and
    uncropped, and on a second call into fresh host memory."""
    import ctypes as C

    from nfgs_b200 import _lib as L

    meta, data = load("small_rho03_buffer")
    s, _ = build(meta, data, dtype)
    s.iterate(max_iter=6, patience=40, verbose=False)
    lib = L.lib()
    for crop in (1, 0):
        dims = (C.c_int32 * 3)()
        n_full = 6 * s.Nz * s.Ny * s.Nx
        ref = np.zeros(n_full)
        L.check(lib.nfgs_fields(s._h, 0, crop, L.dptr(ref), dims))
        n = 6 * dims[0] * dims[1] * dims[2]
        want = ref[:n].astype(np.dtype(dtype))
        for _ in range(2):
            got = np.full(n, np.nan, dtype=np.dtype(dtype))
            dims2 = (C.c_int32 * 3)()
            code = L.NFGS_F32 if dtype == "float32" else L.NFGS_F64
            L.check(lib.nfgs_fields_into(s._h, 0, crop, got.ctypes.data_as(C.c_void_p), code, dims2))
            assert tuple(dims2) == tuple(dims)
            np.testing.assert_array_equal(got, want)
    f = s.fields_to_numpy()
    assert f["Bx"].dtype == np.dtype(dtype)
    with pytest.raises(ValueError):
        L.check(lib.nfgs_fields_into(s._h, 0, 1, np.zeros(4).ctypes.data_as(C.c_void_p), 7, None))

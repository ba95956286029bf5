"""k_h=0 closures on the CPU.

* The oracle's coupled_k0 and constrained_spline_harmonic restatement
  (oracle/k0_oracle.py with OracleNFGS) against fixtures the reference wrote
  (tests/golden/make_k0_golden.py): sigma / energy / divB histories, the stop,
  the selected state's H(z) profile, its cropped fields, the closure's
  diagnostics and the per-step h_k0 diagnostics.
* The library's host-built linear map of the fit (nfgs_k0_operator, no
  device needed) against the oracle's least-squares / KKT solves.
"""

import json
from pathlib import Path

import numpy as np
import pytest

GOLD = Path(__file__).resolve().parent / "golden" / "k0"
SMALL = ["coupled_tiny", "coupled_legacy_mu", "coupled_face_unpadded", "spline_tiny", "spline_buffer_face",
         "spline_unpadded"]


def load(name):
    meta = json.loads((GOLD / f"{name}.json").read_text())
    return meta, np.load(GOLD / f"{name}.npz")


def rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def run_oracle(meta, z):
    from oracle.nfgs_oracle import OracleNFGS

    nx, ny, nz = meta["shape"]
    ctor = {k: v for k, v in meta["ctor"].items() if k != "vertical_current_operator"}
    o = OracleNFGS(nx, ny, nz, *meta["spacing"], **ctor)
    o.set_bottom_vector_boundary(z["bx_in"], z["by_in"], z["bz_in"], zero_net_current=False, ijzbcor=3,
                                 **meta["bnd"])
    return o, o.iterate(**meta["iterate"])


# absolute floor for diagnostics that are round-off by construction (the
# spline's top derivative, the unsmoothed face residual)
ABS = 1e-12


@pytest.mark.parametrize("name", SMALL)
def test_oracle_matches_reference_closure(name):
    meta, z = load(name)
    o, h = run_oracle(meta, z)
    assert h["stop_reason"] == meta["stop_reason"]
    assert h["best_iter"] == meta["best_iter"]
    assert rel(h["sigma"], z["hist_sigma"]) < 1e-10
    assert rel(h["energy"], z["hist_energy"]) < 1e-10
    assert rel(h["divB"], z["hist_divB"]) < 1e-8
    policy = meta["ctor"]["horizontal_zero_mode_policy"]
    sd = h["source_diagnostics"][policy]
    assert rel(sd["profile_by_height"], z["profile"]) < 1e-10
    for key, want in meta["k0_final"].items():
        got = sd[key]
        if isinstance(want, (str, bool)):
            assert got == want, key
        else:
            np.testing.assert_allclose(got, want, rtol=1e-8, atol=ABS, err_msg=key)
    f = o.fields_to_numpy(True)
    for k in ("Bx", "By", "Bz", "Jx", "Jy", "Jz"):
        assert rel(f[k], z["final_" + k]) < 1e-10, k
    for k in z.files:
        if k.startswith("diag_"):
            np.testing.assert_allclose(h[k[5:]], z[k], rtol=1e-8, atol=1e-14, err_msg=k)


def test_spline_state_jz_is_the_face_average():
    """With the constrained spline all three current components come from the
    face current (nfgs_solver.py:5915-5935): the state J_z of an interior
    plane is (J_z(k-1) + 2 J_z(k) + J_z(k+1)) / 4 of the -lap_xy A_z current."""
    from oracle.nfgs_oracle import OracleNFGS, lap_xy

    meta, z = load("spline_tiny")
    nx, ny, nz = meta["shape"]
    ctor = {k: v for k, v in meta["ctor"].items() if k != "vertical_current_operator"}
    o = OracleNFGS(nx, ny, nz, *meta["spacing"], **ctor)
    o.set_bottom_vector_boundary(z["bx_in"], z["by_in"], z["bz_in"], zero_net_current=False, ijzbcor=3,
                                 **meta["bnd"])
    B, J, phi, az, _ = o.compute_initial_conditions()
    jz = -lap_xy(az, o.dx, o.dy)
    jz[0] = o.Jz_T
    jz[-1] = 0.0
    jz[:, :, 0] = jz[:, :, -1] = 0.0
    jz[:, 0, :] = jz[:, -1, :] = 0.0
    jz[0] = o.Jz_T
    want = 0.25 * (jz[:-2] + 2 * jz[1:-1] + jz[2:])
    np.testing.assert_allclose(J[2, 1:-1, 1:-1, 1:-1], want[:, 1:-1, 1:-1], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("spline,legacy,nb,smooth,nz,dz", [
    (0, 0, 8, 1e-3, 9, 1.0), (0, 0, 8, 0.0, 17, 0.5), (0, 1, 8, 1e-2, 12, 0.8),
    (1, 0, 8, 1e-3, 33, 1.0), (1, 0, 5, 1e-2, 7, 1.0), (1, 0, 6, 0.0, 20, 0.37),
])
def test_host_operator_matches_oracle_solves(spline, legacy, nb, smooth, nz, dz):
    import ctypes

    from nfgs_b200 import _lib as L
    from oracle.k0_oracle import CoupledK0, SplineK0

    lib = L.lib()
    G = np.zeros((nz, nz))
    m = np.zeros(nz)
    cond = ctypes.c_double(0.0)
    L.check(lib.nfgs_k0_operator(nz, dz, spline, legacy, nb, smooth, L.dptr(G), L.dptr(m), ctypes.byref(cond)))
    cl = SplineK0(nz, dz, nb, smooth) if spline else CoupledK0(nz, dz, smooth, bool(legacy))
    rng = np.random.default_rng(nz + 7 * nb)
    scale = 0.0
    worst = 0.0
    for _ in range(4):
        q = rng.standard_normal(nz)
        h0 = float(rng.standard_normal())
        want = cl.solve(q, h0)
        got = G @ q + m * h0
        scale = max(scale, np.abs(want).max())
        worst = max(worst, np.abs(got - want).max())
    assert worst <= 1e-10 * scale
    if spline:
        assert cond.value == pytest.approx(float(np.linalg.cond(cl.kkt)), rel=1e-6)
        # the constraints hold for any target: H(0) = h0 and FD2 H'(top) = 0
        q = rng.standard_normal(nz)
        p = G @ q + m * 0.3
        assert p[0] == pytest.approx(0.3, abs=1e-9)
        assert (3 * p[-1] - 4 * p[-2] + p[-3]) / (2 * dz) == pytest.approx(0.0, abs=1e-8 * np.abs(p).max() / dz)
    else:
        assert np.isnan(cond.value)

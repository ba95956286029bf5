"""The oracle's cfcf start against fixtures from the reference itself
(tests/golden/cfcf/, written by tests/golden/make_cfcf_golden.py).

The cfcf start (nfgs_solver.py:6080-6147) projects the Stable-NFPT
curl-free-current state into the NFGS scalars.  Cases: padded grids (the
stable solver's bottom current equals the NFGS one), an unpadded grid (the
stable solver derives its current on the legacy helper grid, so A_z
differs from the gs_cfcf start's), a buffer window, Low-Lou 32^3 with the
BC1 walls and with the potential-pin walls (histories only).
"""

import json
from pathlib import Path

import numpy as np
import pytest

GOLD = Path(__file__).resolve().parent / "golden" / "cfcf"
CASES = sorted(p.stem for p in GOLD.glob("*.json"))


def load(name):
    return json.loads((GOLD / f"{name}.json").read_text()), dict(np.load(GOLD / f"{name}.npz"))


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300))


def oracle(meta, data):
    from oracle.nfgs_oracle import OracleNFGS

    nx, ny, nz = meta["shape"]
    ctor = {k: v for k, v in meta["ctor"].items() if k != "vertical_current_operator"}
    o = OracleNFGS(nx, ny, nz, *meta["spacing"], **ctor)
    o.set_bottom_vector_boundary(data["bx_in"], data["by_in"], data["bz_in"], zero_net_current=False, ijzbcor=3,
                                 **meta["bnd"])
    return o


@pytest.mark.parametrize("name", CASES)
def test_oracle_cfcf_start_matches_reference(name):
    meta, data = load(name)
    o = oracle(meta, data)
    B, J, phi, az, _ = o.compute_initial_conditions(init_mode="cfcf")
    assert [o.Nx, o.Ny, o.Nz] == meta["calc_grid"]
    np.testing.assert_allclose(o.cfcf_diagnostics["stable_cfcf_mean_bcz_by_height"], data["mean_bcz_by_height"],
                               rtol=1e-9, atol=1e-13)
    if "init_phi" in data:
        assert rel(phi, data["init_phi"]) < 1e-11
        assert rel(az, data["init_az"]) < 1e-11
    if "init_B" in data:
        assert rel(B, data["init_B"]) < 1e-11
        assert rel(J, data["init_J"]) < 1e-11
    np.testing.assert_allclose([o.compute_sigma(B, J), o.compute_divB(B), o.compute_energy(B)], data["init_scalars"],
                               rtol=1e-9)


@pytest.mark.parametrize("name", CASES)
def test_oracle_iterate_from_cfcf_matches_reference(name):
    meta, data = load(name)
    o = oracle(meta, data)
    h = o.iterate(init_mode="cfcf", max_iter=meta["iters"], tol=1e-5, mu=1.0, patience=meta["patience"],
                  sigma_improvement_tol=1e-5)
    assert h["stop_reason"] == meta["stop_reason"]
    assert h["best_iter"] == meta["best_iter"]
    np.testing.assert_allclose(h["sigma"], data["hist_sigma"], rtol=1e-8)
    np.testing.assert_allclose(h["energy"], data["hist_energy"], rtol=1e-9)

"""The oracle's per-iteration diagnostics and fixed-point stop against
fixtures from the reference itself (tests/golden/diag/, written by
tests/golden/make_diag_golden.py with record_iteration_diagnostics=True).

Map residuals, PDE residuals (whose exact values are round-off where the
solves are exact), bottom imprints and the alpha-clip / weak-field fractions
of every step (nfgs_solver.py:6806-6933); the fixed_point_criteria_met
column, the fixed_point stop and its selected state (the final accepted
iterate, nfgs_solver.py:3707-3776, 3815-3818).
"""

import json
from pathlib import Path

import numpy as np
import pytest

GOLD = Path(__file__).resolve().parent / "golden" / "diag"
CASES = sorted(p.stem for p in GOLD.glob("*.json"))
# keys whose reference values are round-off of exact identities (the
# scalar PDE rows the modal solves satisfy exactly, h_k0 terms, the exact
# bottom J_z) are compared with an absolute bound instead
ROUNDOFF = ("poloidal_pde_residual_relative", "toroidal_pde_residual_relative", "h_k0_map_residual_relative",
            "h_k0_update_relative", "bottom_jz_imprint_relative")


def load(name):
    return json.loads((GOLD / f"{name}.json").read_text()), dict(np.load(GOLD / f"{name}.npz"))


@pytest.mark.parametrize("name", CASES)
def test_oracle_diagnostics_match_reference(name):
    from oracle.nfgs_oracle import OracleNFGS

    meta, data = load(name)
    nx, ny, nz = meta["shape"]
    ctor = {k: v for k, v in meta["ctor"].items() if k != "vertical_current_operator"}
    o = OracleNFGS(nx, ny, nz, *meta["spacing"], **ctor)
    o.set_bottom_vector_boundary(data["bx_in"], data["by_in"], data["bz_in"], zero_net_current=False, ijzbcor=3,
                                 **meta["bnd"])
    h = o.iterate(init_mode="gs_cfcf", **meta["iterate"])
    assert h["stop_reason"] == meta["stop_reason"]
    assert h["best_iter"] == meta["best_iter"]
    assert h["final_iter"] == meta["final_iter"]
    assert h["selected_state"] == meta["selected_state"]
    np.testing.assert_allclose(h["sigma"], data["hist_sigma"], rtol=1e-8)
    np.testing.assert_array_equal(h["fixed_point_criteria_met"], data["fixed_point_criteria_met"])
    for key in [k[5:] for k in data if k.startswith("diag_")]:
        want = data["diag_" + key]
        if key in ROUNDOFF:
            assert np.max(np.abs(np.asarray(h[key]) - want)) < 1e-9, key
        else:
            np.testing.assert_allclose(h[key], want, rtol=1e-7, atol=1e-14, err_msg=key)
    if "final_Bx" in data:
        f = o.fields_to_numpy()
        for k in ("Bx", "By", "Bz", "Jx", "Jy", "Jz"):
            assert np.linalg.norm(f[k] - data["final_" + k]) <= 1e-9 * np.linalg.norm(data["final_" + k]), k

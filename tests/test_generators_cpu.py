"""The analytic input generators against the reference's own outputs.

* ``nfgs_b200.synthetic.td99_field`` (the benchmark's TD flux rope) against
  the reference generator ``generate_td_model`` (nfgs/_backend/td.py:370-581)
  evaluated with the same parameters on a small lattice that reaches inside
  the flux tube (tests/golden/td99_points.npz).  The two use different
  complete elliptic integral routines (SciPy's vs the reference's Carlson
  forms), so they agree to rounding, not bitwise.
* ``oracle.lowlou_oracle.lowlou_field`` (the analytic interior of config 1)
  against samples of the reference's ``get_analytic_b_field``
  (nfgs/_backend/util/lnl_io.py:97-153) at 64^3, bitwise: the oracle rebuilds
  the reference's own profile interpolant from the recorded coefficients.
"""

import json
import math
from pathlib import Path

import numpy as np

GOLD = Path(__file__).resolve().parent / "golden"


def test_td99_matches_reference_generator():
    from nfgs_b200.synthetic import td99_field, td_params

    d = np.load(GOLD / "td99_points.npz")
    g = d["grid"]
    xs = np.linspace(g[0], g[1], int(g[2]))
    ys = np.linspace(g[3], g[4], int(g[5]))
    zs = np.linspace(g[6], g[7], int(g[8]))
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    for seed in (1, 5):
        p = td_params(seed)
        np.testing.assert_allclose(d[f"seed{seed}_params"], [p[k] for k in ("R", "a", "d", "L", "q", "I0", "l_i")],
                                   rtol=1e-15)
        want = d[f"seed{seed}_B"]
        got = np.stack(td99_field(X, Y, Z, **{k: p[k] for k in ("R", "a", "d", "L", "q", "I0", "l_i")}))
        inside = np.sqrt(X ** 2 + (np.sqrt(Y ** 2 + (Z + p["d"]) ** 2) - p["R"]) ** 2) < p["a"]
        assert inside.sum() > 20  # the lattice samples the tube interior
        assert np.max(np.abs(got - want)) <= 1e-9 * np.max(np.abs(want))


def test_td_bottom_is_the_td99_plane():
    from nfgs_b200.synthetic import td99_field, td_bottom, td_params

    bx, by, bz = td_bottom(40, 36, seed=1, extent=8.0)
    p = td_params(1)
    y, x = np.meshgrid(np.linspace(-8, 8, 36), np.linspace(-8, 8, 40), indexing="ij")
    want = td99_field(x, y, np.zeros_like(x), **{k: p[k] for k in ("R", "a", "d", "L", "q", "I0", "l_i")})
    for a, b in zip((bx, by, bz), want):
        np.testing.assert_array_equal(a, b)
    assert bx.shape == (36, 40)


def test_lowlou_oracle_matches_reference_samples():
    from oracle.lowlou_oracle import lowlou_field

    meta = json.loads((GOLD / "fp32" / "lowlou64_rho05.json").read_text())
    d = np.load(GOLD / "fp32" / "lowlou64_rho05.npz")
    an = meta["analytic"]
    f = lowlou_field(d["lowlou_breaks"], d["lowlou_coeffs"], float(d["lowlou_a2"][0]), n=an["n"], l=an["l"],
                     psi=an["psi"], resolution=tuple(an["resolution"]), bounds=tuple(an["bounds"]))
    i = d["analytic_sample_idx"]
    np.testing.assert_array_equal(f[i[0], i[1], i[2], :], d["analytic_sample"])
    assert an["psi"] == math.pi / 4
    # the bottom plane handed to the solver is the field's z = 0 plane (zyx layout)
    np.testing.assert_array_equal(np.transpose(f[..., 0, 2]), d["bz_in"])

"""The metrics oracle against the reference's own metric functions
(golden vectors from tests/golden/make_metrics_golden.py)."""

from pathlib import Path

import numpy as np
import pytest

from oracle import metrics_oracle as O

G = np.load(Path(__file__).resolve().parent / "golden" / "metrics_golden.npz")
CASES = ("rope", "poly", "aniso", "thin")


def case(name):
    roi = tuple(int(v) for v in G[name + "/roi"])
    return G[name + "/ref"], G[name + "/sol"], G[name + "/cur"], tuple(G[name + "/spacing"]), roi


@pytest.mark.parametrize("name", CASES)
def test_fd2_curl_and_divergence_match_reference(name):
    _, sol, _, sp, _ = case(name)
    np.testing.assert_allclose(np.stack(O.curl(sol, sp)), G[name + "/curl"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(O.divergence(sol, sp), G[name + "/div"], rtol=0, atol=1e-12)


@pytest.mark.parametrize("name", CASES)
def test_oracle_metrics_match_reference(name):
    ref, sol, cur, sp, roi = case(name)
    m = O.field_metrics(ref, sol, cur, sp, roi)
    for k in ("C_vec", "C_CS", "Eprime_n", "Eprime_m", "epsilon", "sigma_J"):
        assert m[k] == pytest.approx(float(G[name + "/rm_" + k]), rel=1e-12, abs=1e-14), k
        assert m[k] == pytest.approx(float(G[name + "/cm_" + k]), rel=1e-12, abs=1e-14), k
    assert m["divB_normalized"] == pytest.approx(float(G[name + "/cm_divB_normalized"]), rel=1e-11, abs=1e-15)
    assert m["sigma_J_common_fd2"] == pytest.approx(float(G[name + "/sigma_J_common_fd2"]), rel=1e-12)
    nz, ny, nx = sol.shape[1:]
    fw = O.field_metrics(None, sol, cur, sp, O.fortran_box(nz, ny, nx))["sigma_J"]
    assert fw == pytest.approx(float(G[name + "/fortran_cwsin"]), rel=1e-12)


def test_polynomial_curl_is_exact():
    """The reference's FD2 test: curl(-y, x, 1 + xy) = (x, -y, 2), div = 0."""
    _, sol, cur, sp, _ = case("poly")
    j = np.stack(O.curl(sol, sp))
    np.testing.assert_allclose(j, cur, atol=2e-14)
    np.testing.assert_allclose(O.divergence(sol, sp), 0, atol=2e-14)

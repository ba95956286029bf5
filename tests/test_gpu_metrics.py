"""GPU evaluation metrics (nfgs_field_metrics) against the reference's
metric functions (golden vectors) and the FP64 oracle."""

from pathlib import Path

import numpy as np
import pytest

from oracle import metrics_oracle as O

pytestmark = pytest.mark.gpu

G = np.load(Path(__file__).resolve().parent / "golden" / "metrics_golden.npz")
CASES = ("rope", "poly", "aniso", "thin")
KEYS = ("C_vec", "C_CS", "Eprime_n", "Eprime_m", "epsilon", "sigma_J")


def case(name):
    roi = tuple(int(v) for v in G[name + "/roi"])
    sl = (slice(roi[0], roi[1]), slice(roi[2], roi[3]), slice(roi[4], roi[5]))
    return G[name + "/ref"], G[name + "/sol"], G[name + "/cur"], tuple(G[name + "/spacing"]), sl


def golden(name, k):
    if k == "divB_normalized":
        return float(G[name + "/cm_divB_normalized"])
    if k == "sigma_J_common_fd2":
        return float(G[name + "/sigma_J_common_fd2"])
    return float(G[name + "/rm_" + k])


@pytest.mark.parametrize("name", CASES)
def test_metrics_match_reference_fp64(name):
    from nfgs_b200 import metrics as M

    ref, sol, cur, sp, sl = case(name)
    m = M.field_metrics(ref, sol, cur, sp, sl)
    for k in KEYS:
        assert m[k] == pytest.approx(golden(name, k), rel=1e-11, abs=1e-13), k
    assert m["divB_normalized"] == pytest.approx(golden(name, "divB_normalized"), rel=1e-10, abs=1e-14)
    assert m["sigma_J_common_fd2"] == pytest.approx(golden(name, "sigma_J_common_fd2"), rel=1e-11)
    assert m["cells"] == np.prod([s.stop - s.start for s in sl])
    assert m["nonfinite_B"] == 0 and m["nonfinite_J"] == 0
    assert M.fortran_cwsin(sol, cur) == pytest.approx(float(G[name + "/fortran_cwsin"]), rel=1e-11)
    keys = ("Bx", "By", "Bz")
    rm = M.compute_reference_metrics(dict(zip(keys, ref)),
                                     dict(zip(keys + ("Jx", "Jy", "Jz"), np.concatenate([sol, cur]))), sl)
    for k in KEYS:
        assert rm[k] == pytest.approx(golden(name, k), rel=1e-11, abs=1e-13), k
    assert rm["En"] == pytest.approx(float(G[name + "/rm_En"]), rel=1e-11, abs=1e-13)
    assert M.common_fd2_sigma_j(dict(zip(keys, sol)), sp, sl) == pytest.approx(
        golden(name, "sigma_J_common_fd2"), rel=1e-11)


@pytest.mark.parametrize("name", CASES)
def test_metrics_fp32_storage_within_fp32_rounding(name):
    import torch
    from nfgs_b200 import metrics as M

    ref, sol, cur, sp, sl = case(name)
    r32, s32, c32 = (torch.from_numpy(a.astype(np.float32)).cuda() for a in (ref, sol, cur))
    m = M.field_metrics(r32, s32, c32, sp, sl)
    # the oracle on the same FP32-rounded values, in FP64
    roi = tuple(v for s in sl for v in (s.start, s.stop))
    o = O.field_metrics(*(a.astype(np.float32).astype(np.float64) for a in (ref, sol, cur)), sp, roi)
    for k in KEYS + ("sigma_J_common_fd2", "divB_normalized"):
        assert m[k] == pytest.approx(o[k], rel=1e-10, abs=1e-12), k
        # and the reference's FP64 values within FP32 input rounding
        assert m[k] == pytest.approx(golden(name, k), rel=2e-5, abs=1e-6), k


def test_metrics_repeatable_and_large_region():
    """A region of 2.0 M cells over many blocks: bitwise repeatable, and equal
    to the oracle to FP64 summation-order rounding."""
    import torch
    from nfgs_b200 import metrics as M

    rng = np.random.default_rng(5)
    shape = (3, 40, 230, 250)
    ref = rng.standard_normal(shape)
    sol = ref + 0.2 * rng.standard_normal(shape)
    cur = rng.standard_normal(shape)
    sl = (slice(1, 39), slice(3, 227), slice(0, 250))
    t = [torch.from_numpy(a).cuda() for a in (ref, sol, cur)]
    a = M.field_metrics(*t, (0.5, 0.6, 0.7), sl)
    b = M.field_metrics(*t, (0.5, 0.6, 0.7), sl)
    assert a == b
    o = O.field_metrics(ref, sol, cur, (0.5, 0.6, 0.7), (1, 39, 3, 227, 0, 250))
    for k in KEYS + ("sigma_J_common_fd2", "divB_normalized", "sum_b2", "sum_ref2"):
        assert a[k] == pytest.approx(o[k], rel=1e-12), k


def test_nonfinite_and_bad_regions_raise():
    from nfgs_b200 import metrics as M

    ref, sol, cur, sp, sl = case("aniso")
    bad = sol.copy()
    bad[1, 2, 2, 3] = np.nan
    keys = ("Bx", "By", "Bz")
    with pytest.raises(RuntimeError, match="Non-finite values in B"):
        M.compute_reference_metrics(dict(zip(keys, ref)), dict(zip(keys + ("Jx", "Jy", "Jz"),
                                                                   np.concatenate([bad, cur]))), sl)
    badj = cur.copy()
    badj[0, 1, 2, 3] = np.inf
    with pytest.raises(RuntimeError, match="Non-finite values in J"):
        M.compute_reference_metrics(dict(zip(keys, ref)), dict(zip(keys + ("Jx", "Jy", "Jz"),
                                                                   np.concatenate([sol, badj]))), sl)
    with pytest.raises(ValueError):
        M.field_metrics(ref, sol, cur, sp, (slice(0, 6), slice(3, 3), slice(0, 7)))
    with pytest.raises(ValueError):
        M.field_metrics(ref, sol, cur, (1.0, 0.0, 1.0), sl)


def test_solution_metrics_on_device_fields_match_host_export():
    """solution_metrics reads the solver's fields on the device; the same
    metrics from fields_to_numpy through the oracle agree."""
    from nfgs_b200 import NFGSSolverGPU
    from nfgs_b200 import metrics as M
    from nfgs_b200.synthetic import td_bottom

    n, nz, ext = 64, 32, 8.0
    h = 2 * ext / (n - 1)
    bx, by, bz = td_bottom(n, n, seed=3, extent=ext, R=3.0, a=1.0, d=1.5)
    s = NFGSSolverGPU(n, n, nz, h, h, h, dtype="float32", bottom_divergence_robin_weight=0.5,
                      horizontal_zero_mode_policy="frozen_linear_harmonic", vertical_current_operator="staggered_face",
                      d0_zero_mode_policy="project", source_zero_mode_policy="project")
    s.set_bottom_vector_boundary(bx, by, bz, zero_net_current=False, smooth_passes=0, ijzbcor=3)
    hist = s.iterate(max_iter=40, tol=1e-5, patience=40, verbose=False)
    f = s.fields_to_numpy()
    dev = s.fields_to_torch().cpu().numpy()
    for q, k in enumerate(("Bx", "By", "Bz", "Jx", "Jy", "Jz")):
        np.testing.assert_array_equal(dev[q], f[k])
    ref = {k: 1.01 * f[k].astype(np.float64) for k in ("Bx", "By", "Bz")}
    m = M.solution_metrics(s, reference=ref)
    B = np.stack([f[k] for k in ("Bx", "By", "Bz")]).astype(np.float64)
    J = np.stack([f[k] for k in ("Jx", "Jy", "Jz")]).astype(np.float64)
    nzc, nyc, nxc = B.shape[1:]
    o = O.field_metrics(np.stack([ref[k] for k in ("Bx", "By", "Bz")]).astype(np.float32).astype(np.float64), B, J,
                        (h, h, h), (0, nzc, 0, nyc, 0, nxc))
    for k in KEYS + ("sigma_J_common_fd2", "divB_normalized"):
        assert m[k] == pytest.approx(o[k], rel=1e-9, abs=1e-12), k
    assert m["C_vec"] == pytest.approx(1.0, abs=1e-6)
    assert m["epsilon"] == pytest.approx(1 / 1.01 ** 2, rel=1e-5)
    fb = O.fortran_box(nzc, nyc, nxc)
    assert m["sigma_J_fortran_box"] == pytest.approx(O.field_metrics(None, B, J, (h, h, h), fb)["sigma_J"], rel=1e-9)
    assert np.isfinite(hist["best_sigma"])

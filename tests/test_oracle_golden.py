"""Pin the CPU oracle against golden tensors produced by the reference solver.

The fixtures in ``tests/golden`` were written by ``tests/golden/make_golden.py``
running the reference ``NFGSSolverGPU`` in FP64 on CPU.  Every comparison
here is FP64 oracle vs FP64 reference, so the tolerances are round-off level.
"""

import json
from pathlib import Path

import numpy as np
import pytest

from oracle.nfgs_oracle import OracleNFGS

GOLD = Path(__file__).resolve().parent / "golden"
CASES = sorted(p.stem for p in GOLD.glob("*.json"))


def load(name):
    meta = json.loads((GOLD / f"{name}.json").read_text())
    data = dict(np.load(GOLD / f"{name}.npz"))
    return meta, data


def make_oracle(meta, data):
    ctor = {k: v for k, v in meta["ctor"].items() if k != "vertical_current_operator"}
    nx, ny, nz = meta["shape"]
    dx, dy, dz = meta["spacing"]
    o = OracleNFGS(nx, ny, nz, dx, dy, dz, **ctor)
    o.set_bottom_vector_boundary(data["bx_in"], data["by_in"], data["bz_in"], zero_net_current=False,
                                 ijzbcor=3, **meta["bnd"])
    return o


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("name", CASES)
def test_setup_products(name):
    meta, data = load(name)
    o = make_oracle(meta, data)
    assert [o.Nx, o.Ny, o.Nz] == meta["calc_grid"]
    assert o.bottom_current_grid_mode == meta["bottom_current_grid_mode"]
    for key, val in [("Bz_obs", o.Bz_obs), ("Jz_obs", o.Jz_obs), ("Az_bottom", o.Az_bottom), ("Jz_T", o.Jz_T),
                     ("Phi_above_bottom", o.Phi_above_bottom), ("Bz_above", o.Bz_above), ("D0", o.D0),
                     ("bottom_dphi_c_target", o.bottom_dphi_c_target),
                     ("gaussian_above", o.gaussian_above_bottom_field())]:
        assert rel(val, data[key]) < 1e-11, key
    if "B_background" in data:
        assert rel(o.B_background, data["B_background"]) < 1e-11
    if o.H is not None:
        np.testing.assert_allclose(o.H[:, 0], data["H_bottom"], rtol=1e-10, atol=1e-13)
    gd = meta["gaussian_separation_diagnostics"]
    for k, v in gd.items():
        ov = o.gaussian_separation_diagnostics[k]
        # residual-type diagnostics sit at round-off (1e-13); compare them absolutely
        assert abs(ov - v) <= 1e-9 * abs(v) + 1e-11, k


@pytest.mark.parametrize("name", CASES)
def test_init_and_steps(name):
    meta, data = load(name)
    o = make_oracle(meta, data)
    st = o.compute_initial_conditions()
    assert rel(st[2], data["init_phi"]) < 1e-10
    assert rel(st[3], data["init_az"]) < 1e-10
    if "init_B" in data:
        assert rel(st[0], data["init_B"]) < 1e-10
        assert rel(st[1], data["init_J"]) < 1e-9
    sc = [o.compute_sigma(st[0], st[1]), o.compute_divB(st[0]), o.compute_energy(st[0])]
    np.testing.assert_allclose(sc, data["init_scalars"], rtol=1e-9)
    st1 = o.iteration_step(*st, mu=1.0)
    st2 = o.iteration_step(*st1, mu=meta["mu2"])
    for tag, s in (("step1", st1), ("step2", st2)):
        if f"{tag}_phi" not in data:
            continue
        assert rel(s[2], data[f"{tag}_phi"]) < 1e-9, tag
        assert rel(s[3], data[f"{tag}_az"]) < 1e-9, tag
        if f"{tag}_B" in data:
            assert rel(s[0], data[f"{tag}_B"]) < 1e-9
            assert rel(s[1], data[f"{tag}_J"]) < 1e-8
    sc = [o.compute_sigma(st1[0], st1[1]), o.compute_divB(st1[0]), o.compute_energy(st1[0]),
          o.compute_sigma(st2[0], st2[1]), o.compute_divB(st2[0]), o.compute_energy(st2[0])]
    np.testing.assert_allclose(sc, data["step_scalars"], rtol=1e-8)


@pytest.mark.parametrize("name", CASES)
def test_iterate_history_and_fields(name):
    meta, data = load(name)
    o = make_oracle(meta, data)
    h = o.iterate(max_iter=meta["iters"], tol=1e-5, mu=1.0, patience=meta["patience"],
                  sigma_improvement_tol=1e-5, stop_mode="sigma_best")
    assert h["stop_reason"] == meta["stop_reason"]
    assert h["best_iter"] == meta["best_iter"]
    assert h["final_iter"] == meta["final_iter"]
    assert abs(h["best_sigma"] - meta["best_sigma"]) < 1e-8 * meta["best_sigma"]
    assert abs(h["final_sigma"] - meta["final_sigma"]) < 1e-8 * max(meta["final_sigma"], 1e-30)
    np.testing.assert_allclose(h["sigma"], data["hist_sigma"], rtol=1e-7)
    np.testing.assert_allclose(h["energy"], data["hist_energy"], rtol=1e-8)
    np.testing.assert_allclose(h["divB"], data["hist_divB"], rtol=1e-6)
    f = o.fields_to_numpy()
    for k in ("Bx", "By", "Bz", "Jx", "Jy", "Jz"):
        if "final_" + k in data:
            assert rel(f[k], data["final_" + k]) < 1e-7, k
        else:
            assert rel(f[k][::2, ::2, ::2], data["final_" + k + "_s2"]) < 1e-6, k
            assert abs(np.sqrt(np.sum(f[k] ** 2)) - data["final_" + k + "_norm"][0]) < 1e-7 * data["final_" + k + "_norm"][0]
    sd = meta["source_diagnostics"]
    for k, v in h["source_diagnostics"].items():
        if k in sd:
            assert abs(v - sd[k]) <= 1e-6 * abs(sd[k]) + 1e-10, k


@pytest.mark.parametrize("name", ["lowlou64_rho05", "td99_96_rho05"])
def test_oracle_reproduces_reference_runs_of_record(name):
    """The oracle against the reference's FP64 runs of config 1 (Low-Lou 64^3)
    and the reduced config 2 (TD generator, 96x96x48): stop reason, best
    iteration, sigma history, final fields (every 4th cell, stored as FP32),
    div-B fraction, and config 1's metrics against the analytic interior."""
    import json

    from oracle.metrics_oracle import divergence, field_metrics
    from oracle.nfgs_oracle import OracleNFGS

    gold = Path(__file__).resolve().parent / "golden" / "fp32"
    meta = json.loads((gold / f"{name}.json").read_text())
    data = dict(np.load(gold / f"{name}.npz"))
    nx, ny, nz = meta["shape"]
    sp = tuple(meta["spacing"])
    o = OracleNFGS(nx, ny, nz, *sp, **{k: v for k, v in meta["ctor"].items() if k != "vertical_current_operator"})
    o.set_bottom_vector_boundary(data["bx_in"], data["by_in"], data["bz_in"], zero_net_current=False,
                                 smooth_passes=0, ijzbcor=3)
    st = meta["stop"]
    h = o.iterate(max_iter=meta["max_iter"], tol=st["tol"], mu=1.0, patience=st["patience"],
                  sigma_improvement_tol=st["sigma_improvement_tol"])
    assert h["stop_reason"] == meta["fp64"]["stop_reason"]
    assert h["best_iter"] == meta["fp64"]["best_iter"]
    np.testing.assert_allclose(h["sigma"], data["hist_sigma_fp64"], rtol=1e-9)
    f = o.fields_to_numpy()
    for k in ("Bx", "By", "Bz", "Jx", "Jy", "Jz"):
        w = data["final64_" + k + "_s4"].astype(np.float64)
        assert np.linalg.norm(f[k][::4, ::4, ::4] - w) / np.linalg.norm(w) < 1e-7, k
    b = np.stack([f[k] for k in ("Bx", "By", "Bz")])
    bm = np.sqrt(np.sum(b * b, axis=0))
    divb = float(np.abs(divergence(b, sp)).mean() / (6.0 * bm.mean() / min(sp) + 1e-12))
    assert divb == pytest.approx(meta["fp64"]["divB_fraction_final"], rel=1e-9)
    if "fp64_vs_analytic" in meta:
        from oracle.lowlou_oracle import lowlou_field, zyx_components

        an = meta["analytic"]
        fa = lowlou_field(data["lowlou_breaks"], data["lowlou_coeffs"], float(data["lowlou_a2"][0]), n=an["n"],
                          l=an["l"], psi=an["psi"], resolution=tuple(an["resolution"]), bounds=tuple(an["bounds"]))
        ref = np.stack(zyx_components(fa))[:, :b.shape[1]]
        j = np.stack([f[k] for k in ("Jx", "Jy", "Jz")])
        m = field_metrics(ref, b, j, sp, (0, b.shape[1], 0, b.shape[2], 0, b.shape[3]))
        for k in ("C_vec", "C_CS", "Eprime_n", "Eprime_m", "epsilon", "sigma_J"):
            assert m[k] == pytest.approx(meta["fp64_vs_analytic"][k], rel=1e-9), k

"""Field-line tracer and Q maps on the GPU (nfgs_trace_field_lines,
nfgs_qmap_plane) against the oracle and closed-form answers.

FP64 runs the oracle's arithmetic on the device (up to fused multiply-adds):
ends agree to 1e-9 cells, flags exactly, Q to 1e-7 relative.  FP32 (the
reference's tracing precision) is held to closed-form answers and to the
oracle at stated per-comparison bars.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def plane_seeds(nx, ny, z0):
    x, y = np.meshgrid(np.arange(nx, dtype=float), np.arange(ny, dtype=float), indexing="xy")
    return np.stack([x.ravel(), y.ravel(), np.full(x.size, z0)], axis=1)


def gpu_trace(b, seeds, dtype, normal=(0, 0, 1), step=0.125, max_steps=2000):
    import torch

    from nfgs_b200.qmap import trace_field_lines

    bt = torch.as_tensor(b, dtype=dtype, device="cuda")
    st = torch.as_tensor(seeds, dtype=dtype, device="cuda")
    tr = trace_field_lines(bt, st, normal=normal, step_len=step, max_steps=max_steps)
    return tr


def host(tr):
    return {k: (v.cpu().numpy().astype(np.float64) if k != "flags" else v.cpu().numpy())
            for k, v in tr.items() if k != "max_steps"}


@pytest.mark.parametrize("dtype_name", ["float64", "float32"])
def test_hyperbolic_known_answer(dtype_name):
    import torch

    from nfgs_b200.qmap import q_on_plane
    from oracle import trace_oracle as T

    dt = getattr(torch, dtype_name)
    nx, ny, nz, L = 41, 41, 21, 20.0
    tr = gpu_trace(T.hyperbolic_field(nx, ny, nz, L), plane_seeds(nx, ny, 10.0), dt)
    q = q_on_plane(tr, nx, ny).cpu().numpy().astype(np.float64)
    tol = 5e-5 if dtype_name == "float64" else 2e-3
    np.testing.assert_allclose(q[12:29, 12:29], 2.0 * np.cosh(2.0), rtol=tol)
    h = host(tr)
    i = 20 * nx + 25
    np.testing.assert_allclose(h["ends"][0, i], [20.0 + 5.0 * np.exp(0.5), 20.0, 20.0], atol=5e-5 if dt == torch.float64 else 2e-4)
    assert h["flags"][0, i] == 6 and h["flags"][1, i] == 5


def test_dipole_fp64_matches_oracle():
    import torch

    from nfgs_b200.qmap import q_on_plane
    from oracle import trace_oracle as T

    nx, ny, nz = 48, 40, 24
    b = T.dipole_field(nx, ny, nz)
    seeds = plane_seeds(nx, ny, 0.5)
    tr = gpu_trace(b, seeds, torch.float64, max_steps=4000)
    q = q_on_plane(tr, nx, ny).cpu().numpy()
    h = host(tr)
    ends, flags, bn, length = T.trace(b, seeds, (0, 0, 1), 0.125, 4000)
    qo = T.qmap(nx, ny, ends, flags, bn)
    np.testing.assert_array_equal(h["flags"], flags)
    assert set(np.unique(flags)) >= {1, 2, 5}  # closed loops back to the bottom and open side exits
    np.testing.assert_allclose(h["ends"], ends, atol=1e-9)
    np.testing.assert_allclose(h["length"], length, rtol=1e-11, atol=1e-9)
    np.testing.assert_allclose(h["bn"], bn, rtol=1e-11, atol=1e-14, equal_nan=True)
    assert np.array_equal(np.isnan(q), np.isnan(qo))
    fin = np.isfinite(qo)
    assert fin.sum() > 0.5 * q.size
    np.testing.assert_allclose(q[fin], qo[fin], rtol=1e-7)


def test_dipole_fp32_against_oracle():
    """FP32: the same face for >= 99% of line ends; ends within 1e-3 cells where
    the faces agree; Q within 1% for >= 95% of the finite values below 1e3."""
    import torch

    from nfgs_b200.qmap import q_on_plane
    from oracle import trace_oracle as T

    nx, ny, nz = 48, 40, 24
    b = T.dipole_field(nx, ny, nz)
    seeds = plane_seeds(nx, ny, 0.5)
    tr = gpu_trace(b, seeds, torch.float32, max_steps=4000)
    q = q_on_plane(tr, nx, ny).cpu().numpy().astype(np.float64)
    h = host(tr)
    ends, flags, bn, _ = T.trace(b, seeds, (0, 0, 1), 0.125, 4000)
    qo = T.qmap(nx, ny, ends, flags, bn)
    same = h["flags"] == flags
    assert same.mean() >= 0.99
    assert np.abs(h["ends"][same] - ends[same]).max() < 1e-3
    both = np.isfinite(q) & np.isfinite(qo) & (qo < 1e3)
    rel = np.abs(q[both] - qo[both]) / qo[both]
    assert (rel < 1e-2).mean() >= 0.95


def test_exit_rules_and_flags():
    import torch

    b = np.zeros((3, 5, 6, 7))
    b[0] = -1.0
    tr = host(gpu_trace(b, np.array([[3.3, 2.0, 1.5], [0.0, 1.0, 1.0], [9.0, 2.0, 1.5]]), torch.float64,
                        normal=(1, 0, 0), max_steps=500))
    assert tr["flags"][0].tolist() == [1, 1, 1] and tr["flags"][1].tolist() == [2, 2, 2]
    np.testing.assert_allclose(tr["ends"][0, 0], [0.0, 2.0, 1.5], atol=1e-12)
    np.testing.assert_allclose(tr["ends"][1, 0], [6.0, 2.0, 1.5], atol=1e-12)
    np.testing.assert_allclose(tr["length"][:, 0], [3.3, 2.7], atol=1e-12)
    assert tr["length"][0, 1] == 0.0
    np.testing.assert_allclose(tr["ends"][1, 2], [6.0, 2.0, 1.5])  # seed clamped into the box
    z = np.zeros((3, 4, 4, 4))
    t2 = host(gpu_trace(z, np.array([[1.0, 1.0, 1.0]]), torch.float32, max_steps=10))
    assert t2["flags"][:, 0].tolist() == [-1, -1] and np.isnan(t2["bn"][1:, 0]).all()
    t3 = host(gpu_trace(b, np.array([[5.0, 2.0, 1.5]]), torch.float64, max_steps=4))
    assert t3["flags"][0, 0] == 0 and t3["length"][0, 0] == 0.5


def test_reference_helpers_contract():
    """compute_y0_qmap / compute_bottom_qmap: shapes, keys, NaN border,
    argument checks, and the Q-only spectral pre-smoothing against NumPy."""
    import torch

    from nfgs_b200 import qmap as Q
    from oracle import trace_oracle as T

    b = T.dipole_field(33, 28, 17).astype(np.float32)
    r = Q.compute_y0_qmap(b[0], b[1], b[2])
    assert r["q"].shape == (17, 33) and r["start_xyz"].shape == (17, 33, 3) and r["line_len"].shape == (17, 33)
    assert np.isnan(r["q"][0]).all() and np.isnan(r["q"][:, -1]).all()
    assert r["metadata"]["plane_y_index"] == 13.5 and r["metadata"]["plane_is_fractional"]
    assert r["metadata"]["q_method"] == "fastqsl"
    ok = (r["flag_start"] > 0) & (r["flag_start"] <= 6)
    # face ends sit on their face up to the FP32 rounding of FastQSL's end estimates
    assert ok.sum() > 0.5 * ok.size and (r["start_xyz"][ok] >= -1e-3).all()
    rb = Q.compute_bottom_qmap(b[0], b[1], b[2])
    assert rb["q"].shape == (28, 33) and np.isfinite(rb["q"]).sum() > 100
    with pytest.raises(ValueError, match="outside"):
        Q.compute_y0_qmap(b[0], b[1], b[2], y_index=40.0)
    # spectral pre-smoothing (fastqsl_plane.py:82-101) restated in NumPy
    sig = 0.75
    freqs = [np.fft.fftfreq(n) for n in b.shape[1:]]
    grids = np.meshgrid(*freqs, indexing="ij")
    k2 = sum(g ** 2 for g in grids)
    ref = np.fft.ifftn(np.fft.fftn(b[0].astype(np.float64)) * np.exp(-0.5 * (2 * np.pi * sig) ** 2 * k2)).real
    got = Q.spectral_gaussian_lowpass(torch.as_tensor(b, device="cuda"), sig)[0].cpu().numpy()
    np.testing.assert_allclose(got, ref.astype(np.float32), rtol=1e-5, atol=1e-6 * np.abs(ref).max())


def gpu_qperp(b, seeds, dtype, delta=0.25, max_steps=2000):
    import torch

    from nfgs_b200.qmap import trace_qperp

    bt = torch.as_tensor(b, dtype=dtype, device="cuda")
    st = torch.as_tensor(seeds, dtype=dtype, device="cuda")
    return host(trace_qperp(bt, st, delta=delta, step_len=0.125, max_steps=max_steps))


@pytest.mark.parametrize("dtype_name", ["float64", "float32"])
def test_qperp_known_answer_on_the_plane_containing_b(dtype_name):
    import torch

    from oracle import trace_oracle as T

    nx, ny, nz, L = 41, 41, 21, 20.0
    z, x = np.meshgrid(np.arange(nz, dtype=float), np.arange(nx, dtype=float), indexing="ij")
    seeds = np.stack([x.ravel(), np.full(x.size, 20.0), z.ravel()], axis=1)
    r = gpu_qperp(T.hyperbolic_field(nx, ny, nz, L), seeds, getattr(torch, dtype_name))
    q = r["q"].reshape(nz, nx)
    np.testing.assert_allclose(q[3:18, 14:27], 2.0 * np.cosh(2.0), rtol=2e-4 if dtype_name == "float64" else 5e-3)


def test_qperp_fp64_matches_oracle():
    import torch

    from oracle import trace_oracle as T

    nx, ny, nz = 48, 40, 24
    b = T.dipole_field(nx, ny, nz)
    seeds = plane_seeds(nx, ny, 0.5)
    r = gpu_qperp(b, seeds, torch.float64, max_steps=4000)
    q, ends, flags, bn, length = T.qperp(b, seeds, 0.25, 0.125, 4000)
    np.testing.assert_array_equal(r["flags"], flags)
    np.testing.assert_allclose(r["ends"], ends, atol=1e-9)
    np.testing.assert_allclose(r["length"], length, rtol=1e-11, atol=1e-9)
    np.testing.assert_allclose(r["bn"], bn, rtol=1e-11, atol=1e-14, equal_nan=True)
    assert np.array_equal(np.isnan(r["q"]), np.isnan(q))
    fin = np.isfinite(q)
    assert fin.sum() > 0.5 * q.size
    np.testing.assert_allclose(r["q"][fin], q[fin], rtol=1e-6)


def test_y0_helper_qperp_method():
    from nfgs_b200 import qmap as Q
    from oracle import trace_oracle as T

    nx, ny, nz, L = 41, 41, 21, 20.0
    b = T.hyperbolic_field(nx, ny, nz, L).astype(np.float32)
    r = Q.compute_y0_qmap(b[0], b[1], b[2], q_method="perp")  # y index 20: the plane containing B
    assert r["metadata"]["q_method"] == "perp"
    np.testing.assert_allclose(r["q"][3:18, 14:27], 2.0 * np.cosh(2.0), rtol=5e-3)
    rp = Q.compute_y0_qmap(b[0], b[1], b[2], q_method="plane")
    assert not np.isfinite(rp["q"]).any()


@pytest.mark.parametrize("dtype_name", ["float64", "float32"])
def test_twist_known_answer_and_oracle(dtype_name):
    """B = (0, sin ax, cos ax): twist = sin(a) L / (4 pi) per half; FP64 also
    equals the oracle on the dipole field."""
    import torch

    from nfgs_b200.qmap import trace_field_lines, trace_qperp
    from oracle import trace_oracle as T

    dt = getattr(torch, dtype_name)
    nx, ny, nz, al = 12, 20, 20, 0.3
    z, y, x = np.meshgrid(np.arange(nz, dtype=float), np.arange(ny, dtype=float), np.arange(nx, dtype=float),
                          indexing="ij")
    b = np.stack([np.zeros_like(x), np.sin(al * x), np.cos(al * x)])
    seeds = np.array([[xx, 10.0, zz] for xx in range(2, 10) for zz in (4.0, 9.5)])
    bt = torch.as_tensor(b, dtype=dt, device="cuda")
    st = torch.as_tensor(seeds, dtype=dt, device="cuda")
    tr = host(trace_field_lines(bt, st, normal=(0, 1, 0), max_steps=2000, twist=True))
    tol = 1e-12 if dtype_name == "float64" else 2e-5
    np.testing.assert_allclose(tr["twist"], np.sin(al) * tr["length"] / (4 * np.pi), rtol=tol, atol=1e-7)
    qp = host(trace_qperp(bt, st, max_steps=2000, twist=True))
    np.testing.assert_allclose(qp["twist"], tr["twist"], rtol=tol, atol=1e-7)
    if dtype_name == "float64":
        bd = T.dipole_field(30, 26, 16)
        sd = plane_seeds(30, 26, 0.5)
        g = host(trace_field_lines(torch.as_tensor(bd, device="cuda"), torch.as_tensor(sd, device="cuda"),
                                   max_steps=4000, twist=True))
        _, f, _, _, two = T.trace(bd, sd, (0, 0, 1), 0.125, 4000, twist=True)
        np.testing.assert_array_equal(g["flags"], f)
        np.testing.assert_allclose(g["twist"], two, rtol=1e-9, atol=1e-12)


def test_y0_helper_twist_bundle():
    from nfgs_b200 import qmap as Q
    from oracle import trace_oracle as T

    b = T.dipole_field(33, 28, 17).astype(np.float32)
    r = Q.compute_y0_qmap(b[0], b[1], b[2], include_twist=True)
    assert r["twist"].shape == (17, 33) and r["twist"].dtype == np.float64
    assert r["metadata"]["twist_included"]
    assert np.isfinite(r["twist"]).all()

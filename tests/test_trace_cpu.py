"""Known answers for the field-line / Q oracle (oracle/trace_oracle.py).

Parity with the reference's FastQSL maps is unpinned (FastQSL needs CuPy and
is not used as a source); the oracle is pinned by fields whose footpoint maps
are known in closed form.  B is linear in these fields, so trilinear
interpolation is exact and only the RK4 step (1/8 cell) limits accuracy.
"""

import numpy as np

from oracle import trace_oracle as T


def plane_seeds(nx, ny, z0):
    x, y = np.meshgrid(np.arange(nx, dtype=float), np.arange(ny, dtype=float), indexing="xy")
    return np.stack([x.ravel(), y.ravel(), np.full(x.size, z0)], axis=1)


def test_uniform_field_q_is_two():
    b = np.zeros((3, 9, 10, 11))
    b[2] = 1.0
    b[0] = 0.3
    ends, flags, bn, length = T.trace(b, plane_seeds(11, 10, 4.0), (0, 0, 1), 0.125, 1000)
    q = T.qmap(11, 10, ends, flags, bn)
    fin = np.isfinite(q)
    assert fin.sum() > 20
    np.testing.assert_allclose(q[fin], 2.0, rtol=1e-12)
    # a line ending on the top face moved by 0.3 per unit height
    i = 3 * 11 + 2
    assert flags[0, i] == 6 and flags[1, i] == 5
    np.testing.assert_allclose(ends[0, i], [2.0 + 0.3 * 4.0, 3.0, 8.0], atol=1e-12)
    np.testing.assert_allclose(length[:, i], [4.0 * np.sqrt(1.09), 4.0 * np.sqrt(1.09)], rtol=1e-12)


def test_hyperbolic_field():
    """B = ((x-xc)/L, -(y-yc)/L, 1): x - xc scales by e^{dz/L}; Q = 2 cosh(2H/L)."""
    nx, ny, nz, L = 41, 41, 21, 20.0
    b = T.hyperbolic_field(nx, ny, nz, L)
    ends, flags, bn, _ = T.trace(b, plane_seeds(nx, ny, 10.0), (0, 0, 1), 0.125, 2000)
    q = T.qmap(nx, ny, ends, flags, bn)
    c = q[12:29, 12:29]
    np.testing.assert_allclose(c, 2.0 * np.cosh(2.0), rtol=5e-5)
    i = 20 * nx + 25
    np.testing.assert_allclose(ends[0, i], [20.0 + 5.0 * np.exp(0.5), 20.0, 20.0], atol=5e-5)
    np.testing.assert_allclose(ends[1, i], [20.0 + 5.0 * np.exp(-0.5), 20.0, 0.0], atol=5e-5)


def test_converging_field_uses_end_normal_components():
    """B = (-(x-xc)/(2L), -(y-yc)/(2L), 1 + z/L) (divergence-free): the map is an
    isotropic scaling, Q = 2, which needs the |Bn+ Bn-| / Bn0^2 factor."""
    nx, ny, nz, L = 31, 31, 17, 8.0
    z, y, x = np.meshgrid(np.arange(nz, dtype=float), np.arange(ny, dtype=float), np.arange(nx, dtype=float),
                          indexing="ij")
    b = np.stack([-(x - 15.0) / (2 * L), -(y - 15.0) / (2 * L), 1.0 + z / L])
    ends, flags, bn, _ = T.trace(b, plane_seeds(nx, ny, 5.0), (0, 0, 1), 0.125, 2000)
    q = T.qmap(nx, ny, ends, flags, bn)
    np.testing.assert_allclose(q[8:23, 8:23], 2.0, rtol=1e-4)
    assert np.all(flags[0].reshape(ny, nx)[8:23, 8:23] == 6)


def test_exits_and_flags():
    """Exit faces, snapping and the zero-field flag."""
    b = np.zeros((3, 5, 6, 7))
    b[0] = -1.0  # lines run along -x
    ends, flags, bn, length = T.trace(b, np.array([[3.3, 2.0, 1.5], [0.0, 1.0, 1.0]]), (1, 0, 0), 0.125, 500)
    assert flags[0].tolist() == [1, 1] and flags[1].tolist() == [2, 2]
    np.testing.assert_allclose(ends[0, 0], [0.0, 2.0, 1.5], atol=1e-12)
    np.testing.assert_allclose(ends[1, 0], [6.0, 2.0, 1.5], atol=1e-12)
    np.testing.assert_allclose(length[:, 0], [3.3, 2.7], atol=1e-12)
    assert length[0, 1] == 0.0  # the seed on the exit face
    np.testing.assert_allclose(bn[:, 0], [-1.0, 1.0, 1.0])
    z = np.zeros((3, 4, 4, 4))
    _, f, bnz, _ = T.trace(z, np.array([[1.0, 1.0, 1.0]]), (0, 0, 1), 0.125, 10)
    assert f[:, 0].tolist() == [-1, -1] and np.isnan(bnz[1:, 0]).all()
    # max steps: a short budget leaves the line unfinished
    _, f2, _, l2 = T.trace(b, np.array([[5.0, 2.0, 1.5]]), (1, 0, 0), 0.125, 4)
    assert f2[0, 0] == 0 and l2[0, 0] == 0.5


def test_qperp_where_the_seed_plane_contains_b():
    """On the y = yc plane of the hyperbolic field By = 0: the seed-grid form
    has no finite value (it divides by Bn0 = 0), Q_perp gives 2 cosh(2H/L)."""
    nx, ny, nz, L = 41, 41, 21, 20.0
    b = T.hyperbolic_field(nx, ny, nz, L)
    z, x = np.meshgrid(np.arange(nz, dtype=float), np.arange(nx, dtype=float), indexing="ij")
    seeds = np.stack([x.ravel(), np.full(x.size, 20.0), z.ravel()], axis=1)
    q, ends, flags, bn, length = T.qperp(b, seeds, 0.25, 0.125, 2000)
    q = q.reshape(nz, nx)
    np.testing.assert_allclose(q[3:18, 14:27], 2.0 * np.cosh(2.0), rtol=2e-4)
    e, f, bnp, _ = T.trace(b, seeds, (0, 1, 0), 0.125, 2000)
    assert not np.isfinite(T.qmap(nx, nz, e, f, bnp)).any()
    # the central line is the plain trace
    np.testing.assert_array_equal(flags, f)
    np.testing.assert_allclose(ends, e, atol=0)
    np.testing.assert_allclose(bn[0], np.sqrt((T.interp(np.moveaxis(b, 0, -1), seeds) ** 2).sum(axis=1)))


def test_qperp_frame_and_uniform_field():
    B = np.array([[0.0, 0.0, 2.0], [1.0, 1.0, 1.0], [0.3, -2.0, 0.1]])
    bm, e1, e2 = T.perp_frame(B)
    b = B / bm[:, None]
    for v in (e1, e2):
        np.testing.assert_allclose((v * b).sum(axis=1), 0.0, atol=1e-15)
        np.testing.assert_allclose((v * v).sum(axis=1), 1.0, rtol=1e-15)
    np.testing.assert_allclose((e1 * e2).sum(axis=1), 0.0, atol=1e-15)
    bu = np.zeros((3, 9, 10, 11))
    bu[2] = 1.0
    bu[0] = 0.3
    bu[1] = -0.2
    x, y = np.meshgrid(np.arange(3.0, 8.0), np.arange(3.0, 7.0), indexing="xy")
    seeds = np.stack([x.ravel(), y.ravel(), np.full(x.size, 4.0)], axis=1)
    q, *_ = T.qperp(bu, seeds, 0.25, 0.125, 1000)
    np.testing.assert_allclose(q, 2.0, rtol=1e-10)


def test_twist_of_a_linear_force_free_field():
    """B = (0, sin ax, cos ax) has J = a B; with grid differences J.B = sin(a)
    at interior x, so each line's twist is sin(a) L / (4 pi)."""
    nx, ny, nz, al = 12, 20, 20, 0.3
    z, y, x = np.meshgrid(np.arange(nz, dtype=float), np.arange(ny, dtype=float), np.arange(nx, dtype=float),
                          indexing="ij")
    b = np.stack([np.zeros_like(x), np.sin(al * x), np.cos(al * x)])
    seeds = np.array([[xx, 10.0, zz] for xx in range(2, 10) for zz in (4.0, 9.5)])
    ends, flags, bn, length, tw = T.trace(b, seeds, (0, 1, 0), 0.125, 2000, twist=True)
    assert (flags > 0).all()
    np.testing.assert_allclose(tw, np.sin(al) * length / (4 * np.pi), rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(T.curl_grid(b)[2][:, :, 1:-1], np.sin(al) * b[2][:, :, 1:-1], rtol=1e-12, atol=1e-15)


def test_qmap_host_helpers():
    """Host-side rules of nfgs_b200.qmap that need no GPU: the physical
    midplane index (fastqsl_plane.py:49-54) and the input checks made before
    any library call."""
    import pytest
    import torch

    from nfgs_b200 import qmap as Q

    assert Q.physical_midplane_grid_index(256) == 127.5
    assert Q.physical_midplane_grid_index(1) == 0.0
    with pytest.raises(ValueError):
        Q.physical_midplane_grid_index(0)
    cpu = torch.zeros((3, 4, 4, 4))
    with pytest.raises(ValueError, match="CUDA tensor"):
        Q.trace_field_lines(cpu, torch.zeros((1, 3)))
    with pytest.raises(ValueError, match="CUDA tensor"):
        Q.trace_qperp(cpu, torch.zeros((1, 3)))

"""The warp-row fused stencil (fs2::k_stencil2, the default) against the
entry-list fused stencil (fs::k_stencil, NFGS_STENCIL_V1=1).

Both compute the same expressions per cell; only the thread layout, the
tiling (30 x 14 tiles, the last one of an axis shifted back onto the wall,
against 32 x 8 tiles with merged remainders) and the order of the partial
sums differ.  From one gs_cfcf start they must give the same states to
rounding and the same sigma_J / divB / energy, on grids with interior
tiles, wall-only tiles, grids narrower than one tile, several z segments,
and every option the fused pass reads: mu relaxation, polarity masks, the
buffer window, the exact-Jz bottom current, the alpha clip and the
horizontal zero mode.
"""

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BASE = dict(bottom_divergence_robin_weight=0.5, horizontal_zero_mode_policy="frozen_linear_harmonic",
            d0_zero_mode_policy="project", source_zero_mode_policy="project",
            vertical_current_operator="staggered_face")


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _solver(nx, ny, nz, dtype, env, kw, seed):
    from nfgs_b200 import NFGSSolverGPU
    from nfgs_b200.synthetic import td_bottom

    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        h = 16.0 / (nx - 1)
        s = NFGSSolverGPU(nx, ny, nz, h, h, h, dtype=dtype, **kw)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    bx, by, bz = td_bottom(nx, ny, seed=seed, extent=8.0)
    s.set_bottom_vector_boundary(bx, by, bz, zero_net_current=False, smooth_passes=0, ijzbcor=3)
    return s


CASES = [
    # (nx, ny, nz, extra ctor kwargs, nseg, polarity, mu)
    (128, 128, 32, {}, "3", "both", 1.0),
    (128, 100, 24, {"horizontal_zero_mode_policy": "omit"}, "1", "both", 0.7),
    (40, 36, 20, {"buffer_thickness": 3}, "2", "both", 1.0),
    (40, 36, 20, {"bottom_parallel_current_mode": "face_parallel_exact_jz", "alpha_clip_scale": 0.5}, "1",
     "both", 1.0),
    (34, 46, 16, {}, "1", "positive", 1.0),
    (34, 46, 16, {}, "2", "negative", 0.8),
    (15, 13, 9, {"pad_calculation_domain": False}, "1", "both", 1.0),
    (62, 31, 12, {"pad_calculation_domain": False}, "2", "both", 1.0),
]


@pytest.mark.parametrize("dtype", ["float64", "float32"])
@pytest.mark.parametrize("case", range(len(CASES)))
def test_warp_row_stencil_matches_entry_list_stencil(case, dtype):
    nx, ny, nz, extra, nseg, pol, mu = CASES[case]
    kw = dict(BASE)
    kw.update(extra)
    a = _solver(nx, ny, nz, dtype, {"NFGS_STENCIL_NSEG": nseg}, kw, seed=11 + case)
    b = _solver(nx, ny, nz, dtype, {"NFGS_STENCIL_NSEG": nseg, "NFGS_STENCIL_V1": "1"}, kw, seed=11 + case)
    for s in (a, b):
        s.iterate(max_iter=0, verbose=False)
    pa, za, sa = a._get_state(1)
    pb, zb, sb = b._get_state(1)
    assert np.array_equal(pa, pb) and np.array_equal(za, zb)
    np.testing.assert_allclose(sa, sb, rtol=1e-12)
    # the first step: same expressions per cell, so rounding-level agreement
    state_tol = 1e-12 if dtype == "float64" else 1e-5
    for step in range(3):
        a._step(mu, pol)
        b._step(mu, pol)
        pa, za, sa = a._get_state(1)
        pb, zb, sb = b._get_state(1)
        assert rel(pa, pb) < state_tol * (10 ** step), (step, rel(pa, pb))
        assert rel(za, zb) < state_tol * (10 ** step), (step, rel(za, zb))
        if step == 0:
            # sigma_J and energy: sums of the same per-cell terms in another
            # order; divB is a cancellation (|div B| << |B| / h), which FP32
            # rounding of B moves by ~1e-4 relative
            np.testing.assert_allclose(sa[[0, 2]], sb[[0, 2]], rtol=1e-10 if dtype == "float64" else 1e-5)
            np.testing.assert_allclose(sa[1], sb[1], rtol=1e-10 if dtype == "float64" else 2e-3)

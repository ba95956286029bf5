"""Device memory of solver handles: pooled, reused across solvers and
returned by release_cached_memory."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _solve(n=64, nz=32, seed=2):
    from nfgs_b200 import NFGSSolverGPU
    from nfgs_b200.synthetic import td_bottom

    h = 16.0 / (n - 1)
    s = NFGSSolverGPU(n, n, nz, h, h, h, dtype="float32", bottom_divergence_robin_weight=0.5,
                      horizontal_zero_mode_policy="frozen_linear_harmonic", vertical_current_operator="staggered_face",
                      d0_zero_mode_policy="project", source_zero_mode_policy="project")
    bx, by, bz = td_bottom(n, n, seed=seed, extent=8.0, R=3.0, a=1.0, d=1.5)
    s.set_bottom_vector_boundary(bx, by, bz, zero_net_current=False, smooth_passes=0, ijzbcor=3)
    hist = s.iterate(max_iter=20, verbose=False)
    f = s.fields_to_numpy()
    return s, hist, f


def test_reused_memory_gives_identical_solves_and_release_returns_it():
    import gc

    import torch
    from nfgs_b200 import release_cached_memory

    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    s, h1, f1 = _solve()
    del s
    gc.collect()
    # a second solver on the reserved memory gives the same result bit for bit
    s, h2, f2 = _solve()
    assert h1["sigma"] == h2["sigma"]
    for k in f1:
        np.testing.assert_array_equal(f1[k], f2[k])
    del s
    gc.collect()
    release_cached_memory(0)
    free1, _ = torch.cuda.mem_get_info()
    # what the library reserved is back (allow for the CUDA context's own growth)
    assert free1 >= free0 - (64 << 20)
    release_cached_memory(0)  # idempotent
    # a solver made after the release (its matrices uploaded again) repeats the first result
    s, h3, f3 = _solve()
    assert h1["sigma"] == h3["sigma"]
    for k in f1:
        np.testing.assert_array_equal(f1[k], f3[k])
    del s

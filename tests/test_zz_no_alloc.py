"""The allocation-free B^> entry point against the allocating one.

nfgs_gaussian_above_noalloc serves callers that cannot allocate device
memory while they run (their own pool allocator holds the free memory, or
a device-wide synchronisation from cudaMalloc/cudaFree would stall other
work).  It must give the same B^> as nfgs_gaussian_above, call after call,
although every call reuses one static scratch array.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _solver(nx, ny, nz, seed, dtype, **kw):
    from nfgs_b200 import NFGSSolverGPU
    from nfgs_b200.synthetic import bipolar_boundary

    s = NFGSSolverGPU(nx, ny, nz, 1.0, 1.0, 1.0, device="cuda:0", dtype=dtype, d0_zero_mode_policy="project",
                      source_zero_mode_policy="project", **kw)
    bx, by, bz = bipolar_boundary(ny, nx, seed)
    s.set_bottom_vector_boundary(bx, by, bz, zero_net_current=False, smooth_passes=0)
    return s


def _call(lib, s, buf, stream):
    return lib.nfgs_gaussian_above_noalloc(s._h, ctypes.c_void_p(buf.data_ptr()), ctypes.c_void_p(stream))


def test_noalloc_matches_allocating_entry_point_on_repeated_calls():
    import torch

    from nfgs_b200 import _lib as L

    lib = L.lib()
    a = _solver(40, 36, 20, 3, "float64")
    b = _solver(30, 30, 12, 5, "float32", gaussian_horizontal_operator="fd")
    ref = {id(a): a.gaussian_above_bottom_field(), id(b): b.gaussian_above_bottom_field()}
    stream = torch.cuda.current_stream().cuda_stream
    # a, then b (leaves other data in the shared scratch), then a again
    for s in (a, b, a):
        buf = torch.full((3 * s.Ny * s.Nx,), float("nan"), dtype=torch.float64, device="cuda:0")
        assert _call(lib, s, buf, stream) == 0, lib.nfgs_last_error()
        torch.cuda.synchronize()
        got = buf.cpu().numpy().reshape(3, s.Ny, s.Nx)
        want = ref[id(s)]
        assert np.isfinite(got).all()
        assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-11


def test_noalloc_on_a_side_stream_and_fp32_spectral_handle():
    """The call on a caller-owned side stream, read only after that stream is
    synchronised, and an FP32 handle with the default (spectral) Gaussian
    operator, against the allocating entry point; the handle is then given a
    new boundary (which waits for the call) and called again."""
    import torch

    from nfgs_b200 import _lib as L
    from nfgs_b200.synthetic import bipolar_boundary

    lib = L.lib()
    s = _solver(34, 38, 14, 7, "float32")
    want = s.gaussian_above_bottom_field()
    side = torch.cuda.Stream()
    for _ in range(2):
        buf = torch.full((3 * s.Ny * s.Nx,), float("nan"), dtype=torch.float64, device="cuda:0")
        torch.cuda.current_stream().synchronize()
        assert _call(lib, s, buf, side.cuda_stream) == 0, lib.nfgs_last_error()
        side.synchronize()
        got = buf.cpu().numpy().reshape(3, s.Ny, s.Nx)
        assert np.isfinite(got).all()
        assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-11
    bx, by, bz = bipolar_boundary(38, 34, 11)
    buf = torch.full((3 * s.Ny * s.Nx,), float("nan"), dtype=torch.float64, device="cuda:0")
    assert _call(lib, s, buf, side.cuda_stream) == 0, lib.nfgs_last_error()
    s.set_bottom_vector_boundary(bx, by, bz, zero_net_current=False, smooth_passes=0)
    side.synchronize()
    want2 = s.gaussian_above_bottom_field()
    buf2 = torch.full((3 * s.Ny * s.Nx,), float("nan"), dtype=torch.float64, device="cuda:0")
    assert _call(lib, s, buf2, side.cuda_stream) == 0, lib.nfgs_last_error()
    side.synchronize()
    got2 = buf2.cpu().numpy().reshape(3, s.Ny, s.Nx)
    assert np.linalg.norm(got2 - want2) / np.linalg.norm(want2) < 1e-11


def test_noalloc_rejects_planes_beyond_the_static_limit():
    import torch

    from nfgs_b200 import NFGSSolverGPU
    from nfgs_b200 import _lib as L

    lib = L.lib()
    big = NFGSSolverGPU(700, 700, 6, 1.0, 1.0, 1.0, device="cuda:0", dtype="float32")
    assert big.Nx * big.Ny > 419430
    buf = torch.empty(3, dtype=torch.float64, device="cuda:0")
    rc = _call(lib, big, buf, torch.cuda.current_stream().cuda_stream)
    assert rc == L.NFGS_EINVAL
    assert b"static scratch limit" in lib.nfgs_last_error()

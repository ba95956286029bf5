"""DCT-I / DST-I transforms of the CUDA path against SciPy (FP64).

FP32 storage on grids with even N and (N-2)/2 <= 256 runs the tcgen05
tensor-core contractions (above 128 pairs the four-role kernel, which solves
use only on request -- NFGS_TC_WIDE=1 -- and which these tests switch on;
FP16 hi/lo split operands, FP32 accumulation in 32-pair chunks);
their error against the FP64 transform must stay at FP32 level: relative
L2 error <= 2e-6 (forward) and <= 2e-6 (inverse) per volume (measured
1.5e-7 to 6e-7).  FP64 storage
runs the SIMT contractions and must agree to 1e-12.
"""

import ctypes

import numpy as np
import pytest
from scipy import fft

pytestmark = pytest.mark.gpu


def _solver(nx, ny, nz, dtype):
    import os

    from nfgs_b200 import NFGSSolverGPU

    # the wide tensor-core kernel is read from the environment when the handle is made
    old = os.environ.get("NFGS_TC_WIDE")
    os.environ["NFGS_TC_WIDE"] = "1"
    try:
        return NFGSSolverGPU(nx, ny, nz, 1.0, 1.0, 1.0, device="cuda:0", dtype=dtype, pad_calculation_domain=False)
    finally:
        if old is None:
            os.environ.pop("NFGS_TC_WIDE")
        else:
            os.environ["NFGS_TC_WIDE"] = old


def _apply(s, chain, inverse, x):
    from nfgs_b200 import _lib as L

    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros_like(x)
    L.check(L.lib().nfgs_apply_transform(s._h, chain, int(inverse), L.dptr(x), L.dptr(out)))
    return out


def _ref(chain, inverse, x):
    t = 1
    f = fft.idct if inverse else fft.dct
    g = fft.idst if inverse else fft.dst
    if chain == 0:
        return f(f(x, type=t, axis=-1), type=t, axis=-2)
    return g(g(x, type=t, axis=-1), type=t, axis=-2)


@pytest.mark.parametrize("shape", [(18, 18, 5), (66, 34, 4), (130, 258, 3), (258, 258, 5), (194, 258, 3), (66, 66, 65),
                                   (258, 258, 129), (514, 514, 3), (514, 258, 4), (258, 386, 3), (514, 514, 65),
                                   (258, 386, 65)])
@pytest.mark.parametrize("dtype,tol", [("float32", 2e-6), ("float64", 1e-12)])
def test_transforms_match_scipy(shape, dtype, tol):
    nx, ny, nz = shape
    s = _solver(nx, ny, nz, dtype)
    rng = np.random.default_rng(nx * 7 + ny)
    # smooth part + noise, as the sources are
    x = rng.standard_normal((nz, ny, nx)) * 0.1
    yy, xx = np.meshgrid(np.linspace(0, 1, ny), np.linspace(0, 1, nx), indexing="ij")
    x += np.exp(-((xx - 0.4) ** 2 + (yy - 0.6) ** 2) / 0.02)[None]
    for chain in (0, 1):
        xin = x if chain == 0 else x[:, 1:-1, 1:-1].copy()
        for inverse in (0, 1):
            got = _apply(s, chain, inverse, xin)
            want = _ref(chain, inverse, xin.astype(np.float32).astype(np.float64) if dtype == "float32" else xin)
            if chain == 0:
                sl = slice(0, nz) if not inverse else slice(1, nz)
            else:
                sl = slice(1, nz - 1)
            err = np.linalg.norm(got[sl] - want[sl]) / np.linalg.norm(want[sl])
            assert err < tol, (chain, inverse, err)

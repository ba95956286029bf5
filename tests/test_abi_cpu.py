"""CPU-side checks of the C ABI and the host logic (no GPU compute)."""

import ctypes
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from nfgs_b200 import _lib as L
from nfgs_b200.grid import calculation_grid, fortran_grid, mudpack_axis_size, pad_or_crop_center
from oracle import nfgs_oracle as O

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "nfgs_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+(nfgs_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib = L.load()
    names = declared_symbols()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(L.SIGNATURES), set(names) ^ set(L.SIGNATURES)
    assert b"sm_100a" in lib.nfgs_version()


def test_struct_layouts_match_c(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "nfgs_b200.h"\nint main(void){'
                   'printf("%zu %zu %zu %zu %zu\\n", sizeof(NfgsGeom), sizeof(NfgsParams), sizeof(NfgsBoundaryOpts),'
                   ' sizeof(NfgsStop), sizeof(NfgsIterResult)); return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    got = [ctypes.sizeof(s) for s in (L.NfgsGeom, L.NfgsParams, L.NfgsBoundaryOpts, L.NfgsStop, L.NfgsIterResult)]
    assert [int(v) for v in out] == got


def test_no_device_fails_loudly():
    lib = L.load()
    g = L.NfgsGeom(10, 10, 8, 1.0, 1.0, 1.0, 10, 10, 8, 0, 0, 0)
    p = L.NfgsParams()
    h = ctypes.c_void_p()
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    assert lib.nfgs_create(ctypes.byref(g), ctypes.byref(p), ctypes.byref(h)) == L.NFGS_ECUDA
    assert b"no CUDA device" in lib.nfgs_last_error()


@pytest.mark.parametrize("n", list(range(2, 300)) + [511, 512, 513, 514, 1024])
def test_grid_sizing_matches_oracle(n):
    assert mudpack_axis_size(n) == O.mudpack_axis_size(n)
    for sym in (False, True):
        g = fortran_grid(n, n + 3, max(n // 2, 3), symmetric_xy=sym)
        o = O.fortran_grid(n, n + 3, max(n // 2, 3), symmetric_xy=sym)
        assert (g["nx"], g["ny"], g["nz"], g["bfx"], g["bfy"]) == o[:5]


def test_calculation_grid_modes():
    assert calculation_grid(256, 256, 128)["nx"] == 258
    g = calculation_grid(256, 256, 128)
    assert (g["nx"], g["ny"], g["nz"], g["pad_xy"]) == (258, 258, 129, (1, 1))
    g = calculation_grid(64, 64, 64)
    assert (g["nx"], g["ny"], g["nz"]) == (66, 66, 65)
    g = calculation_grid(512, 512, 256)
    assert (g["nx"], g["ny"], g["nz"]) == (514, 514, 257)
    g = calculation_grid(11, 9, 7, calculation_domain_mode="bottom_padding")
    assert (g["nx"], g["ny"], g["nz"], g["pad_xy"]) == (17, 15, 15, (3, 3))
    g = calculation_grid(11, 9, 7, pad_calculation_domain=False)
    assert (g["nx"], g["ny"], g["nz"]) == (11, 9, 7)
    with pytest.raises(ValueError):
        calculation_grid(11, 9, 7, calculation_domain_mode="nope")


@pytest.mark.parametrize("shape,target", [((9, 11), (9, 13)), ((10, 12), (13, 13)), ((20, 20), (13, 17)),
                                          ((5, 7), (9, 9))])
def test_pad_or_crop_matches_oracle(shape, target):
    rng = np.random.default_rng(0)
    a = rng.standard_normal(shape)
    ref, fov = O._pad_or_crop_center_2d(a, *target)
    p = pad_or_crop_center(shape[0], shape[1], *target)
    out = np.zeros(target)
    out[p["dy0"]:p["dy0"] + p["cny"], p["dx0"]:p["dx0"] + p["cnx"]] = \
        a[p["sy0"]:p["sy0"] + p["cny"], p["sx0"]:p["sx0"] + p["cnx"]]
    np.testing.assert_array_equal(out, ref)
    assert (fov[0].start, fov[1].start) == (p["dy0"], p["dx0"])


def test_option_validation_before_device():
    from nfgs_b200 import NFGSSolverGPU
    with pytest.raises(ValueError, match="CUDA only"):
        NFGSSolverGPU(16, 16, 8, 1, 1, 1, device="cpu")
    with pytest.raises(ValueError, match="poisson_z_order"):
        NFGSSolverGPU(16, 16, 8, 1, 1, 1, poisson_z_order=4)
    with pytest.raises(ValueError, match="mutually exclusive"):
        NFGSSolverGPU(16, 16, 8, 1, 1, 1, bottom_divergence_robin_weight=0.5,
                      bottom_divergence_projection_weight=0.5)
    with pytest.raises(ValueError, match="between 0 and 1"):
        NFGSSolverGPU(16, 16, 8, 1, 1, 1, bottom_divergence_robin_weight=1.5)
    with pytest.raises(NotImplementedError):
        NFGSSolverGPU(16, 16, 8, 1, 1, 1, horizontal_zero_mode_policy="external_potential")
    # k_h=0 closure options (nfgs_solver.py:4120-4170, 4252-4270)
    with pytest.raises(ValueError, match="relax_scalars=True"):
        NFGSSolverGPU(16, 16, 8, 1, 1, 1, horizontal_zero_mode_policy="coupled_k0", relax_scalars=False)
    with pytest.raises(ValueError, match="must not exceed Nz"):
        NFGSSolverGPU(16, 16, 8, 1, 1, 1, horizontal_zero_mode_policy="constrained_spline_harmonic",
                      k0_spline_basis_size=500)
    with pytest.raises(ValueError, match=">= 4"):
        NFGSSolverGPU(16, 16, 8, 1, 1, 1, horizontal_zero_mode_policy="constrained_spline_harmonic",
                      k0_spline_basis_size=3)
    with pytest.raises(RuntimeError, match="legacy coupled_k0 operator"):
        NFGSSolverGPU(16, 16, 8, 1, 1, 1, horizontal_zero_mode_policy="constrained_spline_harmonic",
                      coupled_k0_discretization="legacy_plane_centred")
    with pytest.raises(ValueError, match=r"k0_update_mu must be in \(0, 1\]"):
        NFGSSolverGPU(16, 16, 8, 1, 1, 1, horizontal_zero_mode_policy="coupled_k0", k0_update_mu=1.5)
    with pytest.raises(ValueError, match="k0_current_target_placement"):
        NFGSSolverGPU(16, 16, 8, 1, 1, 1, horizontal_zero_mode_policy="coupled_k0",
                      k0_current_target_placement="middle")
    with pytest.raises(ValueError, match="k0_ode_smoothness"):
        NFGSSolverGPU(16, 16, 8, 1, 1, 1, horizontal_zero_mode_policy="coupled_k0", k0_ode_smoothness=-1.0)
    with pytest.raises(NotImplementedError):
        NFGSSolverGPU(16, 16, 8, 1, 1, 1, vertical_current_operator="collocated_centered")
    with pytest.raises(ValueError, match="alpha_clip_scale"):
        NFGSSolverGPU(16, 16, 8, 1, 1, 1, alpha_clip_scale=1.0, alpha_limit_factor=2.0)
    with pytest.raises(TypeError):
        NFGSSolverGPU(16, 16, 8, 1, 1, 1, not_an_option=1)
    with pytest.raises(ValueError, match="soft_cfcf_epsilon"):
        NFGSSolverGPU(16, 16, 8, 1, 1, 1, soft_cfcf_epsilon=-1.0)
    with pytest.raises(ValueError, match="soft_cfcf_normal_ridge"):
        NFGSSolverGPU(16, 16, 8, 1, 1, 1, soft_cfcf_normal_ridge=-1e-3)
    with pytest.raises(ValueError, match="soft_cfcf_mode_batch_size"):
        NFGSSolverGPU(16, 16, 8, 1, 1, 1, soft_cfcf_mode_batch_size=0)


def test_oracle_transforms_are_the_dense_matrices():
    """DCT-I / DST-I as dense matrices equal the oracle's SciPy transforms."""
    rng = np.random.default_rng(1)
    for n in (5, 9, 66):
        x = rng.standard_normal(n)
        k = np.arange(n)[:, None]
        m = np.arange(n)[None, :]
        w = np.where((m == 0) | (m == n - 1), 1.0, 2.0)
        C = w * np.cos(np.pi * k * m / (n - 1))
        np.testing.assert_allclose(C @ x, O.dct1(x, 0), rtol=1e-12, atol=1e-12)
        S = 2 * np.sin(np.pi * (k + 1) * (m + 1) / (n + 1))
        np.testing.assert_allclose(S @ x, O.dst1(x, 0), rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(O.idct1(O.dct1(x, 0), 0), x, atol=1e-12)
        np.testing.assert_allclose(O.idst1(O.dst1(x, 0), 0), x, atol=1e-12)


def test_metric_enum_matches_python_names(tmp_path):
    from nfgs_b200.metrics import METRIC_NAMES

    src = tmp_path / "met.c"
    src.write_text('#include <stdio.h>\n#include "nfgs_b200.h"\nint main(void){printf("%d %d %d %d\\n", '
                   'NFGS_MET_SIGMA_J_FD2, NFGS_MET_DIVB_NORM, NFGS_MET_NONFINITE_J, NFGS_MET_COUNT); return 0;}\n')
    exe = tmp_path / "met"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    assert out == [METRIC_NAMES.index("sigma_J_common_fd2"), METRIC_NAMES.index("divB_normalized"),
                   METRIC_NAMES.index("nonfinite_J"), len(METRIC_NAMES)]
    assert L.NFGS_MET_COUNT == len(METRIC_NAMES)


def test_metric_regions_match_reference_helpers():
    from nfgs_b200 import metrics as M
    from oracle import metrics_oracle as MO

    g = np.load(ROOT / "tests" / "golden" / "metrics_golden.npz")
    assert M.flux_rope_center_from_bottom_jz(g["rope/jz0"]) == tuple(int(v) for v in g["rope/center"])
    nz, ny, nx = g["rope/sol"].shape[1:]
    tx, ty, tz = (int(v) for v in g["rope/test_dims"])
    iy, ix = (int(v) for v in g["rope/center"])
    sl = M.test_domain_slices_zyx(nz, ny, nx, iy, ix, tx, ty, tz)
    assert [v for s in sl for v in (s.start, s.stop)] == [int(v) for v in g["rope/roi"]]
    assert M._roi(M.fortran_box(16, 14, 12), (16, 14, 12)).tolist() == list(MO.fortran_box(16, 14, 12))
    with pytest.raises(ValueError):
        M._roi((slice(0, 3), slice(2, 2), slice(0, 4)), (5, 5, 5))
    with pytest.raises(ValueError):
        M._spacing((1.0, -1.0, 1.0))

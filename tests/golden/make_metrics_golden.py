"""Generate metrics_golden.npz by running the REFERENCE's evaluation metrics.

Run where the reference repository is mounted (default ``/root/reference``,
override with ``NFGS_REFERENCE``):

    python tests/golden/make_metrics_golden.py

For a few seeded field sets it records the outputs of
``nfgs.diagnostics.common_fd2`` (curl, divergence, sigma_j),
``nfgs._backend.util.metrics`` (compute_reference_metrics, fortran_cwsin,
test_domain_slices_zyx, flux_rope_center_from_bottom_jz) and
``compute_metrics`` of ``nfgs/_backend/scripts/recompute_td_referee_diagnostics.py``.
That module imports plotting packages at the top, so only the one function is
taken from its source (by ``ast``) and executed.  The tests never import the
reference.
"""

from __future__ import annotations

import ast
import math
import os
import sys
from pathlib import Path

import numpy as np

REF = os.environ.get("NFGS_REFERENCE", "/root/reference")
sys.path.insert(0, REF)

from nfgs.diagnostics import common_fd2  # noqa: E402
from nfgs._backend.util import metrics as M  # noqa: E402

OUT = Path(__file__).resolve().parent / "metrics_golden.npz"


def _compute_metrics():
    path = Path(REF) / "nfgs/_backend/scripts/recompute_td_referee_diagnostics.py"
    tree = ast.parse(path.read_text())
    fn = next(n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name == "compute_metrics")
    mod = ast.Module(body=[fn], type_ignores=[])
    ns = {"np": np, "math": math}
    exec(compile(mod, str(path), "exec"), ns)
    return ns["compute_metrics"]


def smooth_field(rng, nz, ny, nx, modes=4):
    z, y, x = np.meshgrid(np.linspace(0, 1, nz), np.linspace(0, 1, ny), np.linspace(0, 1, nx), indexing="ij")
    out = np.zeros((3, nz, ny, nx))
    for c in range(3):
        for _ in range(modes):
            kz, ky, kx = rng.uniform(0.5, 3.0, 3)
            ph = rng.uniform(0, 2 * np.pi, 3)
            out[c] += rng.normal() * np.cos(np.pi * kz * z + ph[0]) * np.cos(np.pi * ky * y + ph[1]) * np.cos(
                np.pi * kx * x + ph[2])
    return out


def main():
    compute_metrics = _compute_metrics()
    rng = np.random.default_rng(20260)
    cases = {}

    # flux-rope-like: smooth reference, perturbed solution, independent current
    nz, ny, nx = 16, 14, 12
    ref = smooth_field(rng, nz, ny, nx)
    sol = ref + 0.15 * smooth_field(rng, nz, ny, nx, 6) + 0.01 * rng.standard_normal(ref.shape)
    cur = smooth_field(rng, nz, ny, nx, 5)
    jz0 = np.exp(-((np.arange(ny)[:, None] - 8.3) ** 2 + (np.arange(nx)[None, :] - 5.6) ** 2) / 6.0)
    iy, ix = M.flux_rope_center_from_bottom_jz(jz0)
    roi = M.test_domain_slices_zyx(nz, ny, nx, iy, ix, 8, 6, 10)
    cases["rope"] = dict(ref=ref, sol=sol, cur=cur, spacing=(0.5, 0.5, 0.5), roi=roi, jz0=jz0, center=(iy, ix),
                         test_dims=(8, 6, 10))

    # the anisotropic quadratic bundle of the reference's own FD2 test
    x = np.linspace(-1, 1, 9)
    y = np.linspace(-2, 2, 7)
    z = np.linspace(0, 3, 5)
    zz, yy, xx = np.meshgrid(z, y, x, indexing="ij")
    b = np.stack([-yy, xx, 1 + xx * yy])
    cases["poly"] = dict(ref=b * (1 + 0.1 * zz), sol=b, cur=np.stack([xx, -yy, 2 + 0 * xx]),
                         spacing=(0.25, 4 / 6, 0.75), roi=(slice(0, 5), slice(0, 7), slice(0, 9)))

    # random anisotropic, region touching every wall
    sh = (6, 5, 7)
    cases["aniso"] = dict(ref=rng.standard_normal((3,) + sh), sol=rng.standard_normal((3,) + sh),
                          cur=rng.standard_normal((3,) + sh), spacing=(1.0, 0.8, 1.3),
                          roi=(slice(0, 6), slice(1, 5), slice(0, 7)))

    # one- and two-plane axes (the n == 1 and n == 2 derivative branches)
    sh = (2, 1, 6)
    cases["thin"] = dict(ref=rng.standard_normal((3,) + sh), sol=rng.standard_normal((3,) + sh),
                         cur=rng.standard_normal((3,) + sh), spacing=(0.7, 0.9, 1.1),
                         roi=(slice(0, 2), slice(0, 1), slice(1, 6)))

    store = {}
    for name, c in cases.items():
        ref, sol, cur, sp, roi = c["ref"], c["sol"], c["cur"], c["spacing"], c["roi"]
        keys = ("Bx", "By", "Bz")
        f_ref = dict(zip(keys, ref))
        f_sol = dict(zip(keys, sol))
        f_sol.update(zip(("Jx", "Jy", "Jz"), cur))
        rm = M.compute_reference_metrics(f_ref, f_sol, roi)
        j = common_fd2.curl(dict(zip(keys, sol)), sp)
        div = common_fd2.divergence(dict(zip(keys, sol)), sp)
        h_eff = 3 / sum(1 / h for h in sp)
        cm = compute_metrics(f_ref, dict(zip(keys, sol)), dict(zip(("Jx", "Jy", "Jz"), cur)), div, roi, h_eff)
        sj = common_fd2.sigma_j(dict(zip(keys, sol)), sp, roi)
        fw = M.fortran_cwsin(sol, cur)
        p = name + "/"
        store[p + "ref"], store[p + "sol"], store[p + "cur"] = ref, sol, cur
        store[p + "spacing"] = np.array(sp)
        store[p + "roi"] = np.array([v for s in roi for v in (s.start, s.stop)])
        store[p + "curl"] = np.stack([j["Jx"], j["Jy"], j["Jz"]])
        store[p + "div"] = div
        for k, v in rm.items():
            store[p + "rm_" + k] = np.float64(v)
        for k, v in cm.items():
            store[p + "cm_" + k] = np.float64(v)
        store[p + "sigma_J_common_fd2"] = np.float64(sj)
        store[p + "fortran_cwsin"] = np.float64(fw)
        if "jz0" in c:
            store[p + "jz0"] = c["jz0"]
            store[p + "center"] = np.array(c["center"])
            store[p + "test_dims"] = np.array(c["test_dims"])
    np.savez_compressed(OUT, **store)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes, {len(cases)} cases)")


if __name__ == "__main__":
    main()

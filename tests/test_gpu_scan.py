"""Batched scan: solves advanced together by one CUDA graph give exactly the
histories of the same solves run one by one."""

import pytest

pytestmark = pytest.mark.gpu


def test_scan_matches_serial_solves():
    pytest.importorskip("torch")
    from nfgs_b200.scan import run_scan, run_serial, td_scan_cases

    cases = td_scan_cases(3, rhos=(0.0, 0.5), seed=2, grids=((32, 16), (48, 24)))
    hs, timing = run_scan(cases, iters=4, max_iter=400)
    ss, _ = run_serial(cases, max_iter=400)
    assert timing["graph_launches"] >= 1
    for a, b in zip(hs, ss):
        assert a["sigma"] == b["sigma"]
        assert a["best_iter"] == b["best_iter"]
        assert a["stop_reason"] == b["stop_reason"]


def test_overlapped_scan_matches_serial_solves():
    """Solves joined to the running scan as their set-up finishes
    (nfgs_scan_add between launches) follow the same histories."""
    pytest.importorskip("torch")
    from nfgs_b200.scan import run_scan_overlapped, run_serial, td_scan_cases

    cases = td_scan_cases(4, rhos=(0.0, 0.5, 1.0), seed=3, grids=((32, 16), (48, 24)))
    hs, timing = run_scan_overlapped(cases, iters=4, max_iter=400, workers=4)
    ss, _ = run_serial(cases, max_iter=400)
    assert timing["graph_launches"] >= 1 and timing["joins"] >= 1
    for a, b in zip(hs, ss):
        assert a["sigma"] == b["sigma"]
        assert a["best_iter"] == b["best_iter"]
        assert a["stop_reason"] == b["stop_reason"]


def test_scan_add_rejects_a_handle_twice():
    import ctypes as C

    from nfgs_b200.scan import _solver, td_scan_cases
    from nfgs_b200 import _lib as L

    c = td_scan_cases(1, rhos=(0.5,), seed=4, grids=((32, 16),))[0]
    s = _solver(c)
    ctx = s._iterate_begin(max_iter=20, verbose=False, use_graph=True, tol=1e-5, patience=40,
                           sigma_improvement_tol=1e-5)
    arr = (C.c_void_p * 1)(s._h.value)
    scan = C.c_void_p()
    lib = L.lib()
    L.check(lib.nfgs_scan_create(arr, 1, 2, C.byref(scan)))
    try:
        assert lib.nfgs_scan_add(scan, arr, 1) == L.NFGS_EINVAL
    finally:
        L.check(lib.nfgs_scan_destroy(scan))
    s._iterate_finish(ctx)


def test_scan_rejects_unbegun_handle():
    import ctypes as C

    from nfgs_b200 import NFGSSolverGPU
    from nfgs_b200 import _lib as L

    s = NFGSSolverGPU(16, 14, 10, 1.0, 1.0, 1.0, dtype="float32")
    arr = (C.c_void_p * 1)(s._h.value)
    scan = C.c_void_p()
    assert L.lib().nfgs_scan_create(arr, 1, 2, C.byref(scan)) == L.NFGS_ESTATE

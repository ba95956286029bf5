"""Control flow of the overlapped scan runner without a GPU: the library's
scan calls and the solvers are replaced by fakes that record what the
runner asks for.  Every case must be begun once, joined to the scan once
(the first of each grid shape at creation, the others through
nfgs_scan_add), launched until all have stopped, and finished in case
order."""

import ctypes as C
import threading

import pytest


class _FakeSolver:
    def __init__(self, case, handle):
        self.case = case
        self._h = C.c_void_p(handle)
        self.Nx = self.Ny = case["n"]
        self.Nz = case["nz"]
        self.remaining = case["iters"]
        self.finished = False

    def _iterate_begin(self, **kw):
        assert kw["use_graph"] is True
        return {"handle": self._h.value}

    def _iterate_finish(self, ctx):
        assert ctx["handle"] == self._h.value and self.remaining == 0
        self.finished = True
        return {"sigma": [0.0] * self.case["iters"], "handle": self._h.value}


class _FakeLib:
    """nfgs_scan_*: a launch advances every joined solve by `iters` steps."""

    def __init__(self, solvers):
        self.solvers = solvers  # handle -> solver
        self.joined = []
        self.lock = threading.Lock()
        self.launches = 0
        self.iters = 0

    def nfgs_scan_create(self, arr, n, iters, out):
        self.iters = iters
        self.joined += [arr[i] for i in range(n)]
        C.cast(out, C.POINTER(C.c_void_p))[0] = C.c_void_p(1)
        return 0

    def nfgs_scan_add(self, scan, arr, n):
        new = [arr[i] for i in range(n)]
        assert not set(new) & set(self.joined), "a solve joined twice"
        self.joined += new
        return 0

    def nfgs_scan_launch(self, scan, active):
        self.launches += 1
        n = 0
        for h in self.joined:
            s = self.solvers[h]
            s.remaining = max(0, s.remaining - self.iters)
            n += s.remaining > 0
        C.cast(active, C.POINTER(C.c_int32))[0] = n
        return 0

    def nfgs_scan_destroy(self, scan):
        return 0


def test_overlapped_runner_joins_launches_and_finishes_every_case(monkeypatch):
    torch = pytest.importorskip("torch")
    from nfgs_b200 import scan as S

    cases = [dict(n=n, nz=n // 2, iters=it) for n, it in
             [(32, 9), (48, 5), (32, 17), (32, 3), (48, 12), (64, 7), (48, 1), (32, 25)]]
    made = {}
    lock = threading.Lock()

    def fake_solver(case):
        with lock:
            h = 1000 + len(made)
            made[h] = _FakeSolver(case, h)
            return made[h]

    lib = _FakeLib(made)
    monkeypatch.setattr(S, "_solver", fake_solver)
    monkeypatch.setattr(S.L, "lib", lambda: lib)
    monkeypatch.setattr(S.L, "check", lambda rc: None)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    hists, timing = S.run_scan_overlapped(cases, iters=4, max_iter=100, workers=3)

    assert len(made) == len(cases)                       # each case begun once
    assert sorted(lib.joined) == sorted(made)             # and joined once
    assert all(s.finished for s in made.values())
    # histories come back in case order
    by_handle = {h: s.case for h, s in made.items()}
    assert [by_handle[hh["handle"]] for hh in hists] == cases
    assert timing["graph_launches"] == lib.launches >= max(c["iters"] for c in cases) // 4
    assert timing["cell_iterations"] == sum(c["n"] * c["n"] * (c["n"] // 2) * c["iters"] for c in cases)

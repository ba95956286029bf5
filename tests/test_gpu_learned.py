"""The learned warm start on the GPU: every nfgs_nn_* kernel and the full
network forward / backward against the FP64 CPU oracle, and the solver's
learned-start hand-off (acceptance and the gs_cfcf fallback)."""

import ctypes as C

import numpy as np
import pytest

from oracle import fno_oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.detach().cpu().numpy().astype(np.float64)


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-30))


def P(t):
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


@pytest.fixture(scope="module")
def lib():
    from nfgs_b200 import _lib as L

    return L.lib()


def _ok(rc):
    from nfgs_b200 import _lib as L

    assert rc == L.NFGS_OK, L.lib().nfgs_nn_last_error()


@pytest.mark.parametrize("ci,co", [(32, 32), (6, 32), (32, 2)])
def test_pointwise_forward_backward(lib, ci, co):
    rng = np.random.default_rng(1)
    nv = 3000
    x, W, b, gy = rng.standard_normal((ci, nv)), rng.standard_normal((co, ci)), rng.standard_normal(co), \
        rng.standard_normal((co, nv))
    y = torch.zeros((co, nv), device="cuda")
    xd, Wd, bd, gyd = dev(x), dev(W), dev(b), dev(gy)
    _ok(lib.nfgs_nn_pointwise(P(xd), P(Wd), P(bd), P(y), ci, co, nv, 0, None))
    assert rel(host(y), W @ x + b[:, None]) < 1e-6
    gx = torch.zeros((ci, nv), device="cuda")
    gW = torch.zeros((co, ci), device="cuda")
    gb = torch.zeros(co, device="cuda")
    scratch = torch.empty(((nv + 1023) // 1024) * (co * ci + co), device="cuda")
    _ok(lib.nfgs_nn_pointwise_bwd(P(xd), P(Wd), P(gyd), P(gx), P(gW), P(gb), ci, co, nv, 0, P(scratch),
                                  scratch.numel(), None))
    assert rel(host(gx), W.T @ gy) < 1e-6
    assert rel(host(gW), gy @ x.T) < 1e-5
    assert rel(host(gb), gy.sum(axis=1)) < 1e-5


def test_gelu_forward_backward(lib):
    rng = np.random.default_rng(2)
    x, gy = rng.standard_normal(5000) * 3, rng.standard_normal(5000)
    y = torch.zeros(5000, device="cuda")
    gx = torch.zeros(5000, device="cuda")
    xd, gyd = dev(x), dev(gy)
    _ok(lib.nfgs_nn_gelu(P(xd), P(y), 5000, None))
    _ok(lib.nfgs_nn_gelu_bwd(P(xd), P(gyd), P(gx), 5000, 0, None))
    np.testing.assert_allclose(host(y), O.gelu(x), rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(host(gx), gy * O.gelu_grad(x), rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("shape,modes", [((9, 13, 17), (3, 4, 5)), ((65, 130, 130), (12, 12, 12))])
def test_reduce_expand_modemix(lib, shape, modes):
    rng = np.random.default_rng(3)
    Cc = 4
    nz, ny, nx = shape
    kz, ky, kx = modes
    v = rng.standard_normal((Cc,) + shape)
    Az, Sz = O.cosine_bases(nz, kz)
    Ay, Sy = O.cosine_bases(ny, ky)
    Ax, Sx = O.cosine_bases(nx, kx)
    big = torch.empty(Cc * nz * ny * kx, device="cuda")
    small = torch.empty(Cc * nz * ky * kx, device="cuda")
    a = torch.zeros((Cc, kz, ky, kx), device="cuda")
    vd, Azd, Ayd, Axd, Szd, Syd, Sxd = dev(v), dev(Az), dev(Ay), dev(Ax), dev(Sz), dev(Sy), dev(Sx)
    _ok(lib.nfgs_nn_reduce3(P(vd), P(a), Cc, nz, ny, nx, P(Azd), P(Ayd), P(Axd), kz, ky, kx,
                            P(big), P(small), None))
    aref = O.reduce3(v, Az, Ay, Ax)
    assert rel(host(a), aref) < 2e-6
    base = rng.standard_normal((Cc,) + shape)
    u = dev(base)
    ad = dev(aref)
    _ok(lib.nfgs_nn_expand3(P(ad), P(u), Cc, nz, ny, nx, P(Szd), P(Syd), P(Sxd), kz, ky, kx, 1,
                            P(small), P(big), None))
    assert rel(host(u), base + O.expand3(aref, Sz, Sy, Sx)) < 2e-6
    nm = kz * ky * kx
    W = rng.standard_normal((nm, Cc, 3))
    xh = rng.standard_normal((Cc, nm))
    yh = torch.zeros((3, nm), device="cuda")
    xhd, Wd = dev(xh), dev(W)
    _ok(lib.nfgs_nn_modemix(P(xhd), P(Wd), P(yh), Cc, 3, nm, None))
    assert rel(host(yh), O.modemix(xh, W)) < 1e-6
    gyh = rng.standard_normal((3, nm))
    gxh = torch.zeros((Cc, nm), device="cuda")
    gW = torch.zeros((nm, Cc, 3), device="cuda")
    gyhd = dev(gyh)
    _ok(lib.nfgs_nn_modemix_bwd(P(xhd), P(Wd), P(gyhd), P(gxh), P(gW), Cc, 3, nm, None))
    assert rel(host(gxh), np.einsum("kio,ok->ik", W, gyh)) < 1e-6
    assert rel(host(gW), np.einsum("ik,ok->kio", xh, gyh)) < 1e-6


def test_mse_and_adam(lib):
    rng = np.random.default_rng(4)
    n = 10000
    p, t, m = rng.standard_normal(n), rng.standard_normal(n), (rng.random(n) > 0.3).astype(np.float64)
    g = torch.zeros(n, device="cuda")
    part = torch.zeros((n + 255) // 256, dtype=torch.float64, device="cuda")
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    cnt = float(m.sum())
    pd, td, md = dev(p), dev(t), dev(m)
    _ok(lib.nfgs_nn_mse(P(pd), P(td), P(md), P(g), n, cnt, P(part), P(loss), None))
    d = (p.astype(np.float32) - t.astype(np.float32)).astype(np.float64) * m
    np.testing.assert_allclose(loss.item(), np.sum(d * d) / cnt, rtol=1e-6)
    np.testing.assert_allclose(host(g), 2 * d / cnt, rtol=1e-5, atol=1e-9)
    w, gr = rng.standard_normal(n), rng.standard_normal(n)
    wt, mt, vt = dev(w), torch.zeros(n, device="cuda"), torch.zeros(n, device="cuda")
    grd = dev(gr)
    for step in (1, 2):
        _ok(lib.nfgs_nn_adam(P(wt), P(grd), P(mt), P(vt), n, 1e-2, 0.9, 0.999, 1e-8, 0.0, step, None))
    m1 = 0.1 * gr
    v1 = 0.001 * gr * gr
    w1 = w - 1e-2 * (m1 / 0.1) / (np.sqrt(v1 / 0.001) + 1e-8)
    m2 = 0.9 * m1 + 0.1 * gr
    v2 = 0.999 * v1 + 0.001 * gr * gr
    w2 = w1 - 1e-2 * (m2 / (1 - 0.81)) / (np.sqrt(v2 / (1 - 0.999 ** 2)) + 1e-8)
    np.testing.assert_allclose(host(wt), w2, rtol=1e-5, atol=1e-6)


def test_network_forward_backward_against_oracle():
    """Whole network (production width 32) at a small grid: output and every
    parameter gradient within FP32 tolerance of the FP64 oracle."""
    from nfgs_b200.learned import Config, NeuralOperator, init_params

    cfg = Config(cin=6, width=32, layers=3, modes=(3, 4, 4), hidden=32, cout=2, seed=5, out_modes=(5, 6, 7))
    rng = np.random.default_rng(6)
    params = init_params(cfg)
    params["proj2_W"] = (0.2 * rng.standard_normal(params["proj2_W"].shape)).astype(np.float32)
    for k in params:
        if params[k].ndim == 1:
            params[k] = (0.1 * rng.standard_normal(params[k].shape)).astype(np.float32)
    net = NeuralOperator(cfg, params)
    x = rng.standard_normal((6, 7, 9, 11))
    gy = rng.standard_normal((2, 7, 9, 11))
    y = net.forward(dev(x), cache=True)
    net.zero_grad()
    gx = net.backward(dev(gy))
    ocfg = dict(cin=6, width=32, layers=3, modes=(3, 4, 4), hidden=32, cout=2, out_modes=(5, 6, 7))
    p64 = {k: v.astype(np.float64) for k, v in params.items()}
    yo, cache = O.forward(p64, ocfg, x)
    go, gxo = O.backward(p64, ocfg, cache, gy)
    assert rel(host(y), yo) < 1e-5
    assert rel(host(gx), gxo) < 1e-4
    grads = net.get_grads()
    for k in go:
        assert rel(grads[k], go[k]) < 1e-4, k


def test_training_reduces_loss():
    """A few Adam steps on one sample reduce the masked MSE (kernels compose
    into a working optimiser)."""
    from nfgs_b200.learned import Config, NeuralOperator

    cfg = Config(cin=6, width=32, layers=2, modes=(4, 4, 4), hidden=32, cout=2, seed=7, out_modes=(6, 6, 6))
    net = NeuralOperator(cfg)
    rng = np.random.default_rng(8)
    x = dev(rng.standard_normal((6, 9, 10, 11)))
    zz, yy, xx = np.meshgrid(np.linspace(0, 1, 9), np.linspace(0, 1, 10), np.linspace(0, 1, 11), indexing="ij")
    t = dev(np.stack([np.cos(np.pi * xx) * zz, np.sin(np.pi * yy) * (1 - zz)]))
    mask = torch.ones_like(t)
    losses = []
    for _ in range(40):
        y = net.forward(x, cache=True)
        loss, g = net.mse(y, t, mask)
        net.zero_grad()
        net.backward(g)
        net.adam_step(lr=3e-3)
        losses.append(loss.item())
    assert losses[-1] < 0.3 * losses[0]


def test_learned_start_accepts_better_state_and_falls_back():
    """The solver keeps a supplied start only when its sigma_J is lower: the
    converged state of a plain solve is accepted (and the iteration starts at
    its sigma), a noisy state is rejected and the run equals the plain one."""
    from nfgs_b200 import NFGSSolverGPU
    from nfgs_b200.synthetic import sunspot_magnetogram

    bx, by, bz = sunspot_magnetogram(40, seed=11)
    kw = dict(dtype="float32", bottom_divergence_robin_weight=0.5, d0_zero_mode_policy="project",
              source_zero_mode_policy="project")

    def make():
        s = NFGSSolverGPU(40, 40, 20, 1.0, 1.0, 1.0, **kw)
        s.set_bottom_vector_boundary(bx, by, bz, zero_net_current=False, smooth_passes=0, ijzbcor=3)
        return s

    s = make()
    plain = s.iterate(max_iter=300, tol=1e-5, patience=40, sigma_improvement_tol=1e-5, verbose=False)
    phi_b, az_b, _ = s._get_state(0)
    good = (torch.from_numpy(phi_b.astype(np.float32)).cuda(), torch.from_numpy(az_b.astype(np.float32)).cuda())

    s2 = make()
    h = s2.iterate(max_iter=300, tol=1e-5, patience=40, sigma_improvement_tol=1e-5, verbose=False,
                   init_mode="learned", warm_start=lambda solver, phi, az: good)
    info = h["learned_start"]
    assert info["accepted"]
    np.testing.assert_allclose(info["sigma_learned"], plain["best_sigma"], rtol=2e-3)
    np.testing.assert_allclose(h["initial_sigma"], info["sigma_learned"], rtol=1e-12)
    assert h["best_sigma"] <= plain["best_sigma"] * (1 + 2e-3)

    s3 = make()

    def noisy(solver, phi, az):
        g = torch.Generator(device="cuda").manual_seed(0)
        return (phi + 10.0 * phi.abs().max() * torch.randn(phi.shape, device="cuda", generator=g), az)

    h3 = s3.iterate(max_iter=300, tol=1e-5, patience=40, sigma_improvement_tol=1e-5, verbose=False,
                    init_mode="learned", warm_start=noisy)
    assert not h3["learned_start"]["accepted"]
    assert h3["sigma"] == plain["sigma"]


def test_resampling_between_grids():
    """Trilinear resampling reproduces a linear field exactly; cosine
    resampling of a band-limited field equals its synthesis on the target."""
    from nfgs_b200 import learned as LN

    cfg = LN.Config(cin=2, width=8, layers=1, modes=(3, 3, 3), hidden=8, cout=2, out_modes=(4, 5, 6))
    model = LN.NeuralOperator(cfg)
    src, dst = (9, 14, 17), (5, 8, 10)
    z, y, x = np.meshgrid(*(np.linspace(0, 1, n) for n in src), indexing="ij")
    lin = np.stack([1 + 2 * x - 3 * y + 0.5 * z, x * 0 + 4.0]).astype(np.float32)
    out = LN.resample_linear(model, torch.from_numpy(lin).cuda(), dst).cpu().numpy()
    z2, y2, x2 = np.meshgrid(*(np.linspace(0, 1, n) for n in dst), indexing="ij")
    np.testing.assert_allclose(out[0], 1 + 2 * x2 - 3 * y2 + 0.5 * z2, atol=2e-6)
    np.testing.assert_allclose(out[1], 4.0, atol=1e-6)
    rng = np.random.default_rng(2)
    k = (4, 5, 6)
    coef = rng.normal(size=(2,) + k)

    def synth(shape):
        Sz, Sy, Sx = (LN.cosine_bases(n, kk)[1] for n, kk in zip(shape, k))
        return np.einsum("cabd,ai,bj,dk->cijk", coef, Sz, Sy, Sx)

    f = torch.from_numpy(synth(src).astype(np.float32)).cuda()
    g = LN.resample_modes(model, f, dst, k).cpu().numpy()
    ref = synth(dst)
    np.testing.assert_allclose(g, ref, atol=2e-5 * np.abs(ref).max())


def test_restart_evaluate_only_modes_restore_the_start():
    """Mode 3 evaluates candidates without restoring the start's sources;
    mode 4, or the first advance, restores them: the run then equals the plain
    one bit for bit."""
    import ctypes as C

    from nfgs_b200 import NFGSSolverGPU
    from nfgs_b200 import _lib as L
    from nfgs_b200.learned import start_state_views
    from nfgs_b200.synthetic import sunspot_magnetogram

    bx, by, bz = sunspot_magnetogram(40, seed=12)
    kw = dict(dtype="float32", bottom_divergence_robin_weight=0.5, d0_zero_mode_policy="project",
              source_zero_mode_policy="project")
    stop = dict(max_iter=60, tol=1e-5, patience=40, sigma_improvement_tol=1e-5, verbose=False)

    def make():
        s = NFGSSolverGPU(40, 40, 20, 1.0, 1.0, 1.0, **kw)
        s.set_bottom_vector_boundary(bx, by, bz, zero_net_current=False, smooth_passes=0, ijzbcor=3)
        return s

    plain = make().iterate(**stop)
    for final_mode in (4, None):
        s = make()
        ctx = s._iterate_begin(**stop)
        phi, az = start_state_views(s)
        out = np.zeros(3)
        for scale in (1.5, 0.5):
            cp, ca = (phi * scale).contiguous(), (az * scale).contiguous()
            torch.cuda.synchronize()
            L.check(s._lib.nfgs_iterate_restart_from(s._h, C.c_void_p(cp.data_ptr()), C.c_void_p(ca.data_ptr()),
                                                     3, L.dptr(out)))
            assert np.isfinite(out[0]) and out[2] == 0.0
        if final_mode == 4:
            L.check(s._lib.nfgs_iterate_restart_from(s._h, None, None, 4, L.dptr(out)))
            assert np.isnan(out[0])
        s._iterate_loop(ctx)
        h = s._iterate_finish(ctx)
        assert h["sigma"] == plain["sigma"]

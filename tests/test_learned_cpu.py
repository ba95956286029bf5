"""CPU checks of the learned warm start: the oracle's gradients against
finite differences, the cosine bases, parameter initialisation and masks."""

import numpy as np
import pytest

from oracle import fno_oracle as O

CFG = dict(cin=3, width=4, layers=2, modes=(2, 3, 3), hidden=3, cout=2, out_modes=(3, 4, 4))


def _params(rng):
    from nfgs_b200.learned import Config, init_params

    cfg = Config(cin=3, width=4, layers=2, modes=(2, 3, 3), hidden=3, cout=2, seed=3, out_modes=(3, 4, 4))
    p = {k: v.astype(np.float64) for k, v in init_params(cfg).items()}
    # non-zero output layer and biases so every path carries gradient
    for k in p:
        p[k] = p[k] + 0.3 * rng.standard_normal(p[k].shape)
    return p


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    p = _params(rng)
    x = rng.standard_normal((3, 4, 5, 6))
    gy = rng.standard_normal((2, 4, 5, 6))
    y, cache = O.forward(p, CFG, x)
    g, gx = O.backward(p, CFG, cache, gy)
    assert set(g) == set(p)
    eps = 1e-6
    for name in p:
        d = rng.standard_normal(p[name].shape)
        pp = dict(p)
        pm = dict(p)
        pp[name] = p[name] + eps * d
        pm[name] = p[name] - eps * d
        fd = (np.sum(gy * O.forward(pp, CFG, x)[0]) - np.sum(gy * O.forward(pm, CFG, x)[0])) / (2 * eps)
        an = float(np.sum(g[name] * d))
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (name, fd, an)
    d = rng.standard_normal(x.shape)
    fd = (np.sum(gy * O.forward(p, CFG, x + eps * d)[0]) - np.sum(gy * O.forward(p, CFG, x - eps * d)[0])) / (2 * eps)
    assert abs(fd - float(np.sum(gx * d))) <= 1e-6 * max(1.0, abs(fd))


def test_cosine_bases_match_oracle_and_project_low_modes():
    from nfgs_b200.learned import cosine_bases

    for n, k in ((65, 12), (130, 12), (258, 12), (5, 3)):
        A, S = cosine_bases(n, k)
        Ao, So = O.cosine_bases(n, k)
        np.testing.assert_allclose(A, Ao, rtol=0, atol=1e-7)
        np.testing.assert_allclose(S, So, rtol=1e-6, atol=1e-6)
    # S^T A reproduces a cosine series of degree < k up to the trapezoid-rule error
    n, k = 129, 6
    A, S = O.cosine_bases(n, k)
    t = np.linspace(0.0, 1.0, n)
    f = 0.3 + np.cos(np.pi * t) - 0.5 * np.cos(3 * np.pi * t)
    np.testing.assert_allclose(S.T @ (A @ f), f, atol=1e-12)


def test_init_params_shapes_and_determinism():
    from nfgs_b200.learned import Config, init_params

    cfg = Config()
    a = init_params(cfg)
    b = init_params(cfg)
    n = sum(v.size for v in a.values())
    # 4 spectral layers of 12^3 modes x 32 x 32 dominate
    assert n == 6 * 32 + 32 + 4 * (12 ** 3 * 32 * 32 + 32 * 32 + 32) + 32 * 32 + 32 + 2 * 32 + 2
    for k in a:
        np.testing.assert_array_equal(a[k], b[k])
    assert not np.any(a["proj2_W"])


def test_masks_keep_boundary_values():
    torch = pytest.importorskip("torch")
    from nfgs_b200.learned import masks

    m = masks(5, 6, 7, torch.device("cpu")).numpy()
    assert m.shape == (2, 5, 6, 7)
    assert not m[0, 0].any() and m[0, 1:].all()
    assert not m[1, 0].any() and not m[1, -1].any()
    assert not m[1, :, 0].any() and not m[1, :, :, -1].any()
    assert m[1, 1:-1, 1:-1, 1:-1].all()


def test_start_filter_option_parses():
    from nfgs_b200.learned import NeuralOperator
    from nfgs_b200.warmstart_train import parse_filters

    assert parse_filters("none") == (None,)
    assert parse_filters("none;10,10,10") == (None, (10, 10, 10))
    assert parse_filters("16,12,12") == ((16, 12, 12),)
    assert NeuralOperator.start_filters == (None,)

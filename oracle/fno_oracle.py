"""CPU oracle of the learned warm start's neural operator (test infrastructure).

A plain NumPy (FP64) restatement of the operators and of the full forward and
backward pass that nfgs_b200.learned composes from the nfgs_nn_* CUDA
kernels.  Only tests compare against it.  There is no reference counterpart
for this network (the reference starts every solve from the zero-source
state, nfgs_solver.py:6613-6645); the oracle itself is pinned by
finite-difference checks of its gradients (tests/test_learned_cpu.py).
"""

from __future__ import annotations

import numpy as np
from scipy.special import erf


def cosine_bases(n, k):
    j = np.arange(n, dtype=np.float64)
    m = np.arange(k, dtype=np.float64)[:, None]
    c = np.cos(np.pi * m * j[None, :] / (n - 1))
    w = np.ones(n)
    w[0] = w[-1] = 0.5
    return c * w[None, :] / (n - 1), c * np.where(m == 0, 1.0, 2.0)


def pointwise(x, W, b):
    """x (ci, ...) -> (co, ...)."""
    y = np.tensordot(W, x, axes=([1], [0]))
    if b is not None:
        y = y + b.reshape((-1,) + (1,) * (x.ndim - 1))
    return y


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def reduce3(v, Mz, My, Mx):
    """v (C, nz, ny, nx) -> (C, kz, ky, kx)."""
    return np.einsum("az,by,cx,izyx->iabc", Mz, My, Mx, v, optimize=True)


def expand3(a, Mz, My, Mx):
    """a (C, kz, ky, kx) -> (C, nz, ny, nx)."""
    return np.einsum("az,by,cx,iabc->izyx", Mz, My, Mx, a, optimize=True)


def modemix(a, W):
    """a (ci, nm), W (nm, ci, co) -> (co, nm)."""
    return np.einsum("kio,ik->ok", W, a)


def forward(params, cfg, x):
    """Network output and the cache of the backward pass."""
    L = cfg["layers"]
    kz, ky, kx = cfg["modes"]
    _, nz, ny, nx = x.shape
    Az, Sz = cosine_bases(nz, kz)
    Ay, Sy = cosine_bases(ny, ky)
    Ax, Sx = cosine_bases(nx, kx)
    w = cfg["width"]
    h = pointwise(x, params["lift_W"], params["lift_b"])
    hs, zs, As = [h], [], []
    for l in range(L):
        a = reduce3(h, Az, Ay, Ax).reshape(w, -1)
        b = modemix(a, params[f"spec_W{l}"]).reshape(w, kz, ky, kx)
        z = pointwise(h, params[f"pw_W{l}"], params[f"pw_b{l}"]) + expand3(b, Sz, Sy, Sx)
        h = gelu(z) if l < L - 1 else z
        zs.append(z)
        As.append(a)
        hs.append(h)
    p1 = pointwise(h, params["proj1_W"], params["proj1_b"])
    q1 = gelu(p1)
    y = pointwise(q1, params["proj2_W"], params["proj2_b"])
    out_bases = None
    ko = cfg.get("out_modes", (0, 0, 0))
    if all(k > 0 for k in ko):
        kz2, ky2, kx2 = (min(k, n) for k, n in zip(ko, (nz, ny, nx)))
        (Aoz, Soz), (Aoy, Soy), (Aox, Sox) = cosine_bases(nz, kz2), cosine_bases(ny, ky2), cosine_bases(nx, kx2)
        out_bases = (Aoz, Aoy, Aox, Soz, Soy, Sox)
        y = expand3(reduce3(y, Aoz, Aoy, Aox), Soz, Soy, Sox)
    cache = dict(x=x, hs=hs, zs=zs, As=As, p1=p1, q1=q1, bases=(Az, Ay, Ax, Sz, Sy, Sx), out_bases=out_bases)
    return y, cache


def backward(params, cfg, cache, gy):
    """Gradients of <gy, y> with respect to every parameter and to x."""
    L = cfg["layers"]
    kz, ky, kx = cfg["modes"]
    w = cfg["width"]
    Az, Ay, Ax, Sz, Sy, Sx = cache["bases"]
    g = {}

    def pw_back(x, W, gyy, name):
        g[name + "_W"] = np.tensordot(gyy, x, axes=(list(range(1, x.ndim)), list(range(1, x.ndim))))
        g[name + "_b"] = gyy.sum(axis=tuple(range(1, x.ndim)))
        return np.tensordot(W, gyy, axes=([0], [0]))

    if cache.get("out_bases") is not None:
        Aoz, Aoy, Aox, Soz, Soy, Sox = cache["out_bases"]
        gy = expand3(reduce3(gy, Soz, Soy, Sox), Aoz, Aoy, Aox)
    gq = pw_back(cache["q1"], params["proj2_W"], gy, "proj2")
    gp = gq * gelu_grad(cache["p1"])
    gh = pw_back(cache["hs"][-1], params["proj1_W"], gp, "proj1")
    for l in range(L - 1, -1, -1):
        gz = gh * gelu_grad(cache["zs"][l]) if l < L - 1 else gh
        h = cache["hs"][l]
        gwp = np.tensordot(gz, h, axes=([1, 2, 3], [1, 2, 3]))
        g[f"pw_W{l}"] = gwp
        g[f"pw_b{l}"] = gz.sum(axis=(1, 2, 3))
        ghn = np.tensordot(params[f"pw_W{l}"], gz, axes=([0], [0]))
        gb = reduce3(gz, Sz, Sy, Sx).reshape(w, -1)
        a = cache["As"][l]
        g[f"spec_W{l}"] = np.einsum("ik,ok->kio", a, gb)
        ga = np.einsum("kio,ok->ik", params[f"spec_W{l}"], gb).reshape(w, kz, ky, kx)
        ghn = ghn + expand3(ga, Az, Ay, Ax)
        gh = ghn
    gx = pw_back(cache["x"], params["lift_W"], gh, "lift")
    return g, gx

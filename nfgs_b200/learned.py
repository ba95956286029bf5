"""Learned warm start for the NFGS iteration.

A 3-D neural operator on a truncated cosine basis predicts, from the
gs_cfcf start state and the bottom maps, the correction that takes the
start to the converged (best-sigma) state of the plain iteration.  The solver
starts from gs_cfcf + correction when that start has a lower sigma_J, and
from gs_cfcf otherwise; the plain NFPT iteration and its stop rule are
unchanged.  There is no reference counterpart: the reference always starts
from the zero-source state (nfgs_solver.py:6613-6645).

Every operator runs as a hand-written CUDA kernel of libnfgs_b200 (nfgs_nn_*);
PyTorch only allocates device buffers and supplies the stream.

Network (channel-major activations (C, Nz, Ny, Nx), FP32):
    h0 = lift(x)                                   pointwise cin -> width
    h_{l+1} = gelu(W_l h_l + b_l + S(M_l A h_l))   l = 0..L-1 (no gelu on the last)
    y = P2 gelu(P1 h_L + c1) + c2                  pointwise width -> hid -> cout
with A the analysis and S the synthesis of a cosine series truncated to
(kz, ky, kx) modes per axis, applied as separable per-axis contractions, and
M_l a real per-mode channel mixing.  The cosine basis of a grid of n nodes,
cos(pi k j / (n - 1)), represents the same physical frequencies at every
resolution, so a network trained on 130 x 130 x 65 calculation grids applies
to 258 x 258 x 129 grids unchanged.
"""

from __future__ import annotations

import ctypes as C
import json
import math
from dataclasses import asdict, dataclass, field
from pathlib import Path

import numpy as np

from . import _lib as L


def _torch():
    import torch

    return torch


def cosine_bases(n: int, k: int) -> tuple[np.ndarray, np.ndarray]:
    """Analysis A (k, n) and synthesis S (k, n) of the truncated cosine series.

    A[m, j] = w_j cos(pi m j / (n-1)) / (n-1) with trapezoid weights w,
    S[m, j] = c_m cos(pi m j / (n-1)) with c_0 = 1, c_m = 2, so S^T A is the
    projection onto the first k cosine modes of the node values.
    """
    if n < 2 or k < 1 or k > n:
        raise ValueError("cosine basis needs n >= 2 and 1 <= k <= n")
    j = np.arange(n, dtype=np.float64)
    m = np.arange(k, dtype=np.float64)[:, None]
    c = np.cos(np.pi * m * j[None, :] / (n - 1))
    w = np.ones(n)
    w[0] = w[-1] = 0.5
    A = c * w[None, :] / (n - 1)
    S = c * np.where(m == 0, 1.0, 2.0)
    return A.astype(np.float32), S.astype(np.float32)


@dataclass
class Config:
    cin: int = 6
    width: int = 32
    layers: int = 4
    modes: tuple = (12, 12, 12)   # (kz, ky, kx)
    hidden: int = 32
    cout: int = 2
    seed: int = 0
    # per-channel scales of (phi_c, A_z): inputs are divided by in_scale,
    # outputs multiplied by out_scale (training-set RMS after the field and
    # length scaling of each sample)
    in_scale: tuple = (1.0, 1.0)
    out_scale: tuple = (1.0, 1.0)
    # the output is band-limited to these cosine modes per axis (z, y, x),
    # capped by the grid; (0, 0, 0) leaves it unfiltered
    out_modes: tuple = (24, 24, 24)
    # (nz, ny, nx) of the calculation grids the network was trained on; the
    # learned start evaluates it there (features resampled, output brought
    # back by cosine synthesis); () evaluates it on the solver's grid
    train_shape: tuple = ()

    def param_shapes(self) -> list[tuple[str, tuple]]:
        w, nm = self.width, int(np.prod(self.modes))
        shapes = [("lift_W", (w, self.cin)), ("lift_b", (w,))]
        for l in range(self.layers):
            shapes += [(f"spec_W{l}", (nm, w, w)), (f"pw_W{l}", (w, w)), (f"pw_b{l}", (w,))]
        shapes += [("proj1_W", (self.hidden, w)), ("proj1_b", (self.hidden,)),
                   ("proj2_W", (self.cout, self.hidden)), ("proj2_b", (self.cout,))]
        return shapes


def init_params(cfg: Config) -> dict[str, np.ndarray]:
    """Seeded initial parameters (uniform +-1/sqrt(fan_in); spectral weights
    scaled by 1/width; the output layer starts at zero so the untrained
    network predicts no correction)."""
    rng = np.random.default_rng(cfg.seed)
    out = {}
    for name, shape in cfg.param_shapes():
        if name.startswith("spec_W"):
            v = rng.uniform(-1.0, 1.0, shape) / cfg.width
        elif len(shape) == 1:
            v = np.zeros(shape)
        elif name == "proj2_W":
            v = np.zeros(shape)
        else:
            fan_in = shape[1]
            v = rng.uniform(-1.0, 1.0, shape) / math.sqrt(fan_in)
        out[name] = v.astype(np.float32)
    return out


def _ck(rc: int):
    if rc != L.NFGS_OK:
        msg = L.lib().nfgs_nn_last_error()
        raise RuntimeError(f"nfgs_nn kernel failed ({rc}): {msg.decode() if msg else ''}")


def _p(t) -> C.c_void_p:
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


class Grid:
    """Device bases and scratch for one (nz, ny, nx) grid."""

    def __init__(self, model: "NeuralOperator", nz: int, ny: int, nx: int):
        torch = _torch()
        cfg = model.cfg
        self.nz, self.ny, self.nx = nz, ny, nx
        kz, ky, kx = cfg.modes
        if kz > nz or ky > ny or kx > nx:
            raise ValueError("grid smaller than the retained modes")
        dev = model.device
        self.A = [torch.from_numpy(cosine_bases(n, k)[0]).to(dev) for n, k in ((nz, kz), (ny, ky), (nx, kx))]
        self.S = [torch.from_numpy(cosine_bases(n, k)[1]).to(dev) for n, k in ((nz, kz), (ny, ky), (nx, kx))]
        w = max(cfg.width, cfg.hidden, cfg.cin)
        self.big = torch.empty(w * nz * ny * kx, device=dev)
        self.small = torch.empty(w * nz * ky * kx, device=dev)
        nvox = nz * ny * nx
        npair = w * w + w
        self.pw_scratch = torch.empty(((nvox + 1023) // 1024) * npair, device=dev)
        # band-limiting output filter
        self.ko = None
        if all(k > 0 for k in cfg.out_modes):
            ko = tuple(min(k, n) for k, n in zip(cfg.out_modes, (nz, ny, nx)))
            self.ko = ko
            self.Ao = [torch.from_numpy(cosine_bases(n, k)[0]).to(dev) for n, k in zip((nz, ny, nx), ko)]
            self.So = [torch.from_numpy(cosine_bases(n, k)[1]).to(dev) for n, k in zip((nz, ny, nx), ko)]
            co = cfg.cout
            self.big_o = torch.empty(co * nz * ny * ko[2], device=dev)
            self.small_o = torch.empty(co * nz * ko[1] * ko[2], device=dev)
            self.coef_o = torch.empty(co * ko[0] * ko[1] * ko[2], device=dev)


class NeuralOperator:
    """The warm-start network with its forward and backward pass.

    start_filters: the band limits (cosine modes per axis, or None for the
    unfiltered correction) that learned_start tries by default."""

    start_filters: tuple = (None,)

    def __init__(self, cfg: Config, params: dict[str, np.ndarray] | None = None, device="cuda"):
        torch = _torch()
        self.cfg = cfg
        self.device = torch.device(device)
        self.lib = L.lib()
        shapes = cfg.param_shapes()
        total = sum(int(np.prod(s)) for _, s in shapes)
        self.flat = torch.zeros(total, device=self.device)
        self.grad = torch.zeros(total, device=self.device)
        self.m = torch.zeros(total, device=self.device)
        self.v = torch.zeros(total, device=self.device)
        self.step = 0
        self.P, self.G = {}, {}
        off = 0
        for name, shape in shapes:
            n = int(np.prod(shape))
            self.P[name] = self.flat[off:off + n].view(shape)
            self.G[name] = self.grad[off:off + n].view(shape)
            off += n
        self.set_params(params if params is not None else init_params(cfg))
        self._grids: dict[tuple, Grid] = {}
        self.n_params = total

    # -------------------------------------------------------------- params
    def set_params(self, params: dict[str, np.ndarray]):
        torch = _torch()
        for name, t in self.P.items():
            t.copy_(torch.from_numpy(np.asarray(params[name], dtype=np.float32)).to(self.device).view(t.shape))

    def get_params(self) -> dict[str, np.ndarray]:
        return {k: v.detach().cpu().numpy().copy() for k, v in self.P.items()}

    def get_grads(self) -> dict[str, np.ndarray]:
        return {k: v.detach().cpu().numpy().copy() for k, v in self.G.items()}

    def save(self, path: str | Path):
        p = self.get_params()
        np.savez(path, config=json.dumps(asdict(self.cfg)), **{k: v.astype(np.float16) if k.startswith("spec_W")
                                                                else v for k, v in p.items()})

    @classmethod
    def load(cls, path: str | Path, device="cuda") -> "NeuralOperator":
        d = np.load(path, allow_pickle=False)
        c = json.loads(str(d["config"]))
        for key in ("modes", "in_scale", "out_scale", "out_modes", "train_shape"):
            if key in c:
                c[key] = tuple(c[key])
        cfg = Config(**c)
        params = {k: d[k].astype(np.float32) for k in d.files if k != "config"}
        return cls(cfg, params, device)

    def grid(self, nz, ny, nx) -> Grid:
        key = (nz, ny, nx)
        if key not in self._grids:
            self._grids[key] = Grid(self, nz, ny, nx)
        return self._grids[key]

    # -------------------------------------------------------------- ops
    def _stream(self):
        return C.c_void_p(_torch().cuda.current_stream(self.device).cuda_stream)

    def _pointwise(self, x, W, b, y, ci, co, nvox, acc=0):
        _ck(self.lib.nfgs_nn_pointwise(_p(x), _p(W), _p(b), _p(y), ci, co, nvox, acc, self._stream()))

    def _spectral_fwd(self, g: Grid, h, l, z):
        """z += S(M_l A h); returns the modal coefficients a = A h (cached)."""
        torch = _torch()
        cfg = self.cfg
        w = cfg.width
        kz, ky, kx = cfg.modes
        nm = kz * ky * kx
        a = torch.empty(w * nm, device=self.device)
        b = torch.empty(w * nm, device=self.device)
        _ck(self.lib.nfgs_nn_reduce3(_p(h), _p(a), w, g.nz, g.ny, g.nx, _p(g.A[0]), _p(g.A[1]), _p(g.A[2]),
                                     kz, ky, kx, _p(g.big), _p(g.small), self._stream()))
        _ck(self.lib.nfgs_nn_modemix(_p(a), _p(self.P[f"spec_W{l}"]), _p(b), w, w, nm, self._stream()))
        _ck(self.lib.nfgs_nn_expand3(_p(b), _p(z), w, g.nz, g.ny, g.nx, _p(g.S[0]), _p(g.S[1]), _p(g.S[2]),
                                     kz, ky, kx, 1, _p(g.small), _p(g.big), self._stream()))
        return a

    def _band_limit(self, g: Grid, y, first, second):
        """second^T (first y) over the output modes (the filter, or with the
        bases swapped its transpose)."""
        torch = _torch()
        kz, ky, kx = g.ko
        co = self.cfg.cout
        out = torch.empty_like(y)
        _ck(self.lib.nfgs_nn_reduce3(_p(y), _p(g.coef_o), co, g.nz, g.ny, g.nx, _p(first[0]), _p(first[1]),
                                     _p(first[2]), kz, ky, kx, _p(g.big_o), _p(g.small_o), self._stream()))
        _ck(self.lib.nfgs_nn_expand3(_p(g.coef_o), _p(out), co, g.nz, g.ny, g.nx, _p(second[0]), _p(second[1]),
                                     _p(second[2]), kz, ky, kx, 0, _p(g.small_o), _p(g.big_o), self._stream()))
        return out

    def forward(self, x, cache: bool = False):
        """x: (cin, nz, ny, nx) float32 device tensor -> (cout, nz, ny, nx)."""
        torch = _torch()
        cfg = self.cfg
        _, nz, ny, nx = x.shape
        g = self.grid(nz, ny, nx)
        nvox = nz * ny * nx
        w = cfg.width
        x = x.contiguous()
        h = torch.empty((w, nz, ny, nx), device=self.device)
        self._pointwise(x, self.P["lift_W"], self.P["lift_b"], h, cfg.cin, w, nvox)
        hs, zs, As = [h], [], []
        for l in range(cfg.layers):
            z = torch.empty_like(h)
            self._pointwise(h, self.P[f"pw_W{l}"], self.P[f"pw_b{l}"], z, w, w, nvox)
            a = self._spectral_fwd(g, h, l, z)
            if l < cfg.layers - 1:
                hn = torch.empty_like(z)
                _ck(self.lib.nfgs_nn_gelu(_p(z), _p(hn), z.numel(), self._stream()))
            else:
                hn = z
            zs.append(z)
            As.append(a)
            hs.append(hn)
            h = hn
        p1 = torch.empty((cfg.hidden, nz, ny, nx), device=self.device)
        self._pointwise(h, self.P["proj1_W"], self.P["proj1_b"], p1, w, cfg.hidden, nvox)
        q1 = torch.empty_like(p1)
        _ck(self.lib.nfgs_nn_gelu(_p(p1), _p(q1), p1.numel(), self._stream()))
        y = torch.empty((cfg.cout, nz, ny, nx), device=self.device)
        self._pointwise(q1, self.P["proj2_W"], self.P["proj2_b"], y, cfg.hidden, cfg.cout, nvox)
        if g.ko is not None:
            y = self._band_limit(g, y, g.Ao, g.So)
        if cache:
            self._cache = dict(x=x, hs=hs, zs=zs, As=As, p1=p1, q1=q1, grid=g)
        return y

    def backward(self, gy):
        """Accumulates parameter gradients of <gy, y> into self.grad; returns grad wrt x."""
        torch = _torch()
        cfg = self.cfg
        c = self._cache
        g = c["grid"]
        nz, ny, nx = g.nz, g.ny, g.nx
        nvox = nz * ny * nx
        w = cfg.width
        kz, ky, kx = cfg.modes
        nm = kz * ky * kx
        st = self._stream()
        sl = len(g.pw_scratch)
        gy = gy.contiguous()
        if g.ko is not None:
            gy = self._band_limit(g, gy, g.So, g.Ao)
        gq = torch.empty_like(c["q1"])
        _ck(self.lib.nfgs_nn_pointwise_bwd(_p(c["q1"]), _p(self.P["proj2_W"]), _p(gy.contiguous()), _p(gq),
                                           _p(self.G["proj2_W"]), _p(self.G["proj2_b"]), cfg.hidden, cfg.cout,
                                           nvox, 0, _p(g.pw_scratch), sl, st))
        gp = torch.empty_like(gq)
        _ck(self.lib.nfgs_nn_gelu_bwd(_p(c["p1"]), _p(gq), _p(gp), gp.numel(), 0, st))
        gh = torch.empty((w, nz, ny, nx), device=self.device)
        _ck(self.lib.nfgs_nn_pointwise_bwd(_p(c["hs"][-1]), _p(self.P["proj1_W"]), _p(gp), _p(gh),
                                           _p(self.G["proj1_W"]), _p(self.G["proj1_b"]), w, cfg.hidden, nvox, 0,
                                           _p(g.pw_scratch), sl, st))
        ga = torch.empty(w * nm, device=self.device)
        gb = torch.empty(w * nm, device=self.device)
        for l in range(cfg.layers - 1, -1, -1):
            if l < cfg.layers - 1:
                gz = torch.empty_like(gh)
                _ck(self.lib.nfgs_nn_gelu_bwd(_p(c["zs"][l]), _p(gh), _p(gz), gz.numel(), 0, st))
            else:
                gz = gh
            h = c["hs"][l]
            ghn = torch.empty_like(h)
            _ck(self.lib.nfgs_nn_pointwise_bwd(_p(h), _p(self.P[f"pw_W{l}"]), _p(gz), _p(ghn),
                                               _p(self.G[f"pw_W{l}"]), _p(self.G[f"pw_b{l}"]), w, w, nvox, 0,
                                               _p(g.pw_scratch), sl, st))
            # spectral path: gb = S gz, (ga, gW) = modemix^T, gh += A^T ga
            _ck(self.lib.nfgs_nn_reduce3(_p(gz), _p(gb), w, nz, ny, nx, _p(g.S[0]), _p(g.S[1]), _p(g.S[2]),
                                         kz, ky, kx, _p(g.big), _p(g.small), st))
            _ck(self.lib.nfgs_nn_modemix_bwd(_p(c["As"][l]), _p(self.P[f"spec_W{l}"]), _p(gb), _p(ga),
                                             _p(self.G[f"spec_W{l}"]), w, w, nm, st))
            _ck(self.lib.nfgs_nn_expand3(_p(ga), _p(ghn), w, nz, ny, nx, _p(g.A[0]), _p(g.A[1]), _p(g.A[2]),
                                         kz, ky, kx, 1, _p(g.small), _p(g.big), st))
            gh = ghn
        gx = torch.empty_like(c["x"])
        _ck(self.lib.nfgs_nn_pointwise_bwd(_p(c["x"]), _p(self.P["lift_W"]), _p(gh), _p(gx), _p(self.G["lift_W"]),
                                           _p(self.G["lift_b"]), cfg.cin, w, nvox, 0, _p(g.pw_scratch), sl, st))
        return gx

    def zero_grad(self):
        self.grad.zero_()

    def adam_step(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8, wd=0.0):
        self.step += 1
        _ck(self.lib.nfgs_nn_adam(_p(self.flat), _p(self.grad), _p(self.m), _p(self.v), self.flat.numel(),
                                  float(lr), float(b1), float(b2), float(eps), float(wd), self.step,
                                  self._stream()))

    def mse(self, pred, target, mask):
        """(loss as a device double tensor, gradient wrt pred)."""
        torch = _torch()
        n = pred.numel()
        grad = torch.empty_like(pred)
        part = torch.empty((n + 255) // 256, dtype=torch.float64, device=self.device)
        loss = torch.empty(1, dtype=torch.float64, device=self.device)
        count = float(mask.sum().item()) if mask is not None else float(n)
        _ck(self.lib.nfgs_nn_mse(_p(pred), _p(target), _p(mask), _p(grad), n, count, _p(part), _p(loss),
                                 self._stream()))
        return loss, grad


# ---------------------------------------------------------------------------
# Solver interface: features, masks, targets
# ---------------------------------------------------------------------------
class _DevView:
    """__cuda_array_interface__ over a device pointer owned by the solver."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"data": (int(ptr), False), "shape": tuple(shape), "typestr": typestr,
                                         "version": 2, "strides": None}


def start_state_views(solver):
    """Device views (torch) of the gs_cfcf start state after nfgs_iterate_begin."""
    torch = _torch()
    phi = C.c_void_p()
    az = C.c_void_p()
    L.check(solver._lib.nfgs_iterate_start_state(solver._h, C.byref(phi), C.byref(az)))
    ts = "<f4" if solver._np_dtype == np.float32 else "<f8"
    shape = (solver.Nz, solver.Ny, solver.Nx)
    return (torch.as_tensor(_DevView(phi.value, shape, ts), device="cuda"),
            torch.as_tensor(_DevView(az.value, shape, ts), device="cuda"))


def scales(solver) -> tuple[float, float]:
    """(field scale, length scale) that make features resolution-independent."""
    bz = solver._plane(0)
    bs = float(np.abs(bz).max()) or 1.0
    ls = float((solver.Nx - 1) * solver.dx)
    return bs, ls


def masks(nz, ny, nx, device):
    """Entries the correction may change: phi_c above the bottom plane; A_z
    away from the bottom, top and lateral walls."""
    torch = _torch()
    m = torch.ones((2, nz, ny, nx), device=device)
    m[0, 0] = 0.0
    m[1, 0] = 0.0
    m[1, -1] = 0.0
    m[1, :, 0] = 0.0
    m[1, :, -1] = 0.0
    m[1, :, :, 0] = 0.0
    m[1, :, :, -1] = 0.0
    return m


def features(solver, phi, az, in_scale=(1.0, 1.0)):
    """(6, nz, ny, nx) float32 features: phi_c, A_z of the start state, the
    bottom (Bx, By, Bz) broadcast in height, and the height fraction."""
    torch = _torch()
    bs, ls = scales(solver)
    nz, ny, nx = solver.Nz, solver.Ny, solver.Nx
    dev = phi.device
    x = torch.empty((6, nz, ny, nx), device=dev)
    x[0] = phi.float() / (bs * ls * in_scale[0])
    x[1] = az.float() / (bs * ls * in_scale[1])
    for c, plane in ((2, 1), (3, 2), (4, 0)):
        x[c] = torch.from_numpy((solver._plane(plane) / bs).astype(np.float32)).to(dev).view(1, ny, nx)
    x[5] = torch.linspace(0.0, 1.0, nz, device=dev).view(nz, 1, 1)
    return x


def band_limit(model: NeuralOperator, field, modes):
    """Project a (C, nz, ny, nx) device field onto its first `modes` cosine
    modes per axis (nfgs_nn_reduce3 then nfgs_nn_expand3)."""
    torch = _torch()
    C_, nz, ny, nx = field.shape
    kz, ky, kx = (min(k, n) for k, n in zip(modes, (nz, ny, nx)))
    A = [torch.from_numpy(cosine_bases(n, k)[0]).to(field.device) for n, k in ((nz, kz), (ny, ky), (nx, kx))]
    S = [torch.from_numpy(cosine_bases(n, k)[1]).to(field.device) for n, k in ((nz, kz), (ny, ky), (nx, kx))]
    f = field.float().contiguous()
    coef = torch.empty(C_ * kz * ky * kx, device=field.device)
    big = torch.empty(C_ * nz * ny * kx, device=field.device)
    small = torch.empty(C_ * nz * ky * kx, device=field.device)
    out = torch.empty_like(f)
    st = model._stream()
    _ck(model.lib.nfgs_nn_reduce3(_p(f), _p(coef), C_, nz, ny, nx, _p(A[0]), _p(A[1]), _p(A[2]), kz, ky, kx,
                                  _p(big), _p(small), st))
    _ck(model.lib.nfgs_nn_expand3(_p(coef), _p(out), C_, nz, ny, nx, _p(S[0]), _p(S[1]), _p(S[2]), kz, ky, kx, 0,
                                  _p(small), _p(big), st))
    return out


def resample_linear(model: NeuralOperator, field, shape):
    """Trilinear resampling of a (C, nz, ny, nx) device field onto a node grid
    of `shape` spanning the same box (nfgs_nn_resample_linear)."""
    torch = _torch()
    C_, nz, ny, nx = field.shape
    dst = tuple(int(v) for v in shape)
    f = field.float().contiguous()
    out = torch.empty((C_,) + dst, device=field.device)
    _ck(model.lib.nfgs_nn_resample_linear(_p(f), _p(out), C_, nz, ny, nx, dst[0], dst[1], dst[2], model._stream()))
    return out


def resample_modes(model: NeuralOperator, field, shape, modes):
    """A field band-limited to `modes` cosine modes per axis (x <= 32) moved
    to a node grid of `shape` spanning the same box: analysis on the source
    grid (nfgs_nn_reduce3), synthesis on the target (nfgs_nn_expand3); exact
    for band-limited fields."""
    torch = _torch()
    C_, nz, ny, nx = field.shape
    src, dst = (nz, ny, nx), tuple(int(v) for v in shape)
    k = tuple(max(1, min(int(m), a, b)) for m, a, b in zip(modes, src, dst))
    A = [torch.from_numpy(cosine_bases(n, kk)[0]).to(field.device) for n, kk in zip(src, k)]
    S = [torch.from_numpy(cosine_bases(n, kk)[1]).to(field.device) for n, kk in zip(dst, k)]
    f = field.float().contiguous()
    coef = torch.empty(C_ * k[0] * k[1] * k[2], device=field.device)
    big = torch.empty(C_ * max(nz * ny * k[2], dst[0] * dst[1] * k[2]), device=field.device)
    small = torch.empty(C_ * max(nz * k[1] * k[2], dst[0] * k[1] * k[2]), device=field.device)
    out = torch.empty((C_,) + dst, device=field.device)
    st = model._stream()
    _ck(model.lib.nfgs_nn_reduce3(_p(f), _p(coef), C_, nz, ny, nx, _p(A[0]), _p(A[1]), _p(A[2]), k[0], k[1], k[2],
                                  _p(big), _p(small), st))
    _ck(model.lib.nfgs_nn_expand3(_p(coef), _p(out), C_, dst[0], dst[1], dst[2], _p(S[0]), _p(S[1]), _p(S[2]),
                                  k[0], k[1], k[2], 0, _p(small), _p(big), st))
    return out


def learned_start(solver, model, fallback: bool = True, scales_tried=(1.0, 0.6, 0.35, 0.2),
                  filters_tried=None, eval_shape="train") -> dict:
    """After nfgs_iterate_begin: hand a predicted start to the solver.

    model: a NeuralOperator, or a callable (solver, phi, az) -> (phi, az)
    returning a candidate start state as device tensors of the solver dtype.
    For the network, the predicted correction is tried at the given scales
    and the one with the lowest sigma_J is kept when it beats the gs_cfcf
    start (fallback) -- the plain iteration then runs unchanged.  Each band
    limit of filters_tried (default model.start_filters) is tried with every
    scale.  eval_shape (nz, ny, nx): evaluate the network on that grid from
    trilinearly resampled features, and bring its band-limited output back by
    cosine synthesis; "train" (default): the network's training grid
    (cfg.train_shape, or the solver grid when that is not recorded); None:
    the solver grid."""
    torch = _torch()
    phi, az = start_state_views(solver)
    lib = solver._lib
    out = np.zeros(3)

    def evaluate(cp, ca, mode):
        torch.cuda.current_stream().synchronize()  # the library reads them on its own stream
        L.check(lib.nfgs_iterate_restart_from(solver._h, C.c_void_p(cp.data_ptr()), C.c_void_p(ca.data_ptr()),
                                              mode, L.dptr(out)))
        return float(out[0]), float(out[1]), bool(out[2])

    if not isinstance(model, NeuralOperator):
        cand_phi, cand_az = model(solver, phi, az)
        cand_phi = cand_phi.to(device=phi.device, dtype=phi.dtype).contiguous()
        cand_az = cand_az.to(device=az.device, dtype=az.dtype).contiguous()
        s_new, s_gs, acc = evaluate(cand_phi, cand_az, 1 if fallback else 2)
        return {"sigma_learned": s_new, "sigma_gs_cfcf": s_gs, "accepted": acc}

    x = features(solver, phi, az, model.cfg.in_scale)
    bs, ls = scales(solver)
    if isinstance(eval_shape, str):
        eval_shape = tuple(model.cfg.train_shape) or None
    with torch.no_grad():
        if eval_shape is not None and tuple(eval_shape) != tuple(x.shape[1:]):
            if not all(0 < k <= 32 for k in model.cfg.out_modes[2:]) or not all(k > 0 for k in model.cfg.out_modes):
                raise ValueError("eval_shape needs a network with band-limited output (out_modes, x <= 32)")
            yc = model.forward(resample_linear(model, x, eval_shape))
            y = resample_modes(model, yc, x.shape[1:], model.cfg.out_modes)
        else:
            y = model.forward(x)
        m = masks(solver.Nz, solver.Ny, solver.Nx, x.device)
        osc = torch.tensor(model.cfg.out_scale, device=x.device, dtype=torch.float32).view(2, 1, 1, 1)
        corr = ((y * m) * osc * (bs * ls)).double()
    tried = []
    best = None
    for flt in (model.start_filters if filters_tried is None else filters_tried):
        cf = corr if flt is None else (band_limit(model, corr, flt) * m).double()
        for lam in scales_tried:
            cp = (phi.double() + lam * cf[0]).to(phi.dtype).contiguous()
            ca = (az.double() + lam * cf[1]).to(az.dtype).contiguous()
            s_new, s_gs, _ = evaluate(cp, ca, 3)  # the start's sources are restored once, below
            tried.append((flt, lam, s_new))
            if np.isfinite(s_new) and (best is None or s_new < best[1]):
                best = (lam, s_new, cp, ca, flt)
    accepted = False
    if best is not None and (not fallback or best[1] < s_gs):
        _, _, accepted = evaluate(best[2], best[3], 2)
    else:
        L.check(lib.nfgs_iterate_restart_from(solver._h, None, None, 4, L.dptr(out)))
    return {"sigma_learned": best[1] if best else float("nan"), "sigma_gs_cfcf": s_gs, "accepted": accepted,
            "scale": best[0] if best else None, "filter": best[4] if best else None, "tried": tried}

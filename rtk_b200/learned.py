"""Learned preconditioner for the conjugate-gradient reconstruction.

``UNet`` wraps the C ABI network (``rtkb_unet_*``): a 3-level 3D U-Net with
BF16 tensor-core convolutions whose forward and backward passes and Adam
updates run in librtkb200.  ``make_training_pairs`` draws error volumes e
(seeded Gaussian random fields with correlation lengths of 2-20 mm, mixed with
random-ellipsoid volumes) and applies the plan's own normal operator to get
r = A e; ``train`` fits N(r) ~ c e on random crops; ``ConjugateGradient.
set_preconditioner`` then runs flexible PCG with it, falling back to plain CG
whenever the normal-equation residual stops decreasing.

There is no RTK counterpart: RTK's conjugate gradient is unpreconditioned
(include/rtkConjugateGradientImageFilter.hxx:108-258).
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np

from ._capi import check, load
from .ops import _ptr, _stream

# layer (c_in, c_out) of the ten 3x3x3 convolutions, then the 1x1x1 output
LAYERS = [(1, 16), (16, 16), (16, 32), (32, 32), (32, 64), (64, 64), (96, 32), (32, 32), (48, 16), (16, 16)]


def layer_shapes():
    """Host parameter layout: [(27, c_in, c_out)] * 10 + [(16,)]."""
    return [(27, ci, co) for ci, co in LAYERS] + [(16,)]


class UNet:
    """Handle of a rtkb_unet network (weights live on the current device)."""

    def __init__(self, seed: int = 0):
        self._lib = load()
        h = C.c_void_p()
        check(self._lib.rtkb_unet_create(C.c_ulonglong(seed), C.byref(h)))
        self.handle = h
        self.n = int(self._lib.rtkb_unet_num_parameters(h))

    # -- parameters ------------------------------------------------------------------------------
    def get_parameters(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.float32)
        check(self._lib.rtkb_unet_get_parameters(self.handle, out.ctypes.data_as(C.POINTER(C.c_float)), self.n))
        return out

    def set_parameters(self, flat) -> None:
        flat = np.ascontiguousarray(flat, dtype=np.float32)
        if flat.size != self.n:
            raise ValueError(f"expected {self.n} parameters, got {flat.size}")
        check(self._lib.rtkb_unet_set_parameters(self.handle, flat.ctypes.data_as(C.POINTER(C.c_float)), self.n))

    def get_gradients(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.float32)
        check(self._lib.rtkb_unet_get_gradients(self.handle, out.ctypes.data_as(C.POINTER(C.c_float)), self.n))
        return out

    def split(self, flat):
        """Flat parameter vector -> list of per-layer arrays (layer_shapes())."""
        out, o = [], 0
        for shp in layer_shapes():
            k = int(np.prod(shp))
            out.append(np.asarray(flat[o:o + k]).reshape(shp))
            o += k
        return out

    def save(self, path: str) -> None:
        np.save(path, self.get_parameters())

    def load(self, path: str) -> None:
        self.set_parameters(np.load(path))

    # -- compute -----------------------------------------------------------------------------------
    def forward(self, x, out=None, normalize=True, stream=None):
        """x: float32 CUDA tensor (z, y, x) or (batch, z, y, x), sizes multiples of 4."""
        import torch

        xb = x if x.dim() == 4 else x.unsqueeze(0)
        if out is None:
            out = torch.empty_like(x)
        b, nz, ny, nx = xb.shape
        check(self._lib.rtkb_unet_forward(self.handle, b, nx, ny, nz, _ptr(x), _ptr(out), int(normalize),
                                          _stream(stream)))
        return out

    def train_step(self, x, target, lr=1e-3, update=True, want_loss=True, margin=0, stream=None):
        """One Adam step on mean((N(x) - target)^2) over the voxels at least
        `margin` inside every face; returns the loss (synchronises) or None."""
        b, nz, ny, nx = x.shape
        loss = C.c_double()
        check(self._lib.rtkb_unet_train_step(self.handle, b, nx, ny, nz, _ptr(x), _ptr(target), int(margin),
                                             float(lr), int(update), C.byref(loss) if want_loss else None,
                                             _stream(stream)))
        return loss.value if want_loss else None

    def close(self):
        if getattr(self, "handle", None):
            self._lib.rtkb_unet_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- training data ----------------------------------------------------------------------------------
def gaussian_random_field(shape, spacing_mm, corr_mm, gen, device):
    """Zero-mean, unit-rms Gaussian random field whose autocorrelation is a
    Gaussian of standard deviation corr_mm (white noise filtered in Fourier
    space)."""
    import torch

    nz, ny, nx = shape
    w = torch.randn(shape, generator=gen, device=device, dtype=torch.float32)
    kz = torch.fft.fftfreq(nz, d=spacing_mm[2], device=device)
    ky = torch.fft.fftfreq(ny, d=spacing_mm[1], device=device)
    kx = torch.fft.rfftfreq(nx, d=spacing_mm[0], device=device)
    k2 = kz[:, None, None] ** 2 + ky[None, :, None] ** 2 + kx[None, None, :] ** 2
    filt = torch.exp(-2.0 * (math.pi * corr_mm) ** 2 * k2)
    f = torch.fft.irfftn(torch.fft.rfftn(w) * filt, s=shape)
    return f / f.pow(2).mean().sqrt().clamp_min(1e-30)


def ellipsoid_volume(shape, spacing_mm, origin_mm, n, gen, device, field_mm=200.0):
    """Sum of n random ellipsoids (semi-axes 5-80 mm, centres in a sphere of
    diameter field_mm, random rotations, densities in [-1, 1])."""
    import torch

    nz, ny, nx = shape
    z = origin_mm[2] + spacing_mm[2] * torch.arange(nz, device=device, dtype=torch.float32)
    y = origin_mm[1] + spacing_mm[1] * torch.arange(ny, device=device, dtype=torch.float32)
    x = origin_mm[0] + spacing_mm[0] * torch.arange(nx, device=device, dtype=torch.float32)
    out = torch.zeros(shape, device=device, dtype=torch.float32)
    u = lambda *s: torch.rand(*s, generator=gen, device=device)  # noqa: E731
    for _ in range(n):
        axes = 5.0 + 75.0 * u(3)
        d = torch.randn(3, generator=gen, device=device)
        c = d / d.norm() * (field_mm / 2) * u(1) ** (1 / 3)
        q, _ = torch.linalg.qr(torch.randn(3, 3, generator=gen, device=device))
        dens = 2.0 * u(1) - 1.0
        px = (x - c[0])[None, None, :]
        py = (y - c[1])[None, :, None]
        pz = (z - c[2])[:, None, None]
        acc = 0.0
        for a in range(3):
            la = (q[0, a] * px + q[1, a] * py + q[2, a] * pz) / axes[a]
            acc = acc + la * la
        out += dens * (acc <= 1.0).float()
    return out


def _geometry_of(plan):
    vd = plan.vol_desc
    shape = (vd.size[2], vd.size[1], vd.size[0])
    spacing = tuple(vd.spacing[a] for a in range(3))
    origin = tuple(vd.origin[a] for a in range(3))
    return shape, spacing, origin


def draw_field(shape, spacing, origin, rng, gen, dev, corr_mm=(2.0, 20.0), ellipsoid_fraction=0.5):
    """One error volume: a Gaussian random field with a log-uniform
    correlation length in corr_mm, with probability ellipsoid_fraction scaled
    down and added to 5 random ellipsoids."""
    corr = float(np.exp(rng.uniform(np.log(corr_mm[0]), np.log(corr_mm[1]))))
    e = gaussian_random_field(shape, spacing, corr, gen, dev)
    if rng.uniform() < ellipsoid_fraction:
        e = e * float(rng.uniform(0.1, 1.0)) + ellipsoid_volume(shape, spacing, origin, 5, gen, dev)
    return e.contiguous()


def _finish_pairs(rs, es, sr, se):
    c = float(np.median(np.array(sr) / np.array(se)))
    for e in es:
        e.mul_(c)
    return rs, es, c


def make_training_pairs(plan, n_pairs, seed=20261203 + 5, corr_mm=(2.0, 20.0), ellipsoid_fraction=0.5,
                        stream=None):
    """[(r_i, e_i)] with r_i = A e_i through the plan's own normal operator,
    e_i drawn by draw_field.  Returns (inputs, targets, c): inputs
    r_i / rms(r_i), targets c e_i / rms(r_i), c = median rms(r_i) / rms(e_i),
    so that N ~ c A^-1 with O(1) values (the PCG direction does not depend on
    the scale c)."""
    import torch

    shape, spacing, origin = _geometry_of(plan)
    dev = torch.device("cuda")
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    rng = np.random.default_rng(seed)
    es, rs, sr, se = [], [], [], []
    for _ in range(n_pairs):
        e = draw_field(shape, spacing, origin, rng, gen, dev, corr_mm, ellipsoid_fraction)
        r = torch.empty_like(e)
        plan.apply_operator(e, r, stream=stream)
        s_r = float(r.pow(2).mean().sqrt())
        rs.append(r.div_(s_r))
        se.append(float(e.pow(2).mean().sqrt()))
        es.append(e.div_(s_r))
        sr.append(s_r)
    return _finish_pairs(rs, es, sr, se)


def make_krylov_pairs(plan, n_problems, iterations=20, every=2, seed=20261203 + 6, corr_mm=(2.0, 20.0),
                      ellipsoid_fraction=0.5, stream=None):
    """Pairs (A e, e) whose e are the errors plain CG leaves behind: for each
    synthetic problem x* = draw_field(...), b = A x*, run plain CG from 0 and
    take e_k = x* - x_k (and r_k = A e_k, recomputed exactly) every `every`
    iterations up to `iterations`.  Early e_k are smooth, late ones hold the
    slowly converging components -- the residuals a preconditioner meets.
    Returns (inputs, targets, c) as make_training_pairs."""
    import torch

    shape, spacing, origin = _geometry_of(plan)
    dev = torch.device("cuda")
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    rng = np.random.default_rng(seed)
    es, rs, sr, se = [], [], [], []
    for _ in range(n_problems):
        xs = draw_field(shape, spacing, origin, rng, gen, dev, corr_mm, ellipsoid_fraction)
        b = torch.empty_like(xs)
        plan.apply_operator(xs, b, stream=stream)
        x = torch.zeros_like(xs)
        plan.start_rhs(b, x, stream=stream)
        for k in range(iterations + 1):
            if k % every == 0:
                e = (xs - x).contiguous()
                r = torch.empty_like(e)
                plan.apply_operator(e, r, stream=stream)
                s_r = float(r.pow(2).mean().sqrt())
                if s_r > 0:
                    rs.append(r.div_(s_r))
                    se.append(float(e.pow(2).mean().sqrt()))
                    es.append(e.div_(s_r))
                    sr.append(s_r)
            if k < iterations:
                plan.iterate(1, stream=stream)
        del b, x, xs
    return _finish_pairs(rs, es, sr, se)


def train(net, inputs, targets, steps=1000, batch=4, crop=64, lr=1e-3, lr_final=1e-4, seed=7, log_every=50,
          margin=None, per_crop_scale=True, stream=None):
    """Adam on random crops of the training pairs, scored on each crop's
    interior (margin: default crop // 4, the part of the network's receptive
    field that would otherwise see the crop's zero surroundings).  With
    per_crop_scale each crop's input and target are divided by the rms of the
    target: the network has no biases, so N(a r) = a N(r) for a > 0 and the
    scaling leaves the map to learn unchanged, while the loss becomes a
    relative error per crop (the gain of A^-1 differs by orders of magnitude
    between smooth and rough errors).  Returns the loss history [(step, loss)]
    and the wall time."""
    import torch

    rng = np.random.default_rng(seed)
    nz, ny, nx = inputs[0].shape
    cz, cy, cx = min(crop, nz), min(crop, ny), min(crop, nx)
    if margin is None:
        margin = min(cz, cy, cx) // 4
    xb = torch.empty((batch, cz, cy, cx), device="cuda", dtype=torch.float32)
    tb = torch.empty_like(xb)
    hist = []
    t0 = time.perf_counter()
    for s in range(steps):
        for b in range(batch):
            i = int(rng.integers(len(inputs)))
            z0 = int(rng.integers(0, nz - cz + 1)) & ~3 if nz > cz else 0
            y0 = int(rng.integers(0, ny - cy + 1)) & ~3 if ny > cy else 0
            x0 = int(rng.integers(0, nx - cx + 1)) & ~3 if nx > cx else 0
            xb[b].copy_(inputs[i][z0:z0 + cz, y0:y0 + cy, x0:x0 + cx])
            tb[b].copy_(targets[i][z0:z0 + cz, y0:y0 + cy, x0:x0 + cx])
        if per_crop_scale:
            sc = tb.pow(2).mean(dim=(1, 2, 3), keepdim=True).sqrt().clamp_min(1e-30)
            xb.div_(sc)
            tb.div_(sc)
        f = s / max(1, steps - 1)
        lr_s = lr * (lr_final / lr) ** f  # geometric decay
        want = (s % log_every == 0) or s == steps - 1
        loss = net.train_step(xb, tb, lr=lr_s, update=True, want_loss=want, margin=margin, stream=stream)
        if want:
            hist.append((s, loss))
    torch.cuda.synchronize()
    return hist, time.perf_counter() - t0


def preconditioner_quality(plan, net, inputs, targets):
    """Residual-space relative error of the network on full-volume pairs,
    ||A N(r) - r|| / ||r|| with N's scale fitted by least squares, next to the
    same figure for the best scaled identity (plain CG's preconditioner).
    Returns [(network, identity)] per pair."""
    import torch

    out = []
    for r in inputs:
        z = net.forward(r.contiguous(), normalize=True)
        az = torch.empty_like(r)
        ar = torch.empty_like(r)
        plan.apply_operator(z, az)
        plan.apply_operator(r.contiguous(), ar)
        q = []
        for a in (az, ar):
            g = float((a * r).sum() / (a * a).sum().clamp_min(1e-30))
            q.append(float((g * a - r).pow(2).sum().sqrt() / r.pow(2).sum().sqrt()))
        out.append(tuple(q))
    return out

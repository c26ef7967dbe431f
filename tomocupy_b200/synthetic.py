"""Seeded synthetic tomography data (the reference measures on APS datasets
that are not available here; these inputs have the same shapes, dtypes and
value ranges).

Model: random 3D ellipsoids (analytic parallel-beam line integrals of each
row's elliptical cross-section), Beer-Lambert attenuation of a flat field
1e4*(1+0.02*smooth noise), Poisson photon noise, additive dark current
N(100, 5), optional column gain errors ("stripes", which cause rings), all
clipped to uint16.  Generation runs in torch on any device, in row blocks.
"""
from __future__ import annotations

import math

import numpy as np
import torch


def ellipsoids(count: int, n: int, nz: int, density_max: float, seed: int) -> np.ndarray:
    """[count, 8]: cx, cy, cz, a, b, c, alpha, rho (pixel units, rho per pixel)."""
    rng = np.random.default_rng(seed)
    out = np.empty((count, 8))
    r = n / 2
    for k in range(count):
        rad = 0.7 * r * math.sqrt(rng.uniform())
        ang = rng.uniform(0, 2 * math.pi)
        cx, cy = rad * math.cos(ang), rad * math.sin(ang)
        lim = max(4.0, r - math.hypot(cx, cy))
        a = rng.uniform(0.05, 0.5) * lim + 2
        b = rng.uniform(0.05, 0.5) * lim + 2
        cz = rng.uniform(0, nz)
        c = rng.uniform(0.5, 2.0) * max(nz, 8)
        out[k] = (cx, cy, cz, a, b, c, rng.uniform(0, math.pi), rng.uniform(0, density_max))
    return out


def line_integrals(ell: np.ndarray, theta: torch.Tensor, n: int, rows: torch.Tensor,
                   center: float) -> torch.Tensor:
    """Analytic projections [nrows, nproj, n] (float64) of the ellipsoid cross-sections."""
    dev = theta.device
    th = theta.to(torch.float64)[None, :, None]
    s = (torch.arange(n, dtype=torch.float64, device=dev) + 0.5 - center)[None, None, :]
    z = rows.to(torch.float64)[:, None, None] + 0.5
    out = torch.zeros((rows.numel(), theta.numel(), n), dtype=torch.float64, device=dev)
    for cx, cy, cz, a, b, c, al, rho in ell:
        k2 = 1 - ((z - cz) / c) ** 2
        k = torch.sqrt(torch.clamp(k2, min=0.0))
        ak, bk = a * k, b * k
        r2 = (ak * torch.cos(th - al)) ** 2 + (bk * torch.sin(th - al)) ** 2
        s0 = cx * torch.cos(th) + cy * torch.sin(th)
        d2 = r2 - (s - s0) ** 2
        val = 2 * rho * ak * bk * torch.sqrt(torch.clamp(d2, min=0.0)) / torch.clamp(r2, min=1e-30)
        out += torch.where(d2 > 0, val, torch.zeros((), dtype=torch.float64, device=dev))
    return out


def smooth_field(nz: int, n: int, sigma: float, gen: torch.Generator, device) -> torch.Tensor:
    """Unit-variance Gaussian-blurred noise [nz, n] (blur along both axes)."""
    f = torch.randn((nz, n), generator=gen, device=device, dtype=torch.float32)
    rad = int(3 * sigma)
    x = torch.arange(-rad, rad + 1, device=device, dtype=torch.float32)
    k = torch.exp(-0.5 * (x / sigma) ** 2)
    k = (k / k.sum())[None, None, :]
    g = torch.nn.functional.conv1d(f[:, None, :], k, padding=rad)[:, 0]
    if nz > 1:
        g = torch.nn.functional.conv1d(g.t()[:, None, :], k, padding=rad)[:, 0].t()
    g = g - g.mean()
    return g / (g.std() + 1e-12)


def make_dataset(nproj: int, nz: int, n: int, *, seed: int = 0, n_ell: int = 20,
                 density_max: float = 0.02, photons: float = 1e4, ndark: int = 10,
                 nflat: int = 10, stripes: int = 0, stripe_gain: float = 0.03,
                 theta: np.ndarray | None = None, device="cpu", block: int = 64,
                 center: float | None = None):
    """Return (data uint16 [nproj, nz, n], dark uint16 [ndark, nz, n],
    flat uint16 [nflat, nz, n], theta float32 [nproj], ellipsoid table)."""
    dev = torch.device(device)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    if theta is None:
        theta = (np.arange(nproj) * np.pi / nproj).astype(np.float32)
    th = torch.as_tensor(theta, dtype=torch.float32, device=dev)
    center = n / 2 if center is None else center
    ell = ellipsoids(n_ell, n, nz, density_max, seed + 1)
    gain = 1 + 0.02 * smooth_field(nz, n, 16.0, gen, dev)  # [nz, n]
    col_gain = torch.ones(n, dtype=torch.float32, device=dev)
    if stripes:
        rng = np.random.default_rng(seed + 2)
        cols = rng.choice(n, size=stripes, replace=False)
        g = 1 + rng.uniform(-stripe_gain, stripe_gain, size=stripes)
        col_gain[torch.as_tensor(cols, device=dev)] = torch.as_tensor(g, dtype=torch.float32,
                                                                      device=dev)
    dark = (100 + 5 * torch.randn((ndark, nz, n), generator=gen, device=dev)).round()
    dark = dark.clamp(0, 65535).to(torch.int32).to(torch.uint16) if hasattr(torch, "uint16") \
        else dark
    flat_mean = photons * gain
    flat = torch.poisson(flat_mean[None].expand(nflat, nz, n).contiguous(), generator=gen)
    flat = flat + 100 + 5 * torch.randn((nflat, nz, n), generator=gen, device=dev)
    flat = flat.round().clamp(0, 65535).to(torch.int32).to(torch.uint16)
    data = torch.empty((nproj, nz, n), dtype=torch.uint16, device=dev)
    for z0 in range(0, nz, block):
        z1 = min(nz, z0 + block)
        rows = torch.arange(z0, z1, device=dev)
        p = line_integrals(ell, th, n, rows, center)  # [rows, P, n] float64
        lam = (flat_mean[z0:z1, None, :] * col_gain) * torch.exp(-p).to(torch.float32)
        cnt = torch.poisson(lam, generator=gen)
        cnt = cnt + 100 + 5 * torch.randn(cnt.shape, generator=gen, device=dev)
        data[:, z0:z1] = cnt.round().clamp(0, 65535).to(torch.int32).to(torch.uint16).permute(
            1, 0, 2)
    return data, dark, flat, theta, ell

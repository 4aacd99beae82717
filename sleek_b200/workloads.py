"""Seeded synthetic inputs with the shapes and value distributions of SLEEK's
benchmark inputs (the SDRBench fields the reference's scripts download are not
available offline).

Seeds follow ``seed = 20261203 + 1000 * config + variant`` with numpy
``default_rng`` for every random parameter, so a field is a pure function of
(config, variant, shape).  Fields are evaluated with torch on the requested
device (the large ones on the GPU), always in float64 and then rounded to the
target dtype, so CPU and GPU evaluation give the same values up to the last
float64 bit of the sinusoids; tests that need exact cross-machine agreement use
the committed golden fixtures instead of regenerating.

  c0   f32 1-D, 4 sinusoids (amplitude 1e3) + N(0,1e-3), 0.1 % NaN/+inf/-inf/denormal
  c1   f64 3-D turbulence-like field: 64 Fourier modes, A ~ |k|^(-5/3), + gradient
  c2a  f32 2-D lat/lon field (spherical-harmonic-like sinusoids) + 1 % N(0, 0.01)
  c2b  f32 3-D lognormal density exp(1.5 g), g a k^-3 Gaussian random field
  c2c  f32 1-D particle coordinates U[0,256), sorted in blocks of 4096
"""
from __future__ import annotations

import math

import numpy as np
import torch

BASE_SEED = 20261203


def seed_of(config: int, variant: int = 0) -> int:
    return BASE_SEED + 1000 * config + variant


def _rng(config, variant):
    return np.random.default_rng(seed_of(config, variant))


def c0_signal(n: int = 1 << 24, variant: int = 0, device="cpu", dtype=torch.float32) -> torch.Tensor:
    """Sum of 4 sinusoids + small noise, with 0.1 % special values."""
    rng = _rng(0, variant)
    f = 10 ** rng.uniform(-5, -2, 4)
    ph = rng.uniform(0, 2 * math.pi, 4)
    i = torch.arange(n, device=device, dtype=torch.float64)
    x = torch.zeros(n, device=device, dtype=torch.float64)
    for k in range(4):
        x += 1e3 * torch.sin(2 * math.pi * float(f[k]) * i + float(ph[k]))
    noise = torch.from_numpy(rng.normal(0.0, 1e-3, n)).to(device)
    x = (x + noise).to(dtype)
    nsp = max(1, n // 1000)
    idx = torch.from_numpy(rng.choice(n, nsp, replace=False)).to(device)
    tiny = 3e-41 if dtype == torch.float32 else 5e-320
    sp = torch.tensor([float("nan"), float("inf"), float("-inf"), tiny], dtype=dtype, device=device)
    x[idx] = sp[torch.arange(nsp, device=device) % 4]
    return x


def c1_turbulence(shape=(256, 384, 384), variant: int = 0, device="cpu", dtype=torch.float64) -> torch.Tensor:
    """64 random integer-wavevector Fourier modes with A ~ |k|^(-5/3), unit std, + 0.1 x/256."""
    rng = _rng(1, variant)
    nz, ny, nx = shape
    ks = []
    while len(ks) < 64:
        k = rng.integers(-64, 65, 3)
        m = float(np.sqrt((k * k).sum()))
        if 1 <= m <= 64:
            ks.append(k)
    ks = np.array(ks)
    amp = np.sqrt((ks * ks).sum(1)) ** (-5.0 / 3.0)
    amp = amp / np.sqrt(0.5 * (amp * amp).sum())  # unit std of the sum of cosines
    ph = rng.uniform(0, 2 * math.pi, 64)
    z = torch.arange(nz, device=device, dtype=torch.float64) * (2 * math.pi / nz)
    y = torch.arange(ny, device=device, dtype=torch.float64) * (2 * math.pi / ny)
    xx = torch.arange(nx, device=device, dtype=torch.float64) * (2 * math.pi / nx)
    out = torch.zeros(shape, device=device, dtype=torch.float64)
    for m in range(64):
        kz, ky, kx = (float(v) for v in ks[m])
        ez = torch.polar(torch.ones_like(z), kz * z + float(ph[m]))
        ey = torch.polar(torch.ones_like(y), ky * y)
        ex = torch.polar(torch.ones_like(xx), kx * xx)
        out += float(amp[m]) * (ez[:, None, None] * ey[None, :, None] * ex[None, None, :]).real
    grad = 0.1 * torch.arange(nx, device=device, dtype=torch.float64) / 256.0
    out += grad[None, None, :]
    return out.to(dtype).reshape(-1)


def c2a_latlon(shape=(1800, 3600), variant: int = 0, device="cpu", dtype=torch.float32) -> torch.Tensor:
    """Smooth lat/lon field: sum over l, m <= 8 of a_lm sin(l lat + phi) cos(m lon + psi), + 1 % noise."""
    rng = _rng(2, variant)
    nlat, nlon = shape
    lat = torch.linspace(-math.pi / 2, math.pi / 2, nlat, device=device, dtype=torch.float64)
    lon = torch.linspace(0, 2 * math.pi, nlon + 1, device=device, dtype=torch.float64)[:-1]
    out = torch.zeros(shape, device=device, dtype=torch.float64)
    for l in range(9):
        for m in range(9):
            a = float(rng.normal(0, 1.0 / (1 + l + m)))
            p1, p2 = (float(v) for v in rng.uniform(0, 2 * math.pi, 2))
            out += a * torch.sin(l * lat + p1)[:, None] * torch.cos(m * lon + p2)[None, :]
    n = nlat * nlon
    idx = torch.from_numpy(rng.choice(n, n // 100, replace=False)).to(device)
    noise = torch.from_numpy(rng.normal(0, 0.01, n // 100)).to(device)
    flat = out.reshape(-1)
    flat[idx] += noise
    return flat.to(dtype)


def c2b_lognormal(shape=(512, 512, 512), variant: int = 0, device="cpu", dtype=torch.float32) -> torch.Tensor:
    """exp(1.5 g) with g a unit-variance Gaussian random field of spectrum P(k) ~ k^-3."""
    gen = torch.Generator(device=device).manual_seed(seed_of(2, 100 + variant))
    nz, ny, nx = shape
    w = torch.randn(shape, generator=gen, device=device, dtype=torch.float32)
    fw = torch.fft.rfftn(w)
    kz = torch.fft.fftfreq(nz, device=device)[:, None, None]
    ky = torch.fft.fftfreq(ny, device=device)[None, :, None]
    kx = torch.fft.rfftfreq(nx, device=device)[None, None, :]
    k = torch.sqrt(kz * kz + ky * ky + kx * kx)
    k[0, 0, 0] = 1.0
    fw *= k ** -1.5  # amplitude ~ sqrt(P(k))
    fw[0, 0, 0] = 0
    del k
    g = torch.fft.irfftn(fw, s=shape)
    del fw
    g = (g - g.mean()) / g.std()
    return torch.exp(1.5 * g).to(dtype).reshape(-1)


def c2c_particles(n: int = 1 << 28, variant: int = 0, device="cpu", dtype=torch.float32) -> torch.Tensor:
    """Uniform coordinates in [0, 256), each consecutive block of 4096 sorted ascending."""
    gen = torch.Generator(device=device).manual_seed(seed_of(2, 200 + variant))
    x = torch.rand(n, generator=gen, device=device, dtype=torch.float32) * 256.0
    nb = n // 4096
    if nb:
        head = x[: nb * 4096].view(nb, 4096).sort(dim=1).values.reshape(-1)
        x = torch.cat([head, x[nb * 4096:].sort().values])
    else:
        x = x.sort().values
    return x.to(dtype)


def scaled(config: str, nbytes: int, device="cpu", dtype=None, variant: int = 0) -> torch.Tensor:
    """A field of the given config family with about `nbytes` of data (for tests
    and batched / served workloads, where the sizes vary)."""
    if config == "c0":
        dt = dtype or torch.float32
        n = max(1, nbytes // (torch.finfo(dt).bits // 8))
        return c0_signal(n, variant, device, dt)
    if config == "c1":
        dt = dtype or torch.float64
        n = max(1, nbytes // (torch.finfo(dt).bits // 8))
        side = max(1, int(round(n ** (1 / 3))))
        f = c1_turbulence((side, side, side), variant, device, dt)
        return _fit(f, n)
    if config == "c2":
        dt = dtype or torch.float32
        n = max(1, nbytes // (torch.finfo(dt).bits // 8))
        nlat = max(1, int(math.sqrt(n / 2)))
        f = c2a_latlon((nlat, max(1, 2 * nlat)), variant, device, dt)
        return _fit(f, n)
    raise ValueError(config)


def _fit(f: torch.Tensor, n: int) -> torch.Tensor:
    if f.numel() >= n:
        return f[:n].contiguous()
    reps = (n + f.numel() - 1) // f.numel()
    return f.repeat(reps)[:n].contiguous()


def batched_arrays(n: int = 1000, variant: int = 0, device="cpu", min_bytes: int = 4096,
                   max_bytes: int = 64 << 20):
    """The batched workload: n arrays with sizes log-uniform in [min_bytes, max_bytes]
    (rounded down to the element size), float32 / float64 by a fair coin, generators
    c0 / c1 / c2 in turn; even-index arrays lossless, odd ones lossy with bounds
    log-uniform in [1e-6, 1e-1].  Returns (arrays, error_bounds)."""
    rng = np.random.default_rng(seed_of(3, variant))
    arrays, ebs = [], []
    fams = ("c0", "c1", "c2")
    for i in range(n):
        nbytes = int(np.exp(rng.uniform(np.log(min_bytes), np.log(max_bytes))))
        dt = torch.float32 if rng.random() < 0.5 else torch.float64
        x = scaled(fams[i % 3], nbytes, device=device, dtype=dt, variant=i)
        arrays.append(x)
        ebs.append(None if i % 2 == 0 else float(10 ** rng.uniform(-6, -1)))
    return arrays, ebs

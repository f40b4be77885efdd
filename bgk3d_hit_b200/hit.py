"""Seeded initial velocity fields for decaying homogeneous isotropic turbulence.

The reference only has the Taylor-Green initial condition (SRC/init.F90:83-141);
this generator is new. It produces a random-phase, solenoidal velocity field
with the shell spectrum E(k) ~ k^4 exp(-2 (k/k0)^2), rescaled so that the
per-component rms velocity sqrt(<|u|^2>/3) equals u_rms:

1. three white-noise fields from numpy ``default_rng(seed)`` (standard normal),
2. real-to-complex FFT; every mode is normalised to unit modulus (random phase)
   and multiplied by the amplitude sqrt(E(k) / (4 pi k^2)) ~ k exp(-(k/k0)^2),
3. projection onto the plane perpendicular to k (divergence free); the k = 0
   mode and the Nyquist planes of even extents (where i*k has no real
   counterpart) are removed,
4. inverse FFT and rescaling to u_rms.

Arrays are (nz, ny, nx) in C order, i.e. Fortran order with i fastest, the
layout the C-ABI expects. ``hit_velocity`` is set-up code (host, FP64); its
field is handed to ``bgk_init_velocity``. ``hit_velocity_device`` runs steps
2-4 on the GPU (torch.fft, FP64) and leaves the field there for
``bgk_init_velocity_device``: fed numpy's noise it gives the host field to
rounding (the FFT libraries differ); above 512^3 cells it draws the noise on
the GPU too (torch's generator seeded with the same seed: a field with the
same statistics, not the same realisation), since numpy's noise alone would
take minutes and three host arrays of 8 GB at 1024^3.
"""
from __future__ import annotations

import numpy as np

try:  # threaded pocketfft
    import scipy.fft as _fft

    def _rfftn(a):
        return _fft.rfftn(a, workers=-1)

    def _irfftn(a, s):
        return _fft.irfftn(a, s=s, workers=-1)
except Exception:  # pragma: no cover
    def _rfftn(a):
        return np.fft.rfftn(a)

    def _irfftn(a, s):
        return np.fft.irfftn(a, s=s)


def hit_velocity(n: int | tuple, k0: float, u_rms: float, seed: int):
    """Returns (u, v, w), float64 arrays of shape (nz, ny, nx)."""
    nz, ny, nx = (n, n, n) if np.isscalar(n) else tuple(n)
    rng = np.random.default_rng(seed)
    kz = np.fft.fftfreq(nz, 1.0 / nz).reshape(nz, 1, 1)
    ky = np.fft.fftfreq(ny, 1.0 / ny).reshape(1, ny, 1)
    kx = np.fft.rfftfreq(nx, 1.0 / nx).reshape(1, 1, nx // 2 + 1)
    k2 = kx * kx + ky * ky + kz * kz
    kmag = np.sqrt(k2)
    amp = kmag * np.exp(-((kmag / k0) ** 2))
    for kk, nn in ((kx, nx), (ky, ny), (kz, nz)):
        if nn % 2 == 0:
            amp = np.where(np.abs(kk) == nn // 2, 0.0, amp)
    hat = []
    for _ in range(3):
        f = _rfftn(rng.standard_normal((nz, ny, nx)))
        mod = np.abs(f)
        mod[mod == 0] = 1.0
        hat.append(f / mod * amp)
    k2s = np.where(k2 == 0, 1.0, k2)
    div = (kx * hat[0] + ky * hat[1] + kz * hat[2]) / k2s
    hat = [hat[0] - kx * div, hat[1] - ky * div, hat[2] - kz * div]
    for h in hat:
        h[0, 0, 0] = 0.0
    u, v, w = (_irfftn(h, (nz, ny, nx)) for h in hat)
    rms = np.sqrt((np.mean(u * u) + np.mean(v * v) + np.mean(w * w)) / 3.0)
    s = u_rms / rms
    return u * s, v * s, w * s


def divergence_spectral(u, v, w) -> float:
    """Max |div u| of a periodic field, spectral derivative (test helper)."""
    nz, ny, nx = u.shape
    kz = np.fft.fftfreq(nz, 1.0 / nz).reshape(nz, 1, 1)
    ky = np.fft.fftfreq(ny, 1.0 / ny).reshape(1, ny, 1)
    kx = np.fft.rfftfreq(nx, 1.0 / nx).reshape(1, 1, nx // 2 + 1)
    d = 1j * (kx * _rfftn(u) + ky * _rfftn(v) + kz * _rfftn(w))
    return float(np.max(np.abs(_irfftn(d, (nz, ny, nx)))))


NUMPY_NOISE_MAX_CELLS = 512 ** 3


def hit_velocity_device(n: int | tuple, k0: float, u_rms: float, seed: int, device=0, noise: str = "auto"):
    """The generator of ``hit_velocity`` on the GPU. Returns (u, v, w), float64
    torch tensors of shape (nz, ny, nx) on ``device``. noise: "numpy" (the
    host generator's white noise, uploaded), "device" (torch's CUDA generator
    seeded with ``seed``) or "auto" (numpy up to 512^3 cells)."""
    import torch

    nz, ny, nx = (n, n, n) if np.isscalar(n) else tuple(n)
    dev = torch.device("cuda", device) if isinstance(device, int) else torch.device(device)
    if noise == "auto":
        noise = "numpy" if nx * ny * nz <= NUMPY_NOISE_MAX_CELLS else "device"
    if noise == "numpy":
        rng = np.random.default_rng(seed)

        def white():
            return torch.from_numpy(rng.standard_normal((nz, ny, nx))).to(dev)
    elif noise == "device":
        gen = torch.Generator(device=dev)
        gen.manual_seed(seed)

        def white():
            return torch.randn((nz, ny, nx), generator=gen, dtype=torch.float64, device=dev)
    else:
        raise ValueError(noise)
    f64 = dict(dtype=torch.float64, device=dev)
    kz = torch.fft.fftfreq(nz, 1.0 / nz, **f64).reshape(nz, 1, 1)
    ky = torch.fft.fftfreq(ny, 1.0 / ny, **f64).reshape(1, ny, 1)
    kx = torch.fft.rfftfreq(nx, 1.0 / nx, **f64).reshape(1, 1, nx // 2 + 1)
    k2 = kx * kx + ky * ky + kz * kz
    amp = torch.sqrt(k2)
    amp = amp * torch.exp(-((amp / k0) ** 2))
    for kk, nn in ((kx, nx), (ky, ny), (kz, nz)):
        if nn % 2 == 0:
            amp = torch.where(torch.abs(kk) == nn // 2, torch.zeros((), **f64), amp)
    hat = []
    for _ in range(3):
        f = torch.fft.rfftn(white(), dim=(0, 1, 2))
        mod = torch.abs(f)
        mod = torch.where(mod == 0, torch.ones((), **f64), mod)
        f /= mod
        f *= amp
        del mod
        hat.append(f)
    del amp
    k2 = torch.where(k2 == 0, torch.ones((), **f64), k2)
    div = kx * hat[0]
    div += ky * hat[1]
    div += kz * hat[2]
    div /= k2
    del k2
    out = []
    for h, kk in zip(hat, (kx, ky, kz)):
        h -= kk * div
        h[0, 0, 0] = 0.0
    del div
    for i in range(3):
        out.append(torch.fft.irfftn(hat[i], s=(nz, ny, nx), dim=(0, 1, 2)))
        hat[i] = None
    ms = sum(float(torch.mean(x * x)) for x in out)
    s = u_rms / float(np.sqrt(ms / 3.0))
    for x in out:
        x *= s
    return tuple(out)

"""Initial conditions for the benchmark and test workloads (input preparation,
not the stepping path).

random_phase: the seeded random-phase field of the 512^3 workload -- Fourier
modes with |k| <= k_max get unit amplitude and a uniform random phase, the
field is transformed to real space and rescaled to mean density 1.  The
reference's own random_phase (src/ic.f90:190-252) seeds from the clock and
uses an integer-index cut-off; this is the seeded variant the workloads name.

trapped_random_phase: the ensemble workload's initial condition -- a
random-phase field of |k| <= k_max times the Thomas-Fermi profile
sqrt(max(0, 1 - V)) of the harmonic trap V = omega^2 r^2 / 2 on the grid
x_i = -xr + i h (the reference's get_grid, src/ic.f90:32-69).

vortex_line_pade: a straight vortex line along z through the origin,
psi = r R(r) e^{i atan2(y, x)} with the Pade core R of get_rr
(src/ic.f90:888-901).
"""
from __future__ import annotations

import math

import numpy as np


def random_phase(torch, n: int, h: float, kmax: float, seed: int, device, dtype=None):
    """Returns an (n, n, n) complex tensor on `device` (complex64 unless
    dtype is given); phases from torch's Philox generator with `seed`."""
    dtype = dtype or torch.complex64
    L = n * h
    m = torch.fft.fftfreq(n, d=1.0 / n, device=device, dtype=torch.float64)
    k = 2 * math.pi * m / L
    kz, ky, kx = torch.meshgrid(k, k, k, indexing="ij")
    mask = (kx * kx + ky * ky + kz * kz) <= kmax * kmax
    del kx, ky, kz
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    phase = torch.rand((n, n, n), generator=gen, device=device, dtype=torch.float64)
    a = torch.where(mask, torch.exp(2j * math.pi * phase.to(torch.complex128)),
                    torch.zeros((), dtype=torch.complex128, device=device))
    del phase, mask
    psi = torch.fft.ifftn(a)
    del a
    psi = psi / torch.sqrt(torch.mean(psi.abs() ** 2))
    return psi.to(dtype).contiguous()


def trapped_random_phase(torch, n: int, h: float, omega: float, kmax: float, seed: int, device,
                         dtype=None):
    """(n, n, n) complex tensor: random_phase(...) * sqrt(max(0, 1 - V))."""
    psi = random_phase(torch, n, h, kmax, seed, device, torch.complex128)
    xr = (n - 1) * h / 2
    x = -xr + h * torch.arange(n, device=device, dtype=torch.float64)
    r2 = x[None, None, :] ** 2 + x[None, :, None] ** 2 + x[:, None, None] ** 2
    tf = torch.sqrt(torch.clamp(1.0 - 0.5 * omega * omega * r2, min=0.0))
    return (psi * tf).to(dtype or torch.complex64).contiguous()


def vortex_line_pade(x, y, z):
    """numpy (nz, ny, nx) complex128 field of a Pade-core vortex line."""
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    r = np.sqrt(X ** 2 + Y ** 2)
    rr = np.sqrt((0.3437 + 0.0286 * r ** 2) / (1 + 0.3333 * r ** 2 + 0.0286 * r ** 4))
    return r * rr * np.exp(1j * np.arctan2(Y, X))

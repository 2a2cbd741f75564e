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

vortex_ring_xy: a vortex ring in the xy-plane propagating along z, the
reference's vortex_ring with plane 'xy' (src/ic.f90:352-401): the product of
two Pade-core line vortices at the distances d1, d2 from the ring's two
crossings of each meridional half-plane.

pade_pulse_ring: the Pade approximation of a rarefaction pulse / vortex ring
moving along x (src/ic.f90:513-574; the constants are the reference's
published 'ring' and 'pulse' tables).

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


def _rr(r):
    """The Pade core amplitude R(r)/r of get_rr (src/ic.f90:888-901)."""
    return np.sqrt((0.3437 + 0.0286 * r ** 2) / (1.0 + 0.3333 * r ** 2 + 0.0286 * r ** 4))


def vortex_ring_xy(x, y, z, x0, y0, z0, r0, scal=1.0, amp=0.0, mm=0, r1=0.0, kk=0, direction=1.0):
    """(nz, ny, nx) complex128 vortex ring of radius r0 centred at (x0, y0, z0)
    in the xy-plane, with the optional mode-mm disturbance of amplitude amp
    and helical kk / r1 terms of the reference."""
    Z, Y, X = np.meshgrid(np.asarray(z), np.asarray(y), np.asarray(x), indexing="ij")
    theta = np.arctan2(Y - y0, X - x0)
    s = np.sqrt((X - x0) ** 2 + (Y - y0) ** 2) - r1 * np.sin(kk * theta)
    dist = amp * np.cos(mm * theta)
    pp = Z - r1 * np.cos(kk * theta)
    a = scal * (pp - z0)
    b1 = scal * (s + r0 - dist)
    b2 = scal * (s - r0 - dist)
    d1 = np.sqrt(a ** 2 + b1 ** 2)
    d2 = np.sqrt(a ** 2 + b2 ** 2)
    return _rr(d1) * (a + direction * 1j * b1) * _rr(d2) * (a - direction * 1j * b2)


_PADE = {  # a1..a9, U, m (src/ic.f90:563-576)
    "ring": ((-1.1, 0.0170524, 0.0289452, -0.953, -0.0049767, -0.0594346, 0.04, 0.21, 0.00612),
             0.6, 8.97),
    "pulse": ((-0.79792, 0.00388059, 0.00882276, -0.7981, -0.012783, -0.0574092, 0.0399, 0.199,
               0.0058), 0.63, 8.37),
}


def pade_pulse_ring(x, y, z, which, x0, y0, z0, r0):
    """(nz, ny, nx) complex128 Pade rarefaction pulse / ring moving along x."""
    a, U, m = _PADE[which]
    pow_ = 7.0 / 4.0
    Z, Y, X = np.meshgrid(np.asarray(z), np.asarray(y), np.asarray(x), indexing="ij")
    s = np.sqrt((Y - y0) ** 2 + (Z - z0) ** 2)
    one_2u = 1.0 - 2.0 * U ** 2
    x2 = (X - x0) ** 2
    s2 = (s - r0) ** 2
    q = x2 + one_2u * s2
    denom = (1.0 + a[7] * x2 + a[6] * s2 + a[8] * q ** 2) ** pow_
    uu = 1.0 + (a[0] + a[2] * x2 + a[1] * s2 + m * a[8] ** pow_ * U * (2.0 * x2 - one_2u * s2)) * q / denom
    vv = (X - x0) * (a[3] + a[5] * x2 + a[4] * s2 - m * a[8] ** pow_ * q ** 2) / denom
    return uu + 1j * vv


def vortex_line_pade(x, y, z):
    """numpy (nz, ny, nx) complex128 field of a Pade-core vortex line."""
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    r = np.sqrt(X ** 2 + Y ** 2)
    rr = np.sqrt((0.3437 + 0.0286 * r ** 2) / (1 + 0.3333 * r ** 2 + 0.0286 * r ** 4))
    return r * rr * np.exp(1j * np.arctan2(Y, X))


# --------------------------------------------------------------------------
# The initial-condition functions that the reference's ic.in may combine
# (src/ic.f90), as numpy fields (nz, ny, nx) over the grid x, y, z.  They are
# evaluated on the host once per run and loaded with set_state.

def _grid3(x, y, z):
    return np.meshgrid(np.asarray(z, float), np.asarray(y, float), np.asarray(x, float),
                       indexing="ij")


def _line_guard(ll, a1, a2):
    """safe1, safe2 of get_r / get_theta (src/ic.f90:740-757)."""
    eps = np.finfo(float).eps
    safe1 = safe2 = 0.0
    if abs(ll) < eps:
        if abs(a1) >= eps or abs(a2) >= eps:
            raise ValueError("vortex line disturbance wavelength is zero, but amplitude is "
                             "non-zero")
        safe1 = safe2 = 1.0
    return safe1, safe2


def _line_axes(X, Y, Z, vl, scal):
    """The two displaced transverse coordinates of get_r / get_theta
    (src/ic.f90:730-886): for dir 'z' (x - x0 - a1 sin, y - y0 - a2 cos) of
    2 pi (z - z0) / ll, and the cyclic forms for 'x' and 'y'."""
    s1, s2 = _line_guard(vl["ll"], vl["amp1"], vl["amp2"])
    a1, a2, ll = vl["amp1"], vl["amp2"], vl["ll"]
    x0, y0, z0 = vl["x0"], vl["y0"], vl["z0"]
    d = vl["dir"]
    if d == "x":
        ph1, ph2 = 2.0 * np.pi * (X - x0) / (ll + s1), 2.0 * np.pi * (X - x0) / (ll + s2)
        return Y - y0 - a1 * np.sin(ph1), Z - z0 - a2 * np.cos(ph2)
    if d == "y":
        ph1, ph2 = 2.0 * np.pi * (Y - y0) / (ll + s1), 2.0 * np.pi * (Y - y0) / (ll + s2)
        return Z - z0 - a1 * np.sin(ph1), X - x0 - a2 * np.cos(ph2)
    if d == "z":
        ph1, ph2 = 2.0 * np.pi * (Z - z0) / (ll + s1), 2.0 * np.pi * (Z - z0) / (ll + s2)
        return X - x0 - a1 * np.sin(ph1), Y - y0 - a2 * np.cos(ph2)
    raise ValueError(f"vortex line direction {d!r} is not x, y or z")


def vortex_line(x, y, z, vl: dict, scal: float = 1.0):
    """vortex_line(vl) (src/ic.f90:327-350): exp(i theta), times the core
    amplitude 1 - exp(-0.7 r^1.15) unless vl['imprint_phase'].  vl holds the
    line_param fields x0, y0, z0, amp1, amp2, ll, sgn, dir, imprint_phase."""
    Z, Y, X = _grid3(x, y, z)
    u, v = _line_axes(X, Y, Z, vl, scal)
    theta = vl["sgn"] * np.arctan2(scal * v, scal * u)
    if vl["imprint_phase"]:
        return np.exp(1j * theta)
    # get_r scales the squares, not the coordinates (src/ic.f90:762-788)
    r = np.sqrt(scal * u ** 2 + scal * v ** 2)
    return (1.0 - np.exp(-0.7 * r ** 1.15)) * np.exp(1j * theta)


def vortex_ring(x, y, z, vr: dict, scal: float = 1.0):
    """vortex_ring(vr) (src/ic.f90:352-511) in the plane vr['plane'] ('xy',
    'xz' or 'yz'); vr holds the ring_param fields."""
    Z, Y, X = _grid3(x, y, z)
    plane = vr["plane"]
    # (first in-plane, second in-plane, normal) coordinates and centres
    axes = {"xy": ((X, vr["x0"]), (Y, vr["y0"]), (Z, vr["z0"])),
            "xz": ((X, vr["x0"]), (Z, vr["z0"]), (Y, vr["y0"])),
            "yz": ((Y, vr["y0"]), (Z, vr["z0"]), (X, vr["x0"]))}
    if plane not in axes:
        raise ValueError("Unrecognised vortex ring plane.")
    (p1, c1), (p2, c2), (pn, cn) = axes[plane]
    theta = np.arctan2(p2 - c2, p1 - c1)
    s = np.sqrt((p1 - c1) ** 2 + (p2 - c2) ** 2) - vr["r1"] * np.sin(float(vr["kk"]) * theta)
    dist = vr["amp"] * np.cos(float(vr["mm"]) * theta)
    pp = pn - vr["r1"] * np.cos(float(vr["kk"]) * theta)
    a = scal * (pp - cn)
    b1 = scal * (s + vr["r0"] - dist)
    b2 = scal * (s - vr["r0"] - dist)
    d1 = np.sqrt(a ** 2 + b1 ** 2)
    d2 = np.sqrt(a ** 2 + b2 ** 2)
    return _rr(d1) * (a + vr["dir"] * 1j * b1) * _rr(d2) * (a - vr["dir"] * 1j * b2)


def vtrap(x, y, z, omx, omy, omz):
    """Vtrap (src/ic.f90:708-726)."""
    Z, Y, X = _grid3(x, y, z)
    return 0.5 * ((omx ** 2) * X ** 2 + (omy ** 2) * Y ** 2 + (omz ** 2) * Z ** 2)


def fermi(x, y, z, mu, g, omx, omy, omz):
    """fermi() (src/ic.f90:273-305): sqrt((mu - V)/g) where positive, else 0."""
    f = (mu - vtrap(x, y, z, omx, omy, omz)) / g
    return np.where(f >= 0.0, np.sqrt(np.maximum(f, 0.0)), 0.0).astype(np.complex128)


def vortex_pair(x, y, z):
    """vortex_pair() (src/ic.f90:586-632): the Pade vortex-pair profile in (x, y)."""
    Z, Y, X = _grid3(x, y, z)
    a0, a1, a2 = -1.14026, -0.150112, -0.0294564
    b0, b1, b2 = -0.830953, -0.108296, -0.073641
    c0, c1, c2, c3, c4 = 0.35022, 0.03032, 0.15905, 0.04123, 0.01402
    x2, y2 = X ** 2, Y ** 2
    den = 1.0 + c0 * x2 + c1 * X ** 4 + c2 * y2 + c3 * x2 * y2 + c4 * Y ** 4
    return (1.0 + (a0 + a1 * x2 + a2 * y2) / den) + 1j * (X * (b0 + b1 * x2 + b2 * y2) / den)


def sphere(x, y, z):
    """sphere() (src/ic.f90:635-658): 0.5 (1 + tanh(r - 10 - 2))."""
    Z, Y, X = _grid3(x, y, z)
    return (0.5 * (1.0 + np.tanh(np.sqrt(X ** 2 + Y ** 2 + Z ** 2) - 10.0 - 2.0))).astype(
        np.complex128)


def sphere2(x, y, z):
    """sphere2() (src/ic.f90:661-680): 100 exp(-r^2 / 10)."""
    Z, Y, X = _grid3(x, y, z)
    return (100.0 * np.exp(-(X ** 2 + Y ** 2 + Z ** 2) / 10.0)).astype(np.complex128)


def wall(x, y, z):
    """wall() (src/ic.f90:683-705): 0 for z <= -30, else 1."""
    Z, Y, X = _grid3(x, y, z)
    return np.where(Z <= -30.0, 0.0, 1.0).astype(np.complex128)

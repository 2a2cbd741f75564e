"""CPU restatement (pure Python loops over numpy arrays) of the reference's
random_phase (src/ic.f90:190-269), condensed_particles (src/io.f90:315-404)
and spectrum (src/io.f90:632-725), for small grids.

TEST INFRASTRUCTURE ONLY: the checker for the library's spectral entry
points.  Follows the reference's loops literally (index magnitude rule,
shell test, F accumulation); the FFT is numpy's, with the reference's sign
convention and 1/sqrt(N) normalisation (its FFTW2 call,
src/ic.f90:905-1000).  The reference's unpack of FFTW's transposed output
(src/ic.f90:966-972) indexes the y-slab with ny where nz belongs, so its
transform is the 3-D DFT only for ny = nz; this restatement (and the
library) is the 3-D DFT for every shape.

Parity unpinned: the reference's transforms need FFTW 2 with MPI, which is
not in this image, so no reference outputs of these routines exist here.
spectrum_fast and condensed_fast are vectorised forms for large grids,
checked against the loops on small ones.
"""
from __future__ import annotations

import math

import numpy as np


def _k2(i, n1):
    return i * i if i <= n1 // 2 + 1 else (n1 - i + 1) ** 2


def splitmix_phases(seed, n):
    """Phases of the library's random_phase: SplitMix64 (Steele, Lea and
    Flood, OOPSLA 2014) finaliser of seed + (q+1) * 0x9E3779B97F4A7C15 for
    dense index q, top 53 bits times 2^-53."""
    with np.errstate(over="ignore"):
        q = np.arange(1, n + 1, dtype=np.uint64)
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + q * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * 2.0 ** -53


def random_phase(nx, ny, nz, nv, enerv, phases):
    ev = ((0.5 * nx / math.pi) ** 2) * enerv
    comp_amp = math.sqrt((0.11095279993106999 * nv ** 2.5 * (nx * ny * nz)) / ev ** 1.5)
    kc2 = (1.666666666666666 * ev) / nv
    a = np.zeros((nz, ny, nx), complex)
    for k in range(nz):
        kk2 = _k2(k, nz - 1)
        for j in range(ny):
            jj2 = _k2(j, ny - 1)
            for i in range(nx):
                ii2 = _k2(i, nx - 1)
                if ii2 + jj2 + kk2 <= kc2:
                    a[k, j, i] = comp_amp * np.exp(2j * math.pi * phases[k, j, i])
    return np.fft.fftn(a) / math.sqrt(nx * ny * nz)


def filtered(psi, filter_kc, m=1.0):
    """filtered_surface (src/io.f90:533-628): a = backward transform of psi,
    a *= max(1 - m k2 / filter_kc^2, 0), forward transform."""
    nz, ny, nx = psi.shape
    N = nx * ny * nz
    a = np.fft.ifftn(psi) * N / math.sqrt(N)
    for k in range(nz):
        kk2 = _k2(k, nz - 1)
        for j in range(ny):
            jj2 = _k2(j, ny - 1)
            for i in range(nx):
                k2 = _k2(i, nx - 1) + jj2 + kk2
                a[k, j, i] *= max(1.0 - (m * k2 / filter_kc ** 2), 0.0)
    return np.fft.fftn(a) / math.sqrt(N)


def spectrum(a):
    nz, ny, nx = a.shape
    eta = np.zeros(7)
    nharm = np.zeros(7, int)
    F = np.zeros(nx // 2)
    for k in range(nz):
        kk2 = _k2(k, nz - 1)
        for j in range(ny):
            jj2 = _k2(j, ny - 1)
            for i in range(nx):
                k2 = _k2(i, nx - 1) + jj2 + kk2
                if math.sqrt(k2) == 0.0:
                    continue
                p = abs(a[k, j, i]) ** 2
                for kk in range(1, nx // 2 + 1):
                    if math.sqrt(k2) <= kk:
                        F[kk - 1] += p
                log2k = math.log(0.5 * math.sqrt(k2) / math.pi) / math.log(2.0)
                for m in range(1, 8):
                    if abs(log2k) < m and abs(log2k) >= m - 1:
                        eta[m - 1] += p
                        nharm[m - 1] += 1
                        break
    for m in range(7):
        if eta[m] != 0.0:
            eta[m] /= nharm[m]
    return eta, nharm, F


def condensed_particles(psi, xr, yr, zr):
    nz, ny, nx = psi.shape
    dx, dy, dz = 2 * xr / (nx - 1), 2 * yr / (ny - 1), 2 * zr / (nz - 1)
    V = nx * ny * nz
    # FFTW's backward transform is unnormalised (numpy's ifftn times N); the
    # reference divides by sqrt(N)
    a = np.fft.ifftn(psi) * V / math.sqrt(V)
    n0 = abs(a[0, 0, 0]) ** 2
    M = float(np.sum(np.abs(psi) ** 2)) * dx * dy * dz
    rho0 = n0 / V
    kc = math.pi
    dk = 2.0 * kc / (nx - 1)
    tot = 0.0
    for k in range(nz):
        kz = -kc + k * dk
        for j in range(ny):
            ky = -kc + j * dk
            for i in range(nx):
                kx = -kc + i * dk
                k2 = -(1.0 / 12.0) * (
                    ((-2.0 * math.cos(2.0 * kx * dx) + 32.0 * math.cos(kx * dx) - 30.0) / dx ** 2) +
                    ((-2.0 * math.cos(2.0 * ky * dy) + 32.0 * math.cos(ky * dy) - 30.0) / dy ** 2) +
                    ((-2.0 * math.cos(2.0 * kz * dz) + 32.0 * math.cos(kz * dz) - 30.0) / dz ** 2))
                if k2 == 0.0:
                    continue
                tot += (k2 + rho0) / (k2 * k2 + 2.0 * rho0 * k2)
    temp = (M - n0) / tot
    E0 = (1.0 / (2 * V)) * (M ** 2 + (M - n0) ** 2)
    H = E0 + temp * (V - 1)
    temp2 = ((M / (8.0 * xr * yr * zr)) - (n0 / V)) / tot
    return {"M_density": M / (8.0 * xr * yr * zr), "n0_over_V": n0 / V, "M": M, "n0": n0,
            "temp": temp, "temp2": temp2, "H_over_V": H / V}, a


def k2_grid(nx, ny, nz):
    kx = np.array([_k2(i, nx - 1) for i in range(nx)], np.int64)
    ky = np.array([_k2(j, ny - 1) for j in range(ny)], np.int64)
    kz = np.array([_k2(k, nz - 1) for k in range(nz)], np.int64)
    return kz[:, None, None] + ky[None, :, None] + kx[None, None, :]


def random_phase_fast(nx, ny, nz, nv, enerv, phases):
    ev = ((0.5 * nx / math.pi) ** 2) * enerv
    comp_amp = math.sqrt((0.11095279993106999 * nv ** 2.5 * (nx * ny * nz)) / ev ** 1.5)
    kc2 = (1.666666666666666 * ev) / nv
    a = np.where(k2_grid(nx, ny, nz) <= kc2, comp_amp * np.exp(2j * math.pi * phases), 0.0)
    return np.fft.fftn(a) / math.sqrt(nx * ny * nz)


def spectrum_fast(a):
    nz, ny, nx = a.shape
    k2 = k2_grid(nx, ny, nz).ravel()
    p = (np.abs(a) ** 2).ravel()
    sel = k2 > 0
    k2, p = k2[sel], p[sel]
    kmag = np.sqrt(k2.astype(np.float64))
    # sqrt(k2) <= kk first holds at kk = ceil(sqrt(k2)); F is the running sum
    first = np.ceil(kmag).astype(np.int64)
    F = np.cumsum(np.bincount(first, weights=p, minlength=nx // 2 + 1))[1:nx // 2 + 1]
    l2 = np.abs(np.log(0.5 * kmag / math.pi) / math.log(2.0))
    shell = np.floor(l2).astype(np.int64)
    eta = np.zeros(7)
    nharm = np.zeros(7, int)
    for m in range(7):
        s = shell == m
        nharm[m] = int(s.sum())
        eta[m] = p[s].sum() / nharm[m] if p[s].sum() != 0.0 else 0.0
    return eta, nharm, F


def condensed_fast(psi, xr, yr, zr):
    nz, ny, nx = psi.shape
    dx, dy, dz = 2 * xr / (nx - 1), 2 * yr / (ny - 1), 2 * zr / (nz - 1)
    V = nx * ny * nz
    a = np.fft.ifftn(psi) * V / math.sqrt(V)
    n0 = abs(a[0, 0, 0]) ** 2
    M = float(np.sum(np.abs(psi) ** 2)) * dx * dy * dz
    rho0 = n0 / V
    kc = math.pi
    dk = 2.0 * kc / (nx - 1)

    def axis(n, h):
        k = -kc + np.arange(n) * dk
        return (-2.0 * np.cos(2.0 * k * h) + 32.0 * np.cos(k * h) - 30.0) / h ** 2

    k2 = -(1.0 / 12.0) * ((axis(nx, dx)[None, None, :] + axis(ny, dy)[None, :, None])
                          + axis(nz, dz)[:, None, None])
    k2 = k2[k2 != 0.0]
    tot = float(np.sum((k2 + rho0) / (k2 * k2 + 2.0 * rho0 * k2)))
    temp = (M - n0) / tot
    E0 = (1.0 / (2 * V)) * (M ** 2 + (M - n0) ** 2)
    H = E0 + temp * (V - 1)
    temp2 = ((M / (8.0 * xr * yr * zr)) - (n0 / V)) / tot
    return {"M_density": M / (8.0 * xr * yr * zr), "n0_over_V": n0 / V, "M": M, "n0": n0,
            "temp": temp, "temp2": temp2, "H_over_V": H / V}, a

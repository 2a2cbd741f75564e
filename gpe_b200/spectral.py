"""Spectral initial condition and diagnostics of a resident state, through
the C-ABI (gpe_gpu_random_phase, gpe_gpu_condensed_particles,
gpe_gpu_filtered_field: cuFFT plus the library's own reduction kernels).

random_phase: ics' random_phase (src/ic.f90:190-252) with get_kc_amp
(:256-269).  condensed_particles: src/io.f90:315-404 with spectrum
(:632-725).  filtered_field: the field of filtered_surface
(src/io.f90:533-628).  File writers for their outputs are in
gpe_b200.output.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from ._lib import check, device_field, lib, torch_ready

NSHELLS = 7
MASS_COLUMNS = ("M_density", "n0_over_V", "M", "n0", "temp", "temp2", "H_over_V")


@dataclass
class Condensate:
    """One condensed_particles call: the mass.dat columns 3-9 (row), the
    shell mean occupation numbers and mode counts, and F(kk), kk = 1..nx/2."""
    row: dict
    eta: np.ndarray
    nharm: np.ndarray
    F: np.ndarray


def kc_amp(nx: int, ny: int, nz: int, nv: float, enerv: float):
    """get_kc_amp (src/ic.f90:256-269) -> (comp_amp, kc2)."""
    ek = 0.5 * nx / np.pi
    ev = (ek * ek) * enerv
    comp_amp = np.sqrt((0.11095279993106999 * nv ** 2.5) * float(nx * ny * nz) / ev ** 1.5)
    kc2 = (1.666666666666666 * ev) / nv
    return float(comp_amp), float(kc2)


def random_phase(solver, nv: float, enerv: float, seed: int = 0):
    """Load the random-phase state into the solver; returns (comp_amp, kc2)."""
    amp, kc2 = ctypes.c_double(), ctypes.c_double()
    check(lib().gpe_gpu_random_phase(solver.handle, float(nv), float(enerv),
                                     int(seed) & 0xFFFFFFFFFFFFFFFF, ctypes.byref(amp),
                                     ctypes.byref(kc2)), solver.handle)
    return amp.value, kc2.value


def condensed_particles(solver) -> Condensate:
    nx = solver.prm.nx
    row = np.zeros(7)
    eta = np.zeros(NSHELLS)
    nharm = np.zeros(NSHELLS, dtype=np.int64)
    F = np.zeros(nx // 2)
    dp = ctypes.POINTER(ctypes.c_double)
    check(lib().gpe_gpu_condensed_particles(
        solver.handle, row.ctypes.data_as(dp), eta.ctypes.data_as(dp),
        nharm.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), F.ctypes.data_as(dp), nx // 2),
        solver.handle)
    return Condensate(dict(zip(MASS_COLUMNS, (float(v) for v in row))), eta, nharm, F)


def filtered_field(solver, filter_kc: float, m: float = 1.0, out=None):
    """The filtered field of filtered_surface.  Returns a host array of the
    field's precision, or fills `out` (a contiguous CUDA torch tensor of that
    precision, shape (nz, ny, nx)) and returns it."""
    eb = 16 if solver.prm.precision == 16 else 8
    if out is not None:
        device_field(out, solver.shape, solver.prm.device, "filtered_field(out=)", elem_bytes=eb)
        torch_ready(out)
        check(lib().gpe_gpu_filtered_field(solver.handle, float(filter_kc), float(m),
                                           ctypes.c_void_p(out.data_ptr()), eb, 1), solver.handle)
        return out
    host = np.empty(solver.shape, dtype=np.complex128 if eb == 16 else np.complex64)
    check(lib().gpe_gpu_filtered_field(solver.handle, float(filter_kc), float(m),
                                       host.ctypes.data_as(ctypes.c_void_p), eb, 0), solver.handle)
    return host

"""CPU oracle for the GPE finite-difference time stepper.

TEST INFRASTRUCTURE ONLY.  Imported by ``tests/``, ``__graft_entry__.smoke()``
and the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` -- as the
checker and the timed CPU baseline, never as the product.  The product package
``gpe_b200`` does not import it.

PARITY UNPINNED: the reference (liangjj/gpe, Fortran 90 + MPI + FFTW2) ships no
golden vectors and cannot be compiled in this image.  ``liboracle.so`` restates
src/solve.f90, src/derivs.f90, src/variables.f90 and src/ic.f90 in C (see
gpe_oracle.c for per-routine citations) and is pinned against analytic
known-answer tests and the numpy restatement in ``ref_numpy.py``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

SCHEMES = {"euler": 0, "rk2": 1, "rk4": 2, "rk45": 3}


class _OraParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("xr", ctypes.c_double), ("yr", ctypes.c_double), ("zr", ctypes.c_double),
        ("scheme", ctypes.c_int), ("eqn_to_solve", ctypes.c_int),
        ("bcs", ctypes.c_int), ("order", ctypes.c_int), ("real_time", ctypes.c_int),
        ("Urhs", ctypes.c_double), ("diss_amp", ctypes.c_double),
        ("scal", ctypes.c_double), ("g", ctypes.c_double), ("mu", ctypes.c_double),
        ("nn", ctypes.c_double), ("omx", ctypes.c_double), ("omy", ctypes.c_double),
        ("omz", ctypes.c_double),
    ]


class OraTime(ctypes.Structure):
    _fields_ = [("t", ctypes.c_double), ("im_t", ctypes.c_double),
                ("dt_re", ctypes.c_double), ("dt_im", ctypes.c_double),
                ("p", ctypes.c_int)]


def build(force: bool = False) -> str:
    """Compile liboracle.so with the committed Makefile (gcc, OpenMP)."""
    if force or not os.path.exists(_LIB_PATH) or (
        os.path.getmtime(_LIB_PATH)
        < max(os.path.getmtime(os.path.join(_HERE, f))
              for f in ("gpe_oracle.c", "gpe_oracle.h", "Makefile"))
    ):
        subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        vp, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
        L.ora_create.restype = vp
        L.ora_create.argtypes = [ctypes.POINTER(_OraParams)]
        L.ora_destroy.argtypes = [vp]
        L.ora_set_threads.argtypes = [ctypes.c_int]
        L.ora_get_threads.restype = ctypes.c_int
        L.ora_grid.argtypes = [vp, dp, dp, dp]
        L.ora_solver.restype = ctypes.c_int
        L.ora_solver.argtypes = [vp, dp, dp, ctypes.POINTER(OraTime), dp,
                                 ctypes.POINTER(ctypes.c_int)]
        L.ora_rhs.argtypes = [vp, dp, dp]
        L.ora_laplacian.argtypes = [vp, dp, dp]
        L.ora_deriv.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp, dp]
        L.ora_get_norm.restype = ctypes.c_double
        L.ora_get_norm.argtypes = [vp, dp]
        L.ora_energy.restype = ctypes.c_double
        L.ora_energy.argtypes = [vp, dp]
        L.ora_hamiltonian4.restype = ctypes.c_double
        L.ora_hamiltonian4.argtypes = [vp, dp]
        L.ora_mass.restype = ctypes.c_double
        L.ora_mass.argtypes = [vp, dp]
        L.ora_momentum.restype = None
        L.ora_momentum.argtypes = [vp, dp, dp]
        L.ora_renormalise.argtypes = [vp, dp, ctypes.c_double]
        L.ora_get_rr.restype = ctypes.c_double
        L.ora_get_rr.argtypes = [ctypes.c_double]
        L.ora_ic_vortex_line.argtypes = [vp] + [ctypes.c_double] * 7 + [
            ctypes.c_char, ctypes.c_int, dp]
        L.ora_ic_vortex_ring.argtypes = [vp, ctypes.c_char_p] + [ctypes.c_double] * 5 + [
            ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double, dp]
        L.ora_ic_pade_pulse_ring.argtypes = [vp, ctypes.c_char_p] + [ctypes.c_double] * 4 + [dp]
        L.ora_ic_fermi.argtypes = [vp, dp]
        L.ora_zeros.restype = ctypes.c_longlong
        L.ora_zeros.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp, dp,
                                ctypes.POINTER(ctypes.c_longlong), dp, ctypes.c_longlong]
        L.ora_linelength.restype = ctypes.c_double
        L.ora_linelength.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_double, dp]
        _lib = L
    return _lib


def set_threads(n: int) -> None:
    lib().ora_set_threads(int(n))


def get_threads() -> int:
    return int(lib().ora_get_threads())


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _c128(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.complex128)


@dataclass
class OracleParams:
    """run_params / eqn_params subset (src/parameters.f90:24-55) + grid."""
    nx: int
    ny: int
    nz: int
    xr: float
    yr: float
    zr: float
    scheme: str = "rk4"
    eqn_to_solve: int = 4
    bcs: int = 1
    order: int = 2
    real_time: bool = True
    Urhs: float = 0.0
    diss_amp: float = 0.0
    scal: float = 1.0
    g: float = 1.0
    mu: float = 1.0
    nn: float = 1.0
    omx: float = 0.0
    omy: float = 0.0
    omz: float = 0.0


class Oracle:
    """One oracle context; arrays are complex128 shaped (nz, ny, nx)."""

    def __init__(self, prm: OracleParams):
        self.prm = prm
        c = _OraParams(prm.nx, prm.ny, prm.nz, prm.xr, prm.yr, prm.zr,
                       SCHEMES[prm.scheme], prm.eqn_to_solve, prm.bcs, prm.order,
                       1 if prm.real_time else 0, prm.Urhs, prm.diss_amp, prm.scal,
                       prm.g, prm.mu, prm.nn, prm.omx, prm.omy, prm.omz)
        self._h = lib().ora_create(ctypes.byref(c))
        self.shape = (prm.nz, prm.ny, prm.nx)

    def close(self):
        if self._h:
            lib().ora_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def grid(self):
        x = np.zeros(self.prm.nx); y = np.zeros(self.prm.ny); z = np.zeros(self.prm.nz)
        lib().ora_grid(self._h, _dp(x), _dp(y), _dp(z))
        return x, y, z

    def solver(self, psi, tm: OraTime):
        """One solver() call; returns (psi_new, errmax, attempts)."""
        a = _c128(psi)
        out = np.empty_like(a)
        em = ctypes.c_double(0.0)
        na = ctypes.c_int(0)
        rc = lib().ora_solver(self._h, _dp(a), _dp(out), ctypes.byref(tm),
                              ctypes.byref(em), ctypes.byref(na))
        if rc != 0:
            raise ValueError("ERROR: Unrecognised time stepping scheme.")
        return out, em.value, na.value

    def rhs(self, psi):
        a = _c128(psi); out = np.empty_like(a)
        lib().ora_rhs(self._h, _dp(a), _dp(out)); return out

    def laplacian(self, psi):
        a = _c128(psi); out = np.empty_like(a)
        lib().ora_laplacian(self._h, _dp(a), _dp(out)); return out

    def deriv(self, psi, axis: int, second: bool):
        a = _c128(psi); out = np.empty_like(a)
        lib().ora_deriv(self._h, axis, 1 if second else 0, _dp(a), _dp(out)); return out

    def mass(self, psi) -> float:
        a = _c128(psi); return float(lib().ora_mass(self._h, _dp(a)))

    def momentum(self, psi):
        a = _c128(psi)
        out = np.zeros(3)
        lib().ora_momentum(self._h, _dp(a), _dp(out))
        return out

    def get_norm(self, psi) -> float:
        a = _c128(psi); return float(lib().ora_get_norm(self._h, _dp(a)))

    def energy(self, psi) -> float:
        a = _c128(psi); return float(lib().ora_energy(self._h, _dp(a)))

    def hamiltonian4(self, psi) -> float:
        a = _c128(psi); return float(lib().ora_hamiltonian4(self._h, _dp(a)))

    def renormalise(self, psi, norm: float):
        a = _c128(psi).copy()
        lib().ora_renormalise(self._h, _dp(a), float(norm)); return a

    # initial conditions (src/ic.f90)
    def ic_vortex_line(self, x0, y0, z0, amp1=0.0, amp2=0.0, ll=0.0, sgn=1.0,
                       direction="z", imprint_phase=False):
        out = np.empty(self.shape, np.complex128)
        lib().ora_ic_vortex_line(self._h, x0, y0, z0, amp1, amp2, ll, sgn,
                                 direction.encode(), 1 if imprint_phase else 0, _dp(out))
        return out

    def ic_vortex_ring(self, plane, x0, y0, z0, r0, amp=0.0, mm=0, r1=0.0, kk=0, dir=1.0):
        out = np.empty(self.shape, np.complex128)
        lib().ora_ic_vortex_ring(self._h, plane.encode(), x0, y0, z0, r0, amp, mm, r1, kk,
                                 dir, _dp(out))
        return out

    def ic_pade_pulse_ring(self, which, x0, y0, z0, r0):
        out = np.empty(self.shape, np.complex128)
        lib().ora_ic_pade_pulse_ring(self._h, which.encode(), x0, y0, z0, r0, _dp(out))
        return out

    def ic_fermi(self):
        out = np.empty(self.shape, np.complex128)
        lib().ora_ic_fermi(self._h, _dp(out)); return out


def get_rr(r: float) -> float:
    return float(lib().ora_get_rr(float(r)))


def drive(orc: Oracle, psi, tm: OraTime, nsteps: int, *, renorm=False,
          stop_imag=False, imprint=None):
    """The per-step bookkeeping of the reference time loop (src/gpe.f90:134-278)
    with an explicit step count: solver, get_norm + relnorm (equation 4),
    imaginary-to-real switch at relnorm < 1e-12, renormalise, and with
    imprint (the vortex_line(vl1) field) psi = |psi| * imprint
    (src/gpe.f90:270, src/variables.f90:1149-1163).  Returns
    (psi, list of (t, im_t, norm, relnorm))."""
    prm = orc.prm
    rec = []
    prev_norm = 1.0
    real_time = prm.real_time
    if prm.eqn_to_solve == 4 and not real_time:
        prev_norm = orc.get_norm(psi)
        if renorm:
            psi = orc.renormalise(psi, prev_norm)
    norm = 0.0
    for _ in range(nsteps):
        psi, _, _ = orc.solver(psi, tm)
        relnorm = 0.0
        if prm.eqn_to_solve == 4:
            norm = orc.get_norm(psi)
            relnorm = abs((norm - prev_norm) / prev_norm)
            rec.append((tm.t, tm.im_t, norm, relnorm))
        if prm.eqn_to_solve == 4 and not real_time:
            if relnorm < 1e-12:
                if stop_imag:
                    break
                real_time = True
                tm.im_t = 0.0
                tm.dt_re, tm.dt_im = abs(tm.dt_im), abs(tm.dt_re)
            if renorm:
                psi = orc.renormalise(psi, norm)
            if imprint is not None:
                psi = np.abs(psi) * imprint
        prev_norm = norm
        tm.p += 1
    return psi, rec


def linelength(psi, dx: float, state=None):
    """linelength (src/variables.f90:879-1145) of a single-domain interior
    psi (nz, ny, nx).  state: the 18 carried-over work values x(1:6),
    y(1:6), z(1:6) (zeros by default); returns (length, final state)."""
    a = _c128(psi)
    nz, ny, nx = a.shape
    st = np.zeros(18) if state is None else np.array(state, dtype=np.float64)
    L = float(lib().ora_linelength(_dp(a), nx, ny, nz, float(dx), _dp(st)))
    return L, st


def zeros(psi, x, y, z):
    """get_zeros / get_extra_zeros / get_re_im_zeros (src/io.f90:895-1402)
    of a single-domain interior psi on the grid x, y, z -> (counts[12],
    points (n, 3))."""
    a = _c128(psi)
    nz, ny, nx = a.shape
    xs, ys, zs = (np.ascontiguousarray(v, dtype=np.float64) for v in (x, y, z))
    counts = np.zeros(12, dtype=np.int64)
    cp = counts.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))
    n = int(lib().ora_zeros(_dp(a), nx, ny, nz, _dp(xs), _dp(ys), _dp(zs), cp, None, 0))
    pts = np.zeros((max(n, 1), 3))
    lib().ora_zeros(_dp(a), nx, ny, nz, _dp(xs), _dp(ys), _dp(zs), cp, _dp(pts), n)
    return counts, pts[:n]

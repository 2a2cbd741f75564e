"""Checkpoint / restart in the reference's end_state.dat format.

end_state (src/io.f90:840-862) writes, with stream access (no record
markers), in the run's real kind pr (8 or 4 bytes):

    int32 nx, int32 ny, int32 nz, int32 p, real(pr) t, real(pr) im_t,
    complex(pr) dt, complex(pr) psi(0:nx-1, 0:ny-1, 0:nz-1)   (x fastest)

one file per rank (its own z-slab; a single domain writes the whole grid).
state_restart (src/ic.f90:117-186) reads it back, switches the time
direction of dt when the run's real_time flag differs from the saved step,
keeps the saved dt for rkf45 and otherwise rescales p when dt changed.
The same file is the channel for injecting an initial condition into a run.
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np


class RestartError(ValueError):
    """A missing, truncated or mismatched end_state file."""


@dataclass
class EndState:
    nx: int
    ny: int
    nz: int
    p: int
    t: float
    im_t: float
    dt: complex
    psi: np.ndarray  # (nz, ny, nx) complex


def _types(pr_bytes: int):
    if pr_bytes == 8:
        return np.dtype("<f8"), np.dtype("<c16")
    if pr_bytes == 4:
        return np.dtype("<f4"), np.dtype("<c8")
    raise RestartError(f"pr must be 4 or 8 bytes, not {pr_bytes}")


def file_size(nx: int, ny: int, nz: int, pr_bytes: int) -> int:
    return 4 * 4 + 2 * pr_bytes + 2 * pr_bytes + nx * ny * nz * 2 * pr_bytes


def write_end_state(path: str, psi, p: int, t: float, im_t: float, dt: complex,
                    pr_bytes: int = 8) -> None:
    """Write psi (an (nz, ny, nx) complex array) and the time state."""
    rt, ct = _types(pr_bytes)
    a = np.ascontiguousarray(psi, dtype=ct)
    if a.ndim != 3:
        raise RestartError("psi must be (nz, ny, nx)")
    nz, ny, nx = a.shape
    tmp = path + ".tmp"
    with open(tmp, "wb") as f:
        f.write(np.array([nx, ny, nz, p], dtype="<i4").tobytes())
        f.write(np.array([t, im_t], dtype=rt).tobytes())
        f.write(np.array([dt], dtype=ct).tobytes())
        f.write(a.tobytes())
    os.replace(tmp, path)


def read_end_state(path: str, pr_bytes: int = 8, expect=None) -> EndState:
    """Read an end_state file; `expect` = (nx, ny, nz) checks the grid.
    Raises RestartError for a missing, truncated or mismatched file (the
    reference stops with emergency_stop, src/ic.f90:97-101)."""
    rt, ct = _types(pr_bytes)
    if not os.path.exists(path):
        raise RestartError(f"restart requested but {path} does not exist")
    size = os.path.getsize(path)
    if size < 16:
        raise RestartError(f"{path}: truncated header ({size} bytes)")
    with open(path, "rb") as f:
        head = np.frombuffer(f.read(16), dtype="<i4")
        nx, ny, nz, p = (int(v) for v in head)
        if min(nx, ny, nz) < 1:
            raise RestartError(f"{path}: bad grid {nx}x{ny}x{nz}")
        if expect is not None and tuple(expect) != (nx, ny, nz):
            raise RestartError(f"{path}: grid {nx}x{ny}x{nz} differs from the run's "
                               f"{expect[0]}x{expect[1]}x{expect[2]}")
        want = file_size(nx, ny, nz, pr_bytes)
        if size != want:
            raise RestartError(f"{path}: {size} bytes, expected {want} for a {nx}x{ny}x{nz} "
                               f"grid with {pr_bytes}-byte reals")
        t, im_t = (float(v) for v in np.frombuffer(f.read(2 * rt.itemsize), dtype=rt))
        dt = complex(np.frombuffer(f.read(ct.itemsize), dtype=ct)[0])
        psi = np.frombuffer(f.read(nx * ny * nz * ct.itemsize), dtype=ct).reshape(nz, ny, nx)
    return EndState(nx, ny, nz, p, t, im_t, dt, psi.copy())


def restart_time_state(saved: EndState, real_time: bool, scheme: str, dt: complex):
    """(p, t, im_t, dt) of the restarted run, following state_restart
    (src/ic.f90:160-184): a saved imaginary step becomes real (and im_t is
    reset) when the run is in real time, and the reverse; rkf45 keeps the
    saved dt, other schemes keep their own dt and rescale p."""
    p, t, im_t = saved.p, saved.t, saved.im_t
    dt_prev = saved.dt
    if real_time:
        if dt_prev.real == 0.0:
            dt_prev = complex(-dt_prev.imag, dt_prev.real)
            im_t = 0.0
    else:
        if dt_prev.imag == 0.0:
            dt_prev = complex(dt_prev.imag, -dt_prev.real)
            t = 0.0
    if scheme == "rk45":
        dt = dt_prev
    elif dt_prev != dt:
        # integer p = p * dt_prev / dt with Fortran's truncating conversion
        p = int((p * dt_prev / dt).real)
    return p, t, im_t, dt

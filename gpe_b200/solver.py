"""Host-side mirror of the reference solver module over the C-ABI.

The reference exposes its hot path as Fortran module procedures operating on
module globals (src/solve.f90:21 ``solver``; src/variables.f90 ``get_norm``,
``energy``, ``renormalise``; globals in src/parameters.f90).  ``GpeSolver``
keeps the same names and argument meaning, with the globals held on the
object (``t``, ``im_t``, ``dt``, ``p``) and psi resident on the GPU.

Arrays are the reference's interior layout: complex, x fastest, i.e. numpy
shape (nz, ny, nx) in C order.  Errors raise ``GpeError`` where the
reference would call emergency_stop (src/error.f90:24-46).
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass, fields

import numpy as np

from ._lib import (GpeError, GpeParamsC, GpeStepInfoC, GpeTimeC, GpeTimingC, SCHEMES,
                   TIMING_FAMILIES, check, device_field, lib, torch_ready)


@dataclass
class GpeParams:
    """run_params / eqn_params (src/parameters.f90:24-55) plus the grid and
    storage form.  ``precision`` 16 = complex128, 8 = complex64."""
    nx: int
    ny: int
    nz: int
    xr: float = 1.0
    yr: float = 1.0
    zr: float = 1.0
    scheme: str = "rk4"
    eqn_to_solve: int = 4
    bcs: int = 1
    order: int = 2
    real_time: bool = True
    precision: int = 16
    Urhs: float = 0.0
    diss_amp: float = 0.0
    scal: float = 1.0
    g: float = 1.0
    mu: float = 1.0
    nn: float = 1.0
    omx: float = 0.0
    omy: float = 0.0
    omz: float = 0.0
    kahan: bool = False
    device: int = 0
    tile_y: int = 0
    zchunk: int = 0
    fd_match: float = 0.0  # order 4: Laplacian dispersing like 2nd order at spacing fd_match*h

    def to_c(self) -> GpeParamsC:
        c = GpeParamsC()
        lib().gpe_gpu_default_params(ctypes.byref(c), self.nx, self.ny, self.nz)
        for f in fields(self):
            v = getattr(self, f.name)
            if f.name == "scheme":
                if v not in SCHEMES:
                    # the reference fails only when solver() is called
                    # (src/solve.f90:47-49); keep an invalid code for that
                    v = 99
                else:
                    v = SCHEMES[v]
            elif isinstance(v, bool):
                v = int(v)
            setattr(c, f.name, v)
        return c


def _as_host(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


class GpeSolver:
    """One resident run on one B200 (a ``gpe_ctx``)."""

    def __init__(self, prm: GpeParams, t: float = 0.0, im_t: float = 0.0, p: int = 0,
                 dt: complex | None = None, tau: float | None = None):
        self.prm = prm
        self._ctx = ctypes.c_void_p()
        cp = prm.to_c()
        check(lib().gpe_gpu_create(ctypes.byref(cp), ctypes.byref(self._ctx)), None)
        self.shape = (prm.nz, prm.ny, prm.nx)
        self.t, self.im_t, self.p = float(t), float(im_t), int(p)
        if dt is None:
            # src/gpe.f90:76-80
            tau = 0.0 if tau is None else float(tau)
            dt = complex(tau, 0.0) if prm.real_time else complex(0.0, -tau)
        self.dt = complex(dt)
        self.last_info = None

    # ---- lifetime -------------------------------------------------------
    def close(self) -> None:
        if self._ctx:
            lib().gpe_gpu_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._ctx

    # ---- state ------------------------------------------------------------
    def _elem(self, dtype) -> int:
        return 16 if np.dtype(dtype) == np.complex128 else 8

    def set_state(self, psi) -> None:
        """Load psi (numpy host array or CUDA torch tensor, interior layout)."""
        if hasattr(psi, "is_cuda") and psi.is_cuda:
            t = psi.contiguous()
            eb = device_field(t, self.shape, self.prm.device, "set_state")
            torch_ready(t)
            check(lib().gpe_gpu_set_state_device(self._ctx, ctypes.c_void_p(t.data_ptr()), eb),
                  self._ctx)
            return
        a = np.asarray(psi)
        if a.dtype not in (np.complex64, np.complex128):
            a = a.astype(np.complex128)
        a = np.ascontiguousarray(a)
        if a.shape != self.shape:
            raise GpeError(1, f"state shape {a.shape} != {self.shape}")
        check(lib().gpe_gpu_set_state(self._ctx, a.ctypes.data_as(ctypes.c_void_p),
                                      self._elem(a.dtype)), self._ctx)

    def get_state(self, dtype=np.complex128) -> np.ndarray:
        out = np.empty(self.shape, dtype=dtype)
        check(lib().gpe_gpu_get_state(self._ctx, out.ctypes.data_as(ctypes.c_void_p),
                                      self._elem(dtype)), self._ctx)
        return out

    def get_state_device(self, out) -> None:
        """Copy the state into a contiguous CUDA torch tensor (complex64/128)."""
        eb = device_field(out, self.shape, self.prm.device, "get_state_device")
        torch_ready(out)
        check(lib().gpe_gpu_get_state_device(self._ctx, ctypes.c_void_p(out.data_ptr()), eb),
              self._ctx)

    def get_site(self, i: int, j: int, k: int) -> complex:
        """psi at interior site (i, j, k): the save_time point value."""
        v = np.zeros(2)
        check(lib().gpe_gpu_get_site(self._ctx, int(i), int(j), int(k),
                                     v.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
              self._ctx)
        return complex(v[0], v[1])

    def get_plane(self, k: int, dtype=np.complex128) -> np.ndarray:
        """The z-plane k, (ny, nx): the slice of save_surface."""
        out = np.empty((self.prm.ny, self.prm.nx), dtype=dtype)
        check(lib().gpe_gpu_get_plane(self._ctx, int(k), out.ctypes.data_as(ctypes.c_void_p),
                                      self._elem(dtype)), self._ctx)
        return out

    # ---- the reference's hot-path procedures --------------------------------
    def _tm(self) -> GpeTimeC:
        return GpeTimeC(self.t, self.im_t, self.dt.real, self.dt.imag, self.p, 0)

    def _untm(self, tm: GpeTimeC) -> None:
        self.t, self.im_t, self.p = tm.t, tm.im_t, tm.p
        self.dt = complex(tm.dt_re, tm.dt_im)

    def solver(self) -> GpeStepInfoC:
        """solver(var_in, var_out) (src/solve.f90:25-53) on the resident psi;
        updates t, im_t (and dt for rk45) like the reference."""
        tm = self._tm()
        info = GpeStepInfoC()
        check(lib().gpe_gpu_solver(self._ctx, ctypes.byref(tm), ctypes.byref(info)), self._ctx)
        self._untm(tm)
        self.last_info = info
        return info

    def solver_host(self, var_in: np.ndarray) -> np.ndarray:
        """Literal host-array form: returns var_out for var_in."""
        a = np.ascontiguousarray(var_in)
        out = np.empty_like(a)
        tm = self._tm()
        info = GpeStepInfoC()
        check(lib().gpe_gpu_solver_host(self._ctx, a.ctypes.data_as(ctypes.c_void_p),
                                        out.ctypes.data_as(ctypes.c_void_p),
                                        self._elem(a.dtype), ctypes.byref(tm),
                                        ctypes.byref(info)), self._ctx)
        self._untm(tm)
        self.last_info = info
        return out

    def step_series(self, n: int):
        """(dt taken, attempts) of the first n steps of the last rk45 advance."""
        dts = np.zeros(max(n, 1))
        att = np.zeros(max(n, 1), dtype=np.int32)
        check(lib().gpe_gpu_step_series(self._ctx, int(n),
                                        dts.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                        att.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))),
              self._ctx)
        return dts[:n], att[:n]

    def advance(self, nsteps: int) -> np.ndarray:
        """nsteps solver() calls with the per-step norm (rk45: nsteps accepted
        steps, step control on the device)."""
        norms = np.zeros(max(nsteps, 1), dtype=np.float64)
        tm = self._tm()
        check(lib().gpe_gpu_advance(self._ctx, int(nsteps), ctypes.byref(tm),
                                    norms.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
              self._ctx)
        self._untm(tm)
        return norms[:nsteps]

    def get_norm(self) -> float:
        """get_norm (src/variables.f90:537-559)."""
        v = ctypes.c_double()
        check(lib().gpe_gpu_norm(self._ctx, ctypes.byref(v)), self._ctx)
        return v.value

    def energy(self) -> tuple[float, float]:
        """energy (src/variables.f90:563-587) -> (E, H4)."""
        e, h = ctypes.c_double(), ctypes.c_double()
        check(lib().gpe_gpu_energy(self._ctx, ctypes.byref(e), ctypes.byref(h)), self._ctx)
        return e.value, h.value

    def save_end_state(self, path: str) -> None:
        """Checkpoint in the reference's end_state.dat format (src/io.f90:840-862)."""
        from .restart import write_end_state
        pr = 8 if self.prm.precision == 16 else 4
        write_end_state(path, self.get_state(np.complex128 if pr == 8 else np.complex64),
                        self.p, self.t, self.im_t, self.dt, pr)

    def load_end_state(self, path: str) -> None:
        """Restart from an end_state.dat file (src/ic.f90:117-186)."""
        from .restart import read_end_state, restart_time_state
        pr = 8 if self.prm.precision == 16 else 4
        st = read_end_state(path, pr, expect=(self.prm.nx, self.prm.ny, self.prm.nz))
        sch = self.prm.scheme if isinstance(self.prm.scheme, str) else \
            {v: k for k, v in SCHEMES.items()}.get(self.prm.scheme, "rk4")
        self.p, self.t, self.im_t, self.dt = restart_time_state(st, bool(self.prm.real_time), sch,
                                                               self.dt)
        self.set_state(st.psi)

    def wait_probe(self, limit_ns: int) -> None:
        """Failure-detection self-test: raises GpeError(GPE_ERR_TIMEOUT)."""
        check(lib().gpe_gpu_wait_probe(self._ctx, int(limit_ns)), self._ctx)

    def set_wait_limit(self, limit_ns: int) -> None:
        """Limit of the stage kernels' device-side waits (0: the 2 s default)."""
        check(lib().gpe_gpu_set_wait_limit(self._ctx, int(limit_ns)), self._ctx)

    def test_stall(self, plane: int) -> None:
        """Failure-detection test hook: later stage launches never load `plane`
        of a work item, so their bounded waits run out (-1: off)."""
        check(lib().gpe_gpu_test_stall(self._ctx, int(plane)), self._ctx)

    def diagnostics(self) -> tuple[float, np.ndarray]:
        """mass and momentum (src/variables.f90:590-694) -> (M, (Px, Py, Pz))."""
        m = ctypes.c_double()
        mom = np.zeros(3)
        check(lib().gpe_gpu_diagnostics(self._ctx, ctypes.byref(m),
                                        mom.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
              self._ctx)
        return m.value, mom

    # ---- spectral initial condition and diagnostics (cuFFT) ------------------
    def random_phase(self, nv: float, enerv: float, seed: int = 0):
        """random_phase initial condition (src/ic.f90:190-269) -> (comp_amp, kc2)."""
        from . import spectral
        return spectral.random_phase(self, nv, enerv, seed)

    def condensed_particles(self):
        """condensed_particles + spectrum (src/io.f90:315-404, 632-725)."""
        from . import spectral
        return spectral.condensed_particles(self)

    def filtered_field(self, filter_kc: float, m: float = 1.0, out=None):
        """The filtered field of filtered_surface (src/io.f90:533-628)."""
        from . import spectral
        return spectral.filtered_field(self, filter_kc, m, out)

    def linelength(self, field=None) -> float:
        """linelength (src/variables.f90:879-1145): total vortex line length of
        the state, or of `field` (a contiguous CUDA torch tensor (nz, ny, nx),
        complex64/128), e.g. the filtered field."""
        v = ctypes.c_double()
        if field is None:
            check(lib().gpe_gpu_linelength(self._ctx, ctypes.byref(v)), self._ctx)
        else:
            eb = device_field(field, self.shape, self.prm.device, "linelength")
            torch_ready(field)
            check(lib().gpe_gpu_linelength_field(self._ctx, ctypes.c_void_p(field.data_ptr()), eb,
                                                 ctypes.byref(v)), self._ctx)
        return v.value

    def zeros(self, out: np.ndarray | None = None):
        """get_zeros / get_extra_zeros / get_re_im_zeros (src/io.f90:895-1402)
        -> (counts[12], points (n, 3)), sections in the reference's order.

        The point list can run to gigabytes.  By default it goes to a new
        array; `out` (float64, C-contiguous, shape (cap, 3), cap >= the point
        count) is filled instead and a view of its first n rows returned, so
        a caller that asks repeatedly can keep one page-locked buffer
        (`gpe_b200._lib.pinned_empty`) and copy at the link's full rate
        without locking gigabytes of pages on every call."""
        counts = np.zeros(12, dtype=np.int64)
        P64 = ctypes.POINTER(ctypes.c_int64)
        check(lib().gpe_gpu_zeros(self._ctx, counts.ctypes.data_as(P64), None, 0), self._ctx)
        n = int(counts.sum())
        if out is None:
            pts = np.empty((max(n, 1), 3), np.float64)
        else:
            if (not isinstance(out, np.ndarray) or out.dtype != np.float64 or out.ndim != 2
                    or out.shape[1] != 3 or not out.flags.c_contiguous or not out.flags.writeable):
                raise GpeError(1, "out must be a writeable C-contiguous float64 array of "
                                  "shape (cap, 3)")
            if out.shape[0] < n:
                raise GpeError(1, f"out holds {out.shape[0]} points, {n} found")
            pts = out
        check(lib().gpe_gpu_zeros(self._ctx, counts.ctypes.data_as(P64),
                                  pts.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                  pts.shape[0]), self._ctx)
        return counts, pts[:n]

    def renormalise(self, norm: float) -> None:
        """renormalise (src/variables.f90:698-709)."""
        check(lib().gpe_gpu_renormalise(self._ctx, float(norm)), self._ctx)

    def rhs(self, dtype=np.complex128) -> np.ndarray:
        """get_rhs (src/solve.f90:382-440) of the resident psi."""
        out = np.empty(self.shape, dtype=dtype)
        check(lib().gpe_gpu_rhs(self._ctx, out.ctypes.data_as(ctypes.c_void_p),
                                self._elem(dtype)), self._ctx)
        return out

    def laplacian(self, dtype=np.complex128) -> np.ndarray:
        out = np.empty(self.shape, dtype=dtype)
        check(lib().gpe_gpu_laplacian(self._ctx, out.ctypes.data_as(ctypes.c_void_p),
                                      self._elem(dtype)), self._ctx)
        return out

    def set_real_time(self, on: bool) -> None:
        check(lib().gpe_gpu_set_real_time(self._ctx, 1 if on else 0), self._ctx)
        self.prm.real_time = bool(on)

    def grid(self):
        x = np.zeros(self.prm.nx); y = np.zeros(self.prm.ny); z = np.zeros(self.prm.nz)
        P = ctypes.POINTER(ctypes.c_double)
        check(lib().gpe_gpu_grid(self._ctx, x.ctypes.data_as(P), y.ctypes.data_as(P),
                                 z.ctypes.data_as(P)), self._ctx)
        return x, y, z

    # ---- instrumentation ------------------------------------------------------
    def set_timing(self, on: bool) -> None:
        check(lib().gpe_gpu_set_timing(self._ctx, 1 if on else 0), self._ctx)

    def timing(self) -> dict:
        t = GpeTimingC()
        check(lib().gpe_gpu_get_timing(self._ctx, ctypes.byref(t)), self._ctx)
        return {name: {"ms": t.ms[i], "launches": int(t.launches[i]), "sites": int(t.sites[i])}
                for i, name in enumerate(TIMING_FAMILIES)}

    def launch_count(self) -> int:
        return int(lib().gpe_gpu_launch_count(self._ctx))

    def stream_handle(self) -> int:
        """The context's cudaStream_t as an integer."""
        return int(lib().gpe_gpu_stream(self._ctx) or 0)

    def device_bytes(self) -> int:
        return int(lib().gpe_gpu_device_bytes(self._ctx))


@dataclass
class OutputParams:
    """io_params of run.in (src/parameters.f90:57-90) that drive the loop's
    output cadence (src/gpe.f90:176-226)."""
    save_rate: int = 10        # energy.dat, psi_time.dat, norm.dat every save_rate steps
    save_rate2: float = 50.0   # idl_surface (save_3d) every save_rate2 time units
    save_rate3: float = 50.0   # condensed_particles every save_rate3 time units
    p_save: float = 10.0       # end_state every p_save time units
    save_3d: bool = True
    save_spectrum: bool = True
    save_filter: bool = False
    filter_kc: float = 10.0
    save_ll: bool = False      # linelength.dat every save_rate steps
    save_contour: bool = False  # save_surface slice every save_rate2 time units
    save_zeros: bool = False   # zero finders every save_rate2 time units


def _modulo(a: float, p: float) -> float:
    """Fortran modulo: a - floor(a / p) p."""
    return a - math.floor(a / p) * p


def _pr_bytes(prm) -> int:
    return 8 if prm.precision == 16 else 4


def _idl_surface(s, run_dir):
    from . import output
    output.write_idl_surface(run_dir, s.p, s.t, s.im_t, s.get_state(), s.grid(),
                             pr_bytes=_pr_bytes(s.prm))


def _end_state(s, run_dir):
    from . import output
    d = os.path.join(run_dir, output.proc_dir(0))
    os.makedirs(d, exist_ok=True)
    s.save_end_state(os.path.join(d, "end_state.dat"))


def _cadence_outputs(s, run_dir, io: OutputParams, counters: dict) -> None:
    """The writes before solver in the reference loop (src/gpe.f90:176-226),
    on the current state."""
    from . import output
    prm = s.prm
    t_all = s.t + s.im_t
    adt = abs(s.dt)
    if _modulo(t_all, adt * io.save_rate) < adt:
        E, _ = s.energy()
        output.append(os.path.join(run_dir, "energy.dat"),
                      output.energy_line(s.t, s.im_t, E, prm.nx * prm.ny * prm.nz))
        v = s.get_site(prm.nx // 2, prm.ny // 2, prm.nz // 2)
        output.append(os.path.join(run_dir, "psi_time.dat"), output.psi_time_line(s.t, s.im_t, v))
        if io.save_ll:
            output.append(os.path.join(run_dir, "linelength.dat"),
                          output.e_line(s.t, s.im_t, s.linelength()))
    if t_all >= io.save_rate3 * counters["m"]:
        c = s.condensed_particles()
        output.append(os.path.join(run_dir, "mass.dat"), output.mass_line(s.t, s.im_t, c.row))
        if io.save_spectrum:
            output.write_spectrum(run_dir, s.p, s.t, c)
        if io.save_filter:  # filtered_surface (src/io.f90:398-400, 533-628)
            import torch
            f = torch.empty(s.shape, dtype=torch.complex128 if prm.precision == 16 else
                            torch.complex64, device=torch.device("cuda", prm.device))
            s.filtered_field(io.filter_kc, 1.0, out=f)
            if io.save_ll:  # save_linelength(filtered, 1) (src/io.f90:583-585)
                output.append(os.path.join(run_dir, "filtered_ll.dat"),
                              output.e_line(s.t, s.im_t, s.linelength(f)))
            output.write_filtered_surface(run_dir, s.p, s.t, f.cpu().numpy(), s.grid(),
                                          pr_bytes=_pr_bytes(prm))
        counters["m"] += 1
    if t_all >= io.save_rate2 * counters["n"]:
        if io.save_zeros:
            counts, pts = s.zeros()
            output.write_zeros(run_dir, s.p, counts, pts)
        if io.save_contour:
            output.write_surface_slice(run_dir, s.p, s.get_plane(prm.nz // 2), s.grid())
        if io.save_3d:
            _idl_surface(s, run_dir)
        counters["n"] += 1
    if t_all >= io.p_save * counters["ps"]:
        _end_state(s, run_dir)
        counters["ps"] += 1


def run_loop(s: GpeSolver, nsteps: int, *, renorm: bool = False, stop_imag: bool = False,
             record=None, run_dir: str | None = None, outputs: OutputParams | None = None,
             end_time: float | None = None, imprint=None):
    """The per-step bookkeeping of the reference time loop (src/gpe.f90:134-278)
    with an explicit step count: solver, get_norm + relnorm (equation 4),
    imaginary-to-real switch at relnorm < 1e-12 (:251-268), renormalise.
    With run_dir, the loop also keeps the reference's cooperative controls:
    it stops, writing run_dir/proc00/end_state.dat, when the file RUNNING is
    absent before a step (:136-159), and when a file SAVE appears after a
    step it writes the IDL surface run_dir/proc00/densNNNNNNN.dat and deletes
    SAVE (save_run, src/io.f90:1566-1595).  With outputs as well, it writes
    the reference's files at its cadence: energy.dat and psi_time.dat (and
    norm.dat after the step, and timestep.dat for rk45) every save_rate
    steps, condensed_particles
    (mass.dat, spectra, filtered surface) every save_rate3, idl_surface every
    save_rate2 and end_state every p_save time units, the counters starting
    from the current time (:126-128).
    With end_time, the loop also stops once t + im_t > end_time, the
    reference's loop condition (:134).  With imprint (a host field, the
    vortex_line(vl1) of imprint_vl), every imaginary-time step of equation 4
    ends with psi = |psi| * imprint (imprint_vortex_line,
    src/variables.f90:1149-1163; src/gpe.f90:270).
    Returns the list of (t, im_t, norm, relnorm) after each step."""
    from . import output
    prm = s.prm
    out = [] if record is None else record
    prev_norm = 1.0
    if prm.eqn_to_solve == 4 and not prm.real_time:
        prev_norm = s.get_norm()
        if renorm:
            s.renormalise(prev_norm)
    counters = {}
    if outputs is not None:
        counters = {"ps": int(s.t / outputs.p_save), "n": int(s.t / outputs.save_rate2),
                    "m": int(s.t / outputs.save_rate3)}
    norm = 0.0
    for _ in range(nsteps):
        if end_time is not None and not (s.t + s.im_t <= end_time):
            break
        if run_dir is not None and not os.path.exists(os.path.join(run_dir, "RUNNING")):
            _end_state(s, run_dir)
            break
        if outputs is not None and run_dir is not None:
            _cadence_outputs(s, run_dir, outputs, counters)
        s.solver()
        if outputs is not None and run_dir is not None and prm.scheme == "rk45" and \
                s.p % outputs.save_rate == 0:
            # rkqs writes the next step's size after every save_rate-th step
            output.append(os.path.join(run_dir, "timestep.dat"),
                          output.timestep_line(s.t, s.im_t, s.dt, s.p))
        if run_dir is not None and os.path.exists(os.path.join(run_dir, "SAVE")):
            _idl_surface(s, run_dir)
            os.remove(os.path.join(run_dir, "SAVE"))
        relnorm = 0.0
        if prm.eqn_to_solve == 4:
            norm = s.get_norm()
            relnorm = abs((norm - prev_norm) / prev_norm)
            out.append((s.t, s.im_t, norm, relnorm))
            if outputs is not None and run_dir is not None and \
                    _modulo(s.t + s.im_t, abs(s.dt) * outputs.save_rate) < abs(s.dt):
                output.append(os.path.join(run_dir, "norm.dat"),
                              output.norm_line(s.t, s.im_t, norm, relnorm))
        if prm.eqn_to_solve == 4 and not prm.real_time:
            if relnorm < 1e-12:
                if stop_imag:
                    break
                s.set_real_time(True)
                s.im_t = 0.0
                if outputs is not None:
                    counters = {"ps": int(s.t / outputs.p_save),
                                "n": int(s.t / outputs.save_rate2),
                                "m": int(s.t / outputs.save_rate3)}
                    if outputs.save_3d and run_dir is not None:
                        _idl_surface(s, run_dir)
                s.dt = complex(abs(s.dt.imag), abs(s.dt.real))
            if renorm:
                s.renormalise(norm)
            if imprint is not None:
                s.set_state(np.abs(s.get_state()) * imprint)
        prev_norm = norm
        s.p += 1
    return out

"""The reference's run inputs: run.in, parameters.in and ic.in.

A reference run directory holds three input files, and this module reads all
three so that an existing run directory drives the B200 solver unchanged:

* run.in: four Fortran namelists, read in order by read_run_params
  (src/io.f90:78-114): run_params, eqn_params, io_params and misc_params,
  with the variables of src/parameters.f90:24-86.
* parameters.in: Fortran declarations included verbatim in
  src/parameters.f90:21.  The real kind pr (selected_real_kind(15, 307) is
  double, (6, 37) single), the process grid nyprocs x nzprocs, the grid
  nx, ny, nz, and the named line_param / ring_param constants that ic.in
  refers to.
* ic.in: one Fortran assignment, also included verbatim (src/ic.f90:84-109).
  It is init_cond = a product of the initial-condition functions of
  src/ic.f90, e.g. init_cond = fermi() * vortex_line(vl1).

load_run(run_dir) gathers the three into a RunSetup.  run(run_dir) performs
the reference program's steps (src/gpe.f90:30-278): a GpeSolver with the
run's parameters, the initial condition or the restart state, then the time
loop to end_time writing the reference's output files into run_dir.  The
process grid is recorded but not used: one B200 holds the whole grid.
"""
from __future__ import annotations

import os
import re
from dataclasses import dataclass, field

import numpy as np

from . import ic
from .solver import GpeParams, GpeSolver, OutputParams, run_loop


class InputError(ValueError):
    """A malformed or unsupported input file (the reference stops with
    'ERROR: There was an error reading namelist ...', src/io.f90:103-111)."""


# --------------------------------------------------------------------------
# Fortran literals

_LOGICAL = re.compile(r"^\.?(t|f|true|false)\.?$", re.I)


def _strip_comment(line: str) -> str:
    """Drop a '!' comment that is not inside a quoted string."""
    out, quote = [], None
    for ch in line:
        if quote:
            out.append(ch)
            if ch == quote:
                quote = None
        elif ch in "'\"":
            quote = ch
            out.append(ch)
        elif ch == "!":
            break
        else:
            out.append(ch)
    return "".join(out)


def fortran_value(tok: str):
    """A Fortran literal: logical, character, integer or real (with an
    optional kind suffix such as _pr, and d exponents)."""
    t = tok.strip()
    if not t:
        raise InputError("empty value")
    if t[0] in "'\"":
        if len(t) < 2 or t[-1] != t[0]:
            raise InputError(f"unterminated string {tok!r}")
        return t[1:-1].replace(t[0] * 2, t[0])
    if _LOGICAL.match(t):
        return t.strip(".").lower() in ("t", "true")
    t = re.sub(r"_\w+$", "", t)  # kind suffix
    if re.fullmatch(r"[+-]?\d+", t):
        return int(t)
    try:
        return float(t.replace("d", "e").replace("D", "e"))
    except ValueError as e:
        raise InputError(f"cannot read value {tok!r}") from e


def _split_top(s: str, sep: str = ","):
    """Split at sep outside quotes and parentheses."""
    parts, cur, depth, quote = [], [], 0, None
    for ch in s:
        if quote:
            cur.append(ch)
            if ch == quote:
                quote = None
            continue
        if ch in "'\"":
            quote = ch
        elif ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        elif ch == sep and depth == 0:
            parts.append("".join(cur))
            cur = []
            continue
        cur.append(ch)
    parts.append("".join(cur))
    return [p for p in (q.strip() for q in parts) if p]


# --------------------------------------------------------------------------
# run.in

def parse_namelists(text: str) -> dict:
    """All namelist groups of a file: {group: {name: value}}, names lower
    case.  Entries are name = value, separated by commas or new lines; a
    group runs from &group to '/'."""
    groups = {}
    body = "\n".join(_strip_comment(l) for l in text.splitlines())
    for m in re.finditer(r"&(\w+)(.*?)(?:^\s*/|/\s*$|&end)", body, flags=re.S | re.M):
        name, content = m.group(1).lower(), m.group(2)
        entries = {}
        # name = value pairs; values never contain '=' in these files
        tokens = re.split(r"(\b[A-Za-z_]\w*\s*=)", content)
        key = None
        for tok in tokens:
            if tok.strip().endswith("=") and re.fullmatch(r"[A-Za-z_]\w*\s*=", tok.strip()):
                key = tok.strip()[:-1].strip().lower()
                continue
            if key is None:
                if tok.strip().strip(","):
                    raise InputError(f"namelist {name}: text before the first name: {tok!r}")
                continue
            vals = _split_top(tok.replace("\n", ","))
            if len(vals) != 1:
                raise InputError(f"namelist {name}: {key} needs one value, got {vals}")
            entries[key] = fortran_value(vals[0])
            key = None
        groups[name] = entries
    return groups


RUN_PARAMS = ("tau", "end_time", "xr", "yr", "zr", "scheme", "eqn_to_solve", "bcs", "order",
              "restart", "saved_restart", "renorm", "imprint_vl", "stop_imag", "real_time")
EQN_PARAMS = ("urhs", "diss_amp", "scal", "nv", "enerv", "g", "mu", "nn", "omx", "omy", "omz")
IO_PARAMS = ("save_rate", "save_rate2", "save_rate3", "p_save", "save_contour", "save_3d",
             "save_filter", "filter_kc", "save_average", "save_spectrum", "save_pdf",
             "save_vcf", "save_ll", "save_zeros")
MISC_PARAMS = ("nbins", "diagnostic", "pp_filtered_surface", "nlines", "nfilter", "fscale")
_GROUPS = (("run_params", RUN_PARAMS), ("eqn_params", EQN_PARAMS), ("io_params", IO_PARAMS),
           ("misc_params", MISC_PARAMS))


def read_run_in(path: str) -> dict:
    """run.in as {group: {name: value}}; every group read_run_params reads
    must be present, and only the names src/parameters.f90 declares."""
    with open(path) as f:
        groups = parse_namelists(f.read())
    for g, names in _GROUPS:
        if g not in groups:
            raise InputError(f"There was an error reading namelist {g} in run.in: missing")
        extra = set(groups[g]) - set(names)
        if extra:
            raise InputError(f"There was an error reading namelist {g} in run.in: "
                             f"unknown names {sorted(extra)}")
    return groups


# --------------------------------------------------------------------------
# parameters.in

def parse_parameters_in(text: str) -> dict:
    """pr (bytes of the real kind), nyprocs, nzprocs, nx, ny, nz and the
    named line_param / ring_param constants {name: {field: value}}."""
    lines = [_strip_comment(l) for l in text.splitlines()]
    # join '&' continuation lines
    joined, cur = [], ""
    for l in lines:
        s = l.rstrip()
        if s.endswith("&"):
            cur += s[:-1] + " "
            continue
        s = cur + s.lstrip("& ") if cur else s
        cur = ""
        if s.strip():
            joined.append(s.strip())
    out = {"lines": {}, "rings": {}}
    for s in joined:
        m = re.match(r"integer\s*,\s*parameter\s*::\s*pr\s*=\s*selected_real_kind\s*\(\s*(\d+)",
                     s, re.I)
        if m:
            out["pr"] = 8 if int(m.group(1)) > 6 else 4
            continue
        m = re.match(r"integer\s*,\s*parameter\s*::\s*(\w+)\s*=\s*([+-]?\d+)\s*$", s, re.I)
        if m:
            out[m.group(1).lower()] = int(m.group(2))
            continue
        m = re.match(r"type\s*\(\s*(line_param|ring_param)\s*\)\s*,\s*parameter\s*::\s*(\w+)\s*="
                     r"\s*(line_param|ring_param)\s*\((.*)\)\s*$", s, re.I)
        if m:
            kind = m.group(1).lower()
            vals = [fortran_value(v) for v in _split_top(m.group(4))]
            names = LINE_FIELDS if kind == "line_param" else RING_FIELDS
            if len(vals) != len(names):
                raise InputError(f"{m.group(2)}: {kind} takes {len(names)} values, got "
                                 f"{len(vals)}")
            rec = dict(zip(names, vals))
            for k, v in rec.items():  # reals given as integers
                if k in _REAL_FIELDS and isinstance(v, int) and not isinstance(v, bool):
                    rec[k] = float(v)
            out["lines" if kind == "line_param" else "rings"][m.group(2).lower()] = rec
    for k in ("pr", "nx", "ny", "nz"):
        if k not in out:
            raise InputError(f"parameters.in: no {k}")
    return out


LINE_FIELDS = ("x0", "y0", "z0", "amp1", "amp2", "ll", "sgn", "dir", "imprint_phase")
RING_FIELDS = ("plane", "x0", "y0", "z0", "r0", "amp", "mm", "r1", "kk", "dir")
_REAL_FIELDS = {"x0", "y0", "z0", "amp1", "amp2", "ll", "sgn", "r0", "amp", "r1"}


# --------------------------------------------------------------------------
# ic.in

IC_FUNCTIONS = {"random_phase": 0, "fermi": 0, "vortex_line": 1, "vortex_ring": 1,
                "vortex_pair": 0, "sphere": 0, "sphere2": 0, "wall": 0, "pade_pulse_ring": 5}


def parse_ic_in(text: str) -> list:
    """init_cond = f1(args) * f2(args) * ... -> [(name, [args])], args as
    Fortran literals or the lower-case names of parameter constants."""
    body = " ".join(_strip_comment(l).rstrip().rstrip("&") for l in text.splitlines())
    m = re.search(r"init_cond\s*=\s*(.+)$", body.strip(), re.I)
    if not m:
        raise InputError("ic.in: no 'init_cond = ...' assignment")
    factors = []
    for term in _split_top(m.group(1), "*"):
        t = re.fullmatch(r"(\w+)\s*\((.*)\)", term.strip())
        if not t:
            raise InputError(f"ic.in: cannot read factor {term!r}")
        name = t.group(1).lower()
        if name not in IC_FUNCTIONS:
            raise InputError(f"ic.in: unknown initial condition {name}()")
        args = []
        for a in _split_top(t.group(2)):
            args.append(a.lower() if re.fullmatch(r"[A-Za-z_]\w*", a) else fortran_value(a))
        if len(args) != IC_FUNCTIONS[name]:
            raise InputError(f"ic.in: {name}() takes {IC_FUNCTIONS[name]} arguments")
        factors.append((name, args))
    return factors


# --------------------------------------------------------------------------
# A run

@dataclass
class RunSetup:
    prm: GpeParams
    outputs: OutputParams
    tau: float
    end_time: float
    restart: bool
    renorm: bool
    stop_imag: bool
    imprint_vl: bool
    nv: float
    enerv: float
    ic: list
    consts: dict = field(default_factory=dict)
    procs: tuple = (1, 1)
    namelists: dict = field(default_factory=dict)


def load_run(run_dir: str, device: int = 0, kahan: bool = False) -> RunSetup:
    """run.in, parameters.in and ic.in of run_dir -> RunSetup.  The storage
    precision follows pr (complex128 for double, complex64 for single);
    kahan adds compensated accumulation to a single-precision run."""
    nl = read_run_in(os.path.join(run_dir, "run.in"))
    with open(os.path.join(run_dir, "parameters.in")) as f:
        par = parse_parameters_in(f.read())
    with open(os.path.join(run_dir, "ic.in")) as f:
        factors = parse_ic_in(f.read())
    r, e, o = nl["run_params"], nl["eqn_params"], nl["io_params"]
    precision = 16 if par["pr"] == 8 else 8
    prm = GpeParams(nx=par["nx"], ny=par["ny"], nz=par["nz"], xr=float(r["xr"]),
                    yr=float(r["yr"]), zr=float(r["zr"]), scheme=str(r["scheme"]).strip(),
                    eqn_to_solve=int(r["eqn_to_solve"]), bcs=int(r["bcs"]),
                    order=int(r["order"]), real_time=bool(r["real_time"]), precision=precision,
                    Urhs=float(e["urhs"]), diss_amp=float(e["diss_amp"]), scal=float(e["scal"]),
                    g=float(e["g"]), mu=float(e["mu"]), nn=float(e["nn"]), omx=float(e["omx"]),
                    omy=float(e["omy"]), omz=float(e["omz"]), kahan=bool(kahan and precision == 8),
                    device=device)
    outputs = OutputParams(save_rate=int(o["save_rate"]), save_rate2=float(o["save_rate2"]),
                           save_rate3=float(o["save_rate3"]), p_save=float(o["p_save"]),
                           save_3d=bool(o["save_3d"]), save_spectrum=bool(o["save_spectrum"]),
                           save_filter=bool(o["save_filter"]), filter_kc=float(o["filter_kc"]),
                           save_ll=bool(o["save_ll"]), save_contour=bool(o["save_contour"]),
                           save_zeros=bool(o["save_zeros"]))
    consts = dict(par["lines"])
    consts.update(par["rings"])
    for name, args in factors:
        for a in args:
            if isinstance(a, str) and name in ("vortex_line", "vortex_ring") and a not in consts:
                raise InputError(f"ic.in: {a} is not declared in parameters.in")
    return RunSetup(prm=prm, outputs=outputs, tau=float(r["tau"]), end_time=float(r["end_time"]),
                    restart=bool(r["restart"]), renorm=bool(r["renorm"]),
                    stop_imag=bool(r["stop_imag"]), imprint_vl=bool(r["imprint_vl"]),
                    nv=float(e["nv"]), enerv=float(e["enerv"]), ic=factors, consts=consts,
                    procs=(par.get("nyprocs", 1), par.get("nzprocs", 1)), namelists=nl)


def initial_state(setup: RunSetup, solver: GpeSolver | None = None, seed: int = 0):
    """init_cond of ic.in as a numpy (nz, ny, nx) complex128 field.  A
    random_phase() factor is drawn on the GPU through the solver (the
    reference's random_phase with nv and enerv, seeded); the other factors
    are evaluated on the host."""
    p = setup.prm
    x = -p.xr + np.arange(p.nx) * (2.0 * p.xr / (p.nx - 1))
    y = -p.yr + np.arange(p.ny) * (2.0 * p.yr / (p.ny - 1))
    z = -p.zr + np.arange(p.nz) * (2.0 * p.zr / (p.nz - 1))
    psi = np.ones((p.nz, p.ny, p.nx), dtype=np.complex128)
    for name, args in setup.ic:
        if name == "random_phase":
            if solver is None:
                raise InputError("random_phase() needs a solver on the GPU")
            solver.random_phase(setup.nv, setup.enerv, seed)
            f = solver.get_state()
        elif name == "fermi":
            f = ic.fermi(x, y, z, p.mu, p.g, p.omx, p.omy, p.omz)
        elif name == "vortex_line":
            f = ic.vortex_line(x, y, z, setup.consts[args[0]], p.scal)
        elif name == "vortex_ring":
            f = ic.vortex_ring(x, y, z, setup.consts[args[0]], p.scal)
        elif name == "pade_pulse_ring":
            which = str(args[0]).strip().lower()
            f = ic.pade_pulse_ring(x, y, z, which, *[float(a) for a in args[1:]])
        else:  # vortex_pair, sphere, sphere2, wall
            f = getattr(ic, name)(x, y, z)
        psi = psi * f
    return psi


def run(run_dir: str, *, device: int = 0, kahan: bool = False, seed: int = 0,
        max_steps: int | None = None):
    """The reference program on run_dir (src/gpe.f90:30-278): read the inputs,
    set dt from tau, load the initial condition (or end_state.dat when
    restart = .true.; with restart = .false. an existing end_state.dat is an
    error), write the initial idl_surface, then step while t + im_t <=
    end_time with the reference's cadence of outputs.  Returns (solver,
    records of run_loop); the caller closes the solver."""
    from . import output
    from .restart import RestartError
    setup = load_run(run_dir, device=device, kahan=kahan)
    p = setup.prm
    s = GpeSolver(p, tau=setup.tau)
    state = os.path.join(run_dir, output.proc_dir(0), "end_state.dat")
    if setup.restart:
        if not os.path.exists(state):
            s.close()
            raise RestartError(f"restart=.true. but {state} does not exist.")
        s.load_end_state(state)
    else:
        if os.path.exists(state):
            s.close()
            raise RestartError(f"restart=.false. but {state} exists.")
        s.set_state(initial_state(setup, s, seed))
    if setup.outputs.save_3d:
        output.write_idl_surface(run_dir, s.p, s.t, s.im_t, s.get_state(), s.grid(),
                                 pr_bytes=8 if p.precision == 16 else 4)
    imprint = None
    if setup.imprint_vl and "vl1" in setup.consts:
        x, y, z = s.grid()
        imprint = ic.vortex_line(x, y, z, setup.consts["vl1"], p.scal)
    open(os.path.join(run_dir, "RUNNING"), "a").close()
    rec = run_loop(s, max_steps if max_steps is not None else 2 ** 62, renorm=setup.renorm,
                   stop_imag=setup.stop_imag, run_dir=run_dir, outputs=setup.outputs,
                   end_time=setup.end_time, imprint=imprint)
    return s, rec

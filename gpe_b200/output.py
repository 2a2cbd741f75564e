"""The reference's output files, written in its formats from values computed
on the device.

Text files use Fortran edit descriptors: Ew.d prints a value as
0.ddd...E+ee right-justified in w columns (the exponent letter dropped for
|exponent| > 99), Iw a right-justified integer; a format of n items writes
them without separators, one record (line) per write.

  norm.dat      (4e17.9) t, im_t, norm, relnorm            src/io.f90:407-421
  energy.dat    (3e17.9) t, im_t, E/(nx ny nz)             src/io.f90:199-218
  momentum.dat  (4e17.9) t, Px, Py, Pz                      src/io.f90:425-445
  psi_time.dat  (6e17.9) t, im_t, Re psi, Im psi, |psi|^2, phase at
                (nx/2, ny/2, nz/2)                          src/io.f90:147-195
  mass.dat      (9e17.9) t, im_t, M/(8 xr yr zr), n0/V, M, n0, temp, temp2,
                H/V                                         src/io.f90:369-382
  spectrum/spectrumNNNNNNN.dat (2i9,e17.9) m, nharm, eta    src/io.f90:705-710
  idf/idfNNNNNNN.dat           (i9,e17.9)  kk, F(kk)        src/io.f90:712-717
  eta_time.dat  (4e17.9) t, eta(1:3)                        src/io.f90:719-721
  p_saved.dat   (i10) p                                     src/io.f90:521-525
  linelength.dat (3e17.9) t, im_t, total line length        src/io.f90:1405-1438
  filtered_ll.dat (3e17.9) the same of the filtered field    src/io.f90:583-585
  timestep.dat  (3e17.9,i10) t, im_t, |dt|, p (rk45, every save_rate
                steps, after the step)                      src/solve.f90:234-241

Stream (unformatted, access='stream') files of one process directory
procRR/ (RR = the two-digit rank, src/io.f90:118-143):

  densNNNNNNN.dat (idl_surface, src/io.f90:489-529): real(pr) t+im_t;
    int32 nx, ny, nz; int32 nyprocs, nzprocs; int32 js, je, ks, ke;
    complex(pr) psi(0:nx-1, js:je, ks:ke); real(pr) x(nx), y(ny), z(nz)
  filteredNNNNNNN.dat (filtered_surface flag 0, src/io.f90:595-606): the
    same layout with t in place of t+im_t and the filtered field
  end_state_filtered.dat (flag 1, :607-616): the end_state layout

save_surface (src/io.f90:449-485): procRR/psiNNNNNNN.dat, the plane z = nz/2
as (6e17.9) records x(i), y(j), |psi|^2, phase, Re psi, Im psi, j fastest,
an empty record after each i.

Text files of the zero finders in procRR/ (src/io.f90:895-1402):
zerosNNNNNNN.dat, re_zerosNNNNNNN.dat, im_zerosNNNNNNN.dat, each a list-
directed header line per section (" # i,j,k --> ...") followed by its points
as (3e17.9) records.

NNNNNNN = itos(p), p as seven digits with leading zeros (src/io.f90:29-47).
A single-domain run is process 0 of a 1 x 1 grid: js = ks = 0,
je = ny-1, ke = nz-1.
"""
from __future__ import annotations

import math
import os

import numpy as np


def fortran_e(x: float, w: int = 17, d: int = 9) -> str:
    """Ew.d of a real value."""
    x = float(x)
    if math.isnan(x):
        return "NaN".rjust(w)
    if math.isinf(x):
        return ("-Infinity" if x < 0 else "Infinity").rjust(w)
    if x == 0.0:
        body, exp = "0." + "0" * d, 0
        sign = "-" if math.copysign(1.0, x) < 0 else ""
    else:
        mant, e = f"{abs(x):.{d - 1}e}".split("e")
        digits = mant.replace(".", "")
        body, exp = "0." + digits, int(e) + 1
        sign = "-" if x < 0 else ""
    es = f"E{'+' if exp >= 0 else '-'}{abs(exp):02d}" if abs(exp) <= 99 else \
        f"{'+' if exp >= 0 else '-'}{abs(exp):03d}"
    s = sign + body + es
    return s.rjust(w) if len(s) <= w else "*" * w


def fortran_i(n: int, w: int) -> str:
    s = str(int(n))
    return s.rjust(w) if len(s) <= w else "*" * w


def itos(n: int) -> str:
    """itos (src/io.f90:29-47): the last seven decimal digits of n."""
    return "".join(str(abs(int(n)) // 10 ** i % 10) for i in range(6, -1, -1))


def proc_dir(rank: int) -> str:
    return f"proc{rank:02d}"


def e_line(*values, w: int = 17, d: int = 9) -> str:
    return "".join(fortran_e(v, w, d) for v in values) + "\n"


def append(path: str, line: str) -> None:
    with open(path, "a") as f:
        f.write(line)


# ---- time series -------------------------------------------------------------

def norm_line(t, im_t, norm, relnorm) -> str:
    return e_line(t, im_t, norm, relnorm)


def energy_line(t, im_t, E, nsites) -> str:
    return e_line(t, im_t, E / float(nsites))


def momentum_line(t, mom) -> str:
    return e_line(t, mom[0], mom[1], mom[2])


def phase_of(psi):
    """get_phase (src/variables.f90:362-374): atan2(Im psi + 1e-6, Re psi)."""
    return np.arctan2(np.imag(psi) + 1.0e-6, np.real(psi))


def psi_time_line(t, im_t, value: complex) -> str:
    v = complex(value)
    return e_line(t, im_t, v.real, v.imag, abs(v) ** 2,
                  float(np.arctan2(v.imag + 1.0e-6, v.real)))


def timestep_line(t, im_t, dt, p) -> str:
    return fortran_e(t) + fortran_e(im_t) + fortran_e(abs(dt)) + fortran_i(p, 10) + "\n"


def mass_line(t, im_t, row: dict) -> str:
    return e_line(t, im_t, row["M_density"], row["n0_over_V"], row["M"], row["n0"],
                  row["temp"], row["temp2"], row["H_over_V"])


def spectrum_text(eta, nharm) -> str:
    return "".join(fortran_i(m + 1, 9) + fortran_i(nharm[m], 9) + fortran_e(eta[m]) + "\n"
                   for m in range(len(eta)))


def idf_text(F) -> str:
    return "".join(fortran_i(kk + 1, 9) + fortran_e(F[kk]) + "\n" for kk in range(len(F)))


def eta_time_line(t, eta) -> str:
    return e_line(t, eta[0], eta[1], eta[2])


def write_spectrum(run_dir: str, p: int, t: float, cond) -> None:
    """spectrum/, idf/ and eta_time.dat of one condensed_particles call."""
    for sub in ("spectrum", "idf"):
        os.makedirs(os.path.join(run_dir, sub), exist_ok=True)
    with open(os.path.join(run_dir, "spectrum", f"spectrum{itos(p)}.dat"), "w") as f:
        f.write(spectrum_text(cond.eta, cond.nharm))
    with open(os.path.join(run_dir, "idf", f"idf{itos(p)}.dat"), "w") as f:
        f.write(idf_text(cond.F))
    append(os.path.join(run_dir, "eta_time.dat"), eta_time_line(t, cond.eta))


# ---- stream files ----------------------------------------------------------------

def _types(pr_bytes: int):
    if pr_bytes == 8:
        return np.dtype("<f8"), np.dtype("<c16")
    if pr_bytes == 4:
        return np.dtype("<f4"), np.dtype("<c8")
    raise ValueError("pr must be 4 or 8 bytes")


def surface_bytes(time: float, field, x, y, z, pr_bytes: int = 8,
                  procs=(1, 1), bounds=None) -> bytes:
    """The dens / filtered stream layout of one process."""
    rt, ct = _types(pr_bytes)
    a = np.ascontiguousarray(field, dtype=ct)
    nz, ny, nx = a.shape
    if bounds is None:
        bounds = (0, ny - 1, 0, nz - 1)
    return b"".join([
        np.array([time], dtype=rt).tobytes(),
        np.array([len(x), len(y), len(z)], dtype="<i4").tobytes(),
        np.array(procs, dtype="<i4").tobytes(),
        np.array(bounds, dtype="<i4").tobytes(),
        a.tobytes(),
        np.asarray(x, dtype=rt).tobytes(),
        np.asarray(y, dtype=rt).tobytes(),
        np.asarray(z, dtype=rt).tobytes(),
    ])


def write_idl_surface(run_dir: str, p: int, t: float, im_t: float, psi, grid,
                      pr_bytes: int = 8, rank: int = 0) -> str:
    """idl_surface: procRR/densNNNNNNN.dat and the p_saved.dat line."""
    d = os.path.join(run_dir, proc_dir(rank))
    os.makedirs(d, exist_ok=True)
    path = os.path.join(d, f"dens{itos(p)}.dat")
    x, y, z = grid
    with open(path, "wb") as f:
        f.write(surface_bytes(t + im_t, psi, x, y, z, pr_bytes))
    if rank == 0:
        append(os.path.join(run_dir, "p_saved.dat"), fortran_i(p, 10) + "\n")
    return path


def write_filtered_surface(run_dir: str, p: int, t: float, filtered, grid,
                           pr_bytes: int = 8, rank: int = 0) -> str:
    """filtered_surface flag 0: procRR/filteredNNNNNNN.dat."""
    d = os.path.join(run_dir, proc_dir(rank))
    os.makedirs(d, exist_ok=True)
    path = os.path.join(d, f"filtered{itos(p)}.dat")
    x, y, z = grid
    with open(path, "wb") as f:
        f.write(surface_bytes(t, filtered, x, y, z, pr_bytes))
    return path


def read_surface(path: str, pr_bytes: int = 8):
    """Parse a dens / filtered file -> (time, (nx, ny, nz), procs, bounds,
    field (nz, ny, nx), x, y, z)."""
    rt, ct = _types(pr_bytes)
    raw = open(path, "rb").read()
    off = 0

    def take(dtype, count):
        nonlocal off
        v = np.frombuffer(raw, dtype=dtype, count=count, offset=off)
        off += v.nbytes
        return v

    time = float(take(rt, 1)[0])
    nx, ny, nz = (int(v) for v in take("<i4", 3))
    procs = tuple(int(v) for v in take("<i4", 2))
    js, je, ks, ke = (int(v) for v in take("<i4", 4))
    field = take(ct, nx * (je - js + 1) * (ke - ks + 1)).reshape(ke - ks + 1, je - js + 1, nx)
    x, y, z = take(rt, nx), take(rt, ny), take(rt, nz)
    if off != len(raw):
        raise ValueError(f"{path}: {len(raw) - off} trailing bytes")
    return time, (nx, ny, nz), procs, (js, je, ks, ke), field.copy(), x.copy(), y.copy(), z.copy()


# ---- zero finders ------------------------------------------------------------------

ZERO_HEADERS = [
    "# i,j,k --> i+1,j,k", "# i,j,k --> i,j+1,k", "# i,j,k --> i,j,k+1",
    "# i,j,k --> i+1,j,k --> i+1,j+1,k --> i,j+1,k",
    "# i,j,k --> i+1,j,k --> i+1,j,k+1 --> i,j,k+1",
    "# i,j,k --> i,j,k+1 --> i,j+1,k+1 --> i,j+1,k",
]
# sections of each file, in the order of gpe_gpu_zeros
ZERO_FILES = (("zeros", range(0, 6)), ("re_zeros", range(6, 9)), ("im_zeros", range(9, 12)))


def _header(s: int) -> str:
    # list-directed output of a character constant starts with a blank
    return " " + ZERO_HEADERS[s if s < 6 else (s - 6) % 3] + "\n"


def zeros_texts(counts, points) -> dict:
    """The three files' contents from the 12 sections' counts and points."""
    starts = np.concatenate([[0], np.cumsum(np.asarray(counts, dtype=np.int64))])
    out = {}
    for name, secs in ZERO_FILES:
        parts = []
        for s in secs:
            parts.append(_header(s))
            for q in range(starts[s], starts[s + 1]):
                parts.append(e_line(*points[q]))
        out[name] = "".join(parts)
    return out


def write_zeros(run_dir: str, p: int, counts, points, rank: int = 0) -> list:
    """procRR/zerosNNNNNNN.dat, re_zeros..., im_zeros... of one call."""
    d = os.path.join(run_dir, proc_dir(rank))
    os.makedirs(d, exist_ok=True)
    paths = []
    for name, text in zeros_texts(counts, points).items():
        path = os.path.join(d, f"{name}{itos(p)}.dat")
        with open(path, "w") as f:
            f.write(text)
        paths.append(path)
    return paths


def surface_slice_text(plane, x, y) -> str:
    """save_surface of one z-plane (ny, nx)."""
    parts = []
    nyy, nxx = plane.shape
    for i in range(nxx):
        for j in range(nyy):
            v = complex(plane[j, i])
            parts.append(e_line(x[i], y[j], abs(v) ** 2,
                                float(np.arctan2(v.imag + 1.0e-6, v.real)), v.real, v.imag))
        parts.append("\n")
    return "".join(parts)


def write_surface_slice(run_dir: str, p: int, plane, grid, rank: int = 0) -> str:
    d = os.path.join(run_dir, proc_dir(rank))
    os.makedirs(d, exist_ok=True)
    path = os.path.join(d, f"psi{itos(p)}.dat")
    with open(path, "w") as f:
        f.write(surface_slice_text(plane, grid[0], grid[1]))
    return path

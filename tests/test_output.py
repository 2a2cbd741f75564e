"""The reference's output formats (gpe_b200.output): Fortran Ew.d / Iw text
records and the stream layout of the dens / filtered files."""
import os

import numpy as np
import pytest

from gpe_b200 import output


@pytest.mark.parametrize("x, s", [
    (1.5, "  0.150000000E+01"),
    (-1.5, " -0.150000000E+01"),
    (0.0, "  0.000000000E+00"),
    (1.0, "  0.100000000E+01"),
    (0.5, "  0.500000000E+00"),
    (123456789.123, "  0.123456789E+09"),
    (9.9999999996, "  0.100000000E+02"),   # rounds up into the next decade
    (1.23456789049e-5, "  0.123456789E-04"),
    (-2.5e100, " -0.250000000+101"),        # three-digit exponent drops the E
    (1e-300, "  0.100000000-299"),
])
def test_fortran_e17_9(x, s):
    assert output.fortran_e(x) == s
    assert len(s) == 17


def test_fortran_integer_and_itos():
    assert output.fortran_i(7, 9) == "        7"
    assert output.fortran_i(12345, 10) == "     12345"
    assert output.itos(0) == "0000000"
    assert output.itos(1234) == "0001234"
    assert output.itos(123456789) == "3456789"  # the last seven digits
    assert output.proc_dir(0) == "proc00" and output.proc_dir(12) == "proc12"


def test_record_lines():
    assert output.mass_line(1.0, 0.0, {"M_density": 2.0, "n0_over_V": 3.0, "M": 4.0, "n0": 5.0,
                                       "temp": 6.0, "temp2": 7.0, "H_over_V": 8.0}) == \
        "".join(output.fortran_e(v) for v in (1, 0, 2, 3, 4, 5, 6, 7, 8)) + "\n"
    assert output.spectrum_text([0.25, 0.0], [10, 0]) == \
        "        1       10  0.250000000E+00\n        2        0  0.000000000E+00\n"
    assert output.idf_text([1.0, 3.0]) == \
        "        1  0.100000000E+01\n        2  0.300000000E+01\n"
    line = output.psi_time_line(2.0, 0.5, 3.0 + 4.0j)
    assert len(line) == 6 * 17 + 1
    assert line[4 * 17:5 * 17] == output.fortran_e(25.0)
    assert line[5 * 17:6 * 17] == output.fortran_e(np.arctan2(4.0 + 1e-6, 3.0))


@pytest.mark.parametrize("pr", [8, 4])
def test_surface_stream_layout_round_trip(tmp_path, pr):
    nz, ny, nx = 3, 4, 5
    rng = np.random.default_rng(0)
    psi = rng.standard_normal((nz, ny, nx)) + 1j * rng.standard_normal((nz, ny, nx))
    grid = (np.linspace(-2, 2, nx), np.linspace(-1.5, 1.5, ny), np.linspace(-1, 1, nz))
    path = output.write_idl_surface(str(tmp_path), 42, 1.25, 0.5, psi, grid, pr_bytes=pr)
    assert path.endswith(os.path.join("proc00", "dens0000042.dat"))
    raw = open(path, "rb").read()
    assert len(raw) == pr + 9 * 4 + nx * ny * nz * 2 * pr + (nx + ny + nz) * pr
    assert np.frombuffer(raw, "<i4", 9, pr).tolist() == [nx, ny, nz, 1, 1, 0, ny - 1, 0, nz - 1]
    t, dims, procs, bounds, field, x, y, z = output.read_surface(path, pr)
    assert t == 1.75 and dims == (nx, ny, nz) and procs == (1, 1)
    tol = 0 if pr == 8 else 1e-6
    np.testing.assert_allclose(field, psi, rtol=tol, atol=tol)
    np.testing.assert_allclose(x, grid[0], rtol=tol)
    assert open(tmp_path / "p_saved.dat").read() == "        42\n"


def test_write_spectrum_files(tmp_path):
    from gpe_b200.spectral import Condensate
    c = Condensate({}, np.arange(7) * 0.5, np.arange(7), np.array([1.0, 2.0, 4.0]))
    output.write_spectrum(str(tmp_path), 3, 0.25, c)
    assert (tmp_path / "spectrum" / "spectrum0000003.dat").read_text().count("\n") == 7
    assert (tmp_path / "idf" / "idf0000003.dat").read_text().splitlines()[2] == \
        "        3  0.400000000E+01"
    assert (tmp_path / "eta_time.dat").read_text() == output.e_line(0.25, 0.0, 0.5, 1.0)


def test_surface_slice_layout():
    plane = np.array([[1 + 2j, 3 + 0j], [0 - 1j, 2 + 2j]])  # (ny=2, nx=2)
    text = output.surface_slice_text(plane, [0.0, 0.5], [-1.0, 1.0])
    lines = text.split("\n")
    # i outer, j inner, an empty record after each i
    assert len(lines) == 2 * 3 + 1 and lines[2] == "" and lines[5] == ""
    assert lines[0] == output.e_line(0.0, -1.0, 5.0, np.arctan2(2.0 + 1e-6, 1.0), 1.0,
                                     2.0).rstrip("\n")
    assert lines[1].startswith(output.fortran_e(0.0) + output.fortran_e(1.0))

"""The reference's output cadence driven by the device: point values,
condensate rows, spectra and surfaces written by run_loop from a live
context (src/gpe.f90:176-232, src/io.f90:147-195, 315-404, 489-529)."""
import os

import numpy as np
import pytest

from gpe_b200 import GpeParams, GpeSolver, output
from gpe_b200.solver import OutputParams, run_loop
import oracle
from oracle import spectral_ref as ref

pytestmark = pytest.mark.gpu


def _solver(n=16, precision=16):
    xr = 0.5 * (n - 1)
    prm = GpeParams(nx=n, ny=n, nz=n, xr=xr, yr=xr, zr=xr, scheme="rk4", eqn_to_solve=4, bcs=1,
                    order=2, precision=precision, g=1.0, mu=1.0)
    return GpeSolver(prm, dt=0.01)


@pytest.mark.parametrize("precision", [16, 8])
def test_get_site_matches_the_state(precision):
    with _solver(12, precision) as s:
        s.random_phase(1.0, 5.0, 3)
        psi = s.get_state()
        for ijk in [(0, 0, 0), (6, 6, 6), (11, 3, 7), (5, 11, 0)]:
            i, j, k = ijk
            assert s.get_site(i, j, k) == psi[k, j, i]
        with pytest.raises(Exception):
            s.get_site(12, 0, 0)


def test_run_loop_writes_the_reference_files(tmp_path):
    d = str(tmp_path)
    open(os.path.join(d, "RUNNING"), "w").close()
    with _solver(16) as s:
        s.random_phase(0.75, 0.75, 1)
        psi0 = s.get_state()
        io = OutputParams(save_rate=5, save_rate2=0.1, save_rate3=0.05, p_save=0.1)
        run_loop(s, 12, run_dir=d, outputs=io)
        final = s.get_state()
    # mass.dat: first row is condensed_particles of the initial state
    row0, _ = ref.condensed_fast(psi0, *(0.5 * 15,) * 3)
    first = open(os.path.join(d, "mass.dat")).read().splitlines()[0]
    vals = [float(first[17 * q:17 * (q + 1)]) for q in range(9)]
    assert vals[4] == pytest.approx(row0["M"], rel=1e-8)
    assert vals[5] == pytest.approx(row0["n0"], rel=1e-8)
    # psi_time.dat: the centre point of the initial state
    pt = open(os.path.join(d, "psi_time.dat")).read().splitlines()[0]
    assert float(pt[34:51]) == pytest.approx(psi0[8, 8, 8].real, rel=1e-8, abs=1e-12)
    # the first IDL surface holds the initial state bit for bit
    t, dims, procs, bounds, field, x, y, z = output.read_surface(
        os.path.join(d, "proc00", "dens0000000.dat"))
    assert dims == (16, 16, 16) and procs == (1, 1) and bounds == (0, 15, 0, 15)
    assert np.array_equal(field, psi0) and x[0] == -7.5 and x[-1] == 7.5
    # spectra files and the end state
    assert os.path.exists(os.path.join(d, "spectrum", "spectrum0000000.dat"))
    assert os.path.exists(os.path.join(d, "idf", "idf0000000.dat"))
    from gpe_b200.restart import read_end_state
    st = read_end_state(os.path.join(d, "proc00", "end_state.dat"), expect=(16, 16, 16))
    assert st.p in (10, 11) and not np.array_equal(st.psi, final)  # t = 0.1 up to rounding


def test_run_loop_filtered_surface_and_its_line_length(tmp_path):
    d = str(tmp_path)
    open(os.path.join(d, "RUNNING"), "w").close()
    with _solver(16) as s:
        s.random_phase(0.75, 0.75, 2)
        io = OutputParams(save_rate=100, save_rate2=1e9, save_rate3=1e9, p_save=1e9,
                          save_3d=False, save_spectrum=False, save_filter=True, save_ll=True,
                          filter_kc=6.0)
        run_loop(s, 2, run_dir=d, outputs=io)
        grid = s.grid()
    t, dims, _, _, field, x, _, _ = output.read_surface(
        os.path.join(d, "proc00", "filtered0000000.dat"))
    assert dims == (16, 16, 16) and t == 0.0 and np.array_equal(x, grid[0])
    line = open(os.path.join(d, "filtered_ll.dat")).read().splitlines()
    exp, _ = oracle.linelength(field, 1.0)  # dx = 2 xr / (n - 1) = 1
    assert len(line) == 1 and float(line[0][34:51]) == pytest.approx(exp, rel=1e-8)


@pytest.mark.parametrize("precision", [16, 8])
def test_get_plane_matches_the_state(precision):
    with _solver(12, precision) as s:
        s.random_phase(1.0, 5.0, 6)
        psi = s.get_state()
        for k in (0, 6, 11):
            np.testing.assert_array_equal(s.get_plane(k), psi[k])
        np.testing.assert_array_equal(s.get_plane(3, np.complex64),
                                      s.get_state(np.complex64)[3])
        with pytest.raises(Exception):
            s.get_plane(12)

"""Vortex line length (linelength, src/variables.f90:879-1145): the C
restatement in the oracle on analytic lines, and the library's kernels
against it on B200 (analytic lines, a ring, random fields full of
vortices, both storage precisions)."""
import math

import numpy as np
import pytest

import oracle


def _grid(n, h):
    x = (np.arange(n) - (n - 1) / 2) * h
    return np.meshgrid(x, x, x, indexing="ij")  # Z, Y, X


def test_oracle_straight_and_tilted_lines():
    n, h = 16, 0.5
    Z, Y, X = _grid(n, h)
    L, _ = oracle.linelength((X - 0.13) + 1j * (Y + 0.21), h)
    assert L == pytest.approx((n - 2) * h, rel=1e-14)
    L, _ = oracle.linelength((X - 0.3 * Z - 0.13) + 1j * (Y + 0.21), h)
    assert L == pytest.approx((n - 2) * h * math.sqrt(1.09), rel=1e-12)


def test_oracle_ring_is_close_to_its_circumference():
    n, h, R = 24, 0.5, 3.0
    Z, Y, X = _grid(n, h)
    L, _ = oracle.linelength((np.sqrt(X ** 2 + Y ** 2) - R) + 1j * (Z - 0.1), h)
    assert L == pytest.approx(2 * math.pi * R, rel=0.01)


def test_oracle_carries_its_point_arrays():
    """The work arrays come back changed and feed the next call."""
    rng = np.random.default_rng(0)
    psi = rng.standard_normal((10, 10, 10)) + 1j * rng.standard_normal((10, 10, 10))
    L0, st = oracle.linelength(psi, 1.0)
    assert np.any(st != 0.0) and L0 > 0


# --- on the GPU -------------------------------------------------------------------

def _solver(nz, ny, nx, precision=16, h=0.5):
    from gpe_b200 import GpeParams, GpeSolver
    prm = GpeParams(nx=nx, ny=ny, nz=nz, xr=0.5 * (nx - 1) * h, yr=0.5 * (ny - 1) * h,
                    zr=0.5 * (nz - 1) * h, scheme="rk4", eqn_to_solve=4, bcs=1, order=2,
                    precision=precision, g=1.0, mu=1.0)
    return GpeSolver(prm, dt=0.01)


@pytest.mark.gpu
def test_gpu_analytic_lines_and_ring():
    n, h = 24, 0.5
    Z, Y, X = _grid(n, h)
    fields = [(X - 0.13) + 1j * (Y + 0.21), (X - 0.3 * Z - 0.13) + 1j * (Y + 0.21),
              (np.sqrt(X ** 2 + Y ** 2) - 3.0) + 1j * (Z - 0.1)]
    with _solver(n, n, n, h=h) as s:
        for psi in fields:
            s.set_state(psi)
            exp, _ = oracle.linelength(psi, h)
            assert s.linelength() == pytest.approx(exp, rel=1e-13)


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(16, 16, 16), (18, 20, 24), (9, 17, 33), (40, 36, 64),
                                   (6, 6, 6), (6, 7, 9)])
@pytest.mark.parametrize("precision", [16, 8])
def test_gpu_random_fields_match_oracle(shape, precision):
    """Random fields: vortex lines through most cells, with one-point cells
    that measure to the x(2) carried from an earlier cell."""
    nz, ny, nx = shape
    rng = np.random.default_rng(nx * 7 + ny * 3 + nz)
    psi = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    if precision == 8:
        psi = psi.astype(np.complex64)
    with _solver(nz, ny, nx, precision) as s:
        s.set_state(psi)
        got = s.linelength()
        again = s.linelength()
    exp, _ = oracle.linelength(psi.astype(np.complex128), 0.5)
    assert got == pytest.approx(exp, rel=1e-12, abs=1e-14)
    assert got == again  # fixed reduction order


@pytest.mark.gpu
def test_gpu_smooth_field_at_128():
    """Many blocks: a random-phase state (a tangle of long lines)."""
    n = 128
    with _solver(n, n, n) as s:
        s.random_phase(0.75, 0.75, 2)
        psi = s.get_state()
        got = s.linelength()
    exp, _ = oracle.linelength(psi, 0.5)
    assert exp > 0
    assert got == pytest.approx(exp, rel=1e-12)


# --- zero finders (src/io.f90:895-1402) ----------------------------------------------

def test_oracle_zeros_of_a_straight_line():
    """psi = (x - a) + i (y - b): Re and Im cross together on no edge, the
    xy faces hold the line (each with a NaN point: the reference's slope
    divides by zero there), Re / Im crossings on the x / y edges."""
    n, h = 12, 0.5
    Z, Y, X = _grid(n, h)
    x = (np.arange(n) - (n - 1) / 2) * h
    counts, pts = oracle.zeros((X - 0.13) + 1j * (Y + 0.21), x, x, x)
    assert counts.tolist() == [0, 0, 0, n - 2, 0, 0, (n - 2) ** 2, 0, 0, 0, (n - 2) ** 2, 0]
    face = pts[:n - 2]
    assert np.all(face[:, 2] == x[1:n - 1])
    re_x = pts[n - 2:n - 2 + (n - 2) ** 2]
    np.testing.assert_allclose(re_x[:, 0], 0.13, rtol=1e-12)


def test_zero_files_layout(tmp_path):
    from gpe_b200 import output
    counts = [1, 0, 0, 0, 0, 0, 2, 0, 0, 0, 0, 1]
    pts = np.array([[1.0, 2.0, 3.0], [4.0, 5.0, 6.0], [7.0, 8.0, 9.0], [0.5, 0.25, 0.125]])
    paths = output.write_zeros(str(tmp_path), 7, counts, pts)
    names = sorted(p.split("/")[-1] for p in paths)
    assert names == ["im_zeros0000007.dat", "re_zeros0000007.dat", "zeros0000007.dat"]
    z = open(paths[0]).read().splitlines()
    assert z[0] == " # i,j,k --> i+1,j,k" and z[1] == output.e_line(1, 2, 3).rstrip("\n")
    assert len(z) == 6 + 1 and z[-1] == " # i,j,k --> i,j,k+1 --> i,j+1,k+1 --> i,j+1,k"
    r = open(paths[1]).read().splitlines()
    assert r == [" # i,j,k --> i+1,j,k", output.e_line(4, 5, 6).rstrip("\n"),
                 output.e_line(7, 8, 9).rstrip("\n"), " # i,j,k --> i,j+1,k",
                 " # i,j,k --> i,j,k+1"]
    m = open(paths[2]).read().splitlines()
    assert m[-1] == output.e_line(0.5, 0.25, 0.125).rstrip("\n")


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(16, 16, 16), (18, 20, 24), (6, 7, 9), (40, 36, 64)])
@pytest.mark.parametrize("precision", [16, 8])
def test_gpu_zeros_match_oracle(shape, precision):
    """Every section's points equal the oracle's, in order, bit for bit."""
    nz, ny, nx = shape
    rng = np.random.default_rng(nx + 5 * ny + 11 * nz)
    psi = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    if precision == 8:
        psi = psi.astype(np.complex64)
    with _solver(nz, ny, nx, precision) as s:
        s.set_state(psi)
        counts, pts = s.zeros()
        x, y, z = s.grid()
    ec, ep = oracle.zeros(psi.astype(np.complex128), x, y, z)
    assert counts.tolist() == ec.tolist()
    np.testing.assert_array_equal(pts, ep)


@pytest.mark.gpu
def test_gpu_zeros_of_lines_and_a_random_phase_state():
    n, h = 24, 0.5
    Z, Y, X = _grid(n, h)
    with _solver(n, n, n, h=h) as s:
        for psi in [(X - 0.13) + 1j * (Y + 0.21),
                    (np.sqrt(X ** 2 + Y ** 2) - 3.0) + 1j * (Z - 0.1)]:
            s.set_state(psi)
            counts, pts = s.zeros()
            ec, ep = oracle.zeros(psi, *s.grid())
            assert counts.tolist() == ec.tolist()
            np.testing.assert_array_equal(pts, ep)  # NaN where the oracle has NaN
    with _solver(96, 96, 96) as s:
        s.random_phase(0.75, 0.75, 4)
        psi = s.get_state()
        counts, pts = s.zeros()
        ec, ep = oracle.zeros(psi, *s.grid())
    assert counts.tolist() == ec.tolist() and counts.sum() > 0
    np.testing.assert_array_equal(pts, ep)


@pytest.mark.gpu
def test_gpu_zeros_into_a_kept_buffer():
    from gpe_b200 import GpeError
    from gpe_b200._lib import pinned_empty
    rng = np.random.default_rng(5)
    psi = rng.standard_normal((14, 13, 12)) + 1j * rng.standard_normal((14, 13, 12))
    with _solver(14, 13, 12) as s:
        s.set_state(psi)
        want_c, want_p = s.zeros()
        n = int(want_c.sum())
        buf = pinned_empty((n + 7, 3), np.float64)
        buf[:] = -1.0
        counts, pts = s.zeros(out=buf)
        assert counts.tolist() == want_c.tolist()
        np.testing.assert_array_equal(pts, want_p)
        assert pts.base is not None and np.shares_memory(pts, buf)
        assert np.all(buf[n:] == -1.0)
        for bad in (np.zeros((n - 1, 3)), np.zeros((n, 3), np.float32), np.zeros((n, 4)),
                    np.zeros((3, n)).T):
            with pytest.raises(GpeError):
                s.zeros(out=bad)


@pytest.mark.gpu
def test_gpu_zeros_rejects_a_small_buffer_and_fills_the_counts():
    import ctypes

    from gpe_b200 import GpeError
    from gpe_b200._lib import check, lib
    rng = np.random.default_rng(3)
    psi = rng.standard_normal((12, 12, 12)) + 1j * rng.standard_normal((12, 12, 12))
    with _solver(12, 12, 12) as s:
        s.set_state(psi)
        want, _ = s.zeros()
        counts = np.zeros(12, dtype=np.int64)
        pts = np.zeros((2, 3))
        P64 = ctypes.POINTER(ctypes.c_int64)
        with pytest.raises(GpeError):
            check(lib().gpe_gpu_zeros(s.handle, counts.ctypes.data_as(P64),
                                      pts.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 2),
                  s.handle)
    assert want.sum() > 2 and counts.tolist() == want.tolist()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [16, 8])
def test_gpu_line_length_of_a_device_field(precision):
    """gpe_gpu_linelength_field on a dense device array: the same number as the
    resident state holding the same values, and the oracle's on the filtered
    field (save_linelength(filtered, 1))."""
    import torch
    shape = (20, 18, 24)
    rng = np.random.default_rng(8)
    psi = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    dt = torch.complex128 if precision == 16 else torch.complex64
    with _solver(*shape, precision=precision) as s:
        s.set_state(psi.astype(np.complex128 if precision == 16 else np.complex64))
        here = s.linelength()
        dev = torch.empty(shape, dtype=dt, device="cuda")
        s.get_state_device(dev)
        assert s.linelength(dev) == here
        f = torch.empty(shape, dtype=dt, device="cuda")
        s.filtered_field(6.0, 1.0, out=f)
        got = s.linelength(f)
    exp, _ = oracle.linelength(f.cpu().numpy().astype(np.complex128), 0.5)
    assert got == pytest.approx(exp, rel=1e-12, abs=1e-14)

"""Random-phase initial condition (src/ic.f90:190-269), condensed_particles
and spectrum (src/io.f90:315-404, 632-725) and the filtered field
(src/io.f90:533-628): the library's cuFFT path against the loop restatement
in oracle/spectral_ref.py, plus CPU checks of the oracle itself."""
import math

import numpy as np
import pytest

from oracle import spectral_ref as ref

SMALL = [(8, 8, 8), (12, 10, 10), (9, 7, 7), (16, 6, 6), (10, 8, 6)]


def _rng_field(shape, seed, mean=1.0, amp=0.3):
    rng = np.random.default_rng(seed)
    return mean + amp * (rng.standard_normal(shape) + 1j * rng.standard_normal(shape))


# --- oracle checks (CPU) ---------------------------------------------------------

def test_splitmix_matches_published_sequence():
    # SplitMix64 from state 0: the first three outputs of the published generator
    want = [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F]
    got = ref.splitmix_phases(0, 3)
    assert got.tolist() == [(w >> 11) * 2.0 ** -53 for w in want]


def test_kc_amp_constants():
    from gpe_b200.spectral import kc_amp
    amp, kc2 = kc_amp(128, 128, 128, 0.75, 0.75)
    ev = (64 / math.pi) ** 2 * 0.75
    assert kc2 == pytest.approx(1.666666666666666 * ev / 0.75, rel=1e-15)
    assert amp == pytest.approx(math.sqrt(0.11095279993106999 * 0.75 ** 2.5 * 128 ** 3
                                          / ev ** 1.5), rel=1e-15)


@pytest.mark.parametrize("n", [1, 2, 7, 8, 9, 64])
def test_index_magnitude_rule(n):
    # i <= (n-1)/2 + 1 -> i^2, else (n - i)^2
    assert [ref._k2(i, n - 1) for i in range(n)] == \
        [i * i if i <= (n - 1) // 2 + 1 else (n - i) ** 2 for i in range(n)]


def test_shell_thresholds_are_far_from_integers():
    """The device assigns shells by comparing k2 / (4 pi^2) with powers of 4
    instead of taking logarithms; the two agree unless an integer k2 sits
    within rounding of 4 pi^2 4^s.  None does for |s| <= 7."""
    for s in range(-7, 8):
        t = 4.0 * math.pi ** 2 * 4.0 ** s
        if t < 1:
            continue
        assert abs(t - round(t)) / t > 1e-9


@pytest.mark.parametrize("shape", SMALL)
def test_fast_forms_match_loops(shape):
    nx, ny, nz = shape
    psi = _rng_field((nz, ny, nx), 3)
    xr, yr, zr = 0.5 * (nx - 1), 0.4 * (ny - 1), 0.3 * (nz - 1)
    row, a = ref.condensed_particles(psi, xr, yr, zr)
    frow, fa = ref.condensed_fast(psi, xr, yr, zr)
    np.testing.assert_allclose(fa, a, rtol=0, atol=1e-13 * np.abs(a).max())
    for k, v in row.items():
        assert frow[k] == pytest.approx(v, rel=1e-12), k
    eta, nharm, F = ref.spectrum(a)
    feta, fnharm, fF = ref.spectrum_fast(a)
    assert fnharm.tolist() == nharm.tolist()
    np.testing.assert_allclose(feta, eta, rtol=1e-12)
    np.testing.assert_allclose(fF, F, rtol=1e-12)


def test_random_phase_oracle_properties():
    """|a| = comp_amp inside the cutoff, zero outside; Parseval; a shell
    wholly inside the cutoff has eta = comp_amp^2."""
    n, nv, enerv = 24, 1.0, 8.0
    from gpe_b200.spectral import kc_amp
    amp, kc2 = kc_amp(n, n, n, nv, enerv)
    ph = ref.splitmix_phases(5, n ** 3).reshape(n, n, n)
    psi = ref.random_phase(n, n, n, nv, enerv, ph)
    np.testing.assert_allclose(ref.random_phase_fast(n, n, n, nv, enerv, ph), psi, rtol=0,
                               atol=1e-13 * np.abs(psi).max())
    a = np.fft.ifftn(psi) * n ** 3 / math.sqrt(n ** 3)
    inside = ref.k2_grid(n, n, n) <= kc2
    assert 0 < inside.sum() < n ** 3
    np.testing.assert_allclose(np.abs(a[inside]), amp, rtol=1e-12)
    assert np.abs(a[~inside]).max() < 1e-10 * amp
    assert np.sum(np.abs(psi) ** 2) == pytest.approx(amp ** 2 * inside.sum(), rel=1e-12)
    eta, nharm, _ = ref.spectrum_fast(a)
    assert math.sqrt(kc2) > 4 * math.pi  # shell 1: pi < |k| < 4 pi
    assert eta[0] == pytest.approx(amp ** 2, rel=1e-12)


def test_filter_oracle_is_identity_for_a_wide_filter_band():
    psi = _rng_field((6, 6, 8), 9)
    # m = 0: the filter factor is 1 everywhere
    np.testing.assert_allclose(ref.filtered(psi, 3.0, 0.0), psi, rtol=0, atol=1e-13)


# --- the library on the GPU ------------------------------------------------------

def _solver(shape, precision=16, xr=None):
    from gpe_b200 import GpeParams, GpeSolver
    nx, ny, nz = shape
    xr = xr or (0.5 * (nx - 1), 0.5 * (ny - 1), 0.5 * (nz - 1))
    prm = GpeParams(nx=nx, ny=ny, nz=nz, xr=xr[0], yr=xr[1], zr=xr[2], scheme="rk4",
                    eqn_to_solve=4, bcs=1, order=2, precision=precision, g=1.0, mu=1.0)
    return GpeSolver(prm, dt=0.01)


@pytest.mark.gpu
@pytest.mark.parametrize("shape", SMALL)
def test_gpu_random_phase_matches_oracle(shape):
    nx, ny, nz = shape
    nv, enerv, seed = 1.0, 3.0, 1234
    with _solver(shape) as s:
        amp, kc2 = s.random_phase(nv, enerv, seed)
        got = s.get_state()
    from gpe_b200.spectral import kc_amp
    assert (amp, kc2) == pytest.approx(kc_amp(nx, ny, nz, nv, enerv), rel=1e-15)
    ph = ref.splitmix_phases(seed, nx * ny * nz).reshape(nz, ny, nx)
    exp = ref.random_phase(nx, ny, nz, nv, enerv, ph)
    np.testing.assert_allclose(got, exp, rtol=0, atol=1e-12 * np.abs(exp).max())


@pytest.mark.gpu
@pytest.mark.parametrize("shape", SMALL)
def test_gpu_condensed_particles_matches_oracle(shape):
    nx, ny, nz = shape
    psi = _rng_field((nz, ny, nx), 11)
    xr = (0.5 * (nx - 1), 0.4 * (ny - 1), 0.3 * (nz - 1))
    with _solver(shape, xr=xr) as s:
        s.set_state(psi)
        c = s.condensed_particles()
        assert np.array_equal(s.get_state(), psi)  # the transform only reads psi
    row, a = ref.condensed_particles(psi, *xr)
    for k, v in row.items():
        assert c.row[k] == pytest.approx(v, rel=1e-10), k
    eta, nharm, F = ref.spectrum(a)
    assert c.nharm.tolist() == nharm.tolist()
    np.testing.assert_allclose(c.eta, eta, rtol=1e-11)
    np.testing.assert_allclose(c.F, F, rtol=1e-11)


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(8, 8, 8), (12, 10, 10), (9, 7, 7)])
def test_gpu_filtered_field_matches_oracle(shape):
    nx, ny, nz = shape
    psi = _rng_field((nz, ny, nx), 12)
    with _solver(shape) as s:
        s.set_state(psi)
        got = s.filtered_field(4.0, 1.0)
        state_after = s.get_state()
    np.testing.assert_allclose(got, ref.filtered(psi, 4.0, 1.0), rtol=0, atol=1e-12)
    assert np.array_equal(state_after, psi)  # psi itself is not changed


@pytest.mark.gpu
def test_gpu_random_phase_example_128():
    """The reference's random_phase example (128^3, nv = enerv = 0.75):
    state against the oracle's transform, diagnostics against the vectorised
    oracle, and the same numbers from complex64 storage within its rounding."""
    n, nv, enerv, seed = 128, 0.75, 0.75, 7
    with _solver((n, n, n)) as s:
        amp, kc2 = s.random_phase(nv, enerv, seed)
        psi = s.get_state()
        c = s.condensed_particles()
        c2 = s.condensed_particles()
        mass, _ = s.diagnostics()
        assert np.array_equal(s.get_state(), psi)
    ph = ref.splitmix_phases(seed, n ** 3).reshape(n, n, n)
    a_exp = np.where(ref.k2_grid(n, n, n) <= kc2, amp * np.exp(2j * math.pi * ph), 0.0)
    exp = np.fft.fftn(a_exp) / math.sqrt(n ** 3)
    np.testing.assert_allclose(psi, exp, rtol=0, atol=1e-12 * np.abs(exp).max())
    row, a = ref.condensed_fast(psi, *(0.5 * (n - 1),) * 3)
    for k, v in row.items():
        assert c.row[k] == pytest.approx(v, rel=1e-10), k
    assert c.row["M"] == pytest.approx(mass, rel=1e-12)
    eta, nharm, F = ref.spectrum_fast(a)
    assert c.nharm.tolist() == nharm.tolist()
    # shells outside the cutoff hold only rounding noise (~1e-31): absolute floor
    np.testing.assert_allclose(c.eta, eta, rtol=1e-10, atol=1e-12 * eta.max())
    np.testing.assert_allclose(c.F, F, rtol=1e-10)
    # deterministic reduction: the same numbers bit for bit on a second call
    assert np.array_equal(c.eta, c2.eta) and np.array_equal(c.F, c2.F) and c.row == c2.row
    with _solver((n, n, n), precision=8) as s8:
        s8.random_phase(nv, enerv, seed)
        c8 = s8.condensed_particles()
    assert c8.nharm.tolist() == nharm.tolist()
    np.testing.assert_allclose(c8.eta, eta, rtol=1e-5, atol=1e-6 * eta.max())
    np.testing.assert_allclose(c8.F, F, rtol=1e-5)


@pytest.mark.gpu
def test_gpu_spectral_rejects_bad_arguments():
    from gpe_b200 import GpeError
    with _solver((8, 8, 8)) as s:
        with pytest.raises(GpeError):
            s.random_phase(0.0, 1.0)
        with pytest.raises(GpeError):
            s.filtered_field(0.0)

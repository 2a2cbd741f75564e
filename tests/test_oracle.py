"""CPU tests of the oracle: analytic known-answer tests and the cross-check
against the independent numpy restatement.  The reference ships no golden
vectors, so these are what pin the oracle (see oracle/__init__.py)."""
import itertools
import math

import numpy as np
import pytest

import oracle
from oracle.ref_numpy import NumpyGPE
from tests.conftest import rel_l2, random_field

# ---------------------------------------------------------------------------
# scalar recurrences for plane waves / eigenmodes


def rk_scalar(F, a, dt, scheme):
    if scheme == "euler":
        return a + dt * F(a)
    if scheme == "rk2":
        return a + dt * F(a + 0.5 * dt * F(a))
    if scheme == "rk4":
        k1 = F(a); k2 = F(a + 0.5 * dt * k1); k3 = F(a + 0.5 * dt * k2); k4 = F(a + dt * k3)
        return a + dt * (k1 / 6 + k2 / 3 + k3 / 3 + k4 / 6)
    raise ValueError(scheme)


def symbol2(kh, h, order):
    """-(discrete second derivative) of exp(ikx) / exp(ikx)."""
    if order == 2:
        return (2 - 2 * math.cos(kh)) / h ** 2
    return (30 - 32 * math.cos(kh) + 2 * math.cos(2 * kh)) / (12 * h ** 2)


def symbol1(kh, h, order):
    """(discrete first derivative) of exp(ikx) / (i exp(ikx))."""
    if order == 2:
        return math.sin(kh) / h
    return (8 * math.sin(kh) - math.sin(2 * kh)) / (6 * h)


def make(n, xr, **kw):
    prm = oracle.OracleParams(nx=n[0], ny=n[1], nz=n[2], xr=xr[0], yr=xr[1], zr=xr[2], **kw)
    return oracle.Oracle(prm)


@pytest.mark.parametrize("scheme", ["euler", "rk2", "rk4"])
@pytest.mark.parametrize("order", [2, 4])
@pytest.mark.parametrize("eqn", [1, 2, 4])
def test_plane_wave_periodic(scheme, order, eqn):
    n = (12, 10, 8)
    xr = (3.3, 2.9, 2.1)
    U = 0.37 if eqn in (1, 2) else 0.0
    o = make(n, xr, scheme=scheme, eqn_to_solve=eqn, bcs=1, order=order, g=1.7, mu=0.6,
             Urhs=U)
    x, y, z = o.grid()
    h = [2 * r / (m - 1) for r, m in zip(xr, n)]
    m = (2, -1, 3)
    k = [2 * math.pi * mm / (nn * hh) for mm, nn, hh in zip(m, n, h)]
    kap2 = sum(symbol2(kk * hh, hh, order) for kk, hh in zip(k, h))
    sx = symbol1(k[0] * h[0], h[0], order)
    A = 0.8 + 0.3j
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    phase = np.exp(1j * (k[0] * X + k[1] * Y + k[2] * Z))
    psi = A * phase

    def F(a):
        a2 = abs(a) ** 2
        if eqn == 4:
            return -1j * (0.5 * kap2 + 1.7 * a2 - 0.6) * a
        if eqn == 2:
            return 1j * (-kap2 - a2) * a + U * 1j * sx * a
        return 0.5j * (-kap2 + 1 - a2) * a + U * 1j * sx * a

    dt = 0.013
    tm = oracle.OraTime(0, 0, dt, 0, 0)
    a = A
    for _ in range(5):
        psi, _, _ = o.solver(psi, tm)
        a = rk_scalar(F, a, dt, scheme)
    assert rel_l2(psi, a * phase) < 1e-13
    assert tm.t == pytest.approx(5 * dt, abs=1e-15)


@pytest.mark.parametrize("order", [2, 4])
def test_reflective_cosine_eigenmode(order):
    n = (11, 9, 13)
    xr = (2.5, 2.0, 3.0)
    o = make(n, xr, scheme="rk4", eqn_to_solve=4, bcs=2, order=order, g=0.0, mu=0.4)
    x, y, z = o.grid()
    h = [2 * r / (m - 1) for r, m in zip(xr, n)]
    m = (3, 2, 5)
    Z, Y, X = np.meshgrid(np.arange(n[2]), np.arange(n[1]), np.arange(n[0]), indexing="ij")
    mode = (np.cos(math.pi * m[0] * X / (n[0] - 1)) * np.cos(math.pi * m[1] * Y / (n[1] - 1))
            * np.cos(math.pi * m[2] * Z / (n[2] - 1)))
    kap2 = sum(symbol2(math.pi * mm / (nn - 1), hh, order) for mm, nn, hh in zip(m, n, h))
    lam = -1j * (0.5 * kap2 - 0.4)
    dt = 0.02
    z_ = lam * dt
    R = 1 + z_ + z_ ** 2 / 2 + z_ ** 3 / 6 + z_ ** 4 / 24
    psi = (0.7 - 0.2j) * mode
    tm = oracle.OraTime(0, 0, dt, 0, 0)
    for _ in range(4):
        psi, _, _ = o.solver(psi, tm)
    assert rel_l2(psi, (0.7 - 0.2j) * R ** 4 * mode) < 1e-13


@pytest.mark.parametrize("order,expect", [(2, 2.0), (4, 4.0)])
def test_laplacian_convergence_order(order, expect):
    errs = []
    for n in (16, 32):
        L = 6.0
        h = L / n
        xr = h * (n - 1) / 2
        o = make((n, 6, 6), (xr, 1.0, 1.0), eqn_to_solve=4, bcs=1, order=order)
        x, _, _ = o.grid()
        f = np.broadcast_to(np.sin(2 * math.pi * x / L)[None, None, :], (6, 6, n)) + 0j
        lap = o.laplacian(f)
        exact = -(2 * math.pi / L) ** 2 * f
        errs.append(np.max(np.abs(lap - exact)))
    rate = math.log2(errs[0] / errs[1])
    assert abs(rate - expect) < 0.15


def test_norm_weights_exact_for_constants_and_linear():
    n = (9, 7, 11)
    xr = (2.0, 1.5, 3.0)
    o = make(n, xr)
    x, y, z = o.grid()
    ones = np.ones((n[2], n[1], n[0]), complex)
    vol = 8 * xr[0] * xr[1] * xr[2]
    assert o.get_norm(ones) == pytest.approx(vol, rel=1e-14)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    lin = np.sqrt(np.abs(1.0 + 0.1 * X))  # |psi|^2 = 1 + 0.1 x  (linear)
    assert o.get_norm(lin + 0j) == pytest.approx(vol, rel=1e-13)


def test_norm_of_gaussian():
    n = 48
    xr = 6.0
    o = make((n, n, n), (xr, xr, xr))
    x, y, z = o.grid()
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    psi = np.exp(-(X ** 2 + Y ** 2 + Z ** 2) / 2) + 0j  # |psi|^2 integrates to pi^1.5
    assert o.get_norm(psi) == pytest.approx(math.pi ** 1.5, rel=1e-7)


def test_energy_plane_wave():
    n = (10, 8, 12)
    xr = (2.0, 1.7, 2.4)
    o = make(n, xr, order=4)
    x, y, z = o.grid()
    h = [2 * r / (m - 1) for r, m in zip(xr, n)]
    k = [2 * math.pi * mm / (nn * hh) for mm, nn, hh in zip((1, 2, -1), n, h)]
    kap2 = sum(symbol2(kk * hh, hh, 4) for kk, hh in zip(k, h))
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    A = 0.9
    psi = A * np.exp(1j * (k[0] * X + k[1] * Y + k[2] * Z))
    E = o.energy(psi)
    expect = (kap2 * A ** 2 + 0.5 * A ** 4) * np.prod(n) * h[0] * h[1] * h[2]
    assert E == pytest.approx(expect, rel=1e-12)


COMBOS = list(itertools.product([1, 2, 3, 4], [1, 2], [2, 4], ["euler", "rk2", "rk4", "rk45"],
                                [True, False]))


@pytest.mark.parametrize("eqn,bcs,order,scheme,rt", COMBOS)
def test_oracle_matches_numpy(eqn, bcs, order, scheme, rt):
    n = (12, 10, 9)
    kw = dict(Urhs=0.3, diss_amp=0.2, g=1.3, mu=0.9, omx=0.3, omy=0.2, omz=0.4)
    o = make(n, (5.0, 4.0, 3.5), scheme=scheme, eqn_to_solve=eqn, bcs=bcs, order=order,
             real_time=rt, **kw)
    ref = NumpyGPE(*n, 5.0, 4.0, 3.5, eqn=eqn, bcs=bcs, order=order, real_time=rt, **kw)
    psi = random_field((n[2], n[1], n[0]), seed=eqn * 100 + order)
    dt = 0.01 if rt else -0.01j
    tm = oracle.OraTime(0.0, 0.0, dt.real, dt.imag, 0)
    out, _, _ = o.solver(psi, tm)
    if scheme == "rk45":
        exp, dt_did, dt_next, _ = ref.rkqs(psi, dt)
        # errmax is a max of |embedded difference| / psi_scal: the difference
        # cancels ~8 digits, so two FP64 restatements agree to ~1e-9 in it
        # and in dt_next = 0.9 dt errmax^-0.2
        assert complex(tm.dt_re, tm.dt_im) == pytest.approx(dt_next, rel=1e-8)
    else:
        exp = ref.step(psi, dt, scheme)
    assert rel_l2(out, exp) < 1e-13
    assert o.get_norm(psi) == pytest.approx(ref.norm(psi), rel=1e-13)
    assert o.energy(psi) == pytest.approx(ref.energy(psi), rel=1e-12)


def test_rk45_rejects_and_retries():
    n = (10, 10, 10)
    o = make(n, (4.0, 4.0, 4.0), scheme="rk45", eqn_to_solve=2, bcs=1, order=4)
    ref = NumpyGPE(*n, 4.0, 4.0, 4.0, eqn=2, bcs=1, order=4)
    psi = random_field((10, 10, 10), seed=7, amp=0.5)
    tm = oracle.OraTime(0.0, 0.0, 0.2, 0.0, 0)
    out, errmax, att = o.solver(psi, tm)
    exp, dt_did, dt_next, em = ref.rkqs(psi, 0.2)
    assert att > 1
    assert errmax <= 1.0 and errmax == pytest.approx(em, rel=1e-10)
    assert tm.t == pytest.approx(dt_did.real, rel=1e-13)
    assert rel_l2(out, exp) < 1e-13


def test_imaginary_time_rk45_quirk_and_direction():
    """rkqs adds |Im(dt_next)| to im_t (src/solve.f90:227-229)."""
    n = (8, 8, 8)
    o = make(n, (3.0, 3.0, 3.0), scheme="rk45", eqn_to_solve=4, bcs=2, order=2,
             real_time=False, omx=1.0, omy=1.0, omz=1.0)
    psi = random_field((8, 8, 8), seed=3, amp=0.1)
    tm = oracle.OraTime(0.0, 0.0, 0.0, -1e-3, 0)
    o.solver(psi, tm)
    assert tm.t == 0.0
    assert tm.dt_re == 0.0 and tm.dt_im < 0
    assert tm.im_t == pytest.approx(abs(tm.dt_im), rel=1e-15)


def test_unknown_scheme_rejected():
    prm = oracle.OracleParams(nx=8, ny=8, nz=8, xr=1, yr=1, zr=1)
    o = oracle.Oracle(prm)
    o._h  # context exists
    bad = oracle.OracleParams(nx=8, ny=8, nz=8, xr=1, yr=1, zr=1)
    ob = oracle.Oracle(bad)
    # scheme codes outside 0..3 reach the default branch, like the reference's
    # 'ERROR: Unrecognised time stepping scheme.' (src/solve.f90:47-49)
    import ctypes
    p = oracle._OraParams(8, 8, 8, 1, 1, 1, 7, 4, 1, 2, 1, 0, 0, 1, 1, 1, 1, 0, 0, 0)
    h = oracle.lib().ora_create(ctypes.byref(p))
    psi = np.ones(512, complex)
    out = np.zeros_like(psi)
    tm = oracle.OraTime(0, 0, 0.01, 0, 0)
    rc = oracle.lib().ora_solver(h, oracle._dp(psi.view(np.float64)), oracle._dp(out.view(np.float64)),
                                 ctypes.byref(tm), None, None)
    oracle.lib().ora_destroy(h)
    assert rc == -1
    del o, ob


def test_drive_imaginary_time_renorm():
    """Imaginary-time ground state: norm renormalised to nn each step."""
    n = (10, 10, 10)
    prm = oracle.OracleParams(nx=10, ny=10, nz=10, xr=4, yr=4, zr=4, scheme="rk4", eqn_to_solve=4,
                              bcs=2, order=2, real_time=False, g=1.0, mu=1.0, nn=1.0,
                              omx=1.0, omy=1.0, omz=1.0)
    o = oracle.Oracle(prm)
    psi = o.ic_fermi() + 0.01
    tm = oracle.OraTime(0.0, 0.0, 0.0, -0.005, 0)
    psi, rec = oracle.drive(o, psi, tm, 5, renorm=True)
    assert o.get_norm(psi) == pytest.approx(1.0, rel=1e-12)
    assert len(rec) == 5 and tm.p == 5


def test_product_ring_and_pulse_ics_match_the_oracle():
    """gpe_b200.ic's ring and pulse initial conditions (used by the rkf45
    workload) against the oracle's restatement of src/ic.f90."""
    from gpe_b200 import ic
    n = (20, 18, 16)
    xr, yr, zr = 12.0, 11.0, 9.0
    o = oracle.Oracle(oracle.OracleParams(nx=n[0], ny=n[1], nz=n[2], xr=xr, yr=yr, zr=zr))
    x, y, z = (np.linspace(-xr, xr, n[0]), np.linspace(-yr, yr, n[1]), np.linspace(-zr, zr, n[2]))
    got = ic.vortex_ring_xy(x, y, z, 0.5, -0.3, 0.2, 6.0, amp=0.4, mm=3, r1=0.7, kk=2)
    exp = o.ic_vortex_ring("xy", 0.5, -0.3, 0.2, 6.0, amp=0.4, mm=3, r1=0.7, kk=2)
    np.testing.assert_allclose(got, exp, rtol=1e-13, atol=1e-14)
    for which in ("ring", "pulse"):
        got = ic.pade_pulse_ring(x, y, z, which, -4.0, 0.5, -0.5, 1.5)
        exp = o.ic_pade_pulse_ring(which, -4.0, 0.5, -0.5, 1.5)
        np.testing.assert_allclose(got, exp, rtol=1e-13, atol=1e-14)


def test_mass_and_momentum_restatement():
    """mass (src/variables.f90:590-610) and momentum (:615-694): mass is the
    plain sum times the cell volume; momentum of a plane wave exp(i k x)
    follows from the FD symbol, checked against numpy with the oracle's
    own derivative and the norm's integration weights."""
    n = (16, 12, 10)
    for order, bcs in ((2, 1), (4, 1), (4, 2)):
        o = oracle.Oracle(oracle.OracleParams(nx=n[0], ny=n[1], nz=n[2], xr=6.0, yr=5.0, zr=4.0,
                                              order=order, bcs=bcs))
        rng = np.random.default_rng(order + bcs)
        psi = 1.0 + 0.3 * (rng.standard_normal((n[2], n[1], n[0])) +
                           1j * rng.standard_normal((n[2], n[1], n[0])))
        dx, dy, dz = 12.0 / 15, 10.0 / 11, 8.0 / 9
        assert o.mass(psi) == pytest.approx(np.sum(np.abs(psi) ** 2) * dx * dy * dz, rel=1e-13)
        mom = o.momentum(psi)
        # same integrand and weights through independent numpy code
        w = (np.array([_w_y(k, n[2]) for k in range(n[2])])[:, None, None] *
             np.array([_w_y(j, n[1]) for j in range(n[1])])[None, :, None] *
             _w_x(n[0])[None, None, :])
        for a in range(3):
            d = o.deriv(psi, a, False)
            f = (psi.real - 1.0) * np.imag(np.conj(d)) - psi.imag * d.real
            assert mom[a] == pytest.approx(np.sum(w * f) * dx * dy * dz, rel=1e-12, abs=1e-12)


def _w_x(n):
    w = np.zeros(n)
    w[0] += 3 / 8; w[1] += 7 / 6; w[2] += 23 / 24
    w[3:n - 3] += 1.0
    w[n - 3] += 23 / 24; w[n - 2] += 7 / 6; w[n - 1] += 3 / 8
    return w


def _w_y(i, n):
    w = 1.0
    for idx, val in ((0, 3 / 8), (1, 7 / 6), (2, 23 / 24), (n - 3, 23 / 24), (n - 2, 7 / 6),
                     (n - 1, 3 / 8)):
        if i == idx:
            w = val
    return w

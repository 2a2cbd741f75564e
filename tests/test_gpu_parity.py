"""GPU parity: the CUDA path through the C-ABI against the CPU oracle on the
same seeded inputs.

Tolerances (FP64 storage vs the FP64 oracle): relative L2 of psi <= 1e-12,
relative norm / energy <= 1e-12 -- both compute the same arithmetic in a
different order.  rk45 step sizes: <= 1e-8 relative (the embedded error
estimate cancels ~8 digits, see tests/test_oracle.py).  Complex64 storage:
<= 2e-6 per step against FP64, Kahan runs as stated in each test."""
import itertools
import math

import numpy as np
import pytest

import oracle
from gpe_b200 import GpeError, GpeParams, GpeSolver, run_loop
from tests.conftest import rel_l2, random_field

pytestmark = pytest.mark.gpu

KW = dict(Urhs=0.3, diss_amp=0.2, g=1.3, mu=0.9, omx=0.3, omy=0.2, omz=0.4)


def pair(n, xr, scheme="rk4", eqn=4, bcs=1, order=2, rt=True, precision=16, kahan=False,
         **kw):
    prm = GpeParams(nx=n[0], ny=n[1], nz=n[2], xr=xr[0], yr=xr[1], zr=xr[2], scheme=scheme,
                    eqn_to_solve=eqn, bcs=bcs, order=order, real_time=rt, precision=precision,
                    kahan=kahan, **kw)
    o = oracle.Oracle(oracle.OracleParams(nx=n[0], ny=n[1], nz=n[2], xr=xr[0], yr=xr[1],
                                          zr=xr[2], scheme=scheme, eqn_to_solve=eqn, bcs=bcs,
                                          order=order, real_time=rt, **kw))
    return GpeSolver(prm), o


COMBOS = list(itertools.product([1, 2, 3, 4], [1, 2], [2, 4], ["euler", "rk2", "rk4", "rk45"],
                                [True, False]))


@pytest.mark.parametrize("eqn,bcs,order,scheme,rt", COMBOS)
def test_one_step_matches_oracle(eqn, bcs, order, scheme, rt):
    n = (70, 13, 11)  # two x tiles (second ragged), ragged y tile
    g, o = pair(n, (8.0, 4.0, 3.5), scheme, eqn, bcs, order, rt, **KW)
    psi = random_field((n[2], n[1], n[0]), seed=eqn * 1000 + bcs * 100 + order)
    dt = 0.01 if rt else -0.01j
    g.dt = dt
    g.set_state(psi)
    g.solver()
    tm = oracle.OraTime(0.0, 0.0, dt.real, dt.imag, 0)
    exp, em, att = o.solver(psi, tm)
    out = g.get_state()
    assert rel_l2(out, exp) < 1e-12
    assert g.t == pytest.approx(tm.t, rel=1e-12, abs=1e-15)
    assert g.im_t == pytest.approx(tm.im_t, rel=1e-8, abs=1e-15)
    if scheme == "rk45":
        assert g.dt == pytest.approx(complex(tm.dt_re, tm.dt_im), rel=1e-8)
        assert g.last_info.attempts == att
    assert g.get_norm() == pytest.approx(o.get_norm(exp), rel=1e-12)
    g.close()


PLAIN_COMBOS = list(itertools.product([1, 2, 4], [1, 2], [2, 4], ["euler", "rk2", "rk4", "rk45"],
                                      [True, False]))


@pytest.mark.parametrize("eqn,bcs,order,scheme,rt", PLAIN_COMBOS)
def test_one_step_plain_rhs_matches_oracle(eqn, bcs, order, scheme, rt):
    """No trap, sponge or gradient term: the kernels' folded right-hand side."""
    n = (66, 19, 10)
    g, o = pair(n, (8.0, 4.0, 3.5), scheme, eqn, bcs, order, rt, g=1.3, mu=0.9)
    psi = random_field((n[2], n[1], n[0]), seed=eqn * 77 + bcs * 7 + order)
    dt = 0.01 if rt else -0.01j
    g.dt = dt
    g.set_state(psi)
    g.solver()
    tm = oracle.OraTime(0.0, 0.0, dt.real, dt.imag, 0)
    exp, em, att = o.solver(psi, tm)
    assert rel_l2(g.get_state(), exp) < 1e-12
    if scheme == "rk45":
        assert g.dt == pytest.approx(complex(tm.dt_re, tm.dt_im), rel=1e-8)
    assert g.get_norm() == pytest.approx(o.get_norm(exp), rel=1e-12)
    assert rel_l2(g.rhs(), o.rhs(g.get_state())) < 1e-12
    g.close()


@pytest.mark.parametrize("eqn,bcs,order", list(itertools.product([1, 2, 3, 4], [1, 2], [2, 4])))
def test_rhs_laplacian_norm_energy(eqn, bcs, order):
    n = (67, 17, 9)
    g, o = pair(n, (9.0, 5.0, 3.0), "rk4", eqn, bcs, order, True, **KW)
    psi = random_field((n[2], n[1], n[0]), seed=11 + eqn)
    g.set_state(psi)
    assert rel_l2(g.rhs(), o.rhs(psi)) < 1e-12
    assert rel_l2(g.laplacian(), o.laplacian(psi)) < 1e-12
    assert g.get_norm() == pytest.approx(o.get_norm(psi), rel=1e-12)
    E, H = g.energy()
    assert E == pytest.approx(o.energy(psi), rel=1e-12)
    if eqn == 4:
        assert H == pytest.approx(o.hamiltonian4(psi), rel=1e-12)
    g.close()


def vortex_line_pade(x, y, z):
    """psi = R(r) e^{i atan2(y,x)}, R = r * get_rr(r) (src/ic.f90:888-901)."""
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    r = np.sqrt(X ** 2 + Y ** 2)
    rr = np.sqrt((0.3437 + 0.0286 * r ** 2) / (1 + 0.3333 * r ** 2 + 0.0286 * r ** 4))
    return r * rr * np.exp(1j * np.arctan2(Y, X))


def test_config_64cube_rk4_100_steps():
    """64^3, h=0.5, periodic, 2nd order, RK4 dt=0.01, 100 steps, equation 4
    with g=mu=1, straight Pade vortex line: complex128 GPU vs FP64 oracle."""
    n = 64
    xr = 0.5 * (n - 1) / 2
    g, o = pair((n, n, n), (xr, xr, xr), "rk4", 4, 1, 2, True, g=1.0, mu=1.0)
    x, y, z = o.grid()
    psi0 = vortex_line_pade(x, y, z)
    g.dt = 0.01
    g.set_state(psi0)
    oracle.set_threads(8)
    tm = oracle.OraTime(0.0, 0.0, 0.01, 0.0, 0)
    psi = psi0
    for _ in range(100):
        psi, _, _ = o.solver(psi, tm)
    norms = g.advance(100)
    out = g.get_state()
    assert rel_l2(out, psi) < 1e-12
    assert norms[-1] == pytest.approx(o.get_norm(psi), rel=1e-12)
    assert g.energy()[0] == pytest.approx(o.energy(psi), rel=1e-12)
    assert g.t == pytest.approx(1.0, rel=1e-13)
    g.close()


def test_rk45_reflective_order4_multi_step():
    n = 24
    g, o = pair((n, n, n), (4.6, 4.6, 4.6), "rk45", 4, 2, 4, True, g=1.0, mu=1.0)
    x, y, z = o.grid()
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    psi = np.tanh(np.sqrt((X - 1) ** 2 + Y ** 2) + 0.1) * np.exp(1j * np.arctan2(Y, X - 1))
    g.dt = 0.005
    g.set_state(psi)
    tm = oracle.OraTime(0.0, 0.0, 0.005, 0.0, 0)
    for _ in range(8):
        psi, _, _ = o.solver(psi, tm)
        g.solver()
    assert rel_l2(g.get_state(), psi) < 1e-10
    assert g.t == pytest.approx(tm.t, rel=1e-9)
    assert g.dt.real == pytest.approx(tm.dt_re, rel=1e-7)
    g.close()


def test_complex64_kahan_rk45_one_step_and_run():
    """One rk45 call at equal dt matches FP64 to FP32 accuracy.  Over several
    calls the adaptive dt sequences part: errmax is formed from FP32 stage
    values whose rounding (~1e-9 absolute) is ~1e-3 of the 1e-6 tolerance, so
    each dt_next carries ~1e-3 relative noise; the run is then compared at
    the tolerance that time offset implies."""
    n = (64, 24, 20)
    g, o = pair(n, (8.0, 3.0, 2.5), "rk45", 4, 1, 4, True, precision=8, kahan=True,
                g=1.0, mu=1.0)
    psi = random_field((n[2], n[1], n[0]), seed=5, amp=0.2)
    g.dt = 0.002
    g.set_state(psi)
    tm = oracle.OraTime(0.0, 0.0, 0.002, 0.0, 0)
    g.solver()
    exp, em, att = o.solver(psi, tm)
    assert g.last_info.attempts == att
    assert g.t == pytest.approx(tm.t, rel=1e-12)
    assert rel_l2(g.get_state(), exp) < 2e-6
    assert g.dt.real == pytest.approx(tm.dt_re, rel=2e-2)
    for _ in range(10):
        exp, _, _ = o.solver(exp, tm)
        g.solver()
    assert g.t == pytest.approx(tm.t, rel=2e-2)
    assert rel_l2(g.get_state(), exp) < 5e-3
    g.close()


@pytest.mark.parametrize("scheme", ["euler", "rk2", "rk4"])
def test_complex64_kahan_close_to_fp64(scheme):
    n = (64, 24, 20)
    g, o = pair(n, (8.0, 3.0, 2.5), scheme, 4, 1, 4, True, precision=8, kahan=True,
                g=1.0, mu=1.0)
    psi = random_field((n[2], n[1], n[0]), seed=5, amp=0.2)
    g.dt = 0.002
    g.set_state(psi)
    tm = oracle.OraTime(0.0, 0.0, 0.002, 0.0, 0)
    for _ in range(20):
        psi, _, _ = o.solver(psi, tm)
        g.solver()
    assert rel_l2(g.get_state(), psi) < 5e-6
    g.close()


def test_complex64_plain_one_step():
    n = (40, 20, 12)
    g, o = pair(n, (5.0, 3.0, 2.0), "rk4", 4, 2, 2, True, precision=8, g=1.0, mu=1.0)
    psi = random_field((n[2], n[1], n[0]), seed=9)
    g.dt = 0.01
    g.set_state(psi)
    g.solver()
    exp, _, _ = o.solver(psi, oracle.OraTime(0, 0, 0.01, 0, 0))
    assert rel_l2(g.get_state(), exp) < 2e-6
    g.close()


def test_state_roundtrip_and_dtypes():
    n = (33, 7, 6)
    g, _ = pair(n, (3.0, 2.0, 2.0))
    psi = random_field((n[2], n[1], n[0]), seed=2)
    g.set_state(psi)
    assert np.array_equal(g.get_state(), psi)
    g.set_state(psi.astype(np.complex64))
    assert np.array_equal(g.get_state(np.complex64), psi.astype(np.complex64))
    g.close()


def test_solver_host_is_the_resident_step():
    n = (30, 12, 10)
    g, o = pair(n, (4.0, 2.0, 2.0), "rk4", 4, 2, 4, True, g=1.0, mu=1.0)
    psi = random_field((n[2], n[1], n[0]), seed=21)
    g.dt = 0.01
    out = g.solver_host(psi)
    exp, _, _ = o.solver(psi, oracle.OraTime(0, 0, 0.01, 0, 0))
    assert rel_l2(out, exp) < 1e-12
    g.close()


def test_imaginary_time_loop_matches_oracle_drive():
    n = (20, 20, 20)
    kw = dict(g=1.0, mu=1.0, nn=1.0, omx=1.0, omy=1.0, omz=1.0)
    g, o = pair(n, (4.0, 4.0, 4.0), "rk4", 4, 2, 2, False, **kw)
    psi = o.ic_fermi() + 0.05
    g.dt = -0.005j
    g.set_state(psi)
    rec_g = run_loop(g, 6, renorm=True)
    tm = oracle.OraTime(0.0, 0.0, 0.0, -0.005, 0)
    psi_o, rec_o = oracle.drive(o, psi, tm, 6, renorm=True)
    assert rel_l2(g.get_state(), psi_o) < 1e-12
    for a, b in zip(rec_g, rec_o):
        assert a[2] == pytest.approx(b[2], rel=1e-12)
        assert a[1] == pytest.approx(b[1], rel=1e-12)
    assert g.p == tm.p == 6
    g.close()


def test_renormalise():
    n = (16, 16, 16)
    g, o = pair(n, (3.0, 3.0, 3.0), nn=2.0)
    psi = random_field((16, 16, 16), seed=4)
    g.set_state(psi)
    nrm = g.get_norm()
    g.renormalise(nrm)
    assert g.get_norm() == pytest.approx(2.0, rel=1e-12)
    assert rel_l2(g.get_state(), o.renormalise(psi, nrm)) < 1e-15
    g.close()


def test_unknown_scheme_fails_at_solver_like_the_reference():
    prm = GpeParams(nx=8, ny=8, nz=8, scheme="bogus")
    g = GpeSolver(prm, tau=0.01)
    g.set_state(np.ones((8, 8, 8), complex))
    with pytest.raises(GpeError) as e:
        g.solver()
    assert e.value.code == 2 and "Unrecognised time stepping scheme" in str(e.value)
    g.close()


@pytest.mark.parametrize("n", [(6, 6, 6), (129, 9, 7), (64, 64, 8)])
def test_edge_sizes(n):
    g, o = pair(n, (3.0, 2.0, 1.5), "rk4", 2, 1, 4, True, Urhs=0.2)
    psi = random_field((n[2], n[1], n[0]), seed=sum(n))
    g.dt = 0.003
    g.set_state(psi)
    g.solver()
    exp, _, _ = o.solver(psi, oracle.OraTime(0, 0, 0.003, 0, 0))
    assert rel_l2(g.get_state(), exp) < 1e-12
    g.close()


def test_timing_and_launch_count():
    n = (64, 32, 32)
    g, _ = pair(n, (4.0, 2.0, 2.0), "rk4", 4, 1, 4)
    g.set_state(random_field((32, 32, 64), seed=1))
    g.dt = 0.001
    g.set_timing(True)
    c0 = g.launch_count()
    g.advance(3)
    assert g.launch_count() - c0 == 3 * 5
    t = g.timing()
    assert t["stage_mid"]["launches"] == 6 and t["stage_mid"]["ms"] > 0
    g.close()


def test_c2_rkf45_configuration_matches_oracle():
    """128^3, h=0.4, reflective, order 4, rkf45 from the ring x pulse state:
    the first three adaptive steps (psi, accepted dt, attempts) against the
    oracle."""
    import bench
    psi = bench.c2_initial_state()
    p = bench.c2_params(16, False)
    g = GpeSolver(p, dt=0.005)
    g.set_state(psi)
    o = oracle.Oracle(oracle.OracleParams(nx=p.nx, ny=p.ny, nz=p.nz, xr=p.xr, yr=p.yr, zr=p.zr,
                                          scheme="rk45", eqn_to_solve=4, bcs=2, order=4,
                                          g=1.0, mu=1.0))
    tm = oracle.OraTime(0.0, 0.0, 0.005, 0.0, 0)
    q = psi
    for _ in range(3):
        info = g.solver()
        q, em, att = o.solver(q, tm)
        assert info.attempts == att
        assert g.dt == pytest.approx(complex(tm.dt_re, tm.dt_im), rel=1e-8)
        # t sums the accepted steps, which agree to the rk45 dt tolerance
        assert g.t == pytest.approx(tm.t, rel=1e-8)
    assert rel_l2(g.get_state(), q) < 1e-9
    g.close()


@pytest.mark.parametrize("order,bcs,precision", [(2, 1, 16), (4, 1, 16), (4, 2, 16), (2, 2, 8)])
def test_mass_and_momentum_match_oracle(order, bcs, precision):
    n = (70, 13, 11)
    g, o = pair(n, (8.0, 4.0, 3.5), "rk4", 4, bcs, order, True, precision=precision)
    psi = random_field((n[2], n[1], n[0]), seed=order * 10 + bcs)
    if precision == 8:
        psi = psi.astype(np.complex64).astype(np.complex128)
    g.set_state(psi)
    m, mom = g.diagnostics()
    tol = 1e-12 if precision == 16 else 1e-6
    assert m == pytest.approx(o.mass(psi), rel=tol)
    np.testing.assert_allclose(mom, o.momentum(psi), rtol=tol, atol=tol * np.abs(mom).max())
    g.close()


def test_checkpoint_round_trip_through_the_solver(tmp_path):
    n = (40, 12, 10)
    g, o = pair(n, (8.0, 4.0, 3.5), "rk4", 4, 1, 4, True)
    psi = random_field((n[2], n[1], n[0]), seed=5)
    g.dt = 0.01
    g.set_state(psi)
    g.advance(3)
    g.p = 3
    f = str(tmp_path / "end_state.dat")
    g.save_end_state(f)
    g.advance(2)
    ref = g.get_state()
    h, _ = pair(n, (8.0, 4.0, 3.5), "rk4", 4, 1, 4, True)
    h.dt = 0.01
    h.load_end_state(f)
    assert (h.p, h.t) == (3, pytest.approx(0.03))
    h.advance(2)
    assert np.array_equal(h.get_state(), ref)
    g.close()
    h.close()


def test_device_wait_timeout_is_reported_and_the_context_survives():
    """A device wait on a flag nothing sets runs out after 20 ms, the status
    reaches the host as GPE_ERR_TIMEOUT, and the same context then steps
    exactly as before."""
    from gpe_b200 import GpeError
    n = (24, 10, 8)
    g, o = pair(n, (6.0, 3.0, 2.5), "rk4", 4, 1, 2, True)
    psi = random_field((n[2], n[1], n[0]), seed=3)
    g.dt = 0.01
    g.set_state(psi)
    with pytest.raises(GpeError) as e:
        g.wait_probe(20_000_000)
    assert e.value.code == 6
    g.solver()
    tm = oracle.OraTime(0.0, 0.0, 0.01, 0.0, 0)
    exp, _, _ = o.solver(psi, tm)
    assert rel_l2(g.get_state(), exp) < 1e-12
    g.close()


def test_non_finite_state_is_reported():
    from gpe_b200 import GpeError
    n = (24, 10, 8)
    g, _ = pair(n, (6.0, 3.0, 2.5), "rk4", 4, 1, 2, True)
    psi = random_field((n[2], n[1], n[0]), seed=4)
    psi[3, 4, 5] = np.nan
    g.dt = 0.01
    g.set_state(psi)
    g.solver()
    with pytest.raises(GpeError) as e:
        g.get_norm()
    assert e.value.code == 5
    g.close()


@pytest.mark.parametrize("scheme,order,bcs,kahan", [("rk4", 4, 1, False), ("rk4", 2, 2, True),
                                                    ("rk45", 4, 2, False), ("euler", 2, 1, True)])
def test_stage_kernel_waits_run_out_and_the_context_survives(scheme, order, bcs, kahan):
    """The stage kernels' own pipeline waits run out: with the test hook the
    producer warps never load plane 1, the compute warps' wait for it (limit
    20 ms) runs out and the step returns GPE_ERR_TIMEOUT instead of hanging
    (the recipes with a per-item reduction exercise the compute warps' shared
    barrier on the abort path), energy() too; with the hook off and the
    default limit restored the same context steps exactly like the oracle."""
    from gpe_b200 import GpeError
    n = (130, 24, 20)
    g, o = pair(n, (8.0, 4.0, 3.5), scheme, 4, bcs, order, True,
                precision=8 if kahan else 16, kahan=kahan)
    psi = random_field((n[2], n[1], n[0]), seed=11)
    g.dt = 0.01
    g.set_state(psi)
    g.set_wait_limit(20_000_000)
    g.test_stall(1)
    for _ in range(2):
        with pytest.raises(GpeError) as e:
            g.solver()
        assert e.value.code == 6
    with pytest.raises(GpeError) as e:
        g.energy()
    assert e.value.code == 6
    g.test_stall(-1)
    g.set_wait_limit(0)
    g.t, g.dt = 0.0, 0.01
    g.set_state(psi)
    g.solver()
    tm = oracle.OraTime(0.0, 0.0, 0.01, 0.0, 0)
    exp, _, _ = o.solver(psi, tm)
    assert rel_l2(g.get_state(), exp) < (2e-6 if kahan else 1e-12)
    g.close()


@pytest.mark.parametrize("precision,kahan,bcs,rt", [(16, False, 2, True), (8, True, 1, True),
                                                    (16, False, 1, False)])
def test_rk45_advance_equals_single_steps(precision, kahan, bcs, rt):
    """rk45 advance(n): n accepted steps from captured WHILE-node graphs with
    the step control on the device, bitwise equal to n solver() calls (which
    run the same kernels) and to the host-driven attempt loop (timing on),
    with the per-step dt and attempts recorded."""
    n = (40, 20, 16)
    kw = dict(precision=precision, kahan=kahan, omx=0.3, omy=0.2, omz=0.4, g=1.3, mu=0.9)
    psi = random_field((n[2], n[1], n[0]), seed=21)
    dt0 = 0.02 if rt else -0.02j
    runs = []
    for mode in ("advance", "solver", "timed"):
        g, _ = pair(n, (8.0, 4.0, 3.5), "rk45", 4, bcs, 4, rt, **kw)
        g.dt = dt0
        g.set_state(psi)
        if mode == "timed":
            g.set_timing(True)
        if mode == "solver":
            infos = [g.solver() for _ in range(12)]
            series = ([i.dt_did_re if rt else i.dt_did_im for i in infos],
                      [i.attempts for i in infos])
            norms = None
        else:
            norms = g.advance(12)
            d, a = g.step_series(12)
            series = (list(d), list(a))
        runs.append((g.get_state(np.complex128), g.t, g.im_t, g.dt, series, norms))
        g.close()
    (s0, t0, i0, d0, ser0, n0), (s1, t1, i1, d1, ser1, _), (s2, t2, i2, d2, ser2, n2) = runs
    assert np.array_equal(s0, s1) and np.array_equal(s0, s2)
    assert (t0, i0, d0) == (t1, i1, d1) == (t2, i2, d2)
    if rt:
        assert ser0 == ser1 == ser2
    assert np.array_equal(n0, n2)
    assert max(ser0[1]) >= 1


def test_rk45_advance_halts_on_a_non_finite_error_estimate():
    n = (24, 10, 8)
    g, _ = pair(n, (6.0, 3.0, 2.5), "rk45", 4, 1, 2, True)
    psi = random_field((n[2], n[1], n[0]), seed=4)
    psi[3, 4, 5] = np.nan
    g.dt = 0.01
    g.set_state(psi)
    with pytest.raises(GpeError) as e:
        g.advance(5)
    assert e.value.code == 5
    g.close()


@pytest.mark.parametrize("r", [0.5, 0.8])
def test_dispersion_matched_laplacian(r):
    """fd_match = r: per-axis coefficients c1 = (4 - r^2)/(3 h^2), c2 =
    (r^2 - 1)/(12 h^2) of the 4th-order stencil, checked against numpy on a
    periodic random field, and its symbol against the 2nd-order Laplacian of
    spacing r h on a plane wave to the stated order."""
    n = (24, 20, 16)
    xr = (6.0, 5.0, 4.0)
    h = [2 * a / (m - 1) for a, m in zip(xr, n)]
    prm = GpeParams(nx=n[0], ny=n[1], nz=n[2], xr=xr[0], yr=xr[1], zr=xr[2], order=4, bcs=1,
                    fd_match=r)
    psi = random_field((n[2], n[1], n[0]), seed=3)
    with GpeSolver(prm) as s:
        s.set_state(psi)
        got = s.laplacian()
    exp = np.zeros_like(psi)
    for ax, hh in zip((2, 1, 0), h):
        c1 = (4 - r * r) / (3 * hh * hh)
        c2 = (r * r - 1) / (12 * hh * hh)
        exp += c1 * (np.roll(psi, 1, ax) + np.roll(psi, -1, ax)) + \
            c2 * (np.roll(psi, 2, ax) + np.roll(psi, -2, ax)) - 2 * (c1 + c2) * psi
    assert rel_l2(got, exp) < 1e-12
    with pytest.raises(GpeError):
        GpeSolver(GpeParams(nx=8, ny=8, nz=8, order=2, fd_match=0.5))


@pytest.mark.parametrize("precision,kahan,order,bcs,trap", [(8, True, 4, 1, False),
                                                            (8, False, 2, 2, True),
                                                            (16, False, 4, 2, False)])
def test_launch_shape_does_not_change_the_state(precision, kahan, order, bcs, trap):
    """Every site is computed by the same arithmetic whatever the tile height
    (4 or 8 rows; the complex64 two-field stages then run 2 or 4 warps of two
    rows each), the planes per CTA (a ragged last chunk of 3) or the
    library's own choice, so five rk4 steps leave the same state bit for bit."""
    n = (70, 13, 11)  # two x tiles (second ragged), ragged y tiles
    kw = dict(g=1.3, mu=0.9)
    if trap:
        kw.update(omx=0.3, omy=0.2, omz=0.4)
    psi = random_field((n[2], n[1], n[0]), seed=31 + order)
    if precision == 8:
        psi = psi.astype(np.complex64)
    states = []
    for ty, zc in ((0, 0), (4, 0), (8, 0), (4, 3), (8, 5)):
        prm = GpeParams(nx=n[0], ny=n[1], nz=n[2], xr=8.0, yr=4.0, zr=3.5, scheme="rk4",
                        eqn_to_solve=4, bcs=bcs, order=order, precision=precision, kahan=kahan,
                        tile_y=ty, zchunk=zc, **kw)
        with GpeSolver(prm, dt=0.01) as s:
            s.set_state(psi)
            for _ in range(5):
                s.solver()
            states.append((s.get_state(), s.get_norm()))
    for st, nm in states[1:]:
        assert np.array_equal(st, states[0][0])
        assert nm == pytest.approx(states[0][1], rel=1e-12)

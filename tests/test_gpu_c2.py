"""The C2 configuration held to the oracle over the whole run.

128^3 grid, h = 0.4, reflective boundaries, 4th-order differences, adaptive
rkf45 (Cash-Karp stages + rkqs step control, src/solve.f90:158-378) with
tolerance 1e-6 from dt = 0.005, equation 4 (g = mu = 1), from the vortex ring
(r0 = 8) times the Pade rarefaction pulse at x0 = -10, stepped while
t + im_t <= 20 as the reference loop does (src/gpe.f90:134).

complex128 on the GPU against the FP64 oracle, step by step: the same
attempt count every step, accepted and next dt within 1e-8 (the embedded
error estimate cancels about 8 digits, so two FP64 implementations agree on
errmax to ~1e-9), and at the end psi within 1e-9 relative L2, norm and
energy within 1e-9.  complex64 + Kahan with FP64 step control, on its own
step sequence, against the same oracle state: density within 5e-3 relative
L2 (its FP32 error estimates choose different steps, and its last step ends
at a slightly different time).
"""
import os

import numpy as np
import pytest

import bench
import oracle
from gpe_b200 import GpeSolver
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu

T_END = 20.0


def _oracle(p):
    return oracle.Oracle(oracle.OracleParams(nx=p.nx, ny=p.ny, nz=p.nz, xr=p.xr, yr=p.yr,
                                             zr=p.zr, scheme="rk45", eqn_to_solve=4, bcs=2,
                                             order=4, g=1.0, mu=1.0))


@pytest.fixture(scope="module")
def c2_run():
    """The oracle's whole run with the GPU complex128 run beside it, compared
    step by step."""
    oracle.set_threads(os.cpu_count() or 1)
    psi0 = bench.c2_initial_state()
    p = bench.c2_params(16, False)
    g = GpeSolver(p, dt=0.005)
    g.set_state(psi0)
    o = _oracle(p)
    tm = oracle.OraTime(0.0, 0.0, 0.005, 0.0, 0)
    q = psi0
    steps = attempts = 0
    worst_dt = 0.0
    while tm.t + tm.im_t <= T_END:
        t_before = tm.t
        info = g.solver()
        q, em, att = o.solver(q, tm)
        steps += 1
        attempts += att
        assert info.attempts == att, f"step {steps}: {info.attempts} attempts vs {att}"
        dt_did = tm.t - t_before
        assert info.dt_did_re == pytest.approx(dt_did, rel=1e-8), f"step {steps}"
        assert g.dt == pytest.approx(complex(tm.dt_re, tm.dt_im), rel=1e-8), f"step {steps}"
        worst_dt = max(worst_dt, abs(g.dt.real - tm.dt_re) / tm.dt_re)
    out = {"steps": steps, "attempts": attempts, "t": tm.t, "psi": q, "gpu_psi": g.get_state(),
           "gpu_t": g.t, "gpu_norm": g.get_norm(), "gpu_E": g.energy()[0],
           "norm": o.get_norm(q), "E": o.energy(q), "worst_dt": worst_dt}
    g.close()
    o.close()
    return out


def test_c2_complex128_whole_run_matches_oracle(c2_run):
    r = c2_run
    # the reference run takes about 516 accepted steps in about 529 attempts
    assert 400 < r["steps"] < 700 and r["attempts"] >= r["steps"]
    assert r["gpu_t"] == pytest.approx(r["t"], rel=1e-9)
    assert rel_l2(r["gpu_psi"], r["psi"]) < 1e-9
    assert r["gpu_norm"] == pytest.approx(r["norm"], rel=1e-9)
    assert r["gpu_E"] == pytest.approx(r["E"], rel=1e-9)


def test_c2_complex64_kahan_tracks_the_oracle(c2_run):
    r = c2_run
    psi0 = bench.c2_initial_state()
    s = GpeSolver(bench.c2_params(8, True), dt=0.005)
    s.set_state(psi0.astype(np.complex64))
    steps = 0
    while s.t + s.im_t <= T_END:
        s.solver()
        steps += 1
    got = s.get_state(np.complex128)
    s.close()
    dens = rel_l2(np.abs(got) ** 2, np.abs(r["psi"]) ** 2)
    assert dens < 5e-3, (dens, steps, r["steps"])

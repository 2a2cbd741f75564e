"""A run directory in the reference's input format, driven on the GPU.

tests/golden/run_trap holds run.in / parameters.in / ic.in with the settings
of the reference's trap_vortex example on a 40^3 grid: equation 4 in
imaginary time, rk2, reflective boundaries, a harmonic trap, the initial
condition fermi() * vortex_line(vl1) and imprint_vl (|psi| times the line's
phase after every step).  inputs.run reads the three files and steps it; the
oracle does the same steps from its own restatement of the initial-condition
functions: psi within 1e-12 relative L2, the norms per step within 1e-12,
and the reference's output files written."""
import os
import shutil

import numpy as np
import pytest

import oracle
from gpe_b200 import inputs
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "run_trap")


def test_trap_vortex_run_dir_matches_oracle(tmp_path):
    d = tmp_path / "run"
    shutil.copytree(FIXTURE, d)
    steps = 6
    s, rec = inputs.run(str(d), max_steps=steps)
    got = s.get_state()
    t, im_t = s.t, s.im_t
    s.close()

    p = inputs.load_run(FIXTURE).prm
    o = oracle.Oracle(oracle.OracleParams(nx=p.nx, ny=p.ny, nz=p.nz, xr=p.xr, yr=p.yr, zr=p.zr,
                                          scheme="rk2", eqn_to_solve=4, bcs=2, order=2,
                                          real_time=False, g=p.g, mu=p.mu, omx=p.omx,
                                          omy=p.omy, omz=p.omz))
    line = o.ic_vortex_line(-1.5, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0, "z", True)
    psi0 = o.ic_fermi() * line
    tm = oracle.OraTime(0.0, 0.0, 0.0, -1e-4, 0)
    exp, orec = oracle.drive(o, psi0, tm, steps, stop_imag=True, imprint=line)
    assert len(rec) == len(orec) == steps
    assert rel_l2(got, exp) < 1e-12
    assert im_t == pytest.approx(tm.im_t, rel=1e-12) and t == 0.0
    for (a, b) in zip(rec, orec):
        assert a[2] == pytest.approx(b[2], rel=1e-12)
    for f in ("energy.dat", "norm.dat", "psi_time.dat", "RUNNING"):
        assert (d / f).exists(), f
    dens = sorted(os.listdir(d / "proc00"))
    assert any(n.startswith("dens") for n in dens)

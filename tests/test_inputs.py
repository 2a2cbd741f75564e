"""The reference's run inputs (run.in namelists, parameters.in, ic.in) and the
initial-condition functions of src/ic.f90 that ic.in combines, on CPU.

The initial conditions are checked against the oracle's C restatement of
src/ic.f90 on small grids (<= 1e-13 relative: same formulas, libm against
numpy transcendental rounding).  The reference's own example directories are
parsed when the reference tree is present (it is not on the GPU box)."""
import os
import shutil

import numpy as np
import pytest

import oracle
from gpe_b200 import ic, inputs
from gpe_b200.inputs import InputError, fortran_value, parse_ic_in, parse_namelists

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FIXTURE = os.path.join(ROOT, "tests", "golden", "run_trap")
REF_EXAMPLES = "/root/reference/examples"


def test_fortran_literals():
    assert fortran_value(".true.") is True and fortran_value(".FALSE.") is False
    assert fortran_value("T") is True and fortran_value("f") is False
    assert fortran_value("'rk45'") == "rk45"
    assert fortran_value("'don''t'") == "don't"
    assert fortran_value("12") == 12 and fortran_value("-3") == -3
    assert fortran_value("1.0d-3") == pytest.approx(1e-3)
    assert fortran_value("2.5_pr") == 2.5 and fortran_value("-48.0_pr") == -48.0
    assert fortran_value("1e2") == 100.0
    with pytest.raises(InputError):
        fortran_value("'open")
    with pytest.raises(InputError):
        fortran_value("abc")


def test_namelists_commas_comments_and_case():
    nl = parse_namelists("""
    ! comment
    &RUN_PARAMS tau = 0.5, Scheme='rk4' ! trailing
      bcs = 2
    /
    &eqn_params g=1.0d0, mu=2 /
    """)
    assert nl["run_params"] == {"tau": 0.5, "scheme": "rk4", "bcs": 2}
    assert nl["eqn_params"] == {"g": 1.0, "mu": 2}


def test_fixture_run_dir():
    s = inputs.load_run(FIXTURE)
    p = s.prm
    assert (p.nx, p.ny, p.nz, p.precision) == (40, 40, 40, 16)
    assert (p.scheme, p.eqn_to_solve, p.bcs, p.order, p.real_time) == ("rk2", 4, 2, 2, False)
    assert (p.g, p.mu, p.omz, p.xr) == (5.0, 8.0, 2.0, 12.0)
    assert s.tau == 1e-4 and s.end_time == 10.0 and s.stop_imag and s.imprint_vl
    assert s.outputs.save_rate == 2 and s.outputs.save_3d and not s.outputs.save_ll
    assert s.ic == [("fermi", []), ("vortex_line", ["vl1"])]
    assert s.consts["vl1"] == {"x0": -1.5, "y0": 0.0, "z0": 0.0, "amp1": 0.0, "amp2": 0.0,
                               "ll": 0.0, "sgn": 1.0, "dir": "z", "imprint_phase": True}
    assert s.consts["vr1"]["plane"] == "yz" and s.consts["vr1"]["mm"] == 5
    assert s.procs == (1, 2)


def test_bad_inputs_are_rejected(tmp_path):
    d = tmp_path / "run"
    shutil.copytree(FIXTURE, d)
    run_in = (d / "run.in").read_text()
    (d / "run.in").write_text(run_in.replace("&misc_params", "&misc_paramz"))
    with pytest.raises(InputError, match="misc_params"):
        inputs.load_run(str(d))
    (d / "run.in").write_text(run_in.replace("  g        = 5.0", "  gee      = 5.0"))
    with pytest.raises(InputError, match="unknown names"):
        inputs.load_run(str(d))
    (d / "run.in").write_text(run_in)
    (d / "ic.in").write_text("init_cond = fermi() * vortex_line(vl9)\n")
    with pytest.raises(InputError, match="vl9"):
        inputs.load_run(str(d))
    with pytest.raises(InputError, match="unknown"):
        parse_ic_in("init_cond = tornado()")
    with pytest.raises(InputError, match="arguments"):
        parse_ic_in("init_cond = vortex_ring()")
    with pytest.raises(InputError):
        parse_ic_in("psi = fermi()")


@pytest.mark.skipif(not os.path.isdir(REF_EXAMPLES), reason="reference tree not present")
@pytest.mark.parametrize("name,expect", [
    ("ring", dict(scheme="rk45", eqn=1, pr=16, n=128, ic=[("vortex_ring", ["vr1"])])),
    ("random_phase", dict(scheme="rk45", eqn=2, pr=8, n=128, ic=[("random_phase", [])])),
    ("trap_vortex", dict(scheme="rk2", eqn=4, pr=16, n=120,
                         ic=[("fermi", []), ("vortex_line", ["vl1"])])),
])
def test_reference_examples_parse(tmp_path, name, expect):
    d = tmp_path / name
    d.mkdir()
    for f in ("run.in", "parameters.in", "ic.in"):
        shutil.copy(os.path.join(REF_EXAMPLES, name, f + ".dist"), d / f)
    s = inputs.load_run(str(d))
    assert s.prm.scheme == expect["scheme"] and s.prm.eqn_to_solve == expect["eqn"]
    assert s.prm.precision == expect["pr"] and s.prm.nx == expect["n"]
    assert s.ic == expect["ic"]
    assert "vl1" in s.consts and "vr1" in s.consts


def _orc(n, xr, **kw):
    return oracle.Oracle(oracle.OracleParams(nx=n[0], ny=n[1], nz=n[2], xr=xr[0], yr=xr[1],
                                             zr=xr[2], **kw))


def _axes(n, xr):
    return [-r + np.arange(m) * (2 * r / (m - 1)) for m, r in zip(n, xr)]


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("direction", ["x", "y", "z"])
@pytest.mark.parametrize("imprint", [False, True])
def test_vortex_line_matches_oracle(direction, imprint):
    n, xr = (14, 12, 10), (5.0, 4.0, 3.5)
    o = _orc(n, xr, scal=1.3)
    vl = dict(x0=0.3, y0=-0.4, z0=0.2, amp1=0.5, amp2=0.25, ll=3.0, sgn=-1.0, dir=direction,
              imprint_phase=imprint)
    got = ic.vortex_line(*_axes(n, xr), vl, scal=1.3)
    exp = o.ic_vortex_line(0.3, -0.4, 0.2, 0.5, 0.25, 3.0, -1.0, direction, imprint)
    assert _rel(got, exp) < 1e-13


def test_vortex_line_zero_wavelength_needs_zero_amplitude():
    vl = dict(x0=0.0, y0=0.0, z0=0.0, amp1=0.1, amp2=0.0, ll=0.0, sgn=1.0, dir="z",
              imprint_phase=False)
    with pytest.raises(ValueError, match="wavelength"):
        ic.vortex_line(*_axes((6, 6, 6), (1.0, 1.0, 1.0)), vl)


@pytest.mark.parametrize("plane", ["xy", "xz", "yz"])
def test_vortex_ring_matches_oracle(plane):
    n, xr = (16, 14, 12), (9.0, 8.0, 7.0)
    o = _orc(n, xr, scal=0.9)
    vr = dict(plane=plane, x0=0.5, y0=-0.3, z0=0.2, r0=4.0, amp=0.4, mm=3, r1=0.3, kk=2,
              dir=-1.0)
    got = ic.vortex_ring(*_axes(n, xr), vr, scal=0.9)
    exp = o.ic_vortex_ring(plane, 0.5, -0.3, 0.2, 4.0, 0.4, 3, 0.3, 2, -1.0)
    assert _rel(got, exp) < 1e-13


def test_fermi_matches_oracle():
    n, xr = (12, 10, 8), (6.0, 5.0, 4.0)
    o = _orc(n, xr, g=5.0, mu=8.0, omx=1.0, omy=1.0, omz=2.0)
    got = ic.fermi(*_axes(n, xr), 8.0, 5.0, 1.0, 1.0, 2.0)
    assert _rel(got, o.ic_fermi()) < 1e-14
    assert np.any(got == 0.0) and np.any(got != 0.0)


def test_pade_pulse_ring_matches_oracle():
    n, xr = (12, 10, 8), (8.0, 5.0, 4.0)
    o = _orc(n, xr)
    for which in ("ring", "pulse"):
        got = ic.pade_pulse_ring(*_axes(n, xr), which, -2.0, 0.5, 0.0, 1.5)
        assert _rel(got, o.ic_pade_pulse_ring(which, -2.0, 0.5, 0.0, 1.5)) < 1e-13


def test_initial_state_is_the_product():
    s = inputs.load_run(FIXTURE)
    psi = inputs.initial_state(s)
    x, y, z = _axes((40, 40, 40), (12.0, 12.0, 12.0))
    expect = ic.fermi(x, y, z, 8.0, 5.0, 1.0, 1.0, 2.0) * ic.vortex_line(x, y, z, s.consts["vl1"])
    assert np.array_equal(psi, expect)

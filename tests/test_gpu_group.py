"""The library's multi-slab path with real neighbours, on one GPU.

A SlabGroup holds the z-slabs of a grid as separate contexts split by the
reference's para_range rule (uneven splits), placed with gpe_gpu_set_slab,
stepped together by gpe_group_solver: every stage on every slab, boundary
planes copied into the neighbours' ghost planes, the norm / energy / rk45
error combined across slabs (src/variables.f90:98-358, src/solve.f90:189).
Every site is computed from the same values as in a single-domain context,
so the states are compared bitwise with a single context, and with the
oracle at 1e-12; the norm (a sum in another order) at 1e-12."""
import numpy as np
import pytest

import oracle
from gpe_b200 import GpeError, GpeParams, GpeSolver
from gpe_b200.dist import SlabGroup
from tests.conftest import rel_l2, random_field

pytestmark = pytest.mark.gpu

N = (40, 24, 37)
XR = (8.0, 4.0, 6.0)


def _prm(scheme, bcs, order, precision=16, kahan=False, **kw):
    return GpeParams(nx=N[0], ny=N[1], nz=N[2], xr=XR[0], yr=XR[1], zr=XR[2], scheme=scheme,
                     eqn_to_solve=4, bcs=bcs, order=order, precision=precision, kahan=kahan,
                     g=1.2, mu=0.8, **kw)


# 2 and 3 slabs (12-19 planes): every stage computes the boundary planes
# first and copies them on a side stream while the interior planes run;
# 5 slabs (7-8 planes): slabs under 8 planes step in one launch per stage
@pytest.mark.parametrize("nslabs", [2, 3, 5])
@pytest.mark.parametrize("bcs", [1, 2])
@pytest.mark.parametrize("scheme,order", [("rk4", 4), ("rk45", 4), ("rk2", 2), ("euler", 4)])
def test_group_matches_single_domain_and_oracle(nslabs, bcs, scheme, order):
    prm = _prm(scheme, bcs, order, omx=0.2, omy=0.3, omz=0.25)
    psi = random_field((N[2], N[1], N[0]), seed=nslabs * 10 + bcs)
    dt = 0.02
    with SlabGroup(prm, nslabs, dt=dt) as g, GpeSolver(prm, dt=dt) as s:
        assert [pl.nz for pl in g.plans] == [len(range(*(lambda a, b: (a, b + 1))(*pl.z_range)))
                                             for pl in g.plans]
        g.set_global_state(psi)
        s.set_state(psi)
        o = oracle.Oracle(oracle.OracleParams(nx=N[0], ny=N[1], nz=N[2], xr=XR[0], yr=XR[1],
                                              zr=XR[2], scheme=scheme, eqn_to_solve=4, bcs=bcs,
                                              order=order, g=1.2, mu=0.8, omx=0.2, omy=0.3,
                                              omz=0.25))
        tm = oracle.OraTime(0.0, 0.0, dt, 0.0, 0)
        q = psi
        for _ in range(3):
            gi = g.solver()
            si = s.solver()
            q, em, att = o.solver(q, tm)
            assert gi.attempts == si.attempts == att
            assert g.dt == s.dt
        got = g.get_global_state()
        assert np.array_equal(got, s.get_state())
        assert rel_l2(got, q) < 1e-12
        assert g.get_norm() == pytest.approx(s.get_norm(), rel=1e-12)
        assert g.get_norm() == pytest.approx(o.get_norm(q), rel=1e-12)
        e_g, h_g = g.energy()
        e_s, h_s = s.energy()
        assert e_g == pytest.approx(e_s, rel=1e-12) and h_g == pytest.approx(h_s, rel=1e-12)
        o.close()


@pytest.mark.parametrize("bcs", [1, 2])
def test_group_complex64_kahan_is_bitwise_single_domain(bcs):
    prm = _prm("rk4", bcs, 4, precision=8, kahan=True)
    psi = random_field((N[2], N[1], N[0]), seed=7).astype(np.complex64)
    with SlabGroup(prm, 3, dt=0.02) as g, GpeSolver(prm, dt=0.02) as s:
        g.set_global_state(psi)
        s.set_state(psi)
        for _ in range(5):
            g.solver()
            s.solver()
        assert np.array_equal(g.get_global_state(np.complex64), s.get_state(np.complex64))


@pytest.mark.parametrize("nslabs", [2, 5])
def test_group_stage_launches_boundary_planes_apart_when_slabs_are_deep(nslabs):
    """Slabs of 8 planes or more: each stage is two launches per slab (the
    four boundary planes, then the interior) with the ghost copies between
    them on a side stream; one slab under 8 planes keeps the whole group at
    one launch per stage.  Either way every plane is computed once."""
    prm = _prm("rk4", 1, 4)
    psi = random_field((N[2], N[1], N[0]), seed=3)
    with SlabGroup(prm, nslabs, dt=0.02) as g, GpeSolver(prm, dt=0.02) as s:
        g.set_global_state(psi)
        s.set_state(psi)
        for m in g.members:
            m.set_timing(True)
            m.timing()
        g.solver()
        s.solver()
        deep = all(pl.nz >= 8 for pl in g.plans)
        assert deep == (nslabs == 2)
        for m, pl in zip(g.members, g.plans):
            fam = m.timing()
            for f in ("stage_first", "stage_mid", "stage_last"):
                per_stage = 2 if f == "stage_mid" else 1
                assert fam[f]["launches"] == per_stage * (2 if deep else 1), (f, pl.nz)
                assert fam[f]["sites"] == per_stage * N[0] * N[1] * pl.nz
            m.set_timing(False)
        assert np.array_equal(g.get_global_state(), s.get_state())


@pytest.mark.parametrize("nslabs", [2, 3])
def test_group_rk45_complex64_kahan_is_bitwise_single_domain(nslabs):
    """rk45 in complex64 + Kahan: the group combines the slabs' error maxima
    (a max, independent of order) before its step control, the single context
    reduces its own in the step-control launch; the same attempts, steps and
    states, bit for bit."""
    prm = _prm("rk45", 2, 4, precision=8, kahan=True)
    psi = random_field((N[2], N[1], N[0]), seed=11).astype(np.complex64)
    with SlabGroup(prm, nslabs, dt=0.02) as g, GpeSolver(prm, dt=0.02) as s:
        g.set_global_state(psi)
        s.set_state(psi)
        for _ in range(6):
            gi = g.solver()
            si = s.solver()
            assert gi.attempts == si.attempts
            assert g.dt == s.dt and g.t == s.t
        assert np.array_equal(g.get_global_state(np.complex64), s.get_state(np.complex64))


def test_group_members_refuse_stepping_alone():
    prm = _prm("rk4", 1, 2)
    with SlabGroup(prm, 2, dt=0.01) as g:
        with pytest.raises(GpeError) as e:
            g.members[0].solver()
        assert e.value.code == 1 and "slab group" in str(e.value)
        with pytest.raises(GpeError):
            g.members[1].get_norm()

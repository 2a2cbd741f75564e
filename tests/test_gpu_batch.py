"""Batched ensembles against the same runs stepped one context at a time.

Every member of a batch computes each site with the same arithmetic as a
single-run context of the same right-hand-side form, so fields are compared
BITWISE when all members use the full right-hand side (trap on).  The per-run
norms sum the same per-site values in a different item order: relative
1e-12 (FP64) / 1e-6 (complex64 fields, FP64 sums).  A batch mixing runs with
and without a trap steps all of them with the full right-hand side, where a
lone trap-free run folds the factor i into its coefficients: 1e-13 relative
L2 there (FP64 rounding of the folded coefficients)."""
import numpy as np
import pytest

import oracle
from gpe_b200 import BatchOpts, GpeBatch, GpeParams, GpeSolver
from tests.conftest import rel_l2, random_field

pytestmark = pytest.mark.gpu

DT = 0.01


def member(n, h=0.5, om=0.1, bcs=2, order=2, precision=16, kahan=False, **kw):
    nx, ny, nz = n
    return GpeParams(nx=nx, ny=ny, nz=nz, xr=(nx - 1) * h / 2, yr=(ny - 1) * h / 2,
                     zr=(nz - 1) * h / 2, scheme="rk4", eqn_to_solve=4, bcs=bcs, order=order,
                     real_time=True, precision=precision, kahan=kahan, g=1.0, mu=1.0, omx=om,
                     omy=om, omz=om, **kw)


def states(prms, seed, dtype=np.complex128):
    return [random_field((p.nz, p.ny, p.nx), seed=seed + r).astype(dtype)
            for r, p in enumerate(prms)]


def singles(prms, psis, nsteps):
    out, norms = [], []
    for p, s in zip(prms, psis):
        g = GpeSolver(p, dt=DT)
        g.set_state(s)
        norms.append(g.advance(nsteps))
        out.append(g.get_state(s.dtype))
        g.close()
    return out, np.array(norms)


SHAPES = [(32, 32, 32), (48, 20, 9), (70, 13, 11), (17, 40, 24), (64, 64, 8), (6, 6, 6)]


@pytest.mark.parametrize("bcs,order", [(1, 2), (1, 4), (2, 2), (2, 4)])
def test_fp64_batch_is_bitwise_single_runs(bcs, order):
    prms = [member(n, om=0.05 + 0.02 * r, bcs=bcs, order=order) for r, n in enumerate(SHAPES)]
    psis = states(prms, 100 * bcs + order)
    exp, enorm = singles(prms, psis, 7)
    with GpeBatch(prms, DT) as b:
        b.set_states(psis)
        norms = b.advance(7)
        for r in range(len(prms)):
            got = b[r].get_state()
            assert np.array_equal(got, exp[r]), (r, rel_l2(got, exp[r]))
        np.testing.assert_allclose(norms, enorm, rtol=1e-12)


def test_fp64_batch_matches_oracle():
    prms = [member(n, om=0.12, bcs=2, order=4) for n in [(20, 12, 10), (9, 14, 16)]]
    psis = states(prms, 7)
    with GpeBatch(prms, DT) as b:
        b.set_states(psis)
        norms = b.advance(3)
        for r, p in enumerate(prms):
            o = oracle.Oracle(oracle.OracleParams(
                nx=p.nx, ny=p.ny, nz=p.nz, xr=p.xr, yr=p.yr, zr=p.zr, scheme="rk4",
                eqn_to_solve=4, bcs=2, order=4, g=1.0, mu=1.0, omx=p.omx, omy=p.omy,
                omz=p.omz))
            tm = oracle.OraTime(0.0, 0.0, DT, 0.0, 0)
            psi = psis[r]
            for _ in range(3):
                psi, _, _ = o.solver(psi, tm)
            assert rel_l2(b[r].get_state(), psi) < 1e-12
            assert norms[r, -1] == pytest.approx(o.get_norm(psi), rel=1e-12)


# order 2: the batched two-field stages run two rows per warp, as the single
# contexts do; order 4: one row in the batch against two in the single
# contexts -- the same per-site arithmetic either way
@pytest.mark.parametrize("kahan,order", [(False, 2), (True, 2), (False, 4), (True, 4)])
def test_complex64_batch_is_bitwise_single_runs(kahan, order):
    rng = np.random.default_rng(3)
    sizes = rng.choice([32, 48, 64, 96], size=5)
    prms = [member((int(n),) * 3, om=float(rng.uniform(0.05, 0.15)), precision=8, kahan=kahan,
                   order=order)
            for n in sizes]
    psis = states(prms, 11, np.complex64)
    exp, enorm = singles(prms, psis, 12)
    with GpeBatch(prms, DT) as b:
        b.set_states(psis)
        norms = b.advance(12)
        for r in range(len(prms)):
            got = b[r].get_state(np.complex64)
            assert np.array_equal(got, exp[r]), (r, rel_l2(got, exp[r]))
        np.testing.assert_allclose(norms, enorm, rtol=1e-6)


def test_mixed_trap_and_free_runs():
    prms = [member((40, 24, 16), om=0.1), member((24, 40, 20), om=0.0),
            member((33, 17, 12), om=0.0)]
    psis = states(prms, 21)
    exp, enorm = singles(prms, psis, 5)
    with GpeBatch(prms, DT) as b:
        b.set_states(psis)
        norms = b.advance(5)
        for r in range(3):
            assert rel_l2(b[r].get_state(), exp[r]) < 1e-13
        np.testing.assert_allclose(norms, enorm, rtol=1e-12)


@pytest.mark.parametrize("opts", [BatchOpts(use_graph=False), BatchOpts(tile_y=4),
                                  BatchOpts(zchunk=5), BatchOpts(ctas_per_sm=1, zchunk=3),
                                  BatchOpts(tile_y=4, zchunk=64, ctas_per_sm=2)])
def test_launch_options_do_not_change_results(opts):
    prms = [member(n, om=0.08, order=4) for n in SHAPES[:4]]
    psis = states(prms, 31)
    exp, _ = singles(prms, psis, 4)
    with GpeBatch(prms, DT, opts) as b:
        b.set_states(psis)
        b.advance(4)
        for r in range(len(prms)):
            assert np.array_equal(b[r].get_state(), exp[r])
        info = b.info()
        assert info["items"] >= len(prms) and info["grid"] >= 1
        if opts.tile_y:
            assert info["tile_y"] == opts.tile_y


def test_graph_replays_across_calls_and_dt_change():
    prms = [member(n, om=0.1) for n in [(32, 32, 32), (20, 28, 12)]]
    psis = states(prms, 41)
    # reference: 3 steps at DT then 2 at DT/2, single contexts
    exp = []
    for p, s in zip(prms, psis):
        g = GpeSolver(p, dt=DT)
        g.set_state(s)
        g.advance(3)
        g.dt = DT / 2
        g.advance(2)
        exp.append(g.get_state())
        g.close()
    with GpeBatch(prms, DT) as b:
        b.set_states(psis)
        b.advance(1)
        b.advance(2)
        b.dt = DT / 2
        b.advance(2)
        for r in range(2):
            assert np.array_equal(b[r].get_state(), exp[r])
        assert b.launch_count() == 6 * 5


def test_member_state_reload_between_advances():
    prms = [member(n, om=0.1) for n in [(24, 24, 24), (16, 30, 10)]]
    psis = states(prms, 51)
    with GpeBatch(prms, DT) as b:
        b.set_states(psis)
        first = b.advance(3)
        b.set_states(psis)
        again = b.advance(3)
        np.testing.assert_array_equal(first, again)
        # a member's own norm agrees with the batch's last norm
        assert b[0].get_norm() == pytest.approx(again[0, -1], rel=1e-12)


def test_batch_rejects_mismatched_members():
    from gpe_b200 import GpeError
    with pytest.raises(GpeError):
        GpeBatch([member((16, 16, 16)), member((16, 16, 16), order=4)], DT)
    with pytest.raises(GpeError):
        GpeBatch([member((16, 16, 16), precision=8), member((16, 16, 16))], DT)


def test_autotuner_picks_a_candidate_and_keeps_the_state(tmp_path):
    from gpe_b200.autotune import tune
    prms = [member(n, om=0.1) for n in [(32, 32, 32), (48, 48, 48), (20, 28, 12)]]
    psis = states(prms, 61)
    exp, _ = singles(prms, psis, 3)
    cands = [BatchOpts(tile_y=8, zchunk=16), BatchOpts(tile_y=4, zchunk=8, ctas_per_sm=1)]
    cache = str(tmp_path / "tune.json")
    with GpeBatch(prms, DT) as b:
        b.set_states(psis)
        best, table = tune(b, steps=2, cands=cands, cache_path=cache)
        assert best in cands and len(table) == 2 and all(ms > 0 for _, ms in table)
        assert b.opts == best
        b.advance(3)
        for r in range(len(prms)):
            assert np.array_equal(b[r].get_state(), exp[r])
        # a second tune of the same ensemble is served from the cache
        best2, table2 = tune(b, cands=cands, cache_path=cache)
        assert best2 == best and [t for _, t in table2] == [t for _, t in table]

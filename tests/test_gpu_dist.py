"""The NCCL path of the z-slab decomposition on one GPU.

With one rank and periodic boundaries, both z faces of every stencil field go
through the library's NCCL exchange (the rank sends its boundary planes to
itself) instead of the local wrap, so the result must equal the single-domain
run.  Multi-GPU runs use the same code with real neighbours; the rank plan is
checked against the oracle on CPU ranks in tests/test_dist_cpu.py."""
import numpy as np
import pytest

import oracle
from gpe_b200 import GpeParams, GpeSolver
from gpe_b200.dist import SlabSolver
from tests.conftest import rel_l2, random_field

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scheme,precision,bcs", [("rk4", 16, 1), ("rk45", 16, 1),
                                                   ("rk4", 8, 1), ("rk2", 16, 2)])
def test_single_rank_nccl_exchange_equals_local_ghosts(scheme, precision, bcs):
    n = (66, 12, 14)
    prm = GpeParams(nx=n[0], ny=n[1], nz=n[2], xr=6.0, yr=3.0, zr=3.5, scheme=scheme,
                    eqn_to_solve=4, bcs=bcs, order=4, precision=precision,
                    kahan=(precision == 8), g=1.1, mu=0.9, omz=0.2)
    psi = random_field((n[2], n[1], n[0]), seed=17)
    a = GpeSolver(prm, tau=0.004)
    b = SlabSolver(prm, rank=0, nranks=1, dist=None, tau=0.004)
    a.set_state(psi)
    b.set_global_state(psi)
    for _ in range(4):
        a.solver()
        b.solver()
    assert rel_l2(b.get_state(), a.get_state()) < 1e-15
    assert b.get_norm() == pytest.approx(a.get_norm(), rel=1e-15)
    assert b.t == a.t
    if precision == 16:
        o = oracle.Oracle(oracle.OracleParams(nx=n[0], ny=n[1], nz=n[2], xr=6.0, yr=3.0,
                                              zr=3.5, scheme=scheme, eqn_to_solve=4, bcs=bcs,
                                              order=4, g=1.1, mu=0.9, omz=0.2))
        tm = oracle.OraTime(0.0, 0.0, 0.004, 0.0, 0)
        ref = psi
        for _ in range(4):
            ref, _, _ = o.solver(ref, tm)
        tol = 1e-10 if scheme == "rk45" else 1e-12
        assert rel_l2(b.get_state(), ref) < tol
    a.close()
    b.close()

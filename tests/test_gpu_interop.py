"""Device-pointer hand-off between torch and the library's own streams.

The library steps on non-blocking streams that do not wait for torch's
current stream.  A state produced by a long torch computation (the 256^3
random-phase FFT) and passed straight to set_state must arrive complete;
before the binding ordered the call after torch's queued work, the copy
read a half-written tensor at this size."""
import numpy as np
import pytest

import oracle
from gpe_b200 import GpeParams, GpeSolver
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu


def test_state_from_a_fresh_torch_computation_arrives_complete():
    import torch
    from gpe_b200.ic import random_phase
    n, h = 256, 0.25
    xr = (n - 1) * h / 2
    prm = GpeParams(nx=n, ny=n, nz=n, xr=xr, yr=xr, zr=xr, scheme="rk4", eqn_to_solve=4, bcs=1,
                    order=2, precision=16, g=1.0, mu=1.0)
    s = GpeSolver(prm, dt=0.01)
    psi = random_phase(torch, n, h, 1.0, 100, torch.device("cuda"), torch.complex128)
    s.set_state(psi)  # no synchronisation by the caller
    host = psi.cpu().numpy()
    assert np.array_equal(s.get_state(), host)
    out = torch.zeros_like(psi)
    s.get_state_device(out)
    assert torch.equal(out, psi)
    o = oracle.Oracle(oracle.OracleParams(nx=n, ny=n, nz=n, xr=xr, yr=xr, zr=xr, scheme="rk4",
                                          eqn_to_solve=4, bcs=1, order=2, g=1.0, mu=1.0))
    assert s.energy()[1] == pytest.approx(o.hamiltonian4(host), rel=1e-12)
    s.advance(2)
    tm = oracle.OraTime(0.0, 0.0, 0.01, 0.0, 0)
    q = host
    for _ in range(2):
        q, _, _ = o.solver(q, tm)
    assert rel_l2(s.get_state(), q) < 1e-12
    s.close()

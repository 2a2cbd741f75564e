"""Precision form at full size: complex64 psi with Kahan-compensated RK4
accumulation (FP64 reductions) against complex128 on the same GPU, 512^3
periodic, h = 0.5, 4th order, dt = 0.005, 1000 steps, seeded random-phase
initial condition (|k| <= 1).  Target: relative L2 of the density
|psi|^2 <= 1e-5.  The complex128 path is itself held to the CPU oracle at
1e-12 by tests/test_gpu_parity.py.  Plain complex64 (no compensation) is run
beside it to show what the compensation buys."""
import math

import pytest

from gpe_b200 import GpeParams, GpeSolver
from gpe_b200.ic import random_phase

pytestmark = pytest.mark.gpu

N, H, DT, STEPS = 512, 0.5, 0.005, 1000


def run(torch, psi0, precision, kahan):
    xr = H * (N - 1) / 2
    s = GpeSolver(GpeParams(nx=N, ny=N, nz=N, xr=xr, yr=xr, zr=xr, scheme="rk4",
                            eqn_to_solve=4, bcs=1, order=4, precision=precision,
                            kahan=kahan, g=1.0, mu=1.0), tau=DT)
    s.set_state(psi0)
    norms = s.advance(STEPS)
    out = torch.empty((N, N, N), dtype=torch.complex128 if precision == 16 else torch.complex64,
                      device="cuda:0")
    s.get_state_device(out)
    E, H4 = s.energy()
    s.close()
    return out, norms, H4


def test_complex64_kahan_density_error_1000_steps():
    import torch

    psi0 = random_phase(torch, N, H, 1.0, 0, torch.device("cuda:0"), torch.complex128)
    ref, n64, h64 = run(torch, psi0, 16, False)
    rho_ref = ref.abs() ** 2
    del ref
    k32, n32, h32 = run(torch, psi0, 8, True)
    err_kahan = float(torch.linalg.vector_norm((k32.to(torch.complex128).abs() ** 2) - rho_ref)
                      / torch.linalg.vector_norm(rho_ref))
    del k32
    p32, _, _ = run(torch, psi0, 8, False)
    err_plain = float(torch.linalg.vector_norm((p32.to(torch.complex128).abs() ** 2) - rho_ref)
                      / torch.linalg.vector_norm(rho_ref))
    print(f"density rel L2 after {STEPS} steps: kahan {err_kahan:.3e}, plain {err_plain:.3e}; "
          f"norm drift fp64 {abs(n64[-1] / n64[0] - 1):.2e} kahan {abs(n32[-1] / n32[0] - 1):.2e}")
    assert err_kahan <= 1e-5
    assert math.isfinite(h32) and abs(h32 - h64) / abs(h64) < 1e-5

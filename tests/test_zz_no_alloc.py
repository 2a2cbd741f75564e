"""gpe_gpu_norm_noalloc: get_norm for callers that cannot allocate.

Hosts whose device memory is owned by another allocator -- a framework's
caching allocator, or a driver program that sizes all device memory up front
and treats a later cudaMalloc as an error -- cannot use the context-based
entry points, which allocate their fields and scratch.  gpe_gpu_norm_noalloc
takes the caller's device array and a device output slot and allocates
nothing; its partial sums live in a fixed array compiled into the library.

This file is collected last so that a run stopping at the first failure has
already run every other test.  The device buffers below are allocated by the
test (through torch), never by the entry point.
"""
import ctypes

import numpy as np
import pytest

from gpe_b200 import GpeParams, GpeSolver
from gpe_b200._lib import lib
from tests.conftest import random_field

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [16, 8])
def test_noalloc_norm_matches_context_norm_twice(precision):
    import torch

    n = (70, 13, 11)
    xr = (8.0, 4.0, 3.5)
    psi = random_field((n[2], n[1], n[0]), seed=31)
    host = psi.astype(np.complex128 if precision == 16 else np.complex64)
    s = GpeSolver(GpeParams(nx=n[0], ny=n[1], nz=n[2], xr=xr[0], yr=xr[1], zr=xr[2],
                            precision=precision))
    s.set_state(host)
    expect = s.get_norm()  # the existing, context-based get_norm
    s.close()

    d_psi = torch.from_numpy(host).to("cuda:0")
    d_out = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    L = lib()
    for _ in range(2):  # the shared scratch keeps the last call's contents
        d_out.fill_(-1.0)
        torch.cuda.synchronize()
        rc = L.gpe_gpu_norm_noalloc(ctypes.c_void_p(d_psi.data_ptr()), precision, n[0], n[1],
                                    n[2], xr[0], xr[1], xr[2],
                                    ctypes.cast(ctypes.c_void_p(d_out.data_ptr()),
                                                ctypes.POINTER(ctypes.c_double)), None)
        assert rc == 0, L.gpe_gpu_last_error(None)
        torch.cuda.synchronize()
        assert float(d_out.item()) == pytest.approx(expect, rel=1e-12)


def test_noalloc_rejects_grids_beyond_its_scratch():
    import torch

    d_psi = torch.zeros(16, dtype=torch.complex128, device="cuda:0")
    d_out = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    L = lib()
    limit = 8192  # GPE_NOALLOC_MAX_PLANES
    rc = L.gpe_gpu_norm_noalloc(ctypes.c_void_p(d_psi.data_ptr()), 16, 8, 8, limit + 1,
                                1.0, 1.0, 1.0,
                                ctypes.cast(ctypes.c_void_p(d_out.data_ptr()),
                                            ctypes.POINTER(ctypes.c_double)), None)
    assert rc == 1
    assert b"exceeds the fixed scratch" in L.gpe_gpu_last_error(None)

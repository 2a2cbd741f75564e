"""Device-pointer entry points reject a bad tensor before any launch.

The library reads or writes exactly nx*ny*nz dense complex elements behind a
device pointer.  These CPU tests hand the Python binding tensors that would
make it touch memory outside the allocation (host tensors, other devices,
strided views, wrong shapes or dtypes) and check that GpeError is raised
before the library is called.
"""
import ctypes

import numpy as np
import pytest
import torch

from gpe_b200 import GpeParams, GpeSolver
from gpe_b200._lib import GpeError, device_field
from gpe_b200 import spectral


class FakeCuda:
    """Stands in for a CUDA tensor: only the attributes device_field reads."""

    def __init__(self, shape, dtype=torch.complex128, index=0, contiguous=True):
        self.shape = tuple(shape)
        self.dtype = dtype
        self.device = torch.device("cuda", index)
        self.is_cuda = True
        self._contig = contiguous

    def is_contiguous(self):
        return self._contig

    def contiguous(self):
        return self

    def data_ptr(self):
        raise AssertionError("the pointer must not be taken from a rejected tensor")


SHAPE = (6, 7, 8)


def _solver(precision=16):
    s = object.__new__(GpeSolver)
    s.prm = GpeParams(nx=SHAPE[2], ny=SHAPE[1], nz=SHAPE[0], precision=precision)
    s.shape = SHAPE
    s._ctx = ctypes.c_void_p()
    return s


@pytest.mark.parametrize("t,why", [
    (torch.zeros(SHAPE, dtype=torch.complex128), "CUDA tensor"),
    (FakeCuda(SHAPE, index=1), "cuda:1"),
    (FakeCuda(SHAPE, contiguous=False), "contiguous"),
    (FakeCuda((6, 7, 9)), "shape"),
    (FakeCuda(SHAPE, dtype=torch.float32), "dtype"),
    (FakeCuda(SHAPE, dtype=torch.float64), "dtype"),
])
def test_device_field_rejects(t, why):
    with pytest.raises(GpeError) as e:
        device_field(t, SHAPE, 0, "test")
    assert e.value.code == 1 and why in str(e.value)


def test_device_field_accepts_and_sizes():
    assert device_field(FakeCuda(SHAPE), SHAPE, 0, "t") == 16
    assert device_field(FakeCuda(SHAPE, dtype=torch.complex64), SHAPE, 0, "t") == 8


@pytest.mark.parametrize("bad", [FakeCuda((6, 7, 9)), FakeCuda(SHAPE, contiguous=False),
                                 FakeCuda(SHAPE, dtype=torch.float32), FakeCuda(SHAPE, index=3)])
def test_solver_entry_points_reject_before_the_library(bad):
    s = _solver()
    with pytest.raises(GpeError):
        s.set_state(bad)
    with pytest.raises(GpeError):
        s.get_state_device(bad)
    with pytest.raises(GpeError):
        s.linelength(bad)
    with pytest.raises(GpeError):
        spectral.filtered_field(s, 1.0, out=bad)


def test_filtered_out_must_match_precision():
    # a complex64 out for a complex128 solver would be written past its end
    s = _solver(precision=16)
    with pytest.raises(GpeError) as e:
        spectral.filtered_field(s, 1.0, out=FakeCuda(SHAPE, dtype=torch.complex64))
    assert "precision" in str(e.value)


def test_noalloc_rejects_a_plane_beyond_int_range():
    # nx*ny = 2^31 does not fit the plane loop's index range; the entry
    # point refuses it before any device work (the pointer is never read)
    from gpe_b200._lib import lib
    L = lib()
    out = ctypes.c_double()
    rc = L.gpe_gpu_norm_noalloc(ctypes.c_void_p(0x1000), 16, 65536, 32768, 8,
                                1.0, 1.0, 1.0, ctypes.byref(out), None)
    assert rc == 1
    assert b"nx*ny too large" in L.gpe_gpu_last_error(None)
    assert np.isfinite(out.value)

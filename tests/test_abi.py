"""CPU checks of the C-ABI library: it loads without a GPU, exports exactly
what include/gpe_gpu.h declares, its structs match the ctypes mirror, and
calls without a device fail with a clean status (no compute here)."""
import ctypes
import os
import re
import subprocess

import pytest

from gpe_b200 import _lib
from gpe_b200.build import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gpe_gpu.h")


def declared_functions():
    src = open(HEADER).read() + open(os.path.join(ROOT, "include", "gpe_cnn.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set(re.findall(r"\b(gpe_(?:gpu|batch|cnn|group)_\w+)\s*\(", src))
    return names


@pytest.fixture(scope="module")
def L():
    build()
    return _lib.lib()


def test_every_declared_symbol_is_exported(L):
    names = declared_functions()
    assert len(names) >= 20
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (gpe_(?:gpu|batch|cnn|group)_\w+)", out))
    assert names == exported, (names ^ exported)
    for n in names:
        assert hasattr(L, n)
    assert set(_lib.SIGNATURES) == names


def test_struct_layout_matches_header(L):
    p = _lib.GpeParamsC()
    L.gpe_gpu_default_params(ctypes.byref(p), 16, 16, 16)
    assert p.struct_size == ctypes.sizeof(_lib.GpeParamsC)
    assert (p.nx, p.ny, p.nz, p.scheme, p.eqn_to_solve, p.bcs, p.order) == (16, 16, 16, 2, 4, 1, 2)
    assert p.precision == 16 and p.g == 1.0 and p.nn == 1.0
    assert ctypes.sizeof(_lib.GpeTimeC) == 40
    assert L.gpe_gpu_abi_version() == 1


def test_create_validates_before_touching_a_device(L):
    p = _lib.GpeParamsC()
    L.gpe_gpu_default_params(ctypes.byref(p), 4, 16, 16)
    h = ctypes.c_void_p()
    rc = L.gpe_gpu_create(ctypes.byref(p), ctypes.byref(h))
    assert rc == 1 and not h
    assert b">= 6" in L.gpe_gpu_last_error(None)
    L.gpe_gpu_default_params(ctypes.byref(p), 16, 16, 16)
    p.struct_size = 12
    assert L.gpe_gpu_create(ctypes.byref(p), ctypes.byref(h)) == 1
    L.gpe_gpu_default_params(ctypes.byref(p), 16, 16, 16)
    p.kahan = 1  # kahan needs complex64 storage
    assert L.gpe_gpu_create(ctypes.byref(p), ctypes.byref(h)) == 1


def test_no_device_is_a_clean_error_without_gpu(L):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    p = _lib.GpeParamsC()
    L.gpe_gpu_default_params(ctypes.byref(p), 16, 16, 16)
    h = ctypes.c_void_p()
    rc = L.gpe_gpu_create(ctypes.byref(p), ctypes.byref(h))
    assert rc == 7 and not h
    assert L.gpe_gpu_last_error(None)
    with pytest.raises(_lib.GpeError):
        _lib.check(rc)


def test_null_context_calls_are_rejected(L):
    assert L.gpe_gpu_solver(None, None, None) == 1
    assert L.gpe_gpu_norm(None, None) == 1
    # diagnostics entry points check the context before touching a device
    assert L.gpe_gpu_random_phase(None, 1.0, 1.0, 0, None, None) == 1
    assert L.gpe_gpu_condensed_particles(None, None, None, None, None, 0) == 1
    assert L.gpe_gpu_filtered_field(None, 1.0, 1.0, None, 16, 0) == 1
    assert L.gpe_gpu_linelength(None, None) == 1
    assert L.gpe_gpu_zeros(None, None, None, 0) == 1
    assert L.gpe_gpu_get_site(None, 0, 0, 0, None) == 1
    assert L.gpe_gpu_launch_count(None) == -1
    L.gpe_gpu_destroy(None)


def test_batch_create_validates_members_without_gpu(L):
    p = (_lib.GpeParamsC * 2)()
    for q in p:
        L.gpe_gpu_default_params(ctypes.byref(q), 16, 16, 16)
    o = _lib.GpeBatchOptsC()
    L.gpe_batch_default_opts(ctypes.byref(o))
    assert o.struct_size == ctypes.sizeof(_lib.GpeBatchOptsC) and o.use_graph == 1
    h = ctypes.c_void_p()
    # members must share order / bcs / precision
    p[1].order = 4
    assert L.gpe_batch_create(p, 2, ctypes.byref(o), ctypes.byref(h)) == 1 and not h
    assert b"share" in L.gpe_batch_last_error(None)
    p[1].order = 2
    p[1].scheme = 3  # batches step with rk4 only
    assert L.gpe_batch_create(p, 2, ctypes.byref(o), ctypes.byref(h)) == 1
    p[1].scheme = 2
    o.tile_y = 5
    assert L.gpe_batch_create(p, 2, ctypes.byref(o), ctypes.byref(h)) == 1
    o.tile_y = 0
    o.struct_size = 4
    assert L.gpe_batch_create(p, 2, ctypes.byref(o), ctypes.byref(h)) == 1
    assert L.gpe_batch_create(p, 0, None, ctypes.byref(h)) == 1
    assert L.gpe_batch_advance(None, 1, 0.01, 0.0, None) == 1
    assert L.gpe_batch_launch_count(None) == -1
    L.gpe_batch_destroy(None)


def test_new_entry_points_validate_without_a_device(L):
    # slab groups need >= 2 members; null arguments are refused
    g = ctypes.c_void_p()
    assert L.gpe_group_create(None, 0, ctypes.byref(g)) == 1 and not g
    assert b"2 members" in L.gpe_group_last_error(None)
    arr = (ctypes.c_void_p * 2)(None, None)
    assert L.gpe_group_create(arr, 2, ctypes.byref(g)) == 1
    assert b"null member" in L.gpe_group_last_error(None)
    # per-context hooks refuse a null context
    assert L.gpe_gpu_set_wait_limit(None, 1000) == 1
    assert L.gpe_gpu_test_stall(None, 0) == 1
    assert L.gpe_gpu_step_series(None, 1, None, None) == 1
    # fd_match needs order 4 and 0 < r < 1.5, checked before any device call
    p = _lib.GpeParamsC()
    L.gpe_gpu_default_params(ctypes.byref(p), 16, 16, 16)
    p.order, p.fd_match = 2, 0.5
    h = ctypes.c_void_p()
    assert L.gpe_gpu_create(ctypes.byref(p), ctypes.byref(h)) == 1
    assert b"fd_match" in L.gpe_gpu_last_error(None)
    p.order, p.fd_match = 4, 2.0
    assert L.gpe_gpu_create(ctypes.byref(p), ctypes.byref(h)) == 1

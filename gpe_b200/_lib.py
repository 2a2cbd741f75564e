"""ctypes binding of ``libgpe_gpu.so`` (the C-ABI declared in include/gpe_gpu.h).

The library is loaded from this package directory only.  There is no CPU or
eager fallback: if the shared library is missing, or a call is made without a
B200, the error is raised to the caller.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgpe_gpu.so")

GPE_OK = 0
STATUS_NAMES = {
    1: "GPE_ERR_INVALID", 2: "GPE_ERR_SCHEME", 3: "GPE_ERR_CUDA", 4: "GPE_ERR_OOM",
    5: "GPE_ERR_NAN", 6: "GPE_ERR_TIMEOUT", 7: "GPE_ERR_NODEVICE", 8: "GPE_ERR_UNDERFLOW",
}
SCHEMES = {"euler": 0, "rk2": 1, "rk4": 2, "rk45": 3}
TIMING_FAMILIES = ["stage_first", "stage_mid", "stage_last", "reduce", "energy", "copy", "other",
                   "spectrum"]


class GpeError(RuntimeError):
    def __init__(self, code: int, msg: str):
        self.code = code
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")


class GpeParamsC(ctypes.Structure):
    _fields_ = [
        ("struct_size", ctypes.c_int32),
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("xr", ctypes.c_double), ("yr", ctypes.c_double), ("zr", ctypes.c_double),
        ("scheme", ctypes.c_int32), ("eqn_to_solve", ctypes.c_int32),
        ("bcs", ctypes.c_int32), ("order", ctypes.c_int32), ("real_time", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("Urhs", ctypes.c_double), ("diss_amp", ctypes.c_double), ("scal", ctypes.c_double),
        ("g", ctypes.c_double), ("mu", ctypes.c_double), ("nn", ctypes.c_double),
        ("omx", ctypes.c_double), ("omy", ctypes.c_double), ("omz", ctypes.c_double),
        ("kahan", ctypes.c_int32), ("device", ctypes.c_int32),
        ("tile_y", ctypes.c_int32), ("zchunk", ctypes.c_int32),
        ("fd_match", ctypes.c_double),
    ]


class GpeTimeC(ctypes.Structure):
    _fields_ = [("t", ctypes.c_double), ("im_t", ctypes.c_double),
                ("dt_re", ctypes.c_double), ("dt_im", ctypes.c_double),
                ("p", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class GpeStepInfoC(ctypes.Structure):
    _fields_ = [("errmax", ctypes.c_double), ("dt_did_re", ctypes.c_double),
                ("dt_did_im", ctypes.c_double), ("attempts", ctypes.c_int32),
                ("underflow", ctypes.c_int32)]


class GpeTimingC(ctypes.Structure):
    _fields_ = [("ms", ctypes.c_double * 8), ("launches", ctypes.c_int64 * 8),
                ("sites", ctypes.c_int64 * 8)]


class GpeBatchOptsC(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_int32), ("tile_y", ctypes.c_int32),
                ("zchunk", ctypes.c_int32), ("ctas_per_sm", ctypes.c_int32),
                ("use_graph", ctypes.c_int32)]


class GpeCnnParamsC(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_int32), ("nx", ctypes.c_int32), ("ny", ctypes.c_int32),
                ("nz", ctypes.c_int32), ("device", ctypes.c_int32), ("train", ctypes.c_int32),
                ("out_scale", ctypes.c_float), ("preserve_norm", ctypes.c_int32)]


# Every symbol include/gpe_gpu.h and include/gpe_cnn.h declare, with (restype, argtypes).
_vp, _i32, _i64, _dp = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)
SIGNATURES = {
    "gpe_gpu_abi_version": (_i32, []),
    "gpe_gpu_default_params": (None, [ctypes.POINTER(GpeParamsC), _i32, _i32, _i32]),
    "gpe_gpu_create": (ctypes.c_int, [ctypes.POINTER(GpeParamsC), ctypes.POINTER(_vp)]),
    "gpe_gpu_destroy": (None, [_vp]),
    "gpe_gpu_last_error": (ctypes.c_char_p, [_vp]),
    "gpe_gpu_grid": (ctypes.c_int, [_vp, _dp, _dp, _dp]),
    "gpe_gpu_set_state": (ctypes.c_int, [_vp, _vp, _i32]),
    "gpe_gpu_get_state": (ctypes.c_int, [_vp, _vp, _i32]),
    "gpe_gpu_set_state_device": (ctypes.c_int, [_vp, _vp, _i32]),
    "gpe_gpu_get_state_device": (ctypes.c_int, [_vp, _vp, _i32]),
    "gpe_gpu_solver": (ctypes.c_int, [_vp, ctypes.POINTER(GpeTimeC), ctypes.POINTER(GpeStepInfoC)]),
    "gpe_gpu_solver_host": (ctypes.c_int, [_vp, _vp, _vp, _i32, ctypes.POINTER(GpeTimeC),
                                           ctypes.POINTER(GpeStepInfoC)]),
    "gpe_gpu_advance": (ctypes.c_int, [_vp, _i64, ctypes.POINTER(GpeTimeC), _dp]),
    "gpe_gpu_norm": (ctypes.c_int, [_vp, _dp]),
    "gpe_gpu_energy": (ctypes.c_int, [_vp, _dp, _dp]),
    "gpe_gpu_diagnostics": (ctypes.c_int, [_vp, _dp, _dp]),
    "gpe_gpu_wait_probe": (ctypes.c_int, [_vp, ctypes.c_uint64]),
    "gpe_gpu_set_wait_limit": (ctypes.c_int, [_vp, ctypes.c_uint64]),
    "gpe_gpu_test_stall": (ctypes.c_int, [_vp, _i32]),
    "gpe_gpu_step_series": (ctypes.c_int, [_vp, _i64, _dp, ctypes.POINTER(_i32)]),
    "gpe_group_create": (ctypes.c_int, [ctypes.POINTER(_vp), _i32, ctypes.POINTER(_vp)]),
    "gpe_group_solver": (ctypes.c_int, [_vp, ctypes.POINTER(GpeTimeC),
                                        ctypes.POINTER(GpeStepInfoC)]),
    "gpe_group_norm": (ctypes.c_int, [_vp, _dp]),
    "gpe_group_energy": (ctypes.c_int, [_vp, _dp, _dp]),
    "gpe_group_destroy": (None, [_vp]),
    "gpe_group_last_error": (ctypes.c_char_p, [_vp]),
    "gpe_gpu_linelength": (ctypes.c_int, [_vp, _dp]),
    "gpe_gpu_linelength_field": (ctypes.c_int, [_vp, _vp, _i32, _dp]),
    "gpe_gpu_zeros": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int64), _dp, _i64]),
    "gpe_gpu_get_site": (ctypes.c_int, [_vp, _i32, _i32, _i32, _dp]),
    "gpe_gpu_get_plane": (ctypes.c_int, [_vp, _i32, _vp, _i32]),
    "gpe_gpu_random_phase": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double,
                                            ctypes.c_uint64, _dp, _dp]),
    "gpe_gpu_condensed_particles": (ctypes.c_int, [_vp, _dp, _dp, ctypes.POINTER(ctypes.c_int64),
                                                   _dp, _i32]),
    "gpe_gpu_filtered_field": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, _vp, _i32,
                                              _i32]),
    "gpe_gpu_renormalise": (ctypes.c_int, [_vp, ctypes.c_double]),
    "gpe_gpu_rhs": (ctypes.c_int, [_vp, _vp, _i32]),
    "gpe_gpu_laplacian": (ctypes.c_int, [_vp, _vp, _i32]),
    "gpe_gpu_set_real_time": (ctypes.c_int, [_vp, _i32]),
    "gpe_gpu_set_timing": (ctypes.c_int, [_vp, _i32]),
    "gpe_gpu_get_timing": (ctypes.c_int, [_vp, ctypes.POINTER(GpeTimingC)]),
    "gpe_gpu_launch_count": (_i64, [_vp]),
    "gpe_gpu_device_bytes": (_i64, [_vp]),
    "gpe_gpu_stream": (_vp, [_vp]),
    "gpe_gpu_set_slab": (ctypes.c_int, [_vp, _i32, _i32]),
    "gpe_gpu_comm_unique_id": (ctypes.c_int, [_vp]),
    "gpe_gpu_comm_init": (ctypes.c_int, [_vp, _vp, _i32, _i32]),
    "gpe_gpu_host_alloc": (_vp, [ctypes.c_size_t]),
    "gpe_gpu_host_free": (None, [_vp]),
    "gpe_gpu_norm_noalloc": (ctypes.c_int, [_vp, _i32, _i32, _i32, _i32, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_double, _dp, _vp]),
    "gpe_batch_default_opts": (None, [ctypes.POINTER(GpeBatchOptsC)]),
    "gpe_batch_create": (ctypes.c_int, [ctypes.POINTER(GpeParamsC), _i32,
                                        ctypes.POINTER(GpeBatchOptsC), ctypes.POINTER(_vp)]),
    "gpe_batch_destroy": (None, [_vp]),
    "gpe_batch_last_error": (ctypes.c_char_p, [_vp]),
    "gpe_batch_member": (ctypes.c_int, [_vp, _i32, ctypes.POINTER(_vp)]),
    "gpe_batch_advance": (ctypes.c_int, [_vp, _i64, ctypes.c_double, ctypes.c_double, _dp]),
    "gpe_batch_set_opts": (ctypes.c_int, [_vp, ctypes.POINTER(GpeBatchOptsC)]),
    "gpe_batch_stream": (_vp, [_vp]),
    "gpe_batch_launch_count": (_i64, [_vp]),
    "gpe_batch_info": (ctypes.c_int, [_vp, ctypes.POINTER(_i64), ctypes.POINTER(_i32),
                                      ctypes.POINTER(_i32), ctypes.POINTER(_i32)]),
    "gpe_cnn_default_params": (None, [ctypes.POINTER(GpeCnnParamsC), _i32, _i32, _i32]),
    "gpe_cnn_create": (ctypes.c_int, [ctypes.POINTER(GpeCnnParamsC), ctypes.POINTER(_vp)]),
    "gpe_cnn_destroy": (None, [_vp]),
    "gpe_cnn_last_error": (ctypes.c_char_p, [_vp]),
    "gpe_cnn_set_weights": (ctypes.c_int, [_vp, _fp, _fp]),
    "gpe_cnn_get_weights": (ctypes.c_int, [_vp, _fp, _fp]),
    "gpe_cnn_apply": (ctypes.c_int, [_vp, _vp]),
    "gpe_cnn_attach": (ctypes.c_int, [_vp, _vp]),
    "gpe_cnn_delta": (ctypes.c_int, [_vp, _vp, _vp]),
    "gpe_cnn_grad": (ctypes.c_int, [_vp, _vp, _vp, _i32, _dp, _fp, _fp]),
    "gpe_cnn_train_step": (ctypes.c_int, [_vp, _vp, _vp, _i32, ctypes.c_float, _dp]),
    "gpe_cnn_adam_reset": (ctypes.c_int, [_vp]),
    "gpe_cnn_restrict": (ctypes.c_int, [_vp, _vp, _i32]),
    "gpe_cnn_launch_count": (_i64, [_vp]),
}

_lib = None


def lib():
    """Load the in-tree library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m gpe_b200.build` "
                "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def torch_ready(t) -> None:
    """Order a library call after the work torch has queued on t's device.

    The library runs on its own non-blocking streams, which do not wait for
    torch's current stream: a tensor that torch is still writing (or still
    reading) must be finished before its pointer is handed over."""
    import torch
    torch.cuda.current_stream(t.device).synchronize()


_COMPLEX_EB = {"torch.complex64": 8, "torch.complex128": 16}


def device_field(t, shape, device: int, what: str, elem_bytes: int | None = None,
                 dtypes=_COMPLEX_EB) -> int:
    """Check a tensor before its raw pointer goes to the library, and return
    its element size in bytes.

    The entry points that take a device pointer read or write exactly
    prod(shape) elements of the given size, densely; a host tensor, a tensor
    on another GPU, a strided view, a wrong shape or another dtype would make
    them touch memory outside the allocation.  Raises GpeError(GPE_ERR_INVALID)
    before any launch."""
    if not getattr(t, "is_cuda", False):
        raise GpeError(1, f"{what}: expected a CUDA tensor")
    idx = t.device.index
    if (0 if idx is None else idx) != device:
        raise GpeError(1, f"{what}: tensor is on cuda:{idx}, the solver on cuda:{device}")
    if not t.is_contiguous():
        raise GpeError(1, f"{what}: tensor must be contiguous")
    if tuple(t.shape) != tuple(shape):
        raise GpeError(1, f"{what}: shape {tuple(t.shape)} != {tuple(shape)}")
    eb = dtypes.get(str(t.dtype))
    if eb is None:
        raise GpeError(1, f"{what}: dtype {t.dtype} not in {sorted(dtypes)}")
    if elem_bytes is not None and eb != elem_bytes:
        raise GpeError(1, f"{what}: dtype {t.dtype} does not match the solver's precision "
                          f"({elem_bytes}-byte complex)")
    return eb


class _PinnedBlock:
    """Page-locked host memory from gpe_gpu_host_alloc, freed with the object."""

    def __init__(self, nbytes: int):
        self.ptr = lib().gpe_gpu_host_alloc(max(int(nbytes), 1))
        if not self.ptr:
            raise GpeError(4, f"cudaHostAlloc of {nbytes} bytes failed")

    def __del__(self):
        if getattr(self, "ptr", None):
            lib().gpe_gpu_host_free(self.ptr)
            self.ptr = None


def pinned_empty(shape, dtype):
    """A numpy array in page-locked host memory (device-to-host copies into it
    run at the link's full rate); the memory lives as long as the array."""
    import numpy as np
    dt = np.dtype(dtype)
    n = int(np.prod(shape)) if len(shape) else 1
    blk = _PinnedBlock(n * dt.itemsize)
    buf = (ctypes.c_char * max(n * dt.itemsize, 1)).from_address(blk.ptr)
    buf._block = blk  # keeps the memory alive with the buffer
    return np.frombuffer(buf, dtype=dt, count=n).reshape(shape)


def check(rc: int, ctx=None) -> None:
    if rc != GPE_OK:
        msg = lib().gpe_gpu_last_error(ctx)
        raise GpeError(rc, msg.decode() if msg else "")


def check_cnn(rc: int, cnn=None) -> None:
    if rc != GPE_OK:
        msg = lib().gpe_cnn_last_error(cnn)
        raise GpeError(rc, msg.decode() if msg else "")


def check_group(rc: int, group=None) -> None:
    if rc != GPE_OK:
        msg = lib().gpe_group_last_error(group)
        raise GpeError(rc, msg.decode() if msg else "")


def check_batch(rc: int, batch=None) -> None:
    if rc != GPE_OK:
        msg = lib().gpe_batch_last_error(batch)
        raise GpeError(rc, msg.decode() if msg else "")

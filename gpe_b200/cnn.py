"""The learned coarse-grid correction (include/gpe_cnn.h).

CoarseCorrector holds a 4-layer 3x3x3 conv3d network (2 -> 16 -> 16 -> 16 ->
2 channels, GELU, BF16 weights and activations, FP32 accumulation on the
tcgen05 tensor cores) for one coarse grid.  After a coarse time step it adds
delta = out_scale * net(Re psi, Im psi) to psi; it is trained on pairs the
fine-grid solver generates (restrict(fine(t)) stepped once on the coarse
grid, against restrict(fine(t + dt))).  There is no CPU path: every call
runs the CUDA kernels of libgpe_gpu.so.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from ._lib import GpeCnnParamsC, check_cnn, device_field, lib, torch_ready
from .solver import GpeSolver

LAYERS, TAPS, CH = 4, 27, 16


def init_weights(seed: int = 0):
    """He-normal weights over each layer's real fan-in for layers 0-2, a
    zero last layer (the untrained network is the identity correction),
    zero biases.  Returns (w (4,27,16,16) float32, b (4,16) float32)."""
    rng = np.random.default_rng(seed)
    w = np.zeros((LAYERS, TAPS, CH, CH), dtype=np.float32)
    cin = [2, 16, 16, 16]
    cout = [16, 16, 16, 2]
    for l in range(3):
        std = math.sqrt(2.0 / (TAPS * cin[l]))
        w[l, :, :cout[l], :cin[l]] = rng.normal(0.0, std, size=(TAPS, cout[l], cin[l]))
    b = np.zeros((LAYERS, CH), dtype=np.float32)
    return w, b


def _fptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


class CoarseCorrector:
    def __init__(self, nx: int, ny: int, nz: int, device: int = 0, train: bool = False,
                 out_scale: float = 0.01, preserve_norm: bool = False):
        p = GpeCnnParamsC()
        lib().gpe_cnn_default_params(ctypes.byref(p), nx, ny, nz)
        p.device, p.train, p.out_scale = device, int(bool(train)), float(out_scale)
        p.preserve_norm = int(bool(preserve_norm))
        self._h = ctypes.c_void_p()
        check_cnn(lib().gpe_cnn_create(ctypes.byref(p), ctypes.byref(self._h)), None)
        self.shape = (nz, ny, nx)
        self.device = int(device)
        self.out_scale = float(out_scale)
        self.train = bool(train)

    def close(self) -> None:
        if self._h:
            lib().gpe_cnn_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc):
        check_cnn(rc, self._h)

    def set_weights(self, w, b) -> None:
        w = np.ascontiguousarray(w, dtype=np.float32)
        b = np.ascontiguousarray(b, dtype=np.float32)
        assert w.shape == (LAYERS, TAPS, CH, CH) and b.shape == (LAYERS, CH)
        self._chk(lib().gpe_cnn_set_weights(self._h, _fptr(w), _fptr(b)))

    def get_weights(self):
        w = np.zeros((LAYERS, TAPS, CH, CH), dtype=np.float32)
        b = np.zeros((LAYERS, CH), dtype=np.float32)
        self._chk(lib().gpe_cnn_get_weights(self._h, _fptr(w), _fptr(b)))
        return w, b

    def apply(self, s: GpeSolver) -> None:
        """psi += delta(psi) on the solver's resident field."""
        self._chk(lib().gpe_cnn_apply(self._h, s.handle))

    def attach(self, s: GpeSolver) -> None:
        """Correct after every later step of s."""
        self._chk(lib().gpe_cnn_attach(self._h, s.handle))

    @staticmethod
    def detach(s: GpeSolver) -> None:
        check_cnn(lib().gpe_cnn_attach(None, s.handle), None)

    def delta(self, s: GpeSolver):
        """delta of the solver's psi as a CUDA float32 tensor (nz, ny, nx, 2)."""
        import torch
        out = torch.empty(self.shape + (2,), dtype=torch.float32, device="cuda")
        torch_ready(out)
        self._chk(lib().gpe_cnn_delta(self._h, s.handle, ctypes.c_void_p(out.data_ptr())))
        return out

    def _eb(self, t, what: str) -> int:
        return device_field(t, self.shape, self.device, what)

    def grad(self, s: GpeSolver, target):
        """(loss, dW, db) of the pair (s's psi, target CUDA tensor)."""
        t = target.contiguous()
        eb = self._eb(t, "grad target")
        torch_ready(t)
        loss = ctypes.c_double()
        dw = np.zeros((LAYERS, TAPS, CH, CH), dtype=np.float32)
        db = np.zeros((LAYERS, CH), dtype=np.float32)
        self._chk(lib().gpe_cnn_grad(self._h, s.handle, ctypes.c_void_p(t.data_ptr()),
                                     eb, ctypes.byref(loss), _fptr(dw), _fptr(db)))
        return loss.value, dw, db

    def train_step(self, s: GpeSolver, target, lr: float) -> float:
        t = target.contiguous()
        eb = self._eb(t, "train_step target")
        torch_ready(t)
        loss = ctypes.c_double()
        self._chk(lib().gpe_cnn_train_step(self._h, s.handle, ctypes.c_void_p(t.data_ptr()),
                                           eb, float(lr), ctypes.byref(loss)))
        return loss.value

    def adam_reset(self) -> None:
        self._chk(lib().gpe_cnn_adam_reset(self._h))

    def launch_count(self) -> int:
        return int(lib().gpe_cnn_launch_count(self._h))


def restrict(fine: GpeSolver, out) -> None:
    """2:1 restriction (2x2x2 average) of fine's psi into `out`, a CUDA
    complex64/complex128 tensor of shape (nz/2, ny/2, nx/2)."""
    nz, ny, nx = fine.shape
    eb = device_field(out, (nz // 2, ny // 2, nx // 2), fine.prm.device, "restrict(out)")
    torch_ready(out)
    check_cnn(lib().gpe_cnn_restrict(fine.handle, ctypes.c_void_p(out.data_ptr()), eb), None)

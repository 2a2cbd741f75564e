"""Batched ensembles: many independent runs of uneven grids on one B200.

The reference runs one grid per job (src/gpe.f90).  A parameter scan of
trap frequencies, interaction strengths or grid sizes is then a queue of
small jobs, each too small to fill the GPU.  GpeBatch holds all of them
resident and steps them together: every rk4 stage is one persistent launch
whose CTAs walk a shared work list of (run, tile, z-range) items, largest
first, and one whole step is replayed from a CUDA graph
(include/gpe_gpu.h, gpe_batch_*).  Members are ordinary contexts: each one's
state, norm and energy are read through GpeSolver's methods.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from ._lib import GpeBatchOptsC, GpeParamsC, check_batch, lib
from .solver import GpeParams, GpeSolver


@dataclass
class BatchOpts:
    tile_y: int = 0        # 0 = auto (8); else 4 or 8
    zchunk: int = 0        # 0 = auto (min(nz, 64)) planes per work item
    ctas_per_sm: int = 0   # 0 = as many as fit
    use_graph: bool = True

    def to_c(self) -> GpeBatchOptsC:
        o = GpeBatchOptsC()
        lib().gpe_batch_default_opts(ctypes.byref(o))
        o.tile_y, o.zchunk, o.ctas_per_sm = self.tile_y, self.zchunk, self.ctas_per_sm
        o.use_graph = int(bool(self.use_graph))
        return o


class _Member(GpeSolver):
    """Non-owning GpeSolver view of one batch member."""

    def __init__(self, batch: "GpeBatch", run: int, prm: GpeParams):
        self.prm = prm
        self._batch = batch
        self._ctx = ctypes.c_void_p()
        check_batch(lib().gpe_batch_member(batch.handle, run, ctypes.byref(self._ctx)),
                    batch.handle)
        self.shape = (prm.nz, prm.ny, prm.nx)
        self.t, self.im_t, self.p = 0.0, 0.0, 0
        self.dt = complex(batch.dt)
        self.last_info = None

    def close(self) -> None:
        self._ctx = ctypes.c_void_p()


class GpeBatch:
    """nruns resident runs stepped together with rk4 at one time step dt."""

    def __init__(self, prms: Sequence[GpeParams], dt: complex, opts: BatchOpts | None = None):
        self.prms = list(prms)
        self.dt = complex(dt)
        self.opts = opts or BatchOpts()
        arr = (GpeParamsC * len(self.prms))(*[p.to_c() for p in self.prms])
        o = self.opts.to_c()
        self._b = ctypes.c_void_p()
        check_batch(lib().gpe_batch_create(arr, len(self.prms), ctypes.byref(o),
                                           ctypes.byref(self._b)), None)
        self.members = [_Member(self, r, p) for r, p in enumerate(self.prms)]
        self.t = 0.0
        self.steps = 0

    @property
    def handle(self):
        return self._b

    def __len__(self) -> int:
        return len(self.prms)

    def __getitem__(self, r: int) -> GpeSolver:
        return self.members[r]

    def close(self) -> None:
        if self._b:
            for m in self.members:
                m.close()
            lib().gpe_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_opts(self, opts: BatchOpts) -> None:
        """Re-plan the stage launches (tile height, z-planes per item, CTAs
        per SM); states are kept."""
        o = opts.to_c()
        check_batch(lib().gpe_batch_set_opts(self._b, ctypes.byref(o)), self._b)
        self.opts = opts

    def set_states(self, states) -> None:
        for m, s in zip(self.members, states):
            m.set_state(s)

    def advance(self, nsteps: int, want_norms: bool = True) -> np.ndarray | None:
        """nsteps rk4 steps of every run; returns the (nruns, nsteps) norms."""
        norms = np.zeros((len(self), max(nsteps, 1)), dtype=np.float64) if want_norms else None
        ptr = norms.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if want_norms else None
        check_batch(lib().gpe_batch_advance(self._b, int(nsteps), self.dt.real, self.dt.imag,
                                            ptr), self._b)
        self.steps += nsteps
        self.t += nsteps * self.dt.real
        for m in self.members:
            m.t = self.t
            m.p = self.steps
        return norms[:, :nsteps] if want_norms else None

    def info(self) -> dict:
        s, n, g, ty = ctypes.c_int64(), ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        check_batch(lib().gpe_batch_info(self._b, ctypes.byref(s), ctypes.byref(n),
                                         ctypes.byref(g), ctypes.byref(ty)), self._b)
        return {"sites": s.value, "items": n.value, "grid": g.value, "tile_y": ty.value}

    def launch_count(self) -> int:
        return int(lib().gpe_batch_launch_count(self._b))

    def stream_handle(self) -> int:
        return int(lib().gpe_batch_stream(self._b) or 0)

"""z-slab decomposition across ranks (one process per GPU).

The reference splits its grid over an nyprocs x nzprocs MPI process grid
(src/variables.f90:98-182, para_range :134-150) with a two-plane halo
exchanged after every stage (send_recv_z / pack_y / unpack_y, :186-358) and
MPI_ALLREDUCE of the norm, energy and rk45 error (:581, 772, 816;
src/solve.f90:189).  Here x and y stay whole on every rank and ranks own
consecutive z-slabs: the halo is two contiguous planes per face, sent by the
library with NCCL straight into the neighbour's ghost planes after every
stage, and the reductions are NCCL all-reduces (include/gpe_gpu.h,
gpe_gpu_set_slab / gpe_gpu_comm_init).  This module holds the host-side plan
and the bootstrap.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, replace

import numpy as np

from ._lib import GpeStepInfoC, check, check_group, lib
from .solver import GpeParams, GpeSolver


def para_range(n1: int, n2: int, nprocs: int, irank: int) -> tuple[int, int]:
    """Start and end index (inclusive) of rank irank's share of n1..n2, as
    the reference's para_range (src/variables.f90:134-150): the first
    mod(n, nprocs) ranks get one extra element."""
    n = n2 - n1 + 1
    base, extra = divmod(n, nprocs)
    ista = irank * base + n1 + min(irank, extra)
    iend = ista + base - 1
    if extra > irank:
        iend += 1
    return ista, iend


@dataclass(frozen=True)
class SlabPlan:
    """Rank `rank`'s slab of a global z axis of nz_global planes."""
    nz_global: int
    nranks: int
    rank: int
    bcs: int

    @property
    def z_range(self) -> tuple[int, int]:
        return para_range(0, self.nz_global - 1, self.nranks, self.rank)

    @property
    def z_offset(self) -> int:
        return self.z_range[0]

    @property
    def nz(self) -> int:
        a, b = self.z_range
        return b - a + 1

    @property
    def nbr_lo(self) -> int:
        return (self.rank - 1) % self.nranks

    @property
    def nbr_hi(self) -> int:
        return (self.rank + 1) % self.nranks

    @property
    def exch_lo(self) -> bool:
        """Lower z ghosts come from the neighbour below (periodic wrap
        included); otherwise they are the reflective mirror of own planes."""
        return self.bcs == 1 or self.rank > 0

    @property
    def exch_hi(self) -> bool:
        return self.bcs == 1 or self.rank < self.nranks - 1

    def validate(self) -> None:
        if self.nz < (4 if self.bcs == 2 else 2):
            raise ValueError(f"slab of {self.nz} planes is too thin for bcs={self.bcs}")


def slab_params(prm: GpeParams, plan: SlabPlan, device: int) -> GpeParams:
    """The per-rank parameters: same box (zr is the global half-width), the
    slab's plane count, this rank's device."""
    return replace(prm, nz=plan.nz, device=device)


class SlabSolver(GpeSolver):
    """A GpeSolver holding one z-slab and joined to the ranks' NCCL
    communicator.  `dist` is an initialised torch.distributed module (any
    backend); it is used once, to broadcast the NCCL unique id."""

    def __init__(self, prm: GpeParams, rank: int, nranks: int, dist, device: int = 0,
                 **kw):
        # The library resolves NCCL by soname at run time; importing torch
        # first makes that the NCCL torch was built against, so a later
        # `import torch` in the same process does not meet an older one.
        import torch  # noqa: F401
        self.plan = SlabPlan(prm.nz, nranks, rank, prm.bcs)
        self.plan.validate()
        self.global_prm = prm
        super().__init__(slab_params(prm, self.plan, device), **kw)
        check(lib().gpe_gpu_set_slab(self._ctx, prm.nz, self.plan.z_offset), self._ctx)
        uid = (ctypes.c_char * 128)()
        if rank == 0:
            check(lib().gpe_gpu_comm_unique_id(uid), None)
        obj = [bytes(uid)]
        if nranks > 1:
            dist.broadcast_object_list(obj, src=0)
        uid = (ctypes.c_char * 128).from_buffer_copy(obj[0])
        check(lib().gpe_gpu_comm_init(self._ctx, uid, rank, nranks), self._ctx)

    def set_global_state(self, psi_global) -> None:
        """Load this rank's planes of a global (nz_global, ny, nx) array."""
        a, b = self.plan.z_range
        self.set_state(np.ascontiguousarray(np.asarray(psi_global)[a:b + 1]))


class SlabGroup:
    """The z-slabs of one grid as separate contexts on one GPU, stepped
    together by the library (gpe_group_*): the slab tables, z-ghost rules,
    ghost-plane exchange and cross-slab reductions of the multi-rank path,
    with the planes moved by device copies instead of NCCL.  Members follow
    the reference's para_range split (SlabPlan)."""

    def __init__(self, prm: GpeParams, nslabs: int, *, dt=None, tau=None):
        self.global_prm = prm
        self.plans = [SlabPlan(prm.nz, nslabs, r, prm.bcs) for r in range(nslabs)]
        self.members = []
        try:
            for pl in self.plans:
                pl.validate()
                m = GpeSolver(slab_params(prm, pl, prm.device), dt=dt, tau=tau)
                check(lib().gpe_gpu_set_slab(m.handle, prm.nz, pl.z_offset), m.handle)
                self.members.append(m)
            arr = (ctypes.c_void_p * nslabs)(*[m.handle.value for m in self.members])
            self._g = ctypes.c_void_p()
            check_group(lib().gpe_group_create(arr, nslabs, ctypes.byref(self._g)), None)
        except Exception:
            for m in self.members:
                m.close()
            raise
        m0 = self.members[0]
        self.t, self.im_t, self.p, self.dt = m0.t, m0.im_t, m0.p, m0.dt
        self.last_info = None

    def close(self) -> None:
        if getattr(self, "_g", None):
            lib().gpe_group_destroy(self._g)
            self._g = ctypes.c_void_p()
        for m in self.members:
            m.close()
        self.members = []

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_global_state(self, psi_global) -> None:
        a = np.asarray(psi_global)
        for pl, m in zip(self.plans, self.members):
            lo, hi = pl.z_range
            m.set_state(np.ascontiguousarray(a[lo:hi + 1]))

    def get_global_state(self, dtype=np.complex128) -> np.ndarray:
        return np.concatenate([m.get_state(dtype) for m in self.members], axis=0)

    def solver(self):
        from ._lib import GpeTimeC
        tm = GpeTimeC(self.t, self.im_t, self.dt.real, self.dt.imag, self.p, 0)
        info = GpeStepInfoC()
        check_group(lib().gpe_group_solver(self._g, ctypes.byref(tm), ctypes.byref(info)),
                    self._g)
        self.t, self.im_t, self.p = tm.t, tm.im_t, tm.p
        self.dt = complex(tm.dt_re, tm.dt_im)
        self.last_info = info
        return info

    def get_norm(self) -> float:
        v = ctypes.c_double()
        check_group(lib().gpe_group_norm(self._g, ctypes.byref(v)), self._g)
        return v.value

    def energy(self):
        e, h = ctypes.c_double(), ctypes.c_double()
        check_group(lib().gpe_group_energy(self._g, ctypes.byref(e), ctypes.byref(h)), self._g)
        return e.value, h.value

"""Multi-rank z-slab decomposition on CPU (gloo, world size 2 and 3).

Each rank steps its slab of the global grid with a numpy emulation of the
library's stage loop, built on the product's SlabPlan (gpe_b200/dist.py):
its z range (the reference's para_range), neighbours, which faces are
exchanged and which are mirrored locally, and the global-index norm weights
and trap potential.  Ghost planes travel between ranks with torch.distributed
after every stage, the norm is all-reduced, and rank 0 compares the gathered
field with the single-domain oracle.  This checks the decomposition logic the
NCCL path uses; the NCCL exchange itself runs in tests/test_gpu_dist.py."""
import os
import socket

import numpy as np
import pytest

from gpe_b200.dist import SlabPlan, para_range

NX, NY = 12, 10
XR, YR, ZR = 4.0, 3.0, 5.0
DT = 0.004
STEPS = 3
KW = dict(g=1.2, mu=0.8, omx=0.3, omy=0.25, omz=0.35)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _w(i, n):
    w = 1.0
    if i == 0: w = 3 / 8
    if i == 1: w = 7 / 6
    if i == 2: w = 23 / 24
    if i == n - 3: w = 23 / 24
    if i == n - 2: w = 7 / 6
    if i == n - 1: w = 3 / 8
    return w


def _wx(n):
    w = np.zeros(n)
    w[0] += 3 / 8; w[1] += 7 / 6; w[2] += 23 / 24
    w[3:n - 3] += 1.0
    w[n - 3] += 23 / 24; w[n - 2] += 7 / 6; w[n - 1] += 3 / 8
    return w


class SlabEmu:
    """numpy restatement of one rank's slab stepping (test only)."""

    def __init__(self, plan, bcs, order, dist):
        self.p, self.bcs, self.order, self.dist = plan, bcs, order, dist
        nzg = plan.nz_global
        self.h = (2 * XR / (NX - 1), 2 * YR / (NY - 1), 2 * ZR / (nzg - 1))
        x = -XR + np.arange(NX) * self.h[0]
        y = -YR + np.arange(NY) * self.h[1]
        z = -ZR + (plan.z_offset + np.arange(plan.nz)) * self.h[2]
        Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
        self.V = 0.5 * (KW["omx"] ** 2 * X ** 2 + KW["omy"] ** 2 * Y ** 2 + KW["omz"] ** 2 * Z ** 2)
        self.W = (np.array([_w(plan.z_offset + k, nzg) for k in range(plan.nz)])[:, None, None]
                  * np.array([_w(j, NY) for j in range(NY)])[None, :, None] * _wx(NX)[None, None, :])

    def ghosts(self, U):
        """Fill the z ghosts of U (nz+4 planes): local mirror or exchange."""
        import torch
        p, n = self.p, self.p.nz
        if not p.exch_lo:  # reflective bottom: f(-1)=f(1), f(-2)=f(2)
            U[1], U[0] = U[3], U[4]
        if not p.exch_hi:  # reflective top: f(n)=f(n-2), f(n+1)=f(n-3)
            U[n + 2], U[n + 3] = U[n], U[n - 1]
        if p.nranks == 1:
            if p.exch_lo:
                U[0:2] = U[n:n + 2]
            if p.exch_hi:
                U[n + 2:n + 4] = U[2:4]
            return
        reqs, recv = [], {}
        # library order: send up, send down, receive from below, from above
        if p.exch_hi:
            reqs.append(self.dist.isend(torch.from_numpy(U[n:n + 2].copy()), dst=p.nbr_hi, tag=1))
        if p.exch_lo:
            reqs.append(self.dist.isend(torch.from_numpy(U[2:4].copy()), dst=p.nbr_lo, tag=2))
        if p.exch_lo:
            recv["lo"] = torch.empty((2, NY, NX), dtype=torch.complex128)
            reqs.append(self.dist.irecv(recv["lo"], src=p.nbr_lo, tag=1))
        if p.exch_hi:
            recv["hi"] = torch.empty((2, NY, NX), dtype=torch.complex128)
            reqs.append(self.dist.irecv(recv["hi"], src=p.nbr_hi, tag=2))
        for r in reqs:
            r.wait()
        if "lo" in recv:
            U[0:2] = recv["lo"].numpy()
        if "hi" in recv:
            U[n + 2:n + 4] = recv["hi"].numpy()

    def lap(self, U):
        mode = "wrap" if self.bcs == 1 else "reflect"
        P = np.pad(U, ((0, 0), (2, 2), (2, 2)), mode=mode)
        n = self.p.nz
        c = P[2:n + 2, 2:-2, 2:-2]
        sx = lambda o: P[2:n + 2, 2:-2, 2 + o:P.shape[2] - 2 + o]
        sy = lambda o: P[2:n + 2, 2 + o:P.shape[1] - 2 + o, 2:-2]
        sz = lambda o: P[2 + o:n + 2 + o, 2:-2, 2:-2]
        L = 0
        for s_, h in ((sx, self.h[0]), (sy, self.h[1]), (sz, self.h[2])):
            if self.order == 2:
                L = L + (s_(1) - 2 * c + s_(-1)) / h ** 2
            else:
                L = L + (-s_(2) + 16 * s_(1) - 30 * c + 16 * s_(-1) - s_(-2)) / (12 * h ** 2)
        return L

    def rhs(self, U):
        f = U[2:-2]
        return -1j * (-0.5 * self.lap(U) + self.V * f + KW["g"] * np.abs(f) ** 2 * f - KW["mu"] * f)

    def padded(self, f):
        U = np.zeros((self.p.nz + 4, NY, NX), complex)
        U[2:-2] = f
        self.ghosts(U)
        return U

    def rk4(self, psi):
        k1 = self.rhs(self.padded(psi))
        k2 = self.rhs(self.padded(psi + 0.5 * DT * k1))
        k3 = self.rhs(self.padded(psi + 0.5 * DT * k2))
        k4 = self.rhs(self.padded(psi + DT * k3))
        return psi + DT * (k1 / 6 + k2 / 3 + k3 / 3 + k4 / 6)

    def norm(self, psi):
        import torch
        loc = torch.tensor([float(np.sum(self.W * np.abs(psi) ** 2))], dtype=torch.float64)
        self.dist.all_reduce(loc)
        return float(loc.item()) * self.h[0] * self.h[1] * self.h[2]


def _worker(rank, world, port, nzg, bcs, order, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        plan = SlabPlan(nzg, world, rank, bcs)
        plan.validate()
        emu = SlabEmu(plan, bcs, order, dist)
        rng = np.random.default_rng(5)
        full = 1.0 + 0.3 * (rng.standard_normal((nzg, NY, NX)) + 1j * rng.standard_normal((nzg, NY, NX)))
        a, b = plan.z_range
        psi = full[a:b + 1].copy()
        norms = []
        for _ in range(STEPS):
            psi = emu.rk4(psi)
            norms.append(emu.norm(psi))
        import torch
        parts = [None] * world
        dist.all_gather_object(parts, (a, psi))
        if rank == 0:
            out = np.zeros_like(full)
            for a0, blk in parts:
                out[a0:a0 + blk.shape[0]] = blk
            q.put((full, out, norms))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,nzg,bcs,order", [(2, 12, 1, 4), (2, 12, 2, 4), (3, 13, 1, 2),
                                                 (3, 13, 2, 4)])
def test_slab_decomposition_matches_single_domain(world, nzg, bcs, order):
    import torch.multiprocessing as mp

    import oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, nzg, bcs, order, q))
             for r in range(world)]
    for pr in procs:
        pr.start()
    full, out, norms = q.get(timeout=300)
    for pr in procs:
        pr.join(timeout=120)
        assert pr.exitcode == 0
    o = oracle.Oracle(oracle.OracleParams(nx=NX, ny=NY, nz=nzg, xr=XR, yr=YR, zr=ZR,
                                          scheme="rk4", eqn_to_solve=4, bcs=bcs, order=order,
                                          **KW))
    tm = oracle.OraTime(0.0, 0.0, DT, 0.0, 0)
    psi = full
    for _ in range(STEPS):
        psi, _, _ = o.solver(psi, tm)
    assert np.linalg.norm(out - psi) / np.linalg.norm(psi) < 1e-12
    assert norms[-1] == pytest.approx(o.get_norm(psi), rel=1e-12)


def test_para_range_matches_reference_rule():
    # src/variables.f90:134-150: first mod(n, nprocs) ranks get one extra
    assert [para_range(0, 12, 3, r) for r in range(3)] == [(0, 4), (5, 8), (9, 12)]
    assert [para_range(0, 11, 2, r) for r in range(2)] == [(0, 5), (6, 11)]
    p = SlabPlan(13, 3, 0, 2)
    assert (p.z_offset, p.nz, p.exch_lo, p.exch_hi) == (0, 5, False, True)
    p = SlabPlan(13, 3, 2, 1)
    assert (p.nbr_lo, p.nbr_hi, p.exch_lo, p.exch_hi) == (1, 0, True, True)
    with pytest.raises(ValueError):
        SlabPlan(6, 3, 1, 2).validate()

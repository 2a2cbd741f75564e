"""Launch-shape autotuner for batched ensembles.

A batch's stage launches have three free knobs (include/gpe_gpu.h,
gpe_batch_opts): the tile height (4 or 8 rows of 64 sites), the z-planes per
work item, and the resident CTAs per SM.  Small grids want short items (more
items to balance 148 SMs), large grids want long ones (fewer warm-up planes
per item: an item of zc planes reads zc + 2R planes of its stencil field).
The best point depends on the ensemble's size mix, so it is measured: every
candidate is applied to the live batch with gpe_batch_set_opts, warmed up,
and timed with CUDA events on the batch's stream; the fastest wins.  Results
are cached in a JSON file keyed by the ensemble's signature (member shapes,
order, boundary, precision, device name), so a repeated scan pays once.

The candidate set is small and explicit on purpose: 2 x 4 x 3 = 24 shapes,
each timed over a few steps, costs well under a second for ensembles of tens
of millions of sites.
"""
from __future__ import annotations

import hashlib
import itertools
import json
import os
from dataclasses import asdict
from typing import Iterable

from .batch import BatchOpts, GpeBatch

TILE_Y = (8, 4)
ZCHUNK = (8, 16, 32, 64)
CTAS_PER_SM = (0, 1, 2)


def candidates() -> list[BatchOpts]:
    return [BatchOpts(tile_y=ty, zchunk=zc, ctas_per_sm=cp)
            for ty, zc, cp in itertools.product(TILE_Y, ZCHUNK, CTAS_PER_SM)]


def signature(batch: GpeBatch, device_name: str) -> str:
    p0 = batch.prms[0]
    shapes = sorted((p.nx, p.ny, p.nz) for p in batch.prms)
    key = json.dumps({"shapes": shapes, "order": p0.order, "bcs": p0.bcs,
                      "precision": p0.precision, "kahan": bool(p0.kahan),
                      "device": device_name}, sort_keys=True)
    return hashlib.sha1(key.encode()).hexdigest()[:16]


def time_steps(batch: GpeBatch, steps: int, warmup: int = 2) -> float:
    """Milliseconds per step, CUDA events on the batch's own stream."""
    import torch
    stream = torch.cuda.ExternalStream(batch.stream_handle())
    batch.advance(warmup, want_norms=False)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    batch.advance(steps, want_norms=False)
    b.record(stream)
    b.synchronize()
    return a.elapsed_time(b) / steps


def tune(batch: GpeBatch, *, steps: int = 4, cands: Iterable[BatchOpts] | None = None,
         cache_path: str | None = None, restore_state: bool = True) -> tuple[BatchOpts, list]:
    """Time every candidate on `batch` and leave the fastest applied.

    The members' states are saved first and restored afterwards when
    restore_state is set, so tuning does not advance the simulation.
    Returns (best options, [(options, ms per step), ...])."""
    import torch
    dev = torch.cuda.get_device_name(batch.prms[0].device)
    sig = signature(batch, dev)
    cache = {}
    if cache_path and os.path.exists(cache_path):
        with open(cache_path) as f:
            cache = json.load(f)
    if sig in cache:
        best = BatchOpts(**cache[sig]["best"])
        batch.set_opts(best)
        return best, [(BatchOpts(**o), ms) for o, ms in cache[sig]["table"]]
    saved = [m.get_state(_host_dtype(m)) for m in batch.members] if restore_state else None
    table = []
    for o in (list(cands) if cands is not None else candidates()):
        batch.set_opts(o)
        table.append((o, time_steps(batch, steps)))
    best = min(table, key=lambda t: t[1])[0]
    batch.set_opts(best)
    if saved is not None:
        batch.set_states(saved)
    if cache_path:
        cache[sig] = {"best": asdict(best), "table": [(asdict(o), ms) for o, ms in table]}
        tmp = cache_path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(cache, f, indent=1)
        os.replace(tmp, cache_path)
    return best, table


def _host_dtype(m):
    import numpy as np
    return np.complex64 if m.prm.precision == 8 else np.complex128

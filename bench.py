#!/usr/bin/env python
"""Throughput of the GPE finite-difference time stepper on B200.

Workload (one "step" = one full RK4 time step of every site): 512^3 periodic
grid, h = 0.5, 4th-order centred differences, RK4 with dt = 0.005, equation 4
(g = mu = 1, no trap), complex64 psi with Kahan-compensated accumulation and
FP64 norm reduction every step; seeded random-phase initial condition
(|k| <= 1.0, unit amplitudes, uniform phases, rescaled to mean density 1).
Metric: site-updates/s (sites x steps / device time), whole job.  On one
GPU the same line then carries, under "configs", the short results of the
other workloads measured after it (--workload rkf45, ensemble and learned at
reduced step counts; --no-others skips them).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
  python bench.py --workload ensemble [--steps 500]
  python bench.py --workload rkf45 [--t-end 20]
  python bench.py --workload learned [--steps 200]
  python bench.py --workload spectrum [--grid 512] [--steps 20]

--workload ensemble: 64 independent complex64 runs, cubic grids drawn from
{32,48,64,96,128}^3 with seed 0, h = 0.5, harmonic trap omega ~ U[0.05, 0.15],
random-phase IC (|k| <= 0.8) times the Thomas-Fermi profile, 2nd-order FD,
reflective boundaries, RK4 dt = 0.01, 500 steps; all runs stepped together
by the batched launches (autotuned launch shape), next to the same runs
stepped one context at a time.

N > 1 (launched by torchrun): every rank advances its own 512^3 replica
(weak scaling, no data-path collective); with --decomp slab the ranks share
one 512^3 grid as NCCL z-slabs (strong scaling).  Device time is the max over
ranks.
--impl reference times the CPU restatement of the reference's path (the
reference's Fortran build is unavailable in this image) on the host cores.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "site-updates/s & HBM GB/s at 512^3; time-to-t at <=1e-3 density err vs plain"
N_GRID = 512
H = 0.5
DT = 0.005
KMAX = 1.0
# algorithmic bytes per site per RK4 step with complex64 + Kahan, increment
# form: stage 1 reads psi and writes d2 (2 x 8 B); stages 2-3 read psi and d
# (both as stencils) and write the next d (3 x 8 B each); stage 4 reads psi,
# d4, d2, d3, c and writes psi', c (7 x 8 B) -> 120 B/site (the stage-value +
# accumulator form moves 152)
BYTES_PER_FAMILY = {"stage_first": 16, "stage_mid": 24, "stage_last": 56}
BYTES_PER_STEP = 120
# the plain fine path of the learned workload steps at its largest stable dt
FINE_PATH_DT = 0.02
LAUNCHES_PER_STEP = 5


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic():
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


# --------------------------------------------------------------------------
# clocks sampled during the timed region

class ClockSampler:
    FIELDS = ("index,uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 10:
                    continue
                if self.uuid and self.uuid not in parts[1]:
                    continue
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        mx = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for nm, v in zip(names, r[6:10]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


# --------------------------------------------------------------------------

def cpu_sample(threads: int, min_seconds: float = 10.0, max_steps: int = 50):
    """Times the oracle (CPU restatement of the reference path, FP64, the
    reference's own pass structure) on a 512 x 512 x 8 periodic slab of the
    same workload; returns (site-updates/s, steps, sites, seconds)."""
    import numpy as np

    import oracle

    oracle.set_threads(threads)
    nx = ny = N_GRID
    nz = 8
    xr = H * (nx - 1) / 2
    zr = H * (nz - 1) / 2
    o = oracle.Oracle(oracle.OracleParams(nx=nx, ny=ny, nz=nz, xr=xr, yr=xr, zr=zr,
                                          scheme="rk4", eqn_to_solve=4, bcs=1, order=4,
                                          g=1.0, mu=1.0))
    rng = np.random.default_rng(0)
    psi = np.exp(2j * np.pi * rng.random((nz, ny, nx)))
    tm = oracle.OraTime(0.0, 0.0, DT, 0.0, 0)
    psi, _, _ = o.solver(psi, tm)  # warm-up (page-in)
    steps = 0
    t0 = time.perf_counter()
    while True:
        psi, _, _ = o.solver(psi, tm)
        o.get_norm(psi)
        steps += 1
        el = time.perf_counter() - t0
        if (el >= min_seconds and steps >= 2) or steps >= max_steps:
            break
    sites = nx * ny * nz
    return sites * steps / el, steps, sites, el


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    import numpy as np

    import oracle

    oracle.set_threads(threads)
    nx = ny = N_GRID
    nz = 8
    xr = H * (nx - 1) / 2
    zr = H * (nz - 1) / 2
    o = oracle.Oracle(oracle.OracleParams(nx=nx, ny=ny, nz=nz, xr=xr, yr=xr, zr=zr,
                                          scheme="rk4", eqn_to_solve=4, bcs=1, order=4,
                                          g=1.0, mu=1.0))
    rng = np.random.default_rng(0)
    psi = np.exp(2j * np.pi * rng.random((nz, ny, nx)))
    tm = oracle.OraTime(0.0, 0.0, DT, 0.0, 0)
    for _ in range(args.warmup):
        psi, _, _ = o.solver(psi, tm)
        o.get_norm(psi)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        psi, _, _ = o.solver(psi, tm)
        o.get_norm(psi)
    el = time.perf_counter() - t0
    sites = nx * ny * nz
    v = sites * args.steps / el
    sample = (f"each step = one RK4 step (+ get_norm) of a {nx}x{ny}x{nz} periodic slab of the "
              f"512^3 workload, FP64, {threads} OpenMP threads over z-planes")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "site-updates/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        # timed: one step of the slab; projected: the same rate over the
        # whole 512^3 grid (64 slabs), not a measured time
        "ms_per_step": 1e3 * el / args.steps,
        "ms_per_step_slab": 1e3 * el / args.steps,
        "ms_per_step_512cube_projected": 1e3 * el / args.steps * (N_GRID / nz),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded random phases)",
        "config": dict(workload_config(args.gpus, storage="complex128"),
                       sample_grid=[nx, ny, nz]),
        "cpu_baseline": {"value": v, "unit": "site-updates/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": v, "unit": "site-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "note": ("the reference Fortran/MPI/FFTW2 build cannot be compiled in this image; "
                 "this arm runs the project's C restatement of its path (oracle/), which keeps "
                 "the reference's pass structure"),
    }
    print(json.dumps(line), flush=True)
    return 0


ENS_RUNS = 64
ENS_SIZES = (32, 48, 64, 96, 128)
ENS_DT = 0.01
ENS_KMAX = 0.8
# complex64 without compensation, increment form: stage 1 reads psi, writes
# d2 (16 B); stages 2-3 read psi, d and write the next d (24 B each); stage 4
# reads psi, d4, d2, d3 and writes psi' (40 B)
ENS_BYTES_PER_SITE = 104


def ensemble_members(seed=0):
    import numpy as np

    from gpe_b200 import GpeParams
    rng = np.random.default_rng(seed)
    sizes = rng.choice(ENS_SIZES, size=ENS_RUNS)
    omegas = rng.uniform(0.05, 0.15, size=ENS_RUNS)
    prms = []
    for n, om in zip(sizes, omegas):
        n = int(n)
        xr = H * (n - 1) / 2
        prms.append(GpeParams(nx=n, ny=n, nz=n, xr=xr, yr=xr, zr=xr, scheme="rk4",
                              eqn_to_solve=4, bcs=2, order=2, precision=8, kahan=False,
                              g=1.0, mu=1.0, omx=float(om), omy=float(om), omz=float(om)))
    return prms


def run_ensemble(args):
    print(json.dumps(measure_ensemble(args)), flush=True)
    return 0


def measure_ensemble(args):
    """The batched-ensemble workload (config C4): its JSON line as a dict."""
    import numpy as np
    import torch

    from gpe_b200 import GpeBatch, GpeSolver
    from gpe_b200.autotune import tune
    from gpe_b200.batch import BatchOpts
    from gpe_b200.ic import trapped_random_phase

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(0)
    prms = ensemble_members()
    sites = sum(p.nx * p.ny * p.nz for p in prms)
    host = [trapped_random_phase(torch, p.nx, H, p.omx, ENS_KMAX, 1000 + r, dev).cpu().numpy()
            for r, p in enumerate(prms)]
    b = GpeBatch(prms, ENS_DT)
    b.set_states(host)
    if getattr(args, "ens_shape", None):
        # a fixed launch shape (profiling captures): no tuning pass
        ty, zc, cp = (int(v) for v in args.ens_shape.split(","))
        best = BatchOpts(tile_y=ty, zchunk=zc, ctas_per_sm=cp)
        b.set_opts(best)
        table = []
    else:
        best, table = tune(b, steps=4)
    b.set_states(host)
    b.advance(args.warmup, want_norms=False)
    b.set_states(host)
    stream = torch.cuda.ExternalStream(b.stream_handle())
    sampler = ClockSampler(None)
    sampler.start()
    time.sleep(0.3)
    lc0 = b.launch_count()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    norms = b.advance(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    clocks = sampler.stop()
    launches = b.launch_count() - lc0
    info = b.info()
    final = [b[r].get_state(np.complex64) for r in range(len(prms))]

    # end to end: host ICs in, all steps, norms and final states out
    pin = [torch.from_numpy(h).pin_memory() for h in host]
    t0 = time.perf_counter()
    e0.record(stream)
    b.set_states([p.numpy() for p in pin])
    b.advance(args.steps)
    outs = [b[r].get_state(np.complex64) for r in range(len(prms))]
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    del outs
    b.close()

    # the same runs stepped one context at a time (one grid per job)
    seq_ms = 0.0
    seq_launches = 0
    seq_err = 0.0
    for r, p in enumerate(prms):
        s = GpeSolver(p, dt=ENS_DT)
        s.set_state(host[r])
        s.advance(args.warmup)
        s.set_state(host[r])
        st = torch.cuda.ExternalStream(s.stream_handle())
        l0 = s.launch_count()
        a = torch.cuda.Event(enable_timing=True)
        z = torch.cuda.Event(enable_timing=True)
        a.record(st)
        s.advance(args.steps)
        z.record(st)
        z.synchronize()
        seq_ms += a.elapsed_time(z)
        seq_launches += s.launch_count() - l0
        got = s.get_state(np.complex64)
        seq_err = max(seq_err, float(np.abs(got - final[r]).max()))
        s.close()

    peak, peak_kind = load_peaks()
    value = sites * args.steps / (ms / 1e3)
    gbs = ENS_BYTES_PER_SITE * sites * args.steps / (ms / 1e3) / 1e9
    line = {
        "metric": "site-updates/s (ensemble of 64 uneven trapped runs)", "value": value,
        "unit": "site-updates/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded sizes, traps, phases)",
        "config": {"workload": "64 complex64 runs, cubic n in {32,48,64,96,128} (seed 0), "
                               "h=0.5, trap omega~U[0.05,0.15], random phase |k|<=0.8 x TF, "
                               "order 2, reflective, RK4 dt=0.01",
                   "sizes": sorted(p.nx for p in prms), "sites": sites,
                   "l2": f"inputs larger than L2 ({8 * sites * 4 / 1e9:.2f} GB of fields)"},
        "roofline": {"bound": "hbm", "kernel": "stage_kernel (batched, all four stages)",
                     "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
                     "peak_source": peak_kind, "alg_bytes_per_site_step": ENS_BYTES_PER_SITE,
                     "traffic": None},
        "launch": {"best": vars(best), "items": info["items"], "grid": info["grid"],
                   "table_ms": [(vars(o), t) for o, t in table]},
        "sequential": {"value": sites * args.steps / (seq_ms / 1e3), "ms_per_step":
                       seq_ms / args.steps, "launches": seq_launches,
                       "max_abs_diff_vs_batch": seq_err,
                       "form": "each run in its own context, advanced alone, one after another"},
        "speedup_vs_sequential": seq_ms / ms,
        "e2e": {"value": sites * args.steps / e2e_s, "unit": "site-updates/s",
                "h2d_bytes_per_step": 8 * sites / args.steps,
                "d2h_bytes_per_step": (8 * sites + 8 * len(prms) * args.steps) / args.steps,
                "form": "host ICs -> batch, all steps, per-run norms and final states to host; "
                        "wall clock"},
        "clocks": clocks, "gpu_launches": int(launches),
        "final_norm_min": float(norms[:, -1].min()), "final_norm_max": float(norms[:, -1].max()),
    }
    return line


def run_learned(args):
    print(json.dumps(measure_learned(args)), flush=True)
    return 0


def measure_learned(args):
    """Time to t = 50 of the learned coarse path (128^3 complex64 + Kahan RK4
    at the coarse step the network was trained for, network correction after
    every step) against the plain fine path (256^3, h = 0.25, complex64 +
    Kahan RK4 at its largest stable step dt = 0.02), both timed on the device
    per step and scaled by their steps to t = 50."""
    import numpy as np
    import torch

    from gpe_b200.cnn import CoarseCorrector, init_weights
    from gpe_b200.learned import (LearnedConfig, coarse_solver, config_from_weights,
                                  fine_solver, restricted)

    torch.cuda.set_device(0)
    cfg = LearnedConfig()
    steps = args.steps
    wpath = os.path.join(ROOT, "gpe_b200", "data", "cnn_weights.npz")
    if os.path.exists(wpath):
        z = np.load(wpath)
        w, b = z["w"], z["b"]
        cfg = config_from_weights(z, cfg)
        wsrc = "trained (gpe_b200/data/cnn_weights.npz)"
    else:
        w, b = init_weights(7)
        wsrc = "untrained (He-normal, seed 7); the time does not depend on the values"

    def timed(s, k):
        st = torch.cuda.ExternalStream(s.stream_handle())
        s.advance(args.warmup)
        a = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        a.record(st)
        s.advance(k)
        e.record(st)
        e.synchronize()
        return a.elapsed_time(e) / k

    fine_dt = FINE_PATH_DT
    fine = fine_solver(cfg, 100, precision=8, kahan=True, dt=fine_dt)
    c = coarse_solver(cfg)
    c.set_state(restricted(cfg, fine))
    sampler = ClockSampler(None)
    sampler.start()
    time.sleep(0.3)
    ms_fine = timed(fine, steps)
    ms_plain = timed(c, steps)
    n = cfg.coarse_n
    net = CoarseCorrector(n, n, n, out_scale=cfg.out_scale, preserve_norm=cfg.preserve_norm)
    net.set_weights(w, b)
    st = torch.cuda.ExternalStream(c.stream_handle())
    for _ in range(3):
        net.apply(c)
    a = torch.cuda.Event(enable_timing=True)
    e = torch.cuda.Event(enable_timing=True)
    lc0 = net.launch_count()
    a.record(st)
    for _ in range(steps):
        net.apply(c)
    e.record(st)
    e.synchronize()
    ms_net = a.elapsed_time(e) / steps
    launches_per_apply = (net.launch_count() - lc0) / steps
    net.attach(c)
    ms_learned = timed(c, steps)
    clocks = sampler.stop()
    CoarseCorrector.detach(c)
    net.close()
    c.close()
    fine.close()
    K = int(round(cfg.t_end / cfg.dt))
    K_fine = int(round(cfg.t_end / fine_dt))
    sites_c = n ** 3
    useful_flop = 2 * 27 * (2 * 16 + 16 * 16 + 16 * 16 + 16 * 2) * sites_c
    issued_flop = 2 * 27 * 16 * 16 * 4 * sites_c
    peaks = {}
    pp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pp):
        with open(pp) as f:
            peaks = json.load(f)
    tf_peak = float(peaks.get("bf16_tflops", 1590.0))
    achieved = issued_flop / (ms_net / 1e3) / 1e12
    line = {
        "metric": "time to t=50: learned coarse path vs plain fine path",
        "value": (K_fine * ms_fine) / (K * ms_learned),
        "unit": "x (speed-up)", "n_gpus": 1, "steps": steps, "warmup": args.warmup,
        "ms_per_step": ms_learned, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "bf16 network / f32 stepper",
        "data": "synthetic (seeded random phase |k|<=1.0, held-out seed 100)",
        "config": {"workload": f"fine 256^3 h=0.25 complex64+Kahan RK4 dt={fine_dt} vs coarse "
                               f"128^3 h=0.5 complex64+Kahan RK4 dt={cfg.dt} + 4-layer 3x3x3 "
                               "conv3d (2-16-16-16-2, GELU, bf16) after every step",
                   "weights": wsrc},
        "fine_ms_per_step": ms_fine, "coarse_ms_per_step": ms_plain,
        "network_ms_per_apply": ms_net, "learned_ms_per_step": ms_learned,
        "time_to_t50_s": {"fine": K_fine * ms_fine / 1e3, "learned": K * ms_learned / 1e3,
                          "coarse_plain": K * ms_plain / 1e3},
        "roofline": {"bound": "tensor", "kernel": "conv_fwd_kernel (4 layers + input pack)",
                     "achieved": achieved, "peak": tf_peak, "unit": "TFLOP/s",
                     "frac": achieved / tf_peak, "issued_flop_per_apply": issued_flop,
                     "useful_flop_per_apply": useful_flop,
                     "useful_tflops": useful_flop / (ms_net / 1e3) / 1e12,
                     "note": "issued = channels padded to 16 (N=16, K=16 per tap)"},
        "gpu_launches_per_apply": launches_per_apply,
        "clocks": clocks,
    }
    return line


def c2_params(precision, kahan):
    from gpe_b200 import GpeParams
    n, h = 128, 0.4
    xr = h * (n - 1) / 2
    return GpeParams(nx=n, ny=n, nz=n, xr=xr, yr=xr, zr=xr, scheme="rk45", eqn_to_solve=4,
                     bcs=2, order=4, precision=precision, kahan=kahan, g=1.0, mu=1.0)


def c2_initial_state():
    """Vortex ring of radius 8 in the xy-plane times the 'ring'-table Pade
    rarefaction pulse at x0 = -10 (numpy complex128, (nz, ny, nx))."""
    import numpy as np

    from gpe_b200 import ic
    p = c2_params(16, False)
    x = np.linspace(-p.xr, p.xr, p.nx)
    return ic.vortex_ring_xy(x, x, x, 0.0, 0.0, 0.0, 8.0) * ic.pade_pulse_ring(x, x, x, "ring", -10.0,
                                                                                  0.0, 0.0, 0.0)


def run_rkf45(args):
    print(json.dumps(measure_rkf45(args)), flush=True)
    return 0


def measure_rkf45(args):
    """C2: 128^3 reflective, 4th order, adaptive rkf45 (tolerance 1e-6, initial
    dt 0.005) to t = 20, complex128 and complex64 + Kahan.  An untimed pass
    counts the accepted steps the reference loop takes (while t + im_t <=
    t_end); the timed pass takes them in one advance, the step control on the
    device (no host synchronisation per attempt).  Roofline per attempt: the
    six Cash-Karp stages move 36 fields per site (576 B complex128; 288 B
    complex64, 304 B with the Kahan pair)."""
    import numpy as np
    import torch

    from gpe_b200 import GpeSolver
    torch.cuda.set_device(0)
    psi0 = c2_initial_state()
    t_end = args.t_end
    res = {}
    finals = {}
    sampler = ClockSampler(None)
    sampler.start()
    sites = 128 ** 3
    for name, prec, kahan, bps in (("f64", 16, False, 576), ("f32_kahan", 8, True, 304)):
        s = GpeSolver(c2_params(prec, kahan), dt=0.005)
        host = psi0.astype(np.complex64) if prec == 8 else psi0
        s.set_state(host)
        nsteps = 0
        while s.t + s.im_t <= t_end:
            s.solver()
            nsteps += 1
        for _ in range(max(args.warmup, 1)):  # graphs captured, clocks up
            s.t, s.im_t, s.dt = 0.0, 0.0, 0.005
            s.set_state(host)
            s.advance(min(nsteps, 20))
        s.t, s.im_t, s.dt = 0.0, 0.0, 0.005
        s.set_state(host)
        n0 = s.get_norm()
        st = torch.cuda.ExternalStream(s.stream_handle())
        a = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        lc0 = s.launch_count()
        t0 = time.perf_counter()
        a.record(st)
        s.advance(nsteps)
        e.record(st)
        e.synchronize()
        wall = time.perf_counter() - t0
        ms = a.elapsed_time(e)
        _, att = s.step_series(nsteps)
        attempts = int(att.sum())
        finals[name] = s.get_state(np.complex128)
        gbs = bps * sites * attempts / (ms / 1e3) / 1e9
        res[name] = {"steps": nsteps, "attempts": attempts, "t": s.t, "last_dt": s.dt.real,
                     "device_ms": ms, "wall_s": wall,
                     "norm_rel_change": abs(s.get_norm() - n0) / n0,
                     "site_updates_per_s": sites * nsteps / (ms / 1e3),
                     "alg_bytes_per_site_attempt": bps, "hbm_gbs": gbs,
                     "launches": s.launch_count() - lc0}
        s.close()
    clocks = sampler.stop()
    peak, peak_kind = load_peaks()
    ra, rb = np.abs(finals["f32_kahan"]) ** 2, np.abs(finals["f64"]) ** 2
    dens = float(np.linalg.norm(ra - rb) / np.linalg.norm(rb))
    f32 = res["f32_kahan"]
    line = {
        "metric": "time to t=20 (rkf45, 128^3)", "value": f32["device_ms"] / 1e3,
        "unit": "s", "n_gpus": 1, "steps": f32["steps"], "warmup": args.warmup,
        "ms_per_step": f32["device_ms"] / max(f32["steps"], 1),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (+Kahan)",
        "data": "synthetic (vortex ring r0=8 x Pade pulse at x0=-10)",
        "config": {"workload": "128^3 h=0.4 reflective, order 4, rkf45 tol 1e-6, dt0=0.005, "
                               "to t=%g, eqn 4 g=mu=1" % t_end,
                   "l2": "fields of 17-35 MB: the working set of a stage fits in L2"},
        "runs": res, "density_rel_l2_f32_vs_f64": dens, "clocks": clocks,
        "roofline": {"bound": "hbm", "kernel": "Cash-Karp stage kernels (one attempt = 6 launches)",
                     "achieved": f32["hbm_gbs"], "peak": peak, "unit": "GB/s",
                     "frac": f32["hbm_gbs"] / peak, "peak_source": peak_kind,
                     "f64_achieved": res["f64"]["hbm_gbs"],
                     "f64_frac": res["f64"]["hbm_gbs"] / peak, "traffic": None},
        "gpu_launches": f32["launches"],
        "note": "step control on the device: each step is one CUDA graph (conditional WHILE "
                "node around the attempt); the whole run is one advance call",
    }
    return line


def spectrum_cpu_sample(n: int = 128, min_seconds: float = 10.0, max_calls: int = 20):
    """Times the vectorised oracle (numpy, one thread: pocketfft backward
    transform, condensate row, spectrum) on an n^3 random-phase state;
    returns (sites/s, calls, seconds)."""
    import numpy as np

    from oracle import spectral_ref as ref
    xr = 0.5 * (n - 1)
    ph = ref.splitmix_phases(0, n ** 3).reshape(n, n, n)
    psi = ref.random_phase_fast(n, n, n, 0.75, 0.75, ph)
    calls = 0
    t0 = time.perf_counter()
    while True:
        _, a = ref.condensed_fast(psi, xr, xr, xr)
        ref.spectrum_fast(a)
        calls += 1
        el = time.perf_counter() - t0
        if (el >= min_seconds and calls >= 2) or calls >= max_calls:
            break
    return n ** 3 * calls / el, calls, el


def run_spectrum(args):
    """condensed_particles + spectrum of a resident 512^3 complex128 state
    (the reference's random_phase example parameters nv = enerv = 0.75 on a
    512^3 grid): one call = pack psi, backward cuFFT Z2Z, the spectrum
    reduction pass and its finaliser.  Metric: sites/s."""
    import numpy as np
    import torch

    from gpe_b200 import GpeParams, GpeSolver, lib
    from gpe_b200._lib import check
    torch.cuda.set_device(0)
    n = args.grid
    xr = 0.5 * (n - 1)
    prm = GpeParams(nx=n, ny=n, nz=n, xr=xr, yr=xr, zr=xr, scheme="rk4", eqn_to_solve=4, bcs=1,
                    order=2, precision=16, g=1.0, mu=1.0)
    s = GpeSolver(prm, dt=0.01)
    amp, kc2 = s.random_phase(0.75, 0.75, 0)
    stream = torch.cuda.ExternalStream(s.stream_handle())
    for _ in range(args.warmup):
        c = s.condensed_particles()
    props = torch.cuda.get_device_properties(0)
    uuid = str(getattr(props, "uuid", "") or "")
    sampler = ClockSampler(uuid[-12:] if uuid else None)
    sampler.start()
    time.sleep(0.3)
    s.set_timing(True)
    s.timing()
    lc0 = s.launch_count()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        c = s.condensed_particles()
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    launches = s.launch_count() - lc0
    fam = s.timing()
    s.set_timing(False)
    clocks = sampler.stop()
    sites = n ** 3
    value = sites * args.steps / (ms / 1e3)
    peak, peak_kind = load_peaks()
    d = fam["spectrum"]
    per_launch_ms = d["ms"] / max(d["launches"], 1)
    alg_bytes = 16 * sites  # one read of the transformed complex128 field
    achieved = alg_bytes / (per_launch_ms / 1e3) / 1e9
    traffic = load_traffic().get("spectrum_kernel")
    roofline = {"bound": "hbm", "kernel": "spectrum_kernel<double>", "achieved": achieved,
                "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": traffic, "alg_bytes_per_launch": alg_bytes,
                "per_launch_ms": per_launch_ms, "families": fam}

    # end to end: pinned host state in, condensed_particles, row + spectra out
    nb = sites * 16
    L = lib()
    hin = L.gpe_gpu_host_alloc(nb)
    a_in = np.ctypeslib.as_array(ctypes.cast(hin, ctypes.POINTER(ctypes.c_double)), (2 * sites,))
    a_in[:] = s.get_state().view(np.float64).ravel()
    ke = max(1, args.e2e_steps)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(ke):
        check(L.gpe_gpu_set_state(s.handle, ctypes.c_void_p(hin), 16), s.handle)
        s.condensed_particles()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / ke
    L.gpe_gpu_host_free(ctypes.c_void_p(hin))
    e2e = {"value": sites / (e2e_ms / 1e3), "unit": "sites/s", "h2d_bytes_per_step": nb,
           "d2h_bytes_per_step": 8 * (21 + n // 2), "ms_per_step": e2e_ms,
           "form": "gpe_gpu_set_state (pinned host psi) + gpe_gpu_condensed_particles "
                   "(row, eta, nharm, F to host), per call"}

    # vortex line length of the same state (gpe_gpu_linelength), its own line
    s.linelength()
    s.set_timing(True)
    s.timing()
    e0.record(stream)
    kl = 5
    for _ in range(kl):
        length = s.linelength()
    e1.record(stream)
    torch.cuda.synchronize()
    lfam = s.timing()
    s.set_timing(False)
    line_ms = e0.elapsed_time(e1) / kl
    cells_ms = lfam["other"]["ms"] / max(lfam["other"]["launches"], 1)
    linelen = {"length": length, "ms_per_call": line_ms, "sites_per_s": sites / (line_ms / 1e3),
               "cells_kernel_ms": cells_ms,
               "cells_kernel_gbs": 16 * sites / (cells_ms / 1e3) / 1e9}
    # zero finders of the same state: counts, points to host (wall clock, a host sync per
    # pass), into a new array per call and into one page-locked buffer kept across calls
    from gpe_b200._lib import pinned_empty
    zc, _ = s.zeros()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    zc, zp = s.zeros()
    new_ms = (time.perf_counter() - t0) * 1e3
    del zp
    buf = pinned_empty((int(zc.sum()), 3), np.float64)
    s.zeros(out=buf)
    t0 = time.perf_counter()
    zc, zp = s.zeros(out=buf)
    kept_ms = (time.perf_counter() - t0) * 1e3
    del zp, buf
    zeros = {"points": int(zc.sum()), "per_section": zc.tolist(),
             "ms_per_call_wall": new_ms, "ms_per_call_wall_kept_pinned": kept_ms,
             "note": "two passes (count, write) plus the point list copied to the host: into a "
                     "new array, and into a page-locked buffer reused across calls (out=)"}
    s.close()
    cpu = None
    if not args.no_cpu_baseline:
        v, calls, el = spectrum_cpu_sample()
        cpu = {"value": v, "unit": "sites/s", "cores": 1, "kind": "port",
               "sample": f"{calls} calls on a 128^3 random-phase state (vectorised numpy oracle: "
                         f"backward FFT, condensate row, spectrum), 1 thread, {el:.1f} s"}
        import oracle
        from oracle import spectral_ref as ref
        m = 128
        ph = ref.splitmix_phases(0, m ** 3).reshape(m, m, m)
        small = ref.random_phase_fast(m, m, m, 0.75, 0.75, ph)
        t0 = time.perf_counter()
        oracle.linelength(small, 1.0)
        linelen["cpu_sites_per_s"] = m ** 3 / (time.perf_counter() - t0)
        linelen["cpu_sample"] = "oracle linelength (C, 1 thread) on a 128^3 random-phase state"
    line = {
        "metric": "condensed_particles + spectrum throughput", "value": value, "unit": "sites/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (random_phase IC, nv = enerv = 0.75, SplitMix64 seed 0)",
        "config": {"workload": f"{n}^3 complex128 state: pack, backward cuFFT Z2Z, spectrum "
                               "reduction + finaliser per call",
                   "comp_amp": amp, "kc2": kc2,
                   "l2": f"state {16 * sites / 1e9:.2f} GB > L2, no flush needed"},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
        "gpu_launches": int(launches), "gpu_launches_per_step": launches / args.steps,
        "n0_over_V": c.row["n0_over_V"], "eta": c.eta.tolist(), "nharm": c.nharm.tolist(),
        "linelength": linelen, "zeros": zeros,
    }
    print(json.dumps(line), flush=True)
    return 0


def measure_others(args):
    """C2, C4 and C5 in short form for the default line: each one's metric,
    value, roofline and end-to-end figures from a run of its own workload
    (rkf45 to t = 20; 200 ensemble steps; 200 learned and fine steps)."""
    import torch

    def short(line, keep):
        out = {k: line[k] for k in ("metric", "value", "unit", "ms_per_step", "higher_is_better",
                                    "config", "roofline", "clocks") if k in line}
        out.update({k: line[k] for k in keep if k in line})
        return out

    res = {}
    ns = argparse.Namespace(t_end=20.0, warmup=3)
    res["c2_rkf45"] = short(measure_rkf45(ns), ("runs", "density_rel_l2_f32_vs_f64",
                                                 "gpu_launches"))
    torch.cuda.empty_cache()
    ns = argparse.Namespace(steps=200, warmup=5)
    ens = measure_ensemble(ns)
    ens["launch"] = {k: v for k, v in ens["launch"].items() if k != "table_ms"}
    res["c4_ensemble"] = short(ens, ("sequential", "speedup_vs_sequential", "e2e", "launch",
                                     "gpu_launches"))
    torch.cuda.empty_cache()
    ns = argparse.Namespace(steps=200, warmup=5)
    res["c5_learned"] = short(measure_learned(ns), (
        "fine_ms_per_step", "coarse_ms_per_step", "network_ms_per_apply", "learned_ms_per_step",
        "time_to_t50_s", "gpu_launches_per_apply"))
    torch.cuda.empty_cache()
    return res


def workload_config(ngpus, n=N_GRID, storage="complex64+kahan"):
    form = ("complex64 psi + Kahan compensation" if storage == "complex64+kahan"
            else "complex128 psi (the reference's FP64 path)")
    return {"workload": f"{n}^3 periodic grid, h=0.5, 4th-order FD, RK4 dt=0.005, equation 4 "
                        f"(g=mu=1, V=0), {form}, FP64 norm per step",
            "grid": [n, n, n], "h": H, "dt": DT, "scheme": "rk4", "order": 4,
            "bcs": "periodic", "storage": storage,
            "ic": "random phase, |k|<=1.0, seed 0",
            "l2": f"inputs larger than L2 (each field {8 * (n + 4) ** 3 / 1e9:.2f} GB, "
                  "6 fields) - no flush needed",
            "parallelism": f"replicas x{ngpus}" if ngpus > 1 else "single GPU"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="gpe_b200", choices=["gpe_b200", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=8)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-others", action="store_true",
                    help="default workload: skip the C2 / C4 / C5 measurements that follow C3")
    ap.add_argument("--grid", type=int, default=N_GRID,
                    help="cube edge (default 512; smaller sizes are for profiling captures)")
    ap.add_argument("--workload", default="cube",
                    choices=["cube", "ensemble", "learned", "rkf45", "spectrum"])
    ap.add_argument("--t-end", type=float, default=20.0, help="rkf45 workload end time")
    ap.add_argument("--ens-shape", default=None,
                    help="ensemble workload: fixed launch shape 'tile_y,zchunk,ctas_per_sm' "
                         "instead of the autotuner's choice")
    ap.add_argument("--decomp", default="replicas", choices=["replicas", "slab"],
                    help="N > 1: independent 512^3 replicas per GPU (weak scaling), or one "
                         "512^3 grid split into NCCL z-slabs (strong scaling)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "ensemble":
        if "--steps" not in sys.argv:
            args.steps = 500
        return run_ensemble(args)
    if args.workload == "rkf45":
        return run_rkf45(args)
    if args.workload == "spectrum":
        if "--steps" not in sys.argv:
            args.steps = 20
        return run_spectrum(args)
    if args.workload == "learned":
        if "--steps" not in sys.argv:
            args.steps = 200
        return run_learned(args)

    import numpy as np
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from gpe_b200 import GpeParams, GpeSolver, lib

    n = args.grid
    xr = H * (n - 1) / 2
    prm = GpeParams(nx=n, ny=n, nz=n, xr=xr, yr=xr, zr=xr, scheme="rk4", eqn_to_solve=4, bcs=1,
                    order=4, precision=8, kahan=True, g=1.0, mu=1.0, device=local)
    slab = world > 1 and args.decomp == "slab"
    from gpe_b200.ic import random_phase
    psi0 = random_phase(torch, n, H, KMAX, 0, torch.device("cuda", local))
    if slab:
        # one grid, z-slabs by para_range, NCCL ghost exchange after every
        # stage and all-reduced norms (the reference's MPI decomposition)
        from gpe_b200.dist import SlabSolver
        s = SlabSolver(prm, rank, world, dist, device=local, tau=DT)
        a, b = s.plan.z_range
        s.set_state(psi0[a:b + 1].contiguous())
    else:
        s = GpeSolver(prm, tau=DT)
        s.set_state(psi0)
    del psi0
    torch.cuda.empty_cache()
    stream = torch.cuda.ExternalStream(s.stream_handle(), device=local)

    # warm-up
    s.advance(args.warmup)

    props = torch.cuda.get_device_properties(local)
    uuid = str(getattr(props, "uuid", "") or "")
    sampler = ClockSampler(uuid[-12:] if uuid else None)
    sampler.start()
    time.sleep(0.3)
    s.set_timing(True)
    s.timing()  # reset accumulators
    lc0 = s.launch_count()
    if dist:
        dist.barrier()
    torch.cuda.synchronize(local)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    norms = s.advance(args.steps)
    ev1.record(stream)
    torch.cuda.synchronize(local)
    if dist:
        dist.barrier()
    ms = ev0.elapsed_time(ev1)
    launches = s.launch_count() - lc0
    fam = s.timing()
    s.set_timing(False)
    clocks = sampler.stop()
    ms_max = ms
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
    # sites this rank steps, and the job's site-updates per step
    sites = n * n * (s.plan.nz if slab else n)
    job_sites = n ** 3 if slab else world * n ** 3
    value = job_sites * args.steps / (ms_max / 1e3)

    # roofline of the dominant kernel family and of the whole step
    peak, peak_kind = load_peaks()
    dominant = max(("stage_first", "stage_mid", "stage_last"), key=lambda f: fam[f]["ms"])
    d = fam[dominant]
    per_launch_ms = d["ms"] / max(d["launches"], 1)
    # bytes from the sites the family's launches covered (a slab's stage is
    # two launches when its ghost exchange overlaps the interior planes)
    alg_bytes = BYTES_PER_FAMILY[dominant] * d["sites"] / max(d["launches"], 1)
    achieved = BYTES_PER_FAMILY[dominant] * d["sites"] / (d["ms"] / 1e3) / 1e9
    traffic = load_traffic().get(dominant)
    kernel_ms_step = sum(fam[f]["ms"] for f in ("stage_first", "stage_mid", "stage_last",
                                                "reduce")) / args.steps
    step_gbs = BYTES_PER_STEP * sites / (kernel_ms_step / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": f"stage_kernel ({dominant})",
                "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": traffic, "alg_bytes_per_launch": alg_bytes,
                "per_launch_ms": per_launch_ms,
                "step": {"alg_bytes_per_site": BYTES_PER_STEP, "kernel_ms_per_step": kernel_ms_step,
                         "achieved": step_gbs, "frac": step_gbs / peak,
                         "frac_vs_nominal_8000": step_gbs / 8000.0},
                "families": fam}

    # end to end through the C-ABI with host buffers (pinned), host<->device
    # copies inside the timed region: the literal solver(var_in, var_out) form
    nb = sites * 8
    L = lib()
    hin = L.gpe_gpu_host_alloc(nb)
    hout = L.gpe_gpu_host_alloc(nb)
    a_in = np.ctypeslib.as_array(ctypes.cast(hin, ctypes.POINTER(ctypes.c_float)), (2 * sites,))
    a_out = np.ctypeslib.as_array(ctypes.cast(hout, ctypes.POINTER(ctypes.c_float)), (2 * sites,))
    tmp = s.get_state(np.complex64)
    a_in[:] = tmp.view(np.float32).ravel()
    del tmp
    from gpe_b200._lib import GpeStepInfoC, GpeTimeC, check
    ke = max(1, args.e2e_steps)
    if dist:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(ke):
        tm = GpeTimeC(s.t, s.im_t, s.dt.real, s.dt.imag, s.p, 0)
        info = GpeStepInfoC()
        check(L.gpe_gpu_solver_host(s.handle, ctypes.c_void_p(hin), ctypes.c_void_p(hout), 8,
                                    ctypes.byref(tm), ctypes.byref(info)), s.handle)
        s.t, s.im_t = tm.t, tm.im_t
        hin, hout = hout, hin
    e1.record(stream)
    torch.cuda.synchronize(local)
    e2e_ms = e0.elapsed_time(e1) / ke
    if dist:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    L.gpe_gpu_host_free(ctypes.c_void_p(hin))
    L.gpe_gpu_host_free(ctypes.c_void_p(hout))
    e2e = {"value": job_sites / (e2e_ms / 1e3), "unit": "site-updates/s",
           "h2d_bytes_per_step": nb, "d2h_bytes_per_step": nb, "ms_per_step": e2e_ms,
           "form": "gpe_gpu_solver_host: pinned host psi in -> step -> host psi out, per step"}

    # resident form: the reference loop's per-step calls (solver + get_norm)
    e0.record(stream)
    for _ in range(ke):
        s.solver()
        s.get_norm()
    e1.record(stream)
    torch.cuda.synchronize(local)
    res_ms = e0.elapsed_time(e1) / ke
    e2e_resident = {"value": job_sites / (res_ms / 1e3), "unit": "site-updates/s",
                    "h2d_bytes_per_step": ctypes.sizeof(GpeTimeC), "d2h_bytes_per_step": 8,
                    "ms_per_step": res_ms,
                    "form": "psi resident; per step gpe_gpu_solver + gpe_gpu_norm (8 B read back)"}
    s.close()

    # the other configurations, measured in the same run on the same GPU after
    # the C3 timing: adaptive rkf45 to t = 20 (C2), the 64-run ensemble (C4)
    # and the learned coarse path against the fine path (C5)
    others = None
    if world == 1 and not args.no_others:
        others = measure_others(args)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        v, st, ss, el = cpu_sample(threads)
        cpu = {"value": v, "unit": "site-updates/s", "cores": threads, "kind": "port",
               "sample": f"{st} RK4 steps (+ get_norm) of a 512x512x8 periodic slab of the "
                         f"workload ({ss} sites), FP64 oracle with the reference's pass "
                         f"structure, {threads} OpenMP threads, {el:.1f} s"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "site-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "strong" if slab else "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded random-phase IC, |k|<=1.0, torch Philox seed 0)",
            "config": dict(workload_config(world, n),
                           parallelism=(f"z-slabs x{world} (NCCL)" if slab else
                                        workload_config(world, n)["parallelism"])),
            "hbm_gbs_step": step_gbs,
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "e2e_resident": e2e_resident,
            "clocks": clocks, "gpu_launches": int(launches),
            "gpu_launches_per_step": launches / args.steps,
            "final_norm": float(norms[-1]) if len(norms) else None,
        }
        if others is not None:
            line["configs"] = others
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())

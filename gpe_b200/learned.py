"""Training and evaluation of the learned coarse-grid correction.

Workload (seeded, synthetic): fine grid 256^3, h = 0.25, periodic, 2nd-order
differences, equation 4 with g = mu = 1 and no trap, FP64, RK4 with
dt_f = 0.01; initial condition the random-phase field of |k| <= 1.0
(gpe_b200.ic.random_phase).  Coarse grid 128^3, h = 0.5: the fine field
restricted 2:1 (2x2x2 average, which lands exactly on the coarse nodes),
stepped with complex64 RK4 at dt = 0.02, followed by the network's
correction after every step.

Training pairs come from the fine solver itself: for a fine trajectory
psi_f(t_k), t_k = k dt, the input is one coarse step of R psi_f(t_k) and the
target R psi_f(t_{k+1}); the loss is mean |u + delta(u) - target|^2 and the
network learns what the coarse step misses.  Every forward, backward and
Adam update runs in the library's tcgen05 kernels (gpe_b200.cnn).

Training inputs are also taken on-policy: up to `rollout` corrected coarse
steps from a restricted fine state first, so the network learns to pull its
own drift back (without this the corrected run diverges by t = 50), plus a
little input noise.

Evaluation on held-out seeds: the same fine reference, restricted, against
the coarse run with and without the network: relative L2 error of the
density |psi|^2 on the coarse grid at the checkpoint times, and the drift of
the discrete energy H4 of each run -- next to the coarse-grid H4 of the
restricted fine state itself, which is not conserved (energy moves below the
coarse grid's resolution), so a corrected run that tracks the fine solution
drifts with it.

  python -m gpe_b200.learned --out results.json --weights cnn.npz
"""
from __future__ import annotations

import argparse
import json
import math
import time
from dataclasses import asdict, dataclass, field

import numpy as np

from .cnn import CoarseCorrector, init_weights, restrict
from .ic import random_phase
from .solver import GpeParams, GpeSolver


@dataclass
class LearnedConfig:
    fine_n: int = 256
    fine_h: float = 0.25
    coarse_n: int = 128
    dt: float = 0.04            # coarse step (twice the fine path's largest stable step)
    fine_substeps: int = 4      # fine reference steps per coarse step (dt_f = 0.01)
    kmax: float = 1.0
    out_scale: float = 0.01
    coarse_kahan: bool = True
    train_seeds: list = field(default_factory=lambda: [0, 1, 2, 3])
    t_train: float = 10.0
    iters: int = 6000
    lr: float = 1e-3
    lr_final: float = 1e-4
    rollout: int = 8            # on-policy inputs: up to this many corrected steps first
    noise: float = 0.002        # std of complex Gaussian noise added to training inputs
    eval_seeds: list = field(default_factory=lambda: list(range(100, 116)))
    t_end: float = 50.0
    checkpoints: list = field(default_factory=lambda: [1.0, 5.0, 10.0, 20.0, 50.0])
    device: int = 0
    # coarse base: order 2, or order 4 with coarse_match = r > 0 (a Laplacian
    # that disperses like the 2nd-order one at spacing r h: r = 0.5 matches
    # the fine grid), or plain order 4 with coarse_order = 4, coarse_match = 0
    coarse_order: int = 2
    coarse_match: float = 0.0
    # rescale psi after every correction to the norm of the step it corrects
    preserve_norm: bool = False

    @property
    def coarse_h(self) -> float:
        return self.fine_h * self.fine_n / self.coarse_n


def config_from_weights(z, cfg: LearnedConfig | None = None) -> LearnedConfig:
    """The coarse method a weights file was trained for (its dt, stencil,
    output scale and norm handling), on top of cfg or the defaults."""
    cfg = cfg or LearnedConfig()
    if "out_scale" in z:
        cfg.out_scale = float(z["out_scale"])
    if "dt" in z:
        dt = float(z["dt"])
        cfg.fine_substeps = int(round(dt / (cfg.dt / cfg.fine_substeps)))
        cfg.dt = dt
    if "coarse_order" in z:
        cfg.coarse_order = int(z["coarse_order"])
        cfg.coarse_match = float(z["coarse_match"])
    if "preserve_norm" in z:
        cfg.preserve_norm = bool(z["preserve_norm"])
    return cfg


def params(n: int, h: float, precision: int, kahan: bool = False, device: int = 0,
           order: int = 2, fd_match: float = 0.0) -> GpeParams:
    xr = (n - 1) * h / 2
    return GpeParams(nx=n, ny=n, nz=n, xr=xr, yr=xr, zr=xr, scheme="rk4", eqn_to_solve=4, bcs=1,
                     order=order, precision=precision, kahan=kahan, g=1.0, mu=1.0, device=device,
                     fd_match=fd_match)


def fine_solver(cfg: LearnedConfig, seed: int, precision: int = 16, kahan: bool = False,
                dt: float | None = None) -> GpeSolver:
    import torch
    dev = torch.device("cuda", cfg.device)
    s = GpeSolver(params(cfg.fine_n, cfg.fine_h, precision, kahan, cfg.device),
                  dt=dt if dt is not None else cfg.dt / cfg.fine_substeps)
    psi = random_phase(torch, cfg.fine_n, cfg.fine_h, cfg.kmax, seed, dev,
                       torch.complex128 if precision == 16 else torch.complex64)
    s.set_state(psi)
    del psi
    return s


def coarse_solver(cfg: LearnedConfig) -> GpeSolver:
    return GpeSolver(params(cfg.coarse_n, cfg.coarse_h, 8, cfg.coarse_kahan, cfg.device,
                            cfg.coarse_order, cfg.coarse_match), dt=cfg.dt)


def restricted(cfg: LearnedConfig, fine: GpeSolver):
    import torch
    n = cfg.coarse_n
    out = torch.empty((n, n, n), dtype=torch.complex64, device=torch.device("cuda", cfg.device))
    restrict(fine, out)
    return out


def generate(cfg: LearnedConfig, seed: int, t_end: float):
    """Restricted fine states at t = k dt, k = 0..K (one CUDA tensor)."""
    import torch
    K = int(round(t_end / cfg.dt))
    n = cfg.coarse_n
    seq = torch.empty((K + 1, n, n, n), dtype=torch.complex64,
                      device=torch.device("cuda", cfg.device))
    f = fine_solver(cfg, seed)
    restrict(f, seq[0])
    for k in range(K):
        f.advance(cfg.fine_substeps)
        restrict(f, seq[k + 1])
    f.close()
    return seq


def pair_loss(u, target) -> float:
    """Mean over sites of |u - target|^2 (the loss of the zero correction)."""
    import torch
    return float(torch.mean(torch.abs(u - target) ** 2).item())


def train(cfg: LearnedConfig, net: CoarseCorrector, data, log_every: int = 500) -> dict:
    """Adam on random pairs of the training trajectories; cosine learning
    rate from lr to lr_final.  With cfg.rollout = M > 0, a pair's input is
    the network's own state: m in [0, M] corrected coarse steps from
    R psi_f(t_{k-m}) reach t_k, then one coarse step, against R psi_f(t_{k+1})
    -- the network learns to pull its own drift back to the fine solution.
    Returns the loss history and, every log_every iterations, the loss of
    the zero correction on the same pair."""
    import torch
    rng = np.random.default_rng(1234)
    gen = torch.Generator(device=data[0].device)
    gen.manual_seed(4321)
    c = coarse_solver(cfg)
    roll = None
    if cfg.rollout > 0:
        roll = coarse_solver(cfg)
        net.attach(roll)
    state = torch.empty_like(data[0][0])
    hist, base = [], []
    t0 = time.perf_counter()
    for it in range(cfg.iters):
        s = int(rng.integers(len(data)))
        m = int(rng.integers(cfg.rollout + 1)) if roll is not None else 0
        k = int(rng.integers(m, data[s].shape[0] - 1))
        if m > 0:
            roll.set_state(data[s][k - m])
            roll.advance(m)
            roll.get_state_device(state)
        else:
            state.copy_(data[s][k])
        if cfg.noise > 0:
            z = torch.randn(state.shape, generator=gen, device=state.device, dtype=torch.complex64)
            state.add_(cfg.noise * z)
        c.set_state(state)
        c.solver()
        lr = cfg.lr_final + 0.5 * (cfg.lr - cfg.lr_final) * (1 + math.cos(math.pi * it / cfg.iters))
        loss = net.train_step(c, data[s][k + 1], lr)
        hist.append(loss)
        if it % log_every == 0 or it == cfg.iters - 1:
            u = torch.empty_like(data[s][k + 1])
            c.get_state_device(u)
            base.append((it, k, m, loss, pair_loss(u, data[s][k + 1])))
    c.close()
    if roll is not None:
        roll.close()
    return {"loss": hist, "checks": base, "seconds": time.perf_counter() - t0}


def density_error(a, b) -> float:
    import torch
    da = torch.abs(a) ** 2
    db = torch.abs(b) ** 2
    return float((torch.linalg.vector_norm(da - db) / torch.linalg.vector_norm(db)).item())


def evaluate(cfg: LearnedConfig, net: CoarseCorrector | None, seeds, t_end: float,
             checkpoints) -> list:
    """Per seed: density errors at the checkpoints and H4 drift of the plain
    coarse run and (when net is given) the corrected one."""
    import torch
    out = []
    ck = sorted(t for t in checkpoints if t <= t_end + 1e-9)
    for seed in seeds:
        f = fine_solver(cfg, seed)
        ref0 = restricted(cfg, f)
        runs = {"plain": coarse_solver(cfg)}
        if net is not None:
            runs["learned"] = coarse_solver(cfg)
            net.attach(runs["learned"])
        h0 = {}
        for name, c in runs.items():
            c.set_state(ref0)
            h0[name] = c.energy()[1]
        hf0 = f.energy()[1]
        probe = coarse_solver(cfg)  # coarse-grid H4 of the restricted fine state
        probe.set_state(ref0)
        hr0 = probe.energy()[1]
        rec = {"seed": seed, "t": [], "fine_H4_drift": [], "restricted_H4_drift": []}
        for name in runs:
            rec[name] = {"density_err": [], "H4_drift": []}
        k_done = 0
        for t in ck:
            k = int(round(t / cfg.dt))
            f.advance((k - k_done) * cfg.fine_substeps)
            ref = restricted(cfg, f)
            rec["t"].append(t)
            rec["fine_H4_drift"].append(abs(f.energy()[1] - hf0) / abs(hf0))
            probe.set_state(ref)
            rec["restricted_H4_drift"].append(abs(probe.energy()[1] - hr0) / abs(hr0))
            for name, c in runs.items():
                c.advance(k - k_done)
                u = torch.empty_like(ref)
                c.get_state_device(u)
                rec[name]["density_err"].append(density_error(u, ref))
                rec[name]["H4_drift"].append(abs(c.energy()[1] - h0[name]) / abs(h0[name]))
            k_done = k
        for c in runs.values():
            c.close()
        probe.close()
        f.close()
        out.append(rec)
    return out


def summarize(results: list) -> dict:
    s = {}
    names = [k for k in results[0] if isinstance(results[0][k], dict)]
    ts = results[0]["t"]
    for name in names:
        errs = np.array([r[name]["density_err"] for r in results])
        drift = np.array([r[name]["H4_drift"] for r in results])
        s[name] = {"t": ts, "density_err_median": np.median(errs, axis=0).tolist(),
                   "density_err_max": errs.max(axis=0).tolist(),
                   "H4_drift_median": np.median(drift, axis=0).tolist()}
    s["fine_H4_drift_median"] = np.median([r["fine_H4_drift"] for r in results], axis=0).tolist()
    s["restricted_H4_drift_median"] = np.median([r["restricted_H4_drift"] for r in results],
                                                axis=0).tolist()
    return s


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description="train and evaluate the learned coarse-grid correction")
    ap.add_argument("--out", required=True)
    ap.add_argument("--weights", required=True, help="npz written after training (w, b)")
    ap.add_argument("--load", help="skip training: evaluate these weights")
    ap.add_argument("--iters", type=int)
    ap.add_argument("--t-train", type=float)
    ap.add_argument("--train-seeds", type=int, help="number of training seeds (0, 1, ...)")
    ap.add_argument("--eval-seeds", type=int, help="number of held-out seeds (100, 101, ...)")
    ap.add_argument("--t-end", type=float)
    ap.add_argument("--fine-n", type=int)
    ap.add_argument("--coarse-n", type=int)
    ap.add_argument("--lr", type=float)
    ap.add_argument("--out-scale", type=float)
    ap.add_argument("--rollout", type=int)
    ap.add_argument("--noise", type=float)
    ap.add_argument("--dt", type=float, help="coarse step (a multiple of the fine 0.01)")
    ap.add_argument("--checkpoints", help="comma-separated times, or start:stop:step")
    ap.add_argument("--coarse-order", type=int, choices=[2, 4])
    ap.add_argument("--coarse-match", type=float, help="order-4 dispersion match r (0.5: fine grid)")
    ap.add_argument("--no-net", action="store_true", help="evaluate the coarse base alone")
    ap.add_argument("--preserve-norm", action="store_true",
                    help="keep the stepped norm through every correction")
    a = ap.parse_args(argv)
    cfg = LearnedConfig()
    if a.iters is not None:
        cfg.iters = a.iters
    if a.t_train is not None:
        cfg.t_train = a.t_train
    if a.train_seeds is not None:
        cfg.train_seeds = list(range(a.train_seeds))
    if a.eval_seeds is not None:
        cfg.eval_seeds = list(range(100, 100 + a.eval_seeds))
    if a.t_end is not None:
        cfg.t_end = a.t_end
    if a.fine_n is not None:
        cfg.fine_n = a.fine_n
    if a.coarse_n is not None:
        cfg.coarse_n = a.coarse_n
    if a.lr is not None:
        cfg.lr, cfg.lr_final = a.lr, a.lr / 10
    if a.out_scale is not None:
        cfg.out_scale = a.out_scale
    if a.rollout is not None:
        cfg.rollout = a.rollout
    if a.noise is not None:
        cfg.noise = a.noise
    if a.dt is not None:
        cfg.fine_substeps = int(round(a.dt / (cfg.dt / cfg.fine_substeps)))
        cfg.dt = a.dt
    if a.coarse_match is not None:
        cfg.coarse_order, cfg.coarse_match = 4, a.coarse_match
    if a.coarse_order is not None:
        cfg.coarse_order = a.coarse_order
    if a.preserve_norm:
        cfg.preserve_norm = True
    if a.checkpoints:
        ck = []
        for item in a.checkpoints.split(","):
            if ":" in item:
                t0_, t1_, st_ = (float(v) for v in item.split(":"))
                ck += [round(v, 10) for v in np.arange(t0_, t1_ + 1e-9, st_)]
            else:
                ck.append(float(item))
        cfg.checkpoints = sorted(set(ck))
    import torch
    torch.cuda.set_device(cfg.device)
    n = cfg.coarse_n
    report = {"config": asdict(cfg)}
    if a.no_net:
        res = evaluate(cfg, None, cfg.eval_seeds, cfg.t_end, cfg.checkpoints)
        report["eval"] = res
        report["summary"] = summarize(res)
        with open(a.out, "w") as fh:
            json.dump(report, fh, indent=1)
        print(json.dumps(report["summary"]))
        return 0
    if a.load:
        z = np.load(a.load)
        w, b = z["w"], z["b"]
        if a.dt is None and a.coarse_match is None and a.coarse_order is None:
            cfg = config_from_weights(z, cfg)  # the method the weights were trained for
            cfg.preserve_norm = cfg.preserve_norm or a.preserve_norm
            report["config"] = asdict(cfg)
    else:
        net = CoarseCorrector(n, n, n, cfg.device, train=True, out_scale=cfg.out_scale,
                              preserve_norm=cfg.preserve_norm)
        t0 = time.perf_counter()
        data = [generate(cfg, s, cfg.t_train) for s in cfg.train_seeds]
        report["generate_seconds"] = time.perf_counter() - t0
        w, b = init_weights(7)
        net.set_weights(w, b)
        tr = train(cfg, net, data)
        del data
        torch.cuda.empty_cache()
        h = tr["loss"]
        m = max(1, len(h) // 20)
        report["train"] = {"seconds": tr["seconds"], "iters": cfg.iters,
                           "loss_first": float(np.mean(h[:m])), "loss_last": float(np.mean(h[-m:])),
                           "checks (iter, k, m, loss, zero-correction loss)": tr["checks"]}
        w, b = net.get_weights()
        # the weights carry the coarse method they were trained for
        np.savez_compressed(a.weights, w=w, b=b, out_scale=cfg.out_scale, dt=cfg.dt,
                            coarse_order=cfg.coarse_order, coarse_match=cfg.coarse_match,
                            preserve_norm=cfg.preserve_norm)
        net.close()
    net = CoarseCorrector(n, n, n, cfg.device, out_scale=cfg.out_scale,
                          preserve_norm=cfg.preserve_norm)
    net.set_weights(w, b)
    t0 = time.perf_counter()
    res = evaluate(cfg, net, cfg.eval_seeds, cfg.t_end, cfg.checkpoints)
    report["eval_seconds"] = time.perf_counter() - t0
    report["eval"] = res
    report["summary"] = summarize(res)
    net.close()
    with open(a.out, "w") as fh:
        json.dump(report, fh, indent=1)
    print(json.dumps(report["summary"]))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())

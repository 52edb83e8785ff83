"""Training data, training and evaluation of the learned flux-correction
closure on 3D Kelvin-Helmholtz (triply periodic [0,1]^3, the sharp profile
extruded in x3 with seeded noise on all three velocity components, MUSCL
minmod + HLL + SSPRK3, float32).

Data: seeded fine runs at ``fine``^3 with a fixed step dt_c/f (f = the
filter factor, dt_c the coarse step), box-filtered f^3 to the coarse grid.
At every ``sample_every``-th coarse step the pair (U_bar(t), U_bar(t+dt_c))
gives the defect D = U_bar(t+dt_c) - S_c(U_bar(t)) of one plain coarse step
S_c; the network is trained so that dt_c * (-div dF) matches D (a-priori
loss, per-variable weights 1/mean(D_q^2), so the loss of a zero correction is
5).  Evaluation on held-out seeds: density L2 error at t_end against the
filtered fine run for plain coarse, coarse + closure and plain 2x-coarse
(filtered to the coarse grid), with the device time of each run.

    python -m multiphysics_fvm_b200.closure_train --fine 256 --factor 4 \\
        --train-seeds 32 --eval-seeds 8 --out closure.npz --report closure.json
"""
from __future__ import annotations

import argparse
import json
import math
import time
from dataclasses import asdict, dataclass, field

import numpy as np

from . import backend
from . import closure as CL
from .grid.geometry import build_grid


@dataclass
class Config:
    fine: int = 256
    factor: int = 4
    t_end: float = 1.0
    dt_coarse: float = 2e-3
    sample_every: int = 5
    train_seeds: list = field(default_factory=lambda: list(range(32)))
    eval_seeds: list = field(default_factory=lambda: list(range(1000, 1008)))
    epochs: int = 3
    lr: float = 1e-3
    defect_steps: int = 1   # k: target = (U_bar(t + k dt_c) - S_c^k(U_bar(t))) / k
    beta: float = 0.5
    net_seed: int = 0

    @property
    def coarse(self) -> int:
        return self.fine // self.factor

    @property
    def n_coarse_steps(self) -> int:
        return int(round(self.t_end / self.dt_coarse))


def kh_setup(n: int, seed: int):
    from .setups import kelvin_helmholtz_sharp as kh
    return kh.get_setup(n, n, n, seed=seed, precision="fp32", noise_all=True)


def new_sim(n: int, seed: int, initial_state: bool = True, device_ic: bool = True):
    """A float32 3D KH simulation; the initial state is written on the device
    (counter-based noise) or by the host initializer (NumPy noise) and uploaded."""
    s = kh_setup(n, seed)
    sim = backend.Simulation.from_setup(s)
    if initial_state and device_ic:
        sim.init_kelvin_helmholtz(s["initial_conditions"]["parameters"], seed)
    elif initial_state:
        g = build_grid(s["coordinate_system"], s["grid_config"])
        U = s["physics"].allocate_u(s["grid_config"])
        s["initial_conditions"]["initializer"](U, s["physical_parameters"], g, s["initial_conditions"]["parameters"])
        sim.upload(U)
    sim.set_time(0.0, math.inf, float(s["time_config"]["CFL"]))
    return sim


def generate(cfg: Config, seeds, log=print):
    """Training pairs (U_bar, D) as CUDA tensors (N, 5, n, n, n).  With k =
    defect_steps > 1 the defect is averaged over k coarse steps, which spreads
    the coarse scheme's own relaxation of a freshly filtered state over the
    window and keeps the persistent part that a correction can carry."""
    import torch
    f, nc, k = cfg.factor, cfg.coarse, cfg.defect_steps
    coarse = new_sim(nc, 0, initial_state=False)
    Us, Ds = [], []
    for seed in seeds:
        t0 = time.time()
        fine = new_sim(cfg.fine, seed)
        pending = []  # (coarse step at which the window ends, filtered start state)
        for m in range(cfg.n_coarse_steps + 1):
            if pending and m == pending[0][0]:
                _, ub0 = pending.pop(0)
                ubk = CL.filter_state(fine, f)
                CL.upload_dense(coarse, ub0)
                coarse.step(k, dt=cfg.dt_coarse)
                Ds.append((ubk - CL.download_dense(coarse)) / k)
                Us.append(ub0)
            if m == cfg.n_coarse_steps:
                break
            if m % cfg.sample_every == 0 and m + k <= cfg.n_coarse_steps:
                pending.append((m + k, CL.filter_state(fine, f)))
            fine.step(f, dt=cfg.dt_coarse / f)
        st = fine.status()
        fine.close()
        torch.cuda.synchronize()
        log(f"seed {seed}: {len(Us)} pairs, status {st}, {time.time() - t0:.1f} s")
        if st:
            raise RuntimeError(f"fine run of seed {seed} reported status {st}")
    coarse.close()
    return torch.stack(Us), torch.stack(Ds)


def normalisation(U, D, cfg: Config, gamma: float = 1.4):
    """Feature mean/scale, output scales and loss weights from the data."""
    import torch
    rho = U[:, 0]
    v = U[:, 1:4] / rho[:, None]
    p = (gamma - 1.0) * (U[:, 4] - 0.5 * rho * (v * v).sum(1))
    prim = torch.stack([rho, v[:, 0], v[:, 1], v[:, 2], p], 1)
    mean = prim.mean(dim=(0, 2, 3, 4)).double().cpu().numpy()
    scale = prim.std(dim=(0, 2, 3, 4)).double().cpu().numpy()
    rms = D.double().pow(2).mean(dim=(0, 2, 3, 4)).sqrt().cpu().numpy()
    h = 1.0 / cfg.coarse
    out_scale = rms * h / cfg.dt_coarse
    weight = 1.0 / (rms * rms)
    return dict(gamma=gamma, in_mean=mean, in_scale=np.maximum(scale, 1e-6), out_scale=out_scale,
                loss_weight=weight)


def apriori_loss(net: CL.Closure, U, D, cfg: Config) -> float:
    """Mean a-priori loss over samples (5 = no improvement over the plain step)."""
    h = (1.0 / cfg.coarse,) * 3
    tot = 0.0
    for i in range(U.shape[0]):
        net.features(U[i])
        net.forward()
        net.backward(D[i], cfg.dt_coarse, h)
        tot += net.loss()
    return tot / U.shape[0]


def train(cfg: Config, U, D, log=print, net: CL.Closure | None = None):
    import torch
    nc = cfg.coarse
    if net is None:
        net = CL.Closure((nc, nc, nc), seed=cfg.net_seed)
    nrm = normalisation(U, D, cfg)
    net.set_norm(**nrm)
    h = (1.0 / nc,) * 3
    g = torch.Generator().manual_seed(cfg.net_seed)
    curve = []
    t0 = time.time()
    it = 0
    for ep in range(cfg.epochs):
        order = torch.randperm(U.shape[0], generator=g).tolist()
        run = 0.0
        for k, i in enumerate(order):
            net.train_step(U[i], D[i], cfg.dt_coarse, h, cfg.lr)
            run += net.loss()
            it += 1
            if (k + 1) % 200 == 0 or k + 1 == len(order):
                curve.append((it, run / ((k % 200) + 1)))
                run = 0.0
        log(f"epoch {ep}: loss {curve[-1][1]:.4f} ({time.time() - t0:.1f} s)")
    return net, curve, time.time() - t0


def _rho_err(a, b) -> float:
    return float((a[0] - b[0]).double().pow(2).mean().sqrt().item())


def evaluate(cfg: Config, net: CL.Closure, seeds, betas=None, checkpoints: int = 4, log=print):
    """Per seed: density L2 error against the filtered fine run at
    ``checkpoints`` equally spaced times up to t_end, and the device time (ms)
    of each run, for plain coarse, coarse + closure at each clip factor in
    ``betas`` and plain 2x-coarse (filtered to the coarse grid)."""
    import torch
    betas = [cfg.beta] if betas is None else list(betas)
    f, nc, n = cfg.factor, cfg.coarse, cfg.n_coarse_steps
    seg = n // checkpoints
    nm = cfg.fine // 2
    rows = []
    plain = new_sim(nc, 0, initial_state=False)
    closed = new_sim(nc, 0, initial_state=False)
    mid = new_sim(nm, 0, initial_state=False)
    for seed in seeds:
        fine = new_sim(cfg.fine, seed)
        ic_c = CL.filter_state(fine, f)
        ic_m = CL.filter_state(fine, 2)
        refs, ms_fine = [], 0.0
        for _ in range(checkpoints):
            ms_fine += _timed(fine, seg * f, cfg.dt_coarse / f)
            refs.append(CL.filter_state(fine, f))
        fine.close()
        out = {"seed": seed, "t": [cfg.dt_coarse * seg * (c + 1) for c in range(checkpoints)], "ms_fine": ms_fine}
        runs = [("plain", plain, None, ic_c, 1, cfg.dt_coarse, 1)]
        runs += [(f"closure_b{b:g}", closed, b, ic_c, 1, cfg.dt_coarse, 1) for b in betas]
        runs += [("plain_2x", mid, None, ic_m, 2, cfg.dt_coarse / 2, 2)]
        for name, sim, beta, ic, mult, dt, back in runs:
            if beta is not None:
                net.attach(sim, beta=beta)  # resets the switch counter
            CL.upload_dense(sim, ic)
            sim.clear_status()
            sim.set_time(0.0, math.inf, 0.4)
            errs, ms = [], 0.0
            for c in range(checkpoints):
                ms += _timed(sim, seg * mult, dt)
                res = CL.filter_state(sim, back) if back > 1 else CL.download_dense(sim)
                errs.append(_rho_err(res, refs[c]))
            rec = {"err": errs, "ms": ms, "status": sim.status()}
            if beta is not None:
                rec["switched"] = CL.Closure.switch_count(sim)
                rec["beta"] = beta
            out[name] = rec
        rows.append(out)
        log(json.dumps(out))
        del refs
        torch.cuda.empty_cache()
    for s in (plain, closed, mid):
        s.close()
    return rows


def _timed(sim, steps: int, dt: float) -> float:
    """Advance `steps` fixed steps of size dt; device time in ms."""
    from . import _lib as L
    L.check(sim._lib.fvm_set_dt(sim._h, float(dt)), "fvm_set_dt")
    return sim.time_steps(steps, fixed_dt=True)


def summarise(rows):
    """Mean over seeds of the final-time error and the device time of each run."""
    names = [k for k in rows[0] if isinstance(rows[0][k], dict)]
    out = {"ms_fine": float(np.mean([r["ms_fine"] for r in rows]))}
    for k in names:
        out[f"err_{k}"] = float(np.mean([r[k]["err"][-1] for r in rows]))
        out[f"ms_{k}"] = float(np.mean([r[k]["ms"] for r in rows]))
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--fine", type=int, default=256)
    ap.add_argument("--factor", type=int, default=4)
    ap.add_argument("--t-end", type=float, default=1.0)
    ap.add_argument("--dt-coarse", type=float, default=2e-3)
    ap.add_argument("--sample-every", type=int, default=5)
    ap.add_argument("--train-seeds", type=int, default=32)
    ap.add_argument("--eval-seeds", type=int, default=8)
    ap.add_argument("--epochs", type=int, default=3)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--beta", type=float, default=0.5)
    ap.add_argument("--defect-steps", type=int, default=1)
    ap.add_argument("--betas", default="", help="comma-separated clip factors to evaluate (default: --beta)")
    ap.add_argument("--checkpoints", type=int, default=4)
    ap.add_argument("--weights", default="", help="evaluate these weights instead of training")
    ap.add_argument("--fct", action="store_true", help="flux-corrected transport bound on the corrections")
    ap.add_argument("--out", default="")
    ap.add_argument("--report", required=True)
    a = ap.parse_args(argv)
    cfg = Config(fine=a.fine, factor=a.factor, t_end=a.t_end, dt_coarse=a.dt_coarse, sample_every=a.sample_every,
                 train_seeds=list(range(a.train_seeds)), eval_seeds=list(range(1000, 1000 + a.eval_seeds)),
                 epochs=a.epochs, lr=a.lr, beta=a.beta, defect_steps=a.defect_steps)
    betas = [float(b) for b in a.betas.split(",") if b] or [cfg.beta]
    if a.weights:
        net = CL.Closure((cfg.coarse,) * 3)
        meta = net.load(a.weights)
        net.set_limiter(a.fct)
        rows = evaluate(cfg, net, cfg.eval_seeds, betas, a.checkpoints)
        rep = {"config": asdict(cfg), "fct": a.fct, "weights": a.weights, "weights_meta": meta, "eval": rows,
               "summary": summarise(rows)}
        with open(a.report, "w") as fh:
            json.dump(rep, fh, indent=1)
        print(json.dumps(rep["summary"]))
        return
    if not a.out:
        ap.error("--out is required when training")
    t0 = time.time()
    U, D = generate(cfg, cfg.train_seeds)
    t_gen = time.time() - t0
    nh = max(1, U.shape[0] // 10)
    net, curve, t_train = train(cfg, U, D)
    net.set_limiter(a.fct)
    # held-out a-priori check on the eval seeds' first pairs
    Uv, Dv = generate(Config(**{**asdict(cfg), "t_end": cfg.t_end / 2}), cfg.eval_seeds[:2])
    apri = apriori_loss(net, Uv, Dv, cfg)
    apri_train = apriori_loss(net, U[:nh], D[:nh], cfg)
    rows = evaluate(cfg, net, cfg.eval_seeds, betas, a.checkpoints)
    rep = {"config": asdict(cfg), "fct": a.fct, "pairs": int(U.shape[0]), "seconds_generate": t_gen, "seconds_train": t_train,
           "loss_curve": curve, "apriori_loss_heldout": apri, "apriori_loss_train_subset": apri_train,
           "apriori_loss_plain": 5.0, "eval": rows, "summary": summarise(rows)}
    net.save(a.out, meta={"config": asdict(cfg), "summary": rep["summary"]})
    with open(a.report, "w") as fh:
        json.dump(rep, fh, indent=1)
    print(json.dumps(rep["summary"]))


if __name__ == "__main__":
    main()

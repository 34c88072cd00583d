"""The learned coarse-grid flux correction: data, training and evaluation.

    python -m dev_field_efvm_b200.learned --train 2000 --eval 200 --out learned.json --save model.npz

Family: periodic [0,10]^2 boxes of 2-6 superposed isentropic vortices (strength
beta ~ U[1,4], radius ~ U[0.5,1.5], random centres, minimum-image distances) on a
random mean flow, plus smooth density and pressure modes (wave vectors |k| <= 4,
total amplitude <= 0.1).  The coarse grid is 64^2 (MUSCL-minmod + HLLC-Thornber,
SSP-RK3); the fine grid is 256^2 with a quarter of the coarse time step.

Data: every training trajectory runs on the fine grid in FP64 (batched on the
GPU) and is averaged 4x4 conservatively onto the coarse grid after each coarse
step.  For a coarse snapshot U^k the target residual is
R^k = (avg U_fine(t_{k+1}) - P(U^k)) / dt, with P one plain coarse step (batched
on the GPU).  The network is trained so that the divergence of its face
corrections cancels R (efvm_nn_loss_grad), with Adam, by the library's own
tensor-core kernels.

Evaluation on held-out seeds: density L1 distance to the averaged fine solution
after a number of coarse steps, for the plain 64^2 method, the corrected 64^2
method and the plain 128^2 method (averaged 2x2 onto 64^2), the device time of
each, and the fraction of faces where the sensor fell back to the plain flux.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import abi, cases

L = 10.0
GAMMA = 1.4


def family_state(n: int, seed: int) -> np.ndarray:
    """(n, n, 5) conserved state of the vortex family on the periodic box."""
    rng = np.random.default_rng(seed)
    h = L / n
    x = (np.arange(n) + 0.5) * h
    X, Y = np.meshgrid(x, x)
    u = np.full_like(X, rng.uniform(-0.5, 0.5))
    v = np.full_like(X, rng.uniform(-0.5, 0.5))
    dT = np.zeros_like(X)
    for _ in range(int(rng.integers(2, 7))):
        beta, r = rng.uniform(1.0, 4.0), rng.uniform(0.5, 1.5)
        cx, cy = rng.uniform(0.0, L, 2)
        dx = X - cx
        dx -= L * np.round(dx / L)
        dy = Y - cy
        dy -= L * np.round(dy / L)
        r2 = (dx * dx + dy * dy) / (r * r)
        f = np.exp(0.5 * (1.0 - r2))
        u += -beta / (2 * np.pi) * (dy / r) * f
        v += beta / (2 * np.pi) * (dx / r) * f
        dT += -(GAMMA - 1.0) * beta * beta / (8.0 * GAMMA * np.pi ** 2) * np.exp(1.0 - r2)
    if dT.min() < -0.6:  # overlapping vortices: keep the temperature positive
        dT *= 0.6 / -dT.min()
    T = 1.0 + dT
    modes = []
    for _ in range(2):
        field = np.zeros_like(X)
        amps = rng.uniform(0.0, 1.0, 3)
        amps *= rng.uniform(0.0, 0.1) / max(amps.sum(), 1e-12)
        for a in amps:
            while True:
                kx, ky = rng.integers(-4, 5, 2)
                if 0 < kx * kx + ky * ky <= 16:
                    break
            field += a * np.cos(2 * np.pi * (kx * X + ky * Y) / L + rng.uniform(0, 2 * np.pi))
        modes.append(field)
    rho = T ** (1.0 / (GAMMA - 1.0)) * (1.0 + modes[0])
    p = T ** (GAMMA / (GAMMA - 1.0)) * (1.0 + modes[1])
    return cases.prim_to_cons(rho, u, v, p, GAMMA)


def coarsen(u: np.ndarray, f: int) -> np.ndarray:
    """Conservative f x f block average of an (ny, nx, 5) state."""
    ny, nx, nv = u.shape
    return u.reshape(ny // f, f, nx // f, f, nv).mean(axis=(1, 3))


def grid_params(n: int, dt: float):
    grid, params, _, _ = cases.vortex_case(n, periodic=True, muscl=True, mean=(0.0, 0.0), cfl=0.4,
                                           seam=abi.SEAM_TRUE_PERIODIC)
    params.fixed_dt = dt
    return grid, params


def coarse_dt(seeds, n=64) -> float:
    """One time step for the whole family: CFL 0.4 on the coarse grid, over the
    initial states of `seeds`, times 0.9."""
    lam = 0.0
    h = L / n
    for s in seeds:
        u = coarsen(family_state(256, s), 256 // n)
        r = u[..., 0]
        vx, vy = u[..., 1] / r, u[..., 2] / r
        p = (GAMMA - 1) * (u[..., 4] - 0.5 * r * (vx * vx + vy * vy))
        a = np.sqrt(GAMMA * p / r)
        lam = max(lam, float(np.max((np.abs(vx) + a) / h + (np.abs(vy) + a) / h + a / h)))
    return 0.9 * 0.4 / lam


def run_fine(seeds, dt_c: float, k_steps: int, fine: int = 256, coarse: int = 64, chunk: int = 250):
    """Coarse snapshots [len(seeds), k_steps + 1, 4, coarse, coarse] (rho, m_x,
    m_y, E) of fine FP64 runs, and the device seconds they took."""
    from .device import Batch
    import torch

    f = fine // coarse
    grid, params = grid_params(fine, dt_c / f)
    out = np.zeros((len(seeds), k_steps + 1, 4, coarse, coarse))
    seconds = 0.0
    for c0 in range(0, len(seeds), chunk):
        part = seeds[c0:c0 + chunk]
        b = Batch([grid] * len(part), params)
        for k, s in enumerate(part):
            u = family_state(fine, s)
            b.upload(k, u)
            out[c0 + k, 0] = np.moveaxis(coarsen(u, f)[..., [0, 1, 2, 4]], -1, 0)
        for step in range(1, k_steps + 1):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            b.run(np.full(len(part), (step - 0.5 / f) * dt_c))
            seconds += time.perf_counter() - t0
            for k in range(len(part)):
                out[c0 + k, step] = np.moveaxis(coarsen(b.download(k), f)[..., [0, 1, 2, 4]], -1, 0)
        b.close()
    return out, seconds


def to_state5(q4: np.ndarray) -> np.ndarray:
    """[4, n, n] (rho, m_x, m_y, E) -> (n, n, 5) with rho_w = 0."""
    z = np.zeros(q4.shape[1:])
    return np.stack([q4[0], q4[1], q4[2], z, q4[3]], axis=-1)


def plain_step(states: np.ndarray, dt_c: float, n: int = 64) -> np.ndarray:
    """One plain coarse step of every state [S, 4, n, n] (batched on the GPU)."""
    from .device import Batch

    grid, params = grid_params(n, dt_c)
    out = np.zeros_like(states)
    chunk = 2048
    for c0 in range(0, len(states), chunk):
        part = states[c0:c0 + chunk]
        b = Batch([grid] * len(part), params)
        for k, q in enumerate(part):
            b.upload(k, to_state5(q))
        b.run(np.full(len(part), 0.5 * dt_c))
        for k in range(len(part)):
            out[c0 + k] = np.moveaxis(b.download(k)[..., [0, 1, 2, 4]], -1, 0)
        b.close()
    return out


def make_dataset(seeds, dt_c: float, k_steps: int):
    """Training pairs (U^k, R^k) from the fine trajectories of `seeds`."""
    traj, fine_s = run_fine(seeds, dt_c, k_steps)
    states = traj[:, :-1].reshape(-1, 4, 64, 64)
    targets = traj[:, 1:].reshape(-1, 4, 64, 64)
    resid = (targets - plain_step(states, dt_c)) / dt_c
    return states, resid, fine_s


def train(states, resid, dt_c: float, epochs: int, batch: int = 32, lr: float = 2e-3, seed: int = 0, log=print):
    """Train a FluxNet on the pairs; returns the network and the loss history."""
    import torch
    from .device import FluxNet

    dx = L / 64
    w = 1.0 / np.maximum(np.mean(resid ** 2, axis=(0, 2, 3)), 1e-30)
    w = w / w.sum() * 4.0
    out_scale = float(np.sqrt(np.mean(resid ** 2)) * dx)
    net = FluxNet(out_scale=out_scale, gamma=GAMMA, seed=seed)
    S = torch.tensor(states, device="cuda")
    R = torch.tensor(resid, device="cuda")
    rng = np.random.default_rng(seed)
    hist = []
    steps = 0
    total = epochs * max(1, len(states) // batch)
    for ep in range(epochs):
        order = rng.permutation(len(states))
        losses = []
        for b0 in range(0, len(order) - batch + 1, batch):
            idx = torch.tensor(order[b0:b0 + batch], device="cuda")
            loss = net.loss_grad(S[idx].contiguous(), R[idx].contiguous(), dx, dx, w)
            net.adam(lr * 0.5 * (1 + np.cos(np.pi * steps / total)))
            steps += 1
            losses.append(loss)
        hist.append(float(np.mean(losses)))
        log(f"epoch {ep}: loss {hist[-1]:.4e} ({hist[-1] / hist[0]:.4f} of the first epoch's)")
    return net, hist, {"w": w.tolist(), "out_scale": out_scale}


def evaluate(net, seeds, dt_c: float, k_steps: int, sensor: float = 0.2):
    """Density L1 after k_steps coarse steps against the averaged fine solution."""
    import torch
    from .device import Context

    truth, fine_s = run_fine(seeds, dt_c, k_steps)
    res = {"plain64": [], "learned64": [], "plain128": []}
    secs = {"plain64": 0.0, "learned64": 0.0, "plain128": 0.0, "plain256": fine_s / len(seeds)}
    faces = fallbacks = 0
    g64, p64 = grid_params(64, dt_c)
    g128, p128 = grid_params(128, dt_c / 2)
    for k, s in enumerate(seeds):
        fine = family_state(256, s)
        ref = truth[k, -1, 0]
        for name, grid, params, f, corr in (("plain64", g64, p64, 4, False), ("learned64", g64, p64, 4, True),
                                            ("plain128", g128, p128, 2, False)):
            c = Context(grid, params)
            c.upload(coarsen(fine, f))
            if corr:
                c.set_flux_correction(net, sensor)
            c.step(1)  # warm-up of the graph
            c.upload(coarsen(fine, f))
            c.set_solver_state(abi.EfvmSolverState())
            steps = k_steps * (4 // f)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            c.step(steps)
            c.solver_state()
            secs[name] += (time.perf_counter() - t0) / len(seeds)
            u = c.download()
            rho = coarsen(u, 2)[..., 0] if f == 2 else u[..., 0]
            res[name].append(float(np.mean(np.abs(rho - ref))))
            if corr:
                a, b = c.correction_stats()
                faces += a
                fallbacks += b
            c.close()
    summary = {name: {"l1_mean": float(np.mean(v)), "l1_median": float(np.median(v))} for name, v in res.items()}
    summary["wins_over_plain64"] = float(np.mean(np.array(res["learned64"]) < np.array(res["plain64"])))
    summary["seconds_per_case"] = secs
    summary["fallback_rate"] = fallbacks / max(faces, 1)
    return summary, res


MODEL = __import__("os").path.join(__import__("os").path.dirname(__file__), "models", "flux_net_vortex64.npz")


def load_trained(path: str = MODEL):
    """The network trained by `main` (2000 trajectories, 40 epochs), and its coarse dt."""
    from .device import FluxNet

    d = np.load(path)
    net = FluxNet(out_scale=float(d["out_scale"]), gamma=GAMMA)
    net.set_params(d["params"])
    return net, float(d["dt_coarse"])


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=2000, help="training trajectories")
    ap.add_argument("--eval", type=int, default=200, help="held-out trajectories")
    ap.add_argument("--k-train", type=int, default=4, help="coarse steps per training trajectory")
    ap.add_argument("--k-eval", type=int, default=16, help="coarse steps of the evaluation runs")
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--out", default=None)
    ap.add_argument("--save", default=None, help="write the trained parameters (.npz)")
    args = ap.parse_args()
    train_seeds = list(range(1000, 1000 + args.train))
    eval_seeds = list(range(900000, 900000 + args.eval))
    dt_c = coarse_dt(train_seeds[:64] + eval_seeds[:64])
    t0 = time.perf_counter()
    states, resid, _ = make_dataset(train_seeds, dt_c, args.k_train)
    t_data = time.perf_counter() - t0
    print(f"data: {len(states)} pairs in {t_data:.1f} s (dt {dt_c:.4e})", flush=True)
    t0 = time.perf_counter()
    net, hist, meta = train(states, resid, dt_c, args.epochs)
    t_train = time.perf_counter() - t0
    summary, per_case = evaluate(net, eval_seeds, dt_c, args.k_eval)
    summary.update({"train_trajectories": args.train, "pairs": int(len(states)), "epochs": args.epochs,
                    "loss_history": hist, "data_seconds": t_data, "train_seconds": t_train, "dt_coarse": dt_c,
                    "k_eval": args.k_eval, **meta})
    print(json.dumps(summary), flush=True)
    if args.out:
        json.dump({"summary": summary, "per_case": per_case}, open(args.out, "w"), indent=1)
    if args.save:
        np.savez(args.save, params=net.params(), out_scale=net.out_scale(), dt_coarse=dt_c)


if __name__ == "__main__":
    main()

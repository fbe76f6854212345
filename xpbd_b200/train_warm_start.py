"""Train and evaluate the learned lambda warm start (3-DOF cloth) on the GPU.

    python -m xpbd_b200.train_warm_start --samples 10000000 --out model.pt
    python -m xpbd_b200.train_warm_start --eval model.pt

Data: randomized cloths (n x n, n ~ U{32..128}; spacing 0.02 m, 0.01 kg, two
pinned corners, FLOOR rows at y = 0; compliance log-uniform in [1e-10, 1e-4]),
each run for a random number of frames with the normal solver, then sampled
substep by substep: features at the substep start, target = the multiplier
after 50 plain Jacobi iterations (``learned.collect``).  Training: Adam on the
mean squared error, by the engine's own gradient and Adam kernels.

Evaluation (``evaluate``): a 128 x 128 cloth of the same family at compliance
1e-5 (where the plain Jacobi solve reaches the tolerance; at compliance <= 1e-6
it does not within any practical iteration count, from any start), after it
has been hanging for a while: per sampled substep, the Jacobi iterations the
plain solve (lambda0 = 0) and the warm-started solve need to bring the residual
(hard rows max(0, -C), compliant rows |C + alpha~ lambda|) below 1e-4 m, with
the per-substep fallback to plain when the learned first iteration is worse.
"""

from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from . import scenes
from .learned import WarmStartMLP, collect, iterations_to_tol
from .solver import Solver


def make_cloth(n, compliance, floor=True):
    s = Solver(dt=1 / 60, substeps=15, iterations=2, solve_mode="jacobi")
    scenes.build_cloth(s, res=n, spacing=0.02, mass=0.01, y=1.0, compliance=compliance, floor=floor)
    return s


def generate(n_samples, seed=0, substeps_per_cloth=8, log=print):
    rng = np.random.default_rng(seed)
    F, T = [], []
    total = 0
    t0 = time.time()
    while total < n_samples:
        n = int(rng.integers(32, 129))
        comp = float(10.0 ** rng.uniform(-10, -4))
        s = make_cloth(n, comp)
        for _ in range(int(rng.integers(0, 40))):
            s.step()
        f, t = collect(s, substeps=substeps_per_cloth, iters=50)
        F.append(f)
        T.append(t)
        total += len(t)
        log(f"  cloth {n}x{n} compliance {comp:.2e}: {len(t)} samples (total {total}, {time.time() - t0:.1f} s)")
    return torch.cat(F)[:n_samples], torch.cat(T)[:n_samples]


def train(F, T, epochs=4, batch=8192, lr=2e-3, seed=0, log=print):
    torch.manual_seed(seed)
    m = WarmStartMLP(seed=seed)
    n = len(T)
    for ep in range(epochs):
        perm = torch.randperm(n, device=F.device)
        acc = 0.0
        steps = 0
        for k in range(0, n, batch):
            sel = perm[k:k + batch]
            loss = m.train_step(F[sel], T[sel], lr=lr * (0.5 ** ep))
            if steps % 64 == 0:
                acc += float(loss.item())
            steps += 1
        log(f"  epoch {ep}: mean sampled loss {acc / max(1, (steps + 63) // 64):.5f}")
    return m


def evaluate(m, n=128, compliance=1e-5, frames=30, samples=8, tol=1e-4, max_iters=100):
    s = make_cloth(n, compliance)
    for _ in range(frames):
        s.step()
    rows = []
    for k in range(samples):
        rows.append(iterations_to_tol(s, m, tol=tol, max_iters=max_iters))
        s.step()
    plain = np.array([r["plain"] for r in rows])
    learned = np.array([r["learned_with_fallback"] for r in rows])
    return {"cloth": f"{n}x{n}", "compliance": compliance, "tol_m": tol, "max_iters": max_iters,
            "iters_plain": plain.tolist(), "iters_learned": learned.tolist(),
            "fallbacks": int(sum(r["fallback"] for r in rows)),
            "mean_plain": float(plain.mean()), "mean_learned": float(learned.mean()),
            "ratio": float(plain.mean() / max(learned.mean(), 1e-9))}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--samples", type=int, default=10_000_000)
    ap.add_argument("--epochs", type=int, default=4)
    ap.add_argument("--out", default=None)
    ap.add_argument("--eval", default=None, help="evaluate a saved model instead of training")
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args()
    if a.eval:
        m = WarmStartMLP()
        m.load_state_dict(torch.load(a.eval))
    else:
        t0 = time.time()
        F, T = generate(a.samples, seed=a.seed)
        print(f"generated {len(T)} samples in {time.time() - t0:.1f} s")
        t0 = time.time()
        m = train(F, T, epochs=a.epochs, seed=a.seed)
        print(f"trained in {time.time() - t0:.1f} s")
        if a.out:
            torch.save(m.state_dict(), a.out)
    print(json.dumps(evaluate(m)))


if __name__ == "__main__":
    main()

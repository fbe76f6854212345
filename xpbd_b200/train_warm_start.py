"""Train and evaluate the learned lambda warm start on the GPU.

    python -m xpbd_b200.train_warm_start --samples 10000000 --out weights.npy
    python -m xpbd_b200.train_warm_start --eval weights.npy
    python -m xpbd_b200.train_warm_start --time-infer [ROWS ...]
    python -m xpbd_b200.train_warm_start --time-grads [SAMPLES ...]

Data (half from each family, by sample count):
  * randomized cloths (n x n, n ~ U{32..128}; spacing 0.02 m, 0.01 kg, two
    pinned corners, FLOOR rows at y = 0; compliance log-uniform in
    [1e-10, 1e-4]), each run for a random number of frames, then sampled substep
    by substep: features at the substep start, target = the multiplier after 50
    plain Jacobi iterations (``learned.collect``);
  * randomized box piles (256..1440 boxes on a near-cubic 0.8 m lattice, half
    extents U[0.1, 0.3] m, random orientations, mu 0.6, e 0.2), run for a
    random number of frames, then sampled substep by substep in the same way on
    the floor-corner and manifold-point rows (``learned.collect6``).
In both, the previous substep's converged multiplier is feature 3.  Training:
Adam on the mean squared error, by the engine's own gradient and Adam kernels,
cosine learning-rate decay.

Evaluation (``evaluate_cloth``, ``evaluate_pile``): per sampled substep, the
Jacobi iterations the plain solve (lambda0 = 0) and the warm-started solve need
to bring the max residual (hard rows max(0, -C), compliant rows |C + alpha~
lambda|) below 1e-4 m, with the per-substep fallback to plain when the learned
first iteration is worse.  On the 128 x 128 cloth at compliance 1e-5 the plain
solve reaches 1e-4 m; on the settled 1440-box pile it does not within 50
iterations (averaged Jacobi through a 10-box-high stack converges slowly), so
the pile also reports the iterations each start needs to reach the plain
solve's own 50-iteration residual, and the residual after the configured two.
"""

from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np
import torch

from . import scenes
from .learned import SubstepKit6, WarmStartMLP, collect, collect6, iterations_to_tol, iterations_to_tol6
from .solver import Solver
from .solver_6dof import Solver6DOF

PILE_KW = dict(dt=1 / 60, substeps=15, iterations=2, floor_y=0.0, friction=0.6, restitution=0.2, broadphase="lbvh")


def make_cloth(n, compliance, floor=True):
    s = Solver(dt=1 / 60, substeps=15, iterations=2, solve_mode="jacobi")
    scenes.build_cloth(s, res=n, spacing=0.02, mass=0.01, y=1.0, compliance=compliance, floor=floor)
    return s


def make_pile(k, seed):
    """About k boxes on a near-cubic 0.8 m lattice (config-2 distributions)."""
    nx = max(2, int(round((k / 1.2) ** (1 / 3) * 1.1)))
    ny = max(1, k // (nx * nx))
    s = Solver6DOF(device="cuda:0", **PILE_KW)
    scenes.build_box_pile(s, nx=nx, ny=ny, nz=nx, seed=seed)
    return s


# Plain Jacobi iterations behind a training target (and behind the previous
# multiplier a substep carries into the next one's features, in training and
# in evaluation).
TARGET_ITERS = 50
# Which multiplier a substep carries into the next one's features: "target"
# (the TARGET_ITERS-iteration solve's) or "run" (the solver's own iterations',
# as step() carries it).
CARRY = "target"


def generate(n_samples, seed=0, scenes_per_family=200, substeps_per_cloth=8, pile_frames=1, log=print):
    """Alternates cloths and piles until `n_samples`; each scene contributes a
    random subset of at most n_samples / (2 scenes_per_family) of its rows, so
    the samples span many scenes (compliances, sizes, pile heights, times)."""
    rng = np.random.default_rng(seed)
    gen = torch.Generator(device="cuda").manual_seed(seed)
    per_scene = max(1, n_samples // (2 * scenes_per_family))
    F, T = [], []
    got = {"cloth": 0, "pile": 0}
    t0 = time.time()
    while got["cloth"] + got["pile"] < n_samples:
        if got["cloth"] <= got["pile"]:
            n = int(rng.integers(32, 129))
            comp = float(10.0 ** rng.uniform(-10, -4))
            s = make_cloth(n, comp)
            for _ in range(int(rng.integers(0, 40))):
                s.step()
            f, t = collect(s, substeps=substeps_per_cloth, iters=TARGET_ITERS, carry=CARRY)
            kind, what = "cloth", f"cloth {n}x{n} compliance {comp:.2e}"
        else:
            k = int(rng.integers(256, 1441))
            s = make_pile(k, int(rng.integers(1 << 30)))
            for _ in range(int(rng.integers(30, 300))):
                s.step()
            f, t = collect6(s, frames=pile_frames, iters=TARGET_ITERS, carry=CARRY)
            kind, what = "pile", f"pile {s.num_bodies} boxes"
        if len(t) > per_scene:
            sel = torch.randperm(len(t), device=t.device, generator=gen)[:per_scene]
            f, t = f[sel], t[sel]
        F.append(f)
        T.append(t)
        got[kind] += len(t)
        log(f"  {what}: {len(t)} samples (cloth {got['cloth']}, pile {got['pile']}, {time.time() - t0:.1f} s)")
    return torch.cat(F)[:n_samples], torch.cat(T)[:n_samples]


def train(F, T, epochs=40, batch=8192, lr=2e-3, seed=0, log=print):
    torch.manual_seed(seed)
    m = WarmStartMLP(seed=seed)
    n = len(T)
    for ep in range(epochs):
        perm = torch.randperm(n, device=F.device)
        rate = lr * 0.5 * (1.0 + math.cos(math.pi * ep / epochs))
        losses = []
        for k in range(0, n, batch):
            sel = perm[k:k + batch]
            losses.append(m.train_step(F[sel], T[sel], lr=rate))
        log(f"  epoch {ep}: mean loss {float(torch.stack(losses).mean()):.5f}")
    return m


def evaluate_cloth(m, n=128, compliance=1e-5, frames=30, substeps=16, tol=1e-4, max_iters=200):
    """A hanging n x n cloth after `frames` frames; the next `substeps` substeps
    one by one (the first has no previous converged multiplier and is left out
    of the means)."""
    s = make_cloth(n, compliance)
    for _ in range(frames):
        s.step()
    carry_iters = TARGET_ITERS if CARRY == "target" else s.iterations
    rows = [iterations_to_tol(s, m, tol=tol, max_iters=max_iters, advance=True, classic=True,
                              carry_iters=carry_iters) for _ in range(substeps)][1:]
    plain = np.array([r["plain"] for r in rows])
    learned = np.array([r["learned_with_fallback"] for r in rows])
    classic = np.array([r["classic"] for r in rows])
    pf_plain = np.array([r["to_plain_final"]["plain"] for r in rows])
    pf_fb = np.array([r["to_plain_final"]["plain"] if r["fallback"] else r["to_plain_final"]["learned"] for r in rows])
    return {"scene": f"cloth {n}x{n}", "compliance": compliance, "tol_m": tol, "max_iters": max_iters,
            "substeps": len(rows), "iters_plain": plain.tolist(), "iters_learned": learned.tolist(),
            "fallbacks": int(sum(r["fallback"] for r in rows)),
            "mean_plain": float(plain.mean()), "mean_learned": float(learned.mean()),
            "mean_classic": float(classic.mean()), "iters_classic": classic.tolist(),
            "ratio": float(plain.mean() / max(learned.mean(), 1e-9)),
            "residual_first_iter_mean": {k: float(np.mean([r["residual_first_iter"][k] for r in rows]))
                                         for k in ("plain", "learned", "classic")},
            "residual_second_iter_mean": {
                "plain": float(np.mean([r["residual_plain"][1] for r in rows])),
                "learned": float(np.mean([r["residual_learned"][1] for r in rows]))},
            "iters_to_plain_final": {"plain": float(pf_plain.mean()), "learned_with_fallback": float(pf_fb.mean())},
            "plain_final_residual_mean": float(np.mean([r["residual_plain"][-1] for r in rows]))}


def evaluate_pile(m, frames_before=240, frames=2, tol=1e-4, max_iters=None, seed=0):
    """The 1440-box pile (12 x 10 x 12, seed 0) after `frames_before` frames; the
    next `frames` frames substep by substep (the first substep of the run has no
    previous converged multiplier and is left out of the means)."""
    max_iters = TARGET_ITERS if max_iters is None else max_iters
    s = Solver6DOF(device="cuda:0", **PILE_KW)
    scenes.build_box_pile(s, seed=seed)
    for _ in range(frames_before):
        s.step()
    kit = SubstepKit6(s)
    prev = {"classic lambda_prev": (1.0, lambda k: torch.cat([k.prev_floor, k.prev_pair]))}
    rows = []
    for f in range(frames):
        kit.broadphase()
        for _ in range(s.substeps):
            rows.append(iterations_to_tol6(kit, m, tol=tol, max_iters=max_iters, variants=prev,
                                           carry_iters=None if CARRY == "target" else s.iterations))
    rows = rows[1:]
    pf_plain = np.array([r["to_plain_final"]["plain"] for r in rows])
    pf_learn = np.array([r["to_plain_final"]["learned"] for r in rows])
    fb = np.array([r["fallback"] for r in rows])
    pf_fb = np.where(fb, pf_plain, pf_learn)
    pf_prev = np.array([r["classic lambda_prev"]["to_plain_final"] for r in rows])
    res2 = {"plain": float(np.mean([r["residual_plain"][1] for r in rows])),
            "learned": float(np.mean([r["residual_learned"][1] for r in rows])),
            "classic lambda_prev": float(np.mean([r["classic lambda_prev"]["second"] for r in rows]))}
    return {"scene": f"box pile {s.num_bodies} after {frames_before} frames", "substeps": len(rows),
            "tol_m": tol, "max_iters": max_iters,
            "iters_to_tol": {"plain": float(np.mean([r["plain"] for r in rows])),
                             "learned_with_fallback": float(np.mean([r["learned_with_fallback"] for r in rows]))},
            "plain_final_residual_mean": float(np.mean([r["residual_plain"][-1] for r in rows])),
            "iters_to_plain_final": {"plain": float(pf_plain.mean()), "learned": float(pf_learn.mean()),
                                     "learned_with_fallback": float(pf_fb.mean()),
                                     "classic lambda_prev": float(pf_prev.mean())},
            "fallbacks": int(fb.sum()), "mean_residual_after_2_iters": res2,
            "ratio_with_fallback": float(pf_plain.mean() / max(pf_fb.mean(), 1e-9))}


def _event_ms(fn, reps=20):
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    fn()
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def time_inference(m, rows_list=(2400, 14897, 113410, 1 << 20), reps=50, seed=0):
    """Device time of one ``xpbd_mlp_infer`` launch (tensor-core inference) per
    row count, on random features (mean of `reps` launches, CUDA events)."""
    rng = np.random.default_rng(seed)
    out = {}
    for R in rows_list:
        feats = torch.from_numpy(rng.normal(size=(R, 8)).astype(np.float32)).cuda()
        weff = torch.from_numpy(rng.uniform(1.0, 10.0, R).astype(np.float32)).cuda()
        lam = torch.zeros(R, device="cuda")
        us = _event_ms(lambda: m.infer(feats, weff, R, lam), reps=reps) * 1e3
        if not bool(torch.isfinite(lam).all()):
            raise RuntimeError("non-finite inference output")
        out[str(R)] = {"us": round(us, 2), "rows_per_s": round(R / (us * 1e-6), 1)}
    return out


def time_gradient(m, batches=(65536, 1 << 20), reps=20, seed=0):
    """Device time of one ``xpbd_mlp_grads`` launch (tensor-core training
    kernel) per batch size, on random features and targets (mean of `reps`
    launches, CUDA events)."""
    from . import _native as N
    rng = np.random.default_rng(seed)
    out = {}
    for B in batches:
        feats = torch.from_numpy(rng.normal(size=(B, 8)).astype(np.float32)).cuda()
        targets = torch.from_numpy(rng.normal(size=B).astype(np.float32)).cuda()
        loss = torch.zeros(1, dtype=torch.float32, device="cuda")

        def run():
            N.check(m.F["grads"](N.ptr(feats), N.ptr(targets), B, N.ptr(m.wb), N.ptr(m.G), N.ptr(loss),
                                 N.stream_of("cuda:0")), "xpbd_mlp_grads")
        us = _event_ms(run, reps=reps) * 1e3
        if not bool(torch.isfinite(m.G).all()):
            raise RuntimeError("non-finite gradient")
        m.G.zero_()
        out[str(B)] = {"us": round(us, 1), "samples_per_s": round(B / (us * 1e-6), 1)}
    return out


def time_warm_start(m):
    """Device time of the warm start's extra work per substep (features +
    inference + warm apply) against one plain Jacobi iteration (solve + apply),
    on the 1440-box pile after 240 frames and on the 128 x 128 cloth; each is
    repeated from the same state."""
    from .learned import SubstepKit
    out = {}
    s = Solver6DOF(device="cuda:0", **PILE_KW)
    scenes.build_box_pile(s)
    for _ in range(240):
        s.step()
    kit = SubstepKit6(s)
    kit.broadphase()
    kit.begin()
    snap = kit.snapshot()
    rows = int((kit.weff > 0).sum().item())

    def warm6():
        kit.restore(snap)
        N6 = kit.L
        from . import _native as N
        N.check(N6.xpbd6_features(kit.st, kit.par, N.ptr(kit.prev_floor), N.ptr(kit.prev_pair), N.ptr(kit.feats),
                                  N.ptr(kit.weff), kit.stream()))
        kit.warm(m)

    def iter6():
        kit.restore(snap)
        kit.iterate()
    out["pile"] = {"rows": rows, "warm_start_ms": round(_event_ms(warm6), 4),
                   "iteration_ms": round(_event_ms(iter6), 4)}
    c = make_cloth(128, 1e-5)
    for _ in range(30):
        c.step()
    ck = SubstepKit(c)
    snap3 = c.state_dict()
    ck.integrate()

    def warm3():
        ck.features()
        ck.warm(m)

    def iter3():
        ck.iterate(first=False)
    rows3 = int(c.tensors["n_rows"].item())
    out["cloth"] = {"rows": rows3, "warm_start_ms": round(_event_ms(warm3), 4),
                    "iteration_ms": round(_event_ms(iter3), 4)}
    c.load_state_dict(snap3)
    return out


def product_frames(m, frames=20):
    """Frames through the public ``step()`` with each ``warm_start`` setting on
    the 128 x 128 cloth (compliance 1e-5, Jacobi) and the 1440-box pile (after
    240 frames): ms per frame, M proj/s (rows x substeps x iterations; the
    warm start's extra first iteration is overhead, not counted) and the mean
    max residual after the frames."""
    out = {}
    for name in ("cloth", "pile"):
        for label, ws in (("plain", None), ("previous", "previous"), ("learned", m)):
            if name == "cloth":
                s = Solver(dt=1 / 60, substeps=15, iterations=2, solve_mode="jacobi", warm_start=ws)
                scenes.build_cloth(s, res=128, compliance=1e-5)
                pre = 30
            else:
                s = Solver6DOF(device="cuda:0", warm_start=ws, **PILE_KW)
                scenes.build_box_pile(s)
                s.sync_pairs = False
                pre = 240
            for _ in range(pre):
                s.step()
            torch.cuda.synchronize()
            if name == "pile":
                s.manifold_points(reset=True)
                n_dyn = int((s.tensors["x"][:, 3] > 0).sum().item())
            res = []
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ms = 0.0
            for _ in range(frames):
                e0.record()
                s.step()
                e1.record()
                torch.cuda.synchronize()
                ms += e0.elapsed_time(e1)
                res.append(float(np.max(s.residual())))
            if name == "cloth":
                proj = frames * s.num_constraints * s.substeps * s.iterations
            else:
                pts = s._runner.kit.points_total if ws is not None else s.manifold_points()
                proj = s.iterations * (frames * s.substeps * (8 * n_dyn) + pts)
            used = int(s._runner.learned_used.item()) if ws is not None else 0
            out[f"{name}/{label}"] = {"ms_per_frame": round(ms / frames, 4),
                                      "M_proj_per_s": round(proj / (ms / 1e3) / 1e6, 2),
                                      "mean_max_residual": float(np.mean(res)),
                                      "warm_substeps_kept": used}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--samples", type=int, default=10_000_000)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--out", default=None, help="save the trained weights (float32 .npy)")
    ap.add_argument("--eval", default=None, help="evaluate saved weights instead of training")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--target-iters", type=int, default=50,
                    help="plain Jacobi iterations behind a target and behind the carried previous multiplier")
    ap.add_argument("--carry", choices=["target", "run"], default="target",
                    help="the multiplier a substep carries into the next one's features: the target solve's, "
                         "or the solver's own iterations' (as step())")
    ap.add_argument("--time-infer", type=int, nargs="*", default=None, metavar="ROWS",
                    help="only time the inference launch at these row counts (shipped weights)")
    ap.add_argument("--time-grads", type=int, nargs="*", default=None, metavar="SAMPLES",
                    help="only time the gradient launch at these batch sizes (shipped weights)")
    a = ap.parse_args()
    global TARGET_ITERS, CARRY
    TARGET_ITERS = a.target_iters
    CARRY = a.carry
    report = {"target_iters": TARGET_ITERS, "carry": CARRY}
    if a.time_infer is not None:
        m = WarmStartMLP.pretrained()
        print(json.dumps(time_inference(m, tuple(a.time_infer) or (2400, 14897, 113410, 1 << 20))))
        return
    if a.time_grads is not None:
        m = WarmStartMLP.pretrained()
        print(json.dumps(time_gradient(m, tuple(a.time_grads) or (65536, 1 << 20))))
        return
    if a.eval:
        m = WarmStartMLP()
        m.load_weights(a.eval)
    else:
        t0 = time.time()
        F, T = generate(a.samples, seed=a.seed)
        report["samples"] = len(T)
        report["generate_s"] = round(time.time() - t0, 1)
        t0 = time.time()
        m = train(F, T, epochs=a.epochs, seed=a.seed)
        torch.cuda.synchronize()
        report["train_s"] = round(time.time() - t0, 1)
        report["epochs"] = a.epochs
        if a.out:
            m.save_weights(a.out)
    report["cloth"] = evaluate_cloth(m)
    report["cloth_c1e-4"] = evaluate_cloth(m, compliance=1e-4)
    report["pile"] = evaluate_pile(m)
    report["timing"] = time_warm_start(m)
    report["frames"] = product_frames(m)
    print(json.dumps(report))


if __name__ == "__main__":
    main()

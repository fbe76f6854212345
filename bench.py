#!/usr/bin/env python
"""Benchmark of the XPBD substep engine on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload boxes|spheres|cloth|cloth_jacobi|batch]
    python bench.py --impl reference ...      # the CPU restatement of the reference, timed on the host

A step is one frame (dt = 1/60 s, 15 substeps x 2 iterations) of the workload.
Default workload: the 1440-box pile (12 x 10 x 12 lattice, pitch 0.8 m, half
extents U[0.1, 0.3] m, random orientations, mu = 0.6, e = 0.2, LBVH broad phase),
timed after 60 settling frames.  The metric is constraint projections per second
(rows x substeps x iterations, the reference's benchmark definition,
examples/benchmark.py:126; for 6-DOF rows = 8 floor slots per dynamic body +
manifold points + joints per substep, the points counted on the device every
substep) and ms/frame.  Multi-GPU runs are independent replicas of one scene (no
data exchange), except the batch, whose scenes are split across the ranks by LPT
bin packing: value = sum over ranks of projections / max over ranks of time.

Timing: W untimed frames, then K frames each bracketed by CUDA events on the
solver's stream, with the 126 MB L2 flushed (256 MB memset) between frames
outside the events; barrier + synchronize on both sides; max over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "boxes": "box pile 1440 (12x10x12 lattice pitch 0.8 m, half extents U[0.1,0.3] m, density 1000, random "
             "orientation, mu=0.6, e=0.2), LBVH, 15x2",
    "spheres": "sphere pile 2048 (16x8x16, r=0.05 m, jitter 0.01, floor + self collision mu=0.5), jacobi 15x2",
    "cloth": "cloth 32x32 (spacing 0.02 m, 0.01 kg, 2 pinned corners, 5826 DISTANCE alpha=1e-8 + 1024 FLOOR mu=0.3), gs 15x2",
    "cloth_jacobi": "cloth 32x32 as above, jacobi 15x2",
    "batch": "256 independent scenes from seed 0: 128 cloths n x n (n ~ U{16..128}, gs, per-scene coloring) + "
             "128 box piles of k boxes (k ~ U{64..1024}, LBVH), packed into one 3-DOF and one 6-DOF system, 15x2",
}
SIX_DOF = {"boxes"}
# Frames run before the warm-up (untimed, every leg): the 1440-box pile falls
# for about 80 frames before it has collapsed; the timed frames (and the
# driver autotuning) then see the contact-rich pile rather than boxes in the air.
SETTLE = {"boxes": 60}
BYTES_PER_PROJ = {0: 88, 1: 88, 2: 64, 3: 112}   # DISTANCE, ATTACH, FLOOR, CONTACT (Jacobi)
BYTES_PER_PROJ_GS = {0: 84, 1: 84, 2: 64, 3: 112}
APPLY_BYTES = 60          # per body per iteration (Jacobi averaged apply)
BODY_SUBSTEP_BYTES = 128  # per body per substep (integrate + finalize + clamp)
# 6-DOF per unit: manifold point projection, floor corner, joint, manifold
# generation per pair per substep, body per substep
POINT_BYTES, CORNER_BYTES, JOINT_BYTES, PAIR_GEN_BYTES, BODY6_BYTES = 196, 47, 196, 300, 128


def make_solver(workload, device, solver_cls):
    from xpbd_b200 import scenes
    if workload == "spheres":
        s = solver_cls(dt=1 / 60, substeps=15, iterations=2, solve_mode="jacobi", device=device)
        scenes.build_sphere_pile(s)
    elif workload == "boxes":
        s = solver_cls(dt=1 / 60, substeps=15, iterations=2, floor_y=0.0, friction=0.6, restitution=0.2,
                       broadphase="lbvh", device=device)
        scenes.build_box_pile(s)
    elif workload in ("cloth", "cloth_jacobi"):
        mode = "gs" if workload == "cloth" else "jacobi"
        s = solver_cls(dt=1 / 60, substeps=15, iterations=2, solve_mode=mode, device=device)
        scenes.build_cloth(s)
    else:
        raise SystemExit(f"unknown workload {workload}")
    return s


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_for(workload):
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            return json.load(f).get(workload)
    except Exception:
        return None


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.f = None

    def __enter__(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.f.seek(0)
        rows = [r.split(", ") for r in self.f.read().strip().splitlines() if r.strip()]
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            if len(r) >= 9:
                for k, nm in enumerate(names):
                    if r[5 + k].strip() == "Active":
                        reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def algorithmic_bytes(solver, rows_type_counts, gs):
    S, I, n = solver.substeps, solver.iterations, solver.num_bodies
    table = BYTES_PER_PROJ_GS if gs else BYTES_PER_PROJ
    b = S * I * sum(table[t] * c for t, c in rows_type_counts.items())
    if not gs:
        b += S * I * n * APPLY_BYTES
    b += S * n * BODY_SUBSTEP_BYTES
    return b


def algorithmic_bytes6(S, I, n, n_dyn, n_joints, points_per_substep, pairs):
    """Bytes of one frame of the 6-DOF substep kernel by the per-unit model."""
    return int(S * (I * (points_per_substep * POINT_BYTES + 8 * n_dyn * CORNER_BYTES + n_joints * JOINT_BYTES)
                    + pairs * PAIR_GEN_BYTES + n * BODY6_BYTES))


def sort_launches(n, bits):
    """Kernel launches of prims.cu sort_pairs_u64: one CTA up to 16384 keys;
    above, per 8-bit pass a histogram, a 3-kernel scan and a scatter, plus a copy
    back after an odd number of passes."""
    if n <= 16384:
        return 1
    passes = (bits + 7) // 8
    return 5 * passes + passes % 2


def lbvh_sort_launches(n, n_scenes):
    """The LBVH key sort: 30 Morton bits plus the bits of the largest scene id."""
    bits, ns = 30, n_scenes - 1
    while ns > 0:
        bits += 1
        ns >>= 1
    return sort_launches(n, bits)


def batch_launches_per_frame(b):
    """One frame kernel for the cloths; for the piles the multi-kernel LBVH chain
    (init, AABB, Morton, sort, build, refit, count, 3-kernel scan, write) and one
    substep kernel."""
    n = 0
    if getattr(b, "has_cloth", True):
        n += 1
    if getattr(b, "has_piles", True):
        n += 10 + lbvh_sort_launches(b.piles.num_bodies, b.piles.n_scenes) + 1
    return n


def phase_floor_us(launch, device, rounds=2000, repeats=3):
    """Measured latency floor of one phase on the driver of `launch` (mode,
    blocks, threads): xpbd_phase_floor's dependent L2 load + vector reduction +
    barrier, median of `repeats` runs of `rounds` phases."""
    import ctypes as C

    from xpbd_b200 import _native as N
    mode = {"grid": 0, "shared": 1, "cluster": 2}[launch["mode"]]
    vals = []
    for _ in range(repeats):
        ns = C.c_float(0.0)
        N.check(N.lib().xpbd_phase_floor(mode, int(launch["blocks"]), int(launch["threads"]), rounds,
                                         C.byref(ns), N.stream_of(device)), "xpbd_phase_floor")
        vals.append(ns.value / 1e3)
    return statistics.median(vals)


def latency_model(kernel, kern_ms, barriers, phases, launch, device):
    """Frame kernel time against the phase latency floor: a frame of a scene
    this small is a chain of `phases` dependent phases, each at least one
    barrier plus one dependent L2 round trip."""
    floor = phase_floor_us(launch, device)
    us = kern_ms * 1e3 / max(phases, 1)
    return {"kernel": kernel, "barriers_per_frame": barriers, "phases_per_frame": phases,
            "us_per_phase": round(us, 4), "floor_us_per_phase": round(floor, 4), "frac": round(floor / us, 4),
            "floor_probe": f"{launch['mode']} {launch['blocks']}x{launch['threads']}: one dependent L2 load + "
                           "one vector reduction + the barrier per phase (xpbd_phase_floor)"}


def time_batch(args, device, flush_buf, clocks=None, rank=0, world=1, n_scenes=256, sample=(0, 1, 2, 3)):
    """Aggregate projections/s of the batched scenes (this rank's share when the
    batch is sharded), plus per-scene residual against the same scenes solved
    alone (a sample of this rank's scenes)."""
    import numpy as np
    import torch

    from xpbd_b200.batch import BatchedScenes, batch_specs, rank_scene_ids
    from xpbd_b200.shard import gather_scene_metrics
    specs = batch_specs(n_scenes, seed=0)
    ids = rank_scene_ids(specs, rank, world)
    t0 = time.perf_counter()
    b = BatchedScenes(specs, device=device, scene_ids=ids)
    build_s = time.perf_counter() - t0
    for _ in range(args.warmup):
        b.step()
    # batched against solo: the sampled scenes after the warm-up frames, before
    # the piles' float-atomic order separates two runs of the same pile (a
    # falling pile is chaotic; after ~100 frames two runs differ by metres)
    res_w = b.residuals()
    snap = {i: b.scene_positions(i) for i in sample if i in b.scene_ids}
    tune = b.autotune(frames=2)  # on the warmed-up state (contacts present), restored afterwards
    torch.cuda.synchronize(device)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    stream = torch.cuda.current_stream(device)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    b.reset_projection_count()
    ctx = clocks if clocks is not None else _Null()
    with ctx:
        for k in range(args.steps):
            if flush_buf is not None:
                flush_buf.zero_()
            ev[k][0].record(stream)
            b.step()
            ev[k][1].record(stream)
        torch.cuda.synchronize(device)
    frame_ms = [a.elapsed_time(c) for a, c in ev]
    proj_total = b.projections(args.steps)
    points_total = b.piles.manifold_points() if b.has_piles else 0
    # per-kernel time on further frames (each system alone, L2 flushed), for the roofline
    S, I = b.cloth.substeps, b.cloth.iterations
    kern = {}
    for name, sys_, on in (("cloth", b.cloth, b.has_cloth), ("piles", b.piles, b.has_piles)):
        if not on:
            continue
        kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(5)]
        for e1, e2 in kev:
            if flush_buf is not None:
                flush_buf.zero_()
            e1.record(stream)
            sys_.step()
            e2.record(stream)
        torch.cuda.synchronize(device)
        kern[name] = statistics.mean(a.elapsed_time(c) for a, c in kev)
    res = b.residuals()  # every scene after all frames
    checks = {}
    for i, x_batched in snap.items():
        s = b.solo(i)
        for _ in range(args.warmup):
            s.step()
        torch.cuda.synchronize(device)
        d = float(np.abs(x_batched - s.positions()).max())
        checks[str(i)] = {"kind": b.specs[i].kind, "size": b.specs[i].size, "frames": args.warmup,
                          "residual_batched": float(res_w[i]), "residual_solo": float(s.residual()[0]),
                          "max_abs_dx_vs_solo": d}
    rows3 = b.cloth.num_constraints if b.has_cloth else 0
    n3 = b.cloth.num_bodies if b.has_cloth else 0
    alg3 = S * I * rows3 * BYTES_PER_PROJ_GS[0] + S * n3 * BODY_SUBSTEP_BYTES
    npairs, n6, alg6 = 0, 0, 0
    if b.has_piles:
        T = b.piles.tensors
        npairs = min(b.piles.n_pairs, b.piles.cap)
        n6 = b.piles.num_bodies
        n_dyn6 = int((T["x"][:, 3] > 0).sum().item())
        alg6 = algorithmic_bytes6(S, I, n6, n_dyn6, b.piles.num_joints, points_total / (args.steps * S), npairs)
    # every scene's residual, whichever rank stepped it
    held = [i for i in b.scene_ids]
    all_res = gather_scene_metrics(held, [float(res[i]) for i in held], len(specs))
    hbm, _ = peaks()
    rl = {}
    for name, alg in (("cloth", alg3), ("piles", alg6)):
        if name in kern:
            ach = alg / (kern[name] / 1e3) / 1e9
            rl[name] = {"kernel": "k3_frames (gs, grid)" if name == "cloth" else "LBVH chain + k6_substeps",
                        "alg_bytes_per_frame": int(alg), "ms": round(kern[name], 5), "achieved_gbs": round(ach, 1),
                        "frac": round(ach / hbm, 4), "traffic": traffic_for(f"batch_{name}")}
    return dict(total_ms=sum(frame_ms), frame_ms=frame_ms, kern_ms=frame_ms, proj_total=proj_total,
                rows=rows3, bodies=n3 + n6, status=(b.piles.status() if b.has_piles else 0) |
                (b.cloth.status() if b.has_cloth else 0), alg_bytes=alg3 + alg6,
                launches=args.steps * batch_launches_per_frame(b), kernel="k3_frames (gs) + k6_substeps (whole frame)",
                roofline_parts=rl,
                launch={"cloth": b.cloth.launch_info() if b.has_cloth else None,
                        "piles": b.piles.launch_info() if b.has_piles else None, "autotune": tune,
                        "scenes_this_rank": len(b.scene_ids), "scenes_total": len(specs),
                        "build_s": round(build_s, 1), "residual_max": float(np.nanmax(all_res)),
                        "residual_median": float(np.nanmedian(all_res)),
                        "scenes_with_residual": int(np.isfinite(all_res).sum()), "vs_solo": checks,
                        "cloth_particles": n3, "cloth_rows": rows3, "boxes": n6, "pairs": npairs,
                        "manifold_points_per_substep": round(points_total / max(args.steps * S, 1), 1)})


def time_engine(args, workload, device, rank, world, flush_buf, clocks=None):
    if workload == "batch":
        return time_batch(args, device, flush_buf, clocks, rank, world)
    if workload in SIX_DOF:
        return time_engine6(args, workload, device, world, flush_buf, clocks)
    import ctypes as C

    import numpy as np
    import torch

    from xpbd_b200 import Solver
    from xpbd_b200 import _native as N

    s = make_solver(workload, device, Solver)
    s.sync_contacts = False  # contact-capacity overflow is checked once after the run
    gs = s.solve_mode == "gs"
    L = N.lib()
    stream = torch.cuda.current_stream(device)
    sp = C.c_void_p(stream.cuda_stream)
    # frame kernel + contact build: one fused cluster launch up to 4096 collidable
    # spheres, else init, sanitize, cells, keys, sort (63-bit cell keys), count,
    # scan (3), write
    n_coll = int(s.tensors["collide_idx"].numel()) if s._self_collision else 0
    contact_launches = 1 if n_coll <= 4096 else 9 + sort_launches(n_coll, 63)
    launches_per_frame = 1 + (contact_launches if s._self_collision else 0)

    s._flush()
    for _ in range(args.warmup):
        s.step()
    tune = pin_or_tune(s, args)
    s.step()  # (self collision) attaches the contact rebuild and captures the frame on the tuned launch
    torch.cuda.synchronize(device)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    T = s.tensors
    n_rows_dev = torch.zeros(args.steps, dtype=torch.int32, device=device)
    # a frame: one xpbd3_step; with self collision it replays the captured
    # graph of contact rebuild + frame kernel
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    ctx = clocks if clocks is not None else _Null()
    with ctx:
        for k in range(args.steps):
            if flush_buf is not None:
                flush_buf.zero_()
            e0, e2 = ev[k]
            e0.record(stream)
            N.check(L.xpbd3_step(s._h, 1, sp), "xpbd3_step")
            e2.record(stream)
            n_rows_dev[k:k + 1].copy_(T["n_rows"])  # this frame's live rows (outside the events)
        torch.cuda.synchronize(device)
    frame_ms = [a.elapsed_time(c) for a, c in ev]
    status = s.status()
    rows = s.rows()
    types, counts = np.unique(rows["type"], return_counts=True)
    type_counts = {int(t): int(c) for t, c in zip(types, counts)}
    m = int(len(rows["type"]))
    proj_total = int(n_rows_dev.sum().item()) * s.substeps * s.iterations
    total_ms = sum(frame_ms)
    kern_ms = frame_ms
    if s._self_collision:
        # the frame kernel alone (the roofline's kernel), the contacts rebuilt
        # outside its events, on further frames after the timed ones
        s._detach_contacts()
        kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(min(args.steps, 100))]
        for e1, e2 in kev:
            if flush_buf is not None:
                flush_buf.zero_()
            s._build_contacts(sp)
            e1.record(stream)
            N.check(L.xpbd3_step(s._h, 1, sp), "xpbd3_step")
            e2.record(stream)
        torch.cuda.synchronize(device)
        kern_ms = [a.elapsed_time(c) for a, c in kev]
    alg_bytes = algorithmic_bytes(s, type_counts, gs)
    launch = s.launch_info()
    barriers, phases = s.phases()
    res = dict(total_ms=total_ms, frame_ms=frame_ms, kern_ms=kern_ms, proj_total=proj_total,
               rows=m, bodies=s.num_bodies, status=status, alg_bytes=alg_bytes,
               launches=launches_per_frame * args.steps, solver=s, kernel="k3_frames",
               latency=latency_model("k3_frames", statistics.mean(kern_ms), barriers, phases, launch, device))
    res["launch"] = dict(launch, autotune=tune["ms_per_frame"])
    return res


def time_engine6(args, workload, device, world, flush_buf, clocks=None):
    """Box pile: per frame the device broad phase (LBVH build + pair emission)
    then one persistent launch of all substeps, replayed as one CUDA graph."""
    import torch

    from xpbd_b200 import Solver6DOF
    from xpbd_b200 import _native as N
    from xpbd_b200.solver_6dof import lib6

    s = make_solver(workload, device, Solver6DOF)
    s.sync_pairs = False
    s._flush()
    L = lib6()
    stream = torch.cuda.current_stream(device)
    sp = N.stream_of(device)
    for _ in range(SETTLE.get(workload, 0) + args.warmup):
        N.check(L.xpbd6_step(s._h, 1, sp))
    tune = pin_or_tune(s, args)
    # capture the frame graph on the chosen launch, and warm it: the first
    # replays after the tuner's launches run slower
    N.check(L.xpbd6_step(s._h, max(3, args.warmup), sp))
    torch.cuda.synchronize(device)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    # a frame: one xpbd6_step, the replay of the captured graph of broad phase +
    # substep kernel (what step() runs)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    ctx = clocks if clocks is not None else _Null()
    s.manifold_points(reset=True)
    with ctx:
        for k in range(args.steps):
            if flush_buf is not None:
                flush_buf.zero_()
            e0, e2 = ev[k]
            e0.record(stream)
            N.check(L.xpbd6_step(s._h, 1, sp))
            e2.record(stream)
        torch.cuda.synchronize(device)
    frame_ms = [a.elapsed_time(c) for a, c in ev]
    points_total = s.manifold_points()  # every substep of the timed frames
    n = s.num_bodies
    n_dyn = int((s.tensors["x"][:, 3] > 0).sum().item())
    npairs = min(s.n_pairs, s.cap)
    # the substep kernel alone (the roofline's kernel) and the broad phase, each
    # launched on its own, on further frames after the timed ones
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
            torch.cuda.Event(enable_timing=True)) for _ in range(min(args.steps, 100))]
    for e0, e1, e2 in kev:
        if flush_buf is not None:
            flush_buf.zero_()
        e0.record(stream)
        N.check(L.xpbd6_broadphase(s._h, sp))
        e1.record(stream)
        N.check(L.xpbd6_substeps(s._h, sp))
        e2.record(stream)
    torch.cuda.synchronize(device)
    bp_ms = [a.elapsed_time(b) for a, b, _ in kev]
    kern_ms = [b.elapsed_time(c) for _, b, c in kev]
    status = s.status()
    S, I = s.substeps, s.iterations
    proj_total = I * (args.steps * S * (8 * n_dyn + s.num_joints) + points_total)
    pts_sub = points_total / (args.steps * S)
    alg = algorithmic_bytes6(S, I, n, n_dyn, s.num_joints, pts_sub, npairs)
    kernel = "k6_substeps8" if s.lanes == 8 else "k6_substeps"
    launch = s.launch_info()
    barriers, phases = s.phases()
    return dict(total_ms=sum(frame_ms), frame_ms=frame_ms, kern_ms=kern_ms, proj_total=proj_total,
                rows=int(round(8 * n_dyn + pts_sub + s.num_joints)), bodies=n, status=status, alg_bytes=alg,
                launches=args.steps * 2, solver=s, kernel=kernel,
                latency=latency_model(kernel, statistics.mean(kern_ms), barriers, phases, launch, device),
                launch=dict(launch, pairs_last_frame=npairs, manifold_points_per_substep=round(pts_sub, 1),
                            broadphase_ms=round(statistics.mean(bp_ms), 5),
                            separate_launches_ms_per_frame=round(statistics.mean(bp_ms) + statistics.mean(kern_ms), 5),
                            autotune=tune["ms_per_frame"]))


def time_e2e(args, workload, device):
    """Same metric through the public API with host buffers.  Every frame: the
    state (3-DOF: x, v; 6-DOF: x, q, v, w -- the solver keeps them as the rows
    of one contiguous block, ``tensors["state"]``, so one copy each way) is
    uploaded from pinned host memory, ``step()`` runs, and the state (plus the
    live row count, 3-DOF) is read back into pinned host memory, which feeds
    the next frame; the stream is synchronised each frame.  The region is
    bracketed by CUDA events on the solver's stream."""
    import torch

    from xpbd_b200 import Solver, Solver6DOF
    six = workload in SIX_DOF
    s = make_solver(workload, device, Solver6DOF if six else Solver)
    if six:
        s.sync_pairs = False
    else:
        s.sync_contacts = False
    s._flush()
    T = s.tensors
    keys = ("state",)
    host = {k: T[k].cpu().pin_memory() for k in keys}
    rows_host = torch.zeros(args.steps, dtype=torch.int32).pin_memory()
    stream = torch.cuda.current_stream(device)

    def frame(k=None):
        for key in keys:
            T[key].copy_(host[key], non_blocking=True)
        s.step()
        for key in keys:
            host[key].copy_(T[key], non_blocking=True)
        if k is not None and not six:
            rows_host[k:k + 1].copy_(T["n_rows"], non_blocking=True)
        stream.synchronize()

    # the same frames as the device-timed leg (6-DOF: its warm-up, then the
    # frames that warm the graph after tuning)
    pre = SETTLE.get(workload, 0) + (args.warmup + max(3, args.warmup) if six else max(3, args.warmup))
    for _ in range(pre):
        frame()
    steps = args.steps
    if six:
        s.manifold_points(reset=True)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(steps):
        frame(k)
    e1.record(stream)
    torch.cuda.synchronize(device)
    ms = e0.elapsed_time(e1) / steps
    S, I = s.substeps, s.iterations
    if six:
        n_dyn = int((T["x"][:, 3] > 0).sum().item())
        proj = I * (steps * S * (8 * n_dyn + s.num_joints) + s.manifold_points())
    else:
        proj = int(rows_host.sum().item()) * S * I
    nbytes = sum(host[k].numel() * 4 for k in keys)
    return ms, proj, nbytes, nbytes + (0 if six else 4)


def frame_projections(s):
    """Projections of the oracle's last frame: rows x S x I (3-DOF, the
    reference's definition); I x (S x (8 floor slots per dynamic body + joints)
    + the manifold points of every substep) (6-DOF)."""
    if hasattr(s, "num_constraints"):
        return s.num_constraints * s.substeps * s.iterations
    n_dyn = int((s.inv_mass > 0).sum())
    return s.iterations * (s.substeps * (8 * n_dyn + s.num_joints) + s.frame_points)


def cpu_baseline(workload, seconds, threads=1):
    """The oracle (CPU restatement of the reference) on a bounded sample of the
    same workload: consecutive frames from the same initial state until
    `seconds` of host time have elapsed (at least one frame), its substep loop
    on `threads` host threads (OpenMP; the contact rebuild and row flush stay
    on the Python thread, as in the reference's own host code)."""
    from oracle import oracle as O
    six = workload in SIX_DOF
    s = make_solver(workload, "cpu", O.OracleSolver6DOF if six else O.OracleSolver)
    s.threads = threads
    for _ in range(1 + SETTLE.get(workload, 0)):  # outside the sample: array set-up + the settling frames
        s.step()
    t0 = time.perf_counter()
    frames = 0
    proj = 0
    while True:
        s.step()
        frames += 1
        proj += frame_projections(s)
        if time.perf_counter() - t0 >= seconds:
            break
    dt = time.perf_counter() - t0
    return proj / dt / 1e6, frames, dt


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


def pin_or_tune(s, args):
    """The frame driver for the timed loop: the autotuner on the warmed-up state
    (contacts present; the state is restored afterwards), or the launch given by
    --driver MODE,BLOCKS,THREADS[,LANES] (a profiler's timing would mislead the
    autotuner, so profiles pin the launch the plain run chose)."""
    if not args.driver:
        return s.autotune(frames=3)
    v = [int(t) for t in args.driver.split(",")]
    if len(v) == 4:
        s.lanes = v[3]
    s.set_driver(*v[:3])
    s._bind()
    return {"ms_per_frame": {}, "pinned": args.driver}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    t0 = time.perf_counter()
    from oracle import oracle as O
    six = args.workload in SIX_DOF
    if args.workload == "batch":
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no batched-scene path"}),
              flush=True)
        return
    s = make_solver(args.workload, "cpu", O.OracleSolver6DOF if six else O.OracleSolver)
    threads = O.host_threads()  # every host core (OMP_NUM_THREADS when set)
    s.threads = threads
    for _ in range(SETTLE.get(args.workload, 0) + args.warmup):
        s.step()
    times = []
    proj = 0
    for _ in range(args.steps):
        a = time.perf_counter()
        s.step()
        times.append(time.perf_counter() - a)
        proj += frame_projections(s)
    total = sum(times)
    value = proj / total / 1e6
    line = {
        "impl": "reference", "metric": "constraint projections per second", "value": round(value, 4),
        "unit": "M proj/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(total / args.steps * 1e3, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": WORKLOADS[args.workload], "frames_per_step": 1,
                   "settle_frames": SETTLE.get(args.workload, 0)},
        "cpu_baseline": {"value": round(value, 4), "unit": "M proj/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} consecutive frames after "
                                   f"{SETTLE.get(args.workload, 0) + args.warmup} untimed frames, substep loop "
                                   f"on {threads} OpenMP threads"},
        "e2e": {"value": round(value, 4), "unit": "M proj/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": round(time.perf_counter() - t0, 2),
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--workload", default="boxes", choices=sorted(WORKLOADS))
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-flush", action="store_true")
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--driver", default="",
                    help="pin the frame driver MODE,BLOCKS,THREADS[,LANES] instead of autotuning "
                         "(mode 0 grid, 1 shared, 2 cluster; LANES 1 or 8 for boxes)")
    ap.add_argument("--kernels-only", action="store_true",
                    help="only the device-timed loop (for profiler launch lists): no e2e, CPU baseline or extras")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        return run_reference(args)

    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = f"cuda:{local}"
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device(device))
    flush = None if args.no_flush else torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=device)
    clocks = Clocks(local)
    r = time_engine(args, args.workload, device, rank, world, flush, clocks)
    total_ms = r["total_ms"]
    proj_total = r["proj_total"]
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([total_ms], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        pj = torch.tensor([proj_total], dtype=torch.float64, device=device)
        dist.all_reduce(pj, op=dist.ReduceOp.SUM)
        proj_total = float(pj.item())
    ms_per_step = total_ms / args.steps
    value = proj_total / (total_ms / 1e3) / 1e6
    sharded = args.workload == "batch"
    if rank == 0:
        hbm, peak_kind = peaks()
        kern_ms = statistics.mean(r["kern_ms"])
        achieved = r["alg_bytes"] / (kern_ms / 1e3) / 1e9
        line = {
            "metric": "constraint projections per second", "value": round(value, 4), "unit": "M proj/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 5),
            "higher_is_better": True, "scaling": "strong" if (sharded and world > 1) else "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded numpy default_rng(0))",
            "config": {"workload": WORKLOADS[args.workload], "bodies": r["bodies"],
                       "rows_per_substep": r["rows"], "projections_timed": int(proj_total),
                       "frames_per_step": 1, "settle_frames": SETTLE.get(args.workload, 0),
                       "l2": "flushed between frames (256 MB memset outside the timed events)",
                       "parallelism": (f"batch sharded over {world} ranks (LPT)" if sharded and world > 1
                                       else f"replicas x{world}"), "launch": r["launch"]},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": hbm, "unit": "GB/s",
                         "frac": round(achieved / hbm, 5), "peak_kind": peak_kind,
                         "traffic": traffic_for(args.workload), "kernel": r["kernel"],
                         "kernel_ms": round(kern_ms, 5), "alg_bytes_per_launch": r["alg_bytes"]},
            "gpu_launches": r["launches"],
            "status_bits": r["status"],
        }
        if "latency" in r:
            line["latency"] = r["latency"]
        if "roofline_parts" in r:
            line["roofline"]["parts"] = r["roofline_parts"]
        line["clocks"] = clocks.summary()
        if args.kernels_only or args.workload == "batch":
            print(json.dumps(line), flush=True)
            if world > 1:
                import torch.distributed as dist
                dist.destroy_process_group()
            return
        try:
            e_ms, e_proj, h2d, d2h = time_e2e(args, args.workload, device)
            line["e2e"] = {"value": round(world * e_proj / args.steps / (e_ms / 1e3) / 1e6, 4), "unit": "M proj/s",
                           "ms_per_step": round(e_ms, 5), "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}
        except Exception as e:  # pragma: no cover - reported, never silent
            line["e2e"] = {"error": repr(e)}
        if world == 1:
            from oracle import oracle as O
            threads = O.host_threads()
            v, frames, secs = cpu_baseline(args.workload, args.cpu_seconds, threads)
            v1, frames1, secs1 = cpu_baseline(args.workload, args.cpu_seconds / 2, 1)
            line["cpu_baseline"] = {"value": round(v, 4), "unit": "M proj/s", "cores": threads, "kind": "port",
                                    "sample": f"{frames} consecutive frames of the same workload after "
                                              f"{SETTLE.get(args.workload, 0)} settling frames ({secs:.1f} s), "
                                              f"substep loop on {threads} OpenMP threads",
                                    "single_thread": {"value": round(v1, 4), "cores": 1,
                                                      "sample": f"{frames1} frames ({secs1:.1f} s)"}}
            if not args.no_extras:
                extras = {}
                for wl in WORKLOADS:
                    if wl == args.workload:
                        continue
                    a2 = argparse.Namespace(**vars(args))
                    a2.steps = min(args.steps, 50)
                    rr = time_engine(a2, wl, device, 0, 1, flush, None)
                    ms = rr["total_ms"] / a2.steps
                    km = statistics.mean(rr["kern_ms"])
                    ex = {"ms_per_frame": round(ms, 5),
                          "M_proj_per_s": round(rr["proj_total"] / (rr["total_ms"] / 1e3) / 1e6, 3),
                          "kernel_ms": round(km, 5), "launch": rr["launch"],
                          "roofline": {"kernel": rr["kernel"], "alg_bytes_per_launch": rr["alg_bytes"],
                                       "achieved_gbs": round(rr["alg_bytes"] / (km / 1e3) / 1e9, 2),
                                       "frac": round(rr["alg_bytes"] / (km / 1e3) / 1e9 / hbm, 5),
                                       "traffic": traffic_for(wl)}}
                    if "latency" in rr:
                        ex["latency"] = rr["latency"]
                    if "roofline_parts" in rr:
                        ex["roofline"]["parts"] = rr["roofline_parts"]
                    extras[wl] = ex
                line["other_workloads"] = extras
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

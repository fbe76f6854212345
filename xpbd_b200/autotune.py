"""Driver autotuner for the persistent frame / substep kernels.

For a bound scene it times each candidate launch configuration -- one CTA with
the state in shared memory, one thread-block cluster of 2-16 CTAs (hardware
cluster barrier), or a cooperative grid (bounded global barrier) -- on a copy
of the current state, restores the state, and keeps the fastest.  Results are
cached per scene shape, so a solver rebuilt with the same sizes reuses them.
"""

from __future__ import annotations

import ctypes as C

import torch

from . import _native as N

_CACHE: dict = {}


def _time(run, stream, frames):
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    run()  # warm-up (first launch of a configuration)
    e0.record(stream)
    for _ in range(frames):
        run()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / frames


def tune3(s, frames=3, candidates=None):
    s._flush()
    key = ("3dof", s.num_bodies, s._cap, s.solve_mode, s.substeps, s.iterations, s.num_colors)
    if key in _CACHE and candidates is None:
        s.set_driver(*_CACHE[key][0])
        return _CACHE[key][1]
    if candidates is None:
        candidates = [(1, 0, 0), (2, 16, 512), (2, 8, 512), (2, 4, 512), (2, 16, 256), (0, 0, 256)]
    stream = torch.cuda.current_stream(s.device)
    sp = C.c_void_p(stream.cuda_stream)
    if s._self_collision:
        s._build_contacts(sp)
    snap = s.state_dict()
    results = {}
    for cand in candidates:
        try:
            s.set_driver(*cand)
            info = s.launch_info()
            if cand[0] == 1 and info["mode"] != "shared":
                continue  # does not fit in shared memory
            tag = (info["mode"], info["blocks"], info["threads"])
            if tag in results:
                continue
            ms = _time(lambda: N.check(N.lib().xpbd3_step(s._h, 1, sp)), stream, frames)
            results[tag] = (ms, cand)
        finally:
            s.load_state_dict(snap)
    best_tag = min(results, key=lambda t: results[t][0])
    best = results[best_tag][1]
    s.set_driver(*best)
    report = {"chosen": {"mode": best_tag[0], "blocks": best_tag[1], "threads": best_tag[2]},
              "ms_per_frame": {f"{t[0]}x{t[1]}x{t[2]}": round(v[0], 5) for t, v in results.items()}}
    _CACHE[key] = (best, report)
    return report


def tune6(s, frames=3, candidates=None):
    from .solver_6dof import lib6
    s._flush()
    key = ("6dof", s.num_bodies, s.cap, s.num_joints, s.substeps, s.iterations, s.broadphase)
    if key in _CACHE and candidates is None:
        best = _CACHE[key][0]
        s.lanes = best[3] if len(best) > 3 else 8
        s.set_driver(*best[:3])
        s._bind()  # bind now: callers may drive the handle directly, without step()
        return _CACHE[key][1]
    if candidates is None:
        candidates = [(2, 16, 512, 8), (2, 16, 256, 8), (2, 8, 512, 8), (0, 0, 256, 8), (0, 0, 512, 8),
                      (2, 16, 512, 1), (2, 16, 256, 1), (0, 0, 256, 1)]
    stream = torch.cuda.current_stream(s.device)
    sp = C.c_void_p(stream.cuda_stream)
    L = lib6()
    if s._sig != s._signature():
        s._bind()
    N.check(L.xpbd6_broadphase(s._h, sp))
    snap = s.state_dict()
    results = {}
    for cand in candidates:
        try:
            lanes = cand[3] if len(cand) > 3 else 8
            s.lanes = lanes
            s.set_driver(*cand[:3])
            info = s.launch_info()
            tag = (info["mode"], info["blocks"], info["threads"], lanes)
            if tag in results:
                continue
            ms = _time(lambda: N.check(L.xpbd6_substeps(s._h, sp)), stream, frames)
            results[tag] = (ms, cand)
        finally:
            s.load_state_dict(snap)
    best_tag = min(results, key=lambda t: results[t][0])
    best = results[best_tag][1]
    s.lanes = best[3] if len(best) > 3 else 8
    s.set_driver(*best[:3])
    s._bind()  # bind now: callers may drive the handle directly, without step()
    report = {"chosen": {"mode": best_tag[0], "blocks": best_tag[1], "threads": best_tag[2], "lanes": best_tag[3]},
              "ms_per_frame": {f"{t[0]}x{t[1]}x{t[2]}x{t[3]}": round(v[0], 5) for t, v in results.items()}}
    _CACHE[key] = (best, report)
    return report

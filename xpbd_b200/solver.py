"""3-DOF XPBD particle solver on B200 -- drop-in for the reference ``Solver``
(src/xpbd3d/solver.py:57-508): same constructor arguments, scene-building calls,
``step()``, perturbations and read-back.

Host side: scene lists (as in the reference) are flushed to CUDA tensors in a
packed float4 layout; a C-ABI handle (libxpbd_b200.so) then runs each frame as
one persistent launch (``xpbd3_step``).  With self collision on, contacts are
regenerated on the device every frame (``xpbd3_contacts_build``) in the
reference's row order.  In Gauss-Seidel mode the rows must then be recolored
(Welsh-Powell, as the reference does on the host every frame): with
``sync_contacts = False`` a one-CTA device pass colors them inside the frame's
captured graph (contact rebuild + coloring + frame kernel); with
``sync_contacts = True`` they are colored on the host after one
device-to-host copy, with exact contact-capacity overflow handling.

Differences from the reference, all deliberate:
* ``device`` defaults to ``"cuda:0"``; a CPU device raises (the engine has no
  CPU path -- the CPU restatement lives in ``oracle/`` and is test-only);
* setters update the device tensors in place instead of re-allocating them.
"""

from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _native as N
from .scene import Body, ConstraintHandle, Shape, shape_radius

DISTANCE = 0
ATTACH = 1
FLOOR = 2
CONTACT = 3


@dataclass
class _Row:
    type: int
    body_a: int
    body_b: int = -1
    rest: float = 0.0
    compliance: float = 0.0
    anchor: tuple = (0.0, 0.0, 0.0)
    mu: float = 0.0


class Solver:
    def __init__(self, dt: float = 1.0 / 60.0, substeps: int = 10, iterations: int = 1,
                 gravity=(0.0, -9.81, 0.0), damping: float = 0.0, solve_mode: str = "auto",
                 jacobi_relax: float = 1.0, device: str = "cuda:0", max_speed: float = 40.0, warm_start=None):
        """As the reference's constructor, plus `warm_start` (no reference
        counterpart; the reference restarts every substep from lambda = 0):
        None (the reference's lambda0 = 0), ``"previous"`` (the classical warm
        start from the previous substep's multipliers) or a
        ``learned.WarmStartMLP`` (the learned lambda0).  A warm start drives
        Jacobi solves of fixed rows (no self collision); every substep it also
        runs the plain first iteration and keeps whichever first iteration
        leaves the smaller residual."""
        self.device = N.require_cuda(device)
        self.warm_start = warm_start
        self._runner = None
        self.dt = float(dt)
        self.substeps = int(substeps)
        self.iterations = int(iterations)
        self.gravity = tuple(float(g) for g in gravity)
        self.damping = float(damping)
        self.jacobi_relax = float(jacobi_relax)
        self.max_speed = float(max_speed)
        if solve_mode == "auto":
            solve_mode = "jacobi"
        assert solve_mode in ("gs", "jacobi")
        self.solve_mode = solve_mode
        self._x, self._v, self._mass, self._radius = [], [], [], []
        self._collide, self._friction = [], []
        self._rows: list[_Row] = []
        self._self_collision = False
        self._contact_margin = 0.0
        self._default_friction = 0.0
        self._dirty = True
        self._params_dirty = True
        self._h = None
        self._contacts = None
        self.num_colors = 0
        self.color_counts: dict[int, int] = {}
        self.contact_capacity_per_body = 16
        self.sync_contacts = True  # read the contact count each frame (exact overflow handling)
        self._n_contacts_host = 0
        self._t = {}
        self.driver = (-1, 0, 0)  # (mode, blocks, threads): -1 automatic; see set_driver
        # Row ranges colored independently (batched independent scenes): each
        # scene gets the colors it would get alone, so Gauss-Seidel per scene is
        # the same computation as solving that scene alone.
        self.color_groups: list[tuple[int, int]] | None = None

    # ---- scene building (solver.py:130-228) ---------------------------------------
    def add_particle(self, position, mass, velocity=(0.0, 0.0, 0.0), shape: Shape | None = None,
                     collide: bool = True, radius: float | None = None, friction: float | None = None) -> Body:
        idx = len(self._x)
        self._x.append(tuple(float(v) for v in position))
        self._v.append(tuple(float(v) for v in velocity))
        self._mass.append(float(mass))
        sh = shape or Shape()
        r = float(radius) if radius is not None else shape_radius(sh)
        self._radius.append(r)
        self._collide.append(bool(collide) and r > 0.0 and mass > 0.0)
        mu = float(friction) if friction is not None else self._default_friction
        self._friction.append(max(0.0, mu))
        self._dirty = True
        return Body(index=idx, shape=sh)

    def add_distance(self, body_a: Body, body_b: Body, rest: float | None = None,
                     compliance: float = 0.0) -> ConstraintHandle:
        if rest is None:
            rest = float(np.linalg.norm(np.asarray(self._x[body_a.index]) - np.asarray(self._x[body_b.index])))
        self._rows.append(_Row(DISTANCE, body_a.index, body_b.index, rest=float(rest), compliance=float(compliance)))
        self._dirty = True
        return ConstraintHandle(index=len(self._rows) - 1)

    def add_attach(self, body: Body, world_point, compliance: float = 0.0, rest: float = 0.0) -> ConstraintHandle:
        self._rows.append(_Row(ATTACH, body.index, -1, rest=float(rest), compliance=float(compliance),
                               anchor=tuple(float(p) for p in world_point)))
        self._dirty = True
        return ConstraintHandle(index=len(self._rows) - 1)

    def add_floor_contact(self, body: Body, floor_y: float = 0.0, friction: float | None = None) -> ConstraintHandle:
        mu = float(friction) if friction is not None else self._friction[body.index]
        self._rows.append(_Row(FLOOR, body.index, -1, anchor=(0.0, float(floor_y), 0.0), mu=max(0.0, mu)))
        self._dirty = True
        return ConstraintHandle(index=len(self._rows) - 1)

    def enable_self_collision(self, enabled: bool = True, margin: float = 0.0,
                              default_friction: float | None = None) -> None:
        self._self_collision = bool(enabled)
        self._contact_margin = float(margin)
        if default_friction is not None:
            self._default_friction = max(0.0, float(default_friction))
            for k in range(len(self._friction)):
                if self._friction[k] == 0.0:
                    self._friction[k] = self._default_friction
        self._dirty = True

    # ---- perturbations (solver.py:232-271), in place on the device ----------------
    def set_position(self, body: Body, p) -> None:
        self._flush()
        self._t["x"][body.index, :3] = torch.tensor(p, dtype=torch.float32, device=self.device)

    def set_velocity(self, body: Body, vel) -> None:
        self._flush()
        self._t["v"][body.index, :3] = torch.tensor(vel, dtype=torch.float32, device=self.device)

    def add_impulse(self, body: Body, dv) -> None:
        self._flush()
        self._t["v"][body.index, :3] += torch.tensor(dv, dtype=torch.float32, device=self.device)

    def set_all_compliance(self, value: float, only_distance: bool = True) -> None:
        self._flush()
        for r in self._rows:
            if (not only_distance) or r.type == DISTANCE:
                r.compliance = float(value)
        rt = self._t["row_i"][: len(self._rows), 0]
        sel = (rt == DISTANCE) if only_distance else torch.ones_like(rt, dtype=torch.bool)
        self._t["row_f"][: len(self._rows), 1][sel] = float(value)
        self.rows_changed()

    def set_all_friction(self, mu: float) -> None:
        self._flush()
        self._default_friction = float(mu)
        for k in range(len(self._friction)):
            self._friction[k] = float(mu)
        for r in self._rows:
            if r.type in (FLOOR, CONTACT):
                r.mu = float(mu)
        rt = self._t["row_i"][:, 0]
        self._t["row_f"][:, 2][(rt == FLOOR) | (rt == CONTACT)] = float(mu)
        if "friction" in self._t:
            self._t["friction"].fill_(float(mu))
        self.rows_changed()

    def rows_changed(self) -> None:
        """Row parameters were edited in place on the device (the setters above,
        or a caller writing ``tensors["row_f"]``): Gauss-Seidel frames pack the
        rows in color order again before their next launch."""
        self._flush()
        N.check(N.lib().xpbd3_rows_changed(self._h, N.stream_of(self.device)), "xpbd3_rows_changed")

    # ---- flush: host lists -> device tensors (solver.py:346-408) -------------------
    def _flush(self) -> None:
        if not self._dirty:
            return
        dev = self.device
        n = len(self._x)
        ms = len(self._rows)
        x = np.zeros((n, 4), np.float32)
        v = np.zeros((n, 4), np.float32)
        if n:
            x[:, :3] = np.asarray(self._x, np.float32).reshape(-1, 3)
            v[:, :3] = np.asarray(self._v, np.float32).reshape(-1, 3)
        mass = np.asarray(self._mass, np.float32) if n else np.zeros(0, np.float32)
        x[:, 3] = np.where(mass > 0.0, 1.0 / np.maximum(mass, 1e-20), 0.0).astype(np.float32)
        old = self._t
        if "x" in old and 0 < old["x"].shape[0] <= n:
            k = old["x"].shape[0]
            x[:k, :3] = old["x"][:, :3].cpu().numpy()
            v[:k, :3] = old["v"][:, :3].cpu().numpy()
        collide_idx = np.nonzero(np.asarray(self._collide, bool))[0].astype(np.int32) if n else np.zeros(0, np.int32)
        n_coll = len(collide_idx) if self._self_collision else 0
        cap_contacts = max(1024, self.contact_capacity_per_body * n_coll) if self._self_collision else 0
        cap = ms + cap_contacts
        row_i = np.zeros((max(cap, 1), 4), np.int32)
        row_f = np.zeros((max(cap, 1), 4), np.float32)
        row_a = np.zeros((max(cap, 1), 4), np.float32)
        if ms:
            R = self._rows
            ti = np.fromiter((v for r in R for v in (r.type, r.body_a, r.body_b)), np.int64, 3 * ms).reshape(ms, 3)
            tf = np.fromiter((v for r in R for v in (r.rest, r.compliance, r.mu)), np.float64, 3 * ms).reshape(ms, 3)
            an = np.fromiter((v for r in R for v in r.anchor), np.float64, 3 * ms).reshape(ms, 3)
            bad = (ti[:, 1] < 0) | (ti[:, 1] >= n) | (ti[:, 2] < -1) | (ti[:, 2] >= n) | (
                np.isin(ti[:, 0], (DISTANCE, CONTACT)) & (ti[:, 2] < 0))
            if bad.any():
                raise IndexError(f"constraint row {int(np.nonzero(bad)[0][0])} references a body outside [0, {n})")
            row_i[:ms, :3] = ti
            row_i[:ms, 3] = 1
            row_f[:ms, :3] = tf
            row_f[:ms, 3] = an[:, 1]
            row_a[:ms, :3] = an
        T = {}
        # x and v are the two rows of one contiguous block (`state`), so a caller
        # moving the state to or from the host needs one copy each way
        T["state"] = torch.from_numpy(np.stack([x, v])).to(dev)
        T["x"], T["v"] = T["state"].unbind(0)
        T["x_prev"] = torch.zeros((n, 4), dtype=torch.float32, device=dev)
        T["acc"] = torch.zeros((n, 4), dtype=torch.float32, device=dev)
        T["row_i"] = torch.from_numpy(row_i).to(dev)
        T["row_f"] = torch.from_numpy(row_f).to(dev)
        T["row_anchor"] = torch.from_numpy(row_a).to(dev)
        T["lam"] = torch.zeros(max(cap, 1), dtype=torch.float32, device=dev)
        T["n_rows"] = torch.tensor([ms], dtype=torch.int32, device=dev)
        T["status"] = torch.zeros(1, dtype=torch.int32, device=dev)
        self._n_static = ms
        self._cap = cap
        self._n_contacts_host = 0
        if self._self_collision:
            existing = sorted({(min(r.body_a, r.body_b) * n + max(r.body_a, r.body_b))
                               for r in self._rows if r.body_b >= 0})
            T["radius"] = torch.tensor(np.asarray(self._radius, np.float32), device=dev)
            T["friction"] = torch.tensor(np.asarray(self._friction, np.float32), device=dev)
            T["collide_idx"] = torch.from_numpy(collide_idx).to(dev)
            T["existing"] = torch.tensor(np.asarray(existing, np.int64), device=dev)
            xi = np.zeros((n, 4), np.float32)
            if n:
                xi[:, :3] = np.asarray(self._x, np.float32).reshape(-1, 3)
            T["x_init"] = torch.from_numpy(xi).to(dev)
            self._rmax = float(np.asarray(self._radius, np.float32)[collide_idx].max()) if len(collide_idx) else 0.0
            if self._contacts is not None:
                N.lib().xpbd3_contacts_destroy(self._contacts)
            h = C.c_void_p()
            N.check(N.lib().xpbd3_contacts_create(C.byref(h), n, len(collide_idx)), "xpbd3_contacts_create")
            self._contacts = h
        self._t = T
        if self.solve_mode == "gs":
            self._color(ms)
        else:
            T["color_order"] = torch.zeros(1, dtype=torch.int32, device=dev)
            T["color_starts"] = torch.zeros(2, dtype=torch.int32, device=dev)
            self.num_colors = 1 if ms else 0
            self.color_counts = {}
        self._bind()
        self._dirty = False

    def _color(self, m: int, contacts: np.ndarray | None = None) -> None:
        """Color rows [0, m) (+ optional contact endpoints) on the host (coloring.py:26-89)."""
        T = self._t
        a = np.array([r.body_a for r in self._rows], np.int32)
        b = np.array([r.body_b for r in self._rows], np.int32)
        if contacts is not None and len(contacts):
            a = np.concatenate([a, contacts[:, 0].astype(np.int32)])
            b = np.concatenate([b, contacts[:, 1].astype(np.int32)])
        m = len(a)
        color = np.zeros(max(m, 1), np.int32)
        k = 0
        groups = self.color_groups if (self.color_groups and contacts is None) else [(0, m)]
        for g0, g1 in groups:
            if g1 <= g0:
                continue
            ga = a[g0:g1]
            gb = b[g0:g1]
            lo = int(ga.min())
            hi = int(max(ga.max(), gb.max()))
            ga = np.ascontiguousarray(ga - lo, dtype=np.int32)  # scene-local body ids
            gb = np.ascontiguousarray(np.where(gb >= 0, gb - lo, -1), dtype=np.int32)
            gc = np.zeros(g1 - g0, np.int32)
            kg = N.lib().xpbd_color_constraints(hi - lo + 1, g1 - g0, ga.ctypes.data_as(C.c_void_p),
                                                gb.ctypes.data_as(C.c_void_p), gc.ctypes.data_as(C.c_void_p))
            if kg < 0:
                raise N.XpbdError("coloring failed (row references a body out of range)")
            color[g0:g1] = gc
            k = max(k, kg)
        order = np.zeros(max(m, 1), np.int32)
        starts = np.zeros(k + 1, np.int32)
        if m:
            N.lib().xpbd_color_ranges(m, color.ctypes.data_as(C.c_void_p), order.ctypes.data_as(C.c_void_p),
                                      starts.ctypes.data_as(C.c_void_p))
        T["color_order"] = torch.from_numpy(order).to(self.device)
        T["color_starts"] = torch.from_numpy(starts).to(self.device)
        self.num_colors = int(k)
        self.color_counts = {int(c): int(cnt) for c, cnt in zip(*np.unique(color[:m], return_counts=True))} if m else {}

    def _state(self) -> N.xpbd3_state:
        T = self._t
        s = N.xpbd3_state()
        s.n_bodies = len(self._x)
        s.row_capacity = self._cap
        s.n_rows_static = self._n_static
        for f in ("x", "v", "x_prev", "acc", "row_i", "row_f", "row_anchor", "lam", "n_rows",
                  "color_order", "color_starts"):
            setattr(s, f, N.ptr(T[f]))
        s.num_colors = self.num_colors if self.solve_mode == "gs" else 0
        return s

    def _params(self) -> N.xpbd3_params:
        p = N.xpbd3_params()
        p.dt = self.dt
        p.substeps = self.substeps
        p.iterations = self.iterations
        p.gravity[:] = self.gravity
        p.damping = self.damping
        p.jacobi_relax = self.jacobi_relax
        p.max_speed = self.max_speed if math.isfinite(self.max_speed) else float("inf")
        p.gs = 1 if self.solve_mode == "gs" else 0
        return p

    def set_driver(self, mode: int = -1, blocks: int = 0, threads: int = 0) -> None:
        """Frame driver: -1 automatic, 0 cooperative grid, 1 one CTA with the
        state in shared memory, 2 one thread-block cluster; 0 = automatic size."""
        self.driver = (int(mode), int(blocks), int(threads))
        if self._h is not None and not self._dirty:
            self._bind()

    def launch_info(self) -> dict:
        self._flush()
        b, t, sm = C.c_int(), C.c_int(), C.c_int()
        N.lib().xpbd3_launch_info(self._h, C.byref(b), C.byref(t), C.byref(sm))
        mode = "cluster" if b.value < 0 else ("shared" if sm.value > 0 else "grid")
        return {"mode": mode, "blocks": abs(b.value), "threads": t.value, "smem_bytes": sm.value}

    def phases(self) -> tuple:
        """(barriers, phases) of one frame of the bound frame kernel."""
        self._flush()
        b, ph = C.c_int(), C.c_int()
        N.check(N.lib().xpbd3_phases(self._h, C.byref(b), C.byref(ph)), "xpbd3_phases")
        return b.value, ph.value

    def autotune(self, frames: int = 3, candidates=None) -> dict:
        """Time the frame drivers on the current scene and keep the fastest."""
        from .autotune import tune3
        return tune3(self, frames, candidates)

    def _bind(self) -> None:
        self.binds = getattr(self, "binds", 0) + 1  # handle (re)binds (a bind drops the captured frame)
        self._hooked = False
        L = N.lib()
        if self._h is None:
            h = C.c_void_p()
            N.check(L.xpbd3_create(C.byref(h)), "xpbd3_create")
            self._h = h
        N.check(L.xpbd3_set_driver(self._h, *[int(v) for v in self.driver]), "xpbd3_set_driver")
        self._st = self._state()
        self._par = self._params()
        N.check(L.xpbd3_bind(self._h, C.byref(self._st), C.byref(self._par)), "xpbd3_bind")

    # ---- the step (solver.py:412-442) ----------------------------------------------
    def step(self) -> None:
        self._flush()
        if len(self._x) == 0:
            return
        L = N.lib()
        stream = N.stream_of(self.device)
        if self.warm_start is not None:
            if self._runner is None or self._runner.binds != self.binds:
                from .learned import WarmStartRunner
                self._runner = WarmStartRunner(self, self.warm_start)
            self._runner.step()
            return
        if self._self_collision:
            if not self.sync_contacts:
                # contact rebuild (+ the device coloring of the rows, Gauss-Seidel)
                # + frame kernel as one captured CUDA graph per bind
                if not self._hooked:
                    self._attach_contacts(stream)
                N.check(L.xpbd3_step(self._h, 1, stream), "xpbd3_step")
                return
            self._detach_contacts()
            self._build_contacts(stream)
        N.check(L.xpbd3_step(self._h, 1, stream), "xpbd3_step")

    def _attach_contacts(self, stream) -> None:
        """Hand the contact rebuild to the bound handle, so xpbd3_step runs it
        before every frame inside one captured graph.  One plain rebuild first
        (idempotent on the state) initialises the builder outside the capture."""
        T = self._t
        L = N.lib()
        args = (N.ptr(T["radius"]), N.ptr(T["friction"]), N.ptr(T["collide_idx"]), int(T["collide_idx"].numel()),
                N.ptr(T["existing"]), int(T["existing"].numel()), N.ptr(T["x_init"]),
                C.c_double(self._contact_margin), C.c_double(self.dt), C.c_double(self._rmax), N.ptr(T["status"]))
        N.check(L.xpbd3_contacts_build(self._contacts, C.byref(self._st), *args, stream), "xpbd3_contacts_build")
        N.check(L.xpbd3_attach_contacts(self._h, self._contacts, *args), "xpbd3_attach_contacts")
        self._hooked = True

    def _detach_contacts(self) -> None:
        """xpbd3_step runs the frame kernel alone again (contacts built by the caller)."""
        if self._hooked:
            N.check(N.lib().xpbd3_attach_contacts(self._h, None, None, None, None, 0, None, 0, None, 0.0, 0.0, 0.0,
                                                  None), "xpbd3_attach_contacts")
            self._hooked = False

    def step_frames(self, frames: int) -> None:
        """Advance `frames` frames in one launch (scenes without self collision)."""
        self._flush()
        if len(self._x) == 0 or frames <= 0:
            return
        if self._self_collision:
            for _ in range(frames):
                self.step()
            return
        N.check(N.lib().xpbd3_step(self._h, int(frames), N.stream_of(self.device)), "xpbd3_step")

    def _build_contacts(self, stream) -> None:
        T = self._t
        L = N.lib()
        n_coll = int(T["collide_idx"].numel())
        for _attempt in range(12):
            N.check(L.xpbd3_contacts_build(self._contacts, C.byref(self._st), N.ptr(T["radius"]),
                                           N.ptr(T["friction"]), N.ptr(T["collide_idx"]), n_coll,
                                           N.ptr(T["existing"]), int(T["existing"].numel()), N.ptr(T["x_init"]),
                                           C.c_double(self._contact_margin), C.c_double(self.dt),
                                           C.c_double(self._rmax), N.ptr(T["status"]), stream),
                    "xpbd3_contacts_build")
            if not self.sync_contacts and self.solve_mode != "gs":
                return
            st = int(T["status"].item())
            if st & N.XPBD_ERR_OVERFLOW:
                # grow the contact capacity and regenerate this frame's contacts
                T["status"].zero_()
                self.contact_capacity_per_body = max(1, self.contact_capacity_per_body) * 2
                self._dirty = True
                self._flush()
                T = self._t
                continue
            break
        self._n_contacts_host = int(T["n_rows"].item()) - self._n_static
        if self.solve_mode == "gs":
            k = self._n_contacts_host
            ab = T["row_i"][self._n_static:self._n_static + k, 1:3].cpu().numpy()
            self._color(self._n_static, ab)
            self._st = self._state()
            N.check(L.xpbd3_bind(self._h, C.byref(self._st), C.byref(self._par)), "xpbd3_bind")

    # ---- read-back (solver.py:487-508) ---------------------------------------------
    def positions(self) -> np.ndarray:
        if not self._t:
            return np.asarray(self._x, np.float32).reshape(-1, 3)
        return self._t["x"][:, :3].cpu().numpy()

    def velocities(self) -> np.ndarray:
        if not self._t:
            return np.asarray(self._v, np.float32).reshape(-1, 3)
        return self._t["v"][:, :3].cpu().numpy()

    def lambdas(self) -> np.ndarray:
        if not self._t:
            return np.zeros(len(self._rows), np.float32)
        m = int(self._t["n_rows"].item())
        return self._t["lam"][:m].cpu().numpy()

    def rows(self) -> dict:
        """Live constraint rows (static + generated contacts) as numpy arrays."""
        self._flush()
        m = int(self._t["n_rows"].item())
        ri = self._t["row_i"][:m].cpu().numpy()
        rf = self._t["row_f"][:m].cpu().numpy()
        return dict(type=ri[:, 0], a=ri[:, 1], b=ri[:, 2], rest=rf[:, 0], compliance=rf[:, 1], mu=rf[:, 2])

    def status(self) -> int:
        """Device status bits (XPBD_ERR_*) raised since the last call; clears them."""
        self._flush()
        out = C.c_int(0)
        N.check(N.lib().xpbd3_status(self._h, C.byref(out), N.stream_of(self.device)), "xpbd3_status")
        s = int(self._t["status"].item())
        self._t["status"].zero_()
        return int(out.value) | s

    def residual(self, row_scene=None, n_scenes: int = 1, per_row: bool = False):
        """Max constraint residual of the current state (hard rows max(0, -C),
        compliant rows |C + alpha~ lambda|), per scene when `row_scene` (a device
        int tensor, one scene id per row) is given."""
        self._flush()
        h = self.dt / self.substeps
        out = torch.zeros(max(int(n_scenes), 1), dtype=torch.float32, device=self.device)
        rows = torch.zeros(self._cap, dtype=torch.float32, device=self.device) if per_row else None
        N.check(N.lib().xpbd3_residual(C.byref(self._st), float(h), N.ptr(row_scene), int(n_scenes), N.ptr(out),
                                       N.ptr(rows), N.stream_of(self.device)), "xpbd3_residual")
        res = out.cpu().numpy()
        if per_row:
            return res, rows[: int(self._t["n_rows"].item())].cpu().numpy()
        return res

    def dlpack(self, name: str = "x"):
        """Zero-copy DLPack capsule of one device state tensor (``x``, ``v``, ...,
        see ``tensors``): headless consumers (a viewer, a renderer, another
        framework) read the live state without a host copy.  Float4 records:
        xyz plus the fourth lane of the layout."""
        self._flush()
        return torch.utils.dlpack.to_dlpack(self._t[name])

    def state_dict(self) -> dict:
        self._flush()
        return {k: self._t[k].clone() for k in ("x", "v", "x_prev", "lam", "n_rows")}

    def load_state_dict(self, sd: dict) -> None:
        self._flush()
        for k, v in sd.items():
            self._t[k].copy_(v)

    @property
    def tensors(self) -> dict:
        self._flush()
        return self._t

    @property
    def num_bodies(self) -> int:
        return len(self._x)

    @property
    def num_constraints(self) -> int:
        if self._self_collision and self._t:
            return int(self._t["n_rows"].item())
        return len(self._rows)

    def __del__(self):
        try:
            L = N.lib()
            if self._h is not None:
                L.xpbd3_destroy(self._h)
            if self._contacts is not None:
                L.xpbd3_contacts_destroy(self._contacts)
        except Exception:
            pass

"""6-DOF rigid-body XPBD solver on B200 -- drop-in for the reference
``Solver6DOF`` (src/xpbd3d/solver_6dof.py:79-559): rigid boxes, particles and
compliant joints with the reference's constructor arguments, scene-building
calls, ``step()`` and read-back.

Each frame is a broad phase (``lbvh`` -- the engine's own Morton/radix-sort/
Karras LBVH --, ``hashgrid`` or ``grid``, all on the device) followed by one
persistent launch that runs every substep (``xpbd6_substeps``).

Like the reference (solver_6dof.py:443-453), the default ``step()`` reads the
live pair count once per frame and, if it exceeds the pair capacity
(max(64, 4 n)), grows the capacity by 1.5x and re-emits the pairs.  With
``sync_pairs = False`` the whole frame is one CUDA-graph replay with no host
round trip; an overflow then raises XPBD_ERR_OVERFLOW in ``status()``.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _native as N

BROADPHASES = {"lbvh": 0, "hashgrid": 1, "grid": 2}


@dataclass
class RigidBody:
    index: int
    half_extents: tuple
    color: tuple = (0.6, 0.6, 0.7)
    static: bool = False
    is_particle: bool = False
    group: int = 0


def _box_inv_inertia(he, mass):
    """Diagonal body-frame inverse inertia of a solid box (solver_6dof.py:70-76)."""
    lx, ly, lz = 2.0 * he[0], 2.0 * he[1], 2.0 * he[2]
    ix = mass / 12.0 * (ly * ly + lz * lz)
    iy = mass / 12.0 * (lx * lx + lz * lz)
    iz = mass / 12.0 * (lx * lx + ly * ly)
    return (1.0 / ix, 1.0 / iy, 1.0 / iz)


class DeviceVec3:
    """Read view of an (n, 4) device tensor's xyz columns with ``.numpy()``."""

    def __init__(self, t):
        self._t = t

    def numpy(self):
        return self._t[:, :3].cpu().numpy()

    def __array__(self, dtype=None, copy=None):
        a = self.numpy()
        return a if dtype is None else a.astype(dtype)


_SIGS6 = {
    "xpbd6_create": ([C.POINTER(C.c_void_p)], C.c_int),
    "xpbd6_destroy": ([C.c_void_p], C.c_int),
    "xpbd6_bind": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "xpbd6_broadphase": ([C.c_void_p, C.c_void_p], C.c_int),
    "xpbd6_substeps": ([C.c_void_p, C.c_void_p], C.c_int),
    "xpbd6_step": ([C.c_void_p, C.c_int, C.c_void_p], C.c_int),
    "xpbd6_status": ([C.c_void_p, C.POINTER(C.c_int), C.c_void_p], C.c_int),
    "xpbd6_set_driver": ([C.c_void_p, C.c_int, C.c_int, C.c_int], C.c_int),
    "xpbd6_set_lanes": ([C.c_void_p, C.c_int], C.c_int),
    "xpbd6_manifold8": ([C.c_void_p, C.c_float, C.c_void_p], C.c_int),
    "xpbd6_set_grid_constants": ([C.c_void_p, C.c_double, C.c_double, C.c_double], C.c_int),
    "xpbd6_launch_info": ([C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int),
    "xpbd6_morton": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "xpbd6_integrate": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "xpbd6_manifold": ([C.c_void_p, C.c_float, C.c_void_p], C.c_int),
    "xpbd6_solve_positions": ([C.c_void_p, C.c_void_p, C.c_int, C.c_void_p], C.c_int),
    "xpbd6_apply_jacobi": ([C.c_void_p, C.c_float, C.c_void_p], C.c_int),
    "xpbd6_finalize": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "xpbd6_solve_velocities": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "xpbd6_apply_velocity": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "xpbd6_body_aabb": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "xpbd6_residual": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p], C.c_int),
    "xpbd6_phases": ([C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int),
    "xpbd6_points": ([C.c_void_p, C.POINTER(C.c_ulonglong), C.c_int, C.c_void_p], C.c_int),
}


def lib6():
    L = N.lib()
    if not getattr(L, "_six_sigs", False):
        for name, (args, res) in _SIGS6.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        L._six_sigs = True
    return L


class Solver6DOF:
    MAN_MARGIN = 0.02  # solver_6dof.py:119 manifold clip gap

    def __init__(self, dt: float = 1.0 / 60.0, substeps: int = 15, iterations: int = 1,
                 gravity=(0.0, -9.81, 0.0), floor_y: float = 0.0, friction: float = 0.6,
                 restitution: float = 0.0, lin_damp: float = 0.0, ang_damp: float = 0.0,
                 gyroscopic: bool = False, jacobi_relax: float = 1.0, device: str = "cuda:0",
                 max_speed: float = 60.0, max_omega: float = 60.0, broadphase: str = "lbvh",
                 edge_axes: bool = False, warm_start=None):
        """As the reference's constructor, plus `edge_axes` (the nine edge-edge
        SAT axes, off: the reference's manifold) and `warm_start` (no reference
        counterpart; the reference zeroes the contact multipliers every
        substep): None, ``"previous"`` (the classical warm start from each floor
        corner's and manifold point's multiplier over the previous substep) or a
        ``learned.WarmStartMLP``; a warm-started frame also runs the plain first
        iteration every substep and keeps whichever leaves the smaller residual."""
        self.device = N.require_cuda(device)
        self.warm_start = warm_start
        self._runner = None
        self.dt = float(dt)
        self.substeps = int(substeps)
        self.iterations = int(iterations)
        self.gravity = tuple(float(g) for g in gravity)
        self.floor_y = float(floor_y)
        self.friction = float(friction)
        self.restitution = float(restitution)
        self.lin_damp = float(lin_damp)
        self.ang_damp = float(ang_damp)
        self.gyroscopic = bool(gyroscopic)
        self.jacobi_relax = float(jacobi_relax)
        self.max_speed = float(max_speed)
        self.max_omega = float(max_omega)
        # Not in the reference (kernels_6dof.py:13-15 tests face axes only): also
        # test the nine edge-edge SAT axes, giving crossing edges a one-point
        # manifold with the edge-edge normal.  Off by default (reference results).
        self.edge_axes = bool(edge_axes)
        if broadphase not in BROADPHASES:
            raise ValueError(f"broadphase must be one of {sorted(BROADPHASES)}")
        self.broadphase = str(broadphase)
        self.contact_margin = 0.0
        self._man_margin = self.MAN_MARGIN
        self._x, self._q, self._v, self._w = [], [], [], []
        self._inv_mass, self._inv_I, self._he, self._group = [], [], [], []
        self._scene: list[int] = []  # independent-scene id per body (batched scenes)
        self.bodies: list[RigidBody] = []
        self._j_a, self._j_b, self._j_anchor_a, self._j_anchor_b = [], [], [], []
        self._j_rest, self._j_compliance = [], []
        self._dirty = True
        self._t = {}
        self._h = None
        self._sig = None
        self.cap = 0
        self._n_pairs_host = 0
        self.sync_pairs = True
        self.driver = (-1, 0, 0)  # (mode, blocks, threads): -1 automatic; see set_driver
        self.lanes = 8            # lanes per floor body / contact pair in the substep phases
        self._scene_default = 0

    # ---- scene building (solver_6dof.py:166-229) ----------------------------------
    def _add_body(self, position, half_extents, mass, quaternion, velocity, omega, color, static,
                  is_particle, group):
        idx = len(self._x)
        he = tuple(float(h) for h in half_extents)
        self._x.append(tuple(float(p) for p in position))
        self._q.append(tuple(float(c) for c in quaternion))
        self._v.append(tuple(float(c) for c in velocity))
        self._w.append(tuple(float(c) for c in omega))
        if static or mass <= 0.0:
            self._inv_mass.append(0.0)
            self._inv_I.append((0.0, 0.0, 0.0))
            static = True
        elif is_particle:
            self._inv_mass.append(1.0 / float(mass))
            self._inv_I.append((0.0, 0.0, 0.0))
        else:
            self._inv_mass.append(1.0 / float(mass))
            self._inv_I.append(_box_inv_inertia(he, float(mass)))
        self._he.append(he)
        self._group.append(int(group))
        self._scene.append(self._scene_default)
        self._dirty = True
        rb = RigidBody(index=idx, half_extents=he, color=color, static=static, is_particle=is_particle,
                       group=int(group))
        self.bodies.append(rb)
        return rb

    def add_box(self, position, half_extents, mass, quaternion=(0.0, 0.0, 0.0, 1.0), velocity=(0.0, 0.0, 0.0),
                omega=(0.0, 0.0, 0.0), color=(0.6, 0.6, 0.75), static=False):
        return self._add_body(position, half_extents, mass, quaternion, velocity, omega, color, static,
                              is_particle=False, group=0)

    def add_particle(self, position, mass, radius=0.015, velocity=(0.0, 0.0, 0.0), color=(0.85, 0.3, 0.35),
                     static=False, group=1):
        return self._add_body(position, (radius, radius, radius), mass, (0.0, 0.0, 0.0, 1.0), velocity,
                              (0.0, 0.0, 0.0), color, static, is_particle=True, group=group)

    def begin_scene(self, scene_id: int) -> None:
        """Bodies added from now on belong to independent scene `scene_id`: they
        only collide with bodies of the same scene (batched scenes in one solver)."""
        self._scene_default = int(scene_id)
        self._dirty = True

    def add_joint(self, a, b, compliance=0.0, rest_length=None, anchor_a=(0.0, 0.0, 0.0),
                  anchor_b=(0.0, 0.0, 0.0)):
        ia = a.index if hasattr(a, "index") else int(a)
        ib = b.index if hasattr(b, "index") else int(b)
        aa = np.asarray(anchor_a, np.float64)
        ab = np.asarray(anchor_b, np.float64)
        if rest_length is None:
            xa = np.asarray(self._x[ia])
            xb = np.asarray(self._x[ib])
            rest_length = float(np.linalg.norm((xa + aa) - (xb + ab)))
        self._j_a.append(ia)
        self._j_b.append(ib)
        self._j_anchor_a.append(tuple(float(c) for c in anchor_a))
        self._j_anchor_b.append(tuple(float(c) for c in anchor_b))
        self._j_rest.append(float(rest_length))
        self._j_compliance.append(float(compliance))
        self._dirty = True
        return len(self._j_a) - 1

    # ---- flush (solver_6dof.py:261-355) --------------------------------------------
    def _alloc_pairs(self, cap):
        dev = self.device
        T = self._t
        self.cap = int(cap)
        T["pairs"] = torch.zeros((cap, 2), dtype=torch.int32, device=dev)
        T["m_hdr"] = torch.zeros((cap, 4), dtype=torch.int32, device=dev)
        T["m_normal"] = torch.zeros((cap, 4), dtype=torch.float32, device=dev)
        T["m_off_inc"] = torch.zeros((cap * 8, 4), dtype=torch.float32, device=dev)
        T["m_off_ref"] = torch.zeros((cap * 8, 4), dtype=torch.float32, device=dev)
        T["lam_pair"] = torch.zeros(cap * 8, dtype=torch.float32, device=dev)

    def _flush(self):
        if not self._dirty:
            return
        dev = self.device
        n = len(self._x)
        f4 = lambda a, w=None: torch.from_numpy(np.concatenate(  # noqa: E731
            [np.asarray(a, np.float32).reshape(-1, 3),
             (np.zeros((len(a), 1), np.float32) if w is None else np.asarray(w, np.float32).reshape(-1, 1))],
            axis=1) if len(a) else np.zeros((0, 4), np.float32)).to(dev)
        old = self._t
        x = np.asarray(self._x, np.float32).reshape(-1, 3)
        q = np.asarray(self._q, np.float32).reshape(-1, 4)
        v = np.asarray(self._v, np.float32).reshape(-1, 3)
        w = np.asarray(self._w, np.float32).reshape(-1, 3)
        if "x" in old and 0 < old["x"].shape[0] <= n:
            k = old["x"].shape[0]
            x[:k] = old["x"][:, :3].cpu().numpy()
            q[:k] = old["q"].cpu().numpy()
            v[:k] = old["v"][:, :3].cpu().numpy()
            w[:k] = old["w"][:, :3].cpu().numpy()
        for nm, (a, b) in (("joint", (self._j_a, self._j_b)),):
            for ia, ib in zip(a, b):
                if not (0 <= ia < n and 0 <= ib < n):
                    raise IndexError(f"{nm} references a body outside [0, {n})")
        T = {}
        self._t = T
        # x, q, v, w are the four rows of one contiguous block (`state`), so a
        # caller moving the state to or from the host needs one copy each way
        T["state"] = torch.empty((4, n, 4), dtype=torch.float32, device=dev)
        T["state"][0].copy_(f4(x, self._inv_mass))
        T["state"][1].copy_(torch.from_numpy(q.copy()).to(dev))
        T["state"][2].copy_(f4(v))
        T["state"][3].copy_(f4(w))
        T["x"], T["q"], T["v"], T["w"] = T["state"].unbind(0)
        T["x_prev"] = torch.zeros((n, 4), dtype=torch.float32, device=dev)
        T["q_prev"] = torch.zeros((n, 4), dtype=torch.float32, device=dev)
        T["inv_I"] = f4(self._inv_I)
        T["he"] = f4(self._he)
        T["group"] = torch.tensor(np.asarray(self._group, np.int32), device=dev)
        for k in ("acc_x", "acc_r", "acc_v", "acc_w"):
            T[k] = torch.zeros((n, 4), dtype=torch.float32, device=dev)
        T["lam_floor"] = torch.zeros(max(8 * n, 1), dtype=torch.float32, device=dev)
        T["n_pairs"] = torch.zeros(1, dtype=torch.int32, device=dev)
        nj = len(self._j_a)
        T["j_ab"] = torch.tensor(np.stack([np.asarray(self._j_a, np.int32), np.asarray(self._j_b, np.int32)], 1)
                                 if nj else np.zeros((0, 2), np.int32), device=dev)
        T["j_anchor_a"] = f4(self._j_anchor_a, self._j_rest)
        T["j_anchor_b"] = f4(self._j_anchor_b, self._j_compliance)
        T["lam_joint"] = torch.zeros(max(nj, 1), dtype=torch.float32, device=dev)
        self.n_scenes = (max(self._scene) + 1) if self._scene else 1
        T["scene"] = (torch.tensor(np.asarray(self._scene, np.int32), device=dev) if self.n_scenes > 1
                      else torch.zeros(0, dtype=torch.int32, device=dev))
        # graph mode has no per-frame host check, so it starts with more headroom
        self._alloc_pairs(max(64, n * (4 if self.sync_pairs else 16)))
        he = np.asarray(self._he, np.float32).reshape(-1, 3)
        self._rs_max = float(np.linalg.norm(he, axis=1).max()) if n else 0.0
        self._hg_cell = 2.0 * self._rs_max + self._man_margin
        self._dirty = False
        self._bind()

    def _state(self):
        T = self._t
        s = N.xpbd6_state()
        s.n_bodies = len(self._x)
        s.n_joints = len(self._j_a)
        s.pair_capacity = self.cap
        for f in ("x", "q", "v", "w", "x_prev", "q_prev", "inv_I", "he", "group", "acc_x", "acc_r", "acc_v",
                  "acc_w", "lam_floor", "pairs", "n_pairs", "m_hdr", "m_normal", "m_off_inc", "m_off_ref",
                  "lam_pair", "j_ab", "j_anchor_a", "j_anchor_b", "lam_joint"):
            setattr(s, f, N.ptr(T[f]))
        s.scene = N.ptr(T["scene"])
        s.n_scenes = int(self.n_scenes)
        return s

    def _params(self):
        p = N.xpbd6_params()
        p.dt = self.dt
        p.substeps = self.substeps
        p.iterations = self.iterations
        p.gyroscopic = 1 if self.gyroscopic else 0
        p.gravity[:] = self.gravity
        p.floor_y = self.floor_y
        p.friction = self.friction
        p.restitution = self.restitution
        p.lin_damp = self.lin_damp
        p.ang_damp = self.ang_damp
        p.jacobi_relax = self.jacobi_relax
        p.max_speed = self.max_speed
        p.max_omega = self.max_omega
        p.man_margin = self._man_margin
        p.broadphase = BROADPHASES[self.broadphase]
        p.edge_axes = 1 if self.edge_axes else 0
        return p

    def _signature(self):
        """solver_6dof.py:481-487: parameters baked into a bound handle / graph."""
        return (self.cap, self.substeps, self.iterations, self.gyroscopic, self.dt, self.gravity, self.floor_y,
                self.friction, self.restitution, self.lin_damp, self.ang_damp, self.jacobi_relax, self.max_speed,
                self.max_omega, self._man_margin, self.broadphase, self.driver, self.lanes, self.edge_axes)

    def _bind(self):
        self.binds = getattr(self, "binds", 0) + 1  # handle (re)binds: each one re-captures the frame graph
        L = lib6()
        if self._h is None:
            h = C.c_void_p()
            N.check(L.xpbd6_create(C.byref(h)), "xpbd6_create")
            self._h = h
        self._st = self._state()
        self._par = self._params()
        N.check(L.xpbd6_set_driver(self._h, *[int(v) for v in self.driver]), "xpbd6_set_driver")
        N.check(L.xpbd6_set_lanes(self._h, int(self.lanes)), "xpbd6_set_lanes")
        N.check(L.xpbd6_set_grid_constants(self._h, self._rs_max, self._hg_cell, self._rs_max),
                "xpbd6_set_grid_constants")
        N.check(L.xpbd6_bind(self._h, C.byref(self._st), C.byref(self._par)), "xpbd6_bind")
        self._sig = self._signature()

    def set_driver(self, mode=-1, blocks=0, threads=0):
        """Substep driver: -1 automatic, 0 cooperative grid, 2 one thread-block
        cluster (hardware cluster barrier); blocks/threads 0 = automatic."""
        self.driver = (int(mode), int(blocks), int(threads))
        self._sig = None

    def launch_info(self):
        self._flush()
        if self._sig != self._signature():
            self._bind()
        b, t = C.c_int(), C.c_int()
        lib6().xpbd6_launch_info(self._h, C.byref(b), C.byref(t))
        return {"mode": "cluster" if b.value < 0 else "grid", "blocks": abs(b.value), "threads": t.value}

    def phases(self):
        """(barriers, phases) of one frame of the bound substep kernel."""
        self._flush()
        if self._sig != self._signature():
            self._bind()
        b, ph = C.c_int(), C.c_int()
        N.check(lib6().xpbd6_phases(self._h, C.byref(b), C.byref(ph)), "xpbd6_phases")
        return b.value, ph.value

    def manifold_points(self, reset=False):
        """Manifold points summed over every substep run since the last reset
        (synchronizes the stream)."""
        self._flush()
        out = C.c_ulonglong(0)
        N.check(lib6().xpbd6_points(self._h, C.byref(out), 1 if reset else 0, N.stream_of(self.device)),
                "xpbd6_points")
        return int(out.value)

    def autotune(self, frames=3, candidates=None):
        """Time the substep drivers on the current scene and keep the fastest."""
        from .autotune import tune6
        return tune6(self, frames, candidates)

    def invalidate(self):
        """Re-bind (and re-capture the frame graph) before the next step."""
        self._sig = None

    # ---- step (solver_6dof.py:489-529) ---------------------------------------------
    def step(self):
        self._flush()
        n = len(self._x)
        if n == 0:
            return
        if self._sig != self._signature():
            self._bind()
        L = lib6()
        stream = N.stream_of(self.device)
        if self.warm_start is not None:
            if self._runner is None or self._runner.binds != self.binds:
                from .learned import WarmStartRunner6
                self._runner = WarmStartRunner6(self, self.warm_start)
            self._runner.step()
            return
        if not self.sync_pairs:
            N.check(L.xpbd6_step(self._h, 1, stream), "xpbd6_step")
            return
        N.check(L.xpbd6_broadphase(self._h, stream), "xpbd6_broadphase")
        cnt = int(self._t["n_pairs"].item())
        if cnt > self.cap:  # overflow -> grow + re-emit once (solver_6dof.py:444-453)
            self._alloc_pairs(int(cnt * 1.5))
            self._bind()
            handled = C.c_int(0)  # the overflow is resolved here: clear its status bit
            N.check(L.xpbd6_status(self._h, C.byref(handled), stream), "xpbd6_status")
            N.check(L.xpbd6_broadphase(self._h, stream), "xpbd6_broadphase")
            cnt = int(self._t["n_pairs"].item())
        self._n_pairs_host = cnt
        N.check(L.xpbd6_substeps(self._h, stream), "xpbd6_substeps")

    # ---- perturbation / read-back (solver_6dof.py:532-559) --------------------------
    def set_velocity(self, idx, vel):
        self._flush()
        self._t["v"][int(idx), :3] = torch.tensor(vel, dtype=torch.float32, device=self.device)

    def add_impulse(self, idx, dvel):
        self._flush()
        self._t["v"][int(idx), :3] += torch.tensor(dvel, dtype=torch.float32, device=self.device)

    def set_omega(self, idx, w):
        self._flush()
        self._t["w"][int(idx), :3] = torch.tensor(w, dtype=torch.float32, device=self.device)

    @property
    def omega(self):
        self._flush()
        return DeviceVec3(self._t["w"])

    @omega.setter
    def omega(self, values):
        self._flush()
        a = np.asarray(values.numpy() if hasattr(values, "numpy") else values, np.float32).reshape(-1, 3)
        self._t["w"][:, :3] = torch.from_numpy(a).to(self.device)

    def positions(self):
        if not self._t:
            return np.asarray(self._x, np.float32).reshape(-1, 3)
        return self._t["x"][:, :3].cpu().numpy()

    def orientations(self):
        if not self._t:
            return np.asarray(self._q, np.float32).reshape(-1, 4)
        return self._t["q"].cpu().numpy()

    def velocities(self):
        if not self._t:
            return np.asarray(self._v, np.float32).reshape(-1, 3)
        return self._t["v"][:, :3].cpu().numpy()

    def angular_velocities(self):
        return self.omega.numpy()

    def pairs(self):
        """Candidate pairs of the last broad phase, (n_pairs, 2) int32."""
        k = min(self.n_pairs, self.cap)
        return self._t["pairs"][:k].cpu().numpy()

    def status(self) -> int:
        self._flush()
        out = C.c_int(0)
        N.check(lib6().xpbd6_status(self._h, C.byref(out), N.stream_of(self.device)), "xpbd6_status")
        return int(out.value)

    def residual(self, body_scene=None, n_scenes=1):
        """Max residual of the last frame's constraints (joints |C + alpha~ lambda|,
        floor corners and manifold points max(0, -C)), per scene when
        `body_scene` (device int tensor, one scene id per body) is given."""
        self._flush()
        out = torch.zeros(max(int(n_scenes), 1), dtype=torch.float32, device=self.device)
        N.check(lib6().xpbd6_residual(C.byref(self._st), C.byref(self._par), N.ptr(body_scene), int(n_scenes),
                                      N.ptr(out), N.stream_of(self.device)), "xpbd6_residual")
        return out.cpu().numpy()

    def dlpack(self, name: str = "x"):
        """Zero-copy DLPack capsule of one device state tensor (``x``, ``v``, ...,
        see ``tensors``): headless consumers (a viewer, a renderer, another
        framework) read the live state without a host copy.  Float4 records:
        xyz plus the fourth lane of the layout."""
        self._flush()
        return torch.utils.dlpack.to_dlpack(self._t[name])

    def state_dict(self):
        self._flush()
        return {k: self._t[k].clone() for k in ("x", "q", "v", "w", "x_prev", "q_prev")}

    def load_state_dict(self, sd):
        self._flush()
        for k, v in sd.items():
            self._t[k].copy_(v)

    @property
    def tensors(self):
        self._flush()
        return self._t

    @property
    def n_pairs(self):
        if not self._t:
            return 0
        return int(self._t["n_pairs"].item())

    @property
    def num_bodies(self):
        return len(self._x)

    @property
    def num_joints(self):
        return len(self._j_a)

    def __del__(self):
        try:
            if self._h is not None:
                lib6().xpbd6_destroy(self._h)
        except Exception:
            pass

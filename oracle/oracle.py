"""CPU ORACLE for the XPBD substep hot path -- test infrastructure only.

``OracleSolver`` and ``OracleSolver6DOF`` restate the host orchestration of the
reference classes ``Solver`` (src/xpbd3d/solver.py:57-508) and ``Solver6DOF``
(src/xpbd3d/solver_6dof.py:79-559) over numpy arrays, and run every kernel
through ``liboracle.so`` (``xpbd_oracle.c``), the sequential fp32 C restatement
of the reference kernels.  Same constructor arguments, scene-building calls,
``step()`` and read-back as the reference.

Only the tests, the smoke check and the benchmark's CPU-baseline leg use this
module; the engine (``xpbd_b200``) never imports it.
"""

from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

DISTANCE, ATTACH, FLOOR, CONTACT = 0, 1, 2, 3

_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)
_i64p = C.POINTER(C.c_int64)
_u32p = C.POINTER(C.c_uint32)


def build(force=False):
    """Compile liboracle.so (gcc, fp32 with no contraction)."""
    src = os.path.join(HERE, "xpbd_oracle.c")
    if not force and os.path.exists(LIB_PATH) and os.path.getmtime(LIB_PATH) >= os.path.getmtime(src):
        return LIB_PATH
    cmd = (f"gcc -O2 -ffp-contract=off -fno-fast-math -fopenmp -fPIC -shared -o {LIB_PATH}.tmp {src} -lm"
           f" && mv {LIB_PATH}.tmp {LIB_PATH}")
    if os.system(cmd) != 0:
        raise RuntimeError("failed to build the oracle library")
    return LIB_PATH


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        build()
        _LIB = C.CDLL(LIB_PATH)
        L = _LIB
        L.or_grid_candidate_pairs.restype = C.c_int64
        L.or3_sphere_contacts.restype = C.c_int64
        L.or6_pairs_overlap.restype = C.c_int64
        L.or6_pairs_hashgrid.restype = C.c_int64
        L.or6_pairs_grid.restype = C.c_int64
        L.or3_color_constraints.restype = C.c_int
        L.or3_color_ranges.restype = C.c_int
        L.or3_residual.restype = C.c_float
        L.or6_residual.restype = C.c_float
        L.or6_frame.restype = C.c_int64
        L.or6_frame_mt.restype = C.c_int64
        L.or6_pairs_overlap_mt.restype = C.c_int64
        L.or_max_threads.restype = C.c_int
    return _LIB


def fp(a):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_fp)


def ip(a):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_ip)


class or3_scene(C.Structure):
    _fields_ = [("n_bodies", C.c_int), ("n_rows", C.c_int),
                ("x", _fp), ("v", _fp), ("x_prev", _fp), ("inv_mass", _fp),
                ("r_type", _ip), ("r_a", _ip), ("r_b", _ip), ("r_active", _ip),
                ("r_rest", _fp), ("r_comp", _fp), ("r_anchor", _fp), ("r_mu", _fp),
                ("r_lambda", _fp), ("dx", _fp), ("dn", _ip),
                ("color_order", _ip), ("color_starts", _ip), ("num_colors", C.c_int)]


class or3_params(C.Structure):
    _fields_ = [("dt", C.c_double), ("substeps", C.c_int), ("iterations", C.c_int),
                ("gx", C.c_float), ("gy", C.c_float), ("gz", C.c_float),
                ("damping", C.c_float), ("jacobi_relax", C.c_float), ("max_speed", C.c_float),
                ("gs", C.c_int)]


class or6_scene(C.Structure):
    _fields_ = [("n", C.c_int), ("n_joints", C.c_int), ("cap", C.c_int),
                ("x", _fp), ("q", _fp), ("v", _fp), ("w", _fp), ("x_prev", _fp), ("q_prev", _fp),
                ("inv_mass", _fp), ("inv_I", _fp), ("he", _fp), ("group", _ip),
                ("dx", _fp), ("drot", _fp), ("dv", _fp), ("dw", _fp),
                ("dcount", _ip), ("dvc", _ip), ("lam_floor", _fp),
                ("pair_a", _ip), ("pair_b", _ip), ("n_pairs", C.c_int),
                ("m_count", _ip), ("m_inc", _ip), ("m_ref", _ip),
                ("m_normal", _fp), ("m_off_inc", _fp), ("m_off_ref", _fp), ("lam_pair", _fp),
                ("j_a", _ip), ("j_b", _ip), ("j_anchor_a", _fp), ("j_anchor_b", _fp),
                ("j_rest", _fp), ("j_comp", _fp), ("lam_joint", _fp)]


class or6_params(C.Structure):
    _fields_ = [("dt", C.c_double), ("substeps", C.c_int), ("iterations", C.c_int),
                ("gyroscopic", C.c_int),
                ("gx", C.c_float), ("gy", C.c_float), ("gz", C.c_float), ("floor_y", C.c_float),
                ("friction", C.c_float), ("restitution", C.c_float), ("lin_damp", C.c_float),
                ("ang_damp", C.c_float), ("jacobi_relax", C.c_float), ("max_speed", C.c_float),
                ("max_omega", C.c_float), ("man_margin", C.c_float)]


def _f32(a, shape=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    return a.reshape(shape) if shape is not None else a


def _i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


# ---------------------------------------------------------------------------
# host helpers restated from the reference
# ---------------------------------------------------------------------------
def color_constraints(n_bodies, a, b):
    """coloring.py:26-71."""
    a = _i32(a); b = _i32(b)
    col = np.full(len(a), -1, np.int32)
    if len(a):
        lib().or3_color_constraints(int(n_bodies), len(a), ip(a), ip(b), ip(col))
    return col


def color_ranges(color):
    """coloring.py:74-89."""
    color = _i32(color)
    if len(color) == 0:
        return np.zeros(0, np.int32), np.zeros(1, np.int32), 0
    k = int(color.max()) + 1
    order = np.zeros(len(color), np.int32)
    starts = np.zeros(k + 1, np.int32)
    lib().or3_color_ranges(len(color), ip(color), ip(order), ip(starts))
    return order, starts, k


def grid_candidate_pairs(p, cell):
    """solver.py:520-562 (local indices, reference emission order)."""
    p = _f32(p, (-1, 3))
    m = p.shape[0]
    cap = m * 64 + 1024
    while True:
        a = np.zeros(cap, np.int32); b = np.zeros(cap, np.int32)
        cnt = lib().or_grid_candidate_pairs(m, fp(p), C.c_float(cell), C.c_int64(cap), ip(a), ip(b))
        if cnt <= cap:
            return a[:cnt], b[:cnt]
        cap = int(cnt)


def shape_radius(shape):
    """solver.py:565-575."""
    if shape is None:
        return 0.0
    if shape.kind == "sphere":
        return float(shape.size[0])
    if shape.kind == "cube":
        return float(min(shape.size))
    if shape.kind == "pillar":
        return float(shape.size[0])
    return 0.0


@dataclass
class _Row:
    type: int
    body_a: int
    body_b: int = -1
    rest: float = 0.0
    compliance: float = 0.0
    anchor: tuple = (0.0, 0.0, 0.0)
    mu: float = 0.0


@dataclass
class _Handle:
    index: int
    rows: int = 1


# ---------------------------------------------------------------------------
class OracleSolver:
    """solver.py:57-508 restated over numpy + liboracle."""

    def __init__(self, dt=1.0 / 60.0, substeps=10, iterations=1, gravity=(0.0, -9.81, 0.0),
                 damping=0.0, solve_mode="auto", jacobi_relax=1.0, device="cpu", max_speed=40.0):
        self.device = device
        self.dt = float(dt)
        self.substeps = int(substeps)
        self.iterations = int(iterations)
        self.gravity = tuple(float(g) for g in gravity)
        self.damping = float(damping)
        self.jacobi_relax = float(jacobi_relax)
        self.max_speed = float(max_speed)
        if solve_mode == "auto":
            solve_mode = "jacobi" if str(device).startswith("cuda") else "gs"
        assert solve_mode in ("gs", "jacobi")
        self.solve_mode = solve_mode
        self._x, self._v, self._mass, self._radius = [], [], [], []
        self._collide, self._friction, self._rows = [], [], []
        self._self_collision = False
        self._contact_margin = 0.0
        self._default_friction = 0.0
        self._dirty = True
        self.x = self.v = None
        self.lam = None
        self.num_colors = 0
        self.color_counts = {}
        # host threads of the substep loop: 1 = the sequential parity oracle;
        # more = or3_frame_mt, the timed CPU baseline (Jacobi sums round in
        # another order)
        self.threads = 1

    # scene building (solver.py:130-228)
    def add_particle(self, position, mass, velocity=(0.0, 0.0, 0.0), shape=None, collide=True,
                     radius=None, friction=None):
        idx = len(self._x)
        self._x.append(tuple(float(v) for v in position))
        self._v.append(tuple(float(v) for v in velocity))
        self._mass.append(float(mass))
        r = float(radius) if radius is not None else shape_radius(shape)
        self._radius.append(r)
        self._collide.append(bool(collide) and r > 0.0 and mass > 0.0)
        mu = float(friction) if friction is not None else self._default_friction
        self._friction.append(max(0.0, mu))
        self._dirty = True
        return _Handle(idx)

    def add_distance(self, body_a, body_b, rest=None, compliance=0.0):
        if rest is None:
            rest = float(np.linalg.norm(np.asarray(self._x[body_a.index]) - np.asarray(self._x[body_b.index])))
        self._rows.append(_Row(DISTANCE, body_a.index, body_b.index, rest=float(rest),
                               compliance=float(compliance)))
        self._dirty = True
        return _Handle(len(self._rows) - 1)

    def add_attach(self, body, world_point, compliance=0.0, rest=0.0):
        self._rows.append(_Row(ATTACH, body.index, -1, rest=float(rest), compliance=float(compliance),
                               anchor=tuple(float(p) for p in world_point)))
        self._dirty = True
        return _Handle(len(self._rows) - 1)

    def add_floor_contact(self, body, floor_y=0.0, friction=None):
        mu = float(friction) if friction is not None else self._friction[body.index]
        self._rows.append(_Row(FLOOR, body.index, -1, anchor=(0.0, float(floor_y), 0.0), mu=max(0.0, mu)))
        self._dirty = True
        return _Handle(len(self._rows) - 1)

    def enable_self_collision(self, enabled=True, margin=0.0, default_friction=None):
        self._self_collision = bool(enabled)
        self._contact_margin = float(margin)
        if default_friction is not None:
            self._default_friction = max(0.0, float(default_friction))
            for k in range(len(self._friction)):
                if self._friction[k] == 0.0:
                    self._friction[k] = self._default_friction

    # perturbations (solver.py:232-271)
    def set_position(self, body, p):
        self._flush(); self.x[body.index] = np.asarray(p, np.float32)

    def set_velocity(self, body, vel):
        self._flush(); self.v[body.index] = np.asarray(vel, np.float32)

    def add_impulse(self, body, dv):
        self._flush(); self.v[body.index] += np.asarray(dv, np.float32)

    def set_all_compliance(self, value, only_distance=True):
        self._flush()
        for i, r in enumerate(self._rows):
            if (not only_distance) or r.type == DISTANCE:
                r.compliance = float(value)
                self.r_comp[i] = np.float32(value)

    def set_all_friction(self, mu):
        self._flush()
        self._default_friction = float(mu)
        for k in range(len(self._friction)):
            self._friction[k] = float(mu)
        for i, r in enumerate(self._rows):
            if r.type in (FLOOR, CONTACT):
                r.mu = float(mu)
                self.r_mu[i] = np.float32(mu)

    # solver.py:275-342
    def _rebuild_contacts(self):
        if not self._self_collision:
            return
        self._rows = [r for r in self._rows if r.type != CONTACT]
        existing = set()
        for r in self._rows:
            if r.body_b >= 0:
                a, b = (r.body_a, r.body_b) if r.body_a < r.body_b else (r.body_b, r.body_a)
                existing.add((a, b))
        n = len(self._x)
        pos = self.x if self.x is not None else _f32(self._x, (-1, 3))
        collide = np.asarray(self._collide, dtype=bool)
        idx = _i32(np.nonzero(collide)[0])
        if len(idx) < 2:
            self._dirty = True
            return
        radii = _f32(self._radius)
        friction = _f32(self._friction)
        vmax = float(np.abs(self.v).max()) if self.v is not None else 0.0
        rmax = float(radii[idx].max())
        margin = min(self._contact_margin + 3.0 * self.dt * vmax, rmax)
        cell = float(radii[idx].max()) * 2.0 + margin
        keys = np.array(sorted(a * n + b for a, b in existing), np.int64)
        cap = max(1024, 64 * len(idx))
        while True:
            ra = np.zeros(cap, np.int32); rb = np.zeros(cap, np.int32)
            rest = np.zeros(cap, np.float32); rmu = np.zeros(cap, np.float32)
            cnt = lib().or3_sphere_contacts(n, fp(pos), fp(radii), fp(friction), ip(idx), len(idx),
                                            C.c_float(cell), C.c_float(margin),
                                            keys.ctypes.data_as(_i64p), len(keys), C.c_int64(cap),
                                            ip(ra), ip(rb), fp(rest), fp(rmu))
            if cnt <= cap:
                break
            cap = int(cnt)
        for k in range(int(cnt)):
            self._rows.append(_Row(CONTACT, int(ra[k]), int(rb[k]), rest=float(rest[k]), mu=float(rmu[k])))
        self._dirty = True

    # solver.py:346-408
    def _flush(self):
        if not self._dirty:
            return
        n = len(self._x)
        m = len(self._rows)
        x = _f32(self._x, (-1, 3)) if n else np.zeros((0, 3), np.float32)
        v = _f32(self._v, (-1, 3)) if n else np.zeros((0, 3), np.float32)
        if self.x is not None and 0 < self.x.shape[0] <= n:
            k = self.x.shape[0]
            x[:k] = self.x; v[:k] = self.v
        mass = _f32(self._mass) if n else np.zeros(0, np.float32)
        self.inv_mass = np.where(mass > 0.0, 1.0 / np.maximum(mass, 1e-20), 0.0).astype(np.float32)
        self.x, self.v = x, v
        self.x_prev = np.zeros_like(x)
        self.dx = np.zeros((n, 3), np.float32)
        self.dn = np.zeros(n, np.int32)
        R = self._rows
        self.r_type = _i32([r.type for r in R]); self.r_a = _i32([r.body_a for r in R])
        self.r_b = _i32([r.body_b for r in R])
        self.r_rest = _f32([r.rest for r in R]); self.r_comp = _f32([r.compliance for r in R])
        self.r_anchor = _f32([r.anchor for r in R], (-1, 3)) if m else np.zeros((0, 3), np.float32)
        self.r_mu = _f32([r.mu for r in R])
        self.lam = np.zeros(m, np.float32)
        self.r_active = np.ones(m, np.int32)
        if self.solve_mode == "gs" and m > 0:
            col = color_constraints(n, self.r_a, self.r_b)
            self.color_order, self.color_starts, self.num_colors = color_ranges(col)
            self.color_counts = {int(c): int(k) for c, k in zip(*np.unique(col, return_counts=True))}
        else:
            self.color_order = np.zeros(max(m, 1), np.int32)
            self.color_starts = np.array([0, m], np.int32)
            self.num_colors = 1 if m else 0
            self.color_counts = {}
        self._dirty = False

    def _sanitize_positions(self):
        """solver.py:469-483."""
        if self.x is None or np.all(np.isfinite(self.x)):
            return
        bad = ~np.all(np.isfinite(self.x), axis=1)
        safe = _f32(self._x, (-1, 3))
        self.x[bad] = safe[bad]
        self.v[bad] = 0.0

    def _scene(self):
        sc = or3_scene()
        sc.n_bodies = len(self._x); sc.n_rows = len(self._rows)
        sc.x, sc.v, sc.x_prev, sc.inv_mass = fp(self.x), fp(self.v), fp(self.x_prev), fp(self.inv_mass)
        sc.r_type, sc.r_a, sc.r_b, sc.r_active = ip(self.r_type), ip(self.r_a), ip(self.r_b), ip(self.r_active)
        sc.r_rest, sc.r_comp, sc.r_anchor, sc.r_mu = (fp(self.r_rest), fp(self.r_comp),
                                                      fp(self.r_anchor), fp(self.r_mu))
        sc.r_lambda, sc.dx, sc.dn = fp(self.lam), fp(self.dx), ip(self.dn)
        sc.color_order, sc.color_starts = ip(self.color_order), ip(self.color_starts)
        sc.num_colors = self.num_colors
        return sc

    def _params(self):
        p = or3_params()
        p.dt = self.dt; p.substeps = self.substeps; p.iterations = self.iterations
        p.gx, p.gy, p.gz = self.gravity
        p.damping = self.damping; p.jacobi_relax = self.jacobi_relax
        p.max_speed = self.max_speed if math.isfinite(self.max_speed) else float("inf")
        p.gs = 1 if self.solve_mode == "gs" else 0
        return p

    def step(self):
        """solver.py:412-442."""
        if self._self_collision:
            self._flush()
            self._sanitize_positions()
            self._rebuild_contacts()
        self._flush()
        if len(self._x) == 0:
            return
        if self.threads > 1:
            lib().or3_frame_mt(C.byref(self._scene()), C.byref(self._params()), int(self.threads))
        else:
            lib().or3_frame(C.byref(self._scene()), C.byref(self._params()))

    def positions(self):
        return self.x.copy() if self.x is not None else _f32(self._x, (-1, 3))

    def velocities(self):
        return self.v.copy() if self.v is not None else _f32(self._v, (-1, 3))

    def residual(self, per_row=False):
        """Max residual: hard rows max(0, -C), compliant rows |C + alpha~ lambda|."""
        self._flush()
        rows = np.zeros(max(len(self._rows), 1), np.float32)
        mx = lib().or3_residual(C.byref(self._scene()), C.c_float(self.dt / self.substeps), fp(rows))
        return (float(mx), rows[:len(self._rows)]) if per_row else float(mx)

    def lambdas(self):
        return self.lam.copy() if self.lam is not None else np.zeros(len(self._rows), np.float32)

    @property
    def num_bodies(self):
        return len(self._x)

    @property
    def num_constraints(self):
        return len(self._rows)


# ---------------------------------------------------------------------------
def box_inv_inertia(he, mass):
    """solver_6dof.py:70-76 (fp64 host arithmetic, stored as fp32)."""
    lx, ly, lz = 2.0 * he[0], 2.0 * he[1], 2.0 * he[2]
    ix = mass / 12.0 * (ly * ly + lz * lz)
    iy = mass / 12.0 * (lx * lx + lz * lz)
    iz = mass / 12.0 * (lx * lx + ly * ly)
    return (1.0 / ix, 1.0 / iy, 1.0 / iz)


@dataclass
class RigidBodyHandle:
    index: int
    half_extents: tuple
    color: tuple = (0.6, 0.6, 0.7)
    static: bool = False
    is_particle: bool = False
    group: int = 0


class OracleSolver6DOF:
    """solver_6dof.py:79-559 restated over numpy + liboracle."""

    MAN_MARGIN = 0.02

    def __init__(self, dt=1.0 / 60.0, substeps=15, iterations=1, gravity=(0.0, -9.81, 0.0),
                 floor_y=0.0, friction=0.6, restitution=0.0, lin_damp=0.0, ang_damp=0.0,
                 gyroscopic=False, jacobi_relax=1.0, device="cpu", max_speed=60.0, max_omega=60.0,
                 broadphase="lbvh"):
        self.device = device
        self.dt = float(dt); self.substeps = int(substeps); self.iterations = int(iterations)
        self.gravity = tuple(float(g) for g in gravity)
        self.floor_y = float(floor_y); self.friction = float(friction)
        self.restitution = float(restitution); self.lin_damp = float(lin_damp)
        self.ang_damp = float(ang_damp); self.gyroscopic = bool(gyroscopic)
        self.jacobi_relax = float(jacobi_relax); self.max_speed = float(max_speed)
        self.max_omega = float(max_omega); self.broadphase = str(broadphase)
        self._man_margin = self.MAN_MARGIN
        self._x, self._q, self._v, self._w = [], [], [], []
        self._inv_mass, self._inv_I, self._he, self._group = [], [], [], []
        self.bodies = []
        self._j_a, self._j_b, self._j_aa, self._j_ab, self._j_rest, self._j_comp = [], [], [], [], [], []
        self._dirty = True
        self.x = self.q = self.v = self.omega = None
        self.n_pairs = 0
        self.cap = 0
        self.threads = 1  # > 1: or6_frame_mt and the threaded pair emission (timed CPU baseline)

    def _add_body(self, position, half_extents, mass, quaternion, velocity, omega, color, static,
                  is_particle, group):
        idx = len(self._x)
        he = tuple(float(h) for h in half_extents)
        self._x.append(tuple(float(p) for p in position))
        self._q.append(tuple(float(c) for c in quaternion))
        self._v.append(tuple(float(c) for c in velocity))
        self._w.append(tuple(float(c) for c in omega))
        if static or mass <= 0.0:
            self._inv_mass.append(0.0); self._inv_I.append((0.0, 0.0, 0.0)); static = True
        elif is_particle:
            self._inv_mass.append(1.0 / float(mass)); self._inv_I.append((0.0, 0.0, 0.0))
        else:
            self._inv_mass.append(1.0 / float(mass)); self._inv_I.append(box_inv_inertia(he, float(mass)))
        self._he.append(he)
        self._group.append(int(group))
        self._dirty = True
        rb = RigidBodyHandle(idx, he, color, static, is_particle, int(group))
        self.bodies.append(rb)
        return rb

    def add_box(self, position, half_extents, mass, quaternion=(0.0, 0.0, 0.0, 1.0),
                velocity=(0.0, 0.0, 0.0), omega=(0.0, 0.0, 0.0), color=(0.6, 0.6, 0.75), static=False):
        return self._add_body(position, half_extents, mass, quaternion, velocity, omega, color, static,
                              False, 0)

    def add_particle(self, position, mass, radius=0.015, velocity=(0.0, 0.0, 0.0),
                     color=(0.85, 0.3, 0.35), static=False, group=1):
        return self._add_body(position, (radius, radius, radius), mass, (0.0, 0.0, 0.0, 1.0), velocity,
                              (0.0, 0.0, 0.0), color, static, True, group)

    def add_joint(self, a, b, compliance=0.0, rest_length=None, anchor_a=(0.0, 0.0, 0.0),
                  anchor_b=(0.0, 0.0, 0.0)):
        ia = a.index if hasattr(a, "index") else int(a)
        ib = b.index if hasattr(b, "index") else int(b)
        aa = np.asarray(anchor_a, np.float64); ab = np.asarray(anchor_b, np.float64)
        if rest_length is None:
            rest_length = float(np.linalg.norm((np.asarray(self._x[ia]) + aa) - (np.asarray(self._x[ib]) + ab)))
        self._j_a.append(ia); self._j_b.append(ib)
        self._j_aa.append(tuple(float(c) for c in anchor_a))
        self._j_ab.append(tuple(float(c) for c in anchor_b))
        self._j_rest.append(float(rest_length)); self._j_comp.append(float(compliance))
        self._dirty = True
        return len(self._j_a) - 1

    def _alloc_pairs(self, cap):
        self.cap = int(cap)
        self.pair_a = np.zeros(cap, np.int32); self.pair_b = np.zeros(cap, np.int32)
        self.lam_pair = np.zeros(cap * 8, np.float32)
        self.m_count = np.zeros(cap, np.int32); self.m_inc = np.zeros(cap, np.int32)
        self.m_ref = np.zeros(cap, np.int32)
        self.m_normal = np.zeros((cap, 3), np.float32)
        self.m_off_inc = np.zeros((cap * 8, 3), np.float32)
        self.m_off_ref = np.zeros((cap * 8, 3), np.float32)

    def _flush(self):
        """solver_6dof.py:261-342."""
        if not self._dirty:
            return
        n = len(self._x)
        x = _f32(self._x, (-1, 3)); q = _f32(self._q, (-1, 4))
        v = _f32(self._v, (-1, 3)); w = _f32(self._w, (-1, 3))
        if self.x is not None and 0 < self.x.shape[0] <= n:
            k = self.x.shape[0]
            x[:k] = self.x; q[:k] = self.q; v[:k] = self.v; w[:k] = self.omega
        self.x, self.q, self.v, self.omega = x, q, v, w
        self.x_prev = np.zeros((n, 3), np.float32); self.q_prev = np.zeros((n, 4), np.float32)
        self.inv_mass = _f32(self._inv_mass); self.inv_I = _f32(self._inv_I, (-1, 3))
        self.he = _f32(self._he, (-1, 3)); self.group = _i32(self._group)
        for nm in ("dx", "drot", "dv", "dw"):
            setattr(self, nm, np.zeros((n, 3), np.float32))
        self.dcount = np.zeros(n, np.int32); self.dvc = np.zeros(n, np.int32)
        self.lam_floor = np.zeros(n * 8, np.float32)
        self.n_joints = len(self._j_a)
        self.j_a = _i32(self._j_a); self.j_b = _i32(self._j_b)
        self.j_anchor_a = _f32(self._j_aa, (-1, 3)) if self.n_joints else np.zeros((0, 3), np.float32)
        self.j_anchor_b = _f32(self._j_ab, (-1, 3)) if self.n_joints else np.zeros((0, 3), np.float32)
        self.j_rest = _f32(self._j_rest); self.j_comp = _f32(self._j_comp)
        self.lam_joint = np.zeros(self.n_joints, np.float32)
        self._alloc_pairs(max(64, n * 4))
        self.lowers = np.zeros((max(n, 1), 3), np.float32); self.uppers = np.zeros((max(n, 1), 3), np.float32)
        he_arr = self.he
        self._hg_rsmax = float(np.linalg.norm(he_arr, axis=1).max()) if n else 0.0
        self._hg_cell = 2.0 * self._hg_rsmax + self._man_margin
        self._dirty = False

    def _emit(self, fn):
        cnt = fn(self.cap)
        if cnt > self.cap:
            self._alloc_pairs(int(cnt * 1.5))
            cnt = fn(self.cap)
        return int(cnt)

    def _broadphase(self):
        n = len(self._x)
        L = lib()
        if self.broadphase == "lbvh":
            L.or6_body_aabb(n, fp(self.x), fp(self.q), fp(self.v), fp(self.omega), fp(self.he),
                            C.c_float(self._man_margin), C.c_float(self.dt), fp(self.lowers), fp(self.uppers))
            if self.threads > 1:
                return self._emit(lambda cap: L.or6_pairs_overlap_mt(
                    n, fp(self.lowers), fp(self.uppers), fp(self.inv_mass), ip(self.group), C.c_int64(cap),
                    ip(self.pair_a), ip(self.pair_b), int(self.threads)))
            return self._emit(lambda cap: L.or6_pairs_overlap(n, fp(self.lowers), fp(self.uppers),
                                                              fp(self.inv_mass), ip(self.group),
                                                              C.c_int64(cap), ip(self.pair_a), ip(self.pair_b)))
        if self.broadphase == "hashgrid":
            return self._emit(lambda cap: L.or6_pairs_hashgrid(
                n, fp(self.x), fp(self.q), fp(self.v), fp(self.omega), fp(self.he), fp(self.inv_mass),
                ip(self.group), C.c_float(self._man_margin), C.c_float(self.dt),
                C.c_float(self._hg_rsmax), C.c_float(self._hg_cell), C.c_int64(cap),
                ip(self.pair_a), ip(self.pair_b)))
        # host grid (solver_6dof.py:232-258)
        if n < 2:
            return 0
        aabb = np.zeros((n, 3), np.float32)
        L.or6_world_aabb_half(n, fp(self.q), fp(self.he), fp(aabb))
        vmax = float(np.abs(self.v).max())
        wmax = float(np.abs(self.omega).max())
        rmax = float(aabb.max())
        maxhe = float(np.linalg.norm(self.he, axis=1).max())
        margin = min(self._man_margin + 2.0 * self.dt * (vmax + wmax * maxhe), rmax)
        cell = 2.0 * rmax + margin
        return self._emit(lambda cap: L.or6_pairs_grid(n, fp(self.x), fp(aabb), fp(self.inv_mass),
                                                        ip(self.group), C.c_float(cell), C.c_float(margin),
                                                        C.c_int64(cap), ip(self.pair_a), ip(self.pair_b)))

    def _scene(self):
        s = or6_scene()
        s.n = len(self._x); s.n_joints = self.n_joints; s.cap = self.cap
        for nm in ("x", "q", "v", "x_prev", "q_prev", "inv_mass", "inv_I", "he", "dx", "drot", "dv", "dw",
                   "lam_floor", "m_normal", "m_off_inc", "m_off_ref", "lam_pair", "j_anchor_a",
                   "j_anchor_b", "j_rest", "lam_joint"):
            setattr(s, nm, fp(getattr(self, nm)))
        s.w = fp(self.omega); s.j_comp = fp(self.j_comp)
        for nm in ("group", "dcount", "dvc", "pair_a", "pair_b", "m_count", "m_inc", "m_ref", "j_a", "j_b"):
            setattr(s, nm, ip(getattr(self, nm)))
        s.n_pairs = min(self.n_pairs, self.cap)
        return s

    def _params(self):
        p = or6_params()
        p.dt = self.dt; p.substeps = self.substeps; p.iterations = self.iterations
        p.gyroscopic = 1 if self.gyroscopic else 0
        p.gx, p.gy, p.gz = self.gravity
        p.floor_y = self.floor_y; p.friction = self.friction; p.restitution = self.restitution
        p.lin_damp = self.lin_damp; p.ang_damp = self.ang_damp; p.jacobi_relax = self.jacobi_relax
        p.max_speed = self.max_speed; p.max_omega = self.max_omega; p.man_margin = self._man_margin
        return p

    def step(self):
        """solver_6dof.py:489-529 (device="cpu" branch: _record runs directly)."""
        self._flush()
        if len(self._x) == 0:
            return
        self.n_pairs = self._broadphase()
        # manifold points summed over this frame's substeps (the projection count)
        if self.threads > 1:
            self.frame_points = int(lib().or6_frame_mt(C.byref(self._scene()), C.byref(self._params()),
                                                       int(self.threads)))
        else:
            self.frame_points = int(lib().or6_frame(C.byref(self._scene()), C.byref(self._params())))

    def residual(self):
        """Max residual of the last frame's joints, floor corners and manifold points."""
        self._flush()
        return float(lib().or6_residual(C.byref(self._scene()), C.c_float(self.floor_y),
                                        C.c_float(self.dt / self.substeps)))

    def set_velocity(self, idx, vel):
        self._flush(); self.v[idx] = np.asarray(vel, np.float32)

    def add_impulse(self, idx, dvel):
        self._flush(); self.v[idx] += np.asarray(dvel, np.float32)

    def positions(self):
        return self.x.copy() if self.x is not None else _f32(self._x, (-1, 3))

    def orientations(self):
        return self.q.copy() if self.q is not None else _f32(self._q, (-1, 4))

    def velocities(self):
        return self.v.copy() if self.v is not None else _f32(self._v, (-1, 3))

    @property
    def num_bodies(self):
        return len(self._x)

    @property
    def num_joints(self):
        return len(self._j_a)


def host_threads():
    """Threads the OpenMP runtime offers (OMP_NUM_THREADS, else the host's cores)."""
    return int(lib().or_max_threads())


def morton_codes(lowers, uppers):
    """The engine's own LBVH key definition (see xpbd_oracle.c)."""
    lo = _f32(lowers, (-1, 3)); hi = _f32(uppers, (-1, 3))
    out = np.zeros(lo.shape[0], np.uint32)
    lib().or_morton_codes(lo.shape[0], fp(lo), fp(hi), out.ctypes.data_as(_u32p))
    return out

"""The reference's own acceptance tests (tests/test_solver.py and
tests/test_solver_6dof.py of nanli9/XPBD), run against the B200 engine through
the same public API.  Scenes, step counts and tolerances are the reference's;
the only change is that the device is a CUDA device and that angular velocity
is written through ``Solver6DOF.omega = ...`` instead of replacing a Warp array.
"""

import math

import numpy as np
import pytest

pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle import oracle as O  # noqa: E402
from xpbd_b200 import Body, Shape, Solver, Solver6DOF  # noqa: E402

DEVICE = "cuda:0"


# ---------------------------------------------------------------- tests/test_solver.py
def test_free_fall_matches_analytic():
    s = Solver(dt=1 / 60, substeps=10, iterations=1, device=DEVICE)
    b = s.add_particle((0, 0, 0), mass=1.0, collide=False)
    for _ in range(60):
        s.step()
    t = 1.0
    assert abs(s.velocities()[b.index, 1] - (-9.81 * t)) < 0.05
    assert abs(s.positions()[b.index, 1] - 0.5 * -9.81 * t * t) < 0.05


def test_static_body_never_moves():
    s = Solver(dt=1 / 60, substeps=10, device=DEVICE)
    a = s.add_particle((0, 1, 0), mass=0.0, collide=False)
    for _ in range(30):
        s.step()
    assert np.allclose(s.positions()[a.index], [0, 1, 0])


@pytest.mark.parametrize("mode", ["gs", "jacobi"])
def test_hard_distance_holds_length(mode):
    s = Solver(dt=1 / 60, substeps=15, iterations=2, device=DEVICE, solve_mode=mode)
    a = s.add_particle((0, 2, 0), mass=0.0, collide=False)
    b = s.add_particle((0.5, 2, 0), mass=1.0, collide=False)
    s.add_distance(a, b, rest=0.5, compliance=0.0)
    for _ in range(120):
        s.step()
    L = np.linalg.norm(s.positions()[b.index] - s.positions()[a.index])
    assert abs(L - 0.5) < 1e-3


@pytest.mark.parametrize("iters", [1, 4, 16])
def test_compliance_iteration_independent(iters):
    alpha = 1e-3
    s = Solver(dt=1 / 60, substeps=20, iterations=iters, device=DEVICE, solve_mode="gs", damping=0.05)
    a = s.add_particle((0, 2, 0), mass=0.0, collide=False)
    b = s.add_particle((0, 1, 0), mass=1.0, collide=False)
    s.add_distance(a, b, rest=1.0, compliance=alpha)
    for _ in range(800):
        s.step()
    stretch = np.linalg.norm(s.positions()[b.index] - s.positions()[a.index]) - 1.0
    analytic = 1.0 * 9.81 * alpha
    assert abs(stretch - analytic) < 0.1 * analytic


def test_floor_contact_rest():
    s = Solver(dt=1 / 60, substeps=10, iterations=2, device=DEVICE)
    b = s.add_particle((0, 2, 0), mass=1.0, shape=Shape("sphere", (0.1,)), collide=False)
    s.add_floor_contact(b, floor_y=0.1, friction=0.5)
    for _ in range(180):
        s.step()
    assert abs(s.positions()[b.index, 1] - 0.1) < 1e-3
    assert abs(s.velocities()[b.index, 1]) < 1e-2


@pytest.mark.parametrize("mode", ["gs", "jacobi"])
def test_two_spheres_do_not_overlap(mode):
    s = Solver(dt=1 / 60, substeps=15, iterations=2, device=DEVICE, solve_mode=mode)
    a = s.add_particle((0.0, 1.0, 0), mass=1.0, shape=Shape("sphere", (0.2,)))
    b = s.add_particle((0.15, 0.4, 0), mass=1.0, shape=Shape("sphere", (0.2,)))
    s.add_floor_contact(a, floor_y=0.2, friction=0.4)
    s.add_floor_contact(b, floor_y=0.2, friction=0.4)
    s.enable_self_collision(True, default_friction=0.4)
    for _ in range(240):
        s.step()
    d = np.linalg.norm(s.positions()[a.index] - s.positions()[b.index])
    assert d >= 0.4 - 2e-3


@pytest.mark.parametrize("mode", ["gs", "jacobi"])
def test_stack_column_settles(mode):
    s = Solver(dt=1 / 60, substeps=20, iterations=2, device=DEVICE, solve_mode=mode, max_speed=0.0)
    r = 0.16
    for k in range(4):
        b = s.add_particle((0, r + k * 2.1 * r, 0), mass=1.0, shape=Shape("sphere", (r,)), friction=0.3)
        s.add_floor_contact(b, floor_y=r, friction=0.3)
    s.enable_self_collision(True, margin=0.05, default_friction=0.3)
    for _ in range(220):
        s.step()
    ys = np.sort(s.positions()[:, 1])
    assert ys.max() < 1.5
    assert np.all(np.isfinite(s.positions()))
    assert np.allclose(np.diff(ys), 2 * r, atol=5e-3)


def test_friction_decelerates_slide():
    s = Solver(dt=1 / 60, substeps=10, iterations=2, device=DEVICE)
    b = s.add_particle((0, 0.1, 0), mass=1.0, shape=Shape("sphere", (0.1,)), collide=False)
    s.add_floor_contact(b, floor_y=0.1, friction=0.5)
    s.set_velocity(b, (3.0, 0, 0))
    for _ in range(120):
        s.step()
    assert abs(s.velocities()[b.index, 0]) < 0.5


def test_coloring_is_valid():
    """Engine coloring (host C++ in libxpbd_b200) on the reference test's graph."""
    import ctypes as C

    from xpbd_b200 import _native as N
    rng = np.random.default_rng(0)
    n_bodies = 40
    a = rng.integers(0, n_bodies, 200).astype(np.int32)
    b = rng.integers(0, n_bodies, 200).astype(np.int32)
    b = np.where(b == a, (b + 1) % n_bodies, b).astype(np.int32)
    color = np.zeros(200, np.int32)
    N.lib().xpbd_color_constraints(n_bodies, 200, a.ctypes.data_as(C.c_void_p), b.ctypes.data_as(C.c_void_p),
                                   color.ctypes.data_as(C.c_void_p))
    incident = {}
    for j in range(len(a)):
        for body in (int(a[j]), int(b[j])):
            incident.setdefault(body, []).append(j)
    for body, js in incident.items():
        cols = [int(color[j]) for j in js]
        assert len(cols) == len(set(cols)), f"body {body} has same-color constraints"
    np.testing.assert_array_equal(color, O.color_constraints(n_bodies, a, b))


# ------------------------------------------------------------ tests/test_solver_6dof.py
def test_6dof_free_fall():
    s = Solver6DOF(dt=1 / 60, substeps=10, iterations=1, device=DEVICE, floor_y=-100.0)
    s.add_box((0, 0, 0), (0.2, 0.2, 0.2), mass=1.0)
    for _ in range(60):
        s.step()
    assert abs(s.positions()[0, 1] - 0.5 * -9.81) < 0.05
    assert abs(s.velocities()[0, 1] - (-9.81)) < 0.05


def test_box_rests_on_floor():
    s = Solver6DOF(dt=1 / 60, substeps=15, iterations=1, device=DEVICE, floor_y=0.0, friction=0.6)
    s.add_box((0, 1.0, 0), (0.2, 0.2, 0.2), mass=1.0)
    for _ in range(180):
        s.step()
    p = s.positions()[0]
    q = s.orientations()[0]
    assert abs(p[1] - 0.2) < 2e-3
    assert abs(s.velocities()[0, 1]) < 1e-2
    assert abs(abs(q[3]) - 1.0) < 1e-2


def test_spin_conservation():
    s = Solver6DOF(dt=1 / 60, substeps=10, iterations=1, device=DEVICE, gravity=(0, 0, 0), floor_y=-100.0)
    s.add_box((0, 0, 0), (0.2, 0.1, 0.3), mass=1.0)
    om = s.omega.numpy().copy()
    om[0] = [0, 5.0, 0]
    s.omega = om
    for _ in range(120):
        s.step()
    w = s.omega.numpy()[0]
    assert abs(w[1] - 5.0) < 0.5
    assert np.linalg.norm(w[[0, 2]]) < 0.5


@pytest.mark.parametrize("n", [3, 5])
def test_stack_settles_no_penetration(n):
    s = Solver6DOF(dt=1 / 60, substeps=20, iterations=1, device=DEVICE, floor_y=0.0, friction=0.6)
    h = 0.2
    for k in range(n):
        s.add_box((0, h + k * (2 * h + 0.02), 0), (h, h, h), mass=1.0)
    for _ in range(350):
        s.step()
    ys = np.sort(s.positions()[:, 1])
    assert np.all(np.isfinite(s.positions()))
    assert ys.max() < n * (2 * h) + 0.2
    assert np.allclose(np.diff(ys), 2 * h, atol=8e-3)
    assert np.abs(s.velocities()).max() < 0.1


def test_pile_stable():
    s = Solver6DOF(dt=1 / 60, substeps=18, iterations=1, device=DEVICE, floor_y=0.0, friction=0.6)
    h = 0.16
    rng = np.random.default_rng(0)
    for ly in range(3):
        for ix in range(3):
            for iz in range(3):
                s.add_box((ix * 0.34 + rng.uniform(-2e-3, 2e-3), h + ly * 0.34,
                           iz * 0.34 + rng.uniform(-2e-3, 2e-3)), (h, h, h), mass=1.0)
    for _ in range(400):
        s.step()
    p = s.positions()
    assert np.all(np.isfinite(p))
    assert p[:, 1].max() < 1.2
    assert np.abs(s.velocities()).max() < 0.2


def test_box_tips_and_rests_flat():
    s = Solver6DOF(dt=1 / 60, substeps=20, iterations=1, device=DEVICE, floor_y=0.0, friction=0.7)
    hw, hh, hd = 0.05, 0.25, 0.12
    s.add_box((0, hh, 0), (hw, hh, hd), mass=1.0)
    om = s.omega.numpy().copy()
    om[0] = [0, 0, -3.0]
    s.omega = om
    for _ in range(300):
        s.step()
    p = s.positions()[0]
    assert abs(p[1] - hw) < 0.03
    assert np.linalg.norm(s.omega.numpy()[0]) < 0.2


def test_broadphases_agree():
    def run(bp):
        s = Solver6DOF(dt=1 / 60, substeps=20, iterations=1, device=DEVICE, floor_y=0.0, friction=0.6,
                       broadphase=bp)
        h = 0.2
        for k in range(4):
            s.add_box((0, h + k * (2 * h + 0.02), 0), (h, h, h), mass=1.0)
        for _ in range(300):
            s.step()
        return np.sort(s.positions()[:, 1])
    ref = run("lbvh")
    assert np.allclose(run("grid"), ref, atol=5e-3)
    assert np.allclose(run("hashgrid"), ref, atol=5e-3)


def test_joint_rigid_link():
    s = Solver6DOF(dt=1 / 60, substeps=20, iterations=2, device=DEVICE, floor_y=-100.0)
    anchor = s.add_box((0, 2, 0), (0.05, 0.05, 0.05), mass=0.0, static=True)
    bob = s.add_box((0.6, 2, 0), (0.1, 0.1, 0.1), mass=1.0)
    s.add_joint(anchor, bob, compliance=0.0)
    for _ in range(300):
        s.step()
    p = s.positions()
    assert np.all(np.isfinite(p))
    assert abs(np.linalg.norm(p[bob.index] - p[anchor.index]) - 0.6) < 0.02
    assert p[bob.index, 1] < p[anchor.index, 1]


def test_particle_rests_on_floor():
    s = Solver6DOF(dt=1 / 60, substeps=15, iterations=1, device=DEVICE, floor_y=0.0, friction=0.5)
    r = 0.05
    s.add_particle((0, 1.0, 0), mass=0.1, radius=r)
    for _ in range(200):
        s.step()
    p = s.positions()[0]
    assert abs(p[1] - r) < 5e-3
    assert abs(s.velocities()[0, 1]) < 1e-2


def test_cloth_hangs_from_pins():
    s = Solver6DOF(dt=1 / 60, substeps=15, iterations=2, device=DEVICE, floor_y=-100.0)
    R, sp = 8, 0.1
    idx = np.empty((R, R), np.int64)
    for iy in range(R):
        for ix in range(R):
            pinned = iy == 0
            b = s.add_particle((ix * sp, 2.0, iy * sp), mass=0.0 if pinned else 0.02, radius=0.01, group=1,
                               static=pinned)
            idx[iy, ix] = b.index
    for iy in range(R):
        for ix in range(R):
            if ix + 1 < R:
                s.add_joint(int(idx[iy, ix]), int(idx[iy, ix + 1]), compliance=1e-7)
            if iy + 1 < R:
                s.add_joint(int(idx[iy, ix]), int(idx[iy + 1, ix]), compliance=1e-7)
    for _ in range(250):
        s.step()
    P = s.positions()
    assert np.all(np.isfinite(P))
    assert abs(P[idx[0]][:, 1].mean() - 2.0) < 1e-3
    assert P[idx[R - 1]][:, 1].mean() < 1.85
    assert abs(np.linalg.norm(P[idx[4, 1]] - P[idx[4, 0]]) - sp) < 0.02


def test_unified_rigid_cloth_joints():
    s = Solver6DOF(dt=1 / 60, substeps=18, iterations=2, device=DEVICE, floor_y=0.0, friction=0.6, lin_damp=0.01)
    for k in range(3):
        s.add_box((0, 0.2 + k * 0.42, 0), (0.2, 0.2, 0.2), mass=1.0)
    R, sp = 6, 0.12
    idx = np.empty((R, R), np.int64)
    for iy in range(R):
        for ix in range(R):
            pinned = iy == 0
            b = s.add_particle((1.5 + ix * sp, 1.5, iy * sp), mass=0.0 if pinned else 0.02, radius=0.01,
                               group=1, static=pinned)
            idx[iy, ix] = b.index
    for iy in range(R):
        for ix in range(R):
            if ix + 1 < R:
                s.add_joint(int(idx[iy, ix]), int(idx[iy, ix + 1]), compliance=1e-6)
            if iy + 1 < R:
                s.add_joint(int(idx[iy, ix]), int(idx[iy + 1, ix]), compliance=1e-6)
    assert s.num_joints > 0
    for _ in range(300):
        s.step()
    P = s.positions()
    assert np.all(np.isfinite(P))
    ys = np.sort(P[:3, 1])
    assert np.allclose(np.diff(ys), 0.4, atol=1e-2)
    assert np.abs(s.velocities()).max() < 1.0


def test_domino_cascade():
    s = Solver6DOF(dt=1 / 60, substeps=20, iterations=1, device=DEVICE, floor_y=0.0, friction=0.6)
    hw, hh, hd = 0.04, 0.22, 0.12
    sp = 0.18
    n = 6
    ang = -0.45
    q0 = (0.0, 0.0, math.sin(ang / 2), math.cos(ang / 2))
    for k in range(n):
        q = q0 if k == 0 else (0, 0, 0, 1)
        y = hh * 0.9 if k == 0 else hh
        s.add_box((k * sp, y, 0.0), (hw, hh, hd), mass=1.0, quaternion=q)
    for _ in range(420):
        s.step()
    fell = int(np.sum(s.positions()[:, 1] < hh * 0.6))
    assert fell >= n - 1

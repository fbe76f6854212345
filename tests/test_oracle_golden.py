"""Pins the CPU oracle against the golden fixtures, which were recorded by
running the reference package's own code (src/xpbd3d) through a sequential CPU
stand-in for Warp (``tests/golden/make_golden.py``).  The oracle and the
recorded reference agree bit for bit: same fp32 operations in the same order,
Jacobi accumulation in thread order."""

import numpy as np
import pytest

from oracle import oracle as O
from golden_scenes import fixtures3, fixtures6, kwargs
from xpbd_b200 import scenes


@pytest.mark.parametrize("name,build,frames", fixtures3(), ids=[f[0] for f in fixtures3()])
def test_oracle3_matches_reference(golden, name, build, frames):
    g = golden(name)
    s = O.OracleSolver(device="cpu", **kwargs(g))
    build(s)
    np.testing.assert_array_equal(s.positions(), g["x0"])
    off = 0
    for f in range(frames):
        s.step()
        np.testing.assert_array_equal(s.positions(), g["x"][f])
        np.testing.assert_array_equal(s.velocities(), g["v"][f])
        m = int(g["rows_per_frame"][f])
        np.testing.assert_array_equal(s.lambdas(), g["lam"][off:off + m])
        # contact rows (type, endpoints, rest, mu) in the reference's order
        np.testing.assert_array_equal(s.r_type, g["r_type"][off:off + m])
        np.testing.assert_array_equal(s.r_a, g["r_a"][off:off + m])
        np.testing.assert_array_equal(s.r_b, g["r_b"][off:off + m])
        np.testing.assert_array_equal(s.r_rest, g["r_rest"][off:off + m])
        np.testing.assert_array_equal(s.r_mu, g["r_mu"][off:off + m])
        off += m
    assert s.num_colors == int(g["num_colors"])


@pytest.mark.parametrize("name,build,frames", fixtures6(), ids=[f[0] for f in fixtures6()])
def test_oracle6_matches_reference(golden, name, build, frames):
    g = golden(name)
    s = O.OracleSolver6DOF(device="cpu", **kwargs(g))
    build(s)
    s._flush()
    np.testing.assert_array_equal(s.positions(), g["x0"])
    off = 0
    for f in range(frames):
        s.step()
        np.testing.assert_array_equal(s.positions(), g["x"][f])
        np.testing.assert_array_equal(s.orientations(), g["q"][f])
        np.testing.assert_array_equal(s.velocities(), g["v"][f])
        np.testing.assert_array_equal(s.omega, g["w"][f])
        np.testing.assert_array_equal(s.lam_floor, g["lam_floor"][f])
        assert s.n_pairs == int(g["n_pairs"][f])
        k = s.n_pairs
        np.testing.assert_array_equal(np.stack([s.pair_a[:k], s.pair_b[:k]], 1), g["pairs"][off:off + k])
        off += k


@pytest.mark.parametrize("name", ["coloring_cloth32"] + [f"coloring_rand{i}" for i in range(4)])
def test_oracle_coloring_matches_reference(golden, name):
    g = golden(name)
    col = O.color_constraints(int(g["n_bodies"]), g["a"], g["b"])
    np.testing.assert_array_equal(col, g["color"])
    order, starts, k = O.color_ranges(col)
    np.testing.assert_array_equal(order, g["order"])
    np.testing.assert_array_equal(starts, g["starts"])


def test_oracle_coloring_valid_random():
    """tests/test_solver.py:122-138: same-color rows share no body."""
    rng = np.random.default_rng(0)
    n_bodies = 40
    a = rng.integers(0, n_bodies, 200)
    b = rng.integers(0, n_bodies, 200)
    b = np.where(b == a, (b + 1) % n_bodies, b)
    color = O.color_constraints(n_bodies, a, b)
    incident = {}
    for j in range(len(a)):
        for body in (int(a[j]), int(b[j])):
            incident.setdefault(body, []).append(int(color[j]))
    for cols in incident.values():
        assert len(cols) == len(set(cols))


def test_oracle_sphere_contacts_2048(golden):
    g = golden("sphere_contacts_2048")
    s = O.OracleSolver(device="cpu", solve_mode="jacobi", substeps=15, iterations=2)
    scenes.build_sphere_pile(s)
    s._flush()
    np.testing.assert_array_equal(s.positions(), g["x0"])
    s._rebuild_contacts()
    rows = [r for r in s._rows if r.type == O.CONTACT]
    np.testing.assert_array_equal([r.body_a for r in rows], g["a"])
    np.testing.assert_array_equal([r.body_b for r in rows], g["b"])
    np.testing.assert_array_equal(np.float32([r.rest for r in rows]), g["rest"])
    np.testing.assert_array_equal(np.float32([r.mu for r in rows]), g["mu"])


@pytest.mark.parametrize("bp", ["lbvh", "hashgrid", "grid"])
def test_oracle_pairs_1440(golden, bp):
    g = golden(f"pairs1440_{bp}")
    s = O.OracleSolver6DOF(device="cpu", substeps=15, iterations=2, floor_y=0.0, friction=0.6,
                           restitution=0.2, broadphase=bp)
    scenes.build_box_pile(s)
    s._flush()
    cnt = s._broadphase()
    np.testing.assert_array_equal(s.pair_a[:cnt], g["a"])
    np.testing.assert_array_equal(s.pair_b[:cnt], g["b"])
    if bp == "lbvh":
        np.testing.assert_array_equal(s.lowers, g["lowers"])
        np.testing.assert_array_equal(s.uppers, g["uppers"])
        np.testing.assert_array_equal(s.inv_I, g["inv_I"])
        half = np.zeros_like(s.he)
        O.lib().or6_world_aabb_half(s.num_bodies, O.fp(s.q), O.fp(s.he), O.fp(half))
        np.testing.assert_array_equal(half, g["aabb_half"])


def test_oracle_manifold_kernel(golden):
    g = golden("manifold_kernel")
    n_pairs = len(g["pair_a"])
    x, q, he = g["x"], g["q"], g["he"]
    for p in range(n_pairs):
        cnt = np.zeros(1, np.int32); inc = np.zeros(1, np.int32); ref = np.zeros(1, np.int32)
        nrm = np.zeros(3, np.float32)
        oi = np.zeros((8, 3), np.float32); orf = np.zeros((8, 3), np.float32)
        O.lib().or6_manifold_pair(O.fp(x), O.fp(q), O.fp(he), int(g["pair_a"][p]), int(g["pair_b"][p]),
                                  O.C.c_float(float(g["margin"])), O.ip(cnt), O.ip(inc), O.ip(ref),
                                  O.fp(nrm), O.fp(oi), O.fp(orf))
        k = int(cnt[0])
        assert k == g["m_count"][p]
        if k:
            assert inc[0] == g["m_inc"][p] and ref[0] == g["m_ref"][p]
            np.testing.assert_array_equal(nrm, g["m_normal"][p])
            np.testing.assert_array_equal(oi[:k], g["m_off_inc"][8 * p:8 * p + k])
            np.testing.assert_array_equal(orf[:k], g["m_off_ref"][8 * p:8 * p + k])

"""One substep on identical state at the benchmark sizes: the 2048-sphere pile
at its contact-richest frame of the first 60 (while it lands) and the 1440-box
pile after 100 frames.

The settled state comes from the engine.  Then an engine and an oracle solver
with one substep per frame (dt = h = 1/900 s, the same 2 iterations) are both
seeded with it, and one frame of each is compared: the contact rows (spheres)
or candidate pairs (boxes) bit for bit, positions and orientations within
1e-5 m, and every multiplier within 1e-4 relative (spheres: of the row's own
multiplier; boxes: of the largest multiplier of its kind, as the floor solve
assigns rather than accumulates).  This repeats for three consecutive
substeps, the oracle re-seeded from the engine before each."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle import oracle as O  # noqa: E402
from xpbd_b200 import Solver, Solver6DOF, scenes  # noqa: E402

H = 1.0 / 900.0


def _seed3(eng, orc, x, v):
    T = eng.tensors
    T["x"][:, :3] = torch.from_numpy(x).to(T["x"].device)
    T["v"][:, :3] = torch.from_numpy(v).to(T["v"].device)
    orc._flush()
    orc.x[:] = x
    orc.v[:] = v


def test_one_substep_sphere_pile_2048_settled():
    settle = Solver(device="cuda:0", dt=1 / 60, substeps=15, iterations=2, solve_mode="jacobi")
    scenes.build_sphere_pile(settle)
    # The pile lands after about 0.4 s and then spreads out over the floor (an
    # averaged-Jacobi stack of spheres does not stand), so its contact count
    # peaks while it lands: take the contact-richest of the first 60 frames.
    best = (-1, None, None)
    for _ in range(60):
        settle.step()
        n_c = settle.num_constraints - settle.num_bodies
        if n_c > best[0]:
            best = (n_c, settle.positions(), settle.velocities())
    _, x, v = best
    kw = dict(dt=H, substeps=1, iterations=2, solve_mode="jacobi")
    eng = Solver(device="cuda:0", **kw)
    orc = O.OracleSolver(device="cpu", **kw)
    # a 5 mm contact margin: every pair of resting neighbours gets a row (the
    # settled spheres touch within float rounding, so without a margin only the
    # pairs that happen to overlap do)
    scenes.build_sphere_pile(eng, margin=0.005)
    scenes.build_sphere_pile(orc, margin=0.005)
    eng._flush()
    _seed3(eng, orc, x, v)
    for k in range(3):
        if k:
            orc.x[:] = eng.positions()
            orc.v[:] = eng.velocities()
        eng.step()
        orc.step()
        rows = eng.rows()
        m = len(orc._rows)
        assert len(rows["type"]) == m
        n_contacts = int((rows["type"] == 3).sum())
        assert n_contacts > 2000, n_contacts  # a settled, contact-rich pile
        np.testing.assert_array_equal(rows["type"], orc.r_type)
        np.testing.assert_array_equal(rows["a"], orc.r_a)
        np.testing.assert_array_equal(rows["b"], orc.r_b)
        np.testing.assert_array_equal(rows["rest"], orc.r_rest)
        np.testing.assert_array_equal(rows["mu"], orc.r_mu)
        dx = np.abs(eng.positions() - orc.positions()).max()
        assert dx <= 1e-5, (k, dx)
        lam_e, lam_o = eng.lambdas(), orc.lambdas()
        err = np.abs(lam_e - lam_o)
        assert np.all(err <= 1e-4 * np.abs(lam_o) + 1e-7), (k, float(err.max()))


@pytest.mark.parametrize("lanes", [8, 1])
def test_one_substep_box_pile_1440_settled(lanes):
    kw15 = dict(dt=1 / 60, substeps=15, iterations=2, floor_y=0.0, friction=0.6, restitution=0.2,
                broadphase="lbvh")
    settle = Solver6DOF(device="cuda:0", **kw15)
    scenes.build_box_pile(settle)
    settle.sync_pairs = False
    for _ in range(100):
        settle.step()
    x, q, v, w = settle.positions(), settle.orientations(), settle.velocities(), settle.omega.numpy()
    kw = dict(kw15, dt=H, substeps=1)
    eng = Solver6DOF(device="cuda:0", **kw)
    orc = O.OracleSolver6DOF(device="cpu", **kw)
    scenes.build_box_pile(eng)
    scenes.build_box_pile(orc)
    eng.lanes = lanes
    eng._flush()
    orc._flush()
    T = eng.tensors
    n = eng.num_bodies
    for k in range(3):
        if k:
            x, q, v, w = eng.positions(), eng.orientations(), eng.velocities(), eng.omega.numpy()
        T["x"][:, :3] = torch.from_numpy(x).to(T["x"].device)
        T["q"][:] = torch.from_numpy(q).to(T["q"].device)
        T["v"][:, :3] = torch.from_numpy(v).to(T["v"].device)
        T["w"][:, :3] = torch.from_numpy(w).to(T["w"].device)
        orc.x[:], orc.q[:], orc.v[:], orc.omega[:] = x, q, v, w
        eng.step()
        orc.step()
        n_pairs = orc.n_pairs
        assert eng.n_pairs == n_pairs and n_pairs > 2000, (eng.n_pairs, n_pairs)
        np.testing.assert_array_equal(eng.pairs(), np.stack([orc.pair_a[:n_pairs], orc.pair_b[:n_pairs]], 1))
        hdr = T["m_hdr"][:n_pairs].cpu().numpy()
        np.testing.assert_array_equal(hdr[:, 0], orc.m_count[:n_pairs])
        assert int(hdr[:, 0].sum()) > 1000
        dx = np.abs(eng.positions() - orc.positions()).max()
        dq = np.abs(eng.orientations() - orc.orientations()).max()
        assert dx <= 1e-5 and dq <= 1e-5, (k, dx, dq)
        for got, want in ((T["lam_floor"][: 8 * n], orc.lam_floor[: 8 * n]),
                          (T["lam_pair"][: 8 * n_pairs], orc.lam_pair[: 8 * n_pairs])):
            got = got.cpu().numpy()
            scale = max(float(np.abs(want).max()), 1e-12)
            assert np.abs(got - want).max() <= 1e-4 * scale, (k, float(np.abs(got - want).max()), scale)

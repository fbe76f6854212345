"""The threaded CPU frames (OpenMP) that the benchmark times as the CPU
baseline: Gauss-Seidel and the pair emission are bit-identical to the
sequential oracle; Jacobi and the 6-DOF frame, whose sums round in another
order, agree to float rounding."""

import numpy as np

from oracle import oracle as O
from xpbd_b200 import scenes


def _pair3(mode, build, threads=4):
    kw = dict(dt=1 / 60, substeps=15, iterations=2, solve_mode=mode)
    a, b = O.OracleSolver(**kw), O.OracleSolver(**kw)
    build(a)
    build(b)
    b.threads = threads
    return a, b


def test_gs_cloth_threads_bit_identical():
    a, b = _pair3("gs", lambda s: scenes.build_cloth(s, res=20, y=0.01, velocity=(0.1, -0.5, 0.0)))
    for _ in range(3):
        a.step()
        b.step()
    np.testing.assert_array_equal(a.positions(), b.positions())
    np.testing.assert_array_equal(a.lambdas(), b.lambdas())


def test_jacobi_sphere_pile_threads_close():
    a, b = _pair3("jacobi", lambda s: scenes.build_sphere_pile(s, nx=8, ny=4, nz=8, pitch=0.098, y0=0.06))
    a.step()
    b.step()
    assert np.abs(a.positions() - b.positions()).max() <= 1e-5
    assert len(a._rows) == len(b._rows)


def test_box_pile_threads_close_and_pairs_identical():
    # one substep per frame: over a whole frame of this overlapping pile the
    # rounding difference can move a contact across a threshold (see the
    # engine's one-substep parity tests)
    kw = dict(dt=1 / 900, substeps=1, iterations=2, floor_y=0.0, friction=0.6, restitution=0.2, broadphase="lbvh")
    a, b = O.OracleSolver6DOF(**kw), O.OracleSolver6DOF(**kw)
    for s in (a, b):
        scenes.build_box_pile(s, nx=5, ny=3, nz=5, pitch=0.45, y0=0.35)
    b.threads = 3
    a.step()
    b.step()
    assert a.n_pairs == b.n_pairs > 0
    np.testing.assert_array_equal(a.pair_a[:a.n_pairs], b.pair_a[:b.n_pairs])
    np.testing.assert_array_equal(a.pair_b[:a.n_pairs], b.pair_b[:b.n_pairs])
    # the manifolds of later substeps see positions that differ by rounding
    assert a.frame_points > 0 and abs(a.frame_points - b.frame_points) <= 0.01 * a.frame_points
    assert np.abs(a.positions() - b.positions()).max() <= 1e-5
    assert np.abs(a.orientations() - b.orientations()).max() <= 1e-5

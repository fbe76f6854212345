"""Max constraint residual after 120 frames, engine against the oracle, on the
full-size benchmark scenes: the 32x32 cloth (Gauss-Seidel and Jacobi), the
2048-sphere pile and the 1440-box pile.  The residual is hard rows max(0, -C),
compliant rows |C + alpha~ lambda|, evaluated on the state after the last
substep.  The two must agree within 5 %.

The cloths run free for all 120 frames.  The piles are chaotic at the
millimetre level over 120 frames (float-atomic rounding moves contacts across
their thresholds, see test_gpu_solver6), and their per-frame max residual
swings by 2-10x from one frame to the next, so one free-running pair of runs
measures the chaos, not the solver.  The piles are therefore checked three
ways:
* after 119 free frames the oracle is seeded with the engine's state, and the
  residual of frame 120, computed from that identical state, agrees within 5 %;
* free running, every frame agrees within 5 % until the trajectories part
  (measured on 16 seeds: the first 5 % departure comes at frame 4-11 for the
  sphere pile and 8-37 for the box pile), checked on the first frames;
* statistically: the per-frame max residual over frames 60-120, pooled over
  many seeds (sphere pile 24, box pile 16), has the same mean on the engine as
  on the oracle.  Measured on 16 seeds the ratio was 0.996 (spheres) and 1.000
  (boxes), while a single seed's ratio ranges 0.33-3.4 (spheres) and 0.78-1.2
  (boxes); halves of 8 seeds deviated by up to 6.7 % and 3.3 %.  The bounds are
  15 % (spheres) and 8 % (boxes)."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle import oracle as O  # noqa: E402
from xpbd_b200 import Solver, Solver6DOF, scenes  # noqa: E402

FRAMES = 120


def _cloth(mode):
    kw = dict(dt=1 / 60, substeps=15, iterations=2, solve_mode=mode)
    return Solver, O.OracleSolver, kw, scenes.build_cloth


CASES = {
    "cloth_gs": _cloth("gs"),
    "cloth_jacobi": _cloth("jacobi"),
    "spheres": (Solver, O.OracleSolver, dict(dt=1 / 60, substeps=15, iterations=2, solve_mode="jacobi"),
                scenes.build_sphere_pile),
    "boxes": (Solver6DOF, O.OracleSolver6DOF, dict(dt=1 / 60, substeps=15, iterations=2, floor_y=0.0, friction=0.6,
                                                   restitution=0.2, broadphase="lbvh"), scenes.build_box_pile),
}


@pytest.mark.parametrize("name", list(CASES))
def test_residual_after_120_frames(name):
    cls, ocls, kw, build = CASES[name]
    eng = cls(device="cuda:0", **kw)
    orc = ocls(device="cpu", **kw)
    build(eng)
    build(orc)
    for _ in range(FRAMES - 1):
        eng.step()
        orc.step()
    if name in ("spheres", "boxes"):
        orc.x[:] = eng.positions()
        orc.v[:] = eng.velocities()
        if name == "boxes":
            orc.q[:] = eng.orientations()
            orc.omega[:] = eng.omega.numpy()
    eng.step()
    orc.step()
    r_eng = float(np.max(eng.residual()))
    r_orc = float(orc.residual())
    assert np.isfinite(r_eng) and np.isfinite(r_orc)
    assert abs(r_eng - r_orc) <= 0.05 * max(r_orc, 1e-6), (r_eng, r_orc)


STAT_SEEDS = {"spheres": 24, "boxes": 16}
STAT_BOUND = {"spheres": 0.15, "boxes": 0.08}
EARLY_FRAMES = {"spheres": 3, "boxes": 7}  # free-running frames compared one by one


@pytest.mark.parametrize("name", ["spheres", "boxes"])
def test_pile_residual_statistics_over_seeds(name):
    cls, ocls, kw, build = CASES[name]
    eng_all, orc_all = [], []
    for seed in range(STAT_SEEDS[name]):
        eng = cls(device="cuda:0", **kw)
        orc = ocls(device="cpu", **kw)
        build(eng, seed=seed)
        build(orc, seed=seed)
        for f in range(FRAMES):
            eng.step()
            orc.step()
            if f < EARLY_FRAMES[name] or f >= 59:
                r_eng = float(np.max(eng.residual()))
                r_orc = float(orc.residual())
                assert np.isfinite(r_eng) and np.isfinite(r_orc)
                if f < EARLY_FRAMES[name]:  # the trajectories have not parted yet
                    assert abs(r_eng - r_orc) <= 0.05 * max(r_orc, 1e-6), (seed, f, r_eng, r_orc)
                else:
                    eng_all.append(r_eng)
                    orc_all.append(r_orc)
    ratio = float(np.mean(eng_all) / np.mean(orc_all))
    assert abs(ratio - 1.0) <= STAT_BOUND[name], ratio


@pytest.mark.parametrize("six", [False, True], ids=["3dof", "6dof"])
def test_residual_reports_a_non_finite_state_as_infinite(six):
    """A state that blew up (one body's position NaN) must not read as a small
    residual: a NaN constraint value fails the hard rows' C < 0 test and a
    maximum with fmaxf drops NaN operands, so the residual kernels map every
    non-finite row to +inf.  The warm-start fallback relies on it."""
    if six:
        s = Solver6DOF(device="cuda:0", dt=1 / 60, substeps=15, iterations=2, floor_y=0.0)
        scenes.build_box_pile(s, nx=3, ny=2, nz=3)
    else:
        s = Solver(device="cuda:0", dt=1 / 60, substeps=15, iterations=2, solve_mode="jacobi")
        scenes.build_cloth(s, res=8)
    s.step()
    assert np.all(np.isfinite(s.residual()))
    s.tensors["x"][2, 1] = float("nan")
    r = s.residual()
    assert np.isinf(r[0]) and r[0] > 0, r

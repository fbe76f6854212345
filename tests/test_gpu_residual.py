"""Max constraint residual after 120 frames, engine against the oracle, on the
full-size benchmark scenes: the 32x32 cloth (Gauss-Seidel and Jacobi), the
2048-sphere pile and the 1440-box pile.  The residual is hard rows max(0, -C),
compliant rows |C + alpha~ lambda|, evaluated on the state after the last
substep.  The two must agree within 5 %.

The cloths run free for all 120 frames.  The piles are chaotic at the
millimetre level over 120 frames (float-atomic rounding moves contacts across
their thresholds, see test_gpu_solver6), and their per-frame max residual
swings by 2-10x from one frame to the next, so a free-running comparison would
measure the chaos, not the solver: after 119 free frames the oracle is seeded
with the engine's state and the residual of frame 120, computed from that
identical state, is compared."""

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

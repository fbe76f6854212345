"""Measurement hooks of the benchmark, on the GPU: the phase latency probe
(xpbd_phase_floor), the per-frame phase counts of the frame kernels
(xpbd3_phases / xpbd6_phases) and the device count of manifold points per
substep (xpbd6_points) that the 6-DOF projection count uses."""

import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from xpbd_b200 import Solver, Solver6DOF, scenes  # noqa: E402
from xpbd_b200 import _native as N  # noqa: E402
from xpbd_b200.solver_6dof import lib6  # noqa: E402


@pytest.mark.parametrize("mode,blocks,threads", [(0, 296, 256), (1, 1, 1024), (2, 16, 256)])
def test_phase_floor_probe(mode, blocks, threads):
    ns = C.c_float(0.0)
    N.check(N.lib().xpbd_phase_floor(mode, blocks, threads, 500, C.byref(ns), N.stream_of("cuda:0")),
            "xpbd_phase_floor")
    # a barrier plus one dependent L2 round trip: well above 50 ns, well below 50 us
    assert 50.0 < ns.value < 50000.0, ns.value


def test_phase_floor_rejects_bad_shapes():
    ns = C.c_float(0.0)
    sp = N.stream_of("cuda:0")
    L = N.lib()
    assert L.xpbd_phase_floor(2, 17, 256, 10, C.byref(ns), sp) == N.XPBD_ERR_BAD_ARG
    assert L.xpbd_phase_floor(1, 2, 256, 10, C.byref(ns), sp) == N.XPBD_ERR_BAD_ARG
    assert L.xpbd_phase_floor(0, 4, 100, 10, C.byref(ns), sp) == N.XPBD_ERR_BAD_ARG
    assert L.xpbd_phase_floor(0, 1 << 20, 256, 10, C.byref(ns), sp) == N.XPBD_ERR_BAD_ARG


def test_phase_counts_of_the_frame_kernels():
    s = Solver(device="cuda:0", dt=1 / 60, substeps=15, iterations=2, solve_mode="jacobi")
    scenes.build_sphere_pile(s)
    s.set_driver(2, 16, 256)
    s.sync_contacts = False
    s.step()
    # folded Jacobi with the folded substep boundary: I barriers per substep and a closing pass
    assert s.phases() == (30, 31)
    c = Solver(device="cuda:0", dt=1 / 60, substeps=15, iterations=2, solve_mode="gs")
    scenes.build_cloth(c)
    c.set_driver(1, 1, 1024)
    c.step()
    assert c.phases() == (1 + 15 * (1 + 2 * c.num_colors),) * 2
    b = Solver6DOF(device="cuda:0", dt=1 / 60, substeps=15, iterations=2)
    scenes.build_box_pile(b, nx=3, ny=2, nz=3)
    b.step()
    # the integrate pass + 7 per substep, for both lane widths
    assert b.phases() == (1 + 15 * 7,) * 2
    b.lanes = 1
    b.step()
    assert b.phases() == (1 + 15 * 7,) * 2


@pytest.mark.parametrize("lanes", [8, 1])
def test_manifold_point_counter(lanes):
    """One substep per frame: the counter grows by the manifold points the
    substep generated (the headers' counts after the frame)."""
    s = Solver6DOF(device="cuda:0", dt=1 / 900, substeps=1, iterations=2)
    scenes.build_box_pile(s, nx=4, ny=3, nz=4, pitch=0.45)
    s.lanes = lanes
    s.sync_pairs = True
    for _ in range(30):
        s.step()
    s.manifold_points(reset=True)
    total = 0
    for _ in range(5):
        s.step()
        torch.cuda.synchronize()
        npairs = min(s.n_pairs, s.cap)
        total += int(s.tensors["m_hdr"][:npairs, 0].sum().item())
    assert total > 0
    assert s.manifold_points() == total

"""Edge-edge SAT axes in the box manifold (``Solver6DOF(edge_axes=True)``; no
reference counterpart: the reference tests the six face axes only,
kernels_6dof.py:13-15).

Two unit cubes, A turned 45 degrees about z and B 45 degrees about x, so that
A's top edge (along z) crosses B's bottom edge (along x).  Every face axis
overlaps whether or not the edges touch; only the edge-edge axis y tells.
"""

import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from xpbd_b200 import Solver6DOF, scenes  # noqa: E402

H = 0.5
R2 = math.sqrt(2.0) * H  # half diagonal of a face: the edges' distance from the centre
QA = (0.0, 0.0, math.sin(math.pi / 8), math.cos(math.pi / 8))  # 45 degrees about z
QB = (math.sin(math.pi / 8), 0.0, 0.0, math.cos(math.pi / 8))  # 45 degrees about x


def _rot(q):
    x, y, z, w = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def _crossing_edges(gap, edge_axes, lanes=8):
    """One manifold generation (one substep, no iterations, no gravity) for the
    two cubes with their edges `gap` apart (negative: penetrating)."""
    s = Solver6DOF(device="cuda:0", substeps=1, iterations=0, gravity=(0.0, 0.0, 0.0), edge_axes=edge_axes)
    s.lanes = lanes
    s.add_box((0.0, 0.0, 0.0), (H, H, H), 1.0, quaternion=QA)
    s.add_box((0.0, 2 * R2 + gap, 0.0), (H, H, H), 1.0, quaternion=QB)
    s.step()
    assert s.status() == 0
    assert s.n_pairs == 1
    T = s.tensors
    hdr = T["m_hdr"][0].cpu().numpy()
    normal = T["m_normal"][0, :3].cpu().numpy()
    x = s.positions()
    depths = []
    for c in range(hdr[0]):
        inc, ref = hdr[1], hdr[2]
        p_inc = x[inc] + _rot(s.orientations()[inc]) @ T["m_off_inc"][c, :3].cpu().numpy()
        p_ref = x[ref] + _rot(s.orientations()[ref]) @ T["m_off_ref"][c, :3].cpu().numpy()
        depths.append(float(np.dot(p_inc - p_ref, normal)))
    return hdr, normal, depths


def _face_overlaps(gap):
    """The six face-axis overlaps of the configuration (all positive here)."""
    RA, RB = _rot(QA), _rot(QB)
    d = np.array([0.0, -(2 * R2 + gap), 0.0])
    out = []
    for R0, R1 in ((RA, RB), (RB, RA)):
        for k in range(3):
            L = R0[:, k]
            out.append(H + sum(H * abs(L @ R1[:, m]) for m in range(3)) - abs(L @ d))
    return np.array(out)


@pytest.mark.parametrize("lanes", [8, 1])
def test_separated_edges_have_no_contact(lanes):
    """1 cm apart: no face axis separates the cubes, the edge axis y does."""
    gap = 0.01
    assert np.all(_face_overlaps(gap) > 0.3)
    hdr, _, _ = _crossing_edges(gap, edge_axes=True, lanes=lanes)
    assert hdr[0] == 0


@pytest.mark.parametrize("lanes", [8, 1])
def test_penetrating_edges_get_one_edge_point(lanes):
    gap = -0.01
    hdr_ref, normal_ref, _ = _crossing_edges(gap, edge_axes=False, lanes=lanes)
    assert abs(normal_ref[1]) < 0.99  # the face manifold's normal is tilted 45 degrees
    hdr, normal, depths = _crossing_edges(gap, edge_axes=True, lanes=lanes)
    assert hdr[0] == 1 and hdr[1] == 0 and hdr[2] == 1  # incident A, reference B
    np.testing.assert_allclose(normal, [0.0, -1.0, 0.0], atol=1e-5)  # from B down to A
    assert abs(depths[0] - gap) <= 1e-5


def test_edge_axes_same_manifolds_for_both_phase_widths():
    """With the flag on, the thread-per-pair and eight-lane manifold phases write
    identical manifolds (one substep of a tumbling pile, same start state)."""
    out = {}
    for lanes in (1, 8):
        s = Solver6DOF(device="cuda:0", substeps=15, iterations=2, restitution=0.2, edge_axes=True)
        s.lanes = lanes
        scenes.build_box_pile(s, nx=5, ny=4, nz=5, pitch=0.6, seed=6)
        s.set_driver(2, 16, 512)
        for _ in range(20):  # identical frames for both until the last substep's rounding
            s.step()
        snap = s.state_dict()
        out[lanes] = (s, snap)
    a, sa = out[1]
    b, _ = out[8]
    b.load_state_dict(sa)  # same state into both
    for s in (a, b):
        s.substeps = 1
        s.invalidate()
        s.step()
    k = a.n_pairs
    assert b.n_pairs == k and k > 0
    ha, hb = a.tensors["m_hdr"][:k].cpu().numpy(), b.tensors["m_hdr"][:k].cpu().numpy()
    np.testing.assert_array_equal(ha, hb)
    live = ha[:, 0] > 0
    assert live.sum() > 3
    np.testing.assert_array_equal(a.tensors["m_normal"][:k].cpu().numpy()[live],
                                  b.tensors["m_normal"][:k].cpu().numpy()[live])
    for name in ("m_off_inc", "m_off_ref"):
        oa = a.tensors[name][: 8 * k].cpu().numpy().reshape(k, 8, 4)
        ob = b.tensors[name][: 8 * k].cpu().numpy().reshape(k, 8, 4)
        for p in np.nonzero(live)[0]:
            np.testing.assert_array_equal(oa[p, : ha[p, 0]], ob[p, : ha[p, 0]])


def test_edge_axes_pile_runs():
    """A pile with the edge axes on steps 60 frames without status bits or
    non-finite positions."""
    s = Solver6DOF(device="cuda:0", substeps=15, iterations=2, restitution=0.2, edge_axes=True)
    scenes.build_box_pile(s, nx=6, ny=5, nz=6, pitch=0.6, seed=7)
    for _ in range(60):
        s.step()
    assert s.status() == 0
    assert np.all(np.isfinite(s.positions()))

"""GPU parity of the 6-DOF engine against the CPU oracle (itself pinned bit-exactly
to the reference's recorded outputs).

Pair lists are compared exactly (LBVH and hash grid: sorted by (a, b); host grid:
the reference's grid emission order).  Body state is compared with tolerances:
position corrections are summed with float atomics in an order that varies
between runs (as in the reference), so x agrees to 1e-5 m after one frame and
drifts slowly after that."""

import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle import oracle as O  # noqa: E402
from golden_scenes import fixtures6, kwargs  # noqa: E402
from xpbd_b200 import Solver6DOF, scenes  # noqa: E402
from xpbd_b200 import _native as N  # noqa: E402
from xpbd_b200.solver_6dof import lib6  # noqa: E402


def _pair(build, **kw):
    eng = Solver6DOF(device="cuda:0", **kw)
    orc = O.OracleSolver6DOF(device="cpu", **kw)
    build(eng)
    build(orc)
    return eng, orc


@pytest.mark.parametrize("name,build,frames", fixtures6(), ids=[f[0] for f in fixtures6()])
def test_frames_match_oracle(golden, name, build, frames):
    kw = kwargs(golden(name))
    eng, orc = _pair(build, **kw)
    for f in range(frames):
        eng.step()
        orc.step()
        k = orc.n_pairs
        assert eng.n_pairs == k, (eng.n_pairs, k)
        np.testing.assert_array_equal(eng.pairs(), np.stack([orc.pair_a[:k], orc.pair_b[:k]], 1))
        tol = 1e-5 * (f + 1) ** 2
        assert np.abs(eng.positions() - orc.positions()).max() <= tol
        assert np.abs(eng.orientations() - orc.orientations()).max() <= 10 * tol
        assert np.abs(eng.velocities() - orc.velocities()).max() <= 900 * tol
        assert np.abs(eng.omega.numpy() - orc.omega).max() <= 9000 * tol


@pytest.mark.parametrize("bp", ["lbvh", "hashgrid", "grid"])
def test_pairs_1440_bit_exact(golden, bp):
    g = golden(f"pairs1440_{bp}")
    s = Solver6DOF(device="cuda:0", substeps=15, iterations=2, floor_y=0.0, friction=0.6, restitution=0.2,
                   broadphase=bp)
    scenes.build_box_pile(s)
    s._flush()
    N.check(lib6().xpbd6_broadphase(s._h, N.stream_of(s.device)))
    p = s.pairs()
    np.testing.assert_array_equal(p[:, 0], g["a"])
    np.testing.assert_array_equal(p[:, 1], g["b"])


def test_body_aabb_and_morton_bit_exact(golden):
    g = golden("pairs1440_lbvh")
    s = Solver6DOF(device="cuda:0", substeps=15, iterations=2, broadphase="lbvh")
    scenes.build_box_pile(s)
    s._flush()
    n = s.num_bodies
    lo = torch.zeros((n, 4), device="cuda")
    hi = torch.zeros((n, 4), device="cuda")
    L = lib6()
    N.check(L.xpbd6_body_aabb(C.byref(s._st), C.byref(s._par), N.ptr(lo), N.ptr(hi), N.stream_of(s.device)))
    np.testing.assert_array_equal(lo[:, :3].cpu().numpy(), g["lowers"])
    np.testing.assert_array_equal(hi[:, :3].cpu().numpy(), g["uppers"])
    codes = np.zeros(n, np.uint32)
    N.check(L.xpbd6_morton(s._h, codes.ctypes.data_as(C.c_void_p), N.stream_of(s.device)))
    np.testing.assert_array_equal(codes, O.morton_codes(g["lowers"], g["uppers"]))


def test_graph_frame_equals_synced_frame():
    def run(sync):
        s = Solver6DOF(device="cuda:0", substeps=10, iterations=2, restitution=0.2)
        scenes.build_box_pile(s, nx=3, ny=3, nz=3, pitch=0.55, seed=3)
        s.sync_pairs = sync
        for _ in range(3):
            s.step()
        assert s.status() == 0
        return s.positions(), s.n_pairs
    a, na = run(True)
    b, nb = run(False)
    assert na == nb
    assert np.abs(a - b).max() <= 1e-4


def test_substep_drivers_agree():
    res = {}
    for drv, want in (((2, 16, 512), "cluster"), ((2, 4, 256), "cluster"), ((0, 0, 256), "grid"),
                      ((0, 1, 256), "grid")):
        s = Solver6DOF(device="cuda:0", substeps=10, iterations=2, restitution=0.2)
        s.set_driver(*drv)
        scenes.build_box_pile(s, nx=4, ny=3, nz=4, pitch=0.55, seed=5)
        assert s.launch_info()["mode"] == want
        for _ in range(3):
            s.step()
        assert s.status() == 0
        res[drv] = s.positions()
    ref = res[(2, 16, 512)]
    for drv, x in res.items():
        assert np.abs(x - ref).max() <= 1e-4, drv


def test_autotune6_matches_oracle():
    kw = dict(substeps=10, iterations=2, restitution=0.2)
    eng, orc = _pair(lambda s: scenes.build_box_pile(s, nx=3, ny=3, nz=3, pitch=0.7, seed=8), **kw)
    rep = eng.autotune(frames=2)
    assert rep["chosen"]["mode"] in ("cluster", "grid")
    eng.step()
    orc.step()
    assert np.abs(eng.positions() - orc.positions()).max() <= 1e-5


def test_pair_capacity_overflow_grows():
    """More candidate pairs than max(64, 4 n): the step grows the capacity and
    re-emits, like the reference, and the physics matches the oracle."""
    kw = dict(substeps=5, iterations=1, restitution=0.0)
    eng, orc = _pair(lambda s: scenes.build_box_pile(s, nx=4, ny=4, nz=4, pitch=0.3, seed=2), **kw)
    eng.step()
    orc.step()
    assert orc.n_pairs > 4 * 64
    assert eng.n_pairs == orc.n_pairs
    assert eng.cap >= eng.n_pairs
    assert np.abs(eng.positions() - orc.positions()).max() <= 1e-4


def test_kernel_entry_points_match_oracle(golden):
    """Manifold generation through the C ABI against the reference's recorded
    manifold of 256 random box pairs."""
    g = golden("manifold_kernel")
    n = len(g["x"])
    s = Solver6DOF(device="cuda:0", substeps=1, iterations=1)
    for i in range(n):
        s.add_box(tuple(g["x"][i]), tuple(g["he"][i]), 1.0, quaternion=tuple(g["q"][i]))
    s._flush()
    T = s.tensors
    npair = len(g["pair_a"])
    if s.cap < npair:
        s._alloc_pairs(npair)
        s._bind()
        T = s.tensors
    T["pairs"][:npair] = torch.from_numpy(np.stack([g["pair_a"], g["pair_b"]], 1)).cuda()
    T["n_pairs"].fill_(npair)
    T["q"].copy_(torch.from_numpy(g["q"]).cuda())
    N.check(lib6().xpbd6_manifold(C.byref(s._st), float(g["margin"]), N.stream_of(s.device)))
    hdr = T["m_hdr"][:npair].cpu().numpy()
    np.testing.assert_array_equal(hdr[:, 0], g["m_count"])
    live = g["m_count"] > 0
    np.testing.assert_array_equal(hdr[live, 1], g["m_inc"][live])
    np.testing.assert_array_equal(hdr[live, 2], g["m_ref"][live])
    np.testing.assert_array_equal(T["m_normal"][:npair, :3].cpu().numpy()[live], g["m_normal"][live])
    oi = T["m_off_inc"][: 8 * npair, :3].cpu().numpy()
    orf = T["m_off_ref"][: 8 * npair, :3].cpu().numpy()
    for p in np.nonzero(live)[0]:
        k = g["m_count"][p]
        np.testing.assert_array_equal(oi[8 * p:8 * p + k], g["m_off_inc"][8 * p:8 * p + k])
        np.testing.assert_array_equal(orf[8 * p:8 * p + k], g["m_off_ref"][8 * p:8 * p + k])

"""GPU parity of the 6-DOF engine against the CPU oracle (itself pinned bit-exactly
to the reference's recorded outputs).

Pair lists are compared exactly (LBVH and hash grid: sorted by (a, b); host grid:
the reference's grid emission order).  Body state is compared with tolerances:
position corrections are summed with float atomics (as in the reference), so x
agrees to about 1e-6 m after one frame.  In the colliding piles that rounding
difference eventually moves a contact across one of its discrete thresholds (a
point's depth crossing zero, a manifold point crossing the margin, a near-tie
between SAT axes) and the trajectories part at the millimetre level: the
reference differs from itself between runs in the same way.  Multi-frame
comparisons on piles therefore re-seed the second solver from the first before
every frame and bound the error one frame adds."""

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


def _reseed_oracle(orc, eng):
    orc.x[:] = eng.positions()
    orc.q[:] = eng.orientations()
    orc.v[:] = eng.velocities()
    orc.omega[:] = eng.omega.numpy()


@pytest.mark.parametrize("lanes", [8, 1])
@pytest.mark.parametrize("name,build,frames", fixtures6(), ids=[f[0] for f in fixtures6()])
def test_frames_match_oracle(golden, name, build, frames, lanes):
    """Stacks, joints and the floor box run free against the oracle; the piles
    re-seed the oracle from the engine before every frame (see module doc)."""
    kw = kwargs(golden(name))
    eng, orc = _pair(build, **kw)
    eng.lanes = lanes
    reseed = name.startswith("pile")
    for f in range(frames):
        if reseed and f:
            _reseed_oracle(orc, eng)
        eng.step()
        orc.step()
        k = orc.n_pairs
        assert eng.n_pairs == k, (eng.n_pairs, k)
        np.testing.assert_array_equal(eng.pairs(), np.stack([orc.pair_a[:k], orc.pair_b[:k]], 1))
        tol = 1e-5 * (1 if reseed else (f + 1) ** 2)
        assert np.abs(eng.positions() - orc.positions()).max() <= tol
        assert np.abs(eng.orientations() - orc.orientations()).max() <= 10 * tol
        assert np.abs(eng.velocities() - orc.velocities()).max() <= 900 * tol
        assert np.abs(eng.omega.numpy() - orc.omega).max() <= 9000 * tol


@pytest.mark.parametrize("lanes", [8, 1])
@pytest.mark.parametrize("name", ["pile_lbvh", "stack", "joints"])
def test_one_substep_positions_and_lambdas(golden, name, lanes):
    """One substep at a time on identical state (the oracle re-seeded from the
    engine before each): positions within 1e-5 m, orientations within 1e-5, and
    the floor, manifold and joint multipliers within 1e-4 of the largest
    multiplier of their kind."""
    build = dict((f[0], f[1]) for f in fixtures6())[name]
    kw = kwargs(golden(name))
    kw["dt"] = kw.get("dt", 1 / 60) / kw["substeps"]
    kw["substeps"] = 1
    eng, orc = _pair(build, **kw)
    eng.lanes = lanes
    for k in range(8):
        if k:
            _reseed_oracle(orc, eng)
        eng.step()
        orc.step()
        n_pairs = orc.n_pairs
        assert eng.n_pairs == n_pairs
        np.testing.assert_array_equal(eng.pairs(), np.stack([orc.pair_a[:n_pairs], orc.pair_b[:n_pairs]], 1))
        assert np.abs(eng.positions() - orc.positions()).max() <= 1e-5
        assert np.abs(eng.orientations() - orc.orientations()).max() <= 1e-5
        T = eng.tensors
        n = eng.num_bodies
        for got, want in ((T["lam_floor"][: 8 * n], orc.lam_floor[: 8 * n]),
                          (T["lam_pair"][: 8 * n_pairs], orc.lam_pair[: 8 * n_pairs]),
                          (T["lam_joint"][: eng.num_joints], orc.lam_joint[: eng.num_joints])):
            got = got.cpu().numpy()
            if want.size:
                scale = max(float(np.abs(want).max()), 1e-12)
                assert np.abs(got - want).max() <= 1e-4 * scale, (k, np.abs(got - want).max(), scale)


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


@pytest.mark.parametrize("dims", [(12, 10, 12), (13, 15, 13)], ids=["fused_1440", "multi_kernel_2535"])
def test_lbvh_pairs_match_oracle_both_paths(dims):
    """LBVH pair lists after 40 frames of a falling pile (moving, rotating
    bodies, so the velocity padding matters), against the oracle's pair set:
    up to 2048 bodies the fused single-launch broad phase runs, above it the
    multi-kernel one; both bit for bit, ordered by (a, b)."""
    nx, ny, nz = dims
    kw = dict(substeps=15, iterations=2, floor_y=0.0, friction=0.6, restitution=0.2, broadphase="lbvh")
    eng, orc = _pair(lambda s: scenes.build_box_pile(s, nx=nx, ny=ny, nz=nz, pitch=0.75, seed=4), **kw)
    for _ in range(40):
        eng.step()
    orc._flush()
    orc.x[:] = eng.positions()
    orc.q[:] = eng.orientations()
    orc.v[:] = eng.velocities()
    orc.omega[:] = eng.omega.numpy()
    N.check(lib6().xpbd6_broadphase(eng._h, N.stream_of(eng.device)))
    if eng.n_pairs > eng.cap:  # grow like step() does, then emit again
        eng._alloc_pairs(int(eng.n_pairs * 1.5))
        eng._bind()
        eng.status()
        N.check(lib6().xpbd6_broadphase(eng._h, N.stream_of(eng.device)))
    k = orc._broadphase()
    assert k > eng.num_bodies
    assert eng.n_pairs == k
    np.testing.assert_array_equal(eng.pairs(), np.stack([orc.pair_a[:k], orc.pair_b[:k]], 1))


@pytest.mark.parametrize("count,outlier", [(2, False), (3, False), (97, False), (600, False), (300, True)])
def test_fused_lbvh_dense_overlap_matches_oracle(count, outlier):
    """Every box overlapping nearly every other (a tight random cloud): each
    query walks most of the tree, so the fused broad phase's shared frontier of
    64 nodes per 8-lane group overflows and the overflowing children are walked
    by single lanes.  The pair set must still equal the oracle's, sorted by
    (a, b); 2 and 3 bodies are the smallest trees.  With one far outlier the
    cloud's Morton keys crowd into a few cells of the key space (long shared
    prefixes, a deep and unbalanced tree)."""
    rng = np.random.default_rng(count)
    kw = dict(substeps=15, iterations=2, floor_y=-10.0, friction=0.6, restitution=0.2, broadphase="lbvh")
    boxes = []
    for _ in range(count):
        q = rng.normal(size=4)
        boxes.append((tuple(rng.uniform(-0.3, 0.3, 3)), tuple(rng.uniform(0.2, 0.4, 3)), tuple(q / np.linalg.norm(q))))
    if outlier:
        boxes.append(((40.0, 0.0, 40.0), (0.2, 0.2, 0.2), (0.0, 0.0, 0.0, 1.0)))

    def build(s):
        for x, he, q in boxes:
            s.add_box(x, he, 1.0, quaternion=q)

    eng, orc = _pair(build, **kw)
    eng._flush()
    orc._flush()
    N.check(lib6().xpbd6_broadphase(eng._h, N.stream_of(eng.device)))
    if eng.n_pairs > eng.cap:
        eng._alloc_pairs(int(eng.n_pairs * 1.5))
        eng._bind()
        eng.status()
        N.check(lib6().xpbd6_broadphase(eng._h, N.stream_of(eng.device)))
    assert eng.status() == 0
    k = orc._broadphase()
    assert eng.n_pairs == k
    if count >= 97:
        assert k > 0.8 * count * (count - 1) / 2 * (0.9 if outlier else 1.0)
    np.testing.assert_array_equal(eng.pairs(), np.stack([orc.pair_a[:k], orc.pair_b[:k]], 1))


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
    """The captured frame (pair count stays on the device) and the synced frame
    (pair count read back between broad and narrow phase) run the same physics."""
    solvers = []
    for sync in (True, False):
        s = Solver6DOF(device="cuda:0", substeps=10, iterations=2, restitution=0.2)
        # a pile that starts separated: from overlapping boxes a single frame
        # already moves contacts across their thresholds by float-atomic order
        scenes.build_box_pile(s, nx=3, ny=3, nz=3, pitch=0.7, seed=8)
        s.sync_pairs = sync
        solvers.append(s)
    a, b = solvers
    for f in range(3):
        if f:
            b.load_state_dict(a.state_dict())
        a.step()
        b.step()
        assert a.status() == 0 and b.status() == 0
        assert a.n_pairs == b.n_pairs
        np.testing.assert_array_equal(a.pairs(), b.pairs())
        assert np.abs(a.positions() - b.positions()).max() <= 1e-5


def test_substep_drivers_agree():
    """Cluster / grid drivers and thread-per-item / eight-lane phases all run the
    same substep; from the same state, one frame agrees to float-atomic rounding."""
    runs = {}
    for drv, lanes, want in (((2, 16, 512), 8, "cluster"), ((2, 4, 256), 8, "cluster"), ((0, 0, 256), 8, "grid"),
                             ((0, 1, 256), 8, "grid"), ((2, 16, 512), 1, "cluster"), ((0, 0, 256), 1, "grid")):
        s = Solver6DOF(device="cuda:0", substeps=10, iterations=2, restitution=0.2)
        s.set_driver(*drv)
        s.lanes = lanes
        scenes.build_box_pile(s, nx=4, ny=3, nz=4, pitch=0.7, seed=8)
        assert s.launch_info()["mode"] == want
        runs[(drv, lanes)] = s
    ref = runs[((2, 16, 512), 8)]
    for f in range(3):
        if f:
            sd = ref.state_dict()
            for s in runs.values():
                if s is not ref:
                    s.load_state_dict(sd)
        for s in runs.values():
            s.step()
        x = ref.positions()
        for key, s in runs.items():
            assert s.status() == 0, key
            assert s.n_pairs == ref.n_pairs, key
            assert np.abs(s.positions() - x).max() <= 1e-5, (f, key)


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


@pytest.mark.parametrize("entry", ["xpbd6_manifold", "xpbd6_manifold8"])
def test_kernel_entry_points_match_oracle(golden, entry):
    """Manifold generation through the C ABI (thread per pair and eight lanes
    per pair) against the reference's recorded manifold of 256 random box pairs:
    bit for bit."""
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
    N.check(getattr(lib6(), entry)(C.byref(s._st), float(g["margin"]), N.stream_of(s.device)))
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


def test_setters_edit_in_place_without_rebinding():
    """set_velocity / add_impulse / set_omega write the device tensors in place:
    no re-bind (no graph re-capture) between frames, and the edit shows in the
    next frame."""
    s = Solver6DOF(device="cuda:0", substeps=10, iterations=2, gravity=(0.0, 0.0, 0.0))
    s.add_box((0.0, 2.0, 0.0), (0.5, 0.5, 0.5), 1.0)
    s.add_box((3.0, 2.0, 0.0), (0.5, 0.5, 0.5), 1.0)
    s.step()
    binds = s.binds
    s.set_velocity(0, (0.0, 6.0, 0.0))
    s.add_impulse(1, (0.0, 0.0, 6.0))
    s.set_omega(1, (0.0, 2.0, 0.0))
    s.step()
    assert s.binds == binds
    x = s.positions()
    assert abs(x[0, 1] - 2.1) < 1e-3 and abs(x[1, 2] - 0.1) < 1e-3
    assert abs(float(s.orientations()[1, 1]) - np.sin(1 / 60)) < 1e-3  # half of 2 rad/s x 1/60 s


def test_dlpack_export_is_the_live_state():
    s = Solver6DOF(device="cuda:0", substeps=5, iterations=1)
    s.add_box((0.0, 2.0, 0.0), (0.5, 0.5, 0.5), 1.0)
    s.step()
    x = torch.utils.dlpack.from_dlpack(s.dlpack("x"))
    np.testing.assert_array_equal(x[:, :3].cpu().numpy(), s.positions())
    s.step()
    np.testing.assert_array_equal(x[:, :3].cpu().numpy(), s.positions())

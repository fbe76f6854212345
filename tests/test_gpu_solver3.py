"""GPU parity of the 3-DOF engine against the CPU oracle (which is itself pinned
bit-exactly to the reference's recorded outputs).

Tolerances: Gauss-Seidel projects rows in place with no atomics, and the engine
evaluates the same fp32 expressions in the same order as the oracle without
contraction (--fmad=false), so GS agrees to 1e-6 m.  Jacobi accumulates
corrections with float atomics whose order varies between runs (as in the
reference itself), so positions agree to 1e-5 m after one frame and lambdas to
1e-4 relative."""

import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle import oracle as O  # noqa: E402
from golden_scenes import fixtures3, kwargs  # noqa: E402
from xpbd_b200 import Solver, scenes  # noqa: E402
from xpbd_b200.scene import Body  # noqa: E402
from xpbd_b200 import _native as N  # noqa: E402


def _pair(build, **kw):
    eng = Solver(device="cuda:0", **kw)
    orc = O.OracleSolver(device="cpu", **kw)
    build(eng)
    build(orc)
    return eng, orc


def _lam_close(a, b, rel=1e-4, abs_=1e-6):
    return np.all(np.abs(a - b) <= abs_ + rel * np.abs(b))


@pytest.mark.parametrize("name,build,frames", fixtures3(), ids=[f[0] for f in fixtures3()])
def test_frames_match_oracle(golden, name, build, frames):
    kw = kwargs(golden(name))
    eng, orc = _pair(build, **kw)
    gs = kw.get("solve_mode") == "gs"
    for f in range(frames):
        eng.step()
        orc.step()
        dx = np.abs(eng.positions() - orc.positions()).max()
        dv = np.abs(eng.velocities() - orc.velocities()).max()
        tol = 1e-6 if gs else 1e-5 * (f + 1) ** 2
        assert dx <= tol, f"frame {f}: max|dx| {dx}"
        assert dv <= 900 * tol, f"frame {f}: max|dv| {dv}"
        assert eng.num_constraints == orc.num_constraints
        r = eng.rows()
        np.testing.assert_array_equal(r["type"], orc.r_type)
        np.testing.assert_array_equal(r["a"], orc.r_a)
        np.testing.assert_array_equal(r["b"], orc.r_b)
        if f == 0:
            assert _lam_close(eng.lambdas(), orc.lambdas()), np.abs(eng.lambdas() - orc.lambdas()).max()
    if gs:
        assert eng.num_colors == orc.num_colors


_JACOBI = [f for f in fixtures3() if "jacobi" in f[0]]


@pytest.mark.parametrize("name,build,frames", _JACOBI, ids=[f[0] for f in _JACOBI])
def test_jacobi_frames_from_identical_state_match_oracle(golden, name, build, frames):
    """Frame by frame from identical state: before every frame the oracle takes
    the engine's positions and velocities, then both run one whole frame
    (all substeps and iterations).  The free-running comparison above lets its
    bound grow with the frame count, because the Jacobi sums' float-atomic
    order makes two runs drift apart; here the drift cannot accumulate, so one
    flat bound holds on every frame: positions within 1e-5 m, velocities within
    1e-2 m/s (position differences over the 1/900 s substep), the rows bit for
    bit and every multiplier of the frame's last substep within 1e-4 relative."""
    kw = kwargs(golden(name))
    eng, orc = _pair(build, **kw)
    eng._flush()
    orc._flush()
    for f in range(frames):
        orc.x[:] = eng.positions()
        orc.v[:] = eng.velocities()
        eng.step()
        orc.step()
        dx = np.abs(eng.positions() - orc.positions()).max()
        dv = np.abs(eng.velocities() - orc.velocities()).max()
        assert dx <= 1e-5, f"frame {f}: max|dx| {dx}"
        assert dv <= 1e-2, f"frame {f}: max|dv| {dv}"
        r = eng.rows()
        np.testing.assert_array_equal(r["type"], orc.r_type)
        np.testing.assert_array_equal(r["a"], orc.r_a)
        np.testing.assert_array_equal(r["b"], orc.r_b)
        assert _lam_close(eng.lambdas(), orc.lambdas()), (f, np.abs(eng.lambdas() - orc.lambdas()).max())


@pytest.mark.parametrize("drv", [(2, 4, 256), (0, 0, 256)], ids=["cluster", "grid"])
@pytest.mark.parametrize("name", ["cloth6_jacobi", "spheres18_jacobi", "chain_jacobi"])
def test_folded_jacobi_drivers_match_oracle(golden, name, drv):
    """The cluster and grid drivers fold each Jacobi apply into the next
    iteration's position reads (one barrier per iteration instead of two); the
    frames still follow the oracle to float-atomic rounding, multipliers too."""
    build, frames = dict((f[0], (f[1], f[2])) for f in fixtures3())[name]
    kw = kwargs(golden(name))
    eng, orc = _pair(build, **kw)
    eng.set_driver(*drv)
    for f in range(frames):
        eng.step()
        orc.step()
        assert eng.status() == 0
        assert eng.launch_info()["mode"] == ("cluster" if drv[0] == 2 else "grid")
        dx = np.abs(eng.positions() - orc.positions()).max()
        assert dx <= 1e-5 * (f + 1) ** 2, f"frame {f}: max|dx| {dx}"
        if f == 0:
            assert _lam_close(eng.lambdas(), orc.lambdas()), np.abs(eng.lambdas() - orc.lambdas()).max()


def _disjoint_pairs(s):
    """40 distance pairs over a floor with friction, some partners static: no
    particle takes more than two corrections per iteration (its pair row and
    its floor row), so float atomics sum them to the same value in any order."""
    rng = np.random.default_rng(3)
    for k in range(40):
        p = rng.uniform(-1.0, 1.0, 3) * np.array([1.0, 0.0, 1.0]) + np.array([0.0, 0.02 + 0.1 * rng.random(), 0.0])
        a = s.add_particle(tuple(p), mass=1.0, velocity=tuple(rng.normal(0.0, 2.0, 3)))
        b = s.add_particle(tuple(p + np.array([0.1, 0.02, 0.0])), mass=0.0 if k % 7 == 0 else 2.0,
                           velocity=tuple(rng.normal(0.0, 2.0, 3)))
        s.add_distance(a, b, compliance=1e-6)
        s.add_floor_contact(a, friction=0.4)
        s.add_floor_contact(b, friction=0.4)


@pytest.mark.parametrize("drv", [(2, 4, 256), (0, 0, 256)], ids=["cluster", "grid"])
@pytest.mark.parametrize("substeps,iterations", [(15, 2), (4, 2), (5, 3), (4, 4)])
def test_folded_substeps_bit_exact_on_disjoint_pairs(drv, substeps, iterations):
    """The folded drivers read each substep boundary on the fly (apply, finalize,
    clamp, integrate inside the first iteration's reads) and store the frame
    state in one closing pass.  Where atomic order cannot matter they match the
    oracle bit for bit: positions, velocities, substep-start positions and
    multipliers, after every frame (odd and even substep counts end in
    different buffers; two to four iterations, the folded range)."""
    kw = dict(dt=1 / 60, substeps=substeps, iterations=iterations, solve_mode="jacobi", damping=0.01, max_speed=3.0)
    eng, orc = _pair(_disjoint_pairs, **kw)
    eng.set_driver(*drv)
    for f in range(4):
        eng.step()
        orc.step()
        assert eng.status() == 0
        sd = eng.state_dict()
        np.testing.assert_array_equal(eng.positions(), orc.positions())
        np.testing.assert_array_equal(eng.velocities(), orc.velocities())
        np.testing.assert_array_equal(sd["x_prev"][:, :3].cpu().numpy(), orc.x_prev)
        np.testing.assert_array_equal(eng.lambdas(), orc.lambdas())


@pytest.mark.parametrize("mode", ["gs", "jacobi"])
def test_one_substep_cloth32(mode):
    """One substep of the 32 x 32 cloth: x within 1e-5 m, lambda within 1e-4 rel."""
    kw = dict(dt=1 / 900, substeps=1, iterations=2, solve_mode=mode)
    eng, orc = _pair(lambda s: scenes.build_cloth(s, y=0.0005, velocity=(0.1, -0.5, 0.0)), **kw)
    eng.step()
    orc.step()
    assert np.abs(eng.positions() - orc.positions()).max() <= 1e-5
    assert _lam_close(eng.lambdas(), orc.lambdas())


@pytest.mark.parametrize("mode", ["gs", "jacobi"])
def test_frame_drivers_agree(mode):
    """Shared-memory single CTA, thread-block cluster and cooperative grid run
    the same phases: GS must agree exactly, Jacobi to atomic-order rounding."""
    build = lambda s: scenes.build_cloth(s, res=12, spacing=0.05, y=0.01, velocity=(0.2, -1.0, 0.1))  # noqa: E731
    res = {}
    for drv, want in (((1, 0, 0), "shared"), ((2, 16, 1024), "cluster"), ((2, 4, 256), "cluster"),
                      ((0, 0, 256), "grid"), ((0, 1, 256), "grid")):
        s = Solver(device="cuda:0", dt=1 / 60, substeps=15, iterations=2, solve_mode=mode)
        build(s)
        s.set_driver(*drv)
        info = s.launch_info()
        assert info["mode"] == want, info
        for _ in range(3):
            s.step()
        res[drv] = s.positions()
        assert s.status() == 0
    ref = res[(1, 0, 0)]
    for drv, x in res.items():
        d = np.abs(x - ref).max()
        assert d <= (0.0 if mode == "gs" else 1e-4), (drv, d)


def test_autotune_keeps_results():
    o = O.OracleSolver(device="cpu", dt=1 / 60, substeps=15, iterations=2, solve_mode="gs")
    s = Solver(device="cuda:0", dt=1 / 60, substeps=15, iterations=2, solve_mode="gs")
    for t in (s, o):
        scenes.build_cloth(t, res=16, spacing=0.03, y=0.01, velocity=(0.1, -0.5, 0.0))
    rep = s.autotune(frames=2)
    assert rep["chosen"]["mode"] in ("shared", "cluster", "grid")
    for _ in range(2):
        s.step()
        o.step()
    assert np.abs(s.positions() - o.positions()).max() <= 1e-6


def test_multi_frame_launch_equals_single_frames():
    build = lambda s: scenes.build_cloth(s, res=8, spacing=0.05, y=0.01)  # noqa: E731
    a = Solver(device="cuda:0", dt=1 / 60, substeps=10, iterations=2, solve_mode="gs")
    b = Solver(device="cuda:0", dt=1 / 60, substeps=10, iterations=2, solve_mode="gs")
    build(a)
    build(b)
    for _ in range(4):
        a.step()
    b.step_frames(4)
    np.testing.assert_array_equal(a.positions(), b.positions())


def test_kernel_entry_points_match_oracle():
    """Each per-kernel C-ABI entry point against the oracle kernel it restates."""
    rng = np.random.default_rng(7)
    s = Solver(device="cuda:0", dt=1 / 60, substeps=1, iterations=1, solve_mode="jacobi")
    o = O.OracleSolver(device="cpu", dt=1 / 60, substeps=1, iterations=1, solve_mode="jacobi")
    for t in (s, o):
        scenes.build_cloth(t, res=10, spacing=0.05, y=0.002, velocity=(0.3, -1.0, 0.2))
        t._flush()
    n = s.num_bodies
    x = o.x + rng.normal(0, 0.003, o.x.shape).astype(np.float32)
    x[:, 1] -= 0.004
    o.x[:] = x
    s.tensors["x"][:, :3] = torch.from_numpy(x).cuda()
    st = C.byref(s._st)
    L = N.lib()
    h = np.float32(1 / 900)
    stream = N.stream_of(s.device)
    N.check(L.xpbd3_integrate(st, h, 0.0, -9.81, 0.0, stream))
    O.lib().or3_integrate(n, O.fp(o.x), O.fp(o.v), O.fp(o.inv_mass), C.c_float(0), C.c_float(-9.81), C.c_float(0),
                          C.c_float(h), O.fp(o.x_prev))
    np.testing.assert_array_equal(s.positions(), o.x)
    N.check(L.xpbd3_solve_jacobi(st, h, 1, stream))
    o.lam[:] = 0
    O.lib().or3_solve_jacobi_all(C.byref(o._scene()), C.c_float(h))
    acc = s.tensors["acc"].cpu().numpy()
    np.testing.assert_allclose(acc[:, :3], o.dx, atol=1e-6)
    np.testing.assert_array_equal(acc[:, 3].astype(np.int32), o.dn)
    assert _lam_close(s.lambdas(), o.lam)
    N.check(L.xpbd3_apply_jacobi(st, np.float32(0.9), stream))
    O.lib().or3_apply_jacobi(n, O.fp(o.x), O.fp(o.dx), O.ip(o.dn), O.fp(o.inv_mass), C.c_float(0.9))
    assert np.abs(s.positions() - o.x).max() <= 1e-6
    N.check(L.xpbd3_finalize_velocity(st, h, np.float32(0.01), stream))
    O.lib().or3_finalize(n, O.fp(o.x), O.fp(o.x_prev), O.fp(o.inv_mass), C.c_float(h), C.c_float(0.01), O.fp(o.v))
    assert np.abs(s.velocities() - o.v).max() <= 1e-3
    N.check(L.xpbd3_cap_velocity(st, np.float32(0.5), stream))
    O.lib().or3_cap(n, O.fp(o.v), C.c_float(0.5))
    assert np.abs(s.velocities() - o.v).max() <= 1e-3


def test_sphere_contacts_2048_bit_exact(golden):
    """Device contact generation on the 2048-sphere pile reproduces the
    reference's rows (endpoints, rest, mu) in the reference's order."""
    g = golden("sphere_contacts_2048")
    s = Solver(device="cuda:0", dt=1 / 60, substeps=15, iterations=2, solve_mode="jacobi")
    scenes.build_sphere_pile(s)
    s._flush()
    s._build_contacts(N.stream_of(s.device))
    r = s.rows()
    k = s._n_static
    np.testing.assert_array_equal(r["a"][k:], g["a"])
    np.testing.assert_array_equal(r["b"][k:], g["b"])
    np.testing.assert_array_equal(r["rest"][k:], g["rest"])
    np.testing.assert_array_equal(r["mu"][k:], g["mu"])
    assert np.all(r["type"][k:] == 3)


@pytest.mark.parametrize("dims", [(16, 8, 16), (20, 12, 20)], ids=["fused_2048", "multi_kernel_4800"])
def test_sphere_contacts_match_oracle_both_paths(dims):
    """Contact rows for a jittered, overlapping pile with random velocities (so
    the velocity margin matters), against the oracle's restatement of
    solver.py:275-342: up to 4096 collidable spheres the single-CTA fused
    builder runs, above it the multi-kernel one; both bit for bit."""
    nx, ny, nz = dims
    kw = dict(dt=1 / 60, substeps=15, iterations=2, solve_mode="jacobi")
    s = Solver(device="cuda:0", **kw)
    o = O.OracleSolver(device="cpu", **kw)
    for t in (s, o):
        scenes.build_sphere_pile(t, nx=nx, ny=ny, nz=nz, pitch=0.098, seed=3)
    s._flush()
    o._flush()
    v = np.random.default_rng(1).normal(size=(s.num_bodies, 3)).astype(np.float32)
    s.tensors["v"][:, :3] = torch.from_numpy(v).cuda()
    o.v[:] = v
    s._build_contacts(N.stream_of(s.device))
    o._rebuild_contacts()
    r = s.rows()
    k = s._n_static
    want = [row for row in o._rows if row.type == 3]
    assert len(want) > 4 * s.num_bodies
    np.testing.assert_array_equal(r["a"][k:], np.array([row.body_a for row in want]))
    np.testing.assert_array_equal(r["b"][k:], np.array([row.body_b for row in want]))
    np.testing.assert_array_equal(r["rest"][k:], np.array([row.rest for row in want], np.float32))
    np.testing.assert_array_equal(r["mu"][k:], np.array([row.mu for row in want], np.float32))


def test_nan_positions_are_reset_and_flagged():
    s = Solver(device="cuda:0", dt=1 / 60, substeps=4, iterations=1, solve_mode="jacobi")
    scenes.build_sphere_pile(s, nx=2, ny=2, nz=2, pitch=0.12, y0=0.3)
    s._flush()
    s.tensors["x"][3, 0] = float("nan")
    s.step()
    assert np.all(np.isfinite(s.positions()))
    assert s.status() & N.XPBD_ERR_NAN


def test_contact_capacity_overflow_grows():
    s = Solver(device="cuda:0", dt=1 / 60, substeps=4, iterations=1, solve_mode="jacobi")
    scenes.build_sphere_pile(s, nx=6, ny=6, nz=6, pitch=0.06, y0=0.3, jitter=0.0)
    s.contact_capacity_per_body = 0  # forces the minimum capacity of 1024 rows
    o = O.OracleSolver(device="cpu", dt=1 / 60, substeps=4, iterations=1, solve_mode="jacobi")
    scenes.build_sphere_pile(o, nx=6, ny=6, nz=6, pitch=0.06, y0=0.3, jitter=0.0)
    s.step()
    o.step()
    assert s.num_constraints == o.num_constraints > 216 + 1024
    assert np.abs(s.positions() - o.positions()).max() <= 1e-4


def test_primitives_sort_and_scan():
    rng = np.random.default_rng(0)
    L = N.lib()
    # one CTA up to 16384 keys, then tiles over many CTAs (8 passes for 64
    # bits; 5 for 40 bits, which end in the scratch buffers and copy back)
    for n, bits in ((1, 64), (5, 64), (1000, 64), (5000, 64), (20000, 64), (100000, 40), (70001, 64)):
        keys = rng.integers(0, 1 << 40, n, dtype=np.uint64)
        keys[: n // 3] = keys[0]  # ties keep input order
        vals = np.arange(n, dtype=np.uint32)
        tk = torch.from_numpy(keys.view(np.int64)).cuda()
        tv = torch.from_numpy(vals.view(np.int32)).cuda()
        N.check(L.xpbd_sort_pairs_u64(N.ptr(tk), N.ptr(tv), n, bits, N.stream_of("cuda:0")))
        order = np.argsort(keys, kind="stable")
        np.testing.assert_array_equal(tk.cpu().numpy().view(np.uint64), keys[order])
        np.testing.assert_array_equal(tv.cpu().numpy().view(np.uint32), vals[order])
    for n in (1, 7, 4096, 100000):
        a = rng.integers(0, 5, n).astype(np.int32)
        ta = torch.from_numpy(a).cuda()
        out = torch.zeros(n, dtype=torch.int32, device="cuda")
        tot = torch.zeros(1, dtype=torch.int32, device="cuda")
        N.check(L.xpbd_scan_i32(N.ptr(ta), N.ptr(out), n, N.ptr(tot), N.stream_of("cuda:0")))
        np.testing.assert_array_equal(out.cpu().numpy(), np.concatenate([[0], np.cumsum(a)[:-1]]))
        assert int(tot.item()) == int(a.sum())


def test_setters_edit_in_place_without_rebinding():
    """Setters write the device tensors in place: no re-bind (and so no graph
    re-capture) between frames; the edits take effect in the next frame."""
    twins = []
    for kick in (False, True):
        s = Solver(device="cuda:0", dt=1 / 60, substeps=10, iterations=2, solve_mode="jacobi")
        scenes.build_cloth(s, res=8, spacing=0.05, y=1.0)
        s.step()
        binds = s.binds
        if kick:
            s.set_velocity(Body(index=5), (0.0, 3.0, 0.0))
            s.set_all_compliance(1e-4)
            s.set_all_friction(0.2)
        s.step()
        assert s.binds == binds
        twins.append(s)
    assert twins[1].positions()[5, 1] > twins[0].positions()[5, 1] + 0.01  # the kick moved body 5 up
    r = twins[1].rows()
    assert np.all(r["compliance"][r["type"] == 0] == np.float32(1e-4))
    assert np.all(r["mu"][r["type"] == 2] == np.float32(0.2))  # FLOOR rows


def test_dlpack_export_is_the_live_state():
    s = Solver(device="cuda:0", dt=1 / 60, substeps=5, iterations=1, solve_mode="jacobi")
    scenes.build_cloth(s, res=6, spacing=0.05, y=1.0)
    s.step()
    x = torch.utils.dlpack.from_dlpack(s.dlpack("x"))
    np.testing.assert_array_equal(x[:, :3].cpu().numpy(), s.positions())
    s.step()
    np.testing.assert_array_equal(x[:, :3].cpu().numpy(), s.positions())  # zero copy: same memory


def test_captured_frame_with_contacts_matches_host_driven_frames():
    """With sync_contacts off, step() attaches the contact rebuild to the handle
    and replays contact rebuild + frame kernel as one captured graph.  The rows
    of the first frame are identical to the host-driven path's (same start
    state), later frames agree to float-atomic rounding, and turning the host
    check back on detaches."""
    runs = {}
    for graph in (False, True):
        s = Solver(device="cuda:0", dt=1 / 60, substeps=15, iterations=2, solve_mode="jacobi")
        scenes.build_sphere_pile(s, nx=8, ny=4, nz=8, pitch=0.098, y0=0.06, seed=4)
        s.sync_contacts = not graph
        s.step()
        assert s._hooked == graph
        rows1 = s.rows()
        for _ in range(3):
            s.step()
        assert s.status() == 0
        runs[graph] = (rows1, s.positions(), s)
    (ra, xa, _), (rb, xb, sb) = runs[False], runs[True]
    for k in ("type", "a", "b", "rest", "mu"):
        np.testing.assert_array_equal(ra[k], rb[k])
    assert np.abs(xa - xb).max() <= 1e-4
    sb.sync_contacts = True
    sb.step()
    assert not sb._hooked
    binds = sb.binds
    sb.sync_contacts = False
    sb.set_driver(0, 0, 256)  # a re-bind drops the capture; the next step captures the grid driver
    sb.step()
    assert sb._hooked and sb.binds == binds + 1 and sb.launch_info()["mode"] == "grid"
    assert sb.status() == 0


def test_gs_drivers_agree_on_attach_rows():
    """The packed Gauss-Seidel rows keep an ATTACH row's index for its anchor:
    the chain scene (distance rows, an ATTACH row, floor rows) gives the same
    bits on the one-CTA, cluster and grid drivers."""
    import make_golden as MG
    res = {}
    for drv in ((1, 0, 0), (2, 4, 256), (0, 0, 256)):
        s = Solver(device="cuda:0", dt=1 / 60, substeps=10, iterations=2, solve_mode="gs")
        MG.chain_scene(s)
        s.set_driver(*drv)
        for _ in range(3):
            s.step()
        assert s.status() == 0
        res[drv] = (s.positions(), s.lambdas())
    ref = res[(1, 0, 0)]
    assert np.any(ref[1] != 0.0)
    for drv, (x, lam) in res.items():
        np.testing.assert_array_equal(x, ref[0])
        np.testing.assert_array_equal(lam, ref[1])


def test_captured_frame_reports_contact_overflow():
    """Without the per-frame host check the captured frame cannot grow the
    contact capacity: it keeps the rows that fit and raises XPBD_ERR_OVERFLOW in
    the status word instead."""
    s = Solver(device="cuda:0", dt=1 / 60, substeps=4, iterations=1, solve_mode="jacobi")
    scenes.build_sphere_pile(s, nx=6, ny=6, nz=6, pitch=0.06, y0=0.3, jitter=0.0)
    s.contact_capacity_per_body = 0  # the minimum capacity of 1024 rows
    s.sync_contacts = False
    s.step()
    assert s._hooked
    assert s.status() & N.XPBD_ERR_OVERFLOW
    assert s.num_constraints == len(s.rows()["type"]) <= s._cap
    assert np.all(np.isfinite(s.positions()))


def test_gs_packed_rows_follow_the_setters():
    """Gauss-Seidel on the grid driver keeps its rows packed in color order
    across launches and packs them again after a setter: frames before and
    after set_all_compliance / set_all_friction agree bit for bit with the
    one-CTA driver, which stages the rows afresh in every launch."""
    out = []
    for drv in ((0, 4, 256), (1, 0, 0)):
        s = Solver(device="cuda:0", dt=1 / 60, substeps=15, iterations=2, solve_mode="gs")
        scenes.build_cloth(s, res=16, spacing=0.03, y=0.05, velocity=(0.1, -0.5, 0.0))
        s.set_driver(*drv)
        for _ in range(3):
            s.step()
        binds = s.binds
        s.set_all_compliance(1e-5)
        s.set_all_friction(0.05)
        for _ in range(3):
            s.step()
        assert s.binds == binds
        out.append((s.launch_info()["mode"], s.positions(), s.lambdas()))
    assert out[0][0] == "grid" and out[1][0] == "shared"
    np.testing.assert_array_equal(out[0][1], out[1][1])
    np.testing.assert_array_equal(out[0][2], out[1][2])

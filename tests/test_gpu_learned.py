"""Learned lambda warm start: the engine's MLP kernels against the CPU oracle
(forward values and the batch gradient), training lowers the loss, and on a
hanging cloth the trained warm start reaches the residual tolerance in fewer
Jacobi iterations than the plain lambda0 = 0 solve.  For the 6-DOF contact rows:
the feature kernel against a numpy restatement, and on a settled box pile the
trained warm start reaches the plain solve's 50-iteration residual in far fewer
iterations."""

import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle import oracle as O  # noqa: E402
from xpbd_b200 import Solver, Solver6DOF, scenes  # noqa: E402
from xpbd_b200.learned import (SubstepKit, SubstepKit6, WarmStartMLP, collect, collect6,  # noqa: E402
                               iterations_to_tol, iterations_to_tol6)


def _oracle_grads(feats, targets, w):
    B = len(targets)
    G = np.zeros(len(w), np.float64)
    f = np.ascontiguousarray(feats, np.float32)
    t = np.ascontiguousarray(targets, np.float32)
    ww = np.ascontiguousarray(w, np.float32)
    L = O.lib()
    L.or_mlp_grads.restype = C.c_double
    loss = L.or_mlp_grads(O.fp(f), O.fp(t), B, O.fp(ww), G.ctypes.data_as(C.POINTER(C.c_double)))
    return loss, G


def test_mlp_gradient_matches_oracle():
    rng = np.random.default_rng(0)
    B = 300
    feats = rng.normal(size=(B, 8)).astype(np.float32)
    feats[:, 7] = 0
    targets = rng.normal(size=B).astype(np.float32)
    m = WarmStartMLP(seed=3)
    loss, G = m.grads(torch.from_numpy(feats).cuda(), torch.from_numpy(targets).cuda())
    ref_loss, ref_G = _oracle_grads(feats, targets, m.w.cpu().numpy())
    assert abs(loss - ref_loss) <= 1e-4 * max(1.0, abs(ref_loss))
    G = G.cpu().numpy()
    scale = np.abs(ref_G).max()
    assert np.abs(G - ref_G).max() <= 2e-4 * scale, np.abs(G - ref_G).max() / scale


def test_mlp_inference_matches_oracle():
    rng = np.random.default_rng(1)
    m_rows = 500
    feats = rng.normal(size=(m_rows, 8)).astype(np.float32)
    weff = rng.uniform(1.0, 10.0, m_rows).astype(np.float32)
    m = WarmStartMLP(seed=4)
    lam0 = torch.zeros(m_rows, device="cuda")
    m.infer(torch.from_numpy(feats).cuda(), torch.from_numpy(weff).cuda(), m_rows, lam0)
    y = np.zeros(m_rows, np.float32)
    O.lib().or_mlp_forward(O.fp(np.ascontiguousarray(feats)), m_rows, O.fp(m.w.cpu().numpy()), O.fp(y))
    ref = np.sign(y) * np.expm1(np.abs(y)) * 1e-3 / weff
    got = lam0.cpu().numpy()
    assert np.isfinite(got).all()
    rel = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-9)
    # The second layer runs on the tensor cores (bf16 operands, fp32
    # accumulation in an order of its own).  Both sides round the first layer's
    # GELU outputs to bf16; a GELU result (CUDA erff against the host's) within
    # an ulp of a rounding boundary can round to the neighbouring bf16 value
    # (0.4 % of that activation), so a few rows move by up to ~1e-3; the rest
    # agree to the fp32 accumulation.
    assert rel.max() <= 2e-3, rel.max()
    assert np.mean(rel <= 2e-5) >= 0.95, np.quantile(rel, [0.5, 0.95, 0.99])
    st = C.c_int(7)
    from xpbd_b200 import _native as N
    N.check(N.lib().xpbd_mlp_status(C.byref(st), 1), "xpbd_mlp_status")
    assert st.value == 0


@pytest.mark.parametrize("m_rows", [1, 127, 128, 129, 4096 + 77, 300000])
def test_mlp_inference_tiles(m_rows):
    """Row counts around the 128-row tile and above the persistent grid
    (4 CTAs per SM): every row written, rows with weff = 0 get 0."""
    rng = np.random.default_rng(m_rows)
    feats = rng.normal(size=(m_rows, 8)).astype(np.float32)
    weff = rng.uniform(1.0, 10.0, m_rows).astype(np.float32)
    weff[::7] = 0.0
    m = WarmStartMLP(seed=4)
    lam0 = torch.full((m_rows + 5,), 12345.0, device="cuda")
    m.infer(torch.from_numpy(feats).cuda(), torch.from_numpy(weff).cuda(), m_rows, lam0)
    got = lam0.cpu().numpy()
    assert (got[m_rows:] == 12345.0).all()
    got = got[:m_rows]
    assert np.isfinite(got).all()
    assert (got[::7] == 0.0).all()
    k = min(m_rows, 2000)
    y = np.zeros(k, np.float32)
    O.lib().or_mlp_forward(O.fp(np.ascontiguousarray(feats[:k])), k, O.fp(m.w.cpu().numpy()), O.fp(y))
    ref = np.sign(y) * np.expm1(np.abs(y)) * 1e-3 / np.where(weff[:k] == 0, 1.0, weff[:k])
    ref[weff[:k] == 0] = 0.0
    rel = np.abs(got[:k] - ref) / np.maximum(np.abs(ref), 1e-9)
    assert rel.max() <= 2e-3, rel.max()


def test_train_step_entry_point_equals_grads_then_adam():
    """xpbd_mlp_train_step through the C ABI: the same weights as
    xpbd_mlp_grads followed by xpbd_mlp_adam, to the rounding of the gradient's
    float atomics (their order differs between runs)."""
    from xpbd_b200 import _native as N
    rng = np.random.default_rng(2)
    feats = torch.from_numpy(rng.normal(size=(700, 8)).astype(np.float32)).cuda()
    targets = torch.from_numpy(rng.normal(size=700).astype(np.float32)).cuda()
    a, b = WarmStartMLP(seed=9), WarmStartMLP(seed=9)
    for step in (1, 2):
        a.train_step(feats, targets, lr=1e-3)
        loss = torch.zeros(1, dtype=torch.float32, device="cuda")
        fn = N.lib().xpbd_mlp_train_step
        fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int] + [C.c_void_p] * 5 + [C.c_float, C.c_int, C.c_void_p,
                                                                            C.c_void_p]
        fn.restype = C.c_int
        N.check(fn(N.ptr(feats), N.ptr(targets), 700, N.ptr(b.w), N.ptr(b.G), N.ptr(b.M), N.ptr(b.V), N.ptr(b.wb),
                   1e-3, step, N.ptr(loss), N.stream_of("cuda:0")), "xpbd_mlp_train_step")
        torch.cuda.synchronize()
        assert float(loss.item()) > 0.0
    np.testing.assert_allclose(a.w.cpu().numpy(), b.w.cpu().numpy(), rtol=1e-5, atol=1e-7)
    np.testing.assert_allclose(a.wb.float().cpu().numpy(), b.wb.float().cpu().numpy(), rtol=1e-2, atol=1e-6)


def _cloth(res=32, compliance=1e-5):
    """A hanging 32 x 32 cloth (spacing 0.02 m, 0.01 kg) at a compliance where
    the plain Jacobi solve does reach 1e-4 m, slowly (a stiffer cloth never
    reaches it within the iteration cap from any start)."""
    s = Solver(dt=1 / 60, substeps=15, iterations=2, solve_mode="jacobi")
    scenes.build_cloth(s, res=res, spacing=0.02, mass=0.01, y=1.0, compliance=compliance, floor=False)
    return s


def test_training_lowers_loss_and_warm_start_saves_iterations():
    torch.manual_seed(0)
    s = _cloth()
    for _ in range(20):  # let the cloth start to hang
        s.step()
    F, T = collect(s, substeps=30, iters=50)
    m = WarmStartMLP(seed=0)
    first = None
    idx = torch.randperm(len(T), device="cuda")
    for epoch in range(80):
        for k in range(0, len(T), 4096):
            sel = idx[k:k + 4096]
            loss = m.train_step(F[sel], T[sel], lr=2e-3)
        if first is None:
            first = float(loss.item())
    last = float(loss.item())
    assert last < 0.5 * first, (first, last)
    res = iterations_to_tol(s, m, tol=1e-4, max_iters=100)
    assert res["plain"] <= 100, res  # the plain solve converges, slowly
    assert not res["fallback"], res
    assert res["learned_with_fallback"] * 2 <= res["plain"], res


PILE_KW = dict(dt=1 / 60, substeps=15, iterations=2, floor_y=0.0, friction=0.6, restitution=0.2)


def _pile(nx, ny, nz, seed, frames):
    s = Solver6DOF(device="cuda:0", **PILE_KW)
    scenes.build_box_pile(s, nx=nx, ny=ny, nz=nz, seed=seed)
    for _ in range(frames):
        s.step()
    return s


def _qrot(q, v):
    u, w = q[:, :3], q[:, 3:4]
    return v * (2 * w * w - 1) + np.cross(u, v) * (2 * w) + u * (2 * np.sum(u * v, 1, keepdims=True))


def _world_invI_mul(q, inv_I, u):
    qc = q * np.array([-1, -1, -1, 1], np.float32)
    return _qrot(q, _qrot(qc, u) * inv_I)


def _gen_inv_mass(im, q, inv_I, r, n):
    rn = np.cross(r, n)
    return im + np.sum(rn * _world_invI_mul(q, inv_I, rn), 1)


def _slog(x):
    return np.sign(x) * np.log1p(np.abs(x))


def test_pile_features_match_numpy():
    """Features of every floor-corner and manifold-point row, restated in numpy
    from the post-manifold state (float64 here, so compared with tolerances)."""
    s = _pile(4, 3, 4, 5, 60)
    kit = SubstepKit6(s)
    kit.broadphase()
    kit.begin()
    T = {k: v.double().cpu().numpy() if v.is_floating_point() else v.cpu().numpy() for k, v in s.tensors.items()}
    h = s.dt / s.substeps
    n = s.num_bodies
    x, q, v, w, he, inv_I = T["x"][:, :3], T["q"], T["v"][:, :3], T["w"][:, :3], T["he"][:, :3], T["inv_I"][:, :3]
    im = T["x"][:, 3]
    prev = torch.cat([kit.prev_floor, kit.prev_pair]).double().cpu().numpy()
    feats = kit.feats.double().cpu().numpy()
    weff = kit.weff.double().cpu().numpy()
    rows, want_f, want_w = [], [], []
    S = np.array([[0.0, 1.0, 0.0]])
    for i in range(n):
        for c in range(8):
            j = 8 * i + c
            if im[i] == 0:
                rows.append(j); want_f.append(np.zeros(7)); want_w.append(0.0)
                continue
            corner = he[i] * np.array([1 if c & 1 else -1, 1 if c & 2 else -1, 1 if c & 4 else -1])
            r = _qrot(q[i:i + 1], corner[None])
            wg = _gen_inv_mass(im[i], q[i:i + 1], inv_I[i:i + 1], r, S)[0]
            C_ = x[i, 1] + r[0, 1] - s.floor_y
            vn = (v[i] + np.cross(w[i], r[0]))[1]
            rows.append(j); want_w.append(wg)
            want_f.append([_slog(C_ / 1e-3), np.log10(wg), np.log10(1e-12), _slog(prev[j] * wg / 1e-3),
                           _slog(max(-C_, 0) / 1e-3), -1.0, _slog(vn * h / 1e-3)])
    n_pairs = min(s.n_pairs, s.cap)
    hdr = T["m_hdr"]
    live = 0
    for p in range(n_pairs):
        cnt, inc, ref = hdr[p, 0], hdr[p, 1], hdr[p, 2]
        for c in range(cnt):
            live += 1
            slot = 8 * p + c
            Sn = T["m_normal"][p, :3][None]
            ri = _qrot(q[inc:inc + 1], T["m_off_inc"][slot, :3][None])
            rr = _qrot(q[ref:ref + 1], T["m_off_ref"][slot, :3][None])
            C_ = np.sum(((x[inc] + ri[0]) - (x[ref] + rr[0])) * Sn[0])
            wg = (_gen_inv_mass(im[inc], q[inc:inc + 1], inv_I[inc:inc + 1], ri, Sn)[0]
                  + _gen_inv_mass(im[ref], q[ref:ref + 1], inv_I[ref:ref + 1], rr, Sn)[0])
            vrel = (v[inc] + np.cross(w[inc], ri[0])) - (v[ref] + np.cross(w[ref], rr[0]))
            j = 8 * n + slot
            rows.append(j); want_w.append(wg)
            want_f.append([_slog(C_ / 1e-3), np.log10(wg), np.log10(1e-12), _slog(prev[j] * wg / 1e-3),
                           _slog(max(-C_, 0) / 1e-3), -Sn[0, 1], _slog(np.dot(vrel, Sn[0]) * h / 1e-3)])
    assert live > 20
    rows = np.array(rows)
    np.testing.assert_allclose(weff[rows], np.array(want_w), rtol=2e-5, atol=1e-7)
    np.testing.assert_allclose(feats[rows, :7], np.array(want_f), rtol=1e-4, atol=2e-3)
    # rows past each manifold's point count and past the live pairs are inactive
    inactive = np.setdiff1d(np.arange(8 * n, 8 * (n + s.cap)), rows)
    assert np.all(weff[inactive] == 0)


def test_pile_training_lowers_loss():
    """The engine's training kernels on box-pile contact rows."""
    torch.manual_seed(0)
    F, T = collect6(_pile(6, 4, 6, 21, 150), frames=2, iters=50)
    m = WarmStartMLP(seed=0)
    first = None
    for epoch in range(10):
        idx = torch.randperm(len(T), device="cuda")
        for k in range(0, len(T), 4096):
            loss = m.train_step(F[idx[k:k + 4096]], T[idx[k:k + 4096]], lr=2e-3)
        if first is None:
            first = float(loss.item())
    assert float(loss.item()) < 0.5 * first, (first, float(loss.item()))


def test_shipped_weights_save_iterations_on_pile():
    """The shipped network (trained on 10M cloth and pile rows) on a settled
    pile it was not trained on: from its warm start the Jacobi solve reaches the
    plain solve's 50-iteration residual in at most half the iterations on
    average, and from the classical start (the previous multipliers) in at most
    a third.  (The classical start is the stronger of the two, see
    profiles/learned_warm_start.md.)"""
    m = WarmStartMLP.pretrained()
    s = _pile(7, 4, 7, 23, 150)
    kit = SubstepKit6(s)
    kit.broadphase()
    prev = {"classic": (1.0, lambda k: torch.cat([k.prev_floor, k.prev_pair]))}
    rows = [iterations_to_tol6(kit, m, max_iters=50, variants=prev) for _ in range(s.substeps)][1:]
    plain = np.mean([r["to_plain_final"]["plain"] for r in rows])
    learned = np.mean([r["to_plain_final"]["learned"] for r in rows])
    classic = np.mean([r["classic"]["to_plain_final"] for r in rows])
    assert classic * 3 <= plain, (classic, plain)
    assert learned * 2 <= plain, (learned, plain)


def test_shipped_weights_save_iterations_on_cloth():
    """The shipped network on a hanging 32 x 32 cloth (compliance 1e-5): the
    warm-started solve reaches 1e-4 m in fewer iterations than the plain solve,
    the fallback included, on consecutive substeps that carry the previous
    converged multipliers."""
    m = WarmStartMLP.pretrained()
    s = _cloth()
    for _ in range(30):
        s.step()
    rows = [iterations_to_tol(s, m, tol=1e-4, max_iters=150, advance=True) for _ in range(4)][1:]
    plain = np.mean([r["plain"] for r in rows])
    learned = np.mean([r["learned_with_fallback"] for r in rows])
    assert plain <= 150
    assert learned * 1.5 <= plain, (learned, plain)


@pytest.mark.parametrize("ws", ["previous", "learned"])
def test_warm_start_option_on_the_3dof_solver(ws):
    """Solver(warm_start=...) steps through the public step(): frames stay
    finite, the warm start is kept on most substeps of a hanging cloth, and the
    residual after each frame is no worse than the plain solver's by more than
    a few percent (both solve 2 iterations per substep)."""
    model = WarmStartMLP.pretrained() if ws == "learned" else "previous"
    kw = dict(dt=1 / 60, substeps=15, iterations=2, solve_mode="jacobi")
    warm, plain = Solver(warm_start=model, **kw), Solver(**kw)
    for s in (warm, plain):
        scenes.build_cloth(s, res=24, compliance=1e-6)
    for _ in range(12):
        warm.step()
        plain.step()
    torch.cuda.synchronize()
    assert np.all(np.isfinite(warm.positions()))
    assert warm.status() == 0
    kept = int(warm._runner.learned_used.item())
    if ws == "previous":  # the previous multipliers beat lambda0 = 0 on a hanging cloth
        assert kept >= 0.5 * 12 * 15, kept
    r_w, r_p = float(warm.residual()[0]), float(plain.residual()[0])
    assert r_w <= 1.05 * r_p, (r_w, r_p)
    with pytest.raises(ValueError):
        s = Solver(warm_start="previous", **kw)
        scenes.build_sphere_pile(s, nx=2, ny=2, nz=2)
        s.step()


@pytest.mark.parametrize("ws", ["previous", "learned"])
def test_warm_start_option_on_the_6dof_solver(ws):
    """Solver6DOF(warm_start=...) on boxes dropped onto the floor (a 3 x 3
    layer 1.1 m apart, so none starts interpenetrating or stacks): frames stay
    finite, the warm-started boxes come to rest like the plain ones (every body
    below 0.2 m/s after 60 frames, mean height within 2 cm of the plain
    solver's), and the device point count covers every substep."""
    model = WarmStartMLP.pretrained() if ws == "learned" else "previous"
    kw = dict(dt=1 / 60, substeps=15, iterations=2, floor_y=0.0, friction=0.6, restitution=0.2)
    warm, plain = Solver6DOF(warm_start=model, **kw), Solver6DOF(**kw)
    for s in (warm, plain):
        scenes.build_box_pile(s, nx=3, ny=1, nz=3, pitch=1.1, y0=0.5)
    for _ in range(60):
        warm.step()
        plain.step()
    torch.cuda.synchronize()
    assert np.all(np.isfinite(warm.positions())) and np.all(np.isfinite(warm.orientations()))
    assert warm.status() == 0
    assert np.linalg.norm(plain.velocities(), axis=1).max() < 0.2  # the scene itself settles
    speed = np.linalg.norm(warm.velocities(), axis=1).max()
    assert speed < 0.2, speed
    dy = abs(float(warm.positions()[:, 1].mean() - plain.positions()[:, 1].mean()))
    assert dy < 0.02, dy
    assert warm._runner.substeps_run == 60 * 15


@pytest.mark.parametrize("ws", ["previous", "learned"])
def test_6dof_warm_start_graph_replay_matches_eager_frames(ws):
    """WarmStartRunner6 replays one captured graph of a frame's substeps from
    the second frame on; the same frames run eagerly give the same state (to
    the float atomics' order of the per-phase contact sums), the same manifold
    point count and the same number of substeps kept warm."""
    from xpbd_b200.learned import WarmStartRunner6
    model = WarmStartMLP.pretrained() if ws == "learned" else "previous"
    kw = dict(dt=1 / 60, substeps=15, iterations=2, floor_y=0.0, friction=0.6, restitution=0.2)
    a, b = Solver6DOF(**kw), Solver6DOF(**kw)
    for s in (a, b):
        scenes.build_box_pile(s, nx=3, ny=2, nz=3, pitch=0.8, y0=0.4)
    ra, rb = WarmStartRunner6(a, model), WarmStartRunner6(b, model)
    for f in range(8):
        ra.step(use_graph=True)
        rb.step(use_graph=False)
        if f == 0:
            assert ra.graph is None
    torch.cuda.synchronize()
    assert ra.graph is not None
    assert ra.substeps_run == rb.substeps_run == 8 * 15
    assert np.all(np.isfinite(a.positions()))
    np.testing.assert_allclose(a.positions(), b.positions(), atol=1e-3)
    np.testing.assert_allclose(a.orientations(), b.orientations(), atol=1e-2)
    pa, pb = ra.kit.points_total, rb.kit.points_total
    assert pa > 0 and abs(pa - pb) <= 0.02 * pb, (pa, pb)
    assert abs(int(ra.learned_used.item()) - int(rb.learned_used.item())) <= 0.1 * 8 * 15


@pytest.mark.parametrize("six", [False, True], ids=["3dof", "6dof"])
def test_warm_start_that_blows_up_falls_back_to_plain(six):
    """A network whose prediction is absurd but finite (an output bias of 80 in
    the log units: lambda0 near 1e31 on every row, which the warm-start kernels
    apply, unlike a non-finite lambda0, which they drop) must never be kept:
    the warm-started first iteration leaves an enormous or non-finite residual,
    so every substep falls back to the plain solve on the device, and the
    frames stay finite and follow the plain solver's."""
    bad = WarmStartMLP(seed=5)
    bad.w[-1] = 80.0  # the output bias
    bad.wb.copy_(bad.w.to(torch.bfloat16))
    if six:
        kw = dict(dt=1 / 60, substeps=15, iterations=2, floor_y=0.0, friction=0.6, restitution=0.2)
        warm, plain = Solver6DOF(warm_start=bad, **kw), Solver6DOF(**kw)
        for s in (warm, plain):
            scenes.build_box_pile(s, nx=3, ny=1, nz=3, pitch=1.1, y0=0.5)
    else:
        kw = dict(dt=1 / 60, substeps=15, iterations=2, solve_mode="jacobi")
        warm, plain = Solver(warm_start=bad, **kw), Solver(**kw)
        for s in (warm, plain):
            scenes.build_cloth(s, res=16, compliance=1e-6)
    for _ in range(6):
        warm.step()
        plain.step()
    torch.cuda.synchronize()
    assert int(warm._runner.learned_used.item()) == 0
    x = warm.positions()
    assert np.all(np.isfinite(x))
    np.testing.assert_allclose(x, plain.positions(), atol=1e-4)

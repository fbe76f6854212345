"""Device Welsh-Powell coloring (xpbd_color_rows_device, the pass a captured
Gauss-Seidel frame with contacts runs every frame) against the reference's
coloring: the recorded fixtures of coloring.py bit for bit, and the host
restatement (itself pinned to those fixtures) on graphs that reach every path
of the kernel -- more live rows than its shared-memory stage, more bodies than
its shared-memory bitsets, more than 64 colors -- plus the color-count limit.
Then the captured Gauss-Seidel sphere-pile frame against the host-colored one."""

import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from xpbd_b200 import Solver, scenes  # noqa: E402
from xpbd_b200 import _native as N  # noqa: E402

MAX_COLORS = 128


def _device_color(n_bodies, a, b, cap=None):
    m = len(a)
    cap = max(cap or m, 1)
    ri = np.zeros((cap, 4), np.int32)
    ri[:m, 1] = a
    ri[:m, 2] = b
    ri[:m, 3] = 1
    dev = "cuda:0"
    t_ri = torch.from_numpy(ri).to(dev)
    t_m = torch.tensor([m], dtype=torch.int32, device=dev)
    color = torch.full((cap,), -7, dtype=torch.int32, device=dev)
    order = torch.zeros(cap, dtype=torch.int32, device=dev)
    starts = torch.zeros(MAX_COLORS + 1, dtype=torch.int32, device=dev)
    k = torch.zeros(1, dtype=torch.int32, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    rc = N.lib().xpbd_color_rows_device(n_bodies, N.ptr(t_ri), N.ptr(t_m), cap, N.ptr(color), N.ptr(order),
                                        N.ptr(starts), N.ptr(k), N.ptr(status), N.stream_of(dev))
    N.check(rc, "xpbd_color_rows_device")
    kk = int(k.item())
    return (color[:m].cpu().numpy(), order[:m].cpu().numpy(), starts[:kk + 1].cpu().numpy(), kk,
            int(status.item()))


def _host_color(n_bodies, a, b):
    a = np.ascontiguousarray(a, np.int32)
    b = np.ascontiguousarray(b, np.int32)
    col = np.zeros(len(a), np.int32)
    k = N.lib().xpbd_color_constraints(n_bodies, len(a), a.ctypes.data_as(C.c_void_p), b.ctypes.data_as(C.c_void_p),
                                       col.ctypes.data_as(C.c_void_p))
    order = np.argsort(col, kind="stable").astype(np.int32)
    starts = np.zeros(k + 1, np.int32)
    starts[1:] = np.cumsum(np.bincount(col, minlength=k))
    return col, order, starts, k


@pytest.mark.parametrize("name", ["coloring_cloth32"] + [f"coloring_rand{i}" for i in range(4)])
def test_device_coloring_matches_reference_fixtures(golden, name):
    g = golden(name)
    col, order, starts, k, st = _device_color(int(g["n_bodies"]), g["a"], g["b"], cap=len(g["a"]) + 100)
    assert st == 0
    np.testing.assert_array_equal(col, g["color"])
    np.testing.assert_array_equal(order, g["order"])
    np.testing.assert_array_equal(starts, g["starts"])
    assert k == len(g["starts"]) - 1


def _random_rows(rng, n, m, one_body=0.2):
    a = rng.integers(0, n, m).astype(np.int32)
    b = rng.integers(0, n, m).astype(np.int32)
    b[b == a] = (b[b == a] + 1) % n
    b[rng.random(m) < one_body] = -1
    return a, b


@pytest.mark.parametrize("n,m", [(300, 5000), (3000, 12000), (6000, 9000), (9000, 20000)],
                         ids=["smem", "global_stage", "global_bitsets", "both_global"])
def test_device_coloring_matches_host_on_random_graphs(n, m):
    rng = np.random.default_rng(n + m)
    a, b = _random_rows(rng, n, m)
    col, order, starts, k, st = _device_color(n, a, b, cap=m + 333)
    hc, ho, hs, hk = _host_color(n, a, b)
    assert st == 0 and k == hk
    np.testing.assert_array_equal(col, hc)
    np.testing.assert_array_equal(order, ho)
    np.testing.assert_array_equal(starts, hs)


def test_device_coloring_past_64_colors():
    # a hub body shared by 100 rows: 100 colors (the second word of the bitsets)
    n = 200
    a = np.zeros(100, np.int32)
    b = np.arange(1, 101, dtype=np.int32)
    rng = np.random.default_rng(3)
    a2, b2 = _random_rows(rng, n, 400)
    a = np.concatenate([a, a2])
    b = np.concatenate([b, b2])
    col, order, starts, k, st = _device_color(n, a, b)
    hc, ho, hs, hk = _host_color(n, a, b)
    assert st == 0 and k == hk >= 100
    np.testing.assert_array_equal(col, hc)
    np.testing.assert_array_equal(order, ho)


def test_device_coloring_reports_more_than_128_colors():
    a = np.zeros(130, np.int32)
    b = np.arange(1, 131, dtype=np.int32)
    *_, st = _device_color(131, a, b)
    assert st & N.XPBD_ERR_OVERFLOW


def test_captured_gs_frame_with_contacts_matches_host_colored_frames():
    """Gauss-Seidel sphere pile: frames replayed as one captured graph (contact
    rebuild + device coloring + frame kernel) against frames that color the
    contact rows on the host: same rows and, Gauss-Seidel being free of atomics,
    bit-identical positions and multipliers."""
    kw = dict(dt=1 / 60, substeps=15, iterations=2, solve_mode="gs")
    dev, host = Solver(device="cuda:0", **kw), Solver(device="cuda:0", **kw)
    for s in (dev, host):
        scenes.build_sphere_pile(s, nx=10, ny=5, nz=10, pitch=0.098, y0=0.06)
    dev.sync_contacts = False
    for f in range(4):
        dev.step()
        host.step()
        torch.cuda.synchronize()
        rd, rh = dev.rows(), host.rows()
        for key in ("type", "a", "b", "rest", "mu"):
            np.testing.assert_array_equal(rd[key], rh[key])
        np.testing.assert_array_equal(dev.positions(), host.positions())
        np.testing.assert_array_equal(dev.lambdas(), host.lambdas())
    assert dev._hooked
    assert dev.status() == 0

"""Failure detection on the GPU without a fault: the engine's grid barrier gives
up at its time limit, reports XPBD_ERR_BARRIER_TIMEOUT in the status word, and
leaves the context usable.  The failure is a CTA that never arrives (a wait
that nothing satisfies), never a trap, a bad address or an endless loop."""

import ctypes as C
import time

import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from xpbd_b200 import _native as N  # noqa: E402


def _run(blocks, absent, rounds):
    st = C.c_int(-1)
    N.check(N.lib().xpbd_barrier_selftest(blocks, absent, rounds, C.byref(st), N.stream_of("cuda:0")),
            "xpbd_barrier_selftest")
    return st.value


def test_grid_barrier_times_out_and_reports():
    assert _run(8, -1, 50) == 0  # every CTA arrives: no status bit
    t0 = time.monotonic()
    status = _run(8, 3, 3)  # CTA 3 never arrives
    elapsed = time.monotonic() - t0
    assert status & N.XPBD_ERR_BARRIER_TIMEOUT
    assert 1.5 < elapsed < 20.0  # the 2 s limit, not a hang
    assert _run(8, -1, 50) == 0  # the context still works, the count was reset
    x = torch.arange(16, device="cuda:0", dtype=torch.float32)
    assert float((x * 2).sum().item()) == 240.0


def test_selftest_rejects_bad_arguments():
    st = C.c_int(0)
    L = N.lib()
    sp = N.stream_of("cuda:0")
    assert L.xpbd_barrier_selftest(1, -1, 1, C.byref(st), sp) == N.XPBD_ERR_BAD_ARG
    assert L.xpbd_barrier_selftest(8, 8, 1, C.byref(st), sp) == N.XPBD_ERR_BAD_ARG
    assert L.xpbd_barrier_selftest(8, -1, 0, C.byref(st), sp) == N.XPBD_ERR_BAD_ARG
    assert L.xpbd_barrier_selftest(1 << 20, -1, 1, C.byref(st), sp) == N.XPBD_ERR_BAD_ARG

"""The allocation-free contact builder ``xpbd3_contacts_build_noalloc``.

Callers such as a plugin whose host application owns every GPU allocation, or
a fixed-budget simulation thread that must not call cudaMalloc (it can
synchronise the whole device), need a contact builder that allocates nothing.
This entry point uses one fixed device array inside the library as its working
memory.  The test calls it twice in a row through the C ABI, on two different
states, and checks each result against the allocating entry point
``xpbd3_contacts_build`` run on the same state: the contact rows (endpoints,
rest length, friction, order) and the live row count must be identical, as
the two entry points run the same kernels.  It does so at a small size and at
the stated limit (8192 collidable spheres), and checks that inputs above the
limit, or naming more collidable spheres than the state holds, are rejected.

This file is named so that pytest collects it last.
"""

import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from xpbd_b200 import Solver, scenes  # noqa: E402
from xpbd_b200 import _native as N  # noqa: E402

_ARGS = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
         C.c_double, C.c_double, C.c_double, C.c_void_p, C.c_void_p]


def _noalloc():
    fn = N.lib().xpbd3_contacts_build_noalloc
    fn.argtypes = _ARGS
    fn.restype = C.c_int
    return fn


def _rows(s):
    T = s.tensors
    m = int(T["n_rows"].item())
    return (m, T["row_i"][:m].cpu().numpy().copy(), T["row_f"][:m].cpu().numpy().copy())


def _build_both(s):
    """Rows from the allocating builder, then from the allocation-free one."""
    T = s.tensors
    stream = N.stream_of(s.device)
    n_coll = int(T["collide_idx"].numel())
    common = (N.ptr(T["radius"]), N.ptr(T["friction"]), N.ptr(T["collide_idx"]), n_coll,
              N.ptr(T["existing"]), int(T["existing"].numel()), N.ptr(T["x_init"]),
              C.c_double(s._contact_margin), C.c_double(s.dt), C.c_double(s._rmax), N.ptr(T["status"]), stream)
    N.check(N.lib().xpbd3_contacts_build(s._contacts, C.byref(s._st), *common), "xpbd3_contacts_build")
    ref = _rows(s)
    T["n_rows"].fill_(-1)
    T["row_i"][s._n_static:].zero_()
    N.check(_noalloc()(C.byref(s._st), *common), "xpbd3_contacts_build_noalloc")
    got = _rows(s)
    return ref, got


def test_noalloc_contacts_match_allocating_builder_twice():
    s = Solver(device="cuda:0", dt=1 / 60, substeps=15, iterations=2, solve_mode="jacobi")
    scenes.build_sphere_pile(s, nx=12, ny=6, nz=12, pitch=0.098, y0=0.06, seed=9)
    s._flush()
    for call in range(2):
        ref, got = _build_both(s)
        assert got[0] == ref[0] > s._n_static, (call, got[0], ref[0])
        np.testing.assert_array_equal(got[1], ref[1])
        np.testing.assert_array_equal(got[2], ref[2])
        assert int(s.tensors["status"].item()) == 0
        # advance the scene so the second call sees a different state
        N.check(N.lib().xpbd3_step(s._h, 1, N.stream_of(s.device)), "xpbd3_step")


def test_noalloc_contacts_at_the_size_limit():
    """8192 collidable spheres (32 x 8 x 32), the largest accepted input: the
    whole fixed layout (counts and offsets of 14 x 8192 neighbour slots, the
    sort and scan scratch) is in use, and the rows still equal the allocating
    builder's, on two calls in a row."""
    s = Solver(device="cuda:0", dt=1 / 60, substeps=15, iterations=2, solve_mode="jacobi")
    scenes.build_sphere_pile(s, nx=32, ny=8, nz=32, pitch=0.098, y0=0.06, seed=4)
    s._flush()
    assert int(s.tensors["collide_idx"].numel()) == 8192
    for call in range(2):
        ref, got = _build_both(s)
        assert got[0] == ref[0] > s._n_static, (call, got[0], ref[0])
        np.testing.assert_array_equal(got[1], ref[1])
        np.testing.assert_array_equal(got[2], ref[2])
        assert int(s.tensors["status"].item()) == 0
        N.check(N.lib().xpbd3_step(s._h, 1, N.stream_of(s.device)), "xpbd3_step")


def test_noalloc_rejects_inputs_over_the_limit():
    # 8448 collidable spheres in the state, 8193 of them passed: over the limit
    big = Solver(device="cuda:0", dt=1 / 60, substeps=4, iterations=1, solve_mode="jacobi")
    scenes.build_sphere_pile(big, nx=33, ny=8, nz=32)
    big._flush()
    T = big.tensors
    assert int(T["collide_idx"].numel()) > 8193
    rc = _noalloc()(C.byref(big._st), N.ptr(T["radius"]), N.ptr(T["friction"]), N.ptr(T["collide_idx"]), 8193,
                    N.ptr(T["existing"]), 0, N.ptr(T["x_init"]), C.c_double(0.0), C.c_double(1 / 60),
                    C.c_double(big._rmax), N.ptr(T["status"]), N.stream_of(big.device))
    assert rc == N.XPBD_ERR_BAD_ARG
    s = Solver(device="cuda:0", dt=1 / 60, substeps=4, iterations=1, solve_mode="jacobi")
    scenes.build_sphere_pile(s, nx=2, ny=2, nz=2)
    s._flush()
    T = s.tensors
    # more collidable spheres than the state has bodies (the allocating builder's
    # handle rejects this too)
    rc = _noalloc()(C.byref(s._st), N.ptr(T["radius"]), N.ptr(T["friction"]), N.ptr(T["collide_idx"]),
                    s.num_bodies + 1, N.ptr(T["existing"]), 0, N.ptr(T["x_init"]), C.c_double(0.0),
                    C.c_double(1 / 60), C.c_double(s._rmax), N.ptr(T["status"]), N.stream_of(s.device))
    assert rc == N.XPBD_ERR_BAD_ARG

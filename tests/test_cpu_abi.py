"""CPU-side checks of the engine library and host logic (no device calls):
the C ABI loads, exports every function include/xpbd_b200.h declares, and the
host-side coloring matches the oracle (and so the reference)."""

import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from xpbd_b200 import _native as N


def test_library_exports_every_declared_symbol():
    L = N.lib()
    declared = N.declared_symbols()
    assert len(declared) >= 40
    missing = [s for s in declared if not hasattr(L, s)]
    assert missing == []
    assert L.xpbd_version().startswith(b"xpbd_b200")


@pytest.mark.parametrize("name", ["coloring_cloth32"] + [f"coloring_rand{i}" for i in range(4)])
def test_engine_coloring_matches_reference(golden, name):
    g = golden(name)
    a = np.ascontiguousarray(g["a"], np.int32)
    b = np.ascontiguousarray(g["b"], np.int32)
    col = np.zeros(len(a), np.int32)
    k = N.lib().xpbd_color_constraints(int(g["n_bodies"]), len(a), a.ctypes.data_as(C.c_void_p),
                                       b.ctypes.data_as(C.c_void_p), col.ctypes.data_as(C.c_void_p))
    np.testing.assert_array_equal(col, g["color"])
    order = np.zeros(len(a), np.int32)
    starts = np.zeros(k + 1, np.int32)
    N.lib().xpbd_color_ranges(len(a), col.ctypes.data_as(C.c_void_p), order.ctypes.data_as(C.c_void_p),
                              starts.ctypes.data_as(C.c_void_p))
    np.testing.assert_array_equal(order, g["order"])
    np.testing.assert_array_equal(starts, g["starts"])


def test_coloring_rejects_bad_indices():
    a = np.array([0, 5], np.int32)
    b = np.array([1, 2], np.int32)
    col = np.zeros(2, np.int32)
    rc = N.lib().xpbd_color_constraints(3, 2, a.ctypes.data_as(C.c_void_p), b.ctypes.data_as(C.c_void_p),
                                        col.ctypes.data_as(C.c_void_p))
    assert rc == -1


def test_solver_requires_cuda_device():
    from xpbd_b200 import Solver, Solver6DOF
    with pytest.raises(N.XpbdError):
        Solver(device="cpu")
    with pytest.raises(N.XpbdError):
        Solver6DOF(device="cpu")


def test_batch_specs_distribution():
    from xpbd_b200.batch import batch_specs
    sp = batch_specs(256, seed=0)
    cl = [s.size for s in sp if s.kind == "cloth"]
    pi = [s.size for s in sp if s.kind == "pile"]
    assert len(cl) == len(pi) == 128
    assert min(cl) >= 16 and max(cl) <= 128 and min(pi) >= 64 and max(pi) <= 1024


def test_oracle_mlp_gradient_finite_difference():
    """The oracle's MLP gradient against central finite differences of its loss."""
    rng = np.random.default_rng(0)
    B = 16
    feats = rng.normal(size=(B, 8)).astype(np.float32)
    targets = rng.normal(size=B).astype(np.float32)
    w = (rng.normal(size=4737) * 0.2).astype(np.float32)
    L = O.lib()
    L.or_mlp_grads.restype = C.c_double
    L.or_bf16_round.restype = C.c_float
    L.or_bf16_round.argtypes = [C.c_float]
    # bf16-representable weights, so that the perturbations survive the rounding
    w = np.array([L.or_bf16_round(float(v)) for v in w], np.float32)
    G = np.zeros(4737, np.float64)
    f = np.ascontiguousarray(feats)
    t = np.ascontiguousarray(targets)
    # the hidden activations' bf16 rounding makes the loss a step function of
    # the first layer's weights; the gradient formulas are checked without it
    L.or_mlp_round_activations(0)
    try:
        L.or_mlp_grads(O.fp(f), O.fp(t), B, O.fp(w), G.ctypes.data_as(C.POINTER(C.c_double)))
        dummy = np.zeros(4737, np.float64)
        for i in (0, 100, 447, 450, 600, 4000, 4607, 4650, 4700, 4736):
            eps = 2.0 ** (np.floor(np.log2(abs(w[i]) + 1e-3)) - 6)  # a step bf16 can represent
            wp = w.copy(); wp[i] += eps
            wm = w.copy(); wm[i] -= eps
            lp = L.or_mlp_grads(O.fp(f), O.fp(t), B, O.fp(wp), dummy.ctypes.data_as(C.POINTER(C.c_double)))
            lm = L.or_mlp_grads(O.fp(f), O.fp(t), B, O.fp(wm), dummy.ctypes.data_as(C.POINTER(C.c_double)))
            fd = 0.5 * (lp - lm) / (2 * eps)  # loss is mean e^2, G is d(0.5 mean e^2)
            assert abs(fd - G[i]) <= 2e-2 * max(1e-3, abs(G[i])), (i, fd, G[i])
    finally:
        L.or_mlp_round_activations(1)

"""ctypes binding of ``libxpbd_b200.so`` (C ABI declared in include/xpbd_b200.h).

The engine has no CPU fallback: importing a solver on a machine without the
built library, or stepping it without a CUDA device, raises.
"""

from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libxpbd_b200.so")

XPBD_OK = 0
XPBD_ERR_BAD_ARG = 1
XPBD_ERR_CUDA = 2
XPBD_ERR_OVERFLOW = 4
XPBD_ERR_NAN = 8
XPBD_ERR_BARRIER_TIMEOUT = 16
XPBD_ERR_BAD_INDEX = 32

_p = C.c_void_p
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)


class XpbdError(RuntimeError):
    pass


class xpbd3_state(C.Structure):
    _fields_ = [("n_bodies", C.c_int), ("row_capacity", C.c_int), ("n_rows_static", C.c_int),
                ("x", _p), ("v", _p), ("x_prev", _p), ("acc", _p),
                ("row_i", _p), ("row_f", _p), ("row_anchor", _p), ("lam", _p),
                ("n_rows", _p), ("color_order", _p), ("color_starts", _p), ("num_colors", C.c_int)]


class xpbd3_params(C.Structure):
    _fields_ = [("dt", C.c_double), ("substeps", C.c_int), ("iterations", C.c_int),
                ("gravity", C.c_float * 3), ("damping", C.c_float), ("jacobi_relax", C.c_float),
                ("max_speed", C.c_float), ("gs", C.c_int)]


class xpbd6_state(C.Structure):
    _fields_ = [("n_bodies", C.c_int), ("n_joints", C.c_int), ("pair_capacity", C.c_int),
                ("x", _p), ("q", _p), ("v", _p), ("w", _p), ("x_prev", _p), ("q_prev", _p),
                ("inv_I", _p), ("he", _p), ("group", _p),
                ("acc_x", _p), ("acc_r", _p), ("acc_v", _p), ("acc_w", _p), ("lam_floor", _p),
                ("pairs", _p), ("n_pairs", _p), ("m_hdr", _p), ("m_normal", _p),
                ("m_off_inc", _p), ("m_off_ref", _p), ("lam_pair", _p),
                ("j_ab", _p), ("j_anchor_a", _p), ("j_anchor_b", _p), ("lam_joint", _p),
                ("scene", _p), ("n_scenes", C.c_int)]


class xpbd6_params(C.Structure):
    _fields_ = [("dt", C.c_double), ("substeps", C.c_int), ("iterations", C.c_int),
                ("gyroscopic", C.c_int), ("gravity", C.c_float * 3),
                ("floor_y", C.c_float), ("friction", C.c_float), ("restitution", C.c_float),
                ("lin_damp", C.c_float), ("ang_damp", C.c_float), ("jacobi_relax", C.c_float),
                ("max_speed", C.c_float), ("max_omega", C.c_float), ("man_margin", C.c_float),
                ("broadphase", C.c_int), ("edge_axes", C.c_int)]


_SIGS = {
    "xpbd_version": ([], C.c_char_p),
    "xpbd_last_error": ([], C.c_char_p),
    "xpbd3_integrate": ([_p, C.c_float, C.c_float, C.c_float, C.c_float, _p], C.c_int),
    "xpbd3_solve_jacobi": ([_p, C.c_float, C.c_int, _p], C.c_int),
    "xpbd3_apply_jacobi": ([_p, C.c_float, _p], C.c_int),
    "xpbd3_solve_color": ([_p, C.c_int, C.c_int, C.c_float, C.c_int, _p], C.c_int),
    "xpbd3_finalize_velocity": ([_p, C.c_float, C.c_float, _p], C.c_int),
    "xpbd3_cap_velocity": ([_p, C.c_float, _p], C.c_int),
    "xpbd3_create": ([C.POINTER(_p)], C.c_int),
    "xpbd3_destroy": ([_p], C.c_int),
    "xpbd3_bind": ([_p, _p, _p], C.c_int),
    "xpbd3_step": ([_p, C.c_int, _p], C.c_int),
    "xpbd3_status": ([_p, _ip, _p], C.c_int),
    "xpbd3_launch_info": ([_p, _ip, _ip, _ip], C.c_int),
    "xpbd3_set_driver": ([_p, C.c_int, C.c_int, C.c_int], C.c_int),
    "xpbd_color_constraints": ([C.c_int, C.c_int, _p, _p, _p], C.c_int),
    "xpbd_color_ranges": ([C.c_int, _p, _p, _p], C.c_int),
    "xpbd3_contacts_create": ([C.POINTER(_p), C.c_int, C.c_int], C.c_int),
    "xpbd3_contacts_destroy": ([_p], C.c_int),
    "xpbd3_contacts_build": ([_p, _p, _p, _p, _p, C.c_int, _p, C.c_int, _p, C.c_double, C.c_double,
                              C.c_double, _p, _p], C.c_int),
    "xpbd_barrier_selftest": ([C.c_int, C.c_int, C.c_int, _p, _p], C.c_int),
    "xpbd_phase_floor": ([C.c_int, C.c_int, C.c_int, C.c_int, _p, _p], C.c_int),
    "xpbd3_phases": ([_p, _ip, _ip], C.c_int),
    "xpbd3_rows_changed": ([_p, _p], C.c_int),
    "xpbd_color_rows_device": ([C.c_int, _p, _p, C.c_int, _p, _p, _p, _p, _p, _p], C.c_int),
    "xpbd6_phases": ([_p, _ip, _ip], C.c_int),
    "xpbd3_attach_contacts": ([_p, _p, _p, _p, _p, C.c_int, _p, C.c_int, _p, C.c_double, C.c_double,
                               C.c_double, _p], C.c_int),
    "xpbd_sort_pairs_u64": ([_p, _p, C.c_int, C.c_int, _p], C.c_int),
    "xpbd_scan_i32": ([_p, _p, C.c_int, _p, _p], C.c_int),
    "xpbd3_residual": ([_p, C.c_float, _p, C.c_int, _p, _p, _p], C.c_int),
    "xpbd6_residual": ([_p, _p, _p, C.c_int, _p, _p], C.c_int),
    "xpbd_mlp_status": ([_ip, C.c_int], C.c_int),
}

_LIB = None


def lib():
    """Load the engine library (fails loudly when it has not been built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise XpbdError(f"{LIB_PATH} is missing: build it with `python -m xpbd_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            if hasattr(L, name):
                fn = getattr(L, name)
                fn.argtypes = args
                fn.restype = res
        _LIB = L
    return _LIB


def declared_symbols():
    """Names of every function declared in include/xpbd_b200.h."""
    import re
    hdr = os.path.join(os.path.dirname(PKG), "include", "xpbd_b200.h")
    txt = open(hdr).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\*?\s+\*?(xpbd\w+)\s*\(", txt, re.M)))


def check(rc, what="xpbd call"):
    if rc != XPBD_OK:
        msg = lib().xpbd_last_error().decode() if rc == XPBD_ERR_CUDA else ""
        raise XpbdError(f"{what} failed with status {rc} {msg}".strip())
    return rc


def ptr(t):
    """Device pointer of a torch tensor as a ctypes void pointer."""
    return C.c_void_p(t.data_ptr()) if t is not None and t.numel() > 0 else C.c_void_p(0)


def stream_of(device):
    import torch
    return C.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def require_cuda(device):
    import torch
    dev = torch.device(device)
    if dev.type != "cuda":
        raise XpbdError(f"xpbd_b200 runs on CUDA devices only (got device={device!r}); "
                        "the CPU restatement of the reference lives in oracle/ and is test-only")
    if not torch.cuda.is_available():
        raise XpbdError("no CUDA device is available")
    lib()
    return dev

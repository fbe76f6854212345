"""Learned lambda warm start for the 3-DOF solver (no reference counterpart).

The reference restarts every substep from lambda = 0 (solver.py:430-431).  Here a
small MLP (7 -> 64 -> 64 -> 1, GELU, bf16 weights, fp32 accumulation), trained
by the engine's own kernels on (row features -> multiplier after 50 plain
iterations) pairs that the plain solver generates, predicts each row's
multiplier at the start of a substep.  The substep then starts from that
lambda0, with positions pre-corrected by the Jacobi-averaged M^-1 grad C^T
lambda0, instead of from lambda = 0.

The plain solve stays the fallback: in ``WarmStartRunner`` every substep runs the
first iteration both ways and keeps the plain one whenever its residual is not
worse than the learned one's.  The residual (``Solver.residual``) -- hard rows
max(0, -C), compliant rows |C + alpha~ lambda| -- is the judge of both.
"""

from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import _native as N

N_PARAM = 7 * 64 + 64 + 64 * 64 + 64 + 64 + 1
LEN = 1.0e-3  # length unit of the feature / target transforms (1 mm)


def _fn(name, args, res=C.c_int):
    f = getattr(N.lib(), name)
    f.argtypes = args
    f.restype = res
    return f


_p = C.c_void_p


def _sigs():
    return dict(
        features=_fn("xpbd3_features", [_p, C.c_float, C.c_float, C.c_float, C.c_float, _p, _p, _p]),
        infer=_fn("xpbd_mlp_infer", [_p, _p, C.c_int, _p, _p, _p]),
        grads=_fn("xpbd_mlp_grads", [_p, _p, C.c_int, _p, _p, _p, _p]),
        adam=_fn("xpbd_mlp_adam", [_p, _p, _p, _p, _p, C.c_float, C.c_int, _p]),
        warm=_fn("xpbd3_warm_start", [_p, _p, _p]),
        integrate=_fn("xpbd3_integrate", [_p, C.c_float, C.c_float, C.c_float, C.c_float, _p]),
        jacobi=_fn("xpbd3_solve_jacobi", [_p, C.c_float, C.c_int, _p]),
        apply=_fn("xpbd3_apply_jacobi", [_p, C.c_float, _p]),
        finalize=_fn("xpbd3_finalize_velocity", [_p, C.c_float, C.c_float, _p]),
        cap=_fn("xpbd3_cap_velocity", [_p, C.c_float, _p]),
    )


def slog(x):
    return np.sign(x) * np.log1p(np.abs(x))


class WarmStartMLP:
    """Weights (fp32 master + bf16 copy) and Adam state on the device."""

    def __init__(self, device="cuda:0", seed=0):
        self.device = torch.device(device)
        g = torch.Generator().manual_seed(seed)
        w = torch.zeros(N_PARAM, dtype=torch.float32)
        o = 0
        for fan_in, fan_out in ((7, 64), (64, 64), (64, 1)):
            std = math.sqrt(2.0 / fan_in)
            w[o:o + fan_in * fan_out] = torch.randn(fan_in * fan_out, generator=g) * std
            o += fan_in * fan_out + fan_out
        self.w = w.to(self.device)
        self.wb = self.w.to(torch.bfloat16)
        self.G = torch.zeros_like(self.w)
        self.M = torch.zeros_like(self.w)
        self.V = torch.zeros_like(self.w)
        self.step_count = 0
        self.F = _sigs()

    def grads(self, feats, targets):
        """Loss (mean squared error) and d(0.5 mean e^2)/dw of one batch."""
        loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        self.G.zero_()
        N.check(self.F["grads"](N.ptr(feats), N.ptr(targets), int(targets.numel()), N.ptr(self.wb),
                                N.ptr(self.G), N.ptr(loss), N.stream_of(self.device)), "xpbd_mlp_grads")
        return float(loss.item()), self.G.clone()

    def train_step(self, feats, targets, lr=1e-3):
        loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        st = N.stream_of(self.device)
        N.check(self.F["grads"](N.ptr(feats), N.ptr(targets), int(targets.numel()), N.ptr(self.wb),
                                N.ptr(self.G), N.ptr(loss), st), "xpbd_mlp_grads")
        self.step_count += 1
        N.check(self.F["adam"](N.ptr(self.w), N.ptr(self.G), N.ptr(self.M), N.ptr(self.V), N.ptr(self.wb),
                               float(lr), self.step_count, st), "xpbd_mlp_adam")
        return loss

    def infer(self, feats, weff, m, lam0):
        N.check(self.F["infer"](N.ptr(feats), N.ptr(weff), int(m), N.ptr(self.wb), N.ptr(lam0),
                                N.stream_of(self.device)), "xpbd_mlp_infer")

    def state_dict(self):
        return {"w": self.w.cpu(), "step": self.step_count}

    def load_state_dict(self, sd):
        self.w.copy_(sd["w"].to(self.device))
        self.wb.copy_(self.w.to(torch.bfloat16))
        self.step_count = int(sd.get("step", 0))


class SubstepKit:
    """Per-kernel driving of one 3-DOF solver's substep (integrate, features,
    warm start, Jacobi iterations, residual, finalize), used for data
    generation, evaluation and the warm-started frame."""

    def __init__(self, s):
        s._flush()
        self.s = s
        self.F = _sigs()
        cap = max(s._cap, 1)
        dev = s.device
        self.feats = torch.zeros((cap, 8), dtype=torch.float32, device=dev)
        self.weff = torch.zeros(cap, dtype=torch.float32, device=dev)
        self.lam0 = torch.zeros(cap, dtype=torch.float32, device=dev)
        self.h = s.dt / s.substeps

    @property
    def st(self):
        return C.byref(self.s._st)

    def stream(self):
        return N.stream_of(self.s.device)

    def integrate(self):
        g = self.s.gravity
        N.check(self.F["integrate"](self.st, float(self.h), g[0], g[1], g[2], self.stream()))

    def features(self):
        g = self.s.gravity
        N.check(self.F["features"](self.st, float(self.h), g[0], g[1], g[2], N.ptr(self.feats), N.ptr(self.weff),
                                   self.stream()))

    def iterate(self, first):
        N.check(self.F["jacobi"](self.st, float(self.h), 1 if first else 0, self.stream()))
        N.check(self.F["apply"](self.st, float(self.s.jacobi_relax), self.stream()))

    def warm(self, model):
        m = self.s._cap
        model.infer(self.feats, self.weff, m, self.lam0)
        N.check(self.F["warm"](self.st, N.ptr(self.lam0), self.stream()))
        N.check(self.F["apply"](self.st, float(self.s.jacobi_relax), self.stream()))

    def finalize(self):
        s = self.s
        N.check(self.F["finalize"](self.st, float(self.h), float(s.damping), self.stream()))
        if s.max_speed > 0.0 and math.isfinite(s.max_speed):
            N.check(self.F["cap"](self.st, float(s.max_speed), self.stream()))

    def residual(self):
        return float(self.s.residual()[0])

    def targets_from(self, lam):
        """Training target y = slog(lambda (w + alpha~) / 1 mm) per row."""
        return torch.sign(lam * self.weff) * torch.log1p(torch.abs(lam * self.weff) / LEN)


def collect(s, substeps, iters=50, every=1):
    """Generate (features, target) pairs from the plain solver: each substep
    integrates, records the features, solves with `iters` plain Jacobi
    iterations from lambda = 0, records the target from the converged lambda,
    and finalizes (so the scene keeps evolving).  Returns concatenated tensors
    of the rows the warm start acts on."""
    kit = SubstepKit(s)
    F, T = [], []
    m = int(s.tensors["n_rows"].item())
    for k in range(substeps):
        kit.integrate()
        kit.features()
        for it in range(iters):
            kit.iterate(first=(it == 0))
        if k % every == 0:
            live = kit.weff[:m] > 0
            F.append(kit.feats[:m][live].clone())
            T.append(kit.targets_from(s.tensors["lam"][:m])[live].clone())
        kit.finalize()
    return torch.cat(F), torch.cat(T)


def iterations_to_tol(s, model=None, tol=1e-4, max_iters=50):
    """From the current state, one substep: the number of Jacobi iterations the
    plain solve (lambda0 = 0) and the warm-started solve need to bring the
    residual below `tol` (max_iters + 1 if never), with the per-substep fallback
    to plain when the learned first iteration is worse.  The state is restored."""
    kit = SubstepKit(s)
    snap = s.state_dict()
    out = {}

    def run(use_model):
        s.load_state_dict(snap)
        kit.integrate()
        if use_model:
            kit.features()
            kit.warm(model)
        res = []
        for it in range(max_iters):
            kit.iterate(first=(it == 0 and not use_model))
            res.append(kit.residual())
        s.load_state_dict(snap)
        hit = [i + 1 for i, r in enumerate(res) if r < tol]
        return (hit[0] if hit else max_iters + 1), res

    out["plain"], rp = run(False)
    if model is not None:
        out["learned"], rl = run(True)
        out["fallback"] = rl[0] > rp[0]
        out["learned_with_fallback"] = out["plain"] if out["fallback"] else out["learned"]
        out["residual_first_iter"] = {"plain": rp[0], "learned": rl[0]}
    return out


class WarmStartRunner:
    """Steps a 3-DOF Jacobi solver with the learned warm start, keeping the
    plain lambda0 = 0 solve as the per-substep fallback.

    Each substep: integrate; compute the features (with the previous substep's
    multipliers); run the first iteration plain and record its residual; run it
    again from the same predicted state with the warm start and record that
    residual; keep whichever residual is smaller (ties go to plain); run the
    remaining iterations; finalize.  The whole frame is captured once as a CUDA
    graph and replayed."""

    def __init__(self, s, model):
        if s.solve_mode != "jacobi":
            raise ValueError("the warm start drives the Jacobi solve")
        self.s = s
        self.model = model
        self.kit = SubstepKit(s)
        T = s.tensors
        dev = s.device
        self.x_tilde = torch.empty_like(T["x"])
        self.x_plain = torch.empty_like(T["x"])
        self.lam_plain = torch.empty_like(T["lam"])
        self.res_p = torch.zeros(1, dtype=torch.float32, device=dev)
        self.res_l = torch.zeros(1, dtype=torch.float32, device=dev)
        self.learned_used = torch.zeros(1, dtype=torch.int32, device=dev)
        self.graph = None

    def _residual(self, out):
        N.check(N.lib().xpbd3_residual(C.byref(self.s._st), float(self.kit.h), None, 1, N.ptr(out), None,
                                       N.stream_of(self.s.device)), "xpbd3_residual")

    def _substep(self):
        kit, T = self.kit, self.s.tensors
        kit.integrate()
        kit.features()
        self.x_tilde.copy_(T["x"])
        kit.iterate(first=True)
        self._residual(self.res_p)
        self.x_plain.copy_(T["x"])
        self.lam_plain.copy_(T["lam"])
        T["x"].copy_(self.x_tilde)
        kit.warm(self.model)
        kit.iterate(first=False)
        self._residual(self.res_l)
        use_plain = self.res_p <= self.res_l
        T["x"].copy_(torch.where(use_plain, self.x_plain, T["x"]))
        T["lam"].copy_(torch.where(use_plain, self.lam_plain, T["lam"]))
        self.learned_used += (~use_plain).to(torch.int32)
        for _ in range(1, self.s.iterations):
            kit.iterate(first=False)
        kit.finalize()

    def _frame(self):
        for _ in range(self.s.substeps):
            self._substep()

    def step(self, use_graph=True):
        if not use_graph:
            self._frame()
            return
        if self.graph is None:
            side = torch.cuda.Stream(self.s.device)
            side.wait_stream(torch.cuda.current_stream(self.s.device))
            with torch.cuda.stream(side):  # warm-up launch outside capture
                snap = self.s.state_dict()
                used = self.learned_used.clone()
                self._frame()
                self.s.load_state_dict(snap)
                self.learned_used.copy_(used)
            torch.cuda.current_stream(self.s.device).wait_stream(side)
            self.graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(self.graph):
                self._frame()
        self.graph.replay()

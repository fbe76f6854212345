"""Learned lambda warm start for the 3-DOF rows and the 6-DOF contact rows (no
reference counterpart).

The reference restarts every substep from lambda = 0 (solver.py:430-431).  Here a
small MLP (7 -> 64 -> 64 -> 1, GELU, bf16 weights, fp32 accumulation), trained
by the engine's own kernels on (row features -> multiplier after 50 plain
iterations) pairs that the plain solver generates, predicts each row's
multiplier at the start of a substep.  The prediction is residual on the
previous substep's multiplier (in the transformed units: y = f3 + MLP(f)).  The substep then starts from that
lambda0, with positions pre-corrected by the Jacobi-averaged M^-1 grad C^T
lambda0, instead of from lambda = 0.

The plain solve stays the fallback: in ``WarmStartRunner`` every substep runs the
first iteration both ways and keeps the plain one whenever its residual is not
worse than the learned one's.  The residual (``Solver.residual``) -- hard rows
max(0, -C), compliant rows |C + alpha~ lambda| -- decides between them.
"""

from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np
import torch

from . import _native as N

N_PARAM = 7 * 64 + 64 + 64 * 64 + 64 + 64 + 1
LEN = 1.0e-3  # length unit of the feature / target transforms (1 mm)
PRETRAINED = os.path.join(os.path.dirname(os.path.abspath(__file__)), "warm_start_weights.npy")


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

    @classmethod
    def pretrained(cls, device="cuda:0"):
        """The shipped network: trained by ``train_warm_start`` on 10M rows from
        randomized cloths and box piles (``warm_start_weights.npy``)."""
        m = cls(device=device)
        m.load_weights(PRETRAINED)
        return m

    def save_weights(self, path):
        """fp32 master weights as a flat .npy (4737 values)."""
        np.save(path, self.w.cpu().numpy())

    def load_weights(self, path):
        w = np.load(path).astype(np.float32).reshape(-1)
        if w.size != N_PARAM:
            raise ValueError(f"{path}: {w.size} weights, expected {N_PARAM}")
        self.load_state_dict({"w": torch.from_numpy(w)})

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

    def warm(self, model=None, lam0=None):
        """lambda := lambda0 (the network's prediction, or the given per-row
        lambda0) with its Jacobi-averaged correction applied."""
        m = self.s._cap
        if lam0 is None:
            model.infer(self.feats, self.weff, m, self.lam0)
        else:
            self.lam0.copy_(lam0)
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


def collect(s, substeps, iters=50, every=1, carry="target"):
    """Generate (features, target) pairs from the plain solver: each substep
    integrates, records the features, solves with `iters` plain Jacobi
    iterations from lambda = 0 and records the target from that lambda.  With
    carry="target" the scene then finalizes from that solve, so the target is
    also the next substep's previous multiplier (feature 3); with carry="run"
    the solve is undone and the substep runs the solver's own iteration count
    (as ``step()`` does), whose multipliers become the previous ones.  Returns
    concatenated tensors of the rows the warm start acts on."""
    kit = SubstepKit(s)
    F, T = [], []
    X = s.tensors["x"]
    m = int(s.tensors["n_rows"].item())
    for k in range(substeps):
        kit.integrate()
        kit.features()
        x0 = X.clone() if carry == "run" else None
        for it in range(iters):
            kit.iterate(first=(it == 0))
        if k % every == 0:
            live = kit.weff[:m] > 0
            F.append(kit.feats[:m][live].clone())
            T.append(kit.targets_from(s.tensors["lam"][:m])[live].clone())
        if x0 is not None:
            X.copy_(x0)
            for it in range(s.iterations):
                kit.iterate(first=(it == 0))
        kit.finalize()
    return torch.cat(F), torch.cat(T)


def iterations_to_tol(s, model=None, tol=1e-4, max_iters=50, advance=False, carry_iters=50, classic=False):
    """From the current state, one substep: the number of Jacobi iterations the
    plain solve (lambda0 = 0) and the warm-started solve need to bring the
    residual below `tol` (max_iters + 1 if never) and to reach the plain solve's
    final residual, with the per-substep fallback to plain when the learned
    first iteration is worse.  The state's multipliers are the previous
    multipliers of the features.  Without `advance` the state is restored; with
    it the scene completes the substep with its normal iterations and the plain
    solve's multipliers after `carry_iters` iterations become the next
    substep's previous multipliers (the protocol ``collect`` trains on).  With
    `classic` the warm start from the previous multipliers themselves
    (lambda0 = lambda_prev) is measured as well."""
    kit = SubstepKit(s)
    snap = s.state_dict()
    out = {}
    lam_plain = None

    def first_below(res, t):
        hit = [i + 1 for i, r in enumerate(res) if r < t]
        return hit[0] if hit else max_iters + 1

    def run(use_model, lam0=None):
        nonlocal lam_plain
        s.load_state_dict(snap)
        kit.integrate()
        warm = use_model or lam0 is not None
        if warm:
            kit.features()
            kit.warm(model, lam0)
        res = []
        for it in range(max_iters):
            kit.iterate(first=(it == 0 and not warm))
            res.append(kit.residual())
            if not warm and it + 1 == min(carry_iters, max_iters):
                lam_plain = s.tensors["lam"].clone()
        s.load_state_dict(snap)
        return first_below(res, tol), res

    out["plain"], rp = run(False)
    out["residual_plain"] = rp
    if model is not None:
        out["learned"], rl = run(True)
        out["fallback"] = rl[0] > rp[0]
        out["learned_with_fallback"] = out["plain"] if out["fallback"] else out["learned"]
        out["residual_first_iter"] = {"plain": rp[0], "learned": rl[0]}
        out["residual_learned"] = rl
        out["to_plain_final"] = {"plain": first_below(rp, rp[-1] * (1 + 1e-6)),
                                 "learned": first_below(rl, rp[-1] * (1 + 1e-6))}
    if classic:
        out["classic"], rc = run(False, snap["lam"])
        out["residual_first_iter"]["classic"] = rc[0]
    if advance:
        kit.integrate()
        for it in range(s.iterations):
            kit.iterate(first=(it == 0))
        kit.finalize()
        s.tensors["lam"].copy_(lam_plain)
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
        """`model`: a ``WarmStartMLP`` (learned lambda0) or ``"previous"`` (the
        classical warm start: lambda0 = the previous substep's multipliers)."""
        if s.solve_mode != "jacobi":
            raise ValueError("the warm start drives the Jacobi solve")
        if s._self_collision:
            raise ValueError("the 3-DOF warm start needs fixed rows (the contact rows are rebuilt every frame)")
        self.s = s
        self.model = model
        self.classic = isinstance(model, str)
        if self.classic and model != "previous":
            raise ValueError(f"unknown warm start {model!r}")
        self.kit = SubstepKit(s)
        T = s.tensors
        dev = s.device
        self.x_tilde = torch.empty_like(T["x"])
        self.x_plain = torch.empty_like(T["x"])
        self.lam_plain = torch.empty_like(T["lam"])
        self.lam_prev = torch.empty_like(T["lam"])
        self.binds = getattr(s, "binds", 0)
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
        if self.classic:
            self.lam_prev.copy_(T["lam"])
        else:
            kit.features()
        self.x_tilde.copy_(T["x"])
        kit.iterate(first=True)
        self._residual(self.res_p)
        self.x_plain.copy_(T["x"])
        self.lam_plain.copy_(T["lam"])
        T["x"].copy_(self.x_tilde)
        if self.classic:
            kit.warm(lam0=self.lam_prev)
        else:
            kit.warm(self.model)
        kit.iterate(first=False)
        self._residual(self.res_l)
        # plain unless the warm start's residual is strictly smaller (ties and a
        # non-finite warm-started residual keep the plain solve)
        use_plain = ~(self.res_l < self.res_p)
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


# ---- 6-DOF contact rows ---------------------------------------------------------------
def _sigs6():
    from .solver_6dof import lib6
    L = lib6()
    for name, args in (("xpbd6_features", [_p, _p, _p, _p, _p, _p, _p]), ("xpbd6_warm_start", [_p, _p, _p, _p])):
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = C.c_int
    return L


class SubstepKit6:
    """Per-kernel driving of one ``Solver6DOF`` substep (integrate, manifold,
    features, warm start, Jacobi iterations, residual, finalize, velocity pass),
    used for data generation and evaluation of the contact-row warm start.

    Rows: the 8 n floor corner slots, then the 8 cap manifold point slots.  The
    reference's floor solve assigns (not accumulates) a corner's multiplier each
    iteration, so the kit keeps each floor slot's total impulse over the substep
    (``tot_floor``); that total is the floor rows' lambda for features and
    targets.  Run with ``plain_iterations`` iterations per substep the kit steps
    the same physics as the persistent substep kernel."""

    def __init__(self, s):
        s._flush()
        if s._sig != s._signature():
            s._bind()
        self.s = s
        self.L = _sigs6()
        self._alloc()
        self.h = s.dt / s.substeps
        self._carry = None
        self._pair_prev_pending = False  # set by broadphase, consumed by the next begin
        self.np_host = min(s.n_pairs, s.cap)
        # manifold points summed over the substeps begun (the projection count)
        self.points_dev = torch.zeros((), dtype=torch.int64, device=s.device)

    @property
    def points_total(self):
        return int(self.points_dev.item())

    def _alloc(self):
        s, dev = self.s, self.s.device
        self.n = s.num_bodies
        self.cap = s.cap
        self.nf = 8 * self.n
        self.rows = 8 * (self.n + self.cap)
        self.feats = torch.zeros((self.rows, 8), dtype=torch.float32, device=dev)
        self.weff = torch.zeros(self.rows, dtype=torch.float32, device=dev)
        self.lam0 = torch.zeros(self.rows, dtype=torch.float32, device=dev)
        self.prev_floor = torch.zeros(self.nf, dtype=torch.float32, device=dev)
        self.prev_pair = torch.zeros(8 * self.cap, dtype=torch.float32, device=dev)
        self.pair_prev = torch.zeros(8 * self.cap, dtype=torch.float32, device=dev)  # carried across a broad phase
        self.tot_floor = torch.zeros(self.nf, dtype=torch.float32, device=dev)
        self.slot = torch.arange(self.cap, dtype=torch.int32, device=dev)

    @property
    def st(self):
        return C.byref(self.s._st)

    @property
    def par(self):
        return C.byref(self.s._par)

    def stream(self):
        return N.stream_of(self.s.device)

    def broadphase(self):
        """The frame's pair list (grows the pair capacity like ``step``).  The
        pair slots' previous multipliers follow their pair into the new list
        (pairs are matched by their (a, b) key); new pairs start at 0."""
        s, T = self.s, self.s.tensors
        n_old = min(s.n_pairs, self.cap)
        old_keys = T["pairs"][:n_old].long()
        old_keys = old_keys[:, 0] * self.n + old_keys[:, 1]
        src = self._carry[self.nf:] if self._carry is not None else T["lam_pair"][: 8 * self.cap]
        old_lam = src.view(-1, 8)[:n_old].clone()
        old_keys, order = torch.sort(old_keys)  # the host grid emits in grid order
        old_lam = old_lam[order]
        N.check(self.L.xpbd6_broadphase(s._h, self.stream()), "xpbd6_broadphase")
        cnt = s.n_pairs
        if cnt > s.cap:
            s._alloc_pairs(int(cnt * 1.5))
            s._bind()
            handled = C.c_int(0)
            N.check(self.L.xpbd6_status(s._h, C.byref(handled), self.stream()), "xpbd6_status")
            N.check(self.L.xpbd6_broadphase(s._h, self.stream()), "xpbd6_broadphase")
            prev_floor = self._carry[: self.nf].clone() if self._carry is not None else self.prev_floor.clone()
            self._alloc()
            self._carry = None
            self.prev_floor.copy_(prev_floor)
        T = s.tensors
        n_new = min(s.n_pairs, self.cap)
        self.np_host = n_new
        keys = T["pairs"][:n_new].long()
        keys = keys[:, 0] * self.n + keys[:, 1]
        mapped = self.pair_prev.view(self.cap, 8)
        mapped.zero_()
        if n_old and n_new:
            idx = torch.searchsorted(old_keys, keys).clamp_(max=n_old - 1)
            hit = old_keys[idx] == keys
            mapped[:n_new][hit] = old_lam[idx[hit]]
        self._pair_prev_pending = True

    def carry(self, lam_rows):
        """Use these per-row multipliers (for example a converged solve's) as the
        next substep's previous multipliers."""
        self._carry = lam_rows.clone()

    def begin(self):
        """integrate + manifold + features of the next substep."""
        T = self.s.tensors
        if self._carry is not None:
            self.prev_floor.copy_(self._carry[: self.nf])
            self.prev_pair.copy_(self._carry[self.nf:])
            self._carry = None
        else:
            self.prev_pair.copy_(T["lam_pair"][: 8 * self.cap])
        if self._pair_prev_pending:  # first substep on a new pair list
            self.prev_pair.copy_(self.pair_prev)
            self._pair_prev_pending = False
        N.check(self.L.xpbd6_integrate(self.st, self.par, self.stream()), "xpbd6_integrate")
        N.check(self.L.xpbd6_manifold(self.st, float(self.s._man_margin), self.stream()), "xpbd6_manifold")
        # the live pairs' point counts, masked on the device (no host read, so a
        # captured substep counts the pairs of the frame it is replayed in)
        live = self.slot < T["n_pairs"].clamp(max=self.cap)
        self.points_dev += torch.where(live, T["m_hdr"][: self.cap, 0], 0).sum()
        N.check(self.L.xpbd6_features(self.st, self.par, N.ptr(self.prev_floor), N.ptr(self.prev_pair),
                                      N.ptr(self.feats), N.ptr(self.weff), self.stream()), "xpbd6_features")
        self.tot_floor.zero_()

    def iterate(self):
        T = self.s.tensors
        N.check(self.L.xpbd6_solve_positions(self.st, self.par, 0, self.stream()), "xpbd6_solve_positions")
        self.tot_floor += T["lam_floor"][: self.nf]
        N.check(self.L.xpbd6_apply_jacobi(self.st, float(self.s.jacobi_relax), self.stream()), "xpbd6_apply_jacobi")

    def warm(self, model=None, scale=1.0, lam0=None):
        """lambda := scale * lambda0 (the network's prediction, or the given
        per-row lambda0) on the rows in contact, with its correction applied."""
        T = self.s.tensors
        if lam0 is None:
            model.infer(self.feats, self.weff, self.rows, self.lam0)
        else:
            self.lam0.copy_(lam0)
        if scale != 1.0:
            self.lam0.mul_(scale)
        N.check(self.L.xpbd6_warm_start(self.st, self.par, N.ptr(self.lam0), self.stream()), "xpbd6_warm_start")
        self.tot_floor += T["lam_floor"][: self.nf]
        N.check(self.L.xpbd6_apply_jacobi(self.st, float(self.s.jacobi_relax), self.stream()), "xpbd6_apply_jacobi")

    def finish(self):
        """finalize + velocity pass; the substep's floor totals become the next
        substep's previous multipliers."""
        for name in ("xpbd6_finalize", "xpbd6_solve_velocities", "xpbd6_apply_velocity"):
            N.check(getattr(self.L, name)(self.st, self.par, self.stream()), name)
        self.prev_floor.copy_(self.tot_floor)

    def snapshot(self):
        T = self.s.tensors
        return T["x"].clone(), T["q"].clone()

    def restore(self, snap):
        """Back to the state right after ``begin`` (multipliers zero)."""
        T = self.s.tensors
        T["x"].copy_(snap[0])
        T["q"].copy_(snap[1])
        T["lam_floor"].zero_()
        T["lam_pair"].zero_()
        self.tot_floor.zero_()

    def residual(self):
        return float(self.s.residual()[0])

    def lam_rows(self):
        """Every row's multiplier: floor totals, then the manifold points'."""
        return torch.cat([self.tot_floor, self.s.tensors["lam_pair"][: 8 * self.cap]])

    def targets_from(self, lam):
        return torch.sign(lam * self.weff) * torch.log1p(torch.abs(lam * self.weff) / LEN)

    def substep(self, iterations=None):
        self.begin()
        for _ in range(self.s.iterations if iterations is None else iterations):
            self.iterate()
        self.finish()


def collect6(s, frames, iters=50, floor_gap=0.01, carry="target"):
    """(features, target) pairs from the plain solver on a box scene: the scene
    advances with its normal iteration count; at every substep the target is
    the multiplier after `iters` plain iterations from the same post-integrate
    state, and (carry="target") that multiplier is the next substep's previous
    multiplier (feature 3), or (carry="run") the multiplier of the scene's own
    iterations is, as in ``step()``.  Floor slots are kept when the corner is
    within `floor_gap` of the floor or its target is non-zero."""
    kit = SubstepKit6(s)
    F, T = [], []
    gap = float(np.log1p(floor_gap / LEN))
    for _ in range(frames):
        kit.broadphase()
        for _ in range(s.substeps):
            kit.begin()
            snap = kit.snapshot()
            for _ in range(iters):
                kit.iterate()
            lam = kit.lam_rows()
            tgt = kit.targets_from(lam)
            if carry == "target":
                kit.carry(lam)
            keep = kit.weff > 0
            keep[: kit.nf] &= (kit.feats[: kit.nf, 0] < gap) | (tgt[: kit.nf] != 0)
            F.append(kit.feats[keep].clone())
            T.append(tgt[keep].clone())
            kit.restore(snap)
            for _ in range(s.iterations):
                kit.iterate()
            kit.finish()
    return torch.cat(F), torch.cat(T)


def iterations_to_tol6(kit, model=None, tol=1e-4, max_iters=50, scale=1.0, variants=None, carry_iters=None):
    """One substep of a box scene from its current state: the residual after
    every Jacobi iteration of the plain solve (lambda0 = 0) and of the
    warm-started solve, the iterations each needs to reach `tol` (max_iters + 1
    if never) and to reach the plain solve's final residual, and the
    per-substep fallback (plain kept when the learned first iteration is worse).
    The scene then completes the substep with its normal iterations, and the
    plain solve's multipliers after `carry_iters` iterations (default
    `max_iters`) become the next substep's previous multipliers (as in
    ``collect6``)."""
    s = kit.s
    kit.begin()
    snap = kit.snapshot()

    carry_at = max_iters if carry_iters is None else min(carry_iters, max_iters)
    carried = {}

    def run(use_model, sc=scale, lam0=None):
        kit.restore(snap)
        if use_model or lam0 is not None:
            kit.warm(model, sc, lam0)
        res = []
        for k in range(max_iters):
            kit.iterate()
            res.append(kit.residual())
            if k + 1 == carry_at and not (use_model or lam0 is not None):
                carried["plain"] = kit.lam_rows().clone()
        return res

    def first_below(res, t):
        hit = [i + 1 for i, r in enumerate(res) if r < t]
        return hit[0] if hit else max_iters + 1

    out = {}
    rp = run(False)
    lam_plain = carried["plain"]
    out["plain"] = first_below(rp, tol)
    out["residual_plain"] = rp
    if model is not None:
        rl = run(True)
        out["learned"] = first_below(rl, tol)
        out["fallback"] = rl[0] > rp[0]
        out["learned_with_fallback"] = out["plain"] if out["fallback"] else out["learned"]
        target = rp[-1]
        out["to_plain_final"] = {"plain": first_below(rp, target * (1 + 1e-6)),
                                 "learned": first_below(rl, target * (1 + 1e-6))}
        out["residual_learned"] = rl
    for name, (sc, lam0_fn) in (variants or {}).items():
        rv = run(lam0_fn is None, sc, None if lam0_fn is None else lam0_fn(kit))
        out[name] = {"first": rv[0], "second": rv[1], "to_tol": first_below(rv, tol),
                     "to_plain_final": first_below(rv, rp[-1] * (1 + 1e-6)), "final": rv[-1]}
    kit.restore(snap)
    for _ in range(s.iterations):
        kit.iterate()
    kit.finish()
    kit.carry(lam_plain)
    return out


class WarmStartRunner6:
    """Steps a ``Solver6DOF`` frame with a warm-started contact solve, keeping
    the plain lambda0 = 0 solve as the per-substep fallback (decided on the
    device).

    Per frame: the broad phase (the pair slots' previous multipliers follow
    their pairs, ``SubstepKit6.broadphase``); per substep: integrate, manifold,
    features; the first iteration plain, its residual; the same first iteration
    from the same predicted state after the warm start, its residual; whichever
    residual is smaller is kept (ties go to plain); the remaining iterations;
    finalize and the velocity pass.  `model` is a ``WarmStartMLP`` (learned
    lambda0) or ``"previous"`` (lambda0 = each row's multiplier over the
    previous substep).  The same physics as the substep kernel otherwise."""

    def __init__(self, s, model):
        self.s = s
        self.model = model
        self.classic = isinstance(model, str)
        if self.classic and model != "previous":
            raise ValueError(f"unknown warm start {model!r}")
        self.kit = SubstepKit6(s)
        self.binds = getattr(s, "binds", 0)
        dev = s.device
        self.res_p = torch.zeros(1, dtype=torch.float32, device=dev)
        self.res_l = torch.zeros(1, dtype=torch.float32, device=dev)
        self.learned_used = torch.zeros(1, dtype=torch.int32, device=dev)
        self.substeps_run = 0
        self.graph = None
        self.frames_eager = 0

    def _residual(self, out):
        N.check(self.kit.L.xpbd6_residual(C.byref(self.s._st), C.byref(self.s._par), None, 1, N.ptr(out),
                                          N.stream_of(self.s.device)), "xpbd6_residual")

    def _substep(self):
        kit, T = self.kit, self.s.tensors
        kit.begin()
        snap = kit.snapshot()
        kit.iterate()
        self._residual(self.res_p)
        plain = (T["x"].clone(), T["q"].clone(), T["lam_floor"].clone(), T["lam_pair"].clone(),
                 kit.tot_floor.clone())
        kit.restore(snap)
        if self.classic:
            kit.warm(lam0=torch.cat([kit.prev_floor, kit.prev_pair]))
        else:
            kit.warm(self.model)
        kit.iterate()
        self._residual(self.res_l)
        # plain unless the warm start's residual is strictly smaller (ties and a
        # non-finite warm-started residual keep the plain solve)
        use_plain = ~(self.res_l < self.res_p)
        for cur, p in zip((T["x"], T["q"], T["lam_floor"], T["lam_pair"], kit.tot_floor), plain):
            cur.copy_(torch.where(use_plain, p, cur))
        self.learned_used += (~use_plain).to(torch.int32)
        for _ in range(1, self.s.iterations):
            kit.iterate()
        kit.finish()
        # A floor corner's impulse is carried only while the corner is still in
        # contact after the last iteration: the floor solve assigns its
        # multiplier and only pushes (kernels_6dof.py:185-193), so the substep
        # total of a corner that has lifted off is no estimate of the next
        # substep's.  (A separated manifold point's multiplier is already set
        # to 0 by its solve.)
        kit.prev_floor.mul_((T["lam_floor"][: kit.nf] != 0).to(kit.prev_floor.dtype))

    def _frame(self):
        for _ in range(self.s.substeps):
            self._substep()

    def step(self, use_graph=True):
        """The broad phase, then the frame's substeps: eager in the first frame
        (which loads every kernel), afterwards one captured CUDA graph of all
        substeps, replayed every frame.  The substeps read no host value that
        changes between frames (the pair count is masked on the device, the
        carried pair multipliers sit in a persistent buffer), so one capture
        serves every frame until the pair capacity grows or the solver is
        re-bound, which re-captures."""
        cap = self.kit.cap
        self.kit.broadphase()  # may grow the pair capacity (a re-bind the kit has absorbed)
        binds = getattr(self.s, "binds", 0)
        if binds != self.binds or self.kit.cap != cap:
            self.graph = None
        self.binds = binds
        if not use_graph or self.frames_eager == 0:
            self._frame()
            self.frames_eager += 1
        else:
            if self.graph is None:
                self.graph = torch.cuda.CUDAGraph()
                with torch.cuda.graph(self.graph):  # records only: the frame runs in the replay
                    self._frame()
            self.kit._pair_prev_pending = False  # consumed by the replayed first substep
            self.graph.replay()
        self.substeps_run += self.s.substeps

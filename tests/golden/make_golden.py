"""Generate the golden fixtures in this folder by running the REFERENCE package
(nanli9/XPBD ``src/xpbd3d``, from a checkout of the reference project) on the CPU through
``warp_shim`` (a sequential stand-in for the Warp builtins it calls).

Run once in a container that has the reference checked out:

    python tests/golden/make_golden.py --ref <reference checkout>
    XPBD_REFERENCE=<reference checkout> python tests/golden/make_golden.py

Nothing at test time reads the reference; the tests only read the ``.npz`` files
this script writes.  Every fixture records the scene parameters, the initial
state and the reference's outputs (positions, velocities, orientations,
multipliers, contact rows, colors, pair sets, manifolds).
"""

from __future__ import annotations

import argparse
import importlib.abc
import importlib.machinery
import importlib.util
import os
import re
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))  # repo root
sys.path.insert(0, HERE)

import warp_shim  # noqa: E402

from xpbd_b200 import scenes  # noqa: E402

_QUERY_LOOP = re.compile(r"while wp\.(bvh_query_next|hash_grid_query_next)\(query, j\):")


class _RefLoader(importlib.machinery.SourceFileLoader):
    def source_to_code(self, data, path, *, _optimize=-1):
        src = data.decode("utf-8") if isinstance(data, bytes) else data
        src = _QUERY_LOOP.sub("for j in query:", src)
        return compile(src, path, "exec", dont_inherit=True, optimize=_optimize)


class _RefFinder(importlib.abc.MetaPathFinder):
    def __init__(self, src_dir):
        self.src_dir = src_dir

    def find_spec(self, name, path, target=None):
        if name != "xpbd3d" and not name.startswith("xpbd3d."):
            return None
        parts = name.split(".")
        if len(parts) == 1:
            fn = os.path.join(self.src_dir, "xpbd3d", "__init__.py")
            return importlib.util.spec_from_file_location(
                name, fn, loader=_RefLoader(name, fn),
                submodule_search_locations=[os.path.join(self.src_dir, "xpbd3d")])
        fn = os.path.join(self.src_dir, *parts) + ".py"
        if not os.path.exists(fn):
            return None
        return importlib.util.spec_from_file_location(name, fn, loader=_RefLoader(name, fn))


def load_reference(ref_root):
    warp_shim.install()
    sys.meta_path.insert(0, _RefFinder(os.path.join(ref_root, "src")))
    import xpbd3d  # noqa: F401
    from xpbd3d import coloring, kernels_6dof, solver, solver_6dof
    return types.SimpleNamespace(pkg=xpbd3d, coloring=coloring, solver=solver,
                                 solver_6dof=solver_6dof, k6=kernels_6dof)


# ---------------------------------------------------------------------------
def _state3(s):
    return dict(x=s.positions().copy(), v=s.velocities().copy(), lam=s.lambdas().copy())


def _rows3(s):
    R = s._rows
    return dict(r_type=np.array([r.type for r in R], np.int32),
                r_a=np.array([r.body_a for r in R], np.int32),
                r_b=np.array([r.body_b for r in R], np.int32),
                r_rest=np.array([r.rest for r in R], np.float32),
                r_comp=np.array([r.compliance for r in R], np.float32),
                r_anchor=np.array([r.anchor for r in R], np.float32).reshape(-1, 3),
                r_mu=np.array([r.mu for r in R], np.float32))


def run3(ref, name, solver_kw, build, frames, out):
    s = ref.solver.Solver(device="cpu", **solver_kw)
    build(s)
    rec = {"x0": s.positions().copy(), "v0": s.velocities().copy()}
    xs, vs, lams, rowsets = [], [], [], []
    for f in range(frames):
        s.step()
        st = _state3(s)
        xs.append(st["x"]); vs.append(st["v"]); lams.append(st["lam"])
        rowsets.append(_rows3(s))
    rec["x"] = np.stack(xs); rec["v"] = np.stack(vs)
    # rows can change per frame (contacts) -> store per-frame ragged as concatenation
    for k in rowsets[0]:
        rec[k] = np.concatenate([r[k] for r in rowsets])
    rec["rows_per_frame"] = np.array([len(r["r_type"]) for r in rowsets], np.int32)
    rec["lam"] = np.concatenate(lams)
    rec["num_colors"] = np.int32(s.num_colors)
    for k, v in solver_kw.items():
        rec["kw_" + k] = np.asarray(v)
    out[name] = rec
    print(f"  {name}: {frames} frames, rows/frame {rec['rows_per_frame'].tolist()}")


def _state6(s):
    return dict(x=s.positions().copy(), q=s.orientations().copy(),
                v=s.velocities().copy(), w=s.omega.numpy().copy())


def run6(ref, name, solver_kw, build, frames, out):
    s = ref.solver_6dof.Solver6DOF(device="cpu", **solver_kw)
    build(s)
    s._flush()
    rec = {"x0": s.positions().copy(), "q0": s.orientations().copy(),
           "v0": s.velocities().copy(), "w0": s.omega.numpy().copy()}
    keys = ("x", "q", "v", "w")
    hist = {k: [] for k in keys}
    npairs, lam_floor, pairs = [], [], []
    for f in range(frames):
        s.step()
        st = _state6(s)
        for k in keys:
            hist[k].append(st[k])
        npairs.append(s.n_pairs)
        lam_floor.append(s.lam_floor.numpy().copy())
        n = min(s.n_pairs, s.cap)
        pa = s.pair_a.numpy()[:n].copy(); pb = s.pair_b.numpy()[:n].copy()
        pairs.append(np.stack([pa, pb], 1))
    for k in keys:
        rec[k] = np.stack(hist[k])
    rec["n_pairs"] = np.array(npairs, np.int32)
    rec["lam_floor"] = np.stack(lam_floor)
    rec["pairs"] = np.concatenate(pairs) if pairs else np.zeros((0, 2), np.int32)
    for k, v in solver_kw.items():
        rec["kw_" + k] = np.asarray(v)
    out[name] = rec
    print(f"  {name}: {frames} frames, pairs/frame {npairs}")


# ---------------------------------------------------------------------------
def chain_scene(s):
    a = s.add_particle((0.0, 2.0, 0.0), mass=0.0, collide=False)
    prev = a
    for k in range(4):
        b = s.add_particle((0.25 * (k + 1), 2.0 - 0.05 * k, 0.03 * k), mass=0.5 + 0.1 * k,
                           velocity=(0.0, 0.0, 0.4), collide=False)
        s.add_distance(prev, b, compliance=1e-5 if k % 2 else 0.0)
        prev = b
    s.add_attach(prev, (1.2, 1.5, 0.2), compliance=1e-4, rest=0.1)


def cap_scene(s):
    s.add_particle((0.0, 1.0, 0.0), mass=1.0, velocity=(80.0, 10.0, -5.0), collide=False)
    s.add_particle((0.0, 2.0, 0.0), mass=1.0, velocity=(1.0, 0.0, 0.0), collide=False)


def rand_quat(rng):
    q = rng.normal(size=4)
    return tuple(q / np.linalg.norm(q))


def floor_box_scene(s):
    rng = np.random.default_rng(3)
    s.add_box((0.1, 0.25, -0.05), (0.3, 0.15, 0.2), mass=2.0, quaternion=rand_quat(rng),
              velocity=(1.0, -2.0, 0.5), omega=(0.0, 3.0, 1.0))
    s.add_box((2.0, 0.12, 0.0), (0.1, 0.1, 0.1), mass=0.5, velocity=(-0.5, -1.0, 0.0))


def stack_scene(s):
    h = 0.2
    for k in range(4):
        s.add_box((0.01 * k, h + k * (2 * h - 0.006), -0.005 * k), (h, h, h), mass=1.0)


def pile_scene(s):
    rng = np.random.default_rng(11)
    for ly in range(2):
        for ix in range(2):
            for iz in range(2):
                e = rng.uniform(0.1, 0.3, 3)
                s.add_box((ix * 0.45, 0.25 + ly * 0.45, iz * 0.45), tuple(e),
                          float(1000.0 * 8 * e[0] * e[1] * e[2]), quaternion=rand_quat(rng),
                          omega=tuple(rng.normal(size=3)))
    s.add_box((0.2, 0.05, 0.2), (1.0, 0.05, 1.0), mass=0.0, static=True)


def joints_scene(s):
    R, sp = 4, 0.1
    idx = np.empty((R, R), np.int64)
    for iy in range(R):
        for ix in range(R):
            pinned = iy == 0
            b = s.add_particle((ix * sp, 2.0, iy * sp), mass=0.0 if pinned else 0.02,
                               radius=0.01, group=1, static=pinned)
            idx[iy, ix] = b.index
    for iy in range(R):
        for ix in range(R):
            if ix + 1 < R:
                s.add_joint(int(idx[iy, ix]), int(idx[iy, ix + 1]), compliance=1e-6)
            if iy + 1 < R:
                s.add_joint(int(idx[iy, ix]), int(idx[iy + 1, ix]), compliance=1e-6)
    anchor = s.add_box((1.0, 2.0, 0.0), (0.05, 0.05, 0.05), mass=0.0, static=True)
    bob = s.add_box((1.5, 2.0, 0.1), (0.1, 0.2, 0.1), mass=1.0,
                    quaternion=(0.0, 0.0, 0.3826834, 0.9238795))
    s.add_joint(anchor, bob, compliance=0.0, anchor_b=(0.0, 0.2, 0.0))
    bob2 = s.add_box((2.0, 1.8, 0.1), (0.1, 0.1, 0.1), mass=0.5)
    s.add_joint(bob, bob2, compliance=1e-5, rest_length=0.4,
                anchor_a=(0.0, -0.2, 0.0), anchor_b=(0.05, 0.0, 0.0))


def manifold_kernel_fixture(ref, out, n_pairs=256, seed=5):
    """Launch the reference's generate_box_manifold on random overlapping pairs."""
    wp = warp_shim
    rng = np.random.default_rng(seed)
    n = 2 * n_pairs
    x = np.zeros((n, 3), np.float32); q = np.zeros((n, 4), np.float32)
    he = rng.uniform(0.05, 0.4, (n, 3)).astype(np.float32)
    for p in range(n_pairs):
        a, b = 2 * p, 2 * p + 1
        x[a] = rng.uniform(-1, 1, 3)
        d = rng.normal(size=3); d /= np.linalg.norm(d)
        kind = p % 4
        q[a] = rand_quat(rng)
        if kind == 0:      # face-face stacking, axis aligned with tiny tilt
            q[a] = (0, 0, 0, 1)
            q[b] = (0.001 * rng.normal(), 0, 0.001 * rng.normal(), 1)
            x[b] = x[a] + np.array([0.01 * rng.normal(), he[a, 1] + he[b, 1] - 0.01, 0.0])
        else:
            q[b] = rand_quat(rng)
            dist = (np.linalg.norm(he[a]) + np.linalg.norm(he[b])) * rng.uniform(0.3, 0.9)
            x[b] = x[a] + d * dist
    q = (q / np.linalg.norm(q, axis=1, keepdims=True)).astype(np.float32)
    pa = np.arange(0, n, 2, dtype=np.int32); pb = pa + 1
    cap = n_pairs
    X = wp.array(x, dtype=wp.vec3); Q = wp.array(q, dtype=wp.quat); HE = wp.array(he, dtype=wp.vec3)
    PA = wp.array(pa, dtype=int); PB = wp.array(pb, dtype=int)
    cnt = wp.array(np.array([n_pairs], np.int32), dtype=int)
    poly = wp.zeros(cap * 16, dtype=wp.vec3)
    m_count = wp.zeros(cap, dtype=int); m_inc = wp.zeros(cap, dtype=int); m_ref = wp.zeros(cap, dtype=int)
    m_normal = wp.zeros(cap, dtype=wp.vec3)
    m_off_inc = wp.zeros(cap * 8, dtype=wp.vec3); m_off_ref = wp.zeros(cap * 8, dtype=wp.vec3)
    wp.launch(ref.k6.generate_box_manifold, dim=cap,
              inputs=[X, Q, HE, PA, PB, cnt, 0.02, poly],
              outputs=[m_count, m_inc, m_ref, m_normal, m_off_inc, m_off_ref])
    out["manifold_kernel"] = dict(x=x, q=q, he=he, pair_a=pa, pair_b=pb, margin=np.float32(0.02),
                                  m_count=m_count.numpy().copy(), m_inc=m_inc.numpy().copy(),
                                  m_ref=m_ref.numpy().copy(), m_normal=m_normal.numpy().copy(),
                                  m_off_inc=m_off_inc.numpy().copy(), m_off_ref=m_off_ref.numpy().copy())
    print(f"  manifold_kernel: {n_pairs} pairs, points {int(m_count.numpy().sum())}")


def host_fixtures(ref, out):
    # coloring on the 32 x 32 cloth rows and on random graphs (reference test style)
    s = ref.solver.Solver(device="cpu", solve_mode="gs", substeps=15, iterations=2)
    scenes.build_cloth(s)
    a = np.array([r.body_a for r in s._rows], np.int32)
    b = np.array([r.body_b for r in s._rows], np.int32)
    col = ref.coloring.color_constraints(s.num_bodies, a, b)
    order, starts, k = ref.coloring.color_ranges(col)
    out["coloring_cloth32"] = dict(n_bodies=np.int32(s.num_bodies), a=a, b=b, color=col,
                                   order=order, starts=starts)
    print(f"  coloring_cloth32: {len(a)} rows, {k} colors")
    for seed in range(4):
        rng = np.random.default_rng(seed)
        nb = 40 + 20 * seed
        m = 200 + 100 * seed
        ra = rng.integers(0, nb, m)
        rb = rng.integers(0, nb, m)
        rb = np.where(rb == ra, (rb + 1) % nb, rb)
        if seed >= 2:
            rb = np.where(rng.random(m) < 0.2, -1, rb)
        col = ref.coloring.color_constraints(nb, ra, rb)
        order, starts, k = ref.coloring.color_ranges(col)
        out[f"coloring_rand{seed}"] = dict(n_bodies=np.int32(nb), a=ra.astype(np.int32),
                                           b=rb.astype(np.int32), color=col, order=order,
                                           starts=starts)
    # sphere self-collision contact rows on the 2048-sphere pile (first frame)
    s = ref.solver.Solver(device="cpu", solve_mode="jacobi", substeps=15, iterations=2)
    scenes.build_sphere_pile(s)
    s._flush()
    x0 = s.positions().copy()
    s._rebuild_contacts()
    rows = [r for r in s._rows if r.type == ref.solver.CONTACT]
    out["sphere_contacts_2048"] = dict(
        x0=x0, a=np.array([r.body_a for r in rows], np.int32),
        b=np.array([r.body_b for r in rows], np.int32),
        rest=np.array([r.rest for r in rows], np.float32),
        mu=np.array([r.mu for r in rows], np.float32))
    print(f"  sphere_contacts_2048: {len(rows)} contact rows")
    # 6-DOF pair sets on the 1440-box pile (all three broad phases, first frame)
    for bp in ("lbvh", "hashgrid", "grid"):
        s6 = ref.solver_6dof.Solver6DOF(device="cpu", substeps=15, iterations=2, floor_y=0.0,
                                        friction=0.6, restitution=0.2, broadphase=bp)
        scenes.build_box_pile(s6)
        s6._flush()
        if bp == "lbvh":
            cnt = s6._broadphase_gpu(s6.num_bodies)
            pa = s6.pair_a.numpy()[:cnt].copy(); pb = s6.pair_b.numpy()[:cnt].copy()
            lo = s6.lowers.numpy().copy(); hi = s6.uppers.numpy().copy()
        elif bp == "hashgrid":
            cnt = s6._broadphase_hashgrid(s6.num_bodies)
            pa = s6.pair_a.numpy()[:cnt].copy(); pb = s6.pair_b.numpy()[:cnt].copy()
        else:
            pa, pb = s6._rebuild_pairs()
        rec = dict(a=np.asarray(pa, np.int32), b=np.asarray(pb, np.int32))
        if bp == "lbvh":
            rec.update(lowers=lo, uppers=hi, x0=s6.positions().copy(), q0=s6.orientations().copy(),
                       he=np.asarray(s6._he, np.float32), inv_mass=np.asarray(s6._inv_mass, np.float32),
                       inv_I=np.asarray(s6._inv_I, np.float32))
            he = np.asarray(s6._he, np.float32)
            rec["aabb_half"] = ref.solver_6dof._world_aabb_half(s6.q.numpy(), he)
        out[f"pairs1440_{bp}"] = rec
        print(f"  pairs1440_{bp}: {len(pa)} pairs")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("XPBD_REFERENCE"),
                    help="root of the reference checkout (default: $XPBD_REFERENCE)")
    ap.add_argument("--only", default=None)
    args = ap.parse_args()
    if not args.ref:
        ap.error("give the reference checkout with --ref or XPBD_REFERENCE")
    ref = load_reference(args.ref)
    out = {}
    jobs = {
        "host": lambda: host_fixtures(ref, out),
        "manifold": lambda: manifold_kernel_fixture(ref, out),
        "cloth": lambda: [run3(ref, f"cloth6_{m}", dict(dt=1 / 60, substeps=15, iterations=2, solve_mode=m,
                                                         damping=0.01, jacobi_relax=1.0),
                               lambda s: scenes.build_cloth(s, res=6, spacing=0.05, y=0.004,
                                                            compliance=1e-6,
                                                            velocity=(0.3, -1.0, 0.2)), 5, out)
                          for m in ("gs", "jacobi")],
        "spheres": lambda: [run3(ref, f"spheres18_{m}", dict(dt=1 / 60, substeps=15, iterations=2,
                                                             solve_mode=m),
                                 lambda s: scenes.build_sphere_pile(s, nx=3, ny=2, nz=3, pitch=0.095,
                                                                    y0=0.06, margin=0.01, seed=4),
                                 4, out) for m in ("gs", "jacobi")],
        "chain": lambda: [run3(ref, f"chain_{m}", dict(dt=1 / 60, substeps=10, iterations=3, solve_mode=m,
                                                       damping=0.02, jacobi_relax=0.8),
                               chain_scene, 5, out) for m in ("gs", "jacobi")],
        "cap": lambda: run3(ref, "cap", dict(dt=1 / 60, substeps=4, iterations=1, solve_mode="jacobi"),
                            cap_scene, 2, out),
        "floorbox": lambda: run6(ref, "floorbox", dict(dt=1 / 60, substeps=15, iterations=2, floor_y=0.0,
                                                       friction=0.6, restitution=0.3, lin_damp=0.01,
                                                       ang_damp=0.02), floor_box_scene, 5, out),
        "stack": lambda: run6(ref, "stack", dict(dt=1 / 60, substeps=15, iterations=2, floor_y=0.0,
                                                 friction=0.6), stack_scene, 3, out),
        "pile": lambda: [run6(ref, f"pile_{bp}", dict(dt=1 / 60, substeps=15, iterations=2, floor_y=0.0,
                                                       friction=0.6, restitution=0.2, gyroscopic=True,
                                                       broadphase=bp, max_omega=20.0),
                              pile_scene, 3, out) for bp in ("lbvh", "hashgrid", "grid")],
        "joints": lambda: run6(ref, "joints", dict(dt=1 / 60, substeps=12, iterations=2, floor_y=-100.0,
                                                   jacobi_relax=0.9), joints_scene, 4, out),
    }
    for name, job in jobs.items():
        if args.only and name not in args.only.split(","):
            continue
        job()
    for name, rec in out.items():
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **rec)
    print("wrote", len(out), "fixtures")


if __name__ == "__main__":
    main()

"""Batched independent scenes of uneven size, stepped together.

The workload (no reference counterpart): N scenes drawn from a seed, half
cloths of n x n particles (n ~ U{16..128}, the 32 x 32 cloth's spacing, mass,
compliance, pins and floor), half box piles of k boxes (k ~ U{64..1024}, the
1440-box pile's size, density and orientation distributions on a near-cubic
0.8 m lattice).

All cloths are packed into ONE 3-DOF system and all piles into ONE 6-DOF
system.  Scenes never interact:
* cloth rows only join particles of their own cloth, and each cloth is colored
  on its own (``Solver.color_groups``), so in Gauss-Seidel mode every scene is
  projected in exactly the order it would be alone;
* piles carry a scene id per body; the LBVH keys carry the scene id above the
  Morton bits, so every scene is one subtree and each body's query starts at
  its own scene's subtree root -- no cross-scene traversal, no cross-scene pair.
Each system then runs one persistent launch per frame (the piles' broad phase
and substeps replayed as one CUDA graph), so a frame of all scenes is two
launch sequences however many scenes there are.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import scenes
from .solver import Solver
from .solver_6dof import Solver6DOF


@dataclass
class SceneSpec:
    kind: str      # "cloth" or "pile"
    size: int      # cloth side n or pile box count k
    seed: int


def batch_specs(n_scenes=256, seed=0, cloth_range=(16, 128), pile_range=(64, 1024)):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_scenes):
        if i % 2 == 0:
            out.append(SceneSpec("cloth", int(rng.integers(cloth_range[0], cloth_range[1] + 1)), i))
        else:
            out.append(SceneSpec("pile", int(rng.integers(pile_range[0], pile_range[1] + 1)), i))
    return out


def build_pile_k(s, k, seed, pitch=0.8, y0=0.5):
    """k boxes on a near-cubic lattice (side = ceil(k^(1/3))), filled y-major."""
    side = int(np.ceil(k ** (1.0 / 3.0) - 1e-9))
    rng = np.random.default_rng(seed)
    placed = 0
    for ly in range(side):
        for ix in range(side):
            for iz in range(side):
                if placed == k:
                    return
                e = rng.uniform(0.1, 0.3, 3)
                q = rng.normal(size=4)
                q = q / np.linalg.norm(q)
                s.add_box((ix * pitch, y0 + ly * pitch, iz * pitch), tuple(e),
                          float(1000.0 * 8.0 * e[0] * e[1] * e[2]), quaternion=tuple(q))
                placed += 1


def build_cloth_scene(s, n):
    scenes.build_cloth(s, res=n)


CLOTH_KW = dict(dt=1 / 60, substeps=15, iterations=2)
PILE_KW = dict(dt=1 / 60, substeps=15, iterations=2, floor_y=0.0, friction=0.6, restitution=0.2, broadphase="lbvh")


@dataclass
class BatchLayout:
    """Where each scene of a (possibly partial) batch sits in the two packed
    systems: global scene ids, body ranges and cloth row ranges."""
    cloth_ids: list
    pile_ids: list
    cloth_bodies: list   # (b0, b1) per cloth scene, in the 3-DOF system
    cloth_rows: list     # (r0, r1) per cloth scene
    pile_bodies: list    # (b0, b1) per pile scene, in the 6-DOF system


def build_batch(specs, scene_ids, cloth, piles) -> BatchLayout:
    """Add the scenes `scene_ids` (global indices into `specs`, ascending) to a
    3-DOF solver `cloth` and a 6-DOF solver `piles` through the public
    scene-building API.  Each pile is opened as its own scene when the solver
    supports scene ids (``begin_scene``), so no pair ever joins two scenes."""
    lay = BatchLayout([], [], [], [], [])
    pile_scene = 0
    for i in scene_ids:
        sp = specs[i]
        if sp.kind == "cloth":
            b0, r0 = cloth.num_bodies, cloth.num_constraints
            build_cloth_scene(cloth, sp.size)
            lay.cloth_ids.append(i)
            lay.cloth_bodies.append((b0, cloth.num_bodies))
            lay.cloth_rows.append((r0, cloth.num_constraints))
        else:
            b0 = piles.num_bodies
            if hasattr(piles, "begin_scene"):
                piles.begin_scene(pile_scene)
            build_pile_k(piles, sp.size, sp.seed)
            lay.pile_ids.append(i)
            lay.pile_bodies.append((b0, piles.num_bodies))
            pile_scene += 1
    return lay


def rank_scene_ids(specs, rank: int, world: int):
    """The scenes one rank of `world` steps: LPT bin packing of the scenes'
    projection counts (``shard.lpt_partition``), so every scene is stepped by
    exactly one rank and the ranks' loads are balanced."""
    from .shard import lpt_partition, scene_cost
    if world <= 1:
        return list(range(len(specs)))
    return lpt_partition([scene_cost(sp) for sp in specs], world)[rank]


class BatchedScenes:
    def __init__(self, specs, device="cuda:0", cloth_mode="gs", substeps=15, iterations=2, scene_ids=None):
        """`scene_ids`: the global indices of the scenes this instance steps (a
        rank's share of a sharded batch, see ``rank_scene_ids``); None = all."""
        self.specs = list(specs)
        self.scene_ids = list(range(len(self.specs))) if scene_ids is None else sorted(int(i) for i in scene_ids)
        self.device = device
        self.cloth_mode = cloth_mode
        kw3 = dict(CLOTH_KW, substeps=substeps, iterations=iterations)
        kw6 = dict(PILE_KW, substeps=substeps, iterations=iterations)
        self.cloth = Solver(device=device, solve_mode=cloth_mode, **kw3)
        self.piles = Solver6DOF(device=device, **kw6)
        self.piles.sync_pairs = False
        lay = build_batch(self.specs, self.scene_ids, self.cloth, self.piles)
        self.layout = lay
        self.cloth_ids, self.pile_ids = lay.cloth_ids, lay.pile_ids
        self.cloth_rows, self.cloth_bodies, self.pile_bodies = lay.cloth_rows, lay.cloth_bodies, lay.pile_bodies
        groups = list(lay.cloth_rows)
        self.cloth.color_groups = groups
        self.has_cloth = self.cloth.num_bodies > 0
        self.has_piles = self.piles.num_bodies > 0
        if self.has_cloth:
            self.cloth._flush()
        if self.has_piles:
            self.piles._flush()
        row_scene = np.zeros(max(len(self.cloth._rows), 1), np.int32)
        for k, (r0, r1) in enumerate(self.cloth_rows):
            row_scene[r0:r1] = k
        cap = self.cloth._cap
        rs = np.zeros(cap, np.int32)
        rs[:len(row_scene)] = row_scene[:cap]
        self.row_scene = torch.from_numpy(rs).to(device)
        self.body_scene = (self.piles.tensors["scene"] if self.has_piles and self.piles.n_scenes > 1 else None)
        self.stream_piles = torch.cuda.Stream(device)

    def autotune(self, frames=2):
        out = {}
        if self.has_cloth:
            out["cloth"] = self.cloth.autotune(frames)
        if self.has_piles:
            out["piles"] = self.piles.autotune(frames)
        return out

    def step(self):
        """One frame of every scene: cloths on the current stream, piles on a
        second stream, joined before returning."""
        cur = torch.cuda.current_stream(self.device)
        self.stream_piles.wait_stream(cur)
        if self.has_cloth:
            self.cloth.step()
        if self.has_piles:
            with torch.cuda.stream(self.stream_piles):
                self.piles.step()
        cur.wait_stream(self.stream_piles)

    def projections_per_frame(self):
        """Projections of one frame with the manifold points of the last substep
        (an estimate; ``projections`` counts every substep)."""
        S, I = self.cloth.substeps, self.cloth.iterations
        n3 = self.cloth.num_constraints if self.has_cloth else 0
        if not self.has_piles:
            return n3 * S * I
        T = self.piles.tensors
        n_dyn = int((T["x"][:, 3] > 0).sum().item())
        hdr = T["m_hdr"][:min(self.piles.n_pairs, self.piles.cap)].cpu().numpy()
        n6 = 8 * n_dyn + int(hdr[:, 0].sum()) + self.piles.num_joints
        return (n3 + n6) * S * I

    def reset_projection_count(self):
        if self.has_piles:
            self.piles.manifold_points(reset=True)

    def projections(self, frames):
        """Projections of the last `frames` frames since ``reset_projection_count``:
        cloth rows x S x I per frame, and per pile substep I x (8 floor slots per
        dynamic body + that substep's manifold points + joints), the points
        counted on the device (synchronizes)."""
        S, I = self.cloth.substeps, self.cloth.iterations
        total = frames * S * I * (self.cloth.num_constraints if self.has_cloth else 0)
        if self.has_piles:
            T = self.piles.tensors
            n_dyn = int((T["x"][:, 3] > 0).sum().item())
            total += I * (frames * S * (8 * n_dyn + self.piles.num_joints) + self.piles.manifold_points())
        return total

    def residuals(self):
        """Max residual per scene, indexed like `specs` (NaN for scenes this
        instance does not hold)."""
        out = np.full(len(self.specs), np.nan, np.float32)
        rc = self.cloth.residual(self.row_scene, len(self.cloth_ids)) if self.has_cloth else []
        rp = self.piles.residual(self.body_scene, max(len(self.pile_ids), 1)) if self.has_piles else []
        for k, i in enumerate(self.cloth_ids):
            out[i] = rc[k]
        for k, i in enumerate(self.pile_ids):
            out[i] = rp[k]
        return out

    def scene_positions(self, i):
        if i in self.cloth_ids:
            b0, b1 = self.cloth_bodies[self.cloth_ids.index(i)]
            return self.cloth.positions()[b0:b1]
        b0, b1 = self.pile_bodies[self.pile_ids.index(i)]
        return self.piles.positions()[b0:b1]

    def solo(self, i):
        """Scene i built alone in its own solver (same parameters)."""
        sp = self.specs[i]
        if sp.kind == "cloth":
            s = Solver(device=self.device, solve_mode=self.cloth_mode,
                       **dict(CLOTH_KW, substeps=self.cloth.substeps, iterations=self.cloth.iterations))
            build_cloth_scene(s, sp.size)
        else:
            s = Solver6DOF(device=self.device,
                           **dict(PILE_KW, substeps=self.piles.substeps, iterations=self.piles.iterations))
            s.sync_pairs = False
            build_pile_k(s, sp.size, sp.seed)
        return s

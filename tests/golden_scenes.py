"""The small scenes the golden fixtures were recorded on (same builders as
``tests/golden/make_golden.py``), plus helpers to rebuild a solver from a
fixture's recorded constructor arguments."""

import numpy as np

from xpbd_b200 import scenes
import make_golden as MG

SCENES3 = {
    "cloth6": (lambda s: scenes.build_cloth(s, res=6, spacing=0.05, y=0.004, compliance=1e-6,
                                            velocity=(0.3, -1.0, 0.2)), 5),
    "spheres18": (lambda s: scenes.build_sphere_pile(s, nx=3, ny=2, nz=3, pitch=0.095, y0=0.06,
                                                     margin=0.01, seed=4), 4),
    "chain": (MG.chain_scene, 5),
}
SCENES6 = {
    "floorbox": (MG.floor_box_scene, 5),
    "stack": (MG.stack_scene, 3),
    "pile_lbvh": (MG.pile_scene, 3),
    "pile_hashgrid": (MG.pile_scene, 3),
    "pile_grid": (MG.pile_scene, 3),
    "joints": (MG.joints_scene, 4),
}


def kwargs(rec):
    out = {}
    for k, v in rec.items():
        if k.startswith("kw_"):
            out[k[3:]] = v.item() if np.ndim(v) == 0 else tuple(v.tolist())
    return out


def fixtures3():
    out = []
    for base, (build, frames) in SCENES3.items():
        for mode in ("gs", "jacobi"):
            out.append((f"{base}_{mode}", build, frames))
    out.append(("cap", MG.cap_scene, 2))
    return out


def fixtures6():
    return [(name, build, frames) for name, (build, frames) in SCENES6.items()]

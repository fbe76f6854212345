"""Scene-building handles (mirror src/xpbd3d/scene.py:18-43 of the reference).

``Body.shape`` is render metadata; for a ``"sphere"`` it also gives the collision
radius used by sphere-sphere self collision (``_shape_radius``).
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Literal


@dataclass
class Shape:
    kind: Literal["sphere", "cube", "pillar"] = "sphere"
    size: tuple = (0.1,)
    color: tuple = (0.4, 0.6, 0.9)


@dataclass
class Body:
    index: int
    shape: Shape = field(default_factory=Shape)


@dataclass
class ConstraintHandle:
    index: int
    rows: int = 1


def shape_radius(shape: Shape | None) -> float:
    """Bounding-sphere radius for the sphere broad phase (solver.py:565-575)."""
    if shape is None:
        return 0.0
    if shape.kind == "sphere":
        return float(shape.size[0])
    if shape.kind == "cube":
        return float(min(shape.size))
    if shape.kind == "pillar":
        return float(shape.size[0])
    return 0.0

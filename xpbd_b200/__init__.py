"""xpbd_b200 -- B200-native XPBD substep engine.

Drop-in for the hot path of nanli9/XPBD (package ``xpbd3d``): the ``Solver``
(3-DOF particles) and ``Solver6DOF`` (rigid boxes, particles, joints) classes
with the reference's constructor arguments, scene-building calls and
``step()``, backed by hand-written sm_100a CUDA behind a C ABI
(``include/xpbd_b200.h``, ``libxpbd_b200.so``).
"""

from .scene import Body, ConstraintHandle, Shape
from .solver import ATTACH, CONTACT, DISTANCE, FLOOR, Solver
from .solver_6dof import RigidBody, Solver6DOF

__all__ = ["Solver", "Solver6DOF", "RigidBody", "Body", "Shape", "ConstraintHandle",
           "DISTANCE", "ATTACH", "FLOOR", "CONTACT"]

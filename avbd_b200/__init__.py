"""B200 (sm_100a) implementation of the AVBD Solver6DOF substep.

Drop-in for the reference `avbd3d.Solver6DOF` (nanli9/AVBD,
src/avbd3d/solver_6dof.py): same constructor, scene API and getters; the
substep runs in the hand-written CUDA library `libavbd6.so` (C ABI in
include/avbd6.h).
"""

from .solver import (BOX_BOX_CONTACT_6DOF, CONTACT_TANGENT_6DOF, FLOOR_CONTACT_6DOF, PIN_6DOF, RigidBody,
                     Solver6DOF, _obb_sat, box_inertia_local, box_inv_inertia_local)

__all__ = ["Solver6DOF", "RigidBody", "FLOOR_CONTACT_6DOF", "CONTACT_TANGENT_6DOF", "PIN_6DOF",
           "BOX_BOX_CONTACT_6DOF", "box_inertia_local", "box_inv_inertia_local", "_obb_sat"]

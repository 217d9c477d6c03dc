"""B200-native meshless hydro pass (GIZMO density -> gradients -> MFM/MFV force).

The compute path is the sm_100a C-ABI library built from gizmo_b200/csrc/
(include/gizmo_hydro.h); ``gizmo_b200.hydro.HydroPass`` mirrors the
reference's density() / hydro_gradient_calc() / hydro_force() entry points.
"""
from . import abi  # noqa: F401

__all__ = ["abi", "hydro", "ics"]

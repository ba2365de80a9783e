"""B200-native geodesic hot path of BlackHorizon.

A ``b200`` backend for the reference's Kerr-Schild ray tracer: the same
``KerrSpacetime``, ``geodesic_rhs``, ``dormand_prince_step``, ``trace_rays``
and ``PinholeCamera`` call signatures (MegaKruk/BlackHorizon, blackhorizon/
kerr.py, geodesics.py, integrators.py, tracer.py, camera.py), with every
computation in hand-written sm_100a CUDA kernels behind the C ABI of
include/bh_b200.h (libbh_b200.so, loaded with ctypes).
"""

from .backend import b200_available, get_xp, gpu_available, to_numpy, xp_of
from .camera import PinholeCamera
from .geodesics import (GeodesicRhs, build_state, conserved_quantities,
                        coordinate_velocity, geodesic_rhs, hamiltonian,
                        null_momentum_from_velocity, timelike_momentum)
from .integrators import (dormand_prince_step, error_ratio, implicit_midpoint_step,
                          integrate_dense, propagate, rk4_step, step_factor)
from .kerr import KerrSchildGeometry, KerrSpacetime
from .tracer import CameraBatch, CameraScene, RayStatus, TraceResult, trace_cameras, trace_rays

__all__ = [
    "b200_available", "get_xp", "gpu_available", "to_numpy", "xp_of",
    "PinholeCamera", "GeodesicRhs", "build_state", "conserved_quantities",
    "coordinate_velocity", "geodesic_rhs", "hamiltonian",
    "null_momentum_from_velocity", "timelike_momentum", "dormand_prince_step",
    "error_ratio", "implicit_midpoint_step", "integrate_dense", "propagate", "rk4_step",
    "step_factor",
    "KerrSchildGeometry", "KerrSpacetime", "CameraBatch", "CameraScene", "RayStatus",
    "TraceResult", "trace_cameras", "trace_rays",
]

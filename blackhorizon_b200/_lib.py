"""ctypes binding of libbh_b200.so (the C ABI in include/bh_b200.h).

The library is built in-tree by ``python -m blackhorizon_b200.build`` (or
``__graft_entry__.build()``).  Loading fails loudly: there is no CPU or
PyTorch fallback for any compute call of this package.
"""

from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbh_b200.so")

# bh_status (include/bh_b200.h)
BH_OK = 0
BH_ERR_INVALID_ARGUMENT = -1
BH_ERR_CUDA = -2
BH_ERR_TIMEOUT = -3
BH_ERR_ESCAPE_RADIUS = -4
BH_ERR_WORKSPACE = -5
BH_ERR_TAPE = -6

PRECISION = {"fp64": 0, "mixed": 1}
LAYOUT = {"aos": 0, "soa": 1}
TRACE_INTERIOR = 1  # bh_trace_flag BH_TRACE_INTERIOR

_D = ctypes.c_double
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
_P = ctypes.c_void_p
_SZ = ctypes.c_size_t


class Scene(ctypes.Structure):
    _fields_ = [("mass", _D), ("spin", _D), ("capture_radius", _D),
                ("escape_radius", _D)]


class Camera(ctypes.Structure):
    _fields_ = [("position", _D * 3), ("forward", _D * 3), ("right", _D * 3),
                ("up", _D * 3), ("fov_degrees", _D), ("width", _I64),
                ("height", _I64), ("scene", Scene)]


class TraceConfig(ctypes.Structure):
    _fields_ = [("max_steps", _I64), ("rtol", _D), ("atol", _D),
                ("initial_step", _D), ("max_step", _D), ("min_step", _D),
                ("precision", _I32), ("layout", _I32), ("timeout_ns", _I64),
                ("variant", _I32), ("blocks_per_sm", _I32), ("project_every", _I32),
                ("flags", _I32), ("reserved", _I32), ("f64_radius", _D)]


class TraceStats(ctypes.Structure):
    _fields_ = [("iterations", _I64), ("attempts", _I64), ("accepted", _I64),
                ("timed_out", _I32), ("bad_rays", _I32)]


class TileStats(ctypes.Structure):
    _fields_ = [("iterations", _I64), ("attempts", _I64), ("accepted", _I64),
                ("crossings", _I64), ("disk_hits", _I64), ("rounds", _I32),
                ("timed_out", _I32)]


class RealtimeConfig(ctypes.Structure):
    _fields_ = [("max_steps", _I64), ("step_scale", _D), ("min_step", _D), ("max_step", _D),
                ("capture_margin", _D), ("momentum_bailout", _D), ("escape_radius", _D),
                ("disk_inner", _D), ("disk_outer", _D), ("interior_stop", _D),
                ("precision", _I32), ("reserved", _I32)]


class RealtimeShading(ctypes.Structure):
    _fields_ = [("mass", _D), ("spin", _D), ("disk_inner", _D), ("disk_outer", _D),
                ("disk_temperature", _D), ("disk_detail", _D), ("exposure", _D),
                ("observer_lapse", _D), ("bb_log_min", _D), ("bb_log_max", _D),
                ("sky_amplification", _D), ("sheet_radiance", _D), ("whiteout", _D),
                ("background", _I32), ("temperature_size", _I32), ("blackbody_size", _I32),
                ("reserved", _I32)]


class OfflineCamera(ctypes.Structure):
    _fields_ = [("position", _D * 3), ("basis", (_D * 3) * 3), ("tetrad", (_D * 4) * 4),
                ("tan_half", _D), ("tan_half_aspect", _D), ("width", _I64), ("height", _I64),
                ("supersample", _I32), ("use_tetrad", _I32)]


class EmissionConfig(ctypes.Structure):
    _fields_ = [("mass", _D), ("spin", _D), ("disk_inner", _D), ("disk_temperature", _D),
                ("disk_detail", _D), ("observer_lapse", _D), ("bb_log_min", _D),
                ("bb_log_max", _D), ("sheet_rgb", _D * 3), ("temperature_size", _I32),
                ("blackbody_size", _I32), ("supersample", _I32), ("reserved", _I32)]


class Vaidya(ctypes.Structure):
    _fields_ = [("mass", _D), ("charge", _D), ("tail_mass", _D), ("tail_start", _D),
                ("tail_power", _D), ("shell_energy", _D), ("shell_start_v", _D),
                ("shell_start_radius", _D), ("shell_width", _D), ("mass_cap", _D),
                ("shell_v", _P), ("shell_r", _P), ("shell_m2", _P), ("n_shell", _I64)]


_SIGNATURES = {
    "bh_abi_version": (ctypes.c_int, []),
    "bh_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "bh_last_error": (ctypes.c_char_p, []),
    "bh_geometry": (ctypes.c_int, [_D, _D, _P, _P, _P, _I64, _I64, _P, _P, _P, _P, _P, _P]),
    "bh_geodesic_rhs": (ctypes.c_int, [_D, _D, _P, _P, _I64, _P]),
    "bh_hamiltonian": (ctypes.c_int, [_D, _D, _P, _P, _I64, _P]),
    "bh_coordinate_velocity": (ctypes.c_int, [_D, _D, _P, _P, _I64, _P]),
    "bh_null_momentum": (ctypes.c_int, [_D, _D, _P, _P, _P, _I64, _I32, _I32, _P, _P]),
    "bh_camera_states": (ctypes.c_int, [ctypes.POINTER(Camera), _P, _P]),
    "bh_dp5_step": (ctypes.c_int, [_D, _D, _P, _P, _P, _P, _I64, _I32, _P]),
    "bh_error_ratio": (ctypes.c_int, [_P, _P, _P, _D, _D, _P, _I64, _P]),
    "bh_step_factor": (ctypes.c_int, [_P, _P, _I64, _P]),
    "bh_device_math": (ctypes.c_int, [_I32, _P, _P, _I64, _P]),
    "bh_rk4": (ctypes.c_int, [_D, _D, _P, _P, _P, _I64, _I64, _I32, _P]),
    "bh_implicit_midpoint": (ctypes.c_int, [_D, _D, _P, _P, _P, _I64, _I32, _I64, _P]),
    "bh_trace_variant_count": (ctypes.c_int, [_I32]),
    "bh_trace_variant": (ctypes.c_int, [_I32, _I32, ctypes.POINTER(_I32),
                                         ctypes.POINTER(_I32), ctypes.POINTER(_I32),
                                         ctypes.POINTER(_I32), ctypes.POINTER(_I32)]),
    "bh_trace_workspace_bytes": (_SZ, []),
    "bh_trace": (ctypes.c_int, [ctypes.POINTER(TraceConfig), ctypes.POINTER(Scene),
                                _P, _P, _P, _P, _I64, _P, _P]),
    "bh_trace_cameras_workspace_bytes": (_SZ, [_I32]),
    "bh_camera_table_upload": (ctypes.c_int, [ctypes.POINTER(Camera), _I32, _P, _SZ,
                                              ctypes.POINTER(_I64), _P]),
    "bh_trace_cameras": (ctypes.c_int, [ctypes.POINTER(TraceConfig), _I32, _I64, _P,
                                        _P, _P, _P, _SZ, _P]),
    "bh_trace_stats_read": (ctypes.c_int, [_P, ctypes.POINTER(TraceStats), _P]),
    "bh_trace_cameras_noalloc": (ctypes.c_int, [ctypes.POINTER(TraceConfig),
                                                ctypes.POINTER(Camera), _I32, _P, _P, _P,
                                                ctypes.POINTER(TraceStats), _P]),
    "bh_propagate": (ctypes.c_int, [ctypes.POINTER(TraceConfig), _D, _D, _P, _P, _P,
                                    _P, _P, _I64, _I64, _P, _P]),
    "bh_propagate_ordered": (ctypes.c_int, [ctypes.POINTER(TraceConfig), _D, _D, _P, _P, _P,
                                            _P, _P, _P, _I64, _I64, _P, _P]),
    "bh_propagate_order_workspace_bytes": (_SZ, [_I64]),
    "bh_propagate_order": (ctypes.c_int, [_P, _I32, _I64, _P, _P, _SZ, _P]),
    "bh_graph_trace_cameras": (ctypes.c_int, [ctypes.POINTER(TraceConfig), _I32, _I64, _P,
                                              _P, _P, _P, _SZ, ctypes.POINTER(_P)]),
    "bh_graph_launch": (ctypes.c_int, [_P, _P]),
    "bh_graph_destroy": (ctypes.c_int, [_P]),
    "bh_trace_tape": (ctypes.c_int, [ctypes.POINTER(TraceConfig), ctypes.POINTER(Scene),
                                     _P, _P, _P, _P, _I64, _P, _P, _I64, _I32, _P, _P]),
    "bh_adjoint": (ctypes.c_int, [_I32, _D, _D, _P, _P, _P, _I64, _I32, _P, _P, _P, _P, _I64,
                                  _P]),
    "bh_replay": (ctypes.c_int, [_I32, _D, _D, _P, _P, _P, _I64, _P, _I64, _P]),
    "bh_celestial_checkerboard": (ctypes.c_int, [_P, _I64, _I32, _P, _P]),
    "bh_render_image": (ctypes.c_int, [_D, _D, _P, _P, _P, _I64, _I32, _P, _P]),
    "bh_trace_realtime": (ctypes.c_int, [ctypes.POINTER(RealtimeConfig), _D, _D, _P, _P, _P,
                                         _P, _P, _P, _I64, _P, _P]),
    "bh_vaidya_shell_table": (_I64, [ctypes.POINTER(Vaidya), _P, _P, _P, _I64]),
    "bh_vaidya_geometry": (ctypes.c_int, [ctypes.POINTER(Vaidya), _P, _P, _P, _P, _I64, _P, _P,
                                          _P, _P, _P, _P]),
    "bh_vaidya_mass": (ctypes.c_int, [ctypes.POINTER(Vaidya), _P, _P, _I64, _P, _P, _P]),
    "bh_vaidya_rhs": (ctypes.c_int, [ctypes.POINTER(Vaidya), _P, _P, _I64, _P]),
    "bh_vaidya_rk4": (ctypes.c_int, [ctypes.POINTER(Vaidya), _P, _P, _P, _I64, _I64, _P]),
    "bh_vaidya_trace": (ctypes.c_int, [ctypes.POINTER(Vaidya), _P, _I64, _D, _D, _I64, _P, _P,
                                       _P, _P, _P, _P, _P]),
    "bh_trace_tile_workspace_bytes": (_SZ, [_I64]),
    "bh_trace_tile": (ctypes.c_int, [ctypes.POINTER(TraceConfig), ctypes.POINTER(Scene), _D, _D,
                                     _P, _I64, _P, _P, _P, _P, _P, _P, _P, _P, _SZ,
                                     ctypes.POINTER(TileStats), _P]),
    "bh_radial_momentum": (ctypes.c_int, [_D, _D, _P, _D, _P]),
    "bh_plunge_worldline": (_I64, [_D, _D, _D, _D, _D, _D, _I64, _P, _P]),
    "bh_inflation_radiance": (ctypes.c_int, [_D, _P, _P, _P, _I64, _I64, _I32, _P, _P]),
    "bh_realtime_shade": (ctypes.c_int, [ctypes.POINTER(RealtimeShading), _P, _P, _P, _P, _I64,
                                         _I64, _P, _P, _P, _P]),
    "bh_offline_camera_rays": (ctypes.c_int, [_D, _D, ctypes.POINTER(OfflineCamera), _P, _P]),
    "bh_offline_radiance": (ctypes.c_int, [ctypes.POINTER(EmissionConfig), _P, _P, _P, _P, _P,
                                           _I64, _I64, _P, _P, _P, _P, _P]),
    "bh_develop_workspace_bytes": (_SZ, [_I64, _I64]),
    "bh_downsample": (ctypes.c_int, [_P, _I64, _I64, _I32, _P, _P]),
    "bh_frame_bloom_workspace_bytes": (_SZ, [_I64, _I64]),
    "bh_frame_bloom": (ctypes.c_int, [_P, _I64, _I64, _D, _P, _I32, _P, _P, _SZ, _P]),
    "bh_develop": (ctypes.c_int, [_P, _I64, _I64, _D, _D, _D, _P, _I32, _P, _P, _SZ, _P]),
    "bh_fma_peak_launch": (ctypes.c_int, [_I32, _I64, _P, ctypes.POINTER(_I64), _P]),
}

_lib = None


class BHError(RuntimeError):
    """A CUDA-side failure reported by libbh_b200 (status BH_ERR_CUDA,
    BH_ERR_TIMEOUT or BH_ERR_WORKSPACE)."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


def load():
    """Load libbh_b200.so, or raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m blackhorizon_b200.build` "
            "(the b200 backend has no fallback)"
        )
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def exported_symbols():
    return list(_SIGNATURES)


def check(status: int, what: str = "") -> None:
    """Map a bh_status to the reference's exception types: ValueError for
    malformed input (bad arguments, escape radius), RuntimeError otherwise."""
    if status == BH_OK:
        return
    lib = load()
    msg = lib.bh_last_error().decode() or lib.bh_status_string(status).decode()
    if what:
        msg = f"{what}: {msg}"
    if status in (BH_ERR_INVALID_ARGUMENT, BH_ERR_ESCAPE_RADIUS):
        raise ValueError(msg)
    raise BHError(status, msg)

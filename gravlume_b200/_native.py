"""ctypes declarations of the C ABI in include/glc.h (structs, enums and function signatures)."""

from __future__ import annotations

import ctypes
from pathlib import Path

from .build import LIB_PATH

c_double, c_int32, c_uint32, c_uint64, c_void_p = (ctypes.c_double, ctypes.c_int32, ctypes.c_uint32,
                                                   ctypes.c_uint64, ctypes.c_void_p)

GLC_OK = 0
ABI_VERSION = 3  # GLC_ABI_VERSION of include/glc.h these structures mirror
STATUS_NAMES = {
    0: "OK", 1: "INVALID_ARGUMENT", 2: "CUDA", 3: "NON_FINITE", 4: "NON_POSITIVE",
    5: "NON_NORMALIZED", 6: "EXTREMALITY_CHANGED", 7: "NON_STATIONARY", 8: "DEGENERATE_FRAME",
    9: "SURFACE_OUTSIDE_ESCAPE", 10: "INVALID_SURFACE", 11: "INVALID_VIEW", 12: "TIMEOUT",
    13: "CAPACITY", 14: "NO_DEVICE", 15: "UNSUPPORTED",
}

CAMERA_PINHOLE, CAMERA_EQUIRECT, CAMERA_RAYLIST = 0, 1, 2


class SceneInput(ctypes.Structure):
    _fields_ = [
        ("mass", c_double), ("spin", c_double), ("charge", c_double),
        ("chart", c_int32), ("has_surface", c_int32),
        ("observer_txyz", c_double * 4), ("target_txyz", c_double * 4),
        ("up_hint_xyz", c_double * 3), ("measured_frequency", c_double),
        ("width", c_uint32), ("height", c_uint32), ("vertical_fov", c_double),
        ("escape_radius", c_double), ("surface_inner", c_double), ("surface_outer", c_double),
        ("intensity_at_six", c_double), ("horizon_offset", c_double),
        ("emission_model", c_int32), ("has_slab", c_int32), ("temperature_at_six", c_double),
        ("slab_optical_depth", c_double), ("slab_emission", c_double), ("slab_temperature", c_double),
    ]


class Scene(ctypes.Structure):
    _fields_ = [
        ("spin", c_double), ("charge", c_double), ("chart_sign", c_double), ("mass_scale", c_double),
        ("outer_horizon", c_double), ("horizon_event_radius", c_double),
        ("escape_radius", c_double), ("surface_inner", c_double), ("surface_outer", c_double),
        ("intensity_at_six", c_double), ("photon_shell_radius", c_double),
        ("isco_prograde", c_double), ("observer_txyz", c_double * 4),
        ("four_velocity", c_double * 4), ("image_right", c_double * 4),
        ("image_up", c_double * 4), ("arrival", c_double * 4),
        ("metric_covariant", c_double * 16), ("frequency", c_double),
        ("tangent_half_fov", c_double), ("width", c_uint32), ("height", c_uint32),
        ("extremality", c_int32), ("has_horizon", c_int32), ("has_escape", c_int32),
        ("has_surface", c_int32), ("emission_model", c_int32), ("reserved", c_int32),
        ("temperature_at_six", c_double), ("slab_transmittance", c_double), ("slab_emission", c_double),
        ("slab_bands", c_double * 3),
    ]


class Policy(ctypes.Structure):
    _fields_ = [
        ("position_rtol", c_double), ("position_atol", c_double),
        ("momentum_rtol", c_double), ("momentum_atol", c_double),
        ("initial_step", c_double), ("minimum_step", c_double), ("maximum_step", c_double),
        ("safety", c_double), ("minimum_factor", c_double), ("maximum_factor", c_double),
        ("maximum_accepted_steps", c_uint64), ("maximum_consecutive_rejects", c_uint32),
        ("precision", c_int32), ("event_affine_tolerance", c_double),
        ("event_tie_tolerance", c_double), ("event_arming_band", c_double),
        ("singularity_guard", c_double), ("mixed_shell_factor", c_double),
        ("renormalize_null", c_uint32), ("persistent", c_uint32), ("block_threads", c_uint32),
        ("blocks_per_sm", c_uint32), ("tile_w", c_uint32), ("tile_h", c_uint32),
        ("refill_interval", c_uint32), ("rays_per_grab", c_uint32),
        ("refill_min_idle", c_uint32), ("mixed_pair_state", c_uint32), ("capture_certificates", c_uint32),
        ("escape_map", c_uint32), ("mixed_split", c_uint32), ("uncertain_terminals", c_uint32),
        ("uncertain_drift_limit", c_double),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class Camera(ctypes.Structure):
    _fields_ = [
        ("kind", c_int32), ("scene_index", c_int32), ("width", c_uint32), ("height", c_uint32),
        ("subpixel_x", c_double), ("subpixel_y", c_double), ("ray_states", c_void_p),
        ("n_rays", c_uint64), ("affine_direction", c_double), ("result_offset", c_uint64),
        ("tile_origin", c_uint32 * 2), ("tile_count", c_uint32 * 2),
    ]


RESULT_FIELDS = ["code", "branch", "escape", "surface", "redshift_time", "event", "drift_a",
                 "drift_b", "turning", "position_xy", "position_zr", "intensity", "radiance"]
# bytes per ray of each result field (radiance is RGBA16F)
RESULT_BYTES = {name: 16 for name in RESULT_FIELDS} | {"radiance": 8}


class Results(ctypes.Structure):
    _fields_ = [(name, c_void_p) for name in RESULT_FIELDS]


class AdjointScene(ctypes.Structure):
    _fields_ = [("input", SceneInput), ("observer_radius", c_double), ("observer_polar", c_double),
                ("observer_azimuth", c_double)]


class Grads(ctypes.Structure):
    _fields_ = [("ray_momentum", c_void_p), ("ray_params", c_void_p), ("params", c_void_p)]


class LaunchStats(ctypes.Structure):
    _fields_ = [("kernel_launches", c_uint64), ("last_rays", c_uint64), ("last_grid", c_uint32),
                ("last_block", c_uint32), ("last_persistent", c_uint32), ("sm_count", c_uint32)]


# Every symbol include/glc.h declares, with (restype, argtypes).
SIGNATURES = {
    "glc_abi_version": (ctypes.c_int, []),
    "glc_last_error_string": (ctypes.c_char_p, []),
    "glc_status_string": (ctypes.c_char_p, [c_int32]),
    "glc_scene_pack": (c_int32, [ctypes.POINTER(SceneInput), ctypes.POINTER(Scene)]),
    "glc_prograde_isco": (c_int32, [c_double, c_double, ctypes.POINTER(c_double)]),
    "glc_policy_default": (c_int32, [c_int32, c_int32, ctypes.POINTER(Policy)]),
    "glc_flop_model": (c_int32, [c_void_p]),
    "glc_selftest_event_policy": (c_int32, [ctypes.POINTER(Policy), c_void_p, c_void_p]),
    "glc_rhs_host": (c_int32, [ctypes.POINTER(Scene), c_void_p, c_double, c_int32, c_void_p]),
    "glc_create": (c_int32, [c_int32, ctypes.POINTER(c_void_p)]),
    "glc_destroy": (c_int32, [c_void_p]),
    "glc_set_policy": (c_int32, [c_void_p, ctypes.POINTER(Policy)]),
    "glc_get_policy": (c_int32, [c_void_p, ctypes.POINTER(Policy)]),
    "glc_get_stats": (c_int32, [c_void_p, ctypes.POINTER(LaunchStats)]),
    "glc_result_slots": (c_int32, [c_void_p, c_int32, c_void_p, c_int32, ctypes.POINTER(c_uint64)]),
    "glc_trace": (c_int32, [c_void_p, c_void_p, c_int32, c_void_p, c_int32,
                            ctypes.POINTER(Results), c_void_p]),
    "glc_trace_host": (c_int32, [c_void_p, c_void_p, c_int32, c_void_p, c_int32,
                                 ctypes.POINTER(Results)]),
    "glc_graph_capture": (c_int32, [c_void_p, c_void_p, c_int32, c_void_p, c_int32,
                                    ctypes.POINTER(Results), c_void_p, ctypes.POINTER(c_void_p)]),
    "glc_graph_launch": (c_int32, [c_void_p, c_void_p]),
    "glc_graph_destroy": (c_int32, [c_void_p]),
    "glc_autotune": (c_int32, [c_void_p, c_void_p, c_int32, c_void_p, c_int32,
                               ctypes.POINTER(Results), c_void_p, c_int32, ctypes.POINTER(Policy)]),
    "glc_refine_shadow_edges": (c_int32, [c_void_p, c_void_p, c_int32, c_void_p, c_int32, ctypes.POINTER(Results),
                                          c_void_p, c_void_p]),
    "glc_surface_footprint": (c_int32, [c_void_p, c_void_p, c_int32, c_void_p, c_int32, c_int32,
                                        ctypes.POINTER(Results), c_void_p, c_void_p]),
    "glc_forward_ckpt": (c_int32, [c_void_p, ctypes.POINTER(AdjointScene), ctypes.POINTER(Camera), c_int32,
                                   ctypes.POINTER(Results), c_void_p, ctypes.POINTER(c_void_p)]),
    "glc_forward_ckpt_into": (c_int32, [c_void_p, ctypes.POINTER(AdjointScene), ctypes.POINTER(Camera), c_int32,
                                        ctypes.POINTER(Results), c_void_p, c_void_p]),
    "glc_backward": (c_int32, [c_void_p, c_void_p, ctypes.POINTER(Grads), c_void_p]),
    "glc_tape_info": (c_int32, [c_void_p, ctypes.POINTER(c_uint64), ctypes.POINTER(c_uint32),
                                ctypes.POINTER(c_uint64)]),
    "glc_tape_destroy": (c_int32, [c_void_p]),
    "glc_trace_static_scratch": (c_int32, [c_void_p, c_int32, c_void_p, c_int32, ctypes.POINTER(Policy),
                                           ctypes.POINTER(Results), c_void_p]),
}

_lib = None


class GlcError(RuntimeError):
    def __init__(self, status: int, where: str, message: str):
        self.status = status
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}: {message}")


def lib(path: Path | None = None):
    """Load libglc.so. Raises if the CUDA extension is missing: there is no fallback path."""
    global _lib
    if _lib is None:
        p = Path(path or LIB_PATH)
        if not p.exists():
            raise RuntimeError(f"libglc.so is not built ({p}); run gravlume_b200.build(force=True)")
        L = ctypes.CDLL(str(p))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        if L.glc_abi_version() != ABI_VERSION:
            raise RuntimeError(f"{p} has ABI {L.glc_abi_version()}, the bindings expect {ABI_VERSION}: rebuild it")
        _lib = L
    return _lib


def check(status: int, where: str) -> None:
    if status != GLC_OK:
        msg = lib().glc_last_error_string().decode(errors="replace")
        raise GlcError(status, where, msg)

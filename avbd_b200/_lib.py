"""ctypes binding of libavbd6.so (include/avbd6.h)."""

from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libavbd6.so")

MAX_VIOL_ITERS = 256  # AVBD_MAX_VIOL_ITERS (include/avbd6.h)
AVBD_ERR_BARRIER_TIMEOUT = 1
AVBD_ERR_HASH_FULL = 2
AVBD_ERR_PAIR_OVERFLOW = 4
AVBD_ERR_ROW_OVERFLOW = 8
AVBD_ERR_NONFINITE = 16
AVBD_ERR_NBR_OVERFLOW = 32
AVBD_ERR_BVH = 64


class AvbdDims(C.Structure):
    _fields_ = [("n_bodies", C.c_int), ("n_static_groups", C.c_int), ("n_static_rows", C.c_int),
                ("pair_cap", C.c_int), ("dyn_row_cap", C.c_int), ("dyn_group_cap", C.c_int),
                ("hash_cap", C.c_int), ("mlp_floats", C.c_int), ("new_cap", C.c_int),
                ("n_scenes", C.c_int), ("anchor_keys", C.c_int)]


class AvbdParams(C.Structure):
    _fields_ = [("dt", C.c_float), ("iterations", C.c_int), ("gravity", C.c_float * 3), ("alpha", C.c_float),
                ("beta", C.c_float), ("gamma", C.c_float), ("post_stabilize", C.c_int),
                ("max_linear_speed", C.c_float), ("max_angular_speed", C.c_float), ("substeps", C.c_int),
                ("friction_static_mult", C.c_float), ("coloring_mode", C.c_int),
                ("recolor_every_substep", C.c_int), ("self_collide", C.c_int), ("self_friction", C.c_float),
                ("group_size", C.c_int), ("use_graph", C.c_int), ("persistent", C.c_int),
                ("record_violation", C.c_int), ("mlp_warm_start", C.c_int), ("debug_skip_arrive", C.c_int),
                ("blocks_per_sm", C.c_int), ("timing", C.c_int), ("log_new_contacts", C.c_int),
                ("flag_sweep", C.c_int), ("bvh_rebuild_every", C.c_int),
                ("adaptive_lanes", C.c_int), ("resting_floor", C.c_int)]


class AvbdStats(C.Structure):
    _fields_ = [("n_pairs_found", C.c_int), ("n_pairs", C.c_int), ("n_dyn_groups", C.c_int),
                ("n_dyn_rows", C.c_int), ("n_dyn_rows_req", C.c_int), ("n_contacts_req", C.c_int),
                ("n_colors", C.c_int), ("recolored", C.c_int), ("conflicts", C.c_int), ("err", C.c_int),
                ("err_where", C.c_int), ("n_cache_hits", C.c_int), ("n_new_contacts", C.c_int),
                ("max_dg", C.c_int), ("n_viol", C.c_int), ("epoch", C.c_uint), ("graph_state", C.c_int),
                ("capture_err", C.c_int), ("kernels_launched", C.c_longlong), ("viol", C.c_float * MAX_VIOL_ITERS),
                ("n_new_logged", C.c_int), ("n_mlp_applied", C.c_int), ("n_mlp_fallback", C.c_int), ("n_mlp_reverted", C.c_int),
                ("viol_contact", C.c_float * MAX_VIOL_ITERS)]

# Learned warm-start network sizes (avbd6.h AVBD_MLP_*).
MLP_IN = 20
MLP_OUT = 4
MLP_PARAMS = 5764
MLP_FLOATS = 3544


_lib = None


def load():
    """Load libavbd6.so; raises if it is missing (no CPU fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is not built: run `python -m avbd_b200.build` (needs nvcc)")
    L = C.CDLL(LIB_PATH)
    vp, i, sz = C.c_void_p, C.c_int, C.c_size_t
    L.avbd_num_arrays.restype = i
    L.avbd_array_name.restype = C.c_char_p
    L.avbd_array_name.argtypes = [i]
    L.avbd_last_error.restype = C.c_char_p
    L.avbd_layout.argtypes = [C.POINTER(AvbdDims), C.POINTER(sz), C.POINTER(sz)]
    L.avbd_create.argtypes = [C.POINTER(AvbdDims), vp, sz, C.POINTER(vp)]
    L.avbd_destroy.argtypes = [vp]
    L.avbd_set_params.argtypes = [vp, C.POINTER(AvbdParams), vp]
    L.avbd_reset_state.argtypes = [vp, vp]
    L.avbd_mark_color_dirty.argtypes = [vp, vp]
    L.avbd_substep.argtypes = [vp, C.c_float, vp]
    L.avbd_step.argtypes = [vp, vp]
    L.avbd_read_stats.argtypes = [vp, C.POINTER(AvbdStats), vp]
    L.avbd_count_color_conflicts.argtypes = [vp, vp]
    L.avbd_cache_load.argtypes = [vp, i, vp, vp, vp]
    L.avbd_cache_load_keys.argtypes = [vp, i, vp, vp, vp]
    L.avbd_clear_errors.argtypes = [vp, vp]
    L.avbd_step_ms.argtypes = [vp, C.POINTER(C.c_float), C.POINTER(C.c_float)]
    L.avbd_read_phase_marks.argtypes = [vp, vp, vp, i, vp]
    L.avbd_exclusive_scan_noalloc.argtypes = [vp, vp, i, vp]
    L.avbd_exclusive_scan_noalloc.restype = i
    L.avbd_mlp_pack.argtypes = [vp, vp, vp, vp]
    L.avbd_mlp_infer.argtypes = [vp, vp, i, vp, vp]
    L.avbd_mlp_scratch_bytes.argtypes = [i]
    L.avbd_mlp_scratch_bytes.restype = sz
    L.avbd_mlp_loss_grad.argtypes = [vp, vp, vp, i, vp, vp, vp, sz, vp]
    L.avbd_mlp_adam.argtypes = [vp, vp, vp, vp, i, C.c_float, C.c_float, C.c_float, C.c_float, vp]
    L.avbd_profile_next_substep.argtypes = [vp]
    L.avbd_collision_profile.argtypes = [vp, C.POINTER(C.c_float), i]
    L.avbd_collision_stage.argtypes = [vp, i]
    L.avbd_collision_stage.restype = C.c_char_p
    for name in ("avbd_layout", "avbd_create", "avbd_destroy", "avbd_set_params", "avbd_reset_state",
                 "avbd_mark_color_dirty", "avbd_substep", "avbd_step", "avbd_read_stats",
                 "avbd_count_color_conflicts", "avbd_cache_load", "avbd_cache_load_keys", "avbd_clear_errors",
                 "avbd_step_ms",
                 "avbd_read_phase_marks", "avbd_mlp_pack", "avbd_mlp_infer", "avbd_mlp_loss_grad", "avbd_mlp_adam",
                 "avbd_profile_next_substep", "avbd_collision_profile"):
        getattr(L, name).restype = i
    _lib = L
    return L


def check(code: int, what: str) -> int:
    if code < 0:
        msg = load().avbd_last_error().decode(errors="replace")
        raise RuntimeError(f"libavbd6 {what} failed ({code}): {msg}")
    return code


# Exported C symbols declared in include/avbd6.h.
EXPORTED = ["avbd_num_arrays", "avbd_array_name", "avbd_layout", "avbd_create", "avbd_destroy",
            "avbd_set_params", "avbd_reset_state", "avbd_mark_color_dirty", "avbd_substep", "avbd_step",
            "avbd_read_stats", "avbd_count_color_conflicts", "avbd_cache_load", "avbd_cache_load_keys",
            "avbd_clear_errors",
            "avbd_step_ms", "avbd_read_phase_marks", "avbd_exclusive_scan_noalloc", "avbd_mlp_pack",
            "avbd_mlp_infer", "avbd_mlp_scratch_bytes", "avbd_mlp_loss_grad", "avbd_mlp_adam", "avbd_last_error",
            "avbd_profile_next_substep", "avbd_collision_profile", "avbd_collision_stage"]

PHASES = ["start", "gate+prelude", "color reset", "color rounds", "bucket", "predict", "primal", "dual",
          "collect"]

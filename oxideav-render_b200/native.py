"""ctypes bindings of `_lib/libpt_b200.so` (the C ABI in include/pt_b200.h and
include/pt_b200_debug.h).

Loading fails loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libpt_b200.so")

_lock = threading.Lock()
_lib = None


class RenderError(RuntimeError):
    """oxideav_render::Error::Backend (src/error.rs:38-43)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{abi.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


vp = C.c_void_p
u32, i32, u64, f32 = C.c_uint32, C.c_int, C.c_uint64, C.c_float
fp, dp, u8p, u32p, u64p = (C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_uint8),
                           C.POINTER(C.c_uint32), C.POINTER(C.c_uint64))

SIGNATURES = {
    # include/pt_b200.h
    "pt_abi_version": (u32, []),
    "pt_create": (i32, [C.POINTER(vp), i32]),
    "pt_destroy": (None, [vp]),
    "pt_last_error": (C.c_char_p, [vp]),
    "pt_scene_upload": (i32, [vp, C.POINTER(abi.pt_scene_desc), u32p]),
    "pt_scene_release": (i32, [vp, u32]),
    "pt_scene_refit": (i32, [vp, u32, C.POINTER(abi.pt_scene_desc)]),
    "pt_scene_device_bytes": (i32, [vp, u32, u64p]),
    "pt_scene_triangle_count": (i32, [vp, u32, u64p]),
    "pt_tracer_create": (i32, [vp, C.POINTER(vp)]),
    "pt_tracer_destroy": (None, [vp]),
    "pt_tracer_sync": (i32, [vp, u32, C.POINTER(abi.pt_camera), C.POINTER(abi.pt_render_options),
                             C.POINTER(C.c_int)]),
    "pt_tracer_refine": (i32, [vp, u32]),
    "pt_tracer_refine_many": (i32, [vp, C.POINTER(vp), u32p, u32]),
    "pt_batch_stats": (i32, [vp, fp, u32p, u64p]),
    "pt_tracer_samples": (i32, [vp, u32p]),
    "pt_tracer_is_converged": (i32, [vp, C.POINTER(C.c_int)]),
    "pt_tracer_reset": (i32, [vp]),
    "pt_tracer_invalidate_scene": (i32, [vp]),
    "pt_tracer_set_environment": (i32, [vp, C.POINTER(abi.pt_environment)]),
    "pt_tracer_read_hdr": (i32, [vp, fp, C.c_size_t]),
    "pt_tracer_read_image": (i32, [vp, u8p, C.c_size_t]),
    "pt_tracer_read_accum": (i32, [vp, dp, C.c_size_t]),
    "pt_tracer_ray_counts": (i32, [vp, u64p, u64p]),
    "pt_render_hdr": (i32, [vp, u32, C.POINTER(abi.pt_camera), C.POINTER(abi.pt_render_options),
                            C.POINTER(abi.pt_environment), fp, C.c_size_t]),
    "pt_render_image": (i32, [vp, u32, C.POINTER(abi.pt_camera), C.POINTER(abi.pt_render_options),
                              C.POINTER(abi.pt_environment), u8p, C.c_size_t]),
    "pt_refine_noalloc": (i32, [vp, u32, C.POINTER(abi.pt_camera), C.POINTER(abi.pt_render_options), u32, u32,
                                C.c_void_p]),
    "pt_raycast_render": (i32, [vp, u32, C.POINTER(abi.pt_camera), C.POINTER(abi.pt_raycast_options), fp,
                                C.c_size_t, u8p, C.c_size_t]),
    # include/pt_b200_serve.h
    "pt_server_create": (i32, [vp, C.POINTER(abi.pt_server_config), C.POINTER(vp)]),
    "pt_server_destroy": (None, [vp]),
    "pt_server_last_error": (C.c_char_p, [vp]),
    "pt_server_scene_register": (i32, [vp, C.POINTER(abi.pt_scene_desc), C.POINTER(abi.pt_environment), u32p]),
    "pt_server_scene_unregister": (i32, [vp, u32]),
    "pt_server_scene_info": (i32, [vp, u32, u64p, C.POINTER(C.c_int)]),
    "pt_server_submit": (i32, [vp, C.POINTER(abi.pt_server_request), u64p]),
    "pt_server_wait": (i32, [vp, u64, i32, fp, C.c_size_t, C.POINTER(abi.pt_request_stats)]),
    "pt_server_poll": (i32, [vp, u64, fp, C.c_size_t, C.POINTER(abi.pt_request_stats)]),
    "pt_server_cancel": (i32, [vp, u64]),
    "pt_server_debug_fail_allocations": (i32, [vp, u32]),
    "pt_server_release": (i32, [vp, u64]),
    "pt_server_stats_get": (i32, [vp, C.POINTER(abi.pt_server_stats)]),
    # include/pt_b200_debug.h
    "pt_set_bvh_builder": (i32, [vp, u32]),
    "pt_debug_build_bvh": (i32, [fp, u32, u32, dp, vp, u64, vp, u64]),
    "pt_scene_bvh_on_device": (i32, [vp, u32, C.POINTER(C.c_int)]),
    "pt_scene_upload_seconds": (i32, [vp, u32, dp]),
    "pt_debug_scene_texels": (i32, [vp, u32, fp, u64, u64p]),
    "pt_debug_sobol": (i32, [vp, u32, u32, fp]),
    "pt_debug_pattern": (i32, [vp, u32, u32, fp]),
    "pt_debug_primary_hits": (i32, [vp, u32, u32p, fp]),
    "pt_debug_bsdf": (i32, [vp, fp, fp, fp, u32, fp]),
    "pt_tracer_traversal_counts": (i32, [vp, u64p, u64p]),
    "pt_tracer_traversal_split": (i32, [vp, u64p]),
    "pt_set_stage_timing": (i32, [vp, i32]),
    "pt_tracer_stage_ms": (i32, [vp, fp, u32]),
    "pt_batch_counters": (i32, [vp, u64p]),
    "pt_batch_stage_ms": (i32, [vp, fp, u32]),
    "pt_scene_bvh_stats": (i32, [vp, u32, u32p, u32p, u32p, dp, dp]),
    "pt_set_schedule": (i32, [vp, u32]),
    "pt_set_wave_slots": (i32, [vp, u32]),
    "pt_set_node_width": (i32, [vp, u32, u32]),
    "pt_set_material_sort": (i32, [vp, i32]),
    "pt_set_traversal": (i32, [vp, u32, u32]),
    "pt_set_shade_blocks": (i32, [vp, u32]),
    "pt_set_wave_overlap": (i32, [vp, i32]),
    "pt_set_wave_graphs": (i32, [vp, i32]),
    "pt_debug_fail_allocations": (i32, [vp, u32]),
    "pt_debug_prepare_scene": (i32, [C.POINTER(abi.pt_scene_desc), dp, u64p]),
    "pt_autotune": (i32, [vp, vp, u32, C.POINTER(abi.pt_tune_choice)]),
    "pt_tune_lookup": (i32, [vp, vp, C.POINTER(abi.pt_tune_choice)]),
    "pt_tune_reset": (i32, [vp]),
    "pt_tracer_last_kernel_ms": (i32, [vp, fp]),
}


def load():
    """The loaded library (raises FileNotFoundError when it was never built)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise FileNotFoundError(f"{LIB_PATH} is missing: run __graft_entry__.build() first")
            lib = C.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def check(status: int, ctx=None) -> None:
    if status != abi.PT_OK:
        msg = load().pt_last_error(ctx)
        raise RenderError(status, msg.decode() if msg else "")

"""ctypes mirrors of the C ABI structs declared in include/pt_b200.h.

Field order, widths and names follow the header one for one; the CPU test
suite compiles the header with gcc and checks every size and offset against
these classes.
"""
from __future__ import annotations

import ctypes as C

PT_MAX_UV_SETS = 4

PT_OK = 0
(PT_ERR_INVALID_ARG, PT_ERR_OOM, PT_ERR_DEVICE, PT_ERR_TIMEOUT, PT_ERR_EVICTED, PT_ERR_CANCELLED, PT_ERR_NOT_FOUND,
 PT_ERR_NOT_READY) = range(1, 9)
STATUS_NAMES = {
    0: "PT_OK",
    1: "PT_ERR_INVALID_ARG",
    2: "PT_ERR_OOM",
    3: "PT_ERR_DEVICE",
    4: "PT_ERR_TIMEOUT",
    5: "PT_ERR_EVICTED",
    6: "PT_ERR_CANCELLED",
    7: "PT_ERR_NOT_FOUND",
    8: "PT_ERR_NOT_READY",
}

PT_ALPHA_OPAQUE, PT_ALPHA_MASK, PT_ALPHA_BLEND = 0, 1, 2

PT_EXT_SPECULAR = 1 << 0
PT_EXT_TRANSMISSION = 1 << 1
PT_EXT_VOLUME = 1 << 2
PT_EXT_CLEARCOAT = 1 << 3
PT_EXT_SHEEN = 1 << 4
PT_EXT_ANISOTROPY = 1 << 5
PT_EXT_IRIDESCENCE = 1 << 6
PT_EXT_DIFFUSE_TRANSMISSION = 1 << 7
PT_EXT_DISPERSION = 1 << 8

PT_FILTER_NEAREST, PT_FILTER_LINEAR = 0, 1
(PT_MIN_NEAREST, PT_MIN_LINEAR, PT_MIN_NEAREST_MIP_NEAREST, PT_MIN_LINEAR_MIP_NEAREST,
 PT_MIN_NEAREST_MIP_LINEAR, PT_MIN_LINEAR_MIP_LINEAR) = range(6)
PT_WRAP_REPEAT, PT_WRAP_CLAMP, PT_WRAP_MIRROR = 0, 1, 2
PT_PIXELS_RGBA8, PT_PIXELS_RGBA_F32 = 0, 1
PT_LIGHT_DIRECTIONAL, PT_LIGHT_POINT, PT_LIGHT_SPOT = 0, 1, 2
PT_PERSPECTIVE, PT_ORTHOGRAPHIC = 0, 1
PT_MIS, PT_LIGHT_ONLY, PT_BSDF_ONLY = 0, 1, 2
PT_TONE_CLAMP, PT_TONE_REINHARD, PT_TONE_ACES = 0, 1, 2
PT_BVH_BUILD_AUTO, PT_BVH_BUILD_HOST, PT_BVH_BUILD_DEVICE, PT_BVH_BUILD_DEVICE_PLOC = 0, 1, 2, 3
PT_BVH_BUILD_HOST_SPATIAL = 4
# pt_schedule (include/pt_b200_debug.h); a new context runs the wavefront.
PT_SCHEDULE_MEGAKERNEL, PT_SCHEDULE_WAVEFRONT = 0, 1
# A new context's path slots per wave.
PT_DEFAULT_WAVE_SLOTS = 1 << 23

f3 = C.c_float * 3
f4 = C.c_float * 4


class pt_texture_binding(C.Structure):
    _fields_ = [
        ("texture", C.c_int32),
        ("uv_set", C.c_uint32),
        ("has_transform", C.c_uint32),
        ("transform", C.c_float * 6),
    ]


def no_binding() -> pt_texture_binding:
    b = pt_texture_binding()
    b.texture = -1
    return b


class pt_material(C.Structure):
    _fields_ = [
        ("base_color", f4),
        ("base_color_texture", pt_texture_binding),
        ("metallic", C.c_float),
        ("roughness", C.c_float),
        ("metallic_roughness_texture", pt_texture_binding),
        ("normal_texture", pt_texture_binding),
        ("normal_scale", C.c_float),
        ("occlusion_texture", pt_texture_binding),
        ("occlusion_strength", C.c_float),
        ("emissive", f3),
        ("emissive_texture", pt_texture_binding),
        ("alpha_mode", C.c_uint32),
        ("alpha_cutoff", C.c_float),
        ("double_sided", C.c_uint32),
        ("unlit", C.c_uint32),
        ("ior", C.c_float),
        ("ext_flags", C.c_uint32),
        ("specular_factor", C.c_float),
        ("specular_texture", pt_texture_binding),
        ("specular_color_factor", f3),
        ("specular_color_texture", pt_texture_binding),
        ("transmission_factor", C.c_float),
        ("transmission_texture", pt_texture_binding),
        ("thickness_factor", C.c_float),
        ("thickness_texture", pt_texture_binding),
        ("attenuation_distance", C.c_float),
        ("attenuation_color", f3),
        ("clearcoat_factor", C.c_float),
        ("clearcoat_texture", pt_texture_binding),
        ("clearcoat_roughness_factor", C.c_float),
        ("clearcoat_roughness_texture", pt_texture_binding),
        ("clearcoat_normal_texture", pt_texture_binding),
        ("clearcoat_normal_scale", C.c_float),
        ("sheen_color_factor", f3),
        ("sheen_color_texture", pt_texture_binding),
        ("sheen_roughness_factor", C.c_float),
        ("sheen_roughness_texture", pt_texture_binding),
        ("anisotropy_strength", C.c_float),
        ("anisotropy_rotation", C.c_float),
        ("anisotropy_texture", pt_texture_binding),
        ("iridescence_factor", C.c_float),
        ("iridescence_texture", pt_texture_binding),
        ("iridescence_ior", C.c_float),
        ("iridescence_thickness_min", C.c_float),
        ("iridescence_thickness_max", C.c_float),
        ("iridescence_thickness_texture", pt_texture_binding),
        ("diffuse_transmission_factor", C.c_float),
        ("diffuse_transmission_texture", pt_texture_binding),
        ("diffuse_transmission_color_factor", f3),
        ("diffuse_transmission_color_texture", pt_texture_binding),
        ("dispersion", C.c_float),
    ]


class pt_texture(C.Structure):
    _fields_ = [
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("format", C.c_uint32),
        ("pixels", C.c_void_p),
        ("mag_filter", C.c_uint32),
        ("min_filter", C.c_uint32),
        ("wrap_s", C.c_uint32),
        ("wrap_t", C.c_uint32),
    ]


class pt_draw_item(C.Structure):
    _fields_ = [
        ("triangle_count", C.c_uint32),
        ("positions", C.POINTER(C.c_float)),
        ("normals", C.POINTER(C.c_float)),
        ("has_vertex_normals", C.c_uint32),
        ("tangents", C.POINTER(C.c_float)),
        ("uvs", C.POINTER(C.c_float) * PT_MAX_UV_SETS),
        ("colors", C.POINTER(C.c_float)),
        ("material", C.c_uint32),
    ]


class pt_light(C.Structure):
    _fields_ = [
        ("kind", C.c_uint32),
        ("color", f3),
        ("intensity", C.c_float),
        ("position", f3),
        ("direction", f3),
        ("has_range", C.c_uint32),
        ("range", C.c_float),
        ("inner_cone_angle", C.c_float),
        ("outer_cone_angle", C.c_float),
    ]


class pt_scene_desc(C.Structure):
    _fields_ = [
        ("item_count", C.c_uint32),
        ("items", C.POINTER(pt_draw_item)),
        ("material_count", C.c_uint32),
        ("materials", C.POINTER(pt_material)),
        ("texture_count", C.c_uint32),
        ("textures", C.POINTER(pt_texture)),
        ("light_count", C.c_uint32),
        ("lights", C.POINTER(pt_light)),
    ]


class pt_environment(C.Structure):
    _fields_ = [
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("pixels", C.POINTER(C.c_float)),
        ("intensity", C.c_float),
    ]


class pt_camera(C.Structure):
    _fields_ = [
        ("eye", f3),
        ("forward", f3),
        ("side", f3),
        ("up", f3),
        ("half_w", C.c_float),
        ("half_h", C.c_float),
        ("projection", C.c_uint32),
    ]


class pt_path_trace_options(C.Structure):
    _fields_ = [
        ("samples_per_pixel", C.c_uint32),
        ("max_bounces", C.c_uint32),
        ("rr_start", C.c_uint32),
        ("clamp", C.c_float),
        ("seed", C.c_uint32),
        ("strategy", C.c_uint32),
    ]


class pt_render_options(C.Structure):
    _fields_ = [
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("background", C.c_uint8 * 4),
        ("tone_map", C.c_uint32),
        ("exposure", C.c_float),
        ("ambient", C.c_float),
        ("path_trace", pt_path_trace_options),
    ]


PT_SHADE_FLAT, PT_SHADE_GOURAUD, PT_SHADE_PHONG, PT_SHADE_WIREFRAME = 0, 1, 2, 3
PT_SHADE_NORMAL_DEBUG, PT_SHADE_DEPTH_DEBUG, PT_SHADE_PBR = 4, 5, 6


class pt_raycast_options(C.Structure):
    _fields_ = [
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("aa", C.c_uint32),
        ("shading", C.c_uint32),
        ("light_azimuth_deg", C.c_float),
        ("light_elevation_deg", C.c_float),
        ("light_intensity", C.c_float),
        ("background", C.c_uint8 * 4),
        ("tone_map", C.c_uint32),
        ("exposure", C.c_float),
        ("max_ray_depth", C.c_uint32),
        ("near_plane", C.c_float),
        ("far_plane", C.c_float),
        ("ambient", C.c_float),
        ("shadows", C.c_uint32),
        ("reflection_roughness_cutoff", C.c_float),
    ]


# include/pt_b200_serve.h
class pt_server_config(C.Structure):
    _fields_ = [
        ("hbm_budget_bytes", C.c_uint64),
        ("wave_slots", C.c_uint32),
        ("max_active", C.c_uint32),
        ("megakernel", C.c_uint32),
        ("pipeline_depth", C.c_uint32),
        ("node_width_extension", C.c_uint32),
        ("node_width_shadow", C.c_uint32),
        ("autotune", C.c_uint32),
        ("material_sort_off", C.c_uint32),
        ("wave_overlap_off", C.c_uint32),
        ("bvh_binned", C.c_uint32),
    ]


class pt_server_request(C.Structure):
    _fields_ = [
        ("scene", C.c_uint32),
        ("samples", C.c_uint32),
        ("continues", C.c_uint64),
        ("camera", pt_camera),
        ("options", pt_render_options),
        ("deadline_ms", C.c_uint32),
    ]


class pt_request_stats(C.Structure):
    _fields_ = [
        ("queue_ms", C.c_double),
        ("latency_ms", C.c_double),
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("samples", C.c_uint32),
        ("waves", C.c_uint32),
    ]


class pt_server_stats(C.Structure):
    _fields_ = [
        ("submitted", C.c_uint64),
        ("completed", C.c_uint64),
        ("failed", C.c_uint64),
        ("samples", C.c_uint64),
        ("waves", C.c_uint64),
        ("rays", C.c_uint64),
        ("gpu_ms", C.c_double),
        ("scene_uploads", C.c_uint64),
        ("scene_evictions", C.c_uint64),
        ("resident_bytes", C.c_uint64),
        ("peak_resident_bytes", C.c_uint64),
        ("resident_scenes", C.c_uint32),
        ("active", C.c_uint32),
        ("pending", C.c_uint32),
        ("accumulators", C.c_uint32),
        ("tuned_classes", C.c_uint64),
        ("cancelled", C.c_uint64),
        ("timed_out", C.c_uint64),
    ]


# include/pt_b200_debug.h
class pt_tune_choice(C.Structure):
    _fields_ = [
        ("schedule", C.c_uint32),
        ("node_width_extension", C.c_uint32),
        ("node_width_shadow", C.c_uint32),
        ("material_sort", C.c_uint32),
        ("wave_slots", C.c_uint32),
        ("samples_per_s", C.c_float),
        ("shade_blocks_per_sm", C.c_uint32),
        ("wave_arenas", C.c_uint32),
        ("traversal_threads", C.c_uint32),
        ("claim_chunk", C.c_uint32),
    ]


ABI_STRUCTS = [
    pt_texture_binding, pt_material, pt_texture, pt_draw_item, pt_light,
    pt_scene_desc, pt_environment, pt_camera, pt_path_trace_options, pt_render_options, pt_raycast_options,
    pt_server_config, pt_server_request, pt_request_stats, pt_server_stats, pt_tune_choice,
]

"""ctypes binding of include/photon_cuda.h (the C ABI of libphoton_cuda.so).

The library is built in-tree (``build.py``) and loaded from this folder.  There is no CPU
fallback: if the library or a CUDA device is missing, the product API raises.
"""
from __future__ import annotations

import ctypes as C
import pathlib

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "libphoton_cuda.so"

PE_OK, PE_ERR_INVALID, PE_ERR_CUDA, PE_ERR_NO_SCENE, PE_ERR_CANCELLED, PE_ERR_OOM, PE_ERR_DEVICE, PE_ERR_LIMIT = range(8)
STATUS_NAMES = {0: "PE_OK", 1: "PE_ERR_INVALID", 2: "PE_ERR_CUDA", 3: "PE_ERR_NO_SCENE", 4: "PE_ERR_CANCELLED",
                5: "PE_ERR_OOM", 6: "PE_ERR_DEVICE", 7: "PE_ERR_LIMIT"}
PE_MAT_LAMBERT, PE_MAT_DISNEY, PE_MAT_DIELECTRIC, PE_MAT_MIRROR = range(4)
PE_FILTER_BOX, PE_FILTER_TRIANGLE, PE_FILTER_GAUSSIAN, PE_FILTER_BLACKMAN_HARRIS = range(4)
PE_BG_ENVIRONMENT, PE_BG_COLOR, PE_BG_TRANSPARENT = range(3)

F3 = C.c_float * 3


class pe_material(C.Structure):
    _fields_ = [
        ("type", C.c_int32), ("base_color", F3), ("emission", F3),
        ("metallic", C.c_float), ("roughness", C.c_float), ("specular", C.c_float),
        ("clearcoat", C.c_float), ("clearcoat_roughness", C.c_float),
        ("ior", C.c_float), ("spec_transmission", C.c_float), ("coat_ior", C.c_float),
        ("coat_tint", F3), ("sheen_color", F3), ("has_sheen_color", C.c_int32),
        ("anisotropy", C.c_float), ("sheen", C.c_float), ("sheen_roughness", C.c_float),
        ("diffuse_roughness", C.c_float), ("diffuse_transmission", C.c_float),
        ("subsurface", C.c_float), ("subsurface_radius", F3),
        ("subsurface_scale", C.c_float), ("subsurface_anisotropy", C.c_float),
        ("edge_tint", F3), ("thin_film_thickness", C.c_float), ("thin_film_ior", C.c_float),
        ("flake_density", C.c_float), ("flake_size", C.c_float), ("flake_roughness", C.c_float),
        ("flake_color", F3), ("opacity", C.c_float),
        ("glass_roughness", C.c_float), ("abbe", C.c_float), ("absorb_color", F3), ("absorb_distance", C.c_float),
        ("scatter_density", C.c_float), ("scatter_color", F3), ("scatter_anisotropy", C.c_float),
        ("thin_walled", C.c_int32), ("film_thickness", C.c_float),
        ("has_absorption", C.c_int32), ("has_scattering", C.c_int32),
        ("round_edge_radius", C.c_float),
        ("albedo_texture", C.c_int32), ("roughness_texture", C.c_int32), ("metalness_texture", C.c_int32),
        ("normal_texture", C.c_int32), ("texture_mapping", C.c_int32), ("texture_scale", C.c_float),
        ("opacity_texture", C.c_int32),
    ]


class pe_camera(C.Structure):
    _fields_ = [("position", F3), ("lower_left", F3), ("horizontal", F3), ("vertical", F3),
                ("u", F3), ("v", F3), ("forward", F3), ("lens_radius", C.c_float), ("orthographic", C.c_int32), ("blades", C.c_int32), ("blade_rotation", C.c_float),
                ("has_shutter_end", C.c_int32), ("end_position", F3), ("end_lower_left", F3), ("end_horizontal", F3),
                ("end_vertical", F3), ("end_u", F3), ("end_v", F3), ("end_forward", F3), ("end_lens_radius", C.c_float)]


class pe_settings(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("max_bounces", C.c_int32), ("rr_depth", C.c_int32),
                ("shadow_quality", C.c_int32), ("filter_type", C.c_int32), ("filter_width", C.c_float),
                ("clamp_indirect", C.c_float), ("seed", C.c_uint64), ("ao_strength", C.c_float),
                ("adaptive_sampling", C.c_int32), ("noise_threshold", C.c_float), ("min_adaptive_samples", C.c_int32),
                ("motion_blur", C.c_int32)]


class pe_scene_info(C.Structure):
    _fields_ = [("triangles", C.c_uint64), ("bvh_nodes", C.c_uint64), ("bvh_leaves", C.c_uint64),
                ("lights", C.c_uint64), ("light_bvh_nodes", C.c_uint64), ("device_bytes", C.c_uint64),
                ("has_environment", C.c_int32), ("light_sampler_mode", C.c_int32)]


class pe_tuning(C.Structure):
    _fields_ = [("tail_paths", C.c_int64), ("closest_traversal", C.c_int32), ("shade_budget", C.c_int32),
                ("any_traversal", C.c_int32), ("wave_slots", C.c_int64)]


class pe_device_info(C.Structure):
    _fields_ = [("name", C.c_char * 128), ("memory_bytes", C.c_uint64), ("compute_major", C.c_int32),
                ("compute_minor", C.c_int32), ("sm_count", C.c_int32), ("usable", C.c_int32),
                ("feature_aovs", C.c_int32), ("feature_light_passes", C.c_int32), ("feature_adaptive", C.c_int32),
                ("pci_bus_id", C.c_char * 32)]


class pe_render_stats(C.Structure):
    _fields_ = [("paths", C.c_uint64), ("closest_rays", C.c_uint64), ("shadow_rays", C.c_uint64),
                ("rejected", C.c_uint64), ("waves", C.c_uint64), ("ms_total", C.c_float),
                ("ms_intersect", C.c_float), ("ms_shadow", C.c_float), ("ms_shade", C.c_float),
                ("intersect_launches", C.c_uint64), ("node_visits", C.c_uint64), ("tri_tests", C.c_uint64),
                ("error_flags", C.c_uint32), ("kernel_launches", C.c_uint64),
                ("shadow_node_visits", C.c_uint64), ("shadow_tri_tests", C.c_uint64),
                ("tail_paths", C.c_uint64), ("ms_tail", C.c_float), ("pad0", C.c_uint32),
                ("tail_closest_rays", C.c_uint64), ("tail_shadow_rays", C.c_uint64)]


class pe_bsdf_query(C.Structure):
    _fields_ = [("wo", F3), ("wi", F3), ("normal", F3), ("ng", F3), ("tangent", F3), ("point", F3),
                ("front_face", C.c_int32), ("wavelength", C.c_float), ("uc", C.c_float), ("u", C.c_float * 2)]


class pe_bsdf_result(C.Structure):
    _fields_ = [("f", F3), ("pdf", C.c_float), ("sampled", C.c_int32), ("wi", F3), ("sf", F3), ("spdf", C.c_float),
                ("delta", C.c_int32), ("pass_through", C.c_int32), ("subsurface", C.c_int32), ("weight", F3)]


PE_REQ_QUEUED, PE_REQ_ACTIVE, PE_REQ_DONE, PE_REQ_FAILED, PE_REQ_RELEASED = 0, 1, 2, 3, 4
PE_GUIDE_MLP_PARAMS, PE_GUIDE_GRID_PARAMS, PE_GUIDE_OUTPUTS = 15616, 16 * 262144 * 2, 40


class pe_guide_info(C.Structure):
    _fields_ = [("mode", C.c_int32), ("ready", C.c_int32), ("steps", C.c_int64), ("last_loss", C.c_float),
                ("pad", C.c_float)]


class pe_sdtree_info(C.Structure):
    _fields_ = [("ready", C.c_int32), ("refinements", C.c_int32), ("samples", C.c_int32),
                ("spatial_leaves", C.c_int32), ("quad_nodes", C.c_int64), ("energy", C.c_double)]


class pe_aov_films(C.Structure):
    _fields_ = [("albedo_sum", C.POINTER(C.c_float)), ("albedo_count", C.POINTER(C.c_uint32)),
                ("albedo_sum_sq", C.POINTER(C.c_float)), ("normal_sum", C.POINTER(C.c_float)),
                ("normal_count", C.POINTER(C.c_uint32)), ("alpha_sum", C.POINTER(C.c_float)),
                ("alpha_count", C.POINTER(C.c_uint32)), ("alpha_sum_sq", C.POINTER(C.c_float))]


PE_MAX_LIGHT_GROUPS = 16
PE_LIGHT_PASSES = 8


class pe_film_arrays(C.Structure):
    _fields_ = [("sum", C.POINTER(C.c_float)), ("count", C.POINTER(C.c_uint32)), ("sum_sq", C.POINTER(C.c_float))]


class pe_pass_films(C.Structure):
    _fields_ = [("light", pe_film_arrays * PE_LIGHT_PASSES), ("depth", pe_film_arrays), ("position", pe_film_arrays),
                ("object_id", pe_film_arrays), ("material_id", pe_film_arrays), ("n_groups", C.c_int32),
                ("pad", C.c_int32), ("groups", pe_film_arrays * PE_MAX_LIGHT_GROUPS),
                ("crypto_object", C.POINTER(C.c_float)), ("crypto_material", C.POINTER(C.c_float))]


class pe_request_desc(C.Structure):
    _fields_ = [("scene", C.c_int32), ("camera", pe_camera), ("settings", pe_settings), ("spp", C.c_int32),
                ("priority", C.c_int32)]


class pe_request_status(C.Structure):
    _fields_ = [("state", C.c_int32), ("samples_done", C.c_int32), ("submit_ms", C.c_double),
                ("start_ms", C.c_double), ("done_ms", C.c_double), ("paths", C.c_uint64), ("error", C.c_int32),
                ("pad", C.c_int32)]


class pe_server_stats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("queued", C.c_uint64), ("active", C.c_uint64), ("waves", C.c_uint64), ("paths", C.c_uint64),
                ("segments", C.c_uint64), ("busy_ms", C.c_double), ("film_bytes", C.c_uint64),
                ("film_bytes_peak", C.c_uint64), ("budget_bytes", C.c_uint64), ("scene_bytes", C.c_uint64)]


# Every symbol include/photon_cuda.h declares, with its ctypes signature.
P = C.c_void_p
FP = C.POINTER(C.c_float)
IP = C.POINTER(C.c_int32)
UP = C.POINTER(C.c_uint32)
SIGNATURES = {
    "pe_last_error": (C.c_char_p, []),
    "pe_abi_version": (C.c_int32, []),
    "pe_scene_set_shadow_catcher": (C.c_int32, [P, C.c_int32]),
    "pe_scene_set_light_group": (C.c_int32, [P, C.c_int32, C.c_char_p]),
    "pe_scene_light_groups": (C.c_int32, [P, C.c_char_p, C.c_int32]),
    "pe_device_render_passes": (C.c_int32, [P, C.POINTER(pe_camera), C.POINTER(pe_settings), C.c_int32, C.c_int32,
                                            C.POINTER(C.c_int32), C.POINTER(C.c_float), C.POINTER(C.c_uint32),
                                            C.POINTER(C.c_float), C.POINTER(pe_aov_films), C.POINTER(pe_pass_films),
                                            C.POINTER(C.c_uint64)]),
    "pe_device_render_aovs": (C.c_int32, [P, C.POINTER(pe_camera), C.POINTER(pe_settings), C.c_int32, C.c_int32,
                                          C.c_void_p, FP, C.POINTER(C.c_uint32), FP, C.POINTER(pe_aov_films),
                                          C.POINTER(C.c_uint64)]),
    "pe_scene_tag_shape": (C.c_int32, [P, C.c_int32, C.c_uint64]),
    "pe_scene_set_light_link": (C.c_int32, [P, C.c_int32, C.c_int32, C.POINTER(C.c_uint64), C.c_int32, C.c_int32,
                                            C.POINTER(C.c_uint64), C.c_int32]),
    "pe_material_defaults": (None, [C.c_int32, C.POINTER(pe_material)]),
    "pe_scene_create": (P, []),
    "pe_scene_destroy": (None, [P]),
    "pe_scene_add_material": (C.c_int32, [P, C.POINTER(pe_material)]),
    "pe_scene_add_texture": (C.c_int32, [P, C.POINTER(C.c_float), C.c_int32, C.c_int32]),
    "pe_scene_build_texture_mipmaps": (C.c_int32, [P, C.c_int32]),
    "pe_scene_add_texture_u8": (C.c_int32, [P, C.POINTER(C.c_uint8), C.c_int32, C.c_int32, C.c_int32]),
    "pe_scene_set_material": (C.c_int32, [P, C.c_int32, C.POINTER(pe_material)]),
    "pe_scene_set_shape_name": (C.c_int32, [P, C.c_int32, C.c_char_p]),
    "pe_scene_set_shape_visibility": (C.c_int32, [P, C.c_int32, C.c_uint32]),
    "pe_scene_set_material_name": (C.c_int32, [P, C.c_int32, C.c_char_p]),
    "pe_device_update_materials": (C.c_int32, [P, P]),
    "pe_device_update_lights": (C.c_int32, [P, P]),
    "pe_scene_set_area_light_radiance": (C.c_int32, [P, C.c_int32, C.POINTER(C.c_float)]),
    "pe_scene_add_blas": (C.c_int32, [P, FP, C.c_uint32, FP, FP, UP, C.c_uint32]),
    "pe_scene_add_instance": (C.c_int32, [P, C.c_int32, FP, FP, C.c_int32]),
    "pe_scene_set_instance_transform": (C.c_int32, [P, C.c_int32, FP, FP]),
    "pe_scene_refit": (C.c_int32, [P]),
    "pe_scene_set_instance_motion": (C.c_int32, [P, C.c_int32, FP, FP]),
    "pe_mat4_inverse": (None, [FP, FP]),
    "pe_device_trace_rays": (C.c_int32, [P, FP, FP, FP, C.c_int32, C.c_int32, C.c_uint32, C.c_float, IP, IP, FP]),
    "pe_scene_shape_bounds": (C.c_int32, [P, C.c_int32, FP]),
    "pe_device_update_transforms": (C.c_int32, [P, P]),
    "pe_scene_add_sphere": (C.c_int32, [P, C.POINTER(C.c_float), C.c_float, C.c_int32]),
    "pe_scene_add_mesh": (C.c_int32, [P, FP, C.c_uint32, FP, FP, UP, C.c_uint32, C.c_int32]),
    "pe_scene_add_area_light": (C.c_int32, [P, FP, FP, FP, FP, C.c_int32]),
    "pe_scene_set_environment": (C.c_int32, [P, FP, C.c_int32, C.c_int32, C.c_float, C.c_float]),
    "pe_scene_set_sun": (C.c_int32, [P, FP, C.c_float, FP]),
    "pe_scene_set_background": (C.c_int32, [P, C.c_int32, FP]),
    "pe_scene_build": (C.c_int32, [P]),
    "pe_scene_get_info": (C.c_int32, [P, C.POINTER(pe_scene_info)]),
    "pe_camera_perspective": (None, [FP, FP, FP, C.c_float, C.c_float, C.POINTER(pe_camera)]),
    "pe_camera_thin_lens": (None, [FP, FP, FP, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int32, C.c_float,
                                   C.POINTER(pe_camera)]),
    "pe_camera_orthographic": (None, [FP, FP, FP, C.c_float, C.c_float, C.POINTER(pe_camera)]),
    "pe_device_count": (C.c_int32, []),
    "pe_device_create": (P, [C.c_int32, C.c_char_p, C.c_size_t]),
    "pe_device_destroy": (None, [P]),
    "pe_device_info_get": (C.c_int32, [P, C.POINTER(pe_device_info)]),
    "pe_device_set_scene": (C.c_int32, [P, P]),
    "pe_device_has_scene": (C.c_int32, [P]),
    "pe_device_render": (C.c_int32, [P, C.POINTER(pe_camera), C.POINTER(pe_settings), C.c_int32, C.c_int32,
                                     IP, FP, UP, FP, C.POINTER(C.c_uint64)]),
    "pe_device_render_resident": (C.c_int32, [P, C.POINTER(pe_camera), C.POINTER(pe_settings), C.c_int32, C.c_int32, IP]),
    "pe_device_render_region": (C.c_int32, [P, C.POINTER(pe_camera), C.POINTER(pe_settings), C.c_int32, C.c_int32,
                                            C.c_int32, C.c_int32, C.c_int32, C.c_int32, IP, FP, UP, FP,
                                            C.POINTER(C.c_uint64)]),
    "pe_device_film_clear": (C.c_int32, [P]),
    "pe_device_render_tile_noalloc": (C.c_int32, [P, C.POINTER(pe_camera), C.POINTER(pe_settings), C.c_int32,
                                                  C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_void_p,
                                                  C.c_void_p, C.c_void_p]),
    "pe_device_film_read": (C.c_int32, [P, FP, UP, FP]),
    "pe_device_synchronize": (C.c_int32, [P]),
    "pe_device_last_stats": (C.c_int32, [P, C.POINTER(pe_render_stats)]),
    "pe_device_set_counting": (C.c_int32, [P, C.c_int32]),
    "pe_device_set_tail_paths": (C.c_int32, [P, C.c_int64]),
    "pe_device_tail_paths": (C.c_int64, [P]),
    "pe_device_get_tuning": (C.c_int32, [P, C.POINTER(pe_tuning)]),
    "pe_device_set_tuning": (C.c_int32, [P, C.POINTER(pe_tuning)]),
    "pe_device_autotune_log": (C.c_int32, [P, C.c_char_p, C.c_size_t]),
    "pe_device_autotune": (C.c_int32, [P, C.POINTER(pe_camera), C.POINTER(pe_settings), C.c_int32, C.POINTER(C.c_int64)]),
    "pe_device_timer_begin": (C.c_int32, [P]),
    "pe_device_timer_end": (C.c_int32, [P, FP]),
    "pe_device_trace_primary": (C.c_int32, [P, C.POINTER(pe_camera), C.POINTER(pe_settings), C.c_int32, IP, IP, FP]),
    "pe_device_trace_primary_ordered": (C.c_int32, [P, C.POINTER(pe_camera), C.POINTER(pe_settings), C.c_int32, IP, IP,
                                                    FP]),
    "pe_device_sobol": (C.c_int32, [P, C.c_uint64, IP, IP, IP, C.c_size_t, C.c_int32, FP]),
    "pe_device_bsdf_probe": (C.c_int32, [P, C.c_int32, C.POINTER(pe_bsdf_query), C.c_size_t, C.POINTER(pe_bsdf_result)]),
    "pe_device_guide_reset": (C.c_int32, [P, C.c_uint64, FP, FP]),
    "pe_device_guide_get": (C.c_int32, [P, FP, FP]),
    "pe_device_guide_set": (C.c_int32, [P, FP, FP]),
    "pe_device_guide_eval": (C.c_int32, [P, FP, C.c_int64, C.c_int32, FP]),
    "pe_device_guide_grad": (C.c_int32, [P, FP, C.c_int64, C.c_float, FP, FP, FP]),
    "pe_device_set_guiding": (C.c_int32, [P, C.c_int32, C.c_int32, C.c_float]),
    "pe_device_guide_info": (C.c_int32, [P, C.POINTER(pe_guide_info)]),
    "pe_device_sdtree_info": (C.c_int32, [P, C.POINTER(pe_sdtree_info)]),
    "pe_sdtree_probe": (C.c_int32, [FP, FP, C.c_int32, FP, FP, C.c_int32, FP, FP, C.c_int32, FP, FP]),
    "pe_server_create": (P, [P, C.c_uint64, C.c_char_p, C.c_size_t]),
    "pe_server_destroy": (None, [P]),
    "pe_server_add_scene": (C.c_int32, [P, P]),
    "pe_server_submit": (C.c_int64, [P, C.POINTER(pe_request_desc)]),
    "pe_server_status": (C.c_int32, [P, C.c_int64, C.POINTER(pe_request_status)]),
    "pe_server_wait": (C.c_int32, [P, C.c_int64, C.c_int32]),
    "pe_server_take": (C.c_int32, [P, C.c_int64, FP, UP, FP]),
    "pe_server_get_stats": (C.c_int32, [P, C.POINTER(pe_server_stats)]),
}

_lib = None


def load(path: pathlib.Path | str | None = None) -> C.CDLL:
    """Loads libphoton_cuda.so (building nothing); raises if it is absent."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = pathlib.Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"{p} is missing: build it with photon-engine_b200/build.py (no CPU fallback exists)")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


class PhotonError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def check(status: int) -> None:
    if status != PE_OK:
        msg = load().pe_last_error()
        raise PhotonError(status, msg.decode() if msg else "")


def fptr(a):
    return a.ctypes.data_as(FP) if a is not None else None


def uptr(a):
    return a.ctypes.data_as(UP) if a is not None else None


def iptr(a):
    return a.ctypes.data_as(IP) if a is not None else None


def f3(v) -> C.Array:
    return F3(*[float(x) for x in v])

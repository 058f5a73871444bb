"""ctypes binding of libcupbr_b200.so (the C ABI declared in include/cupbr_c.h).

The product path has no fallback: if the shared library is missing or fails
to load, importing this module raises.  Every wrapped call checks the int
status and raises CupbrError with cupbr_last_error().
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcupbr_b200.so")


class CupbrError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"cupbr error {code}: {msg}")
        self.code = code


class Vec3(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]

    @staticmethod
    def of(v) -> "Vec3":
        return Vec3(float(v[0]), float(v[1]), float(v[2]))

    def tuple(self):
        return (self.x, self.y, self.z)


class Material(C.Structure):
    _fields_ = [("type", C.c_int32), ("albedo_e", Vec3), ("albedo_d", Vec3), ("albedo_s", Vec3),
                ("shininess", C.c_float), ("roughness", C.c_float), ("eta", C.c_float),
                ("sigma_s", Vec3), ("sigma_a", Vec3), ("g", C.c_float), ("interface_glass", C.c_int32)]


class Light(C.Structure):
    _fields_ = [("type", C.c_int32), ("position", Vec3), ("intensity", Vec3), ("radiance", Vec3),
                ("half_extend1", Vec3), ("half_extend2", Vec3)]


class Camera(C.Structure):
    _fields_ = [("position", Vec3), ("x_axis", Vec3), ("y_axis", Vec3), ("z_axis", Vec3),
                ("aspect_ratio", C.c_float), ("moved", C.c_int32)]


class MediumDesc(C.Structure):
    _fields_ = [("nx", C.c_uint32), ("ny", C.c_uint32), ("nz", C.c_uint32), ("lo", Vec3), ("hi", Vec3),
                ("majorant", C.c_float), ("albedo", C.c_float), ("g", C.c_float), ("q", C.c_float)]


class View(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("camera", Camera), ("width", C.c_uint32), ("height", C.c_uint32),
                ("spp", C.c_uint32), ("frame0", C.c_uint32), ("device_image", C.c_void_p)]


class CacheDesc(C.Structure):
    _fields_ = [("cache_depth", C.c_uint32), ("train_stride", C.c_uint32), ("batch", C.c_uint32),
                ("samples_per_frame", C.c_uint32), ("learning_rate", C.c_float), ("seed", C.c_uint32),
                ("loss", C.c_uint32), ("weight_average", C.c_float), ("cache_specular", C.c_uint32),
                ("train_suffix", C.c_uint32)]


class BvhParams(C.Structure):
    _fields_ = [("max_leaf_size", C.c_int32), ("traversal_cost", C.c_float), ("top_bfs_levels", C.c_int32),
                ("builder", C.c_int32)]


class SceneInfo(C.Structure):
    _fields_ = [("objects", C.c_uint32), ("lights", C.c_uint32), ("triangles", C.c_uint32), ("spheres", C.c_uint32),
                ("quads", C.c_uint32), ("planes", C.c_uint32), ("bvh_nodes", C.c_uint32),
                ("bvh_leaves", C.c_uint32), ("bvh_depth", C.c_uint32), ("bvh_sah_cost", C.c_double),
                ("device_bytes", C.c_uint64), ("env_width", C.c_uint32), ("env_height", C.c_uint32),
                ("committed", C.c_int32), ("bvh_builder", C.c_int32), ("bvh_build_ms", C.c_double),
                ("commit_ms", C.c_double)]


class ObjectDesc(C.Structure):
    _fields_ = [("type", C.c_int32), ("material", Material), ("p0", Vec3), ("p1", Vec3), ("p2", Vec3),
                ("p3", Vec3), ("radius", C.c_float), ("triangle_begin", C.c_uint32),
                ("triangle_count", C.c_uint32), ("finite_box", C.c_int32), ("box_lo", Vec3), ("box_hi", Vec3)]


_P = C.c_void_p
_F = C.POINTER(C.c_float)
_U32 = C.c_uint32
_I32 = C.c_int32

# name -> argtypes (all return int status unless listed in _RESTYPES)
_PROTOS = {
    "cupbr_last_error": [],
    "cupbr_version": [],
    "cupbr_material_default": [C.POINTER(Material)],
    "cupbr_camera_default": [_U32, _U32, C.POINTER(Camera)],
    "cupbr_scene_load_xml": [C.c_char_p, C.POINTER(_P)],
    "cupbr_scene_load_xml_ex": [C.c_char_p, C.POINTER(BvhParams), C.POINTER(_P)],
    "cupbr_scene_parse_xml": [C.c_char_p, C.POINTER(_P)],
    "cupbr_scene_create": [C.POINTER(_P)],
    "cupbr_scene_add_sphere": [_P, Vec3, C.c_float, C.POINTER(Material), C.POINTER(_U32)],
    "cupbr_scene_add_plane": [_P, Vec3, Vec3, C.POINTER(Material), C.POINTER(_U32)],
    "cupbr_scene_add_quad": [_P, Vec3, Vec3, Vec3, Vec3, C.POINTER(Material), C.POINTER(_U32)],
    "cupbr_scene_add_triangle": [_P, Vec3, Vec3, Vec3, C.POINTER(Material), C.POINTER(_U32)],
    "cupbr_scene_add_mesh": [_P, _P, _U32, _P, _U32, Vec3, Vec3, C.POINTER(Material), C.POINTER(_U32)],
    "cupbr_scene_add_mesh_obj": [_P, C.c_char_p, Vec3, Vec3, C.POINTER(Material), C.POINTER(_U32)],
    "cupbr_scene_add_light": [_P, C.POINTER(Light)],
    "cupbr_scene_set_volume": [_P, Vec3, Vec3, C.c_float],
    "cupbr_scene_set_environment": [_P, _P, _U32, _U32],
    "cupbr_scene_load_environment": [_P, C.c_char_p],
    "cupbr_scene_commit": [_P, C.POINTER(BvhParams)],
    "cupbr_scene_destroy": [_P],
    "cupbr_scene_get_info": [_P, C.POINTER(SceneInfo)],
    "cupbr_scene_get_object": [_P, _U32, C.POINTER(ObjectDesc)],
    "cupbr_scene_get_triangles": [_P, _U32, _P, _U32],
    "cupbr_scene_get_bvh": [_P, _P, _U32, C.POINTER(_U32)],
    "cupbr_scene_get_key_slots": [_P, _P, _U32, C.POINTER(_U32)],
    "cupbr_scene_get_light": [_P, _U32, C.POINTER(Light)],
    "cupbr_scene_trace": [_P, _U32, _P, _P, _P, _P, _P],
    "cupbr_scene_visible": [_P, _U32, _P, _P, _P, _P],
    "cupbr_renderer_create": [_I32, C.POINTER(_P)],
    "cupbr_renderer_destroy": [_P],
    "cupbr_renderer_set_output_size": [_P, _U32, _U32],
    "cupbr_renderer_register_scene": [_P, _P],
    "cupbr_renderer_set_method": [_P, _I32],
    "cupbr_renderer_get_method": [_P, C.POINTER(_I32)],
    "cupbr_renderer_render": [_P, C.POINTER(Camera)],
    "cupbr_renderer_reset": [_P],
    "cupbr_renderer_render_frames": [_P, C.POINTER(Camera), _U32],
    "cupbr_renderer_set_batch_paths": [_P, _U32],
    "cupbr_renderer_set_tail_paths": [_P, _U32],
    "cupbr_renderer_set_pipelined": [_P, _I32],
    "cupbr_renderer_set_russian_roulette": [_P, _I32],
    "cupbr_renderer_set_max_trace_depth": [_P, _U32],
    "cupbr_renderer_get_max_trace_depth": [_P, C.POINTER(_U32)],
    "cupbr_renderer_get_output": [_P, C.POINTER(_P), C.POINTER(_U32), C.POINTER(_U32)],
    "cupbr_renderer_get_gradient_x": [_P, C.POINTER(_P)],
    "cupbr_renderer_get_gradient_y": [_P, C.POINTER(_P)],
    "cupbr_renderer_get_frame_index": [_P, C.POINTER(_U32)],
    "cupbr_renderer_set_frame_index": [_P, _U32],
    "cupbr_renderer_set_stream": [_P, _P],
    "cupbr_renderer_get_error_count": [_P, C.POINTER(_U32)],
    "cupbr_renderer_set_instrumented": [_P, _I32],
    "cupbr_renderer_get_stats": [_P, _P],
    "cupbr_renderer_set_profiling": [_P, _I32],
    "cupbr_renderer_get_stage_times": [_P, _P, C.POINTER(_U32), C.POINTER(_U32)],
    "cupbr_pathtracing": [_P, C.POINTER(Camera), _U32, _U32, _I32, _P, _U32, _U32, _P],
    "cupbr_tonemapper_create": [_I32, C.POINTER(_P)],
    "cupbr_tonemapper_destroy": [_P],
    "cupbr_tonemapper_register_image": [_P, _P, _U32, _U32],
    "cupbr_tonemapper_tonemap": [_P],
    "cupbr_tonemapper_get_render_buffer": [_P, C.POINTER(_P), C.POINTER(_U32), C.POINTER(_U32)],
    "cupbr_tonemapper_get_type": [_P, C.POINTER(_I32)],
    "cupbr_tonemapper_set_type": [_P, _I32],
    "cupbr_tonemapper_set_exposure": [_P, C.c_float],
    "cupbr_tonemapper_set_stream": [_P, _P],
    "cupbr_tonemapper_save_to_file": [_P, C.c_char_p],
    "cupbr_tonemap": [_P, _U32, _U32, _I32, C.c_float, _P, _P],
    "cupbr_tonemap_verify_levels": [_P, _P, _P],
    "cupbr_postprocessor_create": [C.POINTER(_P)],
    "cupbr_postprocessor_destroy": [_P],
    "cupbr_postprocessor_register_image": [_P, _P, _U32, _U32],
    "cupbr_postprocessor_get_buffer": [_P, C.POINTER(_P)],
    "cupbr_postprocessor_bloom": [_P, _F],
    "cupbr_postprocessor_set_stream": [_P, _P],
    "cupbr_postprocessor_bloom_tonemap": [_P, _F, _I32, C.c_float, _P],
    "cupbr_bloom_noalloc": [_P, _U32, _U32, _F, _P, _P],
    "cupbr_scene_get_camera": [_P, _U32, _U32, C.POINTER(Camera)],
    "cupbr_scene_set_camera": [_P, Vec3, C.c_float, C.c_float],
    "cupbr_scene_pick": [_P, C.POINTER(Camera), _U32, _U32, _U32, _U32, C.POINTER(Material), C.POINTER(C.c_int32)],
    "cupbr_scene_update_material": [_P, C.c_int32, C.POINTER(Material)],
    "cupbr_batch_create": [C.POINTER(View), _U32, _U32, C.POINTER(_P)],
    "cupbr_batch_destroy": [_P],
    "cupbr_batch_launch": [_P, _P],
    "cupbr_batch_advance": [_P],
    "cupbr_batch_set_frame0": [_P, _U32, _U32],
    "cupbr_batch_get_info": [_P, C.POINTER(_U32), C.POINTER(C.c_uint64), C.POINTER(_U32), C.POINTER(_U32)],
    "cupbr_batch_configure": [_P, _U32, C.c_float],
    "cupbr_batch_autotune": [_P, _P, C.POINTER(C.c_float)],
    "cupbr_batch_autotune_ex": [_P, _P, _U32, C.POINTER(C.c_float)],
    "cupbr_batch_set_mode": [_P, C.c_int32, _U32, _U32, C.c_int32],
    "cupbr_batch_get_mode": [_P, C.POINTER(C.c_int32), C.POINTER(_U32), C.POINTER(_U32), C.POINTER(C.c_int32)],
    "cupbr_batch_get_error_count": [_P, C.POINTER(_U32)],
    "cupbr_batch_set_barrier_probe": [_P, C.c_uint64],
    "cupbr_batch_backward": [_P, C.POINTER(C.c_uint64), C.c_int32, _P],
    "cupbr_batch_get_texture_gradient": [_P, _P, C.POINTER(_P), C.POINTER(_U32), C.POINTER(_U32)],
    "cupbr_medium_create": [C.POINTER(MediumDesc), C.POINTER(_P)],
    "cupbr_medium_destroy": [_P],
    "cupbr_medium_param_count": [_P, C.POINTER(_U32)],
    "cupbr_medium_forward": [_P, _P, _P, C.POINTER(Camera), _U32, _U32, _U32, _U32, _U32, _P, _P],
    "cupbr_medium_backward": [_P, _P, _P, C.POINTER(Camera), _U32, _U32, _U32, _U32, _U32, _P, _P, _P, _P],
    "cupbr_medium_get_error_count": [_P, C.POINTER(_U32)],
    "cupbr_medium_set_batch_paths": [_P, _U32],
    "cupbr_medium_set_profiling": [_P, C.c_int32],
    "cupbr_medium_get_stage_times": [_P, _F, C.POINTER(_U32), C.POINTER(_U32)],
    "cupbr_medium_set_instrumented": [_P, C.c_int32],
    "cupbr_medium_get_stats": [_P, C.POINTER(C.c_uint64)],
    "cupbr_cache_create": [_P, C.POINTER(CacheDesc), C.POINTER(_P)],
    "cupbr_cache_destroy": [_P],
    "cupbr_cache_param_count": [],
    "cupbr_cache_get_bounds": [_P, _F, _F],
    "cupbr_cache_get_params": [_P, _P],
    "cupbr_cache_set_params": [_P, _P],
    "cupbr_cache_save": [_P, C.c_char_p],
    "cupbr_cache_load": [_P, C.c_char_p],
    "cupbr_cache_infer": [_P, _P, _U32, _P, _P],
    "cupbr_cache_train_step": [_P, _P, _U32, _P],
    "cupbr_cache_get_gradient": [_P, _P],
    "cupbr_cache_get_loss": [_P, C.POINTER(C.c_float), C.POINTER(C.c_float)],
    "cupbr_cache_render": [_P, _P, C.POINTER(Camera), _U32, _U32, _U32, _U32, _U32, _I32, _P, _P],
    "cupbr_cache_get_counters": [_P, C.POINTER(_U32)],
    "cupbr_cache_check": [_P, _P],
    "cupbr_renderer_set_estimator": [_P, C.c_int32],
    "cupbr_renderer_set_persistent": [_P, C.c_int32],
    "cupbr_renderer_get_estimator": [_P, C.POINTER(C.c_int32)],
    "cupbr_scene_set_albedo_texture": [_P, _P, _U32, _U32],
    "cupbr_scene_set_object_texture": [_P, _U32, Vec3, Vec3, Vec3],
    "cupbr_scene_get_albedo_texture": [_P, C.POINTER(_P), C.POINTER(_U32), C.POINTER(_U32)],
    "cupbr_debug_fail_allocation": [C.c_int64],
    "cupbr_gdpt_reconstruct": [_U32, _U32, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P],
    "cupbr_cache_set_wait_probe": [_P, _U32],
    "cupbr_cache_set_profiling": [_P, _I32],
    "cupbr_cache_set_batch_paths": [_P, _U32],
    "cupbr_cache_set_tail_paths": [_P, _U32],
    "cupbr_cache_get_stage_times": [_P, _F, C.POINTER(_U32)],
    "cupbr_device_alloc": [C.POINTER(_P), C.c_size_t],
    "cupbr_device_free": [_P],
    "cupbr_memcpy_h2d": [_P, _P, C.c_size_t, _P],
    "cupbr_memcpy_d2h": [_P, _P, C.c_size_t, _P],
    "cupbr_stream_synchronize": [_P],
    "cupbr_save_bmp": [C.c_char_p, _P, _U32, _U32],
    "cupbr_save_pfm": [C.c_char_p, _P, _U32, _U32],
}
_RESTYPES = {"cupbr_last_error": C.c_char_p, "cupbr_version": C.c_char_p, "cupbr_cache_param_count": C.c_uint32}


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m cupbr_b200.build` "
                          "(there is no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    for name, args in _PROTOS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RESTYPES.get(name, C.c_int)
    return lib


lib = _load()


def check(status: int) -> None:
    if status != 0:
        raise CupbrError(status, lib.cupbr_last_error().decode(errors="replace"))


def call(name: str, *args) -> None:
    check(getattr(lib, name)(*args))


def exported_symbols() -> list[str]:
    return list(_PROTOS)

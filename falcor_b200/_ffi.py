"""ctypes binding of the C-ABI declared in include/fpt.h.

The library (falcor_b200/_lib/libfpt.so) is built in-tree by
``falcor_b200.build.build()``.  Loading fails loudly when it is missing: there
is no Python or CPU fallback for any operation of this package.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libfpt.so"

u32 = C.c_uint32
f32 = C.c_float


class fpt_vertex(C.Structure):
    _fields_ = [("position", f32 * 3), ("normal", f32 * 3), ("tangent", f32 * 4), ("texcoord", f32 * 2)]


class fpt_geometry_instance(C.Structure):
    _fields_ = [("vb_offset", u32), ("ib_offset", u32), ("triangle_count", u32), ("material_id", u32), ("flags", u32)]


class fpt_material(C.Structure):
    _fields_ = [("base_color", f32 * 4), ("specular", f32 * 4), ("emissive", f32 * 3), ("emissive_factor", f32),
                ("ior", f32), ("specular_transmission", f32), ("diffuse_transmission", f32), ("transmission", f32 * 3),
                ("flags", u32)]


class fpt_camera(C.Structure):
    _fields_ = [("position", f32 * 3), ("target", f32 * 3), ("up", f32 * 3), ("focal_length", f32), ("frame_height", f32),
                ("aspect_ratio", f32), ("near_z", f32), ("far_z", f32), ("focal_distance", f32), ("jitter_x", f32),
                ("jitter_y", f32)]


class fpt_camera_data(C.Structure):
    _fields_ = [("posW", f32 * 3), ("cameraU", f32 * 3), ("cameraV", f32 * 3), ("cameraW", f32 * 3), ("nearZ", f32),
                ("farZ", f32), ("jitterX", f32), ("jitterY", f32)]


class fpt_envmap_desc(C.Structure):
    _fields_ = [("width", u32), ("height", u32), ("rgb", C.POINTER(f32)), ("tint", f32 * 3), ("intensity", f32)]


class fpt_texture_desc(C.Structure):
    _fields_ = [("width", u32), ("height", u32), ("format", u32), ("texels", C.c_void_p)]


TEXTURE_RGBA8_UNORM_SRGB, TEXTURE_RGBA8_UNORM, TEXTURE_RGBA32_FLOAT = 0, 1, 2


class fpt_scene_desc(C.Structure):
    _fields_ = [("vertices", C.POINTER(fpt_vertex)), ("vertex_count", u32), ("indices", C.POINTER(u32)), ("index_count", u32),
                ("instances", C.POINTER(fpt_geometry_instance)), ("instance_count", u32),
                ("materials", C.POINTER(fpt_material)), ("material_count", u32), ("camera", fpt_camera),
                ("envmap", C.POINTER(fpt_envmap_desc)), ("textures", C.POINTER(fpt_texture_desc)), ("texture_count", u32),
                ("base_color_textures", C.POINTER(u32))]


class fpt_procedural_params(C.Structure):
    _fields_ = [("kind", u32), ("seed", u32), ("grid_res", u32), ("soup_triangles", u32), ("material_count", u32),
                ("emissive_count", u32), ("sphere_subdiv", u32), ("envmap_width", u32), ("envmap_height", u32),
                ("lambert", u32), ("aspect_ratio", f32)]


class fpt_bsdf_probe(C.Structure):
    _fields_ = [("lobe", u32), ("wi", f32 * 3), ("params", f32 * 4), ("sample_count", u32), ("thread_sample_count", u32),
                ("phi_bins", u32), ("cos_bins", u32), ("bin_sample_count", u32)]


class fpt_hitinfo_bits(C.Structure):
    _fields_ = [("type_bits", u32), ("instance_id_bits", u32), ("primitive_index_bits", u32)]


class fpt_bvh_view(C.Structure):
    _fields_ = [("nodes", C.c_void_p), ("node_count", u32), ("tris", C.c_void_p), ("tri_count", u32),
                ("scene_lo", f32 * 3), ("scene_hi", f32 * 3)]


class fpt_scene_info(C.Structure):
    _fields_ = [("triangle_count", u32), ("instance_count", u32), ("material_count", u32), ("emissive_triangle_count", u32),
                ("bvh_node_count", u32), ("has_envmap", u32), ("hit_bits", fpt_hitinfo_bits), ("bvh_build_seconds", C.c_double),
                ("device_bytes", C.c_uint64), ("camera", fpt_camera_data)]


class fpt_frame_io(C.Structure):
    _fields_ = [("width", u32), ("height", u32), ("frame_index", u32), ("prng_dimension", u32),
                ("vbuffer", C.c_void_p), ("color", C.c_void_p), ("ray_count", C.c_void_p), ("path_length", C.c_void_p),
                ("d_color", C.c_void_p), ("vbuffer_out", C.c_void_p), ("sample_color", C.c_void_p),
                ("src", C.c_void_p), ("dst", C.c_void_p), ("src_width", u32), ("src_height", u32), ("refresh", u32),
                ("depth", C.c_void_p), ("mvec", C.c_void_p), ("view_w", C.c_void_p), ("mask", C.c_void_p),
                ("hit_trace", C.c_void_p)]


class fpt_batch_tuning(C.Structure):
    _fields_ = [("wave_capacity", u32), ("shade_grid_scale", u32), ("fetch_chunk", u32)]


class fpt_grad_buffers(C.Structure):
    _fields_ = [("material", C.c_void_p), ("mesh_position", C.c_void_p), ("material_dim", u32), ("position_dim", u32),
                ("mesh_normal", C.c_void_p), ("mesh_tangent", C.c_void_p), ("normal_dim", u32), ("tangent_dim", u32),
                ("base_color_texture", C.c_void_p), ("texture_dim", u32)]


class fpt_grad_config(C.Structure):
    _fields_ = [("grad_type", u32), ("dim", u32), ("hash_size", u32)]


class fpt_light_bvh_view(C.Structure):
    _fields_ = [("nodes", C.POINTER(u32)), ("node_count", u32), ("triangle_indices", C.POINTER(u32)),
                ("triangle_index_count", u32), ("bitmasks", C.POINTER(C.c_uint64)), ("bitmask_count", u32)]


class fpt_pass_stats(C.Structure):
    _fields_ = [("paths", C.c_uint64), ("rays", C.c_uint64), ("device_error", u32), ("kernel_launches", u32),
                ("adjoint_checkpointed", u32), ("reserved", u32), ("checkpoint_bytes", C.c_uint64)]


class fpt_batch_request(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("width", u32), ("height", u32), ("spp", u32), ("max_bounces", u32), ("seed", u32),
                ("color", C.c_void_p)]


FPT_OK = 0
STATUS_NAMES = {0: "FPT_OK", 1: "FPT_ERR_INVALID_ARG", 2: "FPT_ERR_CUDA", 3: "FPT_ERR_OOM", 4: "FPT_ERR_NO_SCENE",
                5: "FPT_ERR_UNSUPPORTED", 6: "FPT_ERR_DEVICE", 7: "FPT_ERR_TIMEOUT", 8: "FPT_ERR_NO_DEVICE"}

# Every symbol include/fpt.h declares, with (restype, argtypes).
_P = C.c_void_p
SIGNATURES = {
    "fpt_version": (C.c_char_p, []),
    "fpt_last_error": (C.c_char_p, []),
    "fpt_device_count": (C.c_int, []),
    "fpt_procedural_scene": (C.c_int, [C.POINTER(fpt_procedural_params), C.POINTER(_P)]),
    "fpt_scene_host_desc": (C.POINTER(fpt_scene_desc), [_P]),
    "fpt_scene_host_free": (None, [_P]),
    "fpt_camera_compute": (C.c_int, [C.POINTER(fpt_camera), C.POINTER(fpt_camera_data)]),
    "fpt_hitinfo_compute_bits": (C.c_int, [C.POINTER(fpt_scene_desc), C.POINTER(fpt_hitinfo_bits)]),
    "fpt_bvh_build": (C.c_int, [C.POINTER(fpt_scene_desc), C.POINTER(_P)]),
    "fpt_bvh_get_view": (C.c_int, [_P, C.POINTER(fpt_bvh_view), C.POINTER(u32), C.POINTER(C.c_double)]),
    "fpt_bvh_free": (None, [_P]),
    "fpt_scene_create": (C.c_int, [C.POINTER(fpt_scene_desc), C.POINTER(_P)]),
    "fpt_scene_destroy": (None, [_P]),
    "fpt_scene_get_info": (C.c_int, [_P, C.POINTER(fpt_scene_info)]),
    "fpt_scene_set_camera": (C.c_int, [_P, C.POINTER(fpt_camera)]),
    "fpt_scene_get_material_params": (C.c_int, [_P, C.POINTER(u32), u32, C.POINTER(C.c_float)]),
    "fpt_scene_set_material_params": (C.c_int, [_P, C.POINTER(u32), u32, C.POINTER(C.c_float)]),
    "fpt_scene_set_material_params_device": (C.c_int, [_P, C.POINTER(u32), u32, _P, _P]),
    "fpt_scene_set_texture_device": (C.c_int, [_P, u32, _P, _P]),
    "fpt_scene_get_bvh": (C.c_int, [_P, C.POINTER(fpt_bvh_view)]),
    "fpt_scene_get_alias_table": (C.c_int, [_P, C.POINTER(u32), u32, C.POINTER(f32)]),
    "fpt_pass_create": (C.c_int, [C.c_char_p, C.POINTER(_P)]),
    "fpt_pass_destroy": (None, [_P]),
    "fpt_pass_set_property_int": (C.c_int, [_P, C.c_char_p, C.c_int64]),
    "fpt_pass_set_property_float": (C.c_int, [_P, C.c_char_p, C.c_double]),
    "fpt_pass_set_property_string": (C.c_int, [_P, C.c_char_p, C.c_char_p]),
    "fpt_pass_set_properties_json": (C.c_int, [_P, C.c_char_p]),
    "fpt_pass_get_properties_json": (C.c_int, [_P, C.c_char_p, C.c_size_t]),
    "fpt_pass_reflect_json": (C.c_int, [_P, C.c_char_p, C.c_size_t]),
    "fpt_pass_set_scene": (C.c_int, [_P, _P]),
    "fpt_pass_execute": (C.c_int, [_P, C.POINTER(fpt_frame_io), _P]),
    "fpt_pass_reset": (C.c_int, [_P]),
    "fpt_pass_execute_noalloc": (C.c_int, [_P, C.POINTER(fpt_frame_io), _P]),
    "fpt_fmath_eval": (C.c_int, [u32, u32, u32, _P, _P, _P, _P]),
    "fpt_bsdf_probe_run": (C.c_int, [C.POINTER(fpt_bsdf_probe), _P, _P, _P, _P, _P]),
    "fpt_pass_backward": (C.c_int, [_P, C.POINTER(fpt_frame_io), _P, C.POINTER(fpt_grad_buffers), _P]),
    "fpt_scene_gradients_create": (C.c_int, [C.POINTER(fpt_grad_config), u32, C.POINTER(_P)]),
    "fpt_scene_gradients_destroy": (None, [_P]),
    "fpt_scene_gradients_clear": (C.c_int, [_P, u32, _P]),
    "fpt_scene_gradients_aggregate": (C.c_int, [_P, u32, _P]),
    "fpt_scene_gradients_atomic_add": (C.c_int, [_P, u32, u32, _P, _P, _P, _P]),
    "fpt_scene_gradients_get": (C.c_int, [_P, u32, C.POINTER(C.POINTER(C.c_float)), C.POINTER(u32), C.POINTER(u32)]),
    "fpt_pass_set_scene_gradients": (C.c_int, [_P, _P]),
    "fpt_pass_set_dLdI": (C.c_int, [_P, _P]),
    "fpt_pass_set_diff_debug_params": (C.c_int, [_P, u32, u32, u32, u32, C.POINTER(C.c_float)]),
    "fpt_scene_get_mesh_info": (C.c_int, [_P, u32, C.POINTER(u32), C.POINTER(u32)]),
    "fpt_scene_get_light_bvh": (C.c_int, [_P, _P]),
    "fpt_scene_get_mesh_vertices_and_indices": (C.c_int, [_P, u32, _P, _P, _P, _P]),
    "fpt_scene_set_mesh_vertices": (C.c_int, [_P, u32, _P, _P, _P, _P, _P]),
    "fpt_pass_get_stats": (C.c_int, [_P, C.POINTER(fpt_pass_stats), _P]),
    "fpt_pass_get_counters": (C.c_int, [_P, C.POINTER(C.c_uint64), u32, _P]),
    "fpt_pass_get_kernel_times": (C.c_int, [_P, C.POINTER(C.c_double), C.POINTER(C.c_uint64), u32, C.c_int]),
    "fpt_batch_create": (C.c_int, [C.POINTER(_P)]),
    "fpt_batch_destroy": (None, [_P]),
    "fpt_batch_add": (C.c_int, [_P, C.POINTER(fpt_batch_request)]),
    "fpt_batch_set_tuning": (C.c_int, [_P, u32, u32]),
    "fpt_batch_get_tuning": (C.c_int, [_P, C.POINTER(u32), C.POINTER(u32)]),
    "fpt_batch_set_tuning_ex": (C.c_int, [_P, C.POINTER(fpt_batch_tuning)]),
    "fpt_batch_get_tuning_ex": (C.c_int, [_P, C.POINTER(fpt_batch_tuning)]),
    "fpt_batch_autotune": (C.c_int, [_P, _P]),
    "fpt_batch_launch": (C.c_int, [_P, _P]),
    "fpt_batch_launch_sequential": (C.c_int, [_P, _P]),
    "fpt_batch_get_stats": (C.c_int, [_P, C.POINTER(fpt_pass_stats), _P]),
}

_lib = None


class FptError(RuntimeError):
    """A C-ABI call returned a non-zero fpt_status (the message is fpt_last_error())."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def lib() -> C.CDLL:
    """Loads libfpt.so once; raises ImportError if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: run falcor_b200.build.build() (the CUDA library is required)")
        l = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | os.RTLD_LOCAL)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(l, name)
            fn.restype = res
            fn.argtypes = args
        _lib = l
    return _lib


def release(fn_name: str, handle) -> None:
    """Frees a handle from a finaliser; a no-op once the library or the
    interpreter is being torn down (module globals may already be None)."""
    l = _lib
    if l is None or handle is None:
        return
    try:
        getattr(l, fn_name)(handle)
    except Exception:
        pass


def check(status: int) -> None:
    if status != FPT_OK:
        raise FptError(status, lib().fpt_last_error().decode(errors="replace"))

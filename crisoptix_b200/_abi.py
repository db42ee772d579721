"""ctypes mirror of include/crisb.h and numpy dtypes of its record layouts."""
from __future__ import annotations

import ctypes
import os

import numpy as np

c_f = ctypes.c_float
c_u32 = ctypes.c_uint32
c_i32 = ctypes.c_int32
c_u64 = ctypes.c_uint64
c_vp = ctypes.c_void_p

# status codes
OK = 0
ERR_INVALID_ARGUMENT = -1
ERR_OUT_OF_MEMORY = -2
ERR_CUDA = -3
ERR_QUEUE_OVERFLOW = -4
ERR_DEVICE_TIMEOUT = -5
ERR_NOT_SUPPORTED = -6
ERR_DEVICE_FAULT = -7

PATH_TRACER = 0
RESTIR_PT = 1
CONDITIONAL_RESTIR = 2
RADIUS_CONSTANT = 0
RADIUS_PATH_LENGTH = 1
BVH_DEVICE = 0
BVH_HOST = 1
BVH_DEVICE_WIDE4 = 2
BVH_FORMAT_WIDE4 = 0
BVH_FORMAT_COMPRESSED8 = 1
STORAGE_FP32 = 0
STORAGE_FP16 = 1
SPEC_COLOR = 0
SPEC_OCC_ROUGH_METAL = 1
MOTION_NONE = 0
MOTION_VECTORS = 1
MOTION_REPROJECT = 2
INVALID_PRIM = 0xFFFFFFFF

BUF_PREFIX_RES_FRONT = 0
BUF_PREFIX_RES_BACK = 1
BUF_CANON_PREFIX = 2
BUF_SUFFIX_RES_FRONT = 3
BUF_SUFFIX_RES_BACK = 4
BUF_CANON_SUFFIX = 5
BUF_GBUFFER = 6
BUF_NEIGHBORS = 7
BUF_NEIGHBOR_COUNT = 8


class Material(ctypes.Structure):
    _fields_ = [("diffuse", c_f * 3), ("specular", c_f * 3), ("emission", c_f * 3), ("roughness", c_f),
                ("spec_usage", c_i32), ("reserved", c_i32)]


class Mesh(ctypes.Structure):
    _fields_ = [("first_triangle", c_u32), ("num_triangles", c_u32)]


class Instance(ctypes.Structure):
    _fields_ = [("mesh", c_u32), ("material_override", c_i32), ("transform", c_f * 12)]


class Emitter(ctypes.Structure):
    _fields_ = [("color", c_f * 3), ("first_face", c_u32), ("num_faces", c_u32)]


class SceneDesc(ctypes.Structure):
    _fields_ = [("positions", c_vp), ("normals", c_vp), ("num_vertices", c_u32), ("indices", c_vp),
                ("triangle_material", c_vp), ("num_triangles", c_u32), ("materials", c_vp), ("num_materials", c_u32),
                ("meshes", c_vp), ("num_meshes", c_u32), ("instances", c_vp), ("num_instances", c_u32),
                ("emitters", c_vp), ("num_emitters", c_u32), ("emitter_faces", c_vp), ("num_emitter_faces", c_u32),
                ("uvs", c_vp), ("textures", c_vp), ("num_textures", c_u32), ("material_textures", c_vp),
                ("bvh_builder", c_u32)]


class Tuning(ctypes.Structure):
    _fields_ = [("trace_block", c_u32), ("trace_grid", c_u32), ("jobs_per_pixel", c_u32), ("frame_ms", c_f)]


class BvhInfo(ctypes.Structure):
    _fields_ = [("format", c_u32), ("on_device", c_u32), ("num_nodes", c_u32), ("node_bytes", c_u32),
                ("stack_bound", c_i32), ("depth", c_i32), ("inner_children", c_u32), ("leaf_children", c_u32)]


class Texture(ctypes.Structure):
    _fields_ = [("rgba", c_vp), ("width", c_u32), ("height", c_u32)]


class Camera(ctypes.Structure):
    _fields_ = [("pos", c_f * 3), ("view_dir", c_f * 3), ("up", c_f * 3), ("aspect", c_f), ("fov", c_f),
                ("changed", c_i32)]


class CameraData(ctypes.Structure):
    _fields_ = [("pos", c_f * 3), ("u", c_f * 3), ("v", c_f * 3), ("w", c_f * 3)]


class Params(ctypes.Structure):
    _fields_ = [("renderer_type", c_i32), ("nee_prob", c_f), ("max_path_len", c_i32), ("enable_accum", c_i32),
                ("recon_min_roughness", c_f), ("recon_min_distance", c_f), ("prefix_len", c_i32),
                ("prefix_enable_temporal", c_i32), ("prefix_enable_spatial", c_i32), ("prefix_spatial_count", c_i32),
                ("prefix_spatial_rounds", c_i32), ("suffix_enable_temporal", c_i32), ("suffix_enable_spatial", c_i32),
                ("suffix_spatial_count", c_i32), ("suffix_spatial_rounds", c_i32), ("gather_n", c_i32),
                ("gather_m", c_i32), ("gather_radius", c_f), ("gather_radius_type", c_i32), ("window_radius", c_i32),
                ("storage", c_i32), ("motion_mode", c_i32), ("seed", c_u64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class TraceHit(ctypes.Structure):
    _fields_ = [("prim", c_u32), ("t", c_f), ("u", c_f), ("v", c_f)]


class Stats(ctypes.Structure):
    _fields_ = [("prefix_gen_temp_ms", c_f), ("prefix_spatial_ms", c_f), ("suffix_gen_temp_ms", c_f),
                ("suffix_spatial_ms", c_f), ("prefix_store_ms", c_f), ("final_gather_ms", c_f), ("total_ms", c_f),
                ("kernel_launches", c_u32), ("trace_ms", c_f), ("shift_ms", c_f), ("resample_ms", c_f),
                ("search_ms", c_f), ("shade_ms", c_f), ("other_ms", c_f), ("closest_rays", c_u64), ("shadow_rays", c_u64),
                ("shift_closest_rays", c_u64), ("shift_shadow_rays", c_u64), ("shift_jobs", c_u64),
                ("node_visits", c_u64), ("tri_tests", c_u64), ("resample_bytes", c_u64 * 5)]

RESAMPLE_KERNELS = ("prefix_combine", "temporal_combine", "spatial_select", "spatial_combine", "gather_combine")


HIT_DTYPE = np.dtype([("prim", "<u4"), ("bary", "<f4", 2), ("in_dir", "<f4", 3)])
PREFIX_DTYPE = np.dtype([("rng", "<u8"), ("primary", HIT_DTYPE), ("recon", HIT_DTYPE), ("last", HIT_DTYPE),
                         ("flags", "<u4"), ("f", "<f4", 3), ("post_recon_f", "<f4", 3), ("p", "<f4"),
                         ("path_len", "<f4"), ("recon_out_dir", "<f4", 3)])
PREFIX_RES_DTYPE = np.dtype([("sample", PREFIX_DTYPE), ("w_sum", "<f4"), ("confidence", "<f4"), ("pad", "<u4", 2)])
SUFFIX_DTYPE = np.dtype([("rng", "<u8"), ("recon", HIT_DTYPE), ("last_prefix", HIT_DTYPE), ("flags", "<u4"),
                         ("f", "<f4", 3), ("post_recon_f", "<f4", 3), ("p", "<f4"), ("recon_out_dir", "<f4", 3),
                         ("pad", "<u4")])
SUFFIX_RES_DTYPE = np.dtype([("sample", SUFFIX_DTYPE), ("w_sum", "<f4"), ("confidence", "<f4")])
# FP16 reservoir storage (crisb_*_res16_rec)
HIT16_DTYPE = np.dtype([("prim", "<u4"), ("bary", "<u2", 2), ("in_dir_oct", "<u4")])
PREFIX_RES16_DTYPE = np.dtype([("rng", "<u8"), ("flags", "<u4"), ("p", "<f4"), ("path_len", "<f4"),
                               ("primary", HIT16_DTYPE), ("recon", HIT16_DTYPE), ("last", HIT16_DTYPE),
                               ("f", "<u2", 3), ("post_recon_f", "<u2", 3), ("recon_out_dir_oct", "<u4"),
                               ("w_sum", "<f4"), ("confidence", "<f4")])
SUFFIX_RES16_DTYPE = np.dtype([("rng", "<u8"), ("flags", "<u4"), ("p", "<f4"), ("recon", HIT16_DTYPE),
                               ("last_prefix", HIT16_DTYPE), ("f", "<u2", 3), ("post_recon_f", "<u2", 3),
                               ("recon_out_dir_oct", "<u4"), ("w_sum", "<f4"), ("confidence", "<f4")])
OCT_ZERO = 0x80008000
GBUFFER_DTYPE = np.dtype([("rng", "<u8"), ("prev_xy", "<u4"), ("flags", "<u4")])
NEIGHBOR_DTYPE = np.dtype([("pixel", "<u4"), ("dist", "<f4")])
TRACE_HIT_DTYPE = np.dtype([("prim", "<u4"), ("t", "<f4"), ("u", "<f4"), ("v", "<f4")])

BUFFER_DTYPES = {
    BUF_PREFIX_RES_FRONT: PREFIX_RES_DTYPE,
    BUF_PREFIX_RES_BACK: PREFIX_RES_DTYPE,
    BUF_CANON_PREFIX: PREFIX_DTYPE,
    BUF_SUFFIX_RES_FRONT: SUFFIX_RES_DTYPE,
    BUF_SUFFIX_RES_BACK: SUFFIX_RES_DTYPE,
    BUF_CANON_SUFFIX: SUFFIX_DTYPE,
    BUF_GBUFFER: GBUFFER_DTYPE,
    BUF_NEIGHBORS: NEIGHBOR_DTYPE,
    BUF_NEIGHBOR_COUNT: np.dtype("<u4"),
}


def buffer_dtype(buffer_id: int, storage: int = STORAGE_FP32) -> np.dtype:
    """Element type of a debug buffer; reservoirs follow the storage layout."""
    if storage == STORAGE_FP16:
        if buffer_id in (BUF_PREFIX_RES_FRONT, BUF_PREFIX_RES_BACK):
            return PREFIX_RES16_DTYPE
        if buffer_id in (BUF_SUFFIX_RES_FRONT, BUF_SUFFIX_RES_BACK):
            return SUFFIX_RES16_DTYPE
    return BUFFER_DTYPES[buffer_id]


# sizeof order of crisb_abi_sizes
ABI_STRUCTS = [Material, Mesh, Instance, Emitter, SceneDesc, Camera, CameraData, Params, HIT_DTYPE, PREFIX_DTYPE,
               PREFIX_RES_DTYPE, SUFFIX_DTYPE, SUFFIX_RES_DTYPE, GBUFFER_DTYPE, NEIGHBOR_DTYPE, TraceHit, Stats,
               HIT16_DTYPE, PREFIX_RES16_DTYPE, SUFFIX_RES16_DTYPE, Tuning, BvhInfo]


def abi_size(t) -> int:
    return t.itemsize if isinstance(t, np.dtype) else ctypes.sizeof(t)


# every entry point declared in include/crisb.h: name -> (restype, argtypes)
ENTRY_POINTS = {
    "crisb_version": (ctypes.c_char_p, []),
    "crisb_last_error": (c_i32, [ctypes.c_char_p, ctypes.c_size_t]),
    "crisb_params_default": (c_i32, [ctypes.POINTER(Params), c_f]),
    "crisb_camera_get_data": (c_i32, [ctypes.POINTER(Camera), ctypes.POINTER(CameraData)]),
    "crisb_scene_create": (c_i32, [ctypes.POINTER(SceneDesc), ctypes.POINTER(c_vp)]),
    "crisb_scene_destroy": (c_i32, [c_vp]),
    "crisb_scene_size": (c_i32, [c_vp, ctypes.POINTER(c_f)]),
    "crisb_scene_num_triangles": (c_i32, [c_vp, ctypes.POINTER(c_u32)]),
    "crisb_scene_bvh_info": (c_i32, [c_vp, ctypes.POINTER(BvhInfo)]),
    "crisb_scene_read_triangles": (c_i32, [c_vp, c_vp, c_vp, c_vp]),
    "crisb_trace_rays": (c_i32, [c_vp, c_vp, c_vp, c_u32, c_i32, c_vp]),
    "crisb_renderer_create": (c_i32, [c_vp, c_u32, c_u32, ctypes.POINTER(Params), ctypes.POINTER(c_vp)]),
    "crisb_renderer_destroy": (c_i32, [c_vp]),
    "crisb_renderer_set_params": (c_i32, [c_vp, ctypes.POINTER(Params)]),
    "crisb_renderer_get_params": (c_i32, [c_vp, ctypes.POINTER(Params)]),
    "crisb_render_frame": (c_i32, [c_vp, ctypes.POINTER(Camera), c_vp, c_vp]),
    "crisb_scene_get_materials": (c_i32, [c_vp, c_vp, c_u32]),
    "crisb_scene_set_materials": (c_i32, [c_vp, c_vp, c_u32]),
    "crisb_scene_set_emitter_colors": (c_i32, [c_vp, c_vp, c_u32]),
    "crisb_adjoint_create": (c_i32, [c_vp, c_u32, c_u32, ctypes.POINTER(Params), ctypes.POINTER(c_vp)]),
    "crisb_adjoint_destroy": (c_i32, [c_vp]),
    "crisb_adjoint_refreeze": (c_i32, [c_vp]),
    "crisb_adjoint_forward": (c_i32, [c_vp, ctypes.POINTER(Camera), c_u64, c_vp, c_vp]),
    "crisb_adjoint_backward": (c_i32, [c_vp, ctypes.POINTER(Camera), c_u64, c_vp, c_vp, c_vp, c_vp]),
    "crisb_autotune_spatial": (c_i32, [c_vp, ctypes.POINTER(Camera), c_u32, c_f, ctypes.POINTER(c_u32),
                                       ctypes.POINTER(c_f)]),
    "crisb_restir_adjoint_enable": (c_i32, [c_vp, c_i32]),
    "crisb_restir_adjoint_forward": (c_i32, [c_vp, c_vp, c_vp]),
    "crisb_restir_adjoint_backward": (c_i32, [c_vp, c_vp, c_vp, c_vp, c_vp]),
    "crisb_batch_create": (c_i32, [ctypes.POINTER(c_vp), c_u32, ctypes.POINTER(c_vp)]),
    "crisb_batch_destroy": (c_i32, [c_vp]),
    "crisb_batch_render": (c_i32, [c_vp, c_vp, ctypes.POINTER(c_vp), c_vp]),
    "crisb_tonemap_srgb8": (c_i32, [c_vp, c_vp, c_u32, c_vp]),
    "crisb_srgb8_thresholds": (c_i32, [c_vp, c_vp]),
    "crisb_set_srgb_output": (c_i32, [c_vp, c_vp]),
    "crisb_set_motion_vectors": (c_i32, [c_vp, c_vp]),
    "crisb_set_trace_grid": (c_i32, [c_vp, c_u32]),
    "crisb_autotune": (c_i32, [c_vp, ctypes.POINTER(Camera), c_u32, ctypes.POINTER(c_u32)]),
    "crisb_set_graph": (c_i32, [c_vp, c_i32]),
    "crisb_set_job_capacity": (c_i32, [c_vp, c_u32]),
    "crisb_set_trace_block": (c_i32, [c_vp, c_u32]),
    "crisb_autotune_ex": (c_i32, [c_vp, ctypes.POINTER(Camera), c_u32, ctypes.POINTER(Tuning)]),
    "crisb_get_job_capacity": (c_i32, [c_vp, ctypes.POINTER(c_u32)]),
    "crisb_frame_index": (c_i32, [c_vp, ctypes.POINTER(c_u64)]),
    "crisb_frame_random": (c_i32, [c_vp, ctypes.POINTER(c_u32)]),
    "crisb_set_timing": (c_i32, [c_vp, c_i32]),
    "crisb_get_stats": (c_i32, [c_vp, ctypes.POINTER(Stats)]),
    "crisb_check_device_errors": (c_i32, [c_vp]),
    "crisb_debug_read": (c_i32, [c_vp, c_i32, c_vp, ctypes.c_size_t]),
    "crisb_debug_size": (c_i32, [c_vp, c_i32, ctypes.POINTER(ctypes.c_size_t)]),
    "crisb_abi_sizes": (c_i32, [ctypes.POINTER(c_u32), c_u32]),
    "crisb_endpoint_search": (c_i32, [c_vp, c_u32, c_vp, c_u32, c_u32, c_vp, c_vp, c_vp]),
    "crisb_endpoint_search_noalloc": (c_i32, [c_vp, c_u32, c_vp, c_u32, c_u32, c_vp, c_vp, c_vp]),
    "crisb_endpoint_search_status": (c_i32, [c_vp]),
    "crisb_endpoint_search_set_visit_cap": (c_i32, [c_u32]),
    "crisb_selftest_kat": (c_i32, [c_i32, c_vp, c_u32, c_vp, c_vp]),
    "crisb_selftest_sort": (c_i32, [c_vp, c_vp, c_u32, c_vp, ctypes.c_size_t, c_vp]),
    "crisb_selftest_sort_temp_bytes": (ctypes.c_size_t, [c_u32]),
}

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libcrisb.so")
_lib = None


def load(path: str = LIB_PATH):
    """Load libcrisb.so (in-tree build).  Raises if it is missing: there is
    no fallback implementation."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"CUDA library {path} is missing; build it with crisoptix_b200/build.py")
    lib = ctypes.CDLL(path)
    for name, (res, args) in ENTRY_POINTS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class CrisbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"crisb error {code}: {msg}")
        self.code = code


def check(code: int):
    if code != OK:
        buf = ctypes.create_string_buffer(1024)
        load().crisb_last_error(buf, 1024)
        raise CrisbError(code, buf.value.decode(errors="replace"))

"""ctypes binding of libillume_gpu.so (include/illume_gpu.h, include/illume_workloads.h).

The shared library is built in-tree by ``rs_illume_b200/csrc/Makefile``.  There
is no fallback: if the library is missing or cannot run on the device, every
GPU entry point raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libillume_gpu.so")

ILM_OK = 0
ILM_ERR_INVALID_ARGUMENT = -1
ILM_ERR_OUT_OF_MEMORY = -2
ILM_ERR_CUDA = -3
ILM_ERR_TRAVERSAL_LIMIT = -4
ILM_ERR_TIMEOUT = -5
ILM_ERR_NOT_FOUND = -6
ILM_ERR_NO_DEVICE = -7
ILM_FLAG_VALIDATE_RAYS = 1
ILM_FLAG_GRID_SCHEDULE = 2
ILM_FLAG_HIGH_OCCUPANCY = 4
ILM_FLAG_LANE_REFILL = 8
ILM_FLAG_NO_TAIL_SPLIT = 16
ILM_MISS = 0xFFFFFFFF
# cudaStreamLegacy: the explicit handle of the legacy default stream (a NULL
# stream argument selects the context's own stream instead)
CUDA_STREAM_LEGACY = 0x1
ILM_TRAVERSAL_ERROR = 0xFFFFFFFE

STATUS_NAMES = {
    ILM_OK: "ILM_OK",
    ILM_ERR_INVALID_ARGUMENT: "ILM_ERR_INVALID_ARGUMENT",
    ILM_ERR_OUT_OF_MEMORY: "ILM_ERR_OUT_OF_MEMORY",
    ILM_ERR_CUDA: "ILM_ERR_CUDA",
    ILM_ERR_TRAVERSAL_LIMIT: "ILM_ERR_TRAVERSAL_LIMIT",
    ILM_ERR_TIMEOUT: "ILM_ERR_TIMEOUT",
    ILM_ERR_NOT_FOUND: "ILM_ERR_NOT_FOUND",
    ILM_ERR_NO_DEVICE: "ILM_ERR_NO_DEVICE",
}

# numpy views of the C records
RAY_DTYPE = np.dtype([("o", "<f4", (3,)), ("tmin", "<f4"), ("d", "<f4", (3,)), ("tmax", "<f4")])
HIT_DTYPE = np.dtype([("prim", "<u4"), ("t", "<f4"), ("u", "<f4"), ("v", "<f4")])
BIN_NODE_DTYPE = np.dtype([("bmin", "<f4", (3,)), ("bmax", "<f4", (3,)), ("offset", "<i4"),
                           ("n_prims", "<u2"), ("axis", "u1"), ("pad", "u1")])
PRIM_REC_DTYPE = np.dtype([("p0", "<f4", (3,)), ("prim", "<u4"), ("p1", "<f4", (3,)), ("flags", "<u4"),
                           ("p2", "<f4", (3,)), ("aux", "<u4")])
SURFACE_INTERACTION_DTYPE = np.dtype([
    ("p", "<f4", (3,)), ("p_error", "<f4", (3,)), ("n", "<f4", (3,)), ("uv", "<f4", (2,)),
    ("dpdu", "<f4", (3,)), ("dpdv", "<f4", (3,)), ("dndu", "<f4", (3,)), ("dndv", "<f4", (3,)),
    ("shading_n", "<f4", (3,)), ("shading_dpdu", "<f4", (3,)), ("shading_dpdv", "<f4", (3,)),
    ("shading_dndu", "<f4", (3,)), ("shading_dndv", "<f4", (3,)), ("wo", "<f4", (3,)), ("t", "<f4"),
    ("prim", "<u4"), ("kind", "<u4")])
SI_MISS, SI_TRIANGLE, SI_SPHERE = 0, 1, 2
assert RAY_DTYPE.itemsize == 32 and HIT_DTYPE.itemsize == 16 and SURFACE_INTERACTION_DTYPE.itemsize == 176
assert BIN_NODE_DTYPE.itemsize == 32 and PRIM_REC_DTYPE.itemsize == 48


class ilm_config(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("stack_depth", ctypes.c_int32),
                ("block_size", ctypes.c_int32), ("flags", ctypes.c_int32), ("max_iterations", ctypes.c_uint32)]


class ilm_build_opts(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int32), ("max_prims_in_node", ctypes.c_int32)]


class ilm_accel_info(ctypes.Structure):
    _fields_ = [("n_prims", ctypes.c_uint32), ("n_binary_nodes", ctypes.c_uint32),
                ("n_nodes", ctypes.c_uint32), ("width", ctypes.c_uint32),
                ("device_bytes", ctypes.c_uint64), ("build_seconds", ctypes.c_double),
                ("n_leaf_refs", ctypes.c_uint32), ("max_depth", ctypes.c_uint32)]


ILM_LAYOUT_KDTREE = 1


class ilm_kdtree_opts(ctypes.Structure):
    _fields_ = [("isect_cost", ctypes.c_int32), ("traversal_cost", ctypes.c_int32),
                ("empty_bonus", ctypes.c_float), ("max_prims", ctypes.c_uint32), ("max_depth", ctypes.c_int32)]


KD_NODE_DTYPE = np.dtype([("word", "<u4"), ("flags", "<u4")])


class ilm_sphere_desc(ctypes.Structure):
    _fields_ = [("object_to_world", ctypes.c_float * 16), ("world_to_object", ctypes.c_float * 16),
                ("radius", ctypes.c_float), ("z_min", ctypes.c_float), ("z_max", ctypes.c_float),
                ("phi_max_deg", ctypes.c_float), ("reverse_orientation", ctypes.c_int32),
                ("kind", ctypes.c_int32), ("height", ctypes.c_float), ("inner_radius", ctypes.c_float),
                ("p1", ctypes.c_float * 3), ("p2", ctypes.c_float * 3)]


class ilm_curve_desc(ctypes.Structure):
    _fields_ = [("object_to_world", ctypes.c_float * 16), ("world_to_object", ctypes.c_float * 16),
                ("cp", ctypes.c_float * 12), ("width", ctypes.c_float * 2), ("n", ctypes.c_float * 6),
                ("u_min", ctypes.c_float), ("u_max", ctypes.c_float), ("type", ctypes.c_int32),
                ("reverse_orientation", ctypes.c_int32)]


CURVE_TYPES = {"flat": 0, "cylinder": 1, "ribbon": 2}
QUADRICS = {"sphere": 0, "disk": 1, "cylinder": 2, "cone": 3, "paraboloid": 4, "hyperboloid": 5}


class ilm_pt_scene_desc(ctypes.Structure):
    _fields_ = [("prim_material", ctypes.c_void_p), ("albedo", ctypes.c_void_p), ("emission", ctypes.c_void_p),
                ("n_materials", ctypes.c_uint32), ("eye", ctypes.c_float * 3), ("fov_deg", ctypes.c_float),
                ("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("camera_to_world", ctypes.c_float * 9)]


class ilm_filter_desc(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("radius", ctypes.c_float * 2), ("a", ctypes.c_float),
                ("b", ctypes.c_float)]


class ilm_scene_file_info(ctypes.Structure):
    _fields_ = [("n_meshes", ctypes.c_uint32), ("n_triangles", ctypes.c_uint32), ("n_vertices", ctypes.c_uint32),
                ("n_quadrics", ctypes.c_uint32), ("n_materials", ctypes.c_uint32), ("n_emissive", ctypes.c_uint32),
                ("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("spp", ctypes.c_uint32),
                ("max_depth", ctypes.c_uint32), ("eye", ctypes.c_float * 3), ("camera_to_world", ctypes.c_float * 9),
                ("fov_deg", ctypes.c_float), ("filter", ilm_filter_desc), ("accelerator", ctypes.c_int32),
                ("bvh", ilm_build_opts), ("kdtree", ilm_kdtree_opts), ("n_warnings", ctypes.c_uint32),
                ("n_curves", ctypes.c_uint32)]


class ilm_pt_opts(ctypes.Structure):
    _fields_ = [("spp", ctypes.c_uint32), ("max_depth", ctypes.c_uint32), ("rr_depth", ctypes.c_uint32),
                ("seed", ctypes.c_uint64), ("wave_paths", ctypes.c_uint32), ("use_graphs", ctypes.c_int32),
                ("filter", ilm_filter_desc)]


class ilm_pt_stats(ctypes.Structure):
    _fields_ = [("closest_rays", ctypes.c_uint64), ("shadow_rays", ctypes.c_uint64), ("seconds", ctypes.c_double),
                ("waves", ctypes.c_uint32)]


class ilm_nrc_render_opts(ctypes.Structure):
    _fields_ = [("frames", ctypes.c_uint32), ("spp_per_frame", ctypes.c_uint32), ("max_depth", ctypes.c_uint32),
                ("rr_depth", ctypes.c_uint32), ("seed", ctypes.c_uint64), ("spread_c", ctypes.c_float),
                ("train_paths", ctypes.c_uint32), ("train_samples", ctypes.c_uint32),
                ("time_budget_s", ctypes.c_double), ("train", ctypes.c_int32), ("train_steps", ctypes.c_uint32),
                ("train_suffix", ctypes.c_uint32)]


class ilm_nrc_render_stats(ctypes.Structure):
    _fields_ = [("frames", ctypes.c_uint32), ("seconds", ctypes.c_double), ("closest_rays", ctypes.c_uint64),
                ("shadow_rays", ctypes.c_uint64), ("queries", ctypes.c_uint64), ("train_samples", ctypes.c_uint64),
                ("last_loss", ctypes.c_float)]


class ilm_mesh_attrs(ctypes.Structure):
    _fields_ = [("n", ctypes.c_void_p), ("s", ctypes.c_void_p), ("uv", ctypes.c_void_p),
                ("reverse_orientation", ctypes.c_int32)]


class ilm_batch_desc(ctypes.Structure):
    _fields_ = [("accel", ctypes.c_uint32), ("rays", ctypes.c_void_p), ("n", ctypes.c_uint64),
                ("hits", ctypes.c_void_p), ("occluded", ctypes.c_void_p)]


class ilm_launch_opts(ctypes.Structure):
    _fields_ = [("stack_depth", ctypes.c_int32), ("schedule", ctypes.c_int32), ("high_occupancy", ctypes.c_int32)]


class ilm_tune_result(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int32), ("launch", ilm_launch_opts), ("ms", ctypes.c_double),
                ("baseline_ms", ctypes.c_double), ("n_tried", ctypes.c_uint32), ("from_cache", ctypes.c_int32)]


_P = ctypes.c_void_p
_U32 = ctypes.c_uint32
_U64 = ctypes.c_uint64
_I32 = ctypes.c_int32
_F = ctypes.c_float

# name -> (restype, argtypes)
SIGNATURES = {
    "ilm_context_create": (_I32, [ctypes.POINTER(_P), ctypes.POINTER(ilm_config)]),
    "ilm_context_destroy": (_I32, [_P]),
    "ilm_last_error_string": (ctypes.c_char_p, [_P]),
    "ilm_context_set_stage_chunk": (_I32, [_P, _U64]),
    "ilm_mesh_upload": (_I32, [_P, _P, _U32, _P, _U32, ctypes.POINTER(_U32)]),
    "ilm_spheres_upload": (_I32, [_P, _P, _U32, ctypes.POINTER(_U32)]),
    "ilm_curves_upload": (_I32, [_P, _P, _U32, ctypes.POINTER(_U32)]),
    "ilm_mesh_set_attrs": (_I32, [_P, _U32, ctypes.POINTER(ilm_mesh_attrs)]),
    "ilm_surface_interactions": (_I32, [_P, _U32, _P, _P, _U64, _P, _P]),
    "ilm_accel_build": (_I32, [_P, _P, _U32, ctypes.POINTER(ilm_build_opts), ctypes.POINTER(_U32)]),
    "ilm_accel_destroy": (_I32, [_P, _U32]),
    "ilm_accel_world_bound": (_I32, [_P, _U32, _P]),
    "ilm_accel_get_info": (_I32, [_P, _U32, ctypes.POINTER(ilm_accel_info)]),
    "ilm_accel_binary_nodes": (_I32, [_P, _U32, _P, _P]),
    "ilm_host_layout_build": (_I32, [_P, _U32, _P, _U32, _P, _U32, ctypes.POINTER(ilm_build_opts),
                                     ctypes.POINTER(_P)]),
    "ilm_host_layout_info": (_I32, [_P, ctypes.POINTER(ilm_accel_info)]),
    "ilm_host_layout_copy": (_I32, [_P, _P, _P, _P, _P, _P]),
    "ilm_host_layout_destroy": (_I32, [_P]),
    "ilm_kdtree_build": (_I32, [_P, _P, _U32, ctypes.POINTER(ilm_kdtree_opts), ctypes.POINTER(_U32)]),
    "ilm_accel_kd_nodes": (_I32, [_P, _U32, _P, _P]),
    "ilm_host_kdtree_build": (_I32, [_P, _U32, _P, _U32, _P, _U32, ctypes.POINTER(ilm_kdtree_opts), _I32,
                                     ctypes.POINTER(_P)]),
    "ilm_host_layout_kd_index": (_I32, [_P, _P]),
    "ilm_loop_subdivide": (_I32, [_P, _U32, _P, _U32, _U32, ctypes.POINTER(_U32), ctypes.POINTER(_U32), _P, _P, _P]),
    "ilm_scene_file_load": (_I32, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(_P)]),
    "ilm_scene_file_parse": (_I32, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t,
                                    ctypes.POINTER(_P)]),
    "ilm_scene_file_info_get": (_I32, [_P, ctypes.POINTER(ilm_scene_file_info)]),
    "ilm_scene_file_warnings": (ctypes.c_char_p, [_P]),
    "ilm_scene_file_mesh": (_I32, [_P, _U32, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "ilm_scene_file_quadrics": (_I32, [_P, _P, _P]),
    "ilm_scene_file_materials": (_I32, [_P, _P, _P]),
    "ilm_scene_file_curves": (_I32, [_P, _P, _P]),
    "ilm_scene_file_build": (_I32, [_P, _P, ctypes.POINTER(_U32), ctypes.POINTER(_U32)]),
    "ilm_scene_file_destroy": (_I32, [_P]),
    "ilm_scene_syntax": (_I32, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t,
                                ctypes.POINTER(ctypes.c_size_t), ctypes.c_char_p, ctypes.c_size_t]),
    "ilm_intersect_closest": (_I32, [_P, _U32, _P, _U64, _P, _P]),
    "ilm_intersect_any": (_I32, [_P, _U32, _P, _U64, _P, _P]),
    "ilm_intersect_closest_noalloc": (_I32, [_P, _U32, _P, _U64, _P, _P]),
    "ilm_batch_plan_create": (_I32, [_P, _P, _U32, _I32, ctypes.POINTER(_P)]),
    "ilm_batch_plan_launch": (_I32, [_P, _P, _P]),
    "ilm_batch_plan_destroy": (_I32, [_P, _P]),
    "ilm_intersect_batched": (_I32, [_P, _P, _U32, _I32, _P]),
    "ilm_accel_set_launch": (_I32, [_P, _U32, ctypes.POINTER(ilm_launch_opts)]),
    "ilm_autotune": (_I32, [_P, _P, _U32, _P, _U64, _I32, _I32, ctypes.POINTER(ilm_tune_result)]),
    "ilm_pt_scene_create": (_I32, [_P, _U32, ctypes.POINTER(ilm_pt_scene_desc), ctypes.POINTER(_U32)]),
    "ilm_render_pt": (_I32, [_P, _U32, ctypes.POINTER(ilm_pt_opts), _P, ctypes.POINTER(ilm_pt_stats)]),
    "ilm_nrc_create": (_I32, [_P, _P, ctypes.POINTER(_P)]),
    "ilm_nrc_destroy": (_I32, [_P, _P]),
    "ilm_nrc_params": (_I32, [_P, _P, _P, _P]),
    "ilm_nrc_infer": (_I32, [_P, _P, _P, _U64, _P, _P]),
    "ilm_nrc_train_step": (_I32, [_P, _P, _P, _P, _U64, ctypes.POINTER(ctypes.c_float), _P]),
    "ilm_nrc_gradients": (_I32, [_P, _P, _P, _P, _U64, _P, ctypes.POINTER(ctypes.c_float)]),
    "ilm_nrc_encode": (_I32, [_P, _P, _P, _U64, _P]),
    "ilm_render_nrc": (_I32, [_P, _U32, _P, ctypes.POINTER(ilm_nrc_render_opts), _P,
                              ctypes.POINTER(ilm_nrc_render_stats)]),
    "ilm_write_pfm": (_I32, [ctypes.c_char_p, _P, _U32, _U32]),
    "ilm_read_pfm": (_I32, [ctypes.c_char_p, _P, ctypes.POINTER(_U32), ctypes.POINTER(_U32)]),
    "ilm_filter_evaluate": (_I32, [ctypes.POINTER(ilm_filter_desc), _F, _F, ctypes.POINTER(_F)]),
    "ilm_filter_table": (_I32, [ctypes.POINTER(ilm_filter_desc), _P]),
    "ilm_device_errors": (_I32, [_P, ctypes.POINTER(_U32), _I32]),
    "ilm_synchronize": (_I32, [_P, _P, ctypes.c_double]),
    # workloads
    "ilm_wl_rng_floats": (None, [_U64, _U64, _P]),
    "ilm_wl_rng_u32": (None, [_U64, _U64, _P]),
    "ilm_wl_soup": (None, [_U64, _U32, _F, _P, _P]),
    "ilm_wl_icosphere_counts": (None, [_U32, ctypes.POINTER(_U32), ctypes.POINTER(_U32)]),
    "ilm_wl_icosphere": (None, [_U32, _U64, _F, _F, _P, _P, _P]),
    "ilm_wl_camera_rays": (None, [_U32, _U32, _P, _F, _P]),
    "ilm_wl_ball_rays": (None, [_U64, _U64, _U64, _U64, _F, _F, _F, _P]),
    "ilm_wl_cornell_counts": (None, [_U32, ctypes.POINTER(_U32), ctypes.POINTER(_U32)]),
    "ilm_wl_cornell": (None, [_U32, _U64, _P, _P, _P, _P, _P]),
}

_lib = None


class IllumeError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        name = STATUS_NAMES.get(status, str(status))
        super().__init__(f"{where} failed with {name}" + (f": {detail}" if detail else ""))


def load() -> ctypes.CDLL:
    """Loads the library (once).  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C rs_illume_b200/csrc` "
                               "(or __graft_entry__.build())")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def ptr(a) -> int:
    """Address of a C-contiguous numpy array (or a raw integer address)."""
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
        return a.ctypes.data
    if hasattr(a, "data_ptr"):      # torch tensor (device or host)
        return a.data_ptr()
    raise TypeError(f"cannot take the address of {type(a)}")

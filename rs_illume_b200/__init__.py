"""rs_illume_b200: B200-native ray queries and path tracing for rs_illume.

The product is the C ABI in include/illume_gpu.h, implemented by
``libillume_gpu.so`` (CUDA kernels for sm_100a + C++ host code, built from
``csrc/``).  This package is the Python host mirror of the reference's
aggregate interface on top of that ABI.
"""
from ._lib import (HIT_DTYPE, ILM_MISS, ILM_TRAVERSAL_ERROR, RAY_DTYPE, IllumeError, LIB_PATH, load)
from .image import filter_desc, filter_table, read_pfm, write_pfm
from .primitive import (Bounds3f, Context, Curves, GpuBVHAccel, GpuKdTreeAccel, Hit, PathTracer, Ray, Scene, Spheres,
                        TriangleMesh, curve_segments, loop_subdivide, quadric_desc, rays_array, sphere_desc)
from .scene_file import SceneFile

__all__ = [
    "HIT_DTYPE", "ILM_MISS", "ILM_TRAVERSAL_ERROR", "RAY_DTYPE", "IllumeError", "LIB_PATH", "load",
    "Bounds3f", "Context", "Curves", "GpuBVHAccel", "GpuKdTreeAccel", "Hit", "PathTracer", "Ray", "Scene", "Spheres",
    "TriangleMesh", "rays_array",
    "SceneFile", "curve_segments", "loop_subdivide", "sphere_desc", "quadric_desc", "filter_desc", "filter_table",
    "read_pfm", "write_pfm",
]

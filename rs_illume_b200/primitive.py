"""Host-side mirror of rs_illume's aggregate interface for the GPU path.

``GpuBVHAccel`` stands where ``BVHAccel`` (src/accelerators/bvh.rs:24-93)
stands in the reference: it implements the ``Primitive`` surface
(src/core/primitive/mod.rs:9-20) -- ``world_bound``, ``intersect``,
``intersect_p`` and the material/area-light queries that an aggregate answers
with an error (bvh.rs:540-553) -- on top of the C ABI in include/illume_gpu.h.
Batched calls (``intersect_batch`` / ``intersect_p_batch``) are the intended
path; the single-ray methods are batches of one.  ``Scene`` mirrors
src/core/scene.rs:10-53.
"""
from __future__ import annotations

import ctypes
import logging
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import (CUDA_STREAM_LEGACY, HIT_DTYPE, ILM_MISS, RAY_DTYPE, IllumeError, ilm_accel_info, ilm_build_opts,
                   ilm_config, ilm_sphere_desc, ptr)

log = logging.getLogger("rs_illume_b200")

SPLIT_METHODS = ("SAH", "HLBVH", "Middle", "EqualCounts")   # bvh.rs:16-22


@dataclass
class Bounds3f:
    """geometry/bounds3.rs:74-77."""
    min: np.ndarray
    max: np.ndarray


@dataclass
class Ray:
    """geometry/ray.rs:11-19 (o, d, t_max; time/medium/differential unused here)."""
    o: Sequence[float]
    d: Sequence[float]
    t_max: float = float("inf")


@dataclass
class Hit:
    """Closest-hit result: the primitive, t and (u, v); for triangles u = b1 and
    v = b2 of the watertight test (shapes/triangle.rs:232-236)."""
    prim: int
    t: float
    u: float
    v: float

    def point(self, ray: Ray) -> np.ndarray:
        """Ray::point_at_time (ray.rs:35-37)."""
        return np.asarray(ray.o, np.float32) + np.asarray(ray.d, np.float32) * np.float32(self.t)


def rays_array(rays: Sequence[Ray]) -> np.ndarray:
    a = np.zeros(len(rays), RAY_DTYPE)
    for i, r in enumerate(rays):
        a["o"][i] = r.o
        a["d"][i] = r.d
        a["tmax"][i] = r.t_max
    return a


class Context:
    """One ilm_context (device, streams, staging buffers, error word).  The
    keyword flags map to include/illume_gpu.h's ILM_FLAG_* (`tail_split=False`
    is ILM_FLAG_NO_TAIL_SPLIT)."""

    def __init__(self, device: int = 0, stack_depth: int = 0, block_size: int = 0, validate_rays: bool = False,
                 max_iterations: int = 0, grid_schedule: bool = False, high_occupancy: bool = False,
                 lane_refill: bool = False, tail_split: bool = True):
        self._lib = _lib.load()
        flags = (_lib.ILM_FLAG_VALIDATE_RAYS if validate_rays else 0) | \
                (_lib.ILM_FLAG_GRID_SCHEDULE if grid_schedule else 0) | \
                (_lib.ILM_FLAG_HIGH_OCCUPANCY if high_occupancy else 0) | \
                (_lib.ILM_FLAG_LANE_REFILL if lane_refill else 0) | \
                (0 if tail_split else _lib.ILM_FLAG_NO_TAIL_SPLIT)
        cfg = ilm_config(device, stack_depth, block_size, flags, max_iterations)
        h = ctypes.c_void_p()
        st = self._lib.ilm_context_create(ctypes.byref(h), ctypes.byref(cfg))
        if st != _lib.ILM_OK:
            raise IllumeError(st, "ilm_context_create")
        self.handle = h

    def check(self, status: int, where: str) -> None:
        if status != _lib.ILM_OK:
            detail = self._lib.ilm_last_error_string(self.handle)
            raise IllumeError(status, where, detail.decode() if detail else "")

    def device_errors(self, reset: bool = True) -> int:
        flags = ctypes.c_uint32()
        self.check(self._lib.ilm_device_errors(self.handle, ctypes.byref(flags), int(reset)), "ilm_device_errors")
        return flags.value

    def synchronize(self, stream=None, timeout_s: float = 60.0) -> None:
        self.check(self._lib.ilm_synchronize(self.handle, stream, timeout_s), "ilm_synchronize")

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.ilm_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class TriangleMesh:
    """TriangleMesh (shapes/triangle.rs:17-74) with world-space vertices and
    optional per-vertex shading normals n, tangents s (nv x 3) and uv (nv x 2)."""

    def __init__(self, ctx: Context, xyz: np.ndarray, idx: np.ndarray, n=None, s=None, uv=None,
                 reverse_orientation: bool = False):
        xyz = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
        idx = np.ascontiguousarray(idx, np.uint32).reshape(-1, 3)
        mid = ctypes.c_uint32()
        ctx.check(ctx._lib.ilm_mesh_upload(ctx.handle, ptr(xyz), len(xyz), ptr(idx), len(idx), ctypes.byref(mid)),
                  "ilm_mesh_upload")
        self.id = mid.value
        self.n_prims = len(idx)
        if n is not None or s is not None or uv is not None or reverse_orientation:
            arrs = [None if a is None else np.ascontiguousarray(a, np.float32).reshape(len(xyz), -1) for a in (n, s, uv)]
            at = _lib.ilm_mesh_attrs(*(ptr(a) for a in arrs), int(reverse_orientation))
            ctx.check(ctx._lib.ilm_mesh_set_attrs(ctx.handle, self.id, ctypes.byref(at)), "ilm_mesh_set_attrs")


def sphere_desc(radius: float, translate=(0.0, 0.0, 0.0), scale: float = 1.0, z_min: Optional[float] = None,
                z_max: Optional[float] = None, phi_max_deg: float = 360.0, reverse: bool = False) -> ilm_sphere_desc:
    """Sphere::new arguments (shapes/sphere.rs:50-75) for a translate*scale placement."""
    d = ilm_sphere_desc()
    tx, ty, tz = translate
    m = [scale, 0, 0, tx, 0, scale, 0, ty, 0, 0, scale, tz, 0, 0, 0, 1]
    inv = [1.0 / scale, 0, 0, -tx / scale, 0, 1.0 / scale, 0, -ty / scale, 0, 0, 1.0 / scale, -tz / scale, 0, 0, 0, 1]
    for i in range(16):
        d.object_to_world[i] = m[i]
        d.world_to_object[i] = inv[i]
    d.radius = radius
    d.z_min = -radius if z_min is None else z_min
    d.z_max = radius if z_max is None else z_max
    d.phi_max_deg = phi_max_deg
    d.reverse_orientation = int(reverse)
    return d


def quadric_desc(kind, radius: float, matrix, z_min: float = 0.0, z_max: float = 0.0, phi_max_deg: float = 360.0,
                 height: float = 0.0, inner_radius: float = 0.0, reverse: bool = False, p1=(0.0, 0.0, 0.0),
                 p2=(0.0, 0.0, 0.0)) -> ilm_sphere_desc:
    """Arguments of Sphere / Disk / Cylinder / Cone / Paraboloid / Hyperboloid
    ::new (shapes/*.rs) for any 4x4 object-to-world matrix (its inverse taken
    in float64).  `kind` is a name of _lib.QUADRICS or its number."""
    d = ilm_sphere_desc()
    m = np.asarray(matrix, np.float64).reshape(4, 4)
    inv = np.linalg.inv(m)
    for i in range(16):
        d.object_to_world[i] = float(np.float32(m.flat[i]))
        d.world_to_object[i] = float(np.float32(inv.flat[i]))
    d.kind = _lib.QUADRICS[kind] if isinstance(kind, str) else int(kind)
    d.radius, d.z_min, d.z_max, d.phi_max_deg = radius, z_min, z_max, phi_max_deg
    d.height, d.inner_radius, d.reverse_orientation = height, inner_radius, int(reverse)
    for k in range(3):
        d.p1[k], d.p2[k] = p1[k], p2[k]
    return d


def loop_subdivide(xyz, idx, levels: int = 3):
    """Loop subdivision surface (shapes/loop_subdiv.rs): (xyz[nv, 3],
    idx[nt, 3], n[nv, 3]) of the mesh refined `levels` times, on its limit
    surface with limit normals (unnormalised)."""
    lib = _lib.load()
    xyz = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
    idx = np.ascontiguousarray(idx, np.uint32).reshape(-1, 3)
    nv, nt = ctypes.c_uint32(), ctypes.c_uint32()
    st = lib.ilm_loop_subdivide(ptr(xyz), len(xyz), ptr(idx), len(idx), levels, ctypes.byref(nv), ctypes.byref(nt),
                                None, None, None)
    if st != _lib.ILM_OK:
        raise IllumeError(st, "ilm_loop_subdivide")
    p = np.empty((nv.value, 3), np.float32)
    i = np.empty((nt.value, 3), np.uint32)
    n = np.empty((nv.value, 3), np.float32)
    st = lib.ilm_loop_subdivide(ptr(xyz), len(xyz), ptr(idx), len(idx), levels, ctypes.byref(nv), ctypes.byref(nt),
                                ptr(p), ptr(i), ptr(n))
    if st != _lib.ILM_OK:
        raise IllumeError(st, "ilm_loop_subdivide")
    return p, i, n


def curve_segments(cp, width, matrix=None, curve_type="flat", normals=None, split_depth: int = 3,
                   reverse: bool = False):
    """A cubic Bezier curve (shapes/curve.rs) as 2^split_depth ilm_curve_desc
    segments over equal u ranges, as pbrt's curve shape splits it.  cp: 4x3
    control points; width (w0, w1); normals 2x3 for ribbons."""
    m = np.eye(4) if matrix is None else np.asarray(matrix, np.float64).reshape(4, 4)
    inv = np.linalg.inv(m)
    n_seg = 1 << split_depth
    out = []
    for k in range(n_seg):
        d = _lib.ilm_curve_desc()
        for i in range(16):
            d.object_to_world[i] = float(np.float32(m.flat[i]))
            d.world_to_object[i] = float(np.float32(inv.flat[i]))
        for i, v in enumerate(np.asarray(cp, np.float32).reshape(12)):
            d.cp[i] = float(v)
        d.width[0], d.width[1] = width
        if normals is not None:
            for i, v in enumerate(np.asarray(normals, np.float32).reshape(6)):
                d.n[i] = float(v)
        d.u_min, d.u_max = k / n_seg, (k + 1) / n_seg
        d.type = _lib.CURVE_TYPES[curve_type] if isinstance(curve_type, str) else int(curve_type)
        d.reverse_orientation = int(reverse)
        out.append(d)
    return out


class Curves:
    """A set of curve segments (shapes/curve.rs), one primitive each."""

    def __init__(self, ctx: Context, descs):
        arr = (_lib.ilm_curve_desc * len(descs))(*descs)
        mid = ctypes.c_uint32()
        ctx.check(ctx._lib.ilm_curves_upload(ctx.handle, ctypes.addressof(arr), len(descs), ctypes.byref(mid)),
                  "ilm_curves_upload")
        self.id = mid.value
        self.n_prims = len(descs)
        self.descs = list(descs)


class Spheres:
    """A set of Sphere shapes (shapes/sphere.rs)."""

    def __init__(self, ctx: Context, descs: Sequence[ilm_sphere_desc]):
        arr = (ilm_sphere_desc * len(descs))(*descs)
        mid = ctypes.c_uint32()
        ctx.check(ctx._lib.ilm_spheres_upload(ctx.handle, ctypes.addressof(arr), len(descs), ctypes.byref(mid)),
                  "ilm_spheres_upload")
        self.id = mid.value
        self.n_prims = len(descs)
        self.descs = list(descs)


class GpuBVHAccel:
    """GPU drop-in for BVHAccel: same SAH tree, queries on the B200."""

    def __init__(self, ctx: Context, shapes: Sequence, max_prims_in_node: int = 4, split_method: str = "SAH",
                 width: int = 8):
        if split_method not in SPLIT_METHODS:
            raise ValueError(f"unknown split method {split_method!r}")
        if split_method != "SAH":
            raise NotImplementedError("only the SAH split method is built on the GPU path")
        self.ctx = ctx
        ids = (ctypes.c_uint32 * len(shapes))(*[s.id for s in shapes])
        opts = ilm_build_opts(width, max_prims_in_node)
        aid = ctypes.c_uint32()
        ctx.check(ctx._lib.ilm_accel_build(ctx.handle, ids, len(shapes), ctypes.byref(opts), ctypes.byref(aid)),
                  "ilm_accel_build")
        self.id = aid.value
        self.width = width
        self.n_prims = sum(s.n_prims for s in shapes)

    def surface_interactions(self, rays, hits, out=None, stream=None):
        """SurfaceInteraction records (SURFACE_INTERACTION_DTYPE) for the hits
        of intersect_batch: host numpy in/out, or device tensors (stream-ordered)."""
        n = len(rays) if isinstance(rays, np.ndarray) else _count(rays, RAY_DTYPE.itemsize)
        if out is None:
            out = np.empty(n, _lib.SURFACE_INTERACTION_DTYPE)
        s = _stream(stream, rays)
        self.ctx.check(self.ctx._lib.ilm_surface_interactions(self.ctx.handle, self.id, ptr(rays), ptr(hits), n,
                                                              ptr(out), s), "ilm_surface_interactions")
        return out

    # -- Primitive surface (primitive/mod.rs:9-20) -------------------------
    def world_bound(self) -> Bounds3f:
        b = np.zeros(6, np.float32)
        self.ctx.check(self.ctx._lib.ilm_accel_world_bound(self.ctx.handle, self.id, ptr(b)), "ilm_accel_world_bound")
        return Bounds3f(b[:3].copy(), b[3:].copy())

    def intersect(self, ray: Ray) -> Optional[Hit]:
        h = self.intersect_batch(rays_array([ray]))[0]
        if h["prim"] == ILM_MISS:
            return None
        if h["prim"] == _lib.ILM_TRAVERSAL_ERROR:
            raise IllumeError(_lib.ILM_ERR_TRAVERSAL_LIMIT, "intersect")
        return Hit(int(h["prim"]), float(h["t"]), float(h["u"]), float(h["v"]))

    def intersect_p(self, ray: Ray) -> bool:
        occ = self.intersect_p_batch(rays_array([ray]))[0]
        if occ == _lib.ILM_TRAVERSAL_ERROR:
            raise IllumeError(_lib.ILM_ERR_TRAVERSAL_LIMIT, "intersect_p")
        return bool(occ)

    def get_area_light(self):
        log.error("%s::get_area_light() called; should have gone to GeometricPrimitive.", type(self).__name__)
        return None

    def get_material(self):
        log.error("%s::get_material() called; should have gone to GeometricPrimitive.", type(self).__name__)
        return None

    def compute_scattering_function(self, *args, **kwargs):
        log.error("%s::compute_scattering_function() called; should have gone to GeometricPrimitive.",
                  type(self).__name__)

    # -- batched path ------------------------------------------------------
    def intersect_batch(self, rays, hits=None, stream=None):
        """Closest hit for every ray.  `rays` is a RAY_DTYPE numpy array (host)
        or a torch uint8/float tensor on the device holding 32-byte records;
        `hits` likewise (16-byte records).  Host arrays return a HIT_DTYPE array.
        Device tensors run on `stream`, by default torch's current stream."""
        n = _count(rays, 32)
        if hits is None:
            if not isinstance(rays, np.ndarray):
                raise ValueError("device rays need a device `hits` buffer")
            hits = np.empty(n, HIT_DTYPE)
        self.ctx.check(self.ctx._lib.ilm_intersect_closest(self.ctx.handle, self.id, ptr(rays), n, ptr(hits),
                                                           _stream(stream, rays)), "ilm_intersect_closest")
        return hits

    def intersect_p_batch(self, rays, occluded=None, stream=None):
        n = _count(rays, 32)
        if occluded is None:
            if not isinstance(rays, np.ndarray):
                raise ValueError("device rays need a device `occluded` buffer")
            occluded = np.empty(n, np.uint32)
        self.ctx.check(self.ctx._lib.ilm_intersect_any(self.ctx.handle, self.id, ptr(rays), n, ptr(occluded),
                                                       _stream(stream, rays)), "ilm_intersect_any")
        return occluded

    def info(self) -> dict:
        inf = ilm_accel_info()
        self.ctx.check(self.ctx._lib.ilm_accel_get_info(self.ctx.handle, self.id, ctypes.byref(inf)),
                       "ilm_accel_get_info")
        return {k: getattr(inf, k) for k, _ in inf._fields_}

    def binary_nodes(self):
        inf = self.info()
        nodes = np.zeros(inf["n_binary_nodes"], _lib.BIN_NODE_DTYPE)
        order = np.zeros(inf["n_prims"], np.uint32)
        self.ctx.check(self.ctx._lib.ilm_accel_binary_nodes(self.ctx.handle, self.id, ptr(nodes), ptr(order)),
                       "ilm_accel_binary_nodes")
        return nodes, order


class GpuKdTreeAccel(GpuBVHAccel):
    """GPU drop-in for KdTreeAccel (accelerators/kdtreeaccel.rs:25-32): the
    same SAH kd-tree, traversed on the B200.  Queries, surface interactions
    and path tracing work as on GpuBVHAccel."""

    def __init__(self, ctx: Context, shapes: Sequence, isect_cost: int = 80, traversal_cost: int = 1,
                 empty_bonus: float = 0.5, max_prims: int = 1, max_depth: int = -1):
        self.ctx = ctx
        ids = (ctypes.c_uint32 * len(shapes))(*[s.id for s in shapes])
        opts = _lib.ilm_kdtree_opts(isect_cost, traversal_cost, empty_bonus, max_prims, max_depth)
        aid = ctypes.c_uint32()
        ctx.check(ctx._lib.ilm_kdtree_build(ctx.handle, ids, len(shapes), ctypes.byref(opts), ctypes.byref(aid)),
                  "ilm_kdtree_build")
        self.id = aid.value
        self.width = _lib.ILM_LAYOUT_KDTREE
        self.n_prims = sum(s.n_prims for s in shapes)

    def binary_nodes(self):
        raise NotImplementedError("a kd-tree has no BVH nodes; see kd_nodes()")

    def kd_nodes(self):
        """(nodes as KD_NODE_DTYPE, leaf index list as uint32)."""
        inf = self.info()
        nodes = np.zeros(inf["n_nodes"], _lib.KD_NODE_DTYPE)
        index = np.zeros(inf["n_leaf_refs"], np.uint32)
        self.ctx.check(self.ctx._lib.ilm_accel_kd_nodes(self.ctx.handle, self.id, ptr(nodes), ptr(index)),
                       "ilm_accel_kd_nodes")
        return nodes, index


class PathTracer:
    """Wavefront path tracer over a triangle GpuBVHAccel (ilm_pt_scene_create /
    ilm_render_pt): Lambertian materials, one-sided diffuse emitters, a pinhole
    camera looking +z in its own frame (camera_to_world places it)."""

    def __init__(self, accel: GpuBVHAccel, prim_material, albedo, emission, eye, fov_deg: float, width: int,
                 height: int, camera_to_world=None):
        """camera_to_world: 3x3 taking camera-space directions (looking +z,
        up +y) to world space; None = identity."""
        self.accel = accel
        ctx = accel.ctx
        self._mat = np.ascontiguousarray(prim_material, np.uint32)
        self._alb = np.ascontiguousarray(albedo, np.float32).reshape(-1, 3)
        self._emi = np.ascontiguousarray(emission, np.float32).reshape(-1, 3)
        d = _lib.ilm_pt_scene_desc()
        d.prim_material = ptr(self._mat)
        d.albedo = ptr(self._alb)
        d.emission = ptr(self._emi)
        d.n_materials = len(self._alb)
        for k in range(3):
            d.eye[k] = eye[k]
        d.fov_deg = fov_deg
        d.width, d.height = width, height
        if camera_to_world is not None:
            for k, v in enumerate(np.asarray(camera_to_world, np.float32).reshape(9)):
                d.camera_to_world[k] = float(v)
        sid = ctypes.c_uint32()
        ctx.check(ctx._lib.ilm_pt_scene_create(ctx.handle, accel.id, ctypes.byref(d), ctypes.byref(sid)),
                  "ilm_pt_scene_create")
        self.id = sid.value
        self.width, self.height = width, height

    def render(self, spp: int, max_depth: int = 8, rr_depth: int = 3, seed: int = 3, wave_paths: int = 0,
               use_graphs: bool = True, out=None, filter=None):
        """Returns (rgb[h, w, 3] float32 (host) or `out`, stats dict).  `filter`:
        an image.filter_desc (default: each sample in its own pixel)."""
        ctx = self.accel.ctx
        o = _lib.ilm_pt_opts(spp, max_depth, rr_depth, seed, wave_paths, int(use_graphs))
        if filter is not None:
            o.filter = filter
        st = _lib.ilm_pt_stats()
        if out is None:
            out = np.empty((self.height, self.width, 3), np.float32)
        ctx.check(ctx._lib.ilm_render_pt(ctx.handle, self.id, ctypes.byref(o), ptr(out), ctypes.byref(st)),
                  "ilm_render_pt")
        return out, {"closest_rays": st.closest_rays, "shadow_rays": st.shadow_rays, "seconds": st.seconds,
                     "waves": st.waves}

    def render_nrc(self, cache, frames: int = 0, spp_per_frame: int = 1, max_depth: int = 8, rr_depth: int = 3,
                   seed: int = 3, spread_c: float = 0.003, train_paths: int = 16384, train_samples: int = 65536,
                   time_budget_s: float = 0.0, train: bool = True, train_steps: int = 2, train_suffix: int = 1,
                   out=None):
        """Path tracing with a RadianceCache (ilm_render_nrc): frames of
        spp_per_frame samples, the cache answering paths whose spread has
        grown, train_steps Adam steps per frame.  Returns (rgb or `out`, stats)."""
        ctx = self.accel.ctx
        o = _lib.ilm_nrc_render_opts(frames, spp_per_frame, max_depth, rr_depth, seed, spread_c, train_paths,
                                     train_samples, time_budget_s, int(train), train_steps, train_suffix)
        st = _lib.ilm_nrc_render_stats()
        if out is None:
            out = np.empty((self.height, self.width, 3), np.float32)
        ctx.check(ctx._lib.ilm_render_nrc(ctx.handle, self.id, cache.handle, ctypes.byref(o), ptr(out),
                                          ctypes.byref(st)), "ilm_render_nrc")
        return out, {"frames": st.frames, "seconds": st.seconds, "closest_rays": st.closest_rays,
                     "shadow_rays": st.shadow_rays, "queries": st.queries, "train_samples": st.train_samples,
                     "last_loss": st.last_loss}


class Scene:
    """Scene (core/scene.rs:10-53): an aggregate plus lights."""

    def __init__(self, aggregate: GpuBVHAccel, lights: Sequence = ()):
        self.aggregate = aggregate
        self.lights = list(lights)
        self.world_bound = aggregate.world_bound()

    def intersect(self, ray: Ray) -> Optional[Hit]:
        return self.aggregate.intersect(ray)

    def intersect_p(self, ray: Ray) -> bool:
        return self.aggregate.intersect_p(ray)


def _count(buf, rec: int) -> int:
    if isinstance(buf, np.ndarray):
        return buf.nbytes // rec
    return buf.numel() * buf.element_size() // rec


def _stream(stream, buf=None):
    """The cudaStream_t to pass.  With no stream given, a call on torch CUDA
    tensors runs on torch's current stream of their device, so it is ordered
    after the torch work that produced them; a call on host arrays passes NULL
    (the context's own stream)."""
    if stream is None:
        if getattr(buf, "is_cuda", False):
            import torch
            h = torch.cuda.current_stream(buf.device).cuda_stream
            # torch's default stream is the legacy default stream, handle 0;
            # the C ABI reads NULL as the context's stream, so name it by
            # its explicit handle, cudaStreamLegacy (0x1)
            return h if h else CUDA_STREAM_LEGACY
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream     # torch.cuda.Stream

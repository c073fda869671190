"""CPU oracle (test infrastructure only).

ctypes wrapper of ``oracle/liboracle.so``, a scalar C++ restatement of
rs_illume's ray-query hot path (see oracle/oracle.h for the file:line map and
the D1..D24 repairs).  Only tests/, ``__graft_entry__.smoke()`` and bench.py's
CPU-baseline / reference legs use it, as the checker; the product library never
links or calls it.

Parity status: unpinned by the reference's own tests -- the reference has no
tests, golden vectors or fixtures for this path and cannot be compiled here.
The restatement is pinned to analytic known-answer cases instead
(tests/test_oracle_kat.py).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")

RAY_DTYPE = np.dtype([("o", "<f4", (3,)), ("tmin", "<f4"), ("d", "<f4", (3,)), ("tmax", "<f4")])
HIT_DTYPE = np.dtype([("prim", "<u4"), ("t", "<f4"), ("u", "<f4"), ("v", "<f4")])
KD_NODE_DTYPE = np.dtype([("word", "<u4"), ("flags", "<u4")])
BIN_NODE_DTYPE = np.dtype([("bmin", "<f4", (3,)), ("bmax", "<f4", (3,)), ("offset", "<i4"),
                           ("n_prims", "<u2"), ("axis", "u1"), ("pad", "u1")])


class orc_sphere_desc(ctypes.Structure):
    _fields_ = [("object_to_world", ctypes.c_float * 16), ("world_to_object", ctypes.c_float * 16),
                ("radius", ctypes.c_float), ("z_min", ctypes.c_float), ("z_max", ctypes.c_float),
                ("phi_max_deg", ctypes.c_float), ("reverse_orientation", ctypes.c_int32),
                ("kind", ctypes.c_int32), ("height", ctypes.c_float), ("inner_radius", ctypes.c_float),
                ("p1", ctypes.c_float * 3), ("p2", ctypes.c_float * 3)]


class orc_curve_desc(ctypes.Structure):
    _fields_ = [("object_to_world", ctypes.c_float * 16), ("world_to_object", ctypes.c_float * 16),
                ("cp", ctypes.c_float * 12), ("width", ctypes.c_float * 2), ("n", ctypes.c_float * 6),
                ("u_min", ctypes.c_float), ("u_max", ctypes.c_float), ("type", ctypes.c_int32),
                ("reverse_orientation", ctypes.c_int32)]


_P = ctypes.c_void_p
_SIG = {
    "orc_gamma": (ctypes.c_float, [ctypes.c_int]),
    "orc_next_float_up": (ctypes.c_float, [ctypes.c_float]),
    "orc_next_float_down": (ctypes.c_float, [ctypes.c_float]),
    "orc_rng_u32": (None, [ctypes.c_uint64, ctypes.c_uint64, _P]),
    "orc_rng_floats": (None, [ctypes.c_uint64, ctypes.c_uint64, _P]),
    "orc_rng_floats_advanced": (None, [ctypes.c_uint64, ctypes.c_int64, ctypes.c_uint64, _P]),
    "orc_scene_create": (_P, [_P, ctypes.c_uint32, _P, ctypes.c_uint32, _P, ctypes.c_uint32, ctypes.c_int]),
    "orc_scene_destroy": (None, [_P]),
    "orc_scene_create_curves": (_P, [_P, ctypes.c_uint32, _P, ctypes.c_uint32, _P, ctypes.c_uint32, _P,
                                     ctypes.c_uint32, ctypes.c_int]),
    "orc_curve_intersect": (ctypes.c_int, [_P, _P, _P]),
    "orc_scene_node_count": (ctypes.c_uint32, [_P]),
    "orc_scene_nodes": (None, [_P, _P]),
    "orc_scene_prim_order": (None, [_P, _P]),
    "orc_scene_world_bound": (None, [_P, _P]),
    "orc_scene_build_seconds": (ctypes.c_double, [_P]),
    "orc_intersect": (ctypes.c_int64, [_P, _P, ctypes.c_uint64, _P, _P, _P, ctypes.c_int]),
    "orc_intersect_p": (ctypes.c_int64, [_P, _P, ctypes.c_uint64, _P, _P, _P, ctypes.c_int]),
    "orc_triangle_intersect": (ctypes.c_int, [_P, _P, _P, _P, ctypes.c_int, _P]),
    "orc_surface_interaction": (ctypes.c_int, [_P, _P, _P, _P, ctypes.c_int, _P, _P]),
    "orc_render_pt_filtered": (ctypes.c_int, [_P, _P, _P, ctypes.c_uint32, _P, _P, _P, _P, ctypes.c_float,
                                              ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                              ctypes.c_uint32, ctypes.c_uint64, _P, ctypes.c_float, ctypes.c_float,
                                              ctypes.c_int, _P, _P, _P]),
    "orc_sphere_intersect": (ctypes.c_int, [_P, _P, ctypes.c_int, _P]),
    "orc_sphere_world_bound": (None, [_P, _P]),
    "orc_last_trace_seconds": (ctypes.c_double, []),
    "orc_wl_icosphere_counts": (None, [ctypes.c_uint32, _P, _P]),
    "orc_wl_icosphere": (None, [ctypes.c_uint32, ctypes.c_uint64, ctypes.c_float, ctypes.c_float, _P, _P, _P]),
    "orc_wl_ball_rays": (None, [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_float,
                                ctypes.c_float, ctypes.c_float, _P]),
    "orc_wl_soup": (None, [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_float, _P, _P]),
    "orc_wl_camera_rays": (None, [ctypes.c_uint32, ctypes.c_uint32, _P, ctypes.c_float, _P]),
    "orc_kdtree_create": (_P, [_P, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_uint32, ctypes.c_int]),
    "orc_kdtree_destroy": (None, [_P]),
    "orc_kdtree_node_count": (ctypes.c_uint32, [_P]),
    "orc_kdtree_index_count": (ctypes.c_uint32, [_P]),
    "orc_kdtree_max_depth": (ctypes.c_int, [_P]),
    "orc_kdtree_nodes": (None, [_P, _P]),
    "orc_kdtree_indices": (None, [_P, _P]),
    "orc_kdtree_intersect": (ctypes.c_int64, [_P, _P, ctypes.c_uint64, _P, _P, _P, ctypes.c_int]),
    "orc_kdtree_intersect_p": (ctypes.c_int64, [_P, _P, ctypes.c_uint64, _P, _P, _P, ctypes.c_int]),
    "orc_render_pt": (ctypes.c_int, [_P, _P, _P, ctypes.c_uint32, _P, _P, _P, _P, ctypes.c_float, ctypes.c_uint32,
                                     ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                     ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                     ctypes.c_uint32, ctypes.c_int, _P, _P]),
}

_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C oracle`")
        lib = ctypes.CDLL(LIB_PATH)
        for k, (r, a) in _SIG.items():
            f = getattr(lib, k)
            f.restype = r
            f.argtypes = a
        _lib = lib
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def gamma(n: int) -> float:
    return load().orc_gamma(n)


def rng_floats(seq: int, n: int, advance: int = 0) -> np.ndarray:
    out = np.empty(n, np.float32)
    if advance:
        load().orc_rng_floats_advanced(seq, advance, n, _p(out))
    else:
        load().orc_rng_floats(seq, n, _p(out))
    return out


def rng_u32(seq: int, n: int) -> np.ndarray:
    out = np.empty(n, np.uint32)
    load().orc_rng_u32(seq, n, _p(out))
    return out


def quadric_desc(kind: int, radius: float, matrix, z_min: float = 0.0, z_max: float = 0.0,
                 phi_max_deg: float = 360.0, height: float = 0.0, inner_radius: float = 0.0,
                 reverse: bool = False, p1=(0.0, 0.0, 0.0), p2=(0.0, 0.0, 0.0)) -> orc_sphere_desc:
    """Any quadric (kind 0 sphere, 1 disk, 2 cylinder, 3 cone, 4 paraboloid,
    5 hyperboloid) under a 4x4 object-to-world matrix (its inverse computed in
    float64)."""
    m = np.asarray(matrix, np.float64).reshape(4, 4)
    inv = np.linalg.inv(m)
    d = orc_sphere_desc()
    for i in range(16):
        d.object_to_world[i] = float(np.float32(m.flat[i]))
        d.world_to_object[i] = float(np.float32(inv.flat[i]))
    d.kind, d.radius, d.z_min, d.z_max = kind, radius, z_min, z_max
    d.phi_max_deg, d.height, d.inner_radius, d.reverse_orientation = phi_max_deg, height, inner_radius, int(reverse)
    for k in range(3):
        d.p1[k], d.p2[k] = p1[k], p2[k]
    return d


def sphere_desc(radius: float, translate=(0.0, 0.0, 0.0), scale: float = 1.0, z_min=None, z_max=None,
                phi_max_deg: float = 360.0, reverse: bool = False) -> orc_sphere_desc:
    d = orc_sphere_desc()
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


class Scene:
    """BVHAccel over triangles (ids 0..nt-1) followed by spheres."""

    def __init__(self, xyz, idx, spheres=(), max_prims_in_node: int = 4, curves=()):
        lib = load()
        self._xyz = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
        self._idx = np.ascontiguousarray(idx, np.uint32).reshape(-1, 3)
        sph = (orc_sphere_desc * max(1, len(spheres)))(*spheres)
        cur = (orc_curve_desc * max(1, len(curves)))(*curves)
        self.n_prims = len(self._idx) + len(spheres) + len(curves)
        self.h = lib.orc_scene_create_curves(_p(self._xyz), len(self._xyz), _p(self._idx), len(self._idx),
                                             ctypes.addressof(sph), len(spheres), ctypes.addressof(cur), len(curves),
                                             max_prims_in_node)

    def __del__(self):
        if getattr(self, "h", None):
            load().orc_scene_destroy(self.h)
            self.h = None

    @property
    def build_seconds(self) -> float:
        return load().orc_scene_build_seconds(self.h)

    def nodes(self) -> np.ndarray:
        n = load().orc_scene_node_count(self.h)
        out = np.zeros(n, BIN_NODE_DTYPE)
        load().orc_scene_nodes(self.h, _p(out))
        return out

    def prim_order(self) -> np.ndarray:
        out = np.zeros(self.n_prims, np.uint32)
        load().orc_scene_prim_order(self.h, _p(out))
        return out

    def world_bound(self) -> np.ndarray:
        out = np.zeros(6, np.float32)
        load().orc_scene_world_bound(self.h, _p(out))
        return out

    def intersect(self, rays: np.ndarray, threads: int = 0, counters: bool = False):
        rays = np.ascontiguousarray(rays)
        hits = np.empty(len(rays), HIT_DTYPE)
        nv = np.empty(len(rays), np.uint32) if counters else None
        nt = np.empty(len(rays), np.uint32) if counters else None
        ovf = load().orc_intersect(self.h, _p(rays), len(rays), _p(hits), _p(nv), _p(nt), threads)
        assert ovf == 0, f"{ovf} rays overflowed the 64-entry traversal stack"
        return (hits, nv, nt) if counters else hits

    def intersect_p(self, rays: np.ndarray, threads: int = 0, counters: bool = False):
        rays = np.ascontiguousarray(rays)
        occ = np.empty(len(rays), np.uint8)
        nv = np.empty(len(rays), np.uint32) if counters else None
        nt = np.empty(len(rays), np.uint32) if counters else None
        ovf = load().orc_intersect_p(self.h, _p(rays), len(rays), _p(occ), _p(nv), _p(nt), threads)
        assert ovf == 0, f"{ovf} rays overflowed the 64-entry traversal stack"
        return (occ, nv, nt) if counters else occ


class KdTree:
    """KdTreeAccel (accelerators/kdtreeaccel.rs:25-465) over a Scene's
    primitives, with the same primitive ids."""

    def __init__(self, scene: Scene, isect_cost: int = 80, traversal_cost: int = 1, empty_bonus: float = 0.5,
                 max_prims: int = 1, max_depth: int = -1):
        self.scene = scene          # the tree's primitive tests read the scene
        self.h = load().orc_kdtree_create(scene.h, isect_cost, traversal_cost, empty_bonus, max_prims, max_depth)

    def __del__(self):
        if getattr(self, "h", None):
            load().orc_kdtree_destroy(self.h)
            self.h = None

    @property
    def max_depth(self) -> int:
        return load().orc_kdtree_max_depth(self.h)

    def nodes(self) -> np.ndarray:
        out = np.zeros(load().orc_kdtree_node_count(self.h), KD_NODE_DTYPE)
        load().orc_kdtree_nodes(self.h, _p(out))
        return out

    def indices(self) -> np.ndarray:
        out = np.zeros(load().orc_kdtree_index_count(self.h), np.uint32)
        load().orc_kdtree_indices(self.h, _p(out))
        return out

    def intersect(self, rays: np.ndarray, threads: int = 0, counters: bool = False):
        rays = np.ascontiguousarray(rays)
        hits = np.empty(len(rays), HIT_DTYPE)
        nv = np.empty(len(rays), np.uint32) if counters else None
        nt = np.empty(len(rays), np.uint32) if counters else None
        ovf = load().orc_kdtree_intersect(self.h, _p(rays), len(rays), _p(hits), _p(nv), _p(nt), threads)
        assert ovf == 0, f"{ovf} rays overflowed the 64-entry kd-tree stack"
        return (hits, nv, nt) if counters else hits

    def intersect_p(self, rays: np.ndarray, threads: int = 0, counters: bool = False):
        rays = np.ascontiguousarray(rays)
        occ = np.empty(len(rays), np.uint8)
        nv = np.empty(len(rays), np.uint32) if counters else None
        nt = np.empty(len(rays), np.uint32) if counters else None
        ovf = load().orc_kdtree_intersect_p(self.h, _p(rays), len(rays), _p(occ), _p(nv), _p(nt), threads)
        assert ovf == 0, f"{ovf} rays overflowed the 64-entry kd-tree stack"
        return (occ, nv, nt) if counters else occ


def render_pt(scene: "Scene", xyz, idx, mat, albedo, emission, eye, fov_deg, width, height, spp, max_depth=8,
              rr_depth=3, seed=3, window=None, threads=0, traversal_counts=False):
    """Path-traced image (oracle/pt.cpp).  Returns (rgb[h, w, 3], (closest rays, shadow rays)), and with
    traversal_counts a third item: (closest node visits, closest triangle tests, shadow node visits,
    shadow triangle tests), summed over the rays on the binary SAH BVH."""
    x0, y0, x1, y1 = window if window else (0, 0, width, height)
    xyz = np.ascontiguousarray(xyz, np.float32)
    idx = np.ascontiguousarray(idx, np.uint32)
    mat = np.ascontiguousarray(mat, np.uint32)
    albedo = np.ascontiguousarray(albedo, np.float32)
    emission = np.ascontiguousarray(emission, np.float32)
    eye = np.asarray(eye, np.float32)
    out = np.zeros((y1 - y0, x1 - x0, 3), np.float32)
    counts = np.zeros(6, np.uint64)
    st = load().orc_render_pt(scene.h, _p(xyz), _p(idx), len(idx), _p(mat), _p(albedo), _p(emission), _p(eye),
                              fov_deg, width, height, spp, max_depth, rr_depth, seed, x0, y0, x1, y1, threads,
                              _p(out), _p(counts))
    assert st == 0, "invalid render arguments"
    if traversal_counts:
        return out, (int(counts[0]), int(counts[1])), tuple(int(c) for c in counts[2:])
    return out, (int(counts[0]), int(counts[1]))


def render_pt_filtered(scene: "Scene", xyz, idx, mat, albedo, emission, eye, fov_deg, width, height, spp,
                       table, radius, max_depth=8, rr_depth=3, seed=3, threads=0, camera_to_world=None):
    """Full-frame render through a filtered film (16 x 16 weight table,
    radius (rx, ry)).  Returns (rgb[h, w, 3], (closest rays, shadow rays))."""
    xyz = np.ascontiguousarray(xyz, np.float32)
    idx = np.ascontiguousarray(idx, np.uint32)
    mat = np.ascontiguousarray(mat, np.uint32)
    albedo = np.ascontiguousarray(albedo, np.float32)
    emission = np.ascontiguousarray(emission, np.float32)
    eye = np.asarray(eye, np.float32)
    table = np.ascontiguousarray(table, np.float32)
    out = np.zeros((height, width, 3), np.float32)
    counts = np.zeros(2, np.uint64)
    cam = None if camera_to_world is None else np.ascontiguousarray(camera_to_world, np.float32).reshape(9)
    st = load().orc_render_pt_filtered(scene.h, _p(xyz), _p(idx), len(idx.reshape(-1, 3)), _p(mat), _p(albedo),
                                       _p(emission), _p(eye), fov_deg, width, height, spp, max_depth, rr_depth, seed,
                                       _p(table), radius[0], radius[1], threads, _p(out), _p(counts), _p(cam))
    assert st == 0
    return out, (int(counts[0]), int(counts[1]))


def last_trace_seconds() -> float:
    return load().orc_last_trace_seconds()


def triangle_intersect(p0, p1, p2, o, d, tmax=float("inf"), closest=True):
    """Returns (t, b0, b1, b2) or None."""
    r = np.zeros(1, RAY_DTYPE)
    r["o"][0] = o
    r["d"][0] = d
    r["tmax"][0] = tmax
    pts = [np.asarray(p, np.float32) for p in (p0, p1, p2)]
    out = np.zeros(4, np.float32)
    ok = load().orc_triangle_intersect(_p(pts[0]), _p(pts[1]), _p(pts[2]), _p(r), int(closest), _p(out))
    return tuple(float(x) for x in out) if ok else None


SI_DTYPE = np.dtype([
    ("p", "<f4", (3,)), ("p_error", "<f4", (3,)), ("n", "<f4", (3,)), ("uv", "<f4", (2,)),
    ("dpdu", "<f4", (3,)), ("dpdv", "<f4", (3,)), ("dndu", "<f4", (3,)), ("dndv", "<f4", (3,)),
    ("shading_n", "<f4", (3,)), ("shading_dpdu", "<f4", (3,)), ("shading_dpdv", "<f4", (3,)),
    ("shading_dndu", "<f4", (3,)), ("shading_dndv", "<f4", (3,)), ("wo", "<f4", (3,)), ("t", "<f4"),
    ("prim", "<u4"), ("kind", "<u4")])


def surface_interaction(p, o, d, tmax=float("inf"), n=None, s=None, uv=None, reverse=False):
    """The SurfaceInteraction of the hit on triangle p (3 x 3 vertices)
    (oracle/interaction.cpp); None on a miss."""
    p = np.ascontiguousarray(p, np.float32).reshape(9)
    arrs = [None if a is None else np.ascontiguousarray(a, np.float32).ravel() for a in (n, s, uv)]
    r = np.zeros(1, RAY_DTYPE)
    r["o"], r["d"], r["tmax"] = o, d, tmax
    out = np.zeros(1, SI_DTYPE)
    hit = load().orc_surface_interaction(_p(p), *(_p(a) if a is not None else None for a in arrs), int(reverse),
                                         _p(r), _p(out))
    return out[0] if hit else None


def curve_desc(cp, width, matrix=None, curve_type: int = 0, normals=None, u_range=(0.0, 1.0),
               reverse: bool = False) -> orc_curve_desc:
    """One curve segment: cp 4x3 control points, width (w0, w1), optional
    4x4 object-to-world (inverse taken in float64), type 0 flat, 1 cylinder,
    2 ribbon (normals 2x3)."""
    m = np.eye(4) if matrix is None else np.asarray(matrix, np.float64).reshape(4, 4)
    inv = np.linalg.inv(m)
    d = orc_curve_desc()
    for i in range(16):
        d.object_to_world[i] = float(np.float32(m.flat[i]))
        d.world_to_object[i] = float(np.float32(inv.flat[i]))
    for i, v in enumerate(np.asarray(cp, np.float32).reshape(12)):
        d.cp[i] = float(v)
    d.width[0], d.width[1] = width
    if normals is not None:
        for i, v in enumerate(np.asarray(normals, np.float32).reshape(6)):
            d.n[i] = float(v)
    d.u_min, d.u_max = u_range
    d.type = curve_type
    d.reverse_orientation = int(reverse)
    return d


def curve_intersect(desc: orc_curve_desc, o, d, tmax=float("inf")):
    """Returns (t, u, v) or None."""
    r = np.zeros(1, RAY_DTYPE)
    r["o"][0] = o
    r["d"][0] = d
    r["tmax"][0] = tmax
    out = np.zeros(3, np.float32)
    ok = load().orc_curve_intersect(ctypes.byref(desc), _p(r), _p(out))
    return tuple(float(x) for x in out) if ok else None


def sphere_intersect(desc: orc_sphere_desc, o, d, tmax=float("inf")):
    """Returns (t, u, v) or None."""
    r = np.zeros(1, RAY_DTYPE)
    r["o"][0] = o
    r["d"][0] = d
    r["tmax"][0] = tmax
    out = np.zeros(3, np.float32)
    ok = load().orc_sphere_intersect(ctypes.byref(desc), _p(r), 1, _p(out))
    return tuple(float(x) for x in out) if ok else None


# --- the oracle's own copy of the benchmark inputs (oracle/workloads.cpp) ---

def icosphere(level: int, seed: int, amplitude: float = 0.05, radius: float = 1.0, centre=(0.0, 0.0, 0.0)):
    nv, nt = ctypes.c_uint32(), ctypes.c_uint32()
    load().orc_wl_icosphere_counts(level, ctypes.byref(nv), ctypes.byref(nt))
    xyz = np.empty((nv.value, 3), np.float32)
    idx = np.empty((nt.value, 3), np.uint32)
    c = np.asarray(centre, np.float32)
    load().orc_wl_icosphere(level, seed, amplitude, radius, _p(c), _p(xyz), _p(idx))
    return xyz, idx


def ball_rays(seed: int, skip: int, n: int, n_closest: int, radius: float = 3.0, tmax_lo: float = 0.1,
              tmax_hi: float = 4.0) -> np.ndarray:
    out = np.empty(n, RAY_DTYPE)
    load().orc_wl_ball_rays(seed, skip, n, n_closest, radius, tmax_lo, tmax_hi, _p(out))
    return out


def soup(seed: int = 1, n: int = 32768, spread: float = 0.02):
    xyz = np.empty((3 * n, 3), np.float32)
    idx = np.empty((n, 3), np.uint32)
    load().orc_wl_soup(seed, n, spread, _p(xyz), _p(idx))
    return xyz, idx


def camera_rays(width: int = 256, height: int = 256, eye=(0.5, 0.5, -1.5), fov_deg: float = 45.0) -> np.ndarray:
    out = np.empty(width * height, RAY_DTYPE)
    e = np.asarray(eye, np.float32)
    load().orc_wl_camera_rays(width, height, _p(e), fov_deg, _p(out))
    return out


def incoherent_workload(n_rays: int = 4194304, level: int = 8):
    """Displaced icosphere (seed 2) + ball rays (first half closest, second half shadow)."""
    xyz, idx = icosphere(level, 2, 0.05, 1.0)
    return xyz, idx, ball_rays(2, 4, n_rays, n_rays // 2, 3.0, 0.1, 4.0)


def coherent_workload():
    """32,768-triangle soup (seed 1) + 256x256 primary rays."""
    xyz, idx = soup(1, 32768, 0.02)
    return xyz, idx, camera_rays(256, 256, (0.5, 0.5, -1.5), 45.0)

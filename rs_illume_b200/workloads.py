"""Seeded synthetic inputs for the benchmark configurations.

The reference ships no benchmark inputs, so scenes and rays are generated
procedurally with the reference's PCG32 (src/core/rng.rs) by the C++ generators
in csrc/workloads.cpp (declared in include/illume_workloads.h).

  coherent      32,768-triangle soup in the unit cube (centre ~ U[0,1]^3, vertex
                offsets ~ U[-0.02, 0.02]^3, seed 1), 256x256 pinhole primary rays
                from (0.5, 0.5, -1.5) looking +z, 45 degree vertical fov.
  incoherent    displaced icosphere level 8 (1,310,720 triangles, seed 2);
                4,194,304 rays from a radius-3 ball with uniform directions;
                the first half closest-hit (tmax = inf), the second half shadow
                rays with tmax ~ U[0.1, 4].
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib
from ._lib import RAY_DTYPE, ptr


def rng_floats(seq: int, n: int) -> np.ndarray:
    out = np.empty(n, np.float32)
    _lib.load().ilm_wl_rng_floats(seq, n, ptr(out))
    return out


def rng_u32(seq: int, n: int) -> np.ndarray:
    out = np.empty(n, np.uint32)
    _lib.load().ilm_wl_rng_u32(seq, n, ptr(out))
    return out


def soup(seed: int = 1, n: int = 32768, spread: float = 0.02):
    xyz = np.empty((3 * n, 3), np.float32)
    idx = np.empty((n, 3), np.uint32)
    _lib.load().ilm_wl_soup(seed, n, spread, ptr(xyz), ptr(idx))
    return xyz, idx


def icosphere_counts(level: int):
    nv, nt = ctypes.c_uint32(), ctypes.c_uint32()
    _lib.load().ilm_wl_icosphere_counts(level, ctypes.byref(nv), ctypes.byref(nt))
    return nv.value, nt.value


def icosphere(level: int, seed: int, amplitude: float = 0.05, radius: float = 1.0, centre=(0.0, 0.0, 0.0)):
    nv, nt = icosphere_counts(level)
    xyz = np.empty((nv, 3), np.float32)
    idx = np.empty((nt, 3), np.uint32)
    c = np.asarray(centre, np.float32)
    _lib.load().ilm_wl_icosphere(level, seed, amplitude, radius, ptr(c), ptr(xyz), ptr(idx))
    return xyz, idx


def camera_rays(width: int = 256, height: int = 256, eye=(0.5, 0.5, -1.5), fov_deg: float = 45.0) -> np.ndarray:
    out = np.empty(width * height, RAY_DTYPE)
    e = np.asarray(eye, np.float32)
    _lib.load().ilm_wl_camera_rays(width, height, ptr(e), fov_deg, ptr(out))
    return out


def ball_rays(seed: int = 2, skip: int = 4, n: int = 4194304, n_closest: int | None = None, radius: float = 3.0,
              tmax_lo: float = 0.1, tmax_hi: float = 4.0) -> np.ndarray:
    if n_closest is None:
        n_closest = n // 2
    out = np.empty(n, RAY_DTYPE)
    _lib.load().ilm_wl_ball_rays(seed, skip, n, n_closest, radius, tmax_lo, tmax_hi, ptr(out))
    return out


CORNELL_CAMERA = {"eye": (0.5, 0.5, -1.37), "fov_deg": 40.0}


def cornell(ico_level: int = 6, seed: int = 3):
    """Procedural Cornell box (include/illume_workloads.h): returns
    (xyz, idx, material per triangle, albedo[4,3], emission[4,3])."""
    lib = _lib.load()
    nv, nt = ctypes.c_uint32(), ctypes.c_uint32()
    lib.ilm_wl_cornell_counts(ico_level, ctypes.byref(nv), ctypes.byref(nt))
    xyz = np.empty((nv.value, 3), np.float32)
    idx = np.empty((nt.value, 3), np.uint32)
    mat = np.empty(nt.value, np.uint32)
    albedo = np.empty((4, 3), np.float32)
    emission = np.empty((4, 3), np.float32)
    lib.ilm_wl_cornell(ico_level, seed, ptr(xyz), ptr(idx), ptr(mat), ptr(albedo), ptr(emission))
    return xyz, idx, mat, albedo, emission


def batched_workload(seed: int = 5, n_scenes: int = 32, tris=(1e3, 2e6), rays=(1e4, 4e6)):
    """Uneven multi-scene workload: per scene (draws of Rng::new(seed), 4 per
    scene) a kind (icosphere or triangle soup), a triangle count and a ray
    count, both log-uniform in the given ranges, and a ray mix of one third
    primary pinhole rays, one third incoherent ball rays (tmax = inf) and one
    third shadow rays (tmax ~ U[0.1, 4]).  Icospheres take the subdivision
    level nearest the target count (at most 8); soups keep their triangle
    size proportional to count^(-1/3).  Returns a list of dicts."""
    u = rng_floats(seed, 4 * n_scenes).astype(np.float64)
    out = []
    for k in range(n_scenes):
        uk, ut, ur, us = u[4 * k: 4 * k + 4]
        t = math.exp(math.log(tris[0]) + ut * (math.log(tris[1]) - math.log(tris[0])))
        r = int(math.exp(math.log(rays[0]) + ur * (math.log(rays[1]) - math.log(rays[0]))))
        sub_seed = 1000 + 16 * seed + k
        if uk < 0.5:
            level = int(min(8, max(1, round(math.log(t / 20.0, 4)))))
            xyz, idx = icosphere(level, sub_seed, 0.05, 1.0)
            eye, radius = (0.0, 0.0, -3.5), 3.0
        else:
            n = int(t)
            xyz, idx = soup(sub_seed, n, 0.02 * (32768.0 / n) ** (1.0 / 3.0))
            eye, radius = (0.5, 0.5, -1.5), 1.5
        n1 = r // 3
        side = max(1, int(math.ceil(math.sqrt(n1))))
        prim = camera_rays(side, side, eye, 45.0)[:n1]
        inc = ball_rays(sub_seed, 0, r - n1, (r - n1) // 2, radius, 0.1, 4.0)
        if uk >= 0.5:   # soups live in the unit cube: centre the ball rays on it
            inc["o"] += np.float32(0.5)
        rays_k = np.ascontiguousarray(np.concatenate([prim, inc]))
        out.append({"kind": "icosphere" if uk < 0.5 else "soup", "xyz": xyz, "idx": idx, "rays": rays_k,
                    "seed": sub_seed})
    return out


def coherent_workload():
    """32,768-triangle soup + 65,536 primary rays."""
    xyz, idx = soup(1, 32768, 0.02)
    return xyz, idx, camera_rays(256, 256, (0.5, 0.5, -1.5), 45.0)


def incoherent_workload(n_rays: int = 4194304, level: int = 8):
    """Displaced icosphere + ball rays (first half closest, second half shadow)."""
    xyz, idx = icosphere(level, 2, 0.05, 1.0)
    rays = ball_rays(2, 4, n_rays, n_rays // 2, 3.0, 0.1, 4.0)
    return xyz, idx, rays

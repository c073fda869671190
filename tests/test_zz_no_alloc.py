"""The allocation-free closest-hit entry point (ilm_intersect_closest_noalloc).

It exists for callers that cannot call cudaMalloc once set up (a render loop
with a fixed memory budget, a process whose device memory belongs to a caching
allocator, a thread that must not stall the device).  Its results must equal
ilm_intersect_closest's -- the same traversal kernel, with its scratch taken
from the library's fixed array -- on two calls in a row, since the array
keeps the previous call's contents.  This file is collected last so that a run
stopping at the first failure has already run every other test; it also passes
on its own in a fresh process (the first call on the device does the set-up).
"""
import ctypes

import numpy as np
import pytest

import rs_illume_b200 as rb
from rs_illume_b200 import _lib
from rs_illume_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def call_noalloc(ctx, acc, rays, hits, stream=None):
    return ctx._lib.ilm_intersect_closest_noalloc(ctx.handle, acc.id, _lib.ptr(rays), len(rays) if isinstance(
        rays, np.ndarray) else rays.numel() // 32, _lib.ptr(hits), stream)


def test_noalloc_matches_allocating_entry_point_twice():
    ctx = rb.Context(0)
    xyz, idx = wl.icosphere(6, 2)
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx)], width=8)
    for seed in (2, 3):            # two calls in a row, different rays
        rays = wl.ball_rays(seed, 0, 65536, 32768)
        want = acc.intersect_batch(rays)                       # ilm_intersect_closest
        got = np.empty(len(rays), _lib.HIT_DTYPE)
        st = call_noalloc(ctx, acc, rays, got)
        assert st == _lib.ILM_OK, ctx._lib.ilm_last_error_string(ctx.handle)
        # same kernel and arithmetic: the records are identical
        assert got.tobytes() == want.tobytes()
        assert np.sum(got["prim"] != rb.ILM_MISS) > 1000
    ctx.close()


def test_noalloc_device_buffers_and_limit():
    import torch
    ctx = rb.Context(0)
    xyz, idx, rays = wl.coherent_workload()                    # exactly 65,536 rays
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx)], width=8)
    want = acc.intersect_batch(rays)
    d_rays = torch.from_numpy(rays.view(np.uint8)).cuda()
    for _ in range(2):
        d_hits = torch.zeros(len(rays) * 16, dtype=torch.uint8, device="cuda")
        assert call_noalloc(ctx, acc, d_rays, d_hits) == _lib.ILM_OK
        torch.cuda.synchronize()
        assert d_hits.cpu().numpy().tobytes() == want.tobytes()
    # beyond the fixed scratch: refused with a clear message, nothing launched
    big = wl.ball_rays(1, 0, 65537, 65537)
    out = np.empty(len(big), _lib.HIT_DTYPE)
    assert call_noalloc(ctx, acc, big, out) == _lib.ILM_ERR_INVALID_ARGUMENT
    assert b"fixed scratch limit" in ctx._lib.ilm_last_error_string(ctx.handle)
    ctx.close()


def _sphere_scene(ctx):
    rng = np.random.default_rng(5)
    centres = rng.uniform(-1, 1, (32, 3))
    radii = rng.uniform(0.05, 0.2, 32)
    xyz, idx = wl.icosphere(3, 7, 0.05, 0.3, (0.0, 0.0, 1.5))
    spheres = [rb.sphere_desc(float(r), tuple(c)) for c, r in zip(centres, radii)]
    return [rb.TriangleMesh(ctx, xyz, idx), rb.Spheres(ctx, spheres)]


@pytest.mark.parametrize("width,spheres,grid", [(2, False, False), (4, False, False), (8, True, False),
                                                (8, False, True), (2, True, False)])
def test_noalloc_layouts_and_schedules(width, spheres, grid):
    """Binary and wide layouts, scenes with analytic shapes, and the
    one-thread-per-ray schedule: the records equal ilm_intersect_closest's."""
    ctx = rb.Context(0, grid_schedule=grid)
    if spheres:
        shapes = _sphere_scene(ctx)
    else:
        xyz, idx = wl.icosphere(5, 3)
        shapes = [rb.TriangleMesh(ctx, xyz, idx)]
    acc = rb.GpuBVHAccel(ctx, shapes, width=width)
    rays = wl.ball_rays(11, 0, 40000, 40000, 2.5)
    want = acc.intersect_batch(rays)
    got = np.empty(len(rays), _lib.HIT_DTYPE)
    assert call_noalloc(ctx, acc, rays, got) == _lib.ILM_OK, ctx._lib.ilm_last_error_string(ctx.handle)
    assert got.tobytes() == want.tobytes()
    assert np.sum(got["prim"] != rb.ILM_MISS) > 500
    assert ctx.device_errors() == 0
    ctx.close()


def test_noalloc_follows_the_accels_launch_choices():
    """An accel set to a 32-entry stack on a context whose default is 64:
    both entry points run the 32-entry kernel, so the same rays (if any)
    overflow and the records are byte-identical."""
    ctx = rb.Context(0, stack_depth=64)
    xyz, idx = wl.icosphere(6, 2)
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx)], width=8)
    o = _lib.ilm_launch_opts(32, 0, 1)
    ctx.check(ctx._lib.ilm_accel_set_launch(ctx.handle, acc.id, ctypes.byref(o)), "ilm_accel_set_launch")
    rays = wl.ball_rays(4, 0, 65536, 65536)
    want = acc.intersect_batch(rays)
    got = np.empty(len(rays), _lib.HIT_DTYPE)
    assert call_noalloc(ctx, acc, rays, got) == _lib.ILM_OK
    assert got.tobytes() == want.tobytes()
    ctx.close()


def test_noalloc_traversal_limit_is_reported():
    """A context with a 3-step iteration cap: the kernel gives up on long rays
    (a bounded loop, nothing waits), marks their records, sets the context's
    error word, and the host-buffer call returns ILM_ERR_TRAVERSAL_LIMIT."""
    ctx = rb.Context(0, max_iterations=3)
    xyz, idx, rays = wl.coherent_workload()
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx)], width=8)
    got = np.empty(len(rays), _lib.HIT_DTYPE)
    assert call_noalloc(ctx, acc, rays, got) == _lib.ILM_ERR_TRAVERSAL_LIMIT
    assert b"traversal limit" in ctx._lib.ilm_last_error_string(ctx.handle)
    marked = got["prim"] == rb.ILM_TRAVERSAL_ERROR
    assert marked.sum() > 1000
    assert ctx.device_errors() != 0          # the context's word, as for ilm_intersect_closest
    # the allocating entry point marks the same records
    want = np.empty(len(rays), _lib.HIT_DTYPE)
    st = ctx._lib.ilm_intersect_closest(ctx.handle, acc.id, _lib.ptr(rays), len(rays), _lib.ptr(want), None)
    assert st == _lib.ILM_OK
    assert np.array_equal(want["prim"] == rb.ILM_TRAVERSAL_ERROR, marked)
    ctx.close()


def test_noalloc_validates_host_rays_like_the_allocating_call():
    ctx = rb.Context(0, validate_rays=True)
    xyz, idx = wl.icosphere(4, 3)
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx)], width=8)
    rays = wl.ball_rays(5, 0, 1024, 1024)
    rays["d"][17] = 0.0
    got = np.empty(len(rays), _lib.HIT_DTYPE)
    assert call_noalloc(ctx, acc, rays, got) == _lib.ILM_ERR_INVALID_ARGUMENT
    assert b"ray 17" in ctx._lib.ilm_last_error_string(ctx.handle)
    st = ctx._lib.ilm_intersect_closest(ctx.handle, acc.id, _lib.ptr(rays), len(rays), _lib.ptr(got), None)
    assert st == _lib.ILM_ERR_INVALID_ARGUMENT
    ctx.close()

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

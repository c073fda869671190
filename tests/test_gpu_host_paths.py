"""Host-buffer path of ilm_intersect_closest / ilm_intersect_any: rays and
results in host memory (pinned or pageable, in any mix) go through device
staging chunks that overlap copy-in, trace and copy-out; every chunk size
returns the device path's records bit for bit, including sub-ranges and
counts that are not a multiple of the chunk."""
import ctypes

import numpy as np
import pytest

import rs_illume_b200 as rb
from rs_illume_b200 import workloads as wl
from rs_illume_b200._lib import HIT_DTYPE, RAY_DTYPE

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scene():
    xyz, idx = wl.icosphere(6, 2)
    rays = wl.ball_rays(2, 4, (1 << 20) + 12345, 1 << 19)
    return xyz, idx, rays


def pinned(nbytes):
    import torch
    return torch.empty(nbytes, dtype=torch.uint8).pin_memory()


@pytest.mark.parametrize("chunk", [4096, 65536, 1 << 18, 1 << 22])
def test_host_buffers_match_device_path(scene, chunk):
    import torch
    xyz, idx, rays = scene
    ctx = rb.Context(0, high_occupancy=True)
    ctx.check(ctx._lib.ilm_context_set_stage_chunk(ctx.handle, chunk), "ilm_context_set_stage_chunk")
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx)], width=8)
    n = len(rays)
    d_rays = torch.from_numpy(rays.view(np.uint8)).cuda()
    d_hits = torch.empty(n * 16, dtype=torch.uint8, device="cuda")
    d_occ = torch.empty(n * 4, dtype=torch.uint8, device="cuda")
    acc.intersect_batch(d_rays, d_hits)
    acc.intersect_p_batch(d_rays, d_occ)
    torch.cuda.synchronize()
    want_h = d_hits.cpu().numpy()
    want_o = d_occ.cpu().numpy()
    h_rays = pinned(n * 32)
    h_rays.numpy()[:] = rays.view(np.uint8)
    h_hits = pinned(n * 16)
    h_occ = pinned(n * 4)
    for _ in range(2):                      # twice: the second call reuses every buffer
        h_hits.numpy()[:] = 0xAB
        acc.intersect_batch(h_rays.numpy().view(RAY_DTYPE), h_hits.numpy().view(HIT_DTYPE))
        assert h_hits.numpy().tobytes() == want_h.tobytes()
        acc.intersect_p_batch(h_rays.numpy().view(RAY_DTYPE), h_occ.numpy().view(np.uint32))
        assert h_occ.numpy().tobytes() == want_o.tobytes()
    # a sub-range (offset pointers, a count that is not a multiple of the chunk)
    k0, k = 1000, 70001
    sub_h = np.zeros(k, HIT_DTYPE)
    acc.intersect_batch(h_rays.numpy()[32 * k0: 32 * (k0 + k)].view(RAY_DTYPE), sub_h)
    assert sub_h.tobytes() == want_h[16 * k0: 16 * (k0 + k)].tobytes()
    # pageable rays and results
    pageable = np.empty(n, HIT_DTYPE)
    acc.intersect_batch(np.ascontiguousarray(rays), pageable)
    assert pageable.tobytes() == want_h.tobytes()
    assert ctx.device_errors() == 0
    ctx.close()


def test_stage_chunk_limits():
    ctx = rb.Context(0)
    for bad in (0, 4095, (1 << 24) + 1):
        assert ctx._lib.ilm_context_set_stage_chunk(ctx.handle, bad) == rb._lib.ILM_ERR_INVALID_ARGUMENT
    assert ctx._lib.ilm_context_set_stage_chunk(ctx.handle, 1 << 24) == 0
    ctx.close()

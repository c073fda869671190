"""SurfaceInteraction reconstruction (triangle.rs:264-415, interaction.rs:262-339).

CPU: known answers of the oracle restatement on a unit right triangle (uv
derivatives with the D14 determinant, the geometric normal, reverse
orientation, shading frames from per-vertex normals with face-forwarding).
GPU (marked): ilm_surface_interactions equals the oracle bit for bit on every
field, for closest hits of soups with and without per-vertex normals,
tangents and uvs, through host and device buffers."""
import numpy as np
import pytest

import oracle
from rs_illume_b200 import workloads as wl

TRI = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)


def test_known_answers_default_uv():
    si = oracle.surface_interaction(TRI, (0.25, 0.25, 1.0), (0.0, 0.0, -1.0))
    assert si is not None and si["kind"] == 1
    np.testing.assert_array_equal(si["p"], [0.25, 0.25, 0.0])
    assert si["t"] == 1.0
    np.testing.assert_array_equal(si["n"], [0, 0, 1])          # normalize((p0-p2) x (p1-p2))
    # default uvs (0,0), (1,0), (1,1); b = (0.5, 0.25, 0.25)
    np.testing.assert_allclose(si["uv"], [0.5, 0.25], rtol=1e-6)
    np.testing.assert_allclose(si["dpdu"], [1, 0, 0], atol=1e-7)
    np.testing.assert_allclose(si["dpdv"], [-1, 1, 0], atol=1e-7)
    # geometric shading frame (no per-vertex data)
    np.testing.assert_array_equal(si["shading_n"], si["n"])
    np.testing.assert_array_equal(si["shading_dpdu"], si["dpdu"])
    np.testing.assert_array_equal(si["wo"], [0, 0, 1])
    assert np.all(si["p_error"] >= 0) and np.all(si["p_error"] < 1e-6)
    assert oracle.surface_interaction(TRI, (2.0, 2.0, 1.0), (0.0, 0.0, -1.0)) is None


def test_reverse_orientation_and_shading_normals():
    si = oracle.surface_interaction(TRI, (0.25, 0.25, 1.0), (0.0, 0.0, -1.0), reverse=True)
    np.testing.assert_array_equal(si["n"], [0, 0, -1])
    nn = np.tile([0.0, 0.0, -1.0], (3, 1))
    si = oracle.surface_interaction(TRI, (0.25, 0.25, 1.0), (0.0, 0.0, -1.0), n=nn)
    # ns = (0,0,-1); ss = dpdu = (1,0,0); ts = ss x ns = (0,1,0); ss = ts x ns = (-1,0,0)
    np.testing.assert_allclose(si["shading_n"], [0, 0, -1], atol=1e-7)
    np.testing.assert_allclose(si["shading_dpdu"], [-1, 0, 0], atol=1e-7)
    np.testing.assert_allclose(si["shading_dpdv"], [0, 1, 0], atol=1e-7)
    np.testing.assert_array_equal(si["n"], [0, 0, -1])          # face-forwarded to the shading normal
    np.testing.assert_array_equal(si["shading_dndu"], [0, 0, 0])  # constant normals


def scene(seed, attrs):
    xyz, idx = wl.soup(seed, 2048, 0.05)
    nv = len(xyz)
    rng = np.random.default_rng(seed)
    extra = {}
    if attrs:
        n = rng.normal(size=(nv, 3)).astype(np.float32)
        n /= np.linalg.norm(n, axis=1, keepdims=True)
        extra = dict(n=n, s=rng.normal(size=(nv, 3)).astype(np.float32),
                     uv=rng.random((nv, 2)).astype(np.float32), reverse_orientation=seed % 2 == 1)
    rays = np.ascontiguousarray(np.concatenate([wl.camera_rays(48, 48, (0.5, 0.5, -1.5), 45.0),
                                                wl.ball_rays(seed, 4, 2048, 2048, 1.0, 0.1, 4.0)]))
    rays["o"][48 * 48:] += np.float32(0.5)
    return xyz, idx, rays, extra


def oracle_record(xyz, idx, prim, ray, extra):
    vi = idx[prim]
    kw = {}
    for k in ("n", "s", "uv"):
        if k in extra:
            kw[k] = extra[k][vi]
    return oracle.surface_interaction(xyz[vi], ray["o"], ray["d"], float("inf"), reverse=extra.get(
        "reverse_orientation", False), **kw)


FIELDS = ("p", "p_error", "n", "uv", "dpdu", "dpdv", "shading_n", "shading_dpdu", "shading_dpdv", "shading_dndu",
          "shading_dndv", "wo", "t")


@pytest.mark.gpu
@pytest.mark.parametrize("seed,attrs", [(21, False), (22, True), (23, True)])
def test_gpu_matches_oracle(ctx, seed, attrs):
    import torch
    import rs_illume_b200 as rb
    xyz, idx, rays, extra = scene(seed, attrs)
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx, **extra)], width=8)
    hits = acc.intersect_batch(rays)
    si = acc.surface_interactions(rays, hits)
    hit = hits["prim"] != rb.ILM_MISS
    assert hit.sum() > 500
    assert np.all(si["kind"][~hit] == 0)
    for i in np.nonzero(hit)[0]:
        want = oracle_record(xyz, idx, int(hits["prim"][i]), rays[i], extra)
        assert want is not None and si["kind"][i] == 1 and si["prim"][i] == hits["prim"][i]
        for f in FIELDS:
            assert np.array_equal(si[f][i], want[f]), (i, f, si[f][i], want[f])
    # device buffers, stream-ordered
    d_rays = torch.from_numpy(rays.view(np.uint8)).cuda()
    d_hits = torch.from_numpy(hits.view(np.uint8)).cuda()
    d_out = torch.empty(len(rays) * 176, dtype=torch.uint8, device="cuda")
    s = torch.cuda.Stream()
    acc.surface_interactions(d_rays, d_hits, d_out, stream=s)
    s.synchronize()
    assert d_out.cpu().numpy().tobytes() == si.tobytes()


@pytest.mark.gpu
def test_gpu_attrs_rules(ctx):
    import rs_illume_b200 as rb
    xyz, idx, _, _ = scene(24, False)
    m = rb.TriangleMesh(ctx, xyz, idx)
    rb.GpuBVHAccel(ctx, [m], width=8)
    import ctypes
    at = rb._lib.ilm_mesh_attrs(None, None, None, 1)
    # attributes are fixed once a build has used the mesh
    assert ctx._lib.ilm_mesh_set_attrs(ctx.handle, m.id, ctypes.byref(at)) == rb._lib.ILM_ERR_INVALID_ARGUMENT

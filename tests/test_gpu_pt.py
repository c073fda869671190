"""GPU wavefront path tracer vs the CPU path-tracing oracle (statistical parity).

Both sides are unbiased estimators of the same image with different random
streams, so parity is statistical, at equal spp:
  * relMSE(GPU, oracle) / relMSE(GPU seed a, GPU seed b) ~ 1: matching bias
    and matching noise (relMSE = mean (x - y)^2 / (y^2 + 0.01), eps 0.01);
  * per-channel image means agree within 5 standard errors;
  * 4x4-block means agree within 5 standard errors per block (few outliers);
  * rays per path agree within 3%.
"""
import numpy as np
import pytest

import oracle
import rs_illume_b200 as rb
from rs_illume_b200 import workloads as wl

pytestmark = pytest.mark.gpu

W = H = 64
SPP = 64
EPS = 0.01


def relmse(x, y):
    return float(np.mean((x - y) ** 2 / (y ** 2 + EPS)))


@pytest.fixture(scope="module")
def cornell_small():
    xyz, idx, mat, alb, emi = wl.cornell(4, 3)
    cam = wl.CORNELL_CAMERA
    sc = oracle.Scene(xyz, idx)
    o, (oc, osh) = oracle.render_pt(sc, xyz, idx, mat, alb, emi, cam["eye"], cam["fov_deg"], W, H, SPP, 8, 3, 3)
    ctx = rb.Context(0)
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx)], width=8)
    pt = rb.PathTracer(acc, mat, alb, emi, cam["eye"], cam["fov_deg"], W, H)
    yield pt, o, oc + osh
    ctx.close()


def test_gpu_pt_matches_oracle_statistically(cornell_small):
    pt, o, o_rays = cornell_small
    g1, s1 = pt.render(SPP, seed=3)
    g2, _ = pt.render(SPP, seed=4)
    assert np.all(np.isfinite(g1)) and g1.min() >= 0.0
    r_go, r_gg = relmse(g1, o), relmse(g1, g2)
    assert 0.75 < r_go / r_gg < 1.33, (r_go, r_gg)
    # image means
    npix = W * H
    se = (g1 - g2).reshape(-1, 3).std(axis=0) / np.sqrt(npix) * np.sqrt(1.0)
    diff = g1.reshape(-1, 3).mean(axis=0) - o.reshape(-1, 3).mean(axis=0)
    assert np.all(np.abs(diff) < 5 * se + 1e-6), (diff, se)
    # 4x4 block means
    def blocks(x):
        return x.reshape(H // 4, 4, W // 4, 4, 3).mean(axis=(1, 3))
    dg = blocks(g1) - blocks(o)
    sb = np.sqrt(blocks((g1 - g2) ** 2) / 2.0 / 16.0) + 1e-4    # per-block std of one render's block mean
    z = np.abs(dg) / (np.sqrt(2.0) * sb)
    assert np.mean(z > 5.0) < 0.01
    # the light is seen directly at its emitted radiance on the camera segment
    assert g1[:8, 24:40].max() == pytest.approx(15.0, rel=1e-5)
    # work per path matches the oracle's (same estimator, same termination rule)
    g_rays = s1["closest_rays"] + s1["shadow_rays"]
    assert abs(g_rays / o_rays - 1.0) < 0.03


def test_graph_replay_equals_eager_launches(cornell_small):
    pt, _, _ = cornell_small
    a, sa = pt.render(16, seed=9, use_graphs=True)
    b, sb = pt.render(16, seed=9, use_graphs=False)
    # same random numbers; only the order of the film's float atomics differs
    np.testing.assert_allclose(a, b, rtol=2e-5, atol=2e-6)
    assert sa["closest_rays"] == sb["closest_rays"] and sa["shadow_rays"] == sb["shadow_rays"]


def test_waves_do_not_change_the_image(cornell_small):
    pt, _, _ = cornell_small
    a, sa = pt.render(16, seed=11, wave_paths=1 << 20)
    b, sb = pt.render(16, seed=11, wave_paths=W * H * 3 + 17)     # uneven waves
    assert sb["waves"] > sa["waves"]
    np.testing.assert_allclose(a, b, rtol=2e-5, atol=2e-6)


def test_gpu_pt_converges(cornell_small):
    pt, _, _ = cornell_small
    lo1, _ = pt.render(16, seed=1)
    lo2, _ = pt.render(16, seed=2)
    hi, _ = pt.render(256, seed=3)
    # 16x the samples: relMSE against a 256-spp image falls roughly with spp
    assert relmse(lo1, hi) < 1.5 * relmse(lo1, lo2)
    assert relmse(hi, lo1) > 0.0


def test_render_rejects_bad_options(cornell_small):
    pt, _, _ = cornell_small
    with pytest.raises(rb.IllumeError):
        pt.render(10)          # not a perfect square
    with pytest.raises(rb.IllumeError):
        pt.render(16, max_depth=0)


def test_render_written_as_pfm(cornell_small, tmp_path):
    from rs_illume_b200 import image
    pt, _, _ = cornell_small
    img, _ = pt.render(4, seed=2)
    p = str(tmp_path / "frame.pfm")
    image.write_pfm(p, img)
    assert image.read_pfm(p).tobytes() == img.tobytes()


def test_filtered_film_matches_oracle_statistically():
    """Gaussian film filter (radius 1.5, alpha 2): GPU splats every path
    contribution through the 16x16 table, the oracle splats each sample."""
    from rs_illume_b200 import image
    xyz, idx, mat, alb, emi = wl.cornell(4, 3)
    cam = wl.CORNELL_CAMERA
    w = h = 32
    f = image.filter_desc("gaussian", (1.5, 1.5), 2.0)
    sc = oracle.Scene(xyz, idx)
    o, _ = oracle.render_pt_filtered(sc, xyz, idx, mat, alb, emi, cam["eye"], cam["fov_deg"], w, h, 64,
                                     image.filter_table(f), (1.5, 1.5), seed=3)
    ctx = rb.Context(0)
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx)], width=8)
    pt = rb.PathTracer(acc, mat, alb, emi, cam["eye"], cam["fov_deg"], w, h)
    g1, _ = pt.render(64, seed=3, filter=f)
    g2, _ = pt.render(64, seed=4, filter=f)
    assert np.all(np.isfinite(g1)) and g1.min() >= 0.0
    r_go, r_gg = relmse(g1, o), relmse(g1, g2)
    assert 0.7 < r_go / r_gg < 1.4, (r_go, r_gg)
    se = (g1 - g2).reshape(-1, 3).std(axis=0) / np.sqrt(w * h)
    diff = g1.reshape(-1, 3).mean(axis=0) - o.reshape(-1, 3).mean(axis=0)
    assert np.all(np.abs(diff) < 5 * se + 1e-6), (diff, se)
    # a box of radius 0.5 through the general splat path equals the default film
    b, _ = pt.render(16, seed=9, filter=image.filter_desc("box", (0.5, 0.5)))
    b_general, _ = pt.render(16, seed=9, filter=image.filter_desc("triangle", (0.5, 0.5)))
    d, _ = pt.render(16, seed=9)
    np.testing.assert_allclose(b, d, rtol=1e-5, atol=1e-6)
    assert np.all(np.isfinite(b_general))
    ctx.close()


def test_full_frame_matches_oracle_centre_tile():
    """The path-tracer workload as measured: Cornell box with the level-6
    icosphere (81,920 + 34 triangles), 1024x1024, 64 spp, depth 8, Russian
    roulette from depth 3.  The GPU renders the whole frame twice (two seeds);
    the oracle renders its 256x256 centre tile, the sample of the frame that
    the CPU baseline times.  Statistical parity on the tile as above."""
    xyz, idx, mat, alb, emi = wl.cornell(6, 3)
    cam = wl.CORNELL_CAMERA
    ctx = rb.Context(0)
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx)], width=8)
    pt = rb.PathTracer(acc, mat, alb, emi, cam["eye"], cam["fov_deg"], 1024, 1024)
    g1, _ = pt.render(64, seed=21)
    g2, _ = pt.render(64, seed=22)
    ctx.close()
    sc = oracle.Scene(xyz, idx)
    o, _ = oracle.render_pt(sc, xyz, idx, mat, alb, emi, cam["eye"], cam["fov_deg"], 1024, 1024, 64, 8, 3, 3,
                            window=(384, 384, 640, 640), threads=0)
    t1, t2 = g1[384:640, 384:640], g2[384:640, 384:640]
    assert np.all(np.isfinite(g1)) and g1.min() >= 0.0
    r_go, r_gg = relmse(t1, o), relmse(t1, t2)
    assert 0.75 < r_go / r_gg < 1.33, (r_go, r_gg)
    se = (t1 - t2).reshape(-1, 3).std(axis=0) / np.sqrt(t1.size // 3)
    diff = t1.reshape(-1, 3).mean(axis=0) - o.reshape(-1, 3).mean(axis=0)
    assert np.all(np.abs(diff) < 5 * se + 1e-6), (diff, se)

    def blocks(x):
        return x.reshape(256 // 8, 8, 256 // 8, 8, 3).mean(axis=(1, 3))
    dg = blocks(t1) - blocks(o)
    sb = np.sqrt(blocks((t1 - t2) ** 2) / 2.0 / 64.0) + 1e-4
    z = np.abs(dg) / (np.sqrt(2.0) * sb)
    assert np.mean(z > 5.0) < 0.01

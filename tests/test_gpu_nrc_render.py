"""Path tracing with the radiance cache (ilm_render_nrc) on the Cornell box.

* With the cache never queried (spread threshold out of reach) and training
  off, the estimator is the plain path tracer: same random streams, same
  image up to the order of the film's float atomics, same ray counts.
* With training on, queries and training samples flow, and a network trained
  online on the path tracer's own training paths renders far closer to the
  reference than an untrained one.
* Against a plain-tracer reference (its own noise removed), a 1-spp frame of
  the cache renderer has lower relMSE than the plain tracer at equal device
  time (the gain is printed); relMSE = mean (x - y)^2 / (y^2 + 0.01).
"""
import numpy as np
import pytest

import rs_illume_b200 as rb
from rs_illume_b200 import workloads as wl
from rs_illume_b200.nrc import RadianceCache

pytestmark = pytest.mark.gpu

EPS = 0.01


def relmse(x, y):
    return float(np.mean((x - y) ** 2 / (y ** 2 + EPS)))


def make_tracer(ctx, w, h):
    xyz, idx, mat, alb, emi = wl.cornell(6, 3)
    cam = wl.CORNELL_CAMERA
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx)], width=8)
    return rb.PathTracer(acc, mat, alb, emi, cam["eye"], cam["fov_deg"], w, h), acc.world_bound()


@pytest.fixture(scope="module")
def tracer64():
    ctx = rb.Context(0)
    pt, bound = make_tracer(ctx, 64, 64)
    yield pt, bound, ctx
    ctx.close()


def test_without_queries_equals_plain_tracer(tracer64):
    pt, bound, ctx = tracer64
    cache = RadianceCache(ctx, bound)
    a, sa = pt.render_nrc(cache, frames=1, spp_per_frame=4, seed=5, spread_c=1e30, train=False)
    b, sb = pt.render(4, seed=5)
    assert sa["queries"] == 0
    np.testing.assert_allclose(a, b, rtol=2e-5, atol=2e-6)
    assert sa["closest_rays"] == sb["closest_rays"] and sa["shadow_rays"] == sb["shadow_rays"]
    cache.close()


def test_training_makes_the_cache_useful(tracer64):
    pt, bound, ctx = tracer64
    ref, _ = pt.render(4096, seed=1)
    trained = RadianceCache(ctx, bound, seed=4)
    img, st = pt.render_nrc(trained, frames=96, spp_per_frame=4, seed=7)
    assert np.all(np.isfinite(img)) and img.min() >= 0.0
    assert st["frames"] == 96
    assert st["queries"] > 0 and st["train_samples"] > 0
    assert np.isfinite(st["last_loss"])
    # the light is still seen directly on the camera segment
    assert img[:8, 24:40].max() == pytest.approx(15.0, rel=1e-5)
    # the same inference-only render with the trained and with an untrained network
    fresh = RadianceCache(ctx, bound, seed=4)
    a, _ = pt.render_nrc(trained, frames=16, spp_per_frame=4, seed=8, train=False)
    b, _ = pt.render_nrc(fresh, frames=16, spp_per_frame=4, seed=8, train=False)
    r_trained, r_fresh = relmse(a, ref), relmse(b, ref)
    assert r_trained < 0.5 * r_fresh, (r_trained, r_fresh)
    trained.close()
    fresh.close()


def test_time_budget_stops_the_render(tracer64):
    pt, bound, ctx = tracer64
    cache = RadianceCache(ctx, bound)
    _, st = pt.render_nrc(cache, frames=0, spp_per_frame=4, time_budget_s=0.05)
    assert st["frames"] >= 1 and st["seconds"] >= 0.05
    cache.close()


def test_equal_time_relmse_beats_plain_tracer():
    """Real-time setting at the benchmark resolution: 1-spp frames, the cache
    trained online over earlier frames; each frame's relMSE against an
    equal-time plain render (relMSE * spp is constant for the unbiased plain
    tracer, so its equal-time relMSE is relMSE(1 spp) * t_spp / t_frame)."""
    ctx = rb.Context(0)
    res = 1024
    pt, bound = make_tracer(ctx, res, res)
    ra, _ = pt.render(1024, seed=1)
    rb_, _ = pt.render(1024, seed=2)
    ref = 0.5 * (ra + rb_)
    var_ref = ((ra - rb_) / 2) ** 2

    def rel(x):    # the reference's own noise removed
        return float(np.mean(((x - ref) ** 2 - var_ref) / (ref ** 2 + EPS)))

    pt.render(16, seed=3)
    _, sp = pt.render(16, seed=4)
    t_spp = sp["seconds"] / 16
    r1 = np.mean([rel(pt.render(1, seed=10 + k)[0]) for k in range(4)])
    gains = []
    for rep in range(3):          # independent runs: a fresh cache each
        cache = RadianceCache(ctx, bound, seed=4 + rep)
        pt.render_nrc(cache, frames=200, seed=9 + 1000 * rep)      # online training over earlier frames
        rs, ts = [], []
        for k in range(6):
            img, st = pt.render_nrc(cache, frames=1, seed=100 + 1000 * rep + k)
            assert np.all(np.isfinite(img))
            rs.append(rel(img))
            ts.append(st["seconds"])
        cache.close()
        r_nrc, t_frame = float(np.mean(rs)), float(np.median(ts))
        gains.append(r1 * t_spp / t_frame / r_nrc)
    print(f"\nplain {t_spp * 1e3:.2f} ms/spp, relMSE(1 spp) {r1:.4f}; equal-time gains {np.round(gains, 3)}")
    # at least 2x lower relMSE than the plain tracer at
    # equal time, on average over the runs (measured 3.4-3.6 after 200 frames
    # on B200 with the default settings: spread threshold 0.003, 2 Adam steps
    # of 32,768 rows, weight decay 1; the bench measures after 800 frames,
    # where the gain has settled lower, 2.27-2.38)
    assert np.mean(gains) > 2.0, gains
    ctx.close()

"""CPU checks of the path-tracing oracle (oracle/pt.cpp).

The reference has no path integrator to compare with, so the restatement is
pinned physically: direct lighting of a Lambertian wall by a one-sided
rectangular emitter must equal albedo/pi * E, with the irradiance E integrated
numerically, and a closed furnace-like setup must conserve energy.
"""
import numpy as np
import pytest

import oracle
from rs_illume_b200 import workloads as wl

EYE = (0.0, 0.0, -1.0)


def quad(a, b, c, d):
    return [a, b, c, d], [(0, 1, 2), (0, 2, 3)]


def wall_and_light(albedo=0.8, le=5.0):
    # wall z = 1 facing the camera; light x in [0.3, 0.5], y in [-0.1, 0.1] at z = 0.5,
    # emitting towards +z: (p0-p2)x(p1-p2) must be +z
    wv, wt = quad((-2, -2, 1), (2, -2, 1), (2, 2, 1), (-2, 2, 1))
    lv, lt = quad((0.3, -0.1, 0.5), (0.5, -0.1, 0.5), (0.5, 0.1, 0.5), (0.3, 0.1, 0.5))
    p0, p1, p2 = (np.array(lv[i], float) for i in lt[0])
    n = np.cross(p0 - p2, p1 - p2)
    assert n[2] > 0
    xyz = np.array(wv + lv, np.float32)
    idx = np.array(wt + [(a + 4, b + 4, c + 4) for a, b, c in lt], np.uint32)
    mat = np.array([0, 0, 1, 1], np.uint32)
    alb = np.array([[albedo] * 3, [0, 0, 0]], np.float32)
    emi = np.array([[0, 0, 0], [le] * 3], np.float32)
    return xyz, idx, mat, alb, emi


def irradiance_at_origin_of_wall(le, n=1500):
    # E = Le * integral cos_wall cos_light / r^2 dA over the light, point (0,0,1)
    xs = 0.3 + (np.arange(n) + 0.5) * 0.2 / n
    ys = -0.1 + (np.arange(n) + 0.5) * 0.2 / n
    X, Y = np.meshgrid(xs, ys)
    r2 = X ** 2 + Y ** 2 + 0.25
    integrand = 0.25 / r2 ** 2
    return le * integrand.sum() * (0.2 / n) ** 2


def test_direct_lighting_matches_numerical_irradiance():
    xyz, idx, mat, alb, emi = wall_and_light()
    sc = oracle.Scene(xyz, idx)
    w = 65   # odd: the centre pixel's centre looks exactly at (0, 0, 1)
    img, _ = oracle.render_pt(sc, xyz, idx, mat, alb, emi, EYE, 40.0, w, w, 16384, max_depth=1, rr_depth=3,
                              seed=1, window=(32, 32, 33, 33))
    want = 0.8 / np.pi * irradiance_at_origin_of_wall(5.0)
    got = img[0, 0]
    assert np.allclose(got, got[0])
    assert got[0] == pytest.approx(want, rel=0.02)


def test_mis_halves_are_unbiased_both_ways():
    # the same pixel with max_depth 1 at two seeds agrees within noise, and a
    # brighter emitter scales the result linearly
    xyz, idx, mat, alb, emi = wall_and_light()
    sc = oracle.Scene(xyz, idx)
    a, _ = oracle.render_pt(sc, xyz, idx, mat, alb, emi, EYE, 40.0, 65, 65, 4096, 1, 3, 2, (30, 30, 35, 35))
    emi2 = emi * 3.0
    b, _ = oracle.render_pt(sc, xyz, idx, mat, alb, emi2, EYE, 40.0, 65, 65, 4096, 1, 3, 2, (30, 30, 35, 35))
    np.testing.assert_allclose(b, 3.0 * a, rtol=1e-5)


def test_cornell_render_properties():
    from rs_illume_b200 import workloads as wl
    xyz, idx, mat, alb, emi = wl.cornell(3, 3)
    sc = oracle.Scene(xyz, idx)
    img, (nc, ns) = oracle.render_pt(sc, xyz, idx, mat, alb, emi, wl.CORNELL_CAMERA["eye"],
                                     wl.CORNELL_CAMERA["fov_deg"], 32, 32, 16)
    assert np.all(np.isfinite(img)) and img.min() >= 0.0
    # the light is visible at the top centre at its emitted radiance
    assert img[:6, 12:20].max() == pytest.approx(15.0, rel=1e-6)
    # red wall on the left, green wall on the right
    left, right = img[8:24, 1:4].mean(axis=(0, 1)), img[8:24, 28:31].mean(axis=(0, 1))
    assert left[0] > 2 * left[1] and right[1] > 2 * right[0]
    assert nc > 32 * 32 * 16 and ns > 0


def test_filtered_film_box_equals_pixel_mean():
    """A box of radius 0.5 through the filtered film is the per-pixel mean."""
    import numpy as np
    from rs_illume_b200 import image
    xyz, idx, mat, alb, emi = wl.cornell(2, 3)
    cam = wl.CORNELL_CAMERA
    sc = oracle.Scene(xyz, idx)
    plain, _ = oracle.render_pt(sc, xyz, idx, mat, alb, emi, cam["eye"], cam["fov_deg"], 12, 12, 4, 8, 3, 5)
    table = image.filter_table(image.filter_desc("box", (0.5, 0.5)))
    filt, _ = oracle.render_pt_filtered(sc, xyz, idx, mat, alb, emi, cam["eye"], cam["fov_deg"], 12, 12, 4, table,
                                        (0.5, 0.5), seed=5)
    np.testing.assert_allclose(filt, plain, rtol=1e-6, atol=1e-7)


def test_filtered_film_gaussian_is_smoother():
    import numpy as np
    from rs_illume_b200 import image
    xyz, idx, mat, alb, emi = wl.cornell(2, 3)
    cam = wl.CORNELL_CAMERA
    sc = oracle.Scene(xyz, idx)
    box, _ = oracle.render_pt(sc, xyz, idx, mat, alb, emi, cam["eye"], cam["fov_deg"], 16, 16, 4, 8, 3, 5)
    f = image.filter_desc("gaussian", (1.5, 1.5), 2.0)
    g, _ = oracle.render_pt_filtered(sc, xyz, idx, mat, alb, emi, cam["eye"], cam["fov_deg"], 16, 16, 4,
                                     image.filter_table(f), (1.5, 1.5), seed=5)
    assert np.all(np.isfinite(g)) and g.min() >= 0
    # same mean radiance, less pixel-to-pixel variation
    assert abs(g.mean() / box.mean() - 1) < 0.05
    assert np.abs(np.diff(g, axis=1)).mean() < np.abs(np.diff(box, axis=1)).mean()

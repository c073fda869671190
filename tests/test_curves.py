"""Curves (shapes/curve.rs): cubic Bezier segments of flat, cylinder and
ribbon type beside triangles and quadrics in one BVH or kd-tree.

CPU: the oracle's restatement against known answers (a straight curve of
constant and of tapered width, end caps, ribbons seen edge-on) and against
float64 geometry on curved segments: a hit lies within half the local width
(plus the refinement's flatness tolerance) of the curve point at its u, and
rays through curve points hit.  GPU (marked): ids, t, u, v and any-hit flags
of the B200 kernels against the oracle, every layout."""
import ctypes

import numpy as np
import pytest

import oracle
from rs_illume_b200 import _lib

STRAIGHT = [[0, 0, 0], [1, 0, 0], [2, 0, 0], [3, 0, 0]]


def bez(u, P):
    P = np.asarray(P, np.float64)
    return (1 - u) ** 3 * P[0] + 3 * (1 - u) ** 2 * u * P[1] + 3 * (1 - u) * u * u * P[2] + u ** 3 * P[3]


def test_straight_curve_known_answers():
    d = oracle.curve_desc(STRAIGHT, (0.2, 0.2))
    t, u, v = oracle.curve_intersect(d, (1.5, 0.05, 5.0), (0.0, 0.0, -1.0))
    assert t == pytest.approx(5.0, rel=1e-6) and u == pytest.approx(0.5) and v == pytest.approx(0.25)
    t, u, v = oracle.curve_intersect(d, (1.5, -0.05, 5.0), (0.0, 0.0, -1.0))
    assert v == pytest.approx(0.75)
    assert oracle.curve_intersect(d, (1.5, 0.11, 5.0), (0.0, 0.0, -1.0)) is None      # outside the half width
    assert oracle.curve_intersect(d, (-0.05, 0.0, 5.0), (0.0, 0.0, -1.0)) is None     # before the start cap
    assert oracle.curve_intersect(d, (3.05, 0.0, 5.0), (0.0, 0.0, -1.0)) is None      # past the end cap
    assert oracle.curve_intersect(d, (1.5, 0.0, 5.0), (0.0, 0.0, -1.0), tmax=4.0) is None
    # a segment covers only its u range; u stays global
    seg = oracle.curve_desc(STRAIGHT, (0.2, 0.2), u_range=(0.5, 0.75))
    assert oracle.curve_intersect(seg, (1.0, 0.0, 5.0), (0.0, 0.0, -1.0)) is None
    t, u, v = oracle.curve_intersect(seg, (1.8, 0.0, 5.0), (0.0, 0.0, -1.0))
    assert u == pytest.approx(0.6, abs=1e-6)
    # a tapered curve: half width 0.05 at u = 0, 0.25 at u = 1
    tap = oracle.curve_desc(STRAIGHT, (0.1, 0.5))
    assert oracle.curve_intersect(tap, (0.3, 0.1, 5.0), (0.0, 0.0, -1.0)) is None     # half width 0.07 at u 0.1
    assert oracle.curve_intersect(tap, (2.7, 0.2, 5.0), (0.0, 0.0, -1.0)) is not None  # half width 0.23 at u 0.9


def test_ribbon_width_follows_its_normal():
    n = [[0, 0, 1], [0, 0, 1]]
    rib = oracle.curve_desc(STRAIGHT, (0.2, 0.2), curve_type=2, normals=n)
    # seen along its normal: full width
    assert oracle.curve_intersect(rib, (1.5, 0.09, 5.0), (0.0, 0.0, -1.0)) is not None
    # seen at 60 degrees from the normal: half the width
    d = np.array([0.0, np.sin(np.radians(60)), -np.cos(np.radians(60))])
    o = np.array([1.5, 0.0, 0.0]) - 5.0 * d
    assert oracle.curve_intersect(rib, o + [0, 0, 0.04], d) is not None
    assert oracle.curve_intersect(rib, o + [0, 0, 0.06 / np.cos(np.radians(60)) * 0.5 + 0.03], d) is None
    # the normal turning along the curve
    twist = oracle.curve_desc(STRAIGHT, (0.2, 0.2), curve_type=2, normals=[[0, 0, 1], [0, 1, 0]])
    assert oracle.curve_intersect(twist, (0.3, 0.09, 5.0), (0.0, 0.0, -1.0)) is not None
    assert oracle.curve_intersect(twist, (2.7, 0.09, 5.0), (0.0, 0.0, -1.0)) is None


def random_curve(rng):
    cp = rng.uniform(-1, 1, (4, 3))
    w = rng.uniform(0.02, 0.15, 2)
    return cp, w


def test_curved_segments_against_float64():
    rng = np.random.default_rng(3)
    checked = hits = 0
    for _ in range(60):
        cp, w = random_curve(rng)
        d = oracle.curve_desc(cp, tuple(w))
        for _ in range(20):
            u0 = rng.uniform(0.05, 0.95)
            target = bez(u0, cp)
            dirn = rng.normal(size=3)
            dirn /= np.linalg.norm(dirn)
            o = target - 3.0 * dirn
            r = oracle.curve_intersect(d, o, dirn)
            checked += 1
            if r is None:
                continue
            hits += 1
            t, u, v = r
            p = o + t * dirn
            local_w = (1 - u) * w[0] + u * w[1]
            # the refinement flattens the curve to within width / 20
            assert np.linalg.norm(p - bez(u, cp)) <= 0.5 * local_w * 1.6 + 0.05 * max(w) + 1e-4
            assert 0.0 <= u <= 1.0 and -1e-3 <= v <= 1.0 + 1e-3
    # rays through curve points hit unless the curve bends back in front
    assert checked == 1200 and hits > 0.85 * checked, hits


def gpu_desc(od):
    g = _lib.ilm_curve_desc()
    ctypes.memmove(ctypes.addressof(g), ctypes.addressof(od), ctypes.sizeof(g))
    return g


def curve_scene(seed):
    rng = np.random.default_rng(seed)
    from rs_illume_b200 import workloads as wl
    xyz, idx = wl.soup(seed, 300, 0.2)
    xyz = (xyz - 0.5) * 3.0
    curves = []
    for k in range(40):
        cp, w = random_curve(rng)
        cp = cp * 0.8 + rng.uniform(-1.2, 1.2, 3)
        typ = k % 3
        nrm = rng.normal(size=(2, 3)) if typ == 2 else None
        m = np.eye(4)
        m[:3, :3] *= rng.uniform(0.7, 1.3)
        for s in range(4):   # split depth 2
            curves.append(oracle.curve_desc(cp, tuple(w), m, typ, nrm, (s / 4, (s + 1) / 4)))
    quads = [oracle.sphere_desc(0.3, tuple(rng.uniform(-1, 1, 3))) for _ in range(6)]
    return xyz.astype(np.float32), idx, quads, curves


@pytest.mark.gpu
@pytest.mark.parametrize("layout", [2, 4, 8, "kd"])
def test_gpu_curves_match_oracle(ctx, layout):
    import rs_illume_b200 as rb
    from rs_illume_b200 import workloads as wl
    from tests.test_kdtree import compare
    xyz, idx, quads, curves = curve_scene(41)
    sc = oracle.Scene(xyz, idx, quads, curves=curves)
    gq = []
    for q in quads:
        g = _lib.ilm_sphere_desc()
        ctypes.memmove(ctypes.addressof(g), ctypes.addressof(q), ctypes.sizeof(g))
        gq.append(g)
    shapes = [rb.TriangleMesh(ctx, xyz, idx), rb.Spheres(ctx, gq), rb.Curves(ctx, [gpu_desc(c) for c in curves])]
    acc = rb.GpuKdTreeAccel(ctx, shapes) if layout == "kd" else rb.GpuBVHAccel(ctx, shapes, width=layout)
    rays = wl.ball_rays(9, 0, 1 << 17, 1 << 17, 2.5, 0.05, 4.0)
    want = sc.intersect(rays)
    got = acc.intersect_batch(rays)
    n_tq = len(idx) + len(quads)
    assert np.sum((want["prim"] >= n_tq) & (want["prim"] != 0xFFFFFFFF)) > 500
    assert compare(got, want, f"curves {layout}", tol_uv=1e-5) <= 1e-3 * len(rays)
    assert np.array_equal(acc.intersect_p_batch(rays).astype(np.uint8), sc.intersect_p(rays))
    wb = acc.world_bound()
    np.testing.assert_array_equal(np.concatenate([wb.min, wb.max]), sc.world_bound())


def test_scene_file_curves():
    import rs_illume_b200 as rb
    sf = rb.SceneFile.parse('''WorldBegin Translate 0 0 2
        Shape "curve" "point P" [0 0 0 1 1 0 2 -1 0 3 0 0] "float width0" 0.2 "float width1" 0.1
        Shape "curve" "point P" [0 0 0 1 1 0 2 -1 0 3 0 0] "string type" "ribbon"
              "normal N" [0 0 1 0 1 0] "integer splitdepth" 1
        Shape "curve" "point P" [0 0 0 1 1 0 2 -1 0 3 0 0] "normal N" [0 0 1 0 1 0] "integer splitdepth" 0
        WorldEnd''')
    c, mat = sf.curves()
    assert sf.info.n_curves == 8 + 2 + 1 and len(c) == 11 and len(mat) == 11
    assert [(s.u_min, s.u_max) for s in c[:8]] == [(k / 8, (k + 1) / 8) for k in range(8)]
    assert tuple(c[0].width) == (pytest.approx(0.2), pytest.approx(0.1)) and c[0].type == 0
    assert c[8].type == 2 and list(c[8].n) == [0, 0, 1, 0, 1, 0]
    assert c[0].object_to_world[11] == 2.0 and c[0].world_to_object[11] == -2.0
    assert any("only used with ribbon" in w for w in sf.warnings)
    with pytest.raises(rb.IllumeError, match="two normals"):
        rb.SceneFile.parse('Shape "curve" "point P" [0 0 0 1 1 0 2 -1 0 3 0 0] "string type" "ribbon"')
    with pytest.raises(rb.IllumeError, match="4 control points"):
        rb.SceneFile.parse('Shape "curve" "point P" [0 0 0 1 1 0 2 -1 0]')


@pytest.mark.gpu
def test_gpu_scene_file_curves_answer_as_direct(ctx):
    import rs_illume_b200 as rb
    from rs_illume_b200 import workloads as wl
    sf = rb.SceneFile.parse('''WorldBegin
        Shape "curve" "point P" [-1 0 0 -0.3 1 0.2 0.3 -1 -0.2 1 0 0] "float width0" 0.2 "float width1" 0.05
        Shape "curve" "point P" [-1 0.5 0 0 0.5 1 0 0.5 -1 1 0.5 0] "string type" "ribbon"
              "normal N" [0 1 0 0 0 1] "float width" 0.15
        WorldEnd''')
    acc, pt = sf.build(ctx)
    assert pt is None
    c, _ = sf.curves()
    direct = rb.GpuBVHAccel(ctx, [rb.Curves(ctx, c)], width=8)
    rays = wl.ball_rays(12, 0, 1 << 16, 1 << 16, 2.0, 0.0, 4.0)
    got = acc.intersect_batch(rays)
    assert got.tobytes() == direct.intersect_batch(rays).tobytes()
    assert np.sum(got["prim"] != 0xFFFFFFFF) > 100

"""Known-answer tests pinning the C++ oracle.

The reference has no tests or golden vectors for this path (and cannot be
compiled here), so the oracle is pinned to (1) hand-derived cases with exact
answers, (2) a second, vectorised numpy restatement of the watertight triangle
test written directly from shapes/triangle.rs:156-262, compared bit for bit on
random cases, and (3) the constants of core/pbrt.rs and core/rng.rs.
"""
import math

import numpy as np
import pytest

import oracle

INF = float("inf")


# --------------------------------------------------------------- constants
def test_gamma_matches_formula_and_device_literals():
    eps = np.float32(np.finfo(np.float32).eps) * np.float32(0.5)
    for n in (1, 2, 3, 5, 7):
        nf = np.float32(n)
        want = (nf * eps) / (np.float32(1) - nf * eps)
        assert np.float32(oracle.gamma(n)) == want
    # the literals hard-coded in rs_illume_b200/csrc/shapes.cuh
    assert oracle.gamma(2) == float.fromhex("0x1.000002p-23")
    assert oracle.gamma(3) == float.fromhex("0x1.800004p-23")
    assert oracle.gamma(5) == float.fromhex("0x1.400006p-22")
    robust = np.float32(1) + np.float32(2) * np.float32(oracle.gamma(3))
    assert float(robust) == float.fromhex("0x1.000006p+0")


def test_next_float():
    lib = oracle.load()
    assert lib.orc_next_float_up(1.0) == np.nextafter(np.float32(1), np.float32(2))
    assert lib.orc_next_float_down(1.0) == np.nextafter(np.float32(1), np.float32(0))
    # both zeros step to the smallest denormal of the right sign (pbrt.rs:129-169)
    assert lib.orc_next_float_up(-0.0) == np.float32(1.4e-45)
    assert lib.orc_next_float_down(0.0) == -np.float32(1.4e-45)
    assert lib.orc_next_float_up(INF) == INF
    assert lib.orc_next_float_down(-INF) == -INF


def test_pcg32_stream_and_float_mapping():
    u = oracle.rng_u32(0, 4)
    f = oracle.rng_floats(0, 4)
    # uniform_float = min(u32 * 2^-32, 1 - 2^-24) (rng.rs:60-63)
    assert np.array_equal(f, np.minimum(u.astype(np.float32) * np.float32(2.0 ** -32), np.float32(1 - 2 ** -24)))
    # PCG32 recurrence re-derived in Python (rng.rs:30-49)
    M = 0x5851f42d4c957f2d
    mask = (1 << 64) - 1

    def pcg(seq, n):
        state, inc = 0, ((seq << 1) | 1) & mask
        out = []

        def step():
            nonlocal state
            old = state
            state = (old * M + inc) & mask
            xs = (((old >> 18) ^ old) >> 27) & 0xFFFFFFFF
            rot = old >> 59
            return ((xs >> rot) | (xs << ((-rot) & 31))) & 0xFFFFFFFF

        step()
        state = (state + 0x853c49e6748fea9b) & mask
        step()
        for _ in range(n):
            out.append(step())
        return out

    for seq in (0, 1, 2, 12345):
        assert list(oracle.rng_u32(seq, 16)) == pcg(seq, 16)


def test_pcg32_advance_repaired():
    # D18: advance(k) followed by draws equals the stream shifted by k.
    base = oracle.rng_floats(5, 300)
    for k in (1, 2, 3, 64, 199):
        assert np.array_equal(oracle.rng_floats(5, 50, advance=k), base[k:k + 50])


# --------------------------------------------------------------- triangle KATs
P0, P1, P2 = (0, 0, 5), (1, 0, 5), (0, 1, 5)


def tri(o, d, tmax=INF, pts=(P0, P1, P2), closest=True):
    return oracle.triangle_intersect(*pts, o, d, tmax, closest)


def test_triangle_interior_exact():
    assert tri((0.25, 0.25, 0), (0, 0, 1)) == (5.0, 0.5, 0.25, 0.25)


def test_triangle_backface_hits():
    r = tri((0.25, 0.25, 0), (0, 0, 1), pts=(P0, P2, P1))
    assert r == (5.0, 0.5, 0.25, 0.25)


def test_triangle_tmax_cut():
    assert tri((0.25, 0.25, 0), (0, 0, 1), tmax=4.999) is None
    assert tri((0.25, 0.25, 0), (0, 0, 1), tmax=5.0) is not None   # t_scaled > t_max*det is strict


def test_triangle_behind_and_on_plane_miss():
    assert tri((0.25, 0.25, 10), (0, 0, 1)) is None
    assert tri((0.25, 0.25, 5), (0, 0, 1)) is None       # t = 0 fails t > delta_t
    assert tri((0.6, 0.6, 0), (0, 0, 1)) is None         # outside


def test_triangle_watertight_shared_edge_and_vertex():
    # a ray through the shared edge p1-p2 hits both triangles of the quad
    q = ((1, 0, 5), (1, 1, 5), (0, 1, 5))
    a = tri((0.5, 0.5, 0), (0, 0, 1))
    b = tri((0.5, 0.5, 0), (0, 0, 1), pts=q)
    assert a is not None and b is not None
    assert a[0] == 5.0 and a[1] == 0.0
    # through a vertex
    v = tri((0, 0, 0), (0, 0, 1))
    assert v == (5.0, 1.0, 0.0, 0.0)


def test_triangle_parallel_ray_misses():
    assert tri((-1, 0.25, 5), (1, 0, 0)) is None


def test_ray_in_bounding_plane_finds_edge_hit():
    # D26: the triangle's edge (0,0,5)-(0,1,6) lies in the plane x = 0, which is
    # also its bounding box's min-x plane.  A ray with d.x = 0 travelling in that
    # plane makes the slab distance (0 - 0) * inf = NaN; the reference's box
    # test would reject the box, although the watertight test accepts the edge hit.
    xyz = np.array([[0, 0, 5], [1, 0, 5], [0, 1, 6]], np.float32)
    idx = np.array([[0, 1, 2]], np.uint32)
    sc = oracle.Scene(xyz, idx)
    r = np.zeros(1, oracle.RAY_DTYPE)
    r["o"][0] = (0.0, 0.25, 0.0)
    r["d"][0] = (0.0, 0.0, 1.0)
    r["tmax"][0] = np.inf
    direct = oracle.triangle_intersect(*xyz, (0.0, 0.25, 0.0), (0.0, 0.0, 1.0))
    assert direct is not None and direct[0] == 5.25 and direct[2] == 0.0
    h = sc.intersect(r)[0]
    assert h["prim"] == 0 and h["t"] == 5.25
    assert sc.intersect_p(r)[0] == 1


# numpy restatement of the watertight test (triangle.rs:156-262)
def watertight_np(p0, p1, p2, o, d, tmax):
    f = np.float32
    g = [oracle.gamma(n) for n in range(8)]
    g = [f(x) for x in g]
    n = len(o)
    ad = np.abs(d)
    kz = np.where(ad[:, 0] > ad[:, 1], np.where(ad[:, 0] > ad[:, 2], 0, 2), np.where(ad[:, 1] > ad[:, 2], 1, 2))
    kx = (kz + 1) % 3
    ky = (kx + 1) % 3
    rows = np.arange(n)

    def perm(v):
        return v[rows, kx], v[rows, ky], v[rows, kz]

    a = perm(p0 - o)
    b = perm(p1 - o)
    c = perm(p2 - o)
    dx, dy, dz = perm(d)
    with np.errstate(all="ignore"):
        sx = -dx / dz
        sy = -dy / dz
        sz = f(1) / dz
        ax = a[0] + sx * a[2]; ay = a[1] + sy * a[2]
        bx = b[0] + sx * b[2]; by = b[1] + sy * b[2]
        cx = c[0] + sx * c[2]; cy = c[1] + sy * c[2]
        e0 = bx * cy - by * cx
        e1 = cx * ay - cy * ax
        e2 = ax * by - ay * bx
        fb = (e0 == 0) | (e1 == 0) | (e2 == 0)
        D = np.float64
        e0 = np.where(fb, (D(cy) * D(bx) - D(cx) * D(by)).astype(f), e0)
        e1 = np.where(fb, (D(ay) * D(cx) - D(ax) * D(cy)).astype(f), e1)
        e2 = np.where(fb, (D(by) * D(ax) - D(bx) * D(ay)).astype(f), e2)
        ok = ~(((e0 < 0) | (e1 < 0) | (e2 < 0)) & ((e0 > 0) | (e1 > 0) | (e2 > 0)))
        det = e0 + e1 + e2
        ok &= det != 0
        az = a[2] * sz; bz = b[2] * sz; cz = c[2] * sz
        ts = e0 * az + e1 * bz + e2 * cz
        tmd = tmax * det
        ok &= ~((det < 0) & ((ts >= 0) | (ts < tmd)))
        ok &= ~((det > 0) & ((ts <= 0) | (ts > tmd)))
        inv = f(1) / det
        b0 = e0 * inv; b1 = e1 * inv; b2 = e2 * inv
        t = ts * inv
        mz = np.maximum(np.maximum(np.abs(az), np.abs(bz)), np.abs(cz))
        mx = np.maximum(np.maximum(np.abs(ax), np.abs(bx)), np.abs(cx))
        my = np.maximum(np.maximum(np.abs(ay), np.abs(by)), np.abs(cy))
        dz_ = g[3] * mz
        dx_ = g[5] * (mx + mz)
        dy_ = g[5] * (my + mz)
        de = f(2) * (g[2] * mx * my + dy_ * mx + dx_ * my)
        me = np.maximum(np.maximum(np.abs(e0), np.abs(e1)), np.abs(e2))
        dt = f(3) * (g[3] * me * mz + de * mz + dz_ * me) * np.abs(inv)
        ok &= ~(t <= dt)
    return ok, t, b0, b1, b2


def test_triangle_matches_numpy_restatement_bitwise():
    rng = np.random.default_rng(11)
    n = 4000
    f = np.float32
    p0 = rng.uniform(-1, 1, (n, 3)).astype(f)
    p1 = (p0 + rng.uniform(-0.5, 0.5, (n, 3))).astype(f)
    p2 = (p0 + rng.uniform(-0.5, 0.5, (n, 3))).astype(f)
    o = rng.uniform(-3, 3, (n, 3)).astype(f)
    # aim most rays at the triangle so that hits are frequent
    w = rng.dirichlet((1, 1, 1), n).astype(f)
    target = w[:, :1] * p0 + w[:, 1:2] * p1 + w[:, 2:] * p2
    d = (target - o).astype(f)
    d[::7] = rng.normal(size=(len(d[::7]), 3)).astype(f)
    d[::11, 0] = 0.0          # zero direction components
    # grid-snapped cases exercise the f64 edge fallback
    k = slice(0, n, 5)
    p0[k] = np.round(p0[k] * 4) / 4
    p1[k] = np.round(p1[k] * 4) / 4
    p2[k] = np.round(p2[k] * 4) / 4
    o[k] = np.round(o[k] * 4) / 4
    d[k] = np.round(d[k] * 4) / 4
    d[k][np.all(d[k] == 0, axis=1)] = (0, 0, 1)
    tmax = np.full(n, np.inf, f)
    tmax[::3] = rng.uniform(0.1, 3.0, len(tmax[::3])).astype(f)
    ok, t, b0, b1, b2 = watertight_np(p0, p1, p2, o, d, tmax)
    hits = 0
    for i in range(n):
        if np.all(d[i] == 0):
            continue
        r = oracle.triangle_intersect(p0[i], p1[i], p2[i], o[i], d[i], float(tmax[i]), closest=False)
        assert (r is not None) == bool(ok[i]), i
        if r is not None:
            hits += 1
            assert np.float32(r[0]) == t[i] and np.float32(r[2]) == b1[i] and np.float32(r[3]) == b2[i], i
    assert hits > n // 4


# --------------------------------------------------------------- sphere KATs
def test_sphere_unit_from_outside_and_inside():
    s = oracle.sphere_desc(1.0)
    # transform_ray_with_error moves the object-space origin forward by its
    # error bound (transform.rs:392-435), so t is a few ulps short of 4
    t, u, v = oracle.sphere_intersect(s, (0, 0, -5), (0, 0, 1))
    assert t == pytest.approx(4.0, rel=1e-6) and t <= 4.0 and u == 0.0 and v == 0.0
    t, u, v = oracle.sphere_intersect(s, (0, 0, 0), (0, 0, 1))
    assert t == pytest.approx(1.0, rel=1e-6)
    assert oracle.sphere_intersect(s, (0, 0, -5), (0, 0, 1), tmax=3.9) is None
    assert oracle.sphere_intersect(s, (2, 0, -5), (0, 0, 1)) is None


def test_sphere_translated():
    s = oracle.sphere_desc(0.5, translate=(2.0, 0.0, 0.0))
    t, u, v = oracle.sphere_intersect(s, (-1, 0, 0), (1, 0, 0))
    assert t == pytest.approx(2.5, rel=1e-6)


def test_sphere_partial_clipping_uses_far_root():
    s = oracle.sphere_desc(1.0, z_max=0.5)
    r = oracle.sphere_intersect(s, (0, 0, 5), (0, 0, -1))
    assert r is not None and r[0] == pytest.approx(6.0, rel=1e-6)
    half = oracle.sphere_desc(1.0, phi_max_deg=180.0)
    # hits at y < 0 (phi > pi) are clipped; a ray along -x... first root at x=1 (phi=0) kept
    r = oracle.sphere_intersect(half, (5, 0.0, 0.0), (-1, 0, 0))
    assert r is not None and r[0] == pytest.approx(4.0, rel=1e-6)
    assert oracle.sphere_intersect(half, (0.0, -5.0, 0.3), (0, 1, 0)) is not None   # far root at y=+r
    r = oracle.sphere_intersect(half, (0.0, -5.0, 0.3), (0, 1, 0))
    assert r[0] == pytest.approx(5.0 + math.sqrt(1 - 0.09), rel=1e-5)


def test_sphere_world_bound():
    lib = oracle.load()
    s = oracle.sphere_desc(0.5, translate=(1.0, 2.0, 3.0))
    out = np.zeros(6, np.float32)
    import ctypes
    lib.orc_sphere_world_bound(ctypes.byref(s), out.ctypes.data)
    assert np.allclose(out, [0.5, 1.5, 2.5, 1.5, 2.5, 3.5])

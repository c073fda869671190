"""Disks, cylinders, cones, paraboloids and hyperboloids (shapes/disk.rs,
cylinder.rs, cone.rs, paraboloid.rs, hyperboloid.rs) beside spheres and
triangles in one BVH.

CPU: the oracle's tests against an independent float64 solution of each
quadric (plane, x^2 + y^2 = r^2, x^2 + y^2 = (r/h)^2 (z - h)^2,
z = (z_max / r^2)(x^2 + y^2), ah (x^2 + y^2) - ch z^2 = 1 with clipping by
radius, z and phi) on random rays and transforms (rays that graze a clipping
boundary are skipped); this also pins the repairs (the cone's b coefficient,
the cylinder's phi_max in radians, the hyperboloid's constructor swap, c
coefficient and first phi).
GPU (marked): closest hits and any-hit flags of the B200 path equal the
oracle's (ids and t bit-exact, (u, v) within 1e-5) on mixed scenes."""
import math

import numpy as np
import pytest

import oracle
from rs_illume_b200 import workloads as wl

KINDS = {"sphere": 0, "disk": 1, "cylinder": 2, "cone": 3, "paraboloid": 4, "hyperboloid": 5}


def rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def random_quadric(rng, kind):
    m = np.eye(4)
    m[:3, :3] = rotation(rng) * rng.uniform(0.5, 1.5)
    m[:3, 3] = rng.uniform(-0.5, 0.5, 3)
    r = float(rng.uniform(0.3, 1.0))
    phi = float(rng.choice([360.0, rng.uniform(90, 359)]))
    if kind == "disk":
        p = dict(height=float(rng.uniform(-0.3, 0.3)), inner_radius=float(rng.choice([0.0, r * rng.uniform(0.1, 0.6)])))
    elif kind == "cylinder":
        z0, z1 = sorted(rng.uniform(-1, 1, 2))
        p = dict(z_min=float(z0), z_max=float(z1) + 0.1)
    elif kind == "cone":
        p = dict(height=float(rng.uniform(0.3, 1.5)))
    elif kind == "paraboloid":
        z0, z1 = sorted(rng.uniform(0.0, 1.2, 2))
        p = dict(z_min=float(z0), z_max=float(z1) + 0.2)
    elif kind == "hyperboloid":
        a = rng.uniform(0, 2 * np.pi, 2)
        r1, r2 = rng.uniform(0.2, 0.9, 2)
        z1, z2 = rng.uniform(-0.9, -0.1), rng.uniform(0.1, 0.9)
        p = dict(p1=(float(r1 * np.cos(a[0])), float(r1 * np.sin(a[0])), float(z1)),
                 p2=(float(r2 * np.cos(a[1])), float(r2 * np.sin(a[1])), float(z2)))
    else:
        p = dict(z_min=-r, z_max=r)
    return m, r, phi, p


def hyperboloid_coefficients(p1, p2):
    """Hyperboloid::new's implicit form in float64, with pbrt's swap."""
    p1, p2 = np.array(p1, np.float64), np.array(p2, np.float64)
    if p2[2] == 0.0:
        p1, p2 = p2, p1
    pp = p1.copy()
    ah = ch = np.inf
    while not (np.isfinite(ah) and np.isfinite(ch)):
        pp = pp + 2.0 * (p2 - p1)
        xy1 = pp[0] ** 2 + pp[1] ** 2
        xy2 = p2[0] ** 2 + p2[1] ** 2
        ah = (1.0 / xy1 - pp[2] ** 2 / (xy1 * p2[2] ** 2)) / (1.0 - xy2 * pp[2] ** 2 / (xy1 * p2[2] ** 2))
        ch = (ah * xy2 - 1.0) / p2[2] ** 2
    return p1, p2, ah, ch


def analytic(kind, m, r, phi_max_deg, p, o, d, tmax=np.inf):
    """float64 nearest hit t (or None), and whether a clip boundary is close."""
    inv = np.linalg.inv(m)
    oo = inv[:3, :3] @ o + inv[:3, 3]
    dd = inv[:3, :3] @ d
    phimax = math.radians(min(max(phi_max_deg, 0.0), 360.0))
    cands = []
    if kind == "disk":
        if dd[2] != 0:
            cands = [(p["height"] - oo[2]) / dd[2]]
    else:
        if kind == "cylinder":
            a = dd[0] ** 2 + dd[1] ** 2
            b = 2 * (dd[0] * oo[0] + dd[1] * oo[1])
            c = oo[0] ** 2 + oo[1] ** 2 - r * r
        elif kind == "cone":
            h = p["height"]
            k = (r / h) ** 2
            a = dd[0] ** 2 + dd[1] ** 2 - k * dd[2] ** 2
            b = 2 * (dd[0] * oo[0] + dd[1] * oo[1] - k * dd[2] * (oo[2] - h))
            c = oo[0] ** 2 + oo[1] ** 2 - k * (oo[2] - h) ** 2
        elif kind == "paraboloid":
            k = p["z_max"] / r ** 2
            a = k * (dd[0] ** 2 + dd[1] ** 2)
            b = 2 * k * (dd[0] * oo[0] + dd[1] * oo[1]) - dd[2]
            c = k * (oo[0] ** 2 + oo[1] ** 2) - oo[2]
        elif kind == "hyperboloid":
            hp1, hp2, ah, ch = hyperboloid_coefficients(p["p1"], p["p2"])
            a = ah * (dd[0] ** 2 + dd[1] ** 2) - ch * dd[2] ** 2
            b = 2 * (ah * (dd[0] * oo[0] + dd[1] * oo[1]) - ch * dd[2] * oo[2])
            c = ah * (oo[0] ** 2 + oo[1] ** 2) - ch * oo[2] ** 2 - 1.0
        else:
            a = dd @ dd
            b = 2 * dd @ oo
            c = oo @ oo - r * r
        disc = b * b - 4 * a * c
        if a != 0 and disc >= 0:
            sq = math.sqrt(disc)
            cands = sorted([(-b - sq) / (2 * a), (-b + sq) / (2 * a)])
    near = False
    for t in cands:
        if not (t > 1e-6 and t < tmax):
            continue
        q = oo + t * dd
        phi = math.atan2(q[1], q[0]) % (2 * math.pi)
        if kind == "hyperboloid":
            v = (q[2] - hp1[2]) / (hp2[2] - hp1[2])
            pr = (1 - v) * hp1 + v * hp2
            phi = math.atan2(pr[0] * q[1] - q[0] * pr[1], q[0] * pr[0] + q[1] * pr[1]) % (2 * math.pi)
        ok = phi <= phimax
        near |= abs(phi - phimax) < 1e-3 or phi < 1e-3 or phi > 2 * math.pi - 1e-3
        if kind == "disk":
            rr = math.hypot(q[0], q[1])
            ok &= p["inner_radius"] <= rr <= r
            near |= abs(rr - r) < 1e-3 or abs(rr - p["inner_radius"]) < 1e-3
        elif kind == "cylinder":
            ok &= p["z_min"] <= q[2] <= p["z_max"]
            near |= abs(q[2] - p["z_min"]) < 1e-3 or abs(q[2] - p["z_max"]) < 1e-3
        elif kind == "cone":
            ok &= 0 <= q[2] <= p["height"]
            near |= abs(q[2]) < 1e-3 or abs(q[2] - p["height"]) < 1e-3
        elif kind in ("paraboloid", "hyperboloid"):
            z0, z1 = (p["z_min"], p["z_max"]) if kind == "paraboloid" else sorted((p["p1"][2], p["p2"][2]))
            ok &= z0 <= q[2] <= z1
            near |= abs(q[2] - z0) < 1e-3 or abs(q[2] - z1) < 1e-3
        else:
            ok &= p["z_min"] <= q[2] <= p["z_max"]
        if ok:
            return t, near
    return None, near


@pytest.mark.parametrize("kind", ["disk", "cylinder", "cone", "paraboloid", "hyperboloid"])
def test_oracle_quadrics_against_float64(kind):
    rng = np.random.default_rng(KINDS[kind])
    checked = hits = 0
    for _ in range(40):
        m, r, phi, p = random_quadric(rng, kind)
        desc = oracle.quadric_desc(KINDS[kind], r, m, phi_max_deg=phi, **p)
        for _ in range(50):
            o = rng.uniform(-2.5, 2.5, 3)
            target = m[:3, 3] + rng.normal(scale=0.6, size=3)
            d = target - o
            d /= np.linalg.norm(d)
            want, near = analytic(kind, m, r, phi, p, o, d)
            if near:
                continue
            got = oracle.sphere_intersect(desc, o.astype(np.float32), d.astype(np.float32))
            checked += 1
            if want is None:
                assert got is None, (kind, o, d, got)
            else:
                hits += 1
                assert got is not None, (kind, o, d, want)
                assert got[0] == pytest.approx(want, rel=2e-4, abs=2e-5)
                assert 0.0 <= got[1] <= 1.0 + 1e-6 and -1e-6 <= got[2] <= 1.0 + 1e-6
    assert checked > 1000 and hits > 200, (checked, hits)


def test_quadric_known_answers():
    eye = np.eye(4)
    disk = oracle.quadric_desc(1, 1.0, eye, height=0.5, inner_radius=0.25)
    # (transform_ray_with_error moves the origin by its error bound, so t is a few ulps short)
    t, u, v = oracle.sphere_intersect(disk, (0.5, 0.0, 2.0), (0.0, 0.0, -1.0))
    assert t == pytest.approx(1.5, rel=1e-6) and u == 0.0 and v == pytest.approx((1.0 - 0.5) / (1.0 - 0.25))
    assert oracle.sphere_intersect(disk, (0.1, 0.0, 2.0), (0.0, 0.0, -1.0)) is None     # inside the hole
    cyl = oracle.quadric_desc(2, 1.0, eye, z_min=-1.0, z_max=1.0, phi_max_deg=360.0)
    t, u, v = oracle.sphere_intersect(cyl, (-3.0, 0.0, 0.5), (1.0, 0.0, 0.0))
    assert t == pytest.approx(2.0, rel=1e-6) and v == pytest.approx(0.75)
    half = oracle.quadric_desc(2, 1.0, eye, z_min=-1.0, z_max=1.0, phi_max_deg=180.0)
    # the near side (phi = pi) passes; from +y the near side (phi = pi/2) is kept
    assert oracle.sphere_intersect(half, (0.0, 3.0, 0.0), (0.0, -1.0, 0.0))[0] == pytest.approx(2.0, rel=1e-6)
    # from -y the near side has phi = 3pi/2 > pi: the far side at t = 4 answers
    assert oracle.sphere_intersect(half, (0.0, -3.0, 0.0), (0.0, 1.0, 0.0))[0] == pytest.approx(4.0, rel=1e-6)
    cone = oracle.quadric_desc(3, 1.0, eye, height=2.0)
    # along -x at z = 1 the cone's radius is 0.5: hit at x = 0.5
    t, u, v = oracle.sphere_intersect(cone, (3.0, 0.0, 1.0), (-1.0, 0.0, 0.0))
    assert t == pytest.approx(2.5, rel=1e-6) and v == pytest.approx(0.5)
    # z = x^2 + y^2 (k = z_max / r^2 = 1): straight down at x = 0.5 meets z = 0.25
    par = oracle.quadric_desc(4, 1.0, eye, z_min=0.0, z_max=1.0)
    t, u, v = oracle.sphere_intersect(par, (0.5, 0.0, 5.0), (0.0, 0.0, -1.0))
    assert t == pytest.approx(4.75, rel=1e-6) and u == 0.0 and v == pytest.approx(0.25)
    # p1 = (1, 0, -1), p2 = (1, 0, 1) sweep the unit cylinder: ah = 1, ch = 0
    hyp = oracle.quadric_desc(5, 0.0, eye, p1=(1.0, 0.0, -1.0), p2=(1.0, 0.0, 1.0))
    t, u, v = oracle.sphere_intersect(hyp, (-3.0, 0.0, 0.5), (1.0, 0.0, 0.0))
    assert t == pytest.approx(2.0, rel=1e-6) and u == pytest.approx(0.5) and v == pytest.approx(0.75)
    # p2.z == 0 swaps the points (pbrt; the reference swaps otherwise and never
    # leaves its loop): a cone-like sheet through (1, 0, 0) and (0.5, 0, 1)
    hyp2 = oracle.quadric_desc(5, 0.0, eye, p1=(0.5, 0.0, 1.0), p2=(1.0, 0.0, 0.0))
    assert oracle.sphere_intersect(hyp2, (-3.0, 0.0, 0.0), (1.0, 0.0, 0.0)) is not None


def mixed_scene(seed):
    rng = np.random.default_rng(seed)
    xyz, idx = wl.soup(seed, 256, 0.2)
    xyz = (xyz - 0.5) * 3.0
    quads = []
    for k in range(36):
        kind = list(KINDS)[k % 6]
        m, r, phi, p = random_quadric(rng, kind)
        m[:3, :3] *= 0.5
        m[:3, 3] *= 3.0
        quads.append((KINDS[kind], r, m, phi, p))
    rays = wl.ball_rays(seed, 4, 8192, 4096, 2.5, 0.1, 4.0)
    return xyz.astype(np.float32), idx, quads, rays


@pytest.mark.gpu
@pytest.mark.parametrize("width", [2, 4, 8])
def test_gpu_quadrics_match_oracle(ctx, width):
    import rs_illume_b200 as rb
    from tests.test_gpu_trace import compare_closest
    xyz, idx, quads, rays = mixed_scene(31)
    odescs = [oracle.quadric_desc(k, r, m, phi_max_deg=phi, **p) for k, r, m, phi, p in quads]
    gdescs = []
    for od in odescs:
        g = rb._lib.ilm_sphere_desc()
        import ctypes
        ctypes.memmove(ctypes.addressof(g), ctypes.addressof(od), ctypes.sizeof(g))
        gdescs.append(g)
    sc = oracle.Scene(xyz, idx, odescs)
    want = sc.intersect(rays)
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx), rb.Spheres(ctx, gdescs)], width=width)
    got = acc.intersect_batch(rays)
    quad_hits = int(np.sum((want["prim"] >= len(idx)) & (want["prim"] != rb.ILM_MISS)))
    assert quad_hits > 300, quad_hits
    compare_closest(got, want, tol_uv=1e-5, label=f"w{width}")
    assert np.array_equal(acc.intersect_p_batch(rays).astype(np.uint8), sc.intersect_p(rays))


def test_product_bounds_equal_oracle():
    """World bounds of the product's records (Transform::transform_bounds of
    each kind's object box) equal the oracle's, through the host-only build."""
    import ctypes
    from rs_illume_b200 import _lib
    from tests.layout_utils import host_layout
    rng = np.random.default_rng(41)
    for k in range(30):
        kind = list(KINDS)[k % 6]
        m, r, phi, p = random_quadric(rng, kind)
        od = oracle.quadric_desc(KINDS[kind], r, m, phi_max_deg=phi, **p)
        gd = _lib.ilm_sphere_desc()
        ctypes.memmove(ctypes.addressof(gd), ctypes.addressof(od), ctypes.sizeof(gd))
        lay = host_layout(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.uint32), 2, 4, spheres=[gd])
        sc = oracle.Scene(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.uint32), [od])
        assert np.array_equal(lay["bound"], sc.world_bound()), kind
    # a hyperboloid whose points give no finite implicit form is rejected
    bad = _lib.ilm_sphere_desc()
    ctypes.memmove(ctypes.addressof(bad), ctypes.addressof(oracle.quadric_desc(
        5, 0.0, np.eye(4), p1=(1.0, 0.0, 0.0), p2=(2.0, 0.0, 0.0))), ctypes.sizeof(bad))
    assert host_layout(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.uint32), 2, 4,
                       spheres=[bad]) == _lib.ILM_ERR_INVALID_ARGUMENT

"""kd-tree aggregate (KdTreeAccel, accelerators/kdtreeaccel.rs:11-596).

CPU: the product's host build equals the oracle's restatement node for node
and index for index, for any thread count and parameter set; structural
properties of the tree; the oracle's kd-tree answers every ray as the oracle's
BVH does (closest hits equal up to documented near-ties, any-hit flags
exact), which anchors the kd restatement on the BVH restatement and its known
answers.
GPU (marked): closest hits and any-hit flags of the B200 kd traversal equal the
oracle kd-tree's and the B200 BVH's; the no-alloc form, surface interactions
and the path tracer give the BVH accel's results on a kd accel.
"""
import numpy as np
import pytest

import oracle
from rs_illume_b200 import _lib
from rs_illume_b200 import workloads as wl
from tests.layout_utils import host_kdtree

MISS = 0xFFFFFFFF
TIE_REL = 1e-6


def compare(g, o, label="", tol_uv=0.0):
    """Closest hits equal except near-ties (both hit, |dt| <= 1e-6 t).  With
    tol_uv (GPU against CPU on quadrics, whose (u, v) go through atan2 / acos of
    either side's math library) t and (u, v) agree within 1e-5 relative and
    tol_uv absolute; otherwise bit for bit."""
    same = g["prim"] == o["prim"]
    for i in np.nonzero(~same)[0]:
        assert g["prim"][i] != MISS and o["prim"][i] != MISS, (label, i, g[i], o[i])
        assert abs(float(g["t"][i]) - float(o["t"][i])) <= TIE_REL * float(o["t"][i]), (label, i, g[i], o[i])
    hit = same & (o["prim"] != MISS)
    if tol_uv:
        np.testing.assert_allclose(g["t"][hit], o["t"][hit], rtol=1e-5)
        np.testing.assert_allclose(g["u"][hit], o["u"][hit], rtol=1e-5, atol=tol_uv)
        np.testing.assert_allclose(g["v"][hit], o["v"][hit], rtol=1e-5, atol=tol_uv)
    else:
        assert np.array_equal(g["t"][hit], o["t"][hit]), label
        assert np.array_equal(g["u"][hit], o["u"][hit]), label
        assert np.array_equal(g["v"][hit], o["v"][hit]), label
    return int((~same).sum())


def quadrics(seed, n):
    rng = np.random.default_rng(seed)
    out_o, out_g = [], []
    for k in range(n):
        c = rng.uniform(-1.0, 1.0, 3)
        r = float(rng.uniform(0.05, 0.25))
        m = np.eye(4)
        m[:3, 3] = c
        kind = k % 4
        kw = {0: dict(z_min=-r, z_max=r), 1: dict(height=0.0, inner_radius=0.3 * r),
              2: dict(z_min=-r, z_max=r), 3: dict(height=2 * r)}[kind]
        d = oracle.quadric_desc(kind, r, m, phi_max_deg=float(rng.choice([360.0, 250.0])), **kw)
        g = _lib.ilm_sphere_desc()
        import ctypes
        ctypes.memmove(ctypes.addressof(g), ctypes.addressof(d), ctypes.sizeof(g))
        out_o.append(d)
        out_g.append(g)
    return out_o, out_g


SCENES = {
    "soup": lambda: (*wl.soup(11, 3000, 0.08), 0),
    "icosphere": lambda: (*wl.icosphere(4, 5), 0),
    "cornell": lambda: (*wl.cornell(3, 3)[:2], 0),
    "mixed": lambda: (*wl.soup(12, 1500, 0.1), 24),
}


def scene(name):
    xyz, idx, nq = SCENES[name]()
    xyz = np.asarray(xyz, np.float32)
    if name in ("soup", "mixed"):
        xyz = (xyz - 0.5) * 2.0
    qo, qg = quadrics(7, nq) if nq else ([], [])
    return xyz, idx, qo, qg


@pytest.mark.parametrize("name", list(SCENES))
@pytest.mark.parametrize("params", [dict(), dict(max_prims=4, empty_bonus=0.2), dict(isect_cost=20, max_depth=9),
                                    dict(traversal_cost=5, max_prims=2)])
def test_product_build_equals_oracle(name, params):
    xyz, idx, qo, qg = scene(name)
    sc = oracle.Scene(xyz, idx, qo)
    kd = oracle.KdTree(sc, **params)
    for threads in (1, 8):
        st, lay = host_kdtree(xyz, idx, qg, threads=threads, **params)
        assert st == 0
        assert np.array_equal(lay["nodes"], kd.nodes()), (name, params, threads)
        assert np.array_equal(lay["index"], kd.indices()), (name, params, threads)
        assert lay["info"].max_depth == kd.max_depth
        assert lay["info"].width == _lib.ILM_LAYOUT_KDTREE
    # records are stored by primitive id
    assert np.array_equal(lay["records"]["prim"], np.arange(len(idx) + len(qg), dtype=np.uint32))


def walk(nodes, index):
    """(leaf prim lists with their depth, interior count); checks links."""
    leaves, interior = [], 0
    stack = [(0, 0)]
    seen = np.zeros(len(nodes), bool)
    while stack:
        i, depth = stack.pop()
        assert not seen[i]
        seen[i] = True
        w, f = int(nodes["word"][i]), int(nodes["flags"][i])
        if f & 3 == 3:
            n = f >> 2
            prims = [] if n == 0 else ([w] if n == 1 else list(index[w:w + n]))
            leaves.append((prims, depth))
        else:
            interior += 1
            above = f >> 2
            assert i + 1 < above < len(nodes)
            stack.append((i + 1, depth + 1))
            stack.append((above, depth + 1))
    assert seen.all()                          # every node reachable exactly once
    return leaves, interior


def test_structure_and_defaults():
    xyz, idx = wl.soup(13, 4000, 0.05)
    st, lay = host_kdtree(xyz, idx)
    assert st == 0
    nodes, index = lay["nodes"], lay["index"]
    leaves, interior = walk(nodes, index)
    assert len(leaves) == interior + 1
    n = len(idx)
    assert lay["info"].max_depth == round(8 + 1.3 * np.log2(n))
    assert max(d for _, d in leaves) <= lay["info"].max_depth
    refs = np.concatenate([np.asarray(p, np.int64) for p, _ in leaves if p])
    assert set(refs.tolist()) == set(range(n))            # every primitive sits in some leaf
    assert sum(len(p) for p, _ in leaves if len(p) > 1) == len(index)
    # with max_prims 1 most leaves hold at most one primitive
    assert np.mean([len(p) <= 1 for p, _ in leaves]) > 0.6


def test_known_answer_two_triangles():
    # two triangles far apart along x: one split along x at an edge between them
    xyz = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [10, 0, 0], [11, 0, 0], [10, 1, 0]], np.float32)
    idx = np.array([[0, 1, 2], [3, 4, 5]], np.uint32)
    st, lay = host_kdtree(xyz, idx)
    nodes = lay["nodes"]
    assert len(nodes) == 3 and len(lay["index"]) == 0
    assert nodes["flags"][0] & 3 == 0 and nodes["flags"][0] >> 2 == 2
    split = nodes["word"][:1].view(np.float32)[0]
    assert split in (1.0, 10.0)                # the end of the first or the start of the second
    assert nodes["flags"][1] == 3 | (1 << 2) and nodes["word"][1] == 0
    assert nodes["flags"][2] == 3 | (1 << 2) and nodes["word"][2] == 1
    np.testing.assert_array_equal(lay["bound"], [0, 0, 0, 11, 1, 0])


def test_degenerate_inputs():
    # empty scene: no nodes
    st, lay = host_kdtree(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.uint32))
    assert st == 0 and len(lay["nodes"]) == 0
    # one primitive: a single leaf
    xyz = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    st, lay = host_kdtree(xyz, np.array([[0, 1, 2]], np.uint32))
    assert list(lay["nodes"]["flags"]) == [3 | 4] and list(lay["nodes"]["word"]) == [0]
    # identical bounds: no edge lies strictly inside the node on any axis -> one leaf of all
    xyz = np.tile(np.array([[0, 0, 0], [1, 0, 0], [0, 1, 1]], np.float32), (5, 1))
    idx = np.arange(15, dtype=np.uint32).reshape(5, 3)
    st, lay = host_kdtree(xyz, idx)
    assert len(lay["nodes"]) == 1 and lay["nodes"]["flags"][0] == 3 | (5 << 2)
    assert list(lay["index"]) == [0, 1, 2, 3, 4]
    # rejected parameters
    assert host_kdtree(xyz, idx, max_depth=65)[0] == _lib.ILM_ERR_INVALID_ARGUMENT
    assert host_kdtree(xyz, idx, empty_bonus=1.5)[0] == _lib.ILM_ERR_INVALID_ARGUMENT
    assert host_kdtree(xyz, idx, isect_cost=-1)[0] == _lib.ILM_ERR_INVALID_ARGUMENT


def axis_rays(seed, n):
    rng = np.random.default_rng(seed)
    r = np.zeros(6 * n, _lib.RAY_DTYPE)
    dirs = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], np.float32)
    for k in range(6):
        sl = slice(n * k, n * (k + 1))
        r["o"][sl] = rng.uniform(-1, 1, (n, 3)) - 3.0 * dirs[k]
        r["d"][sl] = dirs[k]
        r["d"][sl][::5, (k // 2 + 1) % 3] = -0.0      # a negative zero off the axis
        r["tmax"][sl] = np.inf
    r["tmax"][::9] = 0.0
    return r


@pytest.mark.parametrize("name", list(SCENES))
def test_oracle_kdtree_answers_as_the_bvh(name):
    xyz, idx, qo, _ = scene(name)
    sc = oracle.Scene(xyz, idx, qo)
    kd = oracle.KdTree(sc)
    rays = np.concatenate([wl.ball_rays(5, 0, 40000, 40000, 2.5, 0.05, 4.0), axis_rays(6, 500)])
    # near-ties come from coplanar overlapping triangles (the Cornell box's
    # walls and blocks), where visit order decides between equal distances
    ties = compare(kd.intersect(rays), sc.intersect(rays), name)
    assert ties <= 1e-3 * len(rays), ties
    assert np.array_equal(kd.intersect_p(rays), sc.intersect_p(rays))
    # a tighter leaf size and a shallow depth limit change the tree, not the answers
    for params in (dict(max_prims=4), dict(max_depth=6)):
        k2 = oracle.KdTree(sc, **params)
        compare(k2.intersect(rays), sc.intersect(rays), name)
        assert np.array_equal(k2.intersect_p(rays), sc.intersect_p(rays))


# ----------------------------------------------------------------------- GPU

@pytest.mark.gpu
@pytest.mark.parametrize("name", list(SCENES))
def test_gpu_kdtree_matches_oracle(ctx, name):
    import rs_illume_b200 as rb
    xyz, idx, qo, qg = scene(name)
    shapes = [rb.TriangleMesh(ctx, xyz, idx)] + ([rb.Spheres(ctx, qg)] if qg else [])
    acc = rb.GpuKdTreeAccel(ctx, shapes)
    sc = oracle.Scene(xyz, idx, qo)
    kd = oracle.KdTree(sc)
    n0, i0 = acc.kd_nodes()
    assert np.array_equal(n0, kd.nodes()) and np.array_equal(i0, kd.indices())
    rays = np.concatenate([wl.ball_rays(8, 0, 131072, 131072, 2.5, 0.05, 4.0), axis_rays(9, 2000)])
    g = acc.intersect_batch(rays)
    tol = 1e-5 if qg else 0.0
    assert compare(g, kd.intersect(rays), name, tol) <= 1e-3 * len(rays)
    assert np.array_equal(acc.intersect_p_batch(rays).astype(np.uint8), kd.intersect_p(rays))
    # the BVH accel over the same shapes answers the same
    bvh = rb.GpuBVHAccel(ctx, shapes, width=8)
    compare(g, bvh.intersect_batch(rays), name)
    wb = acc.world_bound()
    assert np.array_equal(np.concatenate([wb.min, wb.max]), np.asarray(sc.world_bound()))


@pytest.mark.gpu
@pytest.mark.parametrize("n", [40000, 700001])
def test_gpu_kdtree_split_tail_agrees(n):
    """The kd-tree's split tail (idle lanes take a deferred subtree with its
    range) against the lone traversal, device buffers: any-hit flags equal,
    closest hits equal up to exact ties in t.  700,001 rays run the pooled
    persistent kernel well past its claims; 40,000 is a short queue."""
    import torch
    import rs_illume_b200 as rb
    xyz, idx = wl.icosphere(6, 4)
    rays = wl.ball_rays(6, 4, n, n // 2)
    d_rays = torch.from_numpy(rays.view(np.uint8)).cuda()
    out = []
    for split in (False, True):
        c = rb.Context(0, high_occupancy=True, tail_split=split)
        kd = rb.GpuKdTreeAccel(c, [rb.TriangleMesh(c, xyz, idx)])
        d_hits = torch.full((n * 16,), 0xAB, dtype=torch.uint8, device="cuda")
        d_occ = torch.full((n * 4,), 0xAB, dtype=torch.uint8, device="cuda")
        kd.intersect_batch(d_rays, d_hits)
        kd.intersect_p_batch(d_rays, d_occ)
        torch.cuda.synchronize()
        out.append((d_hits.cpu().numpy().view(_lib.HIT_DTYPE), d_occ.cpu().numpy().view(np.uint32)))
        assert c.device_errors() == 0
        c.close()
    assert np.array_equal(out[0][1], out[1][1])
    assert np.all(out[1][1] <= 1)
    compare(out[1][0], out[0][0], "kd split tail")
    assert np.mean(out[0][0]["prim"] != MISS) > 0.05


@pytest.mark.gpu
def test_gpu_kdtree_device_buffers_noalloc_and_interactions(ctx):
    import torch
    import rs_illume_b200 as rb
    xyz, idx = wl.icosphere(6, 4)
    mesh = rb.TriangleMesh(ctx, xyz, idx)
    kd = rb.GpuKdTreeAccel(ctx, [mesh])
    bvh = rb.GpuBVHAccel(ctx, [mesh], width=8)
    rays = wl.ball_rays(3, 4, 1 << 18, 1 << 18)
    host = kd.intersect_batch(rays)
    d_rays = torch.from_numpy(rays.view(np.uint8)).cuda()
    d_hits = torch.empty(len(rays) * 16, dtype=torch.uint8, device="cuda")
    s = torch.cuda.Stream()
    kd.intersect_batch(d_rays, d_hits, stream=s)
    s.synchronize()
    assert d_hits.cpu().numpy().tobytes() == host.tobytes()
    na = np.empty(4096, _lib.HIT_DTYPE)
    ctx.check(ctx._lib.ilm_intersect_closest_noalloc(ctx.handle, kd.id, _lib.ptr(rays[:4096]), 4096, _lib.ptr(na),
                                                     None), "noalloc")
    assert na.tobytes() == host[:4096].tobytes()
    compare(host, bvh.intersect_batch(rays), "icosphere")
    si_kd = kd.surface_interactions(rays[:8192], host[:8192])
    si_bvh = bvh.surface_interactions(rays[:8192], host[:8192])
    assert si_kd.tobytes() == si_bvh.tobytes()
    info = kd.info()
    assert info["width"] == _lib.ILM_LAYOUT_KDTREE and info["n_leaf_refs"] > 0


@pytest.mark.gpu
def test_gpu_path_tracer_on_kdtree(ctx):
    import rs_illume_b200 as rb
    xyz, idx, mat, alb, emi = wl.cornell(4, 3)
    cam = wl.CORNELL_CAMERA
    mesh = rb.TriangleMesh(ctx, xyz, idx)
    imgs = []
    for acc in (rb.GpuKdTreeAccel(ctx, [mesh]), rb.GpuBVHAccel(ctx, [mesh], width=8)):
        pt = rb.PathTracer(acc, mat, alb, emi, cam["eye"], cam["fov_deg"], 64, 64)
        img, st = pt.render(16, seed=5)
        imgs.append(img)
    # same closest hits -> the same paths: pixels agree up to the order of the
    # film's atomic accumulation; a near-tie between coplanar triangles may
    # change a rare path
    bad = ~np.isclose(imgs[0], imgs[1], rtol=1e-4, atol=1e-6)
    assert bad.mean() < 0.01, bad.mean()
    assert np.allclose(imgs[0].mean(), imgs[1].mean(), rtol=1e-3)

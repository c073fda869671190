"""GPU parity tests for the ray-query kernels (through the C ABI).

Bar (from the hot-path contract): primitive ids bit-exact except near-ties with
|dt| <= 1e-6 * t; t and (u, v) within 1e-5 relative (triangles are in fact
bit-identical because the kernels use the reference's rounding sequence);
any-hit booleans exact.  The CPU oracle is the checker.
"""
import numpy as np
import pytest

import oracle
import rs_illume_b200 as rb
from rs_illume_b200 import workloads as wl
from rs_illume_b200._lib import HIT_DTYPE, ILM_MISS, ILM_TRAVERSAL_ERROR, RAY_DTYPE

pytestmark = pytest.mark.gpu

MISS = ILM_MISS
TIE_REL = 1e-6
VAL_REL = 1e-5


def compare_closest(g, o, tol_uv=0.0, label=""):
    """Returns the number of documented near-ties; asserts everything else."""
    assert len(g) == len(o)
    same = g["prim"] == o["prim"]
    diff = np.nonzero(~same)[0]
    ties = 0
    for i in diff:
        # both must hit, at t equal to within 1e-6 relative (near-tie rule)
        assert g["prim"][i] != MISS and o["prim"][i] != MISS, (label, i, g[i], o[i])
        assert abs(float(g["t"][i]) - float(o["t"][i])) <= TIE_REL * float(o["t"][i]), (label, i, g[i], o[i])
        ties += 1
    hit = same & (o["prim"] != MISS)
    if tol_uv == 0.0:
        assert np.array_equal(g["t"][hit], o["t"][hit]), label
        assert np.array_equal(g["u"][hit], o["u"][hit]), label
        assert np.array_equal(g["v"][hit], o["v"][hit]), label
    else:
        np.testing.assert_allclose(g["t"][hit], o["t"][hit], rtol=VAL_REL)
        np.testing.assert_allclose(g["u"][hit], o["u"][hit], atol=tol_uv, rtol=VAL_REL)
        np.testing.assert_allclose(g["v"][hit], o["v"][hit], atol=tol_uv, rtol=VAL_REL)
    # misses report tmax
    miss = o["prim"] == MISS
    assert np.all(g["prim"][miss & same] == MISS)
    return ties


@pytest.fixture(scope="module")
def coherent():
    xyz, idx, rays = wl.coherent_workload()
    sc = oracle.Scene(xyz, idx)
    return xyz, idx, rays, sc, sc.intersect(rays)


@pytest.fixture(scope="module")
def incoherent():
    xyz, idx = wl.icosphere(8, 2)
    rays = wl.ball_rays(2, 4, 4194304, 2097152)
    sc = oracle.Scene(xyz, idx)
    return xyz, idx, rays, sc


@pytest.mark.parametrize("width", [2, 4, 8])
def test_coherent_closest_parity(ctx, coherent, width):
    xyz, idx, rays, sc, ref = coherent
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx)], width=width)
    g = acc.intersect_batch(rays)
    ties = compare_closest(g, ref, label=f"coherent w{width}")
    assert ties <= 2
    assert 0.3 < np.mean(ref["prim"] != MISS) < 0.9
    assert ctx.device_errors() == 0


@pytest.mark.parametrize("width", [2, 4, 8])
def test_coherent_any_parity(ctx, coherent, width):
    xyz, idx, rays, sc, ref = coherent
    r = rays.copy()
    rng = np.random.default_rng(1)
    r["tmax"] = rng.uniform(1.0, 2.5, len(r)).astype(np.float32)
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx)], width=width)
    g = acc.intersect_p_batch(r)
    o = sc.intersect_p(r)
    assert np.array_equal(g.astype(np.uint8), o)
    assert 0.05 < o.mean() < 0.95


@pytest.mark.parametrize("width", [2, 4, 8])
def test_incoherent_parity_sample(ctx, incoherent, width):
    xyz, idx, rays, sc = incoherent
    rng = np.random.default_rng(width)
    pick_c = np.sort(rng.choice(2097152, 131072, replace=False))
    pick_s = np.sort(rng.choice(2097152, 131072, replace=False)) + 2097152
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx)], width=width)
    rc = np.ascontiguousarray(rays[pick_c])
    ties = compare_closest(acc.intersect_batch(rc), sc.intersect(rc), label=f"incoherent w{width}")
    assert ties <= 4
    rs = np.ascontiguousarray(rays[pick_s])
    assert np.array_equal(acc.intersect_p_batch(rs).astype(np.uint8), sc.intersect_p(rs))


def test_incoherent_full_size_properties(ctx, incoherent):
    """All 4,194,304 rays on the GPU: widths agree, any-hit agrees with
    closest-hit under the same tmax, and every ray's closest hit and
    occlusion flag match the oracle's."""
    xyz, idx, rays, sc = incoherent
    mesh = rb.TriangleMesh(ctx, xyz, idx)
    a8 = rb.GpuBVHAccel(ctx, [mesh], width=8)
    a2 = rb.GpuBVHAccel(ctx, [mesh], width=2)
    h8 = a8.intersect_batch(rays)
    h2 = a2.intersect_batch(rays)
    ties = compare_closest(h8, h2, label="w8 vs w2 full")
    assert ties <= 16
    occ = a8.intersect_p_batch(rays)
    # occluded  <=>  a closest hit exists within the same tmax (no degenerate triangles here)
    assert np.array_equal(occ.astype(bool), h8["prim"] != MISS)
    assert np.all(h8["prim"] != ILM_TRAVERSAL_ERROR)
    ties = compare_closest(h8, sc.intersect(rays), label="full size against the oracle")
    assert ties <= 16, ties
    assert np.array_equal(occ.astype(np.uint8), sc.intersect_p(rays))
    assert ctx.device_errors() == 0


def test_bench_launch_full_size_against_oracle(incoherent):
    """The exact launch the headline measures: a high-occupancy context
    (persistent schedule, 8 resident blocks per SM, 64-entry stack), width 8,
    device-resident rays and results on a stream of the caller.  Every one of
    the 2,097,152 closest-hit and 2,097,152 any-hit answers is checked against
    the oracle (BVHAccel::intersect / intersect_p, accelerators/bvh.rs:563-662)."""
    import torch
    xyz, idx, rays, sc = incoherent
    ctx = rb.Context(0, high_occupancy=True, stack_depth=64)
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx)], width=8)
    half = len(rays) // 2
    closest = np.ascontiguousarray(rays[:half])
    shadow = np.ascontiguousarray(rays[half:])
    d_closest = torch.from_numpy(closest.view(np.uint8)).cuda()
    d_shadow = torch.from_numpy(shadow.view(np.uint8)).cuda()
    d_hits = torch.empty(half * 16, dtype=torch.uint8, device="cuda")
    d_occ = torch.empty(half, dtype=torch.int32, device="cuda")
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    for _ in range(2):     # a relaunch reuses the stream's work counter
        acc.intersect_batch(d_closest, d_hits, stream=s)
        acc.intersect_p_batch(d_shadow, d_occ, stream=s)
    s.synchronize()
    g = d_hits.cpu().numpy().view(HIT_DTYPE)
    ties = compare_closest(g, sc.intersect(closest), label="bench launch, closest")
    assert ties <= 8, ties
    assert np.array_equal(d_occ.cpu().numpy().view(np.uint32).astype(np.uint8), sc.intersect_p(shadow))
    assert ctx.device_errors() == 0
    ctx.close()


@pytest.mark.parametrize("width,n", [(8, 1000003), (4, 600001), (8, 40000)])
def test_pooled_lane_refill_and_grid_schedules_agree(incoherent, width, n):
    """Device buffers: the persistent schedule with warp-filtered chunks and a
    per-warp pool, with per-lane refill, and one thread per ray give
    byte-identical records for closest and any hit.  The pooled schedule's
    split tail (the default: idle lanes take subtrees of their warp's last
    rays; in the one-thread-per-ray kernel, from the start) gives the same
    any-hit flags and the same closest hits up to exact ties in t, where the
    lone traversal keeps the first hit it found and the split keeps the
    smaller primitive id.  The counts are not multiples of a
    chunk, and 40,000 rays is a short queue (one ray per lane per claim).
    Outputs start as a fill pattern, so a ray handed out twice or never
    would show."""
    import torch
    xyz, idx, rays, sc = incoherent
    half = len(rays) // 2                                       # closest (tmax = inf) and shadow rays mixed
    sub = np.ascontiguousarray(np.concatenate([rays[:n // 2], rays[half:half + n - n // 2]]))
    d_rays = torch.from_numpy(sub.view(np.uint8)).cuda()
    out = []
    for kw in ({"high_occupancy": True, "tail_split": False}, {"high_occupancy": True, "lane_refill": True},
               {"grid_schedule": True, "tail_split": False}, {"high_occupancy": True}, {}, {"grid_schedule": True}):
        ctx = rb.Context(0, **kw)
        acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx)], width=width)
        d_hits = torch.full((n * 16,), 0xAB, dtype=torch.uint8, device="cuda")
        d_occ = torch.full((n * 4,), 0xAB, dtype=torch.uint8, device="cuda")
        acc.intersect_batch(d_rays, d_hits)
        acc.intersect_p_batch(d_rays, d_occ)
        torch.cuda.synchronize()
        out.append((d_hits.cpu().numpy().tobytes(), d_occ.cpu().numpy().tobytes()))
        assert ctx.device_errors() == 0
        ctx.close()
    assert out[0] == out[1] == out[2]
    assert np.all(np.frombuffer(out[0][1], np.uint32) <= 1)
    for split in out[3:]:                       # split tail: pooled at 8 blocks per SM and default, grid
        assert split[1] == out[0][1]
        ties = compare_closest(np.frombuffer(split[0], HIT_DTYPE), np.frombuffer(out[0][0], HIT_DTYPE),
                               label="split tail")
        assert ties <= 16
    pick = np.sort(np.random.default_rng(n).choice(n, 20000, replace=False))
    g = np.frombuffer(out[0][0], HIT_DTYPE)[pick]
    compare_closest(g, sc.intersect(np.ascontiguousarray(sub[pick])), label="pooled")


@pytest.mark.parametrize("width", [4, 8])
def test_persistent_and_grid_schedules_agree(incoherent, width):
    """The persistent schedule (work counter, lane refill) and one thread per
    ray must produce byte-identical records, for closest and any hit."""
    xyz, idx, rays, sc = incoherent
    out = []
    for grid in (False, True):
        c = rb.Context(0, grid_schedule=grid, stack_depth=32 if width == 4 else 64)
        acc = rb.GpuBVHAccel(c, [rb.TriangleMesh(c, xyz, idx)], width=width)
        out.append((acc.intersect_batch(rays[:1 << 20]).tobytes(), acc.intersect_p_batch(rays[1 << 21:]).tobytes()))
        assert c.device_errors() == 0
        c.close()
    assert out[0] == out[1]


def sphere_scene():
    rng = np.random.default_rng(5)
    centres = rng.uniform(-1, 1, (64, 3))
    radii = rng.uniform(0.05, 0.2, 64)
    kinds = []
    for i in range(64):
        kw = {}
        if i % 4 == 1:
            kw["z_max"] = 0.3 * radii[i]
        if i % 4 == 2:
            kw["phi_max_deg"] = 200.0
        kinds.append(kw)
    xyz, idx = wl.icosphere(3, 7, 0.05, 0.3, (0.0, 0.0, 1.5))
    return xyz, idx, centres, radii, kinds


@pytest.mark.parametrize("width", [2, 8])
def test_spheres_and_triangles_parity(ctx, width):
    xyz, idx, centres, radii, kinds = sphere_scene()
    gd = [rb.sphere_desc(float(r), tuple(c), **k) for c, r, k in zip(centres, radii, kinds)]
    od = [oracle.sphere_desc(float(r), tuple(c), **k) for c, r, k in zip(centres, radii, kinds)]
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx), rb.Spheres(ctx, gd)], width=width)
    sc = oracle.Scene(xyz, idx, spheres=od)
    rays = wl.ball_rays(17, 0, 65536, 32768, 2.5, 0.1, 4.0)
    g = acc.intersect_batch(rays[:32768])
    o = sc.intersect(rays[:32768])
    compare_closest(g, o, tol_uv=1e-5, label="spheres")
    assert np.sum(o["prim"] >= len(idx)) > 1000          # many sphere hits
    occ = acc.intersect_p_batch(rays[32768:])
    assert np.array_equal(occ.astype(np.uint8), sc.intersect_p(rays[32768:]))


def test_device_pointers_and_stream(ctx, incoherent):
    import torch
    xyz, idx, rays, sc = incoherent
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx)], width=8)
    n = 1 << 20
    host = np.ascontiguousarray(rays[:n])
    d_rays = torch.from_numpy(host.view(np.uint8)).cuda()
    d_hits = torch.empty(n * 16, dtype=torch.uint8, device="cuda")
    s = torch.cuda.Stream()
    acc.intersect_batch(d_rays, d_hits, stream=s)
    s.synchronize()
    g = d_hits.cpu().numpy().view(HIT_DTYPE)
    assert g.tobytes() == acc.intersect_batch(host).tobytes()
    d_occ = torch.empty(n, dtype=torch.int32, device="cuda")
    acc.intersect_p_batch(d_rays, d_occ)
    torch.cuda.synchronize()
    assert np.array_equal(d_occ.cpu().numpy().view(np.uint32), acc.intersect_p_batch(host))


def test_edge_cases(ctx):
    xyz, idx = wl.soup(3, 500, 0.05)
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx)], width=8)
    sc = oracle.Scene(xyz, idx)
    # zero-size batch
    assert len(acc.intersect_batch(np.zeros(0, RAY_DTYPE))) == 0
    # axis-aligned rays (zero direction components, +-inf reciprocals), tmax = 0
    r = np.zeros(6 * 64, RAY_DTYPE)
    rng = np.random.default_rng(3)
    dirs = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], np.float32)
    for k in range(6):
        sl = slice(64 * k, 64 * (k + 1))
        r["o"][sl] = rng.uniform(0, 1, (64, 3)) - 2.0 * dirs[k]
        r["d"][sl] = dirs[k]
        r["tmax"][sl] = np.inf
    r["d"][::5, 0] = -0.0
    r["tmax"][::9] = 0.0
    compare_closest(acc.intersect_batch(r), sc.intersect(r), label="axis rays")
    assert np.array_equal(acc.intersect_p_batch(r).astype(np.uint8), sc.intersect_p(r))
    # single-ray Primitive surface
    h = acc.intersect(rb.Ray((0.5, 0.5, -3.0), (0.0, 0.0, 1.0)))
    o = sc.intersect(rb.rays_array([rb.Ray((0.5, 0.5, -3.0), (0.0, 0.0, 1.0))]))[0]
    assert (h is None and o["prim"] == MISS) or (h.prim == o["prim"] and h.t == o["t"])
    wb = acc.world_bound()
    assert np.array_equal(np.concatenate([wb.min, wb.max]), sc.world_bound())
    assert acc.get_material() is None and acc.get_area_light() is None


def test_empty_scene(ctx):
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, np.zeros((0, 3), np.float32), np.zeros((0, 3), np.uint32))])
    rays = wl.ball_rays(1, 0, 1000, 500)
    h = acc.intersect_batch(rays)
    assert np.all(h["prim"] == MISS)
    assert not acc.intersect_p_batch(rays).any()


def test_iteration_cap_flags_rays_and_context_survives():
    ctx = rb.Context(0, max_iterations=3)
    xyz, idx = wl.icosphere(5, 2)
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx)], width=8)
    rays = wl.ball_rays(2, 4, 4096, 4096)
    h = acc.intersect_batch(rays)
    capped = h["prim"] == ILM_TRAVERSAL_ERROR
    assert capped.any()
    assert ctx.device_errors() & 2
    assert ctx.device_errors() == 0                       # reset by the previous read
    ctx.close()
    # a fresh context with the default cap traces the same rays normally
    c2 = rb.Context(0)
    a2 = rb.GpuBVHAccel(c2, [rb.TriangleMesh(c2, xyz, idx)], width=8)
    h2 = a2.intersect_batch(rays)
    assert not np.any(h2["prim"] == ILM_TRAVERSAL_ERROR)
    c2.close()


def test_host_validation_rejects_bad_rays():
    ctx = rb.Context(0, validate_rays=True)
    xyz, idx = wl.soup(3, 100, 0.05)
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx)])
    rays = wl.ball_rays(1, 0, 100, 100)
    acc.intersect_batch(rays)
    bad = rays.copy()
    bad["d"][7] = (np.nan, 0, 1)
    with pytest.raises(rb.IllumeError) as e:
        acc.intersect_batch(bad)
    assert e.value.status == -1 and "ray 7" in str(e.value)
    bad = rays.copy()
    bad["tmax"][3] = -1.0
    with pytest.raises(rb.IllumeError):
        acc.intersect_p_batch(bad)
    ctx.close()


def test_watchdog_timeout(ctx, incoherent):
    import torch
    xyz, idx, rays, sc = incoherent
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx)], width=2)
    d_rays = torch.from_numpy(rays.view(np.uint8)).cuda()
    d_hits = torch.empty(len(rays) * 16, dtype=torch.uint8, device="cuda")
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    for _ in range(4):
        acc.intersect_batch(d_rays, d_hits, stream=s)
    with pytest.raises(rb.IllumeError) as e:
        ctx.synchronize(s.cuda_stream, timeout_s=0.0)
    assert e.value.status == -5
    ctx.synchronize(s.cuda_stream, timeout_s=60.0)


def test_mixed_pointer_kinds_rejected(ctx):
    import torch
    xyz, idx = wl.soup(3, 100, 0.05)
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx)])
    rays = wl.ball_rays(1, 0, 64, 64)
    d_hits = torch.empty(64 * 16, dtype=torch.uint8, device="cuda")
    with pytest.raises(rb.IllumeError) as e:
        acc.intersect_batch(rays, d_hits)
    assert e.value.status == -1


@pytest.mark.parametrize("grid", [False, True])
def test_batch_beyond_32_bit_offsets(incoherent, grid):
    """138,412,032 rays (4.4 GB of ray records, 2.2 GB of hits): the incoherent
    rays tiled 33 times on the device.  Every copy must answer exactly as the
    first, so ray indices, byte offsets and the persistent schedule's claim
    counter stay correct past 2^32 bytes, for closest and any hit."""
    import torch
    xyz, idx, rays, _ = incoherent
    ctx = rb.Context(0, high_occupancy=True, grid_schedule=grid)
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx)], width=8)
    reps = 33
    one = torch.from_numpy(rays.view(np.uint8)).cuda()
    d_rays = one.repeat(reps)
    n = len(rays) * reps
    assert n * 32 > (1 << 32) and n * 16 > (1 << 31)
    d_hits = torch.empty(n * 16, dtype=torch.uint8, device="cuda")
    d_occ = torch.empty(n * 4, dtype=torch.uint8, device="cuda")
    # no stream given: the calls run on torch's current stream, after repeat()
    acc.intersect_batch(d_rays, d_hits)
    acc.intersect_p_batch(d_rays, d_occ)
    torch.cuda.synchronize()
    del d_rays
    hits = d_hits.view(reps, -1)
    occ = d_occ.view(reps, -1)
    assert bool((hits == hits[0]).all()) and bool((occ == occ[0]).all())
    want = acc.intersect_batch(rays)
    assert hits[0].cpu().numpy().tobytes() == want.tobytes()
    assert ctx.device_errors() == 0
    ctx.close()

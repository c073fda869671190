"""CPU tests of the product's host-side build (SAH tree, wide collapse, records).

The product builder is an independent implementation of BVHAccel::new
(accelerators/bvh.rs:32-93, 95-247, 504-537); it must reproduce the oracle's
binary tree node for node, and its compressed wide layouts must be
conservative and complete.
"""
import numpy as np
import pytest

import oracle
from rs_illume_b200 import workloads as wl
from tests.layout_utils import dequantised_boxes, host_layout


def random_scene(seed, n, spread=0.05, dup=0):
    rng = np.random.default_rng(seed)
    c = rng.uniform(0, 1, (n, 1, 3))
    xyz = (c + rng.uniform(-spread, spread, (n, 3, 3))).astype(np.float32).reshape(-1, 3)
    if dup:
        # identical triangles force zero-extent centroid bounds (bvh.rs:133-141)
        xyz[: 3 * dup] = np.tile(xyz[:3], (dup, 1))
    idx = np.arange(3 * n, dtype=np.uint32).reshape(-1, 3)
    return xyz, idx


SCENES = {
    "coherent_soup": lambda: wl.soup(1, 32768, 0.02),
    "icosphere_l5": lambda: wl.icosphere(5, 2),
    "random_1k": lambda: random_scene(3, 1000),
    "duplicates": lambda: random_scene(4, 300, dup=40),
    "tiny_3": lambda: random_scene(5, 3),
    "single": lambda: random_scene(6, 1),
}


@pytest.mark.parametrize("name", list(SCENES))
@pytest.mark.parametrize("max_prims", [4, 1, 8])
def test_binary_tree_matches_oracle(name, max_prims):
    xyz, idx = SCENES[name]()
    lay = host_layout(xyz, idx, 2, max_prims)
    sc = oracle.Scene(xyz, idx, max_prims_in_node=max_prims)
    assert lay["bin"].tobytes() == sc.nodes().tobytes()
    assert np.array_equal(lay["order"], sc.prim_order())
    assert np.array_equal(lay["bound"], sc.world_bound())


def test_binary_tree_with_spheres_matches_oracle():
    xyz, idx = random_scene(7, 200)
    from rs_illume_b200.primitive import sphere_desc
    sd = [sphere_desc(0.05, translate=(0.1 * i, 0.5, 0.2 * (i % 3))) for i in range(10)]
    od = [oracle.sphere_desc(0.05, translate=(0.1 * i, 0.5, 0.2 * (i % 3))) for i in range(10)]
    lay = host_layout(xyz, idx, 2, 4, spheres=sd)
    sc = oracle.Scene(xyz, idx, spheres=od)
    assert lay["bin"].tobytes() == sc.nodes().tobytes()
    assert np.array_equal(lay["order"], sc.prim_order())
    rec = lay["records"]
    assert np.sum((rec["flags"] & 2) != 0) == 10


def test_binary_tree_invariants():
    xyz, idx = wl.icosphere(4, 9)
    lay = host_layout(xyz, idx, 2)
    nodes = lay["bin"]
    n = len(idx)
    seen = np.zeros(n, int)
    tb = np.stack([xyz[idx].min(1), xyz[idx].max(1)], 1)   # per-triangle bounds
    order = lay["order"]
    for i, nd in enumerate(nodes):
        if nd["n_prims"] > 0:
            assert nd["n_prims"] <= 4
            ids = order[nd["offset"]: nd["offset"] + nd["n_prims"]]
            seen[ids] += 1
            assert np.all(tb[ids, 0] >= nd["bmin"]) and np.all(tb[ids, 1] <= nd["bmax"])
        else:
            for c in (i + 1, nd["offset"]):
                assert np.all(nodes[c]["bmin"] >= nd["bmin"]) and np.all(nodes[c]["bmax"] <= nd["bmax"])
    assert np.all(seen == 1)


@pytest.mark.parametrize("width", [4, 8])
@pytest.mark.parametrize("name", ["coherent_soup", "icosphere_l5", "random_1k", "duplicates", "tiny_3", "single"])
def test_wide_layout_complete_and_conservative(width, name):
    xyz, idx = SCENES[name]()
    lay = host_layout(xyz, idx, width, 4)
    nodes, recs = lay["nodes"], lay["records"]
    n = len(idx)
    assert sorted(recs["prim"].tolist()) == list(range(n))
    tri = np.stack([recs["p0"], recs["p1"], recs["p2"]], 1)
    rec_lo, rec_hi = tri.min(1), tri.max(1)
    # records carry the original vertices
    assert np.array_equal(tri, xyz[idx[recs["prim"]]])
    exact = {}
    used = np.zeros(len(recs), int)
    reached = np.zeros(len(nodes), int)
    reached[0] = 1

    def exact_bound(k):
        if k in exact:
            return exact[k]
        nd = nodes[k]
        lo, hi = np.full(3, np.inf, np.float32), np.full(3, -np.inf, np.float32)
        boxes = dequantised_boxes(nd, width)
        imask = int(nd["packed"]) >> 24
        for c in range(width):
            m = int(nd["meta"][c])
            if m == 0:
                continue
            if (imask >> c) & 1:
                ch = int(nd["child_base"]) + (m & 31)
                reached[ch] += 1
                clo, chi = exact_bound(ch)
            else:
                cnt, off = m >> 5, m & 31
                assert 1 <= cnt <= 4
                r = slice(int(nd["prim_base"]) + off, int(nd["prim_base"]) + off + cnt)
                used[r] += 1
                clo, chi = rec_lo[r].min(0), rec_hi[r].max(0)
            # the dequantised box contains the exact child bounds
            assert np.all(boxes[c, 0] <= clo) and np.all(boxes[c, 1] >= chi), (k, c)
            lo, hi = np.minimum(lo, clo), np.maximum(hi, chi)
        exact[k] = (lo, hi)
        return exact[k]

    import sys
    sys.setrecursionlimit(10000)
    exact_bound(0)
    assert np.all(used == 1)
    assert np.all(reached == 1)


def test_degenerate_flag():
    xyz = np.array([[0, 0, 0], [1, 0, 0], [2, 0, 0], [0, 0, 1], [1, 0, 1], [0, 1, 1]], np.float32)
    idx = np.array([[0, 1, 2], [3, 4, 5]], np.uint32)
    lay = host_layout(xyz, idx, 8)
    rec = lay["records"]
    flags = dict(zip(rec["prim"].tolist(), rec["flags"].tolist()))
    assert flags[0] & 1 and not flags[1] & 1


def test_invalid_inputs_rejected():
    xyz, idx = random_scene(1, 4)
    assert host_layout(xyz, idx, 3) == -1                   # width
    assert host_layout(xyz, idx, 8, 0) == -1                # max prims
    bad = idx.copy()
    bad[0, 0] = 10_000
    assert host_layout(xyz, bad, 8) == -1                   # index out of range
    nan = xyz.copy()
    nan[0, 0] = np.nan
    assert host_layout(nan, idx, 8) == -1                   # non-finite vertex


def test_empty_scene():
    lay = host_layout(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.uint32), 8)
    assert lay["info"].n_nodes == 0 and lay["info"].n_prims == 0

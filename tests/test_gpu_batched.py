"""Batched multi-scene queries (one persistent launch, replayed as a CUDA graph)
and the autotuner.

Every batch must give byte-identical records to the single-scene entry
points (same traversal arithmetic), and a sample of every scene must match the
CPU oracle under the hit-parity rule.
"""
import numpy as np
import pytest

import oracle
import rs_illume_b200 as rb
from rs_illume_b200 import batch as bt
from rs_illume_b200 import workloads as wl
from tests.test_gpu_trace import compare_closest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scenes():
    return wl.batched_workload(7, 8, (1e3, 5e4), (1e4, 1e5))


def device(a):
    import torch
    return torch.from_numpy(a.view(np.uint8)).cuda()


def test_batched_plan_matches_single_scene_and_oracle(ctx, scenes):
    import torch
    accs, entries, any_entries, outs, occs = [], [], [], [], []
    for k, s in enumerate(scenes):
        acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, s["xyz"], s["idx"])], width=8 if k % 2 else 4)
        accs.append(acc)
        d_rays = device(s["rays"])
        out = torch.zeros(len(s["rays"]) * 16, dtype=torch.uint8, device="cuda")
        occ = torch.zeros(len(s["rays"]), dtype=torch.int32, device="cuda")
        outs.append(out)
        occs.append(occ)
        entries.append((acc, d_rays, out))
        any_entries.append((acc, d_rays, occ))
    plan = bt.BatchPlan(ctx, entries)                  # captures and runs once
    aplan = bt.BatchPlan(ctx, any_entries, any_hit=True)
    torch.cuda.synchronize()
    for k, s in enumerate(scenes):
        want = accs[k].intersect_batch(s["rays"])
        got = outs[k].cpu().numpy()
        assert got.tobytes() == want.tobytes(), k
        assert np.array_equal(occs[k].cpu().numpy().view(np.uint32), accs[k].intersect_p_batch(s["rays"])), k
        sc = oracle.Scene(s["xyz"], s["idx"])
        pick = np.random.default_rng(k).choice(len(s["rays"]), 2000, replace=False)
        sub = np.ascontiguousarray(s["rays"][np.sort(pick)])
        compare_closest(got.view(rb.HIT_DTYPE)[np.sort(pick)], sc.intersect(sub), label=f"batch {k}")
    # replay after clearing the outputs: the graph writes them again
    for o in outs:
        o.zero_()
    plan.launch()
    aplan.launch()
    torch.cuda.synchronize()
    for k, s in enumerate(scenes):
        assert outs[k].cpu().numpy().tobytes() == accs[k].intersect_batch(s["rays"]).tobytes()
    assert ctx.device_errors() == 0
    plan.close()
    aplan.close()


def test_bench_batch_sampled_against_oracle(ctx):
    """The batched workload as measured: 32 scenes (seed 5; 1k-2M triangles,
    10k-4M rays each, 15.7M rays), one plan, width 8.  For every scene 3,000
    rays (a third of them from each of the primary, incoherent and shadow
    groups) are checked against the oracle's BVHAccel::intersect
    (accelerators/bvh.rs:563-612), and the any-hit plan against intersect_p
    (bvh.rs:614-662)."""
    import torch
    scenes = wl.batched_workload(5, 32)
    assert len(scenes) == 32
    entries, any_entries, outs, occs = [], [], [], []
    for s in scenes:
        acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, s["xyz"], s["idx"])], width=8)
        d_rays = device(s["rays"])
        out = torch.zeros(len(s["rays"]) * 16, dtype=torch.uint8, device="cuda")
        occ = torch.zeros(len(s["rays"]), dtype=torch.int32, device="cuda")
        outs.append(out)
        occs.append(occ)
        entries.append((acc, d_rays, out))
        any_entries.append((acc, d_rays, occ))
    plan = bt.BatchPlan(ctx, entries)
    aplan = bt.BatchPlan(ctx, any_entries, any_hit=True)
    plan.launch()
    aplan.launch()
    torch.cuda.synchronize()
    assert ctx.device_errors() == 0
    total_hits = 0
    for k, s in enumerate(scenes):
        n = len(s["rays"])
        n1 = n // 3
        rng = np.random.default_rng(100 + k)
        groups = [(0, n1), (n1, n1 + (n - n1) // 2), (n1 + (n - n1) // 2, n)]
        pick = np.sort(np.concatenate([rng.choice(np.arange(a, b), min(1000, b - a), replace=False)
                                       for a, b in groups if b > a]))
        sub = np.ascontiguousarray(s["rays"][pick])
        sc = oracle.Scene(s["xyz"], s["idx"])
        got = outs[k].cpu().numpy().view(rb.HIT_DTYPE)[pick]
        compare_closest(got, sc.intersect(sub), label=f"bench scene {k}")
        total_hits += int(np.sum(got["prim"] != rb.ILM_MISS))
        occ = occs[k].cpu().numpy().view(np.uint32)[pick]
        assert np.array_equal(occ.astype(np.uint8), sc.intersect_p(sub)), k
        del sc
    assert total_hits > 10000
    plan.close()
    aplan.close()


def test_batched_rejects_host_buffers_and_kdtrees(ctx, scenes):
    import torch
    s = scenes[0]
    kd = rb.GpuKdTreeAccel(ctx, [rb.TriangleMesh(ctx, s["xyz"], s["idx"])])
    out = torch.zeros(len(s["rays"]) * 16, dtype=torch.uint8, device="cuda")
    with pytest.raises(rb.IllumeError):
        bt.BatchPlan(ctx, [(kd, device(s["rays"]), out)])
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, s["xyz"], s["idx"])], width=2)
    with pytest.raises(rb.IllumeError):
        bt.BatchPlan(ctx, [(acc, s["rays"], out)])


def test_batched_mixed_widths_and_stack_depths(ctx, scenes):
    """One plan over accels of widths 2, 4 and 8, some set to a 32-entry stack:
    every batch gives the single-scene entry point's records byte for byte
    (closest and any hit) and a sample matches the oracle
    (accelerators/bvh.rs:563-662; binary layout bvh.rs:665-673)."""
    import torch
    accs, entries, any_entries, outs, occs = [], [], [], [], []
    for k, s in enumerate(scenes):
        width = (2, 4, 8)[k % 3]
        acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, s["xyz"], s["idx"])], width=width)
        if width != 2 and k % 2:
            bt.apply_launch(acc, {"stack_depth": 32, "schedule": "persistent", "high_occupancy": True})
        accs.append(acc)
        d_rays = device(s["rays"])
        out = torch.zeros(len(s["rays"]) * 16, dtype=torch.uint8, device="cuda")
        occ = torch.zeros(len(s["rays"]), dtype=torch.int32, device="cuda")
        outs.append(out)
        occs.append(occ)
        entries.append((acc, d_rays, out))
        any_entries.append((acc, d_rays, occ))
    plan = bt.BatchPlan(ctx, entries)
    aplan = bt.BatchPlan(ctx, any_entries, any_hit=True)
    plan.launch()
    aplan.launch()
    torch.cuda.synchronize()
    for k, s in enumerate(scenes):
        got = outs[k].cpu().numpy()
        assert got.tobytes() == accs[k].intersect_batch(s["rays"]).tobytes(), k
        assert np.array_equal(occs[k].cpu().numpy().view(np.uint32), accs[k].intersect_p_batch(s["rays"])), k
        sc = oracle.Scene(s["xyz"], s["idx"])
        pick = np.sort(np.random.default_rng(50 + k).choice(len(s["rays"]), 2000, replace=False))
        compare_closest(got.view(rb.HIT_DTYPE)[pick], sc.intersect(np.ascontiguousarray(s["rays"][pick])),
                        label=f"mixed {k}")
    assert ctx.device_errors() == 0
    plan.close()
    aplan.close()


def test_tuned_plan_sweeps_widths(ctx, scenes):
    """tuned_plan: each scene autotuned over widths 2/4/8, stack depths and
    schedules; the plan's records equal the tuned accels' own queries."""
    import torch
    items, outs = [], []
    for s in scenes[:4]:
        out = torch.zeros(len(s["rays"]) * 16, dtype=torch.uint8, device="cuda")
        outs.append(out)
        items.append(([rb.TriangleMesh(ctx, s["xyz"], s["idx"])], s["rays"], device(s["rays"]), out))
    plan, accs, choices = bt.tuned_plan(ctx, items, sample_rays=8192)
    plan.launch()
    torch.cuda.synchronize()
    for k, s in enumerate(scenes[:4]):
        assert choices[k]["width"] in (2, 4, 8) and choices[k]["n_tried"] >= 3
        assert outs[k].cpu().numpy().tobytes() == accs[k].intersect_batch(s["rays"]).tobytes()
    plan.close()


def test_autotune_picks_a_valid_choice_and_caches(ctx):
    xyz, idx = wl.icosphere(6, 2)
    rays = wl.ball_rays(2, 4, 1 << 18, 1 << 17)
    mesh = rb.TriangleMesh(ctx, xyz, idx)
    r1 = bt.autotune(ctx, [mesh], rays)
    assert r1["width"] in (2, 4, 8) and r1["n_tried"] == 13 and not r1["from_cache"]
    assert r1["ms"] <= r1["baseline_ms"] * 1.05
    r2 = bt.autotune(ctx, [mesh], rays)
    assert r2["from_cache"] and r2["width"] == r1["width"]
    acc, choice = bt.tuned_accel(ctx, [mesh], rays)
    ref = rb.GpuBVHAccel(ctx, [mesh], width=8)
    compare_closest(acc.intersect_batch(rays), ref.intersect_batch(rays), label="tuned vs default")

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


def test_batched_rejects_host_buffers_and_binary_width(ctx, scenes):
    import torch
    s = scenes[0]
    acc2 = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, s["xyz"], s["idx"])], width=2)
    out = torch.zeros(len(s["rays"]) * 16, dtype=torch.uint8, device="cuda")
    with pytest.raises(rb.IllumeError):
        bt.BatchPlan(ctx, [(acc2, device(s["rays"]), out)])


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

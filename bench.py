#!/usr/bin/env python
"""Benchmark: closest-hit Mrays/s on the incoherent workload.

Workload (one step = one pass of the hot path over one batch):
  displaced icosphere, subdivision level 8 (1,310,720 triangles, seed 2), SAH
  BVH with max_prims_in_node = 4; 4,194,304 rays from a radius-3 ball with
  uniform directions; the first 2,097,152 (tmax = inf) are the closest-hit
  batch of a step, the other 2,097,152 (tmax ~ U[0.1, 4]) the any-hit batch
  reported beside it.

Lines printed (rank 0, one JSON line):
  value     device-resident rays and hits, CUDA-event time of the traversal
            launches on the launching stream, L2 flushed between steps.
  e2e       the same metric through the public C ABI with pinned HOST buffers
            (host->device copy of the rays and device->host copy of the hits
            inside the timed region).
  roofline  algorithmic bytes per ray = 32 (ray) + 16 (hit) + 32*N_node +
            36*N_tri, with N_node / N_tri the CPU oracle's mean node visits and
            triangle tests per ray on its binary SAH BVH for the same rays.
  cpu_baseline  the CPU oracle (scalar C++ restatement of BVHAccel::intersect)
            on all host threads, same rays.
Further keys, one per workload of the path (each skippable):
  coherent      32,768-triangle soup with 256x256 primary rays, L2-resident:
                closest-hit Mrays/s against the L2 copy bandwidth measured in
                the same run and the HBM peak.
  path_tracer   wavefront path tracer, Cornell box with the level-6 icosphere
                (81,920 + 34 triangles), 1024x1024, 64 spp stratified, max depth
                8, Russian roulette from depth 3: rays/s and paths/s, with the
                CPU path-tracing oracle timed on a 256x256 tile beside it.
  neural_cache  the same scene with the radiance cache: 1-spp frames at
                1024x1024 after 200 frames of online training; relMSE per frame
                against a 2048-spp plain reference (its own noise removed), and
                the plain tracer's relMSE at the same device time (relMSE(1 spp)
                * t_spp / t_frame); gain = their ratio.  Also the network's
                inference throughput and training-step time.
  kdtree        the kd-tree aggregate (KdTreeAccel) over the headline scene
                and rays: closest-hit and any-hit Mrays/s, build time.
  batched       32 scenes (icospheres and soups, 1k-2M triangles log-uniform)
                with 10k-4M rays each (log-uniform; primary, incoherent, shadow
                thirds), all in one persistent launch per BVH width replayed as
                a CUDA graph: aggregate Mrays/s.
`--impl reference` times the CPU restatement alone (the reference itself is
Rust and cannot be built in this image).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_RAYS = 4194304
N_CLOSEST = 2097152
# Oracle (binary SAH BVH) mean node visits / triangle tests per ray on these
# exact rays; recomputed by the CPU leg of every run as a check.
N_NODE_CLOSEST, N_TRI_CLOSEST = 9.957535, 0.294104
N_NODE_ANY, N_TRI_ANY = 6.984437, 0.182989
BYTES_PER_RAY_CLOSEST = 32 + 16 + 32 * N_NODE_CLOSEST + 36 * N_TRI_CLOSEST
BYTES_PER_RAY_ANY = 32 + 4 + 32 * N_NODE_ANY + 36 * N_TRI_ANY
# DRAM bytes (read + write) of one closest-hit launch on this workload, per
# (width, schedule, occupancy, stack depth): dram__bytes_read.sum +
# dram__bytes_write.sum from an ncu capture of one timed launch after three
# warm-ups (a constant of that capture, not measured by this script).
DRAM_TRAFFIC = {(8, "persistent", "high", 64): 209165312}
TRAFFIC_SOURCE = "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch (captured constant)"
WORKLOAD = ("incoherent closest-hit: displaced icosphere level 8 (1,310,720 tris, seed 2), "
            "2,097,152 closest rays of 4,194,304 ball rays (radius 3, uniform directions)")
# The configuration both arms print (the GPU arm's launch choices go in its
# "launch" key, the CPU arm's threads in its "cpu_baseline" key).
CONFIG = {"workload": WORKLOAD, "accel": "SAH BVH, max_prims_in_node 4, 12 buckets",
          "rays": N_CLOSEST, "l2": "GPU arm: flushed between steps (256 MiB write outside the timed launches)"}
METRIC = "closest-hit Mrays/s"
REF_SPP = 16384   # plain-tracer reference of the radiance-cache comparison
GAIN_REPEATS = 3  # independent radiance-cache runs; the smallest gain is reported
NRC_WARM_FRAMES = 800  # frames of online training before a cache is measured
UNIT = "Mrays/s"


def measured_bf16():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["bf16_tflops"])
    return 1590.0


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    def __init__(self, gpu_index):
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"illume_clocks_{os.getpid()}.csv")
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={gpu_index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) < 9:
                    continue
                try:
                    sm.append(float(p[1]))
                    mx.append(float(p[2]))
                except ValueError:
                    continue
                for k, nm in enumerate(names):
                    if p[5 + k].lower() == "active":
                        reasons.add(nm)
        try:
            os.remove(self.path)
        except OSError:
            pass
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "samples": len(sm),
                "reasons": sorted(reasons)}


def cpu_leg(xyz, idx, rays, threads, steps, warmup):
    """The CPU oracle on the closest-hit batch: Mrays/s with `threads` threads."""
    import oracle
    sc = oracle.Scene(xyz, idx)
    c = np.ascontiguousarray(rays[:N_CLOSEST])
    times = []
    for k in range(warmup + steps):
        sc.intersect(c, threads=threads)
        if k >= warmup:
            times.append(oracle.last_trace_seconds())
    sub = np.ascontiguousarray(c[: 1 << 18])
    _, nv, nt = sc.intersect(sub, threads=threads, counters=True)
    value = len(c) * len(times) / sum(times) / 1e6
    return value, times, float(nv.mean()), float(nt.mean()), sc.build_seconds


def max_over_ranks(values, dist, device):
    """Per-rank timings -> the maximum over ranks (identity on one rank)."""
    if dist is None:
        return list(values)
    import torch
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def replica_throughput(units_per_rank, world, steps, seconds):
    """Whole-job throughput of `world` replicas, each doing units_per_rank per
    step for `steps` steps, timed as the max over ranks (weak scaling)."""
    return world * units_per_rank * steps / seconds


def relmse_fn(ref, var_ref, eps=0.01):
    def f(x):   # the reference's own noise removed: E[(x - ref)^2] = MSE(x) + Var(ref)
        return float(np.mean(((x - ref) ** 2 - var_ref) / (ref ** 2 + eps)))
    return f


# Path tracer (Cornell box, level-6 icosphere, 1024^2, 64 spp, depth 8, RR from
# 3): the oracle's binary-BVH node visits / triangle tests per extension and per
# shadow ray over the whole frame (230,301,469 extension and 125,401,721 shadow
# rays at seed 3).
N_NODE_PT_EXT, N_TRI_PT_EXT = 34.141102, 2.438504
N_NODE_PT_SHADOW, N_TRI_PT_SHADOW = 32.574164, 1.002677
# Path-state bytes per extension ray (one path-bounce): the path record written
# by the camera or shade stage (ray 32, throughput + id 16, PCG state 8, path
# id 4 = 60) and what shade reads for it (throughput + id 16, path id 4, PCG
# state 8, hit 16, ray direction 16, triangle 48, material 16 = 124).
S_PT_EXT = 60 + 124
# Per shadow ray: the entry shade writes (ray 32, contribution + id 16) and
# what accumulate reads (flag 4, contribution 16).
S_PT_SHADOW = 48 + 20
BYTES_PT_EXT = 32 + 16 + 32 * N_NODE_PT_EXT + 36 * N_TRI_PT_EXT + S_PT_EXT
BYTES_PT_SHADOW = 32 + 4 + 32 * N_NODE_PT_SHADOW + 36 * N_TRI_PT_SHADOW + S_PT_SHADOW


def path_tracer_leg(rb, wl, ctx, device, steps, cpu):
    """Cornell box, 1024^2, 64 spp, depth 8, RR from 3."""
    xyz, idx, mat, alb, emi = wl.cornell(6, 3)
    cam = wl.CORNELL_CAMERA
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx)], width=8)
    pt = rb.PathTracer(acc, mat, alb, emi, cam["eye"], cam["fov_deg"], 1024, 1024)
    pt.render(4, seed=1)
    secs, rays, nbytes = [], [], []
    for k in range(max(3, min(steps, 5))):
        _, st = pt.render(64, seed=10 + k)
        secs.append(st["seconds"])
        rays.append(st["closest_rays"] + st["shadow_rays"])
        nbytes.append(st["closest_rays"] * BYTES_PT_EXT + st["shadow_rays"] * BYTES_PT_SHADOW)
    t = sum(secs)
    hbm, kind = measured_peaks()
    ach = sum(nbytes) / t / 1e9
    out = {"value": round(sum(rays) / t / 1e6, 2), "unit": "Mrays/s",
           "paths_per_s": round(len(secs) * 1024 * 1024 * 64 / t / 1e6, 2),
           "ms_per_frame": round(1e3 * t / len(secs), 3), "rays_per_path": round(rays[0] / (1024 * 1024 * 64), 3),
           "roofline": {"bound": "hbm", "achieved": round(ach, 1), "peak": hbm, "unit": "GB/s",
                        "frac": round(ach / hbm, 4), "peak_source": f"{kind} hbm_gbs",
                        "bytes_per_extension_ray": round(BYTES_PT_EXT, 2),
                        "bytes_per_shadow_ray": round(BYTES_PT_SHADOW, 2),
                        "state_bytes": {"per_extension_ray": S_PT_EXT, "per_shadow_ray": S_PT_SHADOW}},
           "config": "Cornell box + level-6 icosphere, 1024x1024, 64 spp, depth 8, RR from 3, wave 2^21 paths"}
    if cpu:
        import oracle
        sc = oracle.Scene(xyz, idx)
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        _, (nc, ns) = oracle.render_pt(sc, xyz, idx, mat, alb, emi, cam["eye"], cam["fov_deg"], 1024, 1024, 64,
                                       8, 3, 3, window=(384, 384, 640, 640), threads=threads)
        tc = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": round((nc + ns) / tc / 1e6, 3), "unit": "Mrays/s", "cores": threads,
                               "kind": "port", "sample": "256x256 centre tile of the same frame, 64 spp "
                                                         "(CPU oracle of PathIntegrator)",
                               "paths_per_s": round(256 * 256 * 64 / tc / 1e6, 4)}
    return out


def neural_cache_leg(rb, wl, ctx, torch, dev):
    from rs_illume_b200.nrc import RadianceCache
    res = 1024
    xyz, idx, mat, alb, emi = wl.cornell(6, 3)
    cam = wl.CORNELL_CAMERA
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx)], width=8)
    pt = rb.PathTracer(acc, mat, alb, emi, cam["eye"], cam["fov_deg"], res, res)
    # reference: the mean of 16 renders of REF_SPP / 16 spp (a perfect square,
    # and 2^30 paths per render, within the 32-bit path ids); the spread
    # between them estimates its own variance
    parts = np.stack([pt.render(REF_SPP // 16, seed=1 + k)[0] for k in range(16)])
    ref = parts.mean(axis=0)
    rel = relmse_fn(ref, parts.var(axis=0, ddof=1) / 16)
    pt.render(16, seed=3)
    _, sp = pt.render(16, seed=4)
    t_spp = sp["seconds"] / 16
    r1 = float(np.mean([rel(pt.render(1, seed=20 + k)[0]) for k in range(4)]))
    # independent repeats: a fresh cache (its own initial weights and frame
    # seeds) trained online; 8 frames measured after 200 frames and again
    # after 800, where the per-frame relMSE has settled (it rises over the
    # first few hundred Adam steps, then holds).  The reported gain is the
    # smallest 800-frame gain; the mean-image bias against the reference is
    # reported beside each measurement.
    def measure(cache, seed0):
        rs, ts, qs, mean = [], [], [], 0.0
        for k in range(8):
            img, st = pt.render_nrc(cache, frames=1, seed=seed0 + k)
            rs.append(rel(img))
            ts.append(st["seconds"])
            qs.append(st["queries"])
            mean += float(np.mean(img)) / 8
        r_nrc, t_frame = float(np.mean(rs)), float(np.median(ts))
        r_plain = r1 * t_spp / t_frame
        return {"gain": round(r_plain / r_nrc, 3), "relmse_cache_frame": round(r_nrc, 5),
                "relmse_plain_equal_time": round(r_plain, 5), "ms_per_frame": round(1e3 * t_frame, 3),
                "queries_per_path": round(float(np.mean(qs)) / res / res, 3),
                "mean_bias": round(mean / float(np.mean(ref)) - 1.0, 4)}

    reps, early = [], []
    for rep in range(GAIN_REPEATS):
        cache = RadianceCache(ctx, acc.world_bound(), seed=4 + rep)
        pt.render_nrc(cache, frames=200, seed=9 + 1000 * rep)
        early.append(measure(cache, 100 + 1000 * rep))
        _, sw = pt.render_nrc(cache, frames=NRC_WARM_FRAMES - 208, seed=20000 + 1000 * rep)
        m = measure(cache, 500 + 1000 * rep)
        m["warm_ms_per_frame"] = round(1e3 * sw["seconds"] / sw["frames"], 3)
        reps.append(m)
        if rep + 1 < GAIN_REPEATS:
            cache.close()
    mlp = mlp_leg(rb, ctx, torch, dev, cache)
    cache.close()
    worst = min(reps, key=lambda r: r["gain"])
    return {"gain": worst["gain"], "gain_repeats": [r["gain"] for r in reps],
            "gain_rule": f"smallest of {GAIN_REPEATS} independent repeats (fresh cache trained online over "
                         f"{NRC_WARM_FRAMES} frames, then 8 measured frames)",
            "relmse_cache_frame": worst["relmse_cache_frame"],
            "relmse_plain_equal_time": worst["relmse_plain_equal_time"], "relmse_plain_1spp": round(r1, 5),
            "ms_per_frame": worst["ms_per_frame"], "plain_ms_per_spp": round(1e3 * t_spp, 3),
            "queries_per_path": worst["queries_per_path"], "warm_frames": NRC_WARM_FRAMES,
            "mean_bias": [r["mean_bias"] for r in reps], "repeats": reps,
            "after_200_frames": {"gain_repeats": [r["gain"] for r in early],
                                 "mean_bias": [r["mean_bias"] for r in early]},
            "mlp": mlp,
            "config": f"Cornell box, 1024x1024, 1-spp frames, spread c 0.003, 16384 training paths and "
                      f"2 Adam steps x 32768 samples per frame (lr 1e-2, decoupled weight decay 1.0), "
                      f"one-vertex self-training suffix, "
                      f"reference {REF_SPP} spp"}


def nrc_frame_leg(rb, wl, ctx):
    """Radiance-cache frames alone (profiling): 1024^2, 3 frames of warm-up
    and one timed 1-spp frame."""
    from rs_illume_b200.nrc import RadianceCache
    xyz, idx, mat, alb, emi = wl.cornell(6, 3)
    cam = wl.CORNELL_CAMERA
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx)], width=8)
    pt = rb.PathTracer(acc, mat, alb, emi, cam["eye"], cam["fov_deg"], 1024, 1024)
    cache = RadianceCache(ctx, acc.world_bound(), seed=4)
    pt.render_nrc(cache, frames=3, seed=9)
    _, st = pt.render_nrc(cache, frames=1, seed=10)
    cache.close()
    return {"ms_per_frame": round(1e3 * st["seconds"], 3), "queries": st["queries"],
            "rays": st["closest_rays"] + st["shadow_rays"]}


def mlp_leg(rb, ctx, torch, dev, cache=None):
    """The network alone on device buffers: inference on 1M rows and a
    training step on 16384 rows, CUDA events on a stream of our own.
    FLOP counts are the algorithmic ones (203 inputs, 3 outputs):
    forward 59,136 per row, training 3x forward."""
    from rs_illume_b200.nrc import RadianceCache
    own = cache is None
    if own:
        cache = RadianceCache(ctx, (0.0, 0.0, 0.0, 1.0, 1.0, 1.0), seed=4)
    rows = 1 << 20
    g = torch.Generator(device="cpu").manual_seed(0)
    x = torch.rand(rows, 12, generator=g)
    x[:, 3:9] = torch.nn.functional.normalize(x[:, 3:9].reshape(-1, 2, 3) - 0.5, dim=2).reshape(-1, 6)
    dx = x.to(dev)
    dy = torch.rand(rows, 3, generator=g).to(dev)
    dout = torch.empty(rows, 3, device=dev)
    # a stream of our own: a null stream handle would select the network's stream
    st_ = torch.cuda.Stream(dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    torch.cuda.synchronize()
    for _ in range(3):
        cache.infer(dx, dout, stream=st_)
        cache.train_step(dx[:16384], dy[:16384], stream=st_, with_loss=False)
    ev[0].record(st_)
    for _ in range(10):
        cache.infer(dx, dout, stream=st_)
    ev[1].record(st_)
    for _ in range(10):
        cache.train_step(dx[:16384], dy[:16384], stream=st_, with_loss=False)
    ev[2].record(st_)
    torch.cuda.synchronize()
    t_inf = ev[0].elapsed_time(ev[1]) / 10 / 1e3
    t_train = ev[1].elapsed_time(ev[2]) / 10 / 1e3
    if own:
        cache.close()
    flops_row = 2 * (203 * 64 + 4 * 64 * 64 + 64 * 3)
    peak = measured_bf16()
    inf_tf = rows * flops_row / t_inf / 1e12
    return {"infer_mrows_per_s": round(rows / t_inf / 1e6, 1), "infer_tflops": round(inf_tf, 2),
            "infer_frac": round(inf_tf / peak, 4), "train_step_ms_16384": round(1e3 * t_train, 4),
            "train_tflops": round(3 * 16384 * flops_row / t_train / 1e12, 2),
            "peak_tflops": peak, "flop_per_row_forward": flops_row,
            "kernels": "inference (two 128-row tiles per warpgroup), training forward and backward: tcgen05.mma "
                       "kind::f16 (bf16, FP32 accumulators in TMEM), M 128 N 64 K 16; weight gradients: "
                       "tcgen05.mma kind::f16, MN-major operands, M 128 N 208/64, split-K over the batch rows"}


# Oracle (binary SAH BVH) node visits / triangle tests per ray over all
# 15,697,303 rays of the 32 batched scenes (total over the scenes / total rays).
N_NODE_BATCHED, N_TRI_BATCHED = 25.283230, 0.976951
BYTES_PER_RAY_BATCHED = 32 + 16 + 32 * N_NODE_BATCHED + 36 * N_TRI_BATCHED


def batched_cpu(scenes):
    """The CPU oracle over every scene's rays (all host threads, one pass;
    builds excluded): aggregate Mrays/s."""
    import oracle
    threads = os.cpu_count() or 1
    secs, n = 0.0, 0
    for s in scenes:
        sc = oracle.Scene(s["xyz"], s["idx"])
        sc.intersect(s["rays"], threads=threads)
        secs += oracle.last_trace_seconds()
        n += len(s["rays"])
        del sc
    return {"value": round(n / secs / 1e6, 3), "unit": "Mrays/s", "cores": threads, "kind": "port",
            "sample": f"all {n:,} rays of the 32 scenes, one pass (CPU oracle, binary SAH BVH per scene)"}


def batched_leg(rb, wl, ctx, torch, dev, steps, cpu=False):
    from rs_illume_b200 import batch as bt
    scenes = wl.batched_workload(5, 32)
    t0 = time.perf_counter()
    entries, keep = [], []
    n_rays = 0
    for s in scenes:
        acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, s["xyz"], s["idx"])], width=8)
        d_rays = torch.from_numpy(s["rays"].view(np.uint8)).to(dev)
        out = torch.empty(len(s["rays"]) * 16, dtype=torch.uint8, device=dev)
        entries.append((acc, d_rays, out))
        keep.append((acc, d_rays, out))
        n_rays += len(s["rays"])
    build_s = time.perf_counter() - t0
    plan = bt.BatchPlan(ctx, entries)
    stream = torch.cuda.Stream(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for _ in range(3):
        plan.launch(stream)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    with torch.cuda.stream(stream):
        for a, b in evs:
            flush.zero_()
            a.record(stream)
            plan.launch(stream)
            b.record(stream)
    torch.cuda.synchronize()
    t = sum(a.elapsed_time(b) for a, b in evs) / 1e3
    plan.close()
    hbm, kind = measured_peaks()
    ach = BYTES_PER_RAY_BATCHED * n_rays / (t / steps) / 1e9
    out = {"value": round(n_rays * steps / t / 1e6, 2), "unit": "Mrays/s", "rays_per_step": n_rays,
           "ms_per_step": round(1e3 * t / steps, 3), "scenes": len(scenes),
           "triangles": int(sum(len(s["idx"]) for s in scenes)), "build_seconds": round(build_s, 2),
           "roofline": {"bound": "hbm", "achieved": round(ach, 1), "peak": hbm, "unit": "GB/s",
                        "frac": round(ach / hbm, 4), "peak_source": f"{kind} hbm_gbs",
                        "bytes_per_ray": round(BYTES_PER_RAY_BATCHED, 3),
                        "bytes_rule": "sum over scenes of 32 + 16 + 32 N_node + 36 N_tri (oracle counts per scene)"},
           "config": "32 scenes, 1k-2M triangles and 10k-4M rays per scene (log-uniform), closest-hit, "
                     "width 8, one persistent launch replayed as a CUDA graph, L2 flushed between steps"}
    del keep, entries
    if cpu:
        out["cpu_baseline"] = batched_cpu(scenes)
    return out


N_NODE_COHERENT, N_TRI_COHERENT = 57.515228, 2.256424
BYTES_PER_RAY_COHERENT = 32 + 16 + 32 * N_NODE_COHERENT + 36 * N_TRI_COHERENT


def l2_copy_gbs(torch, dev):
    """Device-to-device copy of 24 MiB (48 MiB of traffic, resident in the
    126 MB L2) timed with CUDA events: the L2 bandwidth this kernel can see."""
    a = torch.empty(24 << 20, dtype=torch.uint8, device=dev)
    b = torch.empty_like(a)
    for _ in range(5):
        b.copy_(a)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(50):
        b.copy_(a)
    e1.record()
    torch.cuda.synchronize()
    return 2 * a.numel() * 50 / (e0.elapsed_time(e1) / 1e3) / 1e9


def coherent_cpu(xyz, idx, rays, passes=40):
    """The CPU oracle on the coherent rays (all host threads, `passes` passes),
    and the distribution of its binary-BVH node visits per ray: the launch is
    as long as its longest rays."""
    import oracle
    sc = oracle.Scene(xyz, idx)
    threads = os.cpu_count() or 1
    times = []
    for k in range(passes + 2):
        sc.intersect(rays, threads=threads)
        if k >= 2:
            times.append(oracle.last_trace_seconds())
    _, nv, _ = sc.intersect(rays, threads=threads, counters=True)
    q = np.percentile(nv, [50, 90, 99, 99.9])
    return ({"value": round(len(rays) * len(times) / sum(times) / 1e6, 3), "unit": "Mrays/s", "cores": threads,
             "kind": "port", "sample": f"all 65,536 rays x {passes} passes (CPU oracle, binary SAH BVH)"},
            {"mean": round(float(nv.mean()), 3), "p50": float(q[0]), "p90": float(q[1]), "p99": float(q[2]),
             "p99_9": float(q[3]), "max": int(nv.max())})


def coherent_leg(rb, wl, ctx, torch, dev, steps, cpu=False):
    """Config 1: 32,768-triangle soup, 256x256 primary rays (scene and rays
    fully L2-resident): closest-hit Mrays/s and its roofline against the L2
    copy bandwidth measured here and the HBM peak."""
    xyz, idx, rays = wl.coherent_workload()
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx)], width=8)
    d_rays = torch.from_numpy(rays.view(np.uint8)).to(dev)
    d_hits = torch.empty(len(rays) * 16, dtype=torch.uint8, device=dev)
    stream = torch.cuda.Stream(dev)
    for _ in range(5):
        acc.intersect_batch(d_rays, d_hits, stream=stream)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for a, b in evs:
        a.record(stream)
        acc.intersect_batch(d_rays, d_hits, stream=stream)
        b.record(stream)
    torch.cuda.synchronize()
    t = sum(a.elapsed_time(b) for a, b in evs) / 1e3 / steps
    l2 = l2_copy_gbs(torch, dev)
    hbm, kind = measured_peaks()
    ach = BYTES_PER_RAY_COHERENT * len(rays) / t / 1e9
    out = {"value": round(len(rays) / t / 1e6, 2), "unit": "Mrays/s", "us_per_launch": round(t * 1e6, 2),
           "roofline": {"bound": "l2", "achieved": round(ach, 1), "unit": "GB/s",
                        "l2_copy_gbs": round(l2, 1), "frac_of_l2": round(ach / l2, 4),
                        "hbm_peak": hbm, "frac_of_hbm": round(ach / hbm, 4),
                        "bytes_per_ray": round(BYTES_PER_RAY_COHERENT, 2)},
           "config": "32,768-triangle soup (seed 1), 65,536 primary rays 256x256 from (0.5,0.5,-1.5), 45 deg, "
                     "width 8; scene and rays L2-resident (no flush: the workload is the L2 case)"}
    if cpu:
        out["cpu_baseline"], out["oracle_node_visits_per_ray"] = coherent_cpu(xyz, idx, rays)
    return out


# Oracle kd-tree (KdTreeAccel defaults 80 / 1 / 0.5 / 1, depth 34) on the same
# scene and rays: mean node visits / primitive tests per ray.
N_NODE_KD_CLOSEST, N_TRI_KD_CLOSEST = 9.904898, 1.864308
N_NODE_KD_ANY, N_TRI_KD_ANY = 7.529678, 0.806322
BYTES_PER_RAY_KD_CLOSEST = 32 + 16 + 8 * N_NODE_KD_CLOSEST + 36 * N_TRI_KD_CLOSEST
BYTES_PER_RAY_KD_ANY = 32 + 4 + 8 * N_NODE_KD_ANY + 36 * N_TRI_KD_ANY


def kdtree_leg(rb, wl, ctx, torch, dev, steps, warmup, scene=None):
    """The kd-tree aggregate on the headline scene and rays: closest-hit and
    any-hit Mrays/s (device buffers, L2 flushed between launches), host build
    time, and the roofline of the closest-hit launch."""
    xyz, idx, rays = scene if scene is not None else wl.incoherent_workload(N_RAYS)
    t0 = time.perf_counter()
    acc = rb.GpuKdTreeAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx)])
    build_s = time.perf_counter() - t0
    info = acc.info()
    d_closest = torch.from_numpy(np.ascontiguousarray(rays[:N_CLOSEST]).view(np.uint8)).to(dev)
    d_shadow = torch.from_numpy(np.ascontiguousarray(rays[N_CLOSEST:]).view(np.uint8)).to(dev)
    d_hits = torch.empty(N_CLOSEST * 16, dtype=torch.uint8, device=dev)
    d_occ = torch.empty(N_CLOSEST, dtype=torch.int32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.Stream(dev)

    def timed(fn):
        with torch.cuda.stream(stream):
            for _ in range(warmup):
                flush.zero_()
                fn()
            evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
            for a, b in evs:
                flush.zero_()
                a.record(stream)
                fn()
                b.record(stream)
        torch.cuda.synchronize(dev)
        return sum(a.elapsed_time(b) for a, b in evs) / 1e3 / steps

    t = timed(lambda: acc.intersect_batch(d_closest, d_hits, stream=stream))
    t_any = timed(lambda: acc.intersect_p_batch(d_shadow, d_occ, stream=stream))
    hbm, kind = measured_peaks()
    ach = BYTES_PER_RAY_KD_CLOSEST * N_CLOSEST / t / 1e9
    return {"value": round(N_CLOSEST / t / 1e6, 2), "unit": "Mrays/s", "ms_per_launch": round(t * 1e3, 4),
            "anyhit": {"value": round(N_CLOSEST / t_any / 1e6, 2), "unit": "Mrays/s",
                       "achieved_gbs": round(BYTES_PER_RAY_KD_ANY * N_CLOSEST / t_any / 1e9, 1)},
            "roofline": {"bound": "hbm", "achieved": round(ach, 1), "peak": hbm, "unit": "GB/s",
                         "frac": round(ach / hbm, 4), "peak_source": f"{kind} hbm_gbs",
                         "bytes_per_ray": round(BYTES_PER_RAY_KD_CLOSEST, 3)},
            "build_seconds": round(build_s, 3), "n_nodes": int(info["n_nodes"]),
            "n_leaf_refs": int(info["n_leaf_refs"]), "max_depth": int(info["max_depth"]),
            "device_bytes": int(info["device_bytes"]),
            "config": "KdTreeAccel 80/1/0.5/1 over the headline scene; the headline's 2,097,152 closest and "
                      "2,097,152 any-hit rays; persistent schedule, 8 blocks of 128 per SM; L2 flushed between "
                      "launches"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle     # the oracle's own generators: this arm never maps the product library
    xyz, idx, rays = oracle.incoherent_workload(N_RAYS)
    threads = os.cpu_count() or 1
    value, times, nn, nt, build_s = cpu_leg(xyz, idx, rays, threads, args.steps, args.warmup)
    sample = (f"all 2,097,152 closest rays per step x {args.steps} steps "
              f"(CPU restatement of BVHAccel::intersect, binary SAH BVH)")
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * sum(times) / len(times), 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded procedural scene and rays)",
        "config": dict(CONFIG),
        "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample, "bvh": "binary SAH (32-byte LinearBVHNode layout)"},
        "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "oracle_counters": {"n_node": round(nn, 4), "n_tri": round(nt, 4)},
        "build_seconds": round(build_s, 3),
    }
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    import rs_illume_b200 as rb
    from rs_illume_b200 import workloads as wl

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    if args.only and args.only != "closest":
        # one workload alone (profiling runs): its key and nothing else, with
        # the launch choices of the full run
        ctx = rb.Context(local, grid_schedule=(args.schedule == "grid"), high_occupancy=(args.occupancy == "high"),
                         stack_depth=args.stack_depth)
        legs = {"pt": ("path_tracer", lambda: path_tracer_leg(rb, wl, ctx, dev, args.steps, False)),
                "nrc": ("neural_cache", lambda: neural_cache_leg(rb, wl, ctx, torch, dev)),
                "mlp": ("neural_cache", lambda: mlp_leg(rb, ctx, torch, dev)),
                "nrcframe": ("neural_cache", lambda: nrc_frame_leg(rb, wl, ctx)),
                "coherent": ("coherent", lambda: coherent_leg(rb, wl, ctx, torch, dev, args.steps)),
                "batched": ("batched", lambda: batched_leg(rb, wl, ctx, torch, dev, args.steps)),
                "kd": ("kdtree", lambda: kdtree_leg(rb, wl, ctx, torch, dev, args.steps, args.warmup))}
        key, fn = legs[args.only]
        res = fn()
        if rank == 0:
            print(json.dumps({"only": args.only, key: res}), flush=True)
        ctx.close()
        return
    xyz, idx, rays = wl.incoherent_workload(N_RAYS)
    ctx = rb.Context(local, grid_schedule=(args.schedule == "grid"), high_occupancy=(args.occupancy == "high"),
                     stack_depth=args.stack_depth)
    t0 = time.perf_counter()
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx)], width=args.width)
    build_s = time.perf_counter() - t0
    info = acc.info()

    closest = np.ascontiguousarray(rays[:N_CLOSEST])
    shadow = np.ascontiguousarray(rays[N_CLOSEST:])
    d_closest = torch.from_numpy(closest.view(np.uint8)).to(dev)
    d_shadow = torch.from_numpy(shadow.view(np.uint8)).to(dev)
    d_hits = torch.empty(N_CLOSEST * 16, dtype=torch.uint8, device=dev)
    d_occ = torch.empty(N_CLOSEST, dtype=torch.int32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.Stream(dev)

    def barrier():
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def timed(fn, steps, warmup, min_warm_s=0.0):
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        t_start = time.perf_counter()
        k = 0
        # at least `warmup` untimed steps, and at least min_warm_s of them so the
        # clock sampler is running under load before the timed region
        while k < warmup or time.perf_counter() - t_start < min_warm_s:
            with torch.cuda.stream(stream):
                flush.zero_()
                fn()
            if k % 8 == 7:
                stream.synchronize()
            k += 1
        barrier()
        with torch.cuda.stream(stream):
            for a, b in evs:
                flush.zero_()                      # L2 flush, outside the events
                a.record(stream)
                fn()
                b.record(stream)
        barrier()
        return [a.elapsed_time(b) for a, b in evs]

    def trace_closest():
        acc.intersect_batch(d_closest, d_hits, stream=stream)

    def trace_any():
        acc.intersect_p_batch(d_shadow, d_occ, stream=stream)

    sampler = ClockSampler(local) if rank == 0 and not args.no_clocks else None
    ms = timed(trace_closest, args.steps, args.warmup, min_warm_s=1.0 if sampler else 0.0)
    clocks = sampler.stop() if sampler else None
    ms_any = timed(trace_any, args.steps, args.warmup)

    # e2e through the public API with pinned host buffers
    h_rays = torch.from_numpy(closest.view(np.uint8)).pin_memory()
    h_hits = torch.empty(N_CLOSEST * 16, dtype=torch.uint8).pin_memory()
    np_rays = h_rays.numpy().view(rb.RAY_DTYPE)
    np_hits = h_hits.numpy().view(rb.HIT_DTYPE)
    e2e_s = []
    for k in range(args.warmup + args.steps):
        flush.zero_()
        barrier()
        t = time.perf_counter()
        acc.intersect_batch(np_rays, np_hits)
        t = time.perf_counter() - t
        if k >= args.warmup:
            e2e_s.append(t)
    barrier()
    err = ctx.device_errors()
    # the host link alone: plain pinned copies of the same bytes, for context
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    link = []
    for _ in range(3):
        ev[0].record(stream)
        with torch.cuda.stream(stream):
            d_closest.copy_(h_rays, non_blocking=True)
            ev[1].record(stream)
            h_hits.copy_(d_hits, non_blocking=True)
            ev[2].record(stream)
        stream.synchronize()
        link.append((ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])))
    h2d_ms = min(x[0] for x in link)
    d2h_ms = min(x[1] for x in link)

    tot, tot_any, tot_e2e = max_over_ranks([sum(ms) / 1e3, sum(ms_any) / 1e3, sum(e2e_s)], dist, dev)

    if rank == 0:
        value = replica_throughput(N_CLOSEST, world, args.steps, tot) / 1e6
        any_value = replica_throughput(N_CLOSEST, world, args.steps, tot_any) / 1e6
        e2e_value = replica_throughput(N_CLOSEST, world, args.steps, tot_e2e) / 1e6
        peak, peak_kind = measured_peaks()
        avg_launch = tot / args.steps
        achieved = BYTES_PER_RAY_CLOSEST * N_CLOSEST / avg_launch / 1e9
        traffic = DRAM_TRAFFIC.get((args.width, args.schedule, args.occupancy, args.stack_depth))
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1e3 * tot / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded procedural scene and rays)",
            "config": dict(CONFIG),
            "launch": {"bvh_width": args.width, "schedule": args.schedule, "occupancy": args.occupancy,
                       "stack_depth": args.stack_depth,
                       "parallelism": "replicas" if world > 1 else "single GPU"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic,
                         "traffic_source": TRAFFIC_SOURCE if traffic else None,
                         "peak_source": f"{peak_kind} hbm_gbs",
                         "bytes_per_ray": round(BYTES_PER_RAY_CLOSEST, 3)},
            "e2e": {"value": round(e2e_value, 3), "unit": UNIT, "h2d_bytes_per_step": N_CLOSEST * 32,
                    "d2h_bytes_per_step": N_CLOSEST * 16,
                    "pcie_h2d_gbs": round(N_CLOSEST * 32 / h2d_ms / 1e6, 1),
                    "pcie_d2h_gbs": round(N_CLOSEST * 16 / d2h_ms / 1e6, 1),
                    "link_bound_mrays_s": round(N_CLOSEST / max(h2d_ms, d2h_ms) / 1e3, 1)},
            "gpu_launches": args.steps,
            "clocks": clocks,
            "anyhit": {"value": round(any_value, 3), "unit": UNIT, "rays": N_CLOSEST,
                       "ms_per_step": round(1e3 * tot_any / args.steps, 4),
                       "achieved_gbs": round(BYTES_PER_RAY_ANY * N_CLOSEST / (tot_any / args.steps) / 1e9, 1)},
            "build_seconds": round(build_s, 3), "device_bytes": int(info["device_bytes"]),
            "device_error_flags": err,
        }
        if world == 1 and not args.no_cpu:
            threads = os.cpu_count() or 1
            cv, ct, nn, nt, _ = cpu_leg(xyz, idx, rays, threads, 3, 1)
            line["cpu_baseline"] = {"value": round(cv, 3), "unit": UNIT, "cores": threads, "kind": "port",
                                    "sample": "all 2,097,152 closest rays x 3 passes (CPU oracle, binary SAH BVH)",
                                    "n_node_sample": round(nn, 4), "n_tri_sample": round(nt, 4)}
        for key, enabled, fn in (
                ("coherent", not args.only,
                 lambda: coherent_leg(rb, wl, ctx, torch, dev, args.steps, world == 1 and not args.no_cpu)),
                ("kdtree", not args.no_kd and not args.only,
                 lambda: kdtree_leg(rb, wl, ctx, torch, dev, args.steps, args.warmup, (xyz, idx, rays))),
                ("path_tracer", not args.no_pt and not args.only,
                 lambda: path_tracer_leg(rb, wl, ctx, dev, args.steps, world == 1 and not args.no_cpu)),
                ("neural_cache", not args.no_nrc and not args.only, lambda: neural_cache_leg(rb, wl, ctx, torch, dev)),
                ("batched", not args.no_batched and not args.only,
                 lambda: batched_leg(rb, wl, ctx, torch, dev, args.steps, world == 1 and not args.no_cpu))):
            if not enabled:
                continue
            try:
                line[key] = fn()
            except Exception as ex:     # a failed leg is reported, not hidden
                line[key] = {"error": f"{type(ex).__name__}: {ex}"}
        line["gpu_launches"] = args.steps
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--width", type=int, default=8, choices=[2, 4, 8])
    ap.add_argument("--schedule", default="persistent", choices=["persistent", "grid"])
    ap.add_argument("--occupancy", default="high", choices=["high", "default"],
                    help="high: persistent kernel compiled for 7 resident blocks per SM (72 registers)")
    ap.add_argument("--stack-depth", type=int, default=64, choices=[32, 64])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-clocks", action="store_true", help="skip nvidia-smi clock sampling (profiler runs)")
    ap.add_argument("--no-pt", action="store_true", help="skip the path-tracer workload")
    ap.add_argument("--no-nrc", action="store_true", help="skip the radiance-cache workload")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched multi-scene workload")
    ap.add_argument("--no-kd", action="store_true", help="skip the kd-tree workload")
    ap.add_argument("--only", choices=["closest", "coherent", "pt", "nrc", "nrcframe", "mlp", "batched", "kd"],
                    help="run one workload alone (profiling)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

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
`--impl reference` times that CPU restatement alone (the reference itself is
Rust and cannot be built in this image).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
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
# DRAM bytes (read + write) of one closest-hit launch on this workload, from the
# ncu capture summarised in profiles/closest_incoherent_w8.md, per
# (width, schedule, occupancy, stack depth).
DRAM_TRAFFIC = {(8, "persistent", "high", 64): 256464896}
WORKLOAD = ("incoherent closest-hit: displaced icosphere level 8 (1,310,720 tris, seed 2), "
            "2,097,152 closest rays of 4,194,304 ball rays (radius 3, uniform directions)")
METRIC = "closest-hit Mrays/s"
UNIT = "Mrays/s"


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
        self.path = os.path.join(ROOT, "gpurun_out" if os.path.isdir(os.path.join(ROOT, "gpurun_out")) else "",
                                 f".clocks_{os.getpid()}.csv")
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


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from rs_illume_b200 import workloads as wl
    xyz, idx, rays = wl.incoherent_workload(N_RAYS)
    threads = os.cpu_count() or 1
    value, times, nn, nt, build_s = cpu_leg(xyz, idx, rays, threads, args.steps, args.warmup)
    sample = (f"all 2,097,152 closest rays per step x {args.steps} steps "
              f"(CPU restatement of BVHAccel::intersect, binary SAH BVH)")
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * sum(times) / len(times), 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded procedural scene and rays)",
        "config": {"workload": WORKLOAD, "bvh": "binary SAH, max_prims_in_node 4", "threads": threads},
        "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample},
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

    tot = sum(ms) / 1e3
    tot_any = sum(ms_any) / 1e3
    tot_e2e = sum(e2e_s)
    if dist is not None:
        t = torch.tensor([tot, tot_any, tot_e2e], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tot, tot_any, tot_e2e = t.tolist()

    if rank == 0:
        value = world * N_CLOSEST * args.steps / tot / 1e6
        any_value = world * N_CLOSEST * args.steps / tot_any / 1e6
        e2e_value = world * N_CLOSEST * args.steps / tot_e2e / 1e6
        peak, peak_kind = measured_peaks()
        avg_launch = tot / args.steps
        achieved = BYTES_PER_RAY_CLOSEST * N_CLOSEST / avg_launch / 1e9
        traffic = DRAM_TRAFFIC.get((args.width, args.schedule, args.occupancy, args.stack_depth))
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1e3 * tot / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded procedural scene and rays)",
            "config": {"workload": WORKLOAD, "bvh_width": args.width, "max_prims_in_node": 4,
                       "schedule": args.schedule, "occupancy": args.occupancy,
                       "stack_depth": args.stack_depth,
                       "l2": "flushed between steps (256 MiB write outside the timed launches)",
                       "parallelism": "replicas" if world > 1 else "single GPU"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic,
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
                    help="high: persistent kernel compiled for 8 resident blocks per SM (64 registers)")
    ap.add_argument("--stack-depth", type=int, default=64, choices=[32, 64])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-clocks", action="store_true", help="skip nvidia-smi clock sampling (profiler runs)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

"""Batched multi-scene queries and the autotuner (include/illume_gpu.h).

``BatchPlan`` traces many scenes' ray batches of uneven sizes in one
persistent launch per BVH width (2, 4, 8) and stack depth, captured once as a
CUDA graph and replayed; ``tuned_plan`` autotunes every scene first.
``autotune`` times BVH width, stack depth, schedule and occupancy variant on
a sample of rays and returns the fastest; ``tuned_accel`` builds the accel
with that choice applied.  Tuning results are cached in the context and can
be kept across processes with ``save_cache`` / ``load_cache`` (JSON keyed by
GPU name, query kind and size buckets).
"""
from __future__ import annotations

import ctypes
import json
import math
import os
from typing import Sequence

from . import _lib
from ._lib import ilm_batch_desc, ilm_launch_opts, ilm_tune_result, ptr
from .primitive import Context, GpuBVHAccel


def _ray_count(rays) -> int:
    """32-byte ray records in a RAY_DTYPE numpy array or a torch tensor (the
    C ABI refuses host buffers; they are counted so that it can)."""
    if hasattr(rays, "numel"):
        return rays.numel() * rays.element_size() // 32
    return rays.nbytes // 32


class BatchPlan:
    """entries: sequence of (GpuBVHAccel, device rays, device output) where the
    output holds 16-byte hits (closest) or uint32 flags (any_hit)."""

    def __init__(self, ctx: Context, entries: Sequence, any_hit: bool = False):
        self.ctx = ctx
        self.any_hit = any_hit
        descs = (ilm_batch_desc * len(entries))()
        self.total_rays = 0
        for k, (acc, rays, out) in enumerate(entries):
            n = _ray_count(rays)
            descs[k].accel = acc.id
            descs[k].rays = ptr(rays)
            descs[k].n = n
            descs[k].hits = None if any_hit else ptr(out)
            descs[k].occluded = ptr(out) if any_hit else None
            self.total_rays += n
        self._descs = descs
        h = ctypes.c_void_p()
        ctx.check(ctx._lib.ilm_batch_plan_create(ctx.handle, ctypes.addressof(descs), len(entries), int(any_hit),
                                                 ctypes.byref(h)), "ilm_batch_plan_create")
        self.handle = h

    def launch(self, stream=None) -> None:
        s = None if stream is None else (stream if isinstance(stream, int) else stream.cuda_stream)
        self.ctx.check(self.ctx._lib.ilm_batch_plan_launch(self.ctx.handle, self.handle, s), "ilm_batch_plan_launch")

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.ctx._lib.ilm_batch_plan_destroy(self.ctx.handle, self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune(ctx: Context, shapes: Sequence, sample, any_hit: bool = False, force: bool = False) -> dict:
    ids = (ctypes.c_uint32 * len(shapes))(*[s.id for s in shapes])
    n = len(sample) if hasattr(sample, "dtype") and sample.dtype == _lib.RAY_DTYPE else \
        sample.numel() * sample.element_size() // 32
    r = ilm_tune_result()
    ctx.check(ctx._lib.ilm_autotune(ctx.handle, ids, len(shapes), ptr(sample), n, int(any_hit), int(force),
                                    ctypes.byref(r)), "ilm_autotune")
    return {"width": r.width, "stack_depth": r.launch.stack_depth, "schedule": "grid" if r.launch.schedule else
            "persistent", "high_occupancy": bool(r.launch.high_occupancy), "ms": r.ms, "baseline_ms": r.baseline_ms,
            "n_tried": r.n_tried, "from_cache": bool(r.from_cache)}


def apply_launch(acc: GpuBVHAccel, choice: dict) -> None:
    o = ilm_launch_opts(choice["stack_depth"], 1 if choice["schedule"] == "grid" else 0,
                        int(choice["high_occupancy"]))
    acc.ctx.check(acc.ctx._lib.ilm_accel_set_launch(acc.ctx.handle, acc.id, ctypes.byref(o)), "ilm_accel_set_launch")


def tuned_accel(ctx: Context, shapes: Sequence, sample, any_hit: bool = False, cache_path: str | None = None):
    """Autotunes (or reads the JSON cache) and returns (accel, choice)."""
    key = cache_key(shapes, sample, any_hit)
    choice = load_cache(cache_path).get(key) if cache_path else None
    if choice is None:
        choice = autotune(ctx, shapes, sample, any_hit)
        if cache_path:
            save_cache(cache_path, {key: choice})
    acc = GpuBVHAccel(ctx, shapes, width=choice["width"])
    if choice["width"] != 2:
        apply_launch(acc, choice)
    return acc, choice


def tuned_plan(ctx: Context, scenes: Sequence, any_hit: bool = False, sample_rays: int = 1 << 16,
               cache_path: str | None = None):
    """Autotunes every scene on a sample of its rays and builds one plan over
    all of them: scenes: sequence of (shapes, host rays RAY_DTYPE, device rays,
    device output).  Each accel gets its own width (2, 4 or 8) and launch
    choices; the plan groups the scenes by width and stack depth, one
    persistent launch per group.  Returns (plan, accels, choices)."""
    accs, choices, entries = [], [], []
    for shapes, host_rays, d_rays, out in scenes:
        step = max(1, len(host_rays) // sample_rays)
        sample = host_rays[::step][:sample_rays].copy()
        acc, choice = tuned_accel(ctx, shapes, sample, any_hit, cache_path)
        accs.append(acc)
        choices.append(choice)
        entries.append((acc, d_rays, out))
    return BatchPlan(ctx, entries, any_hit), accs, choices


def cache_key(shapes, sample, any_hit: bool) -> str:
    try:
        import torch
        gpu = torch.cuda.get_device_name(0)
    except Exception:
        gpu = "unknown"
    prims = sum(s.n_prims for s in shapes)
    n = len(sample) if hasattr(sample, "dtype") and sample.dtype == _lib.RAY_DTYPE else \
        sample.numel() * sample.element_size() // 32
    return f"{gpu}|{'any' if any_hit else 'closest'}|p{int(math.log2(max(prims, 1)))}|r{int(math.log2(max(n, 1)))}"


def load_cache(path: str | None) -> dict:
    if not path or not os.path.exists(path):
        return {}
    with open(path) as f:
        return json.load(f)


def save_cache(path: str, entries: dict) -> None:
    data = load_cache(path)
    data.update(entries)
    with open(path, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)

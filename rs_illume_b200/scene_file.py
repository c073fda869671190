"""pbrt-v3 scene files on the GPU path (ilm_scene_file_*).

The reference parses these files to a syntax tree (parse_to_ast,
core/parser/mod.rs:19-34) and stops there (core/parser/mod.rs:36-46); this
module loads them into the shapes, materials, camera and render settings that
the B200 accelerators and path tracer take.  `syntax` returns the directive
tree itself, read by the loader's own tokenizer and argument grammar.
"""
from __future__ import annotations

import ctypes
import json
from typing import Optional

import numpy as np

from . import _lib
from ._lib import IllumeError, ptr
from .primitive import Context, GpuBVHAccel, GpuKdTreeAccel, PathTracer


def syntax(text: str, base_dir: str = "") -> dict:
    """The directive tree of `text` without running it (ilm_scene_syntax):
    {"directives": [...], "comments": [...]}, each directive a dict with
    "directive", "file", "line", "num", "str", "params" and, for blocks,
    "children".  Raises IllumeError on a syntax error."""
    lib = _lib.load()
    err = ctypes.create_string_buffer(1024)
    n = ctypes.c_size_t()
    src, base = text.encode(), base_dir.encode()
    st = lib.ilm_scene_syntax(src, base, None, 0, ctypes.byref(n), err, len(err))
    if st != 0:
        raise IllumeError(st, "reading scene syntax", err.value.decode(errors="replace"))
    buf = ctypes.create_string_buffer(n.value + 1)
    st = lib.ilm_scene_syntax(src, base, buf, len(buf), ctypes.byref(n), err, len(err))
    if st != 0:
        raise IllumeError(st, "reading scene syntax", err.value.decode(errors="replace"))
    return json.loads(buf.raw[:n.value].decode())


class SceneFile:
    """A loaded scene file: geometry in world space and its settings."""

    def __init__(self, handle: int):
        self._lib = _lib.load()
        self.handle = handle
        inf = _lib.ilm_scene_file_info()
        self._lib.ilm_scene_file_info_get(handle, ctypes.byref(inf))
        self.info = inf

    @classmethod
    def load(cls, path: str) -> "SceneFile":
        return cls._open(lambda lib, err, h: lib.ilm_scene_file_load(path.encode(), err, len(err), h), path)

    @classmethod
    def parse(cls, text: str, base_dir: str = "") -> "SceneFile":
        return cls._open(lambda lib, err, h: lib.ilm_scene_file_parse(text.encode(), base_dir.encode(), err,
                                                                      len(err), h), "<text>")

    @classmethod
    def _open(cls, call, what):
        lib = _lib.load()
        err = ctypes.create_string_buffer(1024)
        h = ctypes.c_void_p()
        st = call(lib, err, ctypes.byref(h))
        if st != 0:
            raise IllumeError(st, f"loading scene file {what}", err.value.decode(errors="replace"))
        return cls(h.value)

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.ilm_scene_file_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    # -- contents ----------------------------------------------------------
    @property
    def warnings(self) -> list:
        text = self._lib.ilm_scene_file_warnings(self.handle).decode()
        return [w for w in text.split("\n") if w]

    def mesh(self, k: int) -> dict:
        """Triangle mesh k: xyz, idx, and n / s / uv (None when absent), material."""
        nv, nt = ctypes.c_uint32(), ctypes.c_uint32()
        self._check(self._lib.ilm_scene_file_mesh(self.handle, k, ctypes.byref(nv), ctypes.byref(nt), *([None] * 9)))
        xyz = np.zeros((nv.value, 3), np.float32)
        idx = np.zeros((nt.value, 3), np.uint32)
        n = np.zeros((nv.value, 3), np.float32)
        s = np.zeros((nv.value, 3), np.float32)
        uv = np.zeros((nv.value, 2), np.float32)
        hn, hs, huv, mat = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32(), ctypes.c_uint32()
        self._check(self._lib.ilm_scene_file_mesh(self.handle, k, None, None, ptr(xyz), ptr(idx), ptr(n), ptr(s),
                                                  ptr(uv), ctypes.byref(hn), ctypes.byref(hs), ctypes.byref(huv),
                                                  ctypes.byref(mat)))
        return {"xyz": xyz, "idx": idx, "n": n if hn.value else None, "s": s if hs.value else None,
                "uv": uv if huv.value else None, "material": mat.value}

    def quadrics(self):
        """(list of ilm_sphere_desc, material index per quadric)."""
        n = self.info.n_quadrics
        arr = (_lib.ilm_sphere_desc * max(1, n))()
        mat = np.zeros(n, np.uint32)
        self._check(self._lib.ilm_scene_file_quadrics(self.handle, ctypes.addressof(arr), ptr(mat)))
        return list(arr)[:n], mat

    def curves(self):
        """(list of ilm_curve_desc segments, material index per segment)."""
        n = self.info.n_curves
        arr = (_lib.ilm_curve_desc * max(1, n))()
        mat = np.zeros(n, np.uint32)
        self._check(self._lib.ilm_scene_file_curves(self.handle, ctypes.addressof(arr), ptr(mat)))
        return list(arr)[:n], mat

    def materials(self):
        """(albedo[m, 3], emission[m, 3])."""
        m = self.info.n_materials
        alb = np.zeros((m, 3), np.float32)
        emi = np.zeros((m, 3), np.float32)
        self._check(self._lib.ilm_scene_file_materials(self.handle, ptr(alb), ptr(emi)))
        return alb, emi

    def camera(self) -> dict:
        i = self.info
        return {"eye": np.array(i.eye[:], np.float32),
                "camera_to_world": np.array(i.camera_to_world[:], np.float32).reshape(3, 3),
                "fov_deg": i.fov_deg, "width": i.width, "height": i.height}

    # -- GPU ---------------------------------------------------------------
    def build(self, ctx: Context):
        """Uploads the shapes and builds the file's accelerator; returns
        (accel, PathTracer or None).  The path tracer needs triangles only."""
        aid, pid = ctypes.c_uint32(), ctypes.c_uint32()
        ctx.check(self._lib.ilm_scene_file_build(ctx.handle, self.handle, ctypes.byref(aid), ctypes.byref(pid)),
                  "ilm_scene_file_build")
        cls = GpuKdTreeAccel if self.info.accelerator == 1 else GpuBVHAccel
        acc = cls.__new__(cls)
        acc.ctx, acc.id = ctx, aid.value
        acc.width = _lib.ILM_LAYOUT_KDTREE if self.info.accelerator == 1 else self.info.bvh.width
        acc.n_prims = self.info.n_triangles + self.info.n_quadrics + self.info.n_curves
        pt: Optional[PathTracer] = None
        if pid.value:
            pt = PathTracer.__new__(PathTracer)
            pt.accel, pt.id = acc, pid.value
            pt.width, pt.height = self.info.width, self.info.height
        return acc, pt

    def render(self, pt: PathTracer, seed: int = 3, **kw):
        """Renders with the file's sampler and integrator settings (spp,
        maxdepth, pixel filter); keyword arguments override them."""
        i = self.info
        opts = dict(spp=i.spp, max_depth=i.max_depth, seed=seed, filter=i.filter)
        opts.update(kw)
        return pt.render(**opts)

    def _check(self, st):
        if st != 0:
            raise IllumeError(st, "scene file")

"""Film output and film filters (include/illume_gpu.h: ilm_write_pfm,
ilm_read_pfm, ilm_filter_evaluate, ilm_filter_table).  Host-only: no context
or GPU is needed."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import IllumeError, ptr

FILTERS = {"box": 0, "triangle": 1, "gaussian": 2, "mitchell": 3, "lanczos": 4}
TABLE_WIDTH = 16


def _check(st: int, where: str) -> None:
    if st != _lib.ILM_OK:
        raise IllumeError(st, where)


def write_pfm(path: str, rgb: np.ndarray) -> None:
    """rgb: (height, width, 3) float32, row 0 at the top (write_image_pfm,
    core/imageio.rs:264-310)."""
    rgb = np.ascontiguousarray(rgb, np.float32)
    h, w = rgb.shape[:2]
    _check(_lib.load().ilm_write_pfm(path.encode(), ptr(rgb), w, h), "ilm_write_pfm")


def read_pfm(path: str) -> np.ndarray:
    lib = _lib.load()
    w, h = ctypes.c_uint32(), ctypes.c_uint32()
    _check(lib.ilm_read_pfm(path.encode(), None, ctypes.byref(w), ctypes.byref(h)), "ilm_read_pfm")
    out = np.empty((h.value, w.value, 3), np.float32)
    _check(lib.ilm_read_pfm(path.encode(), ptr(out), ctypes.byref(w), ctypes.byref(h)), "ilm_read_pfm")
    return out


def filter_desc(kind: str, radius=(0.5, 0.5), a: float = 0.0, b: float = 0.0) -> _lib.ilm_filter_desc:
    """gaussian: a = alpha; mitchell: a = B, b = C; lanczos: a = tau."""
    d = _lib.ilm_filter_desc()
    d.kind = FILTERS[kind]
    d.radius[0], d.radius[1] = radius
    d.a, d.b = a, b
    return d


def filter_evaluate(desc, x: float, y: float) -> float:
    out = ctypes.c_float()
    _check(_lib.load().ilm_filter_evaluate(ctypes.byref(desc), x, y, ctypes.byref(out)), "ilm_filter_evaluate")
    return out.value


def filter_table(desc) -> np.ndarray:
    """The film's 16 x 16 weight table (core/film.rs:70-82)."""
    out = np.empty((TABLE_WIDTH, TABLE_WIDTH), np.float32)
    _check(_lib.load().ilm_filter_table(ctypes.byref(desc), ptr(out)), "ilm_filter_table")
    return out

"""Helpers to build and decode the product's host layouts in tests."""
import ctypes

import numpy as np

from rs_illume_b200 import _lib

WIDE8 = np.dtype([("origin", "<f4", (3,)), ("packed", "<u4"), ("child_base", "<u4"), ("prim_base", "<u4"),
                  ("meta", "u1", (8,)), ("qlo", "u1", (3, 8)), ("qhi", "u1", (3, 8))])
WIDE4 = np.dtype([("origin", "<f4", (3,)), ("packed", "<u4"), ("child_base", "<u4"), ("prim_base", "<u4"),
                  ("meta", "u1", (4,)), ("qlo", "u1", (3, 4)), ("qhi", "u1", (3, 4)), ("pad", "<u4", (3,))])
assert WIDE8.itemsize == 80 and WIDE4.itemsize == 64


def host_layout(xyz, idx, width=8, max_prims=4, spheres=()):
    lib = _lib.load()
    xyz = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
    idx = np.ascontiguousarray(idx, np.uint32).reshape(-1, 3)
    sph = (_lib.ilm_sphere_desc * max(1, len(spheres)))(*spheres)
    h = ctypes.c_void_p()
    opts = _lib.ilm_build_opts(width, max_prims)
    st = lib.ilm_host_layout_build(_lib.ptr(xyz), len(xyz), _lib.ptr(idx), len(idx), ctypes.addressof(sph),
                                   len(spheres), ctypes.byref(opts), ctypes.byref(h))
    if st != 0:
        return st
    inf = _lib.ilm_accel_info()
    lib.ilm_host_layout_info(h, ctypes.byref(inf))
    nb = {2: 32, 4: 64, 8: 80}[width]
    bn = np.zeros(inf.n_binary_nodes, _lib.BIN_NODE_DTYPE)
    po = np.zeros(inf.n_prims, np.uint32)
    nodes = np.zeros(inf.n_nodes * nb, np.uint8)
    recs = np.zeros(inf.n_prims, _lib.PRIM_REC_DTYPE)
    bound = np.zeros(6, np.float32)
    lib.ilm_host_layout_copy(h, _lib.ptr(bn), _lib.ptr(po), _lib.ptr(nodes), _lib.ptr(recs), _lib.ptr(bound))
    lib.ilm_host_layout_destroy(h)
    if width == 8:
        nodes = nodes.view(WIDE8)
    elif width == 4:
        nodes = nodes.view(WIDE4)
    else:
        nodes = nodes.view(_lib.BIN_NODE_DTYPE)
    return {"info": inf, "bin": bn, "order": po, "nodes": nodes, "records": recs, "bound": bound}


def host_kdtree(xyz, idx, spheres=(), threads=0, isect_cost=80, traversal_cost=1, empty_bonus=0.5, max_prims=1,
                max_depth=-1):
    """The product's host-only kd-tree build: (status, dict)."""
    lib = _lib.load()
    xyz = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
    idx = np.ascontiguousarray(idx, np.uint32).reshape(-1, 3)
    sph = (_lib.ilm_sphere_desc * max(1, len(spheres)))(*spheres)
    h = ctypes.c_void_p()
    opts = _lib.ilm_kdtree_opts(isect_cost, traversal_cost, empty_bonus, max_prims, max_depth)
    st = lib.ilm_host_kdtree_build(_lib.ptr(xyz), len(xyz), _lib.ptr(idx), len(idx), ctypes.addressof(sph),
                                   len(spheres), ctypes.byref(opts), threads, ctypes.byref(h))
    if st != 0:
        return st, None
    inf = _lib.ilm_accel_info()
    lib.ilm_host_layout_info(h, ctypes.byref(inf))
    nodes = np.zeros(inf.n_nodes, _lib.KD_NODE_DTYPE)
    index = np.zeros(inf.n_leaf_refs, np.uint32)
    recs = np.zeros(inf.n_prims, _lib.PRIM_REC_DTYPE)
    bound = np.zeros(6, np.float32)
    lib.ilm_host_layout_copy(h, None, None, _lib.ptr(nodes), _lib.ptr(recs), _lib.ptr(bound))
    lib.ilm_host_layout_kd_index(h, _lib.ptr(index))
    lib.ilm_host_layout_destroy(h)
    return 0, {"info": inf, "nodes": nodes, "index": index, "records": recs, "bound": bound}


def dequantised_boxes(node, width):
    """(W, 2, 3) float32 child boxes of one wide node: fma(2^23 + q, 2^(e-127),
    origin), the origin biased by -2^23 * 2^(e-127).  The sum is exact in
    float64, so one cast to float32 rounds as the fma does."""
    ex = [(int(node["packed"]) >> (8 * a)) & 0xFF for a in range(3)]
    out = np.zeros((width, 2, 3), np.float32)
    for a in range(3):
        s = 2.0 ** (ex[a] - 127)
        o = float(node["origin"][a])
        out[:, 0, a] = (o + (8388608.0 + node["qlo"][a].astype(np.float64)) * s).astype(np.float32)
        out[:, 1, a] = (o + (8388608.0 + node["qhi"][a].astype(np.float64)) * s).astype(np.float32)
    return out

"""Loop subdivision surfaces (shapes/loop_subdiv.rs, pbrt-v3's LoopSubdivide).

The product (C++, float32) against the oracle's Python restatement
(oracle/loop_subdiv.py, float64): identical topology and positions / normals
within float32 rounding, on closed meshes of valence 3, 4, 5 and 6, and on
open meshes whose boundary vertices have valence 2, 3, 4 and more; known
answers (counts per level, planar stays planar, the icosahedron's limit points
on one sphere, outward normals); rejected inputs; the scene-file shape."""
import numpy as np
import pytest

import rs_illume_b200 as rb
from oracle.loop_subdiv import loop_subdivide as oracle_loop

T = (1 + 5 ** 0.5) / 2
ICOSA_V = np.array([[-1, T, 0], [1, T, 0], [-1, -T, 0], [1, -T, 0], [0, -1, T], [0, 1, T], [0, -1, -T], [0, 1, -T],
                    [T, 0, -1], [T, 0, 1], [-T, 0, -1], [-T, 0, 1]])
ICOSA_F = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                    [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                    [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]])
OCTA_V = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]])
OCTA_F = np.array([[0, 2, 4], [2, 1, 4], [1, 3, 4], [3, 0, 4], [2, 0, 5], [1, 2, 5], [3, 1, 5], [0, 3, 5]])
TETRA_V = np.array([[1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]])
TETRA_F = np.array([[0, 1, 2], [0, 3, 1], [0, 2, 3], [1, 3, 2]])


def grid(n):
    v = np.array([[x, y, 0.0] for y in range(n) for x in range(n)])
    f = []
    for y in range(n - 1):
        for x in range(n - 1):
            a = y * n + x
            f += [[a, a + 1, a + n + 1], [a, a + n + 1, a + n]]
    return v, np.array(f)


def fan(k):
    """k triangles around a centre on the boundary: centre valence k + 1."""
    ang = np.linspace(0, np.pi * 1.5, k + 1)
    v = np.r_[[[0.0, 0, 0]], np.c_[np.cos(ang), np.sin(ang), 0.3 * np.sin(3 * ang)]]
    return v, np.array([[0, i + 1, i + 2] for i in range(k)])


MESHES = {"icosahedron": (ICOSA_V, ICOSA_F), "octahedron": (OCTA_V, OCTA_F), "tetrahedron": (TETRA_V, TETRA_F),
          "grid": grid(4), "fan1": fan(1), "fan2": fan(2), "fan5": fan(5)}


@pytest.mark.parametrize("name", list(MESHES))
@pytest.mark.parametrize("levels", [0, 1, 2, 3])
def test_product_equals_oracle(name, levels):
    v, f = MESHES[name]
    p, i, n = rb.loop_subdivide(v, f, levels)
    po, io, no = oracle_loop(v, f, levels)
    assert np.array_equal(i, io)
    scale = np.abs(po).max()
    np.testing.assert_allclose(p, po, atol=2e-6 * scale)
    # normals are cross products of one-ring differences: float32 cancellation
    np.testing.assert_allclose(n, no, atol=2e-5 * max(np.abs(no).max(), 1e-12))


def test_known_answers():
    v, f = ICOSA_V, ICOSA_F
    nv, ne, nf = 12, 30, 20
    for lv in range(4):
        p, i, n = rb.loop_subdivide(v, f, lv)
        assert (len(p), len(i)) == (nv, nf)
        nv, ne, nf = nv + ne, 2 * ne + 3 * nf, 4 * nf
    # the icosahedron's limit points: one sphere at level 0 (every vertex alike)
    p, _, n = rb.loop_subdivide(ICOSA_V, ICOSA_F, 0)
    r = np.linalg.norm(p, axis=1)
    assert r.max() - r.min() < 1e-6
    # on a closed, consistently wound mesh the limit normals all face one way
    # (pbrt's ring order makes them point against the faces' winding normal);
    # around the icosahedron's centre they are radial
    for name in ("icosahedron", "octahedron", "tetrahedron"):
        p, i, n = rb.loop_subdivide(*MESHES[name], 2)
        d = np.sum(p * n, axis=1)
        assert np.all(d < 0), name
        fn = np.cross(p[i[:, 1]] - p[i[:, 0]], p[i[:, 2]] - p[i[:, 0]])
        assert np.all(np.sum(fn * p[i].mean(axis=1), axis=1) > 0), name   # faces wound outward
    p, _, n = rb.loop_subdivide(ICOSA_V, ICOSA_F, 3)
    cos = -np.sum(p * n, axis=1) / np.linalg.norm(p, axis=1) / np.linalg.norm(n, axis=1)
    assert cos.min() > 0.995                  # the limit surface is not a sphere, but close
    # a plane stays a plane, normals along z
    p, _, n = rb.loop_subdivide(*grid(5), 2)
    assert np.all(p[:, 2] == 0.0)
    assert np.all(np.abs(n[:, :2]) <= 1e-6 * np.abs(n[:, 2:]))


def test_rejected_inputs():
    v, f = ICOSA_V, ICOSA_F
    with pytest.raises(rb.IllumeError):
        rb.loop_subdivide(v, f, 11)
    with pytest.raises(rb.IllumeError):
        rb.loop_subdivide(v, np.array([[0, 1, 12]]), 1)      # index out of range
    with pytest.raises(rb.IllumeError):
        rb.loop_subdivide(v, np.array([[0, 0, 1]]), 1)       # degenerate triangle
    with pytest.raises(rb.IllumeError):
        rb.loop_subdivide(v, np.zeros((0, 3), np.uint32), 1)
    # a face wound against its neighbours leaves an edge whose two faces disagree
    f2 = f.copy()
    f2[0] = f2[0][::-1]
    with pytest.raises(rb.IllumeError):
        rb.loop_subdivide(v, f2, 1)


def test_scene_file_loopsubdiv():
    pts = " ".join(repr(float(x)) for x in ICOSA_V.reshape(-1))
    ind = " ".join(str(int(x)) for x in ICOSA_F.reshape(-1))
    sf = rb.SceneFile.parse(f'''WorldBegin Translate 1 2 3
        Shape "loopsubdiv" "integer levels" 2 "point P" [ {pts} ] "integer indices" [ {ind} ]
        WorldEnd''')
    m = sf.mesh(0)
    p, i, n = rb.loop_subdivide(ICOSA_V, ICOSA_F, 2)
    np.testing.assert_allclose(m["xyz"], p + [1, 2, 3], rtol=1e-6)
    assert np.array_equal(m["idx"], i)
    np.testing.assert_allclose(m["n"], n, rtol=1e-6)
    assert sf.warnings == []

"""Loop subdivision restated in Python (TEST INFRASTRUCTURE ONLY).

The algorithm of shapes/loop_subdiv.rs, which is pbrt-v3's LoopSubdivide
(the reference file does not compile; its intent is pbrt's): build face /
vertex adjacency with edges keyed by (min, max) vertex; per level, even
vertices by the one-ring rule (beta = 1/16 when regular, else 3/16 for
valence 3 and 3 / (8 valence)) or the boundary rule (1/8), odd vertices by
3/8, 3/8, 1/8, 1/8 (boundary: 1/2, 1/2), children laid out as the book's
refinement step; finally limit positions (one-ring with gamma = 1 / (valence
+ 3 / (8 beta)), boundary 1/5) and normals from the one-ring tangents.
Float64 arithmetic; the product computes in float32.
"""
import math

import numpy as np

NONE = -1


def _next(i):
    return (i + 1) % 3


def _prev(i):
    return (i + 2) % 3


class _Mesh:
    def __init__(self):
        self.p = []          # vertex positions
        self.start = []      # start face per vertex
        self.child = []
        self.regular = []
        self.boundary = []
        self.fv = []         # [v0, v1, v2] per face
        self.ff = []         # neighbours across (v[i], v[i+1])
        self.fc = []         # children

    def add_vertex(self, p, start=NONE, regular=False, boundary=False):
        self.p.append(np.asarray(p, np.float64))
        self.start.append(start)
        self.child.append(NONE)
        self.regular.append(regular)
        self.boundary.append(boundary)
        return len(self.p) - 1

    def add_face(self):
        self.fv.append([NONE] * 3)
        self.ff.append([NONE] * 3)
        self.fc.append([NONE] * 4)
        return len(self.fv) - 1

    def vnum(self, f, v):
        return self.fv[f].index(v)

    def next_face(self, f, v):
        return self.ff[f][self.vnum(f, v)]

    def prev_face(self, f, v):
        return self.ff[f][_prev(self.vnum(f, v))]

    def next_vert(self, f, v):
        return self.fv[f][_next(self.vnum(f, v))]

    def prev_vert(self, f, v):
        return self.fv[f][_prev(self.vnum(f, v))]

    def other_vert(self, f, a, b):
        return [v for v in self.fv[f] if v != a and v != b][0]

    def valence(self, v):
        f = self.start[v]
        if not self.boundary[v]:
            n = 1
            f = self.next_face(f, v)
            while f != self.start[v]:
                n += 1
                f = self.next_face(f, v)
            return n
        n = 1
        f = self.next_face(f, v)
        while f != NONE:
            n += 1
            f = self.next_face(f, v)
        f = self.prev_face(self.start[v], v)
        while f != NONE:
            n += 1
            f = self.prev_face(f, v)
        return n + 1

    def one_ring(self, v):
        out = []
        f = self.start[v]
        if not self.boundary[v]:
            while True:
                out.append(self.p[self.next_vert(f, v)])
                f = self.next_face(f, v)
                if f == self.start[v]:
                    return out
        while self.next_face(f, v) != NONE:
            f = self.next_face(f, v)
        out.append(self.p[self.next_vert(f, v)])
        while f != NONE:
            out.append(self.p[self.prev_vert(f, v)])
            f = self.prev_face(f, v)
        return out


def _beta(valence):
    return 3.0 / 16.0 if valence == 3 else 3.0 / (8.0 * valence)


def _gamma(valence):
    return 1.0 / (valence + 3.0 / (8.0 * _beta(valence)))


def _one_ring_weight(m, v, beta):
    val = m.valence(v)
    ring = m.one_ring(v)
    return (1.0 - val * beta) * m.p[v] + beta * sum(ring)


def _boundary_weight(m, v, beta):
    val = m.valence(v)
    ring = m.one_ring(v)
    return (1.0 - 2.0 * beta) * m.p[v] + beta * ring[0] + beta * ring[val - 1]


def loop_subdivide(xyz, idx, levels):
    """(positions[nv, 3], indices[nt, 3], normals[nv, 3]) in float64."""
    xyz = np.asarray(xyz, np.float64).reshape(-1, 3)
    idx = np.asarray(idx, np.int64).reshape(-1, 3)
    m = _Mesh()
    for p in xyz:
        m.add_vertex(p)
    for tri in idx:
        f = m.add_face()
        for j in range(3):
            m.fv[f][j] = int(tri[j])
            m.start[int(tri[j])] = f
    open_edges = {}
    for f in range(len(m.fv)):
        for e in range(3):
            a, b = m.fv[f][e], m.fv[f][_next(e)]
            key = (min(a, b), max(a, b))
            if key not in open_edges:
                open_edges[key] = (f, e)
            else:
                f0, e0 = open_edges.pop(key)
                m.ff[f0][e0] = f
                m.ff[f][e] = f0
    for v in range(len(m.p)):
        if m.start[v] == NONE:
            continue
        f = m.next_face(m.start[v], v)
        while f != NONE and f != m.start[v]:
            f = m.next_face(f, v)
        m.boundary[v] = f == NONE
        val = m.valence(v)
        m.regular[v] = (not m.boundary[v] and val == 6) or (m.boundary[v] and val == 4)
    for _ in range(levels):
        c = _Mesh()
        for v in range(len(m.p)):
            m.child[v] = c.add_vertex(np.zeros(3), regular=m.regular[v], boundary=m.boundary[v])
        for f in range(len(m.fv)):
            m.fc[f] = [c.add_face() for _ in range(4)]
        for v in range(len(m.p)):
            if m.start[v] == NONE:
                continue
            if not m.boundary[v]:
                beta = 1.0 / 16.0 if m.regular[v] else _beta(m.valence(v))
                c.p[m.child[v]] = _one_ring_weight(m, v, beta)
            else:
                c.p[m.child[v]] = _boundary_weight(m, v, 1.0 / 8.0)
        edge_verts = {}
        for f in range(len(m.fv)):
            for k in range(3):
                a, b = m.fv[f][k], m.fv[f][_next(k)]
                key = (min(a, b), max(a, b))
                if key in edge_verts:
                    continue
                boundary = m.ff[f][k] == NONE
                if boundary:
                    p = 0.5 * m.p[key[0]] + 0.5 * m.p[key[1]]
                else:
                    p = (3.0 / 8.0 * m.p[key[0]] + 3.0 / 8.0 * m.p[key[1]]
                         + 1.0 / 8.0 * m.p[m.other_vert(f, *key)] + 1.0 / 8.0 * m.p[m.other_vert(m.ff[f][k], *key)])
                edge_verts[key] = c.add_vertex(p, start=m.fc[f][3], regular=True, boundary=boundary)
        for v in range(len(m.p)):
            if m.start[v] != NONE:
                c.start[m.child[v]] = m.fc[m.start[v]][m.vnum(m.start[v], v)]
        for f in range(len(m.fv)):
            ch = m.fc[f]
            for j in range(3):
                c.ff[ch[3]][j] = ch[_next(j)]
                c.ff[ch[j]][_next(j)] = ch[3]
                f2 = m.ff[f][j]
                c.ff[ch[j]][j] = m.fc[f2][m.vnum(f2, m.fv[f][j])] if f2 != NONE else NONE
                f2 = m.ff[f][_prev(j)]
                c.ff[ch[j]][_prev(j)] = m.fc[f2][m.vnum(f2, m.fv[f][j])] if f2 != NONE else NONE
        for f in range(len(m.fv)):
            ch = m.fc[f]
            for j in range(3):
                c.fv[ch[j]][j] = m.child[m.fv[f][j]]
                a, b = m.fv[f][j], m.fv[f][_next(j)]
                ov = edge_verts[(min(a, b), max(a, b))]
                c.fv[ch[j]][_next(j)] = ov
                c.fv[ch[_next(j)]][j] = ov
                c.fv[ch[3]][j] = ov
        m = c
    limit = []
    for v in range(len(m.p)):
        if m.start[v] == NONE:
            limit.append(m.p[v])
        elif m.boundary[v]:
            limit.append(_boundary_weight(m, v, 1.0 / 5.0))
        else:
            limit.append(_one_ring_weight(m, v, _gamma(m.valence(v))))
    m.p = limit
    normals = []
    for v in range(len(m.p)):
        s = np.zeros(3)
        t = np.zeros(3)
        if m.start[v] != NONE:
            val = m.valence(v)
            ring = m.one_ring(v)
            if not m.boundary[v]:
                for j in range(val):
                    s = s + math.cos(2 * math.pi * j / val) * ring[j]
                    t = t + math.sin(2 * math.pi * j / val) * ring[j]
            else:
                s = ring[val - 1] - ring[0]
                if val == 2:
                    t = ring[0] + ring[1] - 2 * m.p[v]
                elif val == 3:
                    t = ring[1] - m.p[v]
                elif val == 4:
                    t = -1 * ring[0] + 2 * ring[1] + 2 * ring[2] - 1 * ring[3] - 2 * m.p[v]
                else:
                    th = math.pi / (val - 1)
                    t = math.sin(th) * (ring[0] + ring[val - 1])
                    for k in range(1, val - 1):
                        t = t + (2 * math.cos(th) - 2) * math.sin(k * th) * ring[k]
                    t = -t
        normals.append(np.cross(s, t))
    return np.array(m.p), np.array(m.fv, np.int64), np.array(normals)

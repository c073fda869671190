"""pbrt-v3 scene files (ilm_scene_file_*), the format of core/parser/ast.rs.

The reference builds a syntax tree and constructs no scene from it
(core/parser/mod.rs:36-46), so there is no reference output to compare with:
the loader is pinned to pbrt-v3's documented semantics by known answers --
transform composition and column order, LookAt frames, the attribute and
transform stacks, orientation flips, normal / tangent / uv handling, shape
and setting defaults, named materials, object instances, Include -- and to
the Cornell workload written as a scene file and read back exactly.
GPU (marked): the file's accel and path tracer give the direct API's answers.
"""
import os

import numpy as np
import pytest

import rs_illume_b200 as rb
from rs_illume_b200 import _lib
from rs_illume_b200 import workloads as wl
from tests.scene_writer import write_triangle_scene

TRI = '"point P" [0 0 0  1 0 0  0 1 0] "integer indices" [0 1 2]'


def load(text, base_dir=""):
    return rb.SceneFile.parse(text, base_dir)


def xform_points(m, p):
    p = np.c_[p, np.ones(len(p))] @ np.asarray(m, np.float64).T
    return (p[:, :3] / p[:, 3:]).astype(np.float32)


def rot(deg, axis):
    a = np.asarray(axis, np.float64) / np.linalg.norm(axis)
    t = np.radians(deg)
    k = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    r = np.eye(4)
    r[:3, :3] = np.cos(t) * np.eye(3) + np.sin(t) * k + (1 - np.cos(t)) * np.outer(a, a)
    return r


def trans(x, y, z):
    m = np.eye(4)
    m[:3, 3] = x, y, z
    return m


def scl(x, y, z):
    return np.diag([x, y, z, 1.0])


P0 = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float64)


def test_settings_and_defaults():
    sf = load("WorldBegin\nWorldEnd\n")
    i = sf.info
    assert (i.width, i.height, i.spp, i.max_depth) == (640, 480, 16, 5)
    assert i.fov_deg == pytest.approx(90.0) and i.accelerator == 0 and i.bvh.max_prims_in_node == 4
    assert i.filter.kind == 0                                        # box
    assert tuple(i.filter.radius) == (0.5, 0.5)
    sf = load('''
        Film "image" "integer xresolution" [ 100 ] "integer yresolution" [ 200 ] "string filename" "x.exr"
        Camera "perspective" "float fov" 30
        Sampler "stratified" "integer xsamples" 3 "integer ysamples" 3 "bool jitter" "true"
        Integrator "path" "integer maxdepth" 9
        PixelFilter "mitchell" "float xwidth" 1.5 "float ywidth" 2.5 "float B" 0.25
        Accelerator "kdtree" "integer intersectcost" 20 "float emptybonus" 0.25 "integer maxprims" 2
        WorldBegin WorldEnd''')
    i = sf.info
    assert (i.width, i.height, i.spp, i.max_depth) == (100, 200, 9, 9)
    # fov spans the shorter (x) axis: the vertical one is wider
    assert i.fov_deg == pytest.approx(np.degrees(2 * np.arctan(np.tan(np.radians(15)) * 2.0)), rel=1e-6)
    assert i.filter.kind == 3 and tuple(i.filter.radius) == (1.5, 2.5)
    assert i.filter.a == pytest.approx(0.25) and i.filter.b == pytest.approx(1 / 3)
    assert i.accelerator == 1 and (i.kdtree.isect_cost, i.kdtree.traversal_cost, i.kdtree.max_prims) == (20, 1, 2)
    assert i.kdtree.empty_bonus == 0.25 and i.kdtree.max_depth == -1
    assert sf.warnings == []
    sf = load('Sampler "halton" "integer pixelsamples" 10 WorldBegin WorldEnd')
    assert sf.info.spp == 16 and any("rounded up to 16" in w for w in sf.warnings)


def test_transform_composition():
    text = f'''WorldBegin
        Translate 1 2 3
        Rotate 30 0 0 1
        Scale 2 3 4
        Shape "trianglemesh" {TRI}
        WorldEnd'''
    m = load(text).mesh(0)
    want = xform_points(trans(1, 2, 3) @ rot(30, (0, 0, 1)) @ scl(2, 3, 4), P0)
    np.testing.assert_allclose(m["xyz"], want, rtol=1e-6, atol=1e-6)
    # Transform / ConcatTransform list the matrix's columns
    t = trans(1, 2, 3) @ rot(40, (1, 1, 0))
    cols = " ".join(repr(float(v)) for v in t.T.reshape(-1))
    for text in (f"WorldBegin Transform [ {cols} ] Shape \"trianglemesh\" {TRI} WorldEnd",
                 f"WorldBegin Translate 9 9 9 Identity ConcatTransform [ {cols} ] Shape \"trianglemesh\" {TRI} WorldEnd"):
        np.testing.assert_allclose(load(text).mesh(0)["xyz"], xform_points(t, P0), rtol=1e-6, atol=1e-6)
    # named coordinate systems
    text = f'''WorldBegin Translate 5 0 0 CoordinateSystem "here" Identity Translate 0 7 0
        CoordSysTransform "here" Shape "trianglemesh" {TRI} WorldEnd'''
    np.testing.assert_allclose(load(text).mesh(0)["xyz"], P0 + [5, 0, 0])


def test_look_at_camera():
    sf = load('LookAt 1 2 3  4 2 3  0 0 1\nCamera "perspective" WorldBegin WorldEnd')
    c = sf.camera()
    np.testing.assert_allclose(c["eye"], [1, 2, 3])
    r = c["camera_to_world"]
    dirn = np.array([1.0, 0, 0])
    right = np.cross([0, 0, 1.0], dirn)
    np.testing.assert_allclose(r[:, 2], dirn, atol=1e-7)        # camera +z looks along dir
    np.testing.assert_allclose(r[:, 0], right, atol=1e-7)       # camera +x is up x dir
    np.testing.assert_allclose(r[:, 1], np.cross(dirn, right), atol=1e-7)
    # a mirrored camera (Scale -1 1 1 before LookAt, as exporters write it)
    sf = load('Scale -1 1 1\nLookAt 0 0 0  0 0 1  0 1 0\nCamera "perspective" WorldBegin WorldEnd')
    np.testing.assert_allclose(sf.camera()["camera_to_world"], np.diag([-1.0, 1, 1]), atol=1e-7)
    # the world block starts from the identity whatever the camera transform
    sf = load(f'Translate 3 3 3 Camera "perspective" WorldBegin Shape "trianglemesh" {TRI} WorldEnd')
    np.testing.assert_allclose(sf.mesh(0)["xyz"], P0)
    np.testing.assert_allclose(sf.camera()["eye"], [-3, -3, -3])


def test_attribute_and_transform_stacks():
    sf = load(f'''WorldBegin
        Material "matte" "rgb Kd" [0.1 0.2 0.3]
        AttributeBegin
          Material "matte" "rgb Kd" [0.9 0.9 0.9]
          AreaLightSource "diffuse" "rgb L" [2 3 4] "rgb scale" [2 2 2]
          Translate 1 0 0
          Shape "trianglemesh" {TRI}
        AttributeEnd
        Shape "trianglemesh" {TRI}
        TransformBegin
          Translate 0 1 0
          Material "matte" "rgb Kd" [0.5 0.6 0.7]
        TransformEnd
        Shape "trianglemesh" {TRI}
        WorldEnd''')
    alb, emi = sf.materials()
    m = [sf.mesh(k) for k in range(3)]
    np.testing.assert_allclose(m[0]["xyz"], P0 + [1, 0, 0])
    np.testing.assert_allclose(alb[m[0]["material"]], [0.9, 0.9, 0.9])
    np.testing.assert_allclose(emi[m[0]["material"]], [4, 6, 8])
    np.testing.assert_allclose(m[1]["xyz"], P0)
    np.testing.assert_allclose(alb[m[1]["material"]], [0.1, 0.2, 0.3])
    assert np.all(emi[m[1]["material"]] == 0)
    # TransformEnd restores the transform only: the material set inside stays
    np.testing.assert_allclose(m[2]["xyz"], P0)
    np.testing.assert_allclose(alb[m[2]["material"]], [0.5, 0.6, 0.7])
    assert sf.info.n_emissive == 1 and sf.info.n_materials == 3


def test_orientation_flips():
    def winding(text):
        return [tuple(load(f"WorldBegin {text} Shape \"trianglemesh\" {TRI} WorldEnd").mesh(0)["idx"][0])]
    assert winding("") == [(0, 1, 2)]
    assert winding("ReverseOrientation") == [(0, 2, 1)]
    assert winding("Scale -1 1 1") == [(0, 2, 1)]                    # a handedness swap
    assert winding("Scale -1 1 1 ReverseOrientation") == [(0, 1, 2)]
    assert winding("AttributeBegin ReverseOrientation AttributeEnd") == [(0, 1, 2)]


def test_normals_tangents_uv():
    sf = load('''WorldBegin Scale 2 1 1
        Shape "trianglemesh" "point P" [0 0 0 1 0 0 0 1 0] "integer indices" [0 1 2]
          "normal N" [1 1 0  1 1 0  1 1 0] "vector S" [1 1 0 1 1 0 1 1 0] "float uv" [0 0 1 0 0 1]
        WorldEnd''')
    m = sf.mesh(0)
    np.testing.assert_allclose(m["n"], [[0.5, 1, 0]] * 3)           # inverse transpose
    np.testing.assert_allclose(m["s"], [[2, 1, 0]] * 3)
    np.testing.assert_allclose(m["uv"], [[0, 0], [1, 0], [0, 1]])
    m = load(f'WorldBegin Shape "trianglemesh" {TRI} WorldEnd').mesh(0)
    assert m["n"] is None and m["s"] is None and m["uv"] is None
    # a single triangle may omit its indices
    m = load('WorldBegin Shape "trianglemesh" "point P" [0 0 0 1 0 0 0 1 0] WorldEnd').mesh(0)
    assert m["idx"].tolist() == [[0, 1, 2]]


def test_quadric_shapes():
    sf = load('''WorldBegin
        Translate 1 0 0
        Shape "sphere"
        Shape "disk" "float height" 0.5 "float innerradius" 0.2
        Shape "cylinder" "float zmin" -2 "float phimax" 180
        ReverseOrientation
        Shape "cone" "float height" 3 "float radius" 0.5
        Shape "paraboloid"
        Shape "hyperboloid" "point p1" [1 0 -1] "point p2" [1 0 1]
        WorldEnd''')
    q, mat = sf.quadrics()
    assert [d.kind for d in q] == [0, 1, 2, 3, 4, 5] and len(mat) == 6
    assert (q[0].radius, q[0].z_min, q[0].z_max, q[0].phi_max_deg) == (1.0, -1.0, 1.0, 360.0)
    assert (q[1].height, q[1].radius, q[1].inner_radius) == (0.5, 1.0, pytest.approx(0.2))
    assert (q[2].z_min, q[2].z_max, q[2].phi_max_deg) == (-2.0, 1.0, 180.0)
    assert (q[3].height, q[3].radius, q[3].reverse_orientation) == (3.0, 0.5, 1)
    assert (q[4].radius, q[4].z_min, q[4].z_max) == (1.0, 0.0, 1.0)
    assert list(q[5].p1) == [1, 0, -1] and list(q[5].p2) == [1, 0, 1]
    assert q[0].reverse_orientation == 0 and q[0].object_to_world[3] == 1.0 and q[0].world_to_object[3] == -1.0


def test_named_materials_instances_and_include(tmp_path):
    inc = tmp_path / "parts" / "tri.pbrt"
    inc.parent.mkdir()
    inc.write_text(f'Shape "trianglemesh" {TRI}\n')
    main = tmp_path / "scene.pbrt"
    main.write_text(f'''WorldBegin
        MakeNamedMaterial "red" "string type" "matte" "rgb Kd" [0.8 0.1 0.1]
        ObjectBegin "thing"
          NamedMaterial "red"
          Translate 0 0 1
          Shape "trianglemesh" {TRI}
        ObjectEnd
        Translate 10 0 0
        ObjectInstance "thing"
        Translate 0 10 0
        ObjectInstance "thing"
        Include "parts/tri.pbrt"
        WorldEnd''')
    sf = rb.SceneFile.load(str(main))
    alb, _ = sf.materials()
    assert sf.info.n_meshes == 3
    np.testing.assert_allclose(sf.mesh(0)["xyz"], P0 + [10, 0, 1])
    np.testing.assert_allclose(sf.mesh(1)["xyz"], P0 + [10, 10, 1])
    np.testing.assert_allclose(sf.mesh(2)["xyz"], P0 + [10, 10, 0])
    np.testing.assert_allclose(alb[sf.mesh(0)["material"]], [0.8, 0.1, 0.1])
    np.testing.assert_allclose(alb[sf.mesh(2)["material"]], [0.5, 0.5, 0.5])   # outside the object block
    assert sf.warnings == []


@pytest.mark.parametrize("text,msg", [
    ("Foo 1 2", "1: unknown directive \"Foo\""),
    ('WorldBegin\nShape "trianglemesh" "point P [0 0 0]', "2: unterminated string"),
    ('WorldBegin\n\nShape "trianglemesh" "point P" [0 0 0 1 0 0 0 1 0', "3: unexpected end of input"),
    ("WorldBegin\nAttributeEnd", "2: unmatched AttributeEnd"),
    ("AttributeBegin\nTransformEnd", "2: TransformEnd closes a block opened by the other kind"),
    ('Transform [1 0 0 0 0 1 0 0 0 0 0 0 0 0 0 1]', "1: Transform matrix is singular"),
    ('WorldBegin NamedMaterial "nope"', "1: named material \"nope\" not defined"),
    ('WorldBegin Shape "trianglemesh" "point P" [0 0 0 1 0 0 0 1 0] "integer indices" [0 1 3]', "index out of range"),
    ('WorldBegin Shape "trianglemesh" "point P" [0 0 0 1 0]', "multiple of 3"),
    ('Translate 1 2 x', "expected a number"),
    ('Shape "sphere" "bogus radius" 1', "unknown parameter type"),
    ('Camera "perspective" "float fov" 180', "fov must lie in (0, 180)"),
    ('ObjectInstance "none"', "object \"none\" not defined"),
])
def test_errors(text, msg):
    with pytest.raises(rb.IllumeError) as e:
        load(text)
    assert msg in str(e.value) and "<text>:" in str(e.value)


def test_missing_file_and_include_depth(tmp_path):
    with pytest.raises(rb.IllumeError, match="cannot open"):
        rb.SceneFile.load(str(tmp_path / "nope.pbrt"))
    loop = tmp_path / "loop.pbrt"
    loop.write_text('Include "loop.pbrt"\n')
    with pytest.raises(rb.IllumeError, match="nested more than 16"):
        rb.SceneFile.load(str(loop))


def test_warnings_for_what_is_not_represented():
    sf = load(f'''
        Camera "orthographic"
        WorldBegin
        LightSource "point" "rgb I" [1 1 1]
        Texture "checks" "spectrum" "checkerboard"
        Material "plastic" "texture Kd" "checks"
        Shape "plymesh" "string filename" "x.ply"
        Shape "trianglemesh" {TRI} "float unusedthing" 3
        WorldEnd''')
    w = "\n".join(sf.warnings)
    for needle in ("rendered as a perspective camera", "light \"point\" is not supported",
                   "texture \"checkerboard\" is not supported", "material \"plastic\" is shaded as matte",
                   "shape \"plymesh\" is not supported", "\"float unusedthing\" unused"):
        assert needle in w, (needle, w)
    assert sf.info.n_meshes == 1 and sf.info.n_warnings == len(sf.warnings)


def test_cornell_written_and_read_back(tmp_path):
    xyz, idx, mat, alb, emi = wl.cornell(3, 3)
    cam = wl.CORNELL_CAMERA
    path = tmp_path / "cornell.pbrt"
    write_triangle_scene(path, xyz, idx, mat, alb, emi, cam["eye"], cam["fov_deg"], 48, 48, spp=16, max_depth=8)
    sf = rb.SceneFile.load(str(path))
    assert sf.warnings == []
    i = sf.info
    assert (i.n_triangles, i.width, i.height, i.spp, i.max_depth) == (len(idx), 48, 48, 16, 8)
    assert i.n_emissive == int(np.sum(np.any(emi[mat] > 0, axis=1)))
    np.testing.assert_array_equal(sf.camera()["eye"], np.float32(cam["eye"]))
    np.testing.assert_array_equal(sf.camera()["camera_to_world"], np.eye(3, dtype=np.float32))
    assert i.fov_deg == np.float32(cam["fov_deg"])
    salb, semi = sf.materials()
    tris, mats = [], []
    for k in range(i.n_meshes):
        m = sf.mesh(k)
        tris.append(m["xyz"][m["idx"]])
        mats += [m["material"]] * len(m["idx"])
    # every triangle, in order, with its vertices bit for bit and its material's values
    np.testing.assert_array_equal(np.concatenate(tris), xyz[idx])
    np.testing.assert_array_equal(salb[mats], alb[mat])
    np.testing.assert_array_equal(semi[mats], emi[mat])


# ----------------------------------------------------------------------- GPU

@pytest.mark.gpu
def test_gpu_scene_file_renders_as_the_direct_api(tmp_path):
    """The Cornell box through a scene file (ids, materials, lights, camera in
    the same order) renders the direct PathTracer's image, up to the order of
    the film's atomic additions; its accel answers rays identically."""
    xyz, idx, mat, alb, emi = wl.cornell(4, 3)
    cam = wl.CORNELL_CAMERA
    w = h = 48
    path = tmp_path / "cornell.pbrt"
    write_triangle_scene(path, xyz, idx, mat, alb, emi, cam["eye"], cam["fov_deg"], w, h, spp=16, max_depth=8)
    ctx = rb.Context(0)
    sf = rb.SceneFile.load(str(path))
    acc_f, pt_f = sf.build(ctx)
    assert pt_f is not None
    img_f, st_f = sf.render(pt_f, seed=5, rr_depth=3)
    acc = rb.GpuBVHAccel(ctx, [rb.TriangleMesh(ctx, xyz, idx)], width=8)
    pt = rb.PathTracer(acc, mat, alb, emi, cam["eye"], cam["fov_deg"], w, h)
    img, st = pt.render(16, max_depth=8, seed=5)
    bad = ~np.isclose(img_f, img, rtol=1e-4, atol=1e-6)
    assert bad.mean() < 0.01, bad.mean()
    assert st_f["closest_rays"] == st["closest_rays"] and st_f["shadow_rays"] == st["shadow_rays"]
    rays = wl.ball_rays(4, 0, 65536, 65536, 1.5, 0.0, 3.0)
    rays["o"] += 0.5
    assert acc_f.intersect_batch(rays).tobytes() == acc.intersect_batch(rays).tobytes()
    ctx.close()


@pytest.mark.gpu
def test_gpu_look_at_camera_matches_oracle(tmp_path):
    """A turned camera (LookAt off the box's axis): the GPU render through the
    file's camera frame and the oracle's render with the same frame agree
    statistically (relMSE ratio and image means, as the path-tracer tests)."""
    import oracle
    xyz, idx, mat, alb, emi = wl.cornell(4, 3)
    w = h = 32
    eye, look = (0.2, 0.6, -1.2), (0.55, 0.45, 0.5)
    path = tmp_path / "turned.pbrt"
    write_triangle_scene(path, xyz, idx, mat, alb, emi, eye, 45.0, w, h, spp=64, max_depth=8, look=look)
    sf = rb.SceneFile.load(str(path))
    c = sf.camera()
    assert not np.allclose(c["camera_to_world"], np.eye(3))
    ctx = rb.Context(0)
    _, pt = sf.build(ctx)
    g1, _ = sf.render(pt, seed=3)
    g2, _ = sf.render(pt, seed=4)
    from rs_illume_b200 import image
    box = image.filter_desc("box", (0.5, 0.5))
    o, _ = oracle.render_pt_filtered(oracle.Scene(xyz, idx), xyz, idx, mat, alb, emi, c["eye"], c["fov_deg"], w, h,
                                     64, image.filter_table(box), (0.5, 0.5), seed=3,
                                     camera_to_world=c["camera_to_world"])

    def relmse(x, y):
        return float(np.mean((x - y) ** 2 / (y ** 2 + 0.01)))
    r_go, r_gg = relmse(g1, o), relmse(g1, g2)
    assert 0.7 < r_go / r_gg < 1.4, (r_go, r_gg)
    se = (g1 - g2).reshape(-1, 3).std(axis=0) / np.sqrt(w * h)
    diff = g1.reshape(-1, 3).mean(axis=0) - o.reshape(-1, 3).mean(axis=0)
    assert np.all(np.abs(diff) < 5 * se + 1e-6), (diff, se)
    ctx.close()


@pytest.mark.gpu
def test_gpu_scene_file_with_quadrics_and_kdtree(ctx):
    """Quadrics and a kd-tree named in the file: the accel is the kd-tree and
    answers as a kd accel built directly; no path-tracing scene is made."""
    sf = load(f'''Accelerator "kdtree"
        WorldBegin
        Shape "trianglemesh" {TRI}
        Translate 0 0 3 Shape "sphere" "float radius" 0.5
        Shape "hyperboloid" "point p1" [1 0 -1] "point p2" [1 0 1]
        WorldEnd''')
    acc, pt = sf.build(ctx)
    assert pt is None and acc.info()["width"] == _lib.ILM_LAYOUT_KDTREE
    q, _ = sf.quadrics()
    m = sf.mesh(0)
    direct = rb.GpuKdTreeAccel(ctx, [rb.TriangleMesh(ctx, m["xyz"], m["idx"]), rb.Spheres(ctx, q)])
    rays = wl.ball_rays(6, 0, 32768, 32768, 2.0, 0.0, 6.0)
    rays["o"] += [0.0, 0.0, 1.5]
    got = acc.intersect_batch(rays)
    assert got.tobytes() == direct.intersect_batch(rays).tobytes()
    assert np.sum(got["prim"] == 1) > 100 and np.sum(got["prim"] == 2) > 100

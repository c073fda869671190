"""The scene-file reader against the reference's own parser tests.

core/parser/parsers/tests.rs holds the reference's known-answer cases for the
pbrt-v3 syntax (numbers, identifiers, strings, transforms, every parameter
type, directive blocks, Include, a whole file).  Each test below feeds the same
input to ilm_scene_syntax, which reads it with the tokenizer and argument
grammar that the loader (ilm_scene_file_parse) runs, and checks the values the
reference's test checks.  The reference tests its sub-parsers one at a time;
here a value reaches the reader inside the smallest directive or parameter
list that carries it.  The file_span.rs tests cover the Rust parser's input
type (slicing, columns, offsets) and have no counterpart.
"""
import numpy as np
import pytest

from rs_illume_b200 import IllumeError
from rs_illume_b200.scene_file import syntax


def top(text, **kw):
    return syntax(text, **kw)["directives"]


def one(text):
    d = top(text)
    assert len(d) == 1
    return d[0]


def param(text):
    """The single parameter of a Shape carrying `text` as its parameter list."""
    ps = one('Shape "s" ' + text)["params"]
    assert len(ps) == 1
    return ps[0]


def test_ws_and_comment():                                   # tests.rs:48-54
    assert syntax(" \t#test\n  ")["comments"] == ["test"]
    assert syntax(" \t\n  ")["comments"] == []
    assert syntax("#test\n#test\n")["comments"] == ["test", "test"]
    assert syntax(" \t\n  ")["directives"] == []


def test_parse_number():                                     # tests.rs:64-73
    p = param('"float v" [3.14 -3.14 3e10 3E10 3e-10 0.5 .5]')
    assert p["num"] == [3.14, -3.14, 3e10, 3e10, 3e-10, 0.5, 0.5]


def test_parse_int():                                        # tests.rs:75-81
    assert param('"integer v" [4 4350 -1 0]')["num"] == [4.0, 4350.0, -1.0, 0.0]
    # integers are -?digits (values.rs parse_int)
    for bad in ("4.5", "1e3", "+4"):
        with pytest.raises(IllumeError, match="takes integers"):
            param(f'"integer v" [{bad}]')


def test_parse_ident():                                      # tests.rs:83-105
    # a bare word, backslash escapes included, is one token
    d = one('ActiveTransform All')
    assert d["str"] == ["All"]
    with pytest.raises(IllumeError, match=r'unknown directive "te\\nst"'):
        syntax("te\\nst")
    with pytest.raises(IllumeError, match='unknown directive "test"'):
        syntax("test")


def test_parse_quoted_string():                              # tests.rs:107-119
    assert one('CoordinateSystem "test"')["str"] == ["test"]


def test_parse_lookat():                                     # tests.rs:121-152
    assert one("LookAt 0 0 0 10 10 10 0 1 0")["num"] == [0, 0, 0, 10, 10, 10, 0, 1, 0]
    d = one("""LookAt 3 4 1.5  # eye
    .5 .5 0  # look at point
    0 0 1    # up vector""")
    assert d["num"] == [3.0, 4.0, 1.5, 0.5, 0.5, 0.0, 0.0, 0.0, 1.0]


def test_parse_translate():                                  # tests.rs:154-163
    assert one("Translate 4 5.5 1.0")["num"] == [4.0, 5.5, 1.0]


def test_parse_scale():                                      # tests.rs:165-174
    assert one("Scale 4 5.5 1.0")["num"] == [4.0, 5.5, 1.0]


def test_parse_rotate():                                     # tests.rs:176-186
    assert one("Rotate 45 4 5.5 1.0")["num"] == [45.0, 4.0, 5.5, 1.0]


def test_parse_coordinate_system():                          # tests.rs:188-195
    d = one('CoordinateSystem "test"')
    assert d["directive"] == "CoordinateSystem" and d["str"] == ["test"]


def test_parse_coord_sys_transform():                        # tests.rs:197-204
    d = one('CoordSysTransform "test"')
    assert d["directive"] == "CoordSysTransform" and d["str"] == ["test"]


@pytest.mark.parametrize("name", ["Transform", "ConcatTransform"])
def test_parse_transform(name):                              # tests.rs:206-252
    vals = " ".join(str(k) for k in range(1, 17))
    assert one(f"{name} {vals}")["num"] == [float(k) for k in range(1, 17)]
    # pbrt-v3 files also bracket the 16 numbers
    assert one(f"{name} [ {vals} ]")["num"] == [float(k) for k in range(1, 17)]
    with pytest.raises(IllumeError):
        syntax(f"{name} 1 2 3")


def test_parse_active_transform():                           # tests.rs:254-271
    for w in ("StartTime", "EndTime", "All"):
        assert one(f"ActiveTransform {w}")["str"] == [w]
    with pytest.raises(IllumeError, match="StartTime, EndTime or All"):
        syntax("ActiveTransform Sometimes")


def test_parse_transform_times():                            # tests.rs:273-278
    assert one("TransformTimes 100 250.6")["num"] == [100.0, 250.6]


def test_parse_integer_parameters():                         # tests.rs:280-339
    p = param('"integer test" 20')
    assert (p["type"], p["name"], p["num"]) == ("integer", "test", [20.0])
    assert param('"integer test" [20]')["num"] == [20.0]
    assert param('"integer test" [20 42 36]')["num"] == [20.0, 42.0, 36.0]


def test_parse_float_parameters():                           # tests.rs:341-376
    p = param('"float test" 20.5')
    assert (p["type"], p["name"], p["num"]) == ("float", "test", [20.5])
    assert param('"float test" [20.5]')["num"] == [20.5]
    assert param('"float test" [20.5 42 36.0]')["num"] == [20.5, 42.0, 36.0]


def test_named_parameter():                                  # tests.rs:378-385
    assert param('"float test" 1')["name"] == "test"
    assert param('"integer   test2" 1')["name"] == "test2"
    # a value that the declared type's grammar does not take is an error
    with pytest.raises(IllumeError, match="expected a number"):
        param('"float test" "string"')
    with pytest.raises(IllumeError, match="takes quoted strings"):
        param('"string test" 1')
    with pytest.raises(IllumeError, match="unknown parameter type"):
        param('"int test2" 1')


@pytest.mark.parametrize("decl,typ", [("point2", "point2"), ("vector2", "vector2")])
def test_parse_2d_parameters(decl, typ):                     # tests.rs:387-405
    p = param(f'"{decl} test" [20.5 10]')
    assert (p["type"], p["num"]) == (typ, [20.5, 10.0])


@pytest.mark.parametrize("decl,typ", [("point3", "point"), ("point", "point"), ("vector3", "vector"),
                                      ("vector", "vector"), ("normal3", "normal"), ("normal", "normal")])
def test_parse_3d_parameters(decl, typ):                     # tests.rs:407-456
    p = param(f'"{decl} test" [20.5 10 0]')
    assert (p["type"], p["name"], p["num"]) == (typ, "test", [20.5, 10.0, 0.0])


def test_parse_spectrum():                                   # tests.rs:458-480
    p = param('"spectrum test" [300 .3 400 .6   410 .65  415 .8  500 .2  600 .1]')
    assert p["type"] == "spectrum" and p["name"] == "test" and p["str"] == []
    assert len(p["num"]) == 12 and p["num"][:2] == [300.0, 0.3]


def test_parse_spectrum_parameter():                         # tests.rs:482-585
    for decl in ("rgb", "color"):
        p = param(f'"{decl} test" [.2 .5 .3]')
        assert (p["type"], p["name"], p["num"]) == (decl, "test", [0.2, 0.5, 0.3])
    p = param('"xyz test" [.4 .5 .6]')
    assert (p["type"], p["num"]) == ("xyz", [0.4, 0.5, 0.6])
    p = param('"spectrum test" [300 .3  400 .6   410 .65  415 .8  500 .2  600 .1]')
    assert len(p["num"]) == 12 and p["num"][:2] == [300.0, 0.3]
    p = param('"blackbody test" [.4 .5]')
    assert (p["type"], p["num"]) == ("blackbody", [0.4, 0.5])
    # a sampled spectrum given by file name
    p = param('"spectrum test" "filename.test"')
    assert (p["type"], p["name"], p["num"], p["str"]) == ("spectrum", "test", [], ["filename.test"])


def test_string_parameter():                                 # tests.rs:587-606
    p = param('"string test" "test value"')
    assert (p["type"], p["name"], p["str"]) == ("string", "test", ["test value"])


def test_boolean_parameter():                                # tests.rs:608-645
    assert param('"bool test" "true"')["str"] == ["true"]
    assert param('"bool test" "false"')["str"] == ["false"]
    with pytest.raises(IllumeError, match='"true" or "false"'):
        param('"bool test" "maybe"')


def test_parse_comment():                                    # tests.rs:647-651
    assert syntax(" \t#test\n")["comments"] == ["test"]


def test_parameter_list():                                   # tests.rs:653-684
    ps = one('Shape "s" "bool test" "true"')["params"]
    assert [(p["type"], p["name"], p["str"]) for p in ps] == [("bool", "test", ["true"])]
    ps = one('Shape "s" "bool test" "true" #test\n#test\n"string test2" "test string"')["params"]
    assert [(p["type"], p["name"], p["str"]) for p in ps] == [("bool", "test", ["true"]),
                                                              ("string", "test2", ["test string"])]


def test_transforms():                                       # tests.rs:686-701
    d = top("Scale 1 2 3#test\nTranslate 1 2 3")
    assert [x["directive"] for x in d] == ["Scale", "Translate"]
    assert d[0]["num"][0] == 1.0 and d[1]["num"][0] == 1.0
    assert [x["line"] for x in d] == [1, 2]


def test_camera():                                           # tests.rs:703-718
    assert one('Camera "realistic"')["str"] == ["realistic"]
    d = one('Camera "realistic" "string test" "test"')
    assert d["str"] == ["realistic"]
    assert [(p["type"], p["name"], p["str"]) for p in d["params"]] == [("string", "test", ["test"])]


SHAPES = '''Shape "sphere" "float radius" 1
            Shape "trianglemesh"
                "integer indices" [0 1 2 0 2 3]
                "point P" [ -20 -20 0   20 -20 0   20 20 0   -20 20 0 ]
                "float st" [ 0 0   1 0    1 1   0 1 ]'''

TEXTURED = '''Texture "checks" "spectrum" "checkerboard"
            "float uscale" [8] "float vscale" [8]
            "rgb tex1" [.1 .1 .1] "rgb tex2" [.8 .8 .8]
    Material "matte" "texture Kd" "checks"
    Translate 0 0 -1
    Shape "trianglemesh"
        "integer indices" [0 1 2 0 2 3]
        "point P" [ -20 -20 0   20 -20 0   20 20 0   -20 20 0 ]
        "float st" [ 0 0   1 0    1 1   0 1 ]'''


def test_object_block():                                     # tests.rs:720-731
    d = one(f'ObjectBegin "shape1"\n{SHAPES}\nObjectEnd')
    assert d["directive"] == "ObjectBegin" and d["str"] == ["shape1"]
    assert len(d["children"]) == 2
    mesh = d["children"][1]
    assert [p["name"] for p in mesh["params"]] == ["indices", "P", "st"]
    assert mesh["params"][1]["num"] == [-20, -20, 0, 20, -20, 0, 20, 20, 0, -20, 20, 0]


def test_attribute_block():                                  # tests.rs:733-747
    d = one(f"AttributeBegin\n{TEXTURED}\nAttributeEnd")
    assert [c["directive"] for c in d["children"]] == ["Texture", "Material", "Translate", "Shape"]
    tex = d["children"][0]
    assert tex["str"] == ["checks", "spectrum", "checkerboard"] and len(tex["params"]) == 4


def test_transform_block():                                  # tests.rs:749-756
    d = one('TransformBegin\n Translate 1 0 1\n Shape "sphere"\nTransformEnd')
    assert [c["directive"] for c in d["children"]] == ["Translate", "Shape"]


WORLD = f'''WorldBegin

        # uniform blue-ish illumination from all directions
        LightSource "infinite" "rgb L" [.4 .45 .5]

        # approximate the sun
        LightSource "distant"  "point from" [ -30 40  100 ]
        "blackbody L" [3000 1.5]

        AttributeBegin
        Material "glass"
        Shape "sphere" "float radius" 1
        AttributeEnd

        AttributeBegin
        {TEXTURED}
        AttributeEnd

    WorldEnd'''


def test_world_directive():                                  # tests.rs:758-788
    d = one(WORLD)
    assert d["directive"] == "WorldBegin"
    assert [c["directive"] for c in d["children"]] == ["LightSource", "LightSource", "AttributeBegin",
                                                       "AttributeBegin"]
    sun = d["children"][1]
    assert [(p["type"], p["name"], p["num"]) for p in sun["params"]] == [("point", "from", [-30, 40, 100]),
                                                                        ("blackbody", "L", [3000, 1.5])]


def test_many_with_include(tmp_path):                        # tests.rs:790-813
    (tmp_path / "shapes.pbrt").write_text(SHAPES)
    d = top('Include "shapes.pbrt"\nShape "sphere" "float radius" 1', base_dir=str(tmp_path))
    assert len(d) == 3
    assert [x["str"][0] for x in d] == ["sphere", "trianglemesh", "sphere"]
    assert d[0]["file"].endswith("shapes.pbrt") and d[2]["file"] == "<text>"
    with pytest.raises(IllumeError, match="cannot open"):
        syntax('Include "missing.pbrt"', base_dir=str(tmp_path))


def test_root():                                             # tests.rs:815-855
    d = top(f'''LookAt 3 4 1.5  # eye
    .5 .5 0  # look at point
    0 0 1    # up vector
Camera "perspective" "float fov" 45

Sampler "halton" "integer pixelsamples" 128
Integrator "path"
Film "image" "string filename" "simple.png"
    "integer xresolution" [400] "integer yresolution" [400]

{WORLD}''')
    assert [x["directive"] for x in d] == ["LookAt", "Camera", "Sampler", "Integrator", "Film", "WorldBegin"]
    assert d[4]["params"][1]["num"] == [400.0]


def test_blocks_must_match():
    """The reference's block parsers need the matching end (directives.rs)."""
    for text, msg in [("AttributeBegin", "without a matching end"), ("AttributeEnd", "unmatched AttributeEnd"),
                      ("AttributeBegin TransformEnd", "unmatched TransformEnd"),
                      ("WorldBegin ObjectBegin \"a\" WorldEnd", "unmatched WorldEnd")]:
        with pytest.raises(IllumeError, match=msg):
            syntax(text)


def test_loader_reads_what_the_syntax_shows(tmp_path):
    """The loader runs the same reader: the root file's settings land in the
    scene's settings, and a parameter the syntax rejects fails the load."""
    from rs_illume_b200 import SceneFile
    sf = SceneFile.parse('''LookAt 3 4 1.5  .5 .5 0  0 0 1
        Camera "perspective" "float fov" 45
        Sampler "halton" "integer pixelsamples" 128
        Film "image" "integer xresolution" [400] "integer yresolution" [400]
        WorldBegin Shape "sphere" "float radius" 1 WorldEnd''')
    assert (sf.info.width, sf.info.height, sf.info.n_quadrics) == (400, 400, 1)
    assert sf.info.spp == 144   # 128 rounded up to a square
    np.testing.assert_allclose(np.array(sf.info.eye), [3, 4, 1.5], rtol=1e-6)
    with pytest.raises(IllumeError, match="takes integers"):
        SceneFile.parse('Film "image" "integer xresolution" [400.5]')
    with pytest.raises(IllumeError, match='"true" or "false"'):
        SceneFile.parse('Sampler "stratified" "bool jitter" "yes"')

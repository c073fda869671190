"""Writes triangle scenes as pbrt-v3 scene files (test helper)."""
import numpy as np


def f32(v) -> str:
    """The shortest decimal that reads back as the same float32."""
    return repr(float(np.float32(v)))


def nums(a) -> str:
    return " ".join(f32(v) for v in np.asarray(a, np.float32).reshape(-1))


def write_triangle_scene(path, xyz, idx, mat, albedo, emission, eye, fov_deg, width, height, spp=16,
                         max_depth=8, look=None, up=(0.0, 1.0, 0.0), extra_world=""):
    """One trianglemesh per run of consecutive triangles sharing a material,
    so primitive ids keep the arrays' order; emissive materials get a diffuse
    area light.  The camera looks along +z from `eye` unless `look` is given."""
    xyz = np.asarray(xyz, np.float32).reshape(-1, 3)
    idx = np.asarray(idx, np.uint32).reshape(-1, 3)
    mat = np.asarray(mat, np.uint32)
    look = (eye[0], eye[1], eye[2] + 1.0) if look is None else look
    out = [f"LookAt {nums(eye)}  {nums(look)}  {nums(up)}",
           f'Camera "perspective" "float fov" [ {f32(fov_deg)} ]',
           f'Film "image" "integer xresolution" [ {width} ] "integer yresolution" [ {height} ]',
           f'Sampler "halton" "integer pixelsamples" {spp}',
           f'Integrator "path" "integer maxdepth" [ {max_depth} ]',
           "WorldBegin"]
    k = 0
    while k < len(idx):
        e = k
        while e < len(idx) and mat[e] == mat[k]:
            e += 1
        m = int(mat[k])
        tri = idx[k:e]
        used, inverse = np.unique(tri.reshape(-1), return_inverse=True)
        out.append("AttributeBegin")
        out.append(f'  Material "matte" "rgb Kd" [ {nums(albedo[m])} ]')
        if np.any(np.asarray(emission[m]) > 0):
            out.append(f'  AreaLightSource "diffuse" "rgb L" [ {nums(emission[m])} ]')
        out.append(f'  Shape "trianglemesh" "point P" [ {nums(xyz[used])} ]')
        out.append(f'    "integer indices" [ {" ".join(str(int(v)) for v in inverse)} ]')
        out.append("AttributeEnd")
        k = e
    out.append(extra_world)
    out.append("WorldEnd")
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")

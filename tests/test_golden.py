"""Golden fixtures (tests/golden/golden.npz, written by make_golden.py).

CPU: the seeded scenes regenerate byte for byte (SHA-256) and the oracle
reproduces every stored answer exactly.  GPU (marked): the B200 path
answers the same rays under the parity bar (ids bit-exact up to documented
near-ties, t and (u, v) within 1e-5 relative, any-hit flags exact)."""
import os

import numpy as np
import pytest

import oracle
from tests.golden import make_golden as mg

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden.npz"))
SETS = ("coherent", "incoherent", "spheres")


def scene_of(name):
    xyz, idx, rays = getattr(mg, name)()
    spheres = mg.sphere_descs(oracle.sphere_desc) if name == "spheres" else ()
    return xyz, idx, rays, spheres


@pytest.mark.parametrize("name", SETS)
def test_oracle_reproduces_golden_queries(name):
    xyz, idx, rays, spheres = scene_of(name)
    assert mg.digest(xyz, idx) == G[f"{name}_scene"].tobytes().decode()
    assert rays.tobytes() == G[f"{name}_rays"].tobytes()
    sc = oracle.Scene(xyz, idx, spheres)
    assert sc.intersect(rays).tobytes() == G[f"{name}_hits"].tobytes()
    assert np.array_equal(sc.intersect_p(rays), G[f"{name}_occ"])


def test_oracle_reproduces_golden_render():
    xyz, idx, mat, alb, emi = mg.pt_scene()
    assert mg.digest(xyz, idx, mat, alb, emi) == G["pt_scene"].tobytes().decode()
    cam = mg.wl.CORNELL_CAMERA
    p = mg.PT
    img, (nc, ns) = oracle.render_pt(oracle.Scene(xyz, idx), xyz, idx, mat, alb, emi, cam["eye"], cam["fov_deg"],
                                     p["w"], p["h"], p["spp"], p["depth"], p["rr"], p["seed"], threads=3)
    assert img.tobytes() == G["pt_image"].tobytes()
    assert [nc, ns] == G["pt_rays"].tolist()


@pytest.mark.gpu
@pytest.mark.parametrize("name", SETS)
@pytest.mark.parametrize("width", [2, 4, 8])
def test_gpu_matches_golden_queries(ctx, name, width):
    import rs_illume_b200 as rb
    from tests.test_gpu_trace import compare_closest
    xyz, idx, rays, _ = scene_of(name)
    shapes = [rb.TriangleMesh(ctx, xyz, idx)]
    if name == "spheres":
        shapes.append(rb.Spheres(ctx, mg.sphere_descs(rb.sphere_desc)))
    acc = rb.GpuBVHAccel(ctx, shapes, width=width)
    hits = acc.intersect_batch(rays)
    compare_closest(hits, G[f"{name}_hits"], tol_uv=1e-5 if name == "spheres" else 0.0, label=f"{name} w{width}")
    assert np.array_equal(acc.intersect_p_batch(rays).astype(np.uint8), G[f"{name}_occ"])


def test_oracle_generators_equal_the_products():
    """The CPU reference leg of the benchmark builds its inputs with the
    oracle's own generators (oracle/workloads.cpp), so it never loads the
    product library; they must give the product generators' bytes."""
    from rs_illume_b200 import workloads as wl
    for a, b in zip(oracle.incoherent_workload(), wl.incoherent_workload()):
        assert a.tobytes() == b.tobytes()
    for a, b in zip(oracle.coherent_workload(), wl.coherent_workload()):
        assert a.tobytes() == b.tobytes()
    for a, b in zip(oracle.icosphere(5, 1021, 0.05, 0.2, (0.66, 0.52, 0.33)),
                    wl.icosphere(5, 1021, 0.05, 0.2, (0.66, 0.52, 0.33))):
        assert a.tobytes() == b.tobytes()
    assert oracle.ball_rays(9, 3, 5000, 1700, 1.5, 0.2, 2.0).tobytes() == \
        wl.ball_rays(9, 3, 5000, 1700, 1.5, 0.2, 2.0).tobytes()
    assert oracle.camera_rays(33, 17, (0.1, 0.2, -3.0), 60.0).tobytes() == \
        wl.camera_rays(33, 17, (0.1, 0.2, -3.0), 60.0).tobytes()

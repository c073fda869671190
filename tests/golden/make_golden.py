"""Writes the golden fixtures of the ray-query and path-tracing path.

    python tests/golden/make_golden.py

The answers come from the CPU oracle (oracle/, the line-by-line restatement
of BVHAccel::intersect / intersect_p, Triangle, Sphere and the PathIntegrator
loop).  The reference ships no test vectors for this path and cannot be built
here, so these fixtures pin the oracle and the GPU path against regressions
on seeded procedural inputs; the scenes are regenerated from their seeds and
the fixture keeps a SHA-256 of their bytes.

Fixtures (golden.npz):
  coherent_*    32,768-triangle soup (seed 1), every 16th of the 256x256
                primary rays: closest hits and any-hit flags
  incoherent_*  displaced icosphere level 5 (20,480 triangles, seed 2),
                2,048 closest + 2,048 shadow ball rays
  spheres_*     four spheres (full, z-clipped, phi-clipped, reversed) and a
                triangle soup, 4,096 ball rays
  pt_*          Cornell box (level-3 icosphere), 24x24, 16 spp, depth 8
pt_tile.pfm holds the same image as a PFM file (ilm_write_pfm).
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from rs_illume_b200 import workloads as wl  # noqa: E402


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def coherent():
    xyz, idx, rays = wl.coherent_workload()
    return xyz, idx, np.ascontiguousarray(rays[::16])


def incoherent():
    xyz, idx = wl.icosphere(5, 2, 0.05, 1.0)
    rays = wl.ball_rays(2, 4, 4096, 2048, 3.0, 0.1, 4.0)
    return xyz, idx, rays


def sphere_descs(desc_fn):
    return [desc_fn(0.3, (0.5, 0.5, 0.5)),
            desc_fn(0.25, (0.2, 0.8, 0.3), z_min=-0.1, z_max=0.2),
            desc_fn(0.2, (0.8, 0.2, 0.7), phi_max_deg=200.0),
            desc_fn(0.15, (0.75, 0.75, 0.2), scale=1.5, reverse=True)]


def spheres():
    xyz, idx = wl.soup(11, 512, 0.05)
    rays = wl.ball_rays(12, 4, 4096, 4096, 1.2, 0.1, 4.0)
    rays["o"] += np.float32(0.5)
    return xyz, idx, rays


PT = dict(w=24, h=24, spp=16, depth=8, rr=3, seed=3, level=3)


def pt_scene():
    xyz, idx, mat, alb, emi = wl.cornell(PT["level"], 3)
    return xyz, idx, mat, alb, emi


def main():
    out = {}
    xyz, idx, rays = coherent()
    sc = oracle.Scene(xyz, idx)
    out.update(coherent_rays=rays, coherent_hits=sc.intersect(rays), coherent_occ=sc.intersect_p(rays),
               coherent_scene=np.frombuffer(digest(xyz, idx).encode(), np.uint8))
    xyz, idx, rays = incoherent()
    sc = oracle.Scene(xyz, idx)
    out.update(incoherent_rays=rays, incoherent_hits=sc.intersect(rays), incoherent_occ=sc.intersect_p(rays),
               incoherent_scene=np.frombuffer(digest(xyz, idx).encode(), np.uint8))
    xyz, idx, rays = spheres()
    sc = oracle.Scene(xyz, idx, sphere_descs(oracle.sphere_desc))
    out.update(spheres_rays=rays, spheres_hits=sc.intersect(rays), spheres_occ=sc.intersect_p(rays),
               spheres_scene=np.frombuffer(digest(xyz, idx).encode(), np.uint8))
    xyz, idx, mat, alb, emi = pt_scene()
    cam = wl.CORNELL_CAMERA
    sc = oracle.Scene(xyz, idx)
    img, (nc, ns) = oracle.render_pt(sc, xyz, idx, mat, alb, emi, cam["eye"], cam["fov_deg"], PT["w"], PT["h"],
                                     PT["spp"], PT["depth"], PT["rr"], PT["seed"])
    out.update(pt_image=img, pt_rays=np.array([nc, ns], np.uint64),
               pt_scene=np.frombuffer(digest(xyz, idx, mat, alb, emi).encode(), np.uint8))
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)
    from rs_illume_b200 import image
    image.write_pfm(os.path.join(HERE, "pt_tile.pfm"), img)
    print("wrote", os.path.join(HERE, "golden.npz"), {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()

"""Regenerates the golden fixtures in tests/golden/ from the reference's own
host code (oracle/_ref/libre_ref.so, built from the reference sources by
oracle/Makefile.ref) and the CPU oracle.

    python tests/golden/make_golden.py

Fixtures:
  perm.npz           RPerlinNoise(seed).permutationTable for several seeds,
                     produced by the reference's PerlinNoise.h.
  ref_soup.npz       a 4096-triangle soup, the reference RKDTreeCPU/RKDThreeGPU
                     build of it (raw 128-byte RKDTreeNodeGPU records and
                     obj_index_list), and the closest hits of a 48x48 primary
                     image traced the way the reference traverses that tree
                     (root-box test, then Moller-Trumbore over the leaf's
                     obj_index_list in order, keeping t < t_exit).
  ref_grid.npz       the same for a 16x16-cell heightfield (shared edges).
  noise.npz          fBm values of the restated Perlin noise at fixed points.
  bunny.npz          real geometry: Sandbox/Meshes/bun_zipper.ply (the Stanford
                     bunny the reference ships, 35,947 vertices, 69,451 faces)
                     as the reference's own rply reader returns it, and the
                     closest-hit distances of a 128x128 primary image of the
                     mesh scaled by 10 (the reference's absolute triangle-test
                     epsilons reject the raw metre-sized model's triangles),
                     traced by the reference's compiled CPU query
                     RKDTreeCPU::singleRayStacklessIntersect.

    python tests/golden/make_golden.py [--only bunny]
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import pyoracle as po  # noqa: E402


class _Cam:
    """Minimal stand-in with re_camera's fields for the oracle binding."""

    def __init__(self, campos, lookat, fov):
        v = np.asarray(lookat, np.float64) - np.asarray(campos, np.float64)
        v /= np.linalg.norm(v)
        self.campos = [float(x) for x in campos]
        self.view = [float(x) for x in v]
        self.camdown = [0.0, -1.0, 0.0]
        self.fov = [float(fov[0]), float(fov[1])]
        self.focial_distance = 1.0


def traced_reference(verts, faces, cam, w, h):
    nodes, idx, root, levels, leaves = po.ref_build(verts, faces)
    rn = po.ref_node_fields(nodes[root])
    assert rn["is_leaf"], "the shipped reference builder makes a single leaf"
    order = idx[rn["first"]: rn["first"] + rn["num_objs"]]
    v0 = verts[faces[order, 0]]
    packed = np.zeros((len(order), 12), np.float32)
    packed[:, 0:3] = v0
    packed[:, 4:7] = verts[faces[order, 1]] - v0
    packed[:, 8:11] = verts[faces[order, 2]] - v0
    hits = po.primary_bruteforce(packed, rn["min"], rn["max"], cam, w, h)
    # map leaf-local positions back to face ids
    ids = hits["id"].copy()
    ids[ids >= 0] = order[ids[ids >= 0]]
    hits["id"] = ids
    return nodes, idx, root, levels, leaves, hits


BUNNY_SCALE = 10.0
BUNNY_CAM = ((0.0, 1.0, 2.5), 45.0)  # offset of the camera from the bunny's centre, fov


def bunny_camera(verts):
    c = (verts.min(0) + verts.max(0)) / 2
    off, fov = BUNNY_CAM
    return _Cam((float(c[0]) + off[0], float(c[1]) + off[1], float(c[2]) + off[2]),
                (float(c[0]), float(c[1]), float(c[2])), (fov, fov))


def bunny():
    from oracle.refpath import reference_file

    path = reference_file("Sandbox", "Meshes", "bun_zipper.ply")
    if path is None or po.ref_ply_lib() is None:
        raise SystemExit("the reference checkout (bun_zipper.ply) or oracle/_ref/libre_ply.so missing")
    ok, verts, faces = po.ref_ply_load(path)
    assert ok and verts.shape == (35947, 3) and faces.shape == (69451, 3)
    sv = (verts * np.float32(BUNNY_SCALE)).astype(np.float32)
    cam = bunny_camera(sv)
    w = h = 128
    o, d = po.camera_rays(cam, w, h, np.arange(w * h))
    tree = po.RefTree(sv, faces)
    t, _, _ = tree.trace(o, d)
    tree.close()
    np.savez_compressed(os.path.join(HERE, "bunny.npz"), verts=verts, faces=faces,
                        scale=np.float32(BUNNY_SCALE), campos=cam.campos, view=cam.view,
                        fov=cam.fov, w=w, h=h, ref_t=t)


def main():
    if po.ref_lib() is None:
        raise SystemExit("oracle/_ref/libre_ref.so missing: make -f oracle/Makefile.ref")
    if "--only" in sys.argv:
        which = sys.argv[sys.argv.index("--only") + 1]
        {"bunny": bunny}[which]()
        print("golden fixture", which, "written to", HERE)
        return
    bunny()
    seeds = np.array([2016, 0, 1, 7, 12345], np.uint32)
    np.savez_compressed(os.path.join(HERE, "perm.npz"), seeds=seeds,
                        tables=np.stack([po.ref_perm(int(s)) for s in seeds]))

    # soup
    n = 4096
    tri = po.soup(3, n)
    verts = tri.reshape(-1, 3)
    faces = np.arange(3 * n, dtype=np.uint32).reshape(n, 3)
    cam = _Cam((0.0, 0.0, 3.0), (0.0, 0.0, 0.0), (60.0, 60.0))
    nodes, idx, root, levels, leaves, hits = traced_reference(verts, faces, cam, 48, 48)
    np.savez_compressed(os.path.join(HERE, "ref_soup.npz"), verts=verts, faces=faces,
                        nodes=nodes, index_list=idx, root=root, levels=levels, leaves=leaves,
                        campos=cam.campos, view=cam.view, fov=cam.fov, w=48, h=48,
                        hits=hits.view(np.int32).reshape(-1, 4))

    # heightfield
    P = po.perm(2016)
    gv, gf = po.heightfield(P, 16, -2.0, 2.0, 6, 0.5)
    cam = _Cam((0.0, 2.0, -3.0), (0.0, 0.0, 0.0), (60.0, 60.0))
    nodes, idx, root, levels, leaves, hits = traced_reference(gv, gf, cam, 40, 40)
    np.savez_compressed(os.path.join(HERE, "ref_grid.npz"), verts=gv, faces=gf, nodes=nodes,
                        index_list=idx, root=root, levels=levels, leaves=leaves,
                        campos=cam.campos, view=cam.view, fov=cam.fov, w=40, h=40,
                        hits=hits.view(np.int32).reshape(-1, 4))

    # noise values
    rng = np.random.default_rng(11)
    pts = np.concatenate([
        rng.uniform(-300, 300, (200, 3)),
        rng.uniform(-2, 2, (200, 3)),
        np.array([[0, 0, 0], [1, 1, 1], [-1, -1, -1], [255, 0, 3], [256, 0, 0], [0.5, 0.5, 0.5]]),
    ]).astype(np.float32)
    vals = {f"fbm{o}": po.fbm_batch(P, pts, o) for o in (1, 6, 8)}
    np.savez_compressed(os.path.join(HERE, "noise.npz"), pts=pts, **vals)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()

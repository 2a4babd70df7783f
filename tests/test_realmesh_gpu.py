"""Real geometry and closed meshes on the GPU.

* The Stanford bunny the reference ships (Sandbox/Meshes/bun_zipper.ply,
  69,451 faces, committed as tests/golden/bunny.npz by make_golden.py from
  the reference's own rply reader), scaled by 10: every primary ray
  bit-exact against the oracle's walk of the same tree, ids against brute
  force (the reference as shipped) under the FP64 edge-margin rule, and hit
  distances against the reference's compiled CPU query
  (RKDTreeCPU::singleRayStacklessIntersect) within 1e-5; an AO frame on it
  bit-exact against the oracle.
* Watertightness of the closed heightfield: vertical rays through every
  interior grid vertex and edge midpoint.  The leaf test is the reference's
  epsilon Moller-Trumbore (ray_functions.cuh:174-223, KDTree.cpp:909-949),
  which is not watertight at shared vertices; the count of rays that pass
  through is printed and must equal brute force's (the kd traversal adds no
  leak of its own).
"""
import os

import numpy as np
import pytest
import torch

import rayengine_b200 as rb
from oracle import pyoracle as po
from test_gpu_parity import _assert_vs_bruteforce, _hits, _kd

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _bunny():
    g = np.load(os.path.join(GOLDEN, "bunny.npz"))
    v = (g["verts"] * g["scale"]).astype(np.float32)
    f = g["faces"]
    campos = [float(x) for x in g["campos"]]
    cam = rb.build_camera(campos, [campos[i] + float(g["view"][i]) for i in range(3)],
                          [float(x) for x in g["fov"]])
    cam.view[:] = [float(x) for x in g["view"]]
    cam.camdir[:] = [float(x) for x in g["view"]]
    return g, v, f, cam


def test_bunny_primary_rays(cuda):
    g, v, f, cam = _bunny()
    w, h = int(g["w"]), int(g["h"])
    packed = rb.pack_triangles(v, f)
    with rb.KDScene.from_mesh(v, f) as sc:
        st, kd = _kd(sc)
        got = _hits(sc.trace_primary(cam, w, h))
    ref = po.primary_kd(kd, cam, w, h)
    assert np.array_equal(got, ref.view(np.int32).reshape(-1, 4))
    hit = got[:, 0] >= 0
    assert 0.25 < hit.mean() < 0.6
    pix = np.arange(w * h, dtype=np.uint32)
    _assert_vs_bruteforce(got, packed, st, cam, w, h, pix, label="bunny 128x128")
    # the reference's compiled query on the same rays (its rays come from the
    # FP64 camera, so grazing rays may differ: exempt by the edge margin)
    rt = g["ref_t"]
    rhit = rt < 1e19
    differ = np.nonzero(rhit != hit)[0]
    if differ.size:
        o, d = po.camera_rays(cam, w, h, differ)
        bf = po.primary_bruteforce(packed, st["bmin"], st["bmax"], cam, w, h, pixels=differ)
        ids = np.where(got[differ, 0] >= 0, got[differ, 0], bf["id"])
        assert np.all(ids >= 0)
        assert np.all(po.edge_margin(packed, ids, o, d) < 1e-5)
    both = rhit & hit
    gt = got[both, 1].view(np.float32).astype(np.float64)
    rel = np.abs(gt - rt[both]) / rt[both]
    print(f"bunny vs the reference's compiled query: {int(both.sum())} hits, "
          f"{differ.size} hit/miss differences (grazing), max rel t {rel.max():.2e}")
    assert rel.max() <= 1e-5


def test_bunny_ao_frame(cuda):
    g, v, f, cam = _bunny()
    w, h = 160, 120
    cam.fov[:] = [45.0, rb.vertical_fov(45.0, w, h)]
    packed = rb.pack_triangles(v, f)
    light = rb.unit((0.3, 1.0, 0.2))
    with rb.KDScene.from_mesh(v, f) as sc:
        st, kd = _kd(sc)
        hits, mask, nsec = sc.render_ao(cam, w, h, light, 0.1, 1e-4, 5)
        hits, mask = _hits(hits), mask.cpu().numpy().view(np.uint32)
    rh, rm, rn = po.frame_ao(kd, packed, cam, w, h, light, 0.1, 1e-4, 5)
    assert np.array_equal(hits, rh.view(np.int32).reshape(-1, 4))
    assert np.array_equal(mask, rm)
    assert int(nsec.item()) == rn > 0
    hit = (rm & 1) == 1
    assert (((rm[hit] >> 2) & 15) != 15).mean() > 0.05  # some AO rays occluded


@pytest.mark.parametrize("cells", [64, 256])
def test_heightfield_edges_and_vertices(cuda, cells):
    cfg = rb.configs.HeightfieldConfig(cells=cells)
    verts, faces = po.heightfield(po.perm(cfg.seed), cfg.cells, cfg.lo, cfg.hi, cfg.octaves,
                                  cfg.amplitude)
    nv = cells + 1
    g = verts.reshape(nv, nv, 3)
    xs, zs = g[0, :, 0], g[:, 0, 2]
    mx = ((xs[:-1] + xs[1:]) / 2).astype(np.float32)
    mz = ((zs[:-1] + zs[1:]) / 2).astype(np.float32)
    pts = []
    for ax, az in ((xs[1:-1], zs[1:-1]), (mx, zs[1:-1]), (xs[1:-1], mz), (mx, mz)):
        X, Z = np.meshgrid(ax, az)
        pts.append(np.stack([X.ravel(), Z.ravel()], 1))
    P = np.concatenate(pts).astype(np.float32)
    n = P.shape[0]
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0], rays[:, 1], rays[:, 2], rays[:, 3], rays[:, 5] = P[:, 0], 10.0, P[:, 1], np.inf, -1.0
    packed = rb.pack_triangles(verts, faces)
    with rb.KDScene.from_mesh(verts, faces) as sc:
        st, kd = _kd(sc)
        got = _hits(sc.trace_rays(torch.from_numpy(rays).cuda()))
    assert np.array_equal(got, po.rays_kd(kd, rays).view(np.int32).reshape(-1, 4))
    # brute force: the same leaf test over every triangle (a one-leaf tree)
    with rb.KDScene.build_host(packed, rb.kd_params(max_depth=1, leaf_size=1 << 30)) as one:
        s1 = one.stats()
        n1, l1, t1 = one.export()
    bf = po.rays_kd(po.KdTree(n1, l1, t1, s1["bmin"], s1["bmax"]), rays)
    leaks = int((got[:, 0] < 0).sum())
    print(f"heightfield {cells}x{cells}: {leaks} of {n} vertical rays through vertices and "
          f"edge midpoints pass through (brute force: {int((bf['id'] < 0).sum())})")
    assert np.array_equal(got[:, 0] < 0, bf["id"] < 0)
    assert leaks <= max(1, n // 10000)

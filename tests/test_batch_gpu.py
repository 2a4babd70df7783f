"""Batched wavefront path tracer on the GPU against the CPU oracle.

Meshes and terrains of different sizes and resolutions in one batch; the
oracle follows each pixel's path with brute-force closest hits and the
exact SDF march, so radiance, primary hits and rays per bounce must agree
bit for bit.
"""
import numpy as np
import pytest
import torch

import rayengine_b200 as rb
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

DEPTH, SEED, BIAS = 4, 11, 1e-4


def _soup(n, seed):
    cfg = rb.configs.SoupConfig(num_tris=n, seed=seed)
    return cfg.packed()


def _heightfield(cells):
    cfg = rb.configs.HeightfieldConfig(cells=cells)
    verts, faces = po.heightfield(po.perm(cfg.seed), cfg.cells, cfg.lo, cfg.hi, cfg.octaves,
                                  cfg.amplitude)
    return rb.pack_triangles(verts, faces), cfg


def _build(cuda):
    specs = []
    meshes = []
    for n, seed, w, h in ((2048, 3, 48, 32), (6000, 4, 33, 21)):
        packed = _soup(n, seed)
        sc = rb.KDScene.from_packed(packed)
        meshes.append(sc)
        cam = rb.build_camera((0, 0, 3), (0, 0, 0), (60.0, rb.vertical_fov(60.0, w, h)))
        specs.append(dict(mesh=sc, packed=packed, camera=cam, width=w, height=h, albedo=0.7))
    packed, hc = _heightfield(24)
    sc = rb.KDScene.from_packed(packed)
    meshes.append(sc)
    hcam = rb.build_camera(hc.campos, hc.lookat, (60.0, rb.vertical_fov(60.0, 40, 30)))
    specs.append(dict(mesh=sc, packed=packed, camera=hcam, width=40, height=30, albedo=0.5))
    for seed, amp, w, h in ((2016, 3.0, 40, 24), (7, 2.0, 24, 18)):
        tc = rb.configs.TerrainConfig(seed=seed, amplitude=amp, width=w, height=h)
        specs.append(dict(terrain=tc.params(), tc=tc, camera=tc.camera(), width=w, height=h,
                          albedo=0.6))
    # interleave kinds so scene boundaries mix meshes and terrains
    order = [0, 3, 1, 4, 2]
    specs = [specs[i] for i in order]
    return specs, meshes


def _oracle(specs, batch):
    scenes = []
    for s in specs:
        if "mesh" in s:
            st = s["mesh"].stats()
            scenes.append(dict(kind=0, tris=s["packed"], bmin=st["bmin"], bmax=st["bmax"],
                               cam=s["camera"], w=s["width"], h=s["height"], albedo=s["albedo"]))
        else:
            f = s["terrain"]
            scenes.append(dict(kind=1, seed=f.seed, octaves=f.octaves, scale=f.scale,
                               amp=f.amplitude, step_factor=f.step_factor, eps=f.eps,
                               tmax=f.tmax, max_steps=f.max_steps, cam=s["camera"],
                               w=s["width"], h=s["height"], albedo=s["albedo"]))
    g = np.arange(batch.total_pixels, dtype=np.uint32)
    return po.batch_path(scenes, batch.offsets, g, DEPTH, SEED, BIAS)


def test_batch_matches_oracle_bit_exact(cuda):
    specs, meshes = _build(cuda)
    with rb.Batch(specs, max_depth=DEPTH, seed=SEED, mesh_bias=BIAS) as b:
        prim = torch.empty((b.total_pixels, 4), dtype=torch.int32, device="cuda")
        rad = b.render(primary=prim).cpu().numpy()
        st = b.stats()
        assert st["error"] == 0
        orad, oprim, onrays = _oracle(specs, b)
        assert np.array_equal(rad.view(np.uint32), orad.view(np.uint32))
        p = prim.cpu().numpy()
        assert np.array_equal(p[:, 0], oprim[:, 0])
        assert np.array_equal(p[:, 1], oprim[:, 1])  # t bits
        mesh_px = np.concatenate([np.arange(b.offsets[i], b.offsets[i] + s["width"] * s["height"])
                                  for i, s in enumerate(specs) if "mesh" in s]).astype(np.int64)
        assert np.array_equal(p[mesh_px, 2:], oprim[mesh_px, 2:])
        # rays per bounce: bounce 0 = every pixel; deeper bounces by scene kind
        kind = np.zeros(b.total_pixels, np.int64)
        for i, s in enumerate(specs):
            if "terrain" in s:
                kind[b.offsets[i]:b.offsets[i] + s["width"] * s["height"]] = 1
        assert st["rays"][0, 0] == b.total_pixels
        for bounce in range(1, DEPTH):
            for k in (0, 1):
                assert st["rays"][bounce, k] == int(((onrays > bounce) & (kind == k)).sum())
        # mesh primary hits equal the single-scene two-sided primary pass
        for i, s in enumerate(specs):
            if "mesh" not in s:
                continue
            w, h = s["width"], s["height"]
            single = s["mesh"].trace_primary(s["camera"], w, h).cpu().numpy()
            assert np.array_equal(single, p[b.offsets[i]:b.offsets[i] + w * h])
    for m in meshes:
        m.close()


def test_graph_replay_and_tunings_give_identical_frames(cuda):
    specs, meshes = _build(cuda)
    with rb.Batch(specs, max_depth=DEPTH, seed=SEED, mesh_bias=BIAS) as b:
        ref = b.render().cpu().numpy()
        out = torch.empty(b.total_pixels, dtype=torch.float32, device="cuda")
        for _ in range(3):  # capture, then replays (counters reset by the kernel itself)
            out.fill_(-1.0)
            b.render(out=out, graph=True)
            assert np.array_equal(out.cpu().numpy(), ref)
            assert b.stats()["error"] == 0
        for bt, rf, sg, sp in ((128, 1, 0, 1), (64, 32, 64, 64), (256, 8, 512, 8)):
            b.set_tuning(bt, rf, sg, sp)
            assert np.array_equal(b.render().cpu().numpy(), ref)
        t = b.autotune()
        assert t["block_threads"] in (128, 256) and t["frame_ms"] > 0
        assert np.array_equal(b.render(graph=True).cpu().numpy(), ref)
        with pytest.raises(rb.RayEngineError):
            b.set_tuning(512, 8, 0)
    for m in meshes:
        m.close()


def test_batch_with_many_terrain_seeds_bit_exact(cuda):
    """More distinct terrain seeds than the word-table limit (16): the
    kernel keeps its noise tables as bytes; the frame must still match the
    oracle bit for bit."""
    specs, meshes = [], []
    packed = _soup(3000, 9)
    sc = rb.KDScene.from_packed(packed)
    meshes.append(sc)
    w, h = 24, 16
    cam = rb.build_camera((0, 0, 3), (0, 0, 0), (60.0, rb.vertical_fov(60.0, w, h)))
    specs.append(dict(mesh=sc, packed=packed, camera=cam, width=w, height=h, albedo=0.7))
    for i in range(18):
        tc = rb.configs.TerrainConfig(seed=100 + i, amplitude=1.5 + 0.1 * i, width=16, height=10)
        specs.append(dict(terrain=tc.params(), tc=tc, camera=tc.camera(), width=16, height=10,
                          albedo=0.6))
    with rb.Batch(specs, max_depth=DEPTH, seed=SEED, mesh_bias=BIAS) as b:
        rad = b.render().cpu().numpy()
        assert b.stats()["error"] == 0
        orad, _, _ = _oracle(specs, b)
        assert np.array_equal(rad.view(np.uint32), orad.view(np.uint32))
        assert np.array_equal(b.render(graph=True).cpu().numpy(), rad)
    for m in meshes:
        m.close()


def test_wait_bounds_run_out_and_the_next_frame_recovers(cuda):
    """The persistent kernel bounds its loop and its polls of queue slots.
    Lowered bounds must make a frame end early with the error flag set (no
    wait runs on), and the next frame with the default bounds must be whole
    again.  Two trips of the loop cannot finish a depth-4 path (each bounce
    ray is claimed in a later trip than the ray that made it), so the
    loop-bound case always trips; the second case also lowers the poll bound."""
    specs, meshes = _build(cuda)
    with rb.Batch(specs, max_depth=DEPTH, seed=SEED, mesh_bias=BIAS) as b:
        ref = b.render().cpu().numpy()
        assert b.stats()["error"] == 0
        for pending, trips in ((0, 2), (64, 4096)):
            b.set_wait_bounds(pending, trips)
            for graph in (False, True):
                b.render(graph=graph)
                torch.cuda.synchronize()
                st = b.stats()
                assert st["error"] == 1, (pending, trips, graph)
            b.set_wait_bounds(0, 0)
            assert np.array_equal(b.render().cpu().numpy(), ref)
            assert b.stats()["error"] == 0
            assert np.array_equal(b.render(graph=True).cpu().numpy(), ref)
            assert b.stats()["error"] == 0
    for m in meshes:
        m.close()

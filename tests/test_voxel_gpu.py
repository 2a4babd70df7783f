"""Voxel SDF on the GPU against the CPU oracle: bake, the three samplers
and the voxel sphere tracer, bit for bit; .rsdf round trip."""
import numpy as np
import pytest
import torch

import rayengine_b200 as rb
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

DIM, SP, ORG = (48, 24, 40), (0.5, 0.5, 0.5), (-12.0, -6.0, -4.0)


def _grid():
    tc = rb.configs.TerrainConfig()
    return tc, rb.VoxelGrid.bake(tc.params(), DIM, SP, ORG)


def test_bake_and_samplers_match_oracle(cuda):
    tc, g = _grid()
    got = g.data.cpu().numpy()
    want = po.voxel_bake(po.perm(tc.seed), tc.octaves, tc.scale, tc.amplitude, DIM, SP, ORG)
    assert np.array_equal(got, want)
    rng = np.random.default_rng(2)
    lo = np.array(ORG, np.float32) - 1.0
    hi = np.array(ORG, np.float32) + np.array(DIM, np.float32) * 0.5 + 1.0
    pts = rng.uniform(lo, hi, (20000, 3)).astype(np.float32)
    d = torch.from_numpy(pts).cuda()
    for q in (rb.VOXEL_LOW, rb.VOXEL_MEDIUM, rb.VOXEL_HIGH):
        s = g.sample(d, q).cpu().numpy()
        assert np.array_equal(s, po.voxel_sample(got, DIM, SP, ORG, q, pts)), q


def test_voxel_trace_matches_oracle_and_file_round_trip(cuda, tmp_path):
    tc, g = _grid()
    w, h = 80, 45
    cam = rb.build_camera((0.0, 6.0, -14.0), (0.0, 0.0, 6.0), (60.0, rb.vertical_fov(60.0, w, h)))
    march = rb.sdf_params(step_factor=0.6, eps=1e-3, tmax=100.0, max_steps=256)
    grid = g.data.cpu().numpy()
    for q in (rb.VOXEL_LOW, rb.VOXEL_MEDIUM, rb.VOXEL_HIGH):
        out = g.trace(q, march, cam, w, h).cpu().numpy()
        ref = po.voxel_trace(grid, DIM, SP, ORG, q, 0.6, 1e-3, 100.0, 256, cam, w, h)
        f = out.view(np.float32).reshape(-1, 8)
        u = out.view(np.uint32).reshape(-1, 8)
        assert np.array_equal(u[:, 7], ref["status"]), q
        assert np.array_equal(u[:, 6], ref["steps"]), q
        hit = ref["status"] == 1
        assert hit.mean() > 0.3
        assert np.array_equal(f[hit, 0:3], ref["pos"][hit])
        assert np.array_equal(f[hit, 3], ref["normal"][hit, 0])
        assert np.array_equal(f[hit, 4:6], ref["normal"][hit, 1:3])
    path = str(tmp_path / "terrain.rsdf")
    g.save(path)
    g2 = rb.VoxelGrid.load(path, origin=ORG)
    assert np.array_equal(g2.data.cpu().numpy(), grid)
    a = g.trace(rb.VOXEL_MEDIUM, march, cam, w, h).cpu().numpy()
    b = g2.trace(rb.VOXEL_MEDIUM, march, cam, w, h).cpu().numpy()
    assert np.array_equal(a, b)


def test_brush_edits_match_oracle(cuda):
    tc, g = _grid()
    grid = g.data.cpu().numpy()
    edits = [(rb.BRUSH_SPHERE_ADD, (0.0, 1.0, 4.0), 2.0, 3.0),
             (rb.BRUSH_SPHERE_SUBTRACT, (2.0, -0.5, 6.0), 1.5, 4.0),
             (rb.BRUSH_CUBE_ADD, (-4.0, 0.5, 8.0), (1.0, 2.0, 1.5), 5.0),
             (rb.BRUSH_CUBE_SUBTRACT, (3.0, 0.0, 2.0), (2.0, 1.0, 1.0), 6.0)]
    for kind, c, e, mat in edits:
        g.brush(kind, c, e, material=mat, smooth=0.1)
        grid = po.voxel_brush(grid, DIM, SP, ORG, kind, c, e, mat, 0.1)
        assert np.array_equal(g.data.cpu().numpy(), grid), kind
    # the edits changed the field
    assert not np.array_equal(grid, po.voxel_bake(po.perm(tc.seed), tc.octaves, tc.scale,
                                                  tc.amplitude, DIM, SP, ORG))

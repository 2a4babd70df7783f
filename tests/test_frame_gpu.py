"""Shaded RGBA8 frame (the reference's render call) against the CPU oracle."""
import numpy as np
import pytest
import torch

import rayengine_b200 as rb
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

LIGHTS = [((2.0, 3.0, 4.0), 20000.0), ((-3.0, 2.0, 1.0), 8000.0)]


def _soup(n=4096):
    packed = rb.configs.SoupConfig(num_tris=n, seed=5).packed()
    return packed, rb.KDScene.from_packed(packed)


def _check(scene, packed, cam, w, h, shade, lights, mode):
    got = scene.render_frame(cam, w, h, lights, shade).cpu().numpy().view(np.uint32)
    st = scene.stats()
    want = po.frame_rgba(packed, st["bmin"], st["bmax"], cam, w, h, lights, list(shade.albedo),
                         list(shade.sky_zenith), list(shade.sky_horizon), mode=mode)
    assert np.array_equal(got, want)
    return got


def test_frame_matches_oracle(cuda):
    packed, sc = _soup()
    with sc:
        w, h = 64, 48
        cam = rb.build_camera((0, 0, 3), (0, 0, 0), (60.0, rb.vertical_fov(60.0, w, h)))
        img = _check(sc, packed, cam, w, h, rb.shade_params(), LIGHTS, 0)
        assert len(np.unique(img)) > 50  # shaded, not flat
        assert np.all(img >> 24 == 255)
        _check(sc, packed, cam, w, h, rb.shade_params(albedo=(0.2, 0.3, 0.1), one_sided=True),
               LIGHTS, 1)
        _check(sc, packed, cam, w, h, rb.shade_params(), [], 0)  # no lights: albedo + sky


def test_frame_heightfield_with_shadows(cuda):
    cfg = rb.configs.HeightfieldConfig(cells=48)
    verts, faces = po.heightfield(po.perm(cfg.seed), cfg.cells, cfg.lo, cfg.hi, cfg.octaves,
                                  cfg.amplitude)
    packed = rb.pack_triangles(verts, faces)
    with rb.KDScene.from_packed(packed) as sc:
        w, h = 80, 45
        cam = rb.build_camera(cfg.campos, cfg.lookat, (60.0, rb.vertical_fov(60.0, w, h)))
        _check(sc, packed, cam, w, h, rb.shade_params(albedo=(0.1, 0.1, 0.1)),
               [((6.0, 5.0, -4.0), 20000.0)], 0)


def test_reference_render_call(cuda):
    packed, sc = _soup(2048)
    with sc:
        w, h = 40, 30
        cam = rb.build_camera((0, 0, 3), (0, 0, 0), (60.0, rb.vertical_fov(60.0, w, h)))
        shade = rb.shade_params()
        sc.bind_frame(cam, LIGHTS, shade, animate_light=True)
        out = torch.zeros(w * h, dtype=torch.int32, device="cuda")
        rb.cuda_render_frame(out, w, h)
        first = sc.render_frame(cam, w, h, LIGHTS, shade).cpu().numpy()
        assert np.array_equal(out.cpu().numpy(), first)
        # the light animation moved light 0 to x = z = 20 cos(0)
        rb.cuda_render_frame(out, w, h)
        moved = [((20.0, 3.0, 20.0), 20000.0), LIGHTS[1]]
        second = sc.render_frame(cam, w, h, moved, shade).cpu().numpy()
        assert np.array_equal(out.cpu().numpy(), second)

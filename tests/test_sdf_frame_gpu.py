"""The shaded SDF terrain frame (the reference's shipped render path,
render_sphere_trace behind cuda_render_frame) against the CPU oracle.

Bar: every RGBA8 pixel equal to the oracle's (the kernel and the oracle
share one operation sequence, including the frame's own e^x, ln x, x^y),
for each combination of the shading switches; at 1920x1080 on a seeded
pixel sample.  The elementary functions are also checked against CUDA's own
expf / logf / powf (their stated error bound).
"""
import numpy as np
import pytest
import torch

import rayengine_b200 as rb
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def test_fmath_bitexact_and_within_bounds(cuda):
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.uniform(-90, 90, 200000), rng.uniform(-1, 1, 100000),
                        [-87.5, -87.0, 0.0, 1e-30, 88.0, 89.0]]).astype(np.float32)
    got = rb.fmath(0, torch.from_numpy(x).cuda()).cpu().numpy()
    assert np.array_equal(got.view(np.uint32), po.fmath(0, x).view(np.uint32))
    ok = (x > -87.0) & (x < 88.0)
    ref = torch.exp(torch.from_numpy(x[ok]).cuda()).cpu().numpy().astype(np.float64)
    assert np.max(np.abs(got[ok] - ref) / ref) < 4e-7
    lx = np.exp(rng.uniform(-80, 80, 300000)).astype(np.float32)
    lx = lx[(lx > 1.2e-38) & np.isfinite(lx)]
    gl = rb.fmath(1, torch.from_numpy(lx).cuda()).cpu().numpy()
    assert np.array_equal(gl.view(np.uint32), po.fmath(1, lx).view(np.uint32))
    ref = torch.log(torch.from_numpy(lx).cuda()).cpu().numpy().astype(np.float64)
    # a few units in the last place: relative for |ln x| > 1, absolute near x = 1
    assert np.all(np.abs(gl - ref) <= 2e-6 + 4e-7 * np.abs(ref))
    y = rng.uniform(0.05, 3.0, lx.size).astype(np.float32)
    px = np.exp(rng.uniform(-20, 3, lx.size)).astype(np.float32)
    gp = rb.fmath(2, torch.from_numpy(px).cuda(), torch.from_numpy(y).cuda()).cpu().numpy()
    assert np.array_equal(gp.view(np.uint32), po.fmath(2, px, y).view(np.uint32))
    ref = torch.pow(torch.from_numpy(px).cuda().double(), torch.from_numpy(y).cuda().double())
    ref = ref.cpu().numpy()
    assert np.max(np.abs(gp - ref) / ref) < 1e-5


FLAG_SETS = [rb.SDF_SHADE, 0, rb.SDF_SHADE | rb.SDF_FOG | rb.SDF_GAMMA | rb.SDF_VIGNETTING,
             rb.SDF_FOG | rb.SDF_VIGNETTING]


@pytest.mark.parametrize("flags", FLAG_SETS)
def test_sdf_frame_small_bitexact(cuda, flags):
    tc = rb.configs.TerrainConfig(width=192, height=108)
    shade = rb.sdf_shade_params(flags=flags)
    img, hits = rb.render_sdf_frame(tc.params(), shade, tc.camera(), tc.width, tc.height)
    got = img.cpu().numpy().view(np.uint32)
    want = po.sdf_frame(po.perm(tc.seed), tc.camera(), tc.width, tc.height, tc.params(), shade)
    assert np.array_equal(got, want)
    assert np.all(got >> 24 == 255)
    assert len(np.unique(got)) > (200 if flags & (rb.SDF_SHADE | rb.SDF_FOG) else 20)
    # the hit record is the plain tracer's
    plain = rb.sphere_trace(tc.params(), tc.camera(), tc.width, tc.height).cpu().numpy()
    assert np.array_equal(hits.cpu().numpy(), plain)


def test_sdf_frame_sky_and_shadow_paths(cuda):
    """A camera that sees both terrain and a large sky, a low sun and a
    light that throws long shadows: every pixel equal to the oracle, and the
    shadow march's evaluation count equal to the oracle's total."""
    tc = rb.configs.TerrainConfig(width=160, height=90, campos=(0.0, 4.0, -20.0),
                                  lookat=(0.0, 4.5, 0.0))
    shade = rb.sdf_shade_params(light_pos=(-30.0, 8.0), sun_dir=(0.0, 0.2, 0.98),
                                shadow_max_steps=256, shadow_tmax=60.0)
    field, cam = tc.params(), tc.camera()
    hits = rb.sphere_trace(field, cam, tc.width, tc.height)
    ev = torch.zeros(1, dtype=torch.int64, device="cuda")
    got = rb.shade_sdf(field, shade, cam, tc.width, tc.height, hits, evals=ev).cpu().numpy()
    want, oev = po.sdf_frame(po.perm(tc.seed), cam, tc.width, tc.height, field, shade, evals=True)
    assert np.array_equal(got.view(np.uint32), want)
    assert int(ev.item()) == int(oev.astype(np.int64).sum())
    st = hits.cpu().numpy()[:, 7].view(np.uint32)
    assert 0.2 < (st == 1).mean() < 0.9  # both sky and terrain in view
    assert oev.max() > 20  # shadow rays march far


def test_sdf_frame_1080p_sampled(cuda):
    tc = rb.configs.TerrainConfig()
    W, H = tc.width, tc.height
    shade = rb.sdf_shade_params(flags=rb.SDF_SHADE | rb.SDF_FOG | rb.SDF_GAMMA |
                                rb.SDF_VIGNETTING)
    img, _ = rb.render_sdf_frame(tc.params(), shade, tc.camera(), W, H)
    img2, _ = rb.render_sdf_frame(tc.params(), shade, tc.camera(), W, H)
    got = img.cpu().numpy().view(np.uint32)
    assert np.array_equal(got, img2.cpu().numpy().view(np.uint32))
    pix = np.random.default_rng(9).choice(W * H, 3000, replace=False).astype(np.uint32)
    want = po.sdf_frame(po.perm(tc.seed), tc.camera(), W, H, tc.params(), shade, pixels=pix)
    assert np.array_equal(got[pix], want)


def test_reference_render_call_sdf_mode(cuda):
    """cuda_render_frame after re_sdf_frame_bind renders the terrain frame
    (the reference's shipped mode) and moves the sun as Craze does; binding
    a mesh scene switches the call back to the kd-tree frame."""
    tc = rb.configs.TerrainConfig(width=96, height=54)
    w, h = tc.width, tc.height
    shade = rb.sdf_shade_params()
    rb.bind_sdf_frame(tc.params(), shade, tc.camera(), animate_sun=True)
    out = torch.zeros(w * h, dtype=torch.int32, device="cuda")
    assert rb.cuda_render_frame(out, w, h) == ""
    first, _ = rb.render_sdf_frame(tc.params(), shade, tc.camera(), w, h)
    assert np.array_equal(out.cpu().numpy(), first.cpu().numpy())
    # after the first frame the sun is (0, cos a, sin a) with a = 0
    rb.cuda_render_frame(out, w, h)
    moved = rb.sdf_shade_params(sun_dir=(0.0, 1.0, 0.0))
    second, _ = rb.render_sdf_frame(tc.params(), moved, tc.camera(), w, h)
    assert np.array_equal(out.cpu().numpy(), second.cpu().numpy())
    assert not np.array_equal(first.cpu().numpy(), second.cpu().numpy())
    # a mesh binding takes the call back to the kd-tree frame
    packed = rb.configs.SoupConfig(num_tris=2048, seed=5).packed()
    with rb.KDScene.from_packed(packed) as sc:
        cam = rb.build_camera((0, 0, 3), (0, 0, 0), (60.0, rb.vertical_fov(60.0, w, h)))
        lights = [((2.0, 3.0, 4.0), 20000.0)]
        sc.bind_frame(cam, lights, rb.shade_params())
        rb.cuda_render_frame(out, w, h)
        mesh = sc.render_frame(cam, w, h, lights, rb.shade_params()).cpu().numpy()
        assert np.array_equal(out.cpu().numpy(), mesh)

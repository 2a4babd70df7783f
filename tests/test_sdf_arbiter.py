"""The FP64 arbiter of SDF hit positions (oracle) on the exact-SDF terrain.

The arbiter marches the same rule as the float tracer (t += 0.6 d) in double
precision and bisects the first crossing it reaches to the density's root.
Without the bisection it reproduces the float march to rounding; with it,
it measures how far the 0.6-step march ends inside the terrain.
"""
import numpy as np

import rayengine_b200 as rb
from oracle import pyoracle as po


def _setup(n=3000):
    tc = rb.configs.TerrainConfig()
    P = po.perm(tc.seed)
    cam = tc.camera()
    pix = np.random.default_rng(3).choice(tc.width * tc.height, n, replace=False).astype(np.uint32)
    o = po.sdf_image(P, cam, tc.width, tc.height, pixels=pix)
    arr = np.zeros((tc.width * tc.height, 8), np.float32)
    arr[pix, 0:3] = o["pos"]
    arr[pix, 7] = o["status"].view(np.float32)
    return tc, P, cam, pix, arr.view(np.int32)


def test_arbiter_reproduces_the_float_march_and_finds_roots():
    tc, P, cam, pix, out = _setup()
    pos, hit = po.sdf_arbiter(P, cam, tc.width, tc.height, pix, refine=False)
    err, mism, both = po.hit_errors(out, pos, hit, pix)
    assert mism == 0 and both > 0.8 * len(pix)
    assert np.median(err) < 1e-5
    rpos, rhit = po.sdf_arbiter(P, cam, tc.width, tc.height, pix, refine=True)
    assert np.array_equal(rhit, hit)
    # the bisected points are on the surface
    d = po.density_d(P, rpos[rhit])
    assert np.abs(d).max() < 1e-9


def test_exact_march_overshoots_the_surface():
    # the 0.6 d step over-estimates the distance where |grad d| > 1/0.6, so
    # the float tracer stops inside the terrain: its median error against
    # the root is well above 1e-3 scene units
    tc, P, cam, pix, out = _setup()
    rpos, rhit = po.sdf_arbiter(P, cam, tc.width, tc.height, pix, refine=True)
    err, mism, both = po.hit_errors(out, rpos, rhit, pix)
    assert mism == 0
    assert np.median(err) > 2e-3

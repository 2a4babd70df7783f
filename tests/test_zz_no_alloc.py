"""re_render_ao_noalloc: the AO frame for callers that cannot allocate device
memory while they render (an engine that owns all device memory through its
own pool, or a frame loop that cannot take cudaMalloc's implicit
synchronisation or an out-of-memory failure mid-frame).

Called through the C ABI and compared with re_render_ao, which grows its
queue with cudaMalloc, on two calls in a row (the fixed scratch keeps the
previous call's contents, so the second call checks that nothing leaks from
the first).  The file name makes pytest collect it last.
"""
import ctypes

import numpy as np
import pytest
import torch

import rayengine_b200 as rb
from rayengine_b200 import _lib
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

MAX_PIXELS = 419430  # RE_NOALLOC_MAX_PIXELS in include/rayengine_b200.h


def _frame(entry, sc, cam, w, h, params):
    primary = torch.empty((h * w, 4), dtype=torch.int32, device="cuda")
    mask = torch.empty(h * w, dtype=torch.int32, device="cuda")
    nsec = torch.zeros(1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    _lib.call(entry, sc.handle, ctypes.byref(cam), w, h, ctypes.byref(params),
              primary.data_ptr(), mask.data_ptr(), nsec.data_ptr(), stream)
    torch.cuda.synchronize()
    return primary.cpu().numpy(), mask.cpu().numpy(), int(nsec.item())


@pytest.mark.parametrize("kind_major", [0, 1, 2])
def test_noalloc_matches_render_ao_twice(cuda, kind_major):
    """Every secondary-queue layout (pixel-major; kind-major and shadow-first,
    whose AO records start at w*h inside the fixed array)."""
    cfg = rb.configs.HeightfieldConfig(cells=128, width=320, height=180)
    verts, faces = po.heightfield(po.perm(cfg.seed), cfg.cells, cfg.lo, cfg.hi, cfg.octaves,
                                  cfg.amplitude)
    cam = cfg.camera()
    with rb.KDScene.from_mesh(verts, faces) as sc:
        t = sc.tuning()
        sc.set_tuning(t["stage_nodes"], kind_major, t["refill_min"])
        for seed in (cfg.ao_seed, cfg.ao_seed + 1):
            params = rb.ao_params(cfg.light_dir, cfg.ao_length, cfg.bias, seed)
            want = _frame("re_render_ao", sc, cam, cfg.width, cfg.height, params)
            got = _frame("re_render_ao_noalloc", sc, cam, cfg.width, cfg.height, params)
            assert np.array_equal(got[0], want[0]), seed
            assert np.array_equal(got[1], want[1]), seed
            assert got[2] == want[2] and got[2] > 0, seed


@pytest.mark.parametrize("kind_major", [0, 1, 2])
def test_noalloc_largest_image(cuda, kind_major):
    """An image of 1024 x 409 = 418,816 pixels, just under the limit, with
    the camera close to the terrain so that almost every pixel hits: the
    queue's last records are written and read."""
    cfg = rb.configs.HeightfieldConfig(cells=128, width=1024, height=409,
                                       campos=(0.0, 3.0, -6.0))
    verts, faces = po.heightfield(po.perm(cfg.seed), cfg.cells, cfg.lo, cfg.hi, cfg.octaves,
                                  cfg.amplitude)
    cam = cfg.camera()
    assert cfg.width * cfg.height <= MAX_PIXELS
    with rb.KDScene.from_mesh(verts, faces) as sc:
        t = sc.tuning()
        sc.set_tuning(t["stage_nodes"], kind_major, t["refill_min"])
        params = rb.ao_params(cfg.light_dir, cfg.ao_length, cfg.bias, cfg.ao_seed)
        want = _frame("re_render_ao", sc, cam, cfg.width, cfg.height, params)
        for _ in range(2):
            got = _frame("re_render_ao_noalloc", sc, cam, cfg.width, cfg.height, params)
            assert np.array_equal(got[0], want[0])
            assert np.array_equal(got[1], want[1])
            assert got[2] == want[2]
        assert want[2] > 0.9 * 5 * cfg.width * cfg.height


def test_noalloc_rejects_images_beyond_its_scratch(cuda):
    cfg = rb.configs.HeightfieldConfig(cells=16)
    verts, faces = po.heightfield(po.perm(cfg.seed), cfg.cells, cfg.lo, cfg.hi, cfg.octaves,
                                  cfg.amplitude)
    with rb.KDScene.from_mesh(verts, faces) as sc:
        params = rb.ao_params(cfg.light_dir)
        w, h = 1024, MAX_PIXELS // 1024 + 1
        with pytest.raises(rb.RayEngineError) as e:
            _lib.call("re_render_ao_noalloc", sc.handle, ctypes.byref(cfg.camera()), w, h,
                      ctypes.byref(params), ctypes.c_void_p(256), ctypes.c_void_p(256), None,
                      None)
        assert e.value.status == 4 and "exceeds the fixed scratch" in str(e.value)

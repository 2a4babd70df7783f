"""Instanced scenes (per-object yaw + location, closest hit over objects)
against the CPU oracle, bit for bit."""
import numpy as np
import pytest

import rayengine_b200 as rb
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", [0, 1])
def test_instances_match_oracle(cuda, mode):
    objs = []
    for n, seed in ((3000, 11), (1500, 12)):
        packed = rb.configs.SoupConfig(num_tris=n, seed=seed).packed()
        objs.append((packed, rb.KDScene.from_packed(packed)))
    placements = [(0, 0.3, (0.8, 0.0, 0.0)), (1, -1.1, (-0.9, 0.2, 0.5)), (0, 2.0, (0.0, -1.2, -0.4))]
    try:
        w, h = 72, 48
        cam = rb.build_camera((0, 0, 4), (0, 0, 0), (60.0, rb.vertical_fov(60.0, w, h)))
        insts = [(objs[i][1], yaw, loc) for i, yaw, loc in placements]
        hits, idx = rb.trace_instances(insts, cam, w, h, flags=mode)
        hits, idx = hits.cpu().numpy(), idx.cpu().numpy()
        oi = []
        for i, yaw, loc in placements:
            st = objs[i][1].stats()
            oi.append((objs[i][0], st["bmin"], st["bmax"], rb.instance_trig(yaw), loc))
        want, widx = po.trace_instances(oi, cam, w, h, mode=mode)
        assert np.array_equal(idx, widx)
        assert np.array_equal(hits.view(po.HIT_DTYPE).reshape(-1).view(np.int32),
                              want.view(np.int32))
        assert len(np.unique(widx)) == 4  # every instance and the background appear
    finally:
        for _, sc in objs:
            sc.close()

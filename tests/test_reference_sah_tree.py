"""The reference arm's configured tree: the checker's binned-SAH builder
(oracle/oracle_kdbuild.c) and the reference's own compiled CPU query
(RKDTreeCPU::singleRayStacklessIntersect) running over it as the
reference's KDNodeCPU objects.  CPU only."""
import numpy as np
import pytest

import rayengine_b200.configs as C
from oracle import pyoracle as po


def _soup(n):
    cfg = C.SoupConfig(num_tris=n)
    verts = po.soup(cfg.seed, cfg.num_tris).reshape(-1, 3)
    faces = np.arange(verts.shape[0], dtype=np.uint32).reshape(-1, 3)
    return cfg, verts, faces


def test_sah_builder_invariants():
    cfg, verts, faces = _soup(4096)
    kd = po.kdb_build(verts, faces, max_depth=24, leaf_size=8)
    nodes = kd.nodes
    leaves = nodes[nodes["axis"] == 3]
    inner = nodes[nodes["axis"] != 3]
    assert len(leaves) == len(inner) + 1  # a full binary tree
    assert kd.depth() <= 24
    # leaves above the size limit only where no plane paid (few, small)
    assert (leaves["count"] <= 8).mean() > 0.95
    # every triangle is in some leaf; indices in range
    assert set(np.unique(kd.index)) == set(range(faces.shape[0]))
    assert leaves["first"].min() >= 0 and (leaves["first"] + leaves["count"]).max() <= len(kd.index)
    # inner splits lie inside the root box on their axis
    for ax in range(3):
        sel = inner[inner["axis"] == ax]["split"]
        assert np.all(sel >= kd.bmin[ax]) and np.all(sel <= kd.bmax[ax])


@pytest.mark.skipif(po.ref_lib() is None, reason="oracle/_ref (the reference's compiled host code) not built")
def test_reference_query_over_sah_tree_equals_its_one_leaf_query():
    """The reference's query keeps the smallest t over every leaf its box
    tests reach, so over a correct tree it returns the t of its own
    one-leaf (brute-force) tree for every ray."""
    cfg, verts, faces = _soup(8192)
    kd = po.kdb_build(verts, faces, max_depth=24, leaf_size=8)
    cam = cfg.camera()
    pix = np.random.default_rng(7).choice(cfg.width * cfg.height, 3000, replace=False)
    o, d = po.camera_rays(cam, cfg.width, cfg.height, pix)
    leaf = po.RefTree(verts, faces)
    sah = po.RefTree.from_kd(verts, faces, kd)
    ta, _, ha = leaf.trace(o, d)
    tb, _, hb = sah.trace(o, d)
    assert ha == hb and ha > 100
    assert np.array_equal(ta, tb)
    leaf.close()
    sah.close()

"""The CPU oracle against the golden fixtures produced by the reference's own
host code (tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

from oracle import pyoracle as po

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _load(name):
    return np.load(os.path.join(GOLDEN, name))


class _Cam:
    def __init__(self, d):
        self.campos = [float(x) for x in d["campos"]]
        self.view = [float(x) for x in d["view"]]
        self.camdown = [0.0, -1.0, 0.0]
        self.fov = [float(x) for x in d["fov"]]
        self.focial_distance = 1.0


def test_permutation_tables_match_reference():
    g = _load("perm.npz")
    for seed, table in zip(g["seeds"], g["tables"]):
        assert np.array_equal(po.perm(int(seed)), table), seed
        assert table[:256].tolist() != list(range(256))
        assert sorted(table[:256].tolist()) == list(range(256))
        assert np.array_equal(table[:256], table[256:])


@pytest.mark.parametrize("fixture", ["ref_soup.npz", "ref_grid.npz"])
def test_reference_tree_is_one_leaf(fixture):
    g = _load(fixture)
    assert g["nodes"].shape == (1, 128)
    assert int(g["levels"]) == 1 and int(g["leaves"]) == 1
    rn = po.ref_node_fields(g["nodes"][0])
    assert rn["is_leaf"] and rn["num_objs"] == g["faces"].shape[0]
    assert np.array_equal(g["index_list"], np.arange(g["faces"].shape[0]))
    v = g["verts"][g["faces"].reshape(-1)]
    assert np.array_equal(rn["min"], v.min(0)) and np.array_equal(rn["max"], v.max(0))


@pytest.mark.parametrize("fixture", ["ref_soup.npz", "ref_grid.npz"])
def test_bruteforce_matches_golden(fixture):
    g = _load(fixture)
    verts, faces = g["verts"], g["faces"]
    packed = np.zeros((faces.shape[0], 12), np.float32)
    v0 = verts[faces[:, 0]]
    packed[:, 0:3] = v0
    packed[:, 4:7] = verts[faces[:, 1]] - v0
    packed[:, 8:11] = verts[faces[:, 2]] - v0
    rn = po.ref_node_fields(g["nodes"][0])
    cam = _Cam(g)
    w, h = int(g["w"]), int(g["h"])
    hits = po.primary_bruteforce(packed, rn["min"], rn["max"], cam, w, h)
    assert np.array_equal(hits.view(np.int32).reshape(-1, 4), g["hits"])
    assert (g["hits"][:, 0] >= 0).sum() > 200


def test_reference_library_reproduces_golden_when_present():
    if po.ref_lib() is None:
        pytest.skip("reference sources not built here")
    g = _load("ref_soup.npz")
    nodes, idx, root, levels, leaves = po.ref_build(g["verts"], g["faces"])
    # compare the initialised fields: a leaf's axis/split_val and the bytes
    # after is_leaf are never written by the reference (KDThreeGPU.cpp:155-181)
    a, b = po.ref_node_fields(nodes[0]), po.ref_node_fields(g["nodes"][0])
    for k in ("min", "max", "is_leaf", "first", "num_objs", "ropes"):
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(idx, g["index_list"])
    gp = _load("perm.npz")
    for seed, table in zip(gp["seeds"], gp["tables"]):
        assert np.array_equal(po.ref_perm(int(seed)), table)


def test_noise_golden_and_identities():
    g = _load("noise.npz")
    P = po.perm(2016)
    for o in (1, 6, 8):
        assert np.array_equal(po.fbm_batch(P, g["pts"], o), g[f"fbm{o}"])
    # improved Perlin noise is zero on the integer lattice
    lattice = np.array([[i, j, k] for i in range(-3, 4) for j in range(-2, 3) for k in (0, 5, 255)],
                       np.float32)
    assert np.all(po.fbm_batch(P, lattice, 1) == 0.0)
    # bounded and continuous
    rng = np.random.default_rng(1)
    pts = rng.uniform(-50, 50, (20000, 3)).astype(np.float32)
    v = po.fbm_batch(P, pts, 1)
    assert np.abs(v).max() <= 2.0
    dv = po.fbm_batch(P, pts + np.float32(1e-3), 1) - v
    assert np.abs(dv).max() < 0.05


def test_sincos_accuracy():
    for u in np.linspace(0, 1, 1001, endpoint=False):
        s, c = po.sincos_2pi(float(np.float32(u)))
        a = 2 * np.pi * np.float64(np.float32(u))
        assert abs(s - np.sin(a)) < 2e-6 and abs(c - np.cos(a)) < 2e-6


def test_hash_is_well_spread():
    vals = np.array([po.hash_u32(7, p, j) for p in range(2000) for j in range(8)], np.uint64)
    hist = np.bincount((vals >> np.uint64(28)).astype(np.int64), minlength=16)
    assert hist.min() > 0.7 * hist.mean()

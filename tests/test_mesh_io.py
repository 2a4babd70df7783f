"""Mesh ingestion (host code, no GPU): PLY and OBJ readers.

Against the reference: where its sources are present, every PLY mesh it
ships is read through its own rply reader compiled from its sources
(oracle/_ref/libre_ply.so, restating RStaticMesh::LoadFromFile) and the
library's reader must give the same arrays (first-triangle mode, the
reference's behaviour).  Generated files cover the encodings and the OBJ
corner forms.
"""
import glob
import os
import struct

import numpy as np
import pytest

import rayengine_b200 as rb
from oracle import pyoracle as po
from oracle.refpath import reference_file

MESHES = reference_file("Sandbox", "Meshes") or ""


def _write_ply(path, verts, polys, fmt):
    hdr = [f"ply", f"format {fmt} 1.0", "comment generated", f"element vertex {len(verts)}",
           "property float x", "property float y", "property float z", "property uchar red",
           f"element face {len(polys)}", "property list uchar int vertex_indices",
           "property float quality", "element extra 1", "property double w", "end_header"]
    with open(path, "wb") as f:
        f.write(("\n".join(hdr) + "\n").encode())
        if fmt == "ascii":
            for v in verts:
                f.write(f"{float(v[0])!r} {float(v[1])!r} {float(v[2])!r} 7\n".encode())
            for p in polys:
                f.write((f"{len(p)} " + " ".join(str(i) for i in p) + " 0.5\n").encode())
            f.write(b"1.25\n")
        else:
            e = "<" if fmt == "binary_little_endian" else ">"
            for v in verts:
                f.write(struct.pack(e + "fffB", *[float(x) for x in v], 7))
            for p in polys:
                f.write(struct.pack(e + "B" + "i" * len(p) + "f", len(p), *p, 0.5))
            f.write(struct.pack(e + "d", 1.25))


@pytest.mark.parametrize("fmt", ["ascii", "binary_little_endian", "binary_big_endian"])
def test_ply_encodings(tmp_path, fmt):
    rng = np.random.default_rng(1)
    verts = rng.normal(size=(7, 3)).astype(np.float32)
    polys = [(0, 1, 2), (2, 3, 4, 5), (1, 5, 6, 0, 3)]
    path = str(tmp_path / "m.ply")
    _write_ply(path, verts, polys, fmt)
    v, f = rb.load_mesh(path)
    assert np.array_equal(v, verts)
    # fan triangulation of every polygon
    assert f.tolist() == [[0, 1, 2], [2, 3, 4], [2, 4, 5], [1, 5, 6], [1, 6, 0], [1, 0, 3]]
    v1, f1 = rb.load_mesh(path, first_triangle_only=True)
    assert f1.tolist() == [[0, 1, 2], [2, 3, 4], [1, 5, 6]]


def test_obj_corners_dedup_and_quads(tmp_path):
    text = """# test
v 0 0 0
v 1 0 0
v 1 1 0
v 0 1 0
v 0.5 0.5 1
vt 0 0
vt 1 0
vn 0 0 1
f 1 2 3
f 1/1 2/2 3/1 4/2
f 1//1 -4//1 5//1
f 2 3 4 5 1
"""
    path = tmp_path / "m.obj"
    path.write_text(text)
    v, f = rb.load_mesh(str(path))
    # one vertex per distinct (p, t, n) corner, in order of first use
    corners = [(1, 0, 0), (2, 0, 0), (3, 0, 0), (1, 1, 0), (2, 2, 0), (3, 1, 0), (4, 2, 0),
               (1, 0, 1), (2, 0, 1), (5, 0, 1), (4, 0, 0), (5, 0, 0)]
    P = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0.5, 0.5, 1]], np.float32)
    assert np.array_equal(v, P[[c[0] - 1 for c in corners]])
    assert f.tolist() == [[0, 1, 2],
                          [3, 4, 5], [6, 3, 5],          # quad (a b c d) -> (a b c), (d a c)
                          [7, 8, 9],
                          [1, 2, 10], [1, 10, 11], [1, 11, 0]]  # pentagon fanned


def test_malformed_files_are_errors(tmp_path):
    bad = tmp_path / "bad.ply"
    bad.write_bytes(b"ply\nformat ascii 1.0\nelement vertex 2\nproperty float x\n"
                    b"property float y\nproperty float z\nend_header\n1 2 3\n")
    with pytest.raises(rb.RayEngineError):
        rb.load_mesh(str(bad))
    idx = tmp_path / "idx.obj"
    idx.write_text("v 0 0 0\nf 1 2 3\n")
    with pytest.raises(rb.RayEngineError):
        rb.load_mesh(str(idx))
    with pytest.raises(rb.RayEngineError):
        rb.load_mesh(str(tmp_path / "missing.ply"))
    with pytest.raises(rb.RayEngineError):
        rb.load_mesh(str(tmp_path / "m.stl"))


needs_ref = pytest.mark.skipif(not os.path.isdir(MESHES) or po.ref_ply_lib() is None,
                               reason="reference meshes or its compiled rply reader absent")


@needs_ref
def test_reference_meshes_read_like_the_reference():
    paths = sorted(glob.glob(os.path.join(MESHES, "*.ply")))
    assert len(paths) >= 10
    for p in paths:
        ok, rv, rf = po.ref_ply_load(p)
        if not ok:  # malformed in the reference's reader too
            with pytest.raises(rb.RayEngineError):
                rb.load_mesh(p, first_triangle_only=True)
            continue
        v, f = rb.load_mesh(p, first_triangle_only=True)
        assert np.array_equal(v, rv), p
        assert np.array_equal(f, rf), p


@needs_ref
def test_bunny_tree_traversal_equals_brute_force():
    # real geometry: the Stanford bunny shipped with the reference (69,451
    # faces), SAH tree built on the host, rope traversal vs brute force
    v, f = rb.load_mesh(os.path.join(MESHES, "bun_zipper.ply"))
    assert v.shape == (35947, 3) and f.shape == (69451, 3)
    # scaled to unit size: the triangle tests' absolute epsilons (|a| < 1e-5)
    # reject the raw model's millimetre triangles
    v = (v * np.float32(10.0)).astype(np.float32)
    packed = rb.pack_triangles(v, f)
    with rb.KDScene.build_host(packed) as sc:
        st = sc.stats()
        nodes, leaves, tris = sc.export()
    kd = po.KdTree(nodes, leaves, tris, st["bmin"], st["bmax"])
    w, h = 96, 96
    c = (v.min(0) + v.max(0)) / 2
    cam = rb.build_camera((float(c[0]), float(c[1]), float(c[2]) + 2.5),
                          (float(c[0]), float(c[1]), float(c[2])), (45.0, 45.0))
    got = po.primary_kd(kd, cam, w, h)
    want = po.primary_bruteforce(packed, st["bmin"], st["bmax"], cam, w, h)
    assert (want["id"] >= 0).mean() > 0.3
    assert np.array_equal(got["id"], want["id"])
    assert np.array_equal(got["t"].view(np.uint32), want["t"].view(np.uint32))

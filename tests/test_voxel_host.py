"""Voxel SDF host parts (no GPU): the .rsdf file format and the oracle's
three samplers on fields whose samples are known exactly."""
import ctypes
import struct

import numpy as np
import pytest

from oracle import pyoracle as po
from rayengine_b200 import _lib
from rayengine_b200._lib import call, RayEngineError


def _desc(dim, spacing, origin=(0, 0, 0)):
    d = _lib.re_voxel_grid()
    d.dim[:] = list(dim)
    d.spacing[:] = [float(x) for x in spacing]
    d.origin[:] = [float(x) for x in origin]
    return d


def test_rsdf_layout_and_round_trip(tmp_path):
    dim, sp = (3, 4, 5), (0.5, 0.25, 2.0)
    n = 3 * 4 * 5
    grid = np.arange(2 * n, dtype=np.float32) * 0.5
    path = str(tmp_path / "g.rsdf")
    call("re_voxel_save", path.encode(), ctypes.byref(_desc(dim, sp)), grid.ctypes.data)
    raw = open(path, "rb").read()
    assert struct.unpack("<3i3f", raw[:24]) == (3, 4, 5, 0.5, 0.25, 2.0)
    assert np.array_equal(np.frombuffer(raw[24:], np.float32), grid)  # x fastest pairs
    d = _lib.re_voxel_grid()
    call("re_voxel_load", path.encode(), ctypes.byref(d), None, 0)
    assert list(d.dim) == list(dim) and list(d.spacing) == list(sp)
    back = np.zeros(2 * n, np.float32)
    call("re_voxel_load", path.encode(), ctypes.byref(d), back.ctypes.data, n)
    assert np.array_equal(back, grid)
    with pytest.raises(RayEngineError):  # buffer too small
        call("re_voxel_load", path.encode(), ctypes.byref(d), back.ctypes.data, n - 1)
    (tmp_path / "t.rsdf").write_bytes(raw[:-8])
    with pytest.raises(RayEngineError):  # truncated
        call("re_voxel_load", str(tmp_path / "t.rsdf").encode(), ctypes.byref(d),
             back.ctypes.data, n)


def test_oracle_samplers_on_exact_fields():
    dim, sp, org = (6, 5, 7), (0.5, 0.5, 0.5), (-1.0, 0.0, 2.0)
    i, j, k = np.meshgrid(np.arange(6), np.arange(5), np.arange(7), indexing="ij")
    # linear field a + b.x on the grid points, stored x fastest
    lin = (0.25 + 0.5 * i - 0.25 * j + 0.125 * k).astype(np.float32)
    grid = np.zeros(2 * lin.size, np.float32)
    grid[0::2] = lin.transpose(2, 1, 0).reshape(-1)
    rng = np.random.default_rng(3)
    # points well inside (away from the clamped edges)
    u = rng.uniform(1.2, 3.8, (500, 3)).astype(np.float32)
    pts = (np.array(org, np.float32) + u * np.float32(0.5)).astype(np.float32)
    uu = (pts - np.array(org, np.float32)) / np.float32(0.5)
    want = 0.25 + 0.5 * uu[:, 0] - 0.25 * uu[:, 1] + 0.125 * uu[:, 2]
    mid = po.voxel_sample(grid, dim, sp, org, 1, pts)
    assert np.abs(mid - want).max() < 1e-5  # trilinear reproduces linear fields
    low = po.voxel_sample(grid, dim, sp, org, 0, pts)
    fl = np.floor(uu).astype(int)
    assert np.array_equal(low, lin[fl[:, 0], fl[:, 1], fl[:, 2]])
    # the cubic B-spline reproduces linear fields too, about voxel centres
    # shifted by half a voxel (the reference's texture-space convention),
    # where none of its 4 x 4 x 4 taps is clamped
    u = rng.uniform(1.5, 3.49, (500, 3)).astype(np.float32)
    pts = (np.array(org, np.float32) + u * np.float32(0.5)).astype(np.float32)
    uu = (pts - np.array(org, np.float32)) / np.float32(0.5)
    high = po.voxel_sample(grid, dim, sp, org, 2, pts)
    want_h = 0.25 + 0.5 * (uu[:, 0] - 0.5) - 0.25 * (uu[:, 1] - 0.5) + 0.125 * (uu[:, 2] - 0.5)
    assert np.abs(high - want_h).max() < 1e-5
    # clamping: far outside reads the edge voxel
    out = po.voxel_sample(grid, dim, sp, org, 0, np.array([[100.0, -100.0, 100.0]], np.float32))
    assert out[0] == lin[5, 0, 6]

"""The C-ABI library loads, exports every declared entry point and validates
arguments without touching a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

import rayengine_b200 as rb
from rayengine_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "rayengine_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"RE_API\s+[\w\s\*]+?\b(re_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "re_trace_primary" in syms and "re_sdf_trace" in syms and len(syms) >= 20


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    # and the Python binding declares a signature for each of them
    assert set(declared_symbols()) <= set(_lib.EXPORTED), set(declared_symbols()) - set(_lib.EXPORTED)


def test_abi_version_and_status_strings():
    assert _lib.lib.re_abi_version() == _lib.ABI_VERSION == 2
    assert _lib.lib.re_status_string(0) == b"ok"
    assert _lib.lib.re_status_string(4) == b"size limit exceeded"


def test_argument_errors_are_reported_not_fatal():
    with pytest.raises(rb.RayEngineError) as e:
        _lib.call("re_scene_create", None, 0, None, 0, None, ctypes.byref(ctypes.c_void_p()))
    assert e.value.status == 1 and "re_scene_create" in str(e.value)
    with pytest.raises(rb.RayEngineError) as e:
        _lib.call("re_gen_grid_faces", 100000, ctypes.c_void_p(1))
    assert e.value.status == 4
    with pytest.raises(rb.RayEngineError):
        _lib.call("re_noise_fbm", None, None, 0, None, None)
    p = rb.sdf_params(max_steps=0)
    with pytest.raises(rb.RayEngineError) as e:
        _lib.call("re_sdf_trace", ctypes.byref(p), ctypes.byref(rb.build_camera((0, 0, 1), (0, 0, 0))),
                  4, 4, ctypes.c_void_p(16), None)
    assert e.value.status in (1, 4)


def test_bad_face_index_rejected():
    verts = np.zeros((3, 3), np.float32)
    faces = np.array([[0, 1, 5]], np.uint32)
    with pytest.raises(rb.RayEngineError) as e:
        rb.KDScene.from_mesh(verts, faces)
    assert e.value.status == 1


def test_host_only_scene_refuses_to_trace():
    packed = rb.configs.SoupConfig(num_tris=64).packed()
    sc = rb.KDScene.build_host(packed)
    with pytest.raises(rb.RayEngineError) as e:
        _lib.call("re_trace_primary", sc.handle, ctypes.byref(rb.build_camera((0, 0, 3), (0, 0, 0))),
                  8, 8, 0, ctypes.c_void_p(16), None)
    assert e.value.status == 5
    sc.close()


def test_tuning_validation():
    """ray_lanes: 1 by default, 0 reads as 1, powers of two up to 8, or 32
    (the warp-cooperative walk)."""
    packed = rb.configs.SoupConfig(num_tris=64).packed()
    with rb.KDScene.build_host(packed) as sc:
        t = sc.tuning()
        assert t["ray_lanes"] == 1 and t["ray_refill_min"] == 32
        for lanes in (2, 4, 8, 32, 1):
            sc.set_tuning(t["stage_nodes"], 0, 8, 32, lanes)
            assert sc.tuning()["ray_lanes"] == lanes
        sc.set_tuning(t["stage_nodes"], 0, 8, 32, 0)
        assert sc.tuning()["ray_lanes"] == 1
        for bad in (3, 6, 16, 64):
            with pytest.raises(rb.RayEngineError) as e:
                sc.set_tuning(t["stage_nodes"], 0, 8, 32, bad)
            assert e.value.status == 1
        assert sc.tuning()["ray_lanes"] == 1


def test_plain_c_caller(tmp_path):
    """The header compiles as C11 and a C program drives the host-only
    entry points through the shared library (the ABI a C or FFI caller
    binds)."""
    import shutil
    import subprocess

    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    lib_dir = os.path.join(root, "rayengine_b200")
    exe = str(tmp_path / "host_only")
    subprocess.run([gcc, "-std=c11", "-Wall", "-Werror", "-O1",
                    "-I", os.path.join(root, "include"),
                    os.path.join(root, "tests", "c_abi", "host_only.c"),
                    "-L", lib_dir, "-lrayengine_b200", "-Wl,-rpath," + lib_dir, "-o", exe],
                   check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr


def test_frame_config_matches_library_defaults():
    """SdfFrameConfig builds re_sdf_shade_params in Python (the benchmark's
    reference arm must not load the library); it equals the library's own
    defaults field for field."""
    a = rb.configs.SdfFrameConfig().shade()
    b = _lib.re_sdf_shade_params()
    _lib.lib.re_sdf_shade_params_default(ctypes.byref(b))
    assert bytes(a) == bytes(b)


def test_measurement_probes_reject_bad_sizes():
    """The roofline probes check their arguments before touching a device."""
    v = ctypes.c_float()
    for nbytes, passes in ((1 << 10, 10), (128 << 20, 10), (32 << 20, 0), (32 << 20, 5000)):
        assert _lib.lib.re_measure_l2_read(nbytes, passes, ctypes.byref(v), None) == 1
    for iters in (0, 1000, (1 << 20) + 1):
        assert _lib.lib.re_measure_fp32_fma(iters, ctypes.byref(v), None) == 1
    assert _lib.lib.re_measure_fp32_fma(1 << 16, None, None) == 1

"""A compiled C++ caller (tests/c_abi/gpu_caller.cpp) drives the library on
the GPU through include/rayengine_b200.h alone: scene upload, primary rays
into its own cudaMalloc'd buffer, and the reference's render call
cuda_render_frame after re_sdf_frame_bind.  Its outputs equal the Python
path's bit for bit."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest
import torch

import rayengine_b200 as rb

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def test_cpp_caller_matches_python_path(cuda, tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no C++ compiler")
    lib_dir = os.path.join(ROOT, "rayengine_b200")
    exe = str(tmp_path / "gpu_caller")
    subprocess.run([gxx, "-std=c++17", "-O1", "-Wall", "-Werror",
                    "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"),
                    os.path.join(ROOT, "tests", "c_abi", "gpu_caller.cpp"),
                    "-L", lib_dir, "-lrayengine_b200", "-Wl,-rpath," + lib_dir,
                    "-L", os.path.join(CUDA, "lib64"), "-lcudart", "-o", exe], check=True)

    soup = rb.configs.SoupConfig(num_tris=4096, width=96, height=80)
    packed = np.ascontiguousarray(soup.packed(), np.float32)
    cam = soup.camera()
    frame = rb.configs.SdfFrameConfig()
    tcfg = frame.terrain
    fw, fh = 64, 36
    fy = rb.vertical_fov(tcfg.fov_x, fw, fh)
    tcam = rb.build_camera(tcfg.campos, tcfg.lookat, (tcfg.fov_x, fy))
    field, shade = tcfg.params(), frame.shade()
    inp = tmp_path / "in.bin"
    with open(inp, "wb") as f:
        f.write(np.uint32(packed.shape[0]).tobytes())
        f.write(packed.tobytes())
        f.write(bytes(cam))
        f.write(np.array([soup.width, soup.height], np.uint32).tobytes())
        f.write(bytes(field))
        f.write(bytes(shade))
        f.write(bytes(tcam))
        f.write(np.array([fw, fh], np.uint32).tobytes())
    outp = tmp_path / "out.bin"
    run = subprocess.run([exe, str(inp), str(outp)], capture_output=True, text=True, timeout=300)
    assert run.returncode == 0 and run.stdout.strip() == "ok", run.stdout + run.stderr
    raw = np.fromfile(outp, np.uint8)
    nh = soup.width * soup.height * 16
    hits = raw[:nh].view(np.int32).reshape(-1, 4)
    rgba = raw[nh:].view(np.uint32)
    assert rgba.size == fw * fh

    with rb.KDScene.from_packed(packed) as sc:
        want = sc.trace_primary(cam, soup.width, soup.height).cpu().numpy()
    assert np.array_equal(hits, want)
    assert (hits[:, 0] >= 0).sum() > 100
    want_rgba, _ = rb.render_sdf_frame(field, shade, tcam, fw, fh)
    assert np.array_equal(rgba, want_rgba.cpu().numpy().view(np.uint32).reshape(-1))

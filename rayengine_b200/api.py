"""Host-side mirror of RayEngine's ray-query interface over the C ABI.

Names follow the reference (hadalhw17/RayEngine, "RE/" = RayEngine/src/):

* ``RCamera`` / ``build_camera``  -- RE/Primitives/Camera.h:7-16,
  RE/Objects/MovableCamera.cpp:101-118 (camdown = (0,-1,0), fov in degrees).
* ``RPerlinNoise``                -- RE/World/PerlinNoise.h:16-52.
* ``KDScene``                     -- RKDTreeCPU + RKDThreeGPU + RTScene +
  copy_memory (RE/Primitives/KDTree.cpp:117-173, RE/Primitives/KDThreeGPU.cpp:9-54,
  RE/World/RTScene.cpp:40-62,179-285, RE/cuda-src/cuda_memory_functions.cuh:58-211),
  with ``trace_primary`` standing for the trace_primary_rays launch
  (RE/cuda-src/renderer.cu:390-410,705-709).
* ``generate_noise`` / ``heightfield`` -- the generate_noise bake
  (RE/cuda-src/renderer.cu:106-126,813-836).
* ``sphere_trace``                -- render_sphere_trace's terrain march
  (RE/cuda-src/renderer.cu:143-235, RE/cuda-src/sphere_tracing.cuh:183-216).

Device buffers are torch CUDA tensors (torch is only the allocator and the
stream provider); every computation runs in librayengine_b200.so.  Errors
raise RayEngineError carrying the library's message.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import RayEngineError, call, lib  # noqa: F401

TRACE_TWO_SIDED = 0
TRACE_ONE_SIDED = 1
TRACE_ANY_HIT = 2

HIT_DTYPE = np.dtype([("id", "<i4"), ("t", "<f4"), ("u", "<f4"), ("v", "<f4")])
SDF_HIT_DTYPE = np.dtype(
    [("pos", "<f4", 3), ("normal", "<f4", 3), ("steps", "<u4"), ("status", "<u4")]
)


def _stream_ptr(stream) -> Optional[int]:
    if stream is None:
        import torch

        return torch.cuda.current_stream().cuda_stream
    return getattr(stream, "cuda_stream", stream)


def _dptr(t) -> int:
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return t.data_ptr()


# ---------------------------------------------------------------- camera
RCamera = _lib.re_camera


def build_camera(campos: Sequence[float], lookat: Sequence[float],
                 fov: Sequence[float] = (60.0, 60.0), focal: float = 1.0) -> RCamera:
    """RMovableCamera::build_camera with the view pointing at ``lookat``."""
    c = RCamera()
    v = np.asarray(lookat, np.float64) - np.asarray(campos, np.float64)
    v = v / np.linalg.norm(v)
    c.campos[:] = [float(x) for x in campos]
    c.view[:] = [float(x) for x in v]
    c.camdir[:] = [float(x) for x in v]
    c.lookat[:] = [float(x) for x in lookat]
    c.camdown[:] = [0.0, -1.0, 0.0]
    c.fov[:] = [float(fov[0]), float(fov[1])]
    c.focial_distance = float(focal)
    c.apertude_radius = 0.0
    return c


def vertical_fov(fov_x_deg: float, width: int, height: int) -> float:
    """Full vertical angle matching fov_x on a width x height image (the
    intent of RMovableCamera::set_fovx, MovableCamera.cpp:38-42)."""
    return math.degrees(2.0 * math.atan(math.tan(math.radians(fov_x_deg) * 0.5) * height / width))


# ----------------------------------------------------------------- noise
class RPerlinNoise:
    """RPerlinNoise(seed): the 512-entry permutation table."""

    def __init__(self, seed: int = 2016):
        self.seed = int(seed)
        tab = np.zeros(512, np.uint32)
        call("re_perlin_permutation", self.seed, tab.ctypes.data)
        self.permutationTable = tab


def fbm_params(seed=2016, octaves=6, lacunarity=2.0, gain=0.5, scale=1.0, amplitude=1.0):
    p = _lib.re_fbm_params()
    p.seed, p.octaves, p.lacunarity, p.gain = seed, octaves, lacunarity, gain
    p.scale, p.amplitude = scale, amplitude
    return p


def generate_noise(params, pts, out=None, stream=None):
    """Batch fBm: out[i] = amplitude * fbm(scale * pts[i]); pts (n,3) float32 CUDA."""
    import torch

    n = pts.shape[0]
    if out is None:
        out = torch.empty(n, dtype=torch.float32, device=pts.device)
    call("re_noise_fbm", ctypes.byref(params), _dptr(pts), n, _dptr(out), _stream_ptr(stream))
    return out


def heightfield(params, cells: int, lo: float, hi: float, out=None, stream=None):
    """(cells+1)^2 x 3 vertex grid with y = amplitude * fbm(x, 0, z)."""
    import torch

    nv = (cells + 1) * (cells + 1)
    if out is None:
        out = torch.empty((nv, 3), dtype=torch.float32, device="cuda")
    call("re_heightfield", ctypes.byref(params), cells, lo, hi, _dptr(out), _stream_ptr(stream))
    return out


def grid_faces(cells: int) -> np.ndarray:
    f = np.empty((2 * cells * cells, 3), np.uint32)
    call("re_gen_grid_faces", cells, f.ctypes.data)
    return f


def triangle_soup(n: int, seed: int = 0) -> np.ndarray:
    """(n, 3, 3) float32 vertices of the seeded soup."""
    v = np.empty((n, 3, 3), np.float32)
    call("re_gen_soup", seed, n, v.ctypes.data)
    return v


def pack_triangles(verts: np.ndarray, faces: np.ndarray) -> np.ndarray:
    """RTScene::init_triangles packing: per face {v0,0, v1-v0,0, v2-v0,0}."""
    v0 = verts[faces[:, 0]]
    p = np.zeros((faces.shape[0], 12), np.float32)
    p[:, 0:3] = v0
    p[:, 4:7] = verts[faces[:, 1]] - v0
    p[:, 8:11] = verts[faces[:, 2]] - v0
    return p


# ------------------------------------------------------------- kd scene
def kd_params(**kw):
    p = _lib.re_kd_params()
    lib.re_kd_params_default(ctypes.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class KDScene:
    """A rope kd-tree scene resident on the current CUDA device."""

    def __init__(self, handle: int):
        self._h = ctypes.c_void_p(handle)

    @classmethod
    def from_mesh(cls, verts: np.ndarray, faces: np.ndarray, params=None) -> "KDScene":
        verts = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
        faces = np.ascontiguousarray(faces, np.uint32).reshape(-1, 3)
        h = ctypes.c_void_p()
        call("re_scene_create", verts.ctypes.data, verts.shape[0], faces.ctypes.data,
             faces.shape[0], ctypes.byref(params) if params is not None else None, ctypes.byref(h))
        return cls(h.value)

    @classmethod
    def from_packed(cls, tris: np.ndarray, params=None) -> "KDScene":
        tris = np.ascontiguousarray(tris, np.float32).reshape(-1, 12)
        h = ctypes.c_void_p()
        call("re_scene_create_packed", tris.ctypes.data, tris.shape[0],
             ctypes.byref(params) if params is not None else None, ctypes.byref(h))
        return cls(h.value)

    @classmethod
    def build_host(cls, tris: np.ndarray, params=None) -> "KDScene":
        """Build the tree on the host only (no device); stats/export work."""
        tris = np.ascontiguousarray(tris, np.float32).reshape(-1, 12)
        h = ctypes.c_void_p()
        call("re_scene_build_host", tris.ctypes.data, tris.shape[0],
             ctypes.byref(params) if params is not None else None, ctypes.byref(h))
        return cls(h.value)

    def close(self) -> None:
        if self._h:
            lib.re_scene_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def stats(self) -> dict:
        s = _lib.re_scene_stats()
        call("re_scene_stats_get", self._h, ctypes.byref(s))
        return {
            "num_tris": s.num_tris, "num_nodes": s.num_nodes, "num_leaves": s.num_leaves,
            "num_refs": s.num_refs, "max_depth": s.max_depth, "max_leaf_size": s.max_leaf_size,
            "bfs_nodes": s.bfs_nodes, "bmin": list(s.bmin), "bmax": list(s.bmax),
            "build_seconds": s.build_seconds, "device_bytes": s.device_bytes,
        }

    def export(self):
        """(nodes uint32 (N,2), leaves uint32 (L,16), tris float32 (R,12))."""
        st = self.stats()
        nodes = np.empty((st["num_nodes"], 2), np.uint32)
        leaves = np.empty((st["num_leaves"], 16), np.uint32)
        tris = np.empty((st["num_refs"], 12), np.float32)
        call("re_scene_export", self._h, nodes.ctypes.data, leaves.ctypes.data, tris.ctypes.data)
        return nodes, leaves, tris

    def export_entry(self):
        """The entry table: uint32 (3, 2, res, res) start nodes per face
        (axis k, side 0 = -k / 1 = +k) and cell (i along the face's lower
        other axis, j along the higher)."""
        res = ctypes.c_uint32()
        call("re_scene_export_entry", self._h, None, ctypes.byref(res))
        r = res.value
        out = np.empty((3, 2, r, r), np.uint32)
        call("re_scene_export_entry", self._h, out.ctypes.data, ctypes.byref(res))
        return out

    def trace_primary(self, cam: RCamera, w: int, h: int, flags: int = TRACE_TWO_SIDED,
                      out=None, stream=None):
        """Closest hits for every pixel -> int32 CUDA tensor (h*w, 4) = re_hit."""
        import torch

        if out is None:
            out = torch.empty((h * w, 4), dtype=torch.int32, device="cuda")
        call("re_trace_primary", self._h, ctypes.byref(cam), w, h, flags, _dptr(out),
             _stream_ptr(stream))
        return out

    def count_primary(self, cam: RCamera, w: int, h: int, flags: int = TRACE_TWO_SIDED,
                      out=None, stream=None):
        """Per-pixel (inner steps, leaf visits, triangle tests, status)."""
        import torch

        if out is None:
            out = torch.empty((h * w, 4), dtype=torch.int32, device="cuda")
        call("re_count_primary", self._h, ctypes.byref(cam), w, h, flags, _dptr(out),
             _stream_ptr(stream))
        return out

    def truncated(self, stream=None) -> int:
        """Rays of the last trace call on this scene that stopped at the
        leaf-visit cap (re_scene_truncated); synchronises the stream."""
        import torch

        t = torch.zeros(1, dtype=torch.int32, device="cuda")
        call("re_scene_truncated", self._h, _dptr(t), _stream_ptr(stream))
        return int(t.item())

    def trace_rays(self, rays, flags: int = TRACE_TWO_SIDED, out=None, stream=None):
        """rays: float32 CUDA tensor (n, 8) = re_ray {o, tmax, d, tag}."""
        import torch

        n = rays.shape[0]
        if out is None:
            out = torch.empty((n, 4), dtype=torch.int32, device="cuda")
        call("re_trace_rays", self._h, _dptr(rays), n, flags, _dptr(out), _stream_ptr(stream))
        return out

    def render_ao(self, cam: RCamera, w: int, h: int, light_dir=(0.3, 1.0, 0.2),
                  ao_length: float = 1.0, bias: float = 1e-4, seed: int = 0,
                  primary=None, mask=None, nsec=None, stream=None):
        """Primary + shadow + 4 AO rays -> (hits (h*w,4) int32, mask (h*w,) int32, n_secondary)."""
        import torch

        if primary is None:
            primary = torch.empty((h * w, 4), dtype=torch.int32, device="cuda")
        if mask is None:
            mask = torch.empty(h * w, dtype=torch.int32, device="cuda")
        if nsec is None:
            nsec = torch.zeros(1, dtype=torch.int32, device="cuda")
        p = ao_params(light_dir, ao_length, bias, seed)
        call("re_render_ao", self._h, ctypes.byref(cam), w, h, ctypes.byref(p), _dptr(primary),
             _dptr(mask), _dptr(nsec), _stream_ptr(stream))
        return primary, mask, nsec

    def render_ao_primary(self, cam: RCamera, w: int, h: int, params, primary, mask,
                          stream=None):
        call("re_render_ao_primary", self._h, ctypes.byref(cam), w, h, ctypes.byref(params),
             _dptr(primary), _dptr(mask), _stream_ptr(stream))

    def render_ao_secondary(self, mask, nsec=None, stream=None):
        call("re_render_ao_secondary", self._h, _dptr(mask),
             _dptr(nsec) if nsec is not None else None, _stream_ptr(stream))

    def tuning(self) -> dict:
        t = _lib.re_tuning()
        call("re_scene_get_tuning", self._h, ctypes.byref(t))
        return {"stage_nodes": t.stage_nodes, "queue_kind_major": t.queue_kind_major,
                "refill_min": t.refill_min, "ray_refill_min": t.ray_refill_min,
                "ray_lanes": t.ray_lanes}

    def set_tuning(self, stage_nodes: int, queue_kind_major: int, refill_min: int,
                   ray_refill_min: int | None = None, ray_lanes: int | None = None) -> None:
        cur = self.tuning()
        if ray_refill_min is None:
            ray_refill_min = cur["ray_refill_min"]
        if ray_lanes is None:
            ray_lanes = cur["ray_lanes"]
        t = _lib.re_tuning(stage_nodes, queue_kind_major, refill_min, ray_refill_min, ray_lanes)
        call("re_scene_set_tuning", self._h, ctypes.byref(t))

    def autotune_ao(self, cam: RCamera, w: int, h: int, params, stream=None) -> dict:
        """Pick staging depth, queue layout and refill threshold by timing the frame."""
        t = _lib.re_tuning()
        ms = ctypes.c_float()
        call("re_autotune_ao", self._h, ctypes.byref(cam), w, h, ctypes.byref(params),
             ctypes.byref(t), ctypes.byref(ms), _stream_ptr(stream))
        return {"stage_nodes": t.stage_nodes, "queue_kind_major": t.queue_kind_major,
                "refill_min": t.refill_min, "frame_ms": round(ms.value, 4)}

    def autotune_primary(self, cam: RCamera, w: int, h: int, flags: int = 0, stream=None) -> dict:
        """Pick staging depth, ray refill threshold and lanes per ray by timing the
        primary pass."""
        t = _lib.re_tuning()
        ms = ctypes.c_float()
        call("re_autotune_primary", self._h, ctypes.byref(cam), w, h, flags, ctypes.byref(t),
             ctypes.byref(ms), _stream_ptr(stream))
        return {"stage_nodes": t.stage_nodes, "ray_refill_min": t.ray_refill_min,
                "ray_lanes": t.ray_lanes, "frame_ms": round(ms.value, 4)}

    def render_frame(self, cam: RCamera, w: int, h: int, lights, shade, out=None, stream=None):
        """Shaded RGBA8 frame -> uint32-valued int32 CUDA tensor (h*w,).

        lights: [(pos xyz, intensity)]; shade: shade_params(...)."""
        import torch

        if out is None:
            out = torch.empty(h * w, dtype=torch.int32, device="cuda")
        arr = _light_array(lights)
        call("re_render_frame", self._h, ctypes.byref(cam), arr, len(lights),
             ctypes.byref(shade), w, h, _dptr(out), _stream_ptr(stream))
        return out

    def bind_frame(self, cam: RCamera, lights, shade, animate_light=False):
        """State for the reference-style cuda_render_frame(output, w, h)."""
        arr = _light_array(lights)
        call("re_frame_bind", self._h, ctypes.byref(cam), arr, len(lights), ctypes.byref(shade),
             1 if animate_light else 0)

    def render_ao_counts(self, cam: RCamera, w: int, h: int, params, stream=None) -> dict:
        """Traversal work of the AO frame (sums over all rays of each pass)."""
        import torch

        t = torch.zeros(8, dtype=torch.int64, device="cuda")
        call("re_render_ao_counts", self._h, ctypes.byref(cam), w, h, ctypes.byref(params),
             _dptr(t), _stream_ptr(stream))
        v = [int(x) for x in t.cpu().tolist()]
        keys = ("inner", "leaf", "tests", "rays")
        return {"primary": dict(zip(keys, v[:4])), "secondary": dict(zip(keys, v[4:]))}


def unit(v) -> list:
    """Unit vector as float32 values (light directions)."""
    v = np.asarray(v, np.float64)
    return [float(x) for x in (v / np.linalg.norm(v)).astype(np.float32)]


def ao_params(light_dir, ao_length=1.0, bias=1e-4, seed=0):
    p = _lib.re_ao_params()
    p.light_dir[:] = unit(light_dir)
    p.ao_length, p.bias, p.seed = ao_length, bias, seed
    return p


# ----------------------------------------------------------- SDF tracing
def sdf_params(seed=2016, octaves=8, scale=0.25, amplitude=3.0, step_factor=0.6, eps=1e-4,
               tmax=200.0, max_steps=512):
    p = _lib.re_sdf_params()
    p.seed, p.octaves, p.scale, p.amplitude = seed, octaves, scale, amplitude
    p.step_factor, p.eps, p.tmax, p.max_steps = step_factor, eps, tmax, max_steps
    return p


def sphere_trace(params, cam: RCamera, w: int, h: int, out=None, stream=None):
    """Exact-SDF march per pixel -> int32 CUDA tensor (h*w, 8) = re_sdf_hit."""
    import torch

    if out is None:
        out = torch.empty((h * w, 8), dtype=torch.int32, device="cuda")
    call("re_sdf_trace", ctypes.byref(params), ctypes.byref(cam), w, h, _dptr(out),
         _stream_ptr(stream))
    return out


# ------------------------------------------------- shaded SDF terrain frame
SDF_SHADE, SDF_FOG, SDF_GAMMA, SDF_VIGNETTING = (_lib.SDF_SHADE, _lib.SDF_FOG, _lib.SDF_GAMMA,
                                                 _lib.SDF_VIGNETTING)


def sdf_shade_params(**kw):
    """re_sdf_shade_params: the library's defaults, overridden by keywords
    (light_pos=(x, y), light_intensity, soft_shadow_k, shadow_tmin,
    shadow_tmax, shadow_max_steps, sun_dir, max_y, fog_density,
    vignetting_k, flags)."""
    p = _lib.re_sdf_shade_params()
    lib.re_sdf_shade_params_default(ctypes.byref(p))
    for k, v in kw.items():
        if k in ("light_pos", "sun_dir"):
            getattr(p, k)[:] = [float(x) for x in v]
        else:
            setattr(p, k, v)
    return p


def render_sdf_frame(field, shade, cam: RCamera, w: int, h: int, hits=None, out=None,
                     stream=None):
    """The shaded terrain frame (render_sphere_trace): trace into `hits`
    ((h*w, 8) int32 = re_sdf_hit) and shade into `out` ((h*w,) int32 RGBA8).
    Returns (out, hits)."""
    import torch

    if hits is None:
        hits = torch.empty((h * w, 8), dtype=torch.int32, device="cuda")
    if out is None:
        out = torch.empty(h * w, dtype=torch.int32, device="cuda")
    call("re_render_sdf_frame", ctypes.byref(field), ctypes.byref(shade), ctypes.byref(cam), w, h,
         _dptr(hits), _dptr(out), _stream_ptr(stream))
    return out, hits


def shade_sdf(field, shade, cam: RCamera, w: int, h: int, hits, out=None, evals=None,
              stream=None):
    """The shading pass alone over a hit record -> RGBA8 (h*w,) int32."""
    import torch

    if out is None:
        out = torch.empty(h * w, dtype=torch.int32, device="cuda")
    call("re_sdf_shade", ctypes.byref(field), ctypes.byref(shade), ctypes.byref(cam), w, h,
         _dptr(hits), _dptr(out), _dptr(evals) if evals is not None else None,
         _stream_ptr(stream))
    return out


def bind_sdf_frame(field, shade, cam: RCamera, animate_sun=False):
    """State for cuda_render_frame() in the reference's shipped SDF mode."""
    call("re_sdf_frame_bind", ctypes.byref(field), ctypes.byref(shade), ctypes.byref(cam),
         1 if animate_sun else 0)


def fmath(fn: int, x, y=None, out=None, stream=None):
    """The frame's elementary functions on CUDA float tensors (0: e^x, 1: ln x, 2: x^y)."""
    import torch

    if out is None:
        out = torch.empty_like(x)
    call("re_fmath", fn, _dptr(x), _dptr(y) if y is not None else None, x.numel(), _dptr(out),
         _stream_ptr(stream))
    return out


# ------------------------------------------------------ neural SDF surrogate
def nsdf_trace_params(lipschitz=1.0, safety=0.9, switch_dist=0.05, min_step=1e-3,
                      max_network_steps=256, max_exact_steps=0, root_steps=4, relax=1.0,
                      exact_only=False, cone_tile=0, cone_coarse=0, normal_taps=6, cone_lanes=1,
                      root_tol=0.0):
    """Neural march / exact phase settings (re_nsdf_trace_params).

    exact_only skips the network: every ray runs the exact phase from the
    camera (the same method without the network).  cone_tile > 0: the
    network marches one cone per cone_tile x cone_tile pixel tile (after a
    first level over cone_coarse tiles when that is set) and every pixel's
    exact phase starts where its tile stopped; cone_lanes lanes evaluate
    successive guessed steps of a cone in one pass.  normal_taps: 6 central
    differences, 4 the tetrahedral normal, 1 the exact field's analytic
    gradient (a second pass over the hits).  root_tol > 0 ends the root
    search once its secant point moves less than that."""
    p = _lib.re_nsdf_trace_params()
    p.lipschitz, p.safety, p.switch_dist, p.min_step = lipschitz, safety, switch_dist, min_step
    p.max_network_steps, p.max_exact_steps = max_network_steps, max_exact_steps
    p.root_steps, p.relax = root_steps, relax
    p.flags = _lib.NSDF_EXACT_ONLY if exact_only else 0
    p.cone_tile, p.cone_coarse, p.normal_taps = cone_tile, cone_coarse, normal_taps
    p.cone_lanes, p.root_tol = cone_lanes, root_tol
    return p


class NeuralSDF:
    """Fourier-feature MLP surrogate of the terrain density (trained and run
    on the device; tensor-core inference)."""

    def __init__(self, box_min, box_max, f0: float = 0.5, seed: int = 1):
        cfg = _lib.re_nsdf_config()
        cfg.box_min[:] = [float(x) for x in box_min]
        cfg.box_max[:] = [float(x) for x in box_max]
        cfg.f0, cfg.seed = f0, seed
        self.box_min, self.box_max, self.f0 = list(cfg.box_min), list(cfg.box_max), f0
        h = ctypes.c_void_p()
        call("re_nsdf_create", ctypes.byref(cfg), ctypes.byref(h))
        self._h = h

    @staticmethod
    def box_for_camera(cam, w, h, tmax, y_lo, y_hi):
        lo = np.zeros(3, np.float32)
        hi = np.zeros(3, np.float32)
        call("re_nsdf_box_for_camera", ctypes.byref(cam), w, h, tmax, y_lo, y_hi,
             lo.ctypes.data, hi.ctypes.data)
        return lo, hi

    @property
    def num_params(self) -> int:
        return int(lib.re_nsdf_num_params())

    def close(self):
        if self._h:
            lib.re_nsdf_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_params(self) -> np.ndarray:
        out = np.empty(self.num_params, np.float32)
        call("re_nsdf_get_params", self._h, out.ctypes.data)
        return out

    def set_params(self, params: np.ndarray) -> None:
        params = np.ascontiguousarray(params, np.float32)
        assert params.shape == (self.num_params,)
        call("re_nsdf_set_params", self._h, params.ctypes.data)

    def generate(self, field, cam, w, h, num_points, seed=1, stream=None):
        call("re_nsdf_generate", self._h, ctypes.byref(field), ctypes.byref(cam), w, h,
             num_points, seed, _stream_ptr(stream))

    def data(self, max_points) -> np.ndarray:
        out = np.empty((max_points, 4), np.float32)
        call("re_nsdf_get_data", self._h, out.ctypes.data, max_points)
        return out

    def train(self, steps, batch=65536, lr=1e-3, stream=None) -> np.ndarray:
        loss = np.empty(steps, np.float32)
        call("re_nsdf_train", self._h, steps, batch, lr, loss.ctypes.data, _stream_ptr(stream))
        return loss

    def loss_grad(self, xyzl, stream=None):
        import torch

        n = xyzl.shape[0]
        g = torch.empty(self.num_params, dtype=torch.float32, device="cuda")
        pred = torch.empty(n, dtype=torch.float32, device="cuda")
        call("re_nsdf_loss_grad", self._h, _dptr(xyzl), n, _dptr(g), _dptr(pred),
             _stream_ptr(stream))
        return g, pred

    def eval(self, pts, out=None, stream=None):
        import torch

        n = pts.shape[0]
        if out is None:
            out = torch.empty(n, dtype=torch.float32, device="cuda")
        call("re_nsdf_eval", self._h, _dptr(pts), n, _dptr(out), _stream_ptr(stream))
        return out

    def eval_reference(self, pts, out=None, stream=None):
        import torch

        n = pts.shape[0]
        if out is None:
            out = torch.empty(n, dtype=torch.float32, device="cuda")
        call("re_nsdf_eval_reference", self._h, _dptr(pts), n, _dptr(out), _stream_ptr(stream))
        return out

    def lipschitz(self, samples=200000, h=1e-2, quantile=1.0, stream=None) -> float:
        """Gradient-norm bound: `quantile` of the finite-difference norms (1 = max)."""
        v = ctypes.c_float()
        call("re_nsdf_lipschitz", self._h, samples, h, quantile, ctypes.byref(v),
             _stream_ptr(stream))
        return float(v.value)

    def trace(self, field, tp, cam, w, h, out=None, stream=None, phase="both"):
        """Neural march + exact phase -> int32 CUDA tensor (h*w, 8) = re_sdf_hit.

        phase "network" / "exact" runs one of the two phases (in that order)."""
        import torch

        if out is None:
            out = torch.empty((h * w, 8), dtype=torch.int32, device="cuda")
        fn = {"both": "re_nsdf_trace", "network": "re_nsdf_trace_network",
              "exact": "re_nsdf_trace_exact"}[phase]
        call(fn, self._h, ctypes.byref(field), ctypes.byref(tp), ctypes.byref(cam), w, h,
             _dptr(out), _stream_ptr(stream))
        return out

    def trace_status(self) -> dict:
        """Counters of the last trace (see re_nsdf_trace_status)."""
        n = ctypes.c_uint32()
        e = ctypes.c_int()
        ev = np.zeros(4, np.uint64)
        call("re_nsdf_trace_status", self._h, ctypes.byref(n), ctypes.byref(e), ev.ctypes.data)
        return {"handed_over": int(n.value), "error": int(e.value),
                "network_evals": int(ev[0]), "exact_evals": int(ev[1]),
                "normal_evals": int(ev[2]), "network_rows": int(ev[3])}

    def save(self, path: str):
        call("re_nsdf_save", self._h, path.encode())

    def load(self, path: str):
        call("re_nsdf_load", self._h, path.encode())


# ------------------------------------------------- batched path tracing
class Batch:
    """Many scenes of uneven size path traced by one persistent launch.

    scenes: dicts with either "mesh" (a KDScene) or "terrain" (sdf_params),
    plus "camera", "width", "height" and "albedo"."""

    def __init__(self, scenes, max_depth=4, seed=0, mesh_bias=1e-4):
        arr = (_lib.re_batch_scene * len(scenes))()
        self._meshes = []
        for i, sc in enumerate(scenes):
            e = arr[i]
            if "mesh" in sc:
                e.kind = _lib.BATCH_MESH
                e.mesh = sc["mesh"]._h.value
                self._meshes.append(sc["mesh"])
            else:
                e.kind = _lib.BATCH_TERRAIN
                e.field = sc["terrain"]
            e.camera = sc["camera"]
            e.width, e.height, e.albedo = sc["width"], sc["height"], sc["albedo"]
        pp = _lib.re_path_params(max_depth, seed, mesh_bias)
        h = ctypes.c_void_p()
        call("re_batch_create", arr, len(scenes), ctypes.byref(pp), ctypes.byref(h))
        self._h = h
        self.max_depth = max_depth
        total = ctypes.c_uint64()
        offs = np.zeros(len(scenes), np.uint64)
        call("re_batch_pixels", self._h, ctypes.byref(total), offs.ctypes.data)
        self.total_pixels = int(total.value)
        self.offsets = offs

    def close(self):
        if self._h:
            lib.re_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def render(self, out=None, primary=None, stream=None, graph=False):
        """One frame -> float32 CUDA tensor of total_pixels radiances."""
        import torch

        if out is None:
            out = torch.empty(self.total_pixels, dtype=torch.float32, device="cuda")
        fn = "re_batch_render_graph" if graph else "re_batch_render"
        call(fn, self._h, _dptr(out), _dptr(primary) if primary is not None else None,
             _stream_ptr(stream))
        return out

    def stats(self) -> dict:
        rays = np.zeros(2 * self.max_depth, np.uint64)
        err = ctypes.c_int()
        call("re_batch_stats_get", self._h, rays.ctypes.data, ctypes.byref(err))
        return {"rays": rays.reshape(self.max_depth, 2).astype(np.int64), "error": int(err.value)}

    def set_wait_bounds(self, pending_polls: int = 0, loop_trips: int = 0) -> None:
        """Lower the kernel's wait bounds (0 = defaults); for error-path tests."""
        call("re_batch_set_wait_bounds", self._h, pending_polls, loop_trips)

    def counts(self, out=None, stream=None) -> dict:
        """Traversal and field-evaluation work of one frame."""
        import torch

        if out is None:
            out = torch.empty(self.total_pixels, dtype=torch.float32, device="cuda")
        v = np.zeros(4, np.uint64)
        call("re_batch_counts", self._h, _dptr(out), _stream_ptr(stream), v.ctypes.data)
        return {"inner": int(v[0]), "leaf": int(v[1]), "tests": int(v[2]),
                "field_evals": int(v[3])}

    @property
    def tuning(self) -> dict:
        t = _lib.re_batch_tuning()
        call("re_batch_get_tuning", self._h, ctypes.byref(t))
        return {"block_threads": t.block_threads, "refill_min": t.refill_min,
                "stage_nodes": t.stage_nodes, "steps_per_trip": t.steps_per_trip}

    def set_tuning(self, block_threads, refill_min, stage_nodes, steps_per_trip=8):
        t = _lib.re_batch_tuning(block_threads, refill_min, stage_nodes, steps_per_trip)
        call("re_batch_set_tuning", self._h, ctypes.byref(t))

    def autotune(self, out=None, stream=None) -> dict:
        import torch

        if out is None:
            out = torch.empty(self.total_pixels, dtype=torch.float32, device="cuda")
        t = _lib.re_batch_tuning()
        ms = ctypes.c_float()
        call("re_batch_autotune", self._h, _dptr(out), _stream_ptr(stream), ctypes.byref(t),
             ctypes.byref(ms))
        return {"block_threads": t.block_threads, "refill_min": t.refill_min,
                "stage_nodes": t.stage_nodes, "steps_per_trip": t.steps_per_trip,
                "frame_ms": round(ms.value, 4)}


# ------------------------------------------------------------ shaded frame
def shade_params(albedo=(0.6, 0.6, 0.6), sky_zenith=(0.35, 0.55, 0.95),
                 sky_horizon=(0.85, 0.9, 1.0), one_sided=False):
    p = _lib.re_shade_params()
    p.albedo[:] = [float(x) for x in albedo]
    p.sky_zenith[:] = [float(x) for x in sky_zenith]
    p.sky_horizon[:] = [float(x) for x in sky_horizon]
    p.flags = TRACE_ONE_SIDED if one_sided else 0
    return p


def _light_array(lights):
    arr = (_lib.re_light * max(1, len(lights)))()
    for i, (pos, inten) in enumerate(lights):
        arr[i].pos[:] = [float(x) for x in pos]
        arr[i].intensity = float(inten)
    return arr


def cuda_render_frame(output, width: int, height: int) -> str:
    """The reference's render call (C++ symbol cuda_render_frame(uint*, const
    uint&, const uint&)) on a CUDA tensor of width*height 32-bit pixels."""
    fn = getattr(lib, "_Z17cuda_render_framePjRKjS1_")
    fn.restype = None
    fn.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32)]
    w, h = ctypes.c_uint32(width), ctypes.c_uint32(height)
    fn(_dptr(output), ctypes.byref(w), ctypes.byref(h))
    err = lib.re_last_error()
    return err.decode() if err else ""


# ------------------------------------------------------------ mesh files
MESH_FIRST_TRIANGLE = 1


def load_mesh(path: str, first_triangle_only: bool = False):
    """(vertices float32 (V,3), faces uint32 (F,3)) from a .ply or .obj file."""
    h = ctypes.c_void_p()
    call("re_mesh_load", str(path).encode(), MESH_FIRST_TRIANGLE if first_triangle_only else 0,
         ctypes.byref(h))
    try:
        nv, nf = ctypes.c_uint32(), ctypes.c_uint32()
        call("re_mesh_info", h, ctypes.byref(nv), ctypes.byref(nf))
        verts = np.empty((nv.value, 3), np.float32)
        faces = np.empty((nf.value, 3), np.uint32)
        call("re_mesh_copy", h, verts.ctypes.data, faces.ctypes.data)
    finally:
        lib.re_mesh_destroy(h)
    return verts, faces


# -------------------------------------------------------------- voxel SDF
VOXEL_LOW, VOXEL_MEDIUM, VOXEL_HIGH = 0, 1, 2
BRUSH_SPHERE_ADD, BRUSH_SPHERE_SUBTRACT, BRUSH_CUBE_ADD, BRUSH_CUBE_SUBTRACT = 0, 1, 2, 3


class VoxelGrid:
    """A voxel SDF on the device: 2 floats {distance, material} per voxel."""

    def __init__(self, dim, spacing, origin=(0.0, 0.0, 0.0), data=None):
        import torch

        self.desc = _lib.re_voxel_grid()
        self.desc.dim[:] = [int(x) for x in dim]
        self.desc.spacing[:] = [float(x) for x in spacing]
        self.desc.origin[:] = [float(x) for x in origin]
        n = int(dim[0]) * int(dim[1]) * int(dim[2])
        if data is None:
            self.data = torch.zeros(2 * n, dtype=torch.float32, device="cuda")
        else:
            self.data = torch.as_tensor(np.ascontiguousarray(data, np.float32).reshape(-1)).cuda()

    @classmethod
    def bake(cls, field, dim, spacing, origin=(0.0, 0.0, 0.0), stream=None):
        g = cls(dim, spacing, origin)
        call("re_voxel_bake", ctypes.byref(field), ctypes.byref(g.desc), _dptr(g.data),
             _stream_ptr(stream))
        return g

    @classmethod
    def load(cls, path: str, origin=(0.0, 0.0, 0.0)):
        d = _lib.re_voxel_grid()
        call("re_voxel_load", str(path).encode(), ctypes.byref(d), None, 0)
        n = d.dim[0] * d.dim[1] * d.dim[2]
        host = np.empty(2 * n, np.float32)
        call("re_voxel_load", str(path).encode(), ctypes.byref(d), host.ctypes.data, n)
        return cls(list(d.dim), list(d.spacing), origin, host)

    def save(self, path: str):
        host = np.ascontiguousarray(self.data.cpu().numpy())
        call("re_voxel_save", str(path).encode(), ctypes.byref(self.desc), host.ctypes.data)

    def sample(self, pts, quality, out=None, stream=None):
        import torch

        n = pts.shape[0]
        if out is None:
            out = torch.empty(n, dtype=torch.float32, device="cuda")
        call("re_voxel_sample", _dptr(self.data), ctypes.byref(self.desc), quality, _dptr(pts), n,
             _dptr(out), _stream_ptr(stream))
        return out

    def brush(self, kind, center, extent, material=0.0, smooth=0.1, stream=None):
        """Edit every voxel: kind in BRUSH_SPHERE_ADD / _SUBTRACT, BRUSH_CUBE_ADD / _SUBTRACT."""
        b = _lib.re_voxel_brush_params()
        b.type = kind
        b.center[:] = [float(x) for x in center]
        ext = list(extent) if hasattr(extent, "__len__") else [extent, extent, extent]
        b.extent[:] = [float(x) for x in ext]
        b.material, b.smooth = float(material), float(smooth)
        call("re_voxel_brush", _dptr(self.data), ctypes.byref(self.desc), ctypes.byref(b),
             _stream_ptr(stream))

    def trace(self, quality, march, cam, w, h, out=None, stream=None):
        import torch

        if out is None:
            out = torch.empty((h * w, 8), dtype=torch.int32, device="cuda")
        call("re_voxel_trace", _dptr(self.data), ctypes.byref(self.desc), quality,
             ctypes.byref(march), ctypes.byref(cam), w, h, _dptr(out), _stream_ptr(stream))
        return out


# ------------------------------------------------------------ instances
def instance_trig(yaw: float):
    """(cos, sin) of a yaw as the instanced tracer computes them."""
    c, s_ = ctypes.c_float(), ctypes.c_float()
    lib.re_instance_trig(ctypes.c_float(yaw), ctypes.byref(c), ctypes.byref(s_))
    return c.value, s_.value


def trace_instances(instances, cam, w, h, flags=TRACE_TWO_SIDED, stream=None):
    """instances: [(KDScene, yaw, location xyz)] -> (re_hit (h*w, 4) int32,
    instance index (h*w,) int32) CUDA tensors."""
    import torch

    arr = (_lib.re_instance * len(instances))()
    for i, (sc, yaw, loc) in enumerate(instances):
        arr[i].mesh = sc._h.value
        arr[i].yaw = float(yaw)
        arr[i].location[:] = [float(x) for x in loc]
    out = torch.empty((h * w, 4), dtype=torch.int32, device="cuda")
    idx = torch.empty(h * w, dtype=torch.int32, device="cuda")
    call("re_trace_instances", arr, len(instances), ctypes.byref(cam), w, h, flags, _dptr(out),
         _dptr(idx), _stream_ptr(stream))
    return out, idx


def measure_l2_read_gbs(nbytes: int = 32 << 20, passes: int = 100, stream=None) -> float:
    """L2 read bandwidth of this GPU in GB/s (re_measure_l2_read)."""
    v = ctypes.c_float()
    call("re_measure_l2_read", nbytes, passes, ctypes.byref(v), _stream_ptr(stream))
    return float(v.value)


def measure_fp32_fma_tops(iters: int = 1 << 16, stream=None) -> float:
    """FP32 fused multiply-adds per second of this GPU, in 10^12
    (re_measure_fp32_fma; one FMA counts as one operation)."""
    v = ctypes.c_float()
    call("re_measure_fp32_fma", iters, ctypes.byref(v), _stream_ptr(stream))
    return float(v.value)

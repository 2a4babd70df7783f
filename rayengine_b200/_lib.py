"""ctypes binding of librayengine_b200.so (declarations: include/rayengine_b200.h).

The shared library is the product: there is no Python or CPU fallback.  If
the library file is missing this module raises at import time.  The library
is mapped into the process on the first call through ``lib`` (not at
import), so code that only uses the package's pure-Python helpers (camera
construction, triangle packing, workload descriptions) never loads it.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librayengine_b200.so")


class RayEngineError(RuntimeError):
    """A C-ABI call returned a non-zero re_status."""

    def __init__(self, status: int, fn: str, message: str):
        super().__init__(f"{fn} failed with status {status}: {message}")
        self.status = status


if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
        "or `make -f rayengine_b200/csrc/Makefile`"
    )

c_float_p = ctypes.POINTER(ctypes.c_float)
c_u32_p = ctypes.POINTER(ctypes.c_uint32)


class re_camera(ctypes.Structure):
    """Same layout as the reference's RCamera (Camera.h:7-16), 88 bytes."""

    _fields_ = [
        ("campos", ctypes.c_float * 3),
        ("camdir", ctypes.c_float * 3),
        ("camright", ctypes.c_float * 3),
        ("camdown", ctypes.c_float * 3),
        ("lookat", ctypes.c_float * 3),
        ("view", ctypes.c_float * 3),
        ("fov", ctypes.c_float * 2),
        ("focial_distance", ctypes.c_float),
        ("apertude_radius", ctypes.c_float),
    ]


class re_kd_params(ctypes.Structure):
    _fields_ = [
        ("max_depth", ctypes.c_uint32),
        ("leaf_size", ctypes.c_uint32),
        ("cost_traversal", ctypes.c_float),
        ("cost_intersect", ctypes.c_float),
        ("empty_bonus", ctypes.c_float),
        ("bfs_levels", ctypes.c_uint32),
        ("threads", ctypes.c_uint32),
        ("max_leaf_visits", ctypes.c_uint32),
    ]


class re_scene_stats(ctypes.Structure):
    _fields_ = [
        ("num_tris", ctypes.c_uint32),
        ("num_nodes", ctypes.c_uint32),
        ("num_leaves", ctypes.c_uint32),
        ("num_refs", ctypes.c_uint32),
        ("max_depth", ctypes.c_uint32),
        ("max_leaf_size", ctypes.c_uint32),
        ("bfs_nodes", ctypes.c_uint32),
        ("pad", ctypes.c_uint32),
        ("bmin", ctypes.c_float * 3),
        ("bmax", ctypes.c_float * 3),
        ("build_seconds", ctypes.c_double),
        ("device_bytes", ctypes.c_uint64),
    ]


class re_tuning(ctypes.Structure):
    _fields_ = [
        ("stage_nodes", ctypes.c_uint32),
        ("queue_kind_major", ctypes.c_uint32),
        ("refill_min", ctypes.c_uint32),
        ("ray_refill_min", ctypes.c_uint32),
        ("ray_lanes", ctypes.c_uint32),
    ]


class re_ao_params(ctypes.Structure):
    _fields_ = [
        ("light_dir", ctypes.c_float * 3),
        ("ao_length", ctypes.c_float),
        ("bias", ctypes.c_float),
        ("seed", ctypes.c_uint32),
    ]


class re_fbm_params(ctypes.Structure):
    _fields_ = [
        ("seed", ctypes.c_uint32),
        ("octaves", ctypes.c_uint32),
        ("lacunarity", ctypes.c_float),
        ("gain", ctypes.c_float),
        ("scale", ctypes.c_float),
        ("amplitude", ctypes.c_float),
    ]


class re_sdf_params(ctypes.Structure):
    _fields_ = [
        ("seed", ctypes.c_uint32),
        ("octaves", ctypes.c_uint32),
        ("scale", ctypes.c_float),
        ("amplitude", ctypes.c_float),
        ("step_factor", ctypes.c_float),
        ("eps", ctypes.c_float),
        ("tmax", ctypes.c_float),
        ("max_steps", ctypes.c_uint32),
    ]


class re_sdf_shade_params(ctypes.Structure):
    _fields_ = [
        ("light_pos", ctypes.c_float * 2),
        ("light_intensity", ctypes.c_float),
        ("soft_shadow_k", ctypes.c_float),
        ("shadow_tmin", ctypes.c_float),
        ("shadow_tmax", ctypes.c_float),
        ("shadow_max_steps", ctypes.c_uint32),
        ("sun_dir", ctypes.c_float * 3),
        ("max_y", ctypes.c_float),
        ("fog_density", ctypes.c_float),
        ("vignetting_k", ctypes.c_float),
        ("flags", ctypes.c_uint32),
    ]


SDF_SHADE, SDF_FOG, SDF_GAMMA, SDF_VIGNETTING = 1, 2, 4, 8


class re_nsdf_config(ctypes.Structure):
    _fields_ = [
        ("box_min", ctypes.c_float * 3),
        ("box_max", ctypes.c_float * 3),
        ("f0", ctypes.c_float),
        ("seed", ctypes.c_uint32),
    ]


class re_nsdf_trace_params(ctypes.Structure):
    _fields_ = [
        ("lipschitz", ctypes.c_float),
        ("safety", ctypes.c_float),
        ("switch_dist", ctypes.c_float),
        ("min_step", ctypes.c_float),
        ("max_network_steps", ctypes.c_uint32),
        ("max_exact_steps", ctypes.c_uint32),
        ("root_steps", ctypes.c_uint32),
        ("relax", ctypes.c_float),
        ("flags", ctypes.c_uint32),
        ("cone_tile", ctypes.c_uint32),
        ("cone_coarse", ctypes.c_uint32),
        ("normal_taps", ctypes.c_uint32),
        ("cone_lanes", ctypes.c_uint32),
        ("root_tol", ctypes.c_float),
    ]


NSDF_EXACT_ONLY = 1


class re_voxel_grid(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_uint32 * 3), ("spacing", ctypes.c_float * 3),
                ("origin", ctypes.c_float * 3)]


class re_instance(ctypes.Structure):
    _fields_ = [("mesh", ctypes.c_void_p), ("yaw", ctypes.c_float),
                ("location", ctypes.c_float * 3)]


class re_voxel_brush_params(ctypes.Structure):
    _fields_ = [("type", ctypes.c_uint32), ("center", ctypes.c_float * 3),
                ("extent", ctypes.c_float * 3), ("material", ctypes.c_float),
                ("smooth", ctypes.c_float)]


class re_light(ctypes.Structure):
    _fields_ = [("pos", ctypes.c_float * 3), ("intensity", ctypes.c_float)]


class re_shade_params(ctypes.Structure):
    _fields_ = [("albedo", ctypes.c_float * 3), ("sky_zenith", ctypes.c_float * 3),
                ("sky_horizon", ctypes.c_float * 3), ("flags", ctypes.c_uint32)]


class re_batch_scene(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_uint32),
        ("mesh", ctypes.c_void_p),
        ("field", re_sdf_params),
        ("camera", re_camera),
        ("width", ctypes.c_uint32),
        ("height", ctypes.c_uint32),
        ("albedo", ctypes.c_float),
    ]


class re_path_params(ctypes.Structure):
    _fields_ = [("max_depth", ctypes.c_uint32), ("seed", ctypes.c_uint32),
                ("mesh_bias", ctypes.c_float)]


class re_batch_tuning(ctypes.Structure):
    _fields_ = [("block_threads", ctypes.c_uint32), ("refill_min", ctypes.c_uint32),
                ("stage_nodes", ctypes.c_uint32), ("steps_per_trip", ctypes.c_uint32)]


BATCH_MESH, BATCH_TERRAIN = 0, 1


_P = ctypes.c_void_p
_U32 = ctypes.c_uint32
_F = ctypes.c_float
_SIGS = {
    "re_abi_version": (ctypes.c_int, []),
    "re_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "re_last_error": (ctypes.c_char_p, []),
    "re_kd_params_default": (None, [ctypes.POINTER(re_kd_params)]),
    "re_scene_create": (ctypes.c_int, [_P, _U32, _P, _U32, ctypes.POINTER(re_kd_params), ctypes.POINTER(_P)]),
    "re_scene_create_packed": (ctypes.c_int, [_P, _U32, ctypes.POINTER(re_kd_params), ctypes.POINTER(_P)]),
    "re_scene_build_host": (ctypes.c_int, [_P, _U32, ctypes.POINTER(re_kd_params), ctypes.POINTER(_P)]),
    "re_scene_stats_get": (ctypes.c_int, [_P, ctypes.POINTER(re_scene_stats)]),
    "re_scene_export": (ctypes.c_int, [_P, _P, _P, _P]),
    "re_scene_export_entry": (ctypes.c_int, [_P, _P, _P]),
    "re_scene_destroy": (ctypes.c_int, [_P]),
    "re_trace_primary": (ctypes.c_int, [_P, ctypes.POINTER(re_camera), _U32, _U32, _U32, _P, _P]),
    "re_trace_rays": (ctypes.c_int, [_P, _P, _U32, _U32, _P, _P]),
    "re_count_primary": (ctypes.c_int, [_P, ctypes.POINTER(re_camera), _U32, _U32, _U32, _P, _P]),
    "re_scene_truncated": (ctypes.c_int, [_P, _P, _P]),
    "re_render_ao": (ctypes.c_int, [_P, ctypes.POINTER(re_camera), _U32, _U32, ctypes.POINTER(re_ao_params), _P, _P, _P, _P]),
    "re_render_ao_primary": (ctypes.c_int, [_P, ctypes.POINTER(re_camera), _U32, _U32, ctypes.POINTER(re_ao_params), _P, _P, _P]),
    "re_render_ao_secondary": (ctypes.c_int, [_P, _P, _P, _P]),
    "re_render_ao_noalloc": (ctypes.c_int, [_P, ctypes.POINTER(re_camera), _U32, _U32, ctypes.POINTER(re_ao_params), _P, _P, _P, _P]),
    "re_autotune_ao": (ctypes.c_int, [_P, ctypes.POINTER(re_camera), _U32, _U32, ctypes.POINTER(re_ao_params), ctypes.POINTER(re_tuning), ctypes.POINTER(ctypes.c_float), _P]),
    "re_autotune_primary": (ctypes.c_int, [_P, ctypes.POINTER(re_camera), _U32, _U32, _U32, ctypes.POINTER(re_tuning), ctypes.POINTER(ctypes.c_float), _P]),
    "re_scene_get_tuning": (ctypes.c_int, [_P, ctypes.POINTER(re_tuning)]),
    "re_scene_set_tuning": (ctypes.c_int, [_P, ctypes.POINTER(re_tuning)]),
    "re_render_ao_counts": (ctypes.c_int, [_P, ctypes.POINTER(re_camera), _U32, _U32, ctypes.POINTER(re_ao_params), _P, _P]),
    "re_perlin_permutation": (ctypes.c_int, [_U32, _P]),
    "re_noise_fbm": (ctypes.c_int, [ctypes.POINTER(re_fbm_params), _P, _U32, _P, _P]),
    "re_heightfield": (ctypes.c_int, [ctypes.POINTER(re_fbm_params), _U32, ctypes.c_float, ctypes.c_float, _P, _P]),
    "re_gen_soup": (ctypes.c_int, [ctypes.c_uint64, _U32, _P]),
    "re_gen_grid_faces": (ctypes.c_int, [_U32, _P]),
    "re_sdf_trace": (ctypes.c_int, [ctypes.POINTER(re_sdf_params), ctypes.POINTER(re_camera), _U32, _U32, _P, _P]),
    "re_sdf_shade_params_default": (None, [ctypes.POINTER(re_sdf_shade_params)]),
    "re_sdf_shade": (ctypes.c_int, [ctypes.POINTER(re_sdf_params), ctypes.POINTER(re_sdf_shade_params), ctypes.POINTER(re_camera), _U32, _U32, _P, _P, _P, _P]),
    "re_render_sdf_frame": (ctypes.c_int, [ctypes.POINTER(re_sdf_params), ctypes.POINTER(re_sdf_shade_params), ctypes.POINTER(re_camera), _U32, _U32, _P, _P, _P]),
    "re_sdf_frame_bind": (ctypes.c_int, [ctypes.POINTER(re_sdf_params), ctypes.POINTER(re_sdf_shade_params), ctypes.POINTER(re_camera), ctypes.c_int]),
    "re_fmath": (ctypes.c_int, [_U32, _P, _P, _U32, _P, _P]),
    "re_nsdf_num_params": (ctypes.c_uint32, []),
    "re_nsdf_box_for_camera": (ctypes.c_int, [ctypes.POINTER(re_camera), _U32, _U32, _F, _F, _F, _P, _P]),
    "re_nsdf_create": (ctypes.c_int, [ctypes.POINTER(re_nsdf_config), ctypes.POINTER(_P)]),
    "re_nsdf_destroy": (ctypes.c_int, [_P]),
    "re_nsdf_get_params": (ctypes.c_int, [_P, _P]),
    "re_nsdf_set_params": (ctypes.c_int, [_P, _P]),
    "re_nsdf_generate": (ctypes.c_int, [_P, ctypes.POINTER(re_sdf_params), ctypes.POINTER(re_camera), _U32, _U32, _U32, _U32, _P]),
    "re_nsdf_get_data": (ctypes.c_int, [_P, _P, _U32]),
    "re_nsdf_train": (ctypes.c_int, [_P, _U32, _U32, _F, _P, _P]),
    "re_nsdf_loss_grad": (ctypes.c_int, [_P, _P, _U32, _P, _P, _P]),
    "re_nsdf_eval": (ctypes.c_int, [_P, _P, _U32, _P, _P]),
    "re_nsdf_eval_reference": (ctypes.c_int, [_P, _P, _U32, _P, _P]),
    "re_nsdf_lipschitz": (ctypes.c_int, [_P, _U32, _F, _F, ctypes.POINTER(_F), _P]),
    "re_nsdf_trace": (ctypes.c_int, [_P, ctypes.POINTER(re_sdf_params), ctypes.POINTER(re_nsdf_trace_params), ctypes.POINTER(re_camera), _U32, _U32, _P, _P]),
    "re_nsdf_trace_network": (ctypes.c_int, [_P, ctypes.POINTER(re_sdf_params), ctypes.POINTER(re_nsdf_trace_params), ctypes.POINTER(re_camera), _U32, _U32, _P, _P]),
    "re_nsdf_trace_exact": (ctypes.c_int, [_P, ctypes.POINTER(re_sdf_params), ctypes.POINTER(re_nsdf_trace_params), ctypes.POINTER(re_camera), _U32, _U32, _P, _P]),
    "re_nsdf_trace_status": (ctypes.c_int, [_P, ctypes.POINTER(_U32), ctypes.POINTER(ctypes.c_int), _P]),
    "re_voxel_bake": (ctypes.c_int, [ctypes.POINTER(re_sdf_params), ctypes.POINTER(re_voxel_grid), _P, _P]),
    "re_voxel_sample": (ctypes.c_int, [_P, ctypes.POINTER(re_voxel_grid), _U32, _P, _U32, _P, _P]),
    "re_voxel_trace": (ctypes.c_int, [_P, ctypes.POINTER(re_voxel_grid), _U32, ctypes.POINTER(re_sdf_params), ctypes.POINTER(re_camera), _U32, _U32, _P, _P]),
    "re_voxel_save": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(re_voxel_grid), _P]),
    "re_voxel_load": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(re_voxel_grid), _P, ctypes.c_uint64]),
    "re_voxel_brush": (ctypes.c_int, [_P, ctypes.POINTER(re_voxel_grid), ctypes.POINTER(re_voxel_brush_params), _P]),
    "re_trace_instances": (ctypes.c_int, [ctypes.POINTER(re_instance), _U32, ctypes.POINTER(re_camera), _U32, _U32, _U32, _P, _P, _P]),
    "re_instance_trig": (None, [_F, ctypes.POINTER(_F), ctypes.POINTER(_F)]),
    "re_measure_l2_read": (ctypes.c_int, [ctypes.c_size_t, _U32, ctypes.POINTER(_F), _P]),
    "re_measure_fp32_fma": (ctypes.c_int, [_U32, ctypes.POINTER(_F), _P]),
    "re_mesh_load": (ctypes.c_int, [ctypes.c_char_p, _U32, ctypes.POINTER(ctypes.c_void_p)]),
    "re_mesh_info": (ctypes.c_int, [_P, ctypes.POINTER(_U32), ctypes.POINTER(_U32)]),
    "re_mesh_copy": (ctypes.c_int, [_P, _P, _P]),
    "re_mesh_destroy": (ctypes.c_int, [_P]),
    "re_render_frame": (ctypes.c_int, [_P, ctypes.POINTER(re_camera), ctypes.POINTER(re_light), _U32, ctypes.POINTER(re_shade_params), _U32, _U32, _P, _P]),
    "re_frame_bind": (ctypes.c_int, [_P, ctypes.POINTER(re_camera), ctypes.POINTER(re_light), _U32, ctypes.POINTER(re_shade_params), ctypes.c_int]),
    "re_batch_create": (ctypes.c_int, [ctypes.POINTER(re_batch_scene), _U32, ctypes.POINTER(re_path_params), ctypes.POINTER(ctypes.c_void_p)]),
    "re_batch_destroy": (ctypes.c_int, [_P]),
    "re_batch_pixels": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_uint64), _P]),
    "re_batch_render": (ctypes.c_int, [_P, _P, _P, _P]),
    "re_batch_render_graph": (ctypes.c_int, [_P, _P, _P, _P]),
    "re_batch_stats_get": (ctypes.c_int, [_P, _P, ctypes.POINTER(ctypes.c_int)]),
    "re_batch_set_wait_bounds": (ctypes.c_int, [_P, _U32, _U32]),
    "re_batch_counts": (ctypes.c_int, [_P, _P, _P, _P]),
    "re_batch_get_tuning": (ctypes.c_int, [_P, ctypes.POINTER(re_batch_tuning)]),
    "re_batch_set_tuning": (ctypes.c_int, [_P, ctypes.POINTER(re_batch_tuning)]),
    "re_batch_autotune": (ctypes.c_int, [_P, _P, _P, ctypes.POINTER(re_batch_tuning), ctypes.POINTER(_F)]),
    "re_nsdf_save": (ctypes.c_int, [_P, ctypes.c_char_p]),
    "re_nsdf_load": (ctypes.c_int, [_P, ctypes.c_char_p]),
}

EXPORTED = tuple(_SIGS)

# RE_ABI_VERSION of include/rayengine_b200.h that the structures above mirror
ABI_VERSION = 2


class _Library:
    """librayengine_b200.so, loaded (and its signatures declared) on first use."""

    def __init__(self):
        self._dll = None

    def _load(self):
        if self._dll is None:
            dll = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in _SIGS.items():
                fn = getattr(dll, name)
                fn.restype = res
                fn.argtypes = args
            abi = dll.re_abi_version()
            if abi != ABI_VERSION:
                raise ImportError(f"{LIB_PATH} has ABI version {abi}, these bindings expect "
                                  f"{ABI_VERSION}: rebuild the library")
            self._dll = dll
        return self._dll

    @property
    def loaded(self) -> bool:
        return self._dll is not None

    def __getattr__(self, name):
        if name.startswith("__"):
            raise AttributeError(name)
        return getattr(self._load(), name)


lib = _Library()


def check(status: int, fn: str) -> None:
    if status != 0:
        msg = lib.re_last_error()
        raise RayEngineError(status, fn, msg.decode() if msg else "")


def call(name: str, *args) -> None:
    check(getattr(lib, name)(*args), name)

"""TEST INFRASTRUCTURE ONLY: ctypes binding of the CPU oracle (liboracle.so).

Imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and
reference legs, as the checker.  The product (rayengine_b200/) never imports
it.  Build with `make -f oracle/Makefile`.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_LIB_PATH = os.path.join(HERE, "_ref", "libre_ref.so")

HIT_DTYPE = np.dtype([("id", "<i4"), ("t", "<f4"), ("u", "<f4"), ("v", "<f4")])
COUNT_DTYPE = np.dtype([("inner", "<u4"), ("leaf", "<u4"), ("tests", "<u4"), ("status", "<u4")])
SDF_DTYPE = np.dtype([("pos", "<f4", 3), ("normal", "<f4", 3), ("steps", "<u4"),
                      ("status", "<u4"), ("t", "<f4"), ("pad", "<f4")])

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} missing: run `make -f oracle/Makefile`")
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.o_ray_tri.restype = ctypes.c_int
        _lib.o_perlin.restype = ctypes.c_float
        _lib.o_perlin.argtypes = [ctypes.c_void_p, ctypes.c_float, ctypes.c_float, ctypes.c_float]
        _lib.o_fbm.restype = ctypes.c_float
        _lib.o_fbm.argtypes = [ctypes.c_void_p, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                               ctypes.c_int, ctypes.c_float, ctypes.c_float]
        _lib.o_hash_u32.restype = ctypes.c_uint32
        _lib.o_hash_u32.argtypes = [ctypes.c_uint32] * 3
        _lib.o_sincos_2pi.argtypes = [ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p]
        _lib.o_max_threads.restype = ctypes.c_int
    return _lib


class OCamera(ctypes.Structure):
    _fields_ = [("campos", ctypes.c_float * 3), ("view", ctypes.c_float * 3),
                ("camdown", ctypes.c_float * 3), ("fov", ctypes.c_float * 2),
                ("focal", ctypes.c_float)]


class OKdTree(ctypes.Structure):
    _fields_ = [("nodes", ctypes.c_void_p), ("leaves", ctypes.c_void_p),
                ("tris", ctypes.c_void_p), ("bmin", ctypes.c_float * 3),
                ("bmax", ctypes.c_float * 3)]


def camera(re_cam) -> OCamera:
    """Oracle camera from a product re_camera (same field values)."""
    c = OCamera()
    c.campos[:] = list(re_cam.campos)
    c.view[:] = list(re_cam.view)
    c.camdown[:] = list(re_cam.camdown)
    c.fov[:] = list(re_cam.fov)
    c.focal = re_cam.focial_distance
    return c


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def threads() -> int:
    return lib().o_max_threads()


def perm(seed: int) -> np.ndarray:
    out = np.zeros(512, np.uint32)
    lib().o_perlin_permutation(ctypes.c_uint32(seed), _p(out))
    return out


def soup(seed: int, n: int) -> np.ndarray:
    v = np.zeros((n, 3, 3), np.float32)
    lib().o_gen_soup(ctypes.c_uint64(seed), ctypes.c_int32(n), _p(v))
    return v


def heightfield(p: np.ndarray, cells: int, lo: float, hi: float, octaves: int, amp: float):
    nv = cells + 1
    verts = np.zeros((nv * nv, 3), np.float32)
    faces = np.zeros((2 * cells * cells, 3), np.uint32)
    lib().o_gen_heightfield(_p(p), ctypes.c_int32(cells), ctypes.c_float(lo), ctypes.c_float(hi),
                            ctypes.c_int(octaves), ctypes.c_float(amp), _p(verts), _p(faces))
    return verts, faces


def fbm_batch(p, pts, octaves, lac=2.0, gain=0.5, scale=1.0, amp=1.0, nthreads=0):
    pts = np.ascontiguousarray(pts, np.float32)
    out = np.zeros(pts.shape[0], np.float32)
    lib().o_batch_fbm(_p(p), _p(pts), ctypes.c_int64(pts.shape[0]), ctypes.c_int(octaves),
                      ctypes.c_float(lac), ctypes.c_float(gain), ctypes.c_float(scale),
                      ctypes.c_float(amp), _p(out), ctypes.c_int(nthreads))
    return out


class KdTree:
    """Oracle view of a flattened tree (arrays from KDScene.export())."""

    def __init__(self, nodes, leaves, tris, bmin, bmax):
        self.nodes = np.ascontiguousarray(nodes, np.uint32)
        self.leaves = np.ascontiguousarray(leaves, np.uint32)
        self.tris = np.ascontiguousarray(tris, np.float32)
        self.s = OKdTree()
        self.s.nodes = self.nodes.ctypes.data
        self.s.leaves = self.leaves.ctypes.data
        self.s.tris = self.tris.ctypes.data
        self.s.bmin[:] = [float(x) for x in bmin]
        self.s.bmax[:] = [float(x) for x in bmax]


def primary_kd(kd: KdTree, cam, w, h, mode=0, max_visits=16384, pixels=None, counts=False,
               nthreads=0):
    pix = None if pixels is None else np.ascontiguousarray(pixels, np.uint32)
    n = w * h if pix is None else pix.shape[0]
    out = np.zeros(n, HIT_DTYPE)
    cnt = np.zeros(n, COUNT_DTYPE) if counts else None
    oc = camera(cam)
    lib().o_batch_primary_kd(ctypes.byref(kd.s), ctypes.byref(oc), ctypes.c_uint32(w),
                             ctypes.c_uint32(h), ctypes.c_int(mode), ctypes.c_uint32(max_visits),
                             _p(pix), ctypes.c_int64(n), _p(out), _p(cnt), ctypes.c_int(nthreads))
    return (out, cnt) if counts else out


def primary_bruteforce(tris_packed, bmin, bmax, cam, w, h, mode=0, pixels=None, nthreads=0):
    tris = np.ascontiguousarray(tris_packed, np.float32)
    pix = None if pixels is None else np.ascontiguousarray(pixels, np.uint32)
    n = w * h if pix is None else pix.shape[0]
    out = np.zeros(n, HIT_DTYPE)
    oc = camera(cam)
    b0 = (ctypes.c_float * 3)(*bmin)
    b1 = (ctypes.c_float * 3)(*bmax)
    lib().o_batch_primary_bruteforce(_p(tris), ctypes.c_int32(tris.shape[0]), b0, b1,
                                     ctypes.byref(oc), ctypes.c_uint32(w), ctypes.c_uint32(h),
                                     ctypes.c_int(mode), _p(pix), ctypes.c_int64(n), _p(out),
                                     ctypes.c_int(nthreads))
    return out


def rays_kd(kd: KdTree, rays, mode=0, anyhit=False, max_visits=16384, nthreads=0):
    rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    out = np.zeros(rays.shape[0], HIT_DTYPE)
    lib().o_batch_rays_kd(ctypes.byref(kd.s), _p(rays), ctypes.c_int64(rays.shape[0]),
                          ctypes.c_int(mode), ctypes.c_int(1 if anyhit else 0),
                          ctypes.c_uint32(max_visits), _p(out), ctypes.c_int(nthreads))
    return out


def frame_ao(kd: KdTree, packed, cam, w, h, light_dir, ao_length, bias, seed, pixels=None,
             max_visits=16384, nthreads=0, totals=False):
    packed = np.ascontiguousarray(packed, np.float32)
    pix = None if pixels is None else np.ascontiguousarray(pixels, np.uint32)
    n = w * h if pix is None else pix.shape[0]
    out = np.zeros(n, HIT_DTYPE)
    mask = np.zeros(n, np.uint32)
    nsec = ctypes.c_uint32(0)
    tot = np.zeros(10, np.uint64)
    oc = camera(cam)
    ld = (ctypes.c_float * 3)(*light_dir)
    lib().o_batch_frame_ao(ctypes.byref(kd.s), _p(packed), ctypes.byref(oc), ctypes.c_uint32(w),
                           ctypes.c_uint32(h), ld, ctypes.c_float(ao_length), ctypes.c_float(bias),
                           ctypes.c_uint32(seed), ctypes.c_uint32(max_visits), _p(pix),
                           ctypes.c_int64(n), _p(out), _p(mask), ctypes.byref(nsec), _p(tot),
                           ctypes.c_int(nthreads))
    if totals:
        return out, mask, nsec.value, tot
    return out, mask, nsec.value


def sdf_image(p, cam, w, h, octaves=8, scale=0.25, amp=3.0, step_factor=0.6, eps=1e-4,
              tmax=200.0, max_steps=512, pixels=None, nthreads=0):
    pix = None if pixels is None else np.ascontiguousarray(pixels, np.uint32)
    n = w * h if pix is None else pix.shape[0]
    out = np.zeros(n, SDF_DTYPE)
    oc = camera(cam)
    lib().o_batch_sdf(_p(p), ctypes.byref(oc), ctypes.c_uint32(w), ctypes.c_uint32(h),
                      ctypes.c_int(octaves), ctypes.c_float(scale), ctypes.c_float(amp),
                      ctypes.c_float(step_factor), ctypes.c_float(eps), ctypes.c_float(tmax),
                      ctypes.c_uint32(max_steps), _p(pix), ctypes.c_int64(n), _p(out),
                      ctypes.c_int(nthreads))
    return out


def sincos_2pi(u: float):
    s = ctypes.c_float()
    c = ctypes.c_float()
    lib().o_sincos_2pi(ctypes.c_float(u), ctypes.byref(s), ctypes.byref(c))
    return s.value, c.value


def hash_u32(a, b, c) -> int:
    return lib().o_hash_u32(a, b, c)


# ---------------------------------------------------------- FP64 arbiter
def edge_margin(packed, ids, o, d):
    """Barycentric margin min(u, v, 1-u-v) of the ray against triangle ids,
    in float64 (the relative edge distance used to exempt grazing rays)."""
    packed = np.asarray(packed, np.float64)
    T = packed[ids]
    v0, e1, e2 = T[:, 0:3], T[:, 4:7], T[:, 8:11]
    o = np.asarray(o, np.float64)
    d = np.asarray(d, np.float64)
    h = np.cross(d, e2)
    a = np.einsum("ij,ij->i", e1, h)
    s = o - v0
    f = 1.0 / a
    u = f * np.einsum("ij,ij->i", s, h)
    q = np.cross(s, e1)
    v = f * np.einsum("ij,ij->i", d, q)
    return np.minimum(np.minimum(u, v), 1.0 - u - v)


def camera_rays(cam, w, h, pixels):
    """Float64 ray origins/directions of the given pixels (arbiter only)."""
    campos = np.array(cam.campos, np.float64)
    view = np.array(cam.view, np.float64)
    view /= np.linalg.norm(view)
    down = np.array(cam.camdown, np.float64)
    down /= np.linalg.norm(down)
    hx = np.cross(view, down)
    hx /= np.linalg.norm(hx)
    vx = np.cross(hx, view)
    vx /= np.linalg.norm(vx)
    th = np.tan(np.radians(cam.fov[0]) * 0.5)
    tv = np.tan(np.radians(cam.fov[1]) * 0.5)
    pixels = np.asarray(pixels)
    x = (pixels % w).astype(np.float64)
    y = (pixels // w).astype(np.float64)
    sx = x / (w - 1.0)
    sy = 1.0 - y / (h - 1.0)
    p = campos + view + hx * th * (2 * sx - 1)[:, None] + vx * tv * (2 * sy - 1)[:, None]
    d = (p - campos) * cam.focial_distance
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.broadcast_to(campos, d.shape).copy(), d


# ---------------------------------------------- the reference, compiled
def ref_lib():
    """The reference's own host code (oracle/_ref/libre_ref.so), or None."""
    if not os.path.exists(REF_LIB_PATH):
        return None
    L = ctypes.CDLL(REF_LIB_PATH)
    L.ref_sizeof_node.restype = ctypes.c_int
    L.ref_build_kdtree.restype = ctypes.c_int
    return L


def ref_build(verts, faces):
    """Reference RKDTreeCPU + RKDThreeGPU over a mesh -> (raw 128-byte node
    records, obj_index_list, root, levels, leaves)."""
    L = ref_lib()
    if L is None:
        raise FileNotFoundError(REF_LIB_PATH)
    verts = np.ascontiguousarray(verts, np.float32)
    faces = np.ascontiguousarray(faces, np.uint32)
    max_nodes = 4 * faces.shape[0] + 16
    nodes = np.zeros((max_nodes, 128), np.uint8)
    idx = np.zeros(64 * faces.shape[0] + 16, np.int32)
    root, nidx, levels, leaves = (ctypes.c_int() for _ in range(4))
    nn = L.ref_build_kdtree(_p(verts), ctypes.c_int(verts.shape[0]), _p(faces),
                            ctypes.c_int(faces.shape[0]), _p(nodes), ctypes.c_int(max_nodes),
                            _p(idx), ctypes.c_int(idx.shape[0]), ctypes.byref(root),
                            ctypes.byref(nidx), ctypes.byref(levels), ctypes.byref(leaves))
    if nn < 0:
        raise RuntimeError("reference tree larger than the buffers")
    return nodes[:nn].copy(), idx[: nidx.value].copy(), root.value, levels.value, leaves.value


class RefTree:
    """The reference's own CPU kd-tree and ray query (RKDTreeCPU built by its
    constructor, KDTree.cpp:117-173, queried with singleRayStacklessIntersect,
    KDTree.cpp:993-1066), compiled from its sources into oracle/_ref.  As
    shipped the tree is one leaf, so a query is Moller-Trumbore over every
    triangle (two-sided, t > 1e-5) keeping the smallest t."""

    def __init__(self, verts, faces):
        L = ref_lib()
        if L is None:
            raise FileNotFoundError(REF_LIB_PATH)
        L.ref_tree_create.restype = ctypes.c_void_p
        L.ref_tree_destroy.argtypes = [ctypes.c_void_p]
        L.ref_tree_trace.restype = ctypes.c_int64
        L.ref_tree_trace.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        L.ref_max_threads.restype = ctypes.c_int
        self._L = L
        v = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
        f = np.ascontiguousarray(faces, np.uint32).reshape(-1, 3)
        self._h = L.ref_tree_create(_p(v), ctypes.c_int(v.shape[0]), _p(f), ctypes.c_int(f.shape[0]))

    @classmethod
    def from_kd(cls, verts, faces, kd):
        """The reference's RKDTreeCPU holding the SAH tree `kd` (a KdbTree)
        as its own KDNodeCPU objects instead of the one leaf its builder
        makes; queries run the reference's compiled code unchanged."""
        self = cls.__new__(cls)
        L = ref_lib()
        if L is None:
            raise FileNotFoundError(REF_LIB_PATH)
        L.ref_tree_from_kd.restype = ctypes.c_void_p
        L.ref_tree_from_kd.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p]
        L.ref_tree_destroy.argtypes = [ctypes.c_void_p]
        L.ref_tree_trace.restype = ctypes.c_int64
        L.ref_tree_trace.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        L.ref_max_threads.restype = ctypes.c_int
        self._L = L
        v = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
        f = np.ascontiguousarray(faces, np.uint32).reshape(-1, 3)
        bmin = np.asarray(kd.bmin, np.float32)
        bmax = np.asarray(kd.bmax, np.float32)
        self._h = L.ref_tree_from_kd(_p(v), ctypes.c_int(v.shape[0]), _p(f), ctypes.c_int(f.shape[0]),
                                     _p(kd.nodes), _p(kd.index), _p(bmin), _p(bmax))
        return self

    def threads(self) -> int:
        return int(self._L.ref_max_threads())

    def trace(self, o, d, nthreads=0):
        """Closest hits of rays (o, d): (t (inf-like 1e20 where none), normals, hit count)."""
        o = np.asarray(o, np.float32).reshape(-1, 3)
        d = np.asarray(d, np.float32).reshape(-1, 3)
        rays = np.ascontiguousarray(np.concatenate([o, d], 1), np.float32)
        n = rays.shape[0]
        t = np.empty(n, np.float32)
        nrm = np.empty((n, 3), np.float32)
        hits = self._L.ref_tree_trace(self._h, _p(rays), ctypes.c_int64(n), _p(t), _p(nrm),
                                      ctypes.c_int(nthreads))
        return t, nrm, int(hits)

    def close(self):
        if self._h:
            self._L.ref_tree_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


KDB_NODE = np.dtype([("axis", "<i4"), ("split", "<f4"), ("left", "<i4"), ("right", "<i4"),
                     ("first", "<i4"), ("count", "<i4")])


class _OKdbTree(ctypes.Structure):
    _fields_ = [("nodes", ctypes.c_void_p), ("n_nodes", ctypes.c_int32),
                ("index", ctypes.c_void_p), ("n_index", ctypes.c_int64),
                ("bmin", ctypes.c_float * 3), ("bmax", ctypes.c_float * 3)]


class KdbTree:
    """The checker's binned-SAH kd-tree (oracle_kdbuild.c): pre-order nodes
    (KDB_NODE), the leaves' triangle lists and the root box."""

    def __init__(self, nodes, index, bmin, bmax):
        self.nodes, self.index, self.bmin, self.bmax = nodes, index, bmin, bmax

    def depth(self) -> int:
        d = np.zeros(len(self.nodes), np.int32)
        for i, n in enumerate(self.nodes):
            if n["axis"] != 3:
                d[n["left"]] = d[n["right"]] = d[i] + 1
        return int(d.max())


def kdb_build(verts, faces, max_depth=24, leaf_size=8, ci=2.0, ct=1.0, empty_bonus=0.15):
    """SAH kd-tree over an indexed mesh (the reference arm's configured tree)."""
    L = lib()
    L.o_kdb_build.restype = ctypes.c_int
    v = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
    f = np.ascontiguousarray(faces, np.uint32).reshape(-1, 3)
    t = _OKdbTree()
    rc = L.o_kdb_build(_p(v), ctypes.c_int32(v.shape[0]), _p(f), ctypes.c_int32(f.shape[0]),
                       ctypes.c_int(max_depth), ctypes.c_int(leaf_size), ctypes.c_float(ci),
                       ctypes.c_float(ct), ctypes.c_float(empty_bonus), ctypes.byref(t))
    if rc != 0:
        raise MemoryError("o_kdb_build failed")
    try:
        nodes = np.ctypeslib.as_array(ctypes.cast(t.nodes, ctypes.POINTER(ctypes.c_int32)),
                                      (t.n_nodes * 6,)).copy().view(KDB_NODE)
        index = np.ctypeslib.as_array(ctypes.cast(t.index, ctypes.POINTER(ctypes.c_int32)),
                                      (int(t.n_index),)).copy() if t.n_index else np.zeros(0, np.int32)
        bmin, bmax = list(t.bmin), list(t.bmax)
    finally:
        L.o_kdb_free(ctypes.byref(t))
    return KdbTree(nodes, index, bmin, bmax)


def ref_perm(seed: int) -> np.ndarray:
    L = ref_lib()
    if L is None:
        raise FileNotFoundError(REF_LIB_PATH)
    out = np.zeros(512, np.uint32)
    L.ref_perlin_permutation(ctypes.c_uint32(seed), _p(out))
    return out


def ref_node_fields(raw: np.ndarray) -> dict:
    """Decode one 128-byte RKDTreeNodeGPU (KDTreeGPUUtills.h:34-46, x86-64
    layout: box 24 B, axis i32, split f32, 5 x size_t, bool, 6 x size_t)."""
    b = raw.tobytes()
    box = np.frombuffer(b[0:24], np.float32)
    axis = int(np.frombuffer(b[24:28], np.int32)[0])
    split = float(np.frombuffer(b[28:32], np.float32)[0])
    left, right, first, num, nnodes = np.frombuffer(b[32:72], np.uint64)
    is_leaf = bool(b[72])
    ropes = np.frombuffer(b[80:128], np.int64)
    return {"min": box[:3].copy(), "max": box[3:].copy(), "axis": axis, "split": split,
            "left": int(left), "right": int(right), "first": int(first), "num_objs": int(num),
            "is_leaf": is_leaf, "ropes": ropes.copy()}


def frame_ao_bruteforce(packed, bmin, bmax, cam, w, h, light_dir, ao_length, bias, seed, pixels,
                        nthreads=0, return_results=False):
    """Reference-as-shipped AO frame on a pixel sample; returns rays traced."""
    packed = np.ascontiguousarray(packed, np.float32)
    pix = np.ascontiguousarray(pixels, np.uint32)
    n = pix.shape[0]
    out = np.zeros(n, HIT_DTYPE)
    mask = np.zeros(n, np.uint32)
    nsec = ctypes.c_uint32(0)
    oc = camera(cam)
    b0 = (ctypes.c_float * 3)(*[float(x) for x in bmin])
    b1 = (ctypes.c_float * 3)(*[float(x) for x in bmax])
    ld = (ctypes.c_float * 3)(*light_dir)
    lib().o_batch_frame_ao_bruteforce(_p(packed), ctypes.c_int32(packed.shape[0]), b0, b1,
                                      ctypes.byref(oc), ctypes.c_uint32(w), ctypes.c_uint32(h), ld,
                                      ctypes.c_float(ao_length), ctypes.c_float(bias),
                                      ctypes.c_uint32(seed), _p(pix), ctypes.c_int64(n), _p(out),
                                      _p(mask), ctypes.byref(nsec), ctypes.c_int(nthreads))
    if return_results:
        return out, mask, nsec.value
    return n + nsec.value


def sdf_arbiter(p, cam, w, h, pixels, octaves=8, scale=0.25, amp=3.0, factor=0.6, tmax=200.0,
              max_steps=4096, refine=True, nthreads=0):
    """FP64 surface points of the given pixels' rays: (n, 3) positions and a hit mask.

    The FP64 march takes the float tracer's steps (t += factor * density); with
    `refine` the first crossing it reaches is bisected to the density's root."""
    pix = np.ascontiguousarray(pixels, np.uint32)
    out = np.zeros((pix.shape[0], 4), np.float64)
    oc = camera(cam)
    lib().o_batch_sdf_arbiter(_p(p), ctypes.byref(oc), ctypes.c_uint32(w), ctypes.c_uint32(h),
                            ctypes.c_int(octaves), ctypes.c_double(scale), ctypes.c_double(amp),
                            ctypes.c_double(factor), ctypes.c_double(tmax), ctypes.c_int(max_steps),
                            ctypes.c_int(1 if refine else 0), _p(pix), ctypes.c_int64(pix.shape[0]), _p(out), ctypes.c_int(nthreads))
    return out[:, :3], out[:, 3] > 0.5


class OSdfField(ctypes.Structure):
    _fields_ = [("octaves", ctypes.c_uint32), ("scale", ctypes.c_float), ("amp", ctypes.c_float),
                ("step_factor", ctypes.c_float), ("eps", ctypes.c_float),
                ("tmax", ctypes.c_float), ("max_steps", ctypes.c_uint32)]


def sdf_frame(p, cam, w, h, field, shade, pixels=None, nthreads=0, evals=False):
    """Oracle RGBA8 values (uint32) of the shaded terrain frame on `pixels`
    (all pixels when None).  field: product re_sdf_params; shade: product
    re_sdf_shade_params (the same bytes as o_sdf_shade)."""
    pix = None if pixels is None else np.ascontiguousarray(pixels, np.uint32)
    n = w * h if pix is None else pix.shape[0]
    out = np.zeros(n, np.uint32)
    ev = np.zeros(n, np.uint32) if evals else None
    f = OSdfField(field.octaves, field.scale, field.amplitude, field.step_factor, field.eps,
                  field.tmax, field.max_steps)
    oc = camera(cam)
    lib().o_batch_sdf_frame(_p(p), ctypes.byref(oc), ctypes.c_uint32(w), ctypes.c_uint32(h),
                            ctypes.byref(f), ctypes.byref(shade), _p(pix), ctypes.c_int64(n),
                            _p(out), _p(ev), ctypes.c_int(nthreads))
    return (out, ev) if evals else out


def fmath(fn, x, y=None):
    """The oracle's elementary functions (0: e^x, 1: ln x, 2: x^y) over float32 arrays."""
    x = np.ascontiguousarray(x, np.float32)
    yy = None if y is None else np.ascontiguousarray(y, np.float32)
    out = np.zeros_like(x)
    lib().o_batch_fmath(ctypes.c_uint32(fn), _p(x), _p(yy), ctypes.c_int64(x.size), _p(out))
    return out


def hit_errors(sdf_out, arbiter_pos, arbiter_hit, pixels):
    """Per-pixel |p_gpu - p_fp64| where both hit, plus hit/miss disagreements."""
    o = np.asarray(sdf_out)
    f = o.view(np.float32).reshape(-1, 8)[pixels]
    status = o.view(np.uint32).reshape(-1, 8)[pixels, 7]
    gpu_hit = status == 1
    both = gpu_hit & arbiter_hit
    err = np.linalg.norm(f[both, 0:3].astype(np.float64) - arbiter_pos[both], axis=1)
    return err, int((gpu_hit != arbiter_hit).sum()), int(both.sum())


def density_d(p, pts, octaves=8, scale=0.25, amp=3.0, nthreads=0):
    """FP64 terrain density p.y - amp * fbm(scale * p) (the arbiter's field)."""
    pts = np.ascontiguousarray(pts, np.float64)
    out = np.zeros(pts.shape[0], np.float64)
    lib().o_batch_density_d(_p(p), _p(pts), ctypes.c_int64(pts.shape[0]), ctypes.c_int(octaves),
                            ctypes.c_double(scale), ctypes.c_double(amp), _p(out),
                            ctypes.c_int(nthreads))
    return out


class OPathScene(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_uint32), ("tris", ctypes.c_void_p), ("ntris", ctypes.c_int32),
                ("bmin", ctypes.c_float * 3), ("bmax", ctypes.c_float * 3),
                ("perm", ctypes.c_void_p), ("octaves", ctypes.c_int),
                ("scale", ctypes.c_float), ("amp", ctypes.c_float),
                ("step_factor", ctypes.c_float), ("eps", ctypes.c_float),
                ("tmax", ctypes.c_float), ("max_steps", ctypes.c_uint32),
                ("cam", OCamera), ("w", ctypes.c_uint32), ("h", ctypes.c_uint32),
                ("albedo", ctypes.c_float)]


def batch_path(scenes, offsets, gpix, depth, seed, mesh_bias, nthreads=0):
    """Oracle radiance, primary hits and rays per path of the batched path tracer.

    scenes: dicts with kind 0 {tris (n,12) float32 in id order, bmin, bmax}
    or kind 1 {seed, octaves, scale, amp, step_factor, eps, tmax, max_steps},
    plus cam (product re_camera), w, h, albedo."""
    keep = []
    arr = (OPathScene * len(scenes))()
    for i, s in enumerate(scenes):
        o = arr[i]
        o.kind = s["kind"]
        if s["kind"] == 0:
            tris = np.ascontiguousarray(s["tris"], np.float32)
            keep.append(tris)
            o.tris, o.ntris = tris.ctypes.data, tris.shape[0]
            o.bmin[:] = [float(x) for x in s["bmin"]]
            o.bmax[:] = [float(x) for x in s["bmax"]]
        else:
            P = np.ascontiguousarray(perm(s["seed"]), np.uint32)
            keep.append(P)
            o.perm = P.ctypes.data
            o.octaves, o.scale, o.amp = s["octaves"], s["scale"], s["amp"]
            o.step_factor, o.eps, o.tmax, o.max_steps = (s["step_factor"], s["eps"], s["tmax"],
                                                         s["max_steps"])
        o.cam = camera(s["cam"])
        o.w, o.h, o.albedo = s["w"], s["h"], s["albedo"]
    offs = np.ascontiguousarray(offsets, np.uint64)
    g = np.ascontiguousarray(gpix, np.uint32)
    rad = np.zeros(g.shape[0], np.float32)
    prim = np.zeros((g.shape[0], 4), np.int32)
    nrays = np.zeros(g.shape[0], np.uint32)
    lib().o_batch_path(arr, ctypes.c_int(len(scenes)), _p(offs), _p(g), ctypes.c_int64(g.shape[0]),
                       ctypes.c_uint32(depth), ctypes.c_uint32(seed), ctypes.c_float(mesh_bias),
                       _p(rad), _p(prim), _p(nrays), ctypes.c_int(nthreads))
    return rad, prim, nrays


def frame_rgba(packed, bmin, bmax, cam, w, h, lights, albedo, zenith, horizon, mode=0,
               pixels=None, nthreads=0):
    """Packed RGBA8 of the shaded frame. lights: list of (pos xyz, intensity)."""
    tris = np.ascontiguousarray(packed, np.float32)
    lp = np.ascontiguousarray([l[0] for l in lights], np.float32).reshape(-1)
    li = np.ascontiguousarray([l[1] for l in lights], np.float32)
    f3 = lambda v: np.ascontiguousarray(v, np.float32)
    bmin, bmax, albedo, zenith, horizon = map(f3, (bmin, bmax, albedo, zenith, horizon))
    pix = None if pixels is None else np.ascontiguousarray(pixels, np.uint32)
    n = w * h if pix is None else pix.shape[0]
    out = np.zeros(n, np.uint32)
    oc = camera(cam)
    lib().o_batch_frame(_p(tris), ctypes.c_int32(tris.shape[0]), _p(bmin), _p(bmax),
                        ctypes.byref(oc), ctypes.c_uint32(w), ctypes.c_uint32(h), ctypes.c_int(mode),
                        _p(lp) if len(lights) else None, _p(li) if len(lights) else None,
                        ctypes.c_uint32(len(lights)), _p(albedo), _p(zenith), _p(horizon),
                        _p(pix), ctypes.c_int64(n), _p(out), ctypes.c_int(nthreads))
    return out


def ref_ply_lib():
    """oracle/_ref/libre_ply.so (the reference's rply + loader shim) or None."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref", "libre_ply.so")
    if not os.path.exists(path):
        return None
    lib_ = ctypes.CDLL(path)
    lib_.ref_ply_load.restype = ctypes.c_int
    lib_.ref_ply_load.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p),
                                  ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_void_p),
                                  ctypes.POINTER(ctypes.c_long)]
    lib_.ref_ply_free.argtypes = [ctypes.c_void_p]
    return lib_


def ref_ply_load(path):
    """(ok, vertices (V,3) float32, faces (F,3) uint32) read the reference's way."""
    lib_ = ref_ply_lib()
    v, f = ctypes.c_void_p(), ctypes.c_void_p()
    nv, nf = ctypes.c_long(), ctypes.c_long()
    ok = lib_.ref_ply_load(str(path).encode(), ctypes.byref(v), ctypes.byref(nv), ctypes.byref(f),
                           ctypes.byref(nf))
    verts = np.ctypeslib.as_array((ctypes.c_float * (3 * nv.value)).from_address(v.value)).copy() \
        if nv.value else np.zeros(0, np.float32)
    faces = np.ctypeslib.as_array((ctypes.c_uint32 * (3 * nf.value)).from_address(f.value)).copy() \
        if nf.value else np.zeros(0, np.uint32)
    lib_.ref_ply_free(v)
    lib_.ref_ply_free(f)
    return bool(ok), verts.reshape(-1, 3), faces.reshape(-1, 3)


class OVoxel(ctypes.Structure):
    _fields_ = [("v", ctypes.c_void_p), ("dim", ctypes.c_int * 3), ("spacing", ctypes.c_float * 3),
                ("origin", ctypes.c_float * 3)]


def _ovoxel(grid, dim, spacing, origin):
    g = OVoxel()
    g.v = grid.ctypes.data
    g.dim[:] = [int(x) for x in dim]
    g.spacing[:] = [float(x) for x in spacing]
    g.origin[:] = [float(x) for x in origin]
    return g


def voxel_bake(p, octaves, scale, amp, dim, spacing, origin, nthreads=0):
    """(2 * voxels) float32: FP32 density at the grid points, material 0."""
    n = int(dim[0]) * int(dim[1]) * int(dim[2])
    out = np.zeros(2 * n, np.float32)
    d = np.ascontiguousarray(dim, np.int32)
    s = np.ascontiguousarray(spacing, np.float32)
    o = np.ascontiguousarray(origin, np.float32)
    lib().o_batch_voxel_bake(_p(p), ctypes.c_int(octaves), ctypes.c_float(scale),
                             ctypes.c_float(amp), _p(d), _p(s), _p(o), _p(out),
                             ctypes.c_int(nthreads))
    return out


def voxel_sample(grid, dim, spacing, origin, quality, pts, nthreads=0):
    grid = np.ascontiguousarray(grid, np.float32)
    pts = np.ascontiguousarray(pts, np.float32)
    out = np.zeros(pts.shape[0], np.float32)
    g = _ovoxel(grid, dim, spacing, origin)
    lib().o_batch_voxel_sample(ctypes.byref(g), ctypes.c_uint32(quality), _p(pts),
                               ctypes.c_int64(pts.shape[0]), _p(out), ctypes.c_int(nthreads))
    return out


def voxel_trace(grid, dim, spacing, origin, quality, step_factor, eps, tmax, max_steps, cam, w,
                h, pixels=None, nthreads=0):
    """Records like sdf_image: pos, normal, steps, status."""
    grid = np.ascontiguousarray(grid, np.float32)
    g = _ovoxel(grid, dim, spacing, origin)
    pix = None if pixels is None else np.ascontiguousarray(pixels, np.uint32)
    n = w * h if pix is None else pix.shape[0]
    out = np.zeros(n, SDF_DTYPE)
    oc = camera(cam)
    lib().o_batch_voxel_trace(ctypes.byref(g), ctypes.c_uint32(quality), ctypes.c_float(step_factor),
                              ctypes.c_float(eps), ctypes.c_float(tmax), ctypes.c_uint32(max_steps),
                              ctypes.byref(oc), ctypes.c_uint32(w), ctypes.c_uint32(h), _p(pix),
                              ctypes.c_int64(n), _p(out), ctypes.c_int(nthreads))
    return out


def trace_instances(instances, cam, w, h, mode=0, nthreads=0):
    """instances: [(packed (n,12), bmin, bmax, (cos, sin), location)] ->
    (hits HIT_DTYPE (w*h,), instance index (w*h,))."""
    n = len(instances)
    keep = [np.ascontiguousarray(x[0], np.float32) for x in instances]
    ptrs = (ctypes.c_void_p * n)(*[k.ctypes.data for k in keep])
    nt = np.array([k.shape[0] for k in keep], np.int32)
    bmin = np.ascontiguousarray([x[1] for x in instances], np.float32)
    bmax = np.ascontiguousarray([x[2] for x in instances], np.float32)
    cs = np.ascontiguousarray([x[3] for x in instances], np.float32)
    loc = np.ascontiguousarray([x[4] for x in instances], np.float32)
    out = np.zeros(w * h, HIT_DTYPE)
    inst = np.zeros(w * h, np.int32)
    oc = camera(cam)
    lib().o_batch_instances(ptrs, _p(nt), _p(bmin), _p(bmax), _p(cs), _p(loc), ctypes.c_int32(n),
                            ctypes.byref(oc), ctypes.c_uint32(w), ctypes.c_uint32(h),
                            ctypes.c_int(mode), _p(out), _p(inst), ctypes.c_int(nthreads))
    return out, inst


def voxel_brush(grid, dim, spacing, origin, kind, center, extent, material=0.0, smooth=0.1):
    g = np.ascontiguousarray(grid, np.float32).copy()
    d = np.ascontiguousarray(dim, np.int32)
    s = np.ascontiguousarray(spacing, np.float32)
    o = np.ascontiguousarray(origin, np.float32)
    c = np.ascontiguousarray(center, np.float32)
    e = np.ascontiguousarray(extent if hasattr(extent, "__len__") else [extent] * 3, np.float32)
    lib().o_voxel_brush(_p(g), _p(d), _p(s), _p(o), ctypes.c_uint32(kind), _p(c), _p(e),
                        ctypes.c_float(material), ctypes.c_float(smooth))
    return g

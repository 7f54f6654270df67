"""libsvo_b200 -- B200-native treelet ray cast behind the libsvo C ABI.

Python mirror of the reference's host interface for the ray-cast path:
``TreeletMemoryManagerCuda`` keeps the method names of
``TreeletMemoryManager`` / ``TreeletMemoryManagerCl`` (src/TreeletMemoryManager.h,
src/TreeletMemoryManagerCl.h), ``render`` is the renderToBuffer launch.  All
work is done by ``_lib/libsvo_b200.so`` (C ABI in include/libsvo_b200.h);
importing this package fails loudly when that library is missing.
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
# LIBSVO_B200_LIB selects another build of the same library (same C ABI)
LIB_PATH = Path(os.environ.get("LIBSVO_B200_LIB", str(_PKG / "_lib" / "libsvo_b200.so")))

if not LIB_PATH.is_file():
    raise ImportError(
        f"libsvo_b200: native library {LIB_PATH} is missing; build it with "
        "`python -c 'import __graft_entry__ as g; g.build()'` (or python libsvo_b200/_build.py)")

_L = ctypes.CDLL(str(LIB_PATH))

# ---- status codes ----------------------------------------------------------
SVO_OK = 0
SVO_ERR_NOENT = -2
SVO_ERR_IO = -5
SVO_ERR_NOMEM = -12
SVO_ERR_BUSY = -16
SVO_ERR_INVALID = -22
SVO_ERR_RANGE = -34
SVO_ERR_NOTSUP = -95
SVO_ERR_TIMEOUT = -110
SVO_ERR_CANCELED = -125
SVO_ERR_CUDA = -1000

_ERR_NAMES = {v: k for k, v in dict(globals()).items() if k.startswith("SVO_ERR_")}

UPLOAD_COALESCED = 0
UPLOAD_PACKED = 1
UPLOAD_PINNED = 2
TRAVERSAL_TREELET = 0
TRAVERSAL_FLAT = 1
HITFLAG_CAPPED = 1
HITFLAG_BOUNDS = 2
HITFLAG_BOXMISS = 4

HIT_DTYPE = np.dtype(
    [("node", "<u4"), ("t", "<f4"), ("depth", "<u2"), ("hit", "u1"), ("flags", "u1"), ("loops", "<u2"),
     ("fetches", "<u2")]
)


class SvoError(RuntimeError):
    def __init__(self, code: int, what: str):
        self.code = code
        msg = f"{what}: {_ERR_NAMES.get(code, code)}"
        if code == SVO_ERR_CUDA:
            msg += f" ({_L.svo_last_error().decode()})"
        super().__init__(msg)


def _check(code: int, what: str) -> int:
    if code != SVO_OK:
        raise SvoError(code, what)
    return code


# ---- C structs -------------------------------------------------------------
class svo_frame_params(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32),
                ("t_scale_ratio", ctypes.c_float), ("mode", ctypes.c_int32),
                ("pixel_far_h", ctypes.c_float * 4), ("pixel_far_v", ctypes.c_float * 4),
                ("far_lower_left", ctypes.c_float * 4), ("camera_position", ctypes.c_float * 4)]


class svo_trace_cfg(ctypes.Structure):
    _fields_ = [("traversal", ctypes.c_int32), ("stack_size", ctypes.c_int32)]


class svo_stats(ctypes.Structure):
    _fields_ = [("capped_rays", ctypes.c_uint32), ("bounds_errors", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32 * 2)]


class svo_scene_info(ctypes.Structure):
    _fields_ = [("num_treelets", ctypes.c_uint32), ("treelet_bytes", ctypes.c_uint32),
                ("nodes_per_treelet", ctypes.c_uint32), ("max_depth", ctypes.c_uint32),
                ("total_nodes", ctypes.c_uint64), ("leaf_voxels", ctypes.c_uint64)]


class svo_mm_info(ctypes.Structure):
    _fields_ = [("num_treelets", ctypes.c_uint32), ("treelet_bytes", ctypes.c_uint32),
                ("nodes_per_treelet", ctypes.c_uint32), ("num_slots", ctypes.c_uint32),
                ("free_slots", ctypes.c_uint32), ("slots_to_upload", ctypes.c_uint32),
                ("incore_nodes", ctypes.c_uint64), ("device_bytes", ctypes.c_uint64)]


class svo_slot_info(ctypes.Structure):
    _fields_ = [("treelet_gid", ctypes.c_int32), ("visibility", ctypes.c_int32),
                ("error", ctypes.c_float)]


class svo_octree_desc(ctypes.Structure):
    _fields_ = [("d_nodes", ctypes.c_void_p), ("d_attribs", ctypes.c_void_p),
                ("num_nodes", ctypes.c_uint64), ("traversal", ctypes.c_int32),
                ("stack_size", ctypes.c_int32)]


class svo_view_desc(ctypes.Structure):
    _fields_ = [("params", svo_frame_params), ("octree", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32), ("d_rgba", ctypes.c_void_p), ("d_hits", ctypes.c_void_p)]


class svo_batch_cfg(ctypes.Structure):
    _fields_ = [("tile_w", ctypes.c_uint32), ("tile_h", ctypes.c_uint32),
                ("block_threads", ctypes.c_uint32), ("blocks_per_sm", ctypes.c_uint32),
                ("top_nodes", ctypes.c_uint32), ("use_graph", ctypes.c_uint32),
                ("rays_per_lane", ctypes.c_uint32)]


class svo_shadow_cfg(ctypes.Structure):
    _fields_ = [("light_direction", ctypes.c_float * 3), ("t_scale_ratio", ctypes.c_float),
                ("normal_offset", ctypes.c_float), ("reserved", ctypes.c_uint32)]


assert ctypes.sizeof(svo_frame_params) == 80
assert ctypes.sizeof(svo_view_desc) == 104
assert ctypes.sizeof(svo_shadow_cfg) == 24

_vp, _u32, _u64, _i32, _f32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int32, ctypes.c_float
_P = ctypes.POINTER

_SIGS = {
    "svo_version": ([], ctypes.c_char_p),
    "svo_last_error": ([], ctypes.c_char_p),
    "svo_scene_build_menger": ([_u32, _u32, _u64, _u32, _u32, _P(_vp)], ctypes.c_int),
    "svo_scene_build_mesh": ([_vp, _u64, _vp, _u64, _u32, _u32, _u32, _i32, _P(_vp)], ctypes.c_int),
    "svo_mesh_icosphere_size": ([_u32, _P(_u64), _P(_u64)], ctypes.c_int),
    "svo_mesh_icosphere": ([_u32, _f32, _u32, _f32, _f32, _u64, _vp, _vp], ctypes.c_int),
    "svo_mesh_terrain_size": ([_u32, _P(_u64), _P(_u64)], ctypes.c_int),
    "svo_mesh_terrain": ([_u32, _u32, _f32, _f32, _f32, _u64, _vp, _vp], ctypes.c_int),
    "svo_scene_write": ([_vp, ctypes.c_char_p], ctypes.c_int),
    "svo_scene_read": ([ctypes.c_char_p, _P(_vp)], ctypes.c_int),
    "svo_scene_info_get": ([_vp, _P(svo_scene_info)], ctypes.c_int),
    "svo_scene_treelet": ([_vp, _u32, _P(_u32), _P(_u32), _P(_i32), _P(_i32), _P(_i32), _P(_i32)], ctypes.c_int),
    "svo_scene_flatten": ([_vp, _vp, _vp, _u64, _P(_u64)], ctypes.c_int),
    "svo_scene_destroy": ([_vp], None),
    "svo_mm_create": ([ctypes.c_char_p, _u64, _vp, _P(_vp)], ctypes.c_int),
    "svo_mm_create_from_scene": ([_vp, _u64, _vp, _P(_vp)], ctypes.c_int),
    "svo_mm_destroy": ([_vp], None),
    "svo_mm_init_device_buffer": ([_vp], ctypes.c_int),
    "svo_mm_get_device_buffers": ([_vp, _P(_vp), _P(_vp), _P(_u64)], ctypes.c_int),
    "svo_mm_insert_treelet": ([_vp, _i32, _i32, _f32], ctypes.c_int),
    "svo_mm_remove_treelet": ([_vp, _i32], ctypes.c_int),
    "svo_mm_free_incore_position": ([_vp], ctypes.c_int),
    "svo_mm_update_client_side": ([_vp, _vp, _vp, _u32, _vp, _u32], ctypes.c_int),
    "svo_mm_update_device_memory": ([_vp, _P(_u32)], ctypes.c_int),
    "svo_mm_plan_uploads": ([_vp, _vp, _vp, _u32, _P(_u32)], ctypes.c_int),
    "svo_mm_reset": ([_vp], ctypes.c_int),
    "svo_mm_insert_all": ([_vp, _P(_u32)], ctypes.c_int),
    "svo_mm_info_get": ([_vp, _P(svo_mm_info)], ctypes.c_int),
    "svo_mm_get_slot": ([_vp, _u32, _P(svo_slot_info)], ctypes.c_int),
    "svo_mm_treelet_slot": ([_vp, _i32, _P(_i32)], ctypes.c_int),
    "svo_mm_copy_incore": ([_vp, _u64, _u64, _vp, _vp], ctypes.c_int),
    "svo_mm_slots_to_upload": ([_vp, _vp, _u32, _P(_u32)], ctypes.c_int),
    "svo_render": ([_vp, _vp, _u64, _P(svo_frame_params), _P(svo_trace_cfg), _vp, _vp, _vp, _vp], ctypes.c_int),
    "svo_trace_rays": ([_vp, _u64, _vp, _vp, _u64, _f32, _P(svo_trace_cfg), _vp, _vp, _vp], ctypes.c_int),
    "svo_mm_render": ([_vp, _P(svo_frame_params), _P(svo_trace_cfg), _vp, _vp, _vp], ctypes.c_int),
    "svo_mm_render_host": ([_vp, _P(svo_frame_params), _P(svo_trace_cfg), _vp, _vp], ctypes.c_int),
    "svo_mm_sync": ([_vp, _vp, _P(svo_stats)], ctypes.c_int),
    "svo_mm_render_host_async": ([_vp, _P(svo_frame_params), _P(svo_trace_cfg), _vp, _vp], ctypes.c_int),
    "svo_mm_render_shadow_host_async": ([_vp, _P(svo_frame_params), _P(svo_trace_cfg), _P(svo_shadow_cfg), _vp,
                                         _vp], ctypes.c_int),
    "svo_mm_set_upload_policy": ([_vp, _i32], ctypes.c_int),
    "svo_mm_set_upload_ratio": ([_vp, _f32], ctypes.c_int),
    "svo_render_shadow": ([_vp, _vp, _u64, _P(svo_frame_params), _P(svo_trace_cfg), _P(svo_shadow_cfg), _vp, _vp,
                           _vp, _vp, _vp], ctypes.c_int),
    "svo_mm_render_shadow": ([_vp, _P(svo_frame_params), _P(svo_trace_cfg), _P(svo_shadow_cfg), _vp, _vp, _vp,
                              _vp], ctypes.c_int),
    "svo_batcher_create": ([_u32, _u32, _P(_vp)], ctypes.c_int),
    "svo_batcher_destroy": ([_vp], None),
    "svo_batcher_set": ([_vp, _P(svo_octree_desc), _u32, _P(svo_view_desc), _u32, _P(svo_batch_cfg), _vp],
                        ctypes.c_int),
    "svo_batcher_launch": ([_vp, _vp, _vp], ctypes.c_int),
    "svo_batcher_autotune": ([_vp, _u32, _vp, _P(svo_batch_cfg), _P(_f32)], ctypes.c_int),
    "svo_batcher_size": ([_vp, _P(_u64), _P(_u64)], ctypes.c_int),
    "svo_device_scene_build_mesh": ([_vp, _u64, _vp, _u64, _u32, _u32, _vp, _P(_vp)], ctypes.c_int),
    "svo_device_scene_build_mesh_attributed": ([_vp, _vp, _vp, _u64, _vp, _u64, _u32, _u32, _vp, _P(_vp)],
                                               ctypes.c_int),
    "svo_scene_build_mesh_attributed": ([_vp, _vp, _vp, _u64, _vp, _u64, _u32, _u32, _u32, _i32, _P(_vp)],
                                        ctypes.c_int),
    "svo_mesh_vertex_attributes": ([_vp, _u64, _vp, _u64, _u64, _vp, _vp], ctypes.c_int),
    "svo_mesh_load_ply": ([ctypes.c_char_p, _P(_vp)], ctypes.c_int),
    "svo_mesh_info": ([_vp, _P(_u64), _P(_u64), _P(_u32)], ctypes.c_int),
    "svo_mesh_copy": ([_vp, _vp, _vp, _vp, _vp], ctypes.c_int),
    "svo_mesh_destroy": ([_vp], None),
    "svo_mesh_fit_unit_cube": ([_vp, _vp, _u64, _f32], ctypes.c_int),
    "svo_device_scene_info_get": ([_vp, _P(svo_scene_info)], ctypes.c_int),
    "svo_device_scene_buffers": ([_vp, _P(_vp), _P(_vp), _P(_u64)], ctypes.c_int),
    "svo_device_scene_copy": ([_vp, _u64, _u64, _vp, _vp], ctypes.c_int),
    "svo_device_scene_counts": ([_vp, _P(_u64), _P(_u64)], ctypes.c_int),
    "svo_device_scene_destroy": ([_vp], None),
    "svo_render_batch_static": ([_P(svo_octree_desc), _u32, _P(svo_view_desc), _u32, _u32, _u32, _vp, _vp],
                                ctypes.c_int),
}
for _name, (_args, _res) in _SIGS.items():
    _fn = getattr(_L, _name)
    _fn.argtypes = _args
    _fn.restype = _res

lib = _L


def version() -> str:
    return _L.svo_version().decode()


def _np_ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _dptr(t) -> int | None:
    """Device pointer of a torch tensor (or an int address, or None)."""
    if t is None:
        return None
    if isinstance(t, int):
        return t
    return t.data_ptr()


def _stream_ptr(stream) -> int | None:
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


# ---- cameras ---------------------------------------------------------------
@dataclass
class Camera:
    """Pinhole camera producing renderToBuffer's frustum arguments
    (raycast_serialized_opencl.cpp:670-675, 729-733) and the LOD ratio
    tScaleRatio = tan(fov/2) * aspect / (W/2) (:303-304).  ``fov_deg`` is the
    vertical field of view."""

    eye: tuple
    target: tuple
    width: int
    height: int
    fov_deg: float = 60.0
    up: tuple = (0.0, 1.0, 0.0)
    far: float = 20.0

    def frame_params(self, mode: int = 0, t_scale_ratio: float | None = None) -> svo_frame_params:
        eye = np.asarray(self.eye, dtype=np.float64)
        fwd = np.asarray(self.target, dtype=np.float64) - eye
        fwd /= np.linalg.norm(fwd)
        up = np.asarray(self.up, dtype=np.float64)
        right = np.cross(fwd, up)
        if np.linalg.norm(right) < 1e-9:
            right = np.cross(fwd, np.array([1.0, 0.0, 0.0]))
        right /= np.linalg.norm(right)
        true_up = np.cross(right, fwd)
        aspect = self.width / self.height
        half_h = self.far * math.tan(math.radians(self.fov_deg) / 2.0)
        half_w = half_h * aspect
        center = eye + fwd * self.far
        fll = center - right * half_w - true_up * half_h
        flr = center + right * half_w - true_up * half_h
        ful = center - right * half_w + true_up * half_h
        h = (flr - fll) / self.width
        v = (ful - fll) / self.height
        if t_scale_ratio is None:
            t_scale_ratio = math.tan(math.radians(self.fov_deg) / 2.0) * aspect / (self.width * 0.5)
        p = svo_frame_params()
        p.width, p.height = int(self.width), int(self.height)
        p.t_scale_ratio = float(np.float32(t_scale_ratio))
        p.mode = int(mode)
        for dst, src, w in ((p.pixel_far_h, h, 0.0), (p.pixel_far_v, v, 0.0),
                            (p.far_lower_left, fll, 1.0), (p.camera_position, eye, 1.0)):
            for i in range(3):
                dst[i] = float(np.float32(src[i]))
            dst[3] = w
        return p


def params_bytes(p: svo_frame_params) -> bytes:
    return bytes(p)


def orbit_camera(seed: int, width: int, height: int, radius=(1.5, 2.5), fov_deg=60.0,
                 target=(0.0, 0.0, 0.0)) -> Camera:
    """Camera at a seeded random position on a sphere shell around `target`,
    looking at it."""
    rng = np.random.default_rng(seed)
    v = rng.normal(size=3)
    v /= np.linalg.norm(v)
    r = rng.uniform(*radius) if isinstance(radius, tuple) else float(radius)
    eye = np.asarray(target) + v * r
    up = (0.0, 1.0, 0.0) if abs(v[1]) < 0.95 else (1.0, 0.0, 0.0)
    return Camera(tuple(eye), tuple(target), width, height, fov_deg, up)


def trace_cfg(traversal: int = TRAVERSAL_TREELET, stack_size: int = 13) -> svo_trace_cfg:
    c = svo_trace_cfg()
    c.traversal = traversal
    c.stack_size = stack_size
    return c


# ---- meshes ----------------------------------------------------------------
def icosphere(subdivisions: int, radius=0.4, octaves=3, amplitude=0.05, frequency=2.0, seed=1):
    """(vertices float32 (V,3), triangles uint32 (T,3)) of a noise-displaced icosphere."""
    nv, nt = _u64(), _u64()
    _check(_L.svo_mesh_icosphere_size(subdivisions, ctypes.byref(nv), ctypes.byref(nt)),
           "svo_mesh_icosphere_size")
    v = np.zeros((nv.value, 3), dtype=np.float32)
    t = np.zeros((nt.value, 3), dtype=np.uint32)
    _check(_L.svo_mesh_icosphere(subdivisions, radius, octaves, amplitude, frequency, seed,
                                 _np_ptr(v), _np_ptr(t)), "svo_mesh_icosphere")
    return v, t


def terrain(grid: int, octaves=6, base=-0.45, height=0.3, frequency=2.0, seed=1):
    """(vertices, triangles) of an fBm height field over the unit square."""
    nv, nt = _u64(), _u64()
    _check(_L.svo_mesh_terrain_size(grid, ctypes.byref(nv), ctypes.byref(nt)), "svo_mesh_terrain_size")
    v = np.zeros((nv.value, 3), dtype=np.float32)
    t = np.zeros((nt.value, 3), dtype=np.uint32)
    _check(_L.svo_mesh_terrain(grid, octaves, base, height, frequency, seed, _np_ptr(v), _np_ptr(t)),
           "svo_mesh_terrain")
    return v, t


def vertex_attributes(vertices: np.ndarray, triangles: np.ndarray, seed=1):
    """(normals, colours), float32 (V, 3) each: area-weighted vertex normals
    and a seeded smooth colour field (svo_mesh_vertex_attributes)."""
    v = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 3)
    t = np.ascontiguousarray(triangles, dtype=np.uint32).reshape(-1, 3)
    n = np.zeros_like(v)
    c = np.zeros_like(v)
    _check(_L.svo_mesh_vertex_attributes(_np_ptr(v), v.shape[0], _np_ptr(t), t.shape[0], seed, _np_ptr(n),
                                         _np_ptr(c)), "svo_mesh_vertex_attributes")
    return n, c


def read_ply(path) -> dict:
    """A PLY mesh (the reference octree builder's input): {"vertices",
    "triangles", "normals" or None, "colors" or None}, float32 / uint32."""
    h = ctypes.c_void_p()
    _check(_L.svo_mesh_load_ply(str(path).encode(), ctypes.byref(h)), "svo_mesh_load_ply")
    try:
        nv, nt, fl = _u64(), _u64(), _u32()
        _check(_L.svo_mesh_info(h, ctypes.byref(nv), ctypes.byref(nt), ctypes.byref(fl)), "svo_mesh_info")
        v = np.zeros((nv.value, 3), dtype=np.float32)
        t = np.zeros((nt.value, 3), dtype=np.uint32)
        n = np.zeros_like(v) if fl.value & 1 else None
        c = np.zeros_like(v) if fl.value & 2 else None
        _check(_L.svo_mesh_copy(h, _np_ptr(v), None if n is None else _np_ptr(n), None if c is None else _np_ptr(c),
                                _np_ptr(t)), "svo_mesh_copy")
    finally:
        _L.svo_mesh_destroy(h)
    return {"vertices": v, "triangles": t, "normals": n, "colors": c}


def fit_unit_cube(vertices: np.ndarray, normals: np.ndarray | None = None, rotate_x_deg=0.0):
    """The reference octree builder's placement, in place on float32 copies:
    returns (vertices, normals)."""
    v = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 3).copy()
    n = None if normals is None else np.ascontiguousarray(normals, dtype=np.float32).reshape(-1, 3).copy()
    _check(_L.svo_mesh_fit_unit_cube(_np_ptr(v), None if n is None else _np_ptr(n), v.shape[0], rotate_x_deg),
           "svo_mesh_fit_unit_cube")
    return v, n


def _vertex_arrays(normals, colors, nv):
    if (normals is None) != (colors is None):
        raise ValueError("pass both per-vertex normals and colours, or neither")
    if normals is None:
        return None, None
    n = np.ascontiguousarray(normals, dtype=np.float32).reshape(-1, 3)
    c = np.ascontiguousarray(colors, dtype=np.float32).reshape(-1, 3)
    if n.shape[0] != nv or c.shape[0] != nv:
        raise ValueError("one normal and one colour per vertex")
    return n, c


# ---- scenes ----------------------------------------------------------------
class Scene:
    """An octree cut into treelets (what TreeletBuildManager writes)."""

    def __init__(self, handle):
        self._h = ctypes.c_void_p(handle)

    @classmethod
    def menger(cls, level=5, depth=8, seed=1, treelet_levels=0, treelet_bytes=0) -> "Scene":
        h = ctypes.c_void_p()
        _check(_L.svo_scene_build_menger(level, depth, seed, treelet_levels, treelet_bytes,
                                         ctypes.byref(h)), "svo_scene_build_menger")
        return cls(h.value)

    @classmethod
    def from_mesh(cls, vertices: np.ndarray, triangles: np.ndarray, depth: int,
                  treelet_levels=0, treelet_bytes=0, threads=0, normals: np.ndarray | None = None,
                  colors: np.ndarray | None = None) -> "Scene":
        """Voxelises a mesh.  With per-vertex normals and colours the leaves
        get the reference's interpolated attributes; without, face normals."""
        v = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 3)
        t = np.ascontiguousarray(triangles, dtype=np.uint32).reshape(-1, 3)
        n, c = _vertex_arrays(normals, colors, v.shape[0])
        h = ctypes.c_void_p()
        _check(_L.svo_scene_build_mesh_attributed(
            _np_ptr(v), None if n is None else _np_ptr(n), None if c is None else _np_ptr(c), v.shape[0],
            _np_ptr(t), t.shape[0], depth, treelet_levels, treelet_bytes, threads, ctypes.byref(h)),
            "svo_scene_build_mesh")
        return cls(h.value)

    @classmethod
    def read(cls, path_base: str) -> "Scene":
        h = ctypes.c_void_p()
        _check(_L.svo_scene_read(str(path_base).encode(), ctypes.byref(h)), "svo_scene_read")
        return cls(h.value)

    @classmethod
    def from_pool(cls, nodes: np.ndarray, attribs: np.ndarray, num_slots: int, treelet_bytes: int,
                  max_depth: int, leaf_voxels: int = 0) -> "Scene":
        """A fully resident incore pool (treelet g in slot g, as insertAll
        leaves it) back into its treelets (svo_scene_from_pool)."""
        n = np.ascontiguousarray(nodes, dtype=np.uint32)
        a = np.ascontiguousarray(attribs, dtype=np.uint32)
        h = ctypes.c_void_p()
        _check(_L.svo_scene_from_pool(_np_ptr(n), _np_ptr(a), num_slots, treelet_bytes, max_depth, leaf_voxels,
                                      ctypes.byref(h)), "svo_scene_from_pool")
        return cls(h.value)

    def write(self, path_base: str):
        _check(_L.svo_scene_write(self._h, str(path_base).encode()), "svo_scene_write")

    @property
    def info(self) -> svo_scene_info:
        i = svo_scene_info()
        _check(_L.svo_scene_info_get(self._h, ctypes.byref(i)), "svo_scene_info_get")
        return i

    def treelet(self, gid: int) -> dict:
        vals = [_u32(), _u32(), _i32(), _i32(), _i32(), _i32()]
        _check(_L.svo_scene_treelet(self._h, gid, *[ctypes.byref(x) for x in vals]), "svo_scene_treelet")
        keys = ["num_nodes", "num_leaves", "parent_gid", "parent_leaf_position", "parent_leaf_idx",
                "parent_leaf_parent_position"]
        return {k: v.value for k, v in zip(keys, vals)}

    def flatten(self):
        """Flat breadth-first pool with absolute first-child indices
        (SvoBranch::serializeSvo layout): (nodes, attribs) uint32 (N, 2)."""
        n = _u64()
        _check(_L.svo_scene_flatten(self._h, None, None, 0, ctypes.byref(n)), "svo_scene_flatten")
        nodes = np.zeros((n.value, 2), dtype=np.uint32)
        attribs = np.zeros((n.value, 2), dtype=np.uint32)
        _check(_L.svo_scene_flatten(self._h, _np_ptr(nodes), _np_ptr(attribs), n.value, ctypes.byref(n)),
               "svo_scene_flatten")
        return nodes, attribs

    def close(self):
        if self._h and self._h.value:
            _L.svo_scene_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- memory manager ----------------------------------------------------------
class DeviceScene:
    """A mesh voxelised, built, cut into treelets and made fully resident on
    the GPU (svo_device_scene_build_mesh): the incore pool the host path
    Scene.from_mesh + TreeletMemoryManagerCuda.insertAll + initDeviceBuffer
    produces, without the host holding the octree."""

    def __init__(self, vertices: np.ndarray, triangles: np.ndarray, depth: int, treelet_levels=0,
                 stream=None, normals: np.ndarray | None = None, colors: np.ndarray | None = None):
        v = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 3)
        t = np.ascontiguousarray(triangles, dtype=np.uint32).reshape(-1, 3)
        n, c = _vertex_arrays(normals, colors, v.shape[0])
        h = ctypes.c_void_p()
        _check(_L.svo_device_scene_build_mesh_attributed(
            _np_ptr(v), None if n is None else _np_ptr(n), None if c is None else _np_ptr(c), v.shape[0],
            _np_ptr(t), t.shape[0], depth, treelet_levels, _stream_ptr(stream), ctypes.byref(h)),
            "svo_device_scene_build_mesh")
        self._h = h

    @property
    def info(self) -> svo_scene_info:
        i = svo_scene_info()
        _check(_L.svo_device_scene_info_get(self._h, ctypes.byref(i)), "svo_device_scene_info_get")
        return i

    def buffers(self):
        """(device node pointer, device attribute pointer, pool records)."""
        n, a, c = ctypes.c_void_p(), ctypes.c_void_p(), _u64()
        _check(_L.svo_device_scene_buffers(self._h, ctypes.byref(n), ctypes.byref(a), ctypes.byref(c)),
               "svo_device_scene_buffers")
        return n.value, a.value, c.value

    def counts(self):
        """(octree nodes over all levels, voxel/triangle overlaps)."""
        o, p = _u64(), _u64()
        _check(_L.svo_device_scene_counts(self._h, ctypes.byref(o), ctypes.byref(p)), "svo_device_scene_counts")
        return o.value, p.value

    def getIncoreBuffer(self, first: int = 0, count: int | None = None):
        total = self.buffers()[2]
        count = total - first if count is None else count
        nodes = np.zeros((count, 2), dtype=np.uint32)
        attribs = np.zeros((count, 2), dtype=np.uint32)
        _check(_L.svo_device_scene_copy(self._h, first, count, _np_ptr(nodes), _np_ptr(attribs)),
               "svo_device_scene_copy")
        return nodes, attribs

    def close(self):
        if self._h and self._h.value:
            _L.svo_device_scene_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class TreeletMemoryManagerCuda:
    """TreeletMemoryManager + TreeletMemoryManagerCl with the incore buffer in
    HBM.  Method names follow the reference; insert/remove/free return bool
    like the reference, other failures raise SvoError."""

    MAX_VISIBILITY = 8

    def __init__(self, scene_or_path, incore_bytes: int, stream=None):
        """scene_or_path: a Scene, a DeviceScene (its pool turned back into
        treelets, svo_mm_create_from_device_scene) or a treelet file base."""
        h = ctypes.c_void_p()
        sp = _stream_ptr(stream)
        if isinstance(scene_or_path, Scene):
            _check(_L.svo_mm_create_from_scene(scene_or_path._h, incore_bytes, sp, ctypes.byref(h)),
                   "svo_mm_create_from_scene")
        elif isinstance(scene_or_path, DeviceScene):
            _check(_L.svo_mm_create_from_device_scene(scene_or_path._h, incore_bytes, sp, ctypes.byref(h)),
                   "svo_mm_create_from_device_scene")
        else:
            _check(_L.svo_mm_create(str(scene_or_path).encode(), incore_bytes, sp, ctypes.byref(h)),
                   "svo_mm_create")
        self._h = h
        self._stream = stream

    # -- reference API --
    def initDeviceBuffer(self):
        _check(_L.svo_mm_init_device_buffer(self._h), "svo_mm_init_device_buffer")

    initClBuffer = initDeviceBuffer

    def getDeviceIncoreBuffer(self):
        """(device node pointer, device attribute pointer, number of nodes)."""
        n, a, c = ctypes.c_void_p(), ctypes.c_void_p(), _u64()
        _check(_L.svo_mm_get_device_buffers(self._h, ctypes.byref(n), ctypes.byref(a), ctypes.byref(c)),
               "svo_mm_get_device_buffers")
        return n.value, a.value, c.value

    def insertTreeletIntoIncoreBuffer(self, gid: int, visibility: int = MAX_VISIBILITY,
                                      error: float = 0.0) -> bool:
        return _L.svo_mm_insert_treelet(self._h, gid, visibility, error) == SVO_OK

    def removeTreeletFromIncoreBuffer(self, gid: int) -> bool:
        return _L.svo_mm_remove_treelet(self._h, gid) == SVO_OK

    def freeIncorePosition(self) -> bool:
        return _L.svo_mm_free_incore_position(self._h) == SVO_OK

    def updateClientSideIncoreBuffer(self, new_gids, new_errors=None, old_gids=()):
        ng = np.ascontiguousarray(new_gids, dtype=np.int32)
        ne = np.ascontiguousarray(new_errors if new_errors is not None else np.zeros(len(ng)),
                                  dtype=np.float32)
        og = np.ascontiguousarray(old_gids, dtype=np.int32)
        return _L.svo_mm_update_client_side(self._h, _np_ptr(ng), _np_ptr(ne), len(ng), _np_ptr(og),
                                            len(og))

    def updateDeviceMemory(self) -> int:
        calls = _u32()
        _check(_L.svo_mm_update_device_memory(self._h, ctypes.byref(calls)), "svo_mm_update_device_memory")
        return calls.value

    def planUploads(self):
        """[(first slot, slot count)] the next updateDeviceMemory copies."""
        n = _u32()
        _check(_L.svo_mm_plan_uploads(self._h, None, None, 0, ctypes.byref(n)), "svo_mm_plan_uploads")
        f = np.zeros(n.value, dtype=np.uint32)
        c = np.zeros(n.value, dtype=np.uint32)
        _check(_L.svo_mm_plan_uploads(self._h, _np_ptr(f), _np_ptr(c), n.value, ctypes.byref(n)),
               "svo_mm_plan_uploads")
        return list(zip(f.tolist(), c.tolist()))

    def setUploadPolicy(self, policy: int):
        """UPLOAD_COALESCED (the reference's ranges, staged), UPLOAD_PACKED
        (dirty slots packed, scatter kernel) or UPLOAD_PINNED (page-locked
        mirror, ranges copied directly)."""
        _check(_L.svo_mm_set_upload_policy(self._h, policy), "svo_mm_set_upload_policy")

    def setUploadRatio(self, ratio: float):
        """The coalescing ratio (the reference's 0.6; 1 = one copy per slot,
        0 = one range over all dirty slots)."""
        _check(_L.svo_mm_set_upload_ratio(self._h, ratio), "svo_mm_set_upload_ratio")

    def resetIncoreBuffer(self):
        _check(_L.svo_mm_reset(self._h), "svo_mm_reset")

    def insertAll(self) -> int:
        n = _u32()
        rc = _L.svo_mm_insert_all(self._h, ctypes.byref(n))
        if rc not in (SVO_OK, SVO_ERR_BUSY):
            _check(rc, "svo_mm_insert_all")
        return n.value

    @property
    def info(self) -> svo_mm_info:
        i = svo_mm_info()
        _check(_L.svo_mm_info_get(self._h, ctypes.byref(i)), "svo_mm_info_get")
        return i

    def getTreeletSizeInByte(self) -> int:
        return self.info.treelet_bytes

    def getNumNodesPerTreelet(self) -> int:
        return self.info.nodes_per_treelet

    def getSlots(self):
        out = []
        s = svo_slot_info()
        for i in range(self.info.num_slots):
            _check(_L.svo_mm_get_slot(self._h, i, ctypes.byref(s)), "svo_mm_get_slot")
            out.append((s.treelet_gid, s.visibility, s.error))
        return out

    def getSlotGid(self, gid: int) -> int:
        s = _i32()
        _check(_L.svo_mm_treelet_slot(self._h, gid, ctypes.byref(s)), "svo_mm_treelet_slot")
        return s.value

    def getIncoreBuffer(self, first: int = 0, count: int | None = None):
        n = self.info.incore_nodes
        count = n - first if count is None else count
        nodes = np.zeros((count, 2), dtype=np.uint32)
        attribs = np.zeros((count, 2), dtype=np.uint32)
        _check(_L.svo_mm_copy_incore(self._h, first, count, _np_ptr(nodes), _np_ptr(attribs)),
               "svo_mm_copy_incore")
        return nodes, attribs

    def getIncoreSlotsToUpload(self):
        c = _u32()
        _check(_L.svo_mm_slots_to_upload(self._h, None, 0, ctypes.byref(c)), "svo_mm_slots_to_upload")
        out = np.zeros(c.value, dtype=np.uint32)
        _check(_L.svo_mm_slots_to_upload(self._h, _np_ptr(out), c.value, ctypes.byref(c)),
               "svo_mm_slots_to_upload")
        return out

    # -- rendering --
    def render(self, params: svo_frame_params, rgba, hits=None, cfg: svo_trace_cfg | None = None,
               stream=None):
        cfg = cfg or trace_cfg()
        _check(_L.svo_mm_render(self._h, ctypes.byref(params), ctypes.byref(cfg), _dptr(rgba),
                                _dptr(hits), _stream_ptr(stream)), "svo_mm_render")

    def render_host(self, params: svo_frame_params, out: np.ndarray | None = None,
                    cfg: svo_trace_cfg | None = None, stream=None) -> np.ndarray:
        cfg = cfg or trace_cfg()
        if out is None:
            out = np.zeros((params.height, params.width), dtype=np.uint32)
        ptr = out.data_ptr() if hasattr(out, "data_ptr") else _np_ptr(out)
        _check(_L.svo_mm_render_host(self._h, ctypes.byref(params), ctypes.byref(cfg), ptr,
                                     _stream_ptr(stream)), "svo_mm_render_host")
        return out

    def render_shadow(self, params: svo_frame_params, rgba, shadow: svo_shadow_cfg | None = None,
                      hits=None, shadow_hits=None, cfg: svo_trace_cfg | None = None, stream=None):
        """Primary plus one shadow ray per hit over the incore buffer."""
        cfg = cfg or trace_cfg()
        shadow = shadow or shadow_cfg()
        _check(_L.svo_mm_render_shadow(self._h, ctypes.byref(params), ctypes.byref(cfg), ctypes.byref(shadow),
                                       _dptr(rgba), _dptr(hits), _dptr(shadow_hits), _stream_ptr(stream)),
               "svo_mm_render_shadow")

    def render_host_async(self, params: svo_frame_params, out, cfg: svo_trace_cfg | None = None, stream=None):
        """Non-blocking render_host: `out` (page-locked host memory, e.g. a
        pinned torch tensor) holds the frame after sync()."""
        cfg = cfg or trace_cfg()
        ptr = out.data_ptr() if hasattr(out, "data_ptr") else _np_ptr(out)
        _check(_L.svo_mm_render_host_async(self._h, ctypes.byref(params), ctypes.byref(cfg), ptr,
                                           _stream_ptr(stream)), "svo_mm_render_host_async")

    def render_shadow_host_async(self, params: svo_frame_params, out, shadow: svo_shadow_cfg | None = None,
                                 cfg: svo_trace_cfg | None = None, stream=None):
        """render_host_async for the primary + shadow ray frame."""
        cfg = cfg or trace_cfg()
        shadow = shadow or shadow_cfg()
        ptr = out.data_ptr() if hasattr(out, "data_ptr") else _np_ptr(out)
        _check(_L.svo_mm_render_shadow_host_async(self._h, ctypes.byref(params), ctypes.byref(cfg),
                                                  ctypes.byref(shadow), ptr, _stream_ptr(stream)),
               "svo_mm_render_shadow_host_async")

    def sync(self, stream=None) -> svo_stats:
        s = svo_stats()
        _check(_L.svo_mm_sync(self._h, _stream_ptr(stream), ctypes.byref(s)), "svo_mm_sync")
        return s

    def close(self):
        if self._h and self._h.value:
            _L.svo_mm_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def render(d_nodes, d_attribs, num_nodes: int, params: svo_frame_params, d_rgba, d_hits=None,
           cfg: svo_trace_cfg | None = None, d_stats=None, stream=None):
    """renderToBuffer over a node pool already in device memory."""
    cfg = cfg or trace_cfg()
    _check(_L.svo_render(_dptr(d_nodes), _dptr(d_attribs), num_nodes, ctypes.byref(params),
                         ctypes.byref(cfg), _dptr(d_rgba), _dptr(d_hits), _dptr(d_stats),
                         _stream_ptr(stream)), "svo_render")


def default_light() -> np.ndarray:
    """shade_diffuse_color_shadow's light (opencl/fillFrameBuffer_rgba.cl:506):
    normalize(-0.5, 1.0, 0.6), with normalize = v / sqrt((x*x + y*y) + z*z) in FP32."""
    v = np.array([-0.5, 1.0, 0.6], dtype=np.float32)
    n = np.sqrt((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2], dtype=np.float32)
    return (v / n).astype(np.float32)


def seeded_light(seed: int) -> np.ndarray:
    """A directional light from a seed: a uniform direction on the upper
    hemisphere (y >= 0.2), normalised in FP32 like default_light()."""
    rng = np.random.default_rng(seed)
    while True:
        v = rng.normal(size=3).astype(np.float32)
        v[1] = abs(v[1])
        n = np.sqrt((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2], dtype=np.float32)
        if n > 1e-3 and v[1] / n >= 0.2:
            return (v / n).astype(np.float32)


def shadow_cfg(light=None, t_scale_ratio=0.001, normal_offset=0.01) -> svo_shadow_cfg:
    """Shadow-ray settings; the defaults are shade_diffuse_color_shadow's
    (light normalize(-0.5, 1, 0.6), tScaleRatio 0.001, normal offset 0.01)."""
    c = svo_shadow_cfg()
    light = default_light() if light is None else np.asarray(light, dtype=np.float32)
    for i in range(3):
        c.light_direction[i] = float(light[i])
    c.t_scale_ratio, c.normal_offset, c.reserved = t_scale_ratio, normal_offset, 0
    return c


def render_shadow(d_nodes, d_attribs, num_nodes: int, params: svo_frame_params, d_rgba,
                  shadow: svo_shadow_cfg | None = None, d_hits=None, d_shadow_hits=None,
                  cfg: svo_trace_cfg | None = None, d_stats=None, stream=None):
    """Primary ray plus one shadow ray per hit (shade_diffuse_color_shadow)
    over a node pool already in device memory."""
    cfg = cfg or trace_cfg()
    shadow = shadow or shadow_cfg()
    _check(_L.svo_render_shadow(_dptr(d_nodes), _dptr(d_attribs), num_nodes, ctypes.byref(params),
                                ctypes.byref(cfg), ctypes.byref(shadow), _dptr(d_rgba), _dptr(d_hits),
                                _dptr(d_shadow_hits), _dptr(d_stats), _stream_ptr(stream)),
           "svo_render_shadow")


def trace_rays(d_nodes, num_nodes: int, d_origins, d_dirs, n: int, t_scale_ratio: float,
               d_hits, cfg: svo_trace_cfg | None = None, d_stats=None, stream=None):
    cfg = cfg or trace_cfg()
    _check(_L.svo_trace_rays(_dptr(d_nodes), num_nodes, _dptr(d_origins), _dptr(d_dirs), n,
                             float(t_scale_ratio), ctypes.byref(cfg), _dptr(d_hits), _dptr(d_stats),
                             _stream_ptr(stream)), "svo_trace_rays")


# ---- batched views -------------------------------------------------------------
def batch_cfg(tile_w=8, tile_h=4, block_threads=256, blocks_per_sm=0, top_nodes=0, use_graph=True,
              rays_per_lane=1):
    c = svo_batch_cfg()
    c.tile_w, c.tile_h, c.block_threads = tile_w, tile_h, block_threads
    c.blocks_per_sm, c.top_nodes, c.use_graph = blocks_per_sm, top_nodes, int(bool(use_graph))
    c.rays_per_lane = rays_per_lane
    return c


def octree_desc(d_nodes, d_attribs, num_nodes, traversal=TRAVERSAL_TREELET, stack_size=13):
    o = svo_octree_desc()
    o.d_nodes, o.d_attribs, o.num_nodes = _dptr(d_nodes), _dptr(d_attribs), num_nodes
    o.traversal, o.stack_size = traversal, stack_size
    return o


def octree_of(mm: "TreeletMemoryManagerCuda", stack_size=13) -> svo_octree_desc:
    n, a, c = mm.getDeviceIncoreBuffer()
    return octree_desc(n, a, c, TRAVERSAL_TREELET, stack_size)


def view_desc(params: svo_frame_params, octree: int, d_rgba, d_hits=None) -> svo_view_desc:
    v = svo_view_desc()
    v.params = params
    v.octree = octree
    v.d_rgba = _dptr(d_rgba)
    v.d_hits = _dptr(d_hits)
    return v


class Batcher:
    """A ragged table of views over resident octrees, cast in one persistent
    launch (svo_batcher_* in the C ABI)."""

    def __init__(self, max_views=1024, max_octrees=64):
        h = ctypes.c_void_p()
        _check(_L.svo_batcher_create(max_views, max_octrees, ctypes.byref(h)), "svo_batcher_create")
        self._h = h

    def set(self, octrees, views, cfg: svo_batch_cfg | None = None, stream=None):
        cfg = cfg or batch_cfg()
        oa = (svo_octree_desc * len(octrees))(*octrees)
        va = (svo_view_desc * len(views))(*views)
        _check(_L.svo_batcher_set(self._h, oa, len(octrees), va, len(views), ctypes.byref(cfg),
                                  _stream_ptr(stream)), "svo_batcher_set")

    def launch(self, d_stats=None, stream=None):
        _check(_L.svo_batcher_launch(self._h, _dptr(d_stats), _stream_ptr(stream)), "svo_batcher_launch")

    def autotune(self, reps=5, stream=None):
        best = svo_batch_cfg()
        ms = _f32()
        _check(_L.svo_batcher_autotune(self._h, reps, _stream_ptr(stream), ctypes.byref(best),
                                       ctypes.byref(ms)), "svo_batcher_autotune")
        return best, ms.value

    def size(self):
        t, r = _u64(), _u64()
        _check(_L.svo_batcher_size(self._h, ctypes.byref(t), ctypes.byref(r)), "svo_batcher_size")
        return t.value, r.value

    def close(self):
        if self._h and self._h.value:
            _L.svo_batcher_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def render_batch_static(octrees, views, tile=(8, 4), d_stats=None, stream=None):
    """The batched cast without allocation (svo_render_batch_static): for
    callers whose host owns all device memory or must not stall on
    cudaMalloc.  At most 256 views and 16 octrees; calls that overlap on the
    GPU share one scratch array and race."""
    oa = (svo_octree_desc * len(octrees))(*octrees)
    va = (svo_view_desc * len(views))(*views)
    _check(_L.svo_render_batch_static(oa, len(octrees), va, len(views), tile[0], tile[1],
                                      _dptr(d_stats), _stream_ptr(stream)), "svo_render_batch_static")


# ---- serving -------------------------------------------------------------------
SERVE_BATCHED = 0
SERVE_PLAIN = 1
SERVE_PLAIN_STREAMED = 2


class svo_server_cfg(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_uint64), ("max_inflight_rays", ctypes.c_uint64),
                ("streams", ctypes.c_uint32), ("max_batch_views", ctypes.c_uint32),
                ("mode", ctypes.c_uint32), ("tile_w", ctypes.c_uint32), ("tile_h", ctypes.c_uint32),
                ("block_threads", ctypes.c_uint32)]


class svo_request(ctypes.Structure):
    _fields_ = [("octree", ctypes.c_uint32), ("reserved", ctypes.c_uint32),
                ("params", svo_frame_params), ("d_rgba", ctypes.c_void_p)]


class svo_request_result(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("batch", ctypes.c_uint32), ("submit_s", ctypes.c_double),
                ("launch_s", ctypes.c_double), ("done_s", ctypes.c_double)]


class svo_server_stats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in ("requests_done", "rays_done", "batches", "octree_loads",
                                                "octree_evictions", "treelets_paged_in",
                                                "bytes_uploaded", "resident_bytes")] + \
               [("resident_octrees", ctypes.c_uint32), ("paged_unconverged", ctypes.c_uint32),
                ("analysis_passes", ctypes.c_uint64), ("paging_us", ctypes.c_uint64)]


for _name, (_args, _res) in {
    "svo_server_create": ([_P(svo_server_cfg), _P(_vp)], ctypes.c_int),
    "svo_server_destroy": ([_vp], None),
    "svo_server_add_octree": ([_vp, _vp, _i32, _P(_u32)], ctypes.c_int),
    "svo_server_add_octree_paged": ([_vp, _vp, _i32, _u64, _P(_u32)], ctypes.c_int),
    "svo_scene_from_pool": ([_vp, _vp, _u32, _u32, _u32, _u64, _P(_vp)], ctypes.c_int),
    "svo_mm_set_analysis_budget": ([_vp, _u64], ctypes.c_int),
    "svo_mm_analysis_requested": ([_vp, _P(_u32)], ctypes.c_int),
    "svo_mm_set_eviction": ([_vp, _i32], ctypes.c_int),
    "svo_mm_create_from_device_scene": ([_vp, _u64, _vp, _P(_vp)], ctypes.c_int),
    "svo_server_set_upload_policy": ([_vp, _u32, _i32], ctypes.c_int),
    "svo_server_submit": ([_vp, _P(svo_request), _P(_u64)], ctypes.c_int),
    "svo_server_wait": ([_vp, _u64, _u32, _P(svo_request_result)], ctypes.c_int),
    "svo_server_poll": ([_vp, _u64, _P(svo_request_result)], ctypes.c_int),
    "svo_server_cancel": ([_vp, _u64], ctypes.c_int),
    "svo_server_release": ([_vp, _u64], ctypes.c_int),
    "svo_server_stats_get": ([_vp, _P(svo_server_stats)], ctypes.c_int),
    "svo_server_replay": ([_vp, _P(svo_request), _P(ctypes.c_double), _u32, _u32, _P(svo_request_result)],
                          ctypes.c_int),
}.items():
    _fn = getattr(_L, _name)
    _fn.argtypes = _args
    _fn.restype = _res


def server_cfg(hbm_budget_bytes, max_inflight_rays=64 << 20, streams=4, max_batch_views=256,
               mode=SERVE_BATCHED, tile=(8, 4), block_threads=128) -> svo_server_cfg:
    c = svo_server_cfg()
    c.hbm_budget_bytes, c.max_inflight_rays = int(hbm_budget_bytes), int(max_inflight_rays)
    c.streams, c.max_batch_views, c.mode = streams, max_batch_views, mode
    c.tile_w, c.tile_h, c.block_threads = tile[0], tile[1], block_threads
    return c


def request(octree: int, params: svo_frame_params, d_rgba) -> svo_request:
    r = svo_request()
    r.octree, r.params, r.d_rgba = octree, params, _dptr(d_rgba)
    return r


class Server:
    """Request loop over resident octrees (svo_server_* in the C ABI)."""

    def __init__(self, cfg: svo_server_cfg):
        h = ctypes.c_void_p()
        _check(_L.svo_server_create(ctypes.byref(cfg), ctypes.byref(h)), "svo_server_create")
        self._h = h

    def add_octree(self, scene: Scene, stack_size=13) -> int:
        i = _u32()
        _check(_L.svo_server_add_octree(self._h, scene._h, stack_size, ctypes.byref(i)),
               "svo_server_add_octree")
        return i.value

    def add_octree_paged(self, scene: Scene, region_bytes: int, stack_size=13) -> int:
        """An octree served by treelet paging inside a fixed region of the pool."""
        i = _u32()
        _check(_L.svo_server_add_octree_paged(self._h, scene._h, stack_size, int(region_bytes),
                                              ctypes.byref(i)), "svo_server_add_octree_paged")
        return i.value

    def set_upload_policy(self, octree: int, policy: int):
        """UPLOAD_PINNED: page-lock the octree's host copy so that its loads
        are DMA copies straight from it."""
        _check(_L.svo_server_set_upload_policy(self._h, octree, policy), "svo_server_set_upload_policy")

    def submit(self, req: svo_request) -> int:
        t = _u64()
        _check(_L.svo_server_submit(self._h, ctypes.byref(req), ctypes.byref(t)), "svo_server_submit")
        return t.value

    def wait(self, ticket: int, timeout_ms=10000) -> svo_request_result:
        r = svo_request_result()
        _check(_L.svo_server_wait(self._h, ticket, timeout_ms, ctypes.byref(r)), "svo_server_wait")
        return r

    def poll(self, ticket: int):
        r = svo_request_result()
        rc = _L.svo_server_poll(self._h, ticket, ctypes.byref(r))
        return (r if rc == SVO_OK else None), rc

    def cancel(self, ticket: int) -> int:
        return _L.svo_server_cancel(self._h, ticket)

    def release(self, ticket: int) -> int:
        return _L.svo_server_release(self._h, ticket)

    def stats(self) -> svo_server_stats:
        s = svo_server_stats()
        _check(_L.svo_server_stats_get(self._h, ctypes.byref(s)), "svo_server_stats_get")
        return s

    def replay(self, reqs, arrival_s, timeout_ms=60000):
        n = len(reqs)
        ra = (svo_request * n)(*reqs)
        ta = (ctypes.c_double * n)(*[float(a) for a in arrival_s])
        out = (svo_request_result * n)()
        rc = _L.svo_server_replay(self._h, ra, ta, n, timeout_ms, out)
        # kept when a wait timed out, so callers can see which requests finished
        self.last_replay_results = list(out)
        _check(rc, "svo_server_replay")
        return list(out)

    def close(self):
        if self._h and self._h.value:
            _L.svo_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- analysis pass ---------------------------------------------------------------
class svo_feedback(ctypes.Structure):
    _fields_ = [("node_id", ctypes.c_int32), ("error", ctypes.c_float), ("sub_treelet_gid", ctypes.c_int32),
                ("t_min", ctypes.c_float)]


FEEDBACK_DTYPE = np.dtype([("node_id", "<i4"), ("error", "<f4"), ("sub_treelet_gid", "<i4"), ("t_min", "<f4")])

for _name, (_args, _res) in {
    "svo_feedback_render": ([_vp, _u64, _P(svo_frame_params), _i32, _vp, _vp, _vp], ctypes.c_int),
    "svo_mm_analyse_feedback": ([_vp, _vp, _u64, _u32, _vp, _vp, _u32, _P(_u32), _vp, _vp, _u32, _P(_u32)],
                                ctypes.c_int),
    "svo_mm_analyse_feedback_device": ([_vp, _vp, _u64, _u32, _vp, _vp, _vp, _u32, _P(_u32), _vp, _vp, _u32,
                                        _P(_u32)], ctypes.c_int),
    "svo_mm_analysis_step": ([_vp, _P(svo_frame_params), _u32, _f32, _f32, _i32, _vp, _P(_u32), _P(_u32)],
                             ctypes.c_int),
    "svo_mm_analysis_begin": ([_vp, _P(svo_frame_params), _u32, _f32, _f32, _i32, _vp], ctypes.c_int),
    "svo_mm_analysis_end": ([_vp, _vp, _P(_u32), _P(_u32)], ctypes.c_int),
}.items():
    _fn = getattr(_L, _name)
    _fn.argtypes = _args
    _fn.restype = _res


def feedback_render(d_nodes, num_nodes, params: svo_frame_params, d_feedback, d_rgba=None, stack_size=13,
                    stream=None):
    """renderToFeedbackBuffer over a device node pool (one record per pixel)."""
    _check(_L.svo_feedback_render(_dptr(d_nodes), num_nodes, ctypes.byref(params), stack_size,
                                  _dptr(d_feedback), _dptr(d_rgba), _stream_ptr(stream)), "svo_feedback_render")


def _analyse_feedback(self, records: np.ndarray, max_new: int = 0):
    """performAnalysePass's processing: ([(gid, error)] new, [(gid, error)] old)."""
    rec = np.ascontiguousarray(records).view(np.uint8).reshape(-1)
    n = rec.size // 16
    nn, no = _u32(), _u32()
    rc = _L.svo_mm_analyse_feedback(self._h, _np_ptr(rec), n, max_new, None, None, 0, ctypes.byref(nn),
                                    None, None, 0, ctypes.byref(no))
    _check(rc, "svo_mm_analyse_feedback")
    ng = np.zeros(nn.value, np.int32); ne = np.zeros(nn.value, np.float32)
    og = np.zeros(no.value, np.int32); oe = np.zeros(no.value, np.float32)
    _check(_L.svo_mm_analyse_feedback(self._h, _np_ptr(rec), n, max_new, _np_ptr(ng), _np_ptr(ne), nn.value,
                                      ctypes.byref(nn), _np_ptr(og), _np_ptr(oe), no.value, ctypes.byref(no)),
           "svo_mm_analyse_feedback")
    return list(zip(ng.tolist(), ne.tolist())), list(zip(og.tolist(), oe.tolist()))


def _analyse_feedback_device(self, d_records, n: int, max_new: int = 0, stream=None):
    """The same processing over n records in device memory, folded on the GPU:
    ([(gid, error)] new, [(gid, error)] old)."""
    cap = self.info.num_treelets + 1  # neither list can be longer
    nn, no = _u32(), _u32()
    ng = np.zeros(cap, np.int32); ne = np.zeros(cap, np.float32)
    og = np.zeros(cap, np.int32); oe = np.zeros(cap, np.float32)
    _check(_L.svo_mm_analyse_feedback_device(self._h, _dptr(d_records), n, max_new, _stream_ptr(stream),
                                             _np_ptr(ng), _np_ptr(ne), cap, ctypes.byref(nn), _np_ptr(og),
                                             _np_ptr(oe), cap, ctypes.byref(no)),
           "svo_mm_analyse_feedback_device")
    k, m = nn.value, no.value
    return list(zip(ng[:k].tolist(), ne[:k].tolist())), list(zip(og[:m].tolist(), oe[:m].tolist()))


def _perform_analyse_pass(self, frame: svo_frame_params, divisor=8, jitter=(0.0, 0.0), stack_size=13,
                          stream=None):
    """One dynamic-loading step (analysis pass, insert, upload): (new, old) counts."""
    nn, no = _u32(), _u32()
    _check(_L.svo_mm_analysis_step(self._h, ctypes.byref(frame), divisor, float(jitter[0]), float(jitter[1]),
                                   stack_size, _stream_ptr(stream), ctypes.byref(nn), ctypes.byref(no)),
           "svo_mm_analysis_step")
    return nn.value, no.value


def _begin_analyse_pass(self, frame: svo_frame_params, divisor=8, jitter=(0.0, 0.0), stack_size=13,
                        stream=None):
    """First half of performAnalysePass: the analysis rays and the GPU fold,
    launched on `stream`; endAnalysePass finishes the step."""
    _check(_L.svo_mm_analysis_begin(self._h, ctypes.byref(frame), divisor, float(jitter[0]),
                                    float(jitter[1]), stack_size, _stream_ptr(stream)),
           "svo_mm_analysis_begin")


def _end_analyse_pass(self, after_stream=None):
    """Second half: insert and evict, then upload once the work queued on
    `after_stream` (a frame reading the pool) is done: (new, old) counts."""
    nn, no = _u32(), _u32()
    _check(_L.svo_mm_analysis_end(self._h, _stream_ptr(after_stream), ctypes.byref(nn), ctypes.byref(no)),
           "svo_mm_analysis_end")
    return nn.value, no.value


TreeletMemoryManagerCuda.beginAnalysePass = _begin_analyse_pass
TreeletMemoryManagerCuda.endAnalysePass = _end_analyse_pass
TreeletMemoryManagerCuda.analyseFeedback = _analyse_feedback
TreeletMemoryManagerCuda.analyseFeedbackDevice = _analyse_feedback_device
TreeletMemoryManagerCuda.performAnalysePass = _perform_analyse_pass


def _set_analysis_budget(self, nbytes: int):
    """Bytes of new treelets one analysis pass may place (0: the reference's 12 MB)."""
    _check(_L.svo_mm_set_analysis_budget(self._h, int(nbytes)), "svo_mm_set_analysis_budget")


TreeletMemoryManagerCuda.setAnalysisBudget = _set_analysis_budget


def _last_analysis_requested(self) -> int:
    """Treelets the last analysis pass asked for, placed or not (0: converged)."""
    n = _u32()
    _check(_L.svo_mm_analysis_requested(self._h, ctypes.byref(n)), "svo_mm_analysis_requested")
    return n.value


TreeletMemoryManagerCuda.lastAnalysisRequested = _last_analysis_requested

EVICT_REFERENCE = 0
EVICT_ANY_UNSEEN = 1


def _set_eviction(self, rule: int):
    """EVICT_REFERENCE (the reference's rule) or EVICT_ANY_UNSEEN."""
    _check(_L.svo_mm_set_eviction(self._h, int(rule)), "svo_mm_set_eviction")


TreeletMemoryManagerCuda.setEviction = _set_eviction


# ---- teardown ------------------------------------------------------------------
# Handles still open when the interpreter exits are closed here, before the
# CUDA runtime linked into the library is torn down: a server's dispatcher
# thread must not issue CUDA calls after that.
import atexit as _atexit  # noqa: E402
import weakref as _weakref  # noqa: E402

_live = _weakref.WeakSet()


def _track(obj):
    _live.add(obj)
    return obj


def _close_all():
    objs = list(_live)
    for o in sorted(objs, key=lambda o: 0 if isinstance(o, Server) else 1):
        try:
            o.close()
        except Exception:
            pass


_atexit.register(_close_all)

for _cls in (Scene, DeviceScene, TreeletMemoryManagerCuda, Batcher, Server):
    _orig_init = _cls.__init__

    def _init(self, *a, __orig=_orig_init, **k):
        __orig(self, *a, **k)
        _track(self)

    _cls.__init__ = _init

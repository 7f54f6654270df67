"""CPU oracle for the libsvo per-ray octree cast.

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU-baseline leg.  The product package ``libsvo_b200`` never
imports it.

Two CPU implementations live here:

* ``liboracle.so`` -- ``oracle/oracle.cpp``, a restatement of the reference's
  ``sample()`` (opencl/treeletRenderer_rgba.cl:201-382) and of
  ``CpuRaycasterSingleRay3::traversSvo``
  (src/incore/CpuRaycasterSingleRay3.cpp:159-387).
* ``libsvo_ref_cl.so`` -- the reference's own ``treeletRenderer_rgba.cl``
  compiled for the host (``oracle/build_ref.py``); present only where the
  reference checkout was available at build time.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
BUILD_DIR = HERE / "_build"
LIB = BUILD_DIR / "liboracle.so"

HIT_DTYPE = np.dtype(
    [("node", "<u4"), ("t", "<f4"), ("depth", "<u2"), ("hit", "u1"), ("flags", "u1"), ("loops", "<u2"),
     ("fetches", "<u2")]
)
assert HIT_DTYPE.itemsize == 16

FLAG_CAPPED = 1
FLAG_BOUNDS = 2
FLAG_BOX_MISS = 4


def build(force: bool = False) -> Path:
    """Compiles oracle.cpp (FP32, no FMA contraction) into oracle/_build."""
    src = HERE / "oracle.cpp"
    if LIB.is_file() and not force and LIB.stat().st_mtime >= src.stat().st_mtime:
        return LIB
    BUILD_DIR.mkdir(parents=True, exist_ok=True)
    cmd = [
        "g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
        "-pthread", "-Wall", "-o", str(LIB), str(src),
    ]
    subprocess.run(cmd, check=True)
    return LIB


def build_reference(force: bool = False, reference=None):
    from . import build_ref

    return build_ref.build(force=force, reference=reference)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.is_file():
            build()
        L = ctypes.CDLL(str(LIB))
        vp, u64, i32, f32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_float
        L.oracle_render.argtypes = [vp, vp, u64, vp, i32, i32, vp, vp, vp, i32]
        L.oracle_render.restype = u64
        L.oracle_cast_rays.argtypes = [vp, u64, vp, vp, u64, f32, i32, i32, vp, i32]
        L.oracle_cast_rays.restype = u64
        L.oracle_pixel_rays.argtypes = [vp, vp, vp]
        L.oracle_pixel_rays.restype = None
        L.oracle_feedback.argtypes = [vp, u64, vp, i32, vp, vp, i32]
        L.oracle_feedback.restype = None
        L.oracle_render_shadow.argtypes = [vp, vp, u64, vp, i32, vp, f32, f32, vp, vp, vp, vp, i32]
        L.oracle_render_shadow.restype = u64
        u32 = ctypes.c_uint32
        L.oracle_render_shadow_rows.argtypes = [vp, vp, u64, vp, i32, vp, f32, f32, u32, u32, vp, vp, vp,
                                                vp, i32]
        L.oracle_render_shadow_rows.restype = u64
        assert L.oracle_hit_record_size() == 16
        _lib = L
    return _lib


def reference_lib():
    """The reference's own kernel compiled for the host, or None if absent."""
    global _ref
    if _ref is None:
        p = HERE / "_ref" / "libsvo_ref_cl.so"
        if not p.is_file():
            return None
        L = ctypes.CDLL(str(p))
        vp, u64, i32, f32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_float
        L.ref_sample_rays.argtypes = [vp, vp, vp, u64, f32, vp, i32]
        L.ref_sample_rays.restype = None
        L.ref_render.argtypes = [vp, vp, vp, vp, i32]
        L.ref_render.restype = None
        L.ref_render_rows.argtypes = [vp, vp, vp, ctypes.c_uint32, ctypes.c_uint32, vp, i32]
        L.ref_render_rows.restype = None
        L.ref_feedback.argtypes = [vp, vp, vp, vp, i32]
        L.ref_feedback.restype = None
        L.ref_render_shadow.argtypes = [vp, vp, vp, vp, f32, f32, vp, vp, i32]
        L.ref_render_shadow.restype = None
        L.ref_render_shadow_rows.argtypes = [vp, vp, vp, vp, f32, f32, ctypes.c_uint32, ctypes.c_uint32,
                                             vp, vp, i32]
        L.ref_render_shadow_rows.restype = None
        assert L.ref_hit_record_size() == 16
        _ref = L
    return _ref


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _threads(threads):
    return int(threads if threads else (os.cpu_count() or 1))


def render(nodes: np.ndarray, attribs: np.ndarray, params: bytes, flat: bool = False,
           stack_size: int = 13, want_rgbaf: bool = False, threads: int | None = None):
    """One frame on the CPU.  ``nodes``/``attribs``: uint32 arrays of shape
    (N, 2).  ``params``: the 80-byte svo_frame_params record.  Returns
    (rgba8 [H, W] uint32, hits [H, W] HIT_DTYPE, node_fetches, rgbaf or None)."""
    nodes = np.ascontiguousarray(nodes, dtype=np.uint32)
    attribs = np.ascontiguousarray(attribs, dtype=np.uint32)
    w, h = np.frombuffer(params[:8], dtype=np.uint32)
    pbuf = np.frombuffer(bytearray(params), dtype=np.uint8)
    rgba = np.zeros((h, w), dtype=np.uint32)
    hits = np.zeros((h, w), dtype=HIT_DTYPE)
    rgbaf = np.zeros((h, w, 4), dtype=np.float32) if want_rgbaf else None
    fetches = lib().oracle_render(
        _ptr(nodes), _ptr(attribs), nodes.shape[0], _ptr(pbuf), int(flat), int(stack_size),
        _ptr(rgba), _ptr(rgbaf) if want_rgbaf else None, _ptr(hits), _threads(threads))
    return rgba, hits, int(fetches), rgbaf


def cast_rays(nodes: np.ndarray, origins: np.ndarray, dirs: np.ndarray, t_scale_ratio: float,
              flat: bool = False, stack_size: int = 13, threads: int | None = None):
    nodes = np.ascontiguousarray(nodes, dtype=np.uint32)
    origins = np.ascontiguousarray(origins, dtype=np.float32)
    dirs = np.ascontiguousarray(dirs, dtype=np.float32)
    n = origins.shape[0]
    hits = np.zeros(n, dtype=HIT_DTYPE)
    fetches = lib().oracle_cast_rays(_ptr(nodes), nodes.shape[0], _ptr(origins), _ptr(dirs), n,
                                     float(t_scale_ratio), int(flat), int(stack_size), _ptr(hits),
                                     _threads(threads))
    return hits, int(fetches)


def pixel_rays(params: bytes):
    w, h = np.frombuffer(params[:8], dtype=np.uint32)
    o = np.zeros((h * w, 3), dtype=np.float32)
    d = np.zeros((h * w, 3), dtype=np.float32)
    pbuf = np.frombuffer(bytearray(params), dtype=np.uint8)
    lib().oracle_pixel_rays(_ptr(pbuf), _ptr(o), _ptr(d))
    return o, d


def reference_sample_rays(nodes, origins, dirs, t_scale_ratio, threads=None):
    L = reference_lib()
    if L is None:
        return None
    nodes = np.ascontiguousarray(nodes, dtype=np.uint32)
    origins = np.ascontiguousarray(origins, dtype=np.float32)
    dirs = np.ascontiguousarray(dirs, dtype=np.float32)
    n = origins.shape[0]
    hits = np.zeros(n, dtype=HIT_DTYPE)
    L.ref_sample_rays(_ptr(nodes), _ptr(origins), _ptr(dirs), n, float(t_scale_ratio), _ptr(hits),
                      _threads(threads))
    return hits


def reference_render(nodes, attribs, params: bytes, threads=None, rows=None):
    """renderToBuffer from the reference source: float RGBA [H, W, 4]
    (only rows [rows[0], rows[1]) when ``rows`` is given)."""
    L = reference_lib()
    if L is None:
        return None
    nodes = np.ascontiguousarray(nodes, dtype=np.uint32)
    attribs = np.ascontiguousarray(attribs, dtype=np.uint32)
    w, h = np.frombuffer(params[:8], dtype=np.uint32)
    out = np.zeros((h, w, 4), dtype=np.float32)
    pbuf = np.frombuffer(bytearray(params), dtype=np.uint8)
    if rows is None:
        L.ref_render(_ptr(nodes), _ptr(attribs), _ptr(pbuf), _ptr(out), _threads(threads))
    else:
        L.ref_render_rows(_ptr(nodes), _ptr(attribs), _ptr(pbuf), int(rows[0]), int(rows[1]), _ptr(out),
                          _threads(threads))
    return out


def to_rgba8(rgbaf: np.ndarray) -> np.ndarray:
    """float RGBA -> packed RGBA8 (byte 0 red), round(clamp(c, 0, 1) * 255) in
    FP32, NaN -> 0."""
    c = rgbaf.astype(np.float32)
    c = np.clip(np.where(np.isnan(c), np.float32(0), c), np.float32(0), np.float32(1))
    b = np.floor(c * np.float32(255.0) + np.float32(0.5)).astype(np.uint32)
    return b[..., 0] | (b[..., 1] << 8) | (b[..., 2] << 16) | (b[..., 3] << 24)


FEEDBACK_DTYPE = np.dtype([("node_id", "<i4"), ("error", "<f4"), ("sub_treelet_gid", "<i4"), ("t_min", "<f4")])


def feedback(nodes, params: bytes, stack_size: int = 13, threads=None):
    """renderToFeedbackBuffer on the CPU: (records [H, W], debug rgbaf [H, W, 4])."""
    nodes = np.ascontiguousarray(nodes, dtype=np.uint32)
    w, h = np.frombuffer(params[:8], dtype=np.uint32)
    rec = np.zeros((h, w), dtype=FEEDBACK_DTYPE)
    rgbaf = np.zeros((h, w, 4), dtype=np.float32)
    pbuf = np.frombuffer(bytearray(params), dtype=np.uint8)
    lib().oracle_feedback(_ptr(nodes), nodes.shape[0], _ptr(pbuf), int(stack_size), _ptr(rec), _ptr(rgbaf),
                          _threads(threads))
    return rec, rgbaf


def reference_feedback(nodes, params: bytes, threads=None):
    L = reference_lib()
    if L is None:
        return None
    nodes = np.ascontiguousarray(nodes, dtype=np.uint32)
    w, h = np.frombuffer(params[:8], dtype=np.uint32)
    rec = np.zeros((h, w), dtype=FEEDBACK_DTYPE)
    rgbaf = np.zeros((h, w, 4), dtype=np.float32)
    pbuf = np.frombuffer(bytearray(params), dtype=np.uint8)
    L.ref_feedback(_ptr(nodes), _ptr(pbuf), _ptr(rec), _ptr(rgbaf), _threads(threads))
    return rec, rgbaf


# Light direction of shade_diffuse_color_shadow (opencl/fillFrameBuffer_rgba.cl:
# 506): normalize(-0.5, 1.0, 0.6) with normalize = v / sqrt((x*x + y*y) + z*z).
def default_light():
    v = np.array([-0.5, 1.0, 0.6], dtype=np.float32)
    l = np.sqrt((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2], dtype=np.float32)
    return (v / l).astype(np.float32)


def render_shadow(nodes, attribs, params: bytes, light, shadow_tsr: float = 0.001,
                  offset: float = 0.01, stack_size: int = 13,
                  want_rgbaf: bool = False, threads=None, rows=None):
    """Primary plus shadow rays on the CPU.  Returns (rgba8 [H, W], hits [H, W],
    shadow_hits [H, W], node_fetches, rgbaf or None); with ``rows`` = (y0, y1)
    only those rows, as arrays of y1 - y0 rows."""
    nodes = np.ascontiguousarray(nodes, dtype=np.uint32)
    attribs = np.ascontiguousarray(attribs, dtype=np.uint32)
    light = np.ascontiguousarray(light, dtype=np.float32)
    w, h = (int(v) for v in np.frombuffer(params[:8], dtype=np.uint32))
    y0, y1 = (0, h) if rows is None else (int(rows[0]), min(h, int(rows[1])))
    n = max(0, y1 - y0)
    pbuf = np.frombuffer(bytearray(params), dtype=np.uint8)
    rgba = np.zeros((n, w), dtype=np.uint32)
    hits = np.zeros((n, w), dtype=HIT_DTYPE)
    shits = np.zeros((n, w), dtype=HIT_DTYPE)
    rgbaf = np.zeros((n, w, 4), dtype=np.float32) if want_rgbaf else None
    fetches = lib().oracle_render_shadow_rows(
        _ptr(nodes), _ptr(attribs), nodes.shape[0], _ptr(pbuf), int(stack_size), _ptr(light),
        float(shadow_tsr), float(offset), y0, y1, _ptr(rgba),
        _ptr(rgbaf) if want_rgbaf else None, _ptr(hits), _ptr(shits), _threads(threads))
    return rgba, hits, shits, int(fetches), rgbaf


def reference_render_shadow(nodes, attribs, params: bytes, light, shadow_tsr: float = 0.001,
                            offset: float = 0.01, threads=None, rows=None):
    """The shadow shading over the reference's own sample(): (rgbaf [H, W, 4],
    shadow_hits [H, W]); with ``rows`` = (y0, y1) only those rows."""
    L = reference_lib()
    if L is None:
        return None
    nodes = np.ascontiguousarray(nodes, dtype=np.uint32)
    attribs = np.ascontiguousarray(attribs, dtype=np.uint32)
    light = np.ascontiguousarray(light, dtype=np.float32)
    w, h = (int(v) for v in np.frombuffer(params[:8], dtype=np.uint32))
    y0, y1 = (0, h) if rows is None else (int(rows[0]), min(h, int(rows[1])))
    n = max(0, y1 - y0)
    out = np.zeros((n, w, 4), dtype=np.float32)
    shits = np.zeros((n, w), dtype=HIT_DTYPE)
    pbuf = np.frombuffer(bytearray(params), dtype=np.uint8)
    L.ref_render_shadow_rows(_ptr(nodes), _ptr(attribs), _ptr(pbuf), _ptr(light), float(shadow_tsr),
                             float(offset), y0, y1, _ptr(out), _ptr(shits), _threads(threads))
    return out, shits

"""The C ABI library loads and exports every function include/libsvo_b200.h
declares; argument errors come back as status codes (no GPU needed)."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import libsvo_b200 as L

HEADER = Path(__file__).resolve().parent.parent / "include" / "libsvo_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(svo_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("svo_mm_create", "svo_mm_init_device_buffer", "svo_mm_insert_treelet",
                 "svo_mm_remove_treelet", "svo_mm_update_device_memory", "svo_mm_reset",
                 "svo_render", "svo_mm_render", "svo_mm_sync"):
        assert must in names
    assert len(names) >= 35


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(L.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_null_arguments_are_status_codes():
    lib = L.lib
    assert lib.svo_scene_build_menger(3, 5, 1, 0, 0, None) == L.SVO_ERR_INVALID
    assert lib.svo_mm_create(None, 1 << 20, None, None) == L.SVO_ERR_INVALID
    assert lib.svo_mm_insert_treelet(None, 1, 8, 0.0) == L.SVO_ERR_INVALID
    assert lib.svo_mm_update_device_memory(None, None) == L.SVO_ERR_INVALID
    assert lib.svo_render(None, None, 0, None, None, None, None, None, None) == L.SVO_ERR_INVALID
    p = L.orbit_camera(1, 8, 8).frame_params()
    cfg = L.trace_cfg(stack_size=40)
    assert lib.svo_render(1, 1, 1, ctypes.byref(p), ctypes.byref(cfg), 1, None, None, None) == L.SVO_ERR_RANGE
    cfg = L.trace_cfg(traversal=7)
    assert lib.svo_render(1, 1, 1, ctypes.byref(p), ctypes.byref(cfg), 1, None, None, None) == L.SVO_ERR_NOTSUP
    p.mode = 8
    cfg = L.trace_cfg()
    assert lib.svo_render(1, 1, 1, ctypes.byref(p), ctypes.byref(cfg), 1, None, None, None) == L.SVO_ERR_NOTSUP
    p.mode = 6  # Phong and quality need the treelet traversal's node centre and quality
    cfg = L.trace_cfg(traversal=L.TRAVERSAL_FLAT, stack_size=8)
    assert lib.svo_render(1, 1, 1, ctypes.byref(p), ctypes.byref(cfg), 1, None, None, None) == L.SVO_ERR_NOTSUP
    sc = L.shadow_cfg()
    assert lib.svo_render_shadow(1, 1, 1, ctypes.byref(p), ctypes.byref(cfg), ctypes.byref(sc), 1, None, None, None,
                                 None) == L.SVO_ERR_NOTSUP
    cfg = L.trace_cfg()
    assert lib.svo_render_shadow(1, None, 1, ctypes.byref(p), ctypes.byref(cfg), ctypes.byref(sc), 1, None, None,
                                 None, None) == L.SVO_ERR_INVALID
    assert lib.svo_render_shadow(1, 1, 1, ctypes.byref(p), ctypes.byref(cfg), None, 1, None, None, None,
                                 None) == L.SVO_ERR_INVALID
    sc.reserved = 1
    assert lib.svo_render_shadow(1, 1, 1, ctypes.byref(p), ctypes.byref(cfg), ctypes.byref(sc), 1, None, None, None,
                                 None) == L.SVO_ERR_INVALID
    assert lib.svo_mm_render_shadow(None, ctypes.byref(p), ctypes.byref(cfg), ctypes.byref(sc), 1, None, None,
                                    None) == L.SVO_ERR_INVALID
    assert lib.svo_mm_render_host_async(None, ctypes.byref(p), ctypes.byref(cfg), 1, None) == L.SVO_ERR_INVALID
    assert lib.svo_mm_render_shadow_host_async(None, ctypes.byref(p), ctypes.byref(cfg), ctypes.byref(sc), 1,
                                               None) == L.SVO_ERR_INVALID
    out = ctypes.c_void_p()
    assert lib.svo_device_scene_build_mesh(None, 3, None, 1, 5, 0, None, ctypes.byref(out)) == L.SVO_ERR_INVALID
    v = (ctypes.c_float * 9)()
    t = (ctypes.c_uint32 * 3)(0, 1, 2)
    assert lib.svo_device_scene_build_mesh_attributed(v, v, None, 3, t, 1, 5, 0, None,
                                                      ctypes.byref(out)) == L.SVO_ERR_INVALID
    assert lib.svo_device_scene_info_get(None, None) == L.SVO_ERR_INVALID
    assert lib.svo_device_scene_buffers(None, None, None, None) == L.SVO_ERR_INVALID
    assert lib.svo_device_scene_copy(None, 0, 0, None, None) == L.SVO_ERR_INVALID
    assert lib.svo_mm_set_upload_policy(None, 0) == L.SVO_ERR_INVALID
    assert lib.svo_mm_set_upload_ratio(None, 0.6) == L.SVO_ERR_INVALID
    assert lib.svo_mesh_vertex_attributes(v, 3, t, 1, 1, None, None) == L.SVO_ERR_INVALID
    t_bad = (ctypes.c_uint32 * 3)(0, 1, 3)
    nrm, col = (ctypes.c_float * 9)(), (ctypes.c_float * 9)()
    assert lib.svo_mesh_vertex_attributes(v, 3, t_bad, 1, 1, nrm, col) == L.SVO_ERR_INVALID


def test_manager_without_device_buffer_rejects_renders(menger_scene):
    mm = L.TreeletMemoryManagerCuda(menger_scene, menger_scene.info.treelet_bytes)
    with pytest.raises(L.SvoError) as e:
        mm.render(L.orbit_camera(1, 8, 8).frame_params(), 0)
    assert e.value.code == L.SVO_ERR_INVALID
    with pytest.raises(L.SvoError):
        mm.getDeviceIncoreBuffer()
    with pytest.raises(L.SvoError) as e:  # slot 0 is dirty but there is no device copy yet
        mm.updateDeviceMemory()
    assert e.value.code == L.SVO_ERR_INVALID


def test_version():
    assert L.version().startswith("libsvo_b200")

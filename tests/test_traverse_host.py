"""The kernels' own traversal code (libsvo_b200/csrc/traverse.cuh) compiled
for the host through tests/hostsim/host_shim.h and compared with the oracle
ray by ray, without a GPU.  This checks the restructured traversal (the
{node, tMax} stack, incremental centres, sign-ordered slab distances, node
prefetch) on the CPU; the GPU tests check the same code as compiled by nvcc.
"""
import ctypes
import subprocess
from pathlib import Path

import numpy as np
import pytest

import libsvo_b200 as L
import oracle
from rays import edge_rays, random_octree_pool

HERE = Path(__file__).resolve().parent / "hostsim"
LIB = HERE / "_build" / "libtraverse_host.so"


@pytest.fixture(scope="module")
def host_lib():
    src = HERE / "traverse_host.cpp"
    deps = [src, HERE / "host_shim.h", HERE.parent.parent / "libsvo_b200" / "csrc" / "traverse.cuh"]
    if not LIB.is_file() or any(LIB.stat().st_mtime < d.stat().st_mtime for d in deps):
        LIB.parent.mkdir(parents=True, exist_ok=True)
        subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
                        "-o", str(LIB), str(src)], check=True)
    lib = ctypes.CDLL(str(LIB))
    vp = ctypes.c_void_p
    lib.host_cast_rays.argtypes = [vp, ctypes.c_uint64, vp, vp, ctypes.c_uint64, ctypes.c_float, ctypes.c_int,
                                   ctypes.c_int, vp]
    lib.host_cast_rays.restype = None
    return lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def check(lib, nodes, o, d, tsr, stack_size=13, flat=False):
    nodes = np.ascontiguousarray(nodes, dtype=np.uint32)
    o = np.ascontiguousarray(o, dtype=np.float32)
    d = np.ascontiguousarray(d, dtype=np.float32)
    got = np.zeros(o.shape[0], dtype=oracle.HIT_DTYPE)
    lib.host_cast_rays(_p(nodes), nodes.shape[0], _p(o), _p(d), o.shape[0], float(tsr), int(stack_size),
                       int(flat), _p(got))
    want, _ = oracle.cast_rays(nodes, o, d, tsr, flat=flat, stack_size=stack_size)
    for k in ("node", "depth", "hit", "flags", "loops", "fetches"):
        bad = np.nonzero(got[k] != want[k])[0]
        assert bad.size == 0, f"{k} differs at {bad.size} rays, first {bad[:5]}"
    assert np.array_equal(got["t"].view(np.uint32), want["t"].view(np.uint32))
    return got


@pytest.mark.parametrize("tsr", [0.0, 0.003, 0.05])
def test_menger_rays(host_lib, small_menger_scene, tsr):
    mm = L.TreeletMemoryManagerCuda(small_menger_scene, small_menger_scene.info.treelet_bytes)
    nodes, _ = mm.getIncoreBuffer()
    o, d = edge_rays(n_random=20000, seed=5)
    check(host_lib, nodes, o, d, tsr)
    o, d = oracle.pixel_rays(bytes(L.orbit_camera(2, 160, 120, radius=1.3).frame_params()))
    h = check(host_lib, nodes, o, d, tsr)
    assert h["hit"].sum() > 1000


def test_flat_pool(host_lib, small_menger_scene):
    nodes, _ = small_menger_scene.flatten()
    o, d = edge_rays(n_random=20000, seed=6)
    for tsr in (0.0, 0.01):
        check(host_lib, nodes, o, d, tsr, stack_size=small_menger_scene.info.max_depth, flat=True)


@pytest.mark.parametrize("seed", range(4))
def test_random_octrees(host_lib, seed):
    nodes, _ = random_octree_pool(seed, depth=4 + seed % 3)
    o, d = edge_rays(n_random=5000, seed=seed)
    check(host_lib, nodes, o, d, 0.0)
    check(host_lib, nodes, o, d, 0.02)


def test_icosphere_frame(host_lib):
    from libsvo_b200 import scenes

    wl = scenes.icosphere(subdivisions=4, depth=9, treelet_levels=5, width=160, height=96)
    info = wl.scene.info
    mm = L.TreeletMemoryManagerCuda(wl.scene, info.treelet_bytes * info.num_treelets)
    mm.insertAll()
    nodes, _ = mm.getIncoreBuffer()
    p = wl.cameras[0].frame_params()
    o, d = oracle.pixel_rays(bytes(p))
    check(host_lib, nodes, o, d, p.t_scale_ratio)


def test_long_and_watchdog_rays(host_lib):
    """Every long ray (60 iterations or more) of a 960x540 icosphere frame,
    one of them stopped by the watchdog at (S+1)^2*5 iterations, matches the
    oracle in node, t, depth, flags, loop and fetch counts."""
    from libsvo_b200 import scenes

    wl = scenes.icosphere(subdivisions=5, depth=9, treelet_levels=4, width=960, height=540)
    info = wl.scene.info
    mm = L.TreeletMemoryManagerCuda(wl.scene, info.treelet_bytes * info.num_treelets)
    mm.insertAll()
    nodes, _ = mm.getIncoreBuffer()
    p = wl.cameras[0].frame_params()
    o, d = oracle.pixel_rays(bytes(p))
    want, _ = oracle.cast_rays(nodes, o, d, p.t_scale_ratio)
    long_rays = np.nonzero(want["loops"] >= 60)[0]
    assert long_rays.size > 1000 and (want["flags"][long_rays] & L.HITFLAG_CAPPED).sum() >= 1
    got = check(host_lib, nodes, o[long_rays], d[long_rays], p.t_scale_ratio)
    assert (got["flags"] & L.HITFLAG_CAPPED).sum() == (want["flags"][long_rays] & L.HITFLAG_CAPPED).sum()

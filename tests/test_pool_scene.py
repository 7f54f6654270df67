"""A fully resident incore pool turned back into treelets (svo_scene_from_pool,
svo_mm_create_from_device_scene): every treelet's records and header must be
the ones the pool was filled from, so the treelet files written from both
scenes are equal byte for byte.  CPU cases run the host manager's mirror; the
GPU case starts from a pool built on the GPU."""
import numpy as np
import pytest

import libsvo_b200 as L


def resident_pool(scene):
    info = scene.info
    mm = L.TreeletMemoryManagerCuda(scene, info.treelet_bytes * info.num_treelets)
    assert mm.insertAll() == info.num_treelets - 1
    nodes, attribs = mm.getIncoreBuffer()
    mm.close()
    return nodes, attribs


def assert_same_files(a, b, tmp_path):
    a.write(str(tmp_path / "a"))
    b.write(str(tmp_path / "b"))
    for ext in (".svo", ".ia"):
        assert (tmp_path / ("a" + ext)).read_bytes() == (tmp_path / ("b" + ext)).read_bytes(), ext


@pytest.mark.parametrize("kind", ["menger_levels", "menger_bytes", "icosphere", "terrain"])
def test_pool_back_to_treelets(kind, tmp_path):
    if kind == "menger_levels":
        scene = L.Scene.menger(level=4, depth=7, seed=3, treelet_levels=3)
    elif kind == "menger_bytes":  # the reference's byte-size fill: sub-treelets at any level
        scene = L.Scene.menger(level=3, depth=6, seed=4, treelet_bytes=1024)
    elif kind == "icosphere":
        v, t = L.icosphere(4, seed=2)
        scene = L.Scene.from_mesh(v, t, 8, treelet_levels=3)
    else:
        v, t = L.terrain(65, seed=3)
        scene = L.Scene.from_mesh(v, t, 7, treelet_levels=2)
    info = scene.info
    assert info.num_treelets > 3
    nodes, attribs = resident_pool(scene)
    back = L.Scene.from_pool(nodes, attribs, info.num_treelets, info.treelet_bytes, info.max_depth,
                             info.leaf_voxels)
    assert_same_files(scene, back, tmp_path)
    # and the manager over the recovered scene fills the same pool again
    n2, a2 = resident_pool(back)
    assert np.array_equal(n2, nodes) and np.array_equal(a2, attribs)


def test_corrupt_pool_is_rejected():
    scene = L.Scene.menger(level=3, depth=5, seed=7, treelet_levels=2)
    info = scene.info
    nodes, attribs = resident_pool(scene)
    bad = nodes.copy()
    bad[1, 0] = 0x7FFFFFF0  # a child pointer far outside the pool
    bad[1, 1] |= 0xFF00
    with pytest.raises(L.SvoError):
        L.Scene.from_pool(bad, attribs, info.num_treelets, info.treelet_bytes, info.max_depth)


@pytest.mark.gpu
def test_manager_from_a_gpu_built_pool(cuda, tmp_path):
    """svo_mm_create_from_device_scene: the treelets recovered from a pool
    built on the GPU equal the host builder's, and a manager with a small
    incore buffer over them pages like one over the host scene."""
    v, t = L.icosphere(4, seed=6)
    host = L.Scene.from_mesh(v, t, 9, treelet_levels=3)
    dev = L.DeviceScene(v, t, 9, treelet_levels=3)
    info = host.info
    nodes, attribs = dev.getIncoreBuffer()
    back = L.Scene.from_pool(nodes, attribs, info.num_treelets, info.treelet_bytes, info.max_depth,
                             info.leaf_voxels)
    assert_same_files(host, back, tmp_path)
    small = info.treelet_bytes * max(4, info.num_treelets // 4)
    mm_dev = L.TreeletMemoryManagerCuda(dev, small)
    mm_host = L.TreeletMemoryManagerCuda(host, small)
    for mm in (mm_dev, mm_host):
        mm.initDeviceBuffer()
    p = L.orbit_camera(3, 160, 120, radius=1.4).frame_params()
    for _ in range(6):
        a = mm_dev.performAnalysePass(p, divisor=2)
        b = mm_host.performAnalysePass(p, divisor=2)
        assert a == b
    n1, a1 = mm_dev.getIncoreBuffer()
    n2, a2 = mm_host.getIncoreBuffer()
    assert np.array_equal(n1, n2) and np.array_equal(a1, a2)
    mm_dev.close()
    mm_host.close()
    dev.close()

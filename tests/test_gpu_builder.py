"""The GPU scene builder (svo_device_scene_build_mesh) against the host path:
Scene.from_mesh -> TreeletMemoryManagerCuda -> insertAll must give the same
incore pool, record for record, and the same scene counts."""
import numpy as np
import pytest

import libsvo_b200 as L

pytestmark = pytest.mark.gpu


def host_pool(v, t, depth, treelet_levels, attrs=(None, None)):
    scene = L.Scene.from_mesh(v, t, depth, treelet_levels=treelet_levels, normals=attrs[0], colors=attrs[1])
    info = scene.info
    mm = L.TreeletMemoryManagerCuda(scene, info.treelet_bytes * info.num_treelets)
    mm.insertAll()
    nodes, attribs = mm.getIncoreBuffer()
    mm.close()
    return info, nodes, attribs


def assert_same(v, t, depth, treelet_levels, attrs=(None, None)):
    info, nodes, attribs = host_pool(v, t, depth, treelet_levels, attrs)
    ds = L.DeviceScene(v, t, depth, treelet_levels=treelet_levels, normals=attrs[0], colors=attrs[1])
    di = ds.info
    for k in ("num_treelets", "treelet_bytes", "nodes_per_treelet", "max_depth", "total_nodes", "leaf_voxels"):
        assert getattr(di, k) == getattr(info, k), k
    dn, da = ds.getIncoreBuffer()
    assert dn.shape == nodes.shape
    bad = np.nonzero((dn != nodes).any(axis=1))[0]
    assert bad.size == 0, f"{bad.size} node records differ, first {bad[:5]}: {dn[bad[:3]]} vs {nodes[bad[:3]]}"
    bad = np.nonzero((da != attribs).any(axis=1))[0]
    assert bad.size == 0, f"{bad.size} attribute records differ, first {bad[:5]}"
    ds.close()
    return info


@pytest.mark.parametrize("depth,levels", [(6, 0), (8, 3), (9, 4), (9, 5), (10, 6)])
def test_icosphere_pool_matches_host(cuda, depth, levels):
    v, t = L.icosphere(3 if depth < 9 else 4)
    info = assert_same(v, t, depth, levels)
    assert info.leaf_voxels > 1000


def test_terrain_pool_matches_host(cuda):
    v, t = L.terrain(64)
    assert_same(v, t, 9, 4)


@pytest.mark.parametrize("depth,levels", [(7, 3), (10, 5)])
def test_interpolated_vertex_attributes_match_host(cuda, depth, levels):
    """The reference's interpolated leaf attributes (per-vertex normals and
    colours) come out of both builders bit for bit."""
    v, t = L.icosphere(4)
    info = assert_same(v, t, depth, levels, L.vertex_attributes(v, t, 7))
    assert info.leaf_voxels > 1000
    v, t = L.terrain(48)
    assert_same(v, t, depth, levels, L.vertex_attributes(v, t, 8))


def test_rendering_the_device_pool(cuda):
    """A frame over the device-built pool equals the frame over the host one."""
    import torch

    from libsvo_b200 import scenes

    wl = scenes.icosphere(subdivisions=4, depth=9, treelet_levels=5, width=320, height=200, colour="vertex")
    v, t = L.icosphere(4)  # the mesh scenes.icosphere builds, with its vertex attributes
    vn, vc = L.vertex_attributes(v, t, 1)
    ds = L.DeviceScene(v, t, 9, treelet_levels=5, normals=vn, colors=vc)
    dn, da, n = ds.buffers()
    p = wl.cameras[0].frame_params()
    rgba = torch.empty((p.height, p.width), dtype=torch.int32, device=cuda)
    L.render(dn, da, n, p, rgba)
    torch.cuda.synchronize()
    info = wl.scene.info
    mm = L.TreeletMemoryManagerCuda(wl.scene, info.treelet_bytes * info.num_treelets)
    mm.insertAll()
    mm.initDeviceBuffer()
    host = mm.render_host(p)
    assert np.array_equal(rgba.cpu().numpy().view(np.uint32), host)
    mm.close()
    ds.close()


def test_bad_inputs_are_status_codes(cuda):
    v, t = L.icosphere(1)
    with pytest.raises(L.SvoError) as e:
        L.DeviceScene(v, t, 0)
    assert e.value.code == L.SVO_ERR_RANGE
    t2 = t.copy()
    t2[0, 0] = v.shape[0]
    with pytest.raises(L.SvoError) as e:
        L.DeviceScene(v, t2, 6)
    assert e.value.code == L.SVO_ERR_INVALID


def test_benchmark_icosphere_pool_matches_host(cuda):
    """The 1080p benchmark's octree (81,920 triangles, depth 11, 6-level
    treelets, seeded vertex attributes; the parameters of
    libsvo_b200.scenes.icosphere): 3,175 treelets, record for record."""
    v, t = L.icosphere(6, radius=0.4, octaves=3, amplitude=0.05, frequency=2.0, seed=1)
    info = assert_same(v, t, 11, 6, L.vertex_attributes(v, t, 1))
    assert info.num_treelets > 3000

"""Pins the oracle to the reference: the restated traversal must agree bit for
bit with the reference's own treelet kernel source (opencl/
treeletRenderer_rgba.cl), compiled for the host by oracle/build_ref.py.

These tests need the reference build (oracle/_ref); where it is absent the
committed golden fixtures (tests/test_golden.py) carry the same check.
"""
import numpy as np
import pytest

import libsvo_b200 as L
import oracle
from rays import edge_rays, paged_menger_manager, random_octree_pool

ref_needed = pytest.mark.skipif(oracle.reference_lib() is None,
                                reason="reference kernel build (oracle/_ref) not present")


def check_rays(nodes, o, d, tsr):
    got, _ = oracle.cast_rays(nodes, o, d, tsr)
    want = oracle.reference_sample_rays(nodes, o, d, tsr)
    for k in ("node", "depth", "hit", "loops"):
        bad = np.nonzero(got[k] != want[k])[0]
        assert bad.size == 0, f"{k} differs at {bad.size} rays, first {bad[:5]}"
    assert np.array_equal(got["t"].view(np.uint32), want["t"].view(np.uint32))
    return got


def check_frame(nodes, attribs, params):
    rgba, hits, _, rgbaf = oracle.render(nodes, attribs, bytes(params), want_rgbaf=True)
    ref = oracle.reference_render(nodes, attribs, bytes(params))
    defined = np.ones(hits.shape, dtype=bool)
    if params.mode == 4:
        # pixel-depth shading reads SampleResult.t, which sample() leaves
        # unwritten for rays that miss the root cube (uninitialised in the
        # reference); the library defines t = 0 there
        defined = (hits["flags"] & oracle.FLAG_BOX_MISS) == 0
        assert defined.sum() > 0
    assert np.array_equal(rgbaf[defined].view(np.uint32), ref[defined].view(np.uint32)), \
        "fragment colours differ"
    assert np.array_equal(rgba[defined], oracle.to_rgba8(ref)[defined])
    o, d = oracle.pixel_rays(bytes(params))
    check_rays(nodes, o, d, params.t_scale_ratio)
    return hits


@ref_needed
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_menger_frames(menger_scene, seed):
    mm = L.TreeletMemoryManagerCuda(menger_scene, menger_scene.info.treelet_bytes)
    nodes, attribs = mm.getIncoreBuffer()
    cam = L.orbit_camera(seed, 320, 240)
    for tsr in (None, 0.0, 0.02):
        hits = check_frame(nodes, attribs, cam.frame_params(t_scale_ratio=tsr))
        assert hits["hit"].sum() > 0


@ref_needed
@pytest.mark.parametrize("mode", [0, 1, 2, 3, 4, 5, 6, 7])
def test_view_modes(menger_scene, mode):
    mm = L.TreeletMemoryManagerCuda(menger_scene, menger_scene.info.treelet_bytes)
    nodes, attribs = mm.getIncoreBuffer()
    check_frame(nodes, attribs, L.orbit_camera(4, 160, 100).frame_params(mode=mode))
    # LOD stops give quality 0 in mode 7, leaves a positive or negative one
    check_frame(nodes, attribs, L.orbit_camera(5, 96, 64, radius=1.2).frame_params(mode=mode, t_scale_ratio=0.02))


def small_icosphere_pool():
    from libsvo_b200 import scenes

    wl = scenes.icosphere(subdivisions=4, depth=9, treelet_levels=5, width=160, height=96)
    info = wl.scene.info
    mm = L.TreeletMemoryManagerCuda(wl.scene, info.treelet_bytes * info.num_treelets)
    mm.insertAll()
    nodes, attribs = mm.getIncoreBuffer()
    return wl, nodes, attribs


@ref_needed
@pytest.mark.parametrize("mode", [2, 6, 7])
def test_view_modes_icosphere(mode):
    wl, nodes, attribs = small_icosphere_pool()
    check_frame(nodes, attribs, wl.cameras[0].frame_params(mode=mode))


def check_shadow_frame(nodes, attribs, params, light, tsr=0.001, offset=0.01):
    """The oracle's shadow frame against the same shading over the
    reference's own sample() (oracle/ref_harness.inc)."""
    rgba, hits, shits, _, rgbaf = oracle.render_shadow(nodes, attribs, bytes(params), light, tsr, offset,
                                                       want_rgbaf=True)
    ref, ref_shits = oracle.reference_render_shadow(nodes, attribs, bytes(params), light, tsr, offset)
    assert np.array_equal(rgbaf.view(np.uint32), ref.view(np.uint32)), "shadow fragment colours differ"
    assert np.array_equal(rgba, oracle.to_rgba8(ref))
    for k in ("node", "depth", "hit", "loops"):
        assert np.array_equal(shits[k], ref_shits[k]), f"shadow {k}"
    assert np.array_equal(shits["t"].view(np.uint32), ref_shits["t"].view(np.uint32))
    return hits, shits


@ref_needed
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_shadow_frames_icosphere(seed):
    wl, nodes, attribs = small_icosphere_pool()
    light = L.default_light() if seed == 0 else L.seeded_light(seed)
    for tsr in (None, 0.0):
        hits, shits = check_shadow_frame(nodes, attribs, wl.cameras[0].frame_params(t_scale_ratio=tsr), light)
        assert hits["hit"].sum() > 500
        assert 0 < shits["hit"].sum() < hits["hit"].sum()


@ref_needed
@pytest.mark.parametrize("seed", [1, 2])
def test_shadow_frames_menger_and_random(menger_scene, seed):
    mm = L.TreeletMemoryManagerCuda(menger_scene, menger_scene.info.treelet_bytes)
    nodes, attribs = mm.getIncoreBuffer()
    check_shadow_frame(nodes, attribs, L.orbit_camera(seed, 160, 120, radius=1.4).frame_params(),
                       L.seeded_light(seed))
    nodes, attribs = random_octree_pool(seed, depth=5)
    check_shadow_frame(nodes, attribs, L.orbit_camera(seed, 96, 96, radius=(1.0, 2.0)).frame_params(t_scale_ratio=0.0),
                       L.seeded_light(seed + 5), 0.0, 0.02)


@ref_needed
@pytest.mark.parametrize("tsr", [0.0, 0.003, 0.05])
def test_edge_rays(menger_scene, tsr):
    mm = L.TreeletMemoryManagerCuda(menger_scene, menger_scene.info.treelet_bytes)
    nodes, _ = mm.getIncoreBuffer()
    o, d = edge_rays(n_random=5000)
    check_rays(nodes, o, d, tsr)


@ref_needed
def test_paged_pool():
    _, mm = paged_menger_manager()
    nodes, attribs = mm.getIncoreBuffer()
    assert (nodes[:, 0].view(np.int32) < 0).any()
    check_frame(nodes, attribs, L.orbit_camera(7, 200, 200, radius=1.4).frame_params(t_scale_ratio=0.0))


@ref_needed
@pytest.mark.parametrize("seed", range(8))
def test_random_octrees(seed):
    nodes, attribs = random_octree_pool(seed, depth=3 + seed % 4)
    check_frame(nodes, attribs, L.orbit_camera(seed, 96, 64, radius=(1.0, 2.0)).frame_params(t_scale_ratio=0.0))
    o, d = edge_rays(n_random=2000, seed=seed)
    check_rays(nodes, o, d, 0.0)


@ref_needed
def test_icosphere_frame():
    from libsvo_b200 import scenes

    wl = scenes.icosphere(subdivisions=5, depth=9, treelet_levels=4, width=320, height=180)
    info = wl.scene.info
    mm = L.TreeletMemoryManagerCuda(wl.scene, info.treelet_bytes * info.num_treelets)
    mm.insertAll()
    nodes, attribs = mm.getIncoreBuffer()
    hits = check_frame(nodes, attribs, wl.cameras[0].frame_params())
    assert hits["hit"].mean() > 0.1


def test_unorm8_conversion_is_exact_for_packed_bytes():
    """The colour epilogue maps each packed byte b to b * 0.003921569f and
    back to round(c * 255): every byte survives."""
    b = np.arange(256, dtype=np.float32)
    c = b * np.float32(0.003921569)
    back = np.floor(c * np.float32(255.0) + np.float32(0.5))
    assert np.array_equal(back, b)


def partially_resident_menger():
    """Root and a few top treelets resident: leaves with non-resident
    sub-treelets appear in the pool."""
    scene = L.Scene.menger(level=4, depth=7, seed=3, treelet_levels=3)
    ntl = scene.info.num_treelets
    parents = np.array([scene.treelet(g)["parent_gid"] for g in range(ntl)])
    mm = L.TreeletMemoryManagerCuda(scene, scene.info.treelet_bytes * ntl)
    top = [g for g in range(1, ntl) if parents[g] == 0]
    for g in top[::2]:
        assert mm.insertTreeletIntoIncoreBuffer(g)
    return scene, mm, parents


@ref_needed
@pytest.mark.parametrize("seed", [1, 2, 3, 4])
def test_feedback_pass(seed):
    _, mm, _ = partially_resident_menger()
    nodes, _ = mm.getIncoreBuffer()
    for tsr in (0.0, None):
        p = bytes(L.orbit_camera(seed, 120, 80, radius=(1.2, 2.0)).frame_params(t_scale_ratio=tsr))
        rec, img = oracle.feedback(nodes, p)
        ref_rec, ref_img = oracle.reference_feedback(nodes, p)
        assert np.array_equal(rec.view(np.uint8), ref_rec.view(np.uint8))
        assert np.array_equal(img.view(np.uint32), ref_img.view(np.uint32))
        if tsr == 0.0:
            assert (rec["sub_treelet_gid"] > 0).any()

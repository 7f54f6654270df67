"""GPU parity for the shading paths beyond the hit record: view modes 2
(iteration count as a wavelength colour), 6 (Phong) and 7 (LOD quality), and
the primary + shadow ray frame.

Hit records (primary and shadow) are compared bit for bit.  Mode 7 and the
shadow frame use only correctly rounded FP32 arithmetic and are compared
exactly; modes 2 and 6 call pow() (CUDA's powf / pow against the host's), so
their RGBA8 pixels are held to the 1-LSB tolerance per channel.
"""
import numpy as np
import pytest

import libsvo_b200 as L
import oracle
from rays import random_octree_pool
from test_render_gpu import _hits_np, _torch, assert_hits_equal, gpu_frame

pytestmark = pytest.mark.gpu

LSB_TOLERANCE = 1  # RGBA8 units per channel, modes 2 and 6


def assert_rgba_close(got, want, tol, what=""):
    g = got.reshape(-1).view(np.uint8).astype(np.int16)
    w = want.reshape(-1).view(np.uint8).astype(np.int16)
    d = np.abs(g - w)
    assert d.max(initial=0) <= tol, f"{what}: max channel difference {d.max()} at {np.argmax(d) // 4}"


@pytest.fixture(scope="module")
def menger_mm(menger_scene, cuda):
    mm = L.TreeletMemoryManagerCuda(menger_scene, menger_scene.info.treelet_bytes)
    mm.initDeviceBuffer()
    yield mm
    mm.close()


@pytest.fixture(scope="module")
def icosphere_mm(cuda):
    from libsvo_b200 import scenes

    wl = scenes.icosphere(subdivisions=5, depth=9, treelet_levels=4, width=400, height=240)
    info = wl.scene.info
    mm = L.TreeletMemoryManagerCuda(wl.scene, info.treelet_bytes * info.num_treelets)
    mm.insertAll()
    mm.initDeviceBuffer()
    yield wl, mm
    mm.close()


@pytest.mark.parametrize("mode", [2, 6, 7])
@pytest.mark.parametrize("tsr", [None, 0.0, 0.02])
def test_extended_view_modes(menger_mm, mode, tsr):
    p = L.orbit_camera(5, 240, 160, radius=1.3).frame_params(mode=mode, t_scale_ratio=tsr)
    rgba, hits = gpu_frame(menger_mm, p)
    nodes, attribs = menger_mm.getIncoreBuffer()
    o_rgba, o_hits, _, _ = oracle.render(nodes, attribs, bytes(p))
    assert_hits_equal(hits, o_hits, f"mode {mode}")
    if mode == 7:
        assert np.array_equal(rgba, o_rgba)
    else:
        assert_rgba_close(rgba, o_rgba, LSB_TOLERANCE, f"mode {mode}")


@pytest.mark.parametrize("mode", [6, 7])
def test_extended_modes_on_icosphere(icosphere_mm, mode):
    wl, mm = icosphere_mm
    p = wl.cameras[0].frame_params(mode=mode)
    rgba, hits = gpu_frame(mm, p)
    nodes, attribs = mm.getIncoreBuffer()
    o_rgba, o_hits, _, _ = oracle.render(nodes, attribs, bytes(p))
    assert_hits_equal(hits, o_hits, f"mode {mode}")
    assert_rgba_close(rgba, o_rgba, 0 if mode == 7 else LSB_TOLERANCE, f"mode {mode}")


def test_modes_6_7_need_the_treelet_traversal(menger_scene, cuda):
    torch = _torch()
    nodes, attribs = menger_scene.flatten()
    dn = torch.from_numpy(nodes.view(np.int32)).to(cuda)
    da = torch.from_numpy(attribs.view(np.int32)).to(cuda)
    rgba = torch.empty((8, 8), dtype=torch.int32, device=cuda)
    cfg = L.trace_cfg(L.TRAVERSAL_FLAT, menger_scene.info.max_depth)
    for mode in (6, 7):
        with pytest.raises(L.SvoError) as e:
            L.render(dn, da, nodes.shape[0], L.orbit_camera(1, 8, 8).frame_params(mode=mode), rgba, cfg=cfg)
        assert e.value.code == L.SVO_ERR_NOTSUP
    with pytest.raises(L.SvoError) as e:
        L.render_shadow(dn, da, nodes.shape[0], L.orbit_camera(1, 8, 8).frame_params(), rgba, cfg=cfg)
    assert e.value.code == L.SVO_ERR_NOTSUP


def gpu_shadow_frame(mm, params, shadow):
    torch = _torch()
    n = params.height * params.width
    rgba = torch.empty((params.height, params.width), dtype=torch.int32, device="cuda")
    hits = torch.empty((n * 16,), dtype=torch.uint8, device="cuda")
    shits = torch.empty((n * 16,), dtype=torch.uint8, device="cuda")
    mm.render_shadow(params, rgba, shadow, hits, shits, stream=torch.cuda.current_stream())
    torch.cuda.synchronize()
    return rgba.cpu().numpy().view(np.uint32), _hits_np(hits), _hits_np(shits)


def check_shadow(mm, params, light, shadow_tsr=0.001, offset=0.01):
    sc = L.shadow_cfg(light, shadow_tsr, offset)
    rgba, hits, shits = gpu_shadow_frame(mm, params, sc)
    nodes, attribs = mm.getIncoreBuffer()
    o_rgba, o_hits, o_shits, _, _ = oracle.render_shadow(nodes, attribs, bytes(params), light,
                                                         shadow_tsr, offset)
    assert_hits_equal(hits, o_hits, "primary")
    assert_hits_equal(shits, o_shits, "shadow")
    assert np.array_equal(rgba, o_rgba)
    return o_hits, o_shits


@pytest.mark.parametrize("seed", [0, 3, 8])
def test_shadow_frame_icosphere(icosphere_mm, seed):
    wl, mm = icosphere_mm
    light = L.default_light() if seed == 0 else L.seeded_light(seed)
    hits, shits = check_shadow(mm, wl.cameras[0].frame_params(), light)
    n_hit = int(hits["hit"].sum())
    n_shadow = int(shits["hit"].sum())
    assert n_hit > 1000
    assert 0 < n_shadow < n_hit  # some hits are lit, some shadowed


def test_shadow_frame_menger(menger_mm):
    for seed, tsr in ((1, None), (2, 0.0)):
        p = L.orbit_camera(seed, 256, 192, radius=1.4).frame_params(t_scale_ratio=tsr)
        check_shadow(menger_mm, p, L.seeded_light(seed))
    # a coarse shadow LOD and a larger offset
    check_shadow(menger_mm, L.orbit_camera(4, 128, 128).frame_params(), L.seeded_light(4), 0.05, 0.03)


@pytest.mark.parametrize("w,h", [(1301, 811), (4099, 257)])
def test_large_ragged_shadow_frames(menger_mm, w, h):
    """Shadow frames of a million pixels or more (many waves of blocks) with
    ragged sizes that leave partial blocks on the right and bottom edges:
    every pixel, primary and shadow record must match the oracle."""
    assert w * h >= 1 << 20
    p = L.orbit_camera(5, w, h, radius=1.6).frame_params()
    hits, shits = check_shadow(menger_mm, p, L.seeded_light(5))
    assert 0 < int(shits["hit"].sum()) < int(hits["hit"].sum())


@pytest.mark.parametrize("seed", range(3))
def test_shadow_random_octrees(cuda, seed):
    torch = _torch()
    nodes, attribs = random_octree_pool(seed, depth=5 + seed % 2)
    dn = torch.from_numpy(nodes.view(np.int32)).to(cuda)
    da = torch.from_numpy(attribs.view(np.int32)).to(cuda)
    p = L.orbit_camera(seed, 160, 120, radius=(1.0, 2.0)).frame_params(t_scale_ratio=0.0)
    n = p.width * p.height
    rgba = torch.empty((p.height, p.width), dtype=torch.int32, device=cuda)
    hits = torch.empty((n * 16,), dtype=torch.uint8, device=cuda)
    shits = torch.empty((n * 16,), dtype=torch.uint8, device=cuda)
    stats = torch.zeros(4, dtype=torch.int32, device=cuda)
    light = L.seeded_light(10 + seed)
    L.render_shadow(dn, da, nodes.shape[0], p, rgba, L.shadow_cfg(light, 0.0, 0.02), hits, shits,
                    d_stats=stats)
    torch.cuda.synchronize()
    o_rgba, o_hits, o_shits, _, _ = oracle.render_shadow(nodes, attribs, bytes(p), light, 0.0, 0.02)
    assert_hits_equal(_hits_np(hits), o_hits, "primary")
    assert_hits_equal(_hits_np(shits), o_shits, "shadow")
    assert np.array_equal(rgba.cpu().numpy().view(np.uint32), o_rgba)
    capped = int((o_hits["flags"] == oracle.FLAG_CAPPED).sum() + (o_shits["flags"] == oracle.FLAG_CAPPED).sum())
    assert int(stats[0].item()) == capped

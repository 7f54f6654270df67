"""GPU parity: the sm_100a ray cast against the CPU oracle, bit for bit.

Every comparison here is exact: node indices, hit flags, depths, loop counts,
the FP32 hit distance t compared as bits, and the RGBA8 pixels.
"""
import numpy as np
import pytest

import libsvo_b200 as L
import oracle
from rays import edge_rays, paged_menger_manager, random_octree_pool

pytestmark = pytest.mark.gpu


def _torch():
    import torch

    return torch


def _hits_np(t):
    return t.cpu().numpy().view(np.uint8).view(L.HIT_DTYPE).reshape(-1)


def assert_hits_equal(got, want, what=""):
    got = got.reshape(-1)
    want = want.reshape(-1)
    for k in ("node", "depth", "hit", "flags", "loops", "fetches"):
        bad = np.nonzero(got[k] != want[k])[0]
        assert bad.size == 0, f"{what}: {k} differs at {bad.size} rays, first {bad[:5]}: " \
                              f"{got[k][bad[:5]]} vs {want[k][bad[:5]]}"
    bt = np.nonzero(got["t"].view(np.uint32) != want["t"].view(np.uint32))[0]
    assert bt.size == 0, f"{what}: t differs at {bt.size} rays: {got['t'][bt[:5]]} vs {want['t'][bt[:5]]}"


def gpu_frame(mm, params, cfg=None):
    torch = _torch()
    rgba = torch.empty((params.height, params.width), dtype=torch.int32, device="cuda")
    hits = torch.empty((params.height * params.width * 16,), dtype=torch.uint8, device="cuda")
    mm.render(params, rgba, hits, cfg=cfg, stream=torch.cuda.current_stream())
    torch.cuda.synchronize()
    return rgba.cpu().numpy().view(np.uint32), _hits_np(hits)


@pytest.fixture(scope="module")
def menger_mm(menger_scene, cuda):
    mm = L.TreeletMemoryManagerCuda(menger_scene, menger_scene.info.treelet_bytes)
    mm.initDeviceBuffer()
    yield mm
    mm.close()


@pytest.mark.parametrize("seed", [1, 2, 3, 4])
def test_menger_frame_matches_oracle(menger_mm, seed):
    cam = L.orbit_camera(seed, 512, 512)
    p = cam.frame_params()
    rgba, hits = gpu_frame(menger_mm, p)
    nodes, attribs = menger_mm.getIncoreBuffer()
    o_rgba, o_hits, _, _ = oracle.render(nodes, attribs, bytes(p))
    assert_hits_equal(hits, o_hits, f"seed {seed}")
    assert np.array_equal(rgba, o_rgba)
    assert o_hits["hit"].sum() > 1000  # the camera sees the sponge


def test_menger_full_depth_and_coarse_lod(menger_mm):
    cam = L.orbit_camera(11, 384, 256, radius=1.2)
    nodes, attribs = menger_mm.getIncoreBuffer()
    for tsr in (0.0, 0.02):
        p = cam.frame_params(t_scale_ratio=tsr)
        rgba, hits = gpu_frame(menger_mm, p)
        o_rgba, o_hits, _, _ = oracle.render(nodes, attribs, bytes(p))
        assert_hits_equal(hits, o_hits, f"tsr {tsr}")
        assert np.array_equal(rgba, o_rgba)


@pytest.mark.parametrize("mode", [1, 3, 4, 5])
def test_view_modes(menger_mm, mode):
    p = L.orbit_camera(5, 200, 120).frame_params(mode=mode)
    rgba, hits = gpu_frame(menger_mm, p)
    nodes, attribs = menger_mm.getIncoreBuffer()
    o_rgba, o_hits, _, _ = oracle.render(nodes, attribs, bytes(p))
    assert np.array_equal(rgba, o_rgba)


@pytest.mark.parametrize("w,h", [(1, 1), (17, 13), (8, 4), (1000, 3)])
def test_ragged_frame_sizes(menger_mm, w, h):
    p = L.orbit_camera(6, w, h, radius=1.6).frame_params()
    rgba, hits = gpu_frame(menger_mm, p)
    nodes, attribs = menger_mm.getIncoreBuffer()
    o_rgba, o_hits, _, _ = oracle.render(nodes, attribs, bytes(p))
    assert_hits_equal(hits, o_hits)
    assert np.array_equal(rgba, o_rgba)


@pytest.mark.parametrize("w,h", [(1301, 811), (4099, 257), (1024, 1024)])
def test_ragged_frames_cast_longest_first(menger_mm, w, h):
    """Frames of a million pixels or more are cast longest first (a per-block
    cost estimate, then the blocks in bucket order); ragged widths and
    heights leave partial blocks on the right and bottom edges.  Every pixel
    must still match the oracle."""
    p = L.orbit_camera(7, w, h, radius=1.8).frame_params()
    assert w * h >= 1 << 20
    rgba, hits = gpu_frame(menger_mm, p)
    nodes, attribs = menger_mm.getIncoreBuffer()
    o_rgba, o_hits, _, _ = oracle.render(nodes, attribs, bytes(p))
    assert_hits_equal(hits, o_hits, f"{w}x{h}")
    assert np.array_equal(rgba, o_rgba.reshape(rgba.shape))


def test_frame_taller_than_one_grid(menger_mm, cuda):
    """600,001 rows: more than one launch's 65,535 block rows of 8 pixels;
    the per-frame, shadow and feedback kernels each cover it in several
    launches."""
    torch = _torch()
    p = L.orbit_camera(7, 3, 600001, radius=1.6, fov_deg=80.0).frame_params()
    rgba, hits = gpu_frame(menger_mm, p)
    nodes, attribs = menger_mm.getIncoreBuffer()
    o_rgba, o_hits, _, _ = oracle.render(nodes, attribs, bytes(p))
    assert_hits_equal(hits, o_hits, "render")
    assert np.array_equal(rgba, o_rgba)
    assert o_hits["hit"].sum() > 1000
    d_nodes, d_attribs, n = menger_mm.getDeviceIncoreBuffer()
    light = L.seeded_light(3)
    img = torch.empty((p.height, p.width), dtype=torch.int32, device=cuda)
    sh = torch.empty(p.width * p.height * 16, dtype=torch.uint8, device=cuda)
    L.render_shadow(d_nodes, d_attribs, n, p, img, L.shadow_cfg(light), None, sh)
    fb = torch.empty(p.width * p.height * 16, dtype=torch.uint8, device=cuda)
    L.feedback_render(d_nodes, n, p, fb)
    torch.cuda.synchronize()
    s_rgba, _, s_sh, _, _ = oracle.render_shadow(nodes, attribs, bytes(p), light)
    assert np.array_equal(img.cpu().numpy().view(np.uint32), s_rgba)
    assert_hits_equal(_hits_np(sh), s_sh.reshape(-1), "shadow rays")
    rec, _ = oracle.feedback(nodes, bytes(p))
    assert np.array_equal(fb.cpu().numpy(), rec.view(np.uint8).reshape(-1))


def test_flat_traversal_matches_oracle(menger_scene, cuda):
    torch = _torch()
    nodes, attribs = menger_scene.flatten()
    depth = menger_scene.info.max_depth
    dn = torch.from_numpy(nodes.view(np.int32)).to(cuda)
    da = torch.from_numpy(attribs.view(np.int32)).to(cuda)
    for seed in (1, 2):
        p = L.orbit_camera(seed, 320, 240).frame_params()
        rgba = torch.empty((p.height, p.width), dtype=torch.int32, device=cuda)
        hits = torch.empty((p.height * p.width * 16,), dtype=torch.uint8, device=cuda)
        L.render(dn, da, nodes.shape[0], p, rgba, hits, cfg=L.trace_cfg(L.TRAVERSAL_FLAT, depth))
        torch.cuda.synchronize()
        o_rgba, o_hits, _, _ = oracle.render(nodes, attribs, bytes(p), flat=True, stack_size=depth)
        assert_hits_equal(_hits_np(hits), o_hits, "flat")
        assert np.array_equal(rgba.cpu().numpy().view(np.uint32), o_rgba)


@pytest.mark.parametrize("tsr", [0.0, 0.003])
def test_explicit_rays_edge_cases(menger_mm, cuda, tsr):
    torch = _torch()
    o, d = edge_rays()
    nodes, _ = menger_mm.getIncoreBuffer()
    dn = torch.from_numpy(nodes.view(np.int32)).to(cuda)
    do = torch.from_numpy(o).to(cuda)
    dd = torch.from_numpy(d).to(cuda)
    hits = torch.empty((o.shape[0] * 16,), dtype=torch.uint8, device=cuda)
    L.trace_rays(dn, nodes.shape[0], do, dd, o.shape[0], tsr, hits)
    torch.cuda.synchronize()
    o_hits, _ = oracle.cast_rays(nodes, o, d, tsr)
    assert_hits_equal(_hits_np(hits), o_hits, "edge rays")


def test_paged_pool_with_relative_indices(cuda):
    scene, mm = paged_menger_manager()
    mm.initDeviceBuffer()
    nodes, attribs = mm.getIncoreBuffer()
    assert (nodes[:, 0].view(np.int32) < 0).any(), "expected negative relative first-child indices"
    for seed in (7, 8):
        p = L.orbit_camera(seed, 256, 256, radius=1.4).frame_params(t_scale_ratio=0.0)
        rgba, hits = gpu_frame(mm, p)
        o_rgba, o_hits, _, _ = oracle.render(nodes, attribs, bytes(p))
        assert_hits_equal(hits, o_hits, "paged")
        assert np.array_equal(rgba, o_rgba)
    mm.close()


def test_bounds_errors_are_reported_not_faulted(cuda):
    torch = _torch()
    nodes = np.zeros((9, 2), dtype=np.uint32)
    nodes[0] = [1, 0xFF00]  # 8 valid inner children
    nodes[1:, 0] = 0x7FFFFFF0  # children point far outside the pool
    nodes[1:, 1] = 0xFF00
    attribs = np.zeros((9, 2), dtype=np.uint32)
    dn = torch.from_numpy(nodes.view(np.int32)).to(cuda)
    da = torch.from_numpy(attribs.view(np.int32)).to(cuda)
    p = L.orbit_camera(1, 64, 64, radius=1.3).frame_params(t_scale_ratio=0.0)
    rgba = torch.empty((64, 64), dtype=torch.int32, device=cuda)
    hits = torch.empty((64 * 64 * 16,), dtype=torch.uint8, device=cuda)
    stats = torch.zeros(4, dtype=torch.int32, device=cuda)
    L.render(dn, da, 9, p, rgba, hits, d_stats=stats)
    torch.cuda.synchronize()
    h = _hits_np(hits)
    o_rgba, o_hits, _, _ = oracle.render(nodes, attribs, bytes(p))
    assert_hits_equal(h, o_hits, "bounds")
    nb = int((h["flags"] == L.HITFLAG_BOUNDS).sum())
    assert nb > 0
    assert int(stats[1].item()) == nb


def test_mm_render_host_matches_device(menger_mm):
    menger_mm.sync()  # clear counters left by earlier tests
    p = L.orbit_camera(2, 300, 200).frame_params()
    host = menger_mm.render_host(p)
    rgba, _ = gpu_frame(menger_mm, p)
    assert np.array_equal(host, rgba)
    st = menger_mm.sync()
    assert st.capped_rays == 0 and st.bounds_errors == 0


@pytest.mark.parametrize("seed", range(6))
def test_random_octrees(cuda, seed):
    torch = _torch()
    nodes, attribs = random_octree_pool(seed, depth=4 + seed % 3)
    dn = torch.from_numpy(nodes.view(np.int32)).to(cuda)
    da = torch.from_numpy(attribs.view(np.int32)).to(cuda)
    p = L.orbit_camera(seed, 160, 120, radius=(1.0, 2.0)).frame_params(t_scale_ratio=0.0)
    rgba = torch.empty((p.height, p.width), dtype=torch.int32, device=cuda)
    hits = torch.empty((p.height * p.width * 16,), dtype=torch.uint8, device=cuda)
    L.render(dn, da, nodes.shape[0], p, rgba, hits)
    torch.cuda.synchronize()
    o_rgba, o_hits, _, _ = oracle.render(nodes, attribs, bytes(p))
    assert_hits_equal(_hits_np(hits), o_hits, "random octree")
    assert np.array_equal(rgba.cpu().numpy().view(np.uint32), o_rgba)


def test_icosphere_frame_matches_oracle(cuda):
    from libsvo_b200 import scenes

    wl = scenes.icosphere(subdivisions=5, depth=9, treelet_levels=4, width=480, height=270)
    info = wl.scene.info
    mm = L.TreeletMemoryManagerCuda(wl.scene, info.treelet_bytes * info.num_treelets)
    assert mm.insertAll() == info.num_treelets - 1
    mm.initDeviceBuffer()
    nodes, attribs = mm.getIncoreBuffer()
    for p in (wl.cameras[0].frame_params(), wl.cameras[0].frame_params(t_scale_ratio=0.0)):
        rgba, hits = gpu_frame(mm, p)
        o_rgba, o_hits, _, _ = oracle.render(nodes, attribs, bytes(p))
        assert_hits_equal(hits, o_hits, "icosphere")
        assert np.array_equal(rgba, o_rgba)
    mm.close()


def test_async_host_frames_match_device(menger_mm):
    """svo_mm_render_host_async: frames of different sizes in a row, each
    copied back on the second stream; every host image equals the device
    render, and the watchdog counters still add up."""
    import torch

    menger_mm.sync()
    frames = [L.orbit_camera(s, w, h).frame_params() for s, (w, h) in
              enumerate([(300, 200), (64, 48), (512, 512), (300, 200), (17, 13)])]
    outs = [torch.empty((p.height, p.width), dtype=torch.int32).pin_memory() for p in frames]
    for p, o in zip(frames, outs):
        menger_mm.render_host_async(p, o)
    st = menger_mm.sync()
    for p, o in zip(frames, outs):
        rgba, _ = gpu_frame(menger_mm, p)
        assert np.array_equal(o.numpy().view(np.uint32), rgba)
    assert st.bounds_errors == 0


def test_async_shadow_host_frames_match_device(menger_mm):
    """svo_mm_render_shadow_host_async, interleaved with
    svo_mm_render_host_async on the manager's two device images: frames of
    different sizes (one of a million pixels) in a row; every host image
    equals the device render of the same kind."""
    import torch

    menger_mm.sync()
    light = L.seeded_light(2)
    sc = L.shadow_cfg(light)
    frames = [(L.orbit_camera(s, w, h, radius=1.6).frame_params(), shadow) for s, (w, h, shadow) in
              enumerate([(300, 200, True), (64, 48, False), (1024, 1024, True), (300, 200, True), (17, 13, False)])]
    outs = [torch.empty((p.height, p.width), dtype=torch.int32).pin_memory() for p, _ in frames]
    for (p, shadow), o in zip(frames, outs):
        if shadow:
            menger_mm.render_shadow_host_async(p, o, sc)
        else:
            menger_mm.render_host_async(p, o)
    st = menger_mm.sync()
    nodes, attribs = menger_mm.getIncoreBuffer()
    for (p, shadow), o in zip(frames, outs):
        if shadow:
            want = torch.empty((p.height, p.width), dtype=torch.int32, device="cuda")
            menger_mm.render_shadow(p, want, sc)
            torch.cuda.synchronize()
            want = want.cpu().numpy().view(np.uint32)
            if p.width * p.height < 100_000:
                assert np.array_equal(want, oracle.render_shadow(nodes, attribs, bytes(p), light)[0])
        else:
            want, _ = gpu_frame(menger_mm, p)
        assert np.array_equal(o.numpy().view(np.uint32), want)
    assert st.bounds_errors == 0
    with pytest.raises(L.SvoError) as e:
        menger_mm.render_shadow_host_async(frames[0][0], outs[0], sc, cfg=L.trace_cfg(L.TRAVERSAL_FLAT))
    assert e.value.code == L.SVO_ERR_NOTSUP

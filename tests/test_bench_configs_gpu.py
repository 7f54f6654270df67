"""Bit-exact parity at the configurations bench.py measures, at full size
(the flat traversal of the headline view included).

* the headline frame: icosphere subdivided 6 times, depth-11 octree in
  6-level treelets, 1920x1080 (2,073,600 rays), every hit record field and
  the RGBA8 image against the oracle, and the image and the reference's own
  sample() results (node, t, depth, loops) against the reference's
  treeletRenderer_rgba.cl compiled for the host (oracle/_ref);
* the batched terrain views: the 64 views of uneven size cast in one
  autotuned batched launch; four of them (the smallest, two middle ones and
  the largest) carry hit records and are compared in full with the oracle,
  and all 64 images with the per-frame kernel's;
* the large primary + shadow frame: the icosphere subdivided 9 times (5.2 M
  triangles) built on the GPU, 3840x2160 primary rays and one shadow ray per
  hit, compared over a band of 96 rows, and the primary frame alone over
  three bands (top, middle, bottom rows).  The test uses the depth-12 octree
  (a 2.6 GB pool, copied to host memory for the CPU side); bench.py's
  large_shadowed measurement makes the same comparison over the depth-14
  pool (40.3 GB) when the host has the memory for its copy.
"""
import numpy as np
import pytest

import libsvo_b200 as L
import oracle

pytestmark = pytest.mark.gpu

FIELDS = ("node", "depth", "hit", "flags", "loops", "fetches")


def _hits(t):
    return t.cpu().numpy().view(np.uint8).view(L.HIT_DTYPE).reshape(-1)


def assert_hits_equal(got, want, what, fields=FIELDS):
    got = got.reshape(-1)
    want = want.reshape(-1)
    for k in fields:
        bad = np.nonzero(got[k] != want[k])[0]
        assert bad.size == 0, f"{what}: {k} differs at {bad.size} rays, first {bad[:5]}"
    bt = np.nonzero(got["t"].view(np.uint32) != want["t"].view(np.uint32))[0]
    assert bt.size == 0, f"{what}: t differs at {bt.size} rays, first {bt[:5]}"


def assert_matches_reference_sample(nodes, params, got, what):
    """The reference's own sample() on the frame's primary rays: node, t,
    depth, hit and loop count per ray (its records carry no fetch count and
    t only where it writes it)."""
    if oracle.reference_lib() is None:
        return
    o, d = oracle.pixel_rays(bytes(params))
    ref = oracle.reference_sample_rays(nodes, o, d, params.t_scale_ratio)
    got = got.reshape(-1)
    for k in ("node", "depth", "hit", "loops"):
        bad = np.nonzero(got[k] != ref[k])[0]
        assert bad.size == 0, f"{what} vs reference sample(): {k} differs at {bad.size} rays"
    defined = ref["hit"] == 1
    assert np.array_equal(got["t"][defined].view(np.uint32), ref["t"][defined].view(np.uint32))


def test_headline_frame_full_size(cuda):
    import torch

    from libsvo_b200 import scenes

    wl = scenes.icosphere()  # subdivisions 6, depth 11, 6-level treelets, 1920x1080
    info = wl.scene.info
    assert (wl.cameras[0].width, wl.cameras[0].height) == (1920, 1080)
    mm = L.TreeletMemoryManagerCuda(wl.scene, info.treelet_bytes * info.num_treelets)
    mm.insertAll()
    mm.initDeviceBuffer()
    nodes, attribs = mm.getIncoreBuffer()
    p = wl.cameras[0].frame_params()
    rgba = torch.empty((p.height, p.width), dtype=torch.int32, device=cuda)
    hits = torch.empty((p.height * p.width * 16,), dtype=torch.uint8, device=cuda)
    mm.render(p, rgba, hits, stream=torch.cuda.current_stream())
    torch.cuda.synchronize()
    got_rgba = rgba.cpu().numpy().view(np.uint32)
    got = _hits(hits)
    o_rgba, o_hits, _, _ = oracle.render(nodes, attribs, bytes(p))
    assert_hits_equal(got, o_hits, "icosphere 1080p")
    assert np.array_equal(got_rgba, o_rgba)
    assert got["hit"].sum() > 400_000
    ref = oracle.reference_render(nodes, attribs, bytes(p))
    if ref is not None:
        assert np.array_equal(got_rgba, oracle.to_rgba8(ref))
    assert_matches_reference_sample(nodes, p, got, "icosphere 1080p")
    mm.close()


def test_batched_terrain_views_full_size(cuda):
    import torch

    from libsvo_b200 import scenes

    wl = scenes.terrain()  # 1024^2 grid, depth 12, 64 views 256^2..2048^2
    info = wl.scene.info
    mm = L.TreeletMemoryManagerCuda(wl.scene, info.treelet_bytes * info.num_treelets)
    mm.insertAll()
    mm.initDeviceBuffer()
    nodes, attribs = mm.getIncoreBuffer()
    ps = [c.frame_params() for c in wl.cameras]
    assert len(ps) == 64
    order = sorted(range(len(ps)), key=lambda i: ps[i].width * ps[i].height)
    checked = [order[0], order[21], order[42], order[63]]
    outs = [torch.empty((p.height, p.width), dtype=torch.int32, device=cuda) for p in ps]
    hits = {i: torch.empty((ps[i].width * ps[i].height * 16,), dtype=torch.uint8, device=cuda)
            for i in checked}
    s = torch.cuda.current_stream()
    b = L.Batcher()
    # the autotuner picks the configuration on the batch without hit records,
    # as bench.py does; the checked launch then adds the records
    b.set([L.octree_of(mm)], [L.view_desc(p, 0, o) for p, o in zip(ps, outs)], L.batch_cfg(), stream=s)
    best, _ = b.autotune(reps=1, stream=s)
    b.set([L.octree_of(mm)], [L.view_desc(p, 0, o, hits.get(i)) for i, (p, o) in enumerate(zip(ps, outs))],
          best, stream=s)
    b.launch(stream=s)
    torch.cuda.synchronize()
    b.close()
    for i in checked:
        p = ps[i]
        o_rgba, o_hits, _, _ = oracle.render(nodes, attribs, bytes(p))
        got = _hits(hits[i])
        assert_hits_equal(got, o_hits, f"terrain view {i} ({p.width}x{p.height})")
        got_rgba = outs[i].cpu().numpy().view(np.uint32)
        assert np.array_equal(got_rgba, o_rgba), f"view {i}"
        ref = oracle.reference_render(nodes, attribs, bytes(p))
        if ref is not None:
            assert np.array_equal(got_rgba, oracle.to_rgba8(ref)), f"view {i} vs reference"
    assert sum(ps[i].width * ps[i].height for i in checked) > 4_000_000
    # all 64 views: the batched images equal the per-frame kernel's, bit for bit
    d_nodes, d_attribs, n = mm.getDeviceIncoreBuffer()
    for i, p in enumerate(ps):
        want = torch.empty((p.height, p.width), dtype=torch.int32, device=cuda)
        L.render(d_nodes, d_attribs, n, p, want)
        assert torch.equal(outs[i], want), f"view {i} ({p.width}x{p.height}) batched vs per-frame"
    mm.close()


def test_large_shadowed_frame_band(cuda):
    import torch

    from libsvo_b200 import scenes

    wl = scenes.large_shadowed(depth=12)  # the depth-14 pool is checked by bench.py
    d_nodes, d_attribs, n = wl.scene.buffers()
    p = wl.camera.frame_params()
    assert (p.width, p.height) == (3840, 2160)
    cfg = L.trace_cfg(L.TRAVERSAL_TREELET, wl.stack_size)
    sc = L.shadow_cfg(wl.light)
    px = p.width * p.height
    rgba = torch.empty((p.height, p.width), dtype=torch.int32, device=cuda)
    hb = torch.empty(px * 16, dtype=torch.uint8, device=cuda)
    sb = torch.empty(px * 16, dtype=torch.uint8, device=cuda)
    L.render_shadow(d_nodes, d_attribs, n, p, rgba, sc, hb, sb, cfg=cfg)
    torch.cuda.synchronize()
    y0, y1 = 1032, 1128  # 96 rows through the middle of the sphere
    got_rgba = rgba.cpu().numpy().view(np.uint32)[y0:y1]
    got = _hits(hb).reshape(p.height, p.width)[y0:y1]
    got_s = _hits(sb).reshape(p.height, p.width)[y0:y1]
    # the primary frame alone: 64,800 blocks cast in estimated-cost order
    # (the sort's per-block costs take 64 KB of shared memory)
    pb = torch.empty(px * 16, dtype=torch.uint8, device=cuda)
    L.render(d_nodes, d_attribs, n, p, rgba, pb, cfg=cfg)
    torch.cuda.synchronize()
    got_p = _hits(pb).reshape(p.height, p.width)
    nodes, attribs = wl.scene.getIncoreBuffer()
    wl.scene.close()
    o, d = oracle.pixel_rays(bytes(p))
    for r0, r1 in ((0, 16), (y0, y1), (p.height - 16, p.height)):
        sl = slice(r0 * p.width, r1 * p.width)
        want, _ = oracle.cast_rays(nodes, o[sl], d[sl], p.t_scale_ratio, stack_size=wl.stack_size)
        assert_hits_equal(got_p[r0:r1], want, f"large primary frame rows {r0}-{r1}")
    assert got_p[y0:y1]["hit"].sum() > 100_000
    o_rgba, o_hits, o_shadow, _, _ = oracle.render_shadow(nodes, attribs, bytes(p), wl.light,
                                                         stack_size=wl.stack_size, rows=(y0, y1))
    assert_hits_equal(got, o_hits, "large frame band, primary rays")
    assert_hits_equal(got_s, o_shadow, "large frame band, shadow rays")
    assert np.array_equal(got_rgba, o_rgba)
    assert got["hit"].sum() > 100_000 and got_s["hit"].sum() > 1000
    ref = oracle.reference_render_shadow(nodes, attribs, bytes(p), wl.light, rows=(y0, y1))
    if ref is not None:
        ref_rgbaf, ref_shadow = ref
        assert np.array_equal(got_rgba, oracle.to_rgba8(ref_rgbaf))
        for k in ("node", "depth", "hit", "loops"):
            assert np.array_equal(got_s[k], ref_shadow[k]), f"shadow rays vs reference sample(): {k}"


def test_flat_traversal_full_size(cuda):
    """The CpuRaycasterSingleRay3 traversal (flat breadth-first pool, absolute
    first-child indices, stack = the octree's depth) on the headline frame at
    full size: the depth-11 icosphere flattened (17.3 M nodes), 1920x1080,
    cast longest first, every hit record and pixel against the oracle's
    traversSvo restatement (parity unpinned: the reference's CPU raycaster
    does not build)."""
    import torch

    from libsvo_b200 import scenes

    wl = scenes.icosphere()
    depth = int(wl.scene.info.max_depth)
    nodes, attribs = wl.scene.flatten()
    dn = torch.from_numpy(nodes.view(np.int32)).to(cuda)
    da = torch.from_numpy(attribs.view(np.int32)).to(cuda)
    p = wl.cameras[0].frame_params()
    rgba = torch.empty((p.height, p.width), dtype=torch.int32, device=cuda)
    hits = torch.empty(p.width * p.height * 16, dtype=torch.uint8, device=cuda)
    L.render(dn, da, nodes.shape[0], p, rgba, hits, cfg=L.trace_cfg(L.TRAVERSAL_FLAT, depth))
    torch.cuda.synchronize()
    o_rgba, o_hits, _, _ = oracle.render(nodes, attribs, bytes(p), flat=True, stack_size=depth)
    assert_hits_equal(_hits(hits), o_hits, "flat icosphere 1080p")
    assert np.array_equal(rgba.cpu().numpy().view(np.uint32), o_rgba)
    assert _hits(hits)["hit"].sum() > 400_000


def test_analysis_records_full_size(cuda):
    """The analysis (feedback) kernel at full resolution on the headline frame
    — the pass that treelet-paged serving runs per request — over a partly
    resident pool (a third of the treelets, placed by two analysis steps):
    every 16-byte record against the oracle's renderToFeedbackBuffer, and
    against the reference's own sampleAnalyse where it was built."""
    import torch

    from libsvo_b200 import scenes

    wl = scenes.icosphere()
    info = wl.scene.info
    p = wl.cameras[0].frame_params()
    mm = L.TreeletMemoryManagerCuda(wl.scene, info.treelet_bytes * (info.num_treelets // 3))
    mm.setEviction(L.EVICT_ANY_UNSEEN)
    mm.initDeviceBuffer()
    for _ in range(2):
        mm.performAnalysePass(p, divisor=8)
    torch.cuda.synchronize()
    d_nodes, _, n = mm.getDeviceIncoreBuffer()
    nodes, _ = mm.getIncoreBuffer()
    fb = torch.empty(p.width * p.height * 16, dtype=torch.uint8, device=cuda)
    L.feedback_render(d_nodes, n, p, fb)
    torch.cuda.synchronize()
    got = fb.cpu().numpy().view(oracle.FEEDBACK_DTYPE).reshape(p.height, p.width)
    rec, _ = oracle.feedback(nodes, bytes(p))
    assert np.array_equal(got.view(np.uint8), rec.view(np.uint8))
    ref = oracle.reference_feedback(nodes, bytes(p))
    if ref is not None:
        assert np.array_equal(got.view(np.uint8), ref[0].view(np.uint8))
    mm.close()

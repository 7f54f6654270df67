"""Batched views: one persistent launch over a ragged table of views and
several octrees must give, view by view, the per-frame kernel's pixels and
hit records bit for bit (and the oracle's)."""
import numpy as np
import pytest

import libsvo_b200 as L
import oracle

pytestmark = pytest.mark.gpu


def _torch():
    import torch

    return torch


@pytest.fixture(scope="module")
def octrees(cuda):
    torch = _torch()
    out = {}
    s1 = L.Scene.menger(level=5, depth=8, seed=1)
    m1 = L.TreeletMemoryManagerCuda(s1, s1.info.treelet_bytes)
    m1.initDeviceBuffer()
    v, t = L.icosphere(4, seed=3)
    s2 = L.Scene.from_mesh(v, t, 8, treelet_levels=3)
    m2 = L.TreeletMemoryManagerCuda(s2, s2.info.treelet_bytes * s2.info.num_treelets)
    m2.insertAll()
    m2.initDeviceBuffer()
    fn, fa = L.Scene.menger(level=4, depth=7, seed=5).flatten()
    dn = torch.from_numpy(fn.view(np.int32)).to(cuda)
    da = torch.from_numpy(fa.view(np.int32)).to(cuda)
    out["descs"] = [L.octree_of(m1), L.octree_of(m2),
                    L.octree_desc(dn, da, fn.shape[0], L.TRAVERSAL_FLAT, 7)]
    out["host"] = [m1.getIncoreBuffer(), m2.getIncoreBuffer(), (fn, fa)]
    out["keep"] = [m1, m2, dn, da]
    yield out
    m1.close()
    m2.close()


VIEWS = [  # (octree, width, height, mode, seed, tsr)
    (0, 256, 256, 0, 1, None), (1, 1, 1, 0, 2, None), (1, 17, 13, 0, 3, 0.0), (0, 100, 37, 3, 4, None),
    (2, 64, 64, 0, 5, None), (1, 333, 211, 5, 6, None), (0, 8, 4, 0, 7, 0.0), (2, 120, 90, 4, 8, 0.0),
    (0, 512, 288, 0, 9, None), (1, 64, 300, 1, 10, None),
]


def make_views(cuda):
    torch = _torch()
    views, bufs, params = [], [], []
    for k, (o, w, h, mode, seed, tsr) in enumerate(VIEWS):
        p = L.orbit_camera(seed, w, h, radius=(1.3, 2.0)).frame_params(mode=mode, t_scale_ratio=tsr)
        rgba = torch.full((h, w), -1, dtype=torch.int32, device=cuda)
        hits = torch.zeros((h * w * 16,), dtype=torch.uint8, device=cuda) if k % 2 == 0 else None
        views.append(L.view_desc(p, o, rgba, hits))
        bufs.append((rgba, hits))
        params.append(p)
    return views, bufs, params


def per_frame(octrees, o, p, cuda):
    torch = _torch()
    d = octrees["descs"][o]
    rgba = torch.empty((p.height, p.width), dtype=torch.int32, device=cuda)
    hits = torch.empty((p.height * p.width * 16,), dtype=torch.uint8, device=cuda)
    L.render(d.d_nodes, d.d_attribs, d.num_nodes, p, rgba, hits,
             cfg=L.trace_cfg(d.traversal, d.stack_size))
    torch.cuda.synchronize()
    return rgba.cpu().numpy(), hits.cpu().numpy()


def check_batch(octrees, bufs, params, cuda, oracle_too=False):
    for k, ((rgba, hits), p) in enumerate(zip(bufs, params)):
        o = VIEWS[k][0]
        want_rgba, want_hits = per_frame(octrees, o, p, cuda)
        assert np.array_equal(rgba.cpu().numpy(), want_rgba), f"view {k}"
        if hits is not None:
            assert np.array_equal(hits.cpu().numpy(), want_hits), f"view {k} hits"
        if oracle_too:
            n, a = octrees["host"][o]
            d = octrees["descs"][o]
            o_rgba, _, _, _ = oracle.render(n, a, bytes(p), flat=d.traversal == L.TRAVERSAL_FLAT,
                                            stack_size=d.stack_size)
            assert np.array_equal(rgba.cpu().numpy().view(np.uint32), o_rgba), f"view {k} oracle"


@pytest.mark.parametrize("tile", [(8, 4), (16, 2), (4, 8), (32, 1)])
def test_mixed_batch_matches_per_frame(octrees, cuda, tile):
    torch = _torch()
    views, bufs, params = make_views(cuda)
    b = L.Batcher(max_views=64, max_octrees=8)
    stats = torch.zeros(4, dtype=torch.int32, device=cuda)
    b.set(octrees["descs"], views, L.batch_cfg(*tile, use_graph=False))
    b.launch(stats)
    torch.cuda.synchronize()
    check_batch(octrees, bufs, params, cuda, oracle_too=tile == (8, 4))
    tiles, rays = b.size()
    assert rays == sum(w * h for _, w, h, *_ in VIEWS)
    assert tiles >= rays // 32
    b.close()


@pytest.mark.parametrize("tile,rays_per_lane", [((8, 4), 2), ((16, 2), 4), ((32, 1), 4), ((4, 8), 2)])
def test_rays_per_lane_matches_per_frame(octrees, cuda, tile, rays_per_lane):
    """A lane casting 2 or 4 rays of a taller tile: same pixels and hit records
    as the per-frame kernel (views whose height is no multiple of the tile's
    included)."""
    torch = _torch()
    views, bufs, params = make_views(cuda)
    b = L.Batcher(max_views=64, max_octrees=8)
    b.set(octrees["descs"], views, L.batch_cfg(*tile, use_graph=False, rays_per_lane=rays_per_lane))
    b.launch()
    torch.cuda.synchronize()
    check_batch(octrees, bufs, params, cuda)
    tiles, rays = b.size()
    assert rays == sum(w * h for _, w, h, *_ in VIEWS)
    assert tiles >= rays // (32 * rays_per_lane)
    b.close()


def test_graph_replay_and_staged_top_nodes(octrees, cuda):
    torch = _torch()
    views, bufs, params = make_views(cuda)
    b = L.Batcher()
    b.set(octrees["descs"], views, L.batch_cfg(top_nodes=1024, block_threads=128, use_graph=True))
    for _ in range(3):
        for rgba, _ in bufs:
            rgba.fill_(-1)
        b.launch()
        torch.cuda.synchronize()
        check_batch(octrees, bufs, params, cuda)
    b.close()


def test_autotune_keeps_results(octrees, cuda):
    torch = _torch()
    views, bufs, params = make_views(cuda)
    b = L.Batcher()
    b.set(octrees["descs"], views, L.batch_cfg())
    best, ms = b.autotune(reps=2)
    assert ms > 0 and best.tile_w * best.tile_h == 32
    for rgba, _ in bufs:
        rgba.fill_(-1)
    b.launch()
    torch.cuda.synchronize()
    check_batch(octrees, bufs, params, cuda)
    b.close()


def test_batch_argument_errors(octrees, cuda):
    torch = _torch()
    views, bufs, params = make_views(cuda)
    b = L.Batcher(max_views=4, max_octrees=2)
    with pytest.raises(L.SvoError) as e:
        b.set(octrees["descs"], views)
    assert e.value.code == L.SVO_ERR_RANGE
    with pytest.raises(L.SvoError) as e:
        b.set(octrees["descs"][:2], views[:1], L.batch_cfg(rays_per_lane=3))
    assert e.value.code == L.SVO_ERR_RANGE
    bad = L.view_desc(params[0], 7, bufs[0][0])
    with pytest.raises(L.SvoError) as e:
        b.set(octrees["descs"][:2], [bad])
    assert e.value.code == L.SVO_ERR_INVALID
    with pytest.raises(L.SvoError) as e:
        b.launch()
    b.close()

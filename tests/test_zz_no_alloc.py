"""svo_render_batch_static: the batched cast for callers that may not
allocate device memory (their host owns all of HBM, or cudaMalloc/cudaFree
could stall their loop).  Its scratch is a fixed device array inside the
library, so this test calls it twice in a row through the C ABI and checks
both results against the allocating entry points (per-frame svo_render and
svo_batcher_launch), bit for bit like the other parity tests.

This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import libsvo_b200 as L

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pools():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    s1 = L.Scene.menger(level=4, depth=7, seed=11)
    m1 = L.TreeletMemoryManagerCuda(s1, s1.info.treelet_bytes)
    m1.initDeviceBuffer()
    v, t = L.icosphere(3, seed=5)
    s2 = L.Scene.from_mesh(v, t, 7, treelet_levels=3)
    m2 = L.TreeletMemoryManagerCuda(s2, s2.info.treelet_bytes * s2.info.num_treelets)
    m2.insertAll()
    m2.initDeviceBuffer()
    # a flat (CpuRaycasterSingleRay3) pool: absolute first-child indices, stack = depth
    fn, fa = s1.flatten()
    dn = torch.from_numpy(fn.view(np.int32)).cuda()
    da = torch.from_numpy(fa.view(np.int32)).cuda()
    flat = L.octree_desc(dn, da, fn.shape[0], L.TRAVERSAL_FLAT, int(s1.info.max_depth))
    yield [L.octree_of(m1), L.octree_of(m2), flat]
    m1.close()
    m2.close()
    del dn, da


# (octree, width, height, view mode, camera seed): the treelet pools in every
# view mode (2, 6 and 7 take the kernel's extended epilogue), the flat pool in
# the modes it supports, and a 1x1 view
SHAPES = [(0, 64, 64, 0, 1), (1, 17, 13, 0, 2), (0, 1, 1, 0, 3), (1, 200, 120, 3, 4), (0, 96, 40, 5, 5),
          (1, 80, 48, 2, 6), (0, 72, 56, 6, 7), (1, 64, 40, 7, 8), (2, 90, 70, 0, 9), (2, 40, 33, 2, 10),
          (1, 33, 65, 1, 11), (0, 48, 48, 4, 12)]


def _outputs(params, device="cuda"):
    import torch

    rgba = [torch.full((p.height, p.width), -1, dtype=torch.int32, device=device) for p in params]
    hits = [torch.full((p.height * p.width * 16,), 255, dtype=torch.uint8, device=device) for p in params]
    return rgba, hits


def test_static_batch_matches_allocating_entry_points(pools):
    import torch

    params = [L.orbit_camera(seed, w, h, radius=(1.3, 2.0)).frame_params(mode=mode)
              for _, w, h, mode, seed in SHAPES]
    # the per-frame entry point
    want = []
    for (o, *_), p in zip(SHAPES, params):
        out = torch.empty((p.height, p.width), dtype=torch.int32, device="cuda")
        d = pools[o]
        L.render(d.d_nodes, d.d_attribs, d.num_nodes, p, out, cfg=L.trace_cfg(d.traversal, d.stack_size))
        want.append(out)
    # the allocating batch entry point, with hit records and counters
    outs_b, hits_b = _outputs(params)
    stats_b = torch.zeros(4, dtype=torch.int32, device="cuda")
    b = L.Batcher(max_views=len(SHAPES), max_octrees=4)
    b.set(pools, [L.view_desc(p, o, t, h) for (o, *_), p, t, h in zip(SHAPES, params, outs_b, hits_b)],
          L.batch_cfg(use_graph=False))
    b.launch(d_stats=stats_b)
    torch.cuda.synchronize()
    for k, (w, got) in enumerate(zip(want, outs_b)):
        assert torch.equal(w, got), f"batcher, view {k}"
    b.close()
    # two calls in a row of the entry point that allocates nothing
    outs, hits = _outputs(params)
    views = [L.view_desc(p, o, t, h) for (o, *_), p, t, h in zip(SHAPES, params, outs, hits)]
    oa = (L.svo_octree_desc * len(pools))(*pools)
    va = (L.svo_view_desc * len(views))(*views)
    stats = torch.zeros(4, dtype=torch.int32, device="cuda")
    for call in range(2):
        for t in outs:
            t.fill_(-1)
        for h in hits:
            h.fill_(255)
        stats.zero_()
        rc = L.lib.svo_render_batch_static(oa, len(pools), va, len(views), 8, 4,
                                           stats.data_ptr(), None)
        assert rc == L.SVO_OK, f"call {call}: {rc}"
        torch.cuda.synchronize()
        for k, (w, got) in enumerate(zip(want, outs)):
            assert torch.equal(w, got), f"call {call}, view {k}"
        for k, (w, got) in enumerate(zip(hits_b, hits)):
            assert torch.equal(w, got), f"call {call}, hit records of view {k}"
        assert torch.equal(stats, stats_b), f"call {call}: counters {stats.tolist()} vs {stats_b.tolist()}"
    # another tile shape through the Python wrapper
    for t in outs:
        t.fill_(-1)
    L.render_batch_static(pools, views, tile=(16, 2))
    torch.cuda.synchronize()
    for w, got in zip(want, outs):
        assert torch.equal(w, got)


def test_static_batch_rejects_sizes_beyond_its_maximum(pools):
    p = L.orbit_camera(1, 8, 8).frame_params()
    views = (L.svo_view_desc * 257)(*[L.view_desc(p, 0, 1) for _ in range(257)])
    oa = (L.svo_octree_desc * len(pools))(*pools)
    assert L.lib.svo_render_batch_static(oa, len(pools), views, 257, 8, 4, None, None) == L.SVO_ERR_RANGE
    many = (L.svo_octree_desc * 17)(*([pools[0]] * 17))
    assert L.lib.svo_render_batch_static(many, 17, views, 1, 8, 4, None, None) == L.SVO_ERR_RANGE
    assert L.lib.svo_render_batch_static(oa, len(pools), views, 1, 5, 4, None, None) == L.SVO_ERR_NOTSUP

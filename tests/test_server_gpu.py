"""Serving: requests of uneven size over several octrees under an HBM budget.

Each request's pixels must be the same whether it is rendered alone (the
per-frame kernel on a fully resident octree) or served in the mix (batched
with others, while octrees are paged in and evicted), bit for bit."""
import numpy as np
import pytest

import libsvo_b200 as L
from libsvo_b200 import scenes as S

pytestmark = pytest.mark.gpu

SMALL = [("icosphere", 3, 7, 3, 1, 0.4), ("terrain", 65, 7, 3, 2, None),
         ("icosphere", 4, 8, 4, 3, 0.35), ("terrain", 129, 8, 4, 4, None)]


@pytest.fixture(scope="module")
def workload(cuda):
    return S.serving(SMALL)


def alone(scene, cam, cuda):
    import torch

    info = scene.info
    mm = L.TreeletMemoryManagerCuda(scene, info.treelet_bytes * info.num_treelets)
    mm.insertAll()
    mm.initDeviceBuffer()
    p = cam.frame_params()
    out = torch.empty((p.height, p.width), dtype=torch.int32, device=cuda)
    mm.render(p, out)
    torch.cuda.synchronize()
    mm.close()
    return out.cpu().numpy()


def footprint(scene):
    i = scene.info
    return 16 * i.treelet_bytes // 8 * i.num_treelets


@pytest.mark.parametrize("mode,upload", [(L.SERVE_BATCHED, None), (L.SERVE_PLAIN, None),
                                         (L.SERVE_PLAIN_STREAMED, None), (L.SERVE_BATCHED, L.UPLOAD_PINNED)])
def test_results_same_alone_and_in_the_mix(workload, cuda, mode, upload):
    """upload: octree loads as DMA copies from page-locked host copies."""
    import torch

    reqs = S.serving_requests(40, len(workload.scenes), seed=5, max_wh=(320, 200))
    # budget for about two of the four octrees: octrees page in and out
    budget = int(1.1 * (footprint(workload.scenes[2]) + footprint(workload.scenes[3])))
    srv = L.Server(L.server_cfg(budget, streams=3, max_batch_views=8, mode=mode))
    ids = [srv.add_octree(s) for s in workload.scenes]
    if upload is not None:
        for i in ids:
            srv.set_upload_policy(i, upload)
    outs, rq = [], []
    for o, cam in reqs:
        p = cam.frame_params()
        t = torch.full((p.height, p.width), -1, dtype=torch.int32, device=cuda)
        outs.append(t)
        rq.append(L.request(ids[o], p, t))
    arrivals = S.poisson_arrivals(len(rq), 2000.0, seed=1)
    res = srv.replay(rq, arrivals, timeout_ms=30000)
    assert all(r.status == L.SVO_OK for r in res)
    assert all(r.submit_s <= r.launch_s <= r.done_s for r in res)
    st = srv.stats()
    assert st.requests_done == len(rq)
    # the budget holds about two octrees: some had to be evicted to serve the rest
    assert st.octree_evictions > 0
    assert st.octree_loads >= len({o for o, _ in reqs})
    torch.cuda.synchronize()
    for (o, cam), t in zip(reqs, outs):
        assert np.array_equal(t.cpu().numpy(), alone(workload.scenes[o], cam, cuda))
    srv.close()


def test_batches_overlap_and_coalesce(workload, cuda):
    import torch

    reqs = S.serving_requests(60, len(workload.scenes), seed=9, max_wh=(256, 160))
    total = sum(footprint(s) for s in workload.scenes)
    srv = L.Server(L.server_cfg(2 * total, streams=4, max_batch_views=16))
    ids = [srv.add_octree(s) for s in workload.scenes]
    outs = [torch.empty((c.height, c.width), dtype=torch.int32, device=cuda) for _, c in reqs]
    rq = [L.request(ids[o], c.frame_params(), t) for (o, c), t in zip(reqs, outs)]
    res = srv.replay(rq, np.zeros(len(rq)), timeout_ms=30000)  # all at once
    assert all(r.status == L.SVO_OK for r in res)
    batches = {r.batch for r in res}
    assert len(batches) < len(rq)  # requests were batched together
    st = srv.stats()
    assert st.octree_evictions == 0 and st.octree_loads == len(set(o for o, _ in reqs))
    srv.close()


def test_cancel_wait_timeout_and_errors(workload, cuda):
    import torch

    total = sum(footprint(s) for s in workload.scenes)
    srv = L.Server(L.server_cfg(total, streams=1, max_batch_views=1, max_inflight_rays=1))
    oid = srv.add_octree(workload.scenes[0])
    cam = L.orbit_camera(1, 128, 128)
    out = torch.empty((128, 128), dtype=torch.int32, device=cuda)
    tickets = [srv.submit(L.request(oid, cam.frame_params(), out)) for _ in range(20)]
    # with one ray in flight at most, later requests are still pending
    assert srv.cancel(tickets[-1]) == L.SVO_OK
    r = srv.wait(tickets[-1])
    assert r.status == L.SVO_ERR_CANCELED
    for t in tickets[:-1]:
        assert srv.wait(t).status == L.SVO_OK
    with pytest.raises(L.SvoError) as e:
        srv.submit(L.request(99, cam.frame_params(), out))
    assert e.value.code == L.SVO_ERR_INVALID
    srv.close()
    # a budget too small for even two treelet slots of an octree: registration fails
    scene = workload.scenes[3]
    tiny = L.Server(L.server_cfg(2 * scene.info.treelet_bytes, streams=1))
    with pytest.raises(L.SvoError) as e:
        tiny.add_octree(scene)
    assert e.value.code == L.SVO_ERR_RANGE
    tiny.close()


def test_octree_larger_than_the_budget_is_paged(workload, cuda):
    """An octree whose pools exceed the whole budget is no longer refused: it
    is served by treelet paging in a quarter of the budget (an eighth of the
    octree), and close views of a small patch of it converge to the fully
    resident image."""
    import torch

    scene = workload.scenes[2]
    srv = L.Server(L.server_cfg(footprint(scene) // 2, streams=2))
    oid = srv.add_octree(scene)
    cams = [L.orbit_camera(k, 96, 64, radius=0.75, fov_deg=20.0) for k in range(3)]
    outs = [torch.full((c.height, c.width), -1, dtype=torch.int32, device=cuda) for c in cams]
    res = srv.replay([L.request(oid, c.frame_params(), t) for c, t in zip(cams, outs)], np.zeros(len(cams)),
                     timeout_ms=60000)
    assert all(r.status == L.SVO_OK for r in res)
    st = srv.stats()
    assert st.treelets_paged_in > 0 and st.octree_loads == 0 and st.paged_unconverged == 0
    torch.cuda.synchronize()
    for c, t in zip(cams, outs):
        assert np.array_equal(t.cpu().numpy(), alone(scene, c, cuda))
    srv.close()


@pytest.mark.parametrize("mode", [L.SERVE_BATCHED, L.SERVE_PLAIN_STREAMED])
def test_treelet_paged_octree_same_alone_and_in_the_mix(workload, cuda, mode):
    """The largest octree served by treelet paging in a region of 3/4 of its
    footprint, the others whole and paged in and out under the rest of the
    budget: every request's image equals its fully resident render, bit for
    bit (the paged requests' analysis passes run to convergence)."""
    import torch

    sizes = [footprint(s) for s in workload.scenes]
    big = int(np.argmax(sizes))
    others = sorted(sizes[i] for i in range(len(sizes)) if i != big)
    region = 3 * sizes[big] // 4
    budget = region + int(1.1 * (others[-1] + others[-2])) + (1 << 20)
    srv = L.Server(L.server_cfg(budget, streams=3, max_batch_views=8, mode=mode))
    ids = [srv.add_octree_paged(s, region) if i == big else srv.add_octree(s)
           for i, s in enumerate(workload.scenes)]
    reqs = S.serving_requests(36, len(workload.scenes), seed=21, max_wh=(256, 160))
    assert sum(o == big for o, _ in reqs) >= 5
    outs = [torch.full((c.height, c.width), -1, dtype=torch.int32, device=cuda) for _, c in reqs]
    rq = [L.request(ids[o], c.frame_params(), t) for (o, c), t in zip(reqs, outs)]
    res = srv.replay(rq, S.poisson_arrivals(len(rq), 1000.0, seed=2), timeout_ms=60000)
    assert all(r.status == L.SVO_OK for r in res)
    st = srv.stats()
    assert st.requests_done == len(rq) and st.treelets_paged_in > 0 and st.paged_unconverged == 0
    # every paged request ran at least one analysis pass (one that asks for
    # nothing more ends it), and the passes were timed
    assert st.analysis_passes >= sum(o == big for o, _ in reqs) and st.paging_us > 0
    torch.cuda.synchronize()
    for (o, cam), t in zip(reqs, outs):
        assert np.array_equal(t.cpu().numpy(), alone(workload.scenes[o], cam, cuda)), f"octree {o}"
    srv.close()


@pytest.mark.parametrize("mode", [L.SERVE_BATCHED, L.SERVE_PLAIN_STREAMED])
def test_repeated_create_serve_destroy(workload, cuda, mode):
    """Teardown right after the last completion, many times over: the server
    must outlive its stream callbacks (batched) and its events (streamed)."""
    import torch

    total = sum(footprint(s) for s in workload.scenes)
    cams = [L.orbit_camera(k, 48 + 8 * k, 40, radius=1.6) for k in range(12)]
    outs = [torch.empty((c.height, c.width), dtype=torch.int32, device=cuda) for c in cams]
    for cycle in range(15):
        srv = L.Server(L.server_cfg(total, streams=4, max_batch_views=3, mode=mode))
        oid = srv.add_octree(workload.scenes[cycle % len(workload.scenes)])
        res = srv.replay([L.request(oid, c.frame_params(), t) for c, t in zip(cams, outs)],
                         np.zeros(len(cams)), timeout_ms=20000)
        assert all(r.status == L.SVO_OK for r in res)
        srv.close()

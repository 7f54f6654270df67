"""Analysis pass on the GPU: the feedback kernel against the oracle bit for
bit, and visibility-driven paging converging to the fully resident image."""
import numpy as np
import pytest

import libsvo_b200 as L
import oracle
from test_oracle_pinning import partially_resident_menger

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_feedback_kernel_matches_oracle(cuda, seed):
    import torch

    _, mm, _ = partially_resident_menger()
    mm.initDeviceBuffer()
    d_nodes, _, n = mm.getDeviceIncoreBuffer()
    nodes, _ = mm.getIncoreBuffer()
    for tsr in (0.0, None):
        p = L.orbit_camera(seed, 150, 100, radius=(1.2, 2.0)).frame_params(t_scale_ratio=tsr)
        fb = torch.empty(p.width * p.height * 16, dtype=torch.uint8, device=cuda)
        img = torch.empty((p.height, p.width), dtype=torch.int32, device=cuda)
        L.feedback_render(d_nodes, n, p, fb, img)
        torch.cuda.synchronize()
        rec, rgbaf = oracle.feedback(nodes, bytes(p))
        got = fb.cpu().numpy().view(oracle.FEEDBACK_DTYPE).reshape(p.height, p.width)
        assert np.array_equal(got.view(np.uint8), rec.view(np.uint8))
        assert np.array_equal(img.cpu().numpy().view(np.uint32), oracle.to_rgba8(rgbaf))
    mm.close()


def render(mm, p, cuda):
    import torch

    rgba = torch.empty((p.height, p.width), dtype=torch.int32, device=cuda)
    hits = torch.empty(p.width * p.height * 16, dtype=torch.uint8, device=cuda)
    mm.render(p, rgba, hits)
    torch.cuda.synchronize()
    return rgba.cpu().numpy(), hits.cpu().numpy().view(L.HIT_DTYPE)


@pytest.mark.parametrize("scene_kind", ["menger", "icosphere"])
def test_paging_by_analysis_converges_to_full_residency(cuda, scene_kind):
    if scene_kind == "menger":
        scene = L.Scene.menger(level=4, depth=7, seed=3, treelet_levels=3)
        cam = L.orbit_camera(5, 160, 120, radius=1.5)
    else:
        v, t = L.icosphere(4, seed=2)
        scene = L.Scene.from_mesh(v, t, 8, treelet_levels=3)
        cam = L.orbit_camera(6, 160, 120, radius=1.6)
    info = scene.info
    p = cam.frame_params(t_scale_ratio=0.0)
    full = L.TreeletMemoryManagerCuda(scene, info.treelet_bytes * info.num_treelets)
    full.insertAll()
    full.initDeviceBuffer()
    want_rgba, want_hits = render(full, p, cuda)
    full.close()

    mm = L.TreeletMemoryManagerCuda(scene, info.treelet_bytes * info.num_treelets)
    mm.initDeviceBuffer()  # only the root treelet is resident
    steps, loaded = 0, 0
    while steps < 60:
        new, old = mm.performAnalysePass(p, divisor=1)
        steps += 1
        loaded += new
        if new == 0:
            break
    assert new == 0 and 0 < loaded < info.num_treelets
    got_rgba, got_hits = render(mm, p, cuda)
    assert np.array_equal(got_rgba, want_rgba)
    for k in ("hit", "depth", "loops"):
        assert np.array_equal(got_hits[k], want_hits[k])
    assert np.array_equal(got_hits["t"].view(np.uint32), want_hits["t"].view(np.uint32))
    # the reference's defaults: 1/8 resolution with jittered far plane
    mm.resetIncoreBuffer()
    rng = np.random.default_rng(1)
    total = 0
    for _ in range(8):
        new, _ = mm.performAnalysePass(p, divisor=8, jitter=tuple(rng.uniform(-1, 1, 2)))
        total += new
    assert total > 0
    mm.close()


def test_analysis_steps_under_memory_pressure(cuda):
    """A pool far smaller than the visible treelets: every step evicts to make
    room, some treelets find no slot or lose their parent to an eviction of
    the same step and are skipped (the reference ignores those insertion
    failures too), and every frame still matches the oracle on the manager's
    host mirror."""
    scene = L.Scene.menger(level=4, depth=7, seed=5, treelet_levels=2)
    info = scene.info
    mm = L.TreeletMemoryManagerCuda(scene, info.treelet_bytes * 40)
    mm.initDeviceBuffer()
    total = 0
    for f in range(20):
        p = L.orbit_camera(100 + f, 96, 80, radius=(1.1, 1.8)).frame_params(t_scale_ratio=0.0)
        new, _ = mm.performAnalysePass(p, divisor=2)
        total += new
        rgba, hits = render(mm, p, cuda)
        nodes, attribs = mm.getIncoreBuffer()
        o_rgba, o_hits, _, _ = oracle.render(nodes, attribs, bytes(p))
        assert np.array_equal(rgba.view(np.uint32), o_rgba), f"frame {f}"
        assert np.array_equal(hits["node"], o_hits.reshape(-1)["node"])
        assert mm.info.free_slots <= 40
    # the pool ran full: the later steps placed treelets only by eviction
    assert mm.info.free_slots == 0 and total >= 39
    mm.close()


@pytest.mark.parametrize("policy", [L.UPLOAD_COALESCED, L.UPLOAD_PINNED])
def test_pipelined_analysis_gives_the_sequential_frames(cuda, policy):
    """The analysis of view k+1 begun beside the cast of frame k (another
    stream) and ended after it: every frame and the counts of placed treelets
    equal the sequential loop's (analysis step, then frame), under paging
    with eviction in a buffer much smaller than the octree."""
    import torch

    v, t = L.icosphere(4, seed=2)
    scene = L.Scene.from_mesh(v, t, 8, treelet_levels=3)
    info = scene.info
    slots = max(8, info.num_treelets // 3)
    from libsvo_b200 import scenes as S

    poses = [S.orbit_pose(2.2 - 0.04 * f, 9.0 * f, 15.0, 192, 128, 30.0).frame_params(t_scale_ratio=0.0)
             for f in range(24)]

    def loop(pipelined):
        mm = L.TreeletMemoryManagerCuda(scene, info.treelet_bytes * slots)
        mm.setUploadPolicy(policy)
        mm.setEviction(L.EVICT_ANY_UNSEEN)
        mm.initDeviceBuffer()
        s, sa = torch.cuda.Stream(), torch.cuda.Stream()
        outs = [torch.empty((p.height, p.width), dtype=torch.int32, device=cuda) for p in poses]
        placed = []
        for p, o in zip(poses, outs):
            if pipelined:
                mm.beginAnalysePass(p, divisor=4, stream=sa)
                placed.append(mm.endAnalysePass(after_stream=s))
            else:
                placed.append(mm.performAnalysePass(p, divisor=4, stream=s))
            mm.render(p, o, stream=s)
        s.synchronize()
        frames = [o.cpu().numpy() for o in outs]
        mm.close()
        return frames, placed

    seq, seq_placed = loop(False)
    pipe, pipe_placed = loop(True)
    assert seq_placed == pipe_placed
    assert sum(n for n, _ in seq_placed) > slots  # treelets were evicted and paged in again
    for k, (a, b) in enumerate(zip(seq, pipe)):
        assert np.array_equal(a, b), f"frame {k}"


def test_analysis_halves_misuse(cuda):
    scene = L.Scene.menger(level=3, depth=6, seed=9, treelet_levels=2)
    mm = L.TreeletMemoryManagerCuda(scene, scene.info.treelet_bytes * 8)
    mm.initDeviceBuffer()
    p = L.orbit_camera(1, 64, 64, radius=1.6).frame_params()
    with pytest.raises(L.SvoError) as e:
        mm.endAnalysePass()
    assert e.value.code == L.SVO_ERR_INVALID
    mm.beginAnalysePass(p, divisor=4)
    with pytest.raises(L.SvoError) as e:
        mm.beginAnalysePass(p, divisor=4)
    assert e.value.code == L.SVO_ERR_BUSY
    # the slots may not change while the analysis is pending
    top = [g for g in range(1, scene.info.num_treelets) if scene.treelet(g)["parent_gid"] == 0]
    assert not mm.insertTreeletIntoIncoreBuffer(top[0])
    assert mm.updateClientSideIncoreBuffer([top[0]]) == L.SVO_ERR_BUSY
    mm.endAnalysePass()
    assert mm.updateClientSideIncoreBuffer([], None, [0]) == L.SVO_OK  # accepted again
    mm.close()

"""Randomised GPU parity: random octrees, cameras inside and outside the
root cube, odd frame sizes, random LOD ratios and view modes, through the
per-frame kernel, the shadow frame and one batched launch over all views;
every hit record bit for bit against the oracle, pixels exact (1 LSB for the
pow-based view modes 2 and 6)."""
import numpy as np
import pytest

import libsvo_b200 as L
import oracle
from rays import random_octree_pool
from test_render_gpu import _hits_np, assert_hits_equal
from test_shading_gpu import LSB_TOLERANCE, assert_rgba_close

pytestmark = pytest.mark.gpu

SEEDS = range(12)


def random_view(rng, seed):
    w, h = int(rng.integers(1, 200)), int(rng.integers(1, 160))
    radius = (0.05, 0.45) if seed % 3 == 0 else (0.8, 3.0)  # every third camera inside the cube
    cam = L.orbit_camera(1000 + seed, w, h, radius=radius, fov_deg=float(rng.uniform(20, 100)))
    tsr = [0.0, None, float(rng.uniform(0.001, 0.05))][seed % 3]
    mode = int(rng.choice([0, 1, 2, 3, 4, 5, 6, 7]))
    return cam.frame_params(mode=mode, t_scale_ratio=tsr)


def check_frame(got_rgba, got_hits, nodes, attribs, p, stack_size=13):
    o_rgba, o_hits, _, _ = oracle.render(nodes, attribs, bytes(p), stack_size=stack_size)
    o_hits = o_hits.reshape(-1)
    assert_hits_equal(got_hits, o_hits, f"mode {p.mode}")
    tol = LSB_TOLERANCE if p.mode in (2, 6) else 0
    assert_rgba_close(got_rgba, o_rgba, tol, f"mode {p.mode}")


@pytest.mark.parametrize("seed", SEEDS)
def test_random_frames(cuda, seed):
    import torch

    rng = np.random.default_rng(seed)
    nodes, attribs = random_octree_pool(seed, depth=3 + seed % 5, fill=float(rng.uniform(0.2, 0.7)))
    dn = torch.from_numpy(nodes.view(np.int32)).to(cuda)
    da = torch.from_numpy(attribs.view(np.int32)).to(cuda)
    p = random_view(rng, seed)
    rgba = torch.empty((p.height, p.width), dtype=torch.int32, device=cuda)
    hits = torch.empty((p.height * p.width * 16,), dtype=torch.uint8, device=cuda)
    L.render(dn, da, nodes.shape[0], p, rgba, hits)
    torch.cuda.synchronize()
    check_frame(rgba.cpu().numpy().view(np.uint32), _hits_np(hits), nodes, attribs, p)
    # the shadow frame of the same view
    light = L.seeded_light(seed)
    sh = torch.empty_like(hits)
    L.render_shadow(dn, da, nodes.shape[0], p, rgba, L.shadow_cfg(light, 0.0, 0.03), hits, sh)
    torch.cuda.synchronize()
    o_rgba, o_hits, o_sh, _, _ = oracle.render_shadow(nodes, attribs, bytes(p), light, 0.0, 0.03)
    assert_hits_equal(_hits_np(hits), o_hits.reshape(-1), "shadow primary")
    assert_hits_equal(_hits_np(sh), o_sh.reshape(-1), "shadow rays")
    assert np.array_equal(rgba.cpu().numpy().view(np.uint32), o_rgba)


def test_random_views_in_one_batch(cuda):
    """All random views of the frames above, over their own octrees, as one
    batched launch, all view modes mixed; then the same table without the
    modes that need the extended instantiation."""
    import torch

    descs, views, checks, keep = [], [], [], []
    for seed in SEEDS:
        rng = np.random.default_rng(seed)
        nodes, attribs = random_octree_pool(seed, depth=3 + seed % 5, fill=float(rng.uniform(0.2, 0.7)))
        p = random_view(rng, seed)
        dn = torch.from_numpy(nodes.view(np.int32)).to(cuda)
        da = torch.from_numpy(attribs.view(np.int32)).to(cuda)
        rgba = torch.empty((p.height, p.width), dtype=torch.int32, device=cuda)
        hits = torch.empty((p.height * p.width * 16,), dtype=torch.uint8, device=cuda)
        descs.append(L.octree_desc(dn, da, nodes.shape[0]))
        views.append(L.view_desc(p, len(descs) - 1, rgba, hits))
        checks.append((nodes, attribs, p, rgba, hits))
        keep += [dn, da]
    b = L.Batcher(max_views=64, max_octrees=64)
    b.set(descs, views, L.batch_cfg(tile_w=8, tile_h=4))
    b.launch()
    torch.cuda.synchronize()
    for nodes, attribs, p, rgba, hits in checks:
        check_frame(rgba.cpu().numpy().view(np.uint32), _hits_np(hits), nodes, attribs, p)
    assert any(c[2].mode in (2, 6, 7) for c in checks)
    for v, c in zip(views, checks):  # modes 0-5 only: the plain instantiation
        if c[2].mode in (2, 6, 7):
            v.params.mode = c[2].mode = 0
    b.set(descs, views, L.batch_cfg(tile_w=16, tile_h=2))
    b.launch()
    torch.cuda.synchronize()
    for nodes, attribs, p, rgba, hits in checks:
        check_frame(rgba.cpu().numpy().view(np.uint32), _hits_np(hits), nodes, attribs, p)
    b.close()

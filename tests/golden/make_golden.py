"""Generates the golden fixtures in this directory from the reference's own
ray cast (opencl/treeletRenderer_rgba.cl compiled for the host by
oracle/build_ref.py).  Needs the reference checkout; run from the repo root:

    python tests/golden/make_golden.py

Each fixture holds a node/attribute pool, frame parameters and rays, and the
reference's outputs for them: renderToBuffer's float RGBA per pixel and
sample()'s hit record per ray (node index, t, depth, hit, loop count).  Some
also hold shadow frames: the shadow shading over the reference's own sample()
(oracle/ref_harness.inc) with its float RGBA and shadow-ray hit records.
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import libsvo_b200 as L  # noqa: E402
import oracle  # noqa: E402
from rays import edge_rays, paged_menger_manager, random_octree_pool  # noqa: E402

HERE = Path(__file__).resolve().parent


def fixture(name, nodes, attribs, frames, rays, tsrs, feedback_frames=(), shadow_frames=()):
    oracle.build_reference()
    assert oracle.reference_lib() is not None, "reference build missing"
    out = {"nodes": nodes, "attribs": attribs}
    for i, p in enumerate(frames):
        out[f"params_{i}"] = np.frombuffer(bytes(p), dtype=np.uint8)
        out[f"rgbaf_{i}"] = oracle.reference_render(nodes, attribs, bytes(p))
    o, d = rays
    out["origins"], out["dirs"] = o, d
    for j, tsr in enumerate(tsrs):
        h = oracle.reference_sample_rays(nodes, o, d, tsr)
        out[f"tsr_{j}"] = np.float32(tsr)
        for k in ("node", "t", "depth", "hit", "loops"):
            out[f"hits_{j}_{k}"] = h[k]
    for k, p in enumerate(feedback_frames):
        out[f"fb_params_{k}"] = np.frombuffer(bytes(p), dtype=np.uint8)
        rec, img = oracle.reference_feedback(nodes, bytes(p))
        out[f"fb_rec_{k}"] = rec.view(np.uint8)
        out[f"fb_img_{k}"] = img
    for k, (p, light, tsr, offset) in enumerate(shadow_frames):
        light = np.asarray(light, dtype=np.float32)
        out[f"sh_params_{k}"] = np.frombuffer(bytes(p), dtype=np.uint8)
        out[f"sh_light_{k}"] = light
        out[f"sh_tsr_{k}"] = np.float32(tsr)
        out[f"sh_offset_{k}"] = np.float32(offset)
        rgbaf, shits = oracle.reference_render_shadow(nodes, attribs, bytes(p), light, tsr, offset)
        out[f"sh_rgbaf_{k}"] = rgbaf
        out[f"sh_hits_{k}"] = shits.view(np.uint8)
    np.savez_compressed(HERE / f"{name}.npz", **out)
    print(name, sum(v.nbytes for v in out.values() if hasattr(v, "nbytes")), "bytes raw")


def main():
    s = L.Scene.menger(level=3, depth=5, seed=7)
    mm = L.TreeletMemoryManagerCuda(s, s.info.treelet_bytes)
    n, a = mm.getIncoreBuffer()
    cams = [L.orbit_camera(1, 64, 48, radius=1.6), L.orbit_camera(2, 40, 40, radius=1.2)]
    frames = [cams[0].frame_params(), cams[0].frame_params(t_scale_ratio=0.0),
              cams[1].frame_params(mode=3), cams[1].frame_params(mode=5, t_scale_ratio=0.01),
              cams[0].frame_params(mode=2), cams[0].frame_params(mode=6),
              cams[1].frame_params(mode=7), cams[1].frame_params(mode=7, t_scale_ratio=0.02)]
    shadows = [(cams[0].frame_params(), L.default_light(), 0.001, 0.04),
               (cams[1].frame_params(t_scale_ratio=0.0), L.seeded_light(3), 0.0, 0.05)]
    fixture("menger_l3_d5", n, a, frames, edge_rays(n_random=3000, seed=1), [0.0, 0.004],
            shadow_frames=shadows)

    n, a = random_octree_pool(11, depth=5)
    cam = L.orbit_camera(3, 48, 48, radius=(1.0, 2.0))
    frames = [cam.frame_params(t_scale_ratio=0.0), cam.frame_params(mode=6),
              cam.frame_params(mode=7, t_scale_ratio=0.01)]
    fixture("random_d5", n, a, frames, edge_rays(n_random=2000, seed=2), [0.0, 0.01],
            shadow_frames=[(cam.frame_params(t_scale_ratio=0.0), L.seeded_light(11), 0.0, 0.02)])

    _, mm = paged_menger_manager()
    n, a = mm.getIncoreBuffer()
    frames = [L.orbit_camera(7, 64, 64, radius=1.4).frame_params(t_scale_ratio=0.0)]
    fixture("menger_paged", n, a, frames, edge_rays(n_random=2000, seed=3), [0.0])

    # analysis pass over a partially resident pool (sub-treelet gids appear)
    from test_oracle_pinning import partially_resident_menger

    _, mm, _ = partially_resident_menger()
    n, a = mm.getIncoreBuffer()
    cam = L.orbit_camera(3, 48, 40, radius=1.3)
    fixture("menger_partial", n, a, [cam.frame_params(t_scale_ratio=0.0)],
            edge_rays(n_random=1000, seed=4), [0.0],
            feedback_frames=[cam.frame_params(t_scale_ratio=0.0), cam.frame_params()])


if __name__ == "__main__":
    main()

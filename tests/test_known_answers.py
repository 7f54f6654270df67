"""Known-answer tests: hand-built pools whose results follow from the
geometry alone, checked on the oracle, on the reference's own sample()
(when its host build is present), on the kernels' traversal built for the
host, and (marked gpu) on the device.

Pools are in the incore layout: node i = {first child relative to i, masks}
with valid bits 8-15 and leaf bits 0-7; child c of a node is
node + first + popcount(valid bits below c), child index 4x + 2y + z.
"""
import numpy as np
import pytest

import libsvo_b200 as L
import oracle
from test_traverse_host import check as host_check, host_lib  # noqa: F401  (fixture)


def one_node_pool():
    return np.array([[0, 0]], dtype=np.uint32)


def depth1_pool(valid_mask):
    """A root whose valid children are all leaves, stored right after it."""
    n = bin(valid_mask).count("1")
    nodes = np.zeros((1 + n, 2), dtype=np.uint32)
    nodes[0] = [1, (valid_mask << 8) | valid_mask]
    return nodes


def rays(*pairs):
    o = np.array([p[0] for p in pairs], dtype=np.float32)
    d = np.array([p[1] for p in pairs], dtype=np.float64)
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    return o, d


TILT = (1e-3, 1e-3, -1.0)  # a ray down the z axis, tilted so that no component is zero


# (pool, ray origin, ray direction, expected (hit, node, t, depth))
CASES = [
    # nothing below the root: a miss that reports the root box's exit distance
    ("one node", one_node_pool(), (0.0, 0.0, 2.0), (0.0, 0.0, -1.0), (0, 0, 2.5, 0)),
    # all eight children: the ray down the z axis at x, y < 0 enters child 1 (z high) first
    ("full depth 1", depth1_pool(0xFF), (-0.25, -0.25, 2.0), (0.0, 0.0, -1.0), (1, 2, 1.5, 1)),
    # child 0 missing: child 1 is then node 1
    ("child 0 missing", depth1_pool(0xFE), (-0.25, -0.25, 2.0), (0.0, 0.0, -1.0), (1, 1, 1.5, 1)),
    # child 1 missing: the ray passes its octant and hits child 0 at the z = 0 plane
    ("child 1 missing", depth1_pool(0xFD), (-0.25, -0.25, 2.0), TILT, (1, 1, 2.0, 1)),
    # the same ray exactly along the axis: OpenCL sign(0) = 0 leaves the zero
    # direction components at 0 (sample(), :231-239), their reciprocals are
    # infinite, the slab distances NaN, and the advance past child 1 leaves
    # the root box: the reference reports a miss at the exit distance
    ("axis ray, NaN slabs", depth1_pool(0xFD), (-0.25, -0.25, 2.0), (0.0, 0.0, -1.0), (0, 0, 2.5, 0)),
    # a ray starting inside the cube: sample() starts at the root box's entry
    # behind the origin, so the leaf behind the origin (child 6) is the hit
    ("origin inside", depth1_pool(0xFF), (0.25, 0.25, 0.25), (0.0, 0.0, 1.0), (1, 7, -0.75, 1)),
    # an axis-parallel ray missing the cube entirely
    ("box miss", depth1_pool(0xFF), (0.75, 0.0, 2.0), (0.0, 0.0, -1.0), (0, 0, 0.0, 0)),
]


@pytest.mark.parametrize("name,pool,o,d,want", CASES, ids=[c[0] for c in CASES])
def test_oracle_known_answers(name, pool, o, d, want):
    ro, rd = rays((o, d))
    h, _ = oracle.cast_rays(pool, ro, rd, 0.0)
    assert_answer(h, want, name)
    ref = oracle.reference_sample_rays(pool, ro, rd, 0.0)
    if ref is not None:
        if name == "box miss":  # sample() leaves t unwritten on a box miss
            ref["t"] = 0.0
        assert_answer(ref, want, name)


def assert_answer(h, want, what):
    got = (int(h["hit"][0]), int(h["node"][0]), int(h["depth"][0]))
    assert got == (want[0], want[1], want[3]), f"{what}: {got}"
    # exact for the axis-aligned rays; the tilted ray's distance to the z = 0
    # plane is 2 / |d_z| with |d_z| = 1 / sqrt(1 + 2e-6)
    assert float(h["t"][0]) == pytest.approx(want[2], rel=2e-6), what


@pytest.mark.parametrize("name,pool,o,d,want", CASES, ids=[c[0] for c in CASES])
def test_kernel_traversal_known_answers(host_lib, name, pool, o, d, want):  # noqa: F811
    ro, rd = rays((o, d))
    h = host_check(host_lib, pool, ro, rd, 0.0)
    assert_answer(h, want, name)


@pytest.mark.gpu
def test_device_known_answers(cuda):
    import torch

    for name, pool, o, d, want in CASES:
        ro, rd = rays((o, d))
        dn = torch.from_numpy(pool.view(np.int32)).to(cuda)
        do, dd = torch.from_numpy(ro).to(cuda), torch.from_numpy(rd).to(cuda)
        hits = torch.empty(16, dtype=torch.uint8, device=cuda)
        L.trace_rays(dn, pool.shape[0], do, dd, 1, 0.0, hits)
        torch.cuda.synchronize()
        h = hits.cpu().numpy().view(L.HIT_DTYPE)
        assert_answer(h, want, name)

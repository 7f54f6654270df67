"""Shared test inputs: edge-case ray sets and paged treelet pools."""
import numpy as np

import libsvo_b200 as L


def edge_rays(n_random=20000, seed=0):
    """Axis-aligned, zero-component, grazing, inside-the-cube, -0.0-origin and
    random rays."""
    rng = np.random.default_rng(seed)
    o, d = [], []
    for origin in ([0.1, 0.2, 3.0], [0.0, 0.0, 2.0], [0.0, 0.0, 0.0], [0.25, -0.25, 0.1],
                   [0.5, 0.5, 2.0], [-0.5, 0.3, -3.0], [-0.0, 0.25, 2.0], [-0.0, -0.0, -2.5]):
        for dirv in ([0, 0, -1], [0, 0, 1], [1, 0, 0], [0, -1, 0], [0, 0.00005, -1], [1e-6, 0, -1],
                     [-0.0, 0.0, -1.0], [0.3, 0.4, -0.866], [-0.3, -0.2, 0.9], [-0.01, 0.02, -1.0]):
            o.append(origin)
            v = np.asarray(dirv, dtype=np.float64)
            d.append(v / np.linalg.norm(v))
    for s in np.linspace(-0.5, 0.5, 11):
        o.append([s, 0.5, 2.0]); d.append([0.0, 0.0, -1.0])
        o.append([0.5, s, -2.0]); d.append([0.0, 0.0, 1.0])
        o.append([-2.0, s, s]); d.append([1.0, 0.0, 0.0])
    eo = rng.normal(size=(n_random, 3))
    eo = eo / np.linalg.norm(eo, axis=1, keepdims=True) * rng.uniform(0.0, 2.5, size=(n_random, 1))
    tgt = rng.uniform(-0.5, 0.5, size=(n_random, 3))
    ed = tgt - eo
    ed /= np.linalg.norm(ed, axis=1, keepdims=True)
    o = np.concatenate([np.asarray(o, dtype=np.float64), eo]).astype(np.float32)
    d = np.concatenate([np.asarray(d, dtype=np.float64), ed]).astype(np.float32)
    return o, d


def paged_menger_manager():
    """A Menger octree cut into 3-level treelets and paged so that child
    treelets sit in slots below their parents: first-child deltas are then
    negative and the index arithmetic wraps mod 2^32."""
    scene = L.Scene.menger(level=4, depth=7, seed=3, treelet_levels=3)
    ntl = scene.info.num_treelets
    parents = np.array([scene.treelet(g)["parent_gid"] for g in range(ntl)])
    top = [g for g in range(1, ntl) if parents[g] == 0]
    mm = L.TreeletMemoryManagerCuda(scene, scene.info.treelet_bytes * ntl)
    for g in top:
        assert mm.insertTreeletIntoIncoreBuffer(g)
    # free the low slots of the first few top treelets, then page in the
    # children of the last ones: they land below their parents
    k = min(8, len(top) // 2)
    for g in top[:k]:
        assert mm.removeTreeletFromIncoreBuffer(g)
    for g in top[::-1][:k]:
        for c in np.nonzero(parents == g)[0]:
            if c != 0:
                assert mm.insertTreeletIntoIncoreBuffer(int(c))
    for g in top[:k]:
        assert mm.insertTreeletIntoIncoreBuffer(g)
    return scene, mm


def random_octree_pool(seed, depth=5, fill=0.5):
    """A random octree serialised breadth first into one treelet pool with
    relative first-child indices (the TreeletBuilderFromFaces layout)."""
    rng = np.random.default_rng(seed)
    nodes = [[0, 0]]
    queue = [(0, 0)]
    head = 0
    while head < len(queue):
        idx, lvl = queue[head]
        head += 1
        if lvl == depth:
            continue
        mask = int(rng.integers(1, 256)) if lvl == 0 else int((rng.random(8) < fill).dot(1 << np.arange(8)))
        if mask == 0:
            mask = 1 << int(rng.integers(0, 8))
        first = len(nodes)
        nodes[idx][0] = first - idx
        nodes[idx][1] = mask << 8
        for c in range(8):
            if (mask >> c) & 1:
                cid = len(nodes)
                nodes.append([0, 0])
                if lvl + 1 == depth:
                    nodes[idx][1] |= 1 << c
                queue.append((cid, lvl + 1))
    n = np.asarray(nodes, dtype=np.int64).astype(np.uint32)
    attribs = np.stack([rng.integers(0, 2**32, size=len(nodes), dtype=np.uint64).astype(np.uint32),
                        rng.integers(0, 2**32, size=len(nodes), dtype=np.uint64).astype(np.uint32)], axis=1)
    return n, attribs

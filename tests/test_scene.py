"""Octree construction, treelet cut, files and flattening (CPU only)."""
import itertools

import numpy as np
import pytest

import libsvo_b200 as L


def menger_cells(level, depth):
    side = 3**level
    off = (2**depth - side) // 2
    ax = np.arange(side)
    digits = np.stack([(ax // 3**k) % 3 == 1 for k in range(level)], axis=1)  # [side, level]
    x, y, z = np.meshgrid(ax, ax, ax, indexing="ij")
    dx, dy, dz = digits[x], digits[y], digits[z]
    holes = ((dx & dy) | (dx & dz) | (dy & dz)).any(axis=-1)
    keep = ~holes
    return set(zip((x[keep] + off).tolist(), (y[keep] + off).tolist(), (z[keep] + off).tolist()))


def decode_flat(nodes):
    """Leaf voxels of a flat pool with absolute first-child indices."""
    out = {}
    stack = [(0, 0, 0, 0, 0)]
    while stack:
        idx, lvl, x, y, z = stack.pop()
        fc, m = int(nodes[idx, 0]), int(nodes[idx, 1])
        rank = 0
        for c in range(8):
            if not (m >> (c + 8)) & 1:
                continue
            cx, cy, cz = 2 * x + ((c >> 2) & 1), 2 * y + ((c >> 1) & 1), 2 * z + (c & 1)
            child = fc + rank
            rank += 1
            if (m >> c) & 1:
                out[(cx, cy, cz)] = lvl + 1
            else:
                stack.append((child, lvl + 1, cx, cy, cz))
    return out


def decode_incore(nodes):
    """Leaf voxels of an incore treelet pool (relative indices, wrapping)."""
    out = {}
    stack = [(0, 0, 0, 0, 0)]
    while stack:
        idx, lvl, x, y, z = stack.pop()
        fc, m = int(nodes[idx, 0]), int(nodes[idx, 1])
        rank = 0
        for c in range(8):
            if not (m >> (c + 8)) & 1:
                continue
            cx, cy, cz = 2 * x + ((c >> 2) & 1), 2 * y + ((c >> 1) & 1), 2 * z + (c & 1)
            child = (idx + fc + rank) & 0xFFFFFFFF
            rank += 1
            if (m >> c) & 1:
                out[(cx, cy, cz)] = lvl + 1
            else:
                stack.append((child, lvl + 1, cx, cy, cz))
    return out


@pytest.mark.parametrize("level,depth", [(2, 4), (3, 5), (3, 6)])
def test_menger_voxels(level, depth):
    s = L.Scene.menger(level=level, depth=depth, seed=1)
    want = menger_cells(level, depth)
    assert s.info.leaf_voxels == len(want) == 20**level
    nodes, _ = s.flatten()
    got = decode_flat(nodes)
    assert set(got) == want
    assert set(got.values()) == {depth}


@pytest.mark.parametrize("levels", [0, 1, 2, 3])
def test_treelet_cut_preserves_octree(levels):
    s = L.Scene.menger(level=3, depth=5, seed=2, treelet_levels=levels)
    info = s.info
    mm = L.TreeletMemoryManagerCuda(s, info.treelet_bytes * info.num_treelets)
    assert mm.insertAll() == info.num_treelets - 1
    nodes, _ = mm.getIncoreBuffer()
    assert set(decode_incore(nodes)) == menger_cells(3, 5)
    n = info.nodes_per_treelet
    for g in range(info.num_treelets):
        t = s.treelet(g)
        assert 1 <= t["num_nodes"] <= n - 7
        if g:
            p = s.treelet(t["parent_gid"])
            assert t["parent_gid"] < g  # breadth-first gids
            assert 0 < t["parent_leaf_position"] < p["num_nodes"]
            assert 0 <= t["parent_leaf_idx"] < 8


def test_treelet_levels_are_aligned_to_the_leaves():
    v, t = L.icosphere(3)
    s = L.Scene.from_mesh(v, t, 7, treelet_levels=3)
    assert s.info.max_depth == 7
    # boundaries at depths 7, 4, 1: the top treelet holds depths 0..1
    top = s.treelet(0)
    assert top["num_nodes"] == 1 + len({(x >> 6, y >> 6, z >> 6) for x, y, z in decode_flat(s.flatten()[0])})


def test_flatten_matches_incore_decode():
    v, t = L.icosphere(3)
    s = L.Scene.from_mesh(v, t, 6, treelet_levels=2)
    flat, fattr = s.flatten()
    mm = L.TreeletMemoryManagerCuda(s, s.info.treelet_bytes * s.info.num_treelets)
    mm.insertAll()
    inc, iattr = mm.getIncoreBuffer()
    assert decode_flat(flat) == decode_incore(inc)
    assert flat.shape[0] == s.info.total_nodes - (s.info.num_treelets - 1)


def test_file_round_trip(tmp_path):
    s = L.Scene.menger(level=3, depth=5, seed=5, treelet_levels=2)
    base = tmp_path / "sponge"
    s.write(base)
    assert (tmp_path / "sponge.svo").stat().st_size == 8 + sum(
        32 + 8 * s.treelet(g)["num_nodes"] for g in range(s.info.num_treelets))
    r = L.Scene.read(base)
    assert r.info.num_treelets == s.info.num_treelets
    assert r.info.max_depth == s.info.max_depth
    for g in range(s.info.num_treelets):
        assert r.treelet(g) == s.treelet(g)
    a, b = s.flatten(), r.flatten()
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    # the manager loads the same files (TreeletMemoryManager(svoFilePath, ...))
    mm = L.TreeletMemoryManagerCuda(str(base), s.info.treelet_bytes * s.info.num_treelets)
    mm.insertAll()
    assert set(decode_incore(mm.getIncoreBuffer()[0])) == menger_cells(3, 5)


def test_file_errors(tmp_path):
    with pytest.raises(L.SvoError) as e:
        L.Scene.read(tmp_path / "missing")
    assert e.value.code == L.SVO_ERR_NOENT
    s = L.Scene.menger(level=2, depth=4, seed=1)
    s.write(tmp_path / "x")
    data = (tmp_path / "x.svo").read_bytes()
    (tmp_path / "x.svo").write_bytes(data[: len(data) // 2])
    with pytest.raises(L.SvoError) as e:
        L.Scene.read(tmp_path / "x")
    assert e.value.code == L.SVO_ERR_IO
    with pytest.raises(L.SvoError) as e:
        L.TreeletMemoryManagerCuda(str(tmp_path / "x"), 1 << 20)
    assert e.value.code == L.SVO_ERR_IO


def test_builder_argument_errors():
    with pytest.raises(L.SvoError):
        L.Scene.menger(level=5, depth=7)  # 243 cells do not fit in 128
    with pytest.raises(L.SvoError):
        L.Scene.menger(level=2, depth=4, treelet_bytes=12)  # not a node multiple
    with pytest.raises(L.SvoError):
        L.Scene.from_mesh(np.zeros((3, 3), np.float32), np.array([[0, 1, 5]], np.uint32), 4)


# ---- triangle voxeliser against a direct separating-axis test -------------

def sat_overlap(c, h, tri):
    v = tri - c
    e = [v[1] - v[0], v[2] - v[1], v[0] - v[2]]
    axes = [np.cross(ei, a) for ei in e for a in np.eye(3)]
    axes += list(np.eye(3))
    axes.append(np.cross(e[0], e[1]))
    for a in axes:
        if not np.any(a):
            continue
        p = v @ a
        r = h * np.abs(a).sum()
        if p.min() > r or p.max() < -r:
            return False
    return True


@pytest.mark.parametrize("seed", range(4))
def test_voxeliser_matches_direct_sat(seed):
    rng = np.random.default_rng(seed)
    depth = 4
    R = 2**depth
    tris = rng.uniform(-0.45, 0.45, size=(3, 3, 3)).astype(np.float32)
    verts = tris.reshape(-1, 3)
    idx = np.arange(9, dtype=np.uint32).reshape(3, 3)
    s = L.Scene.from_mesh(verts, idx, depth)
    got = set(decode_flat(s.flatten()[0]))
    want = set()
    h = 0.5 / R
    for i, j, k in itertools.product(range(R), repeat=3):
        c = np.array([-0.5 + (i + 0.5) / R, -0.5 + (j + 0.5) / R, -0.5 + (k + 0.5) / R])
        if any(sat_overlap(c, h, tris[t].astype(np.float64)) for t in range(3)):
            want.add((i, j, k))
    # float32 vs float64 arithmetic may disagree on boxes the triangle only touches
    assert len(got ^ want) <= max(2, len(want) // 50), (len(got), len(want), len(got ^ want))
    assert len(got & want) >= 0.97 * len(want)


def test_meshes():
    v, t = L.icosphere(2, radius=0.4, amplitude=0.05)
    assert v.shape == (162, 3) and t.shape == (320, 3)
    r = np.linalg.norm(v, axis=1)
    assert r.min() >= 0.35 - 1e-5 and r.max() <= 0.45 + 1e-5
    v6, t6 = L.icosphere(6)
    assert t6.shape[0] == 81920
    v, t = L.terrain(33, octaves=6)
    assert v.shape == (33 * 33, 3) and t.shape == (2 * 32 * 32, 3)
    assert v[:, 1].min() >= -0.45 - 1e-6 and v[:, 1].max() <= -0.15 + 1e-6
    v2, _ = L.terrain(33, octaves=6)
    assert np.array_equal(v, v2)  # seeded, deterministic


def _leaf_attribs(scene):
    mm = L.TreeletMemoryManagerCuda(scene, scene.info.treelet_bytes * scene.info.num_treelets)
    mm.insertAll()
    nodes, attribs = mm.getIncoreBuffer()
    leaf = np.zeros(nodes.shape[0], dtype=bool)
    # children flagged as leaves in their parent's masks
    for i in np.nonzero(nodes[:, 1] & 0xFF)[0]:
        m = int(nodes[i, 1])
        first = (int(i) + int(nodes[i, 0])) & 0xFFFFFFFF
        rank = 0
        for c in range(8):
            if (m >> (8 + c)) & 1:
                if (m >> c) & 1:
                    leaf[first + rank] = True
                rank += 1
    return attribs[leaf]


def test_interpolated_attributes_of_a_flat_triangle():
    """One triangle with equal vertex normals and colours: every leaf carries
    exactly that normal and colour (the interpolation of equal values, whatever
    u and v are); with different vertex colours, every leaf colour lies within
    the vertex colours' range."""
    v = np.array([[-0.4, -0.1, -0.3], [0.4, 0.05, -0.2], [0.0, 0.02, 0.4]], dtype=np.float32)
    t = np.array([[0, 1, 2]], dtype=np.uint32)
    n = np.tile(np.array([0.0, 1.0, 0.0], dtype=np.float32), (3, 1))
    c = np.tile(np.array([0.8, 0.4, 0.2], dtype=np.float32), (3, 1))
    scene = L.Scene.from_mesh(v, t, 6, normals=n, colors=c)
    a = _leaf_attribs(scene)
    assert a.shape[0] > 100
    col = a[:, 1]
    assert ((col >> 24) == 204).all() and (((col >> 16) & 255) == 102).all() and (((col >> 8) & 255) == 51).all()
    nrm = a[:, 0]
    assert (((nrm >> 16) & 255) == 255).all()  # y = 1 -> 1 * 0.5 + 0.5 -> 255
    c2 = np.array([[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]], dtype=np.float32)
    a2 = _leaf_attribs(L.Scene.from_mesh(v, t, 6, normals=n, colors=c2))
    rgb = np.stack([(a2[:, 1] >> 24) & 255, (a2[:, 1] >> 16) & 255, (a2[:, 1] >> 8) & 255], axis=1)
    # the weights (1 - u - v, u, v) sum to 1; u and v are clamped separately,
    # so 1 - u - v may go negative and its channel clamps to 0 (sum above 255)
    assert (rgb.sum(axis=1) >= 253).all()
    assert rgb.max(axis=0).min() > 128  # every vertex colour dominates somewhere


def test_vertex_attribute_arguments():
    v, t = L.icosphere(1)
    n, c = L.vertex_attributes(v, t, 1)
    assert np.allclose(np.linalg.norm(n, axis=1), 1.0, atol=1e-6)
    assert (c >= 0.15).all() and (c <= 0.95).all()
    with pytest.raises(ValueError):
        L.Scene.from_mesh(v, t, 5, normals=n)
    with pytest.raises(L.SvoError) as e:
        L.lib.svo_scene_build_mesh_attributed(v.ctypes.data, n.ctypes.data, None, v.shape[0], t.ctypes.data,
                                             t.shape[0], 5, 0, 0, 0, None) and L._check(-22, "x")
    assert e.value.code == L.SVO_ERR_INVALID

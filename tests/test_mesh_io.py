"""PLY input (the reference octree builder's mesh format) and the builder's
unit-cube placement."""
import numpy as np
import pytest

import libsvo_b200 as L
from oracle.build_ref import reference_root

# the reference's sample scan, where $LIBSVO_REFERENCE names its checkout
REF_PLY = (reference_root() / "data" / "meshes" / "frog2_seperated.ply") if reference_root() else None


def write_ply(path, v, t, n=None, c=None, binary=True, quads=False):
    props = ["property float x", "property float y", "property float z"]
    if n is not None:
        props += ["property float nx", "property float ny", "property float nz"]
    if c is not None:
        props += ["property uchar red", "property uchar green", "property uchar blue", "property uchar alpha"]
    faces = [list(f) for f in t]
    if quads:  # merge triangle pairs (a, b, c), (a, c, d) back into quads where they share the fan edge
        faces = [list(t[i]) + [t[i + 1][2]] for i in range(0, len(t) - 1, 2)]
    head = ["ply", f"format {'binary_little_endian' if binary else 'ascii'} 1.0", "comment test",
            f"element vertex {len(v)}", *props, f"element face {len(faces)}",
            "property list uchar int vertex_indices", "end_header"]
    with open(path, "wb") as f:
        f.write(("\n".join(head) + "\n").encode())
        for i in range(len(v)):
            vals = list(v[i]) + (list(n[i]) if n is not None else [])
            cols = [int(round(x * 255)) for x in c[i]] + [255] if c is not None else []
            if binary:
                f.write(np.asarray(vals, dtype="<f4").tobytes() + bytes(cols))
            else:
                f.write((" ".join(repr(float(x)) for x in vals) + (" " if cols else "") +
                         " ".join(str(x) for x in cols) + "\n").encode())
        for face in faces:
            if binary:
                f.write(bytes([len(face)]) + np.asarray(face, dtype="<i4").tobytes())
            else:
                f.write((f"{len(face)} " + " ".join(str(x) for x in face) + "\n").encode())


@pytest.mark.parametrize("binary", [True, False])
def test_ply_round_trip(tmp_path, binary):
    v, t = L.icosphere(2)
    n, c = L.vertex_attributes(v, t, 4)
    p = tmp_path / "m.ply"
    write_ply(p, v, t, n, c, binary=binary)
    m = L.read_ply(p)
    assert np.array_equal(m["triangles"], t)
    assert np.allclose(m["vertices"], v, atol=0 if binary else 1e-6)
    assert np.allclose(m["normals"], n, atol=0 if binary else 1e-6)
    assert np.allclose(m["colors"], np.round(c * 255) / 255, atol=1e-6)


def test_ply_polygons_become_fans(tmp_path):
    v = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], dtype=np.float32)
    t = np.array([[0, 1, 2], [0, 2, 3]], dtype=np.uint32)
    p = tmp_path / "q.ply"
    write_ply(p, v, t, quads=True)
    m = L.read_ply(p)
    assert m["normals"] is None and m["colors"] is None
    assert np.array_equal(m["triangles"], t)


def test_ply_errors(tmp_path):
    with pytest.raises(L.SvoError) as e:
        L.read_ply(tmp_path / "missing.ply")
    assert e.value.code == L.SVO_ERR_NOENT
    bad = tmp_path / "bad.ply"
    bad.write_bytes(b"ply\nformat binary_big_endian 1.0\nelement vertex 0\nend_header\n")
    with pytest.raises(L.SvoError) as e:
        L.read_ply(bad)
    assert e.value.code == L.SVO_ERR_NOTSUP
    v = np.zeros((3, 3), dtype=np.float32)
    write_ply(tmp_path / "oob.ply", v, np.array([[0, 1, 5]], dtype=np.uint32))
    with pytest.raises(L.SvoError) as e:
        L.read_ply(tmp_path / "oob.ply")
    assert e.value.code == L.SVO_ERR_INVALID


def test_fit_unit_cube():
    rng = np.random.default_rng(1)
    v = (rng.normal(size=(500, 3)) * [3.0, 1.0, 0.5] + [10.0, -4.0, 2.0]).astype(np.float32)
    n = rng.normal(size=(500, 3)).astype(np.float32)
    fv, fn = L.fit_unit_cube(v, n)
    ext = fv.max(axis=0) - fv.min(axis=0)
    assert ext.max() == pytest.approx(1.0, abs=1e-6)
    assert np.allclose(fv.max(axis=0) + fv.min(axis=0), 0.0, atol=1e-6)
    assert np.allclose(np.linalg.norm(fn, axis=1), 1.0, atol=1e-6)
    rv, rn = L.fit_unit_cube(v, n, rotate_x_deg=90.0)  # y -> z, z -> -y
    assert np.allclose(rn[:, 2], fn[:, 1], atol=1e-5) and np.allclose(rn[:, 1], -fn[:, 2], atol=1e-5)


@pytest.mark.skipif(REF_PLY is None or not REF_PLY.is_file(),
                    reason="the reference checkout's sample mesh is not present")
def test_reference_sample_mesh_builds():
    """The reference's own sample mesh (a scanned frog with per-vertex normals
    and colours) through the builder's placement and the attributed build."""
    m = L.read_ply(REF_PLY)
    assert m["vertices"].shape == (19629, 3) and m["normals"] is not None and m["colors"] is not None
    v, n = L.fit_unit_cube(m["vertices"], m["normals"])
    scene = L.Scene.from_mesh(v, m["triangles"], 8, treelet_levels=4, normals=n, colors=m["colors"])
    assert scene.info.leaf_voxels > 10000

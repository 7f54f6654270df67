"""The oracle against golden outputs of the reference's own ray cast.

The fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py from
opencl/treeletRenderer_rgba.cl compiled for the host) hold node pools,
frames, rays and the reference's results; the oracle must reproduce them bit
for bit.  This pins the oracle on machines without the reference checkout.
"""
from pathlib import Path

import numpy as np
import pytest

import oracle

GOLDEN = Path(__file__).resolve().parent / "golden"
FIXTURES = sorted(GOLDEN.glob("*.npz"))


def test_fixtures_present():
    assert len(FIXTURES) >= 4


@pytest.mark.parametrize("path", FIXTURES, ids=[p.stem for p in FIXTURES])
def test_oracle_reproduces_reference_outputs(path):
    z = np.load(path)
    nodes, attribs = z["nodes"], z["attribs"]
    i = 0
    while f"params_{i}" in z:
        params = z[f"params_{i}"].tobytes()
        want = z[f"rgbaf_{i}"]
        _, hits, _, got = oracle.render(nodes, attribs, params, want_rgbaf=True)
        mode = int(np.frombuffer(params[12:16], dtype=np.int32)[0])
        defined = np.ones(hits.shape, dtype=bool)
        if mode == 4:  # t is unwritten by the reference for rays missing the cube
            defined = (hits["flags"] & oracle.FLAG_BOX_MISS) == 0
        assert np.array_equal(got[defined].view(np.uint32), want[defined].view(np.uint32)), f"frame {i}"
        i += 1
    assert i > 0
    j = 0
    while f"tsr_{j}" in z:
        h, _ = oracle.cast_rays(nodes, z["origins"], z["dirs"], float(z[f"tsr_{j}"]))
        for k in ("node", "depth", "hit", "loops"):
            assert np.array_equal(h[k], z[f"hits_{j}_{k}"]), f"{k} at tsr {float(z[f'tsr_{j}'])}"
        assert np.array_equal(h["t"].view(np.uint32), z[f"hits_{j}_t"].view(np.uint32))
        j += 1
    assert j > 0
    k = 0
    while f"fb_params_{k}" in z:
        rec, img = oracle.feedback(nodes, z[f"fb_params_{k}"].tobytes())
        assert np.array_equal(rec.view(np.uint8).reshape(-1), z[f"fb_rec_{k}"].reshape(-1)), f"feedback {k}"
        assert np.array_equal(img.view(np.uint32), z[f"fb_img_{k}"].view(np.uint32))
        k += 1
    k = 0
    while f"sh_params_{k}" in z:
        _, _, shits, _, rgbaf = oracle.render_shadow(
            nodes, attribs, z[f"sh_params_{k}"].tobytes(), z[f"sh_light_{k}"], float(z[f"sh_tsr_{k}"]),
            float(z[f"sh_offset_{k}"]), want_rgbaf=True)
        assert np.array_equal(rgbaf.view(np.uint32), z[f"sh_rgbaf_{k}"].view(np.uint32)), f"shadow frame {k}"
        want = z[f"sh_hits_{k}"].view(oracle.HIT_DTYPE).reshape(shits.shape)
        for f in ("node", "t", "depth", "hit", "loops"):
            assert np.array_equal(shits[f].view(np.uint32) if f == "t" else shits[f],
                                  want[f].view(np.uint32) if f == "t" else want[f]), f"shadow {f}"
        k += 1

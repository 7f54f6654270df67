"""Host side of the analysis pass (RenderPassAnalyse::performAnalysePass,
src/RenderPassAnalyse.cpp:218-356) against a direct restatement, on
feedback records the oracle produces for partially resident pools."""
import numpy as np
import pytest

import libsvo_b200 as L
import oracle
from test_oracle_pinning import partially_resident_menger


def restate(records, slots, parents, N, num_treelets, max_new):
    new, old = {}, {}
    for e in records.reshape(-1):
        node, err, sub = int(e["node_id"]), float(e["error"]), int(e["sub_treelet_gid"])
        if node == 0:
            continue
        if sub != 0:
            if node < 0 or (sub & 0xFFFFFFFF) > num_treelets:
                return None
            if sub not in new or err > new[sub]:
                new[sub] = err
        slot = (node & 0xFFFFFFFF) // N
        if slot > num_treelets or slot >= len(slots):
            return None
        gid = slots[slot]
        if gid < 0 or gid > num_treelets:
            return None
        g = gid
        while g != 0:
            if g not in old or err > old[g]:
                old[g] = err
            g = parents[g]
        old[0] = 99.0
    new_list = sorted(sorted(new.items()), key=lambda kv: -kv[1])[:max_new]
    old_list = sorted(sorted(old.items()), key=lambda kv: -kv[1])
    return new_list, old_list


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_analysis_matches_restatement(seed):
    scene, mm, parents = partially_resident_menger()
    nodes, _ = mm.getIncoreBuffer()
    slots = [s[0] for s in mm.getSlots()]
    N, ntl = mm.getNumNodesPerTreelet(), scene.info.num_treelets
    p = bytes(L.orbit_camera(seed, 96, 96, radius=(1.2, 2.0)).frame_params(t_scale_ratio=0.0))
    rec, _ = oracle.feedback(nodes, p)
    for max_new in (0, 3):
        got_new, got_old = mm.analyseFeedback(rec, max_new=max_new)
        cap = max_new or int((12.0 * 1048576.0) / scene.info.treelet_bytes)
        want_new, want_old = restate(rec, slots, parents, N, ntl, cap)
        assert [g for g, _ in got_new] == [g for g, _ in want_new]
        assert np.allclose([e for _, e in got_new], [e for _, e in want_new], rtol=0, atol=0)
        assert [g for g, _ in got_old] == [g for g, _ in want_old]
        assert got_old[0] == (0, 99.0) or 0 in [g for g, _ in got_old]
    assert len(got_new) > 0 and all(mm.getSlotGid(g) == -1 for g, _ in got_new)


def test_analysis_feeds_update_client_side():
    scene, mm, parents = partially_resident_menger()
    nodes, _ = mm.getIncoreBuffer()
    p = bytes(L.orbit_camera(2, 96, 96, radius=1.4).frame_params(t_scale_ratio=0.0))
    rec, _ = oracle.feedback(nodes, p)
    new, old = mm.analyseFeedback(rec)
    free_before = mm.info.free_slots
    rc = mm.updateClientSideIncoreBuffer([g for g, _ in new], [e for _, e in new], [g for g, _ in old])
    assert rc == L.SVO_OK
    assert mm.info.free_slots == free_before - len(new)
    for g, e in new:
        s = mm.getSlotGid(g)
        assert s >= 0 and mm.getSlots()[s] == (g, 8, pytest.approx(e))


def test_analysis_rejects_what_the_reference_rejects():
    scene, mm, parents = partially_resident_menger()
    ntl = scene.info.num_treelets
    rec = np.zeros(4, dtype=oracle.FEEDBACK_DTYPE)
    rec[0] = (5, 0.1, ntl + 1, 1.0)  # sub-treelet gid beyond the treelet count
    with pytest.raises(L.SvoError) as e:
        mm.analyseFeedback(rec)
    assert e.value.code == L.SVO_ERR_RANGE
    rec[0] = (-3, 0.1, 2, 1.0)  # negative node id with a sub-treelet
    with pytest.raises(L.SvoError):
        mm.analyseFeedback(rec)
    rec[0] = (0, 0.0, 0, 9999999.0)  # empty records: nothing visible
    assert mm.analyseFeedback(rec) == ([], [])

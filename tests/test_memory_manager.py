"""TreeletMemoryManager bookkeeping (host side, no GPU needed).

Follows src/TreeletMemoryManager.cpp: slot stack order, leaf patching with
relative first-child indices (:518-545), removal (:666-700), eviction by
visibility (:561-653), visibility updates (:393-443), and the upload
coalescing of TreeletMemoryManagerCl.cpp:177-211.
"""
import numpy as np
import pytest

import libsvo_b200 as L


@pytest.fixture()
def scene():
    return L.Scene.menger(level=3, depth=6, seed=9, treelet_levels=2)


def children_of(scene, g):
    return [c for c in range(scene.info.num_treelets) if c and scene.treelet(c)["parent_gid"] == g]


def test_reset_state(scene):
    n = scene.info.num_treelets
    mm = L.TreeletMemoryManagerCuda(scene, scene.info.treelet_bytes * 10)
    info = mm.info
    assert info.num_slots == 10 and info.free_slots == 9
    assert mm.getSlots()[0][0] == 0 and mm.getSlots()[0][1] == mm.MAX_VISIBILITY
    assert mm.getSlotGid(0) == 0
    assert all(mm.getSlotGid(g) == -1 for g in range(1, n))
    assert list(mm.getIncoreSlotsToUpload()) == [0]
    assert mm.getTreeletSizeInByte() == scene.info.treelet_bytes


def test_insert_patches_parent_leaf(scene):
    mm = L.TreeletMemoryManagerCuda(scene, scene.info.treelet_bytes * 10)
    N = mm.getNumNodesPerTreelet()
    g = children_of(scene, 0)[3]
    t = scene.treelet(g)
    before, _ = mm.getIncoreBuffer(0, N)
    assert (before[t["parent_leaf_parent_position"], 1] >> t["parent_leaf_idx"]) & 1  # leaf
    assert before[t["parent_leaf_position"], 0] == g  # leaf holds the sub-treelet gid
    assert mm.insertTreeletIntoIncoreBuffer(g, 8, 0.5)
    slot = mm.getSlotGid(g)
    assert slot == 1  # free-slot stack pops 1 after 0
    nodes, _ = mm.getIncoreBuffer()
    leaf = t["parent_leaf_position"]
    root = slot * N
    assert nodes[leaf, 1] == nodes[root, 1]  # root node copied into the leaf
    assert nodes[leaf, 0].view(np.int32) == (root + 1) - leaf  # relative first child
    assert not (nodes[t["parent_leaf_parent_position"], 1] >> t["parent_leaf_idx"]) & 1
    assert list(mm.getIncoreSlotsToUpload()) == [0, 1]
    assert mm.getSlots()[1] == (g, 8, 0.5)
    # remove restores the original leaf and its leaf flag
    assert mm.removeTreeletFromIncoreBuffer(g)
    after, _ = mm.getIncoreBuffer(0, N)
    assert np.array_equal(after, before)
    assert mm.getSlotGid(g) == -1
    assert mm.info.free_slots == 9
    # the freed slot is on top of the stack again
    assert mm.insertTreeletIntoIncoreBuffer(children_of(scene, 0)[0])
    assert mm.getSlotGid(children_of(scene, 0)[0]) == 1


def test_negative_relative_index_after_paging(scene):
    mm = L.TreeletMemoryManagerCuda(scene, scene.info.treelet_bytes * 40)
    N = mm.getNumNodesPerTreelet()
    top = children_of(scene, 0)
    for g in top[:6]:
        assert mm.insertTreeletIntoIncoreBuffer(g)
    assert mm.removeTreeletFromIncoreBuffer(top[0])  # frees slot 1
    deep = children_of(scene, top[5])[0]  # parent in slot 6
    assert mm.insertTreeletIntoIncoreBuffer(deep)
    assert mm.getSlotGid(deep) == 1
    t = scene.treelet(deep)
    leaf = 6 * N + t["parent_leaf_position"]
    nodes, _ = mm.getIncoreBuffer()
    assert int(nodes[leaf, 0].view(np.int32)) == (N + 1) - leaf < 0


def test_insert_errors(scene):
    mm = L.TreeletMemoryManagerCuda(scene, scene.info.treelet_bytes * 3)
    top = children_of(scene, 0)
    grandchild = children_of(scene, top[0])[0]
    assert not mm.insertTreeletIntoIncoreBuffer(grandchild)  # parent not resident
    assert not mm.insertTreeletIntoIncoreBuffer(10**6)
    assert not mm.insertTreeletIntoIncoreBuffer(-1)
    assert mm.insertTreeletIntoIncoreBuffer(top[0])
    assert not mm.insertTreeletIntoIncoreBuffer(top[0])  # already resident
    assert mm.insertTreeletIntoIncoreBuffer(top[1])
    # full, and nothing is evictable (visibility still >= 0)
    assert not mm.insertTreeletIntoIncoreBuffer(top[2])
    assert not mm.removeTreeletFromIncoreBuffer(0)
    assert not mm.removeTreeletFromIncoreBuffer(top[2])
    with pytest.raises(L.SvoError) as e:
        L.TreeletMemoryManagerCuda(scene, scene.info.treelet_bytes - 8)
    assert e.value.code == L.SVO_ERR_RANGE


def test_visibility_driven_eviction(scene):
    mm = L.TreeletMemoryManagerCuda(scene, scene.info.treelet_bytes * 4)
    top = children_of(scene, 0)
    rc = mm.updateClientSideIncoreBuffer(top[:3], [0.1, 0.2, 0.3])
    assert rc == L.SVO_OK
    assert [s[0] for s in mm.getSlots()] == [0, top[0], top[1], top[2]]
    # nine frames without seeing top[1]: its visibility drops below zero,
    # while the root slot (slot 0) is never decremented
    for _ in range(9):
        mm.updateClientSideIncoreBuffer([], None, [top[0], top[2]])
    slots = mm.getSlots()
    assert slots[2][1] < 0 and slots[1][1] == 8 and slots[0][1] == 8
    # evicting needs the parent's visibility below zero as well: root stays 8
    assert not mm.freeIncorePosition()
    # a child of top[1] becomes evictable once both have gone stale
    mm2 = L.TreeletMemoryManagerCuda(scene, scene.info.treelet_bytes * 4)
    gc = children_of(scene, top[1])[0]
    mm2.updateClientSideIncoreBuffer([top[1], gc, top[0]])
    for _ in range(9):
        mm2.updateClientSideIncoreBuffer([], None, [top[0]])
    assert mm2.info.free_slots == 0
    newcomer = top[2]
    assert mm2.insertTreeletIntoIncoreBuffer(newcomer)  # frees gc's slot
    assert mm2.getSlotGid(gc) == -1 and mm2.getSlotGid(newcomer) >= 0


def test_eviction_frees_resident_subtree(scene):
    mm = L.TreeletMemoryManagerCuda(scene, scene.info.treelet_bytes * 8)
    top = children_of(scene, 0)
    a = top[0]
    ca = children_of(scene, a)[:2]
    gca = [c for c in children_of(scene, ca[0])][:1]
    assert mm.updateClientSideIncoreBuffer([a] + ca + gca + [top[1]]) == L.SVO_OK
    nodes_before, _ = mm.getIncoreBuffer(0, mm.getNumNodesPerTreelet())
    for _ in range(9):
        mm.updateClientSideIncoreBuffer([], None, [top[1]])
    # a's parent is the root (always visible), so a itself is not evictable;
    # ca[0] is (parent a stale): freeing it also frees its resident child
    assert mm.freeIncorePosition()
    freed = [g for g in [a] + ca + gca if mm.getSlotGid(g) == -1]
    assert set(freed) in ({ca[0]} | set(gca), {ca[1]})


def test_upload_coalescing_rule(scene):
    """Ranges merge while (treelets+1)/(distance+1) >= 1.2, the reference's
    treeletToSlotRatio 0.6*2 (its first comparison counts the start slot
    twice, which this restatement keeps)."""
    def restate(slots):
        out, i = [], 0
        slots = sorted(slots)
        while i < len(slots):
            start, n_slots, n_tl = slots[i], 1, 1
            while i < len(slots):
                dist = slots[i] - start
                if (n_tl + 1) / (dist + 1) >= 1.2:
                    n_slots, n_tl, i = dist + 1, n_tl + 1, i + 1
                else:
                    break
            out.append((start, n_slots))
        return out

    rng = np.random.default_rng(0)
    top = children_of(scene, 0)
    mm = L.TreeletMemoryManagerCuda(scene, scene.info.treelet_bytes * (len(top) + 1))
    for g in top:
        assert mm.insertTreeletIntoIncoreBuffer(g)
    assert mm.planUploads() == restate(mm.getIncoreSlotsToUpload().tolist())
    # contiguous dirty slots still split every 5 slots: (k+2)/(k+1) >= 1.2 only for k <= 4
    assert mm.planUploads() == [(0, 5), (5, len(top) + 1 - 5)]
    for trial in range(5):
        mm.resetIncoreBuffer()
        sel = sorted(rng.choice(top, size=len(top) // 2, replace=False).tolist())
        for g in sel:
            mm.insertTreeletIntoIncoreBuffer(g)
        for g in sel[::3]:
            mm.removeTreeletFromIncoreBuffer(g)
        dirty = mm.getIncoreSlotsToUpload().tolist()
        assert mm.planUploads() == restate(dirty)
    assert restate([0, 2]) == [(0, 1), (2, 1)]
    assert restate([0, 1, 3]) == [(0, 2), (3, 1)]
    assert restate([0, 1, 2]) == [(0, 3)]


def test_upload_ratio_knob(scene):
    """The coalescing ratio the reference hard-codes (0.6): ratio 1 copies
    every dirty slot alone, ratio 0 one range from the first to the last dirty
    slot; ratios outside [0, 1] are refused (the reference's loop would stop
    advancing above 1)."""
    top = children_of(scene, 0)
    mm = L.TreeletMemoryManagerCuda(scene, scene.info.treelet_bytes * (len(top) + 1))
    for g in top:
        assert mm.insertTreeletIntoIncoreBuffer(g)
    for g in top[1::3]:
        mm.removeTreeletFromIncoreBuffer(g)
    for g in top[1::3]:
        mm.insertTreeletIntoIncoreBuffer(g)
    dirty = mm.getIncoreSlotsToUpload().tolist()
    mm.setUploadRatio(1.0)
    assert mm.planUploads() == [(s, 1) for s in dirty]
    mm.setUploadRatio(0.0)
    assert mm.planUploads() == [(dirty[0], dirty[-1] - dirty[0] + 1)]
    mm.setUploadRatio(0.6)
    assert len(mm.planUploads()) < len(dirty)
    for bad in (-0.1, 1.01, float("nan")):
        with pytest.raises(L.SvoError) as e:
            mm.setUploadRatio(bad)
        assert e.value.code == L.SVO_ERR_RANGE
    with pytest.raises(L.SvoError) as e:
        mm.setUploadPolicy(7)
    assert e.value.code == L.SVO_ERR_NOTSUP
    mm.setUploadPolicy(L.UPLOAD_PACKED)


def test_insert_all_and_reset(scene):
    n = scene.info.num_treelets
    mm = L.TreeletMemoryManagerCuda(scene, scene.info.treelet_bytes * n)
    assert mm.insertAll() == n - 1
    assert mm.info.free_slots == 0
    mm.resetIncoreBuffer()
    assert mm.info.free_slots == n - 1
    small = L.TreeletMemoryManagerCuda(scene, scene.info.treelet_bytes * 5)
    assert small.insertAll() == 4


@pytest.mark.parametrize("evict_any", [False, True])
def test_batched_update_matches_one_insertion_at_a_time(evict_any):
    """updateClientSideIncoreBuffer copies the bodies of the treelets it
    places at the end, in parallel; the mirror (free slots included), the
    slot table and the slots to upload must be those of the same update
    done as a visibility update followed by one insertion at a time.  The
    lists place children after their parents in the same update, under
    eviction pressure, so patches aimed at not-yet-copied slots occur."""
    scene = L.Scene.menger(level=3, depth=7, seed=5, treelet_levels=2)
    n = scene.info.num_treelets
    parent = {c: scene.treelet(c)["parent_gid"] for c in range(1, n)}
    kids = {}
    for c, p in parent.items():
        kids.setdefault(p, []).append(c)
    a = L.TreeletMemoryManagerCuda(scene, scene.info.treelet_bytes * 48)
    b = L.TreeletMemoryManagerCuda(scene, scene.info.treelet_bytes * 48)
    for m in (a, b):
        m.setEviction(L.EVICT_ANY_UNSEEN if evict_any else L.EVICT_REFERENCE)
    rng = np.random.default_rng(11)
    placed_total = 0
    in_batch_children = 0
    for frame in range(100):
        resident = [g for g in range(n) if a.getSlotGid(g) >= 0]
        new = []
        for g in rng.choice(resident, size=min(len(resident), 4), replace=False):
            for c in kids.get(int(g), []):  # children, then some of their children
                if a.getSlotGid(c) < 0 and c not in new:
                    new.append(c)
                    new += [d for d in kids.get(c, [])[:2] if d not in new]
        new = new[:30]
        old = [int(g) for g in rng.choice(resident, size=len(resident) // 8, replace=False) if g]
        errs = rng.random(len(new)).astype(np.float32)
        a.updateClientSideIncoreBuffer(new, errs, old)
        b.updateClientSideIncoreBuffer([], None, old)
        for g, e in zip(new, errs):
            b.insertTreeletIntoIncoreBuffer(g, b.MAX_VISIBILITY, float(e))
        assert a.getSlots() == b.getSlots(), f"frame {frame}"
        na, aa = a.getIncoreBuffer()
        nb, ab = b.getIncoreBuffer()
        assert np.array_equal(na, nb) and np.array_equal(aa, ab), f"frame {frame}"
        assert list(a.getIncoreSlotsToUpload()) == list(b.getIncoreSlotsToUpload())
        placed_total += sum(1 for g in new if a.getSlotGid(g) >= 0)
        in_batch_children += sum(1 for g in new if a.getSlotGid(g) >= 0 and parent[g] in new)
    assert placed_total > 100 and in_batch_children > 10
    a.close()
    b.close()

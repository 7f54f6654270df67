"""Device pools after uploads: every upload policy must leave the device copy
of the incore buffer equal to the host mirror, record for record, through
repeated eviction / insertion cycles that scatter dirty slots."""
import numpy as np
import pytest

import libsvo_b200 as L

pytestmark = pytest.mark.gpu


class _Dev:
    """A raw device range seen as a torch tensor (CUDA array interface)."""

    def __init__(self, ptr, nbytes):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False),
                                         "version": 2}


def device_pool(mm):
    import torch

    d_nodes, d_attribs, n = mm.getDeviceIncoreBuffer()
    torch.cuda.synchronize()
    nodes = torch.as_tensor(_Dev(d_nodes, 8 * n), device="cuda").cpu().numpy().view(np.uint32).reshape(-1, 2)
    attribs = torch.as_tensor(_Dev(d_attribs, 8 * n), device="cuda").cpu().numpy().view(np.uint32).reshape(-1, 2)
    return nodes, attribs


def children(scene):
    kids = {}
    for g in range(1, scene.info.num_treelets):
        kids.setdefault(scene.treelet(g)["parent_gid"], []).append(g)
    return kids


@pytest.mark.parametrize("policy,ratio", [(L.UPLOAD_COALESCED, 0.6), (L.UPLOAD_COALESCED, 1.0),
                                          (L.UPLOAD_COALESCED, 0.0), (L.UPLOAD_PACKED, 0.6),
                                          (L.UPLOAD_PINNED, 0.6)])
def test_device_pool_follows_host_mirror(cuda, policy, ratio):
    scene = L.Scene.menger(level=4, depth=7, seed=5, treelet_levels=2)
    kids = children(scene)
    slots = scene.info.num_treelets // 2
    mm = L.TreeletMemoryManagerCuda(scene, scene.info.treelet_bytes * slots)
    mm.setUploadPolicy(policy)
    mm.setUploadRatio(ratio)
    mm.initDeviceBuffer()
    rng = np.random.default_rng(3)
    resident = {0}
    for cycle in range(6):
        # evict some childless resident treelets, insert treelets whose parent is resident
        leaves = [g for g in resident if g and not any(c in resident for c in kids.get(g, []))]
        for g in rng.permutation(leaves)[: max(1, len(leaves) // 3)].tolist():
            assert mm.removeTreeletFromIncoreBuffer(g)
            resident.discard(g)
        cands = [g for g in range(1, scene.info.num_treelets)
                 if g not in resident and scene.treelet(g)["parent_gid"] in resident]
        for g in rng.permutation(cands).tolist():
            if mm.info.free_slots == 0:
                break
            assert mm.insertTreeletIntoIncoreBuffer(g)
            resident.add(g)
        calls = mm.updateDeviceMemory()
        assert calls > 0
        hn, ha = mm.getIncoreBuffer()
        dn, da = device_pool(mm)
        assert np.array_equal(dn, hn), f"cycle {cycle}: node pool differs"
        assert np.array_equal(da, ha), f"cycle {cycle}: attribute pool differs"
    mm.close()


@pytest.mark.parametrize("policy", [L.UPLOAD_COALESCED, L.UPLOAD_PINNED])
def test_whole_pool_upload(cuda, policy):
    """initDeviceBuffer after insertAll: the whole pool in one upload (staged
    through the ring, or two DMA copies straight from the page-locked
    mirror), then host writes that must wait for that upload."""
    scene = L.Scene.menger(level=4, depth=7, seed=6, treelet_levels=2)
    mm = L.TreeletMemoryManagerCuda(scene, scene.info.treelet_bytes * scene.info.num_treelets)
    mm.setUploadPolicy(policy)
    mm.insertAll()
    mm.initDeviceBuffer()
    hn, ha = mm.getIncoreBuffer()
    dn, da = device_pool(mm)
    assert np.array_equal(dn, hn) and np.array_equal(da, ha)
    mm.resetIncoreBuffer()  # rewrites the mirror right after the upload was issued
    mm.insertAll()
    mm.updateDeviceMemory()
    hn2, ha2 = mm.getIncoreBuffer()
    dn, da = device_pool(mm)
    assert np.array_equal(dn, hn2) and np.array_equal(da, ha2)
    mm.close()

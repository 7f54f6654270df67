"""The analysis pass's record processing on the GPU
(svo_mm_analyse_feedback_device) against the host restatement of
performAnalysePass (svo_mm_analyse_feedback) on the same records: the same
new and visible lists, gids and error bits, in the same order; the same
rejections; and analysis steps driven through the GPU form leave the same
slot table as steps driven through the host form."""
import numpy as np
import pytest

import libsvo_b200 as L

pytestmark = pytest.mark.gpu


def _scene():
    v, t = L.icosphere(4, seed=2)
    return L.Scene.from_mesh(v, t, 8, treelet_levels=3)


def _records(mm, p, cuda):
    import torch

    d_nodes, _, n = mm.getDeviceIncoreBuffer()
    fb = torch.empty(p.width * p.height * 16, dtype=torch.uint8, device=cuda)
    L.feedback_render(d_nodes, n, p, fb)
    torch.cuda.synchronize()
    return fb


def _same(a, b):
    assert [g for g, _ in a] == [g for g, _ in b]
    assert np.array_equal(np.array([e for _, e in a], np.float32).view(np.uint32),
                          np.array([e for _, e in b], np.float32).view(np.uint32))


def test_device_analysis_matches_host(cuda):
    scene = _scene()
    info = scene.info
    mm = L.TreeletMemoryManagerCuda(scene, info.treelet_bytes * info.num_treelets)
    mm.initDeviceBuffer()
    checked = 0
    for f in range(10):
        p = L.orbit_camera(40 + f, 120, 90, radius=(1.2, 2.2)).frame_params(
            t_scale_ratio=[0.0, None, 0.002][f % 3])
        fb = _records(mm, p, cuda)
        rec = fb.cpu().numpy().view(L.FEEDBACK_DTYPE)
        for max_new in (0, 3):
            host = mm.analyseFeedback(rec, max_new)
            dev = mm.analyseFeedbackDevice(fb, rec.size, max_new)
            _same(dev[0], host[0])
            _same(dev[1], host[1])
            checked += len(host[0]) + len(host[1])
        mm.performAnalysePass(p, divisor=2)  # page in, so later frames see deeper treelets
    assert checked > 50
    mm.close()


def test_device_analysis_rejects_what_the_host_rejects(cuda):
    import torch

    scene = _scene()
    info = scene.info
    mm = L.TreeletMemoryManagerCuda(scene, info.treelet_bytes * info.num_treelets)
    mm.initDeviceBuffer()
    p = L.orbit_camera(7, 64, 48, radius=1.5).frame_params(t_scale_ratio=0.0)
    rec = _records(mm, p, cuda).cpu().numpy().view(L.FEEDBACK_DTYPE)
    hit = int(np.nonzero(rec["node_id"] != 0)[0][0])
    for field, value in (("sub_treelet_gid", info.num_treelets + 5), ("sub_treelet_gid", -3),
                         ("node_id", 0x7FFFFFF0)):
        bad = rec.copy()
        bad[field][hit] = value
        d_bad = torch.from_numpy(bad.view(np.uint8).copy()).to(cuda)
        codes = []
        for fn in (lambda: mm.analyseFeedback(bad), lambda: mm.analyseFeedbackDevice(d_bad, bad.size)):
            with pytest.raises(L.SvoError) as e:
                fn()
            codes.append(e.value.code)
        assert codes == [L.SVO_ERR_RANGE, L.SVO_ERR_RANGE], (field, value)
    # no records, or only misses: empty lists
    assert mm.analyseFeedbackDevice(None, 0) == ([], [])
    miss = np.zeros(16, L.FEEDBACK_DTYPE)
    assert mm.analyseFeedbackDevice(torch.from_numpy(miss.view(np.uint8).copy()).to(cuda), 16) == ([], [])
    mm.close()


def test_analysis_steps_match_host_driven_steps(cuda):
    """performAnalysePass (records analysed on the GPU) against the same steps
    with the records read back and analysed on the host."""
    scene = _scene()
    info = scene.info
    a = L.TreeletMemoryManagerCuda(scene, info.treelet_bytes * info.num_treelets)
    b = L.TreeletMemoryManagerCuda(scene, info.treelet_bytes * info.num_treelets)
    a.initDeviceBuffer()
    b.initDeviceBuffer()
    for f in range(12):
        p = L.orbit_camera(60 + f, 100, 80, radius=(1.1, 2.0)).frame_params(t_scale_ratio=0.0)
        placed, _ = a.performAnalysePass(p, divisor=1)
        rec = _records(b, p, cuda).cpu().numpy().view(L.FEEDBACK_DTYPE)
        new, old = b.analyseFeedback(rec)
        assert b.updateClientSideIncoreBuffer([g for g, _ in new], [e for _, e in new],
                                              [g for g, _ in old]) == L.SVO_OK
        b.updateDeviceMemory()
        assert placed == len(new)
        assert a.getSlots() == b.getSlots(), f"step {f}"
    a.close()
    b.close()
